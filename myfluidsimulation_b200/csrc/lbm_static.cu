// Macro-field statistics that allocate no device memory.
//
// lbm_macro_stats_static reduces caller-owned rho/u fields to the FP64 sums of
// the LBM_STAT_* slots (mass, kinetic energy, momentum) with the same
// per-block reduction as the statistics of lbm_step, but its per-block partial
// sums live in one file-scope __device__ array instead of a cudaMalloc'd
// buffer.  It is meant for callers that may not allocate while they run: a
// host loop inside a memory-pool-limited service, a stream that is being
// captured by someone else's code, or a process whose allocator is owned by
// another framework.  No counterpart in the reference (which sums on the host,
// src/bench/main_taylor_green.cpp:157-182).
//
// Limits and contract:
//   * scratch = kMaxRows rows of LBM_NSTAT doubles (2 MiB per device); block b
//     reduces cells [b*kChunk, (b+1)*kChunk), so n <= kMaxRows*kChunk =
//     268,435,456 cells; larger n is rejected with LBM_ERR_SIZE;
//   * nothing has to start at zero: every row a call reads was written by the
//     same call before it is read (two kernels in stream order);
//   * the scratch is shared by every call on a device: two calls that overlap
//     in time (different streams, or different host threads without ordering)
//     race on it and may return mixed sums;
//   * the first call on each device looks up the array's address
//     (cudaGetSymbolAddress) with that device current; make it before any
//     stream capture that will contain later calls.
// The cell assignment to blocks is fixed by kChunk, so the result is the same
// bit for bit on any GPU and from call to call.
#include <mutex>
#include <string>

#include "lbm_capi.h"
#include "lbm_common.cuh"
#include "lbm_internal.h"

namespace lbm {
void set_error(const std::string& msg);
}

namespace {

constexpr int kChunk = 8192;                  // cells per partial row (one block)
constexpr int kMaxRows = 32768;               // rows in the scratch
constexpr int64_t kMaxCells = (int64_t)kChunk * kMaxRows;
constexpr int kMaxDevices = 64;

__device__ __align__(256) double g_stats_scratch[kMaxRows * lbm::NSTAT];

std::mutex g_addr_mu;
double* g_addr[kMaxDevices] = {};

__global__ void __launch_bounds__(256) macro_stats_rows(const float* __restrict__ rho, const float* __restrict__ ux,
                                                        const float* __restrict__ uy, const float* __restrict__ uz,
                                                        const uint8_t* __restrict__ mask, int64_t n,
                                                        double* __restrict__ rows) {
    double acc[lbm::NSTAT];
#pragma unroll
    for (int k = 0; k < lbm::NSTAT; ++k) acc[k] = 0.0;
    const int64_t beg = (int64_t)blockIdx.x * kChunk;
    const int64_t end = beg + kChunk < n ? beg + kChunk : n;
    for (int64_t i = beg + threadIdx.x; i < end; i += blockDim.x) {
        if (mask && mask[i]) continue;            // solid cells are left out, as in lbm_step
        const float r = rho[i], u = ux[i], v = uy[i], w = uz[i];
        acc[0] += (double)r;
        acc[1] += 0.5 * ((double)u * u + (double)v * v + (double)w * w);
        acc[5] += (double)r * u;
        acc[6] += (double)r * v;
        acc[7] += (double)r * w;
    }
    lbm::block_reduce_stats(acc, rows);
}

int scratch_rows(double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        lbm::set_error(std::string("lbm_macro_stats_static: cudaGetDevice: ") + cudaGetErrorString(e));
        return LBM_ERR_CUDA;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        lbm::set_error("lbm_macro_stats_static: device ordinal beyond " + std::to_string(kMaxDevices));
        return LBM_ERR_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lock(g_addr_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_stats_scratch);
        if (e != cudaSuccess || !p) {
            lbm::set_error(std::string("lbm_macro_stats_static: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            return LBM_ERR_CUDA;
        }
        g_addr[dev] = static_cast<double*>(p);
    }
    *out = g_addr[dev];
    return LBM_OK;
}

}  // namespace

extern "C" int lbm_macro_stats_static(const float* d_rho, const float* d_ux, const float* d_uy, const float* d_uz,
                                      const uint8_t* d_mask, int64_t n, double* d_out, void* stream) {
    if (!d_rho || !d_ux || !d_uy || !d_uz || !d_out) {
        lbm::set_error("lbm_macro_stats_static: null field or output pointer");
        return LBM_ERR_INVALID;
    }
    if (n < 0) {
        lbm::set_error("lbm_macro_stats_static: negative cell count");
        return LBM_ERR_INVALID;
    }
    if (n > kMaxCells) {
        lbm::set_error("lbm_macro_stats_static: " + std::to_string(n) + " cells exceed the static scratch limit of " +
                       std::to_string(kMaxCells) + " cells");
        return LBM_ERR_SIZE;
    }
    double* rows = nullptr;
    const int rc = scratch_rows(&rows);
    if (rc != LBM_OK) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int nrows = (int)((n + kChunk - 1) / kChunk);
    if (nrows > 0) macro_stats_rows<<<nrows, 256, 0, s>>>(d_rho, d_ux, d_uy, d_uz, d_mask, n, rows);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = lbm::launch_finalize_stats(rows, nrows, d_out, s);
    if (e != cudaSuccess) {
        lbm::set_error(std::string("lbm_macro_stats_static: launch: ") + cudaGetErrorString(e));
        return LBM_ERR_CUDA;
    }
    return LBM_OK;
}
