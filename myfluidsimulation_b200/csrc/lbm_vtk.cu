// Legacy-ASCII VTK output formatted on the GPU.
//
// The reference writes every field value with `ofstream << float`
// (src/moment_vtk_writer.cu:8-48): the float, widened to double, printed as
// printf "%g" with precision 6 (six significant digits, round-half-even on the
// exact binary value, trailing zeros removed, exponent form below 1e-4 and from
// 1e6 up).  fmt_g6 produces those bytes with integer arithmetic only, so the
// host and the device builds give the same text; a CPU test checks it against
// the C library's printf.
//
// A field of N cells becomes N lines ("v\n", "|u|\n" or "u v w\n").  Two
// kernels: vtk_count formats every line of a block of 256 and stores the
// block's byte count; vtk_scan turns the counts into offsets (one block);
// vtk_emit formats again, scans the line lengths inside the block and stores
// the block's text at its offset.  Formatting costs a few hundred integer
// operations per value, far below the cost of moving the text to the host, so
// formatting twice beats storing per-line lengths.
//
// lbm_vtk_writer runs the whole snapshot asynchronously: the kernels are
// queued on the caller's stream (ordered after the step that produced the
// fields), and a writer thread copies the text to pinned host memory in chunks
// on its own stream and writes the file while the solver keeps stepping.
#include <cuda_runtime.h>

#include <condition_variable>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "lbm_capi.h"
#include "lbm_internal.h"

#define HD __host__ __device__ __forceinline__

namespace lbm {
void set_error(const std::string& msg);
namespace vtk {

// ---- exact "%g" (precision 6) of a float --------------------------------

// unsigned integer of 6 little-endian 32-bit limbs (192 bits: the largest
// product formed below, n * 2^149 with n < 2^21, needs 170)
struct Big {
    uint32_t w[6];
};

HD void big_set(Big& a, uint64_t v) {
    a.w[0] = (uint32_t)v;
    a.w[1] = (uint32_t)(v >> 32);
    a.w[2] = a.w[3] = a.w[4] = a.w[5] = 0;
}

HD void big_mul(Big& a, uint32_t k) {
    uint64_t c = 0;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        const uint64_t t = (uint64_t)a.w[i] * k + c;
        a.w[i] = (uint32_t)t;
        c = t >> 32;
    }
}

HD void big_mul_pow5(Big& a, int k) {
    while (k >= 13) {
        big_mul(a, 1220703125u);   // 5^13
        k -= 13;
    }
    uint32_t p = 1;
    for (int i = 0; i < k; ++i) p *= 5u;
    big_mul(a, p);
}

HD void big_shl(Big& a, int s) {
    const int l = s >> 5, b = s & 31;
    for (int i = 5; i >= 0; --i) {
        const int j = i - l;
        uint32_t hi = j >= 0 ? a.w[j] : 0u;
        uint32_t lo = j - 1 >= 0 ? a.w[j - 1] : 0u;
        a.w[i] = b ? (hi << b) | (lo >> (32 - b)) : hi;
    }
}

HD int big_cmp(const Big& a, const Big& b) {
    for (int i = 5; i >= 0; --i)
        if (a.w[i] != b.w[i]) return a.w[i] < b.w[i] ? -1 : 1;
    return 0;
}

HD void big_sub(Big& a, const Big& b) {
    uint64_t borrow = 0;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        const uint64_t t = (uint64_t)a.w[i] - b.w[i] - borrow;
        a.w[i] = (uint32_t)t;
        borrow = (t >> 63) & 1u;
    }
}

// floor(v * 10^s) for v = m * 2^e as n, with the rest compared to one half:
// half = -1 below, 0 exactly, +1 above.  The value is A / D with
// s >= 0: A = m 5^s 2^max(t,0), D = 2^max(-t,0); s < 0: A = m 2^max(t,0),
// D = 5^-s 2^max(-t,0); t = e + s.  n starts from a double estimate and is
// corrected by exact comparisons.
HD uint32_t scaled_floor(uint32_t m, int e, int s, int& half) {
    const int t = e + s;
    Big A, D;
    big_set(A, m);
    big_set(D, 1);
    if (s >= 0) big_mul_pow5(A, s);
    else big_mul_pow5(D, -s);
    if (t >= 0) big_shl(A, t);
    else big_shl(D, -t);
    // estimate: v * 10^s in double (only a starting point)
    double est = ldexp((double)m, e);
    for (int k = s; k > 0; --k) est *= 10.0;
    for (int k = s; k < 0; ++k) est /= 10.0;
    uint32_t n = est < 1.0 ? 0u : (est > 4.0e9 ? 4000000000u : (uint32_t)est);
    Big nD;
    for (;;) {   // the largest n with n D <= A
        nD = D;
        big_mul(nD, n);
        if (big_cmp(nD, A) > 0) { --n; continue; }
        Big n1;  // (n + 1) D = n D + D
        uint64_t c = 0;
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            const uint64_t x = (uint64_t)nD.w[i] + D.w[i] + c;
            n1.w[i] = (uint32_t)x;
            c = x >> 32;
        }
        if (big_cmp(n1, A) <= 0) { ++n; continue; }
        break;
    }
    Big R = A;
    big_sub(R, nD);
    big_shl(R, 1);
    half = big_cmp(R, D);
    return n;
}

// Bytes of printf("%g", (double)v) into out (at most 12); returns the length.
HD int fmt_g6(float v, char* out) {
    uint32_t bits;
    memcpy(&bits, &v, 4);
    const bool neg = bits >> 31;
    const uint32_t E = (bits >> 23) & 0xffu, F = bits & 0x7fffffu;
    int len = 0;
    if (neg) out[len++] = '-';
    if (E == 0xffu) {
        const char* s = F ? "nan" : "inf";
        out[len++] = s[0]; out[len++] = s[1]; out[len++] = s[2];
        return len;
    }
    if (E == 0 && F == 0) { out[len++] = '0'; return len; }
    const uint32_t m = E ? (F | 0x800000u) : F;
    const int e = (E ? (int)E : 1) - 150;
    // decimal exponent: floor(log10 v), from the bit length, then corrected
    int b = 0;
    for (uint32_t x = m; x; x >>= 1) ++b;
    const int l2 = b - 1 + e;                                  // floor(log2 v)
    int X = (l2 >= 0) ? (l2 * 78913) >> 18 : -((-l2 * 78913 + 262143) >> 18);   // ~ l2 * log10(2)
    uint32_t n = 0;
    int half = 0;
    // fast path: y = v 10^k in double with one correctly rounded operation
    // (10^|k| is exact for |k| <= 22), so |y - exact| <= 2^-33 for y < 2^20;
    // taken only when floor(y) and the side of one half are certain, else the
    // exact path below decides
    bool done = false;
    for (int it = 0; it < 3; ++it) {
        const int k = 5 - X;
        if (k < -22 || k > 22) break;
        double p = 1.0, sq = 10.0;
        for (int a = k < 0 ? -k : k; a; a >>= 1, sq *= sq)
            if (a & 1) p *= sq;
        const double x = ldexp((double)m, e);
        const double y = k >= 0 ? x * p : x / p;
        const double fl = floor(y);
        if (fl >= 1000000.0) { ++X; continue; }
        if (fl < 100000.0) { --X; continue; }
        const double fr = y - fl, tol = 0x1p-30;
        if (fr < tol || fr > 1.0 - tol || fabs(fr - 0.5) < tol) break;
        n = (uint32_t)fl;
        half = fr > 0.5 ? 1 : -1;
        done = true;
        break;
    }
    for (int it = 0; !done && it < 4; ++it) {
        n = scaled_floor(m, e, 5 - X, half);
        if (n >= 1000000u) { ++X; continue; }
        if (n < 100000u) { --X; continue; }
        break;
    }
    if (half > 0 || (half == 0 && (n & 1u))) {
        if (++n == 1000000u) { n = 100000u; ++X; }
    }
    char d[6];
    for (int i = 5; i >= 0; --i) { d[i] = (char)('0' + n % 10u); n /= 10u; }
    int last = 5;                                              // last significant digit kept
    while (last > 0 && d[last] == '0') --last;
    if (X < -4 || X >= 6) {
        out[len++] = d[0];
        if (last > 0) {
            out[len++] = '.';
            for (int i = 1; i <= last; ++i) out[len++] = d[i];
        }
        out[len++] = 'e';
        out[len++] = X < 0 ? '-' : '+';
        const int a = X < 0 ? -X : X;
        out[len++] = (char)('0' + a / 10);
        out[len++] = (char)('0' + a % 10);
    } else if (X >= 0) {
        for (int i = 0; i <= X; ++i) out[len++] = d[i];
        if (last > X) {
            out[len++] = '.';
            for (int i = X + 1; i <= last; ++i) out[len++] = d[i];
        }
    } else {
        out[len++] = '0';
        out[len++] = '.';
        for (int i = 0; i < -X - 1; ++i) out[len++] = '0';
        for (int i = 0; i <= last; ++i) out[len++] = d[i];
    }
    return len;
}

// |u| exactly as speed_kernel computes it (the same expression)
__device__ __forceinline__ float speed3(float u, float v, float w) {
    const float uu = u * u + v * v + w * w;
    return sqrtf(uu);
}

constexpr int LINES = 256;           // lines per block
constexpr int MAXLINE = 39;          // "u v w\n" at 12 bytes per value

template <int KIND>
__device__ __forceinline__ int format_line(const float* a, const float* b, const float* c, int64_t i, char* buf) {
    int len;
    if (KIND == LBM_VTK_SCALAR) {
        len = fmt_g6(a[i], buf);
    } else if (KIND == LBM_VTK_SPEED) {
        len = fmt_g6(speed3(a[i], b[i], c[i]), buf);
    } else {
        len = fmt_g6(a[i], buf);
        buf[len++] = ' ';
        len += fmt_g6(b[i], buf + len);
        buf[len++] = ' ';
        len += fmt_g6(c[i], buf + len);
    }
    buf[len++] = '\n';
    return len;
}

template <int KIND>
__global__ void __launch_bounds__(LINES) vtk_count(const float* a, const float* b, const float* c, int64_t n,
                                                   uint32_t* block_bytes) {
    const int64_t i = (int64_t)blockIdx.x * LINES + threadIdx.x;
    char buf[MAXLINE + 1];
    uint32_t len = i < n ? (uint32_t)format_line<KIND>(a, b, c, i, buf) : 0u;
    // block sum: warp shuffles, then one warp over the 8 warp sums
    for (int o = 16; o; o >>= 1) len += __shfl_xor_sync(0xffffffffu, len, o);
    __shared__ uint32_t ws[LINES / 32];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = len;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t s = 0;
        for (int k = 0; k < LINES / 32; ++k) s += ws[k];
        block_bytes[blockIdx.x] = s;
    }
}

// exclusive scan of the block byte counts (one block of 1024 threads);
// offsets[nb] receives the total
__global__ void __launch_bounds__(1024) vtk_scan(const uint32_t* block_bytes, int64_t nb, uint64_t* offsets) {
    __shared__ uint64_t ws[32];
    __shared__ uint64_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int64_t base = 0; base < nb; base += 1024) {
        const int64_t j = base + threadIdx.x;
        const uint64_t x = j < nb ? block_bytes[j] : 0u;
        uint64_t s = x;   // inclusive warp scan
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t y = __shfl_up_sync(0xffffffffu, s, o);
            if ((threadIdx.x & 31) >= o) s += y;
        }
        if ((threadIdx.x & 31) == 31) ws[threadIdx.x >> 5] = s;
        __syncthreads();
        if (threadIdx.x < 32) {
            uint64_t t = ws[threadIdx.x];
            for (int o = 1; o < 32; o <<= 1) {
                const uint64_t y = __shfl_up_sync(0xffffffffu, t, o);
                if (threadIdx.x >= o) t += y;
            }
            ws[threadIdx.x] = t;
        }
        __syncthreads();
        const uint64_t before = carry + (threadIdx.x >= 32 ? ws[(threadIdx.x >> 5) - 1] : 0u) + s - x;
        if (j < nb) offsets[j] = before;
        __syncthreads();
        if (threadIdx.x == 1023) carry = before + x;
        __syncthreads();
    }
    if (threadIdx.x == 0) offsets[nb] = carry;
}

template <int KIND>
__global__ void __launch_bounds__(LINES) vtk_emit(const float* a, const float* b, const float* c, int64_t n,
                                                  const uint64_t* offsets, char* text) {
    __shared__ char stage[LINES * MAXLINE + 16];
    __shared__ uint32_t ws[LINES / 32];
    const int64_t i = (int64_t)blockIdx.x * LINES + threadIdx.x;
    char buf[MAXLINE + 1];
    const uint32_t len = i < n ? (uint32_t)format_line<KIND>(a, b, c, i, buf) : 0u;
    // exclusive scan of the line lengths inside the block
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t s = len;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
        if (lane >= o) s += y;
    }
    if (lane == 31) ws[warp] = s;
    __syncthreads();
    uint32_t wbase = 0;
    for (int k = 0; k < warp; ++k) wbase += ws[k];
    const uint32_t off = wbase + s - len;
    for (uint32_t k = 0; k < len; ++k) stage[off + k] = buf[k];
    uint32_t total = 0;
    for (int k = 0; k < LINES / 32; ++k) total += ws[k];
    __syncthreads();
    // block text -> global: bytes up to a 4-byte boundary, words, then the tail
    const uint64_t dst = offsets[blockIdx.x];
    const uint32_t head = (uint32_t)((4u - (uint32_t)(dst & 3u)) & 3u);
    const uint32_t h = head < total ? head : total;
    if (threadIdx.x < h) text[dst + threadIdx.x] = stage[threadIdx.x];
    const uint32_t words = (total - h) >> 2;
    uint32_t* tw = reinterpret_cast<uint32_t*>(text + dst + h);
    for (uint32_t k = threadIdx.x; k < words; k += LINES) {
        const uint32_t p = h + 4u * k;
        tw[k] = (uint32_t)(uint8_t)stage[p] | ((uint32_t)(uint8_t)stage[p + 1] << 8) |
                ((uint32_t)(uint8_t)stage[p + 2] << 16) | ((uint32_t)(uint8_t)stage[p + 3] << 24);
    }
    const uint32_t t0 = h + 4u * words;
    if (threadIdx.x < total - t0) text[dst + t0 + threadIdx.x] = stage[t0 + threadIdx.x];
}

int64_t max_line(int kind) { return kind == LBM_VTK_VECTOR ? MAXLINE : 13; }

// Queues the formatting of one field: text[0..total) on the device, total in
// offsets[nb].  scratch: nb uint32 counts; offsets: nb + 1 uint64.
cudaError_t launch_format(int kind, const float* a, const float* b, const float* c, int64_t n, uint32_t* counts,
                          uint64_t* offsets, char* text, cudaStream_t st) {
    const int64_t nb = (n + LINES - 1) / LINES;
    if (nb == 0) return cudaMemsetAsync(offsets, 0, sizeof(uint64_t), st);
    switch (kind) {
        case LBM_VTK_SCALAR: vtk_count<LBM_VTK_SCALAR><<<(unsigned)nb, LINES, 0, st>>>(a, b, c, n, counts); break;
        case LBM_VTK_SPEED: vtk_count<LBM_VTK_SPEED><<<(unsigned)nb, LINES, 0, st>>>(a, b, c, n, counts); break;
        default: vtk_count<LBM_VTK_VECTOR><<<(unsigned)nb, LINES, 0, st>>>(a, b, c, n, counts); break;
    }
    vtk_scan<<<1, 1024, 0, st>>>(counts, nb, offsets);
    switch (kind) {
        case LBM_VTK_SCALAR: vtk_emit<LBM_VTK_SCALAR><<<(unsigned)nb, LINES, 0, st>>>(a, b, c, n, offsets, text); break;
        case LBM_VTK_SPEED: vtk_emit<LBM_VTK_SPEED><<<(unsigned)nb, LINES, 0, st>>>(a, b, c, n, offsets, text); break;
        default: vtk_emit<LBM_VTK_VECTOR><<<(unsigned)nb, LINES, 0, st>>>(a, b, c, n, offsets, text); break;
    }
    return cudaGetLastError();
}

std::string header(int kind, int nx, int ny, int nz) {
    const uint64_t N = (uint64_t)nx * (uint64_t)ny * (uint64_t)nz;
    std::string h = "# vtk DataFile Version 3.0\n";
    h += kind == LBM_VTK_VECTOR ? "vector" : "scalar";
    h += "\nASCII\nDATASET STRUCTURED_POINTS\nDIMENSIONS " + std::to_string(nx) + " " + std::to_string(ny) + " " +
         std::to_string(nz) + "\nORIGIN 0 0 0\nSPACING 1 1 1\nPOINT_DATA " + std::to_string(N) + "\n";
    h += kind == LBM_VTK_VECTOR ? "VECTORS vec float\n" : "SCALARS s float 1\nLOOKUP_TABLE default\n";
    return h;
}

}  // namespace vtk

// One field to one file, synchronously on the legacy default stream (ordered
// after the blocking streams that produced the field, as the reference's
// cudaMemcpy is): format on the device, copy the text back, write it.
int write_vtk_file(int kind, const float* a, const float* b, const float* c, int nx, int ny, int nz,
                   const char* path) {
    const int64_t n = (int64_t)nx * ny * nz;
    const int64_t cap = lbm_vtk_text_bound(kind, n);
    char* d_text = nullptr;
    if (cudaMalloc((void**)&d_text, (size_t)cap) != cudaSuccess) {
        set_error("write_vtk: device allocation failed");
        return LBM_ERR_ALLOC;
    }
    int64_t len = 0;
    int rc = lbm_vtk_format(kind, a, b, c, n, d_text, cap, &len, nullptr);
    std::vector<char> h;
    if (rc == LBM_OK) {
        h.resize((size_t)len);
        if (len > 0 && cudaMemcpy(h.data(), d_text, (size_t)len, cudaMemcpyDeviceToHost) != cudaSuccess) {
            set_error("write_vtk: device copy failed");
            rc = LBM_ERR_CUDA;
        }
    }
    cudaFree(d_text);
    if (rc != LBM_OK) return rc;
    FILE* f = std::fopen(path, "wb");
    if (!f) { set_error(std::string("failed to open VTK file: ") + path); return LBM_ERR_IO; }
    const std::string hd = vtk::header(kind, nx, ny, nz);
    bool ok = std::fwrite(hd.data(), 1, hd.size(), f) == hd.size();
    ok = ok && std::fwrite(h.data(), 1, h.size(), f) == h.size();
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) { set_error(std::string("failed to write VTK file: ") + path); return LBM_ERR_IO; }
    return LBM_OK;
}

}  // namespace lbm

using namespace lbm::vtk;

// ---- asynchronous writer -------------------------------------------------

struct lbm_vtk_writer {
    struct Slot {
        char* d_text = nullptr;
        uint32_t* d_counts = nullptr;
        uint64_t* d_offsets = nullptr;
        cudaEvent_t formatted = nullptr;
        bool busy = false;
    };
    struct Job {
        int slot;
        int kind;
        std::string path;
    };
    int nx = 0, ny = 0, nz = 0, device = 0;
    int64_t n = 0, cap = 0, nb = 0;
    size_t chunk = 0;
    char* h_text = nullptr;          // pinned, two halves of `chunk` bytes (one writer thread)
    uint64_t* h_total = nullptr;     // pinned
    std::vector<Slot> slots;
    cudaStream_t copy = nullptr;
    cudaEvent_t chunk_ev[2] = {nullptr, nullptr};
    std::mutex mu;
    std::condition_variable cv;
    std::deque<Job> jobs;
    bool stop = false;
    int error = LBM_OK;
    std::string error_msg;
    uint64_t bytes_written = 0;
    std::thread th;

    void fail(int code, const std::string& msg) {
        std::lock_guard<std::mutex> g(mu);
        if (error == LBM_OK) { error = code; error_msg = msg; }
    }

    void write_job(const Job& j) {
        Slot& s = slots[j.slot];
        if (cudaEventSynchronize(s.formatted) != cudaSuccess ||
            cudaMemcpyAsync(h_total, s.d_offsets + nb, sizeof(uint64_t), cudaMemcpyDeviceToHost, copy) != cudaSuccess ||
            cudaStreamSynchronize(copy) != cudaSuccess) {
            fail(LBM_ERR_CUDA, "vtk writer: formatting or copy failed");
            return;
        }
        const uint64_t total = *h_total;
        FILE* f = std::fopen(j.path.c_str(), "wb");
        if (!f) { fail(LBM_ERR_IO, "failed to open VTK file: " + j.path); return; }
        const std::string h = header(j.kind, nx, ny, nz);
        bool ok = std::fwrite(h.data(), 1, h.size(), f) == h.size();
        // chunks through two pinned halves: copy k + 1 while k is written
        const uint64_t nch = (total + chunk - 1) / chunk;
        auto issue = [&](uint64_t k) {
            const uint64_t o = k * chunk, len = total - o < chunk ? total - o : chunk;
            cudaMemcpyAsync(h_text + (k & 1) * chunk, s.d_text + o, len, cudaMemcpyDeviceToHost, copy);
            cudaEventRecord(chunk_ev[k & 1], copy);
        };
        if (nch > 0) issue(0);
        for (uint64_t k = 0; k < nch && ok; ++k) {
            if (k + 1 < nch) issue(k + 1);
            if (cudaEventSynchronize(chunk_ev[k & 1]) != cudaSuccess) { ok = false; break; }
            const uint64_t o = k * chunk, len = total - o < chunk ? total - o : chunk;
            ok = std::fwrite(h_text + (k & 1) * chunk, 1, len, f) == len;
            // the half just written is reused by the copy after next: issued
            // only after this fwrite, in stream order behind copy k + 1
        }
        cudaStreamSynchronize(copy);
        ok = (std::fclose(f) == 0) && ok;
        if (!ok) fail(LBM_ERR_IO, "failed to write VTK file: " + j.path);
        else {
            std::lock_guard<std::mutex> g(mu);
            bytes_written += h.size() + total;
        }
    }

    void run() {
        cudaSetDevice(device);
        for (;;) {
            Job j;
            {
                std::unique_lock<std::mutex> g(mu);
                cv.wait(g, [&] { return stop || !jobs.empty(); });
                if (jobs.empty()) return;
                j = jobs.front();
            }
            write_job(j);
            {
                std::lock_guard<std::mutex> g(mu);
                jobs.pop_front();
                slots[j.slot].busy = false;
            }
            cv.notify_all();
        }
    }
};

extern "C" {

int lbm_vtk_writer_create(int32_t nx, int32_t ny, int32_t nz, int32_t depth, lbm_vtk_writer** out) {
    if (!out || nx <= 0 || ny <= 0 || nz <= 0) { lbm::set_error("lbm_vtk_writer_create: bad argument"); return LBM_ERR_INVALID; }
    auto* w = new lbm_vtk_writer();
    w->nx = nx; w->ny = ny; w->nz = nz;
    w->n = (int64_t)nx * ny * nz;
    w->nb = (w->n + LINES - 1) / LINES;
    w->cap = w->n * max_line(LBM_VTK_VECTOR);
    w->chunk = (size_t)std::min<int64_t>(w->cap > 0 ? w->cap : 1, (int64_t)32 << 20);
    cudaGetDevice(&w->device);
    bool ok = cudaStreamCreateWithFlags(&w->copy, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&w->chunk_ev[0], cudaEventDisableTiming) == cudaSuccess &&
              cudaEventCreateWithFlags(&w->chunk_ev[1], cudaEventDisableTiming) == cudaSuccess &&
              cudaHostAlloc((void**)&w->h_text, 2 * w->chunk, cudaHostAllocDefault) == cudaSuccess &&
              cudaHostAlloc((void**)&w->h_total, sizeof(uint64_t), cudaHostAllocDefault) == cudaSuccess;
    w->slots.resize((size_t)(depth < 1 ? 1 : depth));
    for (auto& s : w->slots) {
        ok = ok && cudaMalloc((void**)&s.d_text, (size_t)w->cap + 16) == cudaSuccess &&
             cudaMalloc((void**)&s.d_counts, sizeof(uint32_t) * (size_t)(w->nb + 1)) == cudaSuccess &&
             cudaMalloc((void**)&s.d_offsets, sizeof(uint64_t) * (size_t)(w->nb + 1)) == cudaSuccess &&
             cudaEventCreateWithFlags(&s.formatted, cudaEventDisableTiming) == cudaSuccess;
    }
    if (!ok) {
        lbm_vtk_writer_destroy(w);
        lbm::set_error("lbm_vtk_writer_create: allocation failed");
        return LBM_ERR_ALLOC;
    }
    w->th = std::thread([w] { w->run(); });
    *out = w;
    return LBM_OK;
}

int lbm_vtk_writer_submit(lbm_vtk_writer* w, int32_t kind, const float* d_a, const float* d_b, const float* d_c,
                          const char* path, void* stream) {
    if (!w || !path || !d_a || kind < LBM_VTK_SCALAR || kind > LBM_VTK_VECTOR ||
        (kind != LBM_VTK_SCALAR && (!d_b || !d_c))) {
        lbm::set_error("lbm_vtk_writer_submit: bad argument");
        return LBM_ERR_INVALID;
    }
    int slot = -1;
    {
        std::unique_lock<std::mutex> g(w->mu);
        w->cv.wait(g, [&] {
            for (size_t k = 0; k < w->slots.size(); ++k)
                if (!w->slots[k].busy) { slot = (int)k; return true; }
            return false;
        });
        w->slots[slot].busy = true;
    }
    auto& s = w->slots[slot];
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (launch_format(kind, d_a, d_b, d_c, w->n, s.d_counts, s.d_offsets, s.d_text, st) != cudaSuccess ||
        cudaEventRecord(s.formatted, st) != cudaSuccess) {
        std::lock_guard<std::mutex> g(w->mu);
        s.busy = false;
        lbm::set_error("lbm_vtk_writer_submit: launch failed");
        return LBM_ERR_CUDA;
    }
    {
        std::lock_guard<std::mutex> g(w->mu);
        w->jobs.push_back({slot, kind, path});
    }
    w->cv.notify_all();
    return LBM_OK;
}

int lbm_vtk_writer_flush(lbm_vtk_writer* w) {
    if (!w) { lbm::set_error("lbm_vtk_writer_flush: null writer"); return LBM_ERR_INVALID; }
    std::unique_lock<std::mutex> g(w->mu);
    w->cv.wait(g, [&] { return w->jobs.empty(); });
    const int e = w->error;
    if (e != LBM_OK) {
        lbm::set_error(w->error_msg);
        w->error = LBM_OK;
        w->error_msg.clear();
    }
    return e;
}

int lbm_vtk_writer_bytes(lbm_vtk_writer* w, uint64_t* bytes) {
    if (!w || !bytes) { lbm::set_error("lbm_vtk_writer_bytes: bad argument"); return LBM_ERR_INVALID; }
    std::lock_guard<std::mutex> g(w->mu);
    *bytes = w->bytes_written;
    return LBM_OK;
}

int lbm_vtk_writer_destroy(lbm_vtk_writer* w) {
    if (!w) return LBM_OK;
    if (w->th.joinable()) {
        {
            std::lock_guard<std::mutex> g(w->mu);
            w->stop = true;
        }
        w->cv.notify_all();
        w->th.join();
    }
    for (auto& s : w->slots) {
        cudaFree(s.d_text); cudaFree(s.d_counts); cudaFree(s.d_offsets);
        if (s.formatted) cudaEventDestroy(s.formatted);
    }
    if (w->h_text) cudaFreeHost(w->h_text);
    if (w->h_total) cudaFreeHost(w->h_total);
    if (w->chunk_ev[0]) cudaEventDestroy(w->chunk_ev[0]);
    if (w->chunk_ev[1]) cudaEventDestroy(w->chunk_ev[1]);
    if (w->copy) cudaStreamDestroy(w->copy);
    const int e = w->error;
    delete w;
    return e;
}

int lbm_vtk_format(int32_t kind, const float* d_a, const float* d_b, const float* d_c, int64_t n, char* d_text,
                   int64_t cap, int64_t* len, void* stream) {
    if (!d_text || !len || n < 0 || kind < LBM_VTK_SCALAR || kind > LBM_VTK_VECTOR ||
        (n > 0 && (!d_a || (kind != LBM_VTK_SCALAR && (!d_b || !d_c))))) {
        lbm::set_error("lbm_vtk_format: bad argument");
        return LBM_ERR_INVALID;
    }
    if (cap < lbm_vtk_text_bound(kind, n)) { lbm::set_error("lbm_vtk_format: text buffer too small"); return LBM_ERR_INVALID; }
    const int64_t nb = (n + LINES - 1) / LINES;
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    // scratch from the stream-ordered pool: no device-wide synchronisation
    uint32_t* counts = nullptr;
    uint64_t* offsets = nullptr;
    if (cudaMallocAsync((void**)&counts, sizeof(uint32_t) * (size_t)(nb + 1), st) != cudaSuccess ||
        cudaMallocAsync((void**)&offsets, sizeof(uint64_t) * (size_t)(nb + 1), st) != cudaSuccess) {
        if (counts) cudaFreeAsync(counts, st);
        lbm::set_error("lbm_vtk_format: allocation failed");
        return LBM_ERR_ALLOC;
    }
    uint64_t total = 0;
    const bool ok = launch_format(kind, d_a, d_b, d_c, n, counts, offsets, d_text, st) == cudaSuccess &&
                    cudaMemcpyAsync(&total, offsets + nb, sizeof(uint64_t), cudaMemcpyDeviceToHost, st) == cudaSuccess;
    cudaFreeAsync(counts, st);
    cudaFreeAsync(offsets, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) { lbm::set_error("lbm_vtk_format: kernel failed"); return LBM_ERR_CUDA; }
    if (!ok) { lbm::set_error("lbm_vtk_format: kernel failed"); return LBM_ERR_CUDA; }
    *len = (int64_t)total;
    return LBM_OK;
}

int64_t lbm_vtk_text_bound(int32_t kind, int64_t n) { return n * max_line(kind) + 16; }

int lbm_format_g6(const float* v, int64_t n, char* out, int32_t stride, uint8_t* lens) {
    if ((!v || !out || !lens) && n > 0) { lbm::set_error("lbm_format_g6: null argument"); return LBM_ERR_INVALID; }
    if (stride < 12) { lbm::set_error("lbm_format_g6: stride below 12"); return LBM_ERR_INVALID; }
    for (int64_t i = 0; i < n; ++i) lens[i] = (uint8_t)fmt_g6(v[i], out + i * stride);
    return LBM_OK;
}

}  // extern "C"
