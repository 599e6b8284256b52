// The solver object behind the C-ABI of include/lbm_capi.h.
//
// One lbm_solver replaces the reference's three classes (src/lbm/lbm3d_legacy.hpp,
// lbm3d_home.hpp, lbm3d_hybrid.hpp).  Memory per cell:
//   Legacy/Hybrid: one population buffer (AA pattern), 19 x 4 B (F32) or 19 x 2 B
//                  (F16/BF16), plus rho,u,v,w (16 B), mask, flags (1 B each) and a
//                  link word (4 B); the reference holds two population buffers.
//   HOME:          two moment buffers of 10 x 4 B (or 10 x 2 B), as the reference.
// All launches go to the solver's stream; nothing synchronises except the
// calls documented as synchronous.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "lbm_capi.h"
#include "lbm_common.cuh"
#include "lbm_internal.h"

namespace lbm {

thread_local std::string g_error;
void set_error(const std::string& msg) { g_error = msg; }

}  // namespace lbm

using lbm::set_error;

struct lbm_solver {
    lbm_domain dom{};
    int method = 0, storage = 0, bc = 0, bounce = 0;
    float u_in = 0.f, rho0 = 1.f;
    float omega = 0.f, omega_s = 0.f;
    int64_t N = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    size_t esize = 4;

    void* f = nullptr;          // AA populations (reference bounce: buffer A)
    void* f2 = nullptr;         // reference bounce only: buffer B
    void* m[2] = {nullptr, nullptr};   // HOME moments
    int cur = 0;
    float* macro = nullptr;     // 4*N floats: rho, ux, uy, uz (AA; HOME F16/BF16 export)
    uint8_t* mask = nullptr;    // raw mask as given
    uint8_t* band = nullptr;
    uint8_t* flags = nullptr;
    uint32_t* links = nullptr;
    int32_t* dist = nullptr;
    unsigned long long* dcount = nullptr;
    double* partials = nullptr;
    double* stats = nullptr;
    int max_blocks = 0;
    bool use_flags = false;     // any cell is solid / band / duct boundary
    bool any_solid = false;
    bool any_band = false;
    bool stats_on = false;
    bool macro_out = true;      // write rho,u on the last substep of each lbm_step
    int last_stat_blocks = 0;
    int parity = 0;             // AA: 0 natural layout, 1 swapped; reference bounce: 0 A current, 1 B
    int64_t steps = 0;
    lbm::LaunchCfg cfg_even{0, 256}, cfg_odd{0, 256};
    int home_zchunk = 16;
    bool zghost = false;        // z-slab: planes 0 and nz-1 are ghosts, steps cover 1..nz-2
    uint32_t salt_base = 0;     // narrow stores: index of cell 0 in the whole grid
    // graph cache
    cudaGraphExec_t gexec = nullptr;
    int g_sub = 0, g_parity = -1, g_stats = -1;
    // pipelined host I/O (lbm_stage_from_host, lbm_reinit_from_stage, lbm_read_macros_async)
    cudaStream_t copy_stream = nullptr;
    float* stage[2] = {nullptr, nullptr};
    bool stage_has[2][4] = {};
    int stage_next = 0, stage_ready = -1;
    bool stage_inuse[2] = {false, false};
    cudaEvent_t ev_staged[2] = {nullptr, nullptr}, ev_stage_free[2] = {nullptr, nullptr};
    cudaEvent_t ev_macros = nullptr, ev_read = nullptr;
    bool read_pending = false;
    // HOME F16/BF16/F64: the FP32 macro fields are exported from the state after
    // each lbm_step while macro output is on, else when they are next asked for
    bool macros_stale = false;
};

namespace {

#define CK(call)                                                                   \
    do {                                                                           \
        cudaError_t e_ = (call);                                                   \
        if (e_ != cudaSuccess) {                                                   \
            set_error(std::string(#call) + ": " + cudaGetErrorString(e_));         \
            return LBM_ERR_CUDA;                                                   \
        }                                                                          \
    } while (0)

bool is_aa(const lbm_solver* s) { return s->method != LBM_METHOD_HOME; }
// Legacy/Hybrid with the reference's bounce table run the two-buffer push kernel
bool is_ref_push(const lbm_solver* s) { return is_aa(s) && s->bounce == LBM_BOUNCE_REFERENCE; }
void* cur_pop(const lbm_solver* s) { return (is_ref_push(s) && s->parity) ? s->f2 : s->f; }
void* other_pop(const lbm_solver* s) { return (is_ref_push(s) && s->parity) ? s->f : s->f2; }

void drop_graph(lbm_solver* s) {
    if (s->gexec) { cudaGraphExecDestroy(s->gexec); s->gexec = nullptr; }
    s->g_sub = 0; s->g_parity = -1; s->g_stats = -1;
}

// planes a HOME step covers (a z-slab skips its two ghost planes)
int home_planes(const lbm_solver* s) { return s->zghost ? s->dom.nz - 2 : s->dom.nz; }

float* home_macro_base(lbm_solver* s) {
    // F32 HOME exposes its state directly (d_rho() = m + 0*N, home.cu:355-362)
    return s->storage == LBM_STORE_F32 ? static_cast<float*>(s->m[s->cur]) : s->macro;
}

// the macro fields of the current state: AA writes them in the step; HOME in
// another storage than F32 exports them (now, or when they were skipped)
int macro_fields(lbm_solver* s, float** base) {
    if (is_aa(s)) { *base = s->macro; return LBM_OK; }
    if (s->storage != LBM_STORE_F32 && s->macros_stale) {
        CK(lbm::launch_home_macros(s->m[s->cur], s->storage, s->N, s->rho0, s->macro, s->macro + s->N,
                                   s->macro + 2 * s->N, s->macro + 3 * s->N, s->stream));
        s->macros_stale = false;
    }
    *base = home_macro_base(s);
    return LBM_OK;
}

// after a HOME step in another storage than F32: export the macro fields now
// when macro output is on, else mark them for export on demand
int home_after_step(lbm_solver* s) {
    if (is_aa(s) || s->storage == LBM_STORE_F32) return LBM_OK;
    s->macros_stale = true;
    if (!s->macro_out) return LBM_OK;
    float* b = nullptr;
    return macro_fields(s, &b);
}

int rebuild_flags(lbm_solver* s) {
    s->use_flags = s->any_solid || s->bc == LBM_BC_DUCT || (s->method == LBM_METHOD_HYBRID && s->any_band);
    CK(lbm::launch_build_flags(s->any_solid ? s->mask : nullptr,
                               (s->method == LBM_METHOD_HYBRID && s->any_band) ? s->band : nullptr, s->flags,
                               s->links, s->dom.nx, s->dom.ny, s->dom.nz, s->bc == LBM_BC_DUCT, s->stream));
    drop_graph(s);
    return LBM_OK;
}

lbm::AAParams aa_params(lbm_solver* s, bool macro, bool stats) {
    lbm::AAParams p{};
    p.f = cur_pop(s);
    p.N = s->N;
    p.nx = s->dom.nx; p.ny = s->dom.ny; p.nz = s->dom.nz;
    p.flags = s->use_flags ? s->flags : nullptr;
    p.links = s->links;
    p.omega = s->omega;
    p.omega_h = s->omega;
    p.omega_s = s->omega_s;
    p.hybrid = s->method == LBM_METHOD_HYBRID;
    p.fx = s->dom.force_x; p.fy = s->dom.force_y; p.fz = s->dom.force_z;
    p.duct = s->bc == LBM_BC_DUCT;
    p.u_in = s->u_in;
    p.rho0 = s->rho0;
    p.rho = s->macro; p.ux = s->macro + s->N; p.uy = s->macro + 2 * s->N; p.uz = s->macro + 3 * s->N;
    p.macro = macro;
    p.partials = s->partials;
    p.stats = stats;
    const int64_t plane = (int64_t)s->dom.nx * s->dom.ny;
    p.first = s->zghost ? plane : 0;
    p.cells = s->zghost ? s->N - 2 * plane : s->N;
    p.salt_base = s->salt_base;
    return p;
}

lbm::HomeParams home_params(lbm_solver* s, bool stats) {
    lbm::HomeParams p{};
    p.m = s->m[s->cur];
    p.mn = s->m[s->cur ^ 1];
    p.N = s->N;
    p.nx = s->dom.nx; p.ny = s->dom.ny; p.nz = s->dom.nz;
    p.flags = s->use_flags ? s->flags : nullptr;
    p.links = s->links;
    p.omega = s->omega;
    p.fx = s->dom.force_x; p.fy = s->dom.force_y; p.fz = s->dom.force_z;
    p.duct = s->bc == LBM_BC_DUCT;
    p.u_in = s->u_in;
    p.rho0 = s->rho0;
    p.partials = s->partials;
    p.stats = stats;
    p.zchunk = s->home_zchunk;
    p.ref_bounce = s->bounce == LBM_BOUNCE_REFERENCE;
    p.zb = s->zghost ? 1 : 0;
    p.ze = s->zghost ? s->dom.nz - 1 : s->dom.nz;
    p.salt_base = s->salt_base;
    return p;
}

}  // namespace

// queue n substeps (no sync)
// an asynchronous read of the macro fields must finish before they are rewritten
static int wait_pending_read(lbm_solver* s) {
    if (s->read_pending) {
        CK(cudaStreamWaitEvent(s->stream, s->ev_read, 0));
        s->read_pending = false;
    }
    return LBM_OK;
}

static int enqueue_steps(lbm_solver* s, int n) {
    for (int i = 0; i < n; ++i) {
        const bool last = (i == n - 1);
        const bool st = last && s->stats_on;
        const bool mac = last && (s->macro_out || st);
        // HOME's macro fields are its state: every step rewrites one of the two buffers
        if (mac || !is_aa(s)) {
            const int rc = wait_pending_read(s);
            if (rc != LBM_OK) return rc;
        }
        if (is_ref_push(s)) {
            lbm::AAParams p = aa_params(s, mac, st);
            CK(lbm::launch_ref_push(p, static_cast<const float*>(cur_pop(s)), static_cast<float*>(other_pop(s)),
                                    s->cfg_odd, s->stream));
            s->parity ^= 1;
            if (st) s->last_stat_blocks = s->cfg_odd.blocks;
        } else if (is_aa(s)) {
            lbm::AAParams p = aa_params(s, mac, st);
            const lbm::LaunchCfg cfg = s->parity == 0 ? s->cfg_even : s->cfg_odd;
            CK(lbm::launch_aa_step(p, s->storage, s->parity, cfg, s->stream));
            if (st)
                s->last_stat_blocks = s->parity == 0 ? cfg.blocks
                                                     : (int)lbm::aa_odd_grid(p.nx, p.ny, p.cells / ((int64_t)p.nx * p.ny),
                                                                             p.flags != nullptr, s->storage, cfg);
            s->parity ^= 1;
        } else {
            lbm::HomeParams p = home_params(s, st);
            CK(lbm::launch_home_step(p, s->storage, 8, 3, s->stream));
            s->cur ^= 1;
            if (st) s->last_stat_blocks = lbm::home_num_blocks(s->dom.nx, s->dom.ny, home_planes(s), s->home_zchunk);
        }
        if (st) CK(lbm::launch_finalize_stats(s->partials, s->last_stat_blocks, s->stats, s->stream));
    }
    if (n > 0) {
        const int rc = home_after_step(s);
        if (rc != LBM_OK) return rc;
    }
    s->steps += n;
    return LBM_OK;
}

namespace {
// Phase 1 writes back only what the neighbour's cells wrote: slot q of a
// boundary cell c is written by the cell c - c_q when the link between them
// streams, and by c itself (bounce-back, inlet, outlet) when c's link in
// direction opp(q) does not; a solid c is never written.
template <class T>
__global__ void zslab_merge(T* __restrict__ dst, const T* __restrict__ src, const uint8_t* __restrict__ flags,
                            const uint32_t* __restrict__ links, int64_t n, int back_bit) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (flags && ((flags[i] & lbm::F_SOLID) || ((links[i] >> back_bit) & 1u))) continue;
        dst[i] = src[i];
    }
}
}  // namespace

// One launch for every face of a chain of slabs: job j copies (or, with
// flags, merges) one slot plane.  blockIdx.y is the job.
struct SlabJob {
    void* dst;
    const void* src;
    const uint8_t* flags;     // null: plain copy
    const uint32_t* links;
    int64_t n;                // elements
    int back_bit;
    int pad;
};

template <class T>
__global__ void zslab_jobs(const SlabJob* __restrict__ jobs) {
    const SlabJob j = jobs[blockIdx.y];
    T* __restrict__ dst = static_cast<T*>(j.dst);
    const T* __restrict__ src = static_cast<const T*>(j.src);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < j.n; i += (int64_t)gridDim.x * blockDim.x) {
        if (j.flags && ((j.flags[i] & lbm::F_SOLID) || ((j.links[i] >> j.back_bit) & 1u))) continue;
        dst[i] = src[i];
    }
}

static int merge_slots(lbm_solver* s, int plane, int cz, void* const* src, cudaStream_t st) {
    void* dst[5];
    int64_t b = 0;
    int rc = lbm_zslab_slots(s, plane, cz, dst, &b);
    if (rc != LBM_OK) return rc;
    const int64_t pl = (int64_t)s->dom.nx * s->dom.ny;
    const uint8_t* fl = s->use_flags ? s->flags + plane * pl : nullptr;
    const uint32_t* lk = s->links + plane * pl;
    const int blocks = (int)std::min<int64_t>((pl + 255) / 256, 4096);
    int k = 0;
    for (int q = 0; q < 19; ++q) {
        if (lbm::cz(q) != cz) continue;
        if (s->esize == 4)
            zslab_merge<uint32_t><<<blocks, 256, 0, st>>>(static_cast<uint32_t*>(dst[k]),
                                                          static_cast<const uint32_t*>(src[k]), fl, lk, pl, lbm::opp(q));
        else if (s->esize == 8)
            zslab_merge<uint64_t><<<blocks, 256, 0, st>>>(static_cast<uint64_t*>(dst[k]),
                                                          static_cast<const uint64_t*>(src[k]), fl, lk, pl, lbm::opp(q));
        else
            zslab_merge<uint16_t><<<blocks, 256, 0, st>>>(static_cast<uint16_t*>(dst[k]),
                                                          static_cast<const uint16_t*>(src[k]), fl, lk, pl, lbm::opp(q));
        ++k;
    }
    CK(cudaGetLastError());
    return LBM_OK;
}

extern "C" {

const char* lbm_last_error(void) { return lbm::g_error.c_str(); }
const char* lbm_version(void) { return "lbm_b200 0.1 (sm_100a)"; }

int lbm_create(const lbm_domain* dom, const lbm_options* opts, lbm_solver** out) {
    if (!dom || !out) { set_error("lbm_create: null argument"); return LBM_ERR_INVALID; }
    *out = nullptr;
    if (dom->nx < 1 || dom->ny < 1 || dom->nz < 1) { set_error("lbm_create: dimensions must be >= 1"); return LBM_ERR_INVALID; }
    if (!(dom->tau > 0.5f)) { set_error("lbm_create: tau must be > 0.5"); return LBM_ERR_INVALID; }
    lbm_options o{};
    o.rho0 = 1.0f;
    if (opts) o = *opts;
    if (o.method < 0 || o.method > 2) { set_error("lbm_create: bad method"); return LBM_ERR_INVALID; }
    if (o.storage < 0 || o.storage > 3) { set_error("lbm_create: bad storage"); return LBM_ERR_INVALID; }
    if (o.storage == LBM_STORE_F64 && o.method != LBM_METHOD_HOME && o.bounce == LBM_BOUNCE_REFERENCE) {
        set_error("lbm_create: FP64 storage runs Legacy/Hybrid with halfway bounce-back only");
        return LBM_ERR_UNSUPPORTED;
    }
    if (o.bc < 0 || o.bc > 1) { set_error("lbm_create: bad boundary"); return LBM_ERR_INVALID; }
    if (o.bc == LBM_BC_DUCT && dom->nx < 3) { set_error("lbm_create: a duct needs nx >= 3"); return LBM_ERR_INVALID; }
    if (o.bounce < 0 || o.bounce > 1) { set_error("lbm_create: bad bounce mode"); return LBM_ERR_INVALID; }
    if (o.bounce == LBM_BOUNCE_REFERENCE && o.method != LBM_METHOD_HOME && o.storage != LBM_STORE_F32) {
        set_error("lbm_create: the reference bounce table runs Legacy/Hybrid in F32 storage only");
        return LBM_ERR_UNSUPPORTED;
    }
    const int64_t N = (int64_t)dom->nx * dom->ny * dom->nz;
    // every population index q*N + id and every plane offset stays in int64;
    // the per-row x index and the row counts stay in int
    if (N > ((int64_t)1 << 40) || (int64_t)dom->ny * dom->nz > ((int64_t)1 << 31) - 1) {
        set_error("lbm_create: grid too large");
        return LBM_ERR_SIZE;
    }
    lbm_solver* s = new lbm_solver();
    s->dom = *dom;
    s->method = o.method; s->storage = o.storage; s->bc = o.bc; s->bounce = o.bounce;
    s->u_in = o.inlet_u;
    s->rho0 = (o.rho0 > 0.f) ? o.rho0 : 1.0f;
    s->omega = 1.0f / dom->tau;
    s->omega_s = s->omega;
    s->N = N;
    s->esize = o.storage == LBM_STORE_F32 ? 4 : (o.storage == LBM_STORE_F64 ? 8 : 2);
    auto fail = [&](int code) { lbm_destroy(s); return code; };
    if (o.stream) s->stream = static_cast<cudaStream_t>(o.stream);
    else {
        // a blocking stream: ordered with work on the legacy default stream, which
        // is where the reference's callers (and torch by default) produce inputs
        if (cudaStreamCreate(&s->stream) != cudaSuccess) {
            set_error("lbm_create: cudaStreamCreate failed");
            delete s;
            return LBM_ERR_CUDA;
        }
        s->own_stream = true;
    }
    const int sms = lbm::num_sms();
    s->cfg_even = {sms * 8, 256};
    s->cfg_odd = {sms * 12, 256};
    // HOME: the longest z-chunk (fewest re-built halo planes) that still gives
    // three waves of resident blocks, so the tail of the last wave stays short
    if (o.method == LBM_METHOD_HOME) {
        static const int bps = lbm::home_blocks_per_sm();
        int zc = 4;
        for (int c : {48, 32, 24, 16, 12, 10, 8, 6, 4}) {
            if ((int64_t)lbm::home_num_blocks(dom->nx, dom->ny, dom->nz, std::min(c, dom->nz)) >=
                (int64_t)sms * bps * 3) {
                zc = c;
                break;
            }
        }
        s->home_zchunk = std::min(zc, dom->nz);
    }
    // the z-marching odd step's grid (solvers without a mask)
    const int64_t odd_blocks = lbm::aa_odd_blocks(dom->nx, dom->ny, dom->nz, false, o.storage, s->cfg_odd.threads);
    s->max_blocks = (int)std::max<int64_t>({s->cfg_even.blocks, s->cfg_odd.blocks, odd_blocks,
                                            lbm::home_num_blocks(dom->nx, dom->ny, dom->nz, s->home_zchunk), 1});
    auto dmalloc = [&](void** p, size_t b) { return cudaMalloc(p, b) == cudaSuccess; };
    bool ok = true;
    if (is_aa(s)) ok = ok && dmalloc(&s->f, s->esize * 19 * (size_t)N);
    if (is_ref_push(s)) ok = ok && dmalloc(&s->f2, s->esize * 19 * (size_t)N);
    else ok = ok && dmalloc(&s->m[0], s->esize * 10 * (size_t)N) && dmalloc(&s->m[1], s->esize * 10 * (size_t)N);
    if (is_aa(s) || s->storage != LBM_STORE_F32) ok = ok && dmalloc((void**)&s->macro, sizeof(float) * 4 * (size_t)N);
    ok = ok && dmalloc((void**)&s->mask, (size_t)N) && dmalloc((void**)&s->band, (size_t)N) &&
         dmalloc((void**)&s->flags, (size_t)N) && dmalloc((void**)&s->links, sizeof(uint32_t) * (size_t)N) &&
         dmalloc((void**)&s->partials, sizeof(double) * lbm::NSTAT * (size_t)s->max_blocks) &&
         dmalloc((void**)&s->stats, sizeof(double) * lbm::NSTAT) &&
         dmalloc((void**)&s->dcount, sizeof(unsigned long long));
    if (!ok) {
        set_error("lbm_create: device allocation failed (" + std::to_string(N) + " cells)");
        return fail(LBM_ERR_ALLOC);
    }
    if (cudaMemsetAsync(s->mask, 0, (size_t)N, s->stream) != cudaSuccess ||
        cudaMemsetAsync(s->band, 0, (size_t)N, s->stream) != cudaSuccess ||
        cudaMemsetAsync(s->stats, 0, sizeof(double) * lbm::NSTAT, s->stream) != cudaSuccess ||
        (s->f2 && cudaMemsetAsync(s->f2, 0, s->esize * 19 * (size_t)N, s->stream) != cudaSuccess)) {
        set_error("lbm_create: cudaMemset failed");
        return fail(LBM_ERR_CUDA);
    }
    if (!is_aa(s) && lbm::home_prepare() != cudaSuccess) {
        set_error("lbm_create: cannot set the HOME kernel's shared-memory size");
        return fail(LBM_ERR_CUDA);
    }
    int rc = rebuild_flags(s);
    if (rc == LBM_OK) rc = lbm_reset(s);
    if (rc != LBM_OK) return fail(rc);
    *out = s;
    return LBM_OK;
}

int lbm_destroy(lbm_solver* s) {
    if (!s) return LBM_OK;
    if (s->stream) cudaStreamSynchronize(s->stream);
    drop_graph(s);
    cudaFree(s->f); cudaFree(s->f2); cudaFree(s->m[0]); cudaFree(s->m[1]); cudaFree(s->macro);
    cudaFree(s->mask); cudaFree(s->band); cudaFree(s->flags); cudaFree(s->links);
    cudaFree(s->dist); cudaFree(s->dcount); cudaFree(s->partials); cudaFree(s->stats);
    if (s->copy_stream) cudaStreamSynchronize(s->copy_stream);
    cudaFree(s->stage[0]); cudaFree(s->stage[1]);
    for (cudaEvent_t e : {s->ev_staged[0], s->ev_staged[1], s->ev_stage_free[0], s->ev_stage_free[1], s->ev_macros,
                          s->ev_read})
        if (e) cudaEventDestroy(e);
    if (s->copy_stream) cudaStreamDestroy(s->copy_stream);
    if (s->own_stream && s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return LBM_OK;
}

int lbm_set_solid_mask(lbm_solver* s, const uint8_t* host_mask) {
    if (!s || !host_mask) { set_error("lbm_set_solid_mask: null argument"); return LBM_ERR_INVALID; }
    s->any_solid = false;
    for (int64_t i = 0; i < s->N; ++i)
        if (host_mask[i]) { s->any_solid = true; break; }
    CK(cudaMemcpyAsync(s->mask, host_mask, (size_t)s->N, cudaMemcpyHostToDevice, s->stream));
    CK(cudaStreamSynchronize(s->stream));   // host_mask may be released after return, as in the reference
    return rebuild_flags(s);
}

int lbm_set_legacy_mapping(lbm_solver* s, const uint8_t* host_is_legacy) {
    if (!s) { set_error("lbm_set_legacy_mapping: null solver"); return LBM_ERR_INVALID; }
    if (s->method != LBM_METHOD_HYBRID) { set_error("lbm_set_legacy_mapping: Hybrid only"); return LBM_ERR_INVALID; }
    s->any_band = false;
    if (host_is_legacy) {
        for (int64_t i = 0; i < s->N; ++i)
            if (host_is_legacy[i]) { s->any_band = true; break; }
        CK(cudaMemcpyAsync(s->band, host_is_legacy, (size_t)s->N, cudaMemcpyHostToDevice, s->stream));
        CK(cudaStreamSynchronize(s->stream));
    } else {
        CK(cudaMemsetAsync(s->band, 0, (size_t)s->N, s->stream));
    }
    return rebuild_flags(s);
}

int lbm_build_band(lbm_solver* s, int d0, int64_t* n_band) {
    if (!s) { set_error("lbm_build_band: null solver"); return LBM_ERR_INVALID; }
    if (s->method != LBM_METHOD_HYBRID) { set_error("lbm_build_band: Hybrid only"); return LBM_ERR_INVALID; }
    if (!s->dist && cudaMalloc((void**)&s->dist, sizeof(int32_t) * (size_t)s->N) != cudaSuccess) {
        set_error("lbm_build_band: allocation failed");
        return LBM_ERR_ALLOC;
    }
    CK(lbm::launch_band(s->mask, s->dist, s->band, s->dom.nx, s->dom.ny, s->dom.nz, d0 < 0 ? 0 : d0, s->dcount,
                        s->stream));
    unsigned long long c = 0;
    CK(cudaMemcpyAsync(&c, s->dcount, sizeof(c), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    s->any_band = c > 0;
    if (n_band) *n_band = (int64_t)c;
    return rebuild_flags(s);
}

int lbm_get_band(lbm_solver* s, uint8_t* out) {
    if (!s || !out) { set_error("lbm_get_band: null argument"); return LBM_ERR_INVALID; }
    CK(cudaMemcpyAsync(out, s->band, (size_t)s->N, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return LBM_OK;
}

int lbm_reset(lbm_solver* s) { return lbm_reinit_from_macro(s, nullptr, nullptr, nullptr, nullptr); }

static int reinit_impl(lbm_solver* s, const float* d_rho, const float* d_ux, const float* d_uy, const float* d_uz,
                       bool write_macros);

int lbm_reinit_from_macro(lbm_solver* s, const float* d_rho, const float* d_ux, const float* d_uy,
                          const float* d_uz) {
    if (!s) { set_error("lbm_reinit_from_macro: null solver"); return LBM_ERR_INVALID; }
    const int rc = wait_pending_read(s);
    if (rc != LBM_OK) return rc;
    return reinit_impl(s, d_rho, d_ux, d_uy, d_uz, true);
}

static int reinit_impl(lbm_solver* s, const float* d_rho, const float* d_ux, const float* d_uy, const float* d_uz,
                       bool write_macros) {
    if (is_aa(s)) {
        // Legacy with no rho resets to rho=1, u=0 (legacy.cu:174-178): the same
        // state as feq(1, 0); Hybrid uses rho=1 and the given u (hybrid.cu:76-79).
        if (s->method == LBM_METHOD_LEGACY && !d_rho) d_ux = d_uy = d_uz = nullptr;
        const int form = s->method == LBM_METHOD_LEGACY ? (d_rho ? 0 : 1) : 1;
        void* dst = cur_pop(s);
        float* mo = write_macros ? s->macro : nullptr;
        CK(lbm::launch_aa_reinit(dst, s->storage, s->rho0, s->N, d_rho, d_ux, d_uy, d_uz, mo,
                                 mo ? mo + s->N : nullptr, mo ? mo + 2 * s->N : nullptr, mo ? mo + 3 * s->N : nullptr,
                                 form, s->stream));
        if (is_ref_push(s)) {
            // the reference's Legacy copies f into fnext after reinitialising
            // (legacy.cu:204-206); its reset (null rho) and Hybrid's reinit leave
            // the second buffer as it was
            if (s->method == LBM_METHOD_LEGACY && d_rho)
                CK(cudaMemcpyAsync(other_pop(s), dst, s->esize * 19 * (size_t)s->N, cudaMemcpyDeviceToDevice,
                                   s->stream));
        } else {
            s->parity = 0;
        }
    } else {
        CK(lbm::launch_home_reinit(s->m[0], s->m[1], s->storage, s->rho0, s->N, d_rho, d_ux, d_uy, d_uz, s->stream));
        s->cur = 0;
        if (s->storage != LBM_STORE_F32) {
            s->macros_stale = false;
            CK(lbm::launch_home_macros(s->m[0], s->storage, s->N, s->rho0, s->macro, s->macro + s->N,
                                       s->macro + 2 * s->N, s->macro + 3 * s->N, s->stream));
        }
    }
    s->steps = 0;
    drop_graph(s);
    return LBM_OK;
}

int lbm_reinit_from_host(lbm_solver* s, const float* rho, const float* ux, const float* uy, const float* uz) {
    if (!s) { set_error("lbm_reinit_from_host: null solver"); return LBM_ERR_INVALID; }
    {
        const int rc = wait_pending_read(s);   // the macro buffers are the staging area here
        if (rc != LBM_OK) return rc;
    }
    // stage through the solver's own buffers: AA macro fields, or HOME's next buffer
    float* stage = is_aa(s) ? s->macro : nullptr;
    float* tmp = nullptr;
    if (!stage) {
        if (cudaMallocAsync((void**)&tmp, sizeof(float) * 4 * (size_t)s->N, s->stream) != cudaSuccess) {
            set_error("lbm_reinit_from_host: allocation failed");
            return LBM_ERR_ALLOC;
        }
        stage = tmp;
    }
    const float* src[4] = {rho, ux, uy, uz};
    const float* dptr[4] = {nullptr, nullptr, nullptr, nullptr};
    for (int k = 0; k < 4; ++k) {
        if (!src[k]) continue;
        CK(cudaMemcpyAsync(stage + k * s->N, src[k], sizeof(float) * (size_t)s->N, cudaMemcpyHostToDevice, s->stream));
        dptr[k] = stage + k * s->N;
    }
    const int rc = lbm_reinit_from_macro(s, dptr[0], dptr[1], dptr[2], dptr[3]);
    if (tmp) cudaFreeAsync(tmp, s->stream);
    return rc;
}

static int ensure_copy_path(lbm_solver* s) {
    if (s->copy_stream) return LBM_OK;
    CK(cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking));
    for (int k = 0; k < 2; ++k) {
        CK(cudaEventCreateWithFlags(&s->ev_staged[k], cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&s->ev_stage_free[k], cudaEventDisableTiming));
    }
    CK(cudaEventCreateWithFlags(&s->ev_macros, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&s->ev_read, cudaEventDisableTiming));
    return LBM_OK;
}

int lbm_stage_from_host(lbm_solver* s, const float* rho, const float* ux, const float* uy, const float* uz) {
    if (!s) { set_error("lbm_stage_from_host: null solver"); return LBM_ERR_INVALID; }
    int rc = ensure_copy_path(s);
    if (rc != LBM_OK) return rc;
    const int k = s->stage_next;
    if (!s->stage[k]) CK(cudaMalloc((void**)&s->stage[k], sizeof(float) * 4 * (size_t)s->N));
    // the reinit that last read this buffer must be done with it
    if (s->stage_inuse[k]) CK(cudaStreamWaitEvent(s->copy_stream, s->ev_stage_free[k], 0));
    const float* src[4] = {rho, ux, uy, uz};
    for (int c = 0; c < 4; ++c) {
        s->stage_has[k][c] = src[c] != nullptr;
        if (src[c])
            CK(cudaMemcpyAsync(s->stage[k] + c * s->N, src[c], sizeof(float) * (size_t)s->N, cudaMemcpyHostToDevice,
                               s->copy_stream));
    }
    CK(cudaEventRecord(s->ev_staged[k], s->copy_stream));
    s->stage_ready = k;
    s->stage_next ^= 1;
    return LBM_OK;
}

int lbm_reinit_from_stage(lbm_solver* s) {
    if (!s) { set_error("lbm_reinit_from_stage: null solver"); return LBM_ERR_INVALID; }
    if (s->stage_ready < 0) { set_error("lbm_reinit_from_stage: nothing staged"); return LBM_ERR_INVALID; }
    const int k = s->stage_ready;
    CK(cudaStreamWaitEvent(s->stream, s->ev_staged[k], 0));
    // Legacy/Hybrid leave the macro fields to the next step (so a read of the
    // previous step's fields may still be in flight); HOME's state is rewritten
    if (!is_aa(s)) {
        const int rc = wait_pending_read(s);
        if (rc != LBM_OK) return rc;
    }
    const float* d[4];
    for (int c = 0; c < 4; ++c) d[c] = s->stage_has[k][c] ? s->stage[k] + c * s->N : nullptr;
    const int rc = reinit_impl(s, d[0], d[1], d[2], d[3], !is_aa(s));
    if (rc != LBM_OK) return rc;
    CK(cudaEventRecord(s->ev_stage_free[k], s->stream));
    s->stage_inuse[k] = true;
    s->stage_ready = -1;
    return LBM_OK;
}

int lbm_read_macros_async(lbm_solver* s, float* rho, float* ux, float* uy, float* uz) {
    if (!s) { set_error("lbm_read_macros_async: null solver"); return LBM_ERR_INVALID; }
    int rc = ensure_copy_path(s);
    if (rc != LBM_OK) return rc;
    rc = wait_pending_read(s);   // one read in flight at a time
    if (rc != LBM_OK) return rc;
    float* b = nullptr;
    if ((rc = macro_fields(s, &b)) != LBM_OK) return rc;
    CK(cudaEventRecord(s->ev_macros, s->stream));
    CK(cudaStreamWaitEvent(s->copy_stream, s->ev_macros, 0));
    float* dst[4] = {rho, ux, uy, uz};
    for (int c = 0; c < 4; ++c)
        if (dst[c])
            CK(cudaMemcpyAsync(dst[c], b + c * s->N, sizeof(float) * (size_t)s->N, cudaMemcpyDeviceToHost,
                               s->copy_stream));
    CK(cudaEventRecord(s->ev_read, s->copy_stream));
    s->read_pending = true;
    return LBM_OK;
}

int lbm_wait_reads(lbm_solver* s) {
    if (!s) { set_error("lbm_wait_reads: null solver"); return LBM_ERR_INVALID; }
    if (s->copy_stream) CK(cudaStreamSynchronize(s->copy_stream));
    return LBM_OK;
}

int lbm_step(lbm_solver* s, int substeps) {
    if (!s) { set_error("lbm_step: null solver"); return LBM_ERR_INVALID; }
    if (substeps < 0) { set_error("lbm_step: negative substeps"); return LBM_ERR_INVALID; }
    return enqueue_steps(s, substeps);
}

int lbm_step_graph(lbm_solver* s, int substeps) {
    if (!s) { set_error("lbm_step_graph: null solver"); return LBM_ERR_INVALID; }
    if (substeps <= 0) return lbm_step(s, substeps);
    // A read-back queued on the copy stream (lbm_read_macros_async,
    // lbm_get_stats_async) must end before the replayed steps rewrite the macro
    // fields, the statistics or HOME's moment buffers.  The wait goes on the
    // solver's stream before every launch, outside the graph: the read's event
    // was recorded outside any capture, so it cannot be waited on inside one.
    // Once waited for, read_pending is clear, so a capture below queues no wait.
    {
        const int rc = wait_pending_read(s);
        if (rc != LBM_OK) return rc;
    }
    const int par = is_aa(s) ? s->parity : s->cur;
    if (!s->gexec || s->g_sub != substeps || s->g_parity != par || s->g_stats != (int)s->stats_on) {
        drop_graph(s);
        const int saved_par = s->parity, saved_cur = s->cur;
        const int64_t saved_steps = s->steps;
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
        const int rc = enqueue_steps(s, substeps);
        cudaError_t e = cudaStreamEndCapture(s->stream, &g);
        s->parity = saved_par; s->cur = saved_cur; s->steps = saved_steps;
        if (rc != LBM_OK) { if (g) cudaGraphDestroy(g); return rc; }
        if (e != cudaSuccess) { set_error(std::string("graph capture: ") + cudaGetErrorString(e)); return LBM_ERR_CUDA; }
        e = cudaGraphInstantiate(&s->gexec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) { set_error(std::string("graph instantiate: ") + cudaGetErrorString(e)); return LBM_ERR_CUDA; }
        s->g_sub = substeps; s->g_parity = par; s->g_stats = s->stats_on;
    }
    CK(cudaGraphLaunch(s->gexec, s->stream));
    // advance the host-side state exactly as enqueue_steps would
    if (is_aa(s)) s->parity ^= (substeps & 1);
    else s->cur ^= (substeps & 1);
    if (!is_aa(s) && s->storage != LBM_STORE_F32) s->macros_stale = !s->macro_out;
    s->steps += substeps;
    return LBM_OK;
}

int lbm_synchronize(lbm_solver* s) {
    if (!s) { set_error("lbm_synchronize: null solver"); return LBM_ERR_INVALID; }
    CK(cudaStreamSynchronize(s->stream));
    if (s->copy_stream) CK(cudaStreamSynchronize(s->copy_stream));
    return LBM_OK;
}

int lbm_set_force(lbm_solver* s, float fx, float fy, float fz) {
    if (!s) { set_error("lbm_set_force: null solver"); return LBM_ERR_INVALID; }
    s->dom.force_x = fx; s->dom.force_y = fy; s->dom.force_z = fz;
    drop_graph(s);
    return LBM_OK;
}

int lbm_set_shear_omega(lbm_solver* s, float omega_shear) {
    if (!s) { set_error("lbm_set_shear_omega: null solver"); return LBM_ERR_INVALID; }
    if (s->method != LBM_METHOD_HYBRID) { set_error("lbm_set_shear_omega: Hybrid only"); return LBM_ERR_INVALID; }
    s->omega_s = omega_shear;
    drop_graph(s);
    return LBM_OK;
}

int lbm_set_home_zchunk(lbm_solver* s, int zchunk) {
    if (!s) { set_error("lbm_set_home_zchunk: null solver"); return LBM_ERR_INVALID; }
    if (s->method != LBM_METHOD_HOME) { set_error("lbm_set_home_zchunk: HOME only"); return LBM_ERR_INVALID; }
    if (zchunk < 1) { set_error("lbm_set_home_zchunk: zchunk must be >= 1"); return LBM_ERR_INVALID; }
    const int z = std::min(zchunk, s->dom.nz);
    const int need = lbm::home_num_blocks(s->dom.nx, s->dom.ny, home_planes(s), z);
    if (need > s->max_blocks) {
        // per-block statistics partials: grow once the step queue has drained
        CK(cudaStreamSynchronize(s->stream));
        double* p = nullptr;
        if (cudaMalloc((void**)&p, sizeof(double) * lbm::NSTAT * (size_t)need) != cudaSuccess) {
            set_error("lbm_set_home_zchunk: device allocation failed");
            return LBM_ERR_ALLOC;
        }
        cudaFree(s->partials);
        s->partials = p;
        s->max_blocks = need;
    }
    s->home_zchunk = z;
    drop_graph(s);
    return LBM_OK;
}

// ---- z-slab decomposition ---------------------------------------------------
//
// A slab solver holds its interior planes 1..nz-2 and one ghost plane at each
// end.  The even AA step is local.  In the odd step the slots of plane k with
// c_z = -1 are read and rewritten only by the cells of plane k+1, and those with
// c_z = +1 only by the cells of plane k-1.  So around each odd step the 5 slot
// planes that cross a slab face travel to the neighbour's ghost plane (phase 0)
// and, after it, back into the owner's boundary plane (phase 1).  Nothing else
// is exchanged.


int lbm_set_z_ghosts(lbm_solver* s, int on) {
    if (!s) { set_error("lbm_set_z_ghosts: null solver"); return LBM_ERR_INVALID; }
    if (is_ref_push(s)) {
        set_error("lbm_set_z_ghosts: not for Legacy/Hybrid with the reference's bounce table (two-buffer push)");
        return LBM_ERR_UNSUPPORTED;
    }
    if (on && s->dom.nz < 3) { set_error("lbm_set_z_ghosts: needs nz >= 3 (two ghost planes)"); return LBM_ERR_INVALID; }
    s->zghost = on != 0;
    drop_graph(s);
    return LBM_OK;
}

int lbm_zslab_slots(lbm_solver* s, int plane, int cz, void** ptrs, int64_t* bytes) {
    if (!s || !ptrs || !bytes || (cz != 1 && cz != -1) || plane < 0 || plane >= s->dom.nz) {
        set_error("lbm_zslab_slots: bad argument");
        return LBM_ERR_INVALID;
    }
    if (!is_aa(s) || is_ref_push(s)) { set_error("lbm_zslab_slots: AA solvers only"); return LBM_ERR_UNSUPPORTED; }
    const int64_t pl = (int64_t)s->dom.nx * s->dom.ny;
    char* base = static_cast<char*>(s->f);
    int k = 0;
    for (int q = 0; q < 19; ++q)     // the 5 directions with c_z = cz, in index order
        if (lbm::cz(q) == cz) ptrs[k++] = base + s->esize * ((int64_t)q * s->N + (int64_t)plane * pl);
    *bytes = (int64_t)s->esize * pl;
    return LBM_OK;
}

int lbm_zslab_moment_planes(lbm_solver* s, int plane, void** ptrs, int64_t* bytes) {
    if (!s || !ptrs || !bytes || plane < 0 || plane >= s->dom.nz) {
        set_error("lbm_zslab_moment_planes: bad argument");
        return LBM_ERR_INVALID;
    }
    if (is_aa(s)) { set_error("lbm_zslab_moment_planes: HOME solvers only"); return LBM_ERR_UNSUPPORTED; }
    const int64_t pl = (int64_t)s->dom.nx * s->dom.ny;
    char* base = static_cast<char*>(s->m[s->cur]);
    for (int c = 0; c < 10; ++c) ptrs[c] = base + s->esize * ((int64_t)c * s->N + (int64_t)plane * pl);
    *bytes = (int64_t)s->esize * pl;
    return LBM_OK;
}

int lbm_zslab_step_planes(lbm_solver* s, int z_begin, int z_end, int finish) {
    if (!s) { set_error("lbm_zslab_step_planes: null solver"); return LBM_ERR_INVALID; }
    if (!s->zghost) { set_error("lbm_zslab_step_planes: a z-slab solver (lbm_set_z_ghosts) only"); return LBM_ERR_INVALID; }
    if (is_ref_push(s)) { set_error("lbm_zslab_step_planes: not for the reference bounce table"); return LBM_ERR_UNSUPPORTED; }
    if (z_begin < 1 || z_end > s->dom.nz - 1 || z_begin > z_end) {
        set_error("lbm_zslab_step_planes: planes must satisfy 1 <= z_begin <= z_end <= nz-1");
        return LBM_ERR_INVALID;
    }
    if (z_end > z_begin) {
        if (is_aa(s)) {
            lbm::AAParams p = aa_params(s, false, false);
            const int64_t plane = (int64_t)s->dom.nx * s->dom.ny;
            p.first = (int64_t)z_begin * plane;
            p.cells = (int64_t)(z_end - z_begin) * plane;
            CK(lbm::launch_aa_step(p, s->storage, s->parity, s->parity == 0 ? s->cfg_even : s->cfg_odd, s->stream));
        } else {
            const int rc = wait_pending_read(s);   // HOME's buffers are its macro fields
            if (rc != LBM_OK) return rc;
            lbm::HomeParams p = home_params(s, false);
            p.zb = z_begin;
            p.ze = z_end;
            CK(lbm::launch_home_step(p, s->storage, 8, 3, s->stream));
        }
    }
    if (finish) {
        if (is_aa(s)) {
            s->parity ^= 1;
        } else {
            s->cur ^= 1;
            const int rc = home_after_step(s);
            if (rc != LBM_OK) return rc;
        }
        s->steps += 1;
    }
    return LBM_OK;
}

int lbm_set_index_base(lbm_solver* s, int64_t base) {
    if (!s) { set_error("lbm_set_index_base: null solver"); return LBM_ERR_INVALID; }
    s->salt_base = (uint32_t)(uint64_t)base;
    drop_graph(s);
    return LBM_OK;
}

int lbm_zslab_exchange(lbm_solver* lower, lbm_solver* upper, int phase, void* stream) {
    if (!lower || !upper || (phase != 0 && phase != 1)) { set_error("lbm_zslab_exchange: bad argument"); return LBM_ERR_INVALID; }
    if (!lower->zghost || !upper->zghost || lower->dom.nx != upper->dom.nx || lower->dom.ny != upper->dom.ny ||
        lower->storage != upper->storage || is_aa(lower) != is_aa(upper)) {
        set_error("lbm_zslab_exchange: needs two z-slab solvers of the same method family, x-y size and storage");
        return LBM_ERR_INVALID;
    }
    if (!is_aa(lower)) {
        // HOME pulls whole planes of moments: before each step the boundary
        // planes of the current buffer go to the neighbours' ghosts; nothing
        // comes back after it
        if (phase == 1) return LBM_OK;
        void *lo_top[10], *lo_ghost[10], *up_ghost[10], *up_bot[10];
        int64_t b = 0;
        int rc;
        if ((rc = lbm_zslab_moment_planes(lower, lower->dom.nz - 2, lo_top, &b)) != LBM_OK ||
            (rc = lbm_zslab_moment_planes(lower, lower->dom.nz - 1, lo_ghost, &b)) != LBM_OK ||
            (rc = lbm_zslab_moment_planes(upper, 0, up_ghost, &b)) != LBM_OK ||
            (rc = lbm_zslab_moment_planes(upper, 1, up_bot, &b)) != LBM_OK)
            return rc;
        const cudaStream_t st = static_cast<cudaStream_t>(stream);
        for (int c = 0; c < 10; ++c) {
            CK(cudaMemcpyAsync(up_ghost[c], lo_top[c], (size_t)b, cudaMemcpyDeviceToDevice, st));
            CK(cudaMemcpyAsync(lo_ghost[c], up_bot[c], (size_t)b, cudaMemcpyDeviceToDevice, st));
        }
        return LBM_OK;
    }
    void *lo_top[5], *lo_ghost[5], *up_ghost[5], *up_bot[5];
    int64_t b = 0;
    int rc;
    if ((rc = lbm_zslab_slots(lower, lower->dom.nz - 2, -1, lo_top, &b)) != LBM_OK ||
        (rc = lbm_zslab_slots(lower, lower->dom.nz - 1, 1, lo_ghost, &b)) != LBM_OK ||
        (rc = lbm_zslab_slots(upper, 0, -1, up_ghost, &b)) != LBM_OK ||
        (rc = lbm_zslab_slots(upper, 1, 1, up_bot, &b)) != LBM_OK)
        return rc;
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (phase == 0) {   // boundary planes -> the neighbour's ghosts
        for (int k = 0; k < 5; ++k) {
            CK(cudaMemcpyAsync(up_ghost[k], lo_top[k], (size_t)b, cudaMemcpyDeviceToDevice, st));
            CK(cudaMemcpyAsync(lo_ghost[k], up_bot[k], (size_t)b, cudaMemcpyDeviceToDevice, st));
        }
        return LBM_OK;
    }
    // what the odd step streamed into the ghosts -> their owners
    if ((rc = merge_slots(lower, lower->dom.nz - 2, -1, up_ghost, st)) != LBM_OK) return rc;
    return merge_slots(upper, 1, 1, lo_ghost, st);
}

int lbm_zslab_merge(lbm_solver* s, int plane, int cz, void* const* src, void* stream) {
    if (!s || !src || (cz != 1 && cz != -1)) { set_error("lbm_zslab_merge: bad argument"); return LBM_ERR_INVALID; }
    if (!s->zghost) { set_error("lbm_zslab_merge: not a z-slab solver"); return LBM_ERR_INVALID; }
    return merge_slots(s, plane, cz, src, static_cast<cudaStream_t>(stream));
}

struct lbm_zslab_plan {
    SlabJob* d_jobs[2] = {nullptr, nullptr};   // phase 0 copies, phase 1 merges
    int njobs = 0;
    int esize = 4;
    int64_t elems = 0;
};

int lbm_zslab_plan_create(lbm_solver* const* slabs, int32_t n, lbm_zslab_plan** out) {
    if (!slabs || n < 1 || !out) { set_error("lbm_zslab_plan_create: bad argument"); return LBM_ERR_INVALID; }
    for (int k = 0; k < n; ++k) {
        const lbm_solver* a = slabs[k];
        if (!a || !a->zghost || a->dom.nx != slabs[0]->dom.nx || a->dom.ny != slabs[0]->dom.ny ||
            a->storage != slabs[0]->storage) {
            set_error("lbm_zslab_plan_create: needs z-slab solvers of one x-y size and storage");
            return LBM_ERR_INVALID;
        }
        if (!is_aa(a)) {
            set_error("lbm_zslab_plan_create: Legacy/Hybrid slabs only (HOME uses lbm_zslab_exchange)");
            return LBM_ERR_UNSUPPORTED;
        }
    }
    const int64_t pl = (int64_t)slabs[0]->dom.nx * slabs[0]->dom.ny;
    std::vector<SlabJob> jobs[2];
    for (int k = 0; k < n; ++k) {
        lbm_solver* lo = slabs[k];
        lbm_solver* up = slabs[(k + 1) % n];
        void *lo_top[5], *lo_ghost[5], *up_ghost[5], *up_bot[5];
        int64_t b = 0;
        int rc;
        if ((rc = lbm_zslab_slots(lo, lo->dom.nz - 2, -1, lo_top, &b)) != LBM_OK ||
            (rc = lbm_zslab_slots(lo, lo->dom.nz - 1, 1, lo_ghost, &b)) != LBM_OK ||
            (rc = lbm_zslab_slots(up, 0, -1, up_ghost, &b)) != LBM_OK ||
            (rc = lbm_zslab_slots(up, 1, 1, up_bot, &b)) != LBM_OK)
            return rc;
        const int64_t lo_off = (int64_t)(lo->dom.nz - 2) * pl, up_off = pl;
        int kd = 0, ku = 0;
        for (int q = 0; q < 19; ++q) {
            if (lbm::cz(q) == -1) {
                jobs[0].push_back({up_ghost[kd], lo_top[kd], nullptr, nullptr, pl, 0, 0});
                jobs[1].push_back({lo_top[kd], up_ghost[kd], lo->use_flags ? lo->flags + lo_off : nullptr,
                                   lo->links + lo_off, pl, lbm::opp(q), 0});
                ++kd;
            } else if (lbm::cz(q) == 1) {
                jobs[0].push_back({lo_ghost[ku], up_bot[ku], nullptr, nullptr, pl, 0, 0});
                jobs[1].push_back({up_bot[ku], lo_ghost[ku], up->use_flags ? up->flags + up_off : nullptr,
                                   up->links + up_off, pl, lbm::opp(q), 0});
                ++ku;
            }
        }
    }
    auto* p = new lbm_zslab_plan();
    p->njobs = (int)jobs[0].size();
    p->esize = (int)slabs[0]->esize;
    p->elems = pl;
    for (int ph = 0; ph < 2; ++ph) {
        if (cudaMalloc((void**)&p->d_jobs[ph], sizeof(SlabJob) * jobs[ph].size()) != cudaSuccess ||
            cudaMemcpy(p->d_jobs[ph], jobs[ph].data(), sizeof(SlabJob) * jobs[ph].size(), cudaMemcpyHostToDevice) !=
                cudaSuccess) {
            lbm_zslab_plan_destroy(p);
            set_error("lbm_zslab_plan_create: allocation failed");
            return LBM_ERR_ALLOC;
        }
    }
    *out = p;
    return LBM_OK;
}

int lbm_zslab_plan_exchange(lbm_zslab_plan* p, int phase, void* stream) {
    if (!p || (phase != 0 && phase != 1)) { set_error("lbm_zslab_plan_exchange: bad argument"); return LBM_ERR_INVALID; }
    const dim3 grid((unsigned)std::min<int64_t>((p->elems + 255) / 256, 1024), (unsigned)p->njobs);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (p->esize == 4) zslab_jobs<uint32_t><<<grid, 256, 0, st>>>(p->d_jobs[phase]);
    else if (p->esize == 8) zslab_jobs<uint64_t><<<grid, 256, 0, st>>>(p->d_jobs[phase]);
    else zslab_jobs<uint16_t><<<grid, 256, 0, st>>>(p->d_jobs[phase]);
    CK(cudaGetLastError());
    return LBM_OK;
}

int lbm_zslab_plan_destroy(lbm_zslab_plan* p) {
    if (!p) return LBM_OK;
    cudaFree(p->d_jobs[0]);
    cudaFree(p->d_jobs[1]);
    delete p;
    return LBM_OK;
}

int lbm_step_parity(lbm_solver* s, int* parity) {
    if (!s || !parity) { set_error("lbm_step_parity: null argument"); return LBM_ERR_INVALID; }
    *parity = s->parity;
    return LBM_OK;
}

int lbm_solver_stream(lbm_solver* s, void** stream) {
    if (!s || !stream) { set_error("lbm_solver_stream: null argument"); return LBM_ERR_INVALID; }
    *stream = s->stream;
    return LBM_OK;
}

int lbm_home_zchunk(lbm_solver* s, int* zchunk) {
    if (!s || !zchunk) { set_error("lbm_home_zchunk: null argument"); return LBM_ERR_INVALID; }
    *zchunk = s->home_zchunk;
    return LBM_OK;
}

int lbm_macro_ptrs(lbm_solver* s, float** d_rho, float** d_u, float** d_v, float** d_w) {
    if (!s) { set_error("lbm_macro_ptrs: null solver"); return LBM_ERR_INVALID; }
    float* b = nullptr;
    const int rc = macro_fields(s, &b);
    if (rc != LBM_OK) return rc;
    if (d_rho) *d_rho = b;
    if (d_u) *d_u = b + s->N;
    if (d_v) *d_v = b + 2 * s->N;
    if (d_w) *d_w = b + 3 * s->N;
    return LBM_OK;
}

int lbm_get_macros(lbm_solver* s, float* rho, float* ux, float* uy, float* uz) {
    if (!s) { set_error("lbm_get_macros: null solver"); return LBM_ERR_INVALID; }
    float* b = nullptr;
    const int rc = macro_fields(s, &b);
    if (rc != LBM_OK) return rc;
    float* dst[4] = {rho, ux, uy, uz};
    for (int k = 0; k < 4; ++k)
        if (dst[k]) CK(cudaMemcpyAsync(dst[k], b + k * s->N, sizeof(float) * (size_t)s->N, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return LBM_OK;
}

int lbm_get_state(lbm_solver* s, float* host_out) {
    if (!s || !host_out) { set_error("lbm_get_state: null argument"); return LBM_ERR_INVALID; }
    const int ncomp = is_aa(s) ? 19 : 10;
    float* tmp = nullptr;
    CK(cudaMallocAsync((void**)&tmp, sizeof(float) * ncomp * (size_t)s->N, s->stream));
    cudaError_t e;
    if (is_aa(s)) {
        lbm::AAParams p = aa_params(s, false, false);
        e = lbm::launch_aa_materialize(p, s->storage, is_ref_push(s) ? 0 : s->parity, tmp, s->stream);
    } else {
        e = lbm::launch_home_export(s->m[s->cur], s->storage, s->N, s->rho0, tmp, s->stream);
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(host_out, tmp, sizeof(float) * ncomp * (size_t)s->N, cudaMemcpyDeviceToHost, s->stream);
    cudaFreeAsync(tmp, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) { set_error(std::string("lbm_get_state: ") + cudaGetErrorString(e)); return LBM_ERR_CUDA; }
    return LBM_OK;
}

int lbm_dims(lbm_solver* s, int32_t* nx, int32_t* ny, int32_t* nz, int64_t* n) {
    if (!s) { set_error("lbm_dims: null solver"); return LBM_ERR_INVALID; }
    if (nx) *nx = s->dom.nx;
    if (ny) *ny = s->dom.ny;
    if (nz) *nz = s->dom.nz;
    if (n) *n = s->N;
    return LBM_OK;
}

int lbm_step_count(lbm_solver* s, int64_t* steps) {
    if (!s || !steps) { set_error("lbm_step_count: null argument"); return LBM_ERR_INVALID; }
    *steps = s->steps;
    return LBM_OK;
}

int lbm_enable_stats(lbm_solver* s, int enable) {
    if (!s) { set_error("lbm_enable_stats: null solver"); return LBM_ERR_INVALID; }
    s->stats_on = enable != 0;
    return LBM_OK;
}

int lbm_set_macro_output(lbm_solver* s, int enable) {
    if (!s) { set_error("lbm_set_macro_output: null solver"); return LBM_ERR_INVALID; }
    s->macro_out = enable != 0;
    drop_graph(s);
    return LBM_OK;
}

int lbm_get_stats(lbm_solver* s, double* out) {
    if (!s || !out) { set_error("lbm_get_stats: null argument"); return LBM_ERR_INVALID; }
    CK(cudaMemcpyAsync(out, s->stats, sizeof(double) * lbm::NSTAT, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return LBM_OK;
}

int lbm_get_stats_async(lbm_solver* s, double* out) {
    if (!s || !out) { set_error("lbm_get_stats_async: null argument"); return LBM_ERR_INVALID; }
    // on the copy stream, behind the macro read-back: a device-to-host copy on
    // the solver's stream would wait for the copy engine and stall the steps
    int rc = ensure_copy_path(s);
    if (rc != LBM_OK) return rc;
    CK(cudaEventRecord(s->ev_macros, s->stream));
    CK(cudaStreamWaitEvent(s->copy_stream, s->ev_macros, 0));
    CK(cudaMemcpyAsync(out, s->stats, sizeof(double) * lbm::NSTAT, cudaMemcpyDeviceToHost, s->copy_stream));
    CK(cudaEventRecord(s->ev_read, s->copy_stream));
    s->read_pending = true;   // the next step that writes statistics waits for this copy
    return LBM_OK;
}

int lbm_voxelize(const float* tris, int64_t ntri, const float* bb_in, const lbm_voxel_params* p, uint8_t* mask_out) {
    if (!p || !mask_out || (ntri > 0 && !tris) || ntri < 0) { set_error("lbm_voxelize: bad argument"); return LBM_ERR_INVALID; }
    if (p->nx < 1 || p->ny < 1 || p->nz < 1) { set_error("lbm_voxelize: bad dimensions"); return LBM_ERR_INVALID; }
    const int r = p->refine < 1 ? 1 : p->refine;
    const int64_t NF = (int64_t)p->nx * r * p->ny * r * p->nz * r;
    if (NF > ((int64_t)1 << 36)) { set_error("lbm_voxelize: refined grid too large"); return LBM_ERR_SIZE; }
    float bb[6];
    if (bb_in) std::memcpy(bb, bb_in, sizeof(bb));
    else {
        for (int k = 0; k < 3; ++k) { bb[k] = 3.402823466e+38F; bb[3 + k] = -3.402823466e+38F; }
        for (int64_t i = 0; i < ntri * 3; ++i)
            for (int k = 0; k < 3; ++k) {
                const float v = tris[i * 3 + k];
                if (v < bb[k]) bb[k] = v;
                if (bb[3 + k] < v) bb[3 + k] = v;
            }
    }
    const int64_t N = (int64_t)p->nx * p->ny * p->nz;
    cudaStream_t st = nullptr;
    CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    float* d_tris = nullptr;
    uint8_t* d_mask = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&d_tris, sizeof(float) * 9 * (size_t)(ntri > 0 ? ntri : 1), st);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&d_mask, (size_t)N, st);
    if (e == cudaSuccess && ntri > 0)
        e = cudaMemcpyAsync(d_tris, tris, sizeof(float) * 9 * (size_t)ntri, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = lbm::launch_voxelize(d_tris, ntri, bb, p->nx, p->ny, p->nz, p->uniform_scale, p->translate, r,
                                 p->coverage_threshold, d_mask, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(mask_out, d_mask, (size_t)N, cudaMemcpyDeviceToHost, st);
    if (d_tris) cudaFreeAsync(d_tris, st);
    if (d_mask) cudaFreeAsync(d_mask, st);
    const cudaError_t e2 = cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    if (e == cudaSuccess) e = e2;
    if (e != cudaSuccess) { set_error(std::string("lbm_voxelize: ") + cudaGetErrorString(e)); return LBM_ERR_CUDA; }
    return LBM_OK;
}

}  // extern "C"

// ---- batched instances -------------------------------------------------------
struct lbm_batch {
    std::vector<lbm_solver*> inst;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    lbm::AAParams* d_params = nullptr;
    int4* d_units[2] = {nullptr, nullptr};
    int* d_first[2] = {nullptr, nullptr};
    int nunits[2] = {0, 0};
    int units_threads = 0, units_even = 0, units_odd = 0;   // shape the unit lists were built for
    int storage = LBM_STORE_F32;   // of every instance
    double* partials = nullptr;
    size_t partials_cap = 0;
    double* d_stats = nullptr;
    int parity = 0;
    bool stats_on = false;
    lbm_batch_tuning tune{256, 4, 512, 8, 0.f};
    cudaGraphExec_t gexec = nullptr;
    int g_sub = 0, g_parity = -1, g_stats = -1;
};

namespace {

void batch_drop_graph(lbm_batch* b) {
    if (b->gexec) { cudaGraphExecDestroy(b->gexec); b->gexec = nullptr; }
    b->g_sub = 0; b->g_parity = -1; b->g_stats = -1;
}

int batch_upload_params(lbm_batch* b) {
    for (lbm_solver* s : b->inst)
        if (s->parity != b->inst[0]->parity) {
            set_error("lbm_batch: instances at different step parities");
            return LBM_ERR_INVALID;
        }
    b->parity = b->inst[0]->parity;
    std::vector<lbm::AAParams> h(b->inst.size());
    for (size_t i = 0; i < b->inst.size(); ++i) {
        lbm_solver* s = b->inst[i];
        h[i] = aa_params(s, false, false);
        h[i].flags = s->flags;   // the batched kernels read the flag byte of every instance
    }
    CK(cudaMemcpyAsync(b->d_params, h.data(), sizeof(lbm::AAParams) * h.size(), cudaMemcpyHostToDevice, b->stream));
    CK(cudaStreamSynchronize(b->stream));
    batch_drop_graph(b);
    return LBM_OK;
}

// cells per vector of an instance's batched even step: the width its own step
// takes for its cell count (F16/BF16: 4, 2 or 1; FP32, whose results do not
// depend on it: 2 or 1)
int batch_vec(const lbm_solver* s) {
    if (s->storage == LBM_STORE_F32) return s->N % 2 == 0 ? 2 : 1;
    return s->N % 4 == 0 ? 4 : (s->N % 2 == 0 ? 2 : 1);
}

// unit lists of both parities for the current launch shape
int batch_build_units(lbm_batch* b) {
    const int T = b->tune.threads, E = b->tune.even_unit, O = b->tune.odd_unit;
    if (b->units_threads == T && b->units_even == E && b->units_odd == O && b->d_units[0]) return LBM_OK;
    for (int par = 0; par < 2; ++par) {
        std::vector<int4> u;
        std::vector<int> first;
        for (size_t i = 0; i < b->inst.size(); ++i) {
            const lbm_solver* s = b->inst[i];
            first.push_back((int)u.size());
            // even step: vectors of the width the instance's own step would use
            const int vec = batch_vec(s);
            const int64_t total = par == 0 ? s->N / vec : s->N;
            const int step = par == 0 ? E : O * T;
            for (int64_t f = 0; f < total; f += step)
                u.push_back(make_int4((int)i, (int)f, (int)std::min<int64_t>(step, total - f), par == 0 ? vec : 0));
        }
        first.push_back((int)u.size());
        cudaFree(b->d_units[par]);
        cudaFree(b->d_first[par]);
        b->d_units[par] = nullptr;
        b->d_first[par] = nullptr;
        CK(cudaMalloc((void**)&b->d_units[par], sizeof(int4) * std::max<size_t>(u.size(), 1)));
        CK(cudaMalloc((void**)&b->d_first[par], sizeof(int) * first.size()));
        CK(cudaMemcpy(b->d_units[par], u.data(), sizeof(int4) * u.size(), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(b->d_first[par], first.data(), sizeof(int) * first.size(), cudaMemcpyHostToDevice));
        b->nunits[par] = (int)u.size();
    }
    const size_t need = (size_t)std::max(b->nunits[0], b->nunits[1]) * lbm::NSTAT;
    if (need > b->partials_cap) {
        cudaFree(b->partials);
        b->partials = nullptr;
        CK(cudaMalloc((void**)&b->partials, sizeof(double) * need));
        b->partials_cap = need;
    }
    b->units_threads = T; b->units_even = E; b->units_odd = O;
    batch_drop_graph(b);
    return LBM_OK;
}

int batch_enqueue(lbm_batch* b, int n) {
    const int blocks_cap = lbm::num_sms() * b->tune.blocks_per_sm;
    for (int i = 0; i < n; ++i) {
        const bool st = b->stats_on && i == n - 1;
        const int par = b->parity;
        const int blocks = std::max(1, std::min(blocks_cap, b->nunits[par]));
        CK(lbm::launch_aa_batch(b->d_params, b->d_units[par], b->nunits[par], par, st, b->storage, blocks, b->tune.threads,
                                b->partials, b->stream));
        if (st) CK(lbm::launch_batch_finalize(b->partials, b->d_first[par], (int)b->inst.size(), b->d_stats, b->stream));
        b->parity ^= 1;
    }
    return LBM_OK;
}

void batch_advance_instances(lbm_batch* b, int n) {
    for (lbm_solver* s : b->inst) {
        s->parity ^= (n & 1);
        s->steps += n;
    }
}

}  // namespace

extern "C" {

int lbm_batch_create(lbm_solver* const* solvers, int32_t n, void* stream, lbm_batch** out) {
    if (!solvers || n <= 0 || !out) { set_error("lbm_batch_create: bad argument"); return LBM_ERR_INVALID; }
    *out = nullptr;
    for (int i = 0; i < n; ++i) {
        const lbm_solver* s = solvers[i];
        if (!s) { set_error("lbm_batch_create: null solver"); return LBM_ERR_INVALID; }
        if (!is_aa(s) || is_ref_push(s) || s->storage == LBM_STORE_F64 || s->storage != solvers[0]->storage) {
            set_error("lbm_batch_create: instances must be Legacy/Hybrid, halfway bounce-back, all in one of "
                      "FP32, F16 or BF16 storage");
            return LBM_ERR_UNSUPPORTED;
        }
        if (s->zghost) {
            set_error("lbm_batch_create: z-slab solvers (ghost planes) cannot be batched");
            return LBM_ERR_UNSUPPORTED;
        }
        if ((uint64_t)s->N * 19u >= (1ull << 32)) {
            set_error("lbm_batch_create: instance cell counts must be below 2^32/19");
            return LBM_ERR_SIZE;
        }
        if (s->parity != solvers[0]->parity) {
            set_error("lbm_batch_create: instances at different step parities");
            return LBM_ERR_INVALID;
        }
    }
    lbm_batch* b = new lbm_batch();
    b->inst.assign(solvers, solvers + n);
    b->storage = solvers[0]->storage;
    b->parity = solvers[0]->parity;
    if (stream) b->stream = static_cast<cudaStream_t>(stream);
    else {
        if (cudaStreamCreate(&b->stream) != cudaSuccess) { delete b; set_error("lbm_batch_create: stream"); return LBM_ERR_CUDA; }
        b->own_stream = true;
    }
    // the instances' own streams finish their queued work first
    for (lbm_solver* s : b->inst)
        if (cudaStreamSynchronize(s->stream) != cudaSuccess) { lbm_batch_destroy(b); set_error("lbm_batch_create: sync"); return LBM_ERR_CUDA; }
    if (cudaMalloc((void**)&b->d_params, sizeof(lbm::AAParams) * n) != cudaSuccess ||
        cudaMalloc((void**)&b->d_stats, sizeof(double) * lbm::NSTAT * n) != cudaSuccess) {
        lbm_batch_destroy(b);
        set_error("lbm_batch_create: allocation failed");
        return LBM_ERR_ALLOC;
    }
    cudaMemset(b->d_stats, 0, sizeof(double) * lbm::NSTAT * n);
    int rc = batch_upload_params(b);
    if (rc == LBM_OK) rc = batch_build_units(b);
    if (rc != LBM_OK) { lbm_batch_destroy(b); return rc; }
    *out = b;
    return LBM_OK;
}

int lbm_batch_refresh(lbm_batch* b) {
    if (!b) { set_error("lbm_batch_refresh: null batch"); return LBM_ERR_INVALID; }
    return batch_upload_params(b);
}

int lbm_batch_destroy(lbm_batch* b) {
    if (!b) return LBM_OK;
    if (b->stream) cudaStreamSynchronize(b->stream);
    batch_drop_graph(b);
    cudaFree(b->d_params); cudaFree(b->d_units[0]); cudaFree(b->d_units[1]);
    cudaFree(b->d_first[0]); cudaFree(b->d_first[1]); cudaFree(b->partials); cudaFree(b->d_stats);
    if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return LBM_OK;
}

int lbm_batch_set_tuning(lbm_batch* b, const lbm_batch_tuning* t) {
    if (!b || !t) { set_error("lbm_batch_set_tuning: null argument"); return LBM_ERR_INVALID; }
    if ((t->threads != 128 && t->threads != 256) || t->blocks_per_sm < 1 || t->blocks_per_sm > 16 ||
        t->even_unit < 1 || t->odd_unit < 1) {
        set_error("lbm_batch_set_tuning: threads 128|256, blocks_per_sm 1..16, units >= 1");
        return LBM_ERR_INVALID;
    }
    b->tune = *t;
    return batch_build_units(b);
}

int lbm_batch_get_tuning(lbm_batch* b, lbm_batch_tuning* out) {
    if (!b || !out) { set_error("lbm_batch_get_tuning: null argument"); return LBM_ERR_INVALID; }
    *out = b->tune;
    return LBM_OK;
}

int lbm_batch_tune(lbm_batch* b, int32_t trial_pairs, lbm_batch_tuning* out) {
    if (!b) { set_error("lbm_batch_tune: null batch"); return LBM_ERR_INVALID; }
    if (trial_pairs < 1) trial_pairs = 1;
    const bool saved_stats = b->stats_on;
    b->stats_on = false;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    lbm_batch_tuning best = b->tune;
    float best_ms = 1e30f;
    for (int threads : {128, 256})
        for (int bps : {2, 4, 8})
            for (int ev : {threads, 4 * threads, 16 * threads})
                for (int od : {1, 4, 16}) {
                    if (threads * bps > 2048) continue;
                    lbm_batch_tuning t{threads, bps, ev, od, 0.f};
                    b->tune = t;
                    int rc = batch_build_units(b);
                    if (rc != LBM_OK) return rc;
                    rc = batch_enqueue(b, 2);              // warm-up pair
                    if (rc != LBM_OK) return rc;
                    CK(cudaEventRecord(e0, b->stream));
                    rc = batch_enqueue(b, 2 * trial_pairs);
                    if (rc != LBM_OK) return rc;
                    CK(cudaEventRecord(e1, b->stream));
                    CK(cudaEventSynchronize(e1));
                    float ms = 0.f;
                    CK(cudaEventElapsedTime(&ms, e0, e1));
                    batch_advance_instances(b, 2 + 2 * trial_pairs);
                    if (ms < best_ms) {
                        best_ms = ms;
                        best = t;
                        best.us_per_step = 1e3f * ms / (2 * trial_pairs);
                    }
                }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->tune = best;
    b->stats_on = saved_stats;
    const int rc = batch_build_units(b);
    if (rc != LBM_OK) return rc;
    if (out) *out = best;
    return LBM_OK;
}

int lbm_batch_step(lbm_batch* b, int32_t substeps) {
    if (!b) { set_error("lbm_batch_step: null batch"); return LBM_ERR_INVALID; }
    if (substeps < 0) { set_error("lbm_batch_step: negative substeps"); return LBM_ERR_INVALID; }
    for (const lbm_solver* s : b->inst)
        if (s->parity != b->parity) {
            set_error("lbm_batch_step: an instance was stepped or reinitialised outside the batch; "
                      "call lbm_batch_refresh");
            return LBM_ERR_INVALID;
        }
    if (substeps == 0) return LBM_OK;
    if (substeps == 1) {
        const int rc = batch_enqueue(b, 1);
        if (rc == LBM_OK) batch_advance_instances(b, 1);
        return rc;
    }
    // multi-step calls replay a captured graph of `substeps` persistent launches
    if (!b->gexec || b->g_sub != substeps || b->g_parity != b->parity || b->g_stats != (int)b->stats_on) {
        batch_drop_graph(b);
        const int saved = b->parity;
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        const int rc = batch_enqueue(b, substeps);
        const cudaError_t e = cudaStreamEndCapture(b->stream, &g);
        b->parity = saved;
        if (rc != LBM_OK) { if (g) cudaGraphDestroy(g); return rc; }
        if (e != cudaSuccess) { set_error(std::string("batch graph capture: ") + cudaGetErrorString(e)); return LBM_ERR_CUDA; }
        const cudaError_t e2 = cudaGraphInstantiate(&b->gexec, g, 0);
        cudaGraphDestroy(g);
        if (e2 != cudaSuccess) { set_error(std::string("batch graph: ") + cudaGetErrorString(e2)); return LBM_ERR_CUDA; }
        b->g_sub = substeps; b->g_parity = b->parity; b->g_stats = b->stats_on;
    }
    CK(cudaGraphLaunch(b->gexec, b->stream));
    b->parity ^= (substeps & 1);
    batch_advance_instances(b, substeps);
    return LBM_OK;
}

int lbm_batch_synchronize(lbm_batch* b) {
    if (!b) { set_error("lbm_batch_synchronize: null batch"); return LBM_ERR_INVALID; }
    CK(cudaStreamSynchronize(b->stream));
    return LBM_OK;
}

int lbm_batch_enable_stats(lbm_batch* b, int enable) {
    if (!b) { set_error("lbm_batch_enable_stats: null batch"); return LBM_ERR_INVALID; }
    b->stats_on = enable != 0;
    return LBM_OK;
}

int lbm_batch_get_stats(lbm_batch* b, double* out) {
    if (!b || !out) { set_error("lbm_batch_get_stats: null argument"); return LBM_ERR_INVALID; }
    CK(cudaMemcpyAsync(out, b->d_stats, sizeof(double) * lbm::NSTAT * b->inst.size(), cudaMemcpyDeviceToHost,
                       b->stream));
    CK(cudaStreamSynchronize(b->stream));
    return LBM_OK;
}

}  // extern "C"
