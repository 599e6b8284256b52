// Reference-compatible Legacy / Hybrid step (LBM_BOUNCE_REFERENCE).
//
// The reference's opposite table (src/lbm/lbm3d_legacy.cu:29-32,
// src/lbm/lbm3d_hybrid.cu:28-31) pairs every diagonal direction with its
// mirror image in x (xy and xz diagonals) or y (yz diagonals) instead of its
// opposite.  In the reference's push kernels (legacy.cu:92-108,
// hybrid.cu:140-169) that has two consequences next to solid cells:
//   * a slot (q, y) whose upstream cell y - c_q is solid is written only if the
//     cell's own reflection of direction opp_ref(q) happens to target a solid
//     cell too; otherwise it is never written and keeps what the second buffer
//     held (after the element-wise swap: the populations of the previous step);
//   * a slot written by a neighbour's streaming AND by the cell's own
//     reflection is written twice by two threads (a race in the reference).
// This kernel reproduces that step deterministically: two buffers swapped by
// pointer (the same contents as the reference's swap kernel leaves), unwritten
// slots keep the old buffer's value, and in a doubly written slot the
// reflection wins.  It is the compatibility path, not the fast one: the AA
// kernels (lbm_aa.cu) implement halfway bounce-back with true opposites in
// one buffer.
#include "lbm_common.cuh"
#include "lbm_internal.h"

namespace lbm {
namespace {

__host__ __device__ constexpr int opp_ref(int q) { return opp_tab(q); }

__device__ __forceinline__ int wrapr(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

template <int MODE>
__global__ void __launch_bounds__(256, 2) ref_push(AAParams p, const float* __restrict__ fa, float* __restrict__ fb) {
    constexpr bool MACRO = MODE >= 1, STATS = MODE == 2;
    const int64_t N = p.N;
    const int nx = p.nx, ny = p.ny, nz = p.nz;
    const int bx = blockDim.x;
    const int segs = (nx + bx - 1) / bx;
    const int64_t total = (int64_t)segs * ny * nz;
    const uint8_t* __restrict__ fl = p.flags;
    double acc[NSTAT];
#pragma unroll
    for (int k = 0; k < NSTAT; ++k) acc[k] = 0.0;
    auto solid_at = [&](int x, int y, int z) -> bool {
        // (x may be out of range in a duct: such a cell does not exist)
        if (p.duct && (x < 0 || x >= nx)) return false;
        if (!fl) return false;
        const int64_t t = ((int64_t)wrapr(z, nz) * ny + wrapr(y, ny)) * nx + wrapr(x, nx);
        return (fl[t] & F_SOLID) != 0;
    };

    for (int64_t sg = blockIdx.x; sg < total; sg += gridDim.x) {
        const int64_t row = sg / segs;
        const int x = (int)(sg - row * segs) * bx + threadIdx.x;
        if (x >= nx) continue;
        const int y = (int)(row % ny);
        const int z = (int)(row / ny);
        const int64_t id = row * nx + x;
        const uint32_t f8 = fl ? fl[id] : 0u;
        float c[19];
#pragma unroll
        for (int q = 0; q < 19; ++q) c[q] = fa[q * N + id];
        if (f8 & F_SOLID) {   // legacy.cu:72-76
#pragma unroll
            for (int q = 0; q < 19; ++q) fb[q * N + id] = c[q];
            if (MACRO) { p.rho[id] = 1.f; p.ux[id] = 0.f; p.uy[id] = 0.f; p.uz[id] = 0.f; }
            continue;
        }
        float r = 0.f, jx = 0.f, jy = 0.f, jz = 0.f;
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            r += c[q];
            if (cx(q) > 0) jx += c[q]; else if (cx(q) < 0) jx -= c[q];
            if (cy(q) > 0) jy += c[q]; else if (cy(q) < 0) jy -= c[q];
            if (cz(q) > 0) jz += c[q]; else if (cz(q) < 0) jz -= c[q];
        }
        const float ux = ((r > 0.f) ? jx / r : 0.f) + p.fx;
        const float uy = ((r > 0.f) ? jy / r : 0.f) + p.fy;
        const float uz = ((r > 0.f) ? jz / r : 0.f) + p.fz;
        const bool bgk = !p.hybrid || (f8 & F_BAND);
        float o[19];
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            const float fe = feq_ref(q, r, ux, uy, uz);
            const float fq = c[q];
            if (bgk) o[q] = fq + p.omega * (fe - fq);
            else {
                const float ds = fq - fe;
                o[q] = fq + p.omega_h * (fe - fq) + (p.omega_s - p.omega_h) * (-ds);
            }
        }
        const bool special = (f8 & F_SPECIAL) != 0;
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            const int xt = x + cx(q), yt = y + cy(q), zt = z + cz(q);
            if (p.duct && xt < 0) {                       // inlet (true opposite, as in the AA kernels)
                fb[opp(q) * N + id] = feq_ref(opp(q), r, p.u_in, 0.f, 0.f);
                continue;
            }
            if (p.duct && xt >= nx) {                     // outlet
                fb[opp(q) * N + id] = o[opp(q)];
                continue;
            }
            if (special && solid_at(xt, yt, zt)) {        // reflection into slot opp_ref(q)
                fb[opp_ref(q) * N + id] = o[q];
                if (STATS) {
                    const int64_t t = ((int64_t)wrapr(zt, nz) * ny + wrapr(yt, ny)) * nx + wrapr(xt, nx);
                    if (fl[t] & F_OBST) {
                        acc[2] += (double)(cx(q) - cx(opp_ref(q))) * o[q];
                        acc[3] += (double)(cy(q) - cy(opp_ref(q))) * o[q];
                        acc[4] += (double)(cz(q) - cz(opp_ref(q))) * o[q];
                    }
                }
                continue;
            }
            // the target's own reflection of direction opp_ref(q) lands in the same slot
            if (opp_ref(q) != opp(q) && fl &&
                solid_at(xt + cx(opp_ref(q)), yt + cy(opp_ref(q)), zt + cz(opp_ref(q))))
                continue;
            const int64_t t = ((int64_t)wrapr(zt, nz) * ny + wrapr(yt, ny)) * nx + wrapr(xt, nx);
            fb[q * N + t] = o[q];
        }
        if (MACRO) { p.rho[id] = r; p.ux[id] = ux; p.uy[id] = uy; p.uz[id] = uz; }
        if (STATS) {
            acc[0] += (double)r;
            acc[1] += 0.5 * ((double)ux * ux + (double)uy * uy + (double)uz * uz);
            acc[5] += (double)r * ux;
            acc[6] += (double)r * uy;
            acc[7] += (double)r * uz;
        }
    }
    if constexpr (STATS) block_reduce_stats(acc, p.partials);
}

}  // namespace

cudaError_t launch_ref_push(const AAParams& p, const float* fa, float* fb, LaunchCfg cfg, cudaStream_t s) {
    const int mode = p.stats ? 2 : (p.macro ? 1 : 0);
    if (mode == 0) ref_push<0><<<cfg.blocks, cfg.threads, 0, s>>>(p, fa, fb);
    else if (mode == 1) ref_push<1><<<cfg.blocks, cfg.threads, 0, s>>>(p, fa, fb);
    else ref_push<2><<<cfg.blocks, cfg.threads, 0, s>>>(p, fa, fb);
    return cudaGetLastError();
}

}  // namespace lbm
