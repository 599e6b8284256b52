// Legacy BGK and Hybrid(B0) steps in the AA pattern: one population buffer,
// every population read once and written once per step, in place.
//
// The reference (src/lbm/lbm3d_legacy.cu:59-118, src/lbm/lbm3d_hybrid.cu:89-180)
// pushes into a second buffer and then swaps the two buffers element by element
// (kern_swap), which moves about 473 B per cell-update.  Here:
//   even step: each cell reads its 19 populations (natural layout), collides and
//              writes f*_q into its own slot opp(q)           -> purely local;
//   odd step:  each cell gathers f_q from slot opp(q) of x-c_q, collides and
//              scatters f*_q into slot q of x+c_q             -> natural layout again.
// Both steps read and write the same 19 slots per cell, so no two threads touch
// one slot and no second buffer is needed: 152 B per cell-update in FP32.
//
// A link x -> x+c_q that does not stream (solid target, or the duct's inlet /
// outlet planes) sends its value back into the cell's own slot opp(q), where
// the next odd step's gather (or the next even step's natural read) picks it up:
//   solid target : f*_q                      (halfway bounce-back, legacy.cu:100-104)
//   inlet (x<0)  : feq_opp(q)(rho, u_in)
//   outlet (x>=Nx): f*_opp(q)
// Macro outputs are the moments of the populations the step starts from, as the
// reference's kernels write them before colliding (legacy.cu:78-90,110-113).
#include "lbm_common.cuh"
#include "lbm_internal.h"

namespace lbm {
namespace {

struct Cell {
    float r, ux, uy, uz;
};

// Pre-collision moments with the velocity-shift force (legacy.cu:78-90).  The
// sums run in the reference's q order; the +-1 components add or subtract.
__device__ __forceinline__ Cell moments(const float (&f)[19], float fx, float fy, float fz) {
    float r = 0.f, jx = 0.f, jy = 0.f, jz = 0.f;
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        r += f[q];
        if (cx(q) > 0) jx += f[q]; else if (cx(q) < 0) jx -= f[q];
        if (cy(q) > 0) jy += f[q]; else if (cy(q) < 0) jy -= f[q];
        if (cz(q) > 0) jz += f[q]; else if (cz(q) < 0) jz -= f[q];
    }
    Cell c;
    c.r = r;
    c.ux = ((r > 0.f) ? jx / r : 0.f) + fx;
    c.uy = ((r > 0.f) ? jy / r : 0.f) + fy;
    c.uz = ((r > 0.f) ? jz / r : 0.f) + fz;
    return c;
}

// Post-collision populations.  Band (or Legacy) cells: fq + w(feq - fq)
// (legacy.cu:92-95); Hybrid non-band cells: the algebraic "HOME form" of
// hybrid.cu:148-152, identical to BGK when omega_s == omega_h.
__device__ __forceinline__ void collide(const float (&f)[19], float (&o)[19], const Cell& c,
                                        bool bgk_form, float omega, float omega_h, float omega_s) {
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        const float fe = feq_ref(q, c.r, c.ux, c.uy, c.uz);
        const float fq = f[q];
        if (bgk_form) {
            o[q] = fq + omega * (fe - fq);
        } else {
            const float ds = fq - fe;
            o[q] = fq + omega_h * (fe - fq) + (omega_s - omega_h) * (-ds);
        }
    }
}

__device__ __forceinline__ int wrap(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

// Momentum exchanged with obstacle cells along the solid links of one cell.
__device__ __forceinline__ void add_drag(double (&acc)[NSTAT], const float (&o)[19], uint32_t lk,
                                         const uint8_t* flags, int x, int y, int z, int nx, int ny, int nz,
                                         int duct) {
#pragma unroll
    for (int q = 1; q < 19; ++q) {
        if (!((lk >> q) & 1u)) continue;
        const int xt = x + cx(q);
        if (duct && (xt < 0 || xt >= nx)) continue;
        const int64_t t = ((int64_t)wrap(z + cz(q), nz) * ny + wrap(y + cy(q), ny)) * nx + wrap(xt, nx);
        if (flags[t] & F_OBST) {
            acc[2] += 2.0 * cx(q) * (double)o[q];
            acc[3] += 2.0 * cy(q) * (double)o[q];
            acc[4] += 2.0 * cz(q) * (double)o[q];
        }
    }
}

__device__ __forceinline__ void add_cell_stats(double (&acc)[NSTAT], const Cell& c) {
    acc[0] += (double)c.r;
    acc[1] += 0.5 * ((double)c.ux * c.ux + (double)c.uy * c.uy + (double)c.uz * c.uz);
    acc[5] += (double)c.r * c.ux;
    acc[6] += (double)c.r * c.uy;
    acc[7] += (double)c.r * c.uz;
}

// ---------------------------------------------------------------------------
// Even step: local.  VEC consecutive cells per thread (VEC=4: one 16-byte
// (F32) or 8-byte (F16/BF16) access per population and thread).
// ---------------------------------------------------------------------------
// MODE 0: populations only; 1: + macro fields; 2: + macro fields + statistics
template <class ST, bool MASK, int VEC, int MODE>
__global__ void __launch_bounds__(256, 2) aa_even(AAParams p) {
    constexpr bool MACRO = MODE >= 1, STATS = MODE == 2;
    using T = typename ST::T;
    T* __restrict__ f = static_cast<T*>(p.f);
    const int64_t N = p.N;
    const int64_t nvec = N / VEC;
    double acc[NSTAT];
#pragma unroll
    for (int k = 0; k < NSTAT; ++k) acc[k] = 0.0;

    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nvec;
         v += (int64_t)gridDim.x * blockDim.x) {
        const int64_t id = v * VEC;
        float a[19][VEC];
#pragma unroll
        for (int q = 0; q < 19; ++q) ldv<ST, VEC>(f + q * N + id, q, p.rho0, a[q]);
        uint32_t fl4 = 0;
        if constexpr (MASK) {
            if constexpr (VEC == 4) fl4 = *reinterpret_cast<const uint32_t*>(p.flags + id);
            else if constexpr (VEC == 2) fl4 = *reinterpret_cast<const uint16_t*>(p.flags + id);
            else fl4 = p.flags[id];
        }
        int x0 = 0;
        if (p.duct) x0 = (int)(id % p.nx);
        float mr[VEC], mu[VEC], mv[VEC], mw[VEC];
#pragma unroll
        for (int l = 0; l < VEC; ++l) {
            const uint32_t fl = (fl4 >> (8 * l)) & 0xffu;
            float c[19];
#pragma unroll
            for (int q = 0; q < 19; ++q) c[q] = a[q][l];
            if (MASK && (fl & F_SOLID)) {
                // frozen (legacy.cu:72-76): slot opp(q) gets its own value back
#pragma unroll
                for (int q = 0; q < 19; ++q) a[q][l] = c[opp(q)];
                mr[l] = 1.f; mu[l] = mv[l] = mw[l] = 0.f;
                continue;
            }
            const Cell m = moments(c, p.fx, p.fy, p.fz);
            float o[19];
            const bool bgk = !p.hybrid || (fl & F_BAND);
            collide(c, o, m, bgk, p.omega, p.omega_h, p.omega_s);
            if (STATS) {
                add_cell_stats(acc, m);
                if (MASK && (fl & F_TOUCH)) {
                    const int64_t x = id + l;
                    const int xi = (int)(x % p.nx);
                    const int64_t row = x / p.nx;
                    add_drag(acc, o, p.links[id + l], p.flags, xi, (int)(row % p.ny), (int)(row / p.ny),
                             p.nx, p.ny, p.nz, p.duct);
                }
            }
            if (p.duct) {
                const int x = x0 + l;
                if (x == 0) {
#pragma unroll
                    for (int q = 0; q < 19; ++q)
                        if (cx(q) < 0) o[q] = feq_ref(opp(q), m.r, p.u_in, 0.f, 0.f);
                } else if (x == p.nx - 1) {
#pragma unroll
                    for (int q = 0; q < 19; ++q)
                        if (cx(q) > 0) o[q] = o[opp(q)];
                }
            }
#pragma unroll
            for (int q = 0; q < 19; ++q) a[q][l] = o[q];
            mr[l] = m.r; mu[l] = m.ux; mv[l] = m.uy; mw[l] = m.uz;
        }
#pragma unroll
        for (int q = 0; q < 19; ++q) stv<ST, VEC>(f + opp(q) * N + id, q, p.rho0, a[q]);
        if constexpr (MACRO) {
            stv<StoreF32, VEC>(p.rho + id, 0, 0.f, mr);
            stv<StoreF32, VEC>(p.ux + id, 0, 0.f, mu);
            stv<StoreF32, VEC>(p.uy + id, 0, 0.f, mv);
            stv<StoreF32, VEC>(p.uz + id, 0, 0.f, mw);
        }
    }
    if constexpr (STATS) block_reduce_stats(acc, p.partials);
}

// Neighbour addressing of one cell: 9 row bases (dy,dz in -1..1, periodic in
// y and z) and 3 x positions (periodic in x; in a duct the out-of-range ones
// are never used because those links are marked as not streaming).
struct Nbr {
    int64_t r[3][3];   // [dy+1][dz+1]
    int xs[3];         // [dx+1]
    __device__ __forceinline__ void init(int x, int y, int z, int nx, int ny, int nz) {
        const int ym = y == 0 ? ny - 1 : y - 1, yp = y == ny - 1 ? 0 : y + 1;
        const int zm = z == 0 ? nz - 1 : z - 1, zp = z == nz - 1 ? 0 : z + 1;
        const int yy[3] = {ym, y, yp};
        const int zz[3] = {zm, z, zp};
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) r[a][b] = ((int64_t)zz[b] * ny + yy[a]) * nx;
        xs[0] = x == 0 ? nx - 1 : x - 1;
        xs[1] = x;
        xs[2] = x == nx - 1 ? 0 : x + 1;
    }
    __device__ __forceinline__ int64_t at(int dx, int dy, int dz) const { return r[dy + 1][dz + 1] + xs[dx + 1]; }
};

// ---------------------------------------------------------------------------
// Odd step: one cell per thread, rows of blockDim.x cells per block iteration.
// ---------------------------------------------------------------------------
template <class ST, bool MASK, int MODE>
__global__ void __launch_bounds__(256, 2) aa_odd(AAParams p) {
    constexpr bool MACRO = MODE >= 1, STATS = MODE == 2;
    using T = typename ST::T;
    T* __restrict__ f = static_cast<T*>(p.f);
    const int64_t N = p.N;
    const int nx = p.nx, ny = p.ny, nz = p.nz;
    const int bx = blockDim.x;
    const int segs = (nx + bx - 1) / bx;
    const int64_t total = (int64_t)segs * ny * nz;
    double acc[NSTAT];
#pragma unroll
    for (int k = 0; k < NSTAT; ++k) acc[k] = 0.0;

    for (int64_t sg = blockIdx.x; sg < total; sg += gridDim.x) {
        const int64_t row = sg / segs;
        const int x = (int)(sg - row * segs) * bx + threadIdx.x;
        if (x >= nx) continue;
        const int y = (int)(row % ny);
        const int z = (int)(row / ny);
        const int64_t id = row * nx + x;
        const uint32_t fl = MASK ? p.flags[id] : 0u;
        if (MASK && (fl & F_SOLID)) {
            if (MACRO) { p.rho[id] = 1.f; p.ux[id] = 0.f; p.uy[id] = 0.f; p.uz[id] = 0.f; }
            continue;
        }
        Nbr nb;
        nb.init(x, y, z, nx, ny, nz);
        const bool special = MASK && (fl & F_SPECIAL);
        const uint32_t lk = special ? p.links[id] : 0u;
        float c[19];
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            // incoming q travels the link x -> x + c_opp(q)
            if (special && ((lk >> opp(q)) & 1u)) c[q] = ST::ld(f + q * N + id, q, p.rho0);
            else c[q] = ST::ld(f + opp(q) * N + nb.at(-cx(q), -cy(q), -cz(q)), q, p.rho0);
        }
        const Cell m = moments(c, p.fx, p.fy, p.fz);
        float o[19];
        const bool bgk = !p.hybrid || (fl & F_BAND);
        collide(c, o, m, bgk, p.omega, p.omega_h, p.omega_s);
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            if (special && ((lk >> q) & 1u)) {
                float v = o[q];                                   // bounce-back
                if (p.duct) {
                    const int xt = x + cx(q);
                    if (xt < 0) v = feq_ref(opp(q), m.r, p.u_in, 0.f, 0.f);   // inlet
                    else if (xt >= nx) v = o[opp(q)];                          // outlet
                }
                ST::st(f + opp(q) * N + id, q, p.rho0, v);
            } else {
                ST::st(f + q * N + nb.at(cx(q), cy(q), cz(q)), q, p.rho0, o[q]);
            }
        }
        if (MACRO) { p.rho[id] = m.r; p.ux[id] = m.ux; p.uy[id] = m.uy; p.uz[id] = m.uz; }
        if (STATS) {
            add_cell_stats(acc, m);
            if (MASK && (fl & F_TOUCH)) add_drag(acc, o, lk, p.flags, x, y, z, nx, ny, nz, p.duct);
        }
    }
    if constexpr (STATS) block_reduce_stats(acc, p.partials);
}

// The natural-layout populations f^n (the reference's d_f after n steps).
template <class ST>
__global__ void aa_materialize(AAParams p, int parity, float* __restrict__ out) {
    using T = typename ST::T;
    const T* __restrict__ f = static_cast<const T*>(p.f);
    const int64_t N = p.N;
    for (int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; id < N;
         id += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t fl = p.flags ? p.flags[id] : 0u;
        if (parity == 0 || (fl & F_SOLID)) {
            for (int q = 0; q < 19; ++q) out[q * N + id] = ST::ld(f + q * N + id, q, p.rho0);
            continue;
        }
        const int x = (int)(id % p.nx);
        const int64_t row = id / p.nx;
        Nbr nb;
        nb.init(x, (int)(row % p.ny), (int)(row / p.ny), p.nx, p.ny, p.nz);
        const uint32_t lk = (fl & F_SPECIAL) ? p.links[id] : 0u;
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            float v;
            if ((lk >> opp(q)) & 1u) v = ST::ld(f + q * N + id, q, p.rho0);
            else v = ST::ld(f + opp(q) * N + nb.at(-cx(q), -cy(q), -cz(q)), q, p.rho0);
            out[q * N + id] = v;
        }
    }
}

template <class ST, int MODE>
void launch_mode(const AAParams& p, int parity, LaunchCfg cfg, cudaStream_t s) {
    const bool mask = p.flags != nullptr;
    // two consecutive cells per thread: 8-byte (F32) or 4-byte (F16/BF16) accesses
    constexpr int V = 2;
    if (parity == 0) {
        if (p.N % V == 0) {
            if (mask) aa_even<ST, true, V, MODE><<<cfg.blocks, cfg.threads, 0, s>>>(p);
            else aa_even<ST, false, V, MODE><<<cfg.blocks, cfg.threads, 0, s>>>(p);
        } else {
            if (mask) aa_even<ST, true, 1, MODE><<<cfg.blocks, cfg.threads, 0, s>>>(p);
            else aa_even<ST, false, 1, MODE><<<cfg.blocks, cfg.threads, 0, s>>>(p);
        }
    } else {
        if (mask) aa_odd<ST, true, MODE><<<cfg.blocks, cfg.threads, 0, s>>>(p);
        else aa_odd<ST, false, MODE><<<cfg.blocks, cfg.threads, 0, s>>>(p);
    }
}

template <class ST>
cudaError_t launch_typed(const AAParams& p, int parity, LaunchCfg cfg, cudaStream_t s) {
    const int mode = p.stats ? 2 : (p.macro ? 1 : 0);
    if (mode == 0) launch_mode<ST, 0>(p, parity, cfg, s);
    else if (mode == 1) launch_mode<ST, 1>(p, parity, cfg, s);
    else launch_mode<ST, 2>(p, parity, cfg, s);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_aa_step(const AAParams& p, int storage, int parity, LaunchCfg cfg, cudaStream_t s) {
    switch (storage) {
        case 0: return launch_typed<StoreF32>(p, parity, cfg, s);
        case 1: return launch_typed<StoreF16>(p, parity, cfg, s);
        case 2: return launch_typed<StoreBF16>(p, parity, cfg, s);
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_aa_materialize(const AAParams& p, int storage, int parity, float* out, cudaStream_t s) {
    const int blocks = num_sms() * 8;
    switch (storage) {
        case 0: aa_materialize<StoreF32><<<blocks, 256, 0, s>>>(p, parity, out); break;
        case 1: aa_materialize<StoreF16><<<blocks, 256, 0, s>>>(p, parity, out); break;
        case 2: aa_materialize<StoreBF16><<<blocks, 256, 0, s>>>(p, parity, out); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace lbm
