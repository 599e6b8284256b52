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
//   solid target : f*_q                      (halfway bounce-back)
//   inlet (x<0)  : feq_opp(q)(rho, (u_in,0,0)) = w_q rho (1 + 3 u_in + 3 u_in^2)
//   outlet (x>=Nx): f*_opp(q)
// Link handling is branch-free: per direction the address and the value are
// selected, so a warp holding one boundary cell does not run a second path.
// Macro outputs are the moments of the populations the step starts from, as the
// reference's kernels write them before colliding (legacy.cu:78-90,110-113).
#include "lbm_common.cuh"
#include "lbm_internal.h"

namespace lbm {
namespace {

template <class R>
struct CellT {
    R r, ux, uy, uz;
};
using Cell = CellT<float>;

__device__ __forceinline__ float rfma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double rfma(double a, double b, double c) { return fma(a, b, c); }

// Pre-collision moments with the velocity-shift force (legacy.cu:78-90).
// Opposite pairs are summed first: s = f_q + f_opp, d = f_q - f_opp.
// R: float, or double for the FP64 reference form.
template <class R>
__device__ __forceinline__ CellT<R> moments(const R (&f)[19], R fx, R fy, R fz) {
    // pairs with their positive member: (1,2) x, (3,4) y, (5,6) z, (7,10) +x+y,
    // (9,8) +x-y, (11,14) +x+z, (13,12) +x-z, (15,18) +y+z, (17,16) +y-z
    const R s12 = f[1] + f[2], d12 = f[1] - f[2];
    const R s34 = f[3] + f[4], d34 = f[3] - f[4];
    const R s56 = f[5] + f[6], d56 = f[5] - f[6];
    const R s7 = f[7] + f[10], d7 = f[7] - f[10];
    const R s9 = f[9] + f[8], d9 = f[9] - f[8];
    const R s11 = f[11] + f[14], d11 = f[11] - f[14];
    const R s13 = f[13] + f[12], d13 = f[13] - f[12];
    const R s15 = f[15] + f[18], d15 = f[15] - f[18];
    const R s17 = f[17] + f[16], d17 = f[17] - f[16];
    CellT<R> c;
    c.r = f[0] + ((s12 + s34) + (s56 + s7)) + ((s9 + s11) + (s13 + s15) + s17);
    const R jx = (d12 + d7) + (d9 + d11) + d13;
    const R jy = (d34 + d7) - d9 + (d15 + d17);
    const R jz = (d56 + d11) - d13 + (d15 - d17);
    const R inv = c.r > R(0) ? R(1) / c.r : R(0);
    c.ux = jx * inv + fx;
    c.uy = jy * inv + fy;
    c.uz = jz * inv + fz;
    return c;
}

// BGK collision f* = f + w (feq - f) for every direction, the equilibrium
// evaluated per opposite pair: feq_(+-) = w rho (1 - 1.5u^2 + 4.5 t^2) +- 3 w rho t.
// (The Hybrid's "HOME form" of hybrid.cu:148-152 is this with w = omega_shear.)
template <class R>
__device__ __forceinline__ void collide(R (&f)[19], const CellT<R>& c, R omega) {
    const R A = R(1) - R(1.5) * (c.ux * c.ux + c.uy * c.uy + c.uz * c.uz);
    // w_q rho with the weights' own rounding compensated (mulk): no mass or momentum bias per step
    const R r0 = mulk(c.r, K3_HI, K3_LO), r1 = mulk(c.r, K18_HI, K18_LO), r2 = mulk(c.r, K36_HI, K36_LO);
    auto pair = [&](int qp, int qm, R t, R wr) {
        const R sym = wr * rfma(R(4.5) * t, t, A);
        const R asym = R(3) * wr * t;
        f[qp] = rfma(omega, (sym + asym) - f[qp], f[qp]);
        f[qm] = rfma(omega, (sym - asym) - f[qm], f[qm]);
    };
    f[0] = rfma(omega, r0 * A - f[0], f[0]);
    pair(1, 2, c.ux, r1);
    pair(3, 4, c.uy, r1);
    pair(5, 6, c.uz, r1);
    pair(7, 10, c.ux + c.uy, r2);
    pair(9, 8, c.ux - c.uy, r2);
    pair(11, 14, c.ux + c.uz, r2);
    pair(13, 12, c.ux - c.uz, r2);
    pair(15, 18, c.uy + c.uz, r2);
    pair(17, 16, c.uy - c.uz, r2);
}

// The same two functions in the stored units of the narrow forms,
// g_q = (f_q - w_q rho0) S: sum g = S (rho - rho0) and sum c g = S rho u (the
// weights' first moment vanishes), and the equilibrium in those units is
//   geq_(+-) = S [w (rho - rho0) + w rho (4.5 t^2 - 1.5 u^2)] +- 3 S w rho t.
// The populations are never converted back to f, so a step costs no
// conversion arithmetic per population and rho - rho0 keeps its low bits.
__device__ __forceinline__ Cell moments_g(const float (&g)[19], float fx, float fy, float fz, float r0, float invS,
                                          float& dr) {
    const float s12 = g[1] + g[2], d12 = g[1] - g[2];
    const float s34 = g[3] + g[4], d34 = g[3] - g[4];
    const float s56 = g[5] + g[6], d56 = g[5] - g[6];
    const float s7 = g[7] + g[10], d7 = g[7] - g[10];
    const float s9 = g[9] + g[8], d9 = g[9] - g[8];
    const float s11 = g[11] + g[14], d11 = g[11] - g[14];
    const float s13 = g[13] + g[12], d13 = g[13] - g[12];
    const float s15 = g[15] + g[18], d15 = g[15] - g[18];
    const float s17 = g[17] + g[16], d17 = g[17] - g[16];
    Cell c;
    dr = (g[0] + ((s12 + s34) + (s56 + s7)) + ((s9 + s11) + (s13 + s15) + s17)) * invS;
    c.r = r0 + dr;
    const float jx = ((d12 + d7) + (d9 + d11) + d13) * invS;
    const float jy = ((d34 + d7) - d9 + (d15 + d17)) * invS;
    const float jz = ((d56 + d11) - d13 + (d15 - d17)) * invS;
    const float inv = c.r > 0.f ? 1.0f / c.r : 0.f;
    c.ux = jx * inv + fx;
    c.uy = jy * inv + fy;
    c.uz = jz * inv + fz;
    return c;
}

__device__ __forceinline__ void collide_g(float (&g)[19], const Cell& c, float dr, float omega, float S) {
    const float A1 = -1.5f * (c.ux * c.ux + c.uy * c.uy + c.uz * c.uz);
    const float r0 = mulk(c.r, K3_HI, K3_LO), r1 = mulk(c.r, K18_HI, K18_LO), r2 = mulk(c.r, K36_HI, K36_LO);
    const float d0 = mulk(dr, K3_HI, K3_LO), d1 = mulk(dr, K18_HI, K18_LO), d2 = mulk(dr, K36_HI, K36_LO);
    auto pair = [&](int qp, int qm, float t, float wr, float wd) {
        const float sym = S * fmaf(wr, fmaf(4.5f * t, t, A1), wd);
        const float asym = S * (3.0f * wr * t);
        g[qp] = fmaf(omega, (sym + asym) - g[qp], g[qp]);
        g[qm] = fmaf(omega, (sym - asym) - g[qm], g[qm]);
    };
    g[0] = fmaf(omega, S * fmaf(r0, A1, d0) - g[0], g[0]);
    pair(1, 2, c.ux, r1, d1);
    pair(3, 4, c.uy, r1, d1);
    pair(5, 6, c.uz, r1, d1);
    pair(7, 10, c.ux + c.uy, r2, d2);
    pair(9, 8, c.ux - c.uy, r2, d2);
    pair(11, 14, c.ux + c.uz, r2, d2);
    pair(13, 12, c.ux - c.uz, r2, d2);
    pair(15, 18, c.uy + c.uz, r2, d2);
    pair(17, 16, c.uy - c.uz, r2, d2);
}

__device__ __forceinline__ int wrap(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

// Momentum exchanged with obstacle cells along the solid links of one cell.
template <class R>
__device__ __noinline__ void add_drag(double* acc, const R* o, uint32_t lk, const uint8_t* flags, int x, int y,
                                      int z, int nx, int ny, int nz, int duct) {
    for (int q = 1; q < 19; ++q) {
        if (!((lk >> q) & 1u)) continue;
        const int ex = cx(q), ey = cy(q), ez = cz(q);
        const int xt = x + ex;
        if (duct && (xt < 0 || xt >= nx)) continue;
        const int64_t t = ((int64_t)wrap(z + ez, nz) * ny + wrap(y + ey, ny)) * nx + wrap(xt, nx);
        if (flags[t] & F_OBST) {
            acc[2] += 2.0 * ex * (double)o[q];
            acc[3] += 2.0 * ey * (double)o[q];
            acc[4] += 2.0 * ez * (double)o[q];
        }
    }
}

// add_drag for populations in stored units (narrow forms): f = g / S + w rho0.
__device__ __noinline__ void add_drag_g(double* acc, const float* o, float invS, float r0, uint32_t lk,
                                        const uint8_t* flags, int x, int y, int z, int nx, int ny, int nz, int duct) {
    float f[19];
    for (int q = 0; q < 19; ++q) f[q] = o[q] * invS + wq(q) * r0;
    add_drag(acc, f, lk, flags, x, y, z, nx, ny, nz, duct);
}

template <class R>
__device__ __forceinline__ void add_cell_stats(double (&acc)[NSTAT], const CellT<R>& c) {
    acc[0] += (double)c.r;
    acc[1] += 0.5 * ((double)c.ux * c.ux + (double)c.uy * c.uy + (double)c.uz * c.uz);
    acc[5] += (double)c.r * c.ux;
    acc[6] += (double)c.r * c.uy;
    acc[7] += (double)c.r * c.uz;
}

// Inlet replacement for the incoming direction opp(q): the equilibrium at
// (rho, (u_in,0,0)) of a direction with c_x = +1 is w rho (1 + 3u + 3u^2);
// `kin` = 1 + 3u + 3u^2.
__device__ __forceinline__ float inlet_value(int q, float r, float kin) { return wq(q) * r * kin; }
__device__ __forceinline__ double inlet_value(int q, double r, double kin) {
    return (q == 0 ? 1.0 / 3.0 : (q <= 6 ? 1.0 / 18.0 : 1.0 / 36.0)) * r * kin;
}
// the same in stored units: S w (rho kin - rho0)
__device__ __forceinline__ float inlet_g(int q, float r, float kin, float r0, float S) {
    return S * (wq(q) * fmaf(r, kin, -r0));
}

// ---------------------------------------------------------------------------
// Even step: local.  VEC consecutive cells per thread.
// MODE 0: populations only; 1: + macro fields; 2: + macro fields + statistics
// ---------------------------------------------------------------------------
// One even-step unit: the VEC consecutive cells v*VEC .. v*VEC+VEC-1.
template <class ST, bool MASK, int VEC, int MODE, class IDX>
__device__ __forceinline__ void even_unit(const AAParams& p, IDX v, double (&acc)[NSTAT]) {
    constexpr bool MACRO = MODE >= 1, STATS = MODE == 2;
    using T = typename ST::T;
    using R = typename Real<ST>::type;
    T* __restrict__ f = static_cast<T*>(p.f);
    const IDX N = (IDX)p.N;
    const R kin = R(1) + R(3) * p.u_in + R(3) * p.u_in * p.u_in;
    {
        constexpr bool SH = kNarrow<ST>;    // narrow forms: compute in stored units
        const IDX id = v * VEC;
        R a[19][VEC];
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            if constexpr (SH) ldv_raw<ST, VEC>(f + (IDX)q * N + id, a[q]);
            else ldv<ST, VEC>(f + (IDX)q * N + id, q, p.rho0, a[q]);
        }
        // narrow forms: stochastically rounded stores, random words from one
        // hash of the first cell's global index and its loaded rest population
        const uint32_t hsr = SH ? sr_seed((uint32_t)id + p.salt_base, (float)a[0][0]) : 0u;
        uint32_t fl4 = 0;
        if constexpr (MASK) {
            if constexpr (VEC == 4) fl4 = *reinterpret_cast<const uint32_t*>(p.flags + id);
            else if constexpr (VEC == 2) fl4 = *reinterpret_cast<const uint16_t*>(p.flags + id);
            else fl4 = p.flags[id];
        }
        int x0 = 0;
        if (p.duct) x0 = (int)(id % (IDX)p.nx);
        float mr[VEC], mu[VEC], mv[VEC], mw[VEC];
#pragma unroll
        for (int l = 0; l < VEC; ++l) {
            const uint32_t fl = (fl4 >> (8 * l)) & 0xffu;
            R c[19];
#pragma unroll
            for (int q = 0; q < 19; ++q) c[q] = a[q][l];
            R dr = 0;
            CellT<R> m;
            if constexpr (SH) m = moments_g(c, p.fx, p.fy, p.fz, p.rho0, Raw<ST>::invS, dr);
            else m = moments<R>(c, p.fx, p.fy, p.fz);
            const bool solid = MASK && (fl & F_SOLID);
            const float om = (p.hybrid && !(fl & F_BAND)) ? p.omega_s : p.omega;
            R o[19];
#pragma unroll
            for (int q = 0; q < 19; ++q) o[q] = c[q];
            if constexpr (SH) collide_g(o, m, dr, om, Raw<ST>::S);
            else collide<R>(o, m, R(om));
            if (STATS && !solid) {
                add_cell_stats(acc, m);
                if (MASK && (fl & F_TOUCH)) {
                    const IDX xg = id + l;
                    const int xi = (int)(xg % (IDX)p.nx);
                    const IDX row = xg / (IDX)p.nx;
                    if constexpr (SH)
                        add_drag_g(acc, o, Raw<ST>::invS, p.rho0, p.links[xg], p.flags, xi, (int)(row % (IDX)p.ny),
                                   (int)(row / (IDX)p.ny), p.nx, p.ny, p.nz, p.duct);
                    else
                        add_drag(acc, o, p.links[xg], p.flags, xi, (int)(row % (IDX)p.ny), (int)(row / (IDX)p.ny),
                                 p.nx, p.ny, p.nz, p.duct);
                }
            }
            // a vector may run past the end of its row when nx is not a multiple of
            // VEC (l conditional subtractions cover any nx >= 1)
            int x = x0 + l;
#pragma unroll
            for (int k = 0; k < l; ++k) x = x >= p.nx ? x - p.nx : x;
            const bool at_in = p.duct && x == 0, at_out = p.duct && x == p.nx - 1;
#pragma unroll
            for (int q = 0; q < 19; ++q) {
                R v = o[q];
                if constexpr (SH) {
                    if (cx(q) < 0) v = at_in ? inlet_g(q, m.r, kin, p.rho0, Raw<ST>::S) : v;
                } else {
                    if (cx(q) < 0) v = at_in ? inlet_value(q, m.r, kin) : v;
                }
                if (cx(q) > 0) v = at_out ? o[opp(q)] : v;
                // a solid cell keeps its populations (legacy.cu:72-76): slot opp(q) gets its own value
                a[q][l] = solid ? c[opp(q)] : v;
            }
            mr[l] = solid ? 1.f : (float)m.r;
            mu[l] = solid ? 0.f : (float)m.ux;
            mv[l] = solid ? 0.f : (float)m.uy;
            mw[l] = solid ? 0.f : (float)m.uz;
        }
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            if constexpr (SH) stv_raw_sr<ST, VEC>(f + (IDX)opp(q) * N + id, a[q], hsr, q);
            else stv<ST, VEC>(f + (IDX)opp(q) * N + id, q, p.rho0, a[q]);
        }
        if constexpr (MACRO) {
            stv<StoreF32, VEC>(p.rho + id, 0, 0.f, mr);
            stv<StoreF32, VEC>(p.ux + id, 0, 0.f, mu);
            stv<StoreF32, VEC>(p.uy + id, 0, 0.f, mv);
            stv<StoreF32, VEC>(p.uz + id, 0, 0.f, mw);
        }
    }
}

template <class ST, bool MASK, int VEC, int MODE, class IDX>
__global__ void __launch_bounds__(256, 2) aa_even(AAParams p) {
    constexpr bool STATS = MODE == 2;
    const IDX v0 = (IDX)(p.first / VEC), v1 = (IDX)((p.first + p.cells) / VEC);
    double acc[NSTAT];
#pragma unroll
    for (int k = 0; k < NSTAT; ++k) acc[k] = 0.0;
    for (IDX v = v0 + (IDX)blockIdx.x * blockDim.x + threadIdx.x; v < v1; v += (IDX)gridDim.x * blockDim.x)
        even_unit<ST, MASK, VEC, MODE, IDX>(p, v, acc);
    if constexpr (STATS) block_reduce_stats(acc, p.partials);
}

// Neighbour addressing of one cell: 9 row bases (dy,dz in -1..1, periodic in
// y and z) and 3 x positions (periodic in x; in a duct the out-of-range ones
// are never used because those links are marked as not streaming).
template <class IDX>
struct Nbr {
    IDX r[3][3];   // [dy+1][dz+1]
    int xs[3];     // [dx+1]
    __device__ __forceinline__ void init(int x, int y, int z, int nx, int ny, int nz) {
        const int ym = y == 0 ? ny - 1 : y - 1, yp = y == ny - 1 ? 0 : y + 1;
        const int zm = z == 0 ? nz - 1 : z - 1, zp = z == nz - 1 ? 0 : z + 1;
        const int yy[3] = {ym, y, yp};
        const int zz[3] = {zm, z, zp};
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) r[a][b] = ((IDX)zz[b] * ny + yy[a]) * nx;
        xs[0] = x == 0 ? nx - 1 : x - 1;
        xs[1] = x;
        xs[2] = x == nx - 1 ? 0 : x + 1;
    }
    __device__ __forceinline__ IDX at(int dx, int dy, int dz) const { return r[dy + 1][dz + 1] + xs[dx + 1]; }
};

// Element offsets of the 19 population planes, for the odd step's gathers
// (plane opp(q)) and scatters (plane q), computed once per launch (or unit).
template <class IDX>
struct PlaneOffs {
    IDX g[19], s[19];
    __device__ __forceinline__ void init(IDX N) {
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            g[q] = (IDX)opp(q) * N;
            s[q] = (IDX)q * N;
        }
    }
};

// ---------------------------------------------------------------------------
// Odd step
// ---------------------------------------------------------------------------
// One fluid odd-step cell `id` = (x, y, z) with flag byte `fl`; nb gives its
// neighbours' cell indices (nb.at(dx, dy, dz)).
template <class ST, bool MASK, int MODE, class IDX, class NB>
__device__ __forceinline__ void odd_core(const AAParams& p, const PlaneOffs<IDX>& po, IDX id, int x, int y, int z,
                                         uint32_t fl, const NB& nb, double (&acc)[NSTAT]) {
    constexpr bool MACRO = MODE >= 1, STATS = MODE == 2;
    constexpr bool SH = kNarrow<ST>;    // narrow forms: compute in stored units
    using T = typename ST::T;
    using R = typename Real<ST>::type;
    T* __restrict__ f = static_cast<T*>(p.f);
    const int nx = p.nx, ny = p.ny, nz = p.nz;
    const R kin = R(1) + R(3) * p.u_in + R(3) * p.u_in * p.u_in;
    {
        uint32_t lk = 0u;
        if (MASK && (fl & F_SPECIAL)) lk = p.links[id];
        R c[19];
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            // incoming q travels the link x -> x + c_opp(q); if that link does not
            // stream, the value was left in the cell's own slot q
            const bool nn = (lk >> opp(q)) & 1u;
            const IDX src = nn ? (po.s[q] + id) : (po.g[q] + nb.at(-cx(q), -cy(q), -cz(q)));
            if constexpr (SH) c[q] = Raw<ST>::ld(f + src);
            else c[q] = ST::ld(f + src, q, p.rho0);
        }
        R dr = 0;
        CellT<R> m;
        if constexpr (SH) m = moments_g(c, p.fx, p.fy, p.fz, p.rho0, Raw<ST>::invS, dr);
        else m = moments<R>(c, p.fx, p.fy, p.fz);
        const uint32_t hsr = SH ? sr_seed((uint32_t)id + p.salt_base, (float)c[0]) : 0u;   // stochastic rounding
        const float om = (p.hybrid && !(fl & F_BAND)) ? p.omega_s : p.omega;
        R o[19];
#pragma unroll
        for (int q = 0; q < 19; ++q) o[q] = c[q];
        if constexpr (SH) collide_g(o, m, dr, om, Raw<ST>::S);
        else collide<R>(o, m, R(om));
        const bool at_in = p.duct && x == 0, at_out = p.duct && x == nx - 1;
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            const bool nn = (lk >> q) & 1u;
            R v = o[q];
            if constexpr (SH) {
                if (cx(q) < 0) v = (nn && at_in) ? inlet_g(q, m.r, kin, p.rho0, Raw<ST>::S) : v;
            } else {
                if (cx(q) < 0) v = (nn && at_in) ? inlet_value(q, m.r, kin) : v;
            }
            if (cx(q) > 0) v = (nn && at_out) ? o[opp(q)] : v;
            const IDX dst = nn ? (po.g[q] + id) : (po.s[q] + nb.at(cx(q), cy(q), cz(q)));
            if constexpr (SH) Raw<ST>::st_sr(f + dst, v, sr_word(hsr, 2 * q));
            else ST::st(f + dst, q, p.rho0, v);
        }
        if (MACRO) { p.rho[id] = (float)m.r; p.ux[id] = (float)m.ux; p.uy[id] = (float)m.uy; p.uz[id] = (float)m.uz; }
        if (STATS) {
            add_cell_stats(acc, m);
            if (MASK && (fl & F_TOUCH)) {
                if constexpr (SH) add_drag_g(acc, o, Raw<ST>::invS, p.rho0, lk, p.flags, x, y, z, nx, ny, nz, p.duct);
                else add_drag(acc, o, lk, p.flags, x, y, z, nx, ny, nz, p.duct);
            }
        }
    }
}

// A solid cell's odd step: frozen populations, rest-state macro fields.
template <int MODE, class IDX>
__device__ __forceinline__ void odd_solid(const AAParams& p, IDX id) {
    if (MODE >= 1) { p.rho[id] = 1.f; p.ux[id] = 0.f; p.uy[id] = 0.f; p.uz[id] = 0.f; }
}

// One odd-step cell (x, y, z).
template <class ST, bool MASK, int MODE, class IDX>
__device__ __forceinline__ void odd_cell_at(const AAParams& p, const PlaneOffs<IDX>& po, int x, int y, int z,
                                            double (&acc)[NSTAT]) {
    const IDX id = ((IDX)z * (IDX)p.ny + (IDX)y) * (IDX)p.nx + (IDX)x;
    const uint32_t fl = MASK ? p.flags[id] : 0u;
    if (MASK && (fl & F_SOLID)) {
        odd_solid<MODE>(p, id);
        return;
    }
    Nbr<IDX> nb;
    nb.init(x, y, z, p.nx, p.ny, p.nz);
    odd_core<ST, MASK, MODE, IDX>(p, po, id, x, y, z, fl, nb, acc);
}

// One odd-step cell given by its row (= z*ny + y) and x (the batched step's form).
template <class ST, bool MASK, int MODE, class IDX>
__device__ __forceinline__ void odd_cell(const AAParams& p, const PlaneOffs<IDX>& po, IDX row, int x,
                                         double (&acc)[NSTAT]) {
    odd_cell_at<ST, MASK, MODE, IDX>(p, po, x, (int)(row % p.ny), (int)(row / p.ny), acc);
}

// Neighbour addressing of a thread that marches along z at a fixed (x, y): the
// three row offsets and x positions are formed once, and the three plane bases
// (periodic in z) roll forward by one plane per step.
template <class IDX>
struct NbrZ {
    IDX zb[3];     // [dz+1]: first cell of planes z-1, z, z+1
    IDX yo[3];     // [dy+1]: first cell of rows y-1, y, y+1 inside a plane (periodic)
    int xs[3];     // [dx+1]: x-1, x, x+1 (periodic)
    __device__ __forceinline__ void init(int x, int y, int z, int nx, int ny, int nz) {
        yo[0] = (IDX)(y == 0 ? ny - 1 : y - 1) * (IDX)nx;
        yo[1] = (IDX)y * (IDX)nx;
        yo[2] = (IDX)(y == ny - 1 ? 0 : y + 1) * (IDX)nx;
        xs[0] = x == 0 ? nx - 1 : x - 1;
        xs[1] = x;
        xs[2] = x == nx - 1 ? 0 : x + 1;
        const IDX plane = (IDX)nx * (IDX)ny;
        zb[0] = (IDX)(z == 0 ? nz - 1 : z - 1) * plane;
        zb[1] = (IDX)z * plane;
        zb[2] = (IDX)(z == nz - 1 ? 0 : z + 1) * plane;
    }
    // from plane z to plane z + 1
    __device__ __forceinline__ void advance(int z, int nz, IDX plane) {
        zb[0] = zb[1];
        zb[1] = zb[2];
        zb[2] = z + 2 >= nz ? (IDX)(z + 2 - nz) * plane : zb[2] + plane;
    }
    __device__ __forceinline__ IDX at(int dx, int dy, int dz) const { return zb[dz + 1] + yo[dy + 1] + (IDX)xs[dx + 1]; }
    __device__ __forceinline__ IDX id() const { return zb[1] + yo[1] + (IDX)xs[1]; }
};

// Odd step of grids without a solid mask: a block owns blockDim.x cells of one
// row segment (one y) over a run of p.zrun consecutive planes and marches along
// z, one cell per thread and plane.  The grid holds every (segment, y, run) once (aa_odd_blocks), so the
// hardware balances the runs over the SMs; the neighbour addressing costs a few
// instructions per plane instead of a division and nine row products per cell.
template <class ST, bool MASK, int MODE, class IDX>
__global__ void __launch_bounds__(256, ST::kId == 3 ? 2 : (MASK ? 4 : 3)) aa_odd(AAParams p) {
    constexpr bool STATS = MODE == 2;
    const int bx = blockDim.x;
    const int segs = (p.nx + bx - 1) / bx;
    const IDX plane = (IDX)p.nx * (IDX)p.ny;
    const int zlo = (int)(p.first / (int64_t)plane);
    const int zhi = (int)((p.first + p.cells) / (int64_t)plane);
    int b = (int)blockIdx.x;
    const int seg = b % segs;
    b /= segs;
    const int y = b % p.ny;
    const int z0 = zlo + (b / p.ny) * p.zrun;
    const int z1 = min(zhi, z0 + p.zrun);
    const int x = seg * bx + (int)threadIdx.x;
    double acc[NSTAT];
#pragma unroll
    for (int k = 0; k < NSTAT; ++k) acc[k] = 0.0;
    if (x < p.nx) {
        PlaneOffs<IDX> po;
        po.init((IDX)p.N);
        NbrZ<IDX> nb;
        nb.init(x, y, z0, p.nx, p.ny, p.nz);
        for (int z = z0; z < z1; ++z) {
            const IDX id = nb.id();
            const uint32_t fl = MASK ? p.flags[id] : 0u;
            if (MASK && (fl & F_SOLID)) odd_solid<MODE>(p, id);
            else odd_core<ST, MASK, MODE, IDX>(p, po, id, x, y, z, fl, nb, acc);
            nb.advance(z, p.nz, plane);
        }
    }
    if constexpr (STATS) block_reduce_stats(acc, p.partials);
}

// Odd step over rows, for grids with a solid mask: one cell per thread; a block
// takes every gridDim.x-th row of its x segment (blockIdx.y), and steps the row's
// (y, z) by a fixed stride instead of dividing per cell.  At the 64 registers
// of 4 blocks/SM that the mask's flag and link reads leave, the z-marching
// form's rolling addresses measured more instructions per cell (20.6 against
// 17.6 warp-instructions) and a slower step on the duct.
template <class ST, int MODE, class IDX>
__global__ void __launch_bounds__(256, ST::kId == 3 ? 2 : 4) aa_odd_rows(AAParams p) {
    constexpr bool STATS = MODE == 2;
    const int x = (int)blockIdx.y * (int)blockDim.x + (int)threadIdx.x;
    const int rows = (int)(p.cells / p.nx);
    const int z0 = (int)(p.first / ((int64_t)p.nx * p.ny));
    const int S = (int)gridDim.x;
    const int sy = S % p.ny, sz = S / p.ny;           // the stride in (y, z)
    int y = (int)blockIdx.x % p.ny, z = z0 + (int)blockIdx.x / p.ny;
    double acc[NSTAT];
#pragma unroll
    for (int k = 0; k < NSTAT; ++k) acc[k] = 0.0;
    if (x < p.nx) {
        PlaneOffs<IDX> po;
        po.init((IDX)p.N);
        for (int r = (int)blockIdx.x; r < rows; r += S) {
            odd_cell_at<ST, true, MODE, IDX>(p, po, x, y, z, acc);
            y += sy;
            z += sz;
            if (y >= p.ny) { y -= p.ny; ++z; }
        }
    }
    if constexpr (STATS) block_reduce_stats(acc, p.partials + (size_t)blockIdx.y * gridDim.x * NSTAT);
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
        Nbr<int64_t> nb;
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

}  // namespace

// Planes per block of the odd step: the longest run (at most 8) that still
// leaves about eight waves of resident blocks, so the hardware's block
// scheduling keeps the SMs evenly loaded to the end of the launch.
int aa_odd_zrun(int nx, int ny, int64_t planes, bool mask, int storage, int threads) {
    const int64_t segs = (nx + threads - 1) / threads;
    const int bps = storage == 3 ? 2 : (mask ? 4 : 3);     // aa_odd's launch bounds
    const int64_t target = (int64_t)num_sms() * bps * 8;
    const int64_t run = segs * ny * planes / std::max<int64_t>(target, 1);
    return (int)std::min<int64_t>(std::max<int64_t>(run, 1), 8);
}

int64_t aa_odd_blocks(int nx, int ny, int64_t planes, bool mask, int storage, int threads) {
    const int64_t segs = (nx + threads - 1) / threads;
    const int run = aa_odd_zrun(nx, ny, planes, mask, storage, threads);
    return segs * ny * ((planes + run - 1) / run);
}

int64_t aa_odd_grid(int nx, int ny, int64_t planes, bool mask, int storage, LaunchCfg cfg) {
    if (!mask) return aa_odd_blocks(nx, ny, planes, false, storage, cfg.threads);
    const int segs = (nx + cfg.threads - 1) / cfg.threads;
    return (int64_t)std::max(1, cfg.blocks / segs) * segs;
}

namespace {

template <class ST, int MODE, class IDX>
void launch_mode(const AAParams& p, int parity, LaunchCfg cfg, cudaStream_t s) {
    const bool mask = p.flags != nullptr;
    // consecutive cells per thread: four in FP32 (16-byte accesses; two, with 8-byte accesses,
    // when the launch also writes macro fields or statistics, which would spill at four), four
    // in F16/BF16 (8-byte accesses), one in FP64 (8-byte accesses)
    constexpr int V = ST::kId == 0 ? (MODE == 0 ? 4 : 2) : (ST::kId == 3 ? 1 : 4);
    if (parity == 0) {
        const int64_t span = p.first | p.cells;      // both must be multiples of the vector width
        if (V == 4 && span % 4 != 0 && span % 2 == 0) {
            if (mask) aa_even<ST, true, 2, MODE, IDX><<<cfg.blocks, cfg.threads, 0, s>>>(p);
            else aa_even<ST, false, 2, MODE, IDX><<<cfg.blocks, cfg.threads, 0, s>>>(p);
        } else if (span % V == 0) {
            if (mask) aa_even<ST, true, V, MODE, IDX><<<cfg.blocks, cfg.threads, 0, s>>>(p);
            else aa_even<ST, false, V, MODE, IDX><<<cfg.blocks, cfg.threads, 0, s>>>(p);
        } else {
            if (mask) aa_even<ST, true, 1, MODE, IDX><<<cfg.blocks, cfg.threads, 0, s>>>(p);
            else aa_even<ST, false, 1, MODE, IDX><<<cfg.blocks, cfg.threads, 0, s>>>(p);
        }
    } else {
        if (mask) {
            const int segs = (p.nx + cfg.threads - 1) / cfg.threads;
            const dim3 grid((unsigned)std::max(1, cfg.blocks / segs), (unsigned)segs);
            aa_odd_rows<ST, MODE, IDX><<<grid, cfg.threads, 0, s>>>(p);
            return;
        }
        const int64_t planes = p.cells / ((int64_t)p.nx * p.ny);
        AAParams q = p;
        q.zrun = aa_odd_zrun(p.nx, p.ny, planes, false, ST::kId, cfg.threads);
        const int64_t blocks = aa_odd_blocks(p.nx, p.ny, planes, false, ST::kId, cfg.threads);
        if (blocks <= 0) return;
        aa_odd<ST, false, MODE, IDX><<<(unsigned)blocks, cfg.threads, 0, s>>>(q);
    }
}

template <class ST, class IDX>
void launch_idx(const AAParams& p, int parity, LaunchCfg cfg, cudaStream_t s) {
    const int mode = p.stats ? 2 : (p.macro ? 1 : 0);
    if (mode == 0) launch_mode<ST, 0, IDX>(p, parity, cfg, s);
    else if (mode == 1) launch_mode<ST, 1, IDX>(p, parity, cfg, s);
    else launch_mode<ST, 2, IDX>(p, parity, cfg, s);
}

template <class ST>
cudaError_t launch_typed(const AAParams& p, int parity, LaunchCfg cfg, cudaStream_t s) {
    // 32-bit element offsets while every slot index 19*N fits in them
    if ((uint64_t)p.N * 19u < (1ull << 32)) launch_idx<ST, uint32_t>(p, parity, cfg, s);
    else launch_idx<ST, int64_t>(p, parity, cfg, s);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Batched step: many independent instances (each its own AAParams: grid,
// populations, flags, rates, boundary) advanced by ONE persistent launch.  The
// work is a list of units {instance, first, count, -}: even steps count
// two-cell vectors, odd steps count cells.  Blocks
// take units round-robin; with statistics each unit's FP64 sums go to its own
// slot and batch_finalize adds the slots of each instance in order.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void block_reduce_into(double (&acc)[NSTAT], double* out) {
    __shared__ double red[32][NSTAT];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < NSTAT; ++k) {
        double v = acc[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[warp][k] = v;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < NSTAT; ++k) {
            double v = lane < nw ? red[lane][k] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if (lane == 0) out[k] = v;
        }
    }
    __syncthreads();
}

// Even units count vectors of w.w cells: the single solver's vector width for
// the instance's cell count (F16/BF16: 4, 2 or 1; FP32: 2 or 1), so the
// stochastic rounding draws the same bits as stepping the instance alone.
template <class ST, int MODE>
__global__ void __launch_bounds__(256, 2) aa_batch_even(const AAParams* __restrict__ inst, const int4* __restrict__ units,
                                                     int nunits, double* __restrict__ partials) {
    constexpr bool STATS = MODE == 2;
    __shared__ AAParams p;   // the unit's instance, read by every thread (broadcast)
    for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
        const int4 w = units[u];
        __syncthreads();
        if (threadIdx.x == 0) p = inst[w.x];
        __syncthreads();
        double acc[NSTAT];
#pragma unroll
        for (int k = 0; k < NSTAT; ++k) acc[k] = 0.0;
        for (int v = w.y + threadIdx.x; v < w.y + w.z; v += blockDim.x) {
            if (kNarrow<ST> && w.w == 4) {
                if constexpr (kNarrow<ST>) even_unit<ST, true, 4, MODE, uint32_t>(p, (uint32_t)v, acc);
            } else if (w.w == 2) {
                even_unit<ST, true, 2, MODE, uint32_t>(p, (uint32_t)v, acc);
            } else {
                even_unit<ST, true, 1, MODE, uint32_t>(p, (uint32_t)v, acc);
            }
        }
        if constexpr (STATS) block_reduce_into(acc, partials + (size_t)u * NSTAT);
    }
}

template <class ST, int MODE>
__global__ void __launch_bounds__(256, 4) aa_batch_odd(const AAParams* __restrict__ inst, const int4* __restrict__ units,
                                                       int nunits, double* __restrict__ partials) {
    constexpr bool STATS = MODE == 2;
    __shared__ AAParams p;   // the unit's instance, read by every thread (broadcast)
    for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
        const int4 w = units[u];
        __syncthreads();
        if (threadIdx.x == 0) p = inst[w.x];
        __syncthreads();
        double acc[NSTAT];
#pragma unroll
        for (int k = 0; k < NSTAT; ++k) acc[k] = 0.0;
        PlaneOffs<uint32_t> po;
        po.init((uint32_t)p.N);
        // consecutive cells across row ends, so narrow rows leave no thread idle
        for (int c = w.y + (int)threadIdx.x; c < w.y + w.z; c += (int)blockDim.x) {
            const int row = c / p.nx;
            odd_cell<ST, true, MODE, uint32_t>(p, po, (uint32_t)row, c - row * p.nx, acc);
        }
        if constexpr (STATS) block_reduce_into(acc, partials + (size_t)u * NSTAT);
    }
}

// out[i*NSTAT + k] = sum of partials[u*NSTAT + k] over the units u of instance i,
// which are the contiguous range first[i] .. first[i+1]-1 (fixed order)
__global__ void batch_finalize(const double* __restrict__ partials, const int* __restrict__ first, int n,
                               double* __restrict__ out) {
    const int i = blockIdx.x;
    if (i >= n) return;
    double acc[NSTAT];
#pragma unroll
    for (int k = 0; k < NSTAT; ++k) acc[k] = 0.0;
    for (int u = first[i] + threadIdx.x; u < first[i + 1]; u += blockDim.x)
#pragma unroll
        for (int k = 0; k < NSTAT; ++k) acc[k] += partials[(size_t)u * NSTAT + k];
    block_reduce_into(acc, out + (size_t)i * NSTAT);
}

}  // namespace

template <class ST>
void launch_batch_typed(const AAParams* d_inst, const int4* d_units, int nunits, int parity, int stats, int blocks,
                        int threads, double* partials, cudaStream_t s) {
    if (parity == 0) {
        if (stats) aa_batch_even<ST, 2><<<blocks, threads, 0, s>>>(d_inst, d_units, nunits, partials);
        else aa_batch_even<ST, 0><<<blocks, threads, 0, s>>>(d_inst, d_units, nunits, partials);
    } else {
        if (stats) aa_batch_odd<ST, 2><<<blocks, threads, 0, s>>>(d_inst, d_units, nunits, partials);
        else aa_batch_odd<ST, 0><<<blocks, threads, 0, s>>>(d_inst, d_units, nunits, partials);
    }
}

cudaError_t launch_aa_batch(const AAParams* d_inst, const int4* d_units, int nunits, int parity, int stats,
                            int storage, int blocks, int threads, double* partials, cudaStream_t s) {
    if (nunits <= 0) return cudaSuccess;
    switch (storage) {
        case 0: launch_batch_typed<StoreF32>(d_inst, d_units, nunits, parity, stats, blocks, threads, partials, s); break;
        case 1: launch_batch_typed<StoreF16>(d_inst, d_units, nunits, parity, stats, blocks, threads, partials, s); break;
        case 2: launch_batch_typed<StoreBF16>(d_inst, d_units, nunits, parity, stats, blocks, threads, partials, s); break;
        default: return cudaErrorInvalidValue;   // the batch runs FP32, F16 or BF16 populations
    }
    return cudaGetLastError();
}

cudaError_t launch_batch_finalize(const double* partials, const int* d_first, int n, double* out, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    batch_finalize<<<n, 256, 0, s>>>(partials, d_first, n, out);
    return cudaGetLastError();
}

cudaError_t launch_aa_step(const AAParams& p, int storage, int parity, LaunchCfg cfg, cudaStream_t s) {
    switch (storage) {
        case 0: return launch_typed<StoreF32>(p, parity, cfg, s);
        case 1: return launch_typed<StoreF16>(p, parity, cfg, s);
        case 2: return launch_typed<StoreBF16>(p, parity, cfg, s);
        case 3: return launch_typed<StoreF64>(p, parity, cfg, s);
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_aa_materialize(const AAParams& p, int storage, int parity, float* out, cudaStream_t s) {
    const int blocks = num_sms() * 8;
    switch (storage) {
        case 0: aa_materialize<StoreF32><<<blocks, 256, 0, s>>>(p, parity, out); break;
        case 1: aa_materialize<StoreF16><<<blocks, 256, 0, s>>>(p, parity, out); break;
        case 2: aa_materialize<StoreBF16><<<blocks, 256, 0, s>>>(p, parity, out); break;
        case 3: aa_materialize<StoreF64><<<blocks, 256, 0, s>>>(p, parity, out); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace lbm
