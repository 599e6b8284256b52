// HOME moment-only step (src/lbm/lbm3d_home.cu:37-286): the state is 10
// moments per cell [rho, ux, uy, uz, Sxx, Sxy, Sxz, Syy, Syz, Szz]; every step
// rebuilds each neighbour's post-collision population from its moments,
// gathers the 19 incoming populations and stores their moments.
//
// The reference rebuilds f_q 19 times per cell from global loads of the
// neighbour's 10 moments (190 loads and ~1.1 kFLOP per cell).  Here a block
// owns a 32 x 8 tile of an (x,y) plane and marches along z over a chunk of
// planes.  Every thread handles TWO x-adjacent cells, so the arithmetic runs on
// Blackwell's paired FP32 instructions (FFMA2/FADD2/FMUL2: one issue slot for
// both cells) and every global access moves 8 bytes (FP32) or 4 bytes
// (F16/BF16) of two cells at once.  Warps 0-3 hold the tile (16 pairs per
// row, two rows per warp), warp 4 the two halo rows (pairs) and warp 5 the two
// halo columns and the four corners (single cells).
//   * When a plane's moments arrive (requested one plane ahead), every
//     position rebuilds its post-collision populations ONCE from the identity
//         f*_q = w_q [rho + 3 c_q.(rho u) + 4.5 Q_q : (rho u u + (1-w) S)],
//     Q_q = c_q c_q - I/3 (src/lbm/lbm3d_home.cu:57-80 rearranged:
//     4.5 (c.u)^2 - 1.5 u^2 = 4.5 Q:uu), in opposite-pair form.
//   * It writes f*_q straight into the shared ring slot of the cell that will
//     gather it, (x + c_x, y + c_y) in the tile (destination indexing): the
//     ring holds exactly one 32 x 8 plane per population and slot, and the
//     gather reads all 19 populations of a pair from its own position with
//     aligned 8-byte loads.  The ring is grouped by c_z: the up-going group
//     lives 3 planes, the in-plane group 2 and the down-going group 1
//     (38 planes of 256 floats: 38.9 KB per block).
//   * Sources write unconditionally (a solid source or a halo position outside
//     a duct writes a value nobody uses).  A link that does not stream (solid
//     neighbour, duct inlet/outlet) is resolved by the gathering cell itself,
//     which is the only reader of its slot: it replaces the ring value by the
//     bounce-back, inlet or outlet population computed from its own moments.
//   * The populations are shifted, g_q = f*_q - w_q rho0 (see Coef), and every
//     product with 1/3, 1/6 or 1/18 is rounded as if the constant were exact
//     (mulk), so FP32 rounding adds no drift of mass, momentum or stress.
//   * F16/BF16 moments are stored with stochastic rounding (cvt.rs), the two
//     cells of a pair in one conversion.
// DRAM traffic is the 10 moments read once and written once (80 B per cell in
// FP32, 40 B in F16/BF16) plus the halo re-reads that L2 does not absorb.
#include <type_traits>

#include "lbm_common.cuh"
#include "lbm_internal.h"

namespace lbm {
namespace {

constexpr int TX = 32;                 // tile width (cells), 16 pairs
constexpr int TY = 8;                  // tile height (rows)
constexpr int NCW = TY / 2;            // tile warps: two rows of 16 pairs each
constexpr int NT = (NCW + 2) * 32;     // + the halo-row warp + the halo-column warp
constexpr int PL = TX * TY;            // positions per population plane of the ring

// shared ring (destination-indexed), grouped by c_z: UP[3][5][PL], MID[2][9][PL], DN[5][PL]
constexpr int UP_SZ = 5 * PL, MID_SZ = 9 * PL, DN_SZ = 5 * PL;
constexpr int MID_OFF = 3 * UP_SZ, DN_OFF = MID_OFF + 2 * MID_SZ;
constexpr int TRASH_OFF = DN_OFF + DN_SZ;           // 4 words that take stores nobody reads
constexpr int SMEM_FLOATS = TRASH_OFF + 4;

// offset of q inside its group (UP: 5,11,12,15,16; MID: 0,1,2,3,4,7,8,9,10; DN: 6,13,14,17,18)
__host__ __device__ constexpr int gofs(int q) {
    constexpr int t[19] = {0, 1, 2, 3, 4, 0, 0, 5, 6, 7, 8, 1, 2, 1, 2, 3, 4, 3, 4};
    return t[q] * PL;
}

// the ring groups that hold the populations leaving plane p (UP slot given:
// the step loop rotates the three UP slots instead of dividing by 3)
template <class E>
struct Ring {
    E* up;
    E* mid;
    E* dn;
    __device__ __forceinline__ Ring(E* sm, int p, int upslot) {
        up = sm + upslot * UP_SZ;
        mid = sm + MID_OFF + (p & 1) * MID_SZ;
        dn = sm + DN_OFF;
    }
    template <int q>
    __device__ __forceinline__ E* at(int pos) const {
        return (cz(q) > 0 ? up : (cz(q) == 0 ? mid : dn)) + gofs(q) + pos;
    }
};

// ---- scalar and paired FP32 arithmetic with identical rounding -------------
__device__ __forceinline__ float vadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float vsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float vmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float vfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ float vsplat(float s, float) { return s; }
__device__ __forceinline__ float2 vadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 vsub(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 vmul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 vfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 vsplat(float s, float2) { return make_float2(s, s); }
// FP64 (the reference form): one double, or a pair of doubles with the same
// interface as float2
struct D2 {
    double x, y;
};
__device__ __forceinline__ double vadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double vsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double vmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double vfma(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ double vsplat(float s, double) { return s; }
__device__ __forceinline__ D2 vadd(D2 a, D2 b) { return {__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y)}; }
__device__ __forceinline__ D2 vsub(D2 a, D2 b) { return {__dsub_rn(a.x, b.x), __dsub_rn(a.y, b.y)}; }
__device__ __forceinline__ D2 vmul(D2 a, D2 b) { return {__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)}; }
__device__ __forceinline__ D2 vfma(D2 a, D2 b, D2 c) { return {__fma_rn(a.x, b.x, c.x), __fma_rn(a.y, b.y, c.y)}; }
__device__ __forceinline__ D2 vsplat(float s, D2) { return {(double)s, (double)s}; }
__device__ __forceinline__ D2 vsplat(double s, D2) { return {s, s}; }
__device__ __forceinline__ double vsplat(double s, double) { return s; }
using lbm::mulk;   // the float, float2 and double forms, next to the pair of doubles below
__device__ __forceinline__ D2 mulk(D2 x, float hi, float lo) { return {lbm::mulk(x.x, hi, lo), lbm::mulk(x.y, hi, lo)}; }

// element type of the ring and of one cell's arithmetic (E), and of a pair (V)
template <class T> struct HomeTypes {
    using E = float;
    using V = float2;
};
template <> struct HomeTypes<double> {
    using E = double;
    using V = D2;
};
// one aligned pair in shared memory
__device__ __forceinline__ void st_pair(float* p, float2 v) { *reinterpret_cast<float2*>(p) = v; }
__device__ __forceinline__ void st_pair(double* p, D2 v) { *reinterpret_cast<double2*>(p) = make_double2(v.x, v.y); }
__device__ __forceinline__ float2 ld_pair(const float* p) { return *reinterpret_cast<const float2*>(p); }
__device__ __forceinline__ D2 ld_pair(const double* p) {
    const double2 v = *reinterpret_cast<const double2*>(p);
    return {v.x, v.y};
}
// 1/r where r > 0, else 0 (u = 0 for an empty cell, home.cu:258-262)
__device__ __forceinline__ float2 vrcp_pos(float2 r) {
    return make_float2(r.x > 0.f ? __frcp_rn(r.x) : 0.f, r.y > 0.f ? __frcp_rn(r.y) : 0.f);
}
__device__ __forceinline__ D2 vrcp_pos(D2 r) { return {r.x > 0.0 ? 1.0 / r.x : 0.0, r.y > 0.0 ? 1.0 / r.y : 0.0}; }
// the inlet population of a direction with c_x = +1, shifted by w_q rho0:
// feq(rho, (u_in, 0, 0)) - w_q rho0 (src/lbm/lbm3d_legacy.cu:54-58 form)
template <int q>
__device__ __forceinline__ float inlet_shifted(float rho, float u_in, float r0) {
    return feq_ref(q, rho, u_in, 0.f, 0.f) - wq(q) * r0;
}
template <int q>
__device__ __forceinline__ double inlet_shifted(double rho, float u_in, float r0) {
    constexpr double w = q == 0 ? 1.0 / 3.0 : (q <= 6 ? 1.0 / 18.0 : 1.0 / 36.0);
    const double u = u_in;
    return w * rho * (1.0 + 3.0 * u + 3.0 * u * u) - w * (double)r0;
}

// Rebuild coefficients of one cell (V = float) or two (V = float2), pre-scaled
// by w1 = 1/18 (w0 = 6 w1, w2 = w1/2):
//   P = w1 (rho - rho0 - 1.5 tr B),  a_k = 3 w1 rho u_k,  b_kk = 4.5 w1 B_kk,
//   b_kl = 9 w1 B_kl,  B = rho u u + (1 - w) S.
// The populations built from them are SHIFTED, g_q = f*_q - w_q rho0: the
// moments gathered from g carry the small deviations from the rest state
// instead of the O(1) constant part (sum g = rho - rho0, sum c c g = Pi -
// rho0/3 I), which keeps the FP32 cancellation in S = Pi - rho/3 I - rho u u
// at the size of the deviations.
template <class V>
struct Coef {
    V P, ax, ay, az, bxx, byy, bzz, bxy, bxz, byz;
    template <class S>
    __device__ __forceinline__ void set(const V (&m)[10], S omw_s, float r0) {
        const V omw = vsplat(omw_s, V{});
        const V r = m[0];
        const V jx = vmul(r, m[1]), jy = vmul(r, m[2]), jz = vmul(r, m[3]);
        const V Bxx = vfma(jx, m[1], vmul(omw, m[4]));
        const V Bxy = vfma(jx, m[2], vmul(omw, m[5]));
        const V Bxz = vfma(jx, m[3], vmul(omw, m[6]));
        const V Byy = vfma(jy, m[2], vmul(omw, m[7]));
        const V Byz = vfma(jy, m[3], vmul(omw, m[8]));
        const V Bzz = vfma(jz, m[3], vmul(omw, m[9]));
        P = mulk(vfma(vsplat(-1.5f, V{}), vadd(vadd(Bxx, Byy), Bzz), vsub(r, vsplat(r0, V{}))), K18_HI, K18_LO);
        const V b45 = vsplat(0.25f, V{}), b9 = vsplat(0.5f, V{});   // 4.5/18 and 9/18, exact
        ax = mulk(jx, K6_HI, K6_LO); ay = mulk(jy, K6_HI, K6_LO); az = mulk(jz, K6_HI, K6_LO);
        bxx = vmul(b45, Bxx); byy = vmul(b45, Byy); bzz = vmul(b45, Bzz);
        bxy = vmul(b9, Bxy); bxz = vmul(b9, Bxz); byz = vmul(b9, Byz);
    }
};

// Post-collision population q from the coefficients: the same expression for
// every position and role (tile cell, halo, bounce-back), in opposite-pair form.
template <int q, class V>
__device__ __forceinline__ V fpost(const Coef<V>& c) {
    const V half = vsplat(0.5f, V{});
    if constexpr (q == 0) {
        return vmul(vsplat(6.0f, V{}), c.P);
    } else if constexpr (q <= 6) {
        constexpr int k = (q - 1) / 2;               // axis
        constexpr bool plus = (q & 1) == 1;
        const V b = vadd(c.P, k == 0 ? c.bxx : (k == 1 ? c.byy : c.bzz));
        const V a = k == 0 ? c.ax : (k == 1 ? c.ay : c.az);
        return plus ? vadd(b, a) : vsub(b, a);
    } else {
        // diagonal in the plane of axes (i, j), i < j; sign s of the second component
        constexpr int X = cx(q), Y = cy(q), Z = cz(q);
        constexpr int i = X != 0 ? 0 : 1;
        constexpr int j = Z != 0 ? 2 : 1;
        constexpr int si = i == 0 ? X : Y;
        constexpr int sj = j == 1 ? Y : Z;
        const V bi = vadd(c.P, i == 0 ? c.bxx : c.byy);          // P + b_ii
        const V b = vadd(bi, j == 1 ? c.byy : c.bzz);             // + b_jj
        const V bij = (i == 0 && j == 1) ? c.bxy : ((i == 0) ? c.bxz : c.byz);
        const V ai = i == 0 ? c.ax : c.ay;
        const V aj = j == 1 ? c.ay : c.az;
        if constexpr (si * sj > 0) {
            const V bp = vadd(b, bij), sp = vadd(ai, aj);
            return vmul(half, si > 0 ? vadd(bp, sp) : vsub(bp, sp));
        } else {
            const V bm = vsub(b, bij), sn = vsub(ai, aj);
            return vmul(half, si > 0 ? vadd(bm, sn) : vsub(bm, sn));
        }
    }
}

template <int q> struct QI { static constexpr int value = q; };
template <int Q0, int Q1, class F>
__device__ __forceinline__ void static_for(F&& fn) {
    if constexpr (Q0 < Q1) {
        fn(QI<Q0>{});
        static_for<Q0 + 1, Q1>(fn);
    }
}

// ---- moment storage: F32 as is; F16/BF16 keep rho - rho0, u and S ---------
// (F16 scaled by 2^10, exact, as the F16 populations are)
template <class T> struct MomStore;
// Moments are read with ld.global.cg (kept in L2, not in L1): each is read once
// per block, and L1 left free measured 1-3 % faster than the read-only path
// (FP32) and than plain loads (F16/BF16)
template <> struct MomStore<float> {
    static constexpr float S = 1.0f, invS = 1.0f;
    __device__ __forceinline__ static float ld(const float* p) { return __ldcg(p); }
    __device__ __forceinline__ static float2 ld2(const float* p) { return __ldcg(reinterpret_cast<const float2*>(p)); }
};
template <> struct MomStore<__half> {
    static constexpr float S = kF16Scale, invS = kF16Inv;
    __device__ __forceinline__ static float ld(const __half* p) { return __half2float(__ldcg(p)); }
    __device__ __forceinline__ static float2 ld2(const __half* p) {
        return __half22float2(__ldcg(reinterpret_cast<const __half2*>(p)));
    }
};
template <> struct MomStore<double> {
    static constexpr float S = 1.0f, invS = 1.0f;
    __device__ __forceinline__ static double ld(const double* p) { return __ldg(p); }
    __device__ __forceinline__ static D2 ld2(const double* p) {
        const double2 v = __ldg(reinterpret_cast<const double2*>(p));
        return {v.x, v.y};
    }
};
template <> struct MomStore<__nv_bfloat16> {
    static constexpr float S = 1.0f, invS = 1.0f;
    __device__ __forceinline__ static float ld(const __nv_bfloat16* p) { return __bfloat162float(__ldcg(p)); }
    __device__ __forceinline__ static float2 ld2(const __nv_bfloat16* p) {
        return __bfloat1622float2(__ldcg(reinterpret_cast<const __nv_bfloat162*>(p)));
    }
};
// stored value -> moment (k = 0 is rho, stored as rho - rho0 in the narrow forms)
template <class T>
__device__ __forceinline__ float mom_of(float v, int k, float r0) {
    if constexpr (sizeof(T) == 4) return v;
    else return __fmaf_rn(v, MomStore<T>::invS, k == 0 ? r0 : 0.f);
}
template <class T>
__device__ __forceinline__ double mom_of(double v, int k, float r0) { return v; }
template <class T>
__device__ __forceinline__ D2 mom_of(D2 v, int k, float r0) { return v; }
template <class T>
__device__ __forceinline__ float2 mom_of(float2 v, int k, float r0) {
    if constexpr (sizeof(T) == 4) return v;
    else {
        const float s = k == 0 ? r0 : 0.f;
        return vfma(v, vsplat(MomStore<T>::invS, float2{}), make_float2(s, s));
    }
}

// The 10 new moments of two cells (FP32: two float2 stores per moment pair;
// F16/BF16: one stochastically rounded conversion of the two cells per moment,
// the ten random words drawn from one hash of the pair's first cell index and
// its first two values).  `both`: both cells stored and the pair 8-byte (or
// 4-byte) aligned; otherwise the cells go one by one as `own0` / `own1` say.
template <class T, class IDX, class V>
__device__ __forceinline__ void store_pair(T* op, IDX N, float r0, const V (&out)[10], uint32_t salt, bool both,
                                           bool own0, bool own1) {
    if constexpr (sizeof(T) == 8) {
        if (both) {
#pragma unroll
            for (int c = 0; c < 10; ++c) *reinterpret_cast<double2*>(op + (IDX)c * N) = make_double2(out[c].x, out[c].y);
        } else {
#pragma unroll
            for (int c = 0; c < 10; ++c) {
                if (own0) op[(IDX)c * N] = out[c].x;
                if (own1) op[(IDX)c * N + 1] = out[c].y;
            }
        }
    } else if constexpr (sizeof(T) == 4) {
        if (both) {
#pragma unroll
            for (int c = 0; c < 10; ++c) *reinterpret_cast<float2*>(op + (IDX)c * N) = out[c];
        } else {
#pragma unroll
            for (int c = 0; c < 10; ++c) {
                if (own0) op[(IDX)c * N] = out[c].x;
                if (own1) op[(IDX)c * N + 1] = out[c].y;
            }
        }
    } else {
        constexpr bool F16 = std::is_same<T, __half>::value;
        const float sc = MomStore<T>::S;
        const uint32_t h = mix32(salt ^ __float_as_uint(out[0].x) ^ (__float_as_uint(out[0].y) * 0x9e3779b9u));
        uint16_t* o = reinterpret_cast<uint16_t*>(op);
#pragma unroll
        for (int c = 0; c < 10; ++c) {
            uint32_t rb = h * (2u * c + 1u) * 0x85ebca6bu;
            rb ^= rb >> 15;
            const float s = c == 0 ? r0 : 0.f;
            const float a = (out[c].x - s) * sc, b = (out[c].y - s) * sc;
            const uint32_t d = F16 ? cvt_rs_f16x2(a, b, rb) : cvt_rs_bf16x2(a, b, rb);
            if (both) {
                *reinterpret_cast<uint32_t*>(o + (IDX)c * N) = d;
            } else {
                if (own0) o[(IDX)c * N] = (uint16_t)(d & 0xffffu);
                if (own1) o[(IDX)c * N + 1] = (uint16_t)(d >> 16);
            }
        }
    }
}

// Ring writes of a source pair at tile position (px, py), px even: population
// q goes to (px + c_x, py + c_y) and (px + 1 + c_x, py + c_y), where they are
// inside the tile.  The in-x pair is one aligned 8-byte store; a shifted pair
// is two 4-byte stores.  SEL: a store whose destination lies outside the tile
// goes to the trash words instead of being skipped (selects, no branches; the
// FP32 form, where it measured 2 % faster: the narrow forms spill with it).
template <int q, bool SEL, class E, class V>
__device__ __forceinline__ void put_pair(const Ring<E>& R, int px, int py, V v, E* trash) {
    constexpr int X = cx(q), Y = cy(q);
    const int dy = py + Y;
    if constexpr (SEL) {
        const bool row = Y == 0 || (dy >= 0 && dy < TY);
        E* p = R.template at<q>(dy * TX + px + X);
        if constexpr (X == 0) {
            st_pair(row ? p : trash, v);
        } else if constexpr (X > 0) {
            *(row ? p : trash) = v.x;
            *((row && px + 2 < TX) ? p + 1 : trash) = v.y;
        } else {
            *((row && px > 0) ? p : trash) = v.x;
            *(row ? p + 1 : trash) = v.y;
        }
    } else {
        if (dy < 0 || dy >= TY) return;
        E* p = R.template at<q>(dy * TX + px + X);
        if constexpr (X == 0) {
            st_pair(p, v);
        } else if constexpr (X > 0) {
            p[0] = v.x;
            if (px + 2 < TX) p[1] = v.y;
        } else {
            if (px > 0) p[0] = v.x;
            p[1] = v.y;
        }
    }
}
template <int q, class E>
__device__ __forceinline__ void put_one(const Ring<E>& R, int px, int py, E v) {
    const int dx = px + cx(q), dy = py + cy(q);
    if (dx < 0 || dx >= TX || dy < 0 || dy >= TY) return;
    *R.template at<q>(dy * TX + dx) = v;
}

// halo-row positions build the populations that cross a y edge of the tile;
// halo-column positions and corners those that cross an x edge (the
// destination test drops the ones that stay outside)
#define HOME_ROW_Q 3, 4, 7, 8, 9, 10, 15, 16, 17, 18
#define HOME_COL_Q 1, 2, 7, 8, 9, 10, 11, 12, 13, 14
template <int... Qs, class F>
__device__ __forceinline__ void for_qs(F&& fn) {
    (fn(QI<Qs>{}), ...);
}

// Roles of the threads of a block
enum : int { ROLE_TILE = 0, ROLE_ROW = 1, ROLE_COL = 2, ROLE_IDLE = 3 };

// SLAB: the planes [p.zb, p.ze) of a z-slab and salts offset by p.salt_base;
// otherwise every plane (a separate instantiation keeps the plain step's
// bounds compile-time)
template <class T, bool STATS, class IDX, bool SLAB>
__global__ void __launch_bounds__(NT, sizeof(T) == 8 ? 2 : 4) home_step(HomeParams p) {
    using E = typename HomeTypes<T>::E;
    using V = typename HomeTypes<T>::V;
    extern __shared__ __align__(16) unsigned char smraw[];
    E* sm = reinterpret_cast<E*>(smraw);
    const T* __restrict__ m = static_cast<const T*>(p.m);
    T* __restrict__ mn = static_cast<T*>(p.mn);
    const IDX N = (IDX)p.N;
    const int nx = p.nx, ny = p.ny, nz = p.nz;
    const E omw = E(1) - E(p.omega);    // 1 - omega (in FP64 for the FP64 form)
    const float r0 = p.rho0;

    const int tiles_x = (nx + TX - 1) / TX;
    const int tiles_y = (ny + TY - 1) / TY;
    int b = blockIdx.x;
    const int x0 = (b % tiles_x) * TX; b /= tiles_x;
    const int y0 = (b % tiles_y) * TY; b /= tiles_y;
    const int z0 = (SLAB ? p.zb : 0) + b * p.zchunk;
    const int z1 = min(SLAB ? p.ze : nz, z0 + p.zchunk);
    const uint32_t salt0 = SLAB ? p.salt_base : 0u;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    // this thread's role and tile position (px, py) of its first cell
    int role, px, py;
    if (warp < NCW) { role = ROLE_TILE; px = 2 * (lane & 15); py = 2 * warp + (lane >> 4); }
    else if (warp == NCW) { role = ROLE_ROW; px = 2 * (lane & 15); py = (lane >> 4) ? TY : -1; }
    else if (lane < 2 * TY) { role = ROLE_COL; px = lane < TY ? -1 : TX; py = lane & (TY - 1); }
    else if (lane < 2 * TY + 4) {
        const int k = lane - 2 * TY;
        role = ROLE_COL; px = (k & 1) ? TX : -1; py = (k & 2) ? TY : -1;
    } else { role = ROLE_IDLE; px = 0; py = 0; }
    const bool pair = role == ROLE_TILE || role == ROLE_ROW;
    // the cells it stands for: periodic in y, periodic or absent in x
    const int ly = y0 + py;
    const int gy = ((ly % ny) + ny) % ny;
    int gx0 = x0 + px, gx1 = gx0 + 1;
    bool e0 = role != ROLE_IDLE, e1 = pair;
    if (p.duct) {
        e0 = e0 && gx0 >= 0 && gx0 < nx;
        e1 = e1 && gx1 < nx;
    } else {
        gx0 = ((gx0 % nx) + nx) % nx;
        gx1 = gx1 % nx;
    }
    // cells that gather and store (tile cells inside the grid)
    const bool own0 = role == ROLE_TILE && ly < ny && x0 + px < nx;
    const bool own1 = role == ROLE_TILE && ly < ny && x0 + px + 1 < nx;
    const IDX plane = (IDX)nx * (IDX)ny;
    const IDX c0 = (IDX)gy * (IDX)nx + (IDX)gx0;
    const IDX c1 = (IDX)gy * (IDX)nx + (IDX)gx1;
    // one aligned vector access for both cells: with nx even every plane, row
    // and moment plane starts at an even cell index, and the pair starts at an even x
    const bool vec = pair && e0 && e1 && c1 == c0 + 1 && (nx & 1) == 0;

    V mreg[10];
#pragma unroll
    for (int c = 0; c < 10; ++c) mreg[c] = vsplat(0.f, V{});
    uint32_t freg = 0;                // flag bytes of the two cells (owners only)
    const uint8_t* __restrict__ flags = p.flags;
    auto load = [&](int z) {
        const int zz = z < 0 ? z + nz : (z >= nz ? z - nz : z);
        const IDX base = (IDX)zz * plane;
        if (vec) {
            const T* q = m + base + c0;
#pragma unroll
            for (int c = 0; c < 10; ++c) mreg[c] = MomStore<T>::ld2(q + (IDX)c * N);
        } else {
            if (e0) {
#pragma unroll
                for (int c = 0; c < 10; ++c) mreg[c].x = MomStore<T>::ld(m + base + c0 + (IDX)c * N);
            }
            if (e1) {
#pragma unroll
                for (int c = 0; c < 10; ++c) mreg[c].y = MomStore<T>::ld(m + base + c1 + (IDX)c * N);
            }
        }
        if (flags && (own0 || own1)) {
            if (vec) freg = *reinterpret_cast<const uint16_t*>(flags + base + c0);
            else freg = (own0 ? flags[base + c0] : 0u) | ((own1 ? flags[base + c1] : 0u) << 8);
        }
    };
    // the moments of plane pz are in mreg: write the populations leaving it
    constexpr bool kSel = std::is_same<T, float>::value;
    auto arrive = [&](int pz, int upslot) {
        if (role == ROLE_IDLE) return;
        const Ring<E> R(sm, pz, upslot);
        if (pair) {
            V mm[10];
#pragma unroll
            for (int c = 0; c < 10; ++c) mm[c] = mom_of<T>(mreg[c], c, r0);
            Coef<V> cf;
            cf.set(mm, omw, r0);
            if (role == ROLE_TILE) {
                static_for<0, 19>([&](auto qi) {
                    constexpr int q = decltype(qi)::value;
                    put_pair<q, kSel>(R, px, py, fpost<q>(cf), sm + TRASH_OFF);
                });
            } else {
                for_qs<HOME_ROW_Q>([&](auto qi) {
                    constexpr int q = decltype(qi)::value;
                    put_pair<q, kSel>(R, px, py, fpost<q>(cf), sm + TRASH_OFF);
                });
            }
        } else {
            E mm[10];
#pragma unroll
            for (int c = 0; c < 10; ++c) mm[c] = mom_of<T>(mreg[c].x, c, r0);
            Coef<E> cf;
            cf.set(mm, omw, r0);
            for_qs<HOME_COL_Q>([&](auto qi) {
                constexpr int q = decltype(qi)::value;
                put_one<q>(R, px, py, fpost<q>(cf));
            });
        }
    };
    auto mod3 = [](int v) { return v < 0 ? v + 3 : v % 3; };   // v >= -1
    int um = mod3(z0 - 1), u0 = mod3(z0), up = mod3(z0 + 1);  // UP slots of planes z-1, z, z+1

    double acc[NSTAT];
#pragma unroll
    for (int k = 0; k < NSTAT; ++k) acc[k] = 0.0;

    load(z0 - 1);
    arrive(z0 - 1, um);
    load(z0);
    arrive(z0, u0);
    uint32_t fcur = freg;          // flags of the cells in the plane being gathered
    load(z0 + 1);
    const int pos = py * TX + px;  // tile position of the first cell (owners)

    for (int z = z0; z < z1; ++z) {
        // 1. plane z+1 arrives (its moments were loaded one iteration ago); z+2 is requested
        arrive(z + 1, up);
        const uint32_t fnext = freg;
        if (z + 2 <= z1) load(z + 2);
        __syncthreads();
        // 2. gather and moments
        if (own0 || own1) {
            const IDX id = (IDX)z * plane + c0;
            const bool sol0 = own0 && (fcur & F_SOLID), sol1 = own1 && ((fcur >> 8) & F_SOLID);
            if (!((sol0 || !own0) && (sol1 || !own1))) {
                const Ring<E> Rm(sm, z - 1, um), Rz(sm, z, u0), Rp(sm, z + 1, up);
                // Links that do not stream: the gathering cell writes the replacement
                // into its own slot, which only it reads.  The (unused) value its
                // source wrote there came before the barrier above.
                const bool sp0 = own0 && (fcur & F_SPECIAL), sp1 = own1 && ((fcur >> 8) & F_SPECIAL);
                if (sp0 || sp1) {
                    const uint32_t lk0 = sp0 ? p.links[id] : 0u;
                    const uint32_t lk1 = sp1 ? p.links[id + 1] : 0u;
                    V om[10];
#pragma unroll
                    for (int c = 0; c < 10; ++c) {
                        om[c].x = sp0 ? mom_of<T>(MomStore<T>::ld(m + id + (IDX)c * N), c, r0) : E(0);
                        om[c].y = sp1 ? mom_of<T>(MomStore<T>::ld(m + id + 1 + (IDX)c * N), c, r0) : E(0);
                    }
                    Coef<V> oc;
                    oc.set(om, omw, r0);
                    const int gxa = x0 + px;
                    static_for<1, 19>([&](auto qi) {
                        constexpr int q = decltype(qi)::value;
                        const bool n0 = (lk0 >> opp(q)) & 1u, n1 = (lk1 >> opp(q)) & 1u;
                        if (n0 || n1) {
                            // own post-collision population of direction bq comes back as q
                            // (home.cu:219-225); bq = opp(q), or the reference's table
                            constexpr int bt = opp(q), br = opp_tab(q);
                            const V bb = p.ref_bounce ? fpost<br>(oc) : fpost<bt>(oc);
                            V v = bb;
                            if (cx(q) != 0 && p.duct) {
                                const V fo = fpost<q>(oc);                 // outlet
                                const int xa = gxa - cx(q), xb = gxa + 1 - cx(q);
                                if (xa < 0) v.x = inlet_shifted<q>(om[0].x, p.u_in, r0);   // inlet
                                else if (xa >= nx) v.x = fo.x;
                                if (xb < 0) v.y = inlet_shifted<q>(om[0].y, p.u_in, r0);
                                else if (xb >= nx) v.y = fo.y;
                            }
                            if (STATS) {
                                constexpr int bq0 = bt, bq1 = br;
                                const int ys = ((gy - cy(q)) % ny + ny) % ny;
                                const int zs = ((z - cz(q)) % nz + nz) % nz;
                                const IDX rowb = (IDX)zs * plane + (IDX)ys * (IDX)nx;
#pragma unroll
                                for (int h = 0; h < 2; ++h) {
                                    if (!(h ? n1 : n0)) continue;
                                    const int xs = gxa + h - cx(q);
                                    if (p.duct && (xs < 0 || xs >= nx)) continue;
                                    const int xw = ((xs % nx) + nx) % nx;
                                    if (flags[rowb + (IDX)xw] & F_OBST) {
                                        const int bq = p.ref_bounce ? bq1 : bq0;
                                        const double fv = (double)(h ? v.y : v.x) + (double)(wq(q) * r0);   // unshifted
                                        acc[2] += (double)(cx(bq) - cx(q)) * fv;
                                        acc[3] += (double)(cy(bq) - cy(q)) * fv;
                                        acc[4] += (double)(cz(bq) - cz(q)) * fv;
                                    }
                                }
                            }
                            const Ring<E>& R = cz(q) > 0 ? Rm : (cz(q) == 0 ? Rz : Rp);
                            E* sl = R.template at<q>(pos);
                            if (n0) sl[0] = v.x;
                            if (n1) sl[1] = v.y;
                        }
                    });
                }
                V fq[19];
                static_for<0, 19>([&](auto qi) {
                    constexpr int q = decltype(qi)::value;
                    const Ring<E>& R = cz(q) > 0 ? Rm : (cz(q) == 0 ? Rz : Rp);
                    fq[q] = ld_pair(R.template at<q>(pos));
                });
                // moments of the gathered (shifted) populations (home.cu:238-273):
                // dr = rho - rho0 = sum g, M = sum c c g = Pi - rho0/3 I; opposite pairs first
                const V s1 = vadd(fq[1], fq[2]), d1 = vsub(fq[1], fq[2]);
                const V s3 = vadd(fq[3], fq[4]), d3 = vsub(fq[3], fq[4]);
                const V s5 = vadd(fq[5], fq[6]), d5 = vsub(fq[5], fq[6]);
                const V s7 = vadd(fq[7], fq[10]), d7 = vsub(fq[7], fq[10]);     // (+1,+1,0)
                const V s9 = vadd(fq[9], fq[8]), d9 = vsub(fq[9], fq[8]);       // (+1,-1,0)
                const V s11 = vadd(fq[11], fq[14]), d11 = vsub(fq[11], fq[14]); // (+1,0,+1)
                const V s13 = vadd(fq[13], fq[12]), d13 = vsub(fq[13], fq[12]); // (+1,0,-1)
                const V s15 = vadd(fq[15], fq[18]), d15 = vsub(fq[15], fq[18]); // (0,+1,+1)
                const V s17 = vadd(fq[17], fq[16]), d17 = vsub(fq[17], fq[16]); // (0,+1,-1)
                const V dr = vadd(fq[0], vadd(vadd(vadd(s1, s3), vadd(s5, s7)),
                                              vadd(vadd(vadd(s9, s11), vadd(s13, s15)), s17)));
                const V jx = vadd(vadd(vadd(d1, d7), vadd(d9, d11)), d13);
                const V jy = vadd(vsub(vadd(d3, d7), d9), vadd(d15, d17));
                const V jz = vadd(vsub(vadd(d5, d11), d13), vsub(d15, d17));
                const V Mxx = vadd(vadd(vadd(s1, s7), vadd(s9, s11)), s13);
                const V Myy = vadd(vadd(vadd(s3, s7), vadd(s9, s15)), s17);
                const V Mzz = vadd(vadd(vadd(s5, s11), vadd(s13, s15)), s17);
                const V Mxy = vsub(s7, s9), Mxz = vsub(s11, s13), Myz = vsub(s15, s17);
                const V r = vadd(dr, vsplat(r0, V{}));
                const V inv = vrcp_pos(r);
                const V ux = vfma(jx, inv, vsplat(p.fx, V{}));
                const V uy = vfma(jy, inv, vsplat(p.fy, V{}));
                const V uz = vfma(jz, inv, vsplat(p.fz, V{}));
                const V r3 = mulk(dr, K3_HI, K3_LO);
                const V rx = vmul(r, ux), ry = vmul(r, uy), rz = vmul(r, uz);
                V out[10] = {r, ux, uy, uz,
                                  vsub(Mxx, vfma(rx, ux, r3)), vsub(Mxy, vmul(rx, uy)), vsub(Mxz, vmul(rx, uz)),
                                  vsub(Myy, vfma(ry, uy, r3)), vsub(Myz, vmul(ry, uz)), vsub(Mzz, vfma(rz, uz, r3))};
                if (sol0 || sol1) {   // a solid cell stores the rest state (home.cu:180-188)
#pragma unroll
                    for (int c = 0; c < 10; ++c) {
                        if (sol0) out[c].x = c == 0 ? E(1) : E(0);
                        if (sol1) out[c].y = c == 0 ? E(1) : E(0);
                    }
                }
                store_pair<T, IDX, V>(mn + id, N, r0, out, (uint32_t)id + salt0, vec && own0 && own1, own0, own1);
                if (STATS) {
                    if (own0 && !sol0) {
                        acc[0] += (double)r.x;
                        acc[1] += 0.5 * ((double)ux.x * ux.x + (double)uy.x * uy.x + (double)uz.x * uz.x);
                        acc[5] += (double)r.x * ux.x;
                        acc[6] += (double)r.x * uy.x;
                        acc[7] += (double)r.x * uz.x;
                    }
                    if (own1 && !sol1) {
                        acc[0] += (double)r.y;
                        acc[1] += 0.5 * ((double)ux.y * ux.y + (double)uy.y * uy.y + (double)uz.y * uz.y);
                        acc[5] += (double)r.y * ux.y;
                        acc[6] += (double)r.y * uy.y;
                        acc[7] += (double)r.y * uz.y;
                    }
                }
            } else {
                // every owned cell is solid: the rest state
                V out[10];
#pragma unroll
                for (int c = 0; c < 10; ++c) out[c] = vsplat(c == 0 ? 1.f : 0.f, V{});
                store_pair<T, IDX, V>(mn + id, N, r0, out, (uint32_t)id + salt0, vec && own0 && own1, own0, own1);
            }
        }
        fcur = fnext;
        {   // plane z+2 takes the slot of plane z-1
            const int t = um;
            um = u0;
            u0 = up;
            up = t;
        }
        __syncthreads();
    }
    if constexpr (STATS) block_reduce_stats(acc, p.partials);
}

template <class T>
__global__ void home_export(const T* __restrict__ m, int64_t N, float r0, float* __restrict__ out) {
    const int64_t tot = 10 * N;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = mom_of<T>(MomStore<T>::ld(m + i), (int)(i / N), r0);
}

template <class T>
__global__ void home_macros(const T* __restrict__ m, int64_t N, float r0, float* rho, float* ux, float* uy,
                            float* uz) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        rho[i] = mom_of<T>(MomStore<T>::ld(m + i), 0, r0);
        ux[i] = mom_of<T>(MomStore<T>::ld(m + N + i), 1, r0);
        uy[i] = mom_of<T>(MomStore<T>::ld(m + 2 * N + i), 2, r0);
        uz[i] = mom_of<T>(MomStore<T>::ld(m + 3 * N + i), 3, r0);
    }
}

template <class T, bool STATS>
void launch_step(const HomeParams& p, cudaStream_t s) {
    const int grid = home_num_blocks(p.nx, p.ny, p.ze - p.zb, p.zchunk);
    const size_t smem = sizeof(typename HomeTypes<T>::E) * SMEM_FLOATS;
    // 32-bit element offsets while every index 10*N fits in them
    const bool slab = p.zb != 0 || p.ze != p.nz || p.salt_base != 0;
    if ((uint64_t)p.N * 10u < (1ull << 32)) {
        if (slab) home_step<T, STATS, uint32_t, true><<<grid, NT, smem, s>>>(p);
        else home_step<T, STATS, uint32_t, false><<<grid, NT, smem, s>>>(p);
    } else {
        if (slab) home_step<T, STATS, int64_t, true><<<grid, NT, smem, s>>>(p);
        else home_step<T, STATS, int64_t, false><<<grid, NT, smem, s>>>(p);
    }
}

template <class T>
cudaError_t launch_home_t(const HomeParams& p, cudaStream_t s) {
    if (p.stats) launch_step<T, true>(p, s);
    else launch_step<T, false>(p, s);
    return cudaGetLastError();
}

}  // namespace

cudaError_t home_prepare() {
    cudaError_t e = cudaSuccess;
    auto set = [&](const void* fn, int esz = 4) {
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, esz * SMEM_FLOATS);
    };
    auto all = [&](auto slab) {
        constexpr bool S = decltype(slab)::value;
        set((const void*)home_step<float, false, uint32_t, S>);
        set((const void*)home_step<float, true, uint32_t, S>);
        set((const void*)home_step<__half, false, uint32_t, S>);
        set((const void*)home_step<__half, true, uint32_t, S>);
        set((const void*)home_step<__nv_bfloat16, false, uint32_t, S>);
        set((const void*)home_step<__nv_bfloat16, true, uint32_t, S>);
        set((const void*)home_step<float, false, int64_t, S>);
        set((const void*)home_step<float, true, int64_t, S>);
        set((const void*)home_step<__half, false, int64_t, S>);
        set((const void*)home_step<__half, true, int64_t, S>);
        set((const void*)home_step<__nv_bfloat16, false, int64_t, S>);
        set((const void*)home_step<__nv_bfloat16, true, int64_t, S>);
        set((const void*)home_step<double, false, uint32_t, S>, 8);
        set((const void*)home_step<double, true, uint32_t, S>, 8);
        set((const void*)home_step<double, false, int64_t, S>, 8);
        set((const void*)home_step<double, true, int64_t, S>, 8);
    };
    all(std::false_type{});
    all(std::true_type{});
    return e;
}

int home_num_blocks(int nx, int ny, int nz, int zchunk) {
    return ((nx + TX - 1) / TX) * ((ny + TY - 1) / TY) * ((nz + zchunk - 1) / zchunk);
}

int home_blocks_per_sm() {
    int n = 0;
    if (home_prepare() != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, home_step<float, false, uint32_t, false>, NT,
                                                      sizeof(float) * SMEM_FLOATS) != cudaSuccess || n < 1)
        return 1;
    return n;
}

cudaError_t launch_home_step(const HomeParams& p, int storage, int tile_y, int blocks_per_sm, cudaStream_t s) {
    (void)tile_y; (void)blocks_per_sm;
    switch (storage) {
        case 0: return launch_home_t<float>(p, s);
        case 1: return launch_home_t<__half>(p, s);
        case 2: return launch_home_t<__nv_bfloat16>(p, s);
        case 3: return launch_home_t<double>(p, s);
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_home_export(const void* m, int storage, int64_t N, float rho0, float* out, cudaStream_t s) {
    const int blocks = num_sms() * 8;
    switch (storage) {
        case 0: home_export<float><<<blocks, 256, 0, s>>>(static_cast<const float*>(m), N, rho0, out); break;
        case 1: home_export<__half><<<blocks, 256, 0, s>>>(static_cast<const __half*>(m), N, rho0, out); break;
        case 2: home_export<__nv_bfloat16><<<blocks, 256, 0, s>>>(static_cast<const __nv_bfloat16*>(m), N, rho0, out); break;
        case 3: home_export<double><<<blocks, 256, 0, s>>>(static_cast<const double*>(m), N, rho0, out); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_home_macros(const void* m, int storage, int64_t N, float rho0, float* rho, float* ux, float* uy,
                               float* uz, cudaStream_t s) {
    const int blocks = num_sms() * 8;
    switch (storage) {
        case 1: home_macros<__half><<<blocks, 256, 0, s>>>(static_cast<const __half*>(m), N, rho0, rho, ux, uy, uz); break;
        case 2: home_macros<__nv_bfloat16><<<blocks, 256, 0, s>>>(static_cast<const __nv_bfloat16*>(m), N, rho0, rho, ux, uy, uz); break;
        case 3: home_macros<double><<<blocks, 256, 0, s>>>(static_cast<const double*>(m), N, rho0, rho, ux, uy, uz); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace lbm
