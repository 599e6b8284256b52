// HOME moment-only step (src/lbm/lbm3d_home.cu:37-286): the state is 10
// moments per cell [rho, ux, uy, uz, Sxx, Sxy, Sxz, Syy, Syz, Szz]; every step
// rebuilds each neighbour's post-collision population from its moments,
// gathers the 19 incoming populations and stores their moments.
//
// The reference rebuilds f_q 19 times per cell from global loads of the
// neighbour's 10 moments (190 loads and ~1.1 kFLOP per cell).  Here a block
// owns a 32 x 8 tile of an (x,y) plane and marches along z over a chunk of
// planes, with one thread per tile cell (8 warps) and 3 warps for the halo:
//   * when the moments of a plane arrive (requested one plane ahead), every
//     position rebuilds its post-collision populations ONCE, from the identity
//         f*_q = w_q [rho + 3 c_q.(rho u) + 4.5 Q_q : (rho u u + (1-w) S)],
//     Q_q = c_q c_q - I/3 (src/lbm/lbm3d_home.cu:57-80 rearranged:
//     4.5 (c.u)^2 - 1.5 u^2 = 4.5 Q:uu), in opposite-pair form, into a shared
//     ring grouped by c_z: the up-going group lives 3 planes, the in-plane group
//     2 and the down-going group 1 (38 floats per position; halo positions write
//     only the 5, or 1, populations that point into the tile, with the same
//     expressions as a tile cell);
//   * the populations are shifted, g_q = f*_q - w_q rho0 (see Coef), and every
//     product with 1/3, 1/6 or 1/18 is rounded as if the constant were exact
//     (mulk), so FP32 rounding adds no drift of mass, momentum or stress;
//   * a link that does not stream (solid neighbour, duct inlet/outlet) is
//     handled by the gathering cell, which writes the replacement into the slot
//     of the source it would have gathered from (each slot has one reader);
//   * the gather is 19 shared-memory loads and pair sums;
//   * F16/BF16 moments are stored with stochastic rounding (cvt.rs).
// DRAM traffic is the 10 moments read once and written once (80 B per cell in
// FP32, 40 B in F16/BF16) plus the halo re-reads that L2 does not absorb.
#include <type_traits>

#include "lbm_common.cuh"
#include "lbm_internal.h"

namespace lbm {
namespace {

constexpr int TX = 32;
constexpr int TY = 8;
constexpr int HX = TX + 2;
constexpr int HY = TY + 2;
constexpr int HC = HX * HY;           // 340 halo-tile positions
constexpr int NWARP = TY + 3;         // 8 tile rows, 2 halo rows, 1 halo-column/corner warp
constexpr int NT = NWARP * 32;        // 352 threads

// shared ring, grouped by c_z: UP[3][5][HC], MID[2][9][HC], DN[5][HC]
constexpr int UP_SZ = 5 * HC, MID_SZ = 9 * HC, DN_SZ = 5 * HC;
constexpr int MID_OFF = 3 * UP_SZ, DN_OFF = MID_OFF + 2 * MID_SZ;
constexpr int SMEM_FLOATS = DN_OFF + DN_SZ;

// offset of q inside its group (UP: 5,11,12,15,16; MID: 0,1,2,3,4,7,8,9,10; DN: 6,13,14,17,18)
__host__ __device__ constexpr int gofs(int q) {
    constexpr int t[19] = {0, 1, 2, 3, 4, 0, 0, 5, 6, 7, 8, 1, 2, 1, 2, 3, 4, 3, 4};
    return t[q] * HC;
}

// the ring groups that hold the populations leaving plane p
struct Ring {
    float* up;
    float* mid;
    float* dn;
    __device__ __forceinline__ Ring(float* sm, int p) {
        up = sm + (p < 0 ? p + 3 : p % 3) * UP_SZ;   // p >= -1
        mid = sm + MID_OFF + (p & 1) * MID_SZ;
        dn = sm + DN_OFF;
    }
    // the same with the UP slot (p mod 3) given: the step loop rotates the
    // three slots instead of dividing by 3 for every ring
    __device__ __forceinline__ Ring(float* sm, int p, int upslot) {
        up = sm + upslot * UP_SZ;
        mid = sm + MID_OFF + (p & 1) * MID_SZ;
        dn = sm + DN_OFF;
    }
    template <int q>
    __device__ __forceinline__ float& at(int pos) const {
        return (cz(q) > 0 ? up : (cz(q) == 0 ? mid : dn))[gofs(q) + pos];
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
    __device__ __forceinline__ void set(const V (&m)[10], float omw_s, float r0) {
        const V omw = vsplat(omw_s, V{});
        const V r = m[0];
        const V jx = vmul(r, m[1]), jy = vmul(r, m[2]), jz = vmul(r, m[3]);
        const V Bxx = vfma(jx, m[1], vmul(omw, m[4]));
        const V Bxy = vfma(jx, m[2], vmul(omw, m[5]));
        const V Bxz = vfma(jx, m[3], vmul(omw, m[6]));
        const V Byy = vfma(jy, m[2], vmul(omw, m[7]));
        const V Byz = vfma(jy, m[3], vmul(omw, m[8]));
        const V Bzz = vfma(jz, m[3], vmul(omw, m[9]));
        constexpr float w1 = 1.0f / 18.0f;
        P = mulk(vfma(vsplat(-1.5f, V{}), vadd(vadd(Bxx, Byy), Bzz), vsub(r, vsplat(r0, V{}))), K18_HI, K18_LO);
        const V b45 = vsplat(4.5f * w1, V{}), b9 = vsplat(9.0f * w1, V{});   // 1/4 and 1/2, exact
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
template <class T> struct MomStore;
template <> struct MomStore<float> {
    __device__ __forceinline__ static float ld(const float* p, int k, float r0) { return __ldg(p); }
    __device__ __forceinline__ static float2 ld2(const float* p, int k, float r0) {
        return __ldg(reinterpret_cast<const float2*>(p));
    }
    __device__ __forceinline__ static void st(float* p, int k, float r0, float v, uint32_t) { *p = v; }
    __device__ __forceinline__ static void st2(float* p, int k, float r0, float2 v, uint32_t) {
        *reinterpret_cast<float2*>(p) = v;
    }
};
// F16: (rho - rho0, u, S) scaled by 2^10 (exact), as the F16 populations are
template <> struct MomStore<__half> {
    __device__ __forceinline__ static float ld(const __half* p, int k, float r0) {
        return __half2float(*p) * kF16Inv + (k == 0 ? r0 : 0.f);
    }
    __device__ __forceinline__ static float2 ld2(const __half* p, int k, float r0) {
        const float2 v = __half22float2(*reinterpret_cast<const __half2*>(p));
        const float s = k == 0 ? r0 : 0.f;
        return make_float2(v.x * kF16Inv + s, v.y * kF16Inv + s);
    }
    // stochastically rounded (see cvt_rs_f16x2); salt: a per-value index
    __device__ __forceinline__ static void st(__half* p, int k, float r0, float v, uint32_t salt) {
        const float a = (k == 0 ? v - r0 : v) * kF16Scale;
        const uint32_t d = cvt_rs_f16x2(a, 0.f, sr_bits(a, 0.f, salt));
        *reinterpret_cast<uint16_t*>(p) = (uint16_t)(d & 0xffffu);
    }
    __device__ __forceinline__ static void st2(__half* p, int k, float r0, float2 v, uint32_t salt) {
        const float s = k == 0 ? r0 : 0.f;
        const float a = (v.x - s) * kF16Scale, b = (v.y - s) * kF16Scale;
        *reinterpret_cast<uint32_t*>(p) = cvt_rs_f16x2(a, b, sr_bits(a, b, salt));
    }
};
template <> struct MomStore<__nv_bfloat16> {
    __device__ __forceinline__ static float ld(const __nv_bfloat16* p, int k, float r0) {
        return __bfloat162float(*p) + (k == 0 ? r0 : 0.f);
    }
    __device__ __forceinline__ static float2 ld2(const __nv_bfloat16* p, int k, float r0) {
        const float2 v = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(p));
        const float s = k == 0 ? r0 : 0.f;
        return make_float2(v.x + s, v.y + s);
    }
    __device__ __forceinline__ static void st(__nv_bfloat16* p, int k, float r0, float v, uint32_t salt) {
        const float a = k == 0 ? v - r0 : v;
        const uint32_t d = cvt_rs_bf16x2(a, 0.f, sr_bits(a, 0.f, salt));
        *reinterpret_cast<uint16_t*>(p) = (uint16_t)(d & 0xffffu);
    }
    __device__ __forceinline__ static void st2(__nv_bfloat16* p, int k, float r0, float2 v, uint32_t salt) {
        const float s = k == 0 ? r0 : 0.f;
        const float a = v.x - s, b = v.y - s;
        *reinterpret_cast<uint32_t*>(p) = cvt_rs_bf16x2(a, b, sr_bits(a, b, salt));
    }
};

// The 10 new moments of one cell.  FP32 stores them as they are; F16/BF16
// convert them two at a time with one stochastic-rounding conversion
// (cvt.rs.*x2) and split the pair into the two planes, drawing the five random
// words from one hash of the cell's index and first two values.
template <class T, class IDX>
__device__ __forceinline__ void store_moments(T* op, IDX N, float r0, const float (&out)[10], uint32_t salt) {
    if constexpr (sizeof(T) == 4) {
#pragma unroll
        for (int c = 0; c < 10; ++c) op[(IDX)c * N] = out[c];
    } else {
        constexpr bool F16 = std::is_same<T, __half>::value;
        const float sc = F16 ? kF16Scale : 1.0f;
        const uint32_t h = mix32(salt ^ __float_as_uint(out[0]) ^ (__float_as_uint(out[1]) * 0x9e3779b9u));
        uint16_t* o = reinterpret_cast<uint16_t*>(op);
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            uint32_t rb = h * (2u * k + 1u) * 0x85ebca6bu;
            rb ^= rb >> 15;
            const float a = (k == 0 ? out[0] - r0 : out[2 * k]) * sc, b = out[2 * k + 1] * sc;
            const uint32_t d = F16 ? cvt_rs_f16x2(a, b, rb) : cvt_rs_bf16x2(a, b, rb);
            o[(IDX)(2 * k) * N] = (uint16_t)(d & 0xffffu);
            o[(IDX)(2 * k + 1) * N] = (uint16_t)(d >> 16);
        }
    }
}

// A tile cell writes all 19 populations leaving its plane; a halo position
// writes only the directions that point into the tile: dir 0 = x-1 column
// (+x), 1 = x+TX column (-x), 2 = y-1 row (+y), 3 = y+TY row (-y), 4..7 =
// corners feeding 7, 8, 9, 10.  The same expression (fpost) for every role.
__device__ __forceinline__ void build(const Ring& R, int pos, int dir, const Coef<float>& c) {
    auto put = [&](auto qi) {
        constexpr int q = decltype(qi)::value;
        R.template at<q>(pos) = fpost<q>(c);
    };
    switch (dir) {
        case -1: static_for<0, 19>(put); break;
        case 0: put(QI<1>{}); put(QI<7>{}); put(QI<9>{}); put(QI<11>{}); put(QI<13>{}); break;
        case 1: put(QI<2>{}); put(QI<8>{}); put(QI<10>{}); put(QI<12>{}); put(QI<14>{}); break;
        case 2: put(QI<3>{}); put(QI<7>{}); put(QI<8>{}); put(QI<15>{}); put(QI<17>{}); break;
        case 3: put(QI<4>{}); put(QI<9>{}); put(QI<10>{}); put(QI<16>{}); put(QI<18>{}); break;
        case 4: put(QI<7>{}); break;
        case 5: put(QI<8>{}); break;
        case 6: put(QI<9>{}); break;
        case 7: put(QI<10>{}); break;
        default: break;
    }
}

// SLAB: the planes [p.zb, p.ze) of a z-slab and salts offset by p.salt_base;
// otherwise every plane (a separate instantiation: the plain step is at its
// register limit, and the two run-time bounds alone cost it spills)
template <class T, bool STATS, class IDX, bool SLAB>
__global__ void __launch_bounds__(NT, 3) home_step(HomeParams p) {
    extern __shared__ float sm[];
    const T* __restrict__ m = static_cast<const T*>(p.m);
    T* __restrict__ mn = static_cast<T*>(p.mn);
    const IDX N = (IDX)p.N;
    const int nx = p.nx, ny = p.ny, nz = p.nz;
    const float omw = 1.f - p.omega;
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

    // this thread's position in the (TX+2) x (TY+2) halo tile, and its role
    int hx, hy, dir;   // dir: -1 tile cell, 0..7 halo (see build_halo), -2 idle
    if (warp < TY) { hx = lane + 1; hy = warp + 1; dir = -1; }
    else if (warp == TY) { hx = lane + 1; hy = 0; dir = 2; }
    else if (warp == TY + 1) { hx = lane + 1; hy = TY + 1; dir = 3; }
    else if (lane < TY) { hx = 0; hy = lane + 1; dir = 0; }
    else if (lane < 2 * TY) { hx = TX + 1; hy = lane - TY + 1; dir = 1; }
    else if (lane < 2 * TY + 4) {
        const int k = lane - 2 * TY;
        hx = (k & 1) ? TX + 1 : 0; hy = (k & 2) ? TY + 1 : 0; dir = 4 + k;
    } else { hx = 0; hy = 0; dir = -2; }
    const int pos = hy * HX + hx;
    // the cell it stands for (periodic in y, periodic or absent in x)
    const int lx = x0 - 1 + hx, ly = y0 - 1 + hy;
    int gx = lx;
    const int gy = ((ly % ny) + ny) % ny;
    bool exists = dir != -2;
    if (p.duct) exists = exists && lx >= 0 && lx < nx;
    else gx = ((lx % nx) + nx) % nx;
    const bool owner = dir == -1 && lx < nx && ly < ny;   // gathers and stores a cell
    const IDX plane = (IDX)nx * (IDX)ny;
    const IDX coff = (IDX)gy * (IDX)nx + (IDX)gx;

    const uint8_t* __restrict__ flags = p.flags;
    float mreg[10];
#pragma unroll
    for (int c = 0; c < 10; ++c) mreg[c] = 0.f;
    uint32_t freg = 0;
    auto load = [&](int z) {
        if (!exists) return;
        const int zz = z < 0 ? z + nz : (z >= nz ? z - nz : z);
        const IDX id = (IDX)zz * plane + coff;
#pragma unroll
        for (int c = 0; c < 10; ++c) mreg[c] = MomStore<T>::ld(m + (IDX)c * N + id, c, r0);
        freg = flags ? flags[id] : 0u;
    };
    // the moments of plane pz are in mreg/freg: write the populations leaving it
    // (a solid cell writes none; its slots are filled by its fluid neighbours)
    auto arrive = [&](int pz, int upslot) {
        if (exists && !(freg & F_SOLID)) {
            Coef<float> c;
            c.set(mreg, omw, r0);
            build(Ring(sm, pz, upslot), pos, dir, c);
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
    uint32_t fcur = freg;          // this position's flags in the plane being gathered
    load(z0 + 1);

    for (int z = z0; z < z1; ++z) {
        // 1. plane z+1 arrives (its moments were loaded one iteration ago); z+2 is requested
        arrive(z + 1, up);
        const uint32_t fnext = freg;
        if (z + 2 <= z1) load(z + 2);
        // 2. a link that does not stream: the cell writes the replacement into the
        //    slot of the source it would have gathered from (read by nobody else)
        if (owner && (fcur & F_SPECIAL)) {
            const IDX id = (IDX)z * plane + coff;
            const uint32_t lk = p.links[id];
            float own[10];
#pragma unroll
            for (int c = 0; c < 10; ++c) own[c] = MomStore<T>::ld(m + (IDX)c * N + id, c, r0);
            Coef<float> oc;
            oc.set(own, omw, r0);
            const Ring Rm(sm, z - 1, um), Rz(sm, z, u0), Rp(sm, z + 1, up);
            static_for<1, 19>([&](auto qi) {
                constexpr int q = decltype(qi)::value;
                if ((lk >> opp(q)) & 1u) {
                    const int xs = gx - cx(q);
                    float v;
                    if (p.duct && xs < 0) {
                        v = feq_ref(q, own[0], p.u_in, 0.f, 0.f) - wq(q) * r0;         // inlet
                    } else if (p.duct && xs >= nx) {
                        v = fpost<q>(oc);                                                 // outlet
                    } else {
                        // own post-collision population of direction bq comes back as q
                        // (home.cu:219-225); bq = opp(q), or the reference's table
                        constexpr int bt = opp(q), br = opp_tab(q);
                        v = p.ref_bounce ? fpost<br>(oc) : fpost<bt>(oc);
                        if (STATS) {
                            const int bq = p.ref_bounce ? br : bt;
                            const int ys = ((gy - cy(q)) % ny + ny) % ny;
                            const int zs = ((z - cz(q)) % nz + nz) % nz;
                            const int xw = ((xs % nx) + nx) % nx;
                            if (flags[(IDX)zs * plane + (IDX)ys * (IDX)nx + (IDX)xw] & F_OBST) {
                                const double fv = (double)v + (double)(wq(q) * r0);   // unshifted
                                acc[2] += (double)(cx(bq) - cx(q)) * fv;
                                acc[3] += (double)(cy(bq) - cy(q)) * fv;
                                acc[4] += (double)(cz(bq) - cz(q)) * fv;
                            }
                        }
                    }
                    // the source of q sits in plane z - c_z(q)
                    const Ring& R = cz(q) > 0 ? Rm : (cz(q) == 0 ? Rz : Rp);
                    R.template at<q>(pos - cx(q) - HX * cy(q)) = v;
                }
            });
        }
        __syncthreads();
        // 3. gather and moments
        if (owner) {
            const IDX id = (IDX)z * plane + coff;
            T* op = mn + id;
            if (fcur & F_SOLID) {
#pragma unroll
                for (int c = 0; c < 10; ++c)
                    MomStore<T>::st(op + (IDX)c * N, c, r0, c == 0 ? 1.f : 0.f,
                                    ((uint32_t)id + salt0) * 10u + c);
            } else {
                const Ring Rm(sm, z - 1, um), Rz(sm, z, u0), Rp(sm, z + 1, up);
                float fq[19];
                static_for<0, 19>([&](auto qi) {
                    constexpr int q = decltype(qi)::value;
                    const Ring& R = cz(q) > 0 ? Rm : (cz(q) == 0 ? Rz : Rp);
                    fq[q] = R.template at<q>(pos - cx(q) - HX * cy(q));
                });
                // moments of the gathered (shifted) populations (home.cu:238-273):
                // dr = rho - rho0 = sum g, M = sum c c g = Pi - rho0/3 I; opposite pairs first
                const float s1 = fq[1] + fq[2], d1 = fq[1] - fq[2];
                const float s3 = fq[3] + fq[4], d3 = fq[3] - fq[4];
                const float s5 = fq[5] + fq[6], d5 = fq[5] - fq[6];
                const float s7 = fq[7] + fq[10], d7 = fq[7] - fq[10];     // (+1,+1,0)
                const float s9 = fq[9] + fq[8], d9 = fq[9] - fq[8];       // (+1,-1,0)
                const float s11 = fq[11] + fq[14], d11 = fq[11] - fq[14]; // (+1,0,+1)
                const float s13 = fq[13] + fq[12], d13 = fq[13] - fq[12]; // (+1,0,-1)
                const float s15 = fq[15] + fq[18], d15 = fq[15] - fq[18]; // (0,+1,+1)
                const float s17 = fq[17] + fq[16], d17 = fq[17] - fq[16]; // (0,+1,-1)
                const float dr = fq[0] + ((s1 + s3) + (s5 + s7)) + ((s9 + s11) + (s13 + s15) + s17);
                const float jx = (d1 + d7) + (d9 + d11) + d13;
                const float jy = (d3 + d7) - d9 + (d15 + d17);
                const float jz = (d5 + d11) - d13 + (d15 - d17);
                const float Mxx = (s1 + s7) + (s9 + s11) + s13;
                const float Myy = (s3 + s7) + (s9 + s15) + s17;
                const float Mzz = (s5 + s11) + (s13 + s15) + s17;
                const float Mxy = s7 - s9, Mxz = s11 - s13, Myz = s15 - s17;
                const float r = dr + r0;
                const float inv = r > 0.f ? 1.0f / r : 0.f;
                const float ux = fmaf(jx, inv, p.fx), uy = fmaf(jy, inv, p.fy), uz = fmaf(jz, inv, p.fz);
                const float r3 = mulk(dr, K3_HI, K3_LO);
                const float rx = r * ux, ry = r * uy, rz = r * uz;
                const float out[10] = {r, ux, uy, uz,
                                       Mxx - fmaf(rx, ux, r3), Mxy - rx * uy, Mxz - rx * uz,
                                       Myy - fmaf(ry, uy, r3), Myz - ry * uz, Mzz - fmaf(rz, uz, r3)};
#pragma unroll
                store_moments<T, IDX>(op, N, r0, out, (uint32_t)id + salt0);
                if (STATS) {
                    acc[0] += (double)r;
                    acc[1] += 0.5 * ((double)ux * ux + (double)uy * uy + (double)uz * uz);
                    acc[5] += (double)r * ux;
                    acc[6] += (double)r * uy;
                    acc[7] += (double)r * uz;
                }
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
        out[i] = MomStore<T>::ld(m + i, (int)(i / N), r0);
}

template <class T>
__global__ void home_macros(const T* __restrict__ m, int64_t N, float r0, float* rho, float* ux, float* uy,
                            float* uz) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        rho[i] = MomStore<T>::ld(m + i, 0, r0);
        ux[i] = MomStore<T>::ld(m + N + i, 1, r0);
        uy[i] = MomStore<T>::ld(m + 2 * N + i, 2, r0);
        uz[i] = MomStore<T>::ld(m + 3 * N + i, 3, r0);
    }
}

template <class T, bool STATS>
void launch_step(const HomeParams& p, cudaStream_t s) {
    const int grid = home_num_blocks(p.nx, p.ny, p.ze - p.zb, p.zchunk);
    const size_t smem = sizeof(float) * SMEM_FLOATS;
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
    const int smem = (int)(sizeof(float) * SMEM_FLOATS);
    cudaError_t e = cudaSuccess;
    auto set = [&](const void* fn) {
        if (e == cudaSuccess) e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
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
    };
    all(std::false_type{});
    all(std::true_type{});
    return e;
}

int home_num_blocks(int nx, int ny, int nz, int zchunk) {
    return ((nx + TX - 1) / TX) * ((ny + TY - 1) / TY) * ((nz + zchunk - 1) / zchunk);
}

cudaError_t launch_home_step(const HomeParams& p, int storage, int tile_y, int blocks_per_sm, cudaStream_t s) {
    (void)tile_y; (void)blocks_per_sm;
    switch (storage) {
        case 0: return launch_home_t<float>(p, s);
        case 1: return launch_home_t<__half>(p, s);
        case 2: return launch_home_t<__nv_bfloat16>(p, s);
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_home_export(const void* m, int storage, int64_t N, float rho0, float* out, cudaStream_t s) {
    const int blocks = num_sms() * 8;
    switch (storage) {
        case 0: home_export<float><<<blocks, 256, 0, s>>>(static_cast<const float*>(m), N, rho0, out); break;
        case 1: home_export<__half><<<blocks, 256, 0, s>>>(static_cast<const __half*>(m), N, rho0, out); break;
        case 2: home_export<__nv_bfloat16><<<blocks, 256, 0, s>>>(static_cast<const __nv_bfloat16*>(m), N, rho0, out); break;
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
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace lbm
