// Shared device definitions for the D3Q19 kernels (sm_100a).
//
// Velocity set and weights keep the reference's order so that the population
// layout f[q*N + id] and the HOME moment layout m[k*N + id] stay the same as
// the reference's buffers (src/lbm/lbm3d_legacy.cu:16-35,
// src/lbm/lbm3d_home.hpp:57-71).
#pragma once

#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include "lbm_internal.h"

namespace lbm {

// 0:(0,0,0) 1:(+1,0,0) 2:(-1,0,0) 3:(0,+1,0) 4:(0,-1,0) 5:(0,0,+1) 6:(0,0,-1)
// 7:(+1,+1,0) 8:(-1,+1,0) 9:(+1,-1,0) 10:(-1,-1,0) 11:(+1,0,+1) 12:(-1,0,+1)
// 13:(+1,0,-1) 14:(-1,0,-1) 15:(0,+1,+1) 16:(0,-1,+1) 17:(0,+1,-1) 18:(0,-1,-1)
__host__ __device__ constexpr int cx(int q) {
    constexpr int t[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
    return t[q];
}
__host__ __device__ constexpr int cy(int q) {
    constexpr int t[19] = {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1};
    return t[q];
}
__host__ __device__ constexpr int cz(int q) {
    constexpr int t[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1};
    return t[q];
}
// the opposite direction, c_opp(q) = -c_q
__host__ __device__ constexpr int opp(int q) {
    constexpr int t[19] = {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15};
    return t[q];
}
// The reference's opp() table (src/lbm/lbm3d_legacy.cu:29-32): the true
// opposite for the axis directions, the mirror image in x (xy/xz diagonals)
// or y (yz diagonals) for the others.  Used only by LBM_BOUNCE_REFERENCE.
__host__ __device__ constexpr int opp_tab(int q) {
    constexpr int t[19] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17};
    return t[q];
}
// weights as the reference writes them: 1.0f/3.0f, 1.0f/18.0f, 1.0f/36.0f
__host__ __device__ constexpr float wq(int q) {
    return q == 0 ? 1.0f / 3.0f : (q <= 6 ? 1.0f / 18.0f : 1.0f / 36.0f);
}

// Products with the lattice constants 1/3, 1/6, 1/18 and 1/36, rounded as if
// the constant were exact: c x = fma(c_hi, x, c_lo x) with c_hi = float(c) and
// c_lo = float(c - c_hi).  A plain product with float(c) carries the constant's
// own rounding error into every step as a bias (float(1/6) is 3e-8 too large,
// so momentum rebuilt with it grows by 3e-8 per step, 3e-5 after 1000 steps);
// with the split the rounding is that of one correctly rounded product.
constexpr float K3_HI = 0x1.555556p-2f, K3_LO = -0x1.555556p-27f;     // 1/3
constexpr float K6_HI = 0x1.555556p-3f, K6_LO = -0x1.555556p-28f;     // 1/6
constexpr float K18_HI = 0x1.c71c72p-5f, K18_LO = -0x1.c71c72p-32f;   // 1/18
constexpr float K36_HI = 0x1.c71c72p-6f, K36_LO = -0x1.c71c72p-33f;   // 1/36
__device__ __forceinline__ float mulk(float x, float hi, float lo) { return __fmaf_rn(hi, x, __fmul_rn(lo, x)); }
// FP64: the constant itself to 48 bits (hi + lo), one product
__device__ __forceinline__ double mulk(double x, float hi, float lo) { return x * ((double)hi + (double)lo); }
__device__ __forceinline__ float2 mulk(float2 x, float hi, float lo) {
    return __ffma2_rn(make_float2(hi, hi), x, __fmul2_rn(make_float2(lo, lo), x));
}

// ---- stochastic rounding to F16/BF16 pairs (sm_100a cvt.rs) ---------------
// The narrow stores of a smooth field round neighbouring cells the same way,
// so round-to-nearest errors add up coherently over the steps; rounding up or
// down at random, with probability given by the distance to each neighbour,
// makes every store unbiased and the errors independent.  The random bits are a
// hash of the stored values and of a per-value salt (no state, so the step is
// still a pure function of its input and can be replayed in a graph).
__device__ __forceinline__ uint32_t mix32(uint32_t x) {
    x ^= x >> 16; x *= 0x7feb352du; x ^= x >> 15; x *= 0x846ca68bu; x ^= x >> 16;
    return x;
}
__device__ __forceinline__ uint32_t sr_bits(float a, float b, uint32_t salt) {
    return mix32(salt ^ __float_as_uint(a) ^ (__float_as_uint(b) * 0x9e3779b9u));
}
// {lo, hi} -> packed f16x2 (lo in the low half), stochastically rounded
__device__ __forceinline__ uint32_t cvt_rs_f16x2(float lo, float hi, uint32_t rb) {
    uint32_t d;
    asm("cvt.rs.satfinite.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(hi), "f"(lo), "r"(rb));
    return d;
}
__device__ __forceinline__ uint32_t cvt_rs_bf16x2(float lo, float hi, uint32_t rb) {
    uint32_t d;
    asm("cvt.rs.satfinite.bf16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(hi), "f"(lo), "r"(rb));
    return d;
}

// flag byte per cell, built on the device from the solid mask
enum : uint8_t {
    F_SOLID = 1,     // solid cell (frozen populations, macros 1,0,0,0)
    F_BAND = 2,      // Hybrid: BGK-form collision
    F_OBST = 4,      // solid cell that counts for the drag (not a wall)
    F_SPECIAL = 8,   // fluid cell with at least one non-streaming link
    F_TOUCH = 16,    // fluid cell with a link into an obstacle cell
};

// The Legacy equilibrium, written as src/lbm/lbm3d_legacy.cu:54-58 writes it
// (the same expression keeps nvcc's contraction pattern, hence the results, close).
__device__ __forceinline__ float feq_ref(int q, float rho, float ux, float uy, float uz) {
    const float eiu = (float)cx(q) * ux + (float)cy(q) * uy + (float)cz(q) * uz;
    const float uu = ux * ux + uy * uy + uz * uz;
    return wq(q) * rho * (1.0f + 3.0f * eiu + 4.5f * eiu * eiu - 1.5f * uu);
}

// ---- storage traits --------------------------------------------------------
// F32 stores f as is.  F16/BF16 store the shifted value f - w_q*rho0 (all
// arithmetic stays FP32); the shift keeps the small deviations from the rest
// state in the narrow mantissa instead of the large constant part.
struct StoreF32 {
    using T = float;
    static constexpr int kId = 0;
    __device__ __forceinline__ static float ld(const T* p, int q, float r0) { return __ldg(p); }
    // Every population store is streaming (.cs, evict first): nothing reads a
    // stored slot again in the same launch, and the step's state is larger than
    // L2, so the lines L2 keeps are those still to be gathered (the odd step's
    // x-shifted rows are read by two warps).  Measured on B200: the duct's odd
    // step 138.8 -> 134.7 us, the 512^3 F16 even step 1.81 -> 1.71 ms.
    __device__ __forceinline__ static void st(T* p, int q, float r0, float v) { __stcs(p, v); }
    __device__ __forceinline__ static void ld4(const T* p, int q, float r0, float* o) {
        const float4 v = *reinterpret_cast<const float4*>(p);
        o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
    }
    __device__ __forceinline__ static void st4(T* p, int q, float r0, const float* v) {
        __stcs(reinterpret_cast<float4*>(p), make_float4(v[0], v[1], v[2], v[3]));
    }
    __device__ __forceinline__ static void ld2(const T* p, int q, float r0, float* o) {
        const float2 v = *reinterpret_cast<const float2*>(p);
        o[0] = v.x; o[1] = v.y;
    }
    __device__ __forceinline__ static void st2(T* p, int q, float r0, const float* v) {
        __stcs(reinterpret_cast<float2*>(p), make_float2(v[0], v[1]));
    }
};

// FP64 storage and arithmetic: the reference runs the narrower forms are
// measured against.  Plain values, no shift.
struct StoreF64 {
    using T = double;
    static constexpr int kId = 3;
    __device__ __forceinline__ static double ld(const T* p, int q, float r0) { return __ldg(p); }
    __device__ __forceinline__ static void st(T* p, int q, float r0, double v) { __stcs(p, v); }
    __device__ __forceinline__ static void ld2(const T* p, int q, float r0, double* o) {
        const double2 v = *reinterpret_cast<const double2*>(p);
        o[0] = v.x; o[1] = v.y;
    }
    __device__ __forceinline__ static void st2(T* p, int q, float r0, const double* v) {
        __stcs(reinterpret_cast<double2*>(p), make_double2(v[0], v[1]));
    }
    __device__ __forceinline__ static void ld4(const T* p, int q, float r0, double* o) {
        ld2(p, q, r0, o); ld2(p + 2, q, r0, o + 2);
    }
    __device__ __forceinline__ static void st4(T* p, int q, float r0, const double* v) {
        st2(p, q, r0, v); st2(p + 2, q, r0, v + 2);
    }
};

// arithmetic type of a storage form: FP32 for every form but FP64
template <class ST> struct Real { using type = float; };
template <> struct Real<StoreF64> { using type = double; };
// the shifted narrow forms (F16, BF16), which compute in stored units
template <class ST> constexpr bool kNarrow = ST::kId == 1 || ST::kId == 2;

// F16 keeps the shifted value scaled by 2^10 (exact in FP32): |f - w rho0| < 64
// fits, and deviations down to 6e-8 stay normal numbers instead of subnormals.
constexpr float kF16Scale = 1024.0f;
constexpr float kF16Inv = 1.0f / 1024.0f;

struct StoreF16 {
    using T = __half;
    static constexpr int kId = 1;
    __device__ __forceinline__ static float ld(const T* p, int q, float r0) {
        return __half2float(*p) * kF16Inv + wq(q) * r0;
    }
    __device__ __forceinline__ static void st(T* p, int q, float r0, float v) {
        __stcs(reinterpret_cast<unsigned short*>(p), __half_as_ushort(__float2half_rn((v - wq(q) * r0) * kF16Scale)));
    }
    __device__ __forceinline__ static void ld4(const T* p, int q, float r0, float* o) {
        const uint2 raw = *reinterpret_cast<const uint2*>(p);
        const __half2 a = *reinterpret_cast<const __half2*>(&raw.x);
        const __half2 b = *reinterpret_cast<const __half2*>(&raw.y);
        const float s = wq(q) * r0;
        const float2 fa = __half22float2(a), fb = __half22float2(b);
        o[0] = fa.x * kF16Inv + s; o[1] = fa.y * kF16Inv + s; o[2] = fb.x * kF16Inv + s; o[3] = fb.y * kF16Inv + s;
    }
    __device__ __forceinline__ static void st4(T* p, int q, float r0, const float* v) {
        const float s = wq(q) * r0;
        __half2 a = __floats2half2_rn((v[0] - s) * kF16Scale, (v[1] - s) * kF16Scale);
        __half2 b = __floats2half2_rn((v[2] - s) * kF16Scale, (v[3] - s) * kF16Scale);
        uint2 raw;
        raw.x = *reinterpret_cast<uint32_t*>(&a);
        raw.y = *reinterpret_cast<uint32_t*>(&b);
        __stcs(reinterpret_cast<uint2*>(p), raw);
    }
    __device__ __forceinline__ static void ld2(const T* p, int q, float r0, float* o) {
        const float2 f = __half22float2(*reinterpret_cast<const __half2*>(p));
        const float s = wq(q) * r0;
        o[0] = f.x * kF16Inv + s; o[1] = f.y * kF16Inv + s;
    }
    __device__ __forceinline__ static void st2(T* p, int q, float r0, const float* v) {
        const float s = wq(q) * r0;
        *reinterpret_cast<__half2*>(p) = __floats2half2_rn((v[0] - s) * kF16Scale, (v[1] - s) * kF16Scale);
    }
};

struct StoreBF16 {
    using T = __nv_bfloat16;
    static constexpr int kId = 2;
    __device__ __forceinline__ static float ld(const T* p, int q, float r0) {
        return __bfloat162float(*p) + wq(q) * r0;
    }
    __device__ __forceinline__ static void st(T* p, int q, float r0, float v) {
        __stcs(reinterpret_cast<unsigned short*>(p), __bfloat16_as_ushort(__float2bfloat16_rn(v - wq(q) * r0)));
    }
    __device__ __forceinline__ static void ld4(const T* p, int q, float r0, float* o) {
        const uint2 raw = *reinterpret_cast<const uint2*>(p);
        const __nv_bfloat162 a = *reinterpret_cast<const __nv_bfloat162*>(&raw.x);
        const __nv_bfloat162 b = *reinterpret_cast<const __nv_bfloat162*>(&raw.y);
        const float s = wq(q) * r0;
        const float2 fa = __bfloat1622float2(a), fb = __bfloat1622float2(b);
        o[0] = fa.x + s; o[1] = fa.y + s; o[2] = fb.x + s; o[3] = fb.y + s;
    }
    __device__ __forceinline__ static void st4(T* p, int q, float r0, const float* v) {
        const float s = wq(q) * r0;
        __nv_bfloat162 a = __floats2bfloat162_rn(v[0] - s, v[1] - s);
        __nv_bfloat162 b = __floats2bfloat162_rn(v[2] - s, v[3] - s);
        uint2 raw;
        raw.x = *reinterpret_cast<uint32_t*>(&a);
        raw.y = *reinterpret_cast<uint32_t*>(&b);
        __stcs(reinterpret_cast<uint2*>(p), raw);
    }
    __device__ __forceinline__ static void ld2(const T* p, int q, float r0, float* o) {
        const float2 f = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(p));
        const float s = wq(q) * r0;
        o[0] = f.x + s; o[1] = f.y + s;
    }
    __device__ __forceinline__ static void st2(T* p, int q, float r0, const float* v) {
        const float s = wq(q) * r0;
        *reinterpret_cast<__nv_bfloat162*>(p) = __floats2bfloat162_rn(v[0] - s, v[1] - s);
    }
};

// vector load/store of VEC consecutive cells of one population plane
// The narrow forms in their stored units, g = (f - w_q rho0) * S (S = 2^10 for
// F16, 1 for BF16), for steps that compute in those units: no conversion back
// to f on load and none on store, and no cancellation against w_q rho0.
template <class ST> struct Raw;
template <> struct Raw<StoreF32> {   // FP32 stores f itself (S = 1, no shift)
    using T = float;
    static constexpr float S = 1.0f, invS = 1.0f;
    __device__ __forceinline__ static float ld(const T* p) { return __ldg(p); }
    __device__ __forceinline__ static void st(T* p, float g) { __stcs(p, g); }
};
template <> struct Raw<StoreF16> {
    using T = __half;
    static constexpr float S = kF16Scale, invS = kF16Inv;
    __device__ __forceinline__ static float ld(const T* p) { return __half2float(*p); }
    __device__ __forceinline__ static void st(T* p, float g) {
        __stcs(reinterpret_cast<unsigned short*>(p), __half_as_ushort(__float2half_rn(g)));
    }
    __device__ __forceinline__ static void ld4(const T* p, float* o) {
        const uint2 raw = *reinterpret_cast<const uint2*>(p);
        const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&raw.x));
        const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&raw.y));
        o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
    }
    __device__ __forceinline__ static void st4(T* p, const float* v) {
        __half2 a = __floats2half2_rn(v[0], v[1]), b = __floats2half2_rn(v[2], v[3]);
        uint2 raw;
        raw.x = *reinterpret_cast<uint32_t*>(&a);
        raw.y = *reinterpret_cast<uint32_t*>(&b);
        __stcs(reinterpret_cast<uint2*>(p), raw);
    }
    __device__ __forceinline__ static void ld2(const T* p, float* o) {
        const float2 a = __half22float2(*reinterpret_cast<const __half2*>(p));
        o[0] = a.x; o[1] = a.y;
    }
    __device__ __forceinline__ static void st2(T* p, const float* v) {
        *reinterpret_cast<__half2*>(p) = __floats2half2_rn(v[0], v[1]);
    }
    // stochastically rounded stores (rb: random bits, see cvt_rs_f16x2)
    __device__ __forceinline__ static void st_sr(T* p, float g, uint32_t rb) {
        __stcs(reinterpret_cast<unsigned short*>(p), (unsigned short)(cvt_rs_f16x2(g, 0.f, rb) & 0xffffu));
    }
    __device__ __forceinline__ static void st2_sr(T* p, const float* v, uint32_t rb) {
        __stcs(reinterpret_cast<unsigned int*>(p), cvt_rs_f16x2(v[0], v[1], rb));
    }
    __device__ __forceinline__ static void st4_sr(T* p, const float* v, uint32_t rb0, uint32_t rb1) {
        __stcs(reinterpret_cast<uint2*>(p), make_uint2(cvt_rs_f16x2(v[0], v[1], rb0), cvt_rs_f16x2(v[2], v[3], rb1)));
    }
};
template <> struct Raw<StoreBF16> {
    using T = __nv_bfloat16;
    static constexpr float S = 1.0f, invS = 1.0f;
    __device__ __forceinline__ static float ld(const T* p) { return __bfloat162float(*p); }
    __device__ __forceinline__ static void st(T* p, float g) {
        __stcs(reinterpret_cast<unsigned short*>(p), __bfloat16_as_ushort(__float2bfloat16_rn(g)));
    }
    __device__ __forceinline__ static void ld4(const T* p, float* o) {
        const uint2 raw = *reinterpret_cast<const uint2*>(p);
        const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&raw.x));
        const float2 b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&raw.y));
        o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
    }
    __device__ __forceinline__ static void st4(T* p, const float* v) {
        __nv_bfloat162 a = __floats2bfloat162_rn(v[0], v[1]), b = __floats2bfloat162_rn(v[2], v[3]);
        uint2 raw;
        raw.x = *reinterpret_cast<uint32_t*>(&a);
        raw.y = *reinterpret_cast<uint32_t*>(&b);
        __stcs(reinterpret_cast<uint2*>(p), raw);
    }
    __device__ __forceinline__ static void ld2(const T* p, float* o) {
        const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(p));
        o[0] = a.x; o[1] = a.y;
    }
    __device__ __forceinline__ static void st2(T* p, const float* v) {
        *reinterpret_cast<__nv_bfloat162*>(p) = __floats2bfloat162_rn(v[0], v[1]);
    }
    __device__ __forceinline__ static void st_sr(T* p, float g, uint32_t rb) {
        __stcs(reinterpret_cast<unsigned short*>(p), (unsigned short)(cvt_rs_bf16x2(g, 0.f, rb) & 0xffffu));
    }
    __device__ __forceinline__ static void st2_sr(T* p, const float* v, uint32_t rb) {
        __stcs(reinterpret_cast<unsigned int*>(p), cvt_rs_bf16x2(v[0], v[1], rb));
    }
    __device__ __forceinline__ static void st4_sr(T* p, const float* v, uint32_t rb0, uint32_t rb1) {
        __stcs(reinterpret_cast<uint2*>(p),
               make_uint2(cvt_rs_bf16x2(v[0], v[1], rb0), cvt_rs_bf16x2(v[2], v[3], rb1)));
    }
};
// Random words for the stochastically rounded stores of one thread: one hash of
// the (global) index of its first cell and of a value it loaded, then a cheap
// odd-multiplier derivation per stored word k (k < 64).
__device__ __forceinline__ uint32_t sr_seed(uint32_t cell, float v) {
    return mix32(cell ^ (__float_as_uint(v) * 0x9e3779b9u));
}
__device__ __forceinline__ uint32_t sr_word(uint32_t h, int k) {
    uint32_t rb = h * ((2u * (uint32_t)k + 1u) * 0x85ebca6bu);
    return rb ^ (rb >> 15);
}
template <class ST, int VEC>
__device__ __forceinline__ void stv_raw_sr(typename ST::T* p, const float* v, uint32_t h, int q) {
    if constexpr (VEC == 4) Raw<ST>::st4_sr(p, v, sr_word(h, 2 * q), sr_word(h, 2 * q + 1));
    else if constexpr (VEC == 2) Raw<ST>::st2_sr(p, v, sr_word(h, 2 * q));
    else Raw<ST>::st_sr(p, v[0], sr_word(h, 2 * q));
}
template <class ST, int VEC>
__device__ __forceinline__ void ldv_raw(const typename ST::T* p, float* o) {
    if constexpr (VEC == 4) Raw<ST>::ld4(p, o);
    else if constexpr (VEC == 2) Raw<ST>::ld2(p, o);
    else o[0] = Raw<ST>::ld(p);
}
template <class ST, int VEC>
__device__ __forceinline__ void stv_raw(typename ST::T* p, const float* v) {
    if constexpr (VEC == 4) Raw<ST>::st4(p, v);
    else if constexpr (VEC == 2) Raw<ST>::st2(p, v);
    else Raw<ST>::st(p, v[0]);
}

template <class ST, int VEC>
__device__ __forceinline__ void ldv(const typename ST::T* p, int q, float r0, typename Real<ST>::type* o) {
    if constexpr (VEC == 4) ST::ld4(p, q, r0, o);
    else if constexpr (VEC == 2) ST::ld2(p, q, r0, o);
    else o[0] = ST::ld(p, q, r0);
}
template <class ST, int VEC>
__device__ __forceinline__ void stv(typename ST::T* p, int q, float r0, const typename Real<ST>::type* v) {
    if constexpr (VEC == 4) ST::st4(p, q, r0, v);
    else if constexpr (VEC == 2) ST::st2(p, q, r0, v);
    else ST::st(p, q, r0, v[0]);
}

// ---- FP64 block reduction of NSTAT partial sums ---------------------------
// Warp shuffles, then one warp over the per-warp results; thread 0 writes the
// block's NSTAT partials to out[blockIdx.x * NSTAT + k].  Deterministic for a
// fixed launch shape (a fixed tree per block, a fixed block order in the
// final pass).
__device__ __forceinline__ void block_reduce_stats(double (&acc)[NSTAT], double* out) {
    __shared__ double red[32][NSTAT];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nwarps = (blockDim.x + 31) >> 5;
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
            double v = (lane < nwarps) ? red[lane][k] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if (lane == 0) out[(size_t)blockIdx.x * NSTAT + k] = v;
        }
    }
    __syncthreads();
}

}  // namespace lbm
