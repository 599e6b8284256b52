// HOME moment-only step (src/lbm/lbm3d_home.cu:37-286): the state is 10
// moments per cell [rho, ux, uy, uz, Sxx, Sxy, Sxz, Syy, Syz, Szz]; every step
// rebuilds each neighbour's post-collision population from its moments,
// gathers the 19 incoming populations and stores their moments.
//
// The reference rebuilds f_q 19 times per cell from global loads of the
// neighbour's 10 moments (190 loads and ~1.1 kFLOP per cell).  Here each
// block owns a 32 x 8 tile of an (x,y) plane and marches along z over a chunk
// of planes:
//   * the moments of plane z+1 (tile + 1-cell halo) are prefetched into
//     registers one iteration ahead, so their loads overlap the gather of z;
//   * every cell's 19 post-collision populations are built ONCE, from the
//     identity  f*_q = w_q [rho + 3 c_q.(rho u) + 4.5 Q_q : (rho u u + (1-w) S)]
//     with Q_q = c_q c_q - I/3, which is src/lbm/lbm3d_home.cu:57-80
//     rearranged (4.5(c.u)^2 - 1.5u^2 = 4.5 Q:uu), and kept in shared memory,
//     grouped by c_z: the 5 down-going ones of plane z+1, the 9 in-plane ones
//     of planes z and z+1, the 5 up-going ones of planes z-1, z and z+1;
//   * the gather is then 19 shared-memory loads per cell.
// DRAM traffic is the 10 moments read once and written once (80 B per cell in
// FP32) plus the halo re-reads that L2 does not absorb.
#include "lbm_common.cuh"
#include "lbm_internal.h"

namespace lbm {
namespace {

constexpr int TX = 32;
constexpr int TY = 8;
constexpr int HX = TX + 2;
constexpr int HY = TY + 2;
constexpr int HC = HX * HY;       // 340 halo-tile cells
constexpr int NT = TX * TY;       // 256 threads
constexpr int PER = (HC + NT - 1) / NT;   // halo cells per thread (2)

// c_z groups in q order
__host__ __device__ constexpr int grp(int q) { return cz(q) > 0 ? 2 : (cz(q) < 0 ? 0 : 1); }
__host__ __device__ constexpr int gidx(int q) {
    // position of q inside its group
    int k = 0;
    for (int i = 0; i < q; ++i) k += (grp(i) == grp(q));
    return k;
}
// shared layout offsets (floats)
constexpr int DN_OFF = 0;                   // [5][HC]   plane z+1
constexpr int MID_OFF = 5 * HC;             // [2][9][HC] planes by parity
constexpr int UP_OFF = MID_OFF + 18 * HC;   // [3][5][HC] planes mod 3
constexpr int SMEM_FLOATS = UP_OFF + 15 * HC;

// Moment storage: F32 as is; F16/BF16 keep rho - rho0, u and S.
template <class T> struct MomStore;
template <> struct MomStore<float> {
    __device__ __forceinline__ static float ld(const float* p, int k, float r0) { return __ldg(p); }
    __device__ __forceinline__ static void st(float* p, int k, float r0, float v) { *p = v; }
};
template <> struct MomStore<__half> {
    __device__ __forceinline__ static float ld(const __half* p, int k, float r0) {
        return __half2float(*p) + (k == 0 ? r0 : 0.f);
    }
    __device__ __forceinline__ static void st(__half* p, int k, float r0, float v) {
        *p = __float2half_rn(k == 0 ? v - r0 : v);
    }
};
template <> struct MomStore<__nv_bfloat16> {
    __device__ __forceinline__ static float ld(const __nv_bfloat16* p, int k, float r0) {
        return __bfloat162float(*p) + (k == 0 ? r0 : 0.f);
    }
    __device__ __forceinline__ static void st(__nv_bfloat16* p, int k, float r0, float v) {
        *p = __float2bfloat16_rn(k == 0 ? v - r0 : v);
    }
};

// The 10 regularised-rebuild coefficients of one cell.
struct Coef {
    float P, ax, ay, az, bxx, byy, bzz, bxy, bxz, byz;
    __device__ __forceinline__ void from_moments(const float (&m)[10], float omw) {
        const float r = m[0];
        ax = r * m[1]; ay = r * m[2]; az = r * m[3];
        bxx = ax * m[1] + omw * m[4];
        bxy = ax * m[2] + omw * m[5];
        bxz = ax * m[3] + omw * m[6];
        byy = ay * m[2] + omw * m[7];
        byz = ay * m[3] + omw * m[8];
        bzz = az * m[3] + omw * m[9];
        P = r - 1.5f * (bxx + byy + bzz);
    }
    // f*_q = w_q [P + 3 c.a + 4.5 sum_a c_a^2 B_aa + 9 sum_{a<b} c_a c_b B_ab]
    template <int q>
    __device__ __forceinline__ float fpost() const {
        float s = P;
        constexpr int X = cx(q), Y = cy(q), Z = cz(q);
        if (X) s += (X > 0 ? 3.f : -3.f) * ax;
        if (Y) s += (Y > 0 ? 3.f : -3.f) * ay;
        if (Z) s += (Z > 0 ? 3.f : -3.f) * az;
        if (X) s += 4.5f * bxx;
        if (Y) s += 4.5f * byy;
        if (Z) s += 4.5f * bzz;
        if (X && Y) s += (X * Y > 0 ? 9.f : -9.f) * bxy;
        if (X && Z) s += (X * Z > 0 ? 9.f : -9.f) * bxz;
        if (Y && Z) s += (Y * Z > 0 ? 9.f : -9.f) * byz;
        return wq(q) * s;
    }
};

template <int q>
struct QI { static constexpr int value = q; };

template <int Q0, int Q1, class F>
__device__ __forceinline__ void static_for(F&& fn) {
    if constexpr (Q0 < Q1) {
        fn(QI<Q0>{});
        static_for<Q0 + 1, Q1>(fn);
    }
}

template <class T, bool STATS>
__global__ void __launch_bounds__(NT, 2) home_step(HomeParams p) {
    extern __shared__ float sm[];
    const T* __restrict__ m = static_cast<const T*>(p.m);
    T* __restrict__ mn = static_cast<T*>(p.mn);
    const int64_t N = p.N;
    const int nx = p.nx, ny = p.ny, nz = p.nz;
    const float omw = 1.f - p.omega;
    const float r0 = p.rho0;

    const int tiles_x = (nx + TX - 1) / TX;
    const int tiles_y = (ny + TY - 1) / TY;
    int b = blockIdx.x;
    const int tx0 = (b % tiles_x) * TX; b /= tiles_x;
    const int ty0 = (b % tiles_y) * TY; b /= tiles_y;
    const int z0 = b * p.zchunk;
    const int z1 = min(nz, z0 + p.zchunk);
    const int tid = threadIdx.x;

    // halo cells staged by this thread
    int64_t hoff[PER];     // plane-relative offset, -1 if outside / not mine
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const int i = tid + k * NT;
        hoff[k] = -1;
        if (i < HC) {
            int gx = tx0 - 1 + (i % HX);
            int gy = ty0 - 1 + (i / HX);
            gy = ((gy % ny) + ny) % ny;
            bool ok = true;
            if (p.duct) ok = (gx >= 0 && gx < nx);
            else gx = ((gx % nx) + nx) % nx;
            if (ok) hoff[k] = (int64_t)gy * nx + gx;
        }
    }
    const int64_t plane = (int64_t)nx * ny;
    float reg[PER][10];
    auto load_plane = [&](int z) {
        const int zz = ((z % nz) + nz) % nz;
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            if (hoff[k] < 0) continue;
            const int64_t id = (int64_t)zz * plane + hoff[k];
#pragma unroll
            for (int c = 0; c < 10; ++c) reg[k][c] = MomStore<T>::ld(m + c * N + id, c, r0);
        }
    };
    // builds the populations of the staged plane z into shared memory;
    // which = 1: only the up-going group, 2: up-going + in-plane, 3: all
    auto build_plane = [&](int z, int which) {
        float* up = sm + UP_OFF + (((z % 3) + 3) % 3) * 5 * HC;
        float* mid = sm + MID_OFF + (z & 1) * 9 * HC;
        float* dn = sm + DN_OFF;
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const int i = tid + k * NT;
            if (hoff[k] < 0) continue;
            Coef cf;
            cf.from_moments(reg[k], omw);
            static_for<0, 19>([&](auto qi) {
                constexpr int q = decltype(qi)::value;
                constexpr int g = grp(q), j = gidx(q);
                if (g == 2) up[j * HC + i] = cf.template fpost<q>();
                else if (g == 1) { if (which >= 2) mid[j * HC + i] = cf.template fpost<q>(); }
                else { if (which >= 3) dn[j * HC + i] = cf.template fpost<q>(); }
            });
        }
    };

    double acc[NSTAT];
#pragma unroll
    for (int k = 0; k < NSTAT; ++k) acc[k] = 0.0;

    const int lx = tid % TX, ly = tid / TX;
    const int gx = tx0 + lx, gy = ty0 + ly;
    const bool inside = gx < nx && gy < ny;
    const int hc = (ly + 1) * HX + (lx + 1);

    load_plane(z0 - 1);
    build_plane(z0 - 1, 1);
    load_plane(z0);
    build_plane(z0, 2);
    load_plane(z0 + 1);
    for (int z = z0; z < z1; ++z) {
        build_plane(z + 1, 3);
        if (z + 1 < z1) load_plane(z + 2);
        __syncthreads();
        if (inside) {
            const int64_t id = (int64_t)z * plane + (int64_t)gy * nx + gx;
            const uint32_t fl = p.flags ? p.flags[id] : 0u;
            if (fl & F_SOLID) {
                MomStore<T>::st(mn + id, 0, r0, 1.f);
#pragma unroll
                for (int c = 1; c < 10; ++c) MomStore<T>::st(mn + c * N + id, c, r0, 0.f);
            } else {
                const float* up = sm + UP_OFF + (((z - 1) % 3 + 3) % 3) * 5 * HC;
                const float* mid = sm + MID_OFF + (z & 1) * 9 * HC;
                const float* dn = sm + DN_OFF;
                float fq[19];
                static_for<0, 19>([&](auto qi) {
                    constexpr int q = decltype(qi)::value;
                    constexpr int g = grp(q), j = gidx(q);
                    const int src = hc - cx(q) - HX * cy(q);
                    fq[q] = (g == 2 ? up : (g == 1 ? mid : dn))[j * HC + src];
                });
                if (fl & F_SPECIAL) {
                    // links that do not stream: rebuild from the cell's own moments
                    const uint32_t lk = p.links[id];
                    float own[10];
#pragma unroll
                    for (int c = 0; c < 10; ++c) own[c] = MomStore<T>::ld(m + c * N + id, c, r0);
                    Coef oc;
                    oc.from_moments(own, omw);
                    float of[19];
                    static_for<0, 19>([&](auto qi) {
                        constexpr int q = decltype(qi)::value;
                        of[q] = oc.template fpost<q>();
                    });
                    static_for<1, 19>([&](auto qi) {
                        constexpr int q = decltype(qi)::value;
                        if ((lk >> opp(q)) & 1u) {
                            const int xs = gx - cx(q);
                            if (p.duct && xs < 0) {
                                fq[q] = feq_ref(q, own[0], p.u_in, 0.f, 0.f);          // inlet
                            } else if (p.duct && xs >= nx) {
                                fq[q] = of[q];                                           // outlet
                            } else {
                                // own post-collision population of direction b comes back as q
                                // (home.cu:219-225); b = opp(q), or the reference's table
                                constexpr int b_true = opp(q), b_tab = opp_tab(q);
                                const int b = p.ref_bounce ? b_tab : b_true;
                                fq[q] = p.ref_bounce ? of[b_tab] : of[b_true];
                                if (STATS && (fl & F_TOUCH)) {
                                    const int ys = ((gy - cy(q)) % ny + ny) % ny;
                                    const int zs = ((z - cz(q)) % nz + nz) % nz;
                                    const int xw = ((xs % nx) + nx) % nx;
                                    if (p.flags[(int64_t)zs * plane + (int64_t)ys * nx + xw] & F_OBST) {
                                        acc[2] += (double)(cx(b) - cx(q)) * (double)fq[q];
                                        acc[3] += (double)(cy(b) - cy(q)) * (double)fq[q];
                                        acc[4] += (double)(cz(b) - cz(q)) * (double)fq[q];
                                    }
                                }
                            }
                        }
                    });
                }
                // moments of the gathered populations (home.cu:238-273)
                float r = 0.f, jx = 0.f, jy = 0.f, jz = 0.f;
                float Mxx = 0.f, Mxy = 0.f, Mxz = 0.f, Myy = 0.f, Myz = 0.f, Mzz = 0.f;
                static_for<0, 19>([&](auto qi) {
                    constexpr int q = decltype(qi)::value;
                    constexpr int X = cx(q), Y = cy(q), Z = cz(q);
                    const float v = fq[q];
                    r += v;
                    if (X) jx += X > 0 ? v : -v;
                    if (Y) jy += Y > 0 ? v : -v;
                    if (Z) jz += Z > 0 ? v : -v;
                    if (X) Mxx += v;
                    if (Y) Myy += v;
                    if (Z) Mzz += v;
                    if (X && Y) Mxy += X * Y > 0 ? v : -v;
                    if (X && Z) Mxz += X * Z > 0 ? v : -v;
                    if (Y && Z) Myz += Y * Z > 0 ? v : -v;
                });
                float ux = (r > 0.f) ? (jx / r) : 0.f;
                float uy = (r > 0.f) ? (jy / r) : 0.f;
                float uz = (r > 0.f) ? (jz / r) : 0.f;
                ux += p.fx; uy += p.fy; uz += p.fz;
                const float cs2 = 1.0f / 3.0f;
                const float out[10] = {r, ux, uy, uz,
                                       Mxx - (r * cs2 + r * ux * ux), Mxy - r * ux * uy, Mxz - r * ux * uz,
                                       Myy - (r * cs2 + r * uy * uy), Myz - r * uy * uz,
                                       Mzz - (r * cs2 + r * uz * uz)};
#pragma unroll
                for (int c = 0; c < 10; ++c) MomStore<T>::st(mn + c * N + id, c, r0, out[c]);
                if (STATS) {
                    acc[0] += (double)r;
                    acc[1] += 0.5 * ((double)ux * ux + (double)uy * uy + (double)uz * uz);
                    acc[5] += (double)r * ux;
                    acc[6] += (double)r * uy;
                    acc[7] += (double)r * uz;
                }
            }
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

template <class T>
cudaError_t launch_home_t(const HomeParams& p, cudaStream_t s) {
    const int tiles = ((p.nx + TX - 1) / TX) * ((p.ny + TY - 1) / TY);
    const int chunks = (p.nz + p.zchunk - 1) / p.zchunk;
    const size_t smem = sizeof(float) * SMEM_FLOATS;
    if (p.stats) home_step<T, true><<<tiles * chunks, NT, smem, s>>>(p);
    else home_step<T, false><<<tiles * chunks, NT, smem, s>>>(p);
    return cudaGetLastError();
}

}  // namespace

cudaError_t home_prepare() {
    const int smem = (int)(sizeof(float) * SMEM_FLOATS);
    cudaError_t e = cudaSuccess;
    auto set = [&](const void* fn) {
        if (e == cudaSuccess) e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    };
    set((const void*)home_step<float, false>);
    set((const void*)home_step<float, true>);
    set((const void*)home_step<__half, false>);
    set((const void*)home_step<__half, true>);
    set((const void*)home_step<__nv_bfloat16, false>);
    set((const void*)home_step<__nv_bfloat16, true>);
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
