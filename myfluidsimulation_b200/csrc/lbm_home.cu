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
//     only the 5, or 1, populations that point into the tile);
//   * a link that does not stream (solid neighbour, duct inlet/outlet) is
//     handled by the gathering cell, which writes the replacement into the slot
//     of the source it would have gathered from (each slot has one reader);
//   * the gather is 19 shared-memory loads and pair sums.
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
        up = sm + (((p % 3) + 3) % 3) * UP_SZ;
        mid = sm + MID_OFF + (p & 1) * MID_SZ;
        dn = sm + DN_OFF;
    }
    template <int q>
    __device__ __forceinline__ float& at(int pos) const {
        return (cz(q) > 0 ? up : (cz(q) == 0 ? mid : dn))[gofs(q) + pos];
    }
};

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

// Rebuild coefficients of one cell, pre-scaled by w1 = 1/18 (w0 = 6 w1, w2 = w1/2):
//   P = w1 (rho - 1.5 tr B),  a_k = 3 w1 rho u_k,  b_kk = 4.5 w1 B_kk,  b_kl = 9 w1 B_kl,
//   B = rho u u + (1 - w) S.  Then f*_q = P + sum_k c_k a_k + sum_k c_k^2 b_kk
//   + sum_{k<l} c_k c_l b_kl for the axis directions, half of that for the
//   diagonals, and 6 P for the rest direction.
struct Coef {
    float P, ax, ay, az, bxx, byy, bzz, bxy, bxz, byz;
    __device__ __forceinline__ void set(const float (&m)[10], float omw) {
        const float r = m[0];
        const float jx = r * m[1], jy = r * m[2], jz = r * m[3];
        const float Bxx = fmaf(jx, m[1], omw * m[4]);
        const float Bxy = fmaf(jx, m[2], omw * m[5]);
        const float Bxz = fmaf(jx, m[3], omw * m[6]);
        const float Byy = fmaf(jy, m[2], omw * m[7]);
        const float Byz = fmaf(jy, m[3], omw * m[8]);
        const float Bzz = fmaf(jz, m[3], omw * m[9]);
        constexpr float w1 = 1.0f / 18.0f;
        P = w1 * fmaf(-1.5f, Bxx + Byy + Bzz, r);
        ax = (3.0f * w1) * jx; ay = (3.0f * w1) * jy; az = (3.0f * w1) * jz;
        bxx = (4.5f * w1) * Bxx; byy = (4.5f * w1) * Byy; bzz = (4.5f * w1) * Bzz;
        bxy = (9.0f * w1) * Bxy; bxz = (9.0f * w1) * Bxz; byz = (9.0f * w1) * Byz;
    }
    // one population (halo positions and the boundary path)
    template <int q>
    __device__ __forceinline__ float fpost() const {
        constexpr int X = cx(q), Y = cy(q), Z = cz(q);
        if constexpr (q == 0) {
            return 6.0f * P;
        } else {
            float s = P;
            if (X) s += X > 0 ? ax : -ax;
            if (Y) s += Y > 0 ? ay : -ay;
            if (Z) s += Z > 0 ? az : -az;
            if (X) s += bxx;
            if (Y) s += byy;
            if (Z) s += bzz;
            if (X && Y) s += X * Y > 0 ? bxy : -bxy;
            if (X && Z) s += X * Z > 0 ? bxz : -bxz;
            if (Y && Z) s += Y * Z > 0 ? byz : -byz;
            return ((X != 0) + (Y != 0) + (Z != 0)) == 2 ? 0.5f * s : s;
        }
    }
};

template <int q> struct QI { static constexpr int value = q; };
template <int Q0, int Q1, class F>
__device__ __forceinline__ void static_for(F&& fn) {
    if constexpr (Q0 < Q1) {
        fn(QI<Q0>{});
        static_for<Q0 + 1, Q1>(fn);
    }
}

// A tile cell writes all 19 populations leaving its plane.
__device__ __forceinline__ void build_tile_cell(const Ring& R, int pos, const Coef& c) {
    R.at<0>(pos) = 6.0f * c.P;
    const float bx = c.P + c.bxx, by = c.P + c.byy, bz = c.P + c.bzz;
    R.at<1>(pos) = bx + c.ax;
    R.at<2>(pos) = bx - c.ax;
    R.at<3>(pos) = by + c.ay;
    R.at<4>(pos) = by - c.ay;
    R.at<5>(pos) = bz + c.az;
    R.at<6>(pos) = bz - c.az;
    {
        const float b = bx + c.byy, bp = b + c.bxy, bm = b - c.bxy;
        const float sp = c.ax + c.ay, sn = c.ax - c.ay;
        R.at<7>(pos) = 0.5f * (bp + sp);     // (+1,+1,0)
        R.at<10>(pos) = 0.5f * (bp - sp);    // (-1,-1,0)
        R.at<9>(pos) = 0.5f * (bm + sn);     // (+1,-1,0)
        R.at<8>(pos) = 0.5f * (bm - sn);     // (-1,+1,0)
    }
    {
        const float b = bx + c.bzz, bp = b + c.bxz, bm = b - c.bxz;
        const float sp = c.ax + c.az, sn = c.ax - c.az;
        R.at<11>(pos) = 0.5f * (bp + sp);    // (+1,0,+1)
        R.at<14>(pos) = 0.5f * (bp - sp);    // (-1,0,-1)
        R.at<13>(pos) = 0.5f * (bm + sn);    // (+1,0,-1)
        R.at<12>(pos) = 0.5f * (bm - sn);    // (-1,0,+1)
    }
    {
        const float b = by + c.bzz, bp = b + c.byz, bm = b - c.byz;
        const float sp = c.ay + c.az, sn = c.ay - c.az;
        R.at<15>(pos) = 0.5f * (bp + sp);    // (0,+1,+1)
        R.at<18>(pos) = 0.5f * (bp - sp);    // (0,-1,-1)
        R.at<17>(pos) = 0.5f * (bm + sn);    // (0,+1,-1)
        R.at<16>(pos) = 0.5f * (bm - sn);    // (0,-1,+1)
    }
}

// A halo position writes only the directions that point into the tile:
// dir 0 = x-1 column (+x), 1 = x+TX column (-x), 2 = y-1 row (+y),
// 3 = y+TY row (-y), 4..7 = corners feeding 7, 8, 9, 10.
__device__ __forceinline__ void build_halo(const Ring& R, int pos, int dir, const Coef& c) {
    switch (dir) {
        case 0:
            R.at<1>(pos) = c.fpost<1>(); R.at<7>(pos) = c.fpost<7>(); R.at<9>(pos) = c.fpost<9>();
            R.at<11>(pos) = c.fpost<11>(); R.at<13>(pos) = c.fpost<13>();
            break;
        case 1:
            R.at<2>(pos) = c.fpost<2>(); R.at<8>(pos) = c.fpost<8>(); R.at<10>(pos) = c.fpost<10>();
            R.at<12>(pos) = c.fpost<12>(); R.at<14>(pos) = c.fpost<14>();
            break;
        case 2:
            R.at<3>(pos) = c.fpost<3>(); R.at<7>(pos) = c.fpost<7>(); R.at<8>(pos) = c.fpost<8>();
            R.at<15>(pos) = c.fpost<15>(); R.at<17>(pos) = c.fpost<17>();
            break;
        case 3:
            R.at<4>(pos) = c.fpost<4>(); R.at<9>(pos) = c.fpost<9>(); R.at<10>(pos) = c.fpost<10>();
            R.at<16>(pos) = c.fpost<16>(); R.at<18>(pos) = c.fpost<18>();
            break;
        case 4: R.at<7>(pos) = c.fpost<7>(); break;
        case 5: R.at<8>(pos) = c.fpost<8>(); break;
        case 6: R.at<9>(pos) = c.fpost<9>(); break;
        case 7: R.at<10>(pos) = c.fpost<10>(); break;
        default: break;
    }
}

template <class T, bool STATS>
__global__ void __launch_bounds__(NT, 3) home_step(HomeParams p) {
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
    const int x0 = (b % tiles_x) * TX; b /= tiles_x;
    const int y0 = (b % tiles_y) * TY; b /= tiles_y;
    const int z0 = b * p.zchunk;
    const int z1 = min(nz, z0 + p.zchunk);
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
    const int64_t plane = (int64_t)nx * ny;
    const int64_t coff = (int64_t)gy * nx + gx;

    const uint8_t* __restrict__ flags = p.flags;
    float mreg[10];
#pragma unroll
    for (int c = 0; c < 10; ++c) mreg[c] = 0.f;
    uint32_t freg = 0;
    auto load = [&](int z) {
        if (!exists) return;
        const int zz = z < 0 ? z + nz : (z >= nz ? z - nz : z);
        const int64_t id = (int64_t)zz * plane + coff;
        const T* ptr = m + id;
#pragma unroll
        for (int c = 0; c < 10; ++c) {
            mreg[c] = MomStore<T>::ld(ptr, c, r0);
            ptr += N;
        }
        freg = flags ? flags[id] : 0u;
    };
    // the moments of plane pz are in mreg/freg: write the populations leaving it
    // (a solid cell writes none; its slots are filled by its fluid neighbours)
    auto arrive = [&](int pz) {
        if (exists && !(freg & F_SOLID)) {
            Coef c;
            c.set(mreg, omw);
            const Ring R(sm, pz);
            if (dir == -1) build_tile_cell(R, pos, c);
            else build_halo(R, pos, dir, c);
        }
    };

    double acc[NSTAT];
#pragma unroll
    for (int k = 0; k < NSTAT; ++k) acc[k] = 0.0;

    load(z0 - 1);
    arrive(z0 - 1);
    load(z0);
    arrive(z0);
    uint32_t fcur = freg;          // this position's flags in the plane being gathered
    load(z0 + 1);

    for (int z = z0; z < z1; ++z) {
        // 1. plane z+1 arrives (its moments were loaded one iteration ago); z+2 is requested
        arrive(z + 1);
        const uint32_t fnext = freg;
        if (z + 2 <= z1) load(z + 2);
        // 2. a link that does not stream: the cell writes the replacement into the
        //    slot of the source it would have gathered from (read by nobody else)
        if (owner && (fcur & F_SPECIAL)) {
            const int64_t id = (int64_t)z * plane + coff;
            const uint32_t lk = p.links[id];
            float own[10];
            {
                const T* ptr = m + id;
#pragma unroll
                for (int c = 0; c < 10; ++c) { own[c] = MomStore<T>::ld(ptr, c, r0); ptr += N; }
            }
            Coef oc;
            oc.set(own, omw);
            const Ring Rm(sm, z - 1), Rz(sm, z), Rp(sm, z + 1);
            static_for<1, 19>([&](auto qi) {
                constexpr int q = decltype(qi)::value;
                if ((lk >> opp(q)) & 1u) {
                    const int xs = gx - cx(q);
                    float v;
                    if (p.duct && xs < 0) {
                        v = feq_ref(q, own[0], p.u_in, 0.f, 0.f);                      // inlet
                    } else if (p.duct && xs >= nx) {
                        v = oc.template fpost<q>();                                       // outlet
                    } else {
                        // own post-collision population of direction bq comes back as q
                        // (home.cu:219-225); bq = opp(q), or the reference's table
                        constexpr int bt = opp(q), br = opp_tab(q);
                        v = p.ref_bounce ? oc.template fpost<br>() : oc.template fpost<bt>();
                        if (STATS) {
                            const int bq = p.ref_bounce ? br : bt;
                            const int ys = ((gy - cy(q)) % ny + ny) % ny;
                            const int zs = ((z - cz(q)) % nz + nz) % nz;
                            const int xw = ((xs % nx) + nx) % nx;
                            if (flags[(int64_t)zs * plane + (int64_t)ys * nx + xw] & F_OBST) {
                                acc[2] += (double)(cx(bq) - cx(q)) * (double)v;
                                acc[3] += (double)(cy(bq) - cy(q)) * (double)v;
                                acc[4] += (double)(cz(bq) - cz(q)) * (double)v;
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
            const int64_t id = (int64_t)z * plane + coff;
            T* op = mn + id;
            if (fcur & F_SOLID) {
                MomStore<T>::st(op, 0, r0, 1.f);
#pragma unroll
                for (int c = 1; c < 10; ++c) MomStore<T>::st(op + c * N, c, r0, 0.f);
            } else {
                const Ring Rm(sm, z - 1), Rz(sm, z), Rp(sm, z + 1);
                float fq[19];
                static_for<0, 19>([&](auto qi) {
                    constexpr int q = decltype(qi)::value;
                    const Ring& R = cz(q) > 0 ? Rm : (cz(q) == 0 ? Rz : Rp);
                    fq[q] = R.template at<q>(pos - cx(q) - HX * cy(q));
                });
                // moments of the gathered populations (home.cu:238-273), opposite pairs first
                const float s1 = fq[1] + fq[2], d1 = fq[1] - fq[2];
                const float s3 = fq[3] + fq[4], d3 = fq[3] - fq[4];
                const float s5 = fq[5] + fq[6], d5 = fq[5] - fq[6];
                const float s7 = fq[7] + fq[10], d7 = fq[7] - fq[10];     // (+1,+1,0)
                const float s9 = fq[9] + fq[8], d9 = fq[9] - fq[8];       // (+1,-1,0)
                const float s11 = fq[11] + fq[14], d11 = fq[11] - fq[14]; // (+1,0,+1)
                const float s13 = fq[13] + fq[12], d13 = fq[13] - fq[12]; // (+1,0,-1)
                const float s15 = fq[15] + fq[18], d15 = fq[15] - fq[18]; // (0,+1,+1)
                const float s17 = fq[17] + fq[16], d17 = fq[17] - fq[16]; // (0,+1,-1)
                const float r = fq[0] + ((s1 + s3) + (s5 + s7)) + ((s9 + s11) + (s13 + s15) + s17);
                const float jx = (d1 + d7) + (d9 + d11) + d13;
                const float jy = (d3 + d7) - d9 + (d15 + d17);
                const float jz = (d5 + d11) - d13 + (d15 - d17);
                const float Mxx = (s1 + s7) + (s9 + s11) + s13;
                const float Myy = (s3 + s7) + (s9 + s15) + s17;
                const float Mzz = (s5 + s11) + (s13 + s15) + s17;
                const float Mxy = s7 - s9, Mxz = s11 - s13, Myz = s15 - s17;
                const float inv = r > 0.f ? 1.0f / r : 0.f;
                const float ux = jx * inv + p.fx, uy = jy * inv + p.fy, uz = jz * inv + p.fz;
                const float r3 = r * (1.0f / 3.0f);
                const float rx = r * ux, ry = r * uy, rz = r * uz;
                const float out[10] = {r, ux, uy, uz,
                                       Mxx - fmaf(rx, ux, r3), Mxy - rx * uy, Mxz - rx * uz,
                                       Myy - fmaf(ry, uy, r3), Myz - ry * uz, Mzz - fmaf(rz, uz, r3)};
#pragma unroll
                for (int c = 0; c < 10; ++c) {
                    MomStore<T>::st(op, c, r0, out[c]);
                    op += N;
                }
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
