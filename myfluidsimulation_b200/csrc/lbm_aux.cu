// Set-up and helper kernels: equilibrium (re)initialisation, the per-cell
// flag/link words built from the solid mask, the B0 band, the final pass of
// the FP64 statistics, and the reference's free device helpers
// (reinit_equilibrium_from_macro, launch_speed, make_rho_gauss/slab).
#include "lbm_common.cuh"
#include "lbm_internal.h"

namespace lbm {

int num_sms() {
    static int n = 0;
    if (n == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

namespace {

// The cs2 form of src/lbm/lbm_reinit.cu:35-46 (used by Legacy's reinit).
__device__ __forceinline__ float feq_cs2(int q, float r, float u0, float v0, float w0) {
    const float cs2 = 1.f / 3.f;
    const float uu = u0 * u0 + v0 * v0 + w0 * w0;
    const float cu = (float)cx(q) * u0 + (float)cy(q) * v0 + (float)cz(q) * w0;
    return wq(q) * r * (1.f + cu / cs2 + 0.5f * (cu * cu) / (cs2 * cs2) - 0.5f * uu / cs2);
}

template <class ST>
__global__ void aa_reinit(typename ST::T* f, float r0, int64_t N, const float* rho, const float* ux,
                          const float* uy, const float* uz, float* ro, float* uo, float* vo, float* wo,
                          int form) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        const float r = rho ? rho[i] : 1.0f;
        const float u = ux ? ux[i] : 0.0f;
        const float v = uy ? uy[i] : 0.0f;
        const float w = uz ? uz[i] : 0.0f;
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            const float fe = form == 0 ? feq_cs2(q, r, u, v, w) : feq_ref(q, r, u, v, w);
            ST::st(f + q * N + i, q, r0, fe);
        }
        if (ro) { ro[i] = r; uo[i] = u; vo[i] = v; wo[i] = w; }
    }
}

// FP64 storage: the equilibrium of the (FP32) macro fields evaluated in FP64
__global__ void aa_reinit_f64(double* f, int64_t N, const float* rho, const float* ux, const float* uy,
                              const float* uz, float* ro, float* uo, float* vo, float* wo) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        const double r = rho ? rho[i] : 1.0;
        const double u = ux ? ux[i] : 0.0;
        const double v = uy ? uy[i] : 0.0;
        const double w = uz ? uz[i] : 0.0;
        const double uu = u * u + v * v + w * w;
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            const double cu = (double)cx(q) * u + (double)cy(q) * v + (double)cz(q) * w;
            const double wd = q == 0 ? 1.0 / 3.0 : (q <= 6 ? 1.0 / 18.0 : 1.0 / 36.0);
            f[q * N + i] = wd * r * (1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * uu);
        }
        if (ro) { ro[i] = (float)r; uo[i] = (float)u; vo[i] = (float)v; wo[i] = (float)w; }
    }
}

template <class T> __device__ __forceinline__ void st_mom(T* p, int k, float r0, float v);
template <> __device__ __forceinline__ void st_mom<float>(float* p, int k, float r0, float v) { *p = v; }
template <> __device__ __forceinline__ void st_mom<__half>(__half* p, int k, float r0, float v) {
    *p = __float2half_rn((k == 0 ? v - r0 : v) * kF16Scale);   // the HOME F16 layout (lbm_home.cu)
}
template <> __device__ __forceinline__ void st_mom<__nv_bfloat16>(__nv_bfloat16* p, int k, float r0, float v) {
    *p = __float2bfloat16_rn(k == 0 ? v - r0 : v);
}
template <> __device__ __forceinline__ void st_mom<double>(double* p, int k, float r0, float v) { *p = v; }

// src/lbm/lbm3d_home.cu:109-137 (m = mnext = (rho, u, S = 0))
template <class T>
__global__ void home_reinit(T* m, T* mn, float r0, int64_t N, const float* rho, const float* ux, const float* uy,
                            const float* uz) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        const float v[4] = {rho ? rho[i] : 1.0f, ux ? ux[i] : 0.0f, uy ? uy[i] : 0.0f, uz ? uz[i] : 0.0f};
#pragma unroll
        for (int k = 0; k < 10; ++k) {
            const float x = k < 4 ? v[k] : 0.0f;
            st_mom<T>(m + k * N + i, k, r0, x);
            st_mom<T>(mn + k * N + i, k, r0, x);
        }
    }
}

__device__ __forceinline__ int wrapi(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

__global__ void build_flags(const uint8_t* __restrict__ mask, const uint8_t* __restrict__ band,
                            uint8_t* __restrict__ flags, uint32_t* __restrict__ links, int nx, int ny, int nz,
                            int duct) {
    const int64_t N = (int64_t)nx * ny * nz;
    for (int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; id < N; id += (int64_t)gridDim.x * blockDim.x) {
        const uint8_t mk = mask ? mask[id] : 0;
        uint8_t fl = 0;
        uint32_t lk = 0;
        if (mk) {
            fl = F_SOLID | ((mk & 8) ? 0 : F_OBST);
        } else {
            if (band && band[id]) fl |= F_BAND;
            const int x = (int)(id % nx);
            const int64_t row = id / nx;
            const int y = (int)(row % ny), z = (int)(row / ny);
            bool touch = false;
#pragma unroll
            for (int q = 1; q < 19; ++q) {
                const int xt = x + cx(q);
                if (duct && (xt < 0 || xt >= nx)) { lk |= 1u << q; continue; }
                if (!mask) continue;
                const int64_t t = ((int64_t)wrapi(z + cz(q), nz) * ny + wrapi(y + cy(q), ny)) * nx + wrapi(xt, nx);
                const uint8_t m2 = mask[t];
                if (m2) {
                    lk |= 1u << q;
                    if (!(m2 & 8)) touch = true;
                }
            }
            if (lk) fl |= F_SPECIAL;
            if (touch) fl |= F_TOUCH;
        }
        flags[id] = fl;
        links[id] = lk;
    }
}

__global__ void band_init(const uint8_t* __restrict__ mask, int32_t* __restrict__ dist, int64_t N) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x)
        dist[i] = mask[i] ? 0 : -1;
}

// one BFS layer: unlabelled cells next to a cell of layer k-1 get k (6 neighbours, no wrap)
__global__ void band_grow(int32_t* dist, int nx, int ny, int nz, int k) {
    const int64_t N = (int64_t)nx * ny * nz;
    const int64_t sy = nx, sz = (int64_t)nx * ny;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        if (dist[i] != -1) continue;
        const int x = (int)(i % nx);
        const int64_t row = i / nx;
        const int y = (int)(row % ny), z = (int)(row / ny);
        const int want = k - 1;
        bool hit = (x > 0 && dist[i - 1] == want) || (x < nx - 1 && dist[i + 1] == want) ||
                   (y > 0 && dist[i - sy] == want) || (y < ny - 1 && dist[i + sy] == want) ||
                   (z > 0 && dist[i - sz] == want) || (z < nz - 1 && dist[i + sz] == want);
        if (hit) dist[i] = k;
    }
}

__global__ void band_final(const uint8_t* __restrict__ mask, const int32_t* __restrict__ dist,
                           uint8_t* __restrict__ band, int64_t N, int d0, unsigned long long* count) {
    unsigned long long c = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t d = dist[i];
        const uint8_t b = (!mask[i] && d >= 0 && d <= d0) ? 1 : 0;
        band[i] = b;
        c += b;
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}

// Sums the per-block partials in a fixed order (deterministic).
__global__ void finalize_stats(const double* __restrict__ partials, int nblocks, double* __restrict__ out) {
    double acc[NSTAT];
#pragma unroll
    for (int k = 0; k < NSTAT; ++k) acc[k] = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
#pragma unroll
        for (int k = 0; k < NSTAT; ++k) acc[k] += partials[(size_t)b * NSTAT + k];
    __shared__ double red[32][NSTAT];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NSTAT; ++k) {
        double v = acc[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[warp][k] = v;
    }
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
#pragma unroll
        for (int k = 0; k < NSTAT; ++k) {
            double v = lane < nw ? red[lane][k] : 0.0;
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if (lane == 0) out[k] = v;
        }
    }
}

// ---- the reference's free device helpers (same arithmetic) ----------------
__global__ void reinit_eq_kernel(const float* rho, const float* ux, const float* uy, const float* uz, float* f,
                                 int N) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const float r = rho[i];
    const float u0 = ux ? ux[i] : 0.f, v0 = uy ? uy[i] : 0.f, w0 = uz ? uz[i] : 0.f;
#pragma unroll
    for (int q = 0; q < 19; ++q) f[(int64_t)q * N + i] = feq_cs2(q, r, u0, v0, w0);
}

__global__ void speed_kernel(const float* u, const float* v, const float* w, float* out, int N) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) {
        const float uu = u[i] * u[i] + v[i] * v[i] + w[i] * w[i];
        out[i] = sqrtf(uu);
    }
}

__global__ void rho_gauss_kernel(float* rho, int Nx, int Ny, int Nz, float cxp, float cyp, float czp, float sigma,
                                 float amp) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int N = Nx * Ny * Nz;
    if (i >= N) return;
    const int x = i % Nx, y = (i / Nx) % Ny, z = i / (Nx * Ny);
    const float X = (x + 0.5f) / Nx, Y = (y + 0.5f) / Ny, Z = (z + 0.5f) / Nz;
    const float dx = X - cxp, dy = Y - cyp, dz = Z - czp;
    const float r2 = dx * dx + dy * dy + dz * dz;
    rho[i] = 1.0f + amp * __expf(-r2 / (2.f * sigma * sigma));
}

__global__ void rho_slab_kernel(float* rho, int Nx, int Ny, int Nz, int axis, float amp, float center, float width) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int N = Nx * Ny * Nz;
    if (i >= N) return;
    const int x = i % Nx, y = (i / Nx) % Ny, z = i / (Nx * Ny);
    const float s = (axis == 0) ? (x + 0.5f) / Nx : (axis == 1) ? (y + 0.5f) / Ny : (z + 0.5f) / Nz;
    const float val = (fabsf(s - center) < 0.5f * width) ? amp : 0.f;
    rho[i] = 1.0f + val;
}

inline int grid_for(int64_t n, int threads = 256) {
    const int64_t b = (n + threads - 1) / threads;
    const int64_t cap = (int64_t)num_sms() * 16;
    return (int)(b < 1 ? 1 : (b > cap ? cap : b));
}

}  // namespace

cudaError_t launch_aa_reinit(void* f, int storage, float rho0, int64_t N, const float* rho, const float* ux,
                             const float* uy, const float* uz, float* ro, float* uo, float* vo, float* wo,
                             int form, cudaStream_t s) {
    const int g = grid_for(N);
    switch (storage) {
        case 0: aa_reinit<StoreF32><<<g, 256, 0, s>>>((float*)f, rho0, N, rho, ux, uy, uz, ro, uo, vo, wo, form); break;
        case 1: aa_reinit<StoreF16><<<g, 256, 0, s>>>((__half*)f, rho0, N, rho, ux, uy, uz, ro, uo, vo, wo, form); break;
        case 2: aa_reinit<StoreBF16><<<g, 256, 0, s>>>((__nv_bfloat16*)f, rho0, N, rho, ux, uy, uz, ro, uo, vo, wo, form); break;
        case 3: aa_reinit_f64<<<g, 256, 0, s>>>((double*)f, N, rho, ux, uy, uz, ro, uo, vo, wo); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_home_reinit(void* m, void* mn, int storage, float rho0, int64_t N, const float* rho,
                               const float* ux, const float* uy, const float* uz, cudaStream_t s) {
    const int g = grid_for(N);
    switch (storage) {
        case 0: home_reinit<float><<<g, 256, 0, s>>>((float*)m, (float*)mn, rho0, N, rho, ux, uy, uz); break;
        case 1: home_reinit<__half><<<g, 256, 0, s>>>((__half*)m, (__half*)mn, rho0, N, rho, ux, uy, uz); break;
        case 2: home_reinit<__nv_bfloat16><<<g, 256, 0, s>>>((__nv_bfloat16*)m, (__nv_bfloat16*)mn, rho0, N, rho, ux, uy, uz); break;
        case 3: home_reinit<double><<<g, 256, 0, s>>>((double*)m, (double*)mn, rho0, N, rho, ux, uy, uz); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_build_flags(const uint8_t* mask, const uint8_t* band, uint8_t* flags, uint32_t* links, int nx,
                               int ny, int nz, int duct, cudaStream_t s) {
    const int64_t N = (int64_t)nx * ny * nz;
    build_flags<<<grid_for(N), 256, 0, s>>>(mask, band, flags, links, nx, ny, nz, duct);
    return cudaGetLastError();
}

cudaError_t launch_band(const uint8_t* mask, int32_t* dist, uint8_t* band, int nx, int ny, int nz, int d0,
                        unsigned long long* count, cudaStream_t s) {
    const int64_t N = (int64_t)nx * ny * nz;
    const int g = grid_for(N);
    const int max_dist = d0 > 1 ? d0 : 1;   // sim_runner.hpp:221
    band_init<<<g, 256, 0, s>>>(mask, dist, N);
    for (int k = 1; k <= max_dist; ++k) band_grow<<<g, 256, 0, s>>>(dist, nx, ny, nz, k);
    cudaMemsetAsync(count, 0, sizeof(unsigned long long), s);
    band_final<<<g, 256, 0, s>>>(mask, dist, band, N, d0, count);
    return cudaGetLastError();
}

cudaError_t launch_finalize_stats(const double* partials, int nblocks, double* out, cudaStream_t s) {
    finalize_stats<<<1, 256, 0, s>>>(partials, nblocks, out);
    return cudaGetLastError();
}

}  // namespace lbm

// ---- the reference's extern "C" helpers --------------------------------------
extern "C" {

void reinit_equilibrium_from_macro(const float* d_rho, const float* d_ux, const float* d_uy, const float* d_uz,
                                   float* d_f, int N) {
    if (N <= 0) return;
    lbm::reinit_eq_kernel<<<(N + 255) / 256, 256>>>(d_rho, d_ux, d_uy, d_uz, d_f, N);
}

void launch_speed(const float* u, const float* v, const float* w, float* out, int N) {
    if (N <= 0) return;
    lbm::speed_kernel<<<(N + 255) / 256, 256>>>(u, v, w, out, N);
}

void make_rho_gauss(float* d_rho, int Nx, int Ny, int Nz, float cx, float cy, float cz, float sigma, float amp) {
    const int N = Nx * Ny * Nz;
    if (N <= 0) return;
    lbm::rho_gauss_kernel<<<(N + 255) / 256, 256>>>(d_rho, Nx, Ny, Nz, cx, cy, cz, sigma, amp);
}

void make_rho_slab(float* d_rho, int Nx, int Ny, int Nz, int axis, float amp, float center, float width) {
    const int N = Nx * Ny * Nz;
    if (N <= 0) return;
    lbm::rho_slab_kernel<<<(N + 255) / 256, 256>>>(d_rho, Nx, Ny, Nz, axis, amp, center, width);
}

}  // extern "C"
