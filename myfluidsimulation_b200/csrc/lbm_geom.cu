// GPU voxelizer, bit-exact with src/geom/voxelize.cpp:14-243.
//
// The reference runs on one host thread: a separating-axis triangle/box test
// over each triangle's candidate cells, then a queue BFS that marks the
// exterior from the six domain faces.  Here:
//   * one warp per triangle, its lanes striding over the candidate cells;
//     every float operation is spelled with an explicit rounding intrinsic
//     (__fadd_rn, __fmul_rn, ...), so nvcc cannot contract it into an FMA and
//     each result equals the reference's uncontracted x86-64 float result;
//   * the exterior flood fill is a reachability fixed point, computed by
//     rounds of six directional line sweeps (+-x, +-y, +-z) until a round
//     changes nothing; the reachable set is unique, so the mask is identical
//     to the BFS result whatever the visiting order;
//   * the optional refine^3 coverage downsample (voxelize.cpp:187-226) is one
//     thread per coarse cell.
#include "lbm_common.cuh"
#include "lbm_internal.h"

namespace lbm {
namespace {

__device__ __forceinline__ float fmin_ref(float a, float b) { return (b < a) ? b : a; }   // std::min
__device__ __forceinline__ float fmax_ref(float a, float b) { return (a < b) ? b : a; }   // std::max

// a*b - c*d with both products rounded, as GLM's cross evaluates each term
__device__ __forceinline__ float dif2(float a, float b, float c, float d) {
    return __fsub_rn(__fmul_rn(a, b), __fmul_rn(c, d));
}
// ((a0*b0 + a1*b1) + a2*b2) left to right
__device__ __forceinline__ float dot3(float a0, float a1, float a2, float b0, float b1, float b2) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a0, b0), __fmul_rn(a1, b1)), __fmul_rn(a2, b2));
}

// voxelize.cpp:23-81
__device__ bool tri_box(const float c[3], const float h[3], const float v0[3], const float v1[3], const float v2[3]) {
    float t0[3], t1[3], t2[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        t0[k] = __fsub_rn(v0[k], c[k]);
        t1[k] = __fsub_rn(v1[k], c[k]);
        t2[k] = __fsub_rn(v2[k], c[k]);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float mn = fmin_ref(fmin_ref(t0[k], t1[k]), t2[k]);
        const float mx = fmax_ref(fmax_ref(t0[k], t1[k]), t2[k]);
        if (mx < -h[k] || mn > h[k]) return false;
    }
    float e[3][3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        e[0][k] = __fsub_rn(t1[k], t0[k]);
        e[1][k] = __fsub_rn(t2[k], t1[k]);
        e[2][k] = __fsub_rn(t0[k], t2[k]);
    }
    // n = cross(e0, e1): (a.y*b.z - b.y*a.z, a.z*b.x - b.z*a.x, a.x*b.y - b.x*a.y)
    const float n0 = dif2(e[0][1], e[1][2], e[1][1], e[0][2]);
    const float n1 = dif2(e[0][2], e[1][0], e[1][2], e[0][0]);
    const float n2 = dif2(e[0][0], e[1][1], e[1][0], e[0][1]);
    const float r = dot3(h[0], h[1], h[2], fabsf(n0), fabsf(n1), fabsf(n2));
    const float s = fabsf(dot3(n0, n1, n2, t0[0], t0[1], t0[2]));
    if (s > r) return false;
#pragma unroll
    for (int ei = 0; ei < 3; ++ei) {
        const float* ed = e[ei];
        if (__fadd_rn(__fadd_rn(fabsf(ed[0]), fabsf(ed[1])), fabsf(ed[2])) < 1e-12f) continue;
#pragma unroll
        for (int ai = 0; ai < 3; ++ai) {
            const float ax[3] = {ai == 0 ? 1.f : 0.f, ai == 1 ? 1.f : 0.f, ai == 2 ? 1.f : 0.f};
            const float L0 = dif2(ed[1], ax[2], ax[1], ed[2]);
            const float L1 = dif2(ed[2], ax[0], ax[2], ed[0]);
            const float L2 = dif2(ed[0], ax[1], ax[0], ed[1]);
            const float l2 = dot3(L0, L1, L2, L0, L1, L2);
            if (l2 < 1e-20f) continue;
            const float p0 = dot3(L0, L1, L2, t0[0], t0[1], t0[2]);
            const float p1 = dot3(L0, L1, L2, t1[0], t1[1], t1[2]);
            const float p2 = dot3(L0, L1, L2, t2[0], t2[1], t2[2]);
            const float minp = fmin_ref(p0, fmin_ref(p1, p2));
            const float maxp = fmax_ref(p0, fmax_ref(p1, p2));
            const float rp = dot3(h[0], h[1], h[2], fabsf(L0), fabsf(L1), fabsf(L2));
            if (maxp < -rp || minp > rp) return false;
        }
    }
    return true;
}

// voxelize.cpp:83-113: vertex' = s*vertex + trans, per component
__global__ void fit_kernel(const float* __restrict__ in, float* __restrict__ out, int64_t n, float s, float t0,
                           float t1, float t2) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float tr = (i % 3 == 0) ? t0 : ((i % 3 == 1) ? t1 : t2);
        out[i] = __fadd_rn(__fmul_rn(s, in[i]), tr);
    }
}

// voxelize.cpp:115-149: one warp per triangle
__global__ void surface_kernel(const float* __restrict__ vt, int64_t ntri, int nx, int ny, int nz,
                               uint8_t* __restrict__ surf) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    const float h[3] = {__fdiv_rn(0.5f, (float)nx), __fdiv_rn(0.5f, (float)ny), __fdiv_rn(0.5f, (float)nz)};
    const float eps = 1e-6f;
    for (int64_t t = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < ntri; t += warps) {
        const float* p = vt + t * 9;
        const float v0[3] = {p[0], p[1], p[2]}, v1[3] = {p[3], p[4], p[5]}, v2[3] = {p[6], p[7], p[8]};
        int lo[3], hi[3];
        const int n[3] = {nx, ny, nz};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const float mn = __fsub_rn(fmin_ref(v0[k], fmin_ref(v1[k], v2[k])), eps);
            const float mx = __fadd_rn(fmax_ref(v0[k], fmax_ref(v1[k], v2[k])), eps);
            lo[k] = max(0, (int)floorf(__fmul_rn(mn, (float)n[k])));
            hi[k] = min(n[k] - 1, (int)floorf(__fmul_rn(mx, (float)n[k])));
        }
        if (hi[0] < lo[0] || hi[1] < lo[1] || hi[2] < lo[2]) continue;
        const int64_t sx = hi[0] - lo[0] + 1, sy = hi[1] - lo[1] + 1, sz = hi[2] - lo[2] + 1;
        const int64_t cnt = sx * sy * sz;
        for (int64_t c = lane; c < cnt; c += 32) {
            const int x = lo[0] + (int)(c % sx);
            const int y = lo[1] + (int)((c / sx) % sy);
            const int z = lo[2] + (int)(c / (sx * sy));
            const float cc[3] = {__fdiv_rn(__fadd_rn((float)x, 0.5f), (float)nx),
                                 __fdiv_rn(__fadd_rn((float)y, 0.5f), (float)ny),
                                 __fdiv_rn(__fadd_rn((float)z, 0.5f), (float)nz)};
            if (tri_box(cc, h, v0, v1, v2)) surf[((int64_t)z * ny + y) * nx + x] = 1;
        }
    }
}

// seeds: non-surface cells on the six faces (voxelize.cpp:160-163)
__global__ void seed_kernel(const uint8_t* __restrict__ surf, uint8_t* __restrict__ vis, int nx, int ny, int nz) {
    const int64_t N = (int64_t)nx * ny * nz;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % nx);
        const int64_t row = i / nx;
        const int y = (int)(row % ny), z = (int)(row / ny);
        const bool face = x == 0 || x == nx - 1 || y == 0 || y == ny - 1 || z == 0 || z == nz - 1;
        vis[i] = (face && !surf[i]) ? 1 : 0;
    }
}

// One directional sweep: each thread walks one line of the grid along `axis`
// in direction `dir`, carrying "reached" across non-surface cells.
__global__ void sweep_kernel(const uint8_t* __restrict__ surf, uint8_t* __restrict__ vis, int nx, int ny, int nz,
                             int axis, int dir, int* changed) {
    const int n[3] = {nx, ny, nz};
    const int64_t stride[3] = {1, nx, (int64_t)nx * ny};
    const int a1 = axis == 0 ? 1 : 0, a2 = axis == 2 ? 1 : 2;
    const int64_t lines = (int64_t)n[a1] * n[a2];
    int any = 0;
    for (int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; l < lines; l += (int64_t)gridDim.x * blockDim.x) {
        const int i1 = (int)(l % n[a1]), i2 = (int)(l / n[a1]);
        const int64_t base = i1 * stride[a1] + i2 * stride[a2];
        bool carry = false;
        for (int s = 0; s < n[axis]; ++s) {
            const int c = dir > 0 ? s : n[axis] - 1 - s;
            const int64_t id = base + c * stride[axis];
            if (surf[id]) { carry = false; continue; }
            if (vis[id]) { carry = true; continue; }
            if (carry) { vis[id] = 1; any = 1; }
        }
    }
    if (any) atomicOr(changed, 1);
}

__global__ void solid_kernel(const uint8_t* __restrict__ surf, const uint8_t* __restrict__ vis,
                             uint8_t* __restrict__ out, int64_t N) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (surf[i] || !vis[i]) ? 1 : 0;
}

// voxelize.cpp:187-226
__global__ void downsample_kernel(const uint8_t* __restrict__ fine, int r, int nx, int ny, int nz, float thr,
                                  uint8_t* __restrict__ out) {
    const int64_t N = (int64_t)nx * ny * nz;
    const int64_t fx = (int64_t)nx * r, fy = (int64_t)ny * r;
    const int r3 = r * r * r;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % nx);
        const int64_t row = i / nx;
        const int y = (int)(row % ny), z = (int)(row / ny);
        int cnt = 0;
        for (int dz = 0; dz < r; ++dz)
            for (int dy = 0; dy < r; ++dy) {
                const int64_t b = ((int64_t)z * r + dz) * fy * fx + ((int64_t)y * r + dy) * fx + (int64_t)x * r;
                for (int dx = 0; dx < r; ++dx) cnt += fine[b + dx];
            }
        const float cov = __fdiv_rn((float)cnt, (float)r3);
        out[i] = (cov > 0.0f && cov >= thr) ? 1 : 0;
    }
}

}  // namespace

cudaError_t launch_voxelize(const float* d_tris, int64_t ntri, const float* bb, int nx, int ny, int nz, float scale,
                            const float* translate, int refine, float thr, uint8_t* d_mask, cudaStream_t s) {
    if (refine < 1) refine = 1;
    // compute_fit_transform (voxelize.cpp:83-91), float, uncontracted
    const float bs[3] = {bb[3] - bb[0], bb[4] - bb[1], bb[5] - bb[2]};
    const float maxDim = (bs[0] < ((bs[1] < bs[2]) ? bs[2] : bs[1])) ? ((bs[1] < bs[2]) ? bs[2] : bs[1]) : bs[0];
    volatile float sv = (maxDim > 0.0f) ? (scale / maxDim) : 1.0f;
    const float sf = sv;
    float tr[3];
    for (int k = 0; k < 3; ++k) {
        volatile float center = 0.5f * (bb[k] + bb[3 + k]);
        volatile float prod = sf * center;
        tr[k] = translate[k] - prod;
    }
    const int fx = nx * refine, fy = ny * refine, fz = nz * refine;
    const int64_t NF = (int64_t)fx * fy * fz;
    float* vt = nullptr;
    uint8_t *surf = nullptr, *vis = nullptr, *fine = nullptr;
    int* changed = nullptr;
    cudaError_t e = cudaSuccess;
#define VX_CK(x) do { e = (x); if (e != cudaSuccess) goto done; } while (0)
    VX_CK(cudaMallocAsync(&vt, sizeof(float) * 9 * (size_t)(ntri > 0 ? ntri : 1), s));
    VX_CK(cudaMallocAsync(&surf, (size_t)NF, s));
    VX_CK(cudaMallocAsync(&vis, (size_t)NF, s));
    VX_CK(cudaMallocAsync(&changed, sizeof(int), s));
    if (refine > 1) VX_CK(cudaMallocAsync(&fine, (size_t)NF, s));
    VX_CK(cudaMemsetAsync(surf, 0, (size_t)NF, s));
    if (ntri > 0) {
        fit_kernel<<<num_sms() * 4, 256, 0, s>>>(d_tris, vt, ntri * 9, sf, tr[0], tr[1], tr[2]);
        const int64_t blocks = (ntri + 7) / 8;   // 8 warps per block
        surface_kernel<<<(int)(blocks < 65535 ? blocks : 65535), 256, 0, s>>>(vt, ntri, fx, fy, fz, surf);
        VX_CK(cudaGetLastError());
    }
    seed_kernel<<<num_sms() * 8, 256, 0, s>>>(surf, vis, fx, fy, fz);
    VX_CK(cudaGetLastError());
    for (int round = 0; round < 1000000; ++round) {
        VX_CK(cudaMemsetAsync(changed, 0, sizeof(int), s));
        for (int axis = 0; axis < 3; ++axis)
            for (int dir = -1; dir <= 1; dir += 2) {
                const int64_t lines = (axis == 0) ? (int64_t)fy * fz : (axis == 1 ? (int64_t)fx * fz : (int64_t)fx * fy);
                const int64_t b = (lines + 127) / 128;
                sweep_kernel<<<(int)(b < 65535 ? b : 65535), 128, 0, s>>>(surf, vis, fx, fy, fz, axis, dir, changed);
            }
        VX_CK(cudaGetLastError());
        int h = 0;
        VX_CK(cudaMemcpyAsync(&h, changed, sizeof(int), cudaMemcpyDeviceToHost, s));
        VX_CK(cudaStreamSynchronize(s));
        if (!h) break;
    }
    if (refine == 1) {
        solid_kernel<<<num_sms() * 8, 256, 0, s>>>(surf, vis, d_mask, NF);
    } else {
        solid_kernel<<<num_sms() * 8, 256, 0, s>>>(surf, vis, fine, NF);
        const float t = fmaxf(0.0f, fminf(1.0f, thr));
        downsample_kernel<<<num_sms() * 8, 256, 0, s>>>(fine, refine, nx, ny, nz, t, d_mask);
    }
    VX_CK(cudaGetLastError());
done:
#undef VX_CK
    if (vt) cudaFreeAsync(vt, s);
    if (surf) cudaFreeAsync(surf, s);
    if (vis) cudaFreeAsync(vis, s);
    if (fine) cudaFreeAsync(fine, s);
    if (changed) cudaFreeAsync(changed, s);
    return e;
}

}  // namespace lbm
