// Headless volume ray-march of a scalar field into a device RGBA buffer.
//
// The reference draws its 3-D view with a GLSL fragment shader over a
// full-screen quad (src/render/Vis3D.cpp:30-78), fed by glTexSubImage3D of the
// field copied to the host (Vis3D.cpp:118-126).  Here each CUDA thread is one
// fragment of that shader:
//   ndc = (uv*2-1, 0, 1); w = invPV ndc / w.w; dir = normalize(w.xyz - cam);
//   slab test against [0,1]^3; march from max(tNear,0) in steps of uStep,
//   front-to-back, until t >= tFar or alpha >= 0.95;
//   sample: s = trilinear(field) * uScale; colour = 4-segment map of
//   0.5+0.5 clamp(s,-1,1); alpha = smoothstep(uThresh, 1, |s|), 0 below uThresh;
//   frag = (acc.rgb, 1); a discarded fragment keeps the clear colour
//   (0.02, 0.02, 0.03, 1) of main_compare.cpp:988.
// Pixel (x, y) has uv = ((x+0.5)/W, (y+0.5)/H), row 0 at the bottom as in GL.
//
// Two samplers:
//   LBM_FILTER_EXACT: GL_LINEAR / CLAMP_TO_EDGE trilinear in FP32 from global
//     memory, every operation rounded as written (no FMA contraction), so the
//     image equals the C oracle's bit for bit;
//   LBM_FILTER_TEXTURE: the texture unit's trilinear filter on a 3-D CUDA
//     array (8-bit fractional weights, as GL_LINEAR on the same hardware).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <string>
#include <utility>
#include <vector>

#include "lbm_capi.h"

namespace lbm {
void set_error(const std::string& msg);
namespace render {

struct View {
    float m[16];   // inverse(P V), column-major: m[4*col + row]
    float cam[3];
    float step, scale, thresh;
    int width, height;
};

// rounded-as-written FP32 arithmetic (no contraction into FMA)
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float dvd(float a, float b) { return __fdiv_rn(a, b); }
// GLSL: min(x, y) = y < x ? y : x; max(x, y) = x < y ? y : x
__device__ __forceinline__ float gmin(float x, float y) { return y < x ? y : x; }
__device__ __forceinline__ float gmax(float x, float y) { return x < y ? y : x; }
__device__ __forceinline__ float gclamp(float x, float lo, float hi) { return gmin(gmax(x, lo), hi); }
// mix(x, y, a) = x (1 - a) + y a
__device__ __forceinline__ float mix(float x, float y, float a) { return add(mul(x, sub(1.0f, a)), mul(y, a)); }

__device__ __forceinline__ void colormap(float t, float c[3]) {
    t = gclamp(t, 0.0f, 1.0f);
    float a0[3], a1[3], w;
    if (t < 0.25f) {
        a0[0] = 0.02f; a0[1] = 0.02f; a0[2] = 0.2f; a1[0] = 0.0f; a1[1] = 0.7f; a1[2] = 1.0f; w = mul(t, 4.0f);
    } else if (t < 0.50f) {
        a0[0] = 0.0f; a0[1] = 0.7f; a0[2] = 1.0f; a1[0] = 0.0f; a1[1] = 1.0f; a1[2] = 0.3f; w = mul(sub(t, 0.25f), 4.0f);
    } else if (t < 0.75f) {
        a0[0] = 0.0f; a0[1] = 1.0f; a0[2] = 0.3f; a1[0] = 1.0f; a1[1] = 0.9f; a1[2] = 0.0f; w = mul(sub(t, 0.50f), 4.0f);
    } else {
        a0[0] = 1.0f; a0[1] = 0.9f; a0[2] = 0.0f; a1[0] = 1.0f; a1[1] = 0.1f; a1[2] = 0.0f; w = mul(sub(t, 0.75f), 4.0f);
    }
    for (int k = 0; k < 3; ++k) c[k] = mix(a0[k], a1[k], w);
}

// GL_LINEAR, CLAMP_TO_EDGE, normalized coordinates: texel i is centred at (i + 0.5) / n
struct Exact {
    const float* f;
    int nx, ny, nz;
    __device__ __forceinline__ float operator()(float px, float py, float pz) const {
        int i0[3], i1[3];
        float fr[3];
        const float p[3] = {px, py, pz};
        const int n[3] = {nx, ny, nz};
        for (int k = 0; k < 3; ++k) {
            const float u = sub(mul(p[k], (float)n[k]), 0.5f);
            const float fl = floorf(u);
            fr[k] = sub(u, fl);
            const int i = (int)fl;
            i0[k] = i < 0 ? 0 : (i > n[k] - 1 ? n[k] - 1 : i);
            i1[k] = i + 1 < 0 ? 0 : (i + 1 > n[k] - 1 ? n[k] - 1 : i + 1);
        }
        auto T = [&](int x, int y, int z) { return __ldg(f + ((size_t)z * ny + y) * nx + x); };
        const float c00 = mix(T(i0[0], i0[1], i0[2]), T(i1[0], i0[1], i0[2]), fr[0]);
        const float c10 = mix(T(i0[0], i1[1], i0[2]), T(i1[0], i1[1], i0[2]), fr[0]);
        const float c01 = mix(T(i0[0], i0[1], i1[2]), T(i1[0], i0[1], i1[2]), fr[0]);
        const float c11 = mix(T(i0[0], i1[1], i1[2]), T(i1[0], i1[1], i1[2]), fr[0]);
        const float c0 = mix(c00, c10, fr[1]);
        const float c1 = mix(c01, c11, fr[1]);
        return mix(c0, c1, fr[2]);
    }
};

struct Texture {
    cudaTextureObject_t tex;
    __device__ __forceinline__ float operator()(float px, float py, float pz) const {
        return tex3D<float>(tex, px, py, pz);
    }
};

template <class S>
__global__ void __launch_bounds__(256) raymarch(View v, S sample, float4* __restrict__ out) {
    const int x = blockIdx.x * 16 + (threadIdx.x & 15);
    const int y = blockIdx.y * 16 + (threadIdx.x >> 4);
    if (x >= v.width || y >= v.height) return;
    const float ux = dvd(add((float)x, 0.5f), (float)v.width), uy = dvd(add((float)y, 0.5f), (float)v.height);
    const float ndc[4] = {sub(mul(ux, 2.0f), 1.0f), sub(mul(uy, 2.0f), 1.0f), 0.0f, 1.0f};
    float wp[4];
    for (int r = 0; r < 4; ++r)
        wp[r] = add(add(add(mul(v.m[r], ndc[0]), mul(v.m[4 + r], ndc[1])), mul(v.m[8 + r], ndc[2])),
                    mul(v.m[12 + r], ndc[3]));
    float d[3];
    for (int k = 0; k < 3; ++k) d[k] = sub(dvd(wp[k], wp[3]), v.cam[k]);
    const float len = sqrtf(add(add(mul(d[0], d[0]), mul(d[1], d[1])), mul(d[2], d[2])));
    for (int k = 0; k < 3; ++k) d[k] = dvd(d[k], len);
    float t0[3], t1[3];
    for (int k = 0; k < 3; ++k) {
        t0[k] = dvd(sub(0.0f, v.cam[k]), d[k]);
        t1[k] = dvd(sub(1.0f, v.cam[k]), d[k]);
    }
    float tn = gmax(gmax(gmin(t0[0], t1[0]), gmin(t0[1], t1[1])), gmin(t0[2], t1[2]));
    const float tf = gmin(gmin(gmax(t0[0], t1[0]), gmax(t0[1], t1[1])), gmax(t0[2], t1[2]));
    const size_t o = (size_t)y * v.width + x;
    if (tf < 0.0f || tn > tf) {
        out[o] = make_float4(0.02f, 0.02f, 0.03f, 1.0f);
        return;
    }
    tn = gmax(tn, 0.0f);
    float pos[3];
    for (int k = 0; k < 3; ++k) pos[k] = add(v.cam[k], mul(d[k], tn));
    float t = tn;
    float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    const float range = sub(1.0f, v.thresh);
    while (t < tf && acc[3] < 0.95f) {
        const float sc = mul(sample(pos[0], pos[1], pos[2]), v.scale);
        const float tmag = gclamp(fabsf(sc), 0.0f, 1.0f);
        if (!(tmag < v.thresh)) {
            const float tc = add(0.5f, mul(0.5f, gclamp(sc, -1.0f, 1.0f)));
            const float h = gclamp(dvd(sub(tmag, v.thresh), range), 0.0f, 1.0f);
            const float a = mul(mul(h, h), sub(3.0f, mul(2.0f, h)));
            float col[3];
            colormap(tc, col);
            const float rem = sub(1.0f, acc[3]);
            for (int k = 0; k < 3; ++k) acc[k] = add(acc[k], mul(col[k], rem));
            acc[3] = add(acc[3], mul(a, sub(1.0f, acc[3])));
        }
        for (int k = 0; k < 3; ++k) pos[k] = add(pos[k], mul(d[k], v.step));
        t = add(t, v.step);
    }
    out[o] = make_float4(acc[0], acc[1], acc[2], 1.0f);
}

__global__ void diff_kernel(const float* a, const float* b, float* out, int N) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) out[i] = a[i] - b[i];
}
__global__ void shift_kernel(const float* a, float bias, float* out, int N) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) out[i] = a[i] + bias;
}

}  // namespace render
}  // namespace lbm

using namespace lbm::render;

struct lbm_renderer {
    int nx = 0, ny = 0, nz = 0;
    cudaArray_t arr = nullptr;
    cudaTextureObject_t tex = 0;
};

extern "C" {

int lbm_renderer_create(int32_t nx, int32_t ny, int32_t nz, lbm_renderer** out) {
    if (!out || nx <= 0 || ny <= 0 || nz <= 0) { lbm::set_error("lbm_renderer_create: bad argument"); return LBM_ERR_INVALID; }
    auto* r = new lbm_renderer();
    r->nx = nx; r->ny = ny; r->nz = nz;
    *out = r;
    return LBM_OK;
}

int lbm_renderer_destroy(lbm_renderer* r) {
    if (!r) return LBM_OK;
    if (r->tex) cudaDestroyTextureObject(r->tex);
    if (r->arr) cudaFreeArray(r->arr);
    delete r;
    return LBM_OK;
}

int lbm_render_volume(lbm_renderer* r, const float* d_field, const lbm_render_params* p, float* d_rgba,
                      void* stream) {
    if (!r || !d_field || !p || !d_rgba || p->width <= 0 || p->height <= 0 || !(p->step > 0.0f)) {
        lbm::set_error("lbm_render_volume: bad argument");
        return LBM_ERR_INVALID;
    }
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    View v;
    for (int k = 0; k < 16; ++k) v.m[k] = p->inv_pv[k];
    for (int k = 0; k < 3; ++k) v.cam[k] = p->cam_pos[k];
    v.step = p->step; v.scale = p->scale; v.thresh = p->threshold;
    v.width = p->width; v.height = p->height;
    const dim3 grid((unsigned)((p->width + 15) / 16), (unsigned)((p->height + 15) / 16));
    float4* out = reinterpret_cast<float4*>(d_rgba);
    if (p->filter == LBM_FILTER_TEXTURE) {
        if (!r->arr) {
            cudaChannelFormatDesc ch = cudaCreateChannelDesc<float>();
            if (cudaMalloc3DArray(&r->arr, &ch, make_cudaExtent(r->nx, r->ny, r->nz)) != cudaSuccess) {
                lbm::set_error("lbm_render_volume: 3-D array allocation failed");
                return LBM_ERR_ALLOC;
            }
            cudaResourceDesc rd{};
            rd.resType = cudaResourceTypeArray;
            rd.res.array.array = r->arr;
            cudaTextureDesc td{};
            td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeClamp;
            td.filterMode = cudaFilterModeLinear;
            td.readMode = cudaReadModeElementType;
            td.normalizedCoords = 1;
            if (cudaCreateTextureObject(&r->tex, &rd, &td, nullptr) != cudaSuccess) {
                lbm::set_error("lbm_render_volume: texture creation failed");
                return LBM_ERR_CUDA;
            }
        }
        // the field into the array (the reference's glTexSubImage3D, without the host round trip)
        cudaMemcpy3DParms cp{};
        cp.srcPtr = make_cudaPitchedPtr(const_cast<float*>(d_field), sizeof(float) * r->nx, r->nx, r->ny);
        cp.dstArray = r->arr;
        cp.extent = make_cudaExtent(r->nx, r->ny, r->nz);
        cp.kind = cudaMemcpyDeviceToDevice;
        if (cudaMemcpy3DAsync(&cp, st) != cudaSuccess) {
            lbm::set_error("lbm_render_volume: field copy into the 3-D array failed");
            return LBM_ERR_CUDA;
        }
        raymarch<Texture><<<grid, 256, 0, st>>>(v, Texture{r->tex}, out);
    } else if (p->filter == LBM_FILTER_EXACT) {
        raymarch<Exact><<<grid, 256, 0, st>>>(v, Exact{d_field, r->nx, r->ny, r->nz}, out);
    } else {
        lbm::set_error("lbm_render_volume: unknown filter");
        return LBM_ERR_INVALID;
    }
    if (cudaGetLastError() != cudaSuccess) { lbm::set_error("lbm_render_volume: launch failed"); return LBM_ERR_CUDA; }
    return LBM_OK;
}

// Orbit camera of main_compare.cpp:51-60,972-981: eye = target + radius
// (cos p cos y, sin p, cos p sin y); P = perspective(45 deg, w/h, 0.01, 10),
// V = lookAt(eye, target, +y) (right-handed, clip z in [-1, 1]); inverse in FP64.
int lbm_render_orbit_camera(float yaw, float pitch, float radius, const float* target, int32_t width,
                            int32_t height, float* inv_pv, float* cam_pos) {
    if (!target || !inv_pv || !cam_pos || width <= 0 || height <= 0) {
        lbm::set_error("lbm_render_orbit_camera: bad argument");
        return LBM_ERR_INVALID;
    }
    const double cp = std::cos((double)pitch), sp = std::sin((double)pitch);
    const double cy = std::cos((double)yaw), sy = std::sin((double)yaw);
    const double eye[3] = {target[0] + radius * cp * cy, target[1] + radius * sp, target[2] + radius * cp * sy};
    double f[3] = {target[0] - eye[0], target[1] - eye[1], target[2] - eye[2]};
    auto norm = [](double* a) {
        const double l = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
        for (int k = 0; k < 3; ++k) a[k] /= l;
    };
    auto cross = [](const double* a, const double* b, double* c) {
        c[0] = a[1] * b[2] - a[2] * b[1];
        c[1] = a[2] * b[0] - a[0] * b[2];
        c[2] = a[0] * b[1] - a[1] * b[0];
    };
    norm(f);
    const double up[3] = {0, 1, 0};
    double s[3], u[3];
    cross(f, up, s);
    norm(s);
    cross(s, f, u);
    double V[16] = {0}, P[16] = {0}, M[16], I[16];   // column-major
    V[0] = s[0]; V[4] = s[1]; V[8] = s[2];
    V[1] = u[0]; V[5] = u[1]; V[9] = u[2];
    V[2] = -f[0]; V[6] = -f[1]; V[10] = -f[2];
    V[12] = -(s[0] * eye[0] + s[1] * eye[1] + s[2] * eye[2]);
    V[13] = -(u[0] * eye[0] + u[1] * eye[1] + u[2] * eye[2]);
    V[14] = f[0] * eye[0] + f[1] * eye[1] + f[2] * eye[2];
    V[15] = 1.0;
    const double th = std::tan(0.5 * 45.0 * 3.14159265358979323846 / 180.0), zn = 0.01, zf = 10.0;
    const double aspect = (double)width / (double)height;
    P[0] = 1.0 / (aspect * th);
    P[5] = 1.0 / th;
    P[10] = -(zf + zn) / (zf - zn);
    P[11] = -1.0;
    P[14] = -(2.0 * zf * zn) / (zf - zn);
    for (int c = 0; c < 4; ++c)
        for (int r = 0; r < 4; ++r) {
            double a = 0;
            for (int k = 0; k < 4; ++k) a += P[4 * k + r] * V[4 * c + k];
            M[4 * c + r] = a;
        }
    // Gauss-Jordan inverse with partial pivoting (row-major view of M^T is fine: invert the 4x4 as is)
    double A[4][8];
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            A[r][c] = M[4 * c + r];
            A[r][4 + c] = r == c ? 1.0 : 0.0;
        }
    for (int c = 0; c < 4; ++c) {
        int piv = c;
        for (int r = c + 1; r < 4; ++r)
            if (std::fabs(A[r][c]) > std::fabs(A[piv][c])) piv = r;
        if (A[piv][c] == 0.0) { lbm::set_error("lbm_render_orbit_camera: singular view"); return LBM_ERR_INVALID; }
        for (int k = 0; k < 8; ++k) std::swap(A[c][k], A[piv][k]);
        const double d = A[c][c];
        for (int k = 0; k < 8; ++k) A[c][k] /= d;
        for (int r = 0; r < 4; ++r)
            if (r != c) {
                const double m = A[r][c];
                for (int k = 0; k < 8; ++k) A[r][k] -= m * A[c][k];
            }
    }
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) I[4 * c + r] = A[r][4 + c];
    for (int k = 0; k < 16; ++k) inv_pv[k] = (float)I[k];
    for (int k = 0; k < 3; ++k) cam_pos[k] = (float)eye[k];
    return LBM_OK;
}

// Binary PPM (P6) of a host RGBA float image, top row first (the GL image's
// last row), channels clamped to [0, 1] and rounded to 8 bits.
int lbm_write_ppm(const char* path, const float* rgba, int32_t width, int32_t height) {
    if (!path || !rgba || width <= 0 || height <= 0) { lbm::set_error("lbm_write_ppm: bad argument"); return LBM_ERR_INVALID; }
    FILE* f = std::fopen(path, "wb");
    if (!f) { lbm::set_error(std::string("cannot open ") + path); return LBM_ERR_IO; }
    std::fprintf(f, "P6\n%d %d\n255\n", width, height);
    std::vector<unsigned char> row((size_t)width * 3);
    bool ok = true;
    for (int y = height - 1; y >= 0 && ok; --y) {
        for (int x = 0; x < width; ++x)
            for (int k = 0; k < 3; ++k) {
                float c = rgba[((size_t)y * width + x) * 4 + k];
                c = c < 0.f ? 0.f : (c > 1.f ? 1.f : c);
                row[(size_t)x * 3 + k] = (unsigned char)std::lround(c * 255.0f);
            }
        ok = std::fwrite(row.data(), 1, row.size(), f) == row.size();
    }
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) { lbm::set_error(std::string("cannot write ") + path); return LBM_ERR_IO; }
    return LBM_OK;
}

// The viewer's other field helpers (src/fields/field_ops.cu:20-41).
void launch_diff(const float* a, const float* b, float* out, int N) {
    if (N > 0) lbm::render::diff_kernel<<<(N + 255) / 256, 256>>>(a, b, out, N);
}
void launch_shift(const float* a, float bias, float* out, int N) {
    if (N > 0) lbm::render::shift_kernel<<<(N + 255) / 256, 256>>>(a, bias, out, N);
}

}  // extern "C"
