/*
 * Oracle (test infrastructure only -- never linked into the product).
 *
 * CPU restatement of the reference path of yagise/MyFluidSimulation
 * ("FluidSimExtended"):
 *   - D3Q19 LBM steps in FP64 (and an FP32 twin), lbm_oracle_impl.h;
 *   - the B0 band classification, src/apps/sim_runner.hpp:28-91;
 *   - the STL loader, src/geom/stl_loader.cpp:34-122;
 *   - the SAT + flood-fill voxelizer, src/geom/voxelize.cpp:14-243;
 *   - the volume view's fragment shader (src/render/Vis3D.cpp:30-78), in FP32
 *     with every operation rounded as written.  That one is parity unpinned:
 *     the shader needs an OpenGL context, unavailable on this box, so it is
 *     restated from its GLSL source alone.
 * The geometry code computes in float with no contraction (built with
 * -ffp-contract=off), in the reference's operation order, so that masks are
 * bit-exact with the reference compiled by a default x86-64 g++.
 *
 * Pinning: the geometry functions are checked bit-for-bit against the
 * reference's own voxelize.cpp / stl_loader.cpp / sim_runner.hpp compiled
 * here (oracle/build_ref.sh -> oracle/_ref) and against fixtures generated
 * from it (tests/golden); the LBM steps are checked against the reference's
 * CUDA build run on a B200 (fixtures in tests/golden) within float tolerance.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <float.h>

/* D3Q19 velocity set, reference order (src/lbm/lbm3d_legacy.cu:16-32) */
static const int CX[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
static const int CY[19] = {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1};
static const int CZ[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1};
/* the true opposite direction, c_OPP[q] = -c_q */
static const int OPP[19] = {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15};
/* the reference's opp() table (lbm3d_legacy.cu:29-32, lbm3d_home.cu:27-30,
 * lbm3d_hybrid.cu:28-31): correct for the 6 axis directions, but it pairs each
 * diagonal with its mirror image in x (xy/xz diagonals) or y (yz diagonals),
 * e.g. 7 (+1,+1,0) with 8 (-1,+1,0) */
static const int OPP_REF[19] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17};
static const double W_D[19] = {1.0 / 3.0,
    1.0 / 18.0, 1.0 / 18.0, 1.0 / 18.0, 1.0 / 18.0, 1.0 / 18.0, 1.0 / 18.0,
    1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0,
    1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0};
static const float W_F[19] = {1.0f / 3.0f,
    1.0f / 18.0f, 1.0f / 18.0f, 1.0f / 18.0f, 1.0f / 18.0f, 1.0f / 18.0f, 1.0f / 18.0f,
    1.0f / 36.0f, 1.0f / 36.0f, 1.0f / 36.0f, 1.0f / 36.0f, 1.0f / 36.0f, 1.0f / 36.0f,
    1.0f / 36.0f, 1.0f / 36.0f, 1.0f / 36.0f, 1.0f / 36.0f, 1.0f / 36.0f, 1.0f / 36.0f};

#define REAL double
#define SUFFIX f64
#define WQ(q) W_D[q]
#include "lbm_oracle_impl.h"
#undef REAL
#undef SUFFIX
#undef WQ

#define REAL float
#define SUFFIX f32
#define WQ(q) W_F[q]
#include "lbm_oracle_impl.h"
#undef REAL
#undef SUFFIX
#undef WQ

int orc_num_threads(void) {
#ifdef _OPENMP
    extern int omp_get_max_threads(void);
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------------ */
/* B0 band: src/apps/sim_runner.hpp:28-78 (multi-source 6-neighbour BFS from  */
/* every solid cell, non-periodic, cells at maxDist are labelled but not      */
/* expanded) and :79-91 (isLegacy = fluid && 0 <= dist <= d0).               */
/* run_hybrid_b0 calls it with maxDist = max(1, d0) (sim_runner.hpp:221-224). */
/* ------------------------------------------------------------------------ */
void orc_band(const uint8_t* mask, int nx, int ny, int nz, int d0, int32_t* dist, uint8_t* is_legacy) {
    const int64_t N = (int64_t)nx * ny * nz;
    const int max_dist = d0 > 1 ? d0 : 1;
    for (int64_t i = 0; i < N; ++i) dist[i] = -1;
    int64_t* q = (int64_t*)malloc(sizeof(int64_t) * (size_t)(N > 0 ? N : 1));
    int64_t head = 0, tail = 0;
    for (int64_t i = 0; i < N; ++i)
        if (mask[i]) { dist[i] = 0; q[tail++] = i; }
    const int64_t sy = nx, sz = (int64_t)nx * ny;
    while (head < tail) {
        const int64_t id = q[head++];
        const int dc = dist[id];
        if (dc >= max_dist) continue;
        const int z = (int)(id / sz);
        const int64_t rem = id - (int64_t)z * sz;
        const int y = (int)(rem / sy);
        const int x = (int)(rem - (int64_t)y * sy);
        const int nd = dc + 1;
        int64_t nb[6]; int k = 0;
        if (x > 0) nb[k++] = id - 1;
        if (x < nx - 1) nb[k++] = id + 1;
        if (y > 0) nb[k++] = id - sy;
        if (y < ny - 1) nb[k++] = id + sy;
        if (z > 0) nb[k++] = id - sz;
        if (z < nz - 1) nb[k++] = id + sz;
        for (int j = 0; j < k; ++j)
            if (dist[nb[j]] == -1) { dist[nb[j]] = nd; q[tail++] = nb[j]; }
    }
    free(q);
    for (int64_t i = 0; i < N; ++i)
        is_legacy[i] = (!mask[i] && dist[i] >= 0 && dist[i] <= d0) ? 1 : 0;
}

/* ------------------------------------------------------------------------ */
/* STL loader: src/geom/stl_loader.cpp:34-122.  Returns the number of        */
/* triangles (>0), or -1 when the reference's load_stl would return false.   */
/* tris receives 9 floats per triangle (v0 v1 v2), bb = {min xyz, max xyz}.  */
/* The buffer is malloc'd; free it with orc_free.                            */
/* ------------------------------------------------------------------------ */
static void bb_update(float* bb, const float* p) {
    for (int k = 0; k < 3; ++k) {
        if (p[k] < bb[k]) bb[k] = p[k];          /* std::min(a,b): b<a ? b : a */
        if (bb[3 + k] < p[k]) bb[3 + k] = p[k];  /* std::max(a,b): a<b ? b : a */
    }
}

static int64_t parse_binary(const unsigned char* buf, size_t len, float** out, float* bb) {
    if (len < 84) return -1;
    uint32_t ntri;
    memcpy(&ntri, buf + 80, 4);
    for (int k = 0; k < 3; ++k) { bb[k] = FLT_MAX; bb[3 + k] = -FLT_MAX; }
    if ((uint64_t)84 + (uint64_t)ntri * 50u > (uint64_t)len) return -1;   /* truncated record */
    float* t = (float*)malloc(sizeof(float) * 9 * (size_t)(ntri ? ntri : 1));
    for (uint32_t i = 0; i < ntri; ++i) {
        const unsigned char* r = buf + 84 + (size_t)i * 50 + 12;   /* skip the normal */
        memcpy(t + (size_t)i * 9, r, 36);
        for (int v = 0; v < 3; ++v) bb_update(bb, t + (size_t)i * 9 + v * 3);
    }
    *out = t;
    return (int64_t)ntri;
}

static int64_t parse_ascii(const char* s, size_t len, float** out, float* bb) {
    for (int k = 0; k < 3; ++k) { bb[k] = FLT_MAX; bb[3 + k] = -FLT_MAX; }
    size_t cap = 1024, n = 0;
    float* t = (float*)malloc(sizeof(float) * 9 * cap);
    float tri[9]; int nv = 0;
    size_t pos = 0;
    char line[4096];
    while (pos < len) {
        size_t e = pos;
        while (e < len && s[e] != '\n') ++e;
        size_t L = e - pos; if (L > sizeof(line) - 1) L = sizeof(line) - 1;
        memcpy(line, s + pos, L); line[L] = 0;
        pos = e + 1;
        char tok[64]; int used = 0;
        if (sscanf(line, "%63s%n", tok, &used) == 1 && strcmp(tok, "vertex") == 0) {
            /* ss >> x >> y >> z: a failed extraction leaves 0 and stops the rest */
            float v[3] = {0, 0, 0};
            char* p = line + used;
            for (int k = 0; k < 3; ++k) {
                char* e = p;
                const float val = strtof(p, &e);
                if (e == p) break;
                v[k] = val; p = e;
            }
            const float x = v[0], y = v[1], z = v[2];
            tri[nv * 3 + 0] = x; tri[nv * 3 + 1] = y; tri[nv * 3 + 2] = z; ++nv;
            if (nv == 3) {
                if (n == cap) { cap *= 2; t = (float*)realloc(t, sizeof(float) * 9 * cap); }
                memcpy(t + n * 9, tri, sizeof(tri));
                for (int v = 0; v < 3; ++v) bb_update(bb, tri + v * 3);
                ++n; nv = 0;
            }
        }
    }
    if (n == 0) { free(t); return -1; }
    *out = t;
    return (int64_t)n;
}

int64_t orc_load_stl(const char* path, float** tris, float* bb) {
    FILE* fp = fopen(path, "rb");
    if (!fp) return -1;
    fseek(fp, 0, SEEK_END);
    long len = ftell(fp);
    fseek(fp, 0, SEEK_SET);
    unsigned char* buf = (unsigned char*)malloc((size_t)(len > 0 ? len : 1) + 1);
    size_t got = fread(buf, 1, (size_t)len, fp);
    fclose(fp);
    buf[got] = 0;
    int64_t n = -1;
    if (got >= 5 && memcmp(buf, "solid", 5) == 0) {
        n = parse_ascii((const char*)buf, got, tris, bb);
        if (n < 0) n = parse_binary(buf, got, tris, bb);    /* ASCII failed: try binary */
    } else {
        n = parse_binary(buf, got, tris, bb);
    }
    free(buf);
    return n;
}

void orc_free(void* p) { free(p); }

/* ------------------------------------------------------------------------ */
/* Voxelizer: src/geom/voxelize.cpp:14-243                                   */
/* ------------------------------------------------------------------------ */
static float fminf_ref(float a, float b) { return (b < a) ? b : a; }   /* std::min */
static float fmaxf_ref(float a, float b) { return (a < b) ? b : a; }   /* std::max */

/* glm::cross(x, y) = (x.y*y.z - y.y*x.z, x.z*y.x - y.z*x.x, x.x*y.y - y.x*x.y) */
static void cross3(const float* a, const float* b, float* o) {
    o[0] = a[1] * b[2] - b[1] * a[2];
    o[1] = a[2] * b[0] - b[2] * a[0];
    o[2] = a[0] * b[1] - b[0] * a[1];
}

/* voxelize.cpp:23-81 */
static int tri_box_overlap(const float* c, const float* half, const float* v0, const float* v1, const float* v2) {
    float tv0[3], tv1[3], tv2[3];
    for (int k = 0; k < 3; ++k) { tv0[k] = v0[k] - c[k]; tv1[k] = v1[k] - c[k]; tv2[k] = v2[k] - c[k]; }
    for (int k = 0; k < 3; ++k) {
        const float mn = fminf_ref(fminf_ref(tv0[k], tv1[k]), tv2[k]);
        const float mx = fmaxf_ref(fmaxf_ref(tv0[k], tv1[k]), tv2[k]);
        if (mx < -half[k] || mn > half[k]) return 0;
    }
    float e[3][3];
    for (int k = 0; k < 3; ++k) { e[0][k] = tv1[k] - tv0[k]; e[1][k] = tv2[k] - tv1[k]; e[2][k] = tv0[k] - tv2[k]; }
    float n[3];
    cross3(e[0], e[1], n);
    const float r = half[0] * fabsf(n[0]) + half[1] * fabsf(n[1]) + half[2] * fabsf(n[2]);
    const float s = fabsf(n[0] * tv0[0] + n[1] * tv0[1] + n[2] * tv0[2]);
    if (s > r) return 0;
    static const float axes[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    for (int ei = 0; ei < 3; ++ei) {
        const float* ed = e[ei];
        if (fabsf(ed[0]) + fabsf(ed[1]) + fabsf(ed[2]) < 1e-12f) continue;
        for (int ai = 0; ai < 3; ++ai) {
            float L[3];
            cross3(ed, axes[ai], L);
            const float l2 = L[0] * L[0] + L[1] * L[1] + L[2] * L[2];
            if (l2 < 1e-20f) continue;
            const float p0 = L[0] * tv0[0] + L[1] * tv0[1] + L[2] * tv0[2];
            const float p1 = L[0] * tv1[0] + L[1] * tv1[1] + L[2] * tv1[2];
            const float p2 = L[0] * tv2[0] + L[1] * tv2[1] + L[2] * tv2[2];
            const float minp = fminf_ref(p0, fminf_ref(p1, p2));
            const float maxp = fmaxf_ref(p0, fmaxf_ref(p1, p2));
            const float rp = half[0] * fabsf(L[0]) + half[1] * fabsf(L[1]) + half[2] * fabsf(L[2]);
            if (maxp < -rp || minp > rp) return 0;
        }
    }
    return 1;
}

/* voxelize.cpp:83-113: fit to the unit cube, apply to every vertex */
void orc_fit_transform(const float* tris, int64_t ntri, const float* bb, float scale,
                       float tx, float ty, float tz, float* out) {
    float bbsize[3] = {bb[3] - bb[0], bb[4] - bb[1], bb[5] - bb[2]};
    const float maxDim = fmaxf_ref(bbsize[0], fmaxf_ref(bbsize[1], bbsize[2]));
    const float s = (maxDim > 0.0f) ? (scale / maxDim) : 1.0f;
    const float center[3] = {0.5f * (bb[0] + bb[3]), 0.5f * (bb[1] + bb[4]), 0.5f * (bb[2] + bb[5])};
    const float tr[3] = {tx - s * center[0], ty - s * center[1], tz - s * center[2]};
    for (int64_t i = 0; i < ntri * 3; ++i)
        for (int k = 0; k < 3; ++k) out[i * 3 + k] = s * tris[i * 3 + k] + tr[k];
}

/* voxelize.cpp:115-149: surface cells by SAT over each triangle's candidate box */
void orc_surface(const float* vt, int64_t ntri, int nx, int ny, int nz, uint8_t* surf) {
    const float half[3] = {0.5f / (float)nx, 0.5f / (float)ny, 0.5f / (float)nz};
    const float eps = 1e-6f;
    for (int64_t it = 0; it < ntri; ++it) {
        const float* v0 = vt + it * 9;
        const float* v1 = v0 + 3;
        const float* v2 = v0 + 6;
        const float minx = fminf_ref(v0[0], fminf_ref(v1[0], v2[0])) - eps;
        const float miny = fminf_ref(v0[1], fminf_ref(v1[1], v2[1])) - eps;
        const float minz = fminf_ref(v0[2], fminf_ref(v1[2], v2[2])) - eps;
        const float maxx = fmaxf_ref(v0[0], fmaxf_ref(v1[0], v2[0])) + eps;
        const float maxy = fmaxf_ref(v0[1], fmaxf_ref(v1[1], v2[1])) + eps;
        const float maxz = fmaxf_ref(v0[2], fmaxf_ref(v1[2], v2[2])) + eps;
        int x0 = (int)floorf(minx * (float)nx); if (x0 < 0) x0 = 0;
        int y0 = (int)floorf(miny * (float)ny); if (y0 < 0) y0 = 0;
        int z0 = (int)floorf(minz * (float)nz); if (z0 < 0) z0 = 0;
        int x1 = (int)floorf(maxx * (float)nx); if (x1 > nx - 1) x1 = nx - 1;
        int y1 = (int)floorf(maxy * (float)ny); if (y1 > ny - 1) y1 = ny - 1;
        int z1 = (int)floorf(maxz * (float)nz); if (z1 > nz - 1) z1 = nz - 1;
        for (int z = z0; z <= z1; ++z)
        for (int y = y0; y <= y1; ++y)
        for (int x = x0; x <= x1; ++x) {
            const float c[3] = {((float)x + 0.5f) / (float)nx, ((float)y + 0.5f) / (float)ny,
                                ((float)z + 0.5f) / (float)nz};
            if (tri_box_overlap(c, half, v0, v1, v2)) surf[((int64_t)z * ny + y) * nx + x] = 1;
        }
    }
}

/* voxelize.cpp:151-184: exterior = 6-connected flood fill from the six faces */
void orc_fill(const uint8_t* surf, int nx, int ny, int nz, uint8_t* solid) {
    const int64_t N = (int64_t)nx * ny * nz;
    uint8_t* vis = (uint8_t*)calloc((size_t)N, 1);
    int64_t* q = (int64_t*)malloc(sizeof(int64_t) * (size_t)(N > 0 ? N : 1));
    int64_t head = 0, tail = 0;
#define PUSH(X, Y, Z) do { int xx_ = (X), yy_ = (Y), zz_ = (Z); \
        if (xx_ >= 0 && yy_ >= 0 && zz_ >= 0 && xx_ < nx && yy_ < ny && zz_ < nz) { \
            int64_t i_ = ((int64_t)zz_ * ny + yy_) * nx + xx_; \
            if (!vis[i_] && !surf[i_]) { vis[i_] = 1; q[tail++] = i_; } } } while (0)
    for (int y = 0; y < ny; ++y) for (int z = 0; z < nz; ++z) { PUSH(0, y, z); PUSH(nx - 1, y, z); }
    for (int x = 0; x < nx; ++x) for (int z = 0; z < nz; ++z) { PUSH(x, 0, z); PUSH(x, ny - 1, z); }
    for (int x = 0; x < nx; ++x) for (int y = 0; y < ny; ++y) { PUSH(x, y, 0); PUSH(x, y, nz - 1); }
    while (head < tail) {
        const int64_t i = q[head++];
        const int x = (int)(i % nx), y = (int)((i / nx) % ny), z = (int)(i / ((int64_t)nx * ny));
        PUSH(x + 1, y, z); PUSH(x - 1, y, z);
        PUSH(x, y + 1, z); PUSH(x, y - 1, z);
        PUSH(x, y, z + 1); PUSH(x, y, z - 1);
    }
#undef PUSH
    for (int64_t i = 0; i < N; ++i) solid[i] = (surf[i] || !vis[i]) ? 1 : 0;
    free(vis); free(q);
}

/* voxelize.cpp:187-226 */
void orc_downsample(const uint8_t* fine, int refine, int nx, int ny, int nz, float threshold, uint8_t* coarse) {
    const int64_t NxF = (int64_t)nx * refine, NyF = (int64_t)ny * refine;
    const int r3 = refine * refine * refine;
    const float thr = fmaxf_ref(0.0f, fminf_ref(1.0f, threshold));
    for (int cz = 0; cz < nz; ++cz)
    for (int cy = 0; cy < ny; ++cy)
    for (int cx = 0; cx < nx; ++cx) {
        int cnt = 0;
        for (int dz = 0; dz < refine; ++dz)
        for (int dy = 0; dy < refine; ++dy) {
            const int64_t base = ((int64_t)cz * refine + dz) * NyF * NxF + ((int64_t)cy * refine + dy) * NxF + (int64_t)cx * refine;
            for (int dx = 0; dx < refine; ++dx) cnt += fine[base + dx];
        }
        const float cov = (float)cnt / (float)r3;
        coarse[((int64_t)cz * ny + cy) * nx + cx] = (cov > 0.0f && cov >= thr) ? 1 : 0;
    }
}

/* voxelize.cpp:228-243: the public entry (mesh in its own coordinates + its bbox) */
int orc_voxelize(const float* tris, int64_t ntri, const float* bb, int nx, int ny, int nz,
                 float scale, float tx, float ty, float tz, int refine, float thr, uint8_t* mask) {
    if (refine < 1) refine = 1;
    float* vt = (float*)malloc(sizeof(float) * 9 * (size_t)(ntri > 0 ? ntri : 1));
    orc_fit_transform(tris, ntri, bb, scale, tx, ty, tz, vt);
    const int fx = nx * refine, fy = ny * refine, fz = nz * refine;
    const int64_t NF = (int64_t)fx * fy * fz;
    uint8_t* surf = (uint8_t*)calloc((size_t)NF, 1);
    orc_surface(vt, ntri, fx, fy, fz, surf);
    if (refine == 1) {
        orc_fill(surf, nx, ny, nz, mask);
    } else {
        uint8_t* fine = (uint8_t*)malloc((size_t)NF);
        orc_fill(surf, fx, fy, fz, fine);
        orc_downsample(fine, refine, nx, ny, nz, thr, mask);
        free(fine);
    }
    free(surf); free(vt);
    return 0;
}

/* ---- volume view: the fragment shader of src/render/Vis3D.cpp:30-78 ------ */

/* GLSL min/max/clamp/mix as the specification writes them */
static float g_min(float x, float y) { return y < x ? y : x; }
static float g_max(float x, float y) { return x < y ? y : x; }
static float g_clamp(float x, float lo, float hi) { return g_min(g_max(x, lo), hi); }
static float g_mix(float x, float y, float a) { return x * (1.0f - a) + y * a; }

/* colormap(t), Vis3D.cpp:40-46 */
static void vs_colormap(float t, float c[3]) {
    static const float K[5][3] = {{0.02f, 0.02f, 0.2f}, {0.0f, 0.7f, 1.0f}, {0.0f, 1.0f, 0.3f},
                                  {1.0f, 0.9f, 0.0f}, {1.0f, 0.1f, 0.0f}};
    t = g_clamp(t, 0.0f, 1.0f);
    int seg;
    float w;
    if (t < 0.25f) { seg = 0; w = t * 4.0f; }
    else if (t < 0.50f) { seg = 1; w = (t - 0.25f) * 4.0f; }
    else if (t < 0.75f) { seg = 2; w = (t - 0.50f) * 4.0f; }
    else { seg = 3; w = (t - 0.75f) * 4.0f; }
    for (int k = 0; k < 3; ++k) c[k] = g_mix(K[seg][k], K[seg + 1][k], w);
}

/* texture(uTex, p).r with GL_LINEAR and CLAMP_TO_EDGE on an R32F 3-D texture
 * (Vis3D.cpp:82-89): texel i centred at (i + 0.5) / n, lerp in x, y, z */
static float vs_texture(const float* f, int nx, int ny, int nz, const float p[3]) {
    const int n[3] = {nx, ny, nz};
    int i0[3], i1[3];
    float fr[3];
    for (int k = 0; k < 3; ++k) {
        const float u = p[k] * (float)n[k] - 0.5f;
        const float fl = floorf(u);
        const int i = (int)fl;
        fr[k] = u - fl;
        i0[k] = i < 0 ? 0 : (i > n[k] - 1 ? n[k] - 1 : i);
        i1[k] = i + 1 < 0 ? 0 : (i + 1 > n[k] - 1 ? n[k] - 1 : i + 1);
    }
#define TX(x, y, z) f[((size_t)(z) * ny + (y)) * nx + (x)]
    const float c00 = g_mix(TX(i0[0], i0[1], i0[2]), TX(i1[0], i0[1], i0[2]), fr[0]);
    const float c10 = g_mix(TX(i0[0], i1[1], i0[2]), TX(i1[0], i1[1], i0[2]), fr[0]);
    const float c01 = g_mix(TX(i0[0], i0[1], i1[2]), TX(i1[0], i0[1], i1[2]), fr[0]);
    const float c11 = g_mix(TX(i0[0], i1[1], i1[2]), TX(i1[0], i1[1], i1[2]), fr[0]);
#undef TX
    return g_mix(g_mix(c00, c10, fr[1]), g_mix(c01, c11, fr[1]), fr[2]);
}

/* One frame: main() of the shader for every pixel (x, y), uv = ((x+0.5)/W,
 * (y+0.5)/H), row 0 at the bottom; a discarded fragment keeps the clear colour
 * (0.02, 0.02, 0.03, 1) of main_compare.cpp:988.  inv_pv column-major. */
void orc_raymarch_f32(const float* field, int nx, int ny, int nz, const float* inv_pv, const float* cam,
                      float step, float scale, float thresh, int width, int height, float* rgba,
                      int64_t* samples) {
    int64_t total = 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(+:total)
    for (int y = 0; y < height; ++y) {
        for (int x = 0; x < width; ++x) {
            float* o = rgba + ((size_t)y * width + x) * 4;
            const float uvx = ((float)x + 0.5f) / (float)width, uvy = ((float)y + 0.5f) / (float)height;
            const float ndc[4] = {uvx * 2.0f - 1.0f, uvy * 2.0f - 1.0f, 0.0f, 1.0f};
            float w[4];
            for (int r = 0; r < 4; ++r)
                w[r] = inv_pv[r] * ndc[0] + inv_pv[4 + r] * ndc[1] + inv_pv[8 + r] * ndc[2] + inv_pv[12 + r] * ndc[3];
            float dir[3];
            for (int k = 0; k < 3; ++k) dir[k] = w[k] / w[3] - cam[k];
            const float len = sqrtf(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
            for (int k = 0; k < 3; ++k) dir[k] = dir[k] / len;
            float t0[3], t1[3];
            for (int k = 0; k < 3; ++k) {
                t0[k] = (0.0f - cam[k]) / dir[k];
                t1[k] = (1.0f - cam[k]) / dir[k];
            }
            float tnear = g_max(g_max(g_min(t0[0], t1[0]), g_min(t0[1], t1[1])), g_min(t0[2], t1[2]));
            const float tfar = g_min(g_min(g_max(t0[0], t1[0]), g_max(t0[1], t1[1])), g_max(t0[2], t1[2]));
            if (tfar < 0.0f || tnear > tfar) {
                o[0] = 0.02f; o[1] = 0.02f; o[2] = 0.03f; o[3] = 1.0f;
                continue;
            }
            tnear = g_max(tnear, 0.0f);
            float pos[3];
            for (int k = 0; k < 3; ++k) pos[k] = cam[k] + dir[k] * tnear;
            float t = tnear, acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            while (t < tfar && acc[3] < 0.95f) {
                /* sampleVol(pos), Vis3D.cpp:48-57 */
                const float s = vs_texture(field, nx, ny, nz, pos) * scale;
                const float tmag = g_clamp(fabsf(s), 0.0f, 1.0f);
                float sr = 0.0f, sg = 0.0f, sb = 0.0f, sa = 0.0f;
                if (!(tmag < thresh)) {
                    const float tcol = 0.5f + 0.5f * g_clamp(s, -1.0f, 1.0f);
                    const float h = g_clamp((tmag - thresh) / (1.0f - thresh), 0.0f, 1.0f);   /* smoothstep */
                    float c[3];
                    vs_colormap(tcol, c);
                    sr = c[0]; sg = c[1]; sb = c[2];
                    sa = h * h * (3.0f - 2.0f * h);
                }
                const float rem = 1.0f - acc[3];
                acc[0] += sr * rem;
                acc[1] += sg * rem;
                acc[2] += sb * rem;
                acc[3] += sa * (1.0f - acc[3]);
                for (int k = 0; k < 3; ++k) pos[k] += dir[k] * step;
                t += step;
                ++total;
            }
            o[0] = acc[0]; o[1] = acc[1]; o[2] = acc[2]; o[3] = 1.0f;
        }
    }
    if (samples) *samples = total;
}
