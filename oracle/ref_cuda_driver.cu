// Checker / reference arm only: a C-ABI around the reference's own CUDA solver
// classes (src/lbm/lbm3d_legacy.cu, lbm3d_home.cu, lbm3d_hybrid.cu,
// lbm_reinit.cu, src/fields/*.cu, src/moment_vtk_writer.cu), compiled
// unmodified from the reference sources by oracle/build_ref.sh into
// oracle/_ref/libref_cuda.so.  Tests use it to produce golden fields on the
// GPU; bench.py --impl reference times it.  Never part of the product.
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <exception>
#include <stdexcept>
#include <string>
#include <vector>

#include "lbm/lbm3d_legacy.hpp"
#include "lbm/lbm3d_home.hpp"
#include "lbm/lbm3d_hybrid.hpp"

extern "C" void launch_speed(const float* u, const float* v, const float* w, float* out, int N);
extern "C" void write_scalar_vtk(const char* filename, const float* d_field, int Nx, int Ny, int Nz);
extern "C" void write_vector_vtk(const char* filename, const float* d_fx, const float* d_fy,
                                 const float* d_fz, int Nx, int Ny, int Nz);
extern "C" void make_rho_gauss(float* d_rho, int Nx, int Ny, int Nz, float cx, float cy, float cz,
                               float sigma, float amp);
extern "C" void make_rho_slab(float* d_rho, int Nx, int Ny, int Nz, int axis, float amp, float center,
                              float width);

namespace {
std::string g_err;

struct RefSolver {
    int method = 0;  // 0 legacy, 1 home, 2 hybrid
    LBM3D_Legacy* leg = nullptr;
    LBM3D_Home* home = nullptr;
    LBM3D_Hybrid* hyb = nullptr;
    int N = 0, nx = 0, ny = 0, nz = 0;
    ~RefSolver() { delete leg; delete home; delete hyb; }
    float* d_rho() { return leg ? leg->d_rho() : home ? home->d_rho() : hyb->d_rho(); }
    float* d_u() { return leg ? leg->d_u() : home ? home->d_u() : hyb->d_u(); }
    float* d_v() { return leg ? leg->d_v() : home ? home->d_v() : hyb->d_v(); }
    float* d_w() { return leg ? leg->d_w() : home ? home->d_w() : hyb->d_w(); }
};

template <class F>
int guarded(F&& f) {
    try { f(); return 0; }
    catch (const std::exception& e) { g_err = e.what(); return 1; }
}
}  // namespace

extern "C" {

const char* refcu_last_error(void) { return g_err.c_str(); }

void* refcu_create(int method, int nx, int ny, int nz, float tau, float fx, float fy, float fz) {
    RefSolver* s = new RefSolver();
    s->method = method; s->nx = nx; s->ny = ny; s->nz = nz; s->N = nx * ny * nz;
    Domain d; d.Nx = nx; d.Ny = ny; d.Nz = nz; d.tau = tau; d.forceX = fx; d.forceY = fy; d.forceZ = fz;
    int rc = guarded([&] {
        if (method == 0) { s->leg = new LBM3D_Legacy(); s->leg->init(d); }
        else if (method == 1) { s->home = new LBM3D_Home(); s->home->init(d); }
        else { s->hyb = new LBM3D_Hybrid(); s->hyb->init(d, 0); }
    });
    if (rc) { delete s; return nullptr; }
    return s;
}

void refcu_destroy(void* h) { delete static_cast<RefSolver*>(h); }

int refcu_set_mask(void* h, const uint8_t* mask) {
    RefSolver* s = static_cast<RefSolver*>(h);
    return guarded([&] {
        if (s->leg) s->leg->setSolidMask(mask);
        else if (s->home) s->home->setSolidMask(mask);
        else s->hyb->setSolidMask(mask);
    });
}

int refcu_set_legacy(void* h, const uint8_t* is_legacy) {
    RefSolver* s = static_cast<RefSolver*>(h);
    if (!s->hyb) return 2;
    return guarded([&] { s->hyb->setLegacyMapping(is_legacy, nullptr); });
}

// The fluidsim_tgv path: host fields copied into the solver's own macro
// buffers, then reinitEquilibriumFromMacro on them (main_taylor_green.cpp:90-105).
int refcu_init_fields(void* h, const float* rho, const float* ux, const float* uy, const float* uz) {
    RefSolver* s = static_cast<RefSolver*>(h);
    return guarded([&] {
        const size_t b = sizeof(float) * (size_t)s->N;
        if (cudaMemcpy(s->d_rho(), rho, b, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(s->d_u(), ux, b, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(s->d_v(), uy, b, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(s->d_w(), uz, b, cudaMemcpyHostToDevice) != cudaSuccess)
            throw std::runtime_error("H2D failed");
        if (s->leg) s->leg->reinitEquilibriumFromMacro(s->d_rho(), s->d_u(), s->d_v(), s->d_w());
        else if (s->home) s->home->reinitEquilibriumFromMacro(s->d_rho(), s->d_u(), s->d_v(), s->d_w());
        else s->hyb->reinitEquilibriumFromMacro(s->d_rho(), s->d_u(), s->d_v(), s->d_w());
    });
}

// The run_single_solver / run_hybrid_b0 path: a separate device rho buffer,
// reinitEquilibriumFromMacro(d_rhoInit, nullptr, nullptr, nullptr)
// (sim_runner.hpp:135-137,229-231).  rho == NULL uploads ones.
int refcu_init_rho(void* h, const float* rho) {
    RefSolver* s = static_cast<RefSolver*>(h);
    return guarded([&] {
        float* d = nullptr;
        const size_t b = sizeof(float) * (size_t)s->N;
        if (cudaMalloc(&d, b) != cudaSuccess) throw std::runtime_error("cudaMalloc failed");
        std::vector<float> ones;
        if (!rho) { ones.assign((size_t)s->N, 1.0f); rho = ones.data(); }
        cudaMemcpy(d, rho, b, cudaMemcpyHostToDevice);
        if (s->leg) s->leg->reinitEquilibriumFromMacro(d, nullptr, nullptr, nullptr);
        else if (s->home) s->home->reinitEquilibriumFromMacro(d, nullptr, nullptr, nullptr);
        else s->hyb->reinitEquilibriumFromMacro(d, nullptr, nullptr, nullptr);
        cudaFree(d);
    });
}

int refcu_step(void* h, int substeps) {
    RefSolver* s = static_cast<RefSolver*>(h);
    return guarded([&] {
        if (s->leg) s->leg->step(substeps);
        else if (s->home) s->home->step(substeps);
        else s->hyb->step(substeps);
    });
}

// Milliseconds for `calls` calls of step(substeps), cudaEvents on the default
// stream, as the reference's own sweep times it (main_compare.cpp:539-553).
int refcu_time_steps(void* h, int calls, int substeps, float* ms) {
    RefSolver* s = static_cast<RefSolver*>(h);
    return guarded([&] {
        cudaEvent_t a, b;
        cudaEventCreate(&a); cudaEventCreate(&b);
        cudaEventRecord(a, 0);
        for (int i = 0; i < calls; ++i) {
            if (s->leg) s->leg->step(substeps);
            else if (s->home) s->home->step(substeps);
            else s->hyb->step(substeps);
        }
        cudaEventRecord(b, 0);
        cudaEventSynchronize(b);
        cudaEventElapsedTime(ms, a, b);
        cudaEventDestroy(a); cudaEventDestroy(b);
    });
}

int refcu_get_macros(void* h, float* rho, float* u, float* v, float* w) {
    RefSolver* s = static_cast<RefSolver*>(h);
    return guarded([&] {
        const size_t b = sizeof(float) * (size_t)s->N;
        if (rho) cudaMemcpy(rho, s->d_rho(), b, cudaMemcpyDeviceToHost);
        if (u) cudaMemcpy(u, s->d_u(), b, cudaMemcpyDeviceToHost);
        if (v) cudaMemcpy(v, s->d_v(), b, cudaMemcpyDeviceToHost);
        if (w) cudaMemcpy(w, s->d_w(), b, cudaMemcpyDeviceToHost);
        if (cudaDeviceSynchronize() != cudaSuccess) throw std::runtime_error("D2H failed");
    });
}

// Legacy/Hybrid: the 19*N populations d_f (SoA q*N+id).  HOME: its 10*N moments.
int refcu_get_state(void* h, float* out) {
    RefSolver* s = static_cast<RefSolver*>(h);
    return guarded([&] {
        if (s->leg) cudaMemcpy(out, s->leg->d_f(), sizeof(float) * 19 * (size_t)s->N, cudaMemcpyDeviceToHost);
        else if (s->hyb) cudaMemcpy(out, s->hyb->d_f(), sizeof(float) * 19 * (size_t)s->N, cudaMemcpyDeviceToHost);
        else cudaMemcpy(out, s->home->d_rho(), sizeof(float) * 10 * (size_t)s->N, cudaMemcpyDeviceToHost);
        if (cudaDeviceSynchronize() != cudaSuccess) throw std::runtime_error("D2H failed");
    });
}

// The second population buffer d_fnext (Legacy/Hybrid), for inspecting what
// the reference leaves in it.
int refcu_get_fnext(void* h, float* out) {
    RefSolver* s = static_cast<RefSolver*>(h);
    return guarded([&] {
        const float* p = s->leg ? s->leg->d_fnext() : (s->hyb ? s->hyb->d_fnext() : nullptr);
        if (!p) throw std::runtime_error("no fnext for HOME");
        cudaMemcpy(out, p, sizeof(float) * 19 * (size_t)s->N, cudaMemcpyDeviceToHost);
        if (cudaDeviceSynchronize() != cudaSuccess) throw std::runtime_error("D2H failed");
    });
}

// VTK / field helpers of the reference on host arrays (uploaded to a scratch
// device buffer first): launch_speed, make_rho_gauss/slab, write_*_vtk.
int refcu_speed(const float* u, const float* v, const float* w, float* out, int N) {
    return guarded([&] {
        float* d = nullptr;
        cudaMalloc(&d, sizeof(float) * 4 * (size_t)N);
        cudaMemcpy(d, u, sizeof(float) * N, cudaMemcpyHostToDevice);
        cudaMemcpy(d + N, v, sizeof(float) * N, cudaMemcpyHostToDevice);
        cudaMemcpy(d + 2 * (size_t)N, w, sizeof(float) * N, cudaMemcpyHostToDevice);
        launch_speed(d, d + N, d + 2 * (size_t)N, d + 3 * (size_t)N, N);
        cudaMemcpy(out, d + 3 * (size_t)N, sizeof(float) * N, cudaMemcpyDeviceToHost);
        cudaFree(d);
    });
}

int refcu_rho_profile(int kind, int nx, int ny, int nz, const float* p, float* out) {
    return guarded([&] {
        const int N = nx * ny * nz;
        float* d = nullptr;
        cudaMalloc(&d, sizeof(float) * (size_t)N);
        if (kind == 0) make_rho_gauss(d, nx, ny, nz, p[0], p[1], p[2], p[3], p[4]);
        else make_rho_slab(d, nx, ny, nz, (int)p[0], p[1], p[2], p[3]);
        cudaMemcpy(out, d, sizeof(float) * (size_t)N, cudaMemcpyDeviceToHost);
        cudaFree(d);
    });
}

int refcu_write_vtk(const char* path, const float* a, const float* b, const float* c, int nx, int ny, int nz) {
    return guarded([&] {
        const size_t N = (size_t)nx * ny * nz;
        float* d = nullptr;
        cudaMalloc(&d, sizeof(float) * 3 * N);
        cudaMemcpy(d, a, sizeof(float) * N, cudaMemcpyHostToDevice);
        if (b) {
            cudaMemcpy(d + N, b, sizeof(float) * N, cudaMemcpyHostToDevice);
            cudaMemcpy(d + 2 * N, c, sizeof(float) * N, cudaMemcpyHostToDevice);
            write_vector_vtk(path, d, d + N, d + 2 * N, nx, ny, nz);
        } else {
            write_scalar_vtk(path, d, nx, ny, nz);
        }
        cudaFree(d);
    });
}

}  // extern "C"
