// lbm3d_compat.hpp -- the reference's solver classes (LBM3D_Legacy, LBM3D_Home,
// LBM3D_Hybrid and struct Domain) rebuilt as a header-only C++ layer over the
// C-ABI of lbm_capi.h, for C++ callers written against the reference's
// headers (src/lbm/lbm3d_legacy.hpp:19-56, src/lbm/lbm3d_home.hpp:15-46,
// src/lbm/lbm3d_hybrid.hpp:18-58, src/lbm/lbm_common.hpp:6-10).
//
// Semantics kept from the reference:
//   * init(d) allocates and resets (rho=1, u=0); the classes are not copyable;
//   * setSolidMask takes Nx*Ny*Nz host bytes, x fastest, nonzero = solid;
//   * reinitEquilibriumFromMacro takes DEVICE pointers; null velocity
//     components are 0; a null rho resets Legacy and means rho=1 for HOME and
//     Hybrid;
//   * step(substeps) returns after the GPU finished (the reference ends every
//     step with cudaDeviceSynchronize);
//   * d_rho/d_u/d_v/d_w are borrowed device pointers, valid until the next
//     step/reset/reinit (HOME's move on every step, as in the reference);
//   * failures throw std::runtime_error, as the reference's CUDA_CHECK does.
// Differences: the bounce-back defaults to halfway bounce-back with true
// opposite directions (LBM_BOUNCE_HALFWAY); pass LBM_BOUNCE_REFERENCE in the
// options for the reference's own opposite table.  d_f()/d_fnext() are not
// exposed: Legacy/Hybrid keep one in-place population buffer whose layout
// alternates between steps; copyState() returns the reference's layout.
#ifndef LBM3D_COMPAT_HPP
#define LBM3D_COMPAT_HPP

#include <stdexcept>
#include <string>
#include <vector>

#include "lbm_capi.h"

// struct Domain (src/lbm/lbm_common.hpp:6-10): same fields and defaults.
struct Domain {
    int Nx = 128, Ny = 128, Nz = 96;
    float tau = 0.6f;
    float forceX = 0.0f, forceY = 0.0f, forceZ = 0.0f;
};

namespace lbm_compat {

inline void check(int rc, const char* what) {
    if (rc != LBM_OK) throw std::runtime_error(std::string(what) + ": " + lbm_last_error());
}

inline lbm_options default_options(int method) {
    lbm_options o{};
    o.method = method;
    o.storage = LBM_STORE_F32;
    o.bc = LBM_BC_PERIODIC;
    o.bounce = LBM_BOUNCE_HALFWAY;
    o.inlet_u = 0.0f;
    o.rho0 = 1.0f;
    o.stream = nullptr;
    return o;
}

// Shared body of the three classes.
class SolverBase {
public:
    SolverBase(const SolverBase&) = delete;
    SolverBase& operator=(const SolverBase&) = delete;
    ~SolverBase() { release(); }

    // Options used by the next init() (method is fixed by the class).
    void setOptions(const lbm_options& o) {
        const int m = opts_.method;
        opts_ = o;
        opts_.method = m;
    }
    const lbm_options& options() const { return opts_; }

    void init(const Domain& d) {
        release();
        dom_ = d;
        lbm_domain cd{d.Nx, d.Ny, d.Nz, d.tau, d.forceX, d.forceY, d.forceZ};
        check(lbm_create(&cd, &opts_, &h_), "init");
        refresh();
    }
    void release() {
        if (h_) {
            lbm_destroy(h_);
            h_ = nullptr;
        }
    }
    void setSolidMask(const unsigned char* host_mask) {
        check(lbm_set_solid_mask(h(), host_mask), "setSolidMask");
    }
    void reset() {
        check(lbm_reset(h()), "reset");
        check(lbm_synchronize(h()), "reset");
        refresh();
    }
    void reinitEquilibriumFromMacro(const float* d_rho, const float* d_ux, const float* d_uy, const float* d_uz) {
        check(lbm_reinit_from_macro(h(), d_rho, d_ux, d_uy, d_uz), "reinitEquilibriumFromMacro");
        check(lbm_synchronize(h()), "reinitEquilibriumFromMacro");
        refresh();
    }
    void step(int substeps = 1) {
        check(lbm_step(h(), substeps), "step");
        check(lbm_synchronize(h()), "step");
        refresh();
    }
    void setForce(float fx, float fy, float fz) {
        dom_.forceX = fx; dom_.forceY = fy; dom_.forceZ = fz;
        if (h_) check(lbm_set_force(h_, fx, fy, fz), "setForce");
    }

    float* d_rho() const { return rho_; }
    float* d_u() const { return u_; }
    float* d_v() const { return v_; }
    float* d_w() const { return w_; }
    int Nx() const { return dom_.Nx; }
    int Ny() const { return dom_.Ny; }
    int Nz() const { return dom_.Nz; }
    int N() const { return dom_.Nx * dom_.Ny * dom_.Nz; }

    // State in the reference's layout (19*N populations, or 10*N moments for HOME).
    std::vector<float> copyState() {
        int64_t n = 0;
        check(lbm_dims(h(), nullptr, nullptr, nullptr, &n), "copyState");
        std::vector<float> out((size_t)n * (opts_.method == LBM_METHOD_HOME ? 10 : 19));
        check(lbm_get_state(h(), out.data()), "copyState");
        return out;
    }
    lbm_solver* handle() const { return h_; }

protected:
    explicit SolverBase(int method) : opts_(default_options(method)) {}
    lbm_solver* h() const {
        if (!h_) throw std::runtime_error("solver used before init()");
        return h_;
    }
    void refresh() { check(lbm_macro_ptrs(h(), &rho_, &u_, &v_, &w_), "macro pointers"); }

    lbm_options opts_;
    Domain dom_{};
    lbm_solver* h_ = nullptr;
    float* rho_ = nullptr;
    float* u_ = nullptr;
    float* v_ = nullptr;
    float* w_ = nullptr;
};

}  // namespace lbm_compat

// src/lbm/lbm3d_legacy.hpp:19-56
class LBM3D_Legacy : public lbm_compat::SolverBase {
public:
    LBM3D_Legacy() : SolverBase(LBM_METHOD_LEGACY) {}
};

// src/lbm/lbm3d_home.hpp:15-46
class LBM3D_Home : public lbm_compat::SolverBase {
public:
    LBM3D_Home() : SolverBase(LBM_METHOD_HOME) {}
};

// src/lbm/lbm3d_hybrid.hpp:18-58
class LBM3D_Hybrid : public lbm_compat::SolverBase {
public:
    LBM3D_Hybrid() : SolverBase(LBM_METHOD_HYBRID) {}
    // the cell count is ignored, as in the reference (lbm3d_hybrid.cu:210-221)
    void init(const Domain& d, int nLegacyCells = 0) {
        (void)nLegacyCells;
        SolverBase::init(d);
    }
    // isLegacy: Nx*Ny*Nz host bytes, nonzero = BGK band; null clears the band.
    // The slot array is ignored, as in the reference (lbm3d_hybrid.cu:227-235).
    void setLegacyMapping(const unsigned char* h_isLegacy, const int* h_legacySlot) {
        (void)h_legacySlot;
        lbm_compat::check(lbm_set_legacy_mapping(h(), h_isLegacy), "setLegacyMapping");
    }
    // Builds the band on the GPU from the current mask (sim_runner.hpp:28-91
    // with maxDist = max(1, d0)); returns the number of band cells.
    long long buildBand(int d0) {
        int64_t n = 0;
        lbm_compat::check(lbm_build_band(h(), d0, &n), "buildBand");
        return (long long)n;
    }
};

#endif  // LBM3D_COMPAT_HPP
