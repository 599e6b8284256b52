// Host layer of the command-line tools fluidsim_legacy / fluidsim_home /
// fluidsim_hybrid: argument parsing, obstacle build (STL -> GPU voxelizer),
// initial density, VTK cadence and the step loop, all on the C-ABI of
// lbm_capi.h.
//
// Drop-in surface kept from the reference (src/apps/sim_common.hpp:53-283,
// src/apps/sim_runner.hpp:102-270): the same flags and aliases, defaults,
// clamps, "[vtk]"/"[run]" stdout lines, VTK file names
// {rho,speed,vel}_{legacy|home|hybrid}_%06d.vtk, and the behaviour on an
// unreadable STL (a message on stderr, then the run continues without an
// obstacle).  Unknown flags are ignored, as there.
//
// Flags with no reference counterpart (old flags keep their meaning):
//   --precision f32|f16|bf16   storage of populations / moments (FP32 math)
//   --bounce halfway|reference bounce-back with true opposites (default) or
//                              the reference's own opposite table
//   --bc periodic|duct         duct: velocity inlet at x=0, outlet at x=Nx-1
//   --inlet-u U                duct inlet velocity (default 0.05)
//   --walls                    add y/z wall cells (solid, left out of the drag)
//   --stats-every K            print "[stat]" lines (FP64 mass, kinetic
//                              energy, momentum, drag) every K steps
//   --print-config             print the parsed settings and exit (no GPU)
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <filesystem>
#include <string>
#include <vector>

#include "lbm_capi.h"

namespace fsim {

struct Settings {
    // domain (DomainConfig)
    int nx = 200, ny = 150, nz = 120;
    float tau = 0.58f;
    float fx = 0.0f, fy = 0.0f, fz = 0.0f;
    // obstacle (ObstacleConfig)
    std::string stl;
    float voxel_scale = 0.5f;
    float voxel_tr[3] = {0.5f, 0.5f, 0.5f};
    int amr_factor = 1;
    float amr_threshold = 0.5f;
    // run (RunConfig)
    int steps = 200;
    int substeps = 1;
    std::string vtk_dir;
    int vtk_every = 0;
    std::string init = "none";
    float amp = 1e-3f, sigma = 0.08f;
    float center[3] = {0.6f, 0.5f, 0.5f};
    int slab_axis = 0;
    float slab_center = 0.5f, slab_width = 0.2f;
    // hybrid (HybridConfig)
    int band_d0 = 2;
    // extensions
    int storage = LBM_STORE_F32;
    int bounce = LBM_BOUNCE_HALFWAY;
    int bc = LBM_BC_PERIODIC;
    float inlet_u = 0.05f;
    bool walls = false;
    int stats_every = 0;
    bool print_config = false;
};

// One flag of the table: name(s), number of values, action.
inline void parse_args(int argc, char** argv, Settings& s, bool hybrid) {
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        const int left = argc - 1 - i;   // values available after the flag
        auto f = [&]() { return std::stof(argv[++i]); };
        auto n = [&]() { return std::stoi(argv[++i]); };
        if (left >= 1 && a == "--nx") s.nx = n();
        else if (left >= 1 && a == "--ny") s.ny = n();
        else if (left >= 1 && a == "--nz") s.nz = n();
        else if (left >= 1 && a == "--tau") s.tau = f();
        else if (left >= 3 && a == "--force") { s.fx = f(); s.fy = f(); s.fz = f(); }
        else if (left >= 1 && a == "--force-x") s.fx = f();
        else if (left >= 1 && a == "--force-y") s.fy = f();
        else if (left >= 1 && a == "--force-z") s.fz = f();
        else if (left >= 1 && a == "--stl") s.stl = argv[++i];
        else if (left >= 1 && a == "--voxel-scale") s.voxel_scale = f();
        else if (left >= 3 && a == "--voxel-translate") { s.voxel_tr[0] = f(); s.voxel_tr[1] = f(); s.voxel_tr[2] = f(); }
        else if (a == "--amr") s.amr_factor = std::max(s.amr_factor, 2);
        else if (left >= 1 && (a == "--amr-factor" || a == "--amr-refine")) s.amr_factor = std::max(1, n());
        else if (left >= 1 && a == "--amr-threshold") s.amr_threshold = std::clamp(f(), 0.0f, 1.0f);
        else if (left >= 1 && a == "--steps") s.steps = std::max(0, n());
        else if (left >= 1 && a == "--substeps") s.substeps = std::max(1, n());
        else if (left >= 1 && a == "--vtk-dir") s.vtk_dir = argv[++i];
        else if (left >= 1 && (a == "--vtk-every" || a == "--vtk-interval")) s.vtk_every = std::max(0, n());
        else if (left >= 1 && a == "--init") s.init = argv[++i];
        else if (left >= 1 && a == "--amp") s.amp = f();
        else if (left >= 1 && a == "--sigma") s.sigma = f();
        else if (left >= 3 && a == "--center") { s.center[0] = f(); s.center[1] = f(); s.center[2] = f(); }
        else if (left >= 1 && a == "--axis") {
            const char c = argv[++i][0];
            s.slab_axis = c == 'y' ? 1 : (c == 'z' ? 2 : 0);
        }
        else if (left >= 1 && a == "--width") s.slab_width = f();
        else if (left >= 1 && a == "--slab-center") s.slab_center = f();
        else if (left >= 1 && (a == "--hybrid-band" || a == "--hybrid-d0")) {
            const int v = std::max(0, n());
            if (hybrid) s.band_d0 = v;
        }
        // extensions
        else if (left >= 1 && a == "--precision") {
            const std::string v = argv[++i];
            s.storage = v == "f16" ? LBM_STORE_F16 : (v == "bf16" ? LBM_STORE_BF16 : LBM_STORE_F32);
        }
        else if (left >= 1 && a == "--bounce") s.bounce = std::string(argv[++i]) == "reference" ? LBM_BOUNCE_REFERENCE : LBM_BOUNCE_HALFWAY;
        else if (left >= 1 && a == "--bc") s.bc = std::string(argv[++i]) == "duct" ? LBM_BC_DUCT : LBM_BC_PERIODIC;
        else if (left >= 1 && a == "--inlet-u") s.inlet_u = f();
        else if (a == "--walls") s.walls = true;
        else if (left >= 1 && a == "--stats-every") s.stats_every = std::max(0, n());
        else if (a == "--print-config") s.print_config = true;
    }
    // clamps of sim_common.hpp:186-191
    s.nx = std::max(s.nx, 8);
    s.ny = std::max(s.ny, 8);
    s.nz = std::max(s.nz, 1);
    s.tau = std::max(s.tau, 0.51f);
    s.substeps = std::max(s.substeps, 1);
}

// key=value lines; floats with 9 significant digits so two parsers can be compared exactly
inline void print_settings(const Settings& s, FILE* out) {
    std::fprintf(out, "nx=%d\nny=%d\nnz=%d\ntau=%.9g\nforce=%.9g,%.9g,%.9g\n", s.nx, s.ny, s.nz, s.tau, s.fx, s.fy,
                 s.fz);
    std::fprintf(out, "stl=%s\nvoxel_scale=%.9g\nvoxel_translate=%.9g,%.9g,%.9g\namr_factor=%d\namr_threshold=%.9g\n",
                 s.stl.c_str(), s.voxel_scale, s.voxel_tr[0], s.voxel_tr[1], s.voxel_tr[2], s.amr_factor,
                 s.amr_threshold);
    std::fprintf(out, "steps=%d\nsubsteps=%d\nvtk_dir=%s\nvtk_every=%d\ninit=%s\namp=%.9g\nsigma=%.9g\n", s.steps,
                 s.substeps, s.vtk_dir.c_str(), s.vtk_every, s.init.c_str(), s.amp, s.sigma);
    std::fprintf(out, "center=%.9g,%.9g,%.9g\nslab_axis=%d\nslab_center=%.9g\nslab_width=%.9g\nband_d0=%d\n",
                 s.center[0], s.center[1], s.center[2], s.slab_axis, s.slab_center, s.slab_width, s.band_d0);
}

inline std::string vtk_file(const std::filesystem::path& dir, const std::string& stem, int step) {
    char name[64];
    std::snprintf(name, sizeof(name), "%s_%06d.vtk", stem.c_str(), step);
    return (dir / name).string();
}

// Mask of the obstacle (empty vector = none), sim_common.hpp:198-238.
inline std::vector<uint8_t> obstacle_mask(const Settings& s) {
    std::vector<uint8_t> mask((size_t)s.nx * s.ny * s.nz, 0);
    if (s.stl.empty()) return mask;
    float* tris = nullptr;
    int64_t ntri = 0;
    float bb[6];
    if (lbm_load_stl(s.stl.c_str(), &tris, &ntri, bb) != LBM_OK) {
        std::fprintf(stderr, "[error] failed to load STL: %s\n", s.stl.c_str());
        return mask;   // the run continues without an obstacle
    }
    lbm_voxel_params vp{};
    vp.nx = s.nx; vp.ny = s.ny; vp.nz = s.nz;
    vp.uniform_scale = s.voxel_scale;
    vp.translate[0] = s.voxel_tr[0]; vp.translate[1] = s.voxel_tr[1]; vp.translate[2] = s.voxel_tr[2];
    vp.refine = std::max(1, s.amr_factor);
    vp.coverage_threshold = std::clamp(s.amr_threshold, 0.0f, 1.0f);
    const int rc = lbm_voxelize(tris, ntri, bb, &vp, mask.data());
    lbm_free(tris);
    if (rc != LBM_OK) {
        std::fprintf(stderr, "[error] voxelizer: %s\n", lbm_last_error());
        std::fill(mask.begin(), mask.end(), 0);
    }
    return mask;
}

// y/z faces as wall cells (solid, not counted in the drag)
inline void add_walls(const Settings& s, std::vector<uint8_t>& mask) {
    for (int z = 0; z < s.nz; ++z)
        for (int y = 0; y < s.ny; ++y)
            if (y == 0 || y == s.ny - 1 || z == 0 || z == s.nz - 1)
                for (int x = 0; x < s.nx; ++x) {
                    uint8_t& m = mask[((size_t)z * s.ny + y) * s.nx + x];
                    if (!m) m = LBM_MASK_SOLID | LBM_MASK_WALL;
                }
}

// Initial density on the device (sim_common.hpp:242-260).
inline float* initial_rho(const Settings& s) {
    const size_t N = (size_t)s.nx * s.ny * s.nz;
    float* d = nullptr;
    if (cudaMalloc(&d, sizeof(float) * N) != cudaSuccess) return nullptr;
    if (s.init == "gauss") {
        make_rho_gauss(d, s.nx, s.ny, s.nz, s.center[0], s.center[1], s.center[2], s.sigma, s.amp);
    } else if (s.init == "slab") {
        make_rho_slab(d, s.nx, s.ny, s.nz, s.slab_axis, s.amp, s.slab_center, s.slab_width);
    } else {
        std::vector<float> ones(N, 1.0f);
        cudaMemcpy(d, ones.data(), sizeof(float) * N, cudaMemcpyHostToDevice);
    }
    cudaDeviceSynchronize();
    return d;
}

inline int fail(const char* what) {
    std::fprintf(stderr, "[error] %s: %s\n", what, lbm_last_error());
    return 1;
}

// The run of sim_runner.hpp:102-192 (Legacy/HOME) and :201-270 (Hybrid).
inline int run(const Settings& s, int method, const char* tag) {
    std::vector<uint8_t> mask = obstacle_mask(s);
    if (s.walls) add_walls(s, mask);

    lbm_domain d{s.nx, s.ny, s.nz, s.tau, s.fx, s.fy, s.fz};
    lbm_options o{};
    o.method = method;
    o.storage = s.storage;
    o.bc = s.bc;
    o.bounce = s.bounce;
    o.inlet_u = s.inlet_u;
    o.rho0 = 1.0f;
    lbm_solver* h = nullptr;
    if (lbm_create(&d, &o, &h) != LBM_OK) return fail("lbm_create");
    const int N = s.nx * s.ny * s.nz;
    if (lbm_set_solid_mask(h, mask.data()) != LBM_OK) return fail("set mask");
    if (method == LBM_METHOD_HYBRID && lbm_build_band(h, s.band_d0, nullptr) != LBM_OK) return fail("band");

    float* rho0 = initial_rho(s);
    if (!rho0) return fail("initial density");
    if (lbm_reinit_from_macro(h, rho0, nullptr, nullptr, nullptr) != LBM_OK) return fail("reinit");
    lbm_synchronize(h);
    cudaFree(rho0);

    // VTK directory (sim_common.hpp:269-283)
    bool vtk = !s.vtk_dir.empty() && s.vtk_every > 0;
    std::filesystem::path dir(s.vtk_dir);
    if (vtk) {
        std::error_code ec;
        std::filesystem::create_directories(dir, ec);
        if (ec) {
            std::fprintf(stderr, "[vtk] cannot create the output directory: %s (%s)\n", s.vtk_dir.c_str(),
                         ec.message().c_str());
            vtk = false;
        }
    }
    // snapshots: the text is formatted on the GPU, queued on the solver's
    // stream behind the step, and written by the writer's thread while the
    // next steps run (the reference formats on the host and waits)
    lbm_vtk_writer* writer = nullptr;
    void* stream = nullptr;
    lbm_solver_stream(h, &stream);
    if (vtk && lbm_vtk_writer_create(s.nx, s.ny, s.nz, 3, &writer) != LBM_OK) return fail("VTK writer");
    auto dump = [&](int step) {
        if (!vtk) return;
        float *r, *u, *v, *w;
        lbm_macro_ptrs(h, &r, &u, &v, &w);
        const std::string f_rho = vtk_file(dir, std::string("rho_") + tag, step);
        const std::string f_speed = vtk_file(dir, std::string("speed_") + tag, step);
        const std::string f_vel = vtk_file(dir, std::string("vel_") + tag, step);
        if (lbm_vtk_writer_submit(writer, LBM_VTK_SCALAR, r, nullptr, nullptr, f_rho.c_str(), stream) != LBM_OK ||
            lbm_vtk_writer_submit(writer, LBM_VTK_SPEED, u, v, w, f_speed.c_str(), stream) != LBM_OK ||
            lbm_vtk_writer_submit(writer, LBM_VTK_VECTOR, u, v, w, f_vel.c_str(), stream) != LBM_OK)
            std::fprintf(stderr, "[vtk] %s\n", lbm_last_error());
    };
    if (vtk) {
        std::printf("[vtk] %s: dir=%s every=%d\n", tag, dir.string().c_str(), s.vtk_every);
        dump(0);
    }
    if (method == LBM_METHOD_HYBRID)
        std::printf("[run] hybrid(B0)  d0=%d  Nx=%d Ny=%d Nz=%d  tau=%.4g  force=(%.3g,%.3g,%.3g)  steps=%d substeps=%d\n",
                    s.band_d0, s.nx, s.ny, s.nz, s.tau, s.fx, s.fy, s.fz, s.steps, s.substeps);
    else
        std::printf("[run] %s  Nx=%d Ny=%d Nz=%d  tau=%.4g  force=(%.3g,%.3g,%.3g)  steps=%d substeps=%d\n", tag,
                    s.nx, s.ny, s.nz, s.tau, s.fx, s.fy, s.fz, s.steps, s.substeps);
    std::fflush(stdout);

    for (int step = 1; step <= s.steps; ++step) {
        const bool stat = s.stats_every > 0 && step % s.stats_every == 0;
        if (stat) lbm_enable_stats(h, 1);
        if (lbm_step(h, s.substeps) != LBM_OK) return fail("step");
        if (stat) {
            double st[LBM_NSTAT];
            if (lbm_get_stats(h, st) != LBM_OK) return fail("stats");
            lbm_enable_stats(h, 0);
            std::printf("[stat] step=%d mass=%.12e ke_mean=%.12e drag=(%.9e,%.9e,%.9e)\n", step, st[LBM_STAT_MASS],
                        st[LBM_STAT_KE] / (double)N, st[LBM_STAT_DRAG_X], st[LBM_STAT_DRAG_Y], st[LBM_STAT_DRAG_Z]);
        }
        if (vtk && step % s.vtk_every == 0) dump(step);
    }
    if (lbm_synchronize(h) != LBM_OK) return fail("step");
    if (writer) {
        if (lbm_vtk_writer_flush(writer) != LBM_OK) std::fprintf(stderr, "[vtk] %s\n", lbm_last_error());
        lbm_vtk_writer_destroy(writer);
    }
    lbm_destroy(h);
    return 0;
}

// main() of the three tools: parse, optionally print, run.
inline int cli_main(int argc, char** argv, int method, const char* tag) {
    Settings s;
    parse_args(argc, argv, s, method == LBM_METHOD_HYBRID);
    if (s.print_config) {
        print_settings(s, stdout);
        return 0;
    }
    return run(s, method, tag);
}

}  // namespace fsim
