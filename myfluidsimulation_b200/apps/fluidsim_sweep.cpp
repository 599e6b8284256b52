// fluidsim_sweep: the headless B0 sweep of the reference's fluidsim_compare
// (`--hybrid-sweep-max M`, src/main_compare.cpp:505-699) on liblbm_b200,
// without its OpenGL viewer.
//
// For the obstacle of --stl it runs Legacy and HOME once and Hybrid(B0) for
// every d0 = 0..M, each for --hybrid-sweep-steps steps from the same initial
// density, and prints one CSV line per d0 with the reference's header and
// number formats: band size and ratio, mean |u| over the near-wall fluid cells
// (a 6-neighbour is solid, main_compare.cpp:359-386) per method, their mean
// absolute difference to Legacy, mean fluid density, and ms per step (CUDA
// events around the step loop).
//
// Flags kept from fluidsim_compare: --stl, --force (x) / --force-y / --force-z
// (and --forcey/--forcez), --init, --amp, --sigma, --center, --axis, --width,
// --amr, --amr-factor/--amr-refine, --amr-threshold, --hybrid-band/--hybrid-d0,
// --hybrid-sweep-max/--hybrid-sweep, --hybrid-sweep-steps/--sweep-steps.  The
// grid is fluidsim_compare's 200x150x120, tau 0.58, voxel scale 0.5 and
// translate 0.5; --nx/--ny/--nz/--tau/--voxel-scale/--voxel-translate override
// them and --bounce reference selects the reference's opposite table (flags
// with no reference counterpart).
//
// With halfway bounce-back (the default) all Hybrid runs of the sweep advance
// together through the batch (lbm_batch_*): one persistent launch per step over
// the M+1 instances, whose launch shape is tuned first.  Their fields are the
// same bits as one-by-one runs; ms_per_step_hybrid is then the batch's time per
// step divided by M+1.  --no-batch (or --bounce reference, which the batch
// does not take) runs and times them one at a time, as the reference does.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "lbm_capi.h"

namespace {

struct Args {
    int nx = 200, ny = 150, nz = 120;
    float tau = 0.58f;
    float fx = 0.f, fy = 0.f, fz = 0.f;
    std::string stl;
    std::string init = "none";
    float amp = 1e-3f, sigma = 0.08f, cen[3] = {0.6f, 0.5f, 0.5f}, width = 0.2f;
    int axis = 0;
    int amr = 1;
    float amr_thr = 0.5f;
    int band = 2, sweep_max = -1, sweep_steps = 500;
    float vscale = 0.5f, vtr[3] = {0.5f, 0.5f, 0.5f};
    int bounce = LBM_BOUNCE_HALFWAY;
    bool batch = true;
};

void parse(int argc, char** argv, Args& a) {
    for (int i = 1; i < argc; ++i) {
        const std::string s = argv[i];
        const bool v1 = i + 1 < argc;
        if (v1 && s == "--stl") a.stl = argv[++i];
        else if (v1 && s == "--force") a.fx = std::stof(argv[++i]);
        else if (v1 && (s == "--forcey" || s == "--force-y")) a.fy = std::stof(argv[++i]);
        else if (v1 && (s == "--forcez" || s == "--force-z")) a.fz = std::stof(argv[++i]);
        else if (v1 && s == "--init") a.init = argv[++i];
        else if (v1 && s == "--amp") a.amp = std::stof(argv[++i]);
        else if (v1 && s == "--sigma") a.sigma = std::stof(argv[++i]);
        else if (i + 3 < argc && s == "--center") {
            a.cen[0] = std::stof(argv[++i]); a.cen[1] = std::stof(argv[++i]); a.cen[2] = std::stof(argv[++i]);
        }
        else if (v1 && s == "--axis") {
            const char c = argv[++i][0];
            a.axis = c == 'y' ? 1 : (c == 'z' ? 2 : 0);
        }
        else if (v1 && s == "--width") a.width = std::stof(argv[++i]);
        else if (s == "--amr") a.amr = std::max(a.amr, 2);
        else if (v1 && (s == "--amr-factor" || s == "--amr-refine")) a.amr = std::stoi(argv[++i]);
        else if (v1 && s == "--amr-threshold") a.amr_thr = std::stof(argv[++i]);
        else if (v1 && (s == "--hybrid-band" || s == "--hybrid-d0")) a.band = std::max(0, std::stoi(argv[++i]));
        else if (v1 && (s == "--hybrid-sweep-max" || s == "--hybrid-sweep")) a.sweep_max = std::max(0, std::stoi(argv[++i]));
        else if (v1 && (s == "--hybrid-sweep-steps" || s == "--sweep-steps")) a.sweep_steps = std::max(0, std::stoi(argv[++i]));
        // extensions
        else if (v1 && s == "--nx") a.nx = std::max(8, std::stoi(argv[++i]));
        else if (v1 && s == "--ny") a.ny = std::max(8, std::stoi(argv[++i]));
        else if (v1 && s == "--nz") a.nz = std::max(1, std::stoi(argv[++i]));
        else if (v1 && s == "--tau") a.tau = std::max(0.51f, std::stof(argv[++i]));
        else if (v1 && s == "--voxel-scale") a.vscale = std::stof(argv[++i]);
        else if (i + 3 < argc && s == "--voxel-translate") {
            a.vtr[0] = std::stof(argv[++i]); a.vtr[1] = std::stof(argv[++i]); a.vtr[2] = std::stof(argv[++i]);
        }
        else if (s == "--no-batch") a.batch = false;
        else if (v1 && s == "--bounce") {
            const std::string b = argv[++i];
            a.bounce = b == "reference" ? LBM_BOUNCE_REFERENCE : LBM_BOUNCE_HALFWAY;
        }
    }
    if (a.amr < 1) a.amr = 1;
    a.amr_thr = std::clamp(a.amr_thr, 0.0f, 1.0f);
}

int die(const char* what) {
    std::fprintf(stderr, "[error] %s: %s\n", what, lbm_last_error());
    return 1;
}

struct Result {
    std::vector<float> speed;   // |u| at the near-wall cells
    double mean_u = 0, mean_rho = 0, ms = 0;
    int64_t band = 0;
};

}  // namespace

int main(int argc, char** argv) {
    Args a;
    parse(argc, argv, a);
    std::printf("[args] init=%s amp=%.3g sigma=%.3g center=(%.3f,%.3f,%.3f) axis=%d width=%.3f forceX=%.3g\n",
                a.init.c_str(), a.amp, a.sigma, a.cen[0], a.cen[1], a.cen[2], a.axis, a.width, a.fx);
    std::printf("[args] force=(%.3g, %.3g, %.3g)\n", a.fx, a.fy, a.fz);
    std::printf("[amr ] refine=%d threshold=%.2f\n", a.amr, a.amr_thr);
    if (a.sweep_max < 0) {
        std::fprintf(stderr, "[error] only the headless sweep is provided: pass --hybrid-sweep-max M\n");
        return 1;
    }
    const int64_t N = (int64_t)a.nx * a.ny * a.nz;
    std::vector<uint8_t> mask((size_t)N, 0);
    if (!a.stl.empty()) {
        float* tris = nullptr;
        int64_t ntri = 0;
        float bb[6];
        if (lbm_load_stl(a.stl.c_str(), &tris, &ntri, bb) != LBM_OK) {
            std::fprintf(stderr, "Failed to load STL: %s\n", a.stl.c_str());
            return 1;
        }
        lbm_voxel_params vp{};
        vp.nx = a.nx; vp.ny = a.ny; vp.nz = a.nz;
        vp.uniform_scale = a.vscale;
        for (int k = 0; k < 3; ++k) vp.translate[k] = a.vtr[k];
        vp.refine = a.amr;
        vp.coverage_threshold = a.amr_thr;
        const int rc = lbm_voxelize(tris, ntri, bb, &vp, mask.data());
        lbm_free(tris);
        if (rc != LBM_OK) return die("voxelize");
    }
    // near-wall fluid cells: a solid 6-neighbour inside the box (main_compare.cpp:359-386)
    std::vector<int64_t> near;
    int64_t nfluid = 0;
    for (int z = 0; z < a.nz; ++z)
        for (int y = 0; y < a.ny; ++y)
            for (int x = 0; x < a.nx; ++x) {
                const int64_t i = ((int64_t)z * a.ny + y) * a.nx + x;
                if (mask[i]) continue;
                ++nfluid;
                const int64_t sy = a.nx, sz = (int64_t)a.nx * a.ny;
                if ((x > 0 && mask[i - 1]) || (x < a.nx - 1 && mask[i + 1]) || (y > 0 && mask[i - sy]) ||
                    (y < a.ny - 1 && mask[i + sy]) || (z > 0 && mask[i - sz]) || (z < a.nz - 1 && mask[i + sz]))
                    near.push_back(i);
            }
    std::printf("[wall] near-wall fluid cells: %zu\n", near.size());
    {
        // band of the interactive d0 (main_compare.cpp:464-466)
        lbm_domain dom{a.nx, a.ny, a.nz, a.tau, a.fx, a.fy, a.fz};
        lbm_options o{};
        o.method = LBM_METHOD_HYBRID;
        o.rho0 = 1.0f;
        lbm_solver* s = nullptr;
        int64_t nb = 0;
        if (lbm_create(&dom, &o, &s) != LBM_OK || lbm_set_solid_mask(s, mask.data()) != LBM_OK ||
            lbm_build_band(s, a.band, &nb) != LBM_OK)
            return die("band");
        lbm_destroy(s);
        std::printf("[hybrid] B0 band d0=%d -> legacy cells=%d (fluid only)\n", a.band, (int)nb);
    }
    std::printf("[hybrid] B0 sweep enabled: d0=0..%d, steps_per_run=%d\n", a.sweep_max, a.sweep_steps);

    // initial density
    float* d_rho0 = nullptr;
    if (cudaMalloc(&d_rho0, sizeof(float) * N) != cudaSuccess) return die("cudaMalloc");
    if (a.init == "gauss") make_rho_gauss(d_rho0, a.nx, a.ny, a.nz, a.cen[0], a.cen[1], a.cen[2], a.sigma, a.amp);
    else if (a.init == "slab") make_rho_slab(d_rho0, a.nx, a.ny, a.nz, a.axis, a.amp, 0.5f, a.width);
    else {
        std::vector<float> ones((size_t)N, 1.0f);
        cudaMemcpy(d_rho0, ones.data(), sizeof(float) * N, cudaMemcpyHostToDevice);
    }
    cudaDeviceSynchronize();
    float* d_speed = nullptr;
    if (cudaMalloc(&d_speed, sizeof(float) * N) != cudaSuccess) return die("cudaMalloc");
    std::vector<float> h_speed((size_t)N), h_rho((size_t)N);
    cudaStream_t stream = nullptr;
    if (cudaStreamCreate(&stream) != cudaSuccess) return die("cudaStreamCreate");

    auto create = [&](int method, int d0, lbm_solver** out, int64_t* band) -> int {
        lbm_domain dom{a.nx, a.ny, a.nz, a.tau, a.fx, a.fy, a.fz};
        lbm_options o{};
        o.method = method;
        o.rho0 = 1.0f;
        o.bounce = a.bounce;
        o.stream = stream;
        lbm_solver* s = nullptr;
        if (lbm_create(&dom, &o, &s) != LBM_OK) return die("lbm_create");
        *out = s;
        if (lbm_set_solid_mask(s, mask.data()) != LBM_OK) return die("mask");
        if (method == LBM_METHOD_HYBRID && lbm_build_band(s, d0, band) != LBM_OK) return die("band");
        if (lbm_reinit_from_macro(s, d_rho0, nullptr, nullptr, nullptr) != LBM_OK) return die("reinit");
        return 0;
    };
    // |u| at the near-wall cells and the mean fluid density (main_compare.cpp:572-591)
    auto measure = [&](lbm_solver* s, Result& r) {
        float *rho, *u, *v, *w;
        lbm_macro_ptrs(s, &rho, &u, &v, &w);
        launch_speed(u, v, w, d_speed, (int)N);
        cudaMemcpy(h_speed.data(), d_speed, sizeof(float) * N, cudaMemcpyDeviceToHost);
        cudaMemcpy(h_rho.data(), rho, sizeof(float) * N, cudaMemcpyDeviceToHost);
        r.speed.resize(near.size());
        double su = 0.0;
        for (size_t k = 0; k < near.size(); ++k) {
            r.speed[k] = h_speed[near[k]];
            su += (double)r.speed[k];
        }
        r.mean_u = su / (near.empty() ? 1.0 : (double)near.size());
        double sr = 0.0;
        for (int64_t i = 0; i < N; ++i)
            if (!mask[i]) sr += (double)h_rho[i];
        r.mean_rho = nfluid > 0 ? sr / (double)nfluid : 0.0;
    };
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto elapsed = [&]() {
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        return (double)ms;
    };
    // one solver at a time, step(1) per step, timed by events around the loop
    auto run = [&](int method, int d0, Result& r) -> int {
        lbm_solver* s = nullptr;
        if (create(method, d0, &s, &r.band)) return 1;
        lbm_synchronize(s);
        cudaEventRecord(e0, stream);
        for (int k = 0; k < a.sweep_steps; ++k)
            if (lbm_step(s, 1) != LBM_OK) return die("step");
        cudaEventRecord(e1, stream);
        if (lbm_synchronize(s) != LBM_OK) return die("step");
        r.ms = a.sweep_steps > 0 ? elapsed() / a.sweep_steps : 0.0;
        measure(s, r);
        lbm_destroy(s);
        return 0;
    };
    // every d0 at once: one persistent launch per step over all instances
    auto run_batch = [&](std::vector<Result>& rs) -> int {
        const int n = (int)rs.size();
        std::vector<lbm_solver*> ss((size_t)n, nullptr);
        for (int d0 = 0; d0 < n; ++d0)
            if (create(LBM_METHOD_HYBRID, d0, &ss[d0], &rs[d0].band)) return 1;
        lbm_batch* b = nullptr;
        if (lbm_batch_create(ss.data(), n, stream, &b) != LBM_OK) return die("lbm_batch_create");
        // launch shape: timed on the instances themselves, which then restart
        if (lbm_batch_tune(b, 2, nullptr) != LBM_OK) return die("lbm_batch_tune");
        for (lbm_solver* s : ss)
            if (lbm_reinit_from_macro(s, d_rho0, nullptr, nullptr, nullptr) != LBM_OK) return die("reinit");
        if (lbm_batch_refresh(b) != LBM_OK) return die("lbm_batch_refresh");
        lbm_batch_synchronize(b);
        lbm_batch_enable_stats(b, 0);
        cudaEventRecord(e0, stream);
        for (int k = 0; k < a.sweep_steps; ++k) {
            if (k == a.sweep_steps - 1) lbm_batch_enable_stats(b, 1);   // fields of the last step
            if (lbm_batch_step(b, 1) != LBM_OK) return die("lbm_batch_step");
        }
        cudaEventRecord(e1, stream);
        if (lbm_batch_synchronize(b) != LBM_OK) return die("lbm_batch_step");
        const double ms = a.sweep_steps > 0 ? elapsed() / a.sweep_steps / n : 0.0;
        lbm_batch_destroy(b);
        for (int d0 = 0; d0 < n; ++d0) {
            rs[d0].ms = ms;
            measure(ss[d0], rs[d0]);
            lbm_destroy(ss[d0]);
        }
        return 0;
    };
    auto absdiff = [&](const Result& r, const Result& base) {
        double sa = 0.0;
        for (size_t k = 0; k < near.size(); ++k) sa += std::fabs((double)r.speed[k] - (double)base.speed[k]);
        return sa / (near.empty() ? 1.0 : (double)near.size());
    };

    Result leg, home;
    if (run(LBM_METHOD_LEGACY, 0, leg) || run(LBM_METHOD_HOME, 0, home)) return 1;
    const double ad_home = absdiff(home, leg);
    std::printf("d0,legacy_cells,legacy_ratio,"
                "mean_u_legacy,mean_u_home,mean_u_hybrid,"
                "mean_absdiff_home,mean_absdiff_hybrid,"
                "mean_rho_legacy,mean_rho_home,mean_rho_hybrid,"
                "absdiff_rho_home,absdiff_rho_hybrid,"
                "ms_per_step_legacy,ms_per_step_home,ms_per_step_hybrid,"
                "amr_factor,amr_threshold,fluid_cells,near_wall_cells\n");
    // the batch needs halfway bounce-back, an even cell count and room for every
    // instance at once (about 99 bytes per cell each)
    std::vector<Result> hys;
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    const double need = 110.0 * (double)N * (a.sweep_max + 1);
    const bool batched = a.batch && a.bounce == LBM_BOUNCE_HALFWAY && a.sweep_steps > 0 && N % 2 == 0 &&
                         need < 0.8 * (double)free_b;
    if (batched) {
        hys.resize((size_t)a.sweep_max + 1);
        if (run_batch(hys)) return 1;
    }
    for (int d0 = 0; d0 <= a.sweep_max; ++d0) {
        Result hy;
        if (batched) hy = hys[d0];
        else if (run(LBM_METHOD_HYBRID, d0, hy)) return 1;
        const double ratio = nfluid > 0 ? (double)hy.band / (double)nfluid : 0.0;
        std::printf("%d,%d,%.6f,%.9e,%.9e,%.9e,%.9e,%.9e,%.9e,%.9e,%.9e,%.9e,%.9e,%.6f,%.6f,%.6f,%d,%.6f,%d,%zu\n", d0,
                    (int)hy.band, ratio, leg.mean_u, home.mean_u, hy.mean_u, ad_home, absdiff(hy, leg), leg.mean_rho,
                    home.mean_rho, hy.mean_rho, std::fabs(home.mean_rho - leg.mean_rho),
                    std::fabs(hy.mean_rho - leg.mean_rho), leg.ms, home.ms, hy.ms, a.amr, (double)a.amr_thr,
                    (int)nfluid, near.size());
        std::fflush(stdout);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d_speed);
    cudaFree(d_rho0);
    cudaStreamDestroy(stream);
    return 0;
}
