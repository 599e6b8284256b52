// fluidsim_tgv: drop-in for the reference's Taylor-Green vortex bench
// (src/bench/main_taylor_green.cpp:29-350) on liblbm_b200.  Legacy and HOME
// advance in lock-step from the same analytic initial fields; every
// --sample-every steps both are compared with the analytic decay on the host
// in FP64 (mean kinetic energy, velocity L2 and Linf), printed as "[step]"
// lines and written to the CSV with the reference's header and formatting.
//
// Flags kept from the reference: --nx --ny --nz --steps --sample-every --u0
// --tau --k/--wavenumber --vtk-dir --vtk-every/--vtk-interval --csv.
// Added: --precision f32|f16|bf16 (storage of both solvers) and --tgv3d (the
// 3-D vortex u=u0 sin(kx)cos(ky)cos(kz), v=-u0 cos(kx)sin(ky)cos(kz), w=0,
// p=rho0 u0^2/16 (cos2kx+cos2ky)(cos2kz+2), rho=1+3p, with k=2*pi*k/N per
// axis; its "exact" columns are the small-Reynolds-number decay
// exp(-nu k^2 t) of the velocity with k^2 summed over the three axes).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <string>
#include <vector>

#include "lbm_capi.h"

namespace {

constexpr double kPi = 3.14159265358979323846;

struct Tgv {
    int nx = 128, ny = 128, nz = 16;
    int steps = 400, sample_every = 10;
    double tau = 0.58, u0 = 0.06, k = 1.0;
    std::string vtk_dir;
    int vtk_every = 0;
    std::string csv = "out_vtk/tgv_results.csv";
    int storage = LBM_STORE_F32;
    bool three_d = false;
    // derived
    double cs2 = 1.0 / 3.0, kxw = 0, kyw = 0, kzw = 0, k2 = 0, nu = 0;
    int n = 0;
};

struct Exact {
    double u, v, w, rho;
};

// Analytic field at the cell centre (i + 0.5), main_taylor_green.cpp:68-87.
Exact exact(const Tgv& c, int x, int y, int z, double t) {
    const double tx = (x + 0.5) * c.kxw, ty = (y + 0.5) * c.kyw;
    const double dv = std::exp(-c.nu * c.k2 * t), dr = std::exp(-2.0 * c.nu * c.k2 * t);
    Exact e{};
    if (!c.three_d) {
        e.u = c.u0 * std::sin(tx) * std::cos(ty) * dv;
        e.v = -c.u0 * std::cos(tx) * std::sin(ty) * dv;
        e.w = 0.0;
        e.rho = 1.0 + (c.u0 * c.u0 * dr / (4.0 * c.cs2)) * (std::cos(2.0 * tx) + std::cos(2.0 * ty));
    } else {
        const double tz = (z + 0.5) * c.kzw;
        e.u = c.u0 * std::sin(tx) * std::cos(ty) * std::cos(tz) * dv;
        e.v = -c.u0 * std::cos(tx) * std::sin(ty) * std::cos(tz) * dv;
        e.w = 0.0;
        const double p = c.u0 * c.u0 / 16.0 * (std::cos(2.0 * tx) + std::cos(2.0 * ty)) * (std::cos(2.0 * tz) + 2.0) * dr;
        e.rho = 1.0 + p / c.cs2;
    }
    return e;
}

double exact_energy(const Tgv& c, double t) {
    // mean of |u|^2/2 over the periodic box: u0^2/4 (2-D), u0^2/8 (3-D)
    return (c.three_d ? 0.125 : 0.25) * c.u0 * c.u0 * std::exp(-2.0 * c.nu * c.k2 * t);
}

struct Sample {
    double energy = 0, l2 = 0, linf = 0;
};

struct Row {
    int step;
    double time, e_exact;
    Sample legacy, home;
};

void parse(int argc, char** argv, Tgv& c) {
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        const bool v1 = i + 1 < argc;
        if (v1 && a == "--nx") c.nx = std::stoi(argv[++i]);
        else if (v1 && a == "--ny") c.ny = std::stoi(argv[++i]);
        else if (v1 && a == "--nz") c.nz = std::stoi(argv[++i]);
        else if (v1 && a == "--steps") c.steps = std::stoi(argv[++i]);
        else if (v1 && a == "--sample-every") c.sample_every = std::stoi(argv[++i]);
        else if (v1 && a == "--u0") c.u0 = std::stod(argv[++i]);
        else if (v1 && a == "--tau") c.tau = std::stod(argv[++i]);
        else if (v1 && (a == "--k" || a == "--wavenumber")) c.k = std::stod(argv[++i]);
        else if (v1 && a == "--vtk-dir") c.vtk_dir = argv[++i];
        else if (v1 && (a == "--vtk-every" || a == "--vtk-interval")) c.vtk_every = std::stoi(argv[++i]);
        else if (v1 && a == "--csv") c.csv = argv[++i];
        else if (v1 && a == "--precision") {
            const std::string p = argv[++i];
            c.storage = p == "f16" ? LBM_STORE_F16 : (p == "bf16" ? LBM_STORE_BF16 : LBM_STORE_F32);
        } else if (a == "--tgv3d") c.three_d = true;
    }
    // clamps of main_taylor_green.cpp:243-248
    if (c.sample_every <= 0) c.sample_every = 1;
    if (c.vtk_every < 0) c.vtk_every = 0;
    if (c.nz <= 0) c.nz = 1;
    if (c.nx <= 0) c.nx = 16;
    if (c.ny <= 0) c.ny = 16;
    if (c.steps < 0) c.steps = 0;
    c.n = c.nx * c.ny * c.nz;
    c.kxw = 2.0 * kPi * c.k / c.nx;
    c.kyw = 2.0 * kPi * c.k / c.ny;
    c.kzw = 2.0 * kPi * c.k / c.nz;
    c.k2 = c.kxw * c.kxw + c.kyw * c.kyw + (c.three_d ? c.kzw * c.kzw : 0.0);
    c.nu = (c.tau - 0.5) * c.cs2;
}

void die(const char* what) {
    std::cerr << "[error] " << what << ": " << lbm_last_error() << "\n";
    std::exit(1);
}

lbm_solver* make(const Tgv& c, int method, const std::vector<float>& r, const std::vector<float>& u,
                 const std::vector<float>& v, const std::vector<float>& w) {
    lbm_domain d{c.nx, c.ny, c.nz, (float)c.tau, 0.f, 0.f, 0.f};
    lbm_options o{};
    o.method = method;
    o.storage = c.storage;
    o.rho0 = 1.0f;
    lbm_solver* h = nullptr;
    if (lbm_create(&d, &o, &h) != LBM_OK) die("lbm_create");
    const std::vector<uint8_t> mask((size_t)c.n, 0);
    if (lbm_set_solid_mask(h, mask.data()) != LBM_OK) die("set mask");
    if (lbm_reinit_from_host(h, r.data(), u.data(), v.data(), w.data()) != LBM_OK) die("reinit");
    return h;
}

Sample sample(lbm_solver* h, const Tgv& c, double t, std::vector<float>& r, std::vector<float>& u,
              std::vector<float>& v, std::vector<float>& w) {
    if (lbm_get_macros(h, r.data(), u.data(), v.data(), w.data()) != LBM_OK) die("read macros");
    double e = 0, err2 = 0, emax = 0;
    size_t id = 0;
    for (int z = 0; z < c.nz; ++z)
        for (int y = 0; y < c.ny; ++y)
            for (int x = 0; x < c.nx; ++x, ++id) {
                const Exact a = exact(c, x, y, z, t);
                const double du = (double)u[id] - a.u, dv = (double)v[id] - a.v, dw = (double)w[id] - a.w;
                const double q = du * du + dv * dv + dw * dw;
                err2 += q;
                emax = std::max(emax, std::sqrt(q));
                const double U = u[id], V = v[id], W = w[id];
                e += 0.5 * (U * U + V * V + W * W);
            }
    Sample s;
    s.energy = e / c.n;
    s.l2 = std::sqrt(err2 / c.n);
    s.linf = emax;
    return s;
}

std::string vtk_name(const std::string& stem, int step) {
    char b[64];
    std::snprintf(b, sizeof(b), "%s_%06d.vtk", stem.c_str(), step);
    return b;
}

}  // namespace

int main(int argc, char** argv) {
    Tgv c;
    parse(argc, argv, c);

    std::cout << "[cfg ] Nx=" << c.nx << " Ny=" << c.ny << " Nz=" << c.nz << " steps=" << c.steps
              << " sample=" << c.sample_every << "\n";
    std::cout << "[cfg ] tau=" << c.tau << " nu=" << c.nu << " u0=" << c.u0 << " kx_wave=" << c.kxw
              << " ky_wave=" << c.kyw << " k^2=" << c.k2 << "\n";
    if (!c.vtk_dir.empty()) std::cout << "[cfg ] vtk dir=" << c.vtk_dir << " every=" << c.vtk_every << " steps\n";
    std::cout << "[cfg ] csv=" << c.csv << "\n";

    std::vector<float> r((size_t)c.n), u((size_t)c.n), v((size_t)c.n), w((size_t)c.n, 0.0f);
    {
        size_t id = 0;
        for (int z = 0; z < c.nz; ++z)
            for (int y = 0; y < c.ny; ++y)
                for (int x = 0; x < c.nx; ++x, ++id) {
                    const Exact a = exact(c, x, y, z, 0.0);
                    r[id] = (float)a.rho;
                    u[id] = (float)a.u;
                    v[id] = (float)a.v;
                }
    }
    lbm_solver* legacy = make(c, LBM_METHOD_LEGACY, r, u, v, w);
    lbm_solver* home = make(c, LBM_METHOD_HOME, r, u, v, w);

    const bool vtk = !c.vtk_dir.empty() && c.vtk_every > 0;
    float *sp_l = nullptr, *sp_h = nullptr;
    if (vtk && (cudaMalloc(&sp_l, sizeof(float) * c.n) != cudaSuccess ||
                cudaMalloc(&sp_h, sizeof(float) * c.n) != cudaSuccess)) {
        std::cerr << "[error] cudaMalloc failed\n";
        return 1;
    }
    auto dump = [&](int step) {
        if (!vtk) return;
        std::filesystem::create_directories(c.vtk_dir);
        const std::filesystem::path dir(c.vtk_dir);
        float *lr, *lu, *lv, *lw, *hr, *hu, *hv, *hw;
        lbm_macro_ptrs(legacy, &lr, &lu, &lv, &lw);
        lbm_macro_ptrs(home, &hr, &hu, &hv, &hw);
        launch_speed(lu, lv, lw, sp_l, c.n);
        launch_speed(hu, hv, hw, sp_h, c.n);
        write_scalar_vtk((dir / vtk_name("rho_legacy", step)).string().c_str(), lr, c.nx, c.ny, c.nz);
        write_scalar_vtk((dir / vtk_name("rho_home", step)).string().c_str(), hr, c.nx, c.ny, c.nz);
        write_scalar_vtk((dir / vtk_name("speed_legacy", step)).string().c_str(), sp_l, c.nx, c.ny, c.nz);
        write_scalar_vtk((dir / vtk_name("speed_home", step)).string().c_str(), sp_h, c.nx, c.ny, c.nz);
        write_vector_vtk((dir / vtk_name("vel_legacy", step)).string().c_str(), lu, lv, lw, c.nx, c.ny, c.nz);
        write_vector_vtk((dir / vtk_name("vel_home", step)).string().c_str(), hu, hv, hw, c.nx, c.ny, c.nz);
    };

    std::vector<Row> rows;
    auto sample_now = [&](int step) {
        const double t = step;
        Row row{step, t, exact_energy(c, t), {}, {}};
        row.legacy = sample(legacy, c, t, r, u, v, w);
        row.home = sample(home, c, t, r, u, v, w);
        std::cout << "[step " << std::setw(5) << step << "] "
                  << "E_exact=" << std::setw(12) << row.e_exact << "  E_L=" << std::setw(12) << row.legacy.energy
                  << "  E_H=" << std::setw(12) << row.home.energy << "  L2_L=" << row.legacy.l2
                  << "  L2_H=" << row.home.l2 << "\n";
        if (c.vtk_every > 0 && step % c.vtk_every == 0) dump(step);
        rows.push_back(row);
    };

    sample_now(0);
    for (int step = 1; step <= c.steps; ++step) {
        // both solvers advance on their own streams; the sample reads synchronise
        if (lbm_step(legacy, 1) != LBM_OK || lbm_step(home, 1) != LBM_OK) die("step");
        if (step % c.sample_every == 0 || step == c.steps) sample_now(step);
    }

    // CSV, main_taylor_green.cpp:192-208
    std::ofstream csv(c.csv);
    csv << "step,time,energy_exact,energy_legacy,energy_home,l2_legacy,l2_home,linf_legacy,linf_home\n";
    csv << std::scientific << std::setprecision(8);
    for (const Row& x : rows)
        csv << x.step << "," << x.time << "," << x.e_exact << "," << x.legacy.energy << "," << x.home.energy << ","
            << x.legacy.l2 << "," << x.home.l2 << "," << x.legacy.linf << "," << x.home.linf << "\n";
    std::cout << "[write] saved " << rows.size() << " samples to " << c.csv << "\n";

    if (sp_l) cudaFree(sp_l);
    if (sp_h) cudaFree(sp_h);
    lbm_destroy(legacy);
    lbm_destroy(home);
    return 0;
}
