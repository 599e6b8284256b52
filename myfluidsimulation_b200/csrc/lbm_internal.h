// Internal interfaces between the translation units of liblbm_b200.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace lbm {

// number of FP64 statistics slots (see LBM_STAT_* in lbm_capi.h)
constexpr int NSTAT = 8;

// Parameters of one AA-pattern step (Legacy / Hybrid).
struct AAParams {
    void* f;                 // 19 planes of N cells, storage type per `storage`
    int64_t N;
    int nx, ny, nz;
    const uint8_t* flags;    // nullptr: no solid cells anywhere
    const uint32_t* links;   // bit q: link x -> x+c_q does not stream (solid / inlet / outlet)
    float omega;             // BGK rate (Legacy, and the band cells of Hybrid)
    float omega_h, omega_s;  // Hybrid non-band cells: fq + wh(feq-fq) + (ws-wh)(-(fq-feq))
    int hybrid;              // 1: consult F_BAND; 0: BGK form everywhere
    float fx, fy, fz;
    int duct;                // 1: x non-periodic with inlet/outlet
    float u_in;
    float rho0;              // storage shift reference (F16/BF16)
    float* rho; float* ux; float* uy; float* uz;   // macro outputs (written when macro != 0)
    int macro;
    double* partials;        // [gridDim.x][NSTAT] when stats != 0
    int stats;
    // cells stepped by aa_even / aa_odd: [first, first + cells), whole planes;
    // all N, or the interior planes of a z-slab whose first and last planes are
    // ghost copies of the neighbouring slabs' boundary planes
    int64_t first, cells;
    uint32_t salt_base;      // F16/BF16 stochastic rounding: index of cell 0 in the whole grid
    int zrun;                // odd step: planes per block (set by launch_aa_step)
};

// Parameters of one HOME step (moment-only, two buffers).
struct HomeParams {
    const void* m;           // 10 planes [rho,ux,uy,uz,Sxx,Sxy,Sxz,Syy,Syz,Szz]
    void* mn;
    int64_t N;
    int nx, ny, nz;
    const uint8_t* flags;
    const uint32_t* links;
    float omega;
    float fx, fy, fz;
    int duct;
    float u_in;
    float rho0;
    double* partials;
    int stats;
    int zchunk;              // planes per block
    int ref_bounce;          // 1: the reference's opposite table for reflections
    int zb, ze;              // planes stepped: [zb, ze) (all, or a z-slab's interior)
    uint32_t salt_base;      // added to a cell's index in the stochastic-rounding salt:
                             // a slab passes its plane 0's index in the whole grid
};

// Launch configuration chosen by the host (autotuner or defaults).
struct LaunchCfg {
    int blocks;
    int threads;
};

// AA steps.  parity 0: natural layout in (the even, purely local step);
// parity 1: the odd step (gathers from and scatters to neighbours).
cudaError_t launch_aa_step(const AAParams& p, int storage, int parity, LaunchCfg cfg, cudaStream_t s);
// the odd step's grid: blocks of `threads` cells of one row, each over a run of
// aa_odd_zrun planes; one statistics partial per block
int aa_odd_zrun(int nx, int ny, int64_t planes, bool mask, int storage, int threads);
int64_t aa_odd_blocks(int nx, int ny, int64_t planes, bool mask, int storage, int threads);
// blocks of one odd-step launch: the z-marching grid without a mask; with one,
// cfg.blocks rounded down to a multiple of the row segments (a 2-D grid of
// rows x segments)
int64_t aa_odd_grid(int nx, int ny, int64_t planes, bool mask, int storage, LaunchCfg cfg);
// One step of many instances in one persistent launch (FP32 populations, the
// instances' flag bytes required); units: {instance, first, count, -} with
// first/count in two-cell vectors (parity 0) or cells (parity 1).  stats != 0 writes NSTAT sums per unit into partials.
cudaError_t launch_aa_batch(const AAParams* d_inst, const int4* d_units, int nunits, int parity, int stats,
                            int storage, int blocks, int threads, double* partials, cudaStream_t s);
// per-instance sums of the unit partials: units of instance i are first[i]..first[i+1]-1
cudaError_t launch_batch_finalize(const double* partials, const int* d_first, int n, double* out, cudaStream_t s);
// Reference-compatible Legacy/Hybrid step (two buffers, the reference's
// opposite table): fa -> fb.
cudaError_t launch_ref_push(const AAParams& p, const float* fa, float* fb, LaunchCfg cfg, cudaStream_t s);
// Copies the populations into the reference's natural layout (float, 19*N)
// whatever the parity, without advancing.
cudaError_t launch_aa_materialize(const AAParams& p, int storage, int parity, float* out, cudaStream_t s);
// sets the dynamic shared-memory limit of the HOME kernels (call outside graph capture)
cudaError_t home_prepare();
int home_num_blocks(int nx, int ny, int nz, int zchunk);
// resident HOME blocks per SM (occupancy of the FP32 step kernel)
int home_blocks_per_sm();
cudaError_t launch_home_step(const HomeParams& p, int storage, int tile_y, int blocks_per_sm, cudaStream_t s);
// HOME moments (storage type) -> float 10*N
cudaError_t launch_home_export(const void* m, int storage, int64_t N, float rho0, float* out, cudaStream_t s);
// macro pointers of a HOME state in F16/BF16 are exported to float buffers
cudaError_t launch_home_macros(const void* m, int storage, int64_t N, float rho0,
                               float* rho, float* ux, float* uy, float* uz, cudaStream_t s);

// initialisation
cudaError_t launch_aa_reinit(void* f, int storage, float rho0, int64_t N,
                             const float* rho, const float* ux, const float* uy, const float* uz,
                             float* rho_out, float* ux_out, float* uy_out, float* uz_out,
                             int feq_form, cudaStream_t s);
cudaError_t launch_home_reinit(void* m, void* mn, int storage, float rho0, int64_t N,
                               const float* rho, const float* ux, const float* uy, const float* uz,
                               cudaStream_t s);

// flags / links / band
cudaError_t launch_build_flags(const uint8_t* mask, const uint8_t* band, uint8_t* flags, uint32_t* links,
                               int nx, int ny, int nz, int duct, cudaStream_t s);
cudaError_t launch_band(const uint8_t* mask, int32_t* dist, uint8_t* band, int nx, int ny, int nz, int d0,
                        unsigned long long* count, cudaStream_t s);
cudaError_t launch_finalize_stats(const double* partials, int nblocks, double* out, cudaStream_t s);

// geometry
cudaError_t launch_voxelize(const float* d_tris, int64_t ntri, const float* bb, int nx, int ny, int nz,
                            float scale, const float* translate, int refine, float thr, uint8_t* d_mask,
                            cudaStream_t s);

int num_sms();

}  // namespace lbm
