/*
 * lbm_capi.h -- C-ABI of the B200-native D3Q19 lattice-Boltzmann library
 * (liblbm_b200.so).  Plain pointers and sizes only; every call returns an int
 * status (LBM_OK == 0) and never throws; lbm_last_error() holds the message of
 * the last failure on the calling thread.
 *
 * Each entry cites the reference interface (yagise/MyFluidSimulation, path
 * inside that project) that it replaces.  The reference's solver classes
 * LBM3D_Legacy / LBM3D_Home / LBM3D_Hybrid map onto one opaque lbm_solver
 * created with a method; include/lbm3d_compat.hpp rebuilds those classes on
 * top of this ABI for C++ callers.
 *
 * Threading and streams: a solver is bound to one CUDA stream (its own, or
 * the one passed in lbm_options.stream) and is not thread-safe.  lbm_step is
 * asynchronous on that stream; lbm_synchronize waits for it.  Device pointers
 * returned by getters are borrowed and stay valid until the next lbm_step,
 * lbm_reset/lbm_reinit_from_macro or lbm_destroy (the HOME method swaps its
 * moment buffers on every step, as the reference does).
 */
#ifndef LBM_CAPI_H
#define LBM_CAPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
enum {
    LBM_OK = 0,
    LBM_ERR_INVALID = 1,      /* bad argument, size or state */
    LBM_ERR_CUDA = 2,         /* a CUDA runtime call failed */
    LBM_ERR_ALLOC = 3,        /* device or host allocation failed */
    LBM_ERR_SIZE = 4,         /* a size overflows the supported range */
    LBM_ERR_IO = 5,           /* file could not be read or written */
    LBM_ERR_UNSUPPORTED = 6,  /* combination not implemented */
    LBM_ERR_TIMEOUT = 7       /* a bounded device-side wait gave up */
};

/* collision / update method (the reference's three solver classes) */
enum { LBM_METHOD_LEGACY = 0, LBM_METHOD_HOME = 1, LBM_METHOD_HYBRID = 2 };
/* storage of populations (Legacy/Hybrid) or moments (HOME).
 * F16/BF16 keep shifted values (f - w_q rho0; HOME: rho - rho0, u, S) and
 * compute in FP32.  F64 stores and computes in FP64: the reference form the
 * others are measured against (Legacy/Hybrid with halfway bounce-back; HOME). */
enum { LBM_STORE_F32 = 0, LBM_STORE_F16 = 1, LBM_STORE_BF16 = 2, LBM_STORE_F64 = 3 };
/* boundary: fully periodic (the reference), or a duct along x with a
 * velocity inlet at x=0 and a zero-gradient outlet at x=Nx-1 */
enum { LBM_BC_PERIODIC = 0, LBM_BC_DUCT = 1 };
/* bounce-back at solid cells.
 * HALFWAY: link-wise halfway bounce-back, a population leaving along c_q comes
 *   back along -c_q (every population written once per step; the in-place
 *   AA kernels).
 * REFERENCE: the reference's own opposite table (src/lbm/lbm3d_legacy.cu:29-32),
 *   which pairs each diagonal direction with its mirror image in x or y
 *   rather than its opposite.  Legacy/Hybrid then keep the reference's two
 *   buffers: a slot nobody writes keeps the previous buffer's value, and a slot
 *   written both by streaming and by a reflection (a race in the reference)
 *   takes the reflection.  HOME uses the table deterministically, as the
 *   reference does.  F32 storage only for Legacy/Hybrid. */
enum { LBM_BOUNCE_HALFWAY = 0, LBM_BOUNCE_REFERENCE = 1 };
/* mask byte: any nonzero value is solid (the reference's convention);
 * bit 3 marks a solid cell as a wall that the drag sum leaves out */
enum { LBM_MASK_SOLID = 1, LBM_MASK_WALL = 8 };
/* lbm_get_stats slots */
enum {
    LBM_STAT_MASS = 0,   /* sum of rho over fluid cells */
    LBM_STAT_KE = 1,     /* sum over all cells of |u|^2/2 (divide by N for the mean) */
    LBM_STAT_DRAG_X = 2, /* momentum exchanged with obstacle cells in one step */
    LBM_STAT_DRAG_Y = 3,
    LBM_STAT_DRAG_Z = 4,
    LBM_STAT_MOM_X = 5,  /* sum of rho*u over fluid cells */
    LBM_STAT_MOM_Y = 6,
    LBM_STAT_MOM_Z = 7,
    LBM_NSTAT = 8
};

/* Mirrors struct Domain (src/lbm/lbm_common.hpp:6-10). */
typedef struct lbm_domain {
    int32_t nx, ny, nz;
    float tau;
    float force_x, force_y, force_z;
} lbm_domain;

typedef struct lbm_options {
    int32_t method;    /* LBM_METHOD_* */
    int32_t storage;   /* LBM_STORE_* */
    int32_t bc;        /* LBM_BC_* */
    int32_t bounce;    /* LBM_BOUNCE_* */
    float inlet_u;     /* duct inlet velocity (x) */
    float rho0;        /* reference density of the shifted F16/BF16 storage (default 1) */
    void* stream;      /* cudaStream_t to run on; NULL creates one per solver */
} lbm_options;

typedef struct lbm_solver lbm_solver;

/* Last error message of the calling thread ("" when none). */
const char* lbm_last_error(void);
/* Library version string. */
const char* lbm_version(void);

/* ---- solver lifecycle -------------------------------------------------- */

/* Allocates and resets a solver (rho=1, u=0 equilibrium, no solid cells;
 * with LBM_BOUNCE_REFERENCE the second population buffer starts as zeros).
 * Replaces LBM3D_Legacy::init (src/lbm/lbm3d_legacy.cu:141-147),
 * LBM3D_Home::init (src/lbm/lbm3d_home.cu:301-307) and
 * LBM3D_Hybrid::init (src/lbm/lbm3d_hybrid.cu:210-221). opts may be NULL
 * (Legacy, F32, periodic). */
int lbm_create(const lbm_domain* dom, const lbm_options* opts, lbm_solver** out);
/* Replaces the destructors (~LBM3D_*, lbm3d_legacy.cu:14, home.cu:5, hybrid.cu:5). */
int lbm_destroy(lbm_solver* s);

/* Nx*Ny*Nz bytes, x fastest.  Replaces setSolidMask (lbm3d_legacy.cu:149-151,
 * lbm3d_home.cu:309-311, lbm3d_hybrid.cu:223-225). */
int lbm_set_solid_mask(lbm_solver* s, const uint8_t* host_mask);
/* Hybrid only: per-cell BGK-band flags (NULL clears the band).  Replaces
 * LBM3D_Hybrid::setLegacyMapping (lbm3d_hybrid.cu:227-235); the reference's
 * second (slot) argument is ignored there and has no counterpart here. */
int lbm_set_legacy_mapping(lbm_solver* s, const uint8_t* host_is_legacy);
/* Hybrid only: builds the band on the GPU from the current mask, exactly as
 * build_distance_to_solid_6n + build_legacy_mask_from_distance
 * (src/apps/sim_runner.hpp:28-91) with maxDist=max(1,d0) (sim_runner.hpp:221-224).
 * n_band (may be NULL) receives the number of band cells. */
int lbm_build_band(lbm_solver* s, int d0, int64_t* n_band);
/* Copies the band flags out (Nx*Ny*Nz bytes, 1 = BGK band). */
int lbm_get_band(lbm_solver* s, uint8_t* host_is_legacy);

/* rho=1, u=0 equilibrium.  Replaces reset() (lbm3d_legacy.cu:153-159,
 * lbm3d_home.cu:313-319, lbm3d_hybrid.cu:237-243). */
int lbm_reset(lbm_solver* s);
/* Equilibrium from DEVICE macro fields; NULL velocity components are 0.
 * NULL rho: Legacy resets (lbm3d_legacy.cu:174-178), HOME and Hybrid use rho=1
 * (lbm3d_home.cu:119, lbm3d_hybrid.cu:76).  Replaces reinitEquilibriumFromMacro
 * (lbm3d_legacy.cu:160-208, lbm3d_home.cu:321-333, lbm3d_hybrid.cu:245-257). */
int lbm_reinit_from_macro(lbm_solver* s, const float* d_rho, const float* d_ux,
                          const float* d_uy, const float* d_uz);
/* Same, from HOST arrays (each Nx*Ny*Nz floats; NULL as above): copies them to
 * the solver's macro buffers on its stream, then reinitialises. */
int lbm_reinit_from_host(lbm_solver* s, const float* rho, const float* ux,
                         const float* uy, const float* uz);

/* Pipelined host I/O, for loops that feed every run from host memory and read
 * its result back (host arrays should be pinned for the copies to overlap):
 * lbm_stage_from_host copies the macro fields (NULL: as in
 * lbm_reinit_from_macro) into one of two staging buffers on the solver's copy
 * stream and returns at once; lbm_reinit_from_stage then reinitialises from
 * the last staged fields on the compute stream, after that copy.  For
 * Legacy/Hybrid it leaves the macro fields as they were (the next step
 * rewrites them), so a read of the previous run's fields can still be in
 * flight.  lbm_read_macros_async copies the current macro fields to host on
 * the copy stream; the next call that rewrites them waits for it, and
 * lbm_wait_reads (or lbm_synchronize of both streams) waits for it on the
 * host.  No reference counterpart (the reference copies synchronously,
 * src/bench/main_taylor_green.cpp:90-105,143-156). */
int lbm_stage_from_host(lbm_solver* s, const float* rho, const float* ux, const float* uy, const float* uz);
int lbm_reinit_from_stage(lbm_solver* s);
int lbm_read_macros_async(lbm_solver* s, float* rho, float* ux, float* uy, float* uz);
int lbm_wait_reads(lbm_solver* s);

/* Advances `substeps` steps, asynchronously on the solver's stream.  The
 * macro fields (and, when enabled, the statistics) are those of the last
 * substep, as in the reference, where they hold the moments of the state the
 * step started from (Legacy/Hybrid, lbm3d_legacy.cu:78-113) or of the state it
 * produced (HOME, lbm3d_home.cu:275-285).  Replaces step(int)
 * (lbm3d_legacy.cu:210-224, lbm3d_home.cu:335-354, lbm3d_hybrid.cu:259-283). */
int lbm_step(lbm_solver* s, int substeps);
/* Waits for all work queued on the solver's stream. */
int lbm_synchronize(lbm_solver* s);
/* Replaces setForce (lbm3d_legacy.hpp:36, lbm3d_home.hpp:32, lbm3d_hybrid.hpp:38). */
int lbm_set_force(lbm_solver* s, float fx, float fy, float fz);
/* Hybrid only: the relaxation rate of the non-band ("HOME form") cells'
 * shear term.  The reference fixes it to 1/tau (lbm3d_hybrid.cu:264-267),
 * which is the default here too. */
int lbm_set_shear_omega(lbm_solver* s, float omega_shear);
/* HOME only: planes per block of the moment step (the z-chunk; 1..Nz, larger
 * values are clamped to Nz).  A tuning knob with no reference counterpart:
 * results do not depend on it.  lbm_create picks a value from the grid. */
int lbm_set_home_zchunk(lbm_solver* s, int zchunk);
int lbm_home_zchunk(lbm_solver* s, int* zchunk);

/* Borrowed device pointers of the macro fields.  Replaces d_rho/d_u/d_v/d_w
 * (lbm3d_legacy.cu:229-236, lbm3d_home.cu:355-362, lbm3d_hybrid.hpp:45-52). */
int lbm_macro_ptrs(lbm_solver* s, float** d_rho, float** d_u, float** d_v, float** d_w);
/* Copies the macro fields to host arrays (any may be NULL); synchronous. */
int lbm_get_macros(lbm_solver* s, float* rho, float* ux, float* uy, float* uz);
/* Copies the state to a host array in the reference's layout: Legacy/Hybrid
 * the 19*N populations f[q*N+id] (what d_f() points at, lbm3d_legacy.cu:225);
 * HOME the 10*N moments m[k*N+id] (lbm3d_home.hpp:57-71).  Synchronous. */
int lbm_get_state(lbm_solver* s, float* host_out);
/* Nx, Ny, Nz and N (any may be NULL).  Replaces Nx()/Ny()/Nz()/N(). */
int lbm_dims(lbm_solver* s, int32_t* nx, int32_t* ny, int32_t* nz, int64_t* n);
/* Steps taken since the last reset/reinit. */
int lbm_step_count(lbm_solver* s, int64_t* steps);

/* Enables (1) or disables (0) the FP64 statistics of the last substep of
 * every lbm_step (mass, kinetic energy, momentum, momentum-exchange drag). */
int lbm_enable_stats(lbm_solver* s, int enable);
/* Synchronises and copies the LBM_NSTAT statistics of the last step that
 * computed them.  No reference counterpart (the reference sums on the host,
 * src/bench/main_taylor_green.cpp:157-182). */
int lbm_get_stats(lbm_solver* s, double* out);
/* The same copy without waiting: it is queued on the solver's copy stream
 * after the steps queued so far (as lbm_read_macros_async is), and `out` (host
 * memory, pinned for the copy to be asynchronous) holds their statistics once
 * lbm_wait_reads or lbm_synchronize returns.  For loops that read every step's
 * result without stalling the GPU on each one. */
int lbm_get_stats_async(lbm_solver* s, double* out);

/* Enables (1, the default) or disables (0) the macro-field output of
 * Legacy/Hybrid steps.  Disabled, lbm_step writes only the populations (the
 * macro buffers keep their last values), which saves 16 B per cell on the
 * last substep; statistics, when enabled, still write them.  HOME F32's macro
 * fields are its state and are always current; HOME in F16/BF16/F64 exports
 * them to FP32 after each lbm_step while the output is on, and otherwise when
 * lbm_macro_ptrs, lbm_get_macros or lbm_read_macros_async next asks for them. */
int lbm_set_macro_output(lbm_solver* s, int enable);

/* Captures `substeps` steps into a CUDA graph on first use and replays it;
 * same result as lbm_step.  Invalidated by any setter. */
int lbm_step_graph(lbm_solver* s, int substeps);

/* FP64 sums of DEVICE fields rho, ux, uy, uz of n cells into the DEVICE array
 * d_out[LBM_NSTAT]: MASS, KE and MOM_X/Y/Z as lbm_get_stats defines them (the
 * drag slots are 0).  Cells whose d_mask byte is nonzero are left out (d_mask
 * may be NULL).  Asynchronous on `stream` (NULL: the default stream).
 * Allocates no memory: its partial sums live in a fixed 2 MiB __device__
 * array, so it suits callers that may not allocate while they run.  Limits:
 * n <= 268,435,456 cells (LBM_ERR_SIZE beyond); calls that overlap in time on
 * one device race on the shared array and must be ordered by the caller; the
 * first call on each device does a one-time address lookup and should come
 * before any stream capture.  No counterpart in the reference (it sums on the
 * host, src/bench/main_taylor_green.cpp:157-182). */
int lbm_macro_stats_static(const float* d_rho, const float* d_ux, const float* d_uy, const float* d_uz,
                           const uint8_t* d_mask, int64_t n, double* d_out, void* stream);

/* ---- batched instances ------------------------------------------------- */

/* Many independent Legacy/Hybrid solvers (halfway bounce-back; all in FP32,
 * all in F16 or all in BF16 storage; any sizes, rates, bands and boundaries)
 * advanced together: every substep is ONE persistent launch over all of them,
 * and a multi-step lbm_batch_step is replayed from a captured CUDA graph.  No
 * reference counterpart: the reference runs one solver per process and times
 * each B0 of its sweep separately (src/main_compare.cpp:511-699). */
typedef struct lbm_batch lbm_batch;
/* Launch shape of the batched step, chosen by lbm_batch_tune (or set). */
typedef struct lbm_batch_tuning {
    int32_t threads;         /* threads per block (128 or 256) */
    int32_t blocks_per_sm;   /* persistent blocks per SM */
    int32_t even_unit;       /* vectors (of the width each instance's own step takes: 1, 2 or 4 cells)
                                per work unit of the local step */
    int32_t odd_unit;        /* blocks of `threads` cells per unit of the neighbour step */
    float us_per_step;       /* measured by lbm_batch_tune: mean of one even + one odd launch / 2 */
} lbm_batch_tuning;

/* The solvers must be at the same step parity; they stay owned by the caller,
 * must outlive the batch, and may be read (lbm_get_state, lbm_get_macros)
 * between batch steps.  The batch keeps a snapshot of each solver's settings
 * (mask, band, rates, force, boundary) taken here or by lbm_batch_refresh;
 * after stepping or reinitialising an instance on its own, call
 * lbm_batch_refresh (lbm_batch_step refuses instances out of step). */
int lbm_batch_create(lbm_solver* const* solvers, int32_t n, void* stream, lbm_batch** out);
int lbm_batch_refresh(lbm_batch* b);
int lbm_batch_destroy(lbm_batch* b);
/* Times every candidate launch shape for `trial_pairs` even+odd step pairs on
 * the batch's own instances (which therefore advance by those steps) and keeps
 * the fastest; out (may be NULL) receives it. */
int lbm_batch_tune(lbm_batch* b, int32_t trial_pairs, lbm_batch_tuning* out);
int lbm_batch_set_tuning(lbm_batch* b, const lbm_batch_tuning* t);
int lbm_batch_get_tuning(lbm_batch* b, lbm_batch_tuning* out);
/* Advances every instance by `substeps` steps, asynchronously. */
int lbm_batch_step(lbm_batch* b, int32_t substeps);
int lbm_batch_synchronize(lbm_batch* b);
/* Statistics (and macro fields) of the last substep of every lbm_batch_step. */
int lbm_batch_enable_stats(lbm_batch* b, int enable);
/* Synchronises and copies n x LBM_NSTAT doubles (instance-major). */
int lbm_batch_get_stats(lbm_batch* b, double* out);

/* ---- differentiation ---------------------------------------------------- */

/* A duct problem for lbm_adjoint_run: the Legacy BGK duct step (inlet at x=0
 * with a per-(y,z) velocity profile, zero-gradient outlet, halfway bounce-back
 * on the mask, y and z periodic) from f^0 = feq(1, u0), n_steps steps, and the
 * objective J = mean momentum-exchange drag (x) over the 1-based steps
 * window_begin .. window_end. */
typedef struct lbm_adj_problem {
    int32_t nx, ny, nz;
    double tau;                 /* double, so that FP64 runs see the exact rate */
    double force[3];
    int32_t n_steps;
    int32_t window_begin, window_end;
    int32_t checkpoint_every;   /* forward states kept every k steps, the rest recomputed */
    int32_t precision;          /* 0: FP32, 1: FP64 (state, adjoint and arithmetic) */
} lbm_adj_problem;

/* Objective and, when grad_inlet / grad_u0 are not NULL, its gradient by the
 * hand-written discrete adjoint of the step (reverse pass over checkpointed,
 * recomputed forward states).  host_mask: Nx*Ny*Nz bytes as lbm_set_solid_mask
 * takes them (walls 1|LBM_MASK_WALL are left out of the drag); u_inlet and
 * grad_inlet: Ny*Nz values, index z*Ny + y; u0 and grad_u0: three planes of
 * N values (u_x, u_y, u_z).  Synchronous; allocates its own device memory.  No
 * reference counterpart (the reference has no inlet, drag or gradients). */
int lbm_adjoint_run(const lbm_adj_problem* p, const uint8_t* host_mask, const double* u_inlet,
                    const double* u0, double* objective, double* grad_inlet, double* grad_u0);

/* ---- geometry (host in, host out) ------------------------------------- */

/* STL loader: ASCII when the file starts with "solid" (falls back to binary
 * if no vertex parses), binary otherwise.  Replaces load_stl
 * (src/geom/stl_loader.cpp:102-122).  *tris receives 9 floats per triangle
 * (free with lbm_free); bb receives {min xyz, max xyz}.  LBM_ERR_IO when the
 * reference would return false. */
int lbm_load_stl(const char* path, float** tris, int64_t* ntri, float* bb);
void lbm_free(void* p);

/* Voxel options, mirroring VoxelParams (src/geom/voxelize.hpp:16-24). */
typedef struct lbm_voxel_params {
    int32_t nx, ny, nz;
    float uniform_scale;   /* default 0.9 in VoxelParams, 0.5 on the CLI */
    float translate[3];
    int32_t refine;        /* supersampling factor (AMR), >=1 */
    float coverage_threshold;
} lbm_voxel_params;

/* GPU voxelizer: fit to the unit cube, SAT surface marking, exterior flood
 * fill, optional refine^3 coverage downsample.  Bit-exact with
 * voxelize_mesh_to_mask (src/geom/voxelize.cpp:228-243).  bb may be NULL
 * (computed from the vertices the way the loader does).  mask_out: Nx*Ny*Nz
 * bytes, 1 = solid. */
int lbm_voxelize(const float* tris, int64_t ntri, const float* bb,
                 const lbm_voxel_params* p, uint8_t* mask_out);

/* ---- free functions of the reference (same names and signatures) ------ */

/* f_i = feq(rho,u) for N cells into d_f (SoA q*N+i); NULL u components are 0.
 * src/lbm/lbm_reinit.cu:52-61.  Launches on the default stream. */
void reinit_equilibrium_from_macro(const float* d_rho, const float* d_ux, const float* d_uy,
                                   const float* d_uz, float* d_f, int N);
/* |u| per cell.  src/fields/field_ops.cu:25-28. */
void launch_speed(const float* u, const float* v, const float* w, float* out, int N);
/* Initial density profiles (--init gauss|slab).  src/fields/init_profiles.cu:31-45. */
void make_rho_gauss(float* d_rho, int Nx, int Ny, int Nz, float cx, float cy, float cz,
                    float sigma, float amp);
void make_rho_slab(float* d_rho, int Nx, int Ny, int Nz, int axis, float amp, float center,
                   float width);
/* ASCII legacy VTK (STRUCTURED_POINTS) from a DEVICE field, byte-identical to
 * src/moment_vtk_writer.cu:9-49.  Throwing on an unopenable file, as the
 * reference does, is replaced by an error message on stderr. */
void write_scalar_vtk(const char* filename, const float* d_field, int Nx, int Ny, int Nz);
void write_vector_vtk(const char* filename, const float* d_fx, const float* d_fy,
                      const float* d_fz, int Nx, int Ny, int Nz);
/* Same writers with a status code (LBM_ERR_IO when the file cannot be opened). */
int lbm_write_scalar_vtk(const char* filename, const float* d_field, int Nx, int Ny, int Nz);
int lbm_write_vector_vtk(const char* filename, const float* d_fx, const float* d_fy,
                         const float* d_fz, int Nx, int Ny, int Nz);

/* ---- VTK text on the GPU, asynchronous writer --------------------------- */

/* Line kinds: "v\n" of a scalar field, "|u|\n" computed from (u, v, w) as
 * launch_speed does, "u v w\n" of a vector field.  Values are printed as the
 * reference's `ofstream << float` prints them (src/moment_vtk_writer.cu:22,46). */
enum { LBM_VTK_SCALAR = 0, LBM_VTK_SPEED = 1, LBM_VTK_VECTOR = 2 };
/* Bytes a text buffer needs for n lines of `kind` (no header). */
int64_t lbm_vtk_text_bound(int32_t kind, int64_t n);
/* Formats n lines into device memory d_text (cap bytes, >= lbm_vtk_text_bound)
 * on `stream`, synchronises the stream and returns the text length in *len. */
int lbm_vtk_format(int32_t kind, const float* d_a, const float* d_b, const float* d_c, int64_t n,
                   char* d_text, int64_t cap, int64_t* len, void* stream);
/* Writes whole VTK files (header + text) in the background.  submit queues
 * the formatting on `stream` (after the work already queued there, e.g. the
 * step that produced the fields) and returns; a writer thread copies the text
 * to pinned host memory and writes the file.  At most `depth` fields are in
 * flight; submit waits for a free one.  flush waits for every queued file and
 * returns the first error since the last flush.  No reference counterpart: the
 * reference formats on the host, synchronously. */
typedef struct lbm_vtk_writer lbm_vtk_writer;
int lbm_vtk_writer_create(int32_t nx, int32_t ny, int32_t nz, int32_t depth, lbm_vtk_writer** out);
int lbm_vtk_writer_submit(lbm_vtk_writer* w, int32_t kind, const float* d_a, const float* d_b,
                          const float* d_c, const char* path, void* stream);
int lbm_vtk_writer_flush(lbm_vtk_writer* w);
/* Bytes written to files so far (headers included). */
int lbm_vtk_writer_bytes(lbm_vtk_writer* w, uint64_t* bytes);
int lbm_vtk_writer_destroy(lbm_vtk_writer* w);
/* The same formatting on the host, for checks: value i's text at out + i*stride
 * (stride >= 12), its length in lens[i]. */
int lbm_format_g6(const float* v, int64_t n, char* out, int32_t stride, uint8_t* lens);
/* The CUDA stream a solver runs on (cudaStream_t). */
int lbm_solver_stream(lbm_solver* s, void** stream);
/* Parity of the next AA step (0: the local step, 1: the neighbour step). */
int lbm_step_parity(lbm_solver* s, int* parity);

/* ---- z-slab decomposition ------------------------------------------------ */

/* A slab solver of nz planes steps only planes 1..nz-2; planes 0 and nz-1 are
 * ghost copies of the neighbouring slabs' boundary planes (give them the
 * neighbours' mask, band and initial fields).  Legacy/Hybrid with halfway
 * bounce-back, and HOME.  No reference counterpart: the reference runs one
 * grid on one GPU. */
int lbm_set_z_ghosts(lbm_solver* s, int on);
/* HOME: device addresses of the 10 moment planes of `plane` in the current
 * buffer (they move to the other buffer with every step), each *bytes long. */
int lbm_zslab_moment_planes(lbm_solver* s, int plane, void** ptrs, int64_t* bytes);
/* Index of this solver's cell 0 in the whole grid (a slab: its plane 0).  Only
 * the F16/BF16 stochastic rounding (every method) reads it, so that a slab
 * draws the same random bits for a cell as the whole grid does. */
int lbm_set_index_base(lbm_solver* s, int64_t base);
/* Device addresses of the 5 slot planes of `plane` whose direction has
 * c_z = cz (+1 or -1), in direction order, each *bytes long: what crosses a
 * slab face in an odd step. */
int lbm_zslab_slots(lbm_solver* s, int plane, int cz, void** ptrs, int64_t* bytes);
/* Exchange between two slabs on this device, `lower` below `upper` (periodic
 * wrap: the top slab is `lower` of the bottom one).  Legacy/Hybrid: before
 * each odd step (parity 1) call phase 0 on every face: boundary slots ->
 * neighbour's ghost; after it phase 1: ghost slots -> their owner's boundary
 * plane.  HOME: phase 0 before every step copies the 10 moment planes of each
 * boundary plane to the neighbour's ghost; phase 1 does nothing. */
int lbm_zslab_exchange(lbm_solver* lower, lbm_solver* upper, int phase, void* stream);
/* Phase 1 for slabs on different devices: after receiving a neighbour's ghost
 * slot planes (5 device buffers, direction order) for `plane` / `cz`, take the
 * values its cells wrote: every cell whose link towards that neighbour
 * streams (a cell that bounced its own population back keeps it). */
int lbm_zslab_merge(lbm_solver* s, int plane, int cz, void* const* src, void* stream);
/* One step of a z-slab solver over its planes [z_begin, z_end) only
 * (1 <= z_begin <= z_end <= nz-1), so that the planes next to the ghosts can
 * wait for an exchange while the interior computes: Legacy/Hybrid the current
 * parity's kernel, HOME the moment step.  No statistics and no macro fields
 * (use lbm_step for a step that writes them).  finish != 0 ends the step after
 * this part: the parity flips (HOME: the buffers swap) and the step counts.
 * No reference counterpart. */
int lbm_zslab_step_planes(lbm_solver* s, int z_begin, int z_end, int finish);
/* Every face of a periodic chain of n slabs (slab k below slab k+1, the last
 * below the first) in ONE launch per phase: the transfers of lbm_zslab_exchange
 * for all faces, as a job table built once.  The slabs' buffers must stay in
 * place (no re-creation) while the plan lives.  Capturable in CUDA graphs. */
typedef struct lbm_zslab_plan lbm_zslab_plan;
int lbm_zslab_plan_create(lbm_solver* const* slabs, int32_t n, lbm_zslab_plan** out);
int lbm_zslab_plan_exchange(lbm_zslab_plan* p, int phase, void* stream);
int lbm_zslab_plan_destroy(lbm_zslab_plan* p);

/* ---- headless volume view ------------------------------------------------ */

/* The viewer's other field helpers, same names and signatures
 * (src/fields/field_ops.cu:29-41): out = a - b, out = a + bias. */
void launch_diff(const float* a, const float* b, float* out, int N);
void launch_shift(const float* a, float bias, float* out, int N);

/* Samplers of lbm_render_volume: trilinear in FP32 exactly as written
 * (reproducible, equal to the C oracle), or the texture unit's filter. */
enum { LBM_FILTER_EXACT = 0, LBM_FILTER_TEXTURE = 1 };
/* Uniforms of the reference's volume shader (src/render/Vis3D.cpp:30-78,
 * set at Vis3D.cpp:128-138). */
typedef struct lbm_render_params {
    int32_t width, height;   /* framebuffer (main_compare: 1280 x 720) */
    float inv_pv[16];        /* inverse(P V), column-major */
    float cam_pos[3];
    float step;              /* uStep (0.005 in main_compare.cpp:999) */
    float scale;             /* uScale (150 speed, 1000 rho-1, 2000 difference) */
    float threshold;         /* uThresh (0.15) */
    int32_t filter;          /* LBM_FILTER_* */
} lbm_render_params;
/* Ray-marches the Nx*Ny*Nz device field (x fastest, mapped onto [0,1]^3) into
 * d_rgba (width*height float RGBA, row 0 at the bottom) on `stream`.  Replaces
 * Vis3D::uploadScalar + renderVolume (Vis3D.cpp:118-138) without the host
 * round trip and the GL context. */
typedef struct lbm_renderer lbm_renderer;
int lbm_renderer_create(int32_t nx, int32_t ny, int32_t nz, lbm_renderer** out);
int lbm_render_volume(lbm_renderer* r, const float* d_field, const lbm_render_params* p, float* d_rgba,
                      void* stream);
int lbm_renderer_destroy(lbm_renderer* r);
/* The viewer's orbit camera (main_compare.cpp:51-60,972-981): inverse(P V)
 * and the eye position for yaw/pitch/radius around target. */
int lbm_render_orbit_camera(float yaw, float pitch, float radius, const float* target, int32_t width,
                            int32_t height, float* inv_pv, float* cam_pos);
/* Host RGBA float image -> binary PPM, top row first, 8 bits per channel. */
int lbm_write_ppm(const char* path, const float* rgba, int32_t width, int32_t height);

#ifdef __cplusplus
}  /* extern "C" */
#endif

#endif /* LBM_CAPI_H */
