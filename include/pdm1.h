/*
 * pdm1.h -- C ABI of the B200 (sm_100a) M1 proton dose march.
 *
 * One shared library, libpdm1.so, implements the energy march of
 * proton_solver/numerics/energy.py (WENO-Z reconstruction, HLL fluxes with
 * exact M1 speeds, realizability projection, IF-SSPRK3 / SSPRK3 / Strang /
 * forward-Euler integrators, CSDA stopping power, dose deposit) as CUDA
 * kernels.  Plain C types only: host pointers, device pointers, sizes and a
 * CUDA stream handle.  Every entry point returns a status (PDM1_OK == 0);
 * pdm1_last_error() describes the last failure on the calling thread.
 *
 * Layouts follow the reference: a state U is (4, nx, ny, nz) float64 in C
 * order (z fastest), components (phi, Jx, Jy, Jz); a dose is (nx, ny, nz);
 * a boundary plane is (4, nx, ny); material ids are int32 (nx, ny, nz).
 */
#ifndef PDM1_H
#define PDM1_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *pdm1_stream_t;   /* same type as cudaStream_t */

enum pdm1_status {
    PDM1_OK = 0,
    PDM1_ERR_ARGUMENT = 1,      /* bad shape, pointer or option (reference: ValueError) */
    PDM1_ERR_RANGE = 2,         /* energy outside a coefficient table (ValueError) */
    PDM1_ERR_CUDA = 3,          /* a CUDA runtime call failed */
    PDM1_ERR_MAX_STEPS = 4,     /* the energies buffer is shorter than the march */
    PDM1_ERR_NO_BEAM = 5,       /* the inflow profile is empty (ValueError) */
    PDM1_ERR_UNSUPPORTED = 6,   /* option without a GPU kernel (NotImplementedError) */
    PDM1_ERR_NONFINITE = 7,     /* a non-finite energy step was produced */
    PDM1_ERR_TIMEOUT = 8        /* a bounded wait inside a kernel ran out */
};

enum { PDM1_SCATTERING_OFF = 0, PDM1_SCATTERING_ROSSI = 1, PDM1_SCATTERING_WENTZEL = 2 };
enum { PDM1_INTERP_LINEAR = 0, PDM1_INTERP_PCHIP = 1 };
enum { PDM1_SCHEME_FORWARD_EULER = 0, PDM1_SCHEME_SSPRK3 = 1, PDM1_SCHEME_IF_SSPRK3 = 2 };
enum { PDM1_SPEEDS_EXACT = 0, PDM1_SPEEDS_UNIT = 1 };
enum { PDM1_FP64 = 0, PDM1_FP32_FP64 = 1 };
/* reconstruction (Numerics.spatial_scheme; reconstruction_methods/): ghost widths 3, 1, 2, 2 */
enum { PDM1_SPATIAL_WENO_Z = 0, PDM1_SPATIAL_FIRST_ORDER = 1, PDM1_SPATIAL_MUSCL = 2, PDM1_SPATIAL_WENO3 = 3 };

/* One tabulated coefficient, host memory, strictly increasing energies. */
typedef struct {
    int n_nodes;
    const double *energy;     /* MeV */
    const double *value;
} pdm1_table;

/* One material: physics/stopping_power.py, physics/scattering.py,
 * physics/nuclear.py and physics/materials.py tables. */
typedef struct {
    pdm1_table stopping_power;   /* MeV/m, interpolated by PCHIP */
    pdm1_table transport;        /* Wentzel-VI first transport coefficient, 1/m */
    pdm1_table nuclear;          /* primary nuclear removal coefficient, 1/m */
    double density;              /* kg/m^3 */
    double radiation_length;     /* m (Rossi scattering) */
} pdm1_material;

/* One pencil beam on one voxel phantom.  Mirrors the arguments the reference
 * passes to energy_march (numerics/energy.py:1497-1505): Grid, MaterialMap,
 * BeamInflow and SolverConfig.  All pointers are host memory and are copied
 * into the plan. */
typedef struct {
    int nx, ny, nz;
    double dx, dy, dz;                 /* m */
    int n_materials;                   /* 1 .. 16 */
    const pdm1_material *materials;
    const int32_t *ids;                /* (nx, ny, nz) */
    const double *inflow_spatial;      /* (nx, ny): n_protons * normalised profile,
                                          numerics/boundary.py:30-80 */
    double beam_energy;                /* MeV */
    double energy_spread;              /* MeV, > 0 */
    double angular_spread;             /* rad */
    int scattering, nuclear, interpolation;
    int energy_scheme, wave_speeds;
    double max_energy_step, cfl, energy_min, energy_window_sigma;
    int moving_active_domain;          /* numerics/moving_active_domain.py */
    int vacuum_aware_cfl;
    int active_guard_cells;
    double active_relative_tolerance;  /* exp(-sigma_trunc^2 / 2), energy.py:1305 */
    int precision;                     /* PDM1_FP64 or PDM1_FP32_FP64 */
    int spatial_scheme;                /* PDM1_SPATIAL_*, 0 (WENO-Z) when zero-initialised */
    int phantom_cfl_floor;             /* moving box: bound the CFL step by the vacuum cells of
                                          the whole phantom, as a full-domain march is (no
                                          reference counterpart; 0 = the reference's rule) */
} pdm1_problem;

/* One pencil beam of a field (numerics/boundary.py:63-114): its spectrum and
 * angular spread, and its transverse profile on the phantom's z-min face. */
typedef struct {
    double energy;                  /* MeV */
    double energy_spread;           /* MeV, > 0 */
    double angular_spread;          /* rad */
    const double *inflow_spatial;   /* host (nx, ny): n_protons * normalised profile */
} pdm1_beam;

typedef struct pdm1_plan pdm1_plan;

typedef struct {
    int n_steps;              /* energy steps taken; energies holds n_steps + 1 values */
    int n_snapshots;          /* snapshots written to snap_out */
    int final_state_valid;    /* U holds the final state (full grid) */
    int graph_replays;        /* CUDA graph launches used by the march */
    int kernel_launches;      /* kernels this library launched for the march */
    int stage_launches;       /* launches of the fused stage kernels */
    double stage_ms;          /* their summed device time (CUDA events on the march stream) */
    double cell_steps;        /* sum over energy steps of the cells marched */
    double max_box_cells;     /* largest domain (cells) one beam marched in one step */
    int box_grow_events;      /* learned box: faces grown by the outgoing-flux check */
    int box_fallbacks;        /* learned box: beams that fell back (full domain or heuristic box) */
} pdm1_march_info;

/* Plan: copies the problem to the device and allocates the workspace.
 * Replaces the setup half of energy_march (energy.py:1519-1554). */
int pdm1_plan_create(const pdm1_problem *problem, pdm1_plan **plan);
void pdm1_plan_destroy(pdm1_plan *plan);
size_t pdm1_plan_workspace_bytes(const pdm1_plan *plan);

/* The march: numerics/energy.py:1497-1643 (static domain) and 1262-1494
 * (moving active box).  Device pointers: U (4,nx,ny,nz) in/out, dose
 * (nx,ny,nz) out, energies (max_steps+1) out, snap_out (n_snap,4,nx,ny,nz)
 * out.  Host pointers: snap_targets (n_snap), snap_energies_out (n_snap).
 * Snapshots are written in descending target order, like the reference's
 * snapshot dict.  Synchronises `stream` before returning. */
int pdm1_march(pdm1_plan *plan, double *U, double *dose, double *energies, int max_steps,
               const double *snap_targets, int n_snap, double *snap_out,
               double *snap_energies_out, pdm1_march_info *info, pdm1_stream_t stream);

/* A spot-scanning field: n_beams pencil beams on one phantom, each marching on
 * its own moving active box with its own energy and CFL step, all of them in
 * one persistent launch per stage (no reference counterpart: the reference
 * solves one beam per Solver.solve and never batches).  `phantom` gives the
 * grid, materials, physics and numerics (its beam fields are ignored;
 * moving_active_domain must be set); every beam's compact buffers hold
 * box_capacity_cells cells (0: the whole grid). */
int pdm1_field_plan_create(const pdm1_problem *phantom, const pdm1_beam *beams, int n_beams,
                           size_t box_capacity_cells, pdm1_plan **plan);

/* March every beam of a field plan from zero to energy_min; field_dose
 * (device, (nx,ny,nz)) receives the sum of the beams' doses (FP64 atomic
 * accumulation, so the summation order across beams is not fixed);
 * steps_per_beam (host, n_beams) may be NULL.  Synchronises `stream`. */
int pdm1_field_march(pdm1_plan *plan, double *field_dose, int max_steps, int *steps_per_beam,
                     pdm1_march_info *info, pdm1_stream_t stream);

/* The first `step_limit` steps of the march (a bounded prefix, for timing
 * samples, profiler captures and prefix parity); otherwise as pdm1_march
 * without snapshots.  For a field plan U and energies are not used (may be
 * NULL) and `dose` receives the field dose of those steps. */
int pdm1_march_steps(pdm1_plan *plan, double *U, double *dose, double *energies, int max_steps,
                     int step_limit, pdm1_march_info *info, pdm1_stream_t stream);

/* The march without any allocation by the library (no counterpart in the
 * reference).  For callers that cannot call cudaMalloc: applications that hand
 * the whole device to their own memory pool, plugins whose host forbids device
 * allocation, and paths that must not take an allocation's implicit device
 * synchronisation.  Instead of a plan's workspace, the configuration, tables and
 * stage scratch live in one file-scope __device__ array of 16 MiB that every GPU
 * loading libpdm1.so holds until the process exits; problems that do not fit
 * (roughly more than 130000 cells) are rejected with PDM1_ERR_ARGUMENT.  The
 * caller passes the problem (host), U (device, in/out), dose and energies
 * (device, out) exactly as for pdm1_plan_create + pdm1_march, without snapshots.
 * It marches the full domain in FP64: a problem asking for the moving active
 * box or the FP32 stencil is rejected with PDM1_ERR_UNSUPPORTED.
 * The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) and sets kernel attributes, so make it before any
 * stream capture; first calls from several host threads take turns on a lock.
 * The looked-up address is kept for the life of the process: after a
 * cudaDeviceReset of that device this entry point must not be called again.
 * All calls on a device share the one array and it keeps the
 * last call's contents (the march state is cleared at the start of every
 * call): calls that overlap on the GPU race.  Launches directly on `stream`
 * (no graph, no events) and synchronises it before returning. */
int pdm1_march_noalloc(const pdm1_problem *problem, double *U, double *dose, double *energies,
                       int max_steps, pdm1_march_info *info, pdm1_stream_t stream);

/* Building blocks on the full grid, for operator-level parity checks. */

/* numerics/spatial.py:104-252: rhs = -div F(U), boundary_state (4,nx,ny)
 * device or NULL (then the beam inflow at `energy`). */
int pdm1_spatial_operator(pdm1_plan *plan, const double *U, double energy,
                          const double *boundary_state, double *rhs, pdm1_stream_t stream);

/* numerics/energy.py:539-660: the CFL energy step for state U at `energy`. */
int pdm1_energy_step(pdm1_plan *plan, const double *U, double energy, double *dE_out,
                     pdm1_stream_t stream);

/* One accepted step of the configured integrator (energy.py:1580-1615):
 * U advanced in place, edep (nx,ny,nz) receives the energy deposition in MeV
 * per cell volume and MeV of step (before the MEV_TO_JOULE / rho scaling). */
int pdm1_advance(pdm1_plan *plan, double *U, double energy, double dE, double *edep,
                 pdm1_stream_t stream);

/* Device evaluation of the material coefficients at host energies:
 * out[(e * n_materials + m) * 3 + {0,1,2}] = S, Sigma_tr, Sigma_r (host). */
int pdm1_coefficients(pdm1_plan *plan, const double *energies, int n, double *out);

/* Scalar device functions over device arrays (unit parity). */
int pdm1_weno_batch(const double *v5, double *out, int n, pdm1_stream_t stream);
int pdm1_project_batch(double *u4, int n, pdm1_stream_t stream);
int pdm1_eigen_batch(const double *u4, int axis, double *lo_hi, int n, pdm1_stream_t stream);
int pdm1_hll_batch(const double *left4, const double *right4, int axis, int wave_speeds,
                   double *flux4, int n, pdm1_stream_t stream);
int pdm1_exp_batch(const double *x, double *y, int n, pdm1_stream_t stream);

/* Global 3-D gamma index of `dose_eval` against `dose_ref` (device, same
 * (nx,ny,nz) grid, spacings in mm) as the reference scores doses
 * (proton_solver/metrics.py:542-606, pymedphys.gamma with interp_fraction,
 * max_gamma, global normalisation, lower dose cutoff in percent of it, and
 * skip-once-passed).  gamma_out (device, nx*ny*nz) receives gamma, NaN below
 * the cutoff; *pass_rate_out (host) the percentage of evaluated voxels with
 * gamma <= 1.  Synchronises `stream`. */
int pdm1_gamma(const double *dose_ref, const double *dose_eval, int nx, int ny, int nz,
               double dx_mm, double dy_mm, double dz_mm, double dose_percent,
               double distance_mm, double lower_cutoff_percent, int interp_fraction,
               double max_gamma, double global_normalisation, double *gamma_out,
               double *pass_rate_out, pdm1_stream_t stream);

/* A prescribed energy schedule for a one-beam plan: the march steps through
 * energies[0..n-1] (energies[0] the start energy, strictly decreasing)
 * instead of its CFL steps, then on to energy_min in one step; n = 0 restores
 * the CFL rule.  No reference function; it is the fixed-schedule mode the
 * reference's own harness gets by patching compute_energy_step
 * (numerics/energy.py:539-660): a march given the reference's own energies
 * isolates the per-step arithmetic from the choice of step. */
int pdm1_plan_set_schedule(pdm1_plan *plan, const double *energies, int n);

/* Staging of the FP32 form's stages B and C (no counterpart in the reference;
 * the reference has no GPU tiles): bulk = 1 (the default) copies each z row of
 * the tile and its halo with cp.async.bulk onto a shared-memory mbarrier,
 * bulk = 0 loads cell by cell.  Both fill shared memory with the same values,
 * so the march is the same bit for bit.  No effect on FP64 plans. */
int pdm1_plan_set_staging(pdm1_plan *plan, int bulk);

/* ---- Tile shape of the stage kernels ---------------------------------------
 * No reference counterpart.  The fused stage kernels are built for
 * PDM1_NUM_TILES tile shapes of 256 cells (one per thread): 4x8x8 (the
 * default), 8x8x4 and 2x8x16 (x, y, z; z is the contiguous axis).  The
 * autotuner marches the first `steps` energy steps of the plan's problem with
 * every shape (in scratch buffers it allocates; the plan's results are not
 * touched), measures the stage-kernel time per cell-step with CUDA events,
 * keeps the fastest shape for the plan and reports it in *best_tile and the
 * measurements in ns_per_cell_step (host, PDM1_NUM_TILES, may be NULL). */
#define PDM1_NUM_TILES 3
int pdm1_tile_shape(int tile_id, int *tx, int *ty, int *tz);
int pdm1_plan_set_tile(pdm1_plan *plan, int tile_id);
int pdm1_plan_autotune(pdm1_plan *plan, int steps, int *best_tile, double *ns_per_cell_step,
                       pdm1_stream_t stream);

/* ---- Learned moving box -------------------------------------------------
 * No reference counterpart: the reference's moving box is the fixed heuristic
 * of numerics/moving_active_domain.py:107-193 (significant box plus
 * active_guard_cells on every face).  With a box model, a plan instead extends
 * the significant box on each face by a margin that a small network proposes
 * from the beam's fluence moments at every energy step, and checks every step
 * that the particle current through the box faces stays below
 * leak_tolerance of the beam current; faces that leak more grow by grow_cells,
 * and a beam whose growth passes extra_max falls back to the full domain when
 * its buffers hold it, else to the heuristic box. */
#define PDM1_BOX_FEATURES 16
#define PDM1_BOX_OUTPUTS 6
#define PDM1_BOX_PARAMS 5638      /* 64*16 + 64 + 64*64 + 64 + 6*64 + 6 */
#define PDM1_RECORD_WIDTH 40      /* floats per recorded energy step */

typedef struct {
    const float *params;          /* host: W1 (64x16), b1 (64), W2 (64x64), b2 (64), W3 (6x64), b3 (6);
                                     matrices row-major [out][in]; h = relu(W x + b) */
    float x_mean[PDM1_BOX_FEATURES], x_inv_std[PDM1_BOX_FEATURES];   /* feature normalisation */
    float y_scale[PDM1_BOX_OUTPUTS], y_offset[PDM1_BOX_OUTPUTS];     /* margin = ceil(y * scale + offset) cells;
                                     faces x-, x+, y-, y+, z-, z+ */
    int margin_min, margin_max;   /* clamp of the proposed margins (cells) */
    int grow_cells;               /* growth of a leaking face (cells) */
    int extra_max;                /* total growth of a face beyond which the beam falls back */
    double leak_tolerance;        /* face current / beam current that triggers growth (e.g. 1e-6) */
} pdm1_box_model;

/* Attach (or, with NULL, detach) a box model to a moving-box plan or field plan. */
int pdm1_plan_set_box_model(pdm1_plan *plan, const pdm1_box_model *model);

/* Training data: a one-beam plan on the full domain (moving_active_domain
 * off) with a recorder writes, after every energy step, one row of
 * PDM1_RECORD_WIDTH floats to `rows` (device, max_rows rows):
 *   0 the energy after the step, 1 its dE,
 *   2..7 the significant box (i0, i1, j0, j1, k0, k1: global cells, half-open,
 *        -1 when nothing is significant) at the plan's box tolerance,
 *   8..23 the PDM1_BOX_FEATURES features of the state,
 *   24 the summed fluence, 25 the largest z-plane current, 26 the threshold scale,
 *   27..32 and 33..38 the boxes of the cells above tail_a * scale and
 *        tail_b * scale (the fluence tail at two levels), 39 zero.
 * NULL detaches.  Rows beyond max_rows are dropped; pdm1_march_info.n_steps
 * tells how many steps ran. */
int pdm1_plan_set_recorder(pdm1_plan *plan, float *rows, int max_rows, double tail_a, double tail_b);

/* Training of the proposer network (FP32, on the device; X (n x 16) and Y
 * (n x 6) device, normalised): one fused forward/backward kernel per chunk of
 * 64 samples, Adam updates of theta (device, PDM1_BOX_PARAMS) over `epochs`
 * passes in minibatches of `batch` shuffled with `seed`.  Loss: mean of
 * w (y - target)^2 with w = alpha where the prediction is below the target.
 * loss_per_epoch (host, epochs) may be NULL. */
int pdm1_mlp_train(float *theta, const float *X, const float *Y, int n, int epochs, int batch, float lr,
                   float alpha, unsigned seed, float *loss_per_epoch, pdm1_stream_t stream);
/* Loss (device scalar, may be NULL) and its gradient (device, PDM1_BOX_PARAMS) over all n samples. */
int pdm1_mlp_gradients(const float *theta, const float *X, const float *Y, int n, float alpha, float *grad,
                       float *loss, pdm1_stream_t stream);
/* FP32 forward pass (device arrays). */
int pdm1_mlp_forward(const float *theta, const float *X, int n, float *Y, pdm1_stream_t stream);
/* The march's inference: raw features (device, n x 16) normalised with the
 * model, BF16 tensor-core MLP with FP32 accumulation; out (device, n x 6). */
int pdm1_box_model_infer(const pdm1_box_model *model, const float *features, int n, float *out,
                         pdm1_stream_t stream);

/* Analytical CSDA + straight-streaming dose (proton_solver/analytical.py:173-338),
 * the reference's reduced-model verifier: available without scattering,
 * nuclear removal and angular spread (else PDM1_ERR_ARGUMENT).  Range tables of
 * range_points geometric energies per material (the reference uses 200000),
 * trapezoid rule over energy_points incident energies (128000); `problem` as
 * for pdm1_plan_create; dose (device, (nx, ny, nz)) is overwritten.
 * Synchronises `stream`. */
int pdm1_analytical_csda_dose(const pdm1_problem *problem, int energy_points, int range_points, double *dose,
                              pdm1_stream_t stream);

/* The plans' caching allocator (no reference counterpart: the reference
 * allocates NumPy/CuPy arrays per call).  A destroyed plan's device buffers
 * and pinned blocks stay cached for the next plan of the same sizes;
 * pdm1_pool_cached_bytes: bytes cached for the current device;
 * pdm1_pool_release: synchronise the device and free them. */
size_t pdm1_pool_cached_bytes(void);
int pdm1_pool_release(void);

const char *pdm1_last_error(void);
const char *pdm1_version(void);

#ifdef __cplusplus
}
#endif
#endif
