/*
 * m1_oracle.h -- CPU restatement of the proton_solver M1 energy march.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU baseline load it.
 * The product (proton_dose_m1_b200, libpdm1.so) never links or calls it.
 *
 * Parity is pinned by tests/golden/: vectors and full-march doses produced by
 * importing the unmodified reference proton_solver (tests/golden/make_golden.py)
 * and the deterministic maxima the reference publishes in
 * thesis_results/robustness/coarse_grid_2mm/...
 *
 * Layouts follow the reference: a state U is (4, nx, ny, nz) float64 in
 * C order (z fastest); ids is (nx, ny, nz) int32; a boundary plane is
 * (4, nx, ny).
 */
#ifndef M1_ORACLE_H
#define M1_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Enumerations mirror proton_solver/enums.py. */
enum { ORC_SCATTER_OFF = 0, ORC_SCATTER_ROSSI = 1, ORC_SCATTER_WENTZEL = 2 };
enum { ORC_INTERP_LINEAR = 0, ORC_INTERP_PCHIP = 1 };
enum { ORC_SCHEME_FORWARD_EULER = 0, ORC_SCHEME_SSPRK3 = 1, ORC_SCHEME_IF_SSPRK3 = 2 };
enum { ORC_SPEEDS_EXACT = 0, ORC_SPEEDS_UNIT = 1 };

/* Status codes. */
enum {
    ORC_OK = 0,
    ORC_ERR_ARG = 1,          /* invalid argument (shape, null pointer) */
    ORC_ERR_RANGE = 2,        /* energy outside a coefficient table */
    ORC_ERR_ALLOC = 3,
    ORC_ERR_MAX_STEPS = 4,    /* the caller's energies buffer is too short */
    ORC_ERR_NO_BEAM = 5       /* the inflow profile has zero mass */
};

typedef struct {
    int n_sp;  const double *sp_energy;  const double *sp_value;
    int n_tr;  const double *tr_energy;  const double *tr_value;
    int n_nuc; const double *nuc_energy; const double *nuc_value;
    double density;            /* kg/m^3 */
    double radiation_length;   /* m */
} orc_material_desc;

typedef struct {
    /* grid (numerics/grid.py) */
    int nx, ny, nz;
    double lx, ly, lz;                 /* m */
    /* materials */
    int n_materials;
    const orc_material_desc *materials;
    const int32_t *ids;                /* (nx, ny, nz) */
    /* beam (beam.py) */
    double n_protons, energy, energy_spread;
    double sigma_x, sigma_y, center_x, center_y;
    double angular_spread, cutoff_sigma;
    /* physics (config.py Physics) */
    int scattering, nuclear, interpolation;
    /* numerics (config.py Numerics) */
    int energy_scheme, wave_speeds;
    double max_energy_step, cfl, energy_min, energy_window_sigma;
    int moving_active_domain, vacuum_aware_cfl, active_guard_cells;
    double active_truncation_sigma;
    int store_final_state;
    /* reconstruction (config.py Numerics.spatial_scheme):
     * 0 WENO_Z, 1 FIRST_ORDER, 2 MUSCL, 3 WENO3 */
    int spatial_scheme;
} orc_problem_desc;

typedef struct orc_problem orc_problem;

int  orc_problem_create(const orc_problem_desc *desc, orc_problem **out);
void orc_problem_destroy(orc_problem *p);
const char *orc_last_error(void);

/* ---- scalar kernels (unit parity) ---------------------------------- */
double orc_exp(double x);   /* the double-double exp used by the march */
double orc_weno_left(const double v[5]);
double orc_weno3_left(const double v[3]);
void orc_muscl_faces(double vm, double v0, double vp, double *minus, double *plus);
void   orc_project(double u[4]);
void   orc_eigenvalues(const double u[4], int axis, double *lmin, double *lmax);
void   orc_hll_flux(const double left[4], const double right[4], int axis,
                    int wave_speeds, double flux[4]);

/* ---- material coefficients ----------------------------------------- */
int orc_stopping_power(const orc_problem *p, int material, double energy, double *out);
int orc_transport_coefficient(const orc_problem *p, int material, double energy, double *out);
int orc_nuclear_coefficient(const orc_problem *p, int material, double energy, double *out);
int orc_optical_depths(const orc_problem *p, int material, double energy, double dE,
                       double *scattering_depth, double *nuclear_depth);

/* ---- beam inflow ---------------------------------------------------- */
void orc_inflow_spatial(const orc_problem *p, double *spatial /* (nx, ny) */);
void orc_inflow_state(const orc_problem *p, double energy, double *state /* (4, nx, ny) */);

/* ---- operators on the full grid ------------------------------------- */
int orc_spatial_operator(const orc_problem *p, const double *U, double energy,
                         const double *boundary_state /* (4,nx,ny) or NULL */,
                         double *rhs);
int orc_energy_step(const orc_problem *p, const double *U, double energy, double *dE);
int orc_advance(const orc_problem *p, double *U, double energy, double dE,
                double *energy_deposition /* (nx,ny,nz) */);

/* ---- the march (numerics/energy.py:energy_march) --------------------
 * U: in/out (4,nx,ny,nz); for the moving box U may be NULL (zero start).
 * dose: out (nx,ny,nz).  energies: out, capacity max_steps+1.
 * snap_targets: requested energies; snap_out receives one full state per
 * target actually reached, in descending target order, and
 * snap_energies_out the matching target energies.
 * max_threads <= 0 uses the OpenMP default.
 */
int orc_march(const orc_problem *p, double *U, double *dose,
              double *energies, int max_steps, int *n_steps,
              const double *snap_targets, int n_snap,
              double *snap_out, double *snap_energies_out, int *n_snap_taken,
              int *final_state_written);

/* Bounded sample for timing: run at most `steps` energy steps of the march
 * from the configured start energy and return the number actually run. */
int orc_march_steps(const orc_problem *p, double *U, double *dose, int steps, int *n_done);

/* March through energies[0..n-1] instead of the CFL steps (n = 0: the CFL rule). */
int  orc_set_schedule(orc_problem *p, const double *energies, int n);
void orc_set_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
