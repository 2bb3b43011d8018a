// pdm1_device.cuh -- device-side data of a plan and helpers shared by the
// double-precision march (pdm1_march.cu) and the single-precision stencil
// kernels (pdm1_stage_fp32.cu).
#pragma once

#include "../../include/pdm1.h"
#include "pdm1_math.cuh"

#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace pdm1 {

constexpr int kMaxMat = 16;

// Learned moving box: proposer network 16 -> 64 -> 64 -> 6 (ReLU).
constexpr int kFeat = 16, kHid = 64, kOut = 6, kOutPad = 8;
constexpr int kParams = kHid * kFeat + kHid + kHid * kHid + kHid + kOut * kHid + kOut;

// Device form of a box model: BF16 weights [out][in] (the column-major B
// operand of mma.m16n8k16), FP32 biases, input normalisation and the map of
// the network's outputs to margins in cells.
struct BoxModelDev {
    __nv_bfloat16 W1[kHid * kFeat];
    __nv_bfloat16 W2[kHid * kHid];
    __nv_bfloat16 W3[kOutPad * kHid];
    float b1[kHid], b2[kHid], b3[kOutPad];
    float x_mean[kFeat], x_inv_std[kFeat];
    float y_scale[kOut], y_offset[kOut];
    int margin_min, margin_max, grow_cells, extra_max;
    double leak_tol;
};

int pack_box_model(const pdm1_box_model *m, BoxModelDev &out);

enum { ERR_DEV_RANGE = 1, ERR_DEV_MAXSTEPS = 2, ERR_DEV_NONFINITE = 4, ERR_DEV_CAPACITY = 8, ERR_DEV_TIMEOUT = 16 };
// ---------------------------------------------------------------------------
// Device-side plan data
// ---------------------------------------------------------------------------
struct MatDev {
    TableView sp, tr, nuc;
    double density, X0;
};

// A rectangular domain of the full grid: the whole grid, or the moving active box
// (numerics/moving_active_domain.py), with its tile decomposition.
struct DomainDev {
    int i0, j0, k0;          // origin in the full grid
    int nx, ny, nz;          // extent
    int tx, ty, tz;          // tile shape of the stage kernels
    int tiles_y, tiles_z, ntiles;
    int inflow;              // the domain's z-min face is the beam entrance (k0 == 0)
};

// Tile shape (cells) of the stage kernels; every shape holds one cell per
// thread of a 256-thread CTA.
struct TileDims {
    int x, y, z;
};

// One pencil beam of a march (numerics/boundary.py:63-114): spectrum, angular
// spread, transverse profile on the grid's z-min face, initial moving box.
struct BeamDev {
    double E_beam, sigma_E, rf;     // rf = exp(-angular_spread^2)
    const double *spatial;          // (nx, ny): n_protons * normalised profile
    DomainDev init_box;             // moving_active_domain.py:35-60
};

// What the host polls between graph replays.
struct MarchSummary {
    int active;         // beams that marched in the last step
    int error;          // OR of the beams' error flags
};

struct ConfigDev {
    int nx, ny, nz;
    double dx, dy, dz;
    int nm;
    int scattering, nuclear, interp, scheme, unit_speeds;
    int cfl_floor;       // moving box: CFL bound at least the phantom's vacuum bound
    unsigned present;    // bit m: material m occurs in the phantom
    int spatial;         // PDM1_SPATIAL_*: the reconstruction
    int stencil_radius;  // its ghost width (vacuum-aware CFL masks)
    int use_if;          // integrating factors active (IF_SSPRK3 with sources)
    int strang;          // Strang-split sources around an SSPRK3 / Euler step
    double cfl, max_dE, Emin;
    int max_steps;
    int step_limit;      // >= 0: stop (without error) after this many steps
    int n_targets;
    const int32_t *ids;
    const double *targets;      // descending
    // beams: per-beam buffers hold `cap` cells each (the beam's domain)
    int nbeams;
    size_t cap;
    const BeamDev *beams;
    int *tile_off;              // (nbeams + 1) prefix sums of the active beams' tiles
    MarchSummary *summary;
    // moving active box
    int moving, vacuum_aware, guard;
    double tol;                 // exp(-sigma_trunc^2 / 2)
    double *bufA, *bufB;        // compact-state ping-pong, 4*cap per beam
    unsigned long long *slab;   // max phi per x | y | z slab of the box (double bits), per beam
    unsigned char *active;      // vacuum-aware activity mask on the box, cap per beam
    int grid_ctas;              // persistent grid of the stage kernels
    TileDims tile;              // tile shape of the stage kernels (kTiles[tile_id])
    int tile_id;
    int fp32;                   // FP32-stencil form: float eigenvalues in the CFL bound (not with cfl_floor)
    int bulk_stage;             // FP32 form: stages B and C stage their float4 source by bulk copies
    const double *schedule;     // prescribed energies E_0 .. E_{n-1} (replaces the CFL step), or NULL
    int n_schedule;
    // learned moving box and training-data recorder
    int learned;                // a box model proposes the margins
    const BoxModelDev *model;
    double *acc;                // per beam kAcc doubles: fluence moments and face currents of the box
    double *plane;              // per beam nz doubles: current through each z plane of the box
    float *rec;                 // recorder rows (one-beam full-domain plans), or NULL
    int rec_max;
    double rec_tail_tol[2];     // recorder: the two fluence-tail thresholds
    MatDev mats[kMaxMat];
};

// Layout of a beam's accumulator (cell coordinates are global cell centres,
// in cells): sums over the box of phi, phi x, phi y, phi z, phi x^2, phi y^2,
// phi z^2, Jx, Jy, Jz, |Jx|, |Jy|, then the current |J.n| summed over the
// cells of the box faces x-, x+, y-, y+, z-, z+ that lie inside the phantom
// (the entrance face excluded), then max phi.
enum { ACC_M = 0, ACC_X = 1, ACC_X2 = 4, ACC_J = 7, ACC_JABS = 10, ACC_FACE = 12, ACC_MAX = 18, kAcc = 20 };

struct Coeffs {
    double E, dE, E_next;
    int active;
    int snap_slot;
    double S0[kMaxMat], S1[kMaxMat], S2[kMaxMat];
    double c1p[kMaxMat], c1c[kMaxMat], c1ip[kMaxMat], c1ic[kMaxMat];
    double c2p[kMaxMat], c2c[kMaxMat], c2ip[kMaxMat], c2ic[kMaxMat];
    double Sb[4][kMaxMat];                  // S at E, E-dE/3, E-2dE/3, E-dE
    double fip[4][kMaxMat], fic[4][kMaxMat];   // inverse factors at those depths
    double ed[4];                           // spectrum at those energies
    double ed_next;                         // spectrum at E_next (CFL inflow)
    double hn[kMaxMat], hs[kMaxMat];        // Strang half-step factors
    double S_cfl[kMaxMat];                  // moving box: S at the step's start energy
    double ed_cfl;                          // moving box: spectrum at that energy
};

struct MarchState {
    double E;
    unsigned long long inv_bits;   // CFL max (non-negative double bits)
    double forced_dE;              // > 0: one step with this dE (pdm1_advance)
    int step, done, ti, taken, error;
    DomainDev dom;                 // the domain the stage kernels work on
    DomainDev prev;                // moving box before this step's rebox
    double *Ua;                    // state on `dom`
    double *Uprev;                 // state on `prev`
    int reboxed;
    unsigned long long newmax_bits;   // max phi over the new box (vacuum-aware CFL)
    double pin_max;                // max inflow phi over the new box
    double cell_steps;             // sum over steps of the cells marched (domain volume)
    double max_cells;              // largest domain marched in one step
    // learned box
    int sig[6];                    // significant box (global, half-open); sig[1] < 0: none
    double sig_scale;              // max(phi, phi_in) the threshold was taken from
    int extra[6];                  // growth per face from the outgoing-flux check
    int fallback;                  // 0 learned, 1 full domain, 2 heuristic box
    int grows;                     // faces grown by the check
    int margin[6];                 // margins of the last box
};

__host__ __device__ inline DomainDev make_domain(int i0, int j0, int k0, int nx, int ny, int nz, int inflow,
                                                 TileDims t);


// ---------------------------------------------------------------------------
// Material coefficients (device), mirroring physics/*.py
// ---------------------------------------------------------------------------
__device__ inline bool stopping_power_dev(const MatDev &m, double E, double &out) {
    if (!clip_energy(m.sp, E)) return false;
    if (E == m.sp.E[m.sp.n - 1]) { out = m.sp.v[m.sp.n - 1]; return true; }
    out = pchip_eval(m.sp, E);
    return true;
}

__device__ inline bool transport_dev(const ConfigDev &cf, const MatDev &m, double E, double &out) {
    if (cf.scattering == PDM1_SCATTERING_OFF) { out = 0.0; return true; }
    if (cf.scattering == PDM1_SCATTERING_ROSSI) {
        double e = E > 1.0e-8 ? E : 1.0e-8;
        double M = kProtonRestMev;
        double pv = e * (e + 2.0 * M) / (e + M);
        double r = kRossiEsMev / pv;
        out = r * r / m.X0;
        return true;
    }
    if (!clip_energy(m.tr, E)) return false;
    out = cf.interp == PDM1_INTERP_LINEAR ? linear_eval(m.tr, E) : pchip_eval(m.tr, E);
    return true;
}

__device__ inline bool nuclear_dev(const ConfigDev &cf, const MatDev &m, double E, double &out) {
    if (!clip_energy(m.nuc, E)) return false;
    out = cf.interp == PDM1_INTERP_LINEAR ? linear_eval(m.nuc, E) : pchip_eval(m.nuc, E);
    return true;
}

// numerics/boundary.py:82-114 spectrum factor
__device__ __forceinline__ double energy_density(const BeamDev &bm, double E) {
    double de = E - bm.E_beam;
    double s = bm.sigma_E;
    return dd_exp(-(de * de) / (2.0 * (s * s))) / (sqrt(2.0 * 3.141592653589793) * s);
}

__device__ __forceinline__ void source_factor(double ts, double tn, bool inverse, double &fp, double &fc) {
    double sign = inverse ? 1.0 : -1.0;
    double a = tn < kExpClamp ? tn : kExpClamp;
    double tsum = tn + ts;
    double b = tsum < kExpClamp ? tsum : kExpClamp;
    fp = dd_exp(sign * a);
    fc = dd_exp(sign * b);
}

// ---------------------------------------------------------------------------
// The fused stage kernel
// ---------------------------------------------------------------------------
constexpr int NT = 256;   // threads of a stage CTA = cells of a tile

// A tile shape: the tile's cells, its cross-shaped 3-cell WENO halo (no
// corners: WENO reads along one axis at a time) and its faces.  Shared memory
// holds three arms per component, each the core plus the halo along one axis
// (the core stored three times), so every 6-point stencil is a strided run in
// one arm.
template <int X, int Y, int Z>
struct Tile {
    static constexpr int NT = X * Y * Z;   // threads of the CTA: one cell each
    static_assert(NT == 256 || NT == 512, "256- or 512-cell tiles");
    static constexpr int TX = X, TY = Y, TZ = Z;
    static constexpr int NFX = (X + 1) * Y * Z, NFY = X * (Y + 1) * Z, NFZ = X * Y * (Z + 1);
    static constexpr int NF = NFX + NFY + NFZ;
    static constexpr int SX = (X + 6) * Y * Z;   // x-arm loads (core and x halo)
    static constexpr int SY = X * 6 * Z;         // y halo loads
    static constexpr int SZ = X * Y * 6;         // z halo loads
    static constexpr int AX = (X + 6) * Y * Z;   // arm sizes per component
    static constexpr int AY = X * (Y + 6) * Z;
    static constexpr int AZ = X * Y * (Z + 6);
    template <typename T>
    static constexpr size_t smem_bytes() { return sizeof(T) * 4 * (AX + AY + AZ + NF); }
};

// The tile shapes the stage kernels are built for, the autotuner's candidates.
// (An 8x8x8 tile of 512 threads, 3.375 faces per cell against 3.5-3.7, was
// measured slower: 0.674 against 0.606 ns per cell-step on a 51-spot pelvis batch
// in the FP32 form, with half as many CTAs per SM and twice the warps per barrier.)
constexpr int kNumTiles = 3;
using Tile0 = Tile<4, 8, 8>;
using Tile1 = Tile<8, 8, 4>;
using Tile2 = Tile<2, 8, 16>;
constexpr TileDims kTiles[kNumTiles] = {{4, 8, 8}, {8, 8, 4}, {2, 8, 16}};
constexpr int kMaxTileZ = 16;

__host__ __device__ inline DomainDev make_domain(int i0, int j0, int k0, int nx, int ny, int nz, int inflow,
                                                 TileDims t) {
    DomainDev d;
    d.i0 = i0; d.j0 = j0; d.k0 = k0;
    d.nx = nx; d.ny = ny; d.nz = nz;
    d.tx = t.x; d.ty = t.y; d.tz = t.z;
    d.tiles_y = (ny + t.y - 1) / t.y;
    d.tiles_z = (nz + t.z - 1) / t.z;
    d.ntiles = ((nx + t.x - 1) / t.x) * d.tiles_y * d.tiles_z;
    d.inflow = inflow;
    return d;
}

enum StageMode { MODE_A = 0, MODE_B = 1, MODE_C = 2, MODE_EULER = 3, MODE_RHS = 4,
                 MODE_C_LEARN = 5 };   // launch selector: stage C with the learned box's moments

struct StageArgs {
    const ConfigDev *cf;
    const Coeffs *co;   // per beam
    MarchState *st;     // per beam
    double *U1;         // stage states (on the beam's domain), 4*cap per beam
    double *U2;
    double *V;          // marched variable of stage 1 / 2
    double *qpart;      // (q0 + q1)/6 quadrature part
    double *dose;       // accumulated dose (full grid), or NULL
    double *edep;       // when non-NULL: energy deposition written instead of dose
    double *snap;       // snapshot buffer base (slot * 4N, full grid)
    double *rhs_out;    // MODE_RHS output
    const double *bc_plane;   // MODE_RHS: explicit z-min boundary state (4,nx,ny)
    double rhs_energy_density;
};

template <typename T>
struct SmemT {
    T *X, *Y, *Z, *F;
};


__device__ __forceinline__ size_t global_cell(const ConfigDev &cf, const DomainDev &d, int li, int lj, int lk) {
    return ((size_t)(d.i0 + li) * cf.ny + (d.j0 + lj)) * cf.nz + (d.k0 + lk);
}

// Stencil source value at a domain cell; indices outside the domain are
// clamped (zero-gradient ghosts, numerics/boundary.py:327-397).
template <int MODE>
__device__ __forceinline__ void load_cell(const ConfigDev &cf, const Coeffs &co, const DomainDev &d,
                                          const double *src, int li, int lj, int lk, double out[4]) {
    const int nx = d.nx, ny = d.ny, nz = d.nz;
    const size_t N = (size_t)nx * ny * nz;
    li = li < 0 ? 0 : (li >= nx ? nx - 1 : li);
    lj = lj < 0 ? 0 : (lj >= ny ? ny - 1 : lj);
    lk = lk >= nz ? nz - 1 : lk;
    size_t o = ((size_t)li * ny + lj) * nz + lk;
#pragma unroll
    for (int c = 0; c < 4; ++c) out[c] = src[c * N + o];
    if ((MODE == MODE_A || MODE == MODE_EULER) && cf.strang) {
        int m = cf.ids[global_cell(cf, d, li, lj, lk)];
        double hn = co.hn[m], hs = co.hs[m];
        if (cf.nuclear)
#pragma unroll
            for (int c = 0; c < 4; ++c) out[c] *= hn;
        if (cf.scattering != PDM1_SCATTERING_OFF)
#pragma unroll
            for (int c = 1; c < 4; ++c) out[c] *= hs;
    }
}

// z-min boundary value of component c at domain column (li, lj) for this stage.
// A moving box away from the entrance has zero inflow (moving_active_domain.py:85-95).
template <int MODE>
__device__ __forceinline__ double boundary_value(const StageArgs &a, const ConfigDev &cf, const BeamDev &bm,
                                                 const Coeffs &co, const DomainDev &d, int c, int li, int lj) {
    if (MODE == MODE_RHS && a.bc_plane)
        return a.bc_plane[((size_t)c * d.nx + li) * d.ny + lj];
    if (!d.inflow || c == 1 || c == 2) return 0.0;
    const int gi = d.i0 + li, gj = d.j0 + lj;
    double sp = bm.spatial[(size_t)gi * cf.ny + gj];
    if (MODE == MODE_A || MODE == MODE_EULER || MODE == MODE_RHS) {
        double ed = MODE == MODE_RHS ? a.rhs_energy_density : co.ed[0];
        double phi = sp * ed;
        return c == 0 ? phi : bm.rf * phi;
    }
    // RK-consistent stage traces, numerics/energy.py:348-455 (107-231 without sources)
    int m = cf.ids[((size_t)gi * cf.ny + gj) * cf.nz];
    double V[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        double phi = sp * co.ed[q];
        double x = c == 0 ? phi : bm.rf * phi;
        double B = co.Sb[q][m] * x;
        if (q > 0 && cf.use_if) B *= (c == 0 ? co.fip[q][m] : co.fic[q][m]);
        V[q] = B;
    }
    if (MODE == MODE_B) {
        double vs1 = 0.5 * (-9.0 * V[0] + 18.0 * V[1] - 9.0 * V[2] + 2.0 * V[3]);
        if (cf.use_if) vs1 *= (c == 0 ? co.c1p[m] : co.c1c[m]);
        return vs1 / co.S1[m];
    }
    double vs2 = 0.25 * (11.0 * V[0] - 27.0 * V[1] + 27.0 * V[2] - 7.0 * V[3]);
    if (cf.use_if) vs2 *= (c == 0 ? co.c2p[m] : co.c2c[m]);
    return vs2 / co.S2[m];
}

// One cell's CFL term (numerics/energy.py:539-660): sum over axes of a/(S d).
// `entrance`: the cell is on the domain's z-min layer, where the inflow state
// (zero for a box away from the entrance) joins the z speeds.
// T: the precision of the eigenvalues -- double for the FP64 march, float for
// the FP32-stencil form (its step sequence need not match the FP64 one).
template <typename T>
__device__ __forceinline__ double cfl_term(const ConfigDev &cf, double rf, const double u[4], double s,
                                           bool entrance, double phi_in, const bool use[3]) {
    double a0, a1, a2;
    if (cf.unit_speeds) {
        a0 = a1 = a2 = 1.0;
    } else {
        const T p = T(u[0]), x = T(u[1]), y = T(u[2]), z = T(u[3]);
        T a[3];
        max_abs_speeds3(p, x, y, z, a);
        a0 = double(a[0]);
        a1 = double(a[1]);
        a2 = double(a[2]);
        if (entrance) {
            T pin = T(phi_in);
            T jz = T(rf) * pin;
            double ain = double(max_abs_speed(pin, T(0), T(0), jz, 2));
            if (ain > a2) a2 = ain;
        }
    }
    if (!use[0]) a0 = 0.0;
    if (!use[1]) a1 = 0.0;
    if (!use[2]) a2 = 0.0;
    return a0 / (s * cf.dx) + a1 / (s * cf.dy) + a2 / (s * cf.dz);
}

template <int THREADS = NT>
__device__ __forceinline__ void block_max_atomic(double v, unsigned long long *target) {
    // v >= 0 or NaN; NaN never wins (fmax), like the oracle's comparison loop
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    __shared__ double wmax[THREADS / 32];
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) wmax[w] = v;
    __syncthreads();
    if (w == 0) {
        v = l < THREADS / 32 ? wmax[l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (l == 0 && v > 0.0) atomicMax(target, (unsigned long long)__double_as_longlong(v));
    }
}

__device__ __forceinline__ void atomic_max_double(unsigned long long *target, double v) {
    if (v > 0.0) atomicMax(target, (unsigned long long)__double_as_longlong(v));
}

// Per-slab maxima of phi over one tile (moving box): cell values in `buf`
// (one per cell of the tile, (i, j, k) with k fastest; -1 outside the box).
__device__ __forceinline__ void tile_slab_max(const ConfigDev &cf, unsigned long long *slab, const DomainDev &d,
                                              const double *buf, int i0, int j0, int k0) {
    int t = threadIdx.x;
    const int TX = d.tx, TY = d.ty, TZ = d.tz;
    unsigned long long *sx = slab, *sy = slab + cf.nx, *sz = slab + cf.nx + cf.ny;
    if (t < TX) {
        double m = 0.0;
        for (int e = 0; e < TY * TZ; ++e) m = fmax(m, buf[t * TY * TZ + e]);
        if (i0 + t < d.nx) atomic_max_double(&sx[i0 + t], m);
    } else if (t < TX + TY) {
        int j = t - TX;
        double m = 0.0;
        for (int i = 0; i < TX; ++i)
            for (int k = 0; k < TZ; ++k) m = fmax(m, buf[(i * TY + j) * TZ + k]);
        if (j0 + j < d.ny) atomic_max_double(&sy[j0 + j], m);
    } else if (t < TX + TY + TZ) {
        int k = t - TX - TY;
        double m = 0.0;
        for (int i = 0; i < TX; ++i)
            for (int j = 0; j < TY; ++j) m = fmax(m, buf[(i * TY + j) * TZ + k]);
        if (k0 + k < d.nz) atomic_max_double(&sz[k0 + k], m);
    }
}

// Beam owning global tile t of the step: tile_off holds the exclusive prefix
// sums of the beams' tile counts (beams that do not march have none).
__device__ __forceinline__ int beam_of_tile(const int *tile_off, int nbeams, int t) {
    int lo = 0, hi = nbeams - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (tile_off[mid] <= t) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ unsigned long long *beam_slab(const ConfigDev &cf, int b) {
    return cf.slab + (size_t)b * (cf.nx + cf.ny + cf.nz);
}

// Learned box: one tile's contribution to the beam's fluence moments, face
// currents and z-plane currents (acc, plane) from the state u of each cell
// (cell (li, lj, lk) of domain d, `valid` inside it).  Called by every thread
// of a CTA of THREADS threads laid out as the stage tile (k fastest); `part` and
// `pl` are shared scratch of THREADS/32 x (ACC_MAX + 1) and kMaxTileZ doubles.
template <int THREADS = NT>
__device__ __forceinline__ void tile_moments_cta(const ConfigDev &cf, int b, const DomainDev &d, int k0,
                                                 bool valid, int li, int lj, int lk, const double u[4],
                                                 double (*part)[ACC_MAX + 1], double *pl) {
    constexpr int kSums = ACC_MAX;   // summed entries; max phi separately
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int kk = tid % d.tz;
    if (tid < d.tz) pl[tid] = 0.0;
    double v[kSums + 1];
#pragma unroll
    for (int q = 0; q <= kSums; ++q) v[q] = 0.0;
    if (valid) {
        const double phi = u[0], jx = u[1], jy = u[2], jz = u[3];
        const double gx = d.i0 + li + 0.5, gy = d.j0 + lj + 0.5, gz = d.k0 + lk + 0.5;
        v[ACC_M] = phi;
        v[ACC_X] = phi * gx; v[ACC_X + 1] = phi * gy; v[ACC_X + 2] = phi * gz;
        v[ACC_X2] = phi * gx * gx; v[ACC_X2 + 1] = phi * gy * gy; v[ACC_X2 + 2] = phi * gz * gz;
        v[ACC_J] = jx; v[ACC_J + 1] = jy; v[ACC_J + 2] = jz;
        v[ACC_JABS] = fabs(jx); v[ACC_JABS + 1] = fabs(jy);
        if (li == 0 && d.i0 > 0) v[ACC_FACE + 0] = fabs(jx);
        if (li == d.nx - 1 && d.i0 + d.nx < cf.nx) v[ACC_FACE + 1] = fabs(jx);
        if (lj == 0 && d.j0 > 0) v[ACC_FACE + 2] = fabs(jy);
        if (lj == d.ny - 1 && d.j0 + d.ny < cf.ny) v[ACC_FACE + 3] = fabs(jy);
        if (lk == 0 && d.k0 > 0) v[ACC_FACE + 4] = fabs(jz);
        if (lk == d.nz - 1 && d.k0 + d.nz < cf.nz) v[ACC_FACE + 5] = fabs(jz);
        v[kSums] = phi;
    }
    __syncthreads();   // pl zeroed
    atomicAdd(&pl[kk], v[ACC_J + 2]);
#pragma unroll
    for (int q = 0; q < kSums; ++q)
        for (int w = 16; w > 0; w >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], w);
    for (int w = 16; w > 0; w >>= 1) v[kSums] = fmax(v[kSums], __shfl_xor_sync(0xffffffffu, v[kSums], w));
    if (lane == 0)
        for (int q = 0; q <= kSums; ++q) part[warp][q] = v[q];
    __syncthreads();
    double *acc = cf.acc + (size_t)b * kAcc;
    if (tid < kSums) {
        double s = 0.0;
        for (int w = 0; w < THREADS / 32; ++w) s += part[w][tid];
        if (s != 0.0) atomicAdd(&acc[tid], s);
    } else if (tid == kSums) {
        double m = 0.0;
        for (int w = 0; w < THREADS / 32; ++w) m = fmax(m, part[w][kSums]);
        atomic_max_double(reinterpret_cast<unsigned long long *>(&acc[ACC_MAX]), m);
    } else if (tid >= 32 && tid < 32 + d.tz) {
        const int k = tid - 32;
        if (k0 + k < d.nz && pl[k] != 0.0) atomicAdd(&cf.plane[(size_t)b * cf.nz + d.k0 + k0 + k], pl[k]);
    }
    __syncthreads();
}

// The significant box of desired_box (moving_active_domain.py:107-151):
// scale = max(max phi, max phi_in) (phi_in only while the domain touches
// z = 0), then the first and last x / y / z slab of `d` whose max phi exceeds
// tol * scale (the plan's tolerance for the moving box), an inflow cell above
// it joining the k = 0 layer.  Called by all threads of a CTA of 256 (8
// warps) with `red` = 512 doubles of shared memory; results (local indices,
// hi < 0 when none) in the caller's shared memory.
__device__ inline void significant_box_cta(const ConfigDev &cf, const BeamDev &bm, const DomainDev &d,
                                           const unsigned long long *slab, double ed, double *red, int *s_lo,
                                           int *s_hi, double *s_scale, double tol) {
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const unsigned long long *sx = slab, *sy = slab + cf.nx, *sz = slab + cf.nx + cf.ny;
    auto as_d = [](unsigned long long b) { return __longlong_as_double((long long)b); };
    auto inflow = [&](int i, int j) { return bm.spatial[(size_t)(d.i0 + i) * cf.ny + (d.j0 + j)] * ed; };
    // the state's maximum (slab maxima) and the inflow's over the box's entrance
    double m = 0.0, mi = 0.0;
    for (int i = t; i < d.nx; i += 256) m = fmax(m, as_d(sx[i]));
    if (d.inflow)
        for (int e = t; e < d.nx * d.ny; e += 256) mi = fmax(mi, inflow(e / d.ny, e % d.ny));
    red[t] = m;
    red[256 + t] = mi;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (t < w) {
            red[t] = fmax(red[t], red[t + w]);
            red[256 + t] = fmax(red[256 + t], red[256 + t + w]);
        }
        __syncthreads();
    }
    if (t == 0) {
        *s_scale = fmax(red[0], red[256]);
        for (int q = 0; q < 3; ++q) { s_lo[q] = 0x7fffffff; s_hi[q] = -1; }
    }
    __syncthreads();
    const double scale = *s_scale;
    const double thr = tol * scale;
    // an inflow cell above the threshold exists iff the inflow's maximum is above it
    const bool inflow_on = d.inflow && red[256] > thr;
    if (scale != 0.0) {
        // one warp per x slab (y slab): the slab maximum, or any inflow cell of
        // the slab's entrance row above the threshold
        for (int i = warp; i < d.nx; i += 8) {
            bool act = as_d(sx[i]) > thr;
            if (!act && inflow_on) {
                bool any = false;
                for (int j = lane; j < d.ny; j += 32) any = any || inflow(i, j) > thr;
                act = __any_sync(0xffffffffu, any);
            }
            if (act && lane == 0) { atomicMin(&s_lo[0], i); atomicMax(&s_hi[0], i); }
        }
        for (int j = warp; j < d.ny; j += 8) {
            bool act = as_d(sy[j]) > thr;
            if (!act && inflow_on) {
                bool any = false;
                for (int i = lane; i < d.nx; i += 32) any = any || inflow(i, j) > thr;
                act = __any_sync(0xffffffffu, any);
            }
            if (act && lane == 0) { atomicMin(&s_lo[1], j); atomicMax(&s_hi[1], j); }
        }
        for (int k = t; k < d.nz; k += 256) {
            const bool act = as_d(sz[k]) > thr || (k == 0 && inflow_on);
            if (act) { atomicMin(&s_lo[2], k); atomicMax(&s_hi[2], k); }
        }
    }
    __syncthreads();
}

// Switch a beam to the box `nb` (one thread): the capacity check, the
// compact-state ping-pong, the spectrum for the CFL bound and, for the
// vacuum-aware CFL (energy.py:496-537), the max inflow over the new box.
__device__ inline void switch_box(const ConfigDev &cf, const BeamDev &bm, Coeffs *co, MarchState *st, int b,
                                  DomainDev nb, double ed) {
    const DomainDev d = st->dom;
    bool same = nb.i0 == d.i0 && nb.j0 == d.j0 && nb.k0 == d.k0 && nb.nx == d.nx && nb.ny == d.ny && nb.nz == d.nz;
    if (!same && (size_t)nb.nx * nb.ny * nb.nz > cf.cap) {
        st->error |= ERR_DEV_CAPACITY;   // the box outgrew the beam's buffers
        same = true;
    }
    st->reboxed = same ? 0 : 1;
    if (!same) {
        st->prev = d;
        st->Uprev = st->Ua;
        double *a_buf = cf.bufA + 4 * (size_t)b * cf.cap, *b_buf = cf.bufB + 4 * (size_t)b * cf.cap;
        st->Ua = st->Ua == a_buf ? b_buf : a_buf;
        st->dom = nb;
    }
    st->inv_bits = 0ull;
    co->ed_cfl = ed;
    st->newmax_bits = 0ull;
    double pin = 0.0;
    if (cf.vacuum_aware && nb.inflow)
        for (int e = 0; e < nb.nx * nb.ny; ++e)
            pin = fmax(pin, bm.spatial[(size_t)(nb.i0 + e / nb.ny) * cf.ny + (nb.j0 + e % nb.ny)] * ed);
    st->pin_max = pin;
}

// Learned box and recorder kernels (pdm1_box.cu).
void launch_box_moments(const ConfigDev *d_cf, const MarchState *d_st, int grid, int record, cudaStream_t stream);
void launch_box_learn(const ConfigDev *d_cf, Coeffs *d_co, MarchState *d_st, int nbeams, cudaStream_t stream);
void launch_record(const ConfigDev *d_cf, const Coeffs *d_co, MarchState *d_st, cudaStream_t stream);

// Record an error message for pdm1_last_error() and return `code`.
int report_error(int code, const char *msg);

// The plans' caching allocator (pdm1_pool.cu): device blocks of the current
// device and pinned host blocks, reused by size; pool_free of a pointer the
// pool did not hand out is ignored.
cudaError_t pool_malloc(void **ptr, size_t bytes);
cudaError_t pool_malloc_host(void **ptr, size_t bytes);
void pool_free(void *ptr);

// Single-precision stencil kernels (pdm1_stage_fp32.cu, compiled with fast math).
int stage_fp32_set_attributes();
void launch_stage_fp32(int mode, int tile_id, int grid, const StageArgs &a, cudaStream_t stream);

}  // namespace pdm1
