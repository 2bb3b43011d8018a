// pdm1_march.cu -- the M1 energy march on sm_100a.
//
// Per energy step the device runs
//   prologue   one CTA: CFL step from the previous stage-3 reduction, snapshot
//              landing, per-material stopping powers, optical depths and
//              integrating factors at the stage energies
//              (numerics/energy.py:539-660, 234-455, 878-1130)
//   stage A/B/C  the three IF-SSPRK3 stages, each ONE fused kernel: stage a
//              tile of the stencil source plus its 3-cell WENO halo in shared
//              memory (ghost cells of numerics/boundary.py:117-399 patched in
//              shared memory), WENO-Z + projection + HLL on every face of the
//              tile, divergence, integrating-factor update and projection in
//              registers; stage C also accumulates the dose and reduces the
//              next CFL bound with warp shuffles and one atomic per CTA.
// No host synchronisation inside a step: the energy, dE and all per-step
// coefficients live in device memory, so chunks of steps are captured once
// into a CUDA graph and replayed until the device flags the march done.
#include "../../include/pdm1.h"
#include "pdm1_math.cuh"
#include "pdm1_device.cuh"
#include "pdm1_stage.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

using namespace pdm1;

namespace {

constexpr int kStepsPerGraph = 32;

// fixed-size message buffer: reporting an error allocates nothing
thread_local char g_error[512];

int set_error(int code, const char *msg) {
    snprintf(g_error, sizeof g_error, "%s", msg);
    return code;
}

int set_error(int code, const std::string &msg) { return set_error(code, msg.c_str()); }

#define CUDA_TRY(expr)                                                                    \
    do {                                                                                  \
        cudaError_t e_ = (expr);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return set_error(PDM1_ERR_CUDA, std::string(#expr ": ") + cudaGetErrorString(e_)); \
    } while (0)

// ---------------------------------------------------------------------------
// init: state at the start energy, S and spectrum for the first CFL
// ---------------------------------------------------------------------------
// One CTA per beam.  E0 < 0: each beam starts at its own E + window * sigma_E.
__global__ void init_kernel(const ConfigDev *cfp, Coeffs *cos, MarchState *sts, double *energies,
                            double E0, double ews, double *U, int full_domain) {
    const ConfigDev &cf = *cfp;
    const int b = blockIdx.x;
    const BeamDev &bm = cf.beams[b];
    Coeffs *co = cos + b;
    MarchState *st = sts + b;
    if (E0 < 0.0) E0 = bm.E_beam + ews * bm.sigma_E;
    int t = threadIdx.x;
    if (t < cf.nm) {
        double s;
        if (!stopping_power_dev(cf.mats[t], E0, s)) atomicOr(&st->error, ERR_DEV_RANGE);
        co->S1[t] = s;
    }
    if (t == 0) {
        co->ed_next = energy_density(bm, E0);
        co->E_next = E0;
        st->E = E0;
        st->inv_bits = 0ull;
        st->forced_dE = 0.0;
        st->step = 0;
        st->done = 0;
        st->ti = 0;
        st->taken = 0;
        st->error = 0;
        st->reboxed = 0;
        st->newmax_bits = 0ull;
        st->pin_max = 0.0;
        st->cell_steps = 0.0;
        st->max_cells = 0.0;
        for (int q = 0; q < 6; ++q) { st->sig[q] = -1; st->extra[q] = 0; st->margin[q] = 0; }
        st->sig_scale = 0.0;
        st->fallback = 0;
        st->grows = 0;
        const bool moving = cf.moving && !full_domain;
        st->dom = moving ? bm.init_box : make_domain(0, 0, 0, cf.nx, cf.ny, cf.nz, 1, cf.tile);
        st->prev = st->dom;
        st->Ua = moving ? cf.bufA + 4 * (size_t)b * cf.cap : U;
        st->Uprev = st->Ua;
        if (energies && cf.nbeams == 1) energies[0] = E0;
        if (b == 0) {
            cf.tile_off[0] = 0;
            cf.tile_off[1] = 0;
            cf.summary->active = cf.nbeams;
            cf.summary->error = 0;
        }
    }
}

// Exclusive prefix sums of the marching beams' tile counts, and the summary
// the host polls.  One CTA; beams are processed in chunks of blockDim.x.
__global__ void __launch_bounds__(1024) tiles_kernel(const ConfigDev *cfp, const Coeffs *co,
                                                     const MarchState *st) {
    const ConfigDev &cf = *cfp;
    __shared__ int scan[1024];
    __shared__ int carry, n_active, err;
    const int t = threadIdx.x;
    if (t == 0) { carry = 0; n_active = 0; err = 0; }
    __syncthreads();
    for (int base = 0; base < cf.nbeams; base += blockDim.x) {
        const int b = base + t;
        int n = 0;
        if (b < cf.nbeams) {
            if (co[b].active) {
                n = st[b].dom.ntiles;
                atomicAdd(&n_active, 1);
            }
            if (st[b].error) atomicOr(&err, st[b].error);
        }
        scan[t] = n;
        __syncthreads();
        for (int o = 1; o < (int)blockDim.x; o <<= 1) {
            int v = t >= o ? scan[t - o] : 0;
            __syncthreads();
            scan[t] += v;
            __syncthreads();
        }
        if (b < cf.nbeams) cf.tile_off[b + 1] = carry + scan[t];
        __syncthreads();
        if (t == blockDim.x - 1) carry += scan[t];
        __syncthreads();
    }
    if (t == 0) {
        cf.tile_off[0] = 0;
        cf.summary->active = n_active;
        cf.summary->error = err;
    }
}

// ---------------------------------------------------------------------------
// prologue: one CTA per step
// ---------------------------------------------------------------------------
constexpr int kEvalPerMat = 13;   // 5 stage energies + 8 Gauss points

// One CTA per beam.
__global__ void __launch_bounds__(256) prologue_kernel(const ConfigDev *cfp, Coeffs *cos,
                                                       MarchState *sts, double *energies) {
    const ConfigDev &cf = *cfp;
    const int b = blockIdx.x;
    const BeamDev &bm = cf.beams[b];
    Coeffs *co = cos + b;
    MarchState *st = sts + b;
    if (cf.nbeams > 1) energies = nullptr;
    __shared__ double sE, sdE, sEn;
    __shared__ int sActive, sSlot;
    __shared__ double eS[kMaxMat][kEvalPerMat], eTr[kMaxMat][8], eNu[kMaxMat][8];
    __shared__ double gpt[8];
    int t = threadIdx.x;
    if (t == 0) {
        int active = 0, slot = -1;
        double E = st->E, dE = 0.0, En = E;
        if (!st->done && st->error == 0) {
            if (!(E > cf.Emin) || (cf.step_limit >= 0 && st->step >= cf.step_limit)) {
                st->done = 1;
            } else if (st->step >= cf.max_steps) {
                st->error |= ERR_DEV_MAXSTEPS;
                st->done = 1;
            } else {
                if (st->forced_dE > 0.0) {
                    dE = st->forced_dE;
                } else if (cf.schedule) {
                    // a prescribed energy schedule (another run's steps): the
                    // next energy is taken as given, past its end down to Emin
                    dE = st->step + 1 < cf.n_schedule ? E - cf.schedule[st->step + 1] : E - cf.Emin;
                } else {
                    double inv = __longlong_as_double((long long)st->inv_bits);
                    dE = cf.cfl / inv;
                    dE = cf.max_dE < dE ? cf.max_dE : dE;
                    if (st->ti < cf.n_targets) {
                        double tg = cf.targets[st->ti];
                        if (E > tg && tg >= E - dE) dE = E - tg;
                    }
                    if (E - cf.Emin < dE) dE = E - cf.Emin;
                }
                if (!(dE > 0.0) || !isfinite(dE)) {
                    st->error |= ERR_DEV_NONFINITE;
                    st->done = 1;
                } else {
                    active = 1;
                    En = E - dE;
                    if (cf.schedule && st->forced_dE <= 0.0 && st->step + 1 < cf.n_schedule)
                        En = cf.schedule[st->step + 1];
                    int step = st->step + 1;
                    if (energies) energies[step] = En;
                    if (st->ti < cf.n_targets && fabs(En - cf.targets[st->ti]) <= 1e-12) {
                        slot = st->taken;
                        st->taken += 1;
                        st->ti += 1;
                    }
                    st->step = step;
                    st->E = En;
                    const double cells = (double)st->dom.nx * st->dom.ny * st->dom.nz;
                    st->cell_steps += cells;
                    st->max_cells = fmax(st->max_cells, cells);
                    st->inv_bits = 0ull;
                    if (st->forced_dE > 0.0) st->done = 1;
                }
            }
        }
        sE = E; sdE = dE; sEn = En; sActive = active; sSlot = slot;
        co->E = E; co->dE = dE; co->E_next = En; co->active = active; co->snap_slot = slot;
        if (cf.nbeams == 1) {
            cf.tile_off[0] = 0;
            cf.tile_off[1] = active ? st->dom.ntiles : 0;
            cf.summary->active = active;
            cf.summary->error = st->error;
        }
    }
    __syncthreads();
    if (!sActive) return;
    const double E = sE, dE = sdE;
    // Gauss points for the depths over dE/3, dE/2, 2dE/3, dE (energy.py:919-949)
    if (t < 4) {
        const double width[4] = {dE / 3.0, 0.5 * dE, 2.0 * dE / 3.0, dE};
        double w = width[t];
        double mid = E - 0.5 * w;
        double half = 0.5 * w;
        double off = half / sqrt(3.0);
        gpt[2 * t] = mid - off;
        gpt[2 * t + 1] = mid + off;
    }
    __syncthreads();
    int nm = cf.nm;
    if (t < nm * kEvalPerMat) {
        int m = t / kEvalPerMat, q = t % kEvalPerMat;
        const MatDev &mat = cf.mats[m];
        bool ok = true;
        double e;
        if (q < 5) {
            const double stage_e[5] = {E, E - dE / 3.0, E - 2.0 * dE / 3.0, E - dE, E - 0.5 * dE};
            e = stage_e[q];
        } else {
            e = gpt[q - 5];
            double v = 0.0;
            ok &= transport_dev(cf, mat, e, v);
            eTr[m][q - 5] = v;
            v = 0.0;
            if (cf.nuclear) ok &= nuclear_dev(cf, mat, e, v);
            eNu[m][q - 5] = v;
        }
        double s = 1.0;
        ok &= stopping_power_dev(mat, e, s);
        eS[m][q] = s;
        if (!ok) atomicOr(&st->error, ERR_DEV_RANGE);
    } else if (t >= 224 && t < 229) {
        int q = t - 224;
        const double ed_e[5] = {E, E - dE / 3.0, E - 2.0 * dE / 3.0, E - dE, E - dE};
        double v = energy_density(bm, ed_e[q]);
        if (q < 4) co->ed[q] = v; else co->ed_next = v;
    }
    __syncthreads();
    __shared__ double sTs[kMaxMat][4], sTn[kMaxMat][4];
    if (t < nm) {
        int m = t;
        co->S0[m] = eS[m][0];
        co->S1[m] = eS[m][3];
        co->S2[m] = eS[m][4];
        co->Sb[0][m] = eS[m][0];
        co->Sb[1][m] = eS[m][1];
        co->Sb[2][m] = eS[m][2];
        co->Sb[3][m] = eS[m][3];
        // optical depths, physics/scattering.py:267-306 and nuclear.py:202-233
        // depth index: 0 -> dE/3, 1 -> dE/2, 2 -> 2dE/3, 3 -> dE
        const double width[4] = {dE / 3.0, 0.5 * dE, 2.0 * dE / 3.0, dE};
        for (int d = 0; d < 4; ++d) {
            double half = 0.5 * width[d];
            double ts = 0.0, tn = 0.0;
            if (cf.scattering != PDM1_SCATTERING_OFF)
                ts = half * (eTr[m][2 * d] / eS[m][5 + 2 * d] + eTr[m][2 * d + 1] / eS[m][6 + 2 * d]);
            if (cf.nuclear)
                tn = half * (eNu[m][2 * d] / eS[m][5 + 2 * d] + eNu[m][2 * d + 1] / eS[m][6 + 2 * d]);
            sTs[m][d] = ts;
            sTn[m][d] = tn;
        }
        co->fip[0][m] = 1.0;
        co->fic[0][m] = 1.0;
    }
    __syncthreads();
    // the 16 exponentials per material, one thread each (energy.py:273-310,
    // 1168-1191): integrating factors C(tau) and C(tau)^-1 over dE and dE/2,
    // the inverse factors of the inflow trace at dE/3, 2dE/3, dE, and the
    // Strang half-step factors
    if (t < nm * 16) {
        const int m = t / 16, f = t % 16;
        double ts = 0.0, tn = 0.0, out = 1.0;
        if (f < 14) {
            // which depth, and which factor of source_factor()
            const int depth[14] = {3, 3, 3, 3, 1, 1, 1, 1, 0, 0, 2, 2, 3, 3};
            const bool inv[14] = {false, false, true, true, false, false, true, true, true, true, true, true, true, true};
            const bool cur[14] = {false, true, false, true, false, true, false, true, false, true, false, true, false, true};
            if (cf.use_if) {
                ts = sTs[m][depth[f]];
                tn = sTn[m][depth[f]];
            }
            double sign = inv[f] ? 1.0 : -1.0;
            double a = tn < kExpClamp ? tn : kExpClamp;
            double tsum = tn + ts;
            double b = tsum < kExpClamp ? tsum : kExpClamp;
            out = dd_exp(sign * (cur[f] ? b : a));
            double *dst[14] = {&co->c1p[m], &co->c1c[m], &co->c1ip[m], &co->c1ic[m],
                               &co->c2p[m], &co->c2c[m], &co->c2ip[m], &co->c2ic[m],
                               &co->fip[1][m], &co->fic[1][m], &co->fip[2][m], &co->fic[2][m],
                               &co->fip[3][m], &co->fic[3][m]};
            *dst[f] = out;
        } else if (f == 14) {
            double th = 0.5 * sTn[m][3];
            co->hn[m] = (cf.strang && cf.nuclear) ? dd_exp(-(th < kExpClamp ? th : kExpClamp)) : 1.0;
        } else {
            double th = 0.5 * sTs[m][3];
            co->hs[m] = (cf.strang && cf.scattering != PDM1_SCATTERING_OFF)
                            ? dd_exp(-(th < kExpClamp ? th : kExpClamp)) : 1.0;
        }
    }
}

// Forward Euler writes U1; this copies it back, snapshots, and either reduces
// the CFL bound (static domain) or the slab maxima (moving box).
__global__ void __launch_bounds__(NT) euler_finish_kernel(StageArgs a) {
    const ConfigDev &cf = *a.cf;
    const Coeffs &co = *a.co;
    if (!co.active) return;
    const DomainDev d = a.st->dom;
    double *Ua = a.st->Ua;
    const size_t N = (size_t)d.nx * d.ny * d.nz, NG = (size_t)cf.nx * cf.ny * cf.nz;
    const bool all_axes[3] = {true, true, true};
    double inv = 0.0;
    for (size_t o = (size_t)blockIdx.x * NT + threadIdx.x; o < N; o += (size_t)gridDim.x * NT) {
        double u[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            u[c] = a.U1[c * N + o];
            Ua[c * N + o] = u[c];
        }
        int lk = (int)(o % d.nz), lj = (int)((o / d.nz) % d.ny), li = (int)(o / ((size_t)d.nz * d.ny));
        size_t go = global_cell(cf, d, li, lj, lk);
        if (co.snap_slot >= 0 && a.snap) {
            double *sn = a.snap + (size_t)co.snap_slot * 4 * NG;
#pragma unroll
            for (int c = 0; c < 4; ++c) sn[c * NG + go] = u[c];
        }
        if (cf.moving) {
            atomic_max_double(&cf.slab[li], u[0]);
            atomic_max_double(&cf.slab[cf.nx + lj], u[0]);
            atomic_max_double(&cf.slab[cf.nx + cf.ny + lk], u[0]);
        } else {
            const BeamDev &bm = cf.beams[0];
            double phi_in = 0.0;
            if (lk == 0 && d.inflow) phi_in = bm.spatial[(size_t)(d.i0 + li) * cf.ny + (d.j0 + lj)] * co.ed_next;
            double s = co.S1[cf.ids[go]];
            inv = fmax(inv, cf.fp32 ? cfl_term<float>(cf, bm.rf, u, s, lk == 0, phi_in, all_axes)
                                    : cfl_term<double>(cf, bm.rf, u, s, lk == 0, phi_in, all_axes));
        }
    }
    if (!cf.moving) block_max_atomic(inv, &a.st->inv_bits);
}

// One cell's CFL term on the beam's domain `d` (energy.py:539-660): the
// speeds of the state u and, on the entrance layer, of the inflow state at
// the spectrum value `ed`, over S of the cell's material.  The FP32 form takes
// float speeds, except with the phantom-wide bound, whose purpose is the
// plain method's step sequence.
__device__ __forceinline__ double cell_cfl(const ConfigDev &cf, const BeamDev &bm, const DomainDev &d,
                                           const double *S, double ed, const double u[4], int li, int lj, int lk,
                                           const bool use[3]) {
    double phi_in = 0.0;
    if (lk == 0 && d.inflow) phi_in = bm.spatial[(size_t)(d.i0 + li) * cf.ny + (d.j0 + lj)] * ed;
    const double s = S[cf.ids[global_cell(cf, d, li, lj, lk)]];
    return cf.fp32 && !cf.cfl_floor ? cfl_term<float>(cf, bm.rf, u, s, lk == 0, phi_in, use)
                                    : cfl_term<double>(cf, bm.rf, u, s, lk == 0, phi_in, use);
}

// The phantom-wide bound: the cells outside the box hold no fluence; on the
// full grid they would bound the step with the vacuum speed (wave_speeds.py:
// 36-103) in the material of least stopping power present.
__device__ __forceinline__ double phantom_cfl_floor(const ConfigDev &cf, const double *S) {
    double smin = INFINITY;
    for (int m = 0; m < cf.nm; ++m)
        if (cf.present >> m & 1u) smin = fmin(smin, S[m]);
    const double a = cf.unit_speeds ? 1.0 : 1.0 / sqrt(3.0);
    return a / (smin * cf.dx) + a / (smin * cf.dy) + a / (smin * cf.dz);
}

// CFL bound of the state on the current domain (energy.py:539-660), with S and
// the spectrum at the state's energy: co->S1 / ed_next (static domain, first
// step) or co->S_cfl / ed_cfl (moving box, every step; without vacuum-aware
// masks rebox_kernel computes it while it moves the box).  With vacuum-aware
// masks (energy.py:459-537) a direction counts only within 3 cells, along that
// axis, of an active cell.
__global__ void __launch_bounds__(NT) cfl_kernel(const ConfigDev *cfp, const Coeffs *cos, MarchState *sts,
                                                 int use_box_coeffs) {
    const ConfigDev &cf = *cfp;
    const int b = blockIdx.y;
    const Coeffs *co = cos + b;
    MarchState *st = sts + b;
    const BeamDev &bm = cf.beams[b];
    if (st->done || st->error) return;
    const DomainDev d = st->dom;
    const double *U = st->Ua;
    const size_t N = (size_t)d.nx * d.ny * d.nz;
    const double *S = use_box_coeffs ? co->S_cfl : co->S1;
    const double ed = use_box_coeffs ? co->ed_cfl : co->ed_next;
    bool masks = false;
    if (cf.moving && cf.vacuum_aware && use_box_coeffs) {
        double sc = fmax(__longlong_as_double((long long)st->newmax_bits), st->pin_max);
        masks = sc != 0.0;   // energy.py:518-523: no transported state and no beam -> all directions
    }
    double inv = 0.0;
    for (size_t o = (size_t)blockIdx.x * NT + threadIdx.x; o < N; o += (size_t)gridDim.x * NT) {
        double u[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) u[c] = U[c * N + o];
        int lk = (int)(o % d.nz), lj = (int)((o / d.nz) % d.ny), li = (int)(o / ((size_t)d.nz * d.ny));
        bool use[3] = {true, true, true};
        if (masks) {
            const unsigned char *act = cf.active + (size_t)b * cf.cap;
            for (int ax = 0; ax < 3; ++ax) {
                int lo, hi, pos;
                size_t stride;
                const int r = cf.stencil_radius;   // the reconstruction's ghost width, energy.py:611-622
                if (ax == 0) { pos = li; lo = max(0, li - r); hi = min(d.nx - 1, li + r); stride = (size_t)d.ny * d.nz; }
                else if (ax == 1) { pos = lj; lo = max(0, lj - r); hi = min(d.ny - 1, lj + r); stride = d.nz; }
                else { pos = lk; lo = max(0, lk - r); hi = min(d.nz - 1, lk + r); stride = 1; }
                bool any = false;
                for (int q = lo; q <= hi && !any; ++q) any = act[o + (long long)(q - pos) * (long long)stride] != 0;
                use[ax] = any;
            }
        }
        inv = fmax(inv, cell_cfl(cf, bm, d, S, ed, u, li, lj, lk, use));
    }
    if (cf.cfl_floor && use_box_coeffs && blockIdx.x == 0 && threadIdx.x == 0)
        inv = fmax(inv, phantom_cfl_floor(cf, S));
    block_max_atomic(inv, &st->inv_bits);
}

// ---------------------------------------------------------------------------
// Moving active box (numerics/moving_active_domain.py, energy.py:1262-1494)
// ---------------------------------------------------------------------------

// Start of the march: the initial box, the compact state copied from the
// caller's full-grid U, and the slab maxima of that state.
// blockIdx.y = beam; with Ufull == NULL the beams start from zero.
__global__ void __launch_bounds__(NT) box_init_kernel(const ConfigDev *cfp, MarchState *st, const double *Ufull) {
    const ConfigDev &cf = *cfp;
    const int b = blockIdx.y;
    const DomainDev d = cf.beams[b].init_box;
    const size_t N = (size_t)d.nx * d.ny * d.nz, NG = (size_t)cf.nx * cf.ny * cf.nz;
    double *Ua = cf.bufA + 4 * (size_t)b * cf.cap;
    unsigned long long *slab = beam_slab(cf, b);
    for (size_t o = (size_t)blockIdx.x * NT + threadIdx.x; o < N; o += (size_t)gridDim.x * NT) {
        int lk = (int)(o % d.nz), lj = (int)((o / d.nz) % d.ny), li = (int)(o / ((size_t)d.nz * d.ny));
        size_t go = global_cell(cf, d, li, lj, lk);
        double u0 = 0.0;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            double v = Ufull ? Ufull[c * NG + go] : 0.0;
            Ua[c * N + o] = v;
            if (c == 0) u0 = v;
        }
        atomic_max_double(&slab[li], u0);
        atomic_max_double(&slab[cf.nx + lj], u0);
        atomic_max_double(&slab[cf.nx + cf.ny + lk], u0);
    }
}

// One CTA at the start of every step: desired_box (moving_active_domain.py:
// 107-193) from the slab maxima of the current state and the inflow at the
// step's energy; the switch to the new box; S and spectrum for the CFL.
// One CTA per beam.  With a box model the significant box is kept for
// box_learn_kernel, which chooses the margins and switches the box.
__global__ void __launch_bounds__(256) box_kernel(const ConfigDev *cfp, Coeffs *cos, MarchState *sts) {
    const ConfigDev &cf = *cfp;
    const int b = blockIdx.x;
    const BeamDev &bm = cf.beams[b];
    Coeffs *co = cos + b;
    MarchState *st = sts + b;
    unsigned long long *slab = beam_slab(cf, b);
    __shared__ double red[512];   // significant_box_cta: two reductions
    __shared__ double s_ed, s_scale;
    __shared__ int s_lo[3], s_hi[3];
    __shared__ int s_done;
    const int t = threadIdx.x;
    if (t == 0) s_done = st->done || st->error;
    __syncthreads();
    if (s_done) return;
    const DomainDev d = st->dom;
    const double E = st->E;
    // init_kernel and prologue_kernel leave S1 = S(E_next) and ed_next =
    // spectrum(E_next), with E_next the energy this step starts from
    const bool known = co->E_next == E;
    if (t == 0) s_ed = known ? co->ed_next : energy_density(bm, E);
    if (t < cf.nm) {
        double sv = 1.0;
        if (known) sv = co->S1[t];
        else if (!stopping_power_dev(cf.mats[t], E, sv)) atomicOr(&st->error, ERR_DEV_RANGE);
        co->S_cfl[t] = sv;
    }
    __syncthreads();
    const double ed = s_ed;
    significant_box_cta(cf, bm, d, slab, ed, red, s_lo, s_hi, &s_scale, cf.tol);
    // reset the slab maxima for this step's stage C
    for (int e = t; e < cf.nx + cf.ny + cf.nz; e += 256) slab[e] = 0ull;
    if (t == 0) {
        const double scale = s_scale;
        const bool none = scale == 0.0 || s_hi[0] < 0 || s_hi[1] < 0 || s_hi[2] < 0;
        if (cf.learned) {
            st->sig[0] = none ? -1 : d.i0 + s_lo[0];
            st->sig[1] = none ? -1 : d.i0 + s_hi[0] + 1;
            st->sig[2] = none ? -1 : d.j0 + s_lo[1];
            st->sig[3] = none ? -1 : d.j0 + s_hi[1] + 1;
            st->sig[4] = none ? -1 : d.k0 + s_lo[2];
            st->sig[5] = none ? -1 : d.k0 + s_hi[2] + 1;
            st->sig_scale = scale;
            return;
        }
        DomainDev nb;
        if (none) {
            nb = bm.init_box;
        } else {
            const int g = cf.guard;
            int ai0 = d.i0 + s_lo[0], ai1 = d.i0 + s_hi[0] + 1;
            int aj0 = d.j0 + s_lo[1], aj1 = d.j0 + s_hi[1] + 1;
            int ak0 = d.k0 + s_lo[2], ak1 = d.k0 + s_hi[2] + 1;
            int bi0 = ai0 - g > 0 ? ai0 - g : 0, bi1 = ai1 + g < cf.nx ? ai1 + g : cf.nx;
            int bj0 = aj0 - g > 0 ? aj0 - g : 0, bj1 = aj1 + g < cf.ny ? aj1 + g : cf.ny;
            int bk0 = ak0 - g > 0 ? ak0 - g : 0, bk1 = ak1 + g < cf.nz ? ak1 + g : cf.nz;
            nb = make_domain(bi0, bj0, bk0, bi1 - bi0, bj1 - bj0, bk1 - bk0, bk0 == 0, cf.tile);
        }
        switch_box(cf, bm, co, st, b, nb, ed);
    }
}

// Copy the overlap of the previous box into the new one (zeros elsewhere,
// moving_active_domain.py:196-232); for the vacuum-aware CFL also the max phi
// of the new box.  With `with_cfl` (no vacuum-aware masks) the CFL bound of
// the new box as cfl_kernel computes it, from the values in registers.
// Four CTAs per SM (64 registers, a few spilled to L1): the kernel waits on
// loads and dependent FP64 arithmetic, and at its natural 89 registers only two
// CTAs fit (25 % of the warp slots).
__global__ void __launch_bounds__(NT, 4) rebox_kernel(const ConfigDev *cfp, const Coeffs *cos, MarchState *sts,
                                                   int with_cfl) {
    const ConfigDev &cf = *cfp;
    const int b = blockIdx.y;
    MarchState *st = sts + b;
    if (st->done || st->error) return;
    const DomainDev d = st->dom;
    const bool moved = st->reboxed != 0;
    if (!moved && !cf.vacuum_aware && !with_cfl) return;
    const DomainDev p = st->prev;
    const double *Up = st->Uprev;
    double *Ua = st->Ua;
    const BeamDev &bm = cf.beams[b];
    const double *S = cos[b].S_cfl;
    const double ed = cos[b].ed_cfl;
    const bool all_axes[3] = {true, true, true};
    const size_t N = (size_t)d.nx * d.ny * d.nz, NP = (size_t)p.nx * p.ny * p.nz;
    double m = 0.0, inv = 0.0;
    for (size_t o = (size_t)blockIdx.x * NT + threadIdx.x; o < N; o += (size_t)gridDim.x * NT) {
        // a box holds fewer than 2^32 cells: 32-bit index arithmetic
        const unsigned uo = (unsigned)o, unz = (unsigned)d.nz, uny = (unsigned)d.ny;
        const unsigned row = uo / unz;
        const int lk = (int)(uo - row * unz), lj = (int)(row % uny), li = (int)(row / uny);
        double u[4];
        if (moved) {
            int pi = d.i0 + li - p.i0, pj = d.j0 + lj - p.j0, pk = d.k0 + lk - p.k0;
            bool in = pi >= 0 && pi < p.nx && pj >= 0 && pj < p.ny && pk >= 0 && pk < p.nz;
            size_t po = in ? ((size_t)pi * p.ny + pj) * p.nz + pk : 0;
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                u[c] = in ? Up[c * NP + po] : 0.0;
                Ua[c * N + o] = u[c];
            }
        } else {
#pragma unroll
            for (int c = 0; c < 4; ++c) u[c] = Ua[c * N + o];
        }
        m = fmax(m, u[0]);
        if (with_cfl) inv = fmax(inv, cell_cfl(cf, bm, d, S, ed, u, li, lj, lk, all_axes));
    }
    if (cf.vacuum_aware) block_max_atomic(m, &st->newmax_bits);
    if (with_cfl) {
        if (cf.cfl_floor && blockIdx.x == 0 && threadIdx.x == 0) inv = fmax(inv, phantom_cfl_floor(cf, S));
        block_max_atomic(inv, &st->inv_bits);
    }
}

// Activity mask of the vacuum-aware CFL: phi above tol * max(phi, phi_in),
// plus the inflow at the entrance layer (numerics/energy.py:496-537).
__global__ void __launch_bounds__(NT) mask_kernel(const ConfigDev *cfp, const Coeffs *cos, const MarchState *sts) {
    const ConfigDev &cf = *cfp;
    const int b = blockIdx.y;
    const Coeffs *co = cos + b;
    const MarchState *st = sts + b;
    const BeamDev &bm = cf.beams[b];
    unsigned char *active = cf.active + (size_t)b * cf.cap;
    if (st->done || st->error) return;
    const DomainDev d = st->dom;
    const double *Ua = st->Ua;
    const double scale = fmax(__longlong_as_double((long long)st->newmax_bits), st->pin_max);
    if (scale == 0.0) return;
    const double thr = cf.tol * scale;
    const double ed = co->ed_cfl;
    const size_t N = (size_t)d.nx * d.ny * d.nz;
    for (size_t o = (size_t)blockIdx.x * NT + threadIdx.x; o < N; o += (size_t)gridDim.x * NT) {
        int lk = (int)(o % d.nz), lj = (int)((o / d.nz) % d.ny), li = (int)(o / ((size_t)d.nz * d.ny));
        bool act = Ua[o] > thr;
        if (lk == 0 && d.inflow)
            act = act || bm.spatial[(size_t)(d.i0 + li) * cf.ny + (d.j0 + lj)] * ed > thr;
        active[o] = act ? 1 : 0;
    }
}

// Scatter the compact state into a full-grid array (zeros elsewhere),
// moving_active_domain.py:235-244.
__global__ void __launch_bounds__(NT) embed_kernel(const ConfigDev *cfp, const MarchState *st, double *Ufull) {
    const ConfigDev &cf = *cfp;
    const DomainDev d = st->dom;
    const double *Ua = st->Ua;
    const size_t N = (size_t)d.nx * d.ny * d.nz, NG = (size_t)cf.nx * cf.ny * cf.nz;
    for (size_t go = (size_t)blockIdx.x * NT + threadIdx.x; go < NG; go += (size_t)gridDim.x * NT) {
        int gk = (int)(go % cf.nz), gj = (int)((go / cf.nz) % cf.ny), gi = (int)(go / ((size_t)cf.nz * cf.ny));
        int li = gi - d.i0, lj = gj - d.j0, lk = gk - d.k0;
        bool in = li >= 0 && li < d.nx && lj >= 0 && lj < d.ny && lk >= 0 && lk < d.nz;
        size_t o = ((size_t)li * d.ny + lj) * d.nz + lk;
#pragma unroll
        for (int c = 0; c < 4; ++c) Ufull[c * NG + go] = in ? Ua[c * N + o] : 0.0;
    }
}

// Scalar batches for unit parity checks
__global__ void weno_batch_kernel(const double *v, double *out, int n) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) out[t] = weno_left(v[5 * t], v[5 * t + 1], v[5 * t + 2], v[5 * t + 3], v[5 * t + 4]);
}
__global__ void project_batch_kernel(double *u, int n) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) project(u[4 * t], u[4 * t + 1], u[4 * t + 2], u[4 * t + 3]);
}
__global__ void eigen_batch_kernel(const double *u, int axis, double *out, int n) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) {
        const double *p = u + 4 * t;
        double jn = sqrt(p[1] * p[1] + p[2] * p[2] + p[3] * p[3]);
        double lo, hi;
        eigen(p[0], p[1], p[2], p[3], jn, axis, lo, hi);
        out[2 * t] = lo;
        out[2 * t + 1] = hi;
    }
}
__global__ void hll_batch_kernel(const double *L, const double *R, int axis, int unit, double *F, int n) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) {
        double l[4], r[4], f[4];
        for (int c = 0; c < 4; ++c) { l[c] = L[4 * t + c]; r[c] = R[4 * t + c]; }
        hll_flux(l, r, axis, unit != 0, f);
        for (int c = 0; c < 4; ++c) F[4 * t + c] = f[c];
    }
}
__global__ void exp_batch_kernel(const double *x, double *y, int n) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) y[t] = dd_exp(x[t]);
}
__global__ void coeff_eval_kernel(const ConfigDev *cfp, const double *E, int n, double *out, int *err) {
    const ConfigDev &cf = *cfp;
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * cf.nm) return;
    int e = t / cf.nm, m = t % cf.nm;
    double s = 0, tr = 0, nu = 0;
    bool ok = stopping_power_dev(cf.mats[m], E[e], s);
    ok &= transport_dev(cf, cf.mats[m], E[e], tr);
    ok &= nuclear_dev(cf, cf.mats[m], E[e], nu);
    if (!ok) atomicOr(err, 1);
    out[3 * t] = s;
    out[3 * t + 1] = tr;
    out[3 * t + 2] = nu;
}

// ---------------------------------------------------------------------------
// Host side: tables, plan
// ---------------------------------------------------------------------------
double sign_of(double x) { return (double)((x > 0.0) - (x < 0.0)); }

double pchip_endpoint(double h0, double h1, double d0, double d1) {
    double slope = ((2.0 * h0 + h1) * d0 - h0 * d1) / (h0 + h1);
    if (sign_of(slope) != sign_of(d0)) return 0.0;
    if (sign_of(d0) != sign_of(d1) && std::fabs(slope) > 3.0 * std::fabs(d0)) return 3.0 * d0;
    return slope;
}

// physics/stopping_power.py:94-138 (coefficient_interpolation.py:19-48)
std::vector<double> pchip_slopes(const double *E, const double *v, int n) {
    std::vector<double> h(n - 1), d(n - 1), s(n, 0.0);
    for (int i = 0; i < n - 1; ++i) {
        h[i] = E[i + 1] - E[i];
        d[i] = (v[i + 1] - v[i]) / h[i];
    }
    if (n == 2) {
        s[0] = s[1] = d[0];
        return s;
    }
    for (int k = 1; k < n - 1; ++k) {
        if (d[k - 1] * d[k] > 0.0) {
            double w1 = 2.0 * h[k] + h[k - 1];
            double w2 = h[k] + 2.0 * h[k - 1];
            s[k] = (w1 + w2) / (w1 / d[k - 1] + w2 / d[k]);
        }
    }
    s[0] = pchip_endpoint(h[0], h[1], d[0], d[1]);
    s[n - 1] = pchip_endpoint(h[n - 2], h[n - 3], d[n - 2], d[n - 3]);
    return s;
}

}  // namespace

namespace pdm1 {
int report_error(int code, const char *msg) { return set_error(code, msg); }
std::vector<double> host_pchip_slopes(const double *E, const double *v, int n) { return pchip_slopes(E, v, n); }
}  // namespace pdm1

struct pdm1_plan {
    pdm1_problem p{};
    ConfigDev cf{};
    int nbeams = 1;
    bool field = false;              // created by pdm1_field_plan_create
    size_t cap = 0;
    ConfigDev *d_cf = nullptr;
    Coeffs *d_co = nullptr;         // nbeams
    MarchState *d_st = nullptr;     // nbeams
    MarchState *h_st = nullptr;     // pinned, nbeams
    MarchSummary *d_sum = nullptr;
    MarchSummary *h_sum = nullptr;  // pinned
    BeamDev *d_beams = nullptr;
    int *d_tile_off = nullptr;
    double *d_tables = nullptr;
    int32_t *d_ids = nullptr;
    double *d_spatial = nullptr;    // nbeams x (nx, ny)
    double *d_targets = nullptr;
    double *d_schedule = nullptr;   // prescribed energies (pdm1_plan_set_schedule)
    double *d_U1 = nullptr, *d_U2 = nullptr, *d_V = nullptr, *d_q = nullptr;
    double *d_bufA = nullptr, *d_bufB = nullptr;   // moving box: compact-state ping-pong
    unsigned long long *d_slab = nullptr;
    unsigned char *d_active = nullptr;
    BoxModelDev *d_model = nullptr;  // learned box
    double *d_acc = nullptr;         // nbeams x kAcc
    double *d_plane = nullptr;       // nbeams x nz
    size_t workspace = 0;
    int sms = 148;                   // SMs of the plan's device (stage grid sizing)
    std::vector<BeamDev> h_beams;   // host copy (device spatial pointers)
    // per material: [lo, hi] of the stopping-power, transport, nuclear tables
    std::vector<double> range[3][2];
    cudaStream_t own_stream = nullptr;
    cudaEvent_t ready = nullptr;
    cudaEvent_t ev[2 * kStepsPerGraph] = {};   // stage-kernel timing, one pair per step of a chunk
};

namespace {

bool table_ok(const pdm1_table &t) {
    if (t.n_nodes < 2 || !t.energy || !t.value) return false;
    for (int i = 0; i + 1 < t.n_nodes; ++i)
        if (!(t.energy[i + 1] > t.energy[i])) return false;
    return true;
}

// Upload one table; return its TableView (device pointers patched later).
TableView add_table(std::vector<double> &blob, std::vector<std::pair<size_t, int>> &fix,
                    const pdm1_table &t) {
    TableView v{};
    v.n = t.n_nodes;
    size_t base = blob.size();
    blob.insert(blob.end(), t.energy, t.energy + t.n_nodes);
    blob.insert(blob.end(), t.value, t.value + t.n_nodes);
    std::vector<double> sl = pchip_slopes(t.energy, t.value, t.n_nodes);
    blob.insert(blob.end(), sl.begin(), sl.end());
    fix.push_back({base, t.n_nodes});
    // log-spaced node guess when the spacing in log E is uniform to 1e-9
    double l0 = std::log(t.energy[0]), l1 = std::log(t.energy[t.n_nodes - 1]);
    double step = (l1 - l0) / (t.n_nodes - 1);
    bool uniform = t.energy[0] > 0.0 && step > 0.0;
    for (int i = 0; uniform && i < t.n_nodes; i += 97)
        if (std::fabs(std::log(t.energy[i]) - (l0 + step * i)) > 1e-6 * step) uniform = false;
    v.log_e0 = l0;
    v.inv_log_step = uniform ? 1.0 / step : 0.0;
    return v;
}

// Ghost width of a reconstruction (reconstruction_methods/*.py GHOST_WIDTH)
// and the z cells its inflow extrapolation needs (boundary.py:214-320).
int ghost_width(int scheme) {
    return scheme == PDM1_SPATIAL_FIRST_ORDER ? 1 : (scheme == PDM1_SPATIAL_WENO_Z ? 3 : 2);
}
int min_z_cells(int scheme) {
    return scheme == PDM1_SPATIAL_WENO_Z ? 4 : (scheme == PDM1_SPATIAL_FIRST_ORDER ? 1 : 2);
}
const char *z_cells_message(int scheme) {
    return scheme == PDM1_SPATIAL_WENO_Z ? "WENO-Z inflow extrapolation requires at least four z cells."
                                         : "WENO3 inflow extrapolation requires at least two z cells.";
}

int validate_problem(const pdm1_problem *p) {
    if (!p) return set_error(PDM1_ERR_ARGUMENT, "problem is NULL");
    if (p->nx <= 0 || p->ny <= 0 || p->nz <= 0) return set_error(PDM1_ERR_ARGUMENT, "grid dimensions must be positive");
    if (p->spatial_scheme < PDM1_SPATIAL_WENO_Z || p->spatial_scheme > PDM1_SPATIAL_WENO3)
        return set_error(PDM1_ERR_UNSUPPORTED, "unknown spatial scheme");
    if (p->nz < min_z_cells(p->spatial_scheme)) return set_error(PDM1_ERR_ARGUMENT, z_cells_message(p->spatial_scheme));
    if (p->n_materials < 1 || p->n_materials > kMaxMat) return set_error(PDM1_ERR_ARGUMENT, "n_materials must be in 1..16");
    if (!p->materials || !p->ids) return set_error(PDM1_ERR_ARGUMENT, "NULL materials/ids");
    if (!(p->dx > 0 && p->dy > 0 && p->dz > 0)) return set_error(PDM1_ERR_ARGUMENT, "spacings must be positive");
    if (!(p->cfl > 0.0 && p->cfl <= 1.0)) return set_error(PDM1_ERR_ARGUMENT, "cfl must lie in (0, 1].");
    if (!(p->max_energy_step > 0.0)) return set_error(PDM1_ERR_ARGUMENT, "max_energy_step must be positive.");
    if (p->energy_scheme < 0 || p->energy_scheme > 2) return set_error(PDM1_ERR_UNSUPPORTED, "unknown energy scheme");
    if (p->precision != PDM1_FP64 && p->precision != PDM1_FP32_FP64) return set_error(PDM1_ERR_ARGUMENT, "unknown precision");
    if (p->moving_active_domain && p->active_guard_cells < 0)
        return set_error(PDM1_ERR_ARGUMENT, "active_guard_cells must be non-negative");
    if (p->moving_active_domain && !(p->active_relative_tolerance >= 0.0))
        return set_error(PDM1_ERR_ARGUMENT, "active_relative_tolerance must be non-negative");
    for (int m = 0; m < p->n_materials; ++m) {
        const pdm1_material &mt = p->materials[m];
        if (!table_ok(mt.stopping_power) || !table_ok(mt.transport) || !table_ok(mt.nuclear))
            return set_error(PDM1_ERR_ARGUMENT, "coefficient tables need >= 2 strictly increasing nodes");
        if (!(mt.density > 0.0)) return set_error(PDM1_ERR_ARGUMENT, "density must be positive");
    }
    size_t n = (size_t)p->nx * p->ny * p->nz;
    for (size_t c = 0; c < n; ++c)
        if (p->ids[c] < 0 || p->ids[c] >= p->n_materials) return set_error(PDM1_ERR_ARGUMENT, "material id out of range");
    return PDM1_OK;
}

int validate_beam(const pdm1_beam &b) {
    if (!b.inflow_spatial) return set_error(PDM1_ERR_ARGUMENT, "beam inflow profile is NULL");
    if (!(b.energy_spread > 0.0))
        return set_error(PDM1_ERR_ARGUMENT, "Zero energy spread is not supported by the Gaussian inflow.");
    if (!(b.energy > 0.0)) return set_error(PDM1_ERR_ARGUMENT, "beam energy must be positive");
    return PDM1_OK;
}

bool is_close(double a, double b) { return std::fabs(a - b) <= 1e-8 + 1e-5 * std::fabs(b); }

// Energy range the march will evaluate tables at: [e_lo, e_hi]
int check_energy_range(const pdm1_plan *pl, double e_hi, double e_lo) {
    const pdm1_problem &p = pl->p;
    const bool used[3] = {true, p.scattering == PDM1_SCATTERING_WENTZEL, p.nuclear != 0};
    for (int m = 0; m < p.n_materials; ++m) {
        for (int q = 0; q < 3; ++q) {
            if (!used[q]) continue;
            double lo = pl->range[q][0][m], hi = pl->range[q][1][m];
            if ((e_hi > hi && !is_close(e_hi, hi)) || (e_lo < lo && !is_close(e_lo, lo))) {
                char buf[256];
                snprintf(buf, sizeof buf, "Energy outside coefficient table range [%g, %g] MeV (march spans [%g, %g] MeV).",
                         lo, hi, e_lo, e_hi);
                return set_error(PDM1_ERR_RANGE, buf);
            }
        }
    }
    return PDM1_OK;
}

double beam_start_energy(const pdm1_plan *pl, int b) {
    return pl->h_beams[b].E_beam + pl->p.energy_window_sigma * pl->h_beams[b].sigma_E;
}

StageArgs make_args(pdm1_plan *pl, double *dose, double *edep, double *snap) {
    StageArgs a{};
    a.cf = pl->d_cf;
    a.co = pl->d_co;
    a.st = pl->d_st;
    a.U1 = pl->d_U1;
    a.U2 = pl->d_U2;
    a.V = pl->d_V;
    a.qpart = pl->d_q;
    a.dose = dose;
    a.edep = edep;
    a.snap = snap;
    return a;
}

// blocks of the per-cell kernels, per beam: enough for the largest domain
int cell_blocks(const pdm1_plan *pl) {
    size_t b = (pl->cap + NT - 1) / NT;
    // about 8 CTAs per SM over all beams (at least 64 per beam): these kernels are
    // latency-bound on loads and dependent FP64 arithmetic and want every warp
    const size_t per = pl->nbeams > 1 ? std::max<size_t>(64, (size_t)148 * 8 / pl->nbeams) : (size_t)148 * 8;
    return (int)std::max<size_t>(1, std::min<size_t>(b, per));
}

template <class Tl>
void launch_stage64(int mode, int grid, const StageArgs &a, cudaStream_t stream) {
    const size_t bytes = Tl::template smem_bytes<double>();
    constexpr int nt = Tl::NT;
    switch (mode) {
    case MODE_A: stage_kernel<double, MODE_A, Tl><<<grid, nt, bytes, stream>>>(a); break;
    case MODE_B: stage_kernel<double, MODE_B, Tl><<<grid, nt, bytes, stream>>>(a); break;
    case MODE_C: stage_kernel<double, MODE_C, Tl><<<grid, nt, bytes, stream>>>(a); break;
    case MODE_C_LEARN: stage_kernel<double, MODE_C, Tl, true><<<grid, nt, bytes, stream>>>(a); break;
    case MODE_EULER: stage_kernel<double, MODE_EULER, Tl><<<grid, nt, bytes, stream>>>(a); break;
    default: stage_kernel<double, MODE_RHS, Tl><<<grid, nt, bytes, stream>>>(a); break;
    }
}

// One stage launch in the plan's precision and tile shape.
void launch_stage(const pdm1_plan *pl, int mode, int grid, const StageArgs &a, cudaStream_t stream) {
    if (mode == MODE_C && pl->cf.learned) mode = MODE_C_LEARN;
    if (pl->p.precision == PDM1_FP32_FP64) {
        launch_stage_fp32(mode, pl->cf.tile_id, grid, a, stream);
        return;
    }
    switch (pl->cf.tile_id) {
    case 1: launch_stage64<Tile1>(mode, grid, a, stream); break;
    case 2: launch_stage64<Tile2>(mode, grid, a, stream); break;
    default: launch_stage64<Tile0>(mode, grid, a, stream); break;
    }
}

// The moving box's per-step work ahead of the prologue: desired box, rebox,
// activity mask, CFL bound over the new box -- for every beam at once.
int launch_box_step(pdm1_plan *pl, cudaStream_t stream) {
    const pdm1_problem &p = pl->p;
    const dim3 cells(cell_blocks(pl), pl->nbeams);
    box_kernel<<<pl->nbeams, 256, 0, stream>>>(pl->d_cf, pl->d_co, pl->d_st);
    int n = 3;
    if (pl->cf.learned) {
        // the moments of the state come from the last stage C (tile_moments_cta);
        // before the first step the accumulators hold zeros (no stage C yet)
        launch_box_learn(pl->d_cf, pl->d_co, pl->d_st, pl->nbeams, stream);
        n += 1;
    }
    if (p.vacuum_aware_cfl) {
        rebox_kernel<<<cells, NT, 0, stream>>>(pl->d_cf, pl->d_co, pl->d_st, 0);
        mask_kernel<<<cells, NT, 0, stream>>>(pl->d_cf, pl->d_co, pl->d_st);
        cfl_kernel<<<cells, NT, 0, stream>>>(pl->d_cf, pl->d_co, pl->d_st, 1);
        ++n;
    } else {   // the CFL bound of the new box within the box move
        rebox_kernel<<<cells, NT, 0, stream>>>(pl->d_cf, pl->d_co, pl->d_st, 1);
        --n;
    }
    return n;
}

// One energy step of every beam on `stream`; `slot` >= 0 brackets the stage
// kernels with timing events.  Returns the kernels launched.
int launch_step(pdm1_plan *pl, const StageArgs &a, double *energies, cudaStream_t stream, int slot,
                bool box_step = true) {
    const pdm1_problem &p = pl->p;
    const int grid = pl->cf.grid_ctas;
    int launched = 0;
    if (p.moving_active_domain && box_step) launched += launch_box_step(pl, stream);
    prologue_kernel<<<pl->nbeams, 256, 0, stream>>>(pl->d_cf, pl->d_co, pl->d_st, energies);
    ++launched;
    if (pl->nbeams > 1) {
        tiles_kernel<<<1, 1024, 0, stream>>>(pl->d_cf, pl->d_co, pl->d_st);
        ++launched;
    }
    // external event nodes: real timestamps when the step is replayed from a graph
    if (slot >= 0) cudaEventRecordWithFlags(pl->ev[2 * slot], stream, cudaEventRecordExternal);
    if (p.energy_scheme == PDM1_SCHEME_FORWARD_EULER) {
        launch_stage(pl, MODE_EULER, grid, a, stream);
        ++launched;
    } else {
        launch_stage(pl, MODE_A, grid, a, stream);
        launch_stage(pl, MODE_B, grid, a, stream);
        launch_stage(pl, MODE_C, grid, a, stream);
        launched += 3;
    }
    if (slot >= 0) cudaEventRecordWithFlags(pl->ev[2 * slot + 1], stream, cudaEventRecordExternal);
    if (p.energy_scheme == PDM1_SCHEME_FORWARD_EULER) {
        euler_finish_kernel<<<cell_blocks(pl), NT, 0, stream>>>(a);
        ++launched;
    }
    if (pl->cf.rec) {
        launch_box_moments(pl->d_cf, pl->d_st, grid, 1, stream);
        launch_record(pl->d_cf, pl->d_co, pl->d_st, stream);
        launched += 2;
    }
    return launched;
}

template <class Tl>
cudaError_t set_attributes64() {
    const int bytes = (int)Tl::template smem_bytes<double>();
    const auto attr = cudaFuncAttributeMaxDynamicSharedMemorySize;
    cudaError_t e = cudaFuncSetAttribute(stage_kernel<double, MODE_A, Tl>, attr, bytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(stage_kernel<double, MODE_B, Tl>, attr, bytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(stage_kernel<double, MODE_C, Tl>, attr, bytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(stage_kernel<double, MODE_C, Tl, true>, attr, bytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(stage_kernel<double, MODE_EULER, Tl>, attr, bytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(stage_kernel<double, MODE_RHS, Tl>, attr, bytes);
    return e;
}

int set_smem_attributes() {
    static bool done = false;
    if (done) return PDM1_OK;
    CUDA_TRY(set_attributes64<Tile0>());
    CUDA_TRY(set_attributes64<Tile1>());
    CUDA_TRY(set_attributes64<Tile2>());
    CUDA_TRY((cudaError_t)stage_fp32_set_attributes());
    done = true;
    return PDM1_OK;
}

int device_error_status(int error) {
    if (error & ERR_DEV_RANGE) return set_error(PDM1_ERR_RANGE, "energy outside a coefficient table during the march");
    if (error & ERR_DEV_MAXSTEPS) return set_error(PDM1_ERR_MAX_STEPS, "energies buffer shorter than the march");
    if (error & ERR_DEV_NONFINITE) return set_error(PDM1_ERR_NONFINITE, "non-finite state or non-positive energy step during the march");
    if (error & ERR_DEV_CAPACITY) return set_error(PDM1_ERR_ARGUMENT, "a beam's moving box outgrew the plan's box capacity");
    if (error & ERR_DEV_TIMEOUT) return set_error(PDM1_ERR_TIMEOUT, "a bounded device wait (bulk tile copy) timed out");
    return PDM1_OK;
}

int device_error_status(const MarchState &st) { return device_error_status(st.error); }

// Initial box of a beam from its inflow support (moving_active_domain.py:35-60).
int initial_box(const pdm1_problem &p, const double *spatial, TileDims tile, DomainDev &box) {
    int ilo = -1, ihi = -1, jlo = -1, jhi = -1;
    for (int i = 0; i < p.nx; ++i)
        for (int j = 0; j < p.ny; ++j)
            if (spatial[(size_t)i * p.ny + j] > 0.0) {
                if (ilo < 0 || i < ilo) ilo = i;
                if (i > ihi) ihi = i;
                if (jlo < 0 || j < jlo) jlo = j;
                if (j > jhi) jhi = j;
            }
    if (ilo < 0) return set_error(PDM1_ERR_NO_BEAM, "Beam inflow has empty transverse support.");
    const int g = p.active_guard_cells;
    int i0 = std::max(0, ilo - g), i1 = std::min(p.nx, ihi + 1 + g);
    int j0 = std::max(0, jlo - g), j1 = std::min(p.ny, jhi + 1 + g);
    int k1 = std::min(p.nz, 1 + g);
    box = make_domain(i0, j0, 0, i1 - i0, j1 - j0, k1, 1, tile);
    if (k1 < min_z_cells(p.spatial_scheme)) return set_error(PDM1_ERR_ARGUMENT, z_cells_message(p.spatial_scheme));
    return PDM1_OK;
}

void destroy_plan(pdm1_plan *pl) {
    if (!pl) return;
    // the buffers go back to the pool; wait for the device as cudaFree would
    cudaDeviceSynchronize();
    pool_free(pl->d_cf);
    pool_free(pl->d_co);
    pool_free(pl->d_st);
    pool_free(pl->h_st);
    pool_free(pl->d_sum);
    pool_free(pl->h_sum);
    pool_free(pl->d_beams);
    pool_free(pl->d_tile_off);
    pool_free(pl->d_tables);
    pool_free(pl->d_ids);
    pool_free(pl->d_spatial);
    pool_free(pl->d_targets);
    pool_free(pl->d_schedule);
    pool_free(pl->d_U1);
    pool_free(pl->d_U2);
    pool_free(pl->d_V);
    pool_free(pl->d_q);
    pool_free(pl->d_bufA);
    pool_free(pl->d_bufB);
    pool_free(pl->d_slab);
    pool_free(pl->d_active);
    pool_free(pl->d_model);
    pool_free(pl->d_acc);
    pool_free(pl->d_plane);
    if (pl->ready) cudaEventDestroy(pl->ready);
    for (cudaEvent_t e : pl->ev)
        if (e) cudaEventDestroy(e);
    if (pl->own_stream) cudaStreamDestroy(pl->own_stream);
    delete pl;
}

// Persistent grid of the stage kernels: resident CTAs per SM x SMs, capped by
// the tiles of the full grid.  256-cell tiles: 2 CTAs per SM in double, 4 in
// float (64 registers; 4 x 256 threads hide more of the MUFU and shared-memory
// latency than 3 x 256 at 80 registers: -4 % stage time on field256); a
// 512-cell tile holds half as many CTAs.
int stage_grid(const pdm1_problem &p, TileDims t, int nbeams, int sms) {
    const int per_sm = (p.precision == PDM1_FP32_FP64 ? 4 : 2) * 256 / (t.x * t.y * t.z);
    size_t tiles = (size_t)make_domain(0, 0, 0, p.nx, p.ny, p.nz, 1, t).ntiles * nbeams;
    return (int)std::max<size_t>(1, std::min<size_t>(tiles, (size_t)std::max(1, per_sm) * sms));
}

// A plan for `nbeams` beams on one phantom; every beam's buffers hold `cap` cells.
int create_plan(const pdm1_problem *problem, const pdm1_beam *beams, int nbeams, size_t cap, pdm1_plan **out) {
    int rc = set_smem_attributes();
    if (rc) return rc;
    pdm1_plan *pl = new pdm1_plan();
    pl->p = *problem;
    pl->p.materials = nullptr;   // tables are copied below; host pointers are not kept
    pl->p.ids = nullptr;
    pl->p.inflow_spatial = nullptr;
    pl->nbeams = nbeams;
    pl->cap = cap;
    const pdm1_problem &p = pl->p;
    const size_t N = (size_t)p.nx * p.ny * p.nz, NXY = (size_t)p.nx * p.ny;
    const size_t B = (size_t)nbeams;

    std::vector<double> blob;
    std::vector<std::pair<size_t, int>> fix;
    ConfigDev &cf = pl->cf;
    cf.nx = p.nx; cf.ny = p.ny; cf.nz = p.nz;
    cf.tile = kTiles[0];
    cf.tile_id = 0;
    cf.dx = p.dx; cf.dy = p.dy; cf.dz = p.dz;
    cf.nm = p.n_materials;
    cf.spatial = p.spatial_scheme;
    cf.stencil_radius = ghost_width(p.spatial_scheme);
    cf.cfl_floor = p.moving_active_domain && p.phantom_cfl_floor ? 1 : 0;
    cf.present = 0u;
    cf.scattering = p.scattering;
    cf.nuclear = p.nuclear ? 1 : 0;
    cf.interp = p.interpolation;
    cf.scheme = p.energy_scheme;
    cf.unit_speeds = p.wave_speeds == PDM1_SPEEDS_UNIT;
    bool sources = p.scattering != PDM1_SCATTERING_OFF || p.nuclear;
    cf.use_if = (p.energy_scheme == PDM1_SCHEME_IF_SSPRK3 && sources) ? 1 : 0;
    cf.strang = (p.energy_scheme != PDM1_SCHEME_IF_SSPRK3 && sources) ? 1 : 0;
    cf.cfl = p.cfl;
    cf.max_dE = p.max_energy_step;
    cf.Emin = p.energy_min;
    for (int m = 0; m < p.n_materials; ++m) {
        const pdm1_material &mt = problem->materials[m];
        cf.mats[m].sp = add_table(blob, fix, mt.stopping_power);
        cf.mats[m].tr = add_table(blob, fix, mt.transport);
        cf.mats[m].nuc = add_table(blob, fix, mt.nuclear);
        cf.mats[m].density = mt.density;
        cf.mats[m].X0 = mt.radiation_length;
        const pdm1_table *tabs[3] = {&mt.stopping_power, &mt.transport, &mt.nuclear};
        for (int q = 0; q < 3; ++q) {
            pl->range[q][0].push_back(tabs[q]->energy[0]);
            pl->range[q][1].push_back(tabs[q]->energy[tabs[q]->n_nodes - 1]);
        }
    }
    auto fail = [&](int code) { destroy_plan(pl); return code; };
    // beams: spectrum, angular factor, initial boxes
    pl->h_beams.resize(B);
    for (int b = 0; b < nbeams; ++b) {
        BeamDev &bd = pl->h_beams[b];
        bd.E_beam = beams[b].energy;
        bd.sigma_E = beams[b].energy_spread;
        bd.rf = dd_exp(-(beams[b].angular_spread * beams[b].angular_spread));
        bd.init_box = make_domain(0, 0, 0, p.nx, p.ny, p.nz, 1, cf.tile);
        if (p.moving_active_domain) {
            rc = initial_box(p, beams[b].inflow_spatial, cf.tile, bd.init_box);
            if (rc) return fail(rc);
            if ((size_t)bd.init_box.nx * bd.init_box.ny * bd.init_box.nz > cap)
                return fail(set_error(PDM1_ERR_ARGUMENT, "box capacity smaller than a beam's initial box"));
        }
    }
    for (size_t c = 0; c < N; ++c) cf.present |= 1u << problem->ids[c];
    cudaError_t e;
#define ALLOC(ptr, bytes)                                                      \
    e = pool_malloc((void **)&(ptr), (bytes));                                 \
    if (e != cudaSuccess) {                                                    \
        set_error(PDM1_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e)); \
        return fail(PDM1_ERR_CUDA);                                            \
    }
    ALLOC(pl->d_tables, blob.size() * sizeof(double));
    ALLOC(pl->d_cf, sizeof(ConfigDev));
    ALLOC(pl->d_co, B * sizeof(Coeffs));
    ALLOC(pl->d_st, B * sizeof(MarchState));
    ALLOC(pl->d_sum, sizeof(MarchSummary));
    ALLOC(pl->d_beams, B * sizeof(BeamDev));
    ALLOC(pl->d_tile_off, (B + 1) * sizeof(int));
    ALLOC(pl->d_ids, N * sizeof(int32_t));
    ALLOC(pl->d_spatial, B * NXY * sizeof(double));
    ALLOC(pl->d_targets, 64 * sizeof(double));
    ALLOC(pl->d_U1, B * 4 * cap * sizeof(double));
    ALLOC(pl->d_U2, B * 4 * cap * sizeof(double));
    ALLOC(pl->d_V, B * 4 * cap * sizeof(double));
    ALLOC(pl->d_q, B * cap * sizeof(double));
    ALLOC(pl->d_slab, B * (size_t)(p.nx + p.ny + p.nz) * sizeof(unsigned long long));
    ALLOC(pl->d_acc, B * kAcc * sizeof(double));
    ALLOC(pl->d_plane, B * (size_t)p.nz * sizeof(double));
    if (p.moving_active_domain) {
        ALLOC(pl->d_bufA, B * 4 * cap * sizeof(double));
        ALLOC(pl->d_bufB, B * 4 * cap * sizeof(double));
        ALLOC(pl->d_active, B * cap);
    }
#undef ALLOC
    pl->workspace = B * cap * ((p.moving_active_domain ? 21 : 13) * sizeof(double) + (p.moving_active_domain ? 1 : 0));
    if (pool_malloc_host((void **)&pl->h_st, B * sizeof(MarchState)) != cudaSuccess ||
        pool_malloc_host((void **)&pl->h_sum, sizeof(MarchSummary)) != cudaSuccess ||
        cudaStreamCreateWithFlags(&pl->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&pl->ready, cudaEventDisableTiming) != cudaSuccess)
        return fail(set_error(PDM1_ERR_CUDA, "cudaMallocHost/stream/event creation failed"));
    for (cudaEvent_t &ev : pl->ev)
        if (cudaEventCreate(&ev) != cudaSuccess) return fail(set_error(PDM1_ERR_CUDA, "cudaEventCreate failed"));
    // patch table pointers to device addresses
    int ti = 0;
    for (int m = 0; m < p.n_materials; ++m) {
        TableView *views[3] = {&cf.mats[m].sp, &cf.mats[m].tr, &cf.mats[m].nuc};
        for (TableView *v : views) {
            size_t base = fix[ti++].first;
            v->E = pl->d_tables + base;
            v->v = pl->d_tables + base + v->n;
            v->slope = pl->d_tables + base + 2 * v->n;
        }
    }
    for (int b = 0; b < nbeams; ++b) pl->h_beams[b].spatial = pl->d_spatial + (size_t)b * NXY;
    cf.ids = pl->d_ids;
    cf.targets = pl->d_targets;
    cf.nbeams = nbeams;
    cf.cap = cap;
    cf.beams = pl->d_beams;
    cf.tile_off = pl->d_tile_off;
    cf.summary = pl->d_sum;
    cf.moving = p.moving_active_domain ? 1 : 0;
    cf.fp32 = p.precision == PDM1_FP32_FP64 ? 1 : 0;
    cf.bulk_stage = cf.fp32;
    cf.vacuum_aware = (p.moving_active_domain && p.vacuum_aware_cfl) ? 1 : 0;
    cf.guard = p.active_guard_cells;
    cf.tol = p.active_relative_tolerance;
    cf.bufA = pl->d_bufA;
    cf.bufB = pl->d_bufB;
    cf.slab = pl->d_slab;
    cf.active = pl->d_active;
    cf.learned = 0;
    cf.model = nullptr;
    cf.acc = pl->d_acc;
    cf.plane = pl->d_plane;
    cf.rec = nullptr;
    cf.rec_max = 0;
    {
        int dev = 0, sms = 148;
        if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        // resident CTAs per SM of the stage kernel: 2 in double, 4 in float
        // (64 registers; 4 x 256 threads hide more of the MUFU and shared-memory
        // latency than 3 x 256 at 80 registers: -4 % stage time on field256)
        pl->sms = sms;
        cf.grid_ctas = stage_grid(p, cf.tile, B, sms);
    }
    bool ok = cudaMemcpy(pl->d_tables, blob.data(), blob.size() * sizeof(double), cudaMemcpyHostToDevice) == cudaSuccess &&
              cudaMemcpy(pl->d_ids, problem->ids, N * sizeof(int32_t), cudaMemcpyHostToDevice) == cudaSuccess &&
              cudaMemcpy(pl->d_beams, pl->h_beams.data(), B * sizeof(BeamDev), cudaMemcpyHostToDevice) == cudaSuccess &&
              cudaMemcpy(pl->d_cf, &cf, sizeof(ConfigDev), cudaMemcpyHostToDevice) == cudaSuccess &&
              cudaMemset(pl->d_co, 0, B * sizeof(Coeffs)) == cudaSuccess &&
              cudaMemset(pl->d_st, 0, B * sizeof(MarchState)) == cudaSuccess;
    for (int b = 0; ok && b < nbeams; ++b)
        ok = cudaMemcpy(pl->d_spatial + (size_t)b * NXY, beams[b].inflow_spatial, NXY * sizeof(double),
                        cudaMemcpyHostToDevice) == cudaSuccess;
    if (!ok) return fail(set_error(PDM1_ERR_CUDA, "plan upload failed"));
    *out = pl;
    return PDM1_OK;
}

// The march of every beam of a plan.  One beam: U (full grid, in/out), energies
// and snapshots as numerics/energy.py:energy_march.  Several beams (a field):
// U, energies and snapshots are not used, every beam starts from zero and the
// dose is their sum.
int march_impl(pdm1_plan *pl, double *U, double *dose, double *energies, int max_steps,
               const double *snap_targets, int n_snap, double *snap_out, double *snap_E_out,
               pdm1_march_info *info, pdm1_stream_t stream_, int step_limit, int *steps_per_beam) {
    const bool field = pl->field;
    if (!dose || max_steps < 1 || (!field && (!U || !energies)))
        return set_error(PDM1_ERR_ARGUMENT, "pdm1_march: NULL buffer or max_steps < 1");
    cudaStream_t stream = (cudaStream_t)stream_;
    if (stream == nullptr) {
        // the legacy default stream cannot be captured into a graph: order the
        // plan's own stream after it and march there
        CUDA_TRY(cudaEventRecord(pl->ready, nullptr));
        CUDA_TRY(cudaStreamWaitEvent(pl->own_stream, pl->ready, 0));
        stream = pl->own_stream;
    }
    const pdm1_problem &p = pl->p;
    const int B = pl->nbeams;
    int rc;
    double E0max = 0.0;
    for (int b = 0; b < B; ++b) E0max = std::max(E0max, beam_start_energy(pl, b));
    rc = check_energy_range(pl, E0max, p.energy_min);
    if (rc) return rc;
    // sorted unique targets in [energy_min, E0], descending (energy.py:1531-1538)
    std::vector<double> tg;
    if (!field)
        for (int i = 0; i < n_snap; ++i) {
            double t = snap_targets[i];
            if (p.energy_min <= t && t <= E0max && std::find(tg.begin(), tg.end(), t) == tg.end()) tg.push_back(t);
        }
    std::sort(tg.begin(), tg.end(), [](double a, double b) { return a > b; });
    if (tg.size() > 64) return set_error(PDM1_ERR_ARGUMENT, "at most 64 snapshot energies");
    if (!tg.empty() && !snap_out) return set_error(PDM1_ERR_ARGUMENT, "snap_out is NULL");
    pl->cf.n_targets = (int)tg.size();
    pl->cf.max_steps = max_steps;
    pl->cf.step_limit = step_limit;
    CUDA_TRY(cudaMemcpyAsync(pl->d_cf, &pl->cf, sizeof(ConfigDev), cudaMemcpyHostToDevice, stream));
    if (!tg.empty())
        CUDA_TRY(cudaMemcpyAsync(pl->d_targets, tg.data(), tg.size() * sizeof(double), cudaMemcpyHostToDevice, stream));
    const size_t N = (size_t)p.nx * p.ny * p.nz;
    CUDA_TRY(cudaMemsetAsync(dose, 0, N * sizeof(double), stream));
    if (p.moving_active_domain && !tg.empty())
        CUDA_TRY(cudaMemsetAsync(snap_out, 0, tg.size() * 4 * N * sizeof(double), stream));
    CUDA_TRY(cudaMemsetAsync(pl->d_acc, 0, (size_t)B * kAcc * sizeof(double), stream));
    CUDA_TRY(cudaMemsetAsync(pl->d_plane, 0, (size_t)B * p.nz * sizeof(double), stream));
    CUDA_TRY(cudaMemsetAsync(pl->d_tile_off, 0, (size_t)(B + 1) * sizeof(int), stream));
    if (!p.moving_active_domain)
        CUDA_TRY(cudaMemsetAsync(pl->d_slab, 0, (size_t)B * (p.nx + p.ny + p.nz) * sizeof(unsigned long long), stream));
    (void)cudaGetLastError();   // start from a clean launch-error state
    init_kernel<<<B, 32, 0, stream>>>(pl->d_cf, pl->d_co, pl->d_st, field ? nullptr : energies, -1.0,
                                      p.energy_window_sigma, U, 0);
    if (p.moving_active_domain) {
        CUDA_TRY(cudaMemsetAsync(pl->d_slab, 0, (size_t)B * (p.nx + p.ny + p.nz) * sizeof(unsigned long long), stream));
        box_init_kernel<<<dim3(cell_blocks(pl), B), NT, 0, stream>>>(pl->d_cf, pl->d_st, field ? nullptr : U);
    } else {
        cfl_kernel<<<dim3(cell_blocks(pl), B), NT, 0, stream>>>(pl->d_cf, pl->d_co, pl->d_st, 0);
    }
    CUDA_TRY(cudaGetLastError());
    int launches = 2;
    StageArgs a = make_args(pl, dose, nullptr, snap_out);
    double *step_energies = field ? nullptr : energies;
    // capture a chunk of steps into a graph; replay until no beam marches
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int per_step = 0;
    bool use_graph = true;
    if (cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
        for (int s = 0; s < kStepsPerGraph; ++s) per_step = launch_step(pl, a, step_energies, stream, s);
        if (cudaStreamEndCapture(stream, &graph) != cudaSuccess ||
            cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) {
            use_graph = false;
        }
    } else {
        use_graph = false;
    }
    (void)cudaGetLastError();   // a refused capture falls back to direct launches
    int replays = 0, chunk_steps = 0, stage_launches = 0;
    double stage_ms = 0.0;
    const int stages_per_step = p.energy_scheme == PDM1_SCHEME_FORWARD_EULER ? 1 : 3;
    for (;;) {
        if (use_graph) {
            CUDA_TRY(cudaGraphLaunch(exec, stream));
            replays++;
        } else {
            for (int s = 0; s < kStepsPerGraph; ++s) per_step = launch_step(pl, a, step_energies, stream, s);
            CUDA_TRY(cudaGetLastError());
        }
        launches += kStepsPerGraph * per_step;
        CUDA_TRY(cudaMemcpyAsync(pl->h_sum, pl->d_sum, sizeof(MarchSummary), cudaMemcpyDeviceToHost, stream));
        CUDA_TRY(cudaStreamSynchronize(stream));
        ++chunk_steps;
        for (int s = 0; s < kStepsPerGraph; ++s) {
            float ms = 0.f;
            CUDA_TRY(cudaEventElapsedTime(&ms, pl->ev[2 * s], pl->ev[2 * s + 1]));
            stage_ms += ms;
        }
        stage_launches += kStepsPerGraph * stages_per_step;
        if (pl->h_sum->active == 0 || pl->h_sum->error) break;
    }
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (p.moving_active_domain && !field) {
        embed_kernel<<<cell_blocks(pl), NT, 0, stream>>>(pl->d_cf, pl->d_st, U);
        CUDA_TRY(cudaGetLastError());
        ++launches;
    }
    CUDA_TRY(cudaMemcpyAsync(pl->h_st, pl->d_st, (size_t)B * sizeof(MarchState), cudaMemcpyDeviceToHost, stream));
    CUDA_TRY(cudaStreamSynchronize(stream));
    int err = 0, max_step = 0;
    double cells = 0.0, max_cells = 0.0;
    int grows = 0, fallbacks = 0;
    for (int b = 0; b < B; ++b) {
        grows += pl->h_st[b].grows;
        fallbacks += pl->h_st[b].fallback != 0;
        err |= pl->h_st[b].error;
        max_step = std::max(max_step, pl->h_st[b].step);
        cells += pl->h_st[b].cell_steps;
        max_cells = std::max(max_cells, pl->h_st[b].max_cells);
        if (steps_per_beam) steps_per_beam[b] = pl->h_st[b].step;
    }
    rc = device_error_status(err);
    if (info) {
        info->n_steps = field ? max_step : pl->h_st[0].step;
        info->n_snapshots = field ? 0 : pl->h_st[0].taken;
        info->final_state_valid = field ? 0 : 1;
        info->graph_replays = replays;
        info->kernel_launches = launches;
        // the stage events bracket every step slot of every chunk, including
        // slots after the last beam finished (those kernels return at once)
        info->stage_launches = stage_launches;
        info->stage_ms = stage_ms;
        info->cell_steps = cells;
        info->max_box_cells = max_cells;
        info->box_grow_events = grows;
        info->box_fallbacks = fallbacks;
    }
    if (snap_E_out && !field)
        for (int i = 0; i < pl->h_st[0].taken; ++i) snap_E_out[i] = tg[i];
    (void)chunk_steps;
    return rc;
}

}  // namespace

extern "C" {

const char *pdm1_last_error(void) { return g_error; }
const char *pdm1_version(void) { return "pdm1 0.2 sm_100a"; }

void pdm1_plan_destroy(pdm1_plan *pl) { destroy_plan(pl); }

int pdm1_plan_create(const pdm1_problem *problem, pdm1_plan **out) {
    if (!out) return set_error(PDM1_ERR_ARGUMENT, "out is NULL");
    *out = nullptr;
    int rc = validate_problem(problem);
    if (rc) return rc;
    pdm1_beam beam{problem->beam_energy, problem->energy_spread, problem->angular_spread, problem->inflow_spatial};
    rc = validate_beam(beam);
    if (rc) return rc;
    return create_plan(problem, &beam, 1, (size_t)problem->nx * problem->ny * problem->nz, out);
}

int pdm1_field_plan_create(const pdm1_problem *phantom, const pdm1_beam *beams, int n_beams,
                           size_t box_capacity_cells, pdm1_plan **out) {
    if (!out) return set_error(PDM1_ERR_ARGUMENT, "out is NULL");
    *out = nullptr;
    int rc = validate_problem(phantom);
    if (rc) return rc;
    if (!beams || n_beams < 1) return set_error(PDM1_ERR_ARGUMENT, "a field needs at least one beam");
    if (!phantom->moving_active_domain)
        return set_error(PDM1_ERR_UNSUPPORTED, "a batched field marches every beam on its moving active box");
    if (phantom->energy_scheme == PDM1_SCHEME_FORWARD_EULER)
        return set_error(PDM1_ERR_UNSUPPORTED, "a batched field needs an SSPRK3 integrator");
    for (int b = 0; b < n_beams; ++b) {
        rc = validate_beam(beams[b]);
        if (rc) return rc;
    }
    size_t N = (size_t)phantom->nx * phantom->ny * phantom->nz;
    size_t cap = box_capacity_cells ? std::min(box_capacity_cells, N) : N;
    rc = create_plan(phantom, beams, n_beams, cap, out);
    if (rc == PDM1_OK) (*out)->field = true;
    return rc;
}

int pdm1_field_march(pdm1_plan *pl, double *field_dose, int max_steps, int *steps_per_beam,
                     pdm1_march_info *info, pdm1_stream_t stream) {
    if (!pl) return set_error(PDM1_ERR_ARGUMENT, "plan is NULL");
    if (!pl->field) return set_error(PDM1_ERR_ARGUMENT, "pdm1_field_march takes a field plan");
    return march_impl(pl, nullptr, field_dose, nullptr, max_steps, nullptr, 0, nullptr, nullptr, info, stream,
                      -1, steps_per_beam);
}

size_t pdm1_plan_workspace_bytes(const pdm1_plan *pl) { return pl ? pl->workspace : 0; }

int pdm1_tile_shape(int tile_id, int *tx, int *ty, int *tz) {
    if (tile_id < 0 || tile_id >= kNumTiles) return set_error(PDM1_ERR_ARGUMENT, "unknown tile shape");
    if (tx) *tx = kTiles[tile_id].x;
    if (ty) *ty = kTiles[tile_id].y;
    if (tz) *tz = kTiles[tile_id].z;
    return PDM1_OK;
}

int pdm1_plan_set_tile(pdm1_plan *pl, int tile_id) {
    if (!pl) return set_error(PDM1_ERR_ARGUMENT, "plan is NULL");
    if (tile_id < 0 || tile_id >= kNumTiles) return set_error(PDM1_ERR_ARGUMENT, "unknown tile shape");
    const TileDims t = kTiles[tile_id];
    pl->cf.tile = t;
    pl->cf.tile_id = tile_id;
    pl->cf.grid_ctas = stage_grid(pl->p, t, pl->nbeams, pl->sms);
    for (BeamDev &bd : pl->h_beams) {
        const DomainDev &o = bd.init_box;
        bd.init_box = make_domain(o.i0, o.j0, o.k0, o.nx, o.ny, o.nz, o.inflow, t);
    }
    CUDA_TRY(cudaMemcpy(pl->d_beams, pl->h_beams.data(), pl->h_beams.size() * sizeof(BeamDev), cudaMemcpyHostToDevice));
    return PDM1_OK;
}

int pdm1_plan_set_schedule(pdm1_plan *pl, const double *energies, int n) {
    if (!pl) return set_error(PDM1_ERR_ARGUMENT, "plan is NULL");
    if (n < 0 || (n > 0 && !energies)) return set_error(PDM1_ERR_ARGUMENT, "schedule: NULL energies or n < 0");
    if (pl->nbeams != 1) return set_error(PDM1_ERR_UNSUPPORTED, "a prescribed schedule is for one-beam plans");
    for (int k = 1; k < n; ++k)
        if (!(energies[k] < energies[k - 1]))
            return set_error(PDM1_ERR_ARGUMENT, "schedule: energies must decrease strictly");
    pool_free(pl->d_schedule);
    pl->d_schedule = nullptr;
    pl->cf.schedule = nullptr;
    pl->cf.n_schedule = 0;
    if (n == 0) return PDM1_OK;
    CUDA_TRY(pool_malloc((void **)&pl->d_schedule, (size_t)n * sizeof(double)));
    CUDA_TRY(cudaMemcpy(pl->d_schedule, energies, (size_t)n * sizeof(double), cudaMemcpyHostToDevice));
    pl->cf.schedule = pl->d_schedule;
    pl->cf.n_schedule = n;
    return PDM1_OK;
}

int pdm1_plan_set_staging(pdm1_plan *pl, int bulk) {
    if (!pl) return set_error(PDM1_ERR_ARGUMENT, "plan is NULL");
    pl->cf.bulk_stage = (bulk && pl->cf.fp32) ? 1 : 0;
    return PDM1_OK;
}

int pdm1_plan_autotune(pdm1_plan *pl, int steps, int *best_tile, double *ns_per_cell_step, pdm1_stream_t stream) {
    if (!pl) return set_error(PDM1_ERR_ARGUMENT, "plan is NULL");
    if (steps < 1) return set_error(PDM1_ERR_ARGUMENT, "steps must be >= 1");
    const size_t N = (size_t)pl->p.nx * pl->p.ny * pl->p.nz;
    double *U = nullptr, *dose = nullptr, *energies = nullptr;
    auto release = [&]() { cudaFree(U); cudaFree(dose); cudaFree(energies); };
    if (cudaMalloc(&dose, N * sizeof(double)) != cudaSuccess ||
        (!pl->field && (cudaMalloc(&U, 4 * N * sizeof(double)) != cudaSuccess ||
                        cudaMalloc(&energies, (size_t)(steps + 2) * sizeof(double)) != cudaSuccess))) {
        release();
        return set_error(PDM1_ERR_CUDA, "pdm1_plan_autotune: cudaMalloc failed");
    }
    std::vector<int> per_beam(pl->nbeams);
    double best = 0.0;
    int best_id = 0, rc = PDM1_OK;
    // one untimed pass first (clocks, caches), then every candidate
    for (int pass = -1; pass < kNumTiles && rc == PDM1_OK; ++pass) {
        const int id = pass < 0 ? 0 : pass;
        rc = pdm1_plan_set_tile(pl, id);
        if (rc) break;
        if (U) {
            cudaError_t e = cudaMemsetAsync(U, 0, 4 * N * sizeof(double), (cudaStream_t)stream);
            if (e != cudaSuccess) { rc = set_error(PDM1_ERR_CUDA, cudaGetErrorString(e)); break; }
        }
        pdm1_march_info info{};
        rc = march_impl(pl, U, dose, energies, steps + 1, nullptr, 0, nullptr, nullptr, &info, stream, steps,
                        per_beam.data());
        if (rc) break;
        const double ns = info.cell_steps > 0.0 ? info.stage_ms * 1e6 / info.cell_steps : 0.0;
        if (pass < 0) continue;
        if (ns_per_cell_step) ns_per_cell_step[id] = ns;
        if (pass == 0 || ns < best) { best = ns; best_id = id; }
    }
    release();
    if (rc) return rc;
    if (best_tile) *best_tile = best_id;
    return pdm1_plan_set_tile(pl, best_id);
}

int pdm1_plan_set_box_model(pdm1_plan *pl, const pdm1_box_model *model) {
    if (!pl) return set_error(PDM1_ERR_ARGUMENT, "plan is NULL");
    if (!model) {
        pl->cf.learned = 0;
        pl->cf.model = nullptr;
        return PDM1_OK;
    }
    if (!pl->p.moving_active_domain)
        return set_error(PDM1_ERR_UNSUPPORTED, "a box model needs a plan with moving_active_domain");
    BoxModelDev h;
    int rc = pack_box_model(model, h);
    if (rc) return rc;
    if (!pl->d_model) CUDA_TRY(pool_malloc((void **)&pl->d_model, sizeof(BoxModelDev)));
    CUDA_TRY(cudaMemcpy(pl->d_model, &h, sizeof h, cudaMemcpyHostToDevice));
    pl->cf.learned = 1;
    pl->cf.model = pl->d_model;
    return PDM1_OK;
}

int pdm1_plan_set_recorder(pdm1_plan *pl, float *rows, int max_rows, double tail_a, double tail_b) {
    if (!pl) return set_error(PDM1_ERR_ARGUMENT, "plan is NULL");
    if (!rows) {
        pl->cf.rec = nullptr;
        pl->cf.rec_max = 0;
        return PDM1_OK;
    }
    if (pl->p.moving_active_domain || pl->field || pl->nbeams != 1)
        return set_error(PDM1_ERR_UNSUPPORTED, "the recorder runs on one-beam full-domain plans");
    if (max_rows < 1) return set_error(PDM1_ERR_ARGUMENT, "max_rows must be positive");
    if (!(tail_a > 0.0 && tail_a < 1.0 && tail_b > 0.0 && tail_b < 1.0))
        return set_error(PDM1_ERR_ARGUMENT, "tail tolerances must lie in (0, 1)");
    pl->cf.rec = rows;
    pl->cf.rec_max = max_rows;
    pl->cf.rec_tail_tol[0] = tail_a;
    pl->cf.rec_tail_tol[1] = tail_b;
    return PDM1_OK;
}

int pdm1_march(pdm1_plan *pl, double *U, double *dose, double *energies, int max_steps,
               const double *snap_targets, int n_snap, double *snap_out, double *snap_E_out,
               pdm1_march_info *info, pdm1_stream_t stream) {
    if (!pl) return set_error(PDM1_ERR_ARGUMENT, "plan is NULL");
    if (pl->field) return set_error(PDM1_ERR_ARGUMENT, "pdm1_march takes a one-beam plan; use pdm1_field_march");
    return march_impl(pl, U, dose, energies, max_steps, snap_targets, n_snap, snap_out, snap_E_out,
                      info, stream, -1, nullptr);
}

int pdm1_march_steps(pdm1_plan *pl, double *U, double *dose, double *energies, int max_steps,
                     int step_limit, pdm1_march_info *info, pdm1_stream_t stream) {
    if (!pl) return set_error(PDM1_ERR_ARGUMENT, "plan is NULL");
    if (step_limit < 0) return set_error(PDM1_ERR_ARGUMENT, "step_limit must be >= 0");
    if (pl->field)   // a field plan: the prefix of every beam, the field dose of those steps
        return march_impl(pl, nullptr, dose, nullptr, max_steps, nullptr, 0, nullptr, nullptr, info, stream,
                          step_limit, nullptr);
    return march_impl(pl, U, dose, energies, max_steps, nullptr, 0, nullptr, nullptr, info, stream,
                      step_limit, nullptr);
}

// The building blocks act on the full grid of beam 0 of a one-beam plan.
static int full_domain_state(pdm1_plan *pl, double *U, double energy, double forced_dE, cudaStream_t stream) {
    MarchState st{};
    st.E = energy;
    st.forced_dE = forced_dE;
    st.dom = make_domain(0, 0, 0, pl->p.nx, pl->p.ny, pl->p.nz, 1, pl->cf.tile);
    st.prev = st.dom;
    st.Ua = U;
    st.Uprev = U;
    CUDA_TRY(cudaMemcpyAsync(pl->d_st, &st, sizeof st, cudaMemcpyHostToDevice, stream));
    return PDM1_OK;
}

int pdm1_spatial_operator(pdm1_plan *pl, const double *U, double energy, const double *bc, double *rhs,
                          pdm1_stream_t stream_) {
    (void)cudaGetLastError();
    if (!pl || !U || !rhs || pl->nbeams != 1) return set_error(PDM1_ERR_ARGUMENT, "NULL argument or field plan");
    cudaStream_t stream = (cudaStream_t)stream_;
    int rc = full_domain_state(pl, const_cast<double *>(U), energy, 0.0, stream);
    if (rc) return rc;
    StageArgs a = make_args(pl, nullptr, nullptr, nullptr);
    a.rhs_out = rhs;
    a.bc_plane = bc;
    const BeamDev &bm = pl->h_beams[0];
    double de = energy - bm.E_beam, s = bm.sigma_E;
    a.rhs_energy_density = dd_exp(-(de * de) / (2.0 * (s * s))) / (std::sqrt(2.0 * 3.141592653589793) * s);
    launch_stage(pl, MODE_RHS, pl->cf.grid_ctas, a, stream);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(stream));
    return PDM1_OK;
}

int pdm1_energy_step(pdm1_plan *pl, const double *U, double energy, double *dE_out, pdm1_stream_t stream_) {
    (void)cudaGetLastError();
    if (!pl || !U || !dE_out || pl->nbeams != 1) return set_error(PDM1_ERR_ARGUMENT, "NULL argument or field plan");
    cudaStream_t stream = (cudaStream_t)stream_;
    int rc = check_energy_range(pl, energy, energy);
    if (rc) return rc;
    init_kernel<<<1, 32, 0, stream>>>(pl->d_cf, pl->d_co, pl->d_st, nullptr, energy, pl->p.energy_window_sigma,
                                      const_cast<double *>(U), 1);
    cfl_kernel<<<dim3(cell_blocks(pl), 1), NT, 0, stream>>>(pl->d_cf, pl->d_co, pl->d_st, 0);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(pl->h_st, pl->d_st, sizeof(MarchState), cudaMemcpyDeviceToHost, stream));
    CUDA_TRY(cudaStreamSynchronize(stream));
    rc = device_error_status(*pl->h_st);
    if (rc) return rc;
    double inv = 0.0;
    unsigned long long bits = pl->h_st->inv_bits;
    std::memcpy(&inv, &bits, sizeof inv);
    double dE = pl->p.cfl / inv;
    *dE_out = pl->p.max_energy_step < dE ? pl->p.max_energy_step : dE;
    return PDM1_OK;
}

int pdm1_advance(pdm1_plan *pl, double *U, double energy, double dE, double *edep, pdm1_stream_t stream_) {
    (void)cudaGetLastError();
    if (!pl || !U || !edep || !(dE > 0.0) || pl->nbeams != 1) return set_error(PDM1_ERR_ARGUMENT, "dE must be positive.");
    cudaStream_t stream = (cudaStream_t)stream_;
    int rc = check_energy_range(pl, energy, energy - dE);
    if (rc) return rc;
    pl->cf.n_targets = 0;
    pl->cf.max_steps = 1;
    pl->cf.step_limit = -1;
    CUDA_TRY(cudaMemcpyAsync(pl->d_cf, &pl->cf, sizeof(ConfigDev), cudaMemcpyHostToDevice, stream));
    init_kernel<<<1, 32, 0, stream>>>(pl->d_cf, pl->d_co, pl->d_st, nullptr, energy, pl->p.energy_window_sigma, U, 1);
    rc = full_domain_state(pl, U, energy, dE, stream);
    if (rc) return rc;
    StageArgs a = make_args(pl, nullptr, edep, nullptr);
    launch_step(pl, a, nullptr, stream, -1, false);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(pl->h_st, pl->d_st, sizeof(MarchState), cudaMemcpyDeviceToHost, stream));
    CUDA_TRY(cudaStreamSynchronize(stream));
    return device_error_status(*pl->h_st);
}

int pdm1_coefficients(pdm1_plan *pl, const double *E, int n, double *out) {
    (void)cudaGetLastError();
    if (!pl || !E || !out || n <= 0) return set_error(PDM1_ERR_ARGUMENT, "NULL argument");
    double *dE_ = nullptr, *dout = nullptr;
    int *derr = nullptr;
    int nm = pl->p.n_materials;
    CUDA_TRY(cudaMalloc(&dE_, n * sizeof(double)));
    CUDA_TRY(cudaMalloc(&dout, (size_t)n * nm * 3 * sizeof(double)));
    CUDA_TRY(cudaMalloc(&derr, sizeof(int)));
    CUDA_TRY(cudaMemcpy(dE_, E, n * sizeof(double), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemset(derr, 0, sizeof(int)));
    int total = n * nm;
    coeff_eval_kernel<<<(total + 127) / 128, 128>>>(pl->d_cf, dE_, n, dout, derr);
    CUDA_TRY(cudaGetLastError());
    int herr = 0;
    CUDA_TRY(cudaMemcpy(out, dout, (size_t)total * 3 * sizeof(double), cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost));
    cudaFree(dE_);
    cudaFree(dout);
    cudaFree(derr);
    if (herr) return set_error(PDM1_ERR_RANGE, "energy outside coefficient table range");
    return PDM1_OK;
}

#define BATCH(kernel, ...)                                                 \
    if (n <= 0) return PDM1_OK;                                            \
    (void)cudaGetLastError();                                              \
    kernel<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(__VA_ARGS__); \
    CUDA_TRY(cudaGetLastError());                                          \
    CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));                 \
    return PDM1_OK;

int pdm1_weno_batch(const double *v5, double *out, int n, pdm1_stream_t stream) { BATCH(weno_batch_kernel, v5, out, n) }
int pdm1_project_batch(double *u4, int n, pdm1_stream_t stream) { BATCH(project_batch_kernel, u4, n) }
int pdm1_eigen_batch(const double *u4, int axis, double *lo_hi, int n, pdm1_stream_t stream) {
    BATCH(eigen_batch_kernel, u4, axis, lo_hi, n)
}
int pdm1_hll_batch(const double *l, const double *r, int axis, int ws, double *f, int n, pdm1_stream_t stream) {
    BATCH(hll_batch_kernel, l, r, axis, ws, f, n)
}
int pdm1_exp_batch(const double *x, double *y, int n, pdm1_stream_t stream) { BATCH(exp_batch_kernel, x, y, n) }

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free march.
//
// For callers that must not allocate GPU memory themselves: code running under
// a host application that owns the whole device memory through its own pool,
// plugins whose host forbids cudaMalloc/cudaFree (both synchronise the device
// and can fail once a pool has reserved the memory), and latency-critical
// paths where an allocation's implicit synchronisation is not allowed.  The
// plan data and the stage scratch live in one file-scope __device__ array of
// kNoAllocScratchBytes that every GPU loading this library holds until exit.
// ---------------------------------------------------------------------------
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;   // 16 MiB per GPU
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kNoAllocMaxDevices = 64;
// Device address of g_noalloc_scratch per device: in host code the symbol is
// only a host-side stand-in, so the address comes from cudaGetSymbolAddress.
void *g_noalloc_base[kNoAllocMaxDevices];
std::mutex g_noalloc_setup_mutex;

// PCHIP nodal slopes on the device, the same expressions as pchip_slopes()
// (physics/stopping_power.py:94-138), one thread per node.
__global__ void pchip_slopes_kernel(const double *E, const double *v, double *slope, int n) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    auto h = [&](int i) { return E[i + 1] - E[i]; };
    auto d = [&](int i) { return (v[i + 1] - v[i]) / (E[i + 1] - E[i]); };
    if (n == 2) {
        slope[k] = d(0);
        return;
    }
    auto endpoint = [](double h0, double h1, double d0, double d1) {
        double sl = ((2.0 * h0 + h1) * d0 - h0 * d1) / (h0 + h1);
        double s_sl = (double)((sl > 0.0) - (sl < 0.0)), s_d0 = (double)((d0 > 0.0) - (d0 < 0.0));
        double s_d1 = (double)((d1 > 0.0) - (d1 < 0.0));
        if (s_sl != s_d0) return 0.0;
        if (s_d0 != s_d1 && fabs(sl) > 3.0 * fabs(d0)) return 3.0 * d0;
        return sl;
    };
    if (k == 0) {
        slope[0] = endpoint(h(0), h(1), d(0), d(1));
    } else if (k == n - 1) {
        slope[n - 1] = endpoint(h(n - 2), h(n - 3), d(n - 2), d(n - 3));
    } else {
        double dm = d(k - 1), dk = d(k);
        double out = 0.0;
        if (dm * dk > 0.0) {
            double w1 = 2.0 * h(k) + h(k - 1);
            double w2 = h(k) + 2.0 * h(k - 1);
            out = (w1 + w2) / (w1 / dm + w2 / dk);
        }
        slope[k] = out;
    }
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Table metadata without touching the heap: node count and the log-spacing guess.
TableView table_meta(const pdm1_table &t) {
    TableView v{};
    v.n = t.n_nodes;
    double l0 = std::log(t.energy[0]), l1 = std::log(t.energy[t.n_nodes - 1]);
    double step = (l1 - l0) / (t.n_nodes - 1);
    bool uniform = t.energy[0] > 0.0 && step > 0.0;
    for (int i = 0; uniform && i < t.n_nodes; i += 97)
        if (std::fabs(std::log(t.energy[i]) - (l0 + step * i)) > 1e-6 * step) uniform = false;
    v.log_e0 = l0;
    v.inv_log_step = uniform ? 1.0 / step : 0.0;
    return v;
}

void launch_step_plain(const pdm1_problem &p, ConfigDev *d_cf, Coeffs *d_co, MarchState *d_st,
                       const StageArgs &a, double *energies, int tiles, cudaStream_t stream) {
    prologue_kernel<<<1, 256, 0, stream>>>(d_cf, d_co, d_st, energies);
    if (p.energy_scheme == PDM1_SCHEME_FORWARD_EULER) {
        stage_kernel<double, MODE_EULER, Tile0><<<tiles, NT, Tile0::smem_bytes<double>(), stream>>>(a);
        const size_t N = (size_t)p.nx * p.ny * p.nz;
        euler_finish_kernel<<<(int)std::max<size_t>(1, std::min<size_t>((N + NT - 1) / NT, 148 * 8)), NT, 0, stream>>>(a);
        return;
    }
    stage_kernel<double, MODE_A, Tile0><<<tiles, NT, Tile0::smem_bytes<double>(), stream>>>(a);
    stage_kernel<double, MODE_B, Tile0><<<tiles, NT, Tile0::smem_bytes<double>(), stream>>>(a);
    stage_kernel<double, MODE_C, Tile0><<<tiles, NT, Tile0::smem_bytes<double>(), stream>>>(a);
}

}  // namespace

extern "C" int pdm1_march_noalloc(const pdm1_problem *problem, double *U, double *dose,
                                  double *energies, int max_steps, pdm1_march_info *info,
                                  pdm1_stream_t stream_) {
    if (!U || !dose || !energies || max_steps < 1)
        return set_error(PDM1_ERR_ARGUMENT, "pdm1_march_noalloc: NULL buffer or max_steps < 1");
    int rc = validate_problem(problem);
    if (rc) return rc;
    const pdm1_problem &p = *problem;
    if (p.moving_active_domain)
        return set_error(PDM1_ERR_UNSUPPORTED, "pdm1_march_noalloc: the moving active box needs a plan");
    if (p.precision != PDM1_FP64)
        return set_error(PDM1_ERR_UNSUPPORTED,
                         "pdm1_march_noalloc: marches in FP64 only (the FP32 stencil needs a plan)");
    const size_t N = (size_t)p.nx * p.ny * p.nz;

    // layout of the scratch array
    size_t off = 0;
    const size_t o_cf = off; off = align256(off + sizeof(ConfigDev));
    const size_t o_co = off; off = align256(off + sizeof(Coeffs));
    const size_t o_st = off; off = align256(off + sizeof(MarchState));
    const size_t o_bm = off; off = align256(off + sizeof(BeamDev));
    const size_t o_to = off; off = align256(off + 2 * sizeof(int));
    const size_t o_sm = off; off = align256(off + sizeof(MarchSummary));
    size_t o_tab[kMaxMat][3];
    for (int m = 0; m < p.n_materials; ++m) {
        const pdm1_table *tabs[3] = {&p.materials[m].stopping_power, &p.materials[m].transport,
                                     &p.materials[m].nuclear};
        for (int q = 0; q < 3; ++q) {
            o_tab[m][q] = off;
            off = align256(off + 3 * (size_t)tabs[q]->n_nodes * sizeof(double));
        }
    }
    const size_t o_ids = off; off = align256(off + N * sizeof(int32_t));
    const size_t o_sp = off; off = align256(off + (size_t)p.nx * p.ny * sizeof(double));
    const size_t o_U1 = off; off = align256(off + 4 * N * sizeof(double));
    const size_t o_U2 = off; off = align256(off + 4 * N * sizeof(double));
    const size_t o_V = off; off = align256(off + 4 * N * sizeof(double));
    const size_t o_q = off; off = align256(off + N * sizeof(double));
    if (off > kNoAllocScratchBytes) {
        char msg[256];
        snprintf(msg, sizeof msg,
                 "pdm1_march_noalloc: the problem needs %zu bytes of scratch (%zu cells, %d materials); "
                 "the allocation-free march holds at most %zu bytes (about 130000 cells)",
                 off, N, p.n_materials, kNoAllocScratchBytes);
        return set_error(PDM1_ERR_ARGUMENT, msg);
    }
    double E0 = p.beam_energy + p.energy_window_sigma * p.energy_spread;
    {
        // energy range of the march against the tables (check_energy_range without a plan)
        const bool used[3] = {true, p.scattering == PDM1_SCATTERING_WENTZEL, p.nuclear != 0};
        for (int m = 0; m < p.n_materials; ++m) {
            const pdm1_table *tabs[3] = {&p.materials[m].stopping_power, &p.materials[m].transport,
                                         &p.materials[m].nuclear};
            for (int q = 0; q < 3; ++q) {
                if (!used[q]) continue;
                double lo = tabs[q]->energy[0], hi = tabs[q]->energy[tabs[q]->n_nodes - 1];
                if ((E0 > hi && !is_close(E0, hi)) || (p.energy_min < lo && !is_close(p.energy_min, lo)))
                    return set_error(PDM1_ERR_RANGE, "Energy outside coefficient table range.");
            }
        }
    }

    // once per device, with that device current: the scratch array's device address
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices) return set_error(PDM1_ERR_ARGUMENT, "device ordinal too large");
    // host threads making their first call on a device at the same time take turns
    // (the lock is held for the set-up only, not for the march)
    std::unique_lock<std::mutex> setup_lock(g_noalloc_setup_mutex);
    if (!g_noalloc_base[dev]) {
        void *ptr = nullptr;
        CUDA_TRY(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
        CUDA_TRY(cudaFuncSetAttribute(stage_kernel<double, MODE_A, Tile0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Tile0::smem_bytes<double>()));
        CUDA_TRY(cudaFuncSetAttribute(stage_kernel<double, MODE_B, Tile0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Tile0::smem_bytes<double>()));
        CUDA_TRY(cudaFuncSetAttribute(stage_kernel<double, MODE_C, Tile0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Tile0::smem_bytes<double>()));
        CUDA_TRY(cudaFuncSetAttribute(stage_kernel<double, MODE_EULER, Tile0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Tile0::smem_bytes<double>()));
        g_noalloc_base[dev] = ptr;
    }
    unsigned char *base = static_cast<unsigned char *>(g_noalloc_base[dev]);
    setup_lock.unlock();
    cudaStream_t stream = (cudaStream_t)stream_;
    ConfigDev *d_cf = reinterpret_cast<ConfigDev *>(base + o_cf);
    Coeffs *d_co = reinterpret_cast<Coeffs *>(base + o_co);
    MarchState *d_st = reinterpret_cast<MarchState *>(base + o_st);

    // the configuration, tables, ids and inflow profile go into the scratch array
    ConfigDev cf{};
    cf.nx = p.nx; cf.ny = p.ny; cf.nz = p.nz;
    cf.tile = kTiles[0];
    cf.tile_id = 0;
    cf.dx = p.dx; cf.dy = p.dy; cf.dz = p.dz;
    cf.nm = p.n_materials;
    cf.spatial = p.spatial_scheme;
    cf.stencil_radius = ghost_width(p.spatial_scheme);
    cf.cfl_floor = p.moving_active_domain && p.phantom_cfl_floor ? 1 : 0;
    cf.present = 0u;
    cf.scattering = p.scattering;
    cf.nuclear = p.nuclear ? 1 : 0;
    cf.interp = p.interpolation;
    cf.scheme = p.energy_scheme;
    cf.unit_speeds = p.wave_speeds == PDM1_SPEEDS_UNIT;
    bool sources = p.scattering != PDM1_SCATTERING_OFF || p.nuclear;
    cf.use_if = (p.energy_scheme == PDM1_SCHEME_IF_SSPRK3 && sources) ? 1 : 0;
    cf.strang = (p.energy_scheme != PDM1_SCHEME_IF_SSPRK3 && sources) ? 1 : 0;
    cf.cfl = p.cfl;
    cf.max_dE = p.max_energy_step;
    cf.Emin = p.energy_min;
    cf.max_steps = max_steps;
    cf.step_limit = -1;
    cf.n_targets = 0;
    cf.targets = nullptr;
    {
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cf.grid_ctas = std::max(1, std::min(make_domain(0, 0, 0, p.nx, p.ny, p.nz, 1, kTiles[0]).ntiles, 2 * sms));
    }
    cf.ids = reinterpret_cast<const int32_t *>(base + o_ids);
    cf.nbeams = 1;
    cf.cap = N;
    cf.beams = reinterpret_cast<const BeamDev *>(base + o_bm);
    cf.tile_off = reinterpret_cast<int *>(base + o_to);
    cf.summary = reinterpret_cast<MarchSummary *>(base + o_sm);
    BeamDev bm{};
    bm.E_beam = p.beam_energy;
    bm.sigma_E = p.energy_spread;
    bm.rf = dd_exp(-(p.angular_spread * p.angular_spread));
    bm.spatial = reinterpret_cast<const double *>(base + o_sp);
    bm.init_box = make_domain(0, 0, 0, p.nx, p.ny, p.nz, 1, kTiles[0]);
    for (int m = 0; m < p.n_materials; ++m) {
        const pdm1_material &mt = p.materials[m];
        const pdm1_table *tabs[3] = {&mt.stopping_power, &mt.transport, &mt.nuclear};
        TableView *views[3] = {&cf.mats[m].sp, &cf.mats[m].tr, &cf.mats[m].nuc};
        for (int q = 0; q < 3; ++q) {
            const pdm1_table &t = *tabs[q];
            double *dE_ = reinterpret_cast<double *>(base + o_tab[m][q]);
            *views[q] = table_meta(t);
            views[q]->E = dE_;
            views[q]->v = dE_ + t.n_nodes;
            views[q]->slope = dE_ + 2 * t.n_nodes;
            CUDA_TRY(cudaMemcpyAsync(dE_, t.energy, t.n_nodes * sizeof(double), cudaMemcpyHostToDevice, stream));
            CUDA_TRY(cudaMemcpyAsync(dE_ + t.n_nodes, t.value, t.n_nodes * sizeof(double), cudaMemcpyHostToDevice, stream));
            pchip_slopes_kernel<<<(t.n_nodes + 255) / 256, 256, 0, stream>>>(dE_, dE_ + t.n_nodes, dE_ + 2 * t.n_nodes, t.n_nodes);
        }
        cf.mats[m].density = mt.density;
        cf.mats[m].X0 = mt.radiation_length;
    }
    CUDA_TRY(cudaMemcpyAsync(base + o_ids, p.ids, N * sizeof(int32_t), cudaMemcpyHostToDevice, stream));
    CUDA_TRY(cudaMemcpyAsync(base + o_sp, p.inflow_spatial, (size_t)p.nx * p.ny * sizeof(double), cudaMemcpyHostToDevice, stream));
    CUDA_TRY(cudaMemcpyAsync(d_cf, &cf, sizeof cf, cudaMemcpyHostToDevice, stream));
    CUDA_TRY(cudaMemcpyAsync(base + o_bm, &bm, sizeof bm, cudaMemcpyHostToDevice, stream));
    // the array keeps the previous call's contents: clear what must start at zero
    CUDA_TRY(cudaMemsetAsync(d_co, 0, sizeof(Coeffs), stream));
    CUDA_TRY(cudaMemsetAsync(d_st, 0, sizeof(MarchState), stream));
    CUDA_TRY(cudaMemsetAsync(dose, 0, N * sizeof(double), stream));

    StageArgs a{};
    a.cf = d_cf;
    a.co = d_co;
    a.st = d_st;
    a.U1 = reinterpret_cast<double *>(base + o_U1);
    a.U2 = reinterpret_cast<double *>(base + o_U2);
    a.V = reinterpret_cast<double *>(base + o_V);
    a.qpart = reinterpret_cast<double *>(base + o_q);
    a.dose = dose;

    (void)cudaGetLastError();
    init_kernel<<<1, 32, 0, stream>>>(d_cf, d_co, d_st, energies, E0, p.energy_window_sigma, U, 1);
    const int cblocks = (int)std::max<size_t>(1, std::min<size_t>((N + NT - 1) / NT, 148 * 8));
    cfl_kernel<<<dim3(cblocks, 1), NT, 0, stream>>>(d_cf, d_co, d_st, 0);
    CUDA_TRY(cudaGetLastError());
    int launches = 2 + 3 * p.n_materials, chunks = 0;
    const int per_step = p.energy_scheme == PDM1_SCHEME_FORWARD_EULER ? 3 : 4;
    MarchState hs{};
    for (;;) {
        for (int s = 0; s < kStepsPerGraph; ++s) launch_step_plain(p, d_cf, d_co, d_st, a, energies, cf.grid_ctas, stream);
        CUDA_TRY(cudaGetLastError());
        launches += kStepsPerGraph * per_step;
        ++chunks;
        CUDA_TRY(cudaMemcpyAsync(&hs, d_st, sizeof hs, cudaMemcpyDeviceToHost, stream));
        CUDA_TRY(cudaStreamSynchronize(stream));
        if (hs.done || hs.error) break;
    }
    if (info) {
        info->n_steps = hs.step;
        info->n_snapshots = 0;
        info->final_state_valid = 1;
        info->graph_replays = 0;
        info->kernel_launches = launches;
        info->stage_launches = 0;
        info->stage_ms = 0.0;
        info->cell_steps = hs.cell_steps;
        info->max_box_cells = hs.max_cells;
    }
    (void)chunks;
    return device_error_status(hs);
}
