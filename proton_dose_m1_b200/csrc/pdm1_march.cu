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
__global__ void init_kernel(const ConfigDev *cfp, Coeffs *co, MarchState *st, double *energies,
                            double E0, double *U, int full_domain) {
    const ConfigDev &cf = *cfp;
    int t = threadIdx.x;
    if (t < cf.nm) {
        double s;
        if (!stopping_power_dev(cf.mats[t], E0, s)) atomicOr(&st->error, ERR_DEV_RANGE);
        co->S1[t] = s;
    }
    if (t == 0) {
        co->ed_next = energy_density(cf, E0);
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
        const bool moving = cf.moving && !full_domain;
        st->dom = moving ? cf.init_box : make_domain(0, 0, 0, cf.nx, cf.ny, cf.nz, 1);
        st->prev = st->dom;
        st->Ua = moving ? cf.bufA : U;
        st->Uprev = st->Ua;
        if (energies) energies[0] = E0;
    }
}

// ---------------------------------------------------------------------------
// prologue: one CTA per step
// ---------------------------------------------------------------------------
constexpr int kEvalPerMat = 13;   // 5 stage energies + 8 Gauss points

__global__ void __launch_bounds__(256) prologue_kernel(const ConfigDev *cfp, Coeffs *co,
                                                       MarchState *st, double *energies) {
    const ConfigDev &cf = *cfp;
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
                    int step = st->step + 1;
                    if (energies) energies[step] = En;
                    if (st->ti < cf.n_targets && fabs(En - cf.targets[st->ti]) <= 1e-12) {
                        slot = st->taken;
                        st->taken += 1;
                        st->ti += 1;
                    }
                    st->step = step;
                    st->E = En;
                    st->cell_steps += (double)st->dom.nx * st->dom.ny * st->dom.nz;
                    st->inv_bits = 0ull;
                    if (st->forced_dE > 0.0) st->done = 1;
                }
            }
        }
        sE = E; sdE = dE; sEn = En; sActive = active; sSlot = slot;
        co->E = E; co->dE = dE; co->E_next = En; co->active = active; co->snap_slot = slot;
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
        double v = energy_density(cf, ed_e[q]);
        if (q < 4) co->ed[q] = v; else co->ed_next = v;
    }
    __syncthreads();
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
        double ts[4], tn[4];
        const double width[4] = {dE / 3.0, 0.5 * dE, 2.0 * dE / 3.0, dE};
        for (int d = 0; d < 4; ++d) {
            double half = 0.5 * width[d];
            ts[d] = 0.0;
            tn[d] = 0.0;
            if (cf.scattering != PDM1_SCATTERING_OFF)
                ts[d] = half * (eTr[m][2 * d] / eS[m][5 + 2 * d] + eTr[m][2 * d + 1] / eS[m][6 + 2 * d]);
            if (cf.nuclear)
                tn[d] = half * (eNu[m][2 * d] / eS[m][5 + 2 * d] + eNu[m][2 * d + 1] / eS[m][6 + 2 * d]);
        }
        // depth index: 0 -> dE/3, 1 -> dE/2, 2 -> 2dE/3, 3 -> dE
        double u1 = cf.use_if ? ts[3] : 0.0, n1 = cf.use_if ? tn[3] : 0.0;
        double u2 = cf.use_if ? ts[1] : 0.0, n2 = cf.use_if ? tn[1] : 0.0;
        source_factor(u1, n1, false, co->c1p[m], co->c1c[m]);
        source_factor(u1, n1, true, co->c1ip[m], co->c1ic[m]);
        source_factor(u2, n2, false, co->c2p[m], co->c2c[m]);
        source_factor(u2, n2, true, co->c2ip[m], co->c2ic[m]);
        co->fip[0][m] = 1.0;
        co->fic[0][m] = 1.0;
        const int didx[4] = {0, 0, 2, 3};
        for (int q = 1; q < 4; ++q) {
            double a = cf.use_if ? ts[didx[q]] : 0.0, b = cf.use_if ? tn[didx[q]] : 0.0;
            source_factor(a, b, true, co->fip[q][m], co->fic[q][m]);
        }
        // Strang half steps over the full dE (energy.py:1168-1191, 1194-1260)
        double th = 0.5 * tn[3];
        co->hn[m] = (cf.strang && cf.nuclear) ? dd_exp(-(th < kExpClamp ? th : kExpClamp)) : 1.0;
        th = 0.5 * ts[3];
        co->hs[m] = (cf.strang && cf.scattering != PDM1_SCATTERING_OFF)
                        ? dd_exp(-(th < kExpClamp ? th : kExpClamp)) : 1.0;
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
            double phi_in = 0.0;
            if (lk == 0 && d.inflow) phi_in = cf.spatial[(size_t)(d.i0 + li) * cf.ny + (d.j0 + lj)] * co.ed_next;
            inv = fmax(inv, cfl_term(cf, u, co.S1[cf.ids[go]], lk == 0, phi_in, all_axes));
        }
    }
    if (!cf.moving) block_max_atomic(inv, &a.st->inv_bits);
}

// CFL bound of the state on the current domain (energy.py:539-660), with S and
// the spectrum at the state's energy: co->S1 / ed_next (static domain, first
// step) or co->S_cfl / ed_cfl (moving box, every step).  With vacuum-aware
// masks (energy.py:459-537) a direction counts only within 3 cells, along that
// axis, of an active cell.
__global__ void __launch_bounds__(NT) cfl_kernel(const ConfigDev *cfp, const Coeffs *co, MarchState *st,
                                                 int use_box_coeffs) {
    const ConfigDev &cf = *cfp;
    if (st->done) return;
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
            const unsigned char *act = cf.active;
            for (int ax = 0; ax < 3; ++ax) {
                int lo, hi, pos;
                size_t stride;
                if (ax == 0) { pos = li; lo = max(0, li - 3); hi = min(d.nx - 1, li + 3); stride = (size_t)d.ny * d.nz; }
                else if (ax == 1) { pos = lj; lo = max(0, lj - 3); hi = min(d.ny - 1, lj + 3); stride = d.nz; }
                else { pos = lk; lo = max(0, lk - 3); hi = min(d.nz - 1, lk + 3); stride = 1; }
                bool any = false;
                for (int q = lo; q <= hi && !any; ++q) any = act[o + (long long)(q - pos) * (long long)stride] != 0;
                use[ax] = any;
            }
        }
        double phi_in = 0.0;
        if (lk == 0 && d.inflow) phi_in = cf.spatial[(size_t)(d.i0 + li) * cf.ny + (d.j0 + lj)] * ed;
        inv = fmax(inv, cfl_term(cf, u, S[cf.ids[global_cell(cf, d, li, lj, lk)]], lk == 0, phi_in, use));
    }
    block_max_atomic(inv, &st->inv_bits);
}

// ---------------------------------------------------------------------------
// Moving active box (numerics/moving_active_domain.py, energy.py:1262-1494)
// ---------------------------------------------------------------------------

// Start of the march: the initial box, the compact state copied from the
// caller's full-grid U, and the slab maxima of that state.
__global__ void __launch_bounds__(NT) box_init_kernel(const ConfigDev *cfp, MarchState *st, const double *Ufull) {
    const ConfigDev &cf = *cfp;
    const DomainDev d = cf.init_box;
    const size_t N = (size_t)d.nx * d.ny * d.nz, NG = (size_t)cf.nx * cf.ny * cf.nz;
    for (size_t o = (size_t)blockIdx.x * NT + threadIdx.x; o < N; o += (size_t)gridDim.x * NT) {
        int lk = (int)(o % d.nz), lj = (int)((o / d.nz) % d.ny), li = (int)(o / ((size_t)d.nz * d.ny));
        size_t go = global_cell(cf, d, li, lj, lk);
        double u0 = 0.0;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            double v = Ufull[c * NG + go];
            cf.bufA[c * N + o] = v;
            if (c == 0) u0 = v;
        }
        atomic_max_double(&cf.slab[li], u0);
        atomic_max_double(&cf.slab[cf.nx + lj], u0);
        atomic_max_double(&cf.slab[cf.nx + cf.ny + lk], u0);
    }
}

// One CTA at the start of every step: desired_box (moving_active_domain.py:
// 107-193) from the slab maxima of the current state and the inflow at the
// step's energy; the switch to the new box; S and spectrum for the CFL.
__global__ void __launch_bounds__(256) box_kernel(const ConfigDev *cfp, Coeffs *co, MarchState *st) {
    const ConfigDev &cf = *cfp;
    __shared__ double red[256];
    __shared__ double s_ed, s_scale;
    __shared__ int s_lo[3], s_hi[3];
    __shared__ int s_done;
    const int t = threadIdx.x;
    if (t == 0) s_done = st->done || st->error;
    __syncthreads();
    if (s_done) return;
    const DomainDev d = st->dom;
    const double E = st->E;
    if (t == 0) s_ed = energy_density(cf, E);
    if (t < cf.nm) {
        double sv = 1.0;
        if (!stopping_power_dev(cf.mats[t], E, sv)) atomicOr(&st->error, ERR_DEV_RANGE);
        co->S_cfl[t] = sv;
    }
    __syncthreads();
    const double ed = s_ed;
    const unsigned long long *sx = cf.slab, *sy = cf.slab + cf.nx, *sz = cf.slab + cf.nx + cf.ny;
    auto as_d = [](unsigned long long b) { return __longlong_as_double((long long)b); };
    // scale = max(max phi, max phi_in)   (phi_in only while the box touches z = 0)
    double m = 0.0;
    for (int i = t; i < d.nx; i += 256) m = fmax(m, as_d(sx[i]));
    if (d.inflow)
        for (int e = t; e < d.nx * d.ny; e += 256) {
            int i = e / d.ny, j = e % d.ny;
            m = fmax(m, cf.spatial[(size_t)(d.i0 + i) * cf.ny + (d.j0 + j)] * ed);
        }
    red[t] = m;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (t < w) red[t] = fmax(red[t], red[t + w]);
        __syncthreads();
    }
    if (t == 0) {
        s_scale = red[0];
        for (int q = 0; q < 3; ++q) { s_lo[q] = INT_MAX; s_hi[q] = -1; }
    }
    __syncthreads();
    const double scale = s_scale;
    const double thr = cf.tol * scale;
    if (scale != 0.0) {
        // active x / y indices: slab max above the threshold, or an inflow cell
        // of that row above it (the inflow joins the k = 0 layer)
        for (int i = t; i < d.nx; i += 256) {
            bool act = as_d(sx[i]) > thr;
            if (!act && d.inflow)
                for (int j = 0; j < d.ny && !act; ++j)
                    act = cf.spatial[(size_t)(d.i0 + i) * cf.ny + (d.j0 + j)] * ed > thr;
            if (act) { atomicMin(&s_lo[0], i); atomicMax(&s_hi[0], i); }
        }
        for (int j = t; j < d.ny; j += 256) {
            bool act = as_d(sy[j]) > thr;
            if (!act && d.inflow)
                for (int i = 0; i < d.nx && !act; ++i)
                    act = cf.spatial[(size_t)(d.i0 + i) * cf.ny + (d.j0 + j)] * ed > thr;
            if (act) { atomicMin(&s_lo[1], j); atomicMax(&s_hi[1], j); }
        }
        for (int k = t; k < d.nz; k += 256) {
            bool act = as_d(sz[k]) > thr;
            if (!act && k == 0 && d.inflow)
                for (int e = 0; e < d.nx * d.ny && !act; ++e)
                    act = cf.spatial[(size_t)(d.i0 + e / d.ny) * cf.ny + (d.j0 + e % d.ny)] * ed > thr;
            if (act) { atomicMin(&s_lo[2], k); atomicMax(&s_hi[2], k); }
        }
    }
    __syncthreads();
    // reset the slab maxima for this step's stage C
    for (int e = t; e < cf.nx + cf.ny + cf.nz; e += 256) cf.slab[e] = 0ull;
    if (t == 0) {
        DomainDev nb;
        if (scale == 0.0 || s_hi[0] < 0 || s_hi[1] < 0 || s_hi[2] < 0) {
            nb = cf.init_box;
        } else {
            const int g = cf.guard;
            int ai0 = d.i0 + s_lo[0], ai1 = d.i0 + s_hi[0] + 1;
            int aj0 = d.j0 + s_lo[1], aj1 = d.j0 + s_hi[1] + 1;
            int ak0 = d.k0 + s_lo[2], ak1 = d.k0 + s_hi[2] + 1;
            int bi0 = ai0 - g > 0 ? ai0 - g : 0, bi1 = ai1 + g < cf.nx ? ai1 + g : cf.nx;
            int bj0 = aj0 - g > 0 ? aj0 - g : 0, bj1 = aj1 + g < cf.ny ? aj1 + g : cf.ny;
            int bk0 = ak0 - g > 0 ? ak0 - g : 0, bk1 = ak1 + g < cf.nz ? ak1 + g : cf.nz;
            nb = make_domain(bi0, bj0, bk0, bi1 - bi0, bj1 - bj0, bk1 - bk0, bk0 == 0);
        }
        bool same = nb.i0 == d.i0 && nb.j0 == d.j0 && nb.k0 == d.k0 && nb.nx == d.nx && nb.ny == d.ny && nb.nz == d.nz;
        st->reboxed = same ? 0 : 1;
        if (!same) {
            st->prev = d;
            st->Uprev = st->Ua;
            st->Ua = st->Ua == cf.bufA ? cf.bufB : cf.bufA;
            st->dom = nb;
        }
        st->inv_bits = 0ull;
        co->ed_cfl = ed;
        // vacuum-aware masks (energy.py:496-537) use the inflow of the new box
        st->newmax_bits = 0ull;
        double pin = 0.0;
        if (cf.vacuum_aware && nb.inflow)
            for (int e = 0; e < nb.nx * nb.ny; ++e)
                pin = fmax(pin, cf.spatial[(size_t)(nb.i0 + e / nb.ny) * cf.ny + (nb.j0 + e % nb.ny)] * ed);
        st->pin_max = pin;
    }
}

// Copy the overlap of the previous box into the new one (zeros elsewhere,
// moving_active_domain.py:196-232); for the vacuum-aware CFL also the max phi
// of the new box.
__global__ void __launch_bounds__(NT) rebox_kernel(const ConfigDev *cfp, MarchState *st) {
    const ConfigDev &cf = *cfp;
    if (st->done) return;
    const DomainDev d = st->dom;
    const bool moved = st->reboxed != 0;
    if (!moved && !cf.vacuum_aware) return;
    const DomainDev p = st->prev;
    const double *Up = st->Uprev;
    double *Ua = st->Ua;
    const size_t N = (size_t)d.nx * d.ny * d.nz, NP = (size_t)p.nx * p.ny * p.nz;
    double m = 0.0;
    for (size_t o = (size_t)blockIdx.x * NT + threadIdx.x; o < N; o += (size_t)gridDim.x * NT) {
        if (moved) {
            int lk = (int)(o % d.nz), lj = (int)((o / d.nz) % d.ny), li = (int)(o / ((size_t)d.nz * d.ny));
            int pi = d.i0 + li - p.i0, pj = d.j0 + lj - p.j0, pk = d.k0 + lk - p.k0;
            bool in = pi >= 0 && pi < p.nx && pj >= 0 && pj < p.ny && pk >= 0 && pk < p.nz;
            size_t po = in ? ((size_t)pi * p.ny + pj) * p.nz + pk : 0;
#pragma unroll
            for (int c = 0; c < 4; ++c) Ua[c * N + o] = in ? Up[c * NP + po] : 0.0;
        }
        m = fmax(m, Ua[o]);
    }
    if (cf.vacuum_aware) block_max_atomic(m, &st->newmax_bits);
}

// Activity mask of the vacuum-aware CFL: phi above tol * max(phi, phi_in),
// plus the inflow at the entrance layer (numerics/energy.py:496-537).
__global__ void __launch_bounds__(NT) mask_kernel(const ConfigDev *cfp, const Coeffs *co, const MarchState *st) {
    const ConfigDev &cf = *cfp;
    if (st->done) return;
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
            act = act || cf.spatial[(size_t)(d.i0 + li) * cf.ny + (d.j0 + lj)] * ed > thr;
        cf.active[o] = act ? 1 : 0;
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

struct pdm1_plan {
    pdm1_problem p{};
    ConfigDev cf{};
    ConfigDev *d_cf = nullptr;
    Coeffs *d_co = nullptr;
    MarchState *d_st = nullptr;
    MarchState *h_st = nullptr;   // pinned
    double *d_tables = nullptr;
    int32_t *d_ids = nullptr;
    double *d_spatial = nullptr;
    double *d_targets = nullptr;
    double *d_U1 = nullptr, *d_U2 = nullptr, *d_V = nullptr, *d_q = nullptr;
    double *d_bufA = nullptr, *d_bufB = nullptr;   // moving box: compact-state ping-pong
    unsigned long long *d_slab = nullptr;
    unsigned char *d_active = nullptr;
    size_t workspace = 0;
    std::vector<int32_t> h_ids;
    std::vector<double> h_spatial;
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

// Upload one table; return its TableView (device pointers).
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

int validate_problem(const pdm1_problem *p) {
    if (!p) return set_error(PDM1_ERR_ARGUMENT, "problem is NULL");
    if (p->nx <= 0 || p->ny <= 0 || p->nz <= 0) return set_error(PDM1_ERR_ARGUMENT, "grid dimensions must be positive");
    if (p->nz < 4) return set_error(PDM1_ERR_ARGUMENT, "WENO-Z inflow extrapolation requires at least four z cells.");
    if (p->n_materials < 1 || p->n_materials > kMaxMat) return set_error(PDM1_ERR_ARGUMENT, "n_materials must be in 1..16");
    if (!p->materials || !p->ids || !p->inflow_spatial) return set_error(PDM1_ERR_ARGUMENT, "NULL materials/ids/inflow");
    if (!(p->dx > 0 && p->dy > 0 && p->dz > 0)) return set_error(PDM1_ERR_ARGUMENT, "spacings must be positive");
    if (!(p->energy_spread > 0.0))
        return set_error(PDM1_ERR_ARGUMENT, "Zero energy spread is not supported by the Gaussian inflow.");
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

bool is_close(double a, double b) { return std::fabs(a - b) <= 1e-8 + 1e-5 * std::fabs(b); }

// Energy range the march will evaluate tables at: [energy_min, E_start]
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

int n_tiles(const pdm1_problem &p) {
    return ((p.nx + TX - 1) / TX) * ((p.ny + TY - 1) / TY) * ((p.nz + TZ - 1) / TZ);
}

int cell_blocks(const pdm1_problem &p) {
    size_t n = (size_t)p.nx * p.ny * p.nz;
    size_t b = (n + NT - 1) / NT;
    return (int)std::min<size_t>(b, 148 * 8);
}

// Launch one energy step (prologue + stages) on `stream`; returns launches.
// One stage launch in the plan's precision.
void launch_stage(const pdm1_plan *pl, int mode, int grid, const StageArgs &a, cudaStream_t stream) {
    if (pl->p.precision == PDM1_FP32_FP64) {
        launch_stage_fp32(mode, grid, a, stream);
        return;
    }
    const size_t bytes = stage_smem_bytes<double>();
    switch (mode) {
    case MODE_A: stage_kernel<double, MODE_A><<<grid, NT, bytes, stream>>>(a); break;
    case MODE_B: stage_kernel<double, MODE_B><<<grid, NT, bytes, stream>>>(a); break;
    case MODE_C: stage_kernel<double, MODE_C><<<grid, NT, bytes, stream>>>(a); break;
    case MODE_EULER: stage_kernel<double, MODE_EULER><<<grid, NT, bytes, stream>>>(a); break;
    default: stage_kernel<double, MODE_RHS><<<grid, NT, bytes, stream>>>(a); break;
    }
}

// The moving box's per-step work ahead of the prologue: desired box, rebox,
// activity mask, CFL bound over the new box.
int launch_box_step(pdm1_plan *pl, cudaStream_t stream) {
    const pdm1_problem &p = pl->p;
    box_kernel<<<1, 256, 0, stream>>>(pl->d_cf, pl->d_co, pl->d_st);
    rebox_kernel<<<cell_blocks(p), NT, 0, stream>>>(pl->d_cf, pl->d_st);
    int n = 3;
    if (p.vacuum_aware_cfl) {
        mask_kernel<<<cell_blocks(p), NT, 0, stream>>>(pl->d_cf, pl->d_co, pl->d_st);
        ++n;
    }
    cfl_kernel<<<cell_blocks(p), NT, 0, stream>>>(pl->d_cf, pl->d_co, pl->d_st, 1);
    return n;
}

int launch_step(pdm1_plan *pl, const StageArgs &a, cudaStream_t stream) {
    const pdm1_problem &p = pl->p;
    const int grid = pl->cf.grid_ctas;
    prologue_kernel<<<1, 256, 0, stream>>>(pl->d_cf, pl->d_co, pl->d_st, nullptr);
    if (p.energy_scheme == PDM1_SCHEME_FORWARD_EULER) {
        launch_stage(pl, MODE_EULER, grid, a, stream);
        euler_finish_kernel<<<cell_blocks(p), NT, 0, stream>>>(a);
        return 3;
    }
    launch_stage(pl, MODE_A, grid, a, stream);
    launch_stage(pl, MODE_B, grid, a, stream);
    launch_stage(pl, MODE_C, grid, a, stream);
    return 4;
}

int launch_step_with_energies(pdm1_plan *pl, const StageArgs &a, double *energies, cudaStream_t stream,
                              int slot) {
    const pdm1_problem &p = pl->p;
    const int grid = pl->cf.grid_ctas;
    int launched = 0;
    if (p.moving_active_domain) launched += launch_box_step(pl, stream);
    prologue_kernel<<<1, 256, 0, stream>>>(pl->d_cf, pl->d_co, pl->d_st, energies);
    // external event nodes: real timestamps when the step is replayed from a graph
    cudaEventRecordWithFlags(pl->ev[2 * slot], stream, cudaEventRecordExternal);
    int n;
    if (p.energy_scheme == PDM1_SCHEME_FORWARD_EULER) {
        launch_stage(pl, MODE_EULER, grid, a, stream);
        n = 1;
    } else {
        launch_stage(pl, MODE_A, grid, a, stream);
        launch_stage(pl, MODE_B, grid, a, stream);
        launch_stage(pl, MODE_C, grid, a, stream);
        n = 3;
    }
    cudaEventRecordWithFlags(pl->ev[2 * slot + 1], stream, cudaEventRecordExternal);
    launched += n + 1;
    if (p.energy_scheme == PDM1_SCHEME_FORWARD_EULER) {
        euler_finish_kernel<<<cell_blocks(p), NT, 0, stream>>>(a);
        ++launched;
    }
    return launched;
}

int set_smem_attributes() {
    static bool done = false;
    if (done) return PDM1_OK;
    CUDA_TRY(cudaFuncSetAttribute(stage_kernel<double, MODE_A>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stage_smem_bytes<double>()));
    CUDA_TRY(cudaFuncSetAttribute(stage_kernel<double, MODE_B>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stage_smem_bytes<double>()));
    CUDA_TRY(cudaFuncSetAttribute(stage_kernel<double, MODE_C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stage_smem_bytes<double>()));
    CUDA_TRY(cudaFuncSetAttribute(stage_kernel<double, MODE_EULER>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stage_smem_bytes<double>()));
    CUDA_TRY(cudaFuncSetAttribute(stage_kernel<double, MODE_RHS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stage_smem_bytes<double>()));
    CUDA_TRY((cudaError_t)stage_fp32_set_attributes());
    done = true;
    return PDM1_OK;
}

int device_error_status(const MarchState &st) {
    if (st.error & ERR_DEV_RANGE) return set_error(PDM1_ERR_RANGE, "energy outside a coefficient table during the march");
    if (st.error & ERR_DEV_MAXSTEPS) return set_error(PDM1_ERR_MAX_STEPS, "energies buffer shorter than the march");
    if (st.error & ERR_DEV_NONFINITE) return set_error(PDM1_ERR_NONFINITE, "non-finite state or non-positive energy step during the march");
    return PDM1_OK;
}

}  // namespace

extern "C" {

const char *pdm1_last_error(void) { return g_error; }
const char *pdm1_version(void) { return "pdm1 0.1 sm_100a"; }

void pdm1_plan_destroy(pdm1_plan *pl) {
    if (!pl) return;
    cudaFree(pl->d_cf);
    cudaFree(pl->d_co);
    cudaFree(pl->d_st);
    cudaFreeHost(pl->h_st);
    cudaFree(pl->d_tables);
    cudaFree(pl->d_ids);
    cudaFree(pl->d_spatial);
    cudaFree(pl->d_targets);
    cudaFree(pl->d_U1);
    cudaFree(pl->d_U2);
    cudaFree(pl->d_V);
    cudaFree(pl->d_q);
    cudaFree(pl->d_bufA);
    cudaFree(pl->d_bufB);
    cudaFree(pl->d_slab);
    cudaFree(pl->d_active);
    if (pl->ready) cudaEventDestroy(pl->ready);
    for (cudaEvent_t e : pl->ev)
        if (e) cudaEventDestroy(e);
    if (pl->own_stream) cudaStreamDestroy(pl->own_stream);
    delete pl;
}

int pdm1_plan_create(const pdm1_problem *problem, pdm1_plan **out) {
    if (!out) return set_error(PDM1_ERR_ARGUMENT, "out is NULL");
    *out = nullptr;
    int rc = validate_problem(problem);
    if (rc) return rc;
    rc = set_smem_attributes();
    if (rc) return rc;
    pdm1_plan *pl = new pdm1_plan();
    pl->p = *problem;
    const pdm1_problem &p = pl->p;
    size_t N = (size_t)p.nx * p.ny * p.nz;
    pl->h_ids.assign(problem->ids, problem->ids + N);
    pl->h_spatial.assign(problem->inflow_spatial, problem->inflow_spatial + (size_t)p.nx * p.ny);
    pl->p.ids = pl->h_ids.data();
    pl->p.inflow_spatial = pl->h_spatial.data();
    pl->p.materials = nullptr;   // tables are copied below; host pointers are not kept

    std::vector<double> blob;
    std::vector<std::pair<size_t, int>> fix;
    ConfigDev &cf = pl->cf;
    cf.nx = p.nx; cf.ny = p.ny; cf.nz = p.nz;
    cf.dx = p.dx; cf.dy = p.dy; cf.dz = p.dz;
    cf.nm = p.n_materials;
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
    cf.E_beam = p.beam_energy;
    cf.sigma_E = p.energy_spread;
    cf.rf = dd_exp(-(p.angular_spread * p.angular_spread));
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
    auto fail = [&](int code) { pdm1_plan_destroy(pl); return code; };
    cudaError_t e;
#define ALLOC(ptr, bytes)                                                      \
    e = cudaMalloc((void **)&(ptr), (bytes));                                  \
    if (e != cudaSuccess) {                                                    \
        set_error(PDM1_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e)); \
        return fail(PDM1_ERR_CUDA);                                            \
    }
    ALLOC(pl->d_tables, blob.size() * sizeof(double));
    ALLOC(pl->d_cf, sizeof(ConfigDev));
    ALLOC(pl->d_co, sizeof(Coeffs));
    ALLOC(pl->d_st, sizeof(MarchState));
    ALLOC(pl->d_ids, N * sizeof(int32_t));
    ALLOC(pl->d_spatial, (size_t)p.nx * p.ny * sizeof(double));
    ALLOC(pl->d_targets, 64 * sizeof(double));
    ALLOC(pl->d_U1, 4 * N * sizeof(double));
    ALLOC(pl->d_U2, 4 * N * sizeof(double));
    ALLOC(pl->d_V, 4 * N * sizeof(double));
    ALLOC(pl->d_q, N * sizeof(double));
    if (p.moving_active_domain) {
        ALLOC(pl->d_bufA, 4 * N * sizeof(double));
        ALLOC(pl->d_bufB, 4 * N * sizeof(double));
        ALLOC(pl->d_slab, (size_t)(p.nx + p.ny + p.nz) * sizeof(unsigned long long));
        ALLOC(pl->d_active, N);
    }
#undef ALLOC
    pl->workspace = (13 * N) * sizeof(double);
    if (cudaMallocHost((void **)&pl->h_st, sizeof(MarchState)) != cudaSuccess ||
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
    cf.ids = pl->d_ids;
    cf.spatial = pl->d_spatial;
    cf.targets = pl->d_targets;
    // moving active box: initial box from the inflow support (moving_active_domain.py:35-60)
    cf.moving = p.moving_active_domain ? 1 : 0;
    cf.vacuum_aware = (p.moving_active_domain && p.vacuum_aware_cfl) ? 1 : 0;
    cf.guard = p.active_guard_cells;
    cf.tol = p.active_relative_tolerance;
    cf.bufA = pl->d_bufA;
    cf.bufB = pl->d_bufB;
    cf.slab = pl->d_slab;
    cf.active = pl->d_active;
    if (p.moving_active_domain) {
        int ilo = -1, ihi = -1, jlo = -1, jhi = -1;
        for (int i = 0; i < p.nx; ++i)
            for (int j = 0; j < p.ny; ++j)
                if (pl->h_spatial[(size_t)i * p.ny + j] > 0.0) {
                    if (ilo < 0 || i < ilo) ilo = i;
                    if (i > ihi) ihi = i;
                    if (jlo < 0 || j < jlo) jlo = j;
                    if (j > jhi) jhi = j;
                }
        if (ilo < 0) return fail(set_error(PDM1_ERR_NO_BEAM, "Beam inflow has empty transverse support."));
        const int g = p.active_guard_cells;
        int i0 = std::max(0, ilo - g), i1 = std::min(p.nx, ihi + 1 + g);
        int j0 = std::max(0, jlo - g), j1 = std::min(p.ny, jhi + 1 + g);
        int k1 = std::min(p.nz, 1 + g);
        cf.init_box = make_domain(i0, j0, 0, i1 - i0, j1 - j0, k1, 1);
        if (k1 < 4)
            return fail(set_error(PDM1_ERR_ARGUMENT, "WENO-Z inflow extrapolation requires at least four z cells."));
    }
    {
        int dev = 0, sms = 148;
        if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        int tiles = make_domain(0, 0, 0, p.nx, p.ny, p.nz, 1).ntiles;
        cf.grid_ctas = std::max(1, std::min(tiles, 2 * sms));
    }
    if (cudaMemcpy(pl->d_tables, blob.data(), blob.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(pl->d_ids, pl->h_ids.data(), N * sizeof(int32_t), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(pl->d_spatial, pl->h_spatial.data(), (size_t)p.nx * p.ny * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(pl->d_cf, &cf, sizeof(ConfigDev), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(pl->d_co, 0, sizeof(Coeffs)) != cudaSuccess)
        return fail(set_error(PDM1_ERR_CUDA, "plan upload failed"));
    *out = pl;
    return PDM1_OK;
}

size_t pdm1_plan_workspace_bytes(const pdm1_plan *pl) { return pl ? pl->workspace : 0; }

static int march_impl(pdm1_plan *pl, double *U, double *dose, double *energies, int max_steps,
                      const double *snap_targets, int n_snap, double *snap_out, double *snap_E_out,
                      pdm1_march_info *info, pdm1_stream_t stream_, int step_limit) {
    if (!pl || !U || !dose || !energies || max_steps < 1)
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
    double E0 = p.beam_energy + p.energy_window_sigma * p.energy_spread;
    int rc = check_energy_range(pl, E0, p.energy_min);
    if (rc) return rc;
    // sorted unique targets in [energy_min, E0], descending (energy.py:1531-1538)
    std::vector<double> tg;
    for (int i = 0; i < n_snap; ++i) {
        double t = snap_targets[i];
        if (p.energy_min <= t && t <= E0 && std::find(tg.begin(), tg.end(), t) == tg.end()) tg.push_back(t);
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
    size_t N = (size_t)p.nx * p.ny * p.nz;
    CUDA_TRY(cudaMemsetAsync(dose, 0, N * sizeof(double), stream));
    if (p.moving_active_domain && !tg.empty())
        CUDA_TRY(cudaMemsetAsync(snap_out, 0, tg.size() * 4 * N * sizeof(double), stream));
    (void)cudaGetLastError();   // start from a clean launch-error state
    init_kernel<<<1, 32, 0, stream>>>(pl->d_cf, pl->d_co, pl->d_st, energies, E0, U, 0);
    if (p.moving_active_domain) {
        CUDA_TRY(cudaMemsetAsync(pl->d_slab, 0, (size_t)(p.nx + p.ny + p.nz) * sizeof(unsigned long long), stream));
        box_init_kernel<<<cell_blocks(p), NT, 0, stream>>>(pl->d_cf, pl->d_st, U);
    } else {
        cfl_kernel<<<cell_blocks(p), NT, 0, stream>>>(pl->d_cf, pl->d_co, pl->d_st, 0);
    }
    CUDA_TRY(cudaGetLastError());
    int launches = 2;
    StageArgs a = make_args(pl, dose, nullptr, snap_out);
    // capture a chunk of steps into a graph; replay until the device says done
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int per_step = 0;
    bool use_graph = true;
    if (cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
        for (int s = 0; s < kStepsPerGraph; ++s) per_step = launch_step_with_energies(pl, a, energies, stream, s);
        if (cudaStreamEndCapture(stream, &graph) != cudaSuccess ||
            cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) {
            use_graph = false;
        }
    } else {
        use_graph = false;
    }
    (void)cudaGetLastError();   // a refused capture falls back to direct launches
    int replays = 0, prev_step = 0, stage_launches = 0;
    double stage_ms = 0.0;
    const int stages_per_step = p.energy_scheme == PDM1_SCHEME_FORWARD_EULER ? 1 : 3;
    for (;;) {
        if (use_graph) {
            CUDA_TRY(cudaGraphLaunch(exec, stream));
            replays++;
        } else {
            for (int s = 0; s < kStepsPerGraph; ++s) per_step = launch_step_with_energies(pl, a, energies, stream, s);
            CUDA_TRY(cudaGetLastError());
        }
        CUDA_TRY(cudaMemcpyAsync(pl->h_st, pl->d_st, sizeof(MarchState), cudaMemcpyDeviceToHost, stream));
        CUDA_TRY(cudaStreamSynchronize(stream));
        int ran = pl->h_st->step - prev_step;   // steps of this chunk that did work
        prev_step = pl->h_st->step;
        launches += ran * per_step + (kStepsPerGraph - ran) * per_step;
        for (int s = 0; s < ran && s < kStepsPerGraph; ++s) {
            float ms = 0.f;
            CUDA_TRY(cudaEventElapsedTime(&ms, pl->ev[2 * s], pl->ev[2 * s + 1]));
            stage_ms += ms;
        }
        stage_launches += ran * stages_per_step;
        if (pl->h_st->done || pl->h_st->error) break;
    }
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (p.moving_active_domain) {
        embed_kernel<<<cell_blocks(p), NT, 0, stream>>>(pl->d_cf, pl->d_st, U);
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaStreamSynchronize(stream));
        ++launches;
    }
    rc = device_error_status(*pl->h_st);
    if (info) {
        info->n_steps = pl->h_st->step;
        info->n_snapshots = pl->h_st->taken;
        info->final_state_valid = 1;
        info->graph_replays = replays;
        info->kernel_launches = launches;
        info->stage_launches = stage_launches;
        info->stage_ms = stage_ms;
        info->cell_steps = pl->h_st->cell_steps;
    }
    if (snap_E_out)
        for (int i = 0; i < pl->h_st->taken; ++i) snap_E_out[i] = tg[i];
    return rc;
}

int pdm1_march(pdm1_plan *pl, double *U, double *dose, double *energies, int max_steps,
               const double *snap_targets, int n_snap, double *snap_out, double *snap_E_out,
               pdm1_march_info *info, pdm1_stream_t stream) {
    return march_impl(pl, U, dose, energies, max_steps, snap_targets, n_snap, snap_out, snap_E_out,
                      info, stream, -1);
}

int pdm1_march_steps(pdm1_plan *pl, double *U, double *dose, double *energies, int max_steps,
                     int step_limit, pdm1_march_info *info, pdm1_stream_t stream) {
    if (step_limit < 0) return set_error(PDM1_ERR_ARGUMENT, "step_limit must be >= 0");
    return march_impl(pl, U, dose, energies, max_steps, nullptr, 0, nullptr, nullptr, info, stream,
                      step_limit);
}

int pdm1_spatial_operator(pdm1_plan *pl, const double *U, double energy, const double *bc, double *rhs,
                          pdm1_stream_t stream_) {
    (void)cudaGetLastError();
    if (!pl || !U || !rhs) return set_error(PDM1_ERR_ARGUMENT, "NULL argument");
    cudaStream_t stream = (cudaStream_t)stream_;
    {
        MarchState st{};
        st.dom = make_domain(0, 0, 0, pl->p.nx, pl->p.ny, pl->p.nz, 1);
        st.prev = st.dom;
        st.Ua = const_cast<double *>(U);
        st.Uprev = st.Ua;
        CUDA_TRY(cudaMemcpyAsync(pl->d_st, &st, sizeof st, cudaMemcpyHostToDevice, stream));
    }
    StageArgs a = make_args(pl, nullptr, nullptr, nullptr);
    a.rhs_out = rhs;
    a.bc_plane = bc;
    double de = energy - pl->p.beam_energy, s = pl->p.energy_spread;
    a.rhs_energy_density = dd_exp(-(de * de) / (2.0 * (s * s))) / (std::sqrt(2.0 * 3.141592653589793) * s);
    launch_stage(pl, MODE_RHS, pl->cf.grid_ctas, a, stream);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(stream));
    return PDM1_OK;
}

int pdm1_energy_step(pdm1_plan *pl, const double *U, double energy, double *dE_out, pdm1_stream_t stream_) {
    (void)cudaGetLastError();
    if (!pl || !U || !dE_out) return set_error(PDM1_ERR_ARGUMENT, "NULL argument");
    cudaStream_t stream = (cudaStream_t)stream_;
    int rc = check_energy_range(pl, energy, energy);
    if (rc) return rc;
    init_kernel<<<1, 32, 0, stream>>>(pl->d_cf, pl->d_co, pl->d_st, nullptr, energy, const_cast<double *>(U), 1);
    cfl_kernel<<<cell_blocks(pl->p), NT, 0, stream>>>(pl->d_cf, pl->d_co, pl->d_st, 0);
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
    if (!pl || !U || !edep || !(dE > 0.0)) return set_error(PDM1_ERR_ARGUMENT, "dE must be positive.");
    cudaStream_t stream = (cudaStream_t)stream_;
    int rc = check_energy_range(pl, energy, energy - dE);
    if (rc) return rc;
    pl->cf.n_targets = 0;
    pl->cf.max_steps = 1;
    pl->cf.step_limit = -1;
    CUDA_TRY(cudaMemcpyAsync(pl->d_cf, &pl->cf, sizeof(ConfigDev), cudaMemcpyHostToDevice, stream));
    init_kernel<<<1, 32, 0, stream>>>(pl->d_cf, pl->d_co, pl->d_st, nullptr, energy, U, 1);
    MarchState st{};
    st.E = energy;
    st.forced_dE = dE;
    st.dom = make_domain(0, 0, 0, pl->p.nx, pl->p.ny, pl->p.nz, 1);
    st.prev = st.dom;
    st.Ua = U;
    st.Uprev = U;
    CUDA_TRY(cudaMemcpyAsync(pl->d_st, &st, sizeof st, cudaMemcpyHostToDevice, stream));
    StageArgs a = make_args(pl, nullptr, edep, nullptr);
    launch_step(pl, a, stream);
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
        stage_kernel<double, MODE_EULER><<<tiles, NT, stage_smem_bytes<double>(), stream>>>(a);
        euler_finish_kernel<<<cell_blocks(p), NT, 0, stream>>>(a);
        return;
    }
    stage_kernel<double, MODE_A><<<tiles, NT, stage_smem_bytes<double>(), stream>>>(a);
    stage_kernel<double, MODE_B><<<tiles, NT, stage_smem_bytes<double>(), stream>>>(a);
    stage_kernel<double, MODE_C><<<tiles, NT, stage_smem_bytes<double>(), stream>>>(a);
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
    const size_t N = (size_t)p.nx * p.ny * p.nz;

    // layout of the scratch array
    size_t off = 0;
    const size_t o_cf = off; off = align256(off + sizeof(ConfigDev));
    const size_t o_co = off; off = align256(off + sizeof(Coeffs));
    const size_t o_st = off; off = align256(off + sizeof(MarchState));
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
    if (!g_noalloc_base[dev]) {
        void *ptr = nullptr;
        CUDA_TRY(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
        CUDA_TRY(cudaFuncSetAttribute(stage_kernel<double, MODE_A>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stage_smem_bytes<double>()));
        CUDA_TRY(cudaFuncSetAttribute(stage_kernel<double, MODE_B>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stage_smem_bytes<double>()));
        CUDA_TRY(cudaFuncSetAttribute(stage_kernel<double, MODE_C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stage_smem_bytes<double>()));
        CUDA_TRY(cudaFuncSetAttribute(stage_kernel<double, MODE_EULER>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stage_smem_bytes<double>()));
        g_noalloc_base[dev] = ptr;
    }
    unsigned char *base = static_cast<unsigned char *>(g_noalloc_base[dev]);
    cudaStream_t stream = (cudaStream_t)stream_;
    ConfigDev *d_cf = reinterpret_cast<ConfigDev *>(base + o_cf);
    Coeffs *d_co = reinterpret_cast<Coeffs *>(base + o_co);
    MarchState *d_st = reinterpret_cast<MarchState *>(base + o_st);

    // the configuration, tables, ids and inflow profile go into the scratch array
    ConfigDev cf{};
    cf.nx = p.nx; cf.ny = p.ny; cf.nz = p.nz;
    cf.dx = p.dx; cf.dy = p.dy; cf.dz = p.dz;
    cf.nm = p.n_materials;
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
    cf.E_beam = p.beam_energy;
    cf.sigma_E = p.energy_spread;
    cf.rf = dd_exp(-(p.angular_spread * p.angular_spread));
    cf.max_steps = max_steps;
    cf.step_limit = -1;
    cf.n_targets = 0;
    cf.targets = nullptr;
    {
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cf.grid_ctas = std::max(1, std::min(make_domain(0, 0, 0, p.nx, p.ny, p.nz, 1).ntiles, 2 * sms));
    }
    cf.ids = reinterpret_cast<const int32_t *>(base + o_ids);
    cf.spatial = reinterpret_cast<const double *>(base + o_sp);
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
    init_kernel<<<1, 32, 0, stream>>>(d_cf, d_co, d_st, energies, E0, U, 1);
    cfl_kernel<<<cell_blocks(p), NT, 0, stream>>>(d_cf, d_co, d_st, 0);
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
    }
    (void)chunks;
    return device_error_status(hs);
}
