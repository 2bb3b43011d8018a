// pdm1_stage.cuh -- the fused IF-SSPRK3 stage kernel, templated on the
// arithmetic of the stencil (WENO-Z, interface projection, HLL, divergence):
// double in pdm1_march.cu, float in pdm1_stage_fp32.cu.  The stage update,
// cell projection, CFL bound and dose stay in double in both.
#pragma once

#include "pdm1_device.cuh"

namespace pdm1 {

// Element e of component c's copy of an arm of asz elements.  Double arms are
// [c][e]; float arms hold the components in pairs, [c / 2][e][c % 2], so a
// 64-bit load brings two components of a cell into the packed f32x2 lanes.
template <typename T>
__device__ __forceinline__ T &arm_at(T *arm, int asz, int c, int e) {
    if constexpr (sizeof(T) == sizeof(float)) return arm[((c >> 1) * asz + e) * 2 + (c & 1)];
    else return arm[c * asz + e];
}

// LEARN (stage C of a plan with a learned box): the tile's fluence moments of
// the new state are accumulated for the next step's proposer.
template <typename T, int MODE, class Tl, bool LEARN = false>
__global__ void __launch_bounds__(NT, sizeof(T) == sizeof(double) ? 2 : 4) stage_kernel(StageArgs a) {
    constexpr int TX = Tl::TX, TY = Tl::TY, TZ = Tl::TZ;
    constexpr int NF = Tl::NF, NFX = Tl::NFX, NFY = Tl::NFY;
    constexpr int SX = Tl::SX, SY = Tl::SY, SZ = Tl::SZ;
    constexpr int AX = Tl::AX, AY = Tl::AY, AZ = Tl::AZ;
    const ConfigDev &cf = *a.cf;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *smem = reinterpret_cast<T *>(smem_raw);
    __shared__ double slab_buf[NT];   // moving box: phi of the tile's cells
    SmemT<T> s;
    s.X = smem;            // [c][i + 3][j][k]  (float: [c / 2][i + 3][j][k][c % 2], arm_at)
    s.Y = s.X + 4 * AX;    // [c][i][j + 3][k]
    s.Z = s.Y + 4 * AY;    // [c][i][j][k + 3]
    s.F = s.Z + 4 * AZ;
    const int tid = threadIdx.x;
    const bool unit = cf.unit_speeds != 0;
    const bool all_axes[3] = {true, true, true};
    double cta_inv = 0.0;
    // tiles of all marching beams, back to back (one beam: its domain's tiles)
    const int total = MODE == MODE_RHS ? a.st[0].dom.ntiles : cf.tile_off[cf.nbeams];

    for (int gt = blockIdx.x; gt < total; gt += gridDim.x) {
        const int b = (MODE == MODE_RHS || cf.nbeams == 1) ? 0 : beam_of_tile(cf.tile_off, cf.nbeams, gt);
        const int tile = MODE == MODE_RHS ? gt : gt - cf.tile_off[b];
        const Coeffs &co = a.co[b];
        MarchState &stb = a.st[b];
        const BeamDev &bm = cf.beams[b];
        const DomainDev d = stb.dom;
        double *const Ua = stb.Ua;
        const int nx = d.nx, ny = d.ny, nz = d.nz;
        const size_t N = (size_t)nx * ny * nz;
        const size_t boff = (size_t)b * cf.cap;
        double *const U1 = a.U1 + 4 * boff;
        double *const U2 = a.U2 + 4 * boff;
        double *const Vb = a.V + 4 * boff;
        double *const qb = a.qpart + boff;
        const double *src = (MODE == MODE_B) ? U1 : (MODE == MODE_C ? U2 : Ua);
        const int tz = tile % d.tiles_z, ty = (tile / d.tiles_z) % d.tiles_y, tx = tile / (d.tiles_z * d.tiles_y);
        const int i0 = tx * TX, j0 = ty * TY, k0 = tz * TZ;

        // ---- 1. stage the stencil source + halo (the core into all three arms) ----
        for (int e = tid; e < SX; e += NT) {
            int k = e % TZ, j = (e / TZ) % TY, ii = e / (TZ * TY);
            double u[4];
            load_cell<MODE>(cf, co, d, src, i0 + ii - 3, j0 + j, k0 + k, u);
            const bool core = ii >= 3 && ii < TX + 3;
            const int ex = (ii * TY + j) * TZ + k;
            const int ey = ((ii - 3) * (TY + 6) + j + 3) * TZ + k;
            const int ez = ((ii - 3) * TY + j) * (TZ + 6) + k + 3;
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const T v = T(u[c]);
                arm_at(s.X, AX, c, ex) = v;
                if (core) {
                    arm_at(s.Y, AY, c, ey) = v;
                    arm_at(s.Z, AZ, c, ez) = v;
                }
            }
        }
        for (int e = tid; e < SY; e += NT) {
            int k = e % TZ, jj = (e / TZ) % 6, i = e / (TZ * 6);
            int gj = jj < 3 ? j0 + jj - 3 : j0 + TY + jj - 3;
            int aj = jj < 3 ? jj : TY + jj;   // arm index of local j = gj - j0
            double u[4];
            load_cell<MODE>(cf, co, d, src, i0 + i, gj, k0 + k, u);
#pragma unroll
            for (int c = 0; c < 4; ++c) arm_at(s.Y, AY, c, (i * (TY + 6) + aj) * TZ + k) = T(u[c]);
        }
        for (int e = tid; e < SZ; e += NT) {
            int kk = e % 6, j = (e / 6) % TY, i = e / (6 * TY);
            int gk = kk < 3 ? k0 + kk - 3 : k0 + TZ + kk - 3;
            int ak = kk < 3 ? kk : TZ + kk;
            if (gk < 0) continue;   // z-min ghost, filled below
            double u[4];
            load_cell<MODE>(cf, co, d, src, i0 + i, j0 + j, gk, u);
#pragma unroll
            for (int c = 0; c < 4; ++c) arm_at(s.Z, AZ, c, (i * TY + j) * (TZ + 6) + ak) = T(u[c]);
        }
        __syncthreads();
        // ---- 2. z-min ghost cells: quartic extrapolation through the inflow ----
        if (k0 == 0) {
            for (int e = tid; e < 4 * TX * TY; e += NT) {
                int j = e % TY, i = (e / TY) % TX, c = e / (TX * TY);
                int li = i0 + i, lj = j0 + j;
                if (li >= nx || lj >= ny) continue;
                T ui = T(boundary_value<MODE>(a, cf, bm, co, d, c, li, lj));
                const int ez = (i * TY + j) * (TZ + 6);
                auto z = [&](int kk) -> T & { return arm_at(s.Z, AZ, c, ez + kk); };
                T u0 = z(3), u1 = z(4), u2 = z(5), u3 = z(6);
                if (cf.spatial == PDM1_SPATIAL_WENO_Z) {   // quartic, boundary.py:247-320
                    z(2) = T(5.0) * ui - T(77.0 / 12.0) * u0 + T(43.0 / 12.0) * u1 - T(17.0 / 12.0) * u2 + T(0.25) * u3;
                    z(1) = T(25.0) * ui - T(505.0 / 12.0) * u0 + T(335.0 / 12.0) * u1 - T(145.0 / 12.0) * u2 + T(9.0 / 4.0) * u3;
                    z(0) = T(75.0) * ui - T(545.0 / 4.0) * u0 + T(395.0 / 4.0) * u1 - T(181.0 / 4.0) * u2 + T(35.0 / 4.0) * u3;
                } else if (cf.spatial == PDM1_SPATIAL_FIRST_ORDER) {   // boundary.py:205-212
                    z(2) = ui;
                } else {   // MUSCL / WENO3: quadratic, boundary.py:214-245
                    z(2) = T(3.0) * ui - T(2.5) * u0 + T(0.5) * u1;
                    z(1) = T(9.0) * ui - T(10.5) * u0 + T(2.5) * u1;
                }
            }
            __syncthreads();
        }
        // ---- 3. every face of the tile: WENO-Z, projection, HLL ----
        for (int f = tid; f < NF; f += NT) {
            int axis, i, j, k;
            if (f < NFX) {
                axis = 0; k = f % TZ; j = (f / TZ) % TY; i = f / (TZ * TY);
            } else if (f < NFX + NFY) {
                int u = f - NFX;
                axis = 1; k = u % TZ; j = (u / TZ) % (TY + 1); i = u / (TZ * (TY + 1));
            } else {
                int u = f - NFX - NFY;
                axis = 2; k = u % (TZ + 1); j = (u / (TZ + 1)) % TY; i = u / ((TZ + 1) * TY);
            }
            T L[4], R[4];
            // the six cells along the axis, i - 3 .. i + 2 (face between i - 1 and i),
            // are arm indices i .. i + 5
            T *arm;
            int e0, stride, cs;
            if (axis == 0) {
                arm = s.X; e0 = (i * TY + j) * TZ + k; stride = TY * TZ; cs = AX;
            } else if (axis == 1) {
                arm = s.Y; e0 = (i * (TY + 6) + j) * TZ + k; stride = TZ; cs = AY;
            } else {
                arm = s.Z; e0 = (i * TY + j) * (TZ + 6) + k; stride = 1; cs = AZ;
            }
            if (cf.spatial == PDM1_SPATIAL_WENO_Z) {
                if constexpr (sizeof(T) == sizeof(float)) {
                    // two components per packed reconstruction, L and R from the same loads
                    const float2 *b2 = reinterpret_cast<const float2 *>(arm) + e0;
#pragma unroll
                    for (int pc = 0; pc < 2; ++pc) {
                        float2 w[6];
#pragma unroll
                        for (int q = 0; q < 6; ++q) w[q] = b2[pc * cs + q * stride];
                        const float2 l = weno_left_f32x2(w[0], w[1], w[2], w[3], w[4]);
                        const float2 r = weno_left_f32x2(w[5], w[4], w[3], w[2], w[1]);
                        L[2 * pc] = l.x; L[2 * pc + 1] = l.y;
                        R[2 * pc] = r.x; R[2 * pc + 1] = r.y;
                    }
                } else {
                    const T *base = arm + e0;
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        T w[6];
#pragma unroll
                        for (int q = 0; q < 6; ++q) w[q] = base[c * cs + q * stride];
                        L[c] = weno_left(w[0], w[1], w[2], w[3], w[4]);
                        R[c] = weno_left(w[5], w[4], w[3], w[2], w[1]);
                    }
                }
            } else {
                // the narrower stencils read cells i-2 .. i+1 (arm indices i+1 .. i+4)
                for (int c = 0; c < 4; ++c) {
                    const T wm = arm_at(arm, cs, c, e0 + stride), w0 = arm_at(arm, cs, c, e0 + 2 * stride);
                    const T w1 = arm_at(arm, cs, c, e0 + 3 * stride), wp = arm_at(arm, cs, c, e0 + 4 * stride);
                    if (cf.spatial == PDM1_SPATIAL_FIRST_ORDER) {   // first_order.py:66-111
                        L[c] = w0;
                        R[c] = w1;
                    } else if (cf.spatial == PDM1_SPATIAL_MUSCL) {   // muscl.py:86-145
                        T lo, hi;
                        muscl_faces(wm, w0, w1, lo, hi);
                        L[c] = hi;
                        muscl_faces(w0, w1, wp, lo, hi);
                        R[c] = lo;
                    } else {   // WENO3, weno3.py:108-171
                        L[c] = weno3_left(wm, w0, w1);
                        R[c] = weno3_left(wp, w1, w0);
                    }
                }
            }
            T F[4];
            if constexpr (sizeof(T) == sizeof(float)) {
                face_flux_f32x2(L, R, axis, unit, F);
            } else {
                project(L[0], L[1], L[2], L[3]);
                project(R[0], R[1], R[2], R[3]);
                hll_flux(L, R, axis, unit, F);
            }
#pragma unroll
            for (int c = 0; c < 4; ++c) s.F[c * NF + f] = F[c];
        }
        __syncthreads();
        // ---- 4. divergence and the stage update, one cell per thread ----
        const int k = tid % TZ, j = (tid / TZ) % TY, i = tid / (TZ * TY);
        const int li = i0 + i, lj = j0 + j, lk = k0 + k;
        const bool valid = li < nx && lj < ny && lk < nz;
        double phi_new = -1.0;   // for the moving box's slab maxima
        double um[4] = {0.0, 0.0, 0.0, 0.0};   // the new state, for the learned box's moments
        if (valid) {
            const int fx0 = (i * TY + j) * TZ + k, fx1 = ((i + 1) * TY + j) * TZ + k;
            const int fy0 = NFX + (i * (TY + 1) + j) * TZ + k, fy1 = NFX + (i * (TY + 1) + j + 1) * TZ + k;
            const int fz0 = NFX + NFY + (i * TY + j) * (TZ + 1) + k, fz1 = fz0 + 1;
            double L[4];
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const T *F = s.F + c * NF;
                T gx = (F[fx1] - F[fx0]) / T(cf.dx);
                T gy = (F[fy1] - F[fy0]) / T(cf.dy);
                T gz = (F[fz1] - F[fz0]) / T(cf.dz);
                L[c] = double(-(gx + gy + gz));
            }
            const size_t o = ((size_t)li * ny + lj) * nz + lk;
            if (MODE == MODE_RHS) {
#pragma unroll
                for (int c = 0; c < 4; ++c) a.rhs_out[c * N + o] = L[c];
            } else {
                const size_t go = global_cell(cf, d, li, lj, lk);
                const int m = cf.ids[go];
                const double dE = co.dE;
                // the accepted state at this cell (with the Strang half step applied)
                double un[4];
                if ((MODE == MODE_A || MODE == MODE_EULER) && sizeof(T) == sizeof(double)) {
#pragma unroll
                    for (int c = 0; c < 4; ++c) un[c] = double(s.X[((c * (TX + 6) + (i + 3)) * TY + j) * TZ + k]);
                } else if (MODE == MODE_A || MODE == MODE_EULER) {
                    load_cell<MODE>(cf, co, d, Ua, li, lj, lk, un);   // the state in double
                } else {
                    load_cell<MODE_A>(cf, co, d, Ua, li, lj, lk, un);
                }
                const double s0 = co.S0[m];
                if (MODE == MODE_A) {
                    double u1[4], v1[4];
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        double v0 = s0 * un[c];
                        double v = L[c] * dE + v0;
                        v1[c] = v;
                        double w = v * (c == 0 ? co.c1p[m] : co.c1c[m]);
                        u1[c] = w / co.S1[m];
                    }
                    project(u1[0], u1[1], u1[2], u1[3]);
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        U1[c * N + o] = u1[c];
                        Vb[c * N + o] = v1[c];
                    }
                    double q0 = un[0] * s0, q1 = u1[0] * co.S1[m];
                    qb[o] = 1.0 / 6.0 * q0 + 1.0 / 6.0 * q1;
                } else if (MODE == MODE_B) {
                    double u2[4];
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        double r = L[c] * (c == 0 ? co.c1ip[m] : co.c1ic[m]);
                        r = (r * dE + Vb[c * N + o]) * 0.25;
                        double v = 0.75 * (s0 * un[c]) + r;
                        Vb[c * N + o] = v;
                        double w = v * (c == 0 ? co.c2p[m] : co.c2c[m]);
                        u2[c] = w / co.S2[m];
                    }
                    project(u2[0], u2[1], u2[2], u2[3]);
#pragma unroll
                    for (int c = 0; c < 4; ++c) U2[c * N + o] = u2[c];
                } else {
                    double unew[4];
                    double ed;
                    if (MODE == MODE_C) {
#pragma unroll
                        for (int c = 0; c < 4; ++c) {
                            double r = L[c] * (c == 0 ? co.c2ip[m] : co.c2ic[m]);
                            r = (r * dE + Vb[c * N + o]) * (2.0 / 3.0);
                            double v = 1.0 / 3.0 * (s0 * un[c]) + r;
                            double w = v * (c == 0 ? co.c1p[m] : co.c1c[m]);
                            unew[c] = w / co.S1[m];
                        }
                        project(unew[0], unew[1], unew[2], unew[3]);
                        double u2c = sizeof(T) == sizeof(double)
                                         ? double(s.X[((0 * (TX + 6) + (i + 3)) * TY + j) * TZ + k])
                                         : U2[o];
                        double q2 = u2c * co.S2[m];
                        ed = dE * (qb[o] + 2.0 / 3.0 * q2);
                    } else {   // forward Euler, numerics/energy.py:663-722
#pragma unroll
                        for (int c = 0; c < 4; ++c) {
                            double w = L[c] * dE + s0 * un[c];
                            unew[c] = w / co.S1[m];
                        }
                        project(unew[0], unew[1], unew[2], unew[3]);
                        ed = dE * un[0] * s0;
                    }
                    if (cf.strang) {
                        if (cf.nuclear)
#pragma unroll
                            for (int c = 0; c < 4; ++c) unew[c] *= co.hn[m];
                        if (cf.scattering != PDM1_SCATTERING_OFF)
#pragma unroll
                            for (int c = 1; c < 4; ++c) unew[c] *= co.hs[m];
                    }
                    if (MODE == MODE_C)
#pragma unroll
                        for (int c = 0; c < 4; ++c) um[c] = unew[c];
                    double *dst = MODE == MODE_C ? Ua : U1;
                    bool finite = true;
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        dst[c * N + o] = unew[c];
                        finite = finite && isfinite(unew[c]);
                    }
                    // a non-finite state ends the march with PDM1_ERR_NONFINITE
                    if (!finite) atomicOr(&stb.error, ERR_DEV_NONFINITE);
                    if (a.edep) a.edep[o] = ed;
                    else atomicAdd(&a.dose[go], ed * kMevToJoule / cf.mats[m].density);
                    if (MODE == MODE_C) {
                        if (co.snap_slot >= 0 && a.snap) {
                            const size_t NG = (size_t)cf.nx * cf.ny * cf.nz;
                            double *sn = a.snap + (size_t)co.snap_slot * 4 * NG;
#pragma unroll
                            for (int c = 0; c < 4; ++c) sn[c * NG + go] = unew[c];
                        }
                        if (!cf.moving) {
                            double phi_in = 0.0;
                            if (lk == 0 && d.inflow)
                                phi_in = bm.spatial[(size_t)(d.i0 + li) * cf.ny + (d.j0 + lj)] * co.ed_next;
                            double v = cfl_term<T>(cf, bm.rf, unew, co.S1[m], lk == 0, phi_in, all_axes);
                            cta_inv = fmax(cta_inv, v);
                        }
                        phi_new = unew[0];
                    }
                }
            }
        }
        if (MODE == MODE_C && cf.moving) {
            slab_buf[tid] = phi_new;
            __syncthreads();
            tile_slab_max(cf, beam_slab(cf, b), d, slab_buf, i0, j0, k0);
        }
        if constexpr (LEARN && MODE == MODE_C) {
            // learned box: the moments of the new state feed the next step's proposer
            __shared__ double mom_part[NT / 32][ACC_MAX + 1];
            __shared__ double mom_pl[kMaxTileZ];
            tile_moments_cta(cf, b, d, k0, valid, li, lj, lk, um, mom_part, mom_pl);
        }
        __syncthreads();   // shared memory is reused by the next tile
    }
    if (MODE == MODE_C && !cf.moving) block_max_atomic(cta_inv, &a.st[0].inv_bits);
}

}  // namespace pdm1
