// pdm1_stage.cuh -- the fused IF-SSPRK3 stage kernel, templated on the
// arithmetic of the stencil (WENO-Z, interface projection, HLL, divergence):
// double in pdm1_march.cu, float in pdm1_stage_fp32.cu.  The stage update,
// cell projection, CFL bound and dose stay in double in both.
#pragma once

#include "pdm1_device.cuh"

namespace pdm1 {

// Element e of component c's copy of an arm of asz elements.  Double arms are
// [c][e]; float arms hold a cell's four components together, [e][c] (one
// float4 per cell, the layout of the FP32 form's stage states in HBM), so a
// 128-bit load brings (phi, Jx) and (Jy, Jz) into two packed f32x2 pairs.
template <typename T>
__device__ __forceinline__ T &arm_at(T *arm, int asz, int c, int e) {
    if constexpr (sizeof(T) == sizeof(float)) return arm[e * 4 + c];
    else return arm[c * asz + e];
}

// The FP32 form keeps its stage states U1, U2 as one float4 (phi, Jx, Jy, Jz)
// per cell: stage A writes U1, stage B reads U1 and writes U2, stage C reads
// U2.  The stencil reads them in float in any case, so storing them rounded
// changes no result; the state itself (U^n, V) and the dose stay in double.
template <typename T, int MODE>
constexpr bool kF4Source = sizeof(T) == sizeof(float) && (MODE == MODE_B || MODE == MODE_C);
template <typename T, int MODE>
constexpr bool kF4Dest = sizeof(T) == sizeof(float) && (MODE == MODE_A || MODE == MODE_B);

// ---------------------------------------------------------------------------
// Bulk staging of a float4 tile (cp.async.bulk, the TMA engine's untiled
// copy, completed on a shared-memory mbarrier).  Every z row of every arm is
// one contiguous copy of 16-byte cells; rows outside the domain in x or y
// are the clamped rows (zero-gradient ghosts, numerics/boundary.py:327-397),
// rows are clipped to [0, nz) in z and the z-max ghosts patched afterwards.
// No multicast: each CTA copies from this GPU's own memory into its own
// shared memory.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
    asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(unsigned long long *bar) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(smem_u32(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}

// One row: `bytes` (a multiple of 16) from 16-byte aligned global memory to
// 16-byte aligned shared memory, counted on `bar`.
__device__ __forceinline__ void bulk_row(void *dst, const void *src, unsigned bytes, unsigned long long *bar) {
    mbar_expect_tx(bar, bytes);
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// Issue the rows of one tile (x arm with its x halo, y arm, z arm), each
// thread its share, then arrive once.  The x and y arms hold the tile's own
// z range k0 .. k0 + TZ - 1, the z arm k0 - 3 .. k0 + TZ + 2.
template <class Tl>
__device__ __forceinline__ void bulk_stage_tile(const float4 *src, const DomainDev &d, int i0, int j0, int k0,
                                                float4 *X, float4 *Y, float4 *Z, unsigned long long *bar) {
    constexpr int TX = Tl::TX, TY = Tl::TY, TZ = Tl::TZ;
    constexpr int RX = (TX + 6) * TY, RY = TX * (TY + 6), RZ = TX * TY;
    const int nx = d.nx, ny = d.ny, nz = d.nz;
    // shared memory read or written by the threads before (the last tile) is
    // overwritten by the async proxy next
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    for (int r = threadIdx.x; r < RX + RY + RZ; r += Tl::NT) {
        int li, lj, ka, kb, dst_e;
        float4 *arm;
        if (r < RX) {
            const int j = r % TY, ii = r / TY;
            li = i0 + ii - 3; lj = j0 + j; ka = k0; kb = k0 + TZ;
            arm = X; dst_e = (ii * TY + j) * TZ;
        } else if (r < RX + RY) {
            const int q = r - RX, jj = q % (TY + 6), i = q / (TY + 6);
            li = i0 + i; lj = j0 + jj - 3; ka = k0; kb = k0 + TZ;
            arm = Y; dst_e = (i * (TY + 6) + jj) * TZ;
        } else {
            const int q = r - RX - RY, j = q % TY, i = q / TY;
            li = i0 + i; lj = j0 + j; ka = k0 - 3; kb = k0 + TZ + 3;
            arm = Z; dst_e = (i * TY + j) * (TZ + 6);
        }
        li = li < 0 ? 0 : (li >= nx ? nx - 1 : li);
        lj = lj < 0 ? 0 : (lj >= ny ? ny - 1 : lj);
        const int k_lo = ka < 0 ? 0 : ka, k_hi = kb > nz ? nz : kb;
        if (k_hi > k_lo)
            bulk_row(arm + dst_e + (k_lo - ka), src + ((size_t)li * ny + lj) * nz + k_lo,
                     (unsigned)(k_hi - k_lo) * 16u, bar);
    }
    mbar_arrive(bar);
}

// Wait for the tile's rows; a wait past ~2^31 cycles (about a second) flags
// ERR_DEV_TIMEOUT and lets the march end with an error instead of hanging.
__device__ __forceinline__ void bulk_wait(unsigned long long *bar, unsigned parity, int *error) {
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > (1ll << 31)) {
            atomicOr(error, ERR_DEV_TIMEOUT);
            return;
        }
    }
}

// z-max ghosts of the z arm of a tile whose z range passes nz: the cells
// beyond hold the last cell's value (zero gradient).
template <class Tl>
__device__ __forceinline__ void patch_zmax(const DomainDev &d, int k0, float4 *Z) {
    constexpr int TX = Tl::TX, TY = Tl::TY, TZ = Tl::TZ;
    const int over = k0 + TZ + 3 - d.nz;   // cells of each z-arm row beyond nz
    if (over <= 0) return;
    const int last = d.nz - 1 - (k0 - 3);   // arm index of the domain's last z cell
    for (int e = threadIdx.x; e < TX * TY * over; e += Tl::NT) {
        const int row = e / over, kk = last + 1 + e % over;
        Z[row * (TZ + 6) + kk] = Z[row * (TZ + 6) + last];
    }
}

// LEARN (stage C of a plan with a learned box): the tile's fluence moments of
// the new state are accumulated for the next step's proposer.
template <typename T, int MODE, class Tl, bool LEARN = false>
__global__ void __launch_bounds__(Tl::NT, (sizeof(T) == sizeof(double) ? 2 : 4) * 256 / Tl::NT)
    stage_kernel(StageArgs a) {
    constexpr int NT = Tl::NT;   // threads of this tile shape (one cell each)
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
    // FP32 stages B and C: bulk copies of the float4 stage state, one mbarrier phase per tile
    __shared__ __align__(8) unsigned long long stage_bar;
    unsigned bar_phase = 0;
    if constexpr (kF4Source<T, MODE>) {
        if (cf.bulk_stage) {
            if (tid == 0) mbar_init(&stage_bar, NT);
            __syncthreads();
        }
    }
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
        if constexpr (kF4Source<T, MODE>) {
            // the float4 stage state: bulk copies, or (bulk_stage == 0) one
            // 128-bit load per cell; the arms receive the same values either way
            const float4 *src4 = reinterpret_cast<const float4 *>(src);
            float4 *X4 = reinterpret_cast<float4 *>(s.X), *Y4 = reinterpret_cast<float4 *>(s.Y);
            float4 *Z4 = reinterpret_cast<float4 *>(s.Z);
            if (cf.bulk_stage) {
                bulk_stage_tile<Tl>(src4, d, i0, j0, k0, X4, Y4, Z4, &stage_bar);
                bulk_wait(&stage_bar, bar_phase, &stb.error);
                bar_phase ^= 1u;
                patch_zmax<Tl>(d, k0, Z4);
            } else {
                auto cell = [&](int li, int lj, int lk) {
                    li = li < 0 ? 0 : (li >= nx ? nx - 1 : li);
                    lj = lj < 0 ? 0 : (lj >= ny ? ny - 1 : lj);
                    lk = lk >= nz ? nz - 1 : lk;
                    return src4[((size_t)li * ny + lj) * nz + lk];
                };
                for (int e = tid; e < SX; e += NT) {
                    const int k = e % TZ, j = (e / TZ) % TY, ii = e / (TZ * TY);
                    const float4 v = cell(i0 + ii - 3, j0 + j, k0 + k);
                    X4[(ii * TY + j) * TZ + k] = v;
                    if (ii >= 3 && ii < TX + 3) {
                        Y4[((ii - 3) * (TY + 6) + j + 3) * TZ + k] = v;
                        Z4[((ii - 3) * TY + j) * (TZ + 6) + k + 3] = v;
                    }
                }
                for (int e = tid; e < SY; e += NT) {
                    const int k = e % TZ, jj = (e / TZ) % 6, i = e / (TZ * 6);
                    const int gj = jj < 3 ? j0 + jj - 3 : j0 + TY + jj - 3;
                    const int aj = jj < 3 ? jj : TY + jj;
                    Y4[(i * (TY + 6) + aj) * TZ + k] = cell(i0 + i, gj, k0 + k);
                }
                for (int e = tid; e < SZ; e += NT) {
                    const int kk = e % 6, j = (e / 6) % TY, i = e / (6 * TY);
                    const int gk = kk < 3 ? k0 + kk - 3 : k0 + TZ + kk - 3;
                    const int ak = kk < 3 ? kk : TZ + kk;
                    if (gk < 0) continue;   // z-min ghost, filled below
                    Z4[(i * TY + j) * (TZ + 6) + ak] = cell(i0 + i, j0 + j, gk);
                }
            }
        } else {
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
        }   // the double-precision source
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
                    // two components per packed reconstruction, L and R from the
                    // same six 128-bit loads: (phi, Jx) and (Jy, Jz) of each cell
                    const float4 *b4 = reinterpret_cast<const float4 *>(arm) + e0;
                    float2 w01[6], w23[6];
#pragma unroll
                    for (int q = 0; q < 6; ++q) {
                        const float4 v = b4[q * stride];
                        w01[q] = make_float2(v.x, v.y);
                        w23[q] = make_float2(v.z, v.w);
                    }
                    float2 l = weno_left_f32x2(w01[0], w01[1], w01[2], w01[3], w01[4]);
                    float2 r = weno_left_f32x2(w01[5], w01[4], w01[3], w01[2], w01[1]);
                    L[0] = l.x; L[1] = l.y; R[0] = r.x; R[1] = r.y;
                    l = weno_left_f32x2(w23[0], w23[1], w23[2], w23[3], w23[4]);
                    r = weno_left_f32x2(w23[5], w23[4], w23[3], w23[2], w23[1]);
                    L[2] = l.x; L[3] = l.y; R[2] = r.x; R[3] = r.y;
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
                    if constexpr (kF4Dest<T, MODE>)
                        reinterpret_cast<float4 *>(U1)[o] = make_float4(float(u1[0]), float(u1[1]), float(u1[2]),
                                                                        float(u1[3]));
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        if constexpr (!kF4Dest<T, MODE>) U1[c * N + o] = u1[c];
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
                    if constexpr (kF4Dest<T, MODE>) {
                        reinterpret_cast<float4 *>(U2)[o] = make_float4(float(u2[0]), float(u2[1]), float(u2[2]),
                                                                        float(u2[3]));
                        // the dose quadrature's stage-2 term, from the double state
                        // (stage C reads the sum; the same sum, rounded as it would be there)
                        double q2 = u2[0] * co.S2[m];
                        qb[o] = qb[o] + 2.0 / 3.0 * q2;
                    } else {
#pragma unroll
                        for (int c = 0; c < 4; ++c) U2[c * N + o] = u2[c];
                    }
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
                        if constexpr (sizeof(T) == sizeof(double)) {
                            double u2c = double(s.X[((0 * (TX + 6) + (i + 3)) * TY + j) * TZ + k]);
                            double q2 = u2c * co.S2[m];
                            ed = dE * (qb[o] + 2.0 / 3.0 * q2);
                        } else {
                            ed = dE * qb[o];   // stage B added 2/3 q2
                        }
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
            tile_moments_cta<NT>(cf, b, d, k0, valid, li, lj, lk, um, mom_part, mom_pl);
        }
        __syncthreads();   // shared memory is reused by the next tile
    }
    if (MODE == MODE_C && !cf.moving) block_max_atomic<NT>(cta_inv, &a.st[0].inv_bits);
}

}  // namespace pdm1
