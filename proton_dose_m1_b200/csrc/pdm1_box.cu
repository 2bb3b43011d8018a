// pdm1_box.cu -- the learned moving active box.
//
// A small MLP (16 -> 64 -> 64 -> 6, ReLU) proposes, for every beam at every
// energy step, how many cells the moving box extends beyond the significant
// box on each of its six faces.  This file holds
//   * the fused training kernel (forward, loss and backward of a chunk of
//     samples in one CTA, FP32) and the Adam update, driven by pdm1_mlp_train;
//   * the inference: BF16 operands on the tensor cores (mma.sync m16n8k16,
//     FP32 accumulation), one warp per 16 beams;
//   * the per-step kernels of the learned box and of the training-data
//     recorder (fluence moments of each beam's box, features, margins, the
//     outgoing-flux check).
// The reference has no learned box: its moving box is the fixed heuristic of
// proton_solver/numerics/moving_active_domain.py:107-193 (significant box plus
// a guard of active_guard_cells on every face), which the box kernel in
// pdm1_march.cu reproduces and which this file replaces when a plan holds a
// box model.
#include "../../include/pdm1.h"
#include "pdm1_device.cuh"

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <string>
#include <vector>

namespace pdm1 {

__device__ void mlp_warp16(const BoxModelDev &M, const __nv_bfloat16 *x, __nv_bfloat16 *h, float *out);

namespace {

constexpr int kRows = 64;   // samples per CTA of the training kernel
constexpr int kTrainThreads = 256;
constexpr size_t kTrainSmem =
    sizeof(float) * (kParams + kRows * kFeat + 4 * kRows * kHid + kRows * kOut + kTrainThreads);

#define CUDA_OK(expr)                                                              \
    do {                                                                           \
        cudaError_t e_ = (expr);                                                   \
        if (e_ != cudaSuccess) {                                                   \
            std::string m_ = std::string(#expr ": ") + cudaGetErrorString(e_);     \
            return report_error(PDM1_ERR_CUDA, m_.c_str());                        \
        }                                                                          \
    } while (0)

// Fused training step of one chunk of kRows samples: forward, weighted
// squared loss, backward; the chunk's gradient is added to `grad`.
// theta = W1 (64x16), b1, W2 (64x64), b2, W3 (6x64), b3, rows [out][in].
__global__ void __launch_bounds__(kTrainThreads) mlp_grad_kernel(const float *theta, const float *X,
                                                                 const float *Y, const int *idx, int n_batch,
                                                                 float inv_norm, float alpha, float *grad,
                                                                 float *loss) {
    extern __shared__ float sm[];
    float *P = sm;
    float *x = P + kParams;
    float *h1 = x + kRows * kFeat;
    float *h2 = h1 + kRows * kHid;
    float *d2 = h2 + kRows * kHid;
    float *d1 = d2 + kRows * kHid;
    float *dy = d1 + kRows * kHid;
    float *red = dy + kRows * kOut;
    const int tid = threadIdx.x;
    const int r0 = blockIdx.x * kRows;
    const int nr = min(kRows, n_batch - r0);
    for (int e = tid; e < kParams; e += kTrainThreads) P[e] = theta[e];
    for (int e = tid; e < kRows * kFeat; e += kTrainThreads) {
        int r = e / kFeat, k = e % kFeat;
        x[e] = r < nr ? X[(size_t)idx[r0 + r] * kFeat + k] : 0.f;
    }
    __syncthreads();
    const float *W1 = P, *b1 = W1 + kHid * kFeat, *W2 = b1 + kHid, *b2 = W2 + kHid * kHid;
    const float *W3 = b2 + kHid, *b3 = W3 + kOut * kHid;
    float *gW1 = grad, *gb1 = gW1 + kHid * kFeat, *gW2 = gb1 + kHid, *gb2 = gW2 + kHid * kHid;
    float *gW3 = gb2 + kHid, *gb3 = gW3 + kOut * kHid;
    for (int e = tid; e < kRows * kHid; e += kTrainThreads) {
        int r = e / kHid, n = e % kHid;
        float a = b1[n];
        for (int k = 0; k < kFeat; ++k) a += W1[n * kFeat + k] * x[r * kFeat + k];
        h1[e] = a > 0.f ? a : 0.f;
    }
    __syncthreads();
    for (int e = tid; e < kRows * kHid; e += kTrainThreads) {
        int r = e / kHid, n = e % kHid;
        float a = b2[n];
        for (int k = 0; k < kHid; ++k) a += W2[n * kHid + k] * h1[r * kHid + k];
        h2[e] = a > 0.f ? a : 0.f;
    }
    __syncthreads();
    float lsum = 0.f;
    for (int e = tid; e < kRows * kOut; e += kTrainThreads) {
        int r = e / kOut, o = e % kOut;
        float g = 0.f;
        if (r < nr) {
            float a = b3[o];
            for (int k = 0; k < kHid; ++k) a += W3[o * kHid + k] * h2[r * kHid + k];
            float res = a - Y[(size_t)idx[r0 + r] * kOut + o];
            float w = res < 0.f ? alpha : 1.f;
            lsum += w * res * res;
            g = 2.f * w * res * inv_norm;
        }
        dy[e] = g;
    }
    red[tid] = lsum;
    __syncthreads();
    for (int w = kTrainThreads / 2; w > 0; w >>= 1) {
        if (tid < w) red[tid] += red[tid + w];
        __syncthreads();
    }
    if (tid == 0 && loss) atomicAdd(loss, red[0] * inv_norm);
    // output layer
    for (int e = tid; e < kOut * kHid + kOut; e += kTrainThreads) {
        float s = 0.f;
        if (e < kOut * kHid) {
            int o = e / kHid, k = e % kHid;
            for (int r = 0; r < kRows; ++r) s += dy[r * kOut + o] * h2[r * kHid + k];
            atomicAdd(&gW3[e], s);
        } else {
            int o = e - kOut * kHid;
            for (int r = 0; r < kRows; ++r) s += dy[r * kOut + o];
            atomicAdd(&gb3[o], s);
        }
    }
    for (int e = tid; e < kRows * kHid; e += kTrainThreads) {
        int r = e / kHid, k = e % kHid;
        float s = 0.f;
        for (int o = 0; o < kOut; ++o) s += dy[r * kOut + o] * W3[o * kHid + k];
        d2[e] = h2[e] > 0.f ? s : 0.f;
    }
    __syncthreads();
    // second layer
    for (int e = tid; e < kHid * kHid + kHid; e += kTrainThreads) {
        float s = 0.f;
        if (e < kHid * kHid) {
            int n = e / kHid, k = e % kHid;
            for (int r = 0; r < kRows; ++r) s += d2[r * kHid + n] * h1[r * kHid + k];
            atomicAdd(&gW2[e], s);
        } else {
            int n = e - kHid * kHid;
            for (int r = 0; r < kRows; ++r) s += d2[r * kHid + n];
            atomicAdd(&gb2[n], s);
        }
    }
    for (int e = tid; e < kRows * kHid; e += kTrainThreads) {
        int r = e / kHid, k = e % kHid;
        float s = 0.f;
        for (int n = 0; n < kHid; ++n) s += d2[r * kHid + n] * W2[n * kHid + k];
        d1[e] = h1[e] > 0.f ? s : 0.f;
    }
    __syncthreads();
    // first layer
    for (int e = tid; e < kHid * kFeat + kHid; e += kTrainThreads) {
        float s = 0.f;
        if (e < kHid * kFeat) {
            int n = e / kFeat, k = e % kFeat;
            for (int r = 0; r < kRows; ++r) s += d1[r * kHid + n] * x[r * kFeat + k];
            atomicAdd(&gW1[e], s);
        } else {
            int n = e - kHid * kFeat;
            for (int r = 0; r < kRows; ++r) s += d1[r * kHid + n];
            atomicAdd(&gb1[n], s);
        }
    }
}

// Adam (Kingma & Ba 2015) on the flat parameter vector; clears the gradient.
__global__ void mlp_adam_kernel(float *theta, float *m, float *v, float *grad, int n, float lr, float beta1,
                                float beta2, float eps, float c1, float c2) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float g = grad[i];
    float mi = beta1 * m[i] + (1.f - beta1) * g;
    float vi = beta2 * v[i] + (1.f - beta2) * g * g;
    m[i] = mi;
    v[i] = vi;
    theta[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    grad[i] = 0.f;
}

// Plain FP32 forward, one thread per sample (tests and host-side evaluation).
__global__ void mlp_forward_kernel(const float *theta, const float *X, int n, float *Y) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const float *W1 = theta, *b1 = W1 + kHid * kFeat, *W2 = b1 + kHid, *b2 = W2 + kHid * kHid;
    const float *W3 = b2 + kHid, *b3 = W3 + kOut * kHid;
    float h1[kHid], h2[kHid];
    for (int j = 0; j < kHid; ++j) {
        float a = b1[j];
        for (int k = 0; k < kFeat; ++k) a += W1[j * kFeat + k] * X[(size_t)s * kFeat + k];
        h1[j] = a > 0.f ? a : 0.f;
    }
    for (int j = 0; j < kHid; ++j) {
        float a = b2[j];
        for (int k = 0; k < kHid; ++k) a += W2[j * kHid + k] * h1[k];
        h2[j] = a > 0.f ? a : 0.f;
    }
    for (int o = 0; o < kOut; ++o) {
        float a = b3[o];
        for (int k = 0; k < kHid; ++k) a += W3[o * kHid + k] * h2[k];
        Y[(size_t)s * kOut + o] = a;
    }
}

__global__ void infer_kernel(const BoxModelDev *model, const float *X, int n, float *Y) {
    __shared__ __align__(16) __nv_bfloat16 xs[4][16 * kFeat];
    __shared__ __align__(16) __nv_bfloat16 hs[4][16 * kHid];
    __shared__ float os[4][16 * kOutPad];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int base = (blockIdx.x * 4 + warp) * 16;
    const BoxModelDev &M = *model;
    for (int e = lane; e < 16 * kFeat; e += 32) {
        int r = e / kFeat, k = e % kFeat;
        float v = base + r < n ? (X[(size_t)(base + r) * kFeat + k] - M.x_mean[k]) * M.x_inv_std[k] : 0.f;
        xs[warp][e] = __float2bfloat16_rn(v);
    }
    __syncwarp();
    mlp_warp16(M, xs[warp], hs[warp], os[warp]);
    for (int e = lane; e < 16 * kOut; e += 32) {
        int r = e / kOut, o = e % kOut;
        if (base + r < n) Y[(size_t)(base + r) * kOut + o] = os[warp][r * kOutPad + o];
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// BF16 tensor-core inference of 16 rows by one warp
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t ld_pair(const __nv_bfloat16 *p) {
    return *reinterpret_cast<const uint32_t *>(p);
}

__device__ __forceinline__ void st_pair(__nv_bfloat16 *p, float lo, float hi) {
    *reinterpret_cast<__nv_bfloat162 *>(p) = __floats2bfloat162_rn(lo, hi);
}

// D += A (16x16, row-major) * B (16x8, column-major), BF16 in, FP32 accumulate.
__device__ __forceinline__ void mma_16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// A fragment of rows [0,16) x columns [c0, c0+16) of a row-major bf16 matrix
// with `ld` columns: lane (g = lane/4, t = lane%4) holds (g, c0+2t..+1),
// (g+8, c0+2t..+1), (g, c0+2t+8..+9), (g+8, c0+2t+8..+9).
__device__ __forceinline__ void load_a(uint32_t (&a)[4], const __nv_bfloat16 *m, int ld, int c0, int g, int t) {
    a[0] = ld_pair(m + g * ld + c0 + 2 * t);
    a[1] = ld_pair(m + (g + 8) * ld + c0 + 2 * t);
    a[2] = ld_pair(m + g * ld + c0 + 2 * t + 8);
    a[3] = ld_pair(m + (g + 8) * ld + c0 + 2 * t + 8);
}

__device__ void mlp_warp16(const BoxModelDev &M, const __nv_bfloat16 *x, __nv_bfloat16 *h, float *out) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    uint32_t a[4];
    float acc[8][4];
    // layer 1: (16 x 16) . W1^T -> 16 x 64
    load_a(a, x, kFeat, 0, g, t);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
        const __nv_bfloat16 *w = M.W1 + (8 * j + g) * kFeat + 2 * t;
        mma_16816(acc[j], a, ld_pair(w), ld_pair(w + 8));
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        int c = 8 * j + 2 * t;
        st_pair(h + g * kHid + c, fmaxf(acc[j][0] + M.b1[c], 0.f), fmaxf(acc[j][1] + M.b1[c + 1], 0.f));
        st_pair(h + (g + 8) * kHid + c, fmaxf(acc[j][2] + M.b1[c], 0.f), fmaxf(acc[j][3] + M.b1[c + 1], 0.f));
    }
    __syncwarp();
    // layer 2: (16 x 64) . W2^T -> 16 x 64
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
        load_a(a, h, kHid, 16 * kk, g, t);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const __nv_bfloat16 *w = M.W2 + (8 * j + g) * kHid + 16 * kk + 2 * t;
            mma_16816(acc[j], a, ld_pair(w), ld_pair(w + 8));
        }
    }
    __syncwarp();
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        int c = 8 * j + 2 * t;
        st_pair(h + g * kHid + c, fmaxf(acc[j][0] + M.b2[c], 0.f), fmaxf(acc[j][1] + M.b2[c + 1], 0.f));
        st_pair(h + (g + 8) * kHid + c, fmaxf(acc[j][2] + M.b2[c], 0.f), fmaxf(acc[j][3] + M.b2[c + 1], 0.f));
    }
    __syncwarp();
    // layer 3: (16 x 64) . W3^T -> 16 x 8 (outputs 6, 7 are zero padding)
    float o[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
        load_a(a, h, kHid, 16 * kk, g, t);
        const __nv_bfloat16 *w = M.W3 + g * kHid + 16 * kk + 2 * t;
        mma_16816(o, a, ld_pair(w), ld_pair(w + 8));
    }
    int c = 2 * t;
    out[g * kOutPad + c] = o[0] + M.b3[c];
    out[g * kOutPad + c + 1] = o[1] + M.b3[c + 1];
    out[(g + 8) * kOutPad + c] = o[2] + M.b3[c];
    out[(g + 8) * kOutPad + c + 1] = o[3] + M.b3[c + 1];
    __syncwarp();
}

// ---------------------------------------------------------------------------
// Per-step kernels of the learned box and of the recorder
// ---------------------------------------------------------------------------

// Fluence moments, face currents and z-plane currents of every marching
// beam's box (state at the start of the step, i.e. after the last stage C),
// accumulated into the beam's acc / plane; `record` (one-beam full-domain
// plans) also reduces the slab maxima the significant box is taken from.
__global__ void __launch_bounds__(NT) box_moments_kernel(const ConfigDev *cfp, const MarchState *sts, int record) {
    const ConfigDev &cf = *cfp;
    __shared__ double part[NT / 32][ACC_MAX + 1];
    __shared__ double pl[kMaxTileZ];
    __shared__ double buf[NT];
    const int tid = threadIdx.x;
    const int total = record ? sts[0].dom.ntiles : cf.tile_off[cf.nbeams];
    for (int gt = blockIdx.x; gt < total; gt += gridDim.x) {
        const int b = (record || cf.nbeams == 1) ? 0 : beam_of_tile(cf.tile_off, cf.nbeams, gt);
        const int tile = record ? gt : gt - cf.tile_off[b];
        const MarchState &st = sts[b];
        const DomainDev d = st.dom;
        if (tile >= d.ntiles) continue;   // same for the whole CTA
        const int TX = d.tx, TY = d.ty, TZ = d.tz;
        const int tz = tile % d.tiles_z, ty = (tile / d.tiles_z) % d.tiles_y, tx = tile / (d.tiles_z * d.tiles_y);
        const int i0 = tx * TX, j0 = ty * TY, k0 = tz * TZ;
        const int ii = tid / (TY * TZ), jj = (tid / TZ) % TY, kk = tid % TZ;
        const int li = i0 + ii, lj = j0 + jj, lk = k0 + kk;
        const bool valid = li < d.nx && lj < d.ny && lk < d.nz;
        double u[4] = {0.0, 0.0, 0.0, 0.0};
        if (valid) {
            const size_t N = (size_t)d.nx * d.ny * d.nz, o = ((size_t)li * d.ny + lj) * d.nz + lk;
#pragma unroll
            for (int c = 0; c < 4; ++c) u[c] = st.Ua[c * N + o];
        }
        if (record) {
            buf[tid] = valid ? u[0] : 0.0;
            __syncthreads();
            tile_slab_max(cf, cf.slab, d, buf, i0, j0, k0);
        }
        tile_moments_cta(cf, b, d, k0, valid, li, lj, lk, u, part, pl);
    }
}

// Largest z-plane current density over the planes [k_lo, k_hi), by one warp
// (every lane returns it).
__device__ __forceinline__ double plane_max_warp(const double *plane, int k_lo, int k_hi, int lane) {
    double m = 0.0;
    for (int k = k_lo + lane; k < k_hi; k += 32) m = fmax(m, plane[k]);
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    return m;
}

// Features of a beam's state (one thread): energy, last dE, the significant
// box, and the fluence moments relative to it.  Returns false when the box
// holds no fluence.  plane_max: the largest z-plane current density of the
// box (plane_max_warp); *current receives it as a current (particles per
// MeV).  S_E: the stopping power of material 0 at E when known, else <= 0.
__device__ bool box_features(const ConfigDev &cf, const double *acc, double plane_max, const int sig[6], double E,
                             double dE, double S_E, float *f, double *current) {
    const double I = plane_max * (cf.dx * cf.dy);
    *current = I;
    const double M = acc[ACC_M];
    for (int q = 0; q < kFeat; ++q) f[q] = 0.f;
    if (!(M > 0.0) || sig[1] < 0) return false;
    double S = S_E;
    if (!(S > 0.0) && (!stopping_power_dev(cf.mats[0], E, S) || !(S > 0.0))) S = 1.0;
    f[0] = (float)(E / 100.0);
    f[1] = (float)(dE / cf.max_dE);
    for (int a = 0; a < 3; ++a) {
        const double lo = sig[2 * a], hi = sig[2 * a + 1];
        const double mean = acc[ACC_X + a] / M;
        const double var = fmax(acc[ACC_X2 + a] / M - mean * mean, 0.0);
        f[2 + a] = (float)(0.5 * (hi - lo));
        f[5 + a] = (float)(mean - 0.5 * (lo + hi));
        f[8 + a] = (float)sqrt(var);
    }
    f[11] = (float)(acc[ACC_J + 2] / M);
    f[12] = (float)(acc[ACC_JABS] / M);
    f[13] = (float)(acc[ACC_JABS + 1] / M);
    f[14] = (float)(dE / (S * cf.dz));
    f[15] = (float)(I / (M * cf.dx * cf.dy * cf.dz) * cf.dz);
    return true;
}

// Learned box: features of every beam, the proposer network on the tensor
// cores (one warp per 16 beams), the outgoing-flux check, the new box.
__global__ void __launch_bounds__(128) box_learn_kernel(const ConfigDev *cfp, Coeffs *cos, MarchState *sts) {
    const ConfigDev &cf = *cfp;
    const BoxModelDev &M = *cf.model;
    __shared__ __align__(16) __nv_bfloat16 xs[4][16 * kFeat];
    __shared__ __align__(16) __nv_bfloat16 hs[4][16 * kHid];
    __shared__ float os[4][16 * kOutPad];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int b0 = (blockIdx.x * 4 + warp) * 16, b = b0 + lane;
    const bool mine = lane < 16 && b < cf.nbeams;
    MarchState *st = mine ? sts + b : nullptr;
    const bool live = mine && !(st->done || st->error);
    // the z-plane current maxima of the warp's beams, all 32 lanes per beam;
    // each lane clears the planes it read for the next step's moments
    double pmax = 0.0;
    for (int q = 0; q < 16 && b0 + q < cf.nbeams; ++q) {
        const MarchState &sq = sts[b0 + q];
        if (sq.done || sq.error) continue;   // the same for every lane
        double *pq = cf.plane + (size_t)(b0 + q) * cf.nz;
        const int k_lo = sq.dom.k0, k_hi = sq.dom.k0 + sq.dom.nz;
        const double v = plane_max_warp(pq, k_lo, k_hi, lane);
        for (int k = k_lo + lane; k < k_hi; k += 32) pq[k] = 0.0;
        if (lane == q) pmax = v;
    }
    float f[kFeat];
    double current = 0.0;
    bool valid = false;
    if (live) {
        const double *acc = cf.acc + (size_t)b * kAcc;
        // prologue_kernel left S1 = S(E_next) with E_next the energy of this step
        const double S_E = cos[b].E_next == st->E ? cos[b].S1[0] : 0.0;
        valid = box_features(cf, acc, pmax, st->sig, st->E, cos[b].dE, S_E, f, &current);
    } else {
        for (int q = 0; q < kFeat; ++q) f[q] = 0.f;
    }
    if (lane < 16)
        for (int q = 0; q < kFeat; ++q)
            xs[warp][lane * kFeat + q] = __float2bfloat16_rn(valid ? (f[q] - M.x_mean[q]) * M.x_inv_std[q] : 0.f);
    __syncwarp();
    mlp_warp16(M, xs[warp], hs[warp], os[warp]);
    if (!live) return;
    const BeamDev &bm = cf.beams[b];
    Coeffs *co = cos + b;
    const double ed = co->E_next == st->E ? co->ed_next : energy_density(bm, st->E);
    double *acc = cf.acc + (size_t)b * kAcc;
    DomainDev nb;
    if (st->sig[1] < 0) {
        nb = bm.init_box;
    } else {
        // outgoing-flux check on the box just marched
        const double area[6] = {cf.dy * cf.dz, cf.dy * cf.dz, cf.dx * cf.dz, cf.dx * cf.dz, cf.dx * cf.dy, cf.dx * cf.dy};
        if (current > 0.0)
            for (int q = 0; q < 6; ++q)
                if (acc[ACC_FACE + q] * area[q] > M.leak_tol * current) {
                    st->extra[q] += M.grow_cells;
                    st->grows += 1;
                    if (st->extra[q] > M.extra_max && st->fallback == 0)
                        st->fallback = (size_t)cf.nx * cf.ny * cf.nz <= cf.cap ? 1 : 2;
                }
        int m[6];
        for (int q = 0; q < 6; ++q) {
            int mq = cf.guard;
            if (st->fallback == 0 && valid) {
                float y = os[warp][lane * kOutPad + q] * M.y_scale[q] + M.y_offset[q];
                y = fminf(fmaxf(y, (float)M.margin_min), (float)M.margin_max);
                mq = (int)ceilf(y);
            }
            m[q] = mq + (st->fallback == 2 ? 0 : st->extra[q]);
            st->margin[q] = m[q];
        }
        if (st->fallback == 1) {
            nb = make_domain(0, 0, 0, cf.nx, cf.ny, cf.nz, 1, cf.tile);
        } else {
            int bi0 = max(st->sig[0] - m[0], 0), bi1 = min(st->sig[1] + m[1], cf.nx);
            int bj0 = max(st->sig[2] - m[2], 0), bj1 = min(st->sig[3] + m[3], cf.ny);
            int bk0 = max(st->sig[4] - m[4], 0), bk1 = min(st->sig[5] + m[5], cf.nz);
            nb = make_domain(bi0, bj0, bk0, bi1 - bi0, bj1 - bj0, bk1 - bk0, bk0 == 0, cf.tile);
        }
    }
    for (int q = 0; q < kAcc; ++q) acc[q] = 0.0;
    switch_box(cf, bm, co, st, b, nb, ed);
}

// Recorder (one-beam full-domain plans): after every step, the significant
// box and the features of the new state, one row per step.
__global__ void __launch_bounds__(256) record_kernel(const ConfigDev *cfp, const Coeffs *cos, MarchState *sts) {
    const ConfigDev &cf = *cfp;
    const Coeffs *co = cos;
    MarchState *st = sts;
    const BeamDev &bm = cf.beams[0];
    __shared__ double red[512];   // significant_box_cta: two reductions
    __shared__ double s_scale, s_scale2;
    __shared__ int s_lo[3], s_hi[3], s_lo2[2][3], s_hi2[2][3];
    const int t = threadIdx.x;
    const bool take = co->active != 0;   // uniform: a step ran in this slot
    double *acc = cf.acc;
    unsigned long long *slab = beam_slab(cf, 0);
    if (take) {
        const DomainDev d = st->dom;
        const double ed = energy_density(bm, st->E);
        significant_box_cta(cf, bm, d, slab, ed, red, s_lo, s_hi, &s_scale, cf.tol);
        significant_box_cta(cf, bm, d, slab, ed, red, s_lo2[0], s_hi2[0], &s_scale2, cf.rec_tail_tol[0]);
        significant_box_cta(cf, bm, d, slab, ed, red, s_lo2[1], s_hi2[1], &s_scale2, cf.rec_tail_tol[1]);
        const double pmax = t < 32 ? plane_max_warp(cf.plane, 0, cf.nz, t) : 0.0;
        if (t == 0) {
            const int row = st->step - 1;
            const bool none = s_scale == 0.0 || s_hi[0] < 0 || s_hi[1] < 0 || s_hi[2] < 0;
            int sig[6], tail[2][6];
            for (int a = 0; a < 3; ++a) {
                const int o = a == 0 ? d.i0 : a == 1 ? d.j0 : d.k0;
                sig[2 * a] = none ? -1 : o + s_lo[a];
                sig[2 * a + 1] = none ? -1 : o + s_hi[a] + 1;
                for (int l = 0; l < 2; ++l) {
                    const bool none2 = none || s_hi2[l][0] < 0 || s_hi2[l][1] < 0 || s_hi2[l][2] < 0;
                    tail[l][2 * a] = none2 ? -1 : o + s_lo2[l][a];
                    tail[l][2 * a + 1] = none2 ? -1 : o + s_hi2[l][a] + 1;
                }
            }
            float f[kFeat];
            double current = 0.0;
            box_features(cf, acc, pmax, sig, st->E, co->dE, 0.0, f, &current);
            if (cf.rec && row >= 0 && row < cf.rec_max) {
                float *r = cf.rec + (size_t)row * PDM1_RECORD_WIDTH;
                r[0] = (float)st->E;
                r[1] = (float)co->dE;
                for (int q = 0; q < 6; ++q) r[2 + q] = (float)sig[q];
                for (int q = 0; q < kFeat; ++q) r[8 + q] = f[q];
                r[24] = (float)acc[ACC_M];
                r[25] = (float)current;
                r[26] = (float)s_scale;
                for (int q = 0; q < 6; ++q) r[27 + q] = (float)tail[0][q];
                for (int q = 0; q < 6; ++q) r[33 + q] = (float)tail[1][q];
                r[39] = 0.f;
            }
        }
        __syncthreads();
    }
    for (int q = t; q < kAcc; q += 256) acc[q] = 0.0;
    for (int k = t; k < cf.nz; k += 256) cf.plane[k] = 0.0;
    for (int e = t; e < cf.nx + cf.ny + cf.nz; e += 256) slab[e] = 0ull;
}

void launch_box_moments(const ConfigDev *d_cf, const MarchState *d_st, int grid, int record, cudaStream_t stream) {
    box_moments_kernel<<<grid, NT, 0, stream>>>(d_cf, d_st, record);
}

void launch_box_learn(const ConfigDev *d_cf, Coeffs *d_co, MarchState *d_st, int nbeams, cudaStream_t stream) {
    box_learn_kernel<<<(nbeams + 63) / 64, 128, 0, stream>>>(d_cf, d_co, d_st);
}

void launch_record(const ConfigDev *d_cf, const Coeffs *d_co, MarchState *d_st, cudaStream_t stream) {
    record_kernel<<<1, 256, 0, stream>>>(d_cf, d_co, d_st);
}

// Host: the device form of a box model (BF16 weights, FP32 biases and
// normalisation).
int pack_box_model(const pdm1_box_model *m, BoxModelDev &out) {
    if (!m || !m->params) return report_error(PDM1_ERR_ARGUMENT, "box model without parameters");
    if (m->margin_min < 0 || m->margin_max < m->margin_min || m->grow_cells < 1 || m->extra_max < 0 ||
        !(m->leak_tolerance > 0.0))
        return report_error(PDM1_ERR_ARGUMENT, "box model: invalid margin, growth or leak settings");
    std::memset(&out, 0, sizeof out);
    const float *p = m->params;
    const float *W1 = p, *b1 = W1 + kHid * kFeat, *W2 = b1 + kHid, *b2 = W2 + kHid * kHid;
    const float *W3 = b2 + kHid, *b3 = W3 + kOut * kHid;
    for (int i = 0; i < kParams; ++i)
        if (!std::isfinite(p[i])) return report_error(PDM1_ERR_ARGUMENT, "box model: non-finite parameter");
    for (int i = 0; i < kHid * kFeat; ++i) out.W1[i] = __float2bfloat16_rn(W1[i]);
    for (int i = 0; i < kHid * kHid; ++i) out.W2[i] = __float2bfloat16_rn(W2[i]);
    for (int i = 0; i < kOutPad * kHid; ++i) out.W3[i] = __float2bfloat16_rn(i < kOut * kHid ? W3[i] : 0.f);
    for (int i = 0; i < kHid; ++i) { out.b1[i] = b1[i]; out.b2[i] = b2[i]; }
    for (int i = 0; i < kOutPad; ++i) out.b3[i] = i < kOut ? b3[i] : 0.f;
    for (int i = 0; i < kFeat; ++i) { out.x_mean[i] = m->x_mean[i]; out.x_inv_std[i] = m->x_inv_std[i]; }
    for (int i = 0; i < kOut; ++i) { out.y_scale[i] = m->y_scale[i]; out.y_offset[i] = m->y_offset[i]; }
    out.margin_min = m->margin_min;
    out.margin_max = m->margin_max;
    out.grow_cells = m->grow_cells;
    out.extra_max = m->extra_max;
    out.leak_tol = m->leak_tolerance;
    return PDM1_OK;
}

}  // namespace pdm1

using namespace pdm1;

extern "C" {

int pdm1_mlp_gradients(const float *theta, const float *X, const float *Y, int n, float alpha, float *grad,
                       float *loss, pdm1_stream_t stream_) {
    if (!theta || !X || !Y || !grad || n < 1) return report_error(PDM1_ERR_ARGUMENT, "NULL buffer or n < 1");
    cudaStream_t stream = (cudaStream_t)stream_;
    CUDA_OK(cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrainSmem));
    std::vector<int> idx(n);
    for (int i = 0; i < n; ++i) idx[i] = i;
    int *d_idx = nullptr;
    CUDA_OK(cudaMalloc(&d_idx, n * sizeof(int)));
    cudaError_t e = cudaMemcpyAsync(d_idx, idx.data(), n * sizeof(int), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(grad, 0, kParams * sizeof(float), stream);
    if (e == cudaSuccess && loss) e = cudaMemsetAsync(loss, 0, sizeof(float), stream);
    if (e == cudaSuccess) {
        mlp_grad_kernel<<<(n + kRows - 1) / kRows, kTrainThreads, kTrainSmem, stream>>>(
            theta, X, Y, d_idx, n, 1.f / (float)(n * kOut), alpha, grad, loss);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    cudaFree(d_idx);
    if (e != cudaSuccess) return report_error(PDM1_ERR_CUDA, cudaGetErrorString(e));
    return PDM1_OK;
}

int pdm1_mlp_train(float *theta, const float *X, const float *Y, int n, int epochs, int batch, float lr,
                   float alpha, unsigned seed, float *loss_per_epoch, pdm1_stream_t stream_) {
    if (!theta || !X || !Y || n < 1 || epochs < 1 || batch < 1 || !(lr > 0.f))
        return report_error(PDM1_ERR_ARGUMENT, "pdm1_mlp_train: invalid argument");
    cudaStream_t stream = (cudaStream_t)stream_;
    CUDA_OK(cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrainSmem));
    float *d_m = nullptr, *d_v = nullptr, *d_g = nullptr, *d_loss = nullptr;
    int *d_idx = nullptr;
    auto release = [&]() { cudaFree(d_m); cudaFree(d_v); cudaFree(d_g); cudaFree(d_loss); cudaFree(d_idx); };
    if (cudaMalloc(&d_m, kParams * sizeof(float)) != cudaSuccess || cudaMalloc(&d_v, kParams * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&d_g, kParams * sizeof(float)) != cudaSuccess || cudaMalloc(&d_loss, sizeof(float)) != cudaSuccess ||
        cudaMalloc(&d_idx, (size_t)n * sizeof(int)) != cudaSuccess) {
        release();
        return report_error(PDM1_ERR_CUDA, "pdm1_mlp_train: cudaMalloc failed");
    }
    cudaError_t e = cudaMemsetAsync(d_m, 0, kParams * sizeof(float), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_v, 0, kParams * sizeof(float), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_g, 0, kParams * sizeof(float), stream);
    std::vector<int> perm(n);
    for (int i = 0; i < n; ++i) perm[i] = i;
    std::mt19937 rng(seed);
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    int step = 0;
    for (int ep = 0; ep < epochs && e == cudaSuccess; ++ep) {
        std::shuffle(perm.begin(), perm.end(), rng);
        e = cudaMemcpyAsync(d_idx, perm.data(), (size_t)n * sizeof(int), cudaMemcpyHostToDevice, stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(d_loss, 0, sizeof(float), stream);
        for (int s0 = 0; s0 < n && e == cudaSuccess; s0 += batch) {
            int nb = std::min(batch, n - s0);
            mlp_grad_kernel<<<(nb + kRows - 1) / kRows, kTrainThreads, kTrainSmem, stream>>>(
                theta, X, Y, d_idx + s0, nb, 1.f / (float)(nb * kOut), alpha, d_g, d_loss);
            ++step;
            float c1 = 1.f - std::pow(b1, (float)step), c2 = 1.f - std::pow(b2, (float)step);
            mlp_adam_kernel<<<(kParams + 255) / 256, 256, 0, stream>>>(theta, d_m, d_v, d_g, kParams, lr, b1, b2,
                                                                      eps, c1, c2);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess && loss_per_epoch) {
            float l = 0.f;
            e = cudaMemcpyAsync(&l, d_loss, sizeof l, cudaMemcpyDeviceToHost, stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
            // the per-batch losses are means over their batches: report their mean
            loss_per_epoch[ep] = l / (float)((n + batch - 1) / batch);
        }
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    release();
    if (e != cudaSuccess) return report_error(PDM1_ERR_CUDA, cudaGetErrorString(e));
    return PDM1_OK;
}

int pdm1_mlp_forward(const float *theta, const float *X, int n, float *Y, pdm1_stream_t stream_) {
    if (!theta || !X || !Y || n < 1) return report_error(PDM1_ERR_ARGUMENT, "NULL buffer or n < 1");
    cudaStream_t stream = (cudaStream_t)stream_;
    mlp_forward_kernel<<<(n + 127) / 128, 128, 0, stream>>>(theta, X, n, Y);
    CUDA_OK(cudaGetLastError());
    CUDA_OK(cudaStreamSynchronize(stream));
    return PDM1_OK;
}

int pdm1_box_model_infer(const pdm1_box_model *model, const float *features, int n, float *out,
                         pdm1_stream_t stream_) {
    if (!features || !out || n < 1) return report_error(PDM1_ERR_ARGUMENT, "NULL buffer or n < 1");
    BoxModelDev h;
    int rc = pack_box_model(model, h);
    if (rc) return rc;
    cudaStream_t stream = (cudaStream_t)stream_;
    BoxModelDev *d = nullptr;
    CUDA_OK(cudaMalloc(&d, sizeof h));
    cudaError_t e = cudaMemcpyAsync(d, &h, sizeof h, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) {
        infer_kernel<<<(n + 63) / 64, 128, 0, stream>>>(d, features, n, out);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    cudaFree(d);
    if (e != cudaSuccess) return report_error(PDM1_ERR_CUDA, cudaGetErrorString(e));
    return PDM1_OK;
}

}  // extern "C"
