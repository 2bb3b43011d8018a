// pdm1_gamma.cu -- global 3-D gamma index on the GPU.
//
// The reference scores doses with pymedphys.gamma (pymedphys 0.41.0, called at
// proton_solver/metrics.py:581-594 with interp_fraction=10, max_gamma=1.1,
// local_gamma=False, global_normalisation=max(reference),
// lower_percent_dose_cutoff=10, skip_once_passed=True).  This kernel follows
// the published definition (Low et al., Med. Phys. 25 (1998) 656) with those
// parameters: for every reference voxel at or above the cutoff,
//   gamma = min over evaluation points e within max_gamma * DTA of
//           sqrt(|r - e|^2 / DTA^2 + (D_eval(e) - D_ref(r))^2 / dD^2),
// where the evaluation dose is trilinearly interpolated at points on a lattice
// of spacing DTA / interp_fraction around r (points outside the evaluation
// grid are not candidates) and dD = dose_percent/100 * global normalisation.
// Candidates are visited in order of distance, so the search stops as soon as
// the distance term alone exceeds the best value, or once gamma <= 1.
#include "../../include/pdm1.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>

namespace {

struct Offset {
    double dx, dy, dz;   // mm
    double d2;           // squared distance / DTA^2
};

__device__ __forceinline__ double trilinear(const double *D, int nx, int ny, int nz, double fi, double fj,
                                            double fk) {
    int i = (int)floor(fi), j = (int)floor(fj), k = (int)floor(fk);
    i = i < 0 ? 0 : (i > nx - 2 ? nx - 2 : i);
    j = j < 0 ? 0 : (j > ny - 2 ? ny - 2 : j);
    k = k < 0 ? 0 : (k > nz - 2 ? nz - 2 : k);
    double ti = nx > 1 ? fi - i : 0.0, tj = ny > 1 ? fj - j : 0.0, tk = nz > 1 ? fk - k : 0.0;
    int i1 = nx > 1 ? i + 1 : i, j1 = ny > 1 ? j + 1 : j, k1 = nz > 1 ? k + 1 : k;
    auto at = [&](int a, int b, int c) { return D[((size_t)a * ny + b) * nz + c]; };
    double c00 = at(i, j, k) * (1.0 - tk) + at(i, j, k1) * tk;
    double c01 = at(i, j1, k) * (1.0 - tk) + at(i, j1, k1) * tk;
    double c10 = at(i1, j, k) * (1.0 - tk) + at(i1, j, k1) * tk;
    double c11 = at(i1, j1, k) * (1.0 - tk) + at(i1, j1, k1) * tk;
    double c0 = c00 * (1.0 - tj) + c01 * tj;
    double c1 = c10 * (1.0 - tj) + c11 * tj;
    return c0 * (1.0 - ti) + c1 * ti;
}

__global__ void gamma_kernel(const double *ref, const double *eval, int nx, int ny, int nz, double hx,
                             double hy, double hz, const Offset *off, int n_off, double inv_dd2,
                             double cutoff, double max_gamma, int skip_once_passed, double *gamma,
                             unsigned long long *counts) {
    size_t N = (size_t)nx * ny * nz;
    size_t o = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long pass = 0, valid = 0;
    if (o < N) {
        double dr = ref[o];
        double g = NAN;
        if (dr >= cutoff) {
            int k = (int)(o % nz), j = (int)((o / nz) % ny), i = (int)(o / ((size_t)nz * ny));
            double best = INFINITY;
            for (int q = 0; q < n_off; ++q) {
                const Offset ofs = off[q];
                if (ofs.d2 >= best) break;                    // farther points cannot win
                double fi = i + ofs.dx / hx, fj = j + ofs.dy / hy, fk = k + ofs.dz / hz;
                if (fi < 0.0 || fi > nx - 1 || fj < 0.0 || fj > ny - 1 || fk < 0.0 || fk > nz - 1) continue;
                double de = trilinear(eval, nx, ny, nz, fi, fj, fk) - dr;
                double g2 = ofs.d2 + de * de * inv_dd2;
                if (g2 < best) best = g2;
                if (skip_once_passed && best <= 1.0) break;
            }
            g = sqrt(best);
            if (g > max_gamma) g = max_gamma > 0.0 ? INFINITY : g;
            valid = 1;
            pass = g <= 1.0;
        }
        gamma[o] = g;
    }
    // warp-aggregated counts
    for (int s = 16; s > 0; s >>= 1) {
        pass += __shfl_xor_sync(0xffffffffu, pass, s);
        valid += __shfl_xor_sync(0xffffffffu, valid, s);
    }
    if ((threadIdx.x & 31) == 0 && valid) {
        atomicAdd(&counts[0], pass);
        atomicAdd(&counts[1], valid);
    }
}

}  // namespace

extern "C" int pdm1_gamma(const double *dose_ref, const double *dose_eval, int nx, int ny, int nz,
                          double dx_mm, double dy_mm, double dz_mm, double dose_percent,
                          double distance_mm, double lower_cutoff_percent, int interp_fraction,
                          double max_gamma, double global_normalisation, double *gamma_out,
                          double *pass_rate_out, pdm1_stream_t stream_) {
    if (!dose_ref || !dose_eval || !gamma_out || nx <= 0 || ny <= 0 || nz <= 0 || !(dx_mm > 0) ||
        !(dy_mm > 0) || !(dz_mm > 0) || !(dose_percent > 0) || !(distance_mm > 0) || interp_fraction <= 0 ||
        !(global_normalisation > 0))
        return PDM1_ERR_ARGUMENT;
    cudaStream_t stream = (cudaStream_t)stream_;
    // candidate offsets on the interpolation lattice inside the search sphere, by distance
    const double h = distance_mm / interp_fraction;
    const double R = (max_gamma > 0 ? max_gamma : 1.0) * distance_mm;
    const int m = (int)std::floor(R / h + 1e-9);
    std::vector<Offset> offs;
    for (int a = -m; a <= m; ++a)
        for (int b = -m; b <= m; ++b)
            for (int c = -m; c <= m; ++c) {
                double x = a * h, y = b * h, z = c * h;
                double r2 = x * x + y * y + z * z;
                if (r2 <= R * R * (1.0 + 1e-12)) offs.push_back({x, y, z, r2 / (distance_mm * distance_mm)});
            }
    std::stable_sort(offs.begin(), offs.end(), [](const Offset &p, const Offset &q) { return p.d2 < q.d2; });
    Offset *d_off = nullptr;
    unsigned long long *d_counts = nullptr;
    if (cudaMalloc(&d_off, offs.size() * sizeof(Offset)) != cudaSuccess ||
        cudaMalloc(&d_counts, 2 * sizeof(unsigned long long)) != cudaSuccess) {
        cudaFree(d_off);
        return PDM1_ERR_CUDA;
    }
    cudaMemcpyAsync(d_off, offs.data(), offs.size() * sizeof(Offset), cudaMemcpyHostToDevice, stream);
    cudaMemsetAsync(d_counts, 0, 2 * sizeof(unsigned long long), stream);
    double dD = dose_percent / 100.0 * global_normalisation;
    double cutoff = lower_cutoff_percent / 100.0 * global_normalisation;
    size_t N = (size_t)nx * ny * nz;
    int blocks = (int)((N + 255) / 256);
    gamma_kernel<<<blocks, 256, 0, stream>>>(dose_ref, dose_eval, nx, ny, nz, dx_mm, dy_mm, dz_mm, d_off,
                                             (int)offs.size(), 1.0 / (dD * dD), cutoff, max_gamma, 1,
                                             gamma_out, d_counts);
    unsigned long long counts[2] = {0, 0};
    cudaError_t e = cudaMemcpyAsync(counts, d_counts, sizeof counts, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    cudaFree(d_off);
    cudaFree(d_counts);
    if (e != cudaSuccess) return PDM1_ERR_CUDA;
    if (pass_rate_out) *pass_rate_out = counts[1] ? 100.0 * (double)counts[0] / (double)counts[1] : NAN;
    return PDM1_OK;
}
