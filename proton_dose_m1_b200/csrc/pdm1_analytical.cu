// pdm1_analytical.cu -- the analytical CSDA + straight-streaming dose on the GPU.
//
// The reference's reduced-model verifier (proton_solver/analytical.py:64-326):
// without scattering, nuclear removal or angular spread, every proton keeps
// its transverse position and loses energy along z by the continuous-slowing-
// down range relation R(E_out) = R(E_in) - dz, cell by cell.  The dose of a
// cell is the spectrum-weighted energy lost in it (trapezoid rule over the
// incident energies on [energy_min, E0 + window * sigma_E]) times
// MEV_TO_JOULE / (rho dz), scaled by the beam's transverse fluence.
//
// Range tables (analytical.py:64-106): geometric energy grid from the
// stopping-power table's first node to its last, PCHIP stopping power,
// cumulative trapezoid of 1/S.  Energy <-> range by linear interpolation
// (numpy.interp semantics: clamp below to 0, above to the last value).
// Identical material columns share one column computation, as the
// reference's column cache does; the energies of a column are marched by one
// thread each, the per-cell sums reduced per CTA and added atomically.
#include "../../include/pdm1.h"
#include "pdm1_device.cuh"

#include <cuda_runtime.h>

#include <cmath>
#include <map>
#include <string>
#include <vector>

namespace pdm1 {
std::vector<double> host_pchip_slopes(const double *E, const double *v, int n);
}

using namespace pdm1;

namespace {

constexpr int kThreads = 256;

// numpy.interp with left/right values
__device__ __forceinline__ double interp(double x, const double *xs, const double *ys, int n, double left,
                                         double right) {
    if (!(x >= xs[0])) return left;
    if (x > xs[n - 1]) return right;
    int lo = 0, hi = n - 1;   // xs[lo] <= x <= xs[hi]
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (xs[mid] <= x) lo = mid; else hi = mid;
    }
    double x0 = xs[lo], x1 = xs[hi];
    if (x1 == x0) return ys[hi];
    double t = (x - x0) / (x1 - x0);
    return ys[lo] + t * (ys[hi] - ys[lo]);
}

struct RangeView {
    const double *E, *R;
    int n;
};

// One column per blockIdx.y; energy nodes over blockIdx.x * blockDim.x + threadIdx.x.
__global__ void __launch_bounds__(kThreads) column_kernel(const RangeView *tabs, const int *col_mats, int nz,
                                                          double dz, const double *nodes, const double *weights,
                                                          int n_nodes, double *lost_sum) {
    __shared__ double red[kThreads / 32];
    const int col = blockIdx.y;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double E = i < n_nodes ? nodes[i] : 0.0;
    const double w = i < n_nodes ? weights[i] : 0.0;
    for (int iz = 0; iz < nz; ++iz) {
        const RangeView t = tabs[col_mats[(size_t)col * nz + iz]];
        double lost = 0.0;
        if (E > 0.0) {
            double r_in = interp(E, t.E, t.R, t.n, 0.0, t.R[t.n - 1]);
            double r_out = r_in - dz;
            double e_out = r_out > 0.0 ? interp(r_out, t.R, t.E, t.n, 0.0, t.E[t.n - 1]) : 0.0;
            lost = fmax(E - e_out, 0.0);
            E = e_out;
        }
        double v = w * lost;
        for (int s = 16; s > 0; s >>= 1) v += __shfl_xor_sync(0xffffffffu, v, s);
        if (lane == 0) red[warp] = v;
        __syncthreads();
        if (threadIdx.x == 0) {
            double sum = 0.0;
            for (int q = 0; q < kThreads / 32; ++q) sum += red[q];
            if (sum != 0.0) atomicAdd(&lost_sum[(size_t)col * nz + iz], sum);
        }
        __syncthreads();
    }
}

__global__ void dose_kernel(const int *col_of, const double *lost_sum, const int32_t *ids, const double *inv_rho,
                            const double *spatial, int nx, int ny, int nz, double scale, double *dose) {
    size_t N = (size_t)nx * ny * nz;
    for (size_t o = (size_t)blockIdx.x * blockDim.x + threadIdx.x; o < N; o += (size_t)gridDim.x * blockDim.x) {
        int k = (int)(o % nz);
        size_t xy = o / nz;
        double f = lost_sum[(size_t)col_of[xy] * nz + k] * scale * inv_rho[ids[o]];
        dose[o] = spatial[xy] * f;
    }
}

#define CUDA_OK(expr)                                                              \
    do {                                                                           \
        cudaError_t e_ = (expr);                                                   \
        if (e_ != cudaSuccess) {                                                   \
            std::string m_ = std::string(#expr ": ") + cudaGetErrorString(e_);     \
            return report_error(PDM1_ERR_CUDA, m_.c_str());                        \
        }                                                                          \
    } while (0)

// Host PCHIP (the stopping-power interpolant, physics/stopping_power.py:57-138):
// clamped to the table, searchsorted(side="right") - 1 interval, cubic Hermite.
double pchip_host(const double *E, const double *v, const std::vector<double> &s, int n, double x) {
    if (x <= E[0]) x = E[0];
    if (x >= E[n - 1]) x = E[n - 1];
    int lo = 0, hi = n;   // first index with E > x, minus one
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (E[mid] <= x) lo = mid + 1; else hi = mid;
    }
    int i = lo - 1;
    if (i < 0) i = 0;
    if (i > n - 2) i = n - 2;
    double h = E[i + 1] - E[i], t = (x - E[i]) / h, t2 = t * t, t3 = t2 * t;
    return (2.0 * t3 - 3.0 * t2 + 1.0) * v[i] + (t3 - 2.0 * t2 + t) * h * s[i] + (-2.0 * t3 + 3.0 * t2) * v[i + 1] +
           (t3 - t2) * h * s[i + 1];
}

}  // namespace

extern "C" int pdm1_analytical_csda_dose(const pdm1_problem *p, int energy_points, int range_points, double *dose,
                                         pdm1_stream_t stream_) {
    if (!p || !dose || !p->materials || !p->ids || !p->inflow_spatial)
        return report_error(PDM1_ERR_ARGUMENT, "NULL problem, tables, ids, inflow or dose");
    if (p->scattering != PDM1_SCATTERING_OFF || p->nuclear || p->angular_spread != 0.0)
        return report_error(PDM1_ERR_ARGUMENT, "Analytical reference is not available for this configuration.");
    if (energy_points < 2) return report_error(PDM1_ERR_ARGUMENT, "num_energy_points must be at least 2.");
    if (range_points < 2) return report_error(PDM1_ERR_ARGUMENT, "range_points must be at least 2.");
    if (!(p->energy_spread > 0.0))
        return report_error(PDM1_ERR_ARGUMENT, "Zero energy spread is not supported by the Gaussian inflow.");
    if (p->nx <= 0 || p->ny <= 0 || p->nz <= 0 || p->n_materials < 1 || p->n_materials > kMaxMat)
        return report_error(PDM1_ERR_ARGUMENT, "bad grid or material count");
    cudaStream_t stream = (cudaStream_t)stream_;
    const int nx = p->nx, ny = p->ny, nz = p->nz, nm = p->n_materials;
    const size_t NXY = (size_t)nx * ny, N = NXY * nz;
    for (size_t c = 0; c < N; ++c)
        if (p->ids[c] < 0 || p->ids[c] >= nm) return report_error(PDM1_ERR_ARGUMENT, "material id out of range");
    // range tables per material (analytical.py:64-106)
    std::vector<double> blob;
    std::vector<std::pair<size_t, int>> where(nm);
    std::vector<double> inv_rho(nm);
    for (int m = 0; m < nm; ++m) {
        const pdm1_table &t = p->materials[m].stopping_power;
        if (t.n_nodes < 2) return report_error(PDM1_ERR_ARGUMENT, "stopping-power table needs two nodes");
        std::vector<double> slopes = host_pchip_slopes(t.energy, t.value, t.n_nodes);
        const double a = std::max(t.energy[0], 1e-12), b = t.energy[t.n_nodes - 1];
        const double la = std::log(a), lb = std::log(b);
        std::vector<double> E(range_points), R(range_points, 0.0), S(range_points);
        for (int i = 0; i < range_points; ++i) {
            E[i] = i == 0 ? a : (i == range_points - 1 ? b : std::exp(la + (lb - la) * i / (range_points - 1)));
            S[i] = pchip_host(t.energy, t.value, slopes, t.n_nodes, E[i]);
        }
        for (int i = 1; i < range_points; ++i) R[i] = R[i - 1] + 0.5 * (1.0 / S[i] + 1.0 / S[i - 1]) * (E[i] - E[i - 1]);
        where[m] = {blob.size(), range_points};
        blob.insert(blob.end(), E.begin(), E.end());
        blob.insert(blob.end(), R.begin(), R.end());
        inv_rho[m] = 1.0 / p->materials[m].density;
    }
    // incident energies and trapezoid weights times the spectrum (analytical.py:173-269)
    const double E0 = p->beam_energy + p->energy_window_sigma * p->energy_spread;
    std::vector<double> nodes(energy_points), weights(energy_points);
    for (int i = 0; i < energy_points; ++i)
        nodes[i] = i == energy_points - 1 ? E0
                                         : p->energy_min + (E0 - p->energy_min) * i / (double)(energy_points - 1);
    const double sg = p->energy_spread, norm = std::sqrt(2.0 * 3.141592653589793) * sg;
    for (int i = 0; i < energy_points; ++i) {
        double d = nodes[i] - p->beam_energy;
        double spec = std::exp(-(d * d) / (2.0 * sg * sg)) / norm;
        double left = i > 0 ? nodes[i] - nodes[i - 1] : 0.0, right = i + 1 < energy_points ? nodes[i + 1] - nodes[i] : 0.0;
        weights[i] = 0.5 * (left + right) * spec;
    }
    // distinct material columns (the reference's column cache)
    std::map<std::vector<int32_t>, int> cols;
    std::vector<int> col_of(NXY);
    std::vector<int> col_mats;
    for (size_t xy = 0; xy < NXY; ++xy) {
        std::vector<int32_t> key(p->ids + xy * nz, p->ids + (xy + 1) * nz);
        auto it = cols.find(key);
        if (it == cols.end()) {
            it = cols.emplace(key, (int)cols.size()).first;
            col_mats.insert(col_mats.end(), key.begin(), key.end());
        }
        col_of[xy] = it->second;
    }
    const int ncol = (int)cols.size();
    double *d_blob = nullptr, *d_nodes = nullptr, *d_w = nullptr, *d_lost = nullptr, *d_rho = nullptr, *d_sp = nullptr;
    int *d_cm = nullptr, *d_colof = nullptr;
    int32_t *d_ids = nullptr;
    RangeView *d_tabs = nullptr;
    auto release = [&]() {
        cudaFree(d_blob); cudaFree(d_nodes); cudaFree(d_w); cudaFree(d_lost); cudaFree(d_rho); cudaFree(d_sp);
        cudaFree(d_cm); cudaFree(d_colof); cudaFree(d_ids); cudaFree(d_tabs);
    };
    bool ok = cudaMalloc(&d_blob, blob.size() * sizeof(double)) == cudaSuccess &&
              cudaMalloc(&d_nodes, energy_points * sizeof(double)) == cudaSuccess &&
              cudaMalloc(&d_w, energy_points * sizeof(double)) == cudaSuccess &&
              cudaMalloc(&d_lost, (size_t)ncol * nz * sizeof(double)) == cudaSuccess &&
              cudaMalloc(&d_rho, nm * sizeof(double)) == cudaSuccess &&
              cudaMalloc(&d_sp, NXY * sizeof(double)) == cudaSuccess &&
              cudaMalloc(&d_cm, col_mats.size() * sizeof(int)) == cudaSuccess &&
              cudaMalloc(&d_colof, NXY * sizeof(int)) == cudaSuccess &&
              cudaMalloc(&d_ids, N * sizeof(int32_t)) == cudaSuccess &&
              cudaMalloc(&d_tabs, nm * sizeof(RangeView)) == cudaSuccess;
    if (!ok) {
        release();
        return report_error(PDM1_ERR_CUDA, "pdm1_analytical_csda_dose: cudaMalloc failed");
    }
    std::vector<RangeView> tabs(nm);
    for (int m = 0; m < nm; ++m) tabs[m] = {d_blob + where[m].first, d_blob + where[m].first + where[m].second, where[m].second};
    cudaError_t e = cudaMemcpyAsync(d_blob, blob.data(), blob.size() * sizeof(double), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_nodes, nodes.data(), energy_points * sizeof(double), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_w, weights.data(), energy_points * sizeof(double), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_lost, 0, (size_t)ncol * nz * sizeof(double), stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_rho, inv_rho.data(), nm * sizeof(double), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_sp, p->inflow_spatial, NXY * sizeof(double), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_cm, col_mats.data(), col_mats.size() * sizeof(int), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_colof, col_of.data(), NXY * sizeof(int), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_ids, p->ids, N * sizeof(int32_t), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_tabs, tabs.data(), nm * sizeof(RangeView), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) {
        dim3 grid((energy_points + kThreads - 1) / kThreads, ncol);
        column_kernel<<<grid, kThreads, 0, stream>>>(d_tabs, d_cm, nz, p->dz, d_nodes, d_w, energy_points, d_lost);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        int blocks = (int)std::min<size_t>((N + 255) / 256, 148 * 16);
        dose_kernel<<<blocks, 256, 0, stream>>>(d_colof, d_lost, d_ids, d_rho, d_sp, nx, ny, nz,
                                                kMevToJoule / p->dz, dose);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    release();
    if (e != cudaSuccess) return report_error(PDM1_ERR_CUDA, cudaGetErrorString(e));
    return PDM1_OK;
}
