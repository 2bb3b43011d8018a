// pdm1_math.cuh -- scalar M1 building blocks shared by the march kernels.
//
// Every expression keeps the evaluation order of the reference's FP64 path
// (cited per function, paths relative to the proton_solver project).  The
// double-precision translation unit is compiled with --fmad=false, so each
// product and sum is rounded separately, as NumPy does.
#pragma once

#include <cmath>
#include <cstdint>

#define PDM1_HD __host__ __device__ __forceinline__

namespace pdm1 {

constexpr double kEigEps = 1.0e-10;          // numerics/wave_speeds.py:10
constexpr double kWenoEps = 1.0e-12;         // reconstruction_methods/weno_z.py:8
constexpr double kRealEps = 1.0e-10;         // weno_z.py:10, realizability.py:110
constexpr double kMevToJoule = 1.602176634e-13;   // numerics/energy.py:37
constexpr double kExpClamp = 700.0;          // numerics/energy.py:296-304
constexpr double kProtonRestMev = 938.27208816;   // physics/scattering.py:21
constexpr double kRossiEsMev = 15.0;              // physics/scattering.py:22

// ---------------------------------------------------------------------------
// exp in double-double arithmetic: Cody-Waite reduction with ln 2 held as a
// double-double, exp(r / 2^10) by a degree-9 Taylor series (Dekker/Knuth
// error-free sums, FMA products), ten squarings, scaling by 2^k.  Good to
// about 1e-29 relative before the final rounding, i.e. correctly rounded but
// for rare ties; the same routine runs on the host and the device.
// ---------------------------------------------------------------------------
struct dd { double hi, lo; };

PDM1_HD dd dd_quick(double a, double b) { dd r; r.hi = a + b; r.lo = b - (r.hi - a); return r; }

PDM1_HD dd dd_add(dd a, dd b) {
    double s = a.hi + b.hi;
    double bb = s - a.hi;
    double e = (a.hi - (s - bb)) + (b.hi - bb);
    e += a.lo + b.lo;
    return dd_quick(s, e);
}

PDM1_HD dd dd_mul(dd a, dd b) {
    double p = a.hi * b.hi;
    double e = fma(a.hi, b.hi, -p);
    e += a.hi * b.lo + a.lo * b.hi;
    return dd_quick(p, e);
}

PDM1_HD dd dd_div_d(double a, double b) {
    double q1 = a / b;
    double p = q1 * b;
    double e = fma(q1, b, -p);
    double rem = (a - p) - e;
    return dd_quick(q1, rem / b);
}

PDM1_HD double dd_exp(double x) {
    if (x != x) return x;
    if (x > 709.782712893384) return INFINITY;
    if (x < -745.2) return 0.0;
    const double ln2_hi = 0.6931471805599453094;
    const double ln2_lo = 2.3190468138462996e-17;
    double k = rint(x * 1.4426950408889634);
    double p = k * ln2_hi;
    double pe = fma(k, ln2_hi, -p);
    double s = x - p;
    double t = -pe - k * ln2_lo;
    dd r = dd_quick(s, t);
    r.hi *= 0x1p-10;
    r.lo *= 0x1p-10;
    const double fact[10] = {1.0, 1.0, 2.0, 6.0, 24.0, 120.0, 720.0, 5040.0, 40320.0, 362880.0};
    dd acc = dd_div_d(1.0, fact[9]);
    for (int n = 8; n >= 0; --n) acc = dd_add(dd_mul(acc, r), dd_div_d(1.0, fact[n]));
    for (int q = 0; q < 10; ++q) acc = dd_mul(acc, acc);
    return ldexp(acc.hi + acc.lo, (int)k);
}

// ---------------------------------------------------------------------------
// WENO-Z5 left reconstruction, reconstruction_methods/weno_z.py:12-87
// ---------------------------------------------------------------------------
template <typename T>
PDM1_HD T weno_left(T v0, T v1, T v2, T v3, T v4) {
    // r * r below overflows single precision above r ~ 1.8e19 (reached for
    // fluences of ~1e6 protons); single precision uses weno_left_f32
    static_assert(sizeof(T) == sizeof(double), "weno_left is the FP64 path; use weno_left_f32");
    const T c3 = T(3), c6 = T(6);
    T p0 = v0 / c3 - T(7) * v1 / c6 + T(11) * v2 / c6;
    T p1 = -v1 / c6 + T(5) * v2 / c6 + v3 / c3;
    T p2 = v2 / c3 + T(5) * v3 / c6 - v4 / c6;
    const T k1312 = T(13.0 / 12.0);
    T a, b;
    a = v0 - T(2) * v1 + v2; b = v0 - T(4) * v1 + T(3) * v2;
    T beta0 = k1312 * (a * a) + T(0.25) * (b * b);
    a = v1 - T(2) * v2 + v3; b = v1 - v3;
    T beta1 = k1312 * (a * a) + T(0.25) * (b * b);
    a = v2 - T(2) * v3 + v4; b = T(3) * v2 - T(4) * v3 + v4;
    T beta2 = k1312 * (a * a) + T(0.25) * (b * b);
    T tau5 = fabs(beta2 - beta0);
    T r0 = tau5 / (beta0 + T(kWenoEps));
    T r1 = tau5 / (beta1 + T(kWenoEps));
    T r2 = tau5 / (beta2 + T(kWenoEps));
    // the FP64 path; single precision has its own form, weno_left_f32
    T al0 = T(0.1) * (T(1) + r0 * r0);
    T al1 = T(0.6) * (T(1) + r1 * r1);
    T al2 = T(0.3) * (T(1) + r2 * r2);
    T s = al0 + al1 + al2;
    T w0 = al0 / s, w1 = al1 / s, w2 = al2 / s;
    return w0 * p0 + w1 * p1 + w2 * p2;
}

// Single-precision quotient on the MUFU reciprocal: a * (1/b), two
// instructions, within 2 ulp for |b| below 2^126 (every denominator of the
// float face path: smoothness indicators up to phi^2, weight sums below
// 1e31, |J|, phi, wave-speed denominators of order 1).
PDM1_HD float fast_div(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fdividef(a, b);
#else
    return a / b;
#endif
}

// Single-precision WENO-Z5 with the arithmetic regrouped for fewer
// instructions: the candidate polynomials as integer combinations times 1/6,
// the 1/6 folded into the one reciprocal of the weight sum.  Same weights as
// weno_left; the ratios tau5 / (beta + eps) are held at 1e30 and the alphas
// rescaled by the largest ratio, so that nothing overflows single precision.
PDM1_HD float weno_left_f32(float v0, float v1, float v2, float v3, float v4) {
    const float q0 = 2.0f * v0 - 7.0f * v1 + 11.0f * v2;   // 6 p0
    const float q1 = -v1 + 5.0f * v2 + 2.0f * v3;          // 6 p1
    const float q2 = 2.0f * v2 + 5.0f * v3 - v4;           // 6 p2
    float a = v0 - 2.0f * v1 + v2, b = v0 - 4.0f * v1 + 3.0f * v2;
    const float beta0 = float(13.0 / 12.0) * (a * a) + 0.25f * (b * b);
    a = v1 - 2.0f * v2 + v3; b = v1 - v3;
    const float beta1 = float(13.0 / 12.0) * (a * a) + 0.25f * (b * b);
    a = v2 - 2.0f * v3 + v4; b = 3.0f * v2 - 4.0f * v3 + v4;
    const float beta2 = float(13.0 / 12.0) * (a * a) + 0.25f * (b * b);
    const float tau5 = fabsf(beta2 - beta0);
    // r = tau5 / (beta + eps) reaches phi^2 / eps ~ 1e35 for 1e6 protons
    // and overflows beyond; held at 1e30, where the other weights are 1e-60 of it
    const float r0 = fminf(fast_div(tau5, beta0 + float(kWenoEps)), 1e30f);
    const float r1 = fminf(fast_div(tau5, beta1 + float(kWenoEps)), 1e30f);
    const float r2 = fminf(fast_div(tau5, beta2 + float(kWenoEps)), 1e30f);
    float al0, al1, al2;
    const float rmax = fmaxf(r0, fmaxf(r1, r2));
    if (rmax > 1e15f) {   // r^2 would overflow: divide every alpha by rmax^2
        const float inv = fast_div(1.0f, rmax), e = inv * inv;
        const float t0 = r0 * inv, t1 = r1 * inv, t2 = r2 * inv;
        al0 = 0.1f * (e + t0 * t0);
        al1 = 0.6f * (e + t1 * t1);
        al2 = 0.3f * (e + t2 * t2);
    } else {
        al0 = 0.1f * (1.0f + r0 * r0);
        al1 = 0.6f * (1.0f + r1 * r1);
        al2 = 0.3f * (1.0f + r2 * r2);
    }
    // normalised weights first: al * q itself overflows (al up to 6e29 below
    // the guard, q up to 20 max|v|)
    const float inv = fast_div(1.0f, 6.0f * (al0 + al1 + al2));
    return (al0 * inv) * q0 + (al1 * inv) * q1 + (al2 * inv) * q2;
}

#if defined(__CUDACC__)
// ---------------------------------------------------------------------------
// WENO-Z5 of two components at once on sm_100's packed single-precision
// pipe (fma/mul/add.rn.f32x2: one instruction for both lanes).  Lane x and
// lane y are two state components of the same cells, so the five inputs are
// five 64-bit shared-memory loads.  The arithmetic per lane is that of
// weno_left_f32: the candidate polynomials as integer combinations times 1/6,
// the Jiang-Shu indicators, r = tau5 / (beta + eps) held at 1e30, and, where
// r^2 could overflow (r > 1e15), every alpha rescaled by 1 / max r^2; the
// weights are normalised before they multiply the polynomials.  Quotients
// and the comparisons stay per lane (no packed reciprocal or min/max).
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 pk(float s) { return make_float2(s, s); }
__device__ __forceinline__ float2 pk_fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 pk_mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 pk_add(float2 a, float2 b) { return __fadd2_rn(a, b); }
// approximate reciprocal per lane (MUFU), within 2 ulp for |x| below 2^126
__device__ __forceinline__ float2 pk_rcp(float2 x) { return make_float2(__fdividef(1.0f, x.x), __fdividef(1.0f, x.y)); }
__device__ __forceinline__ float2 pk_sqrt(float2 x) { return make_float2(sqrtf(x.x), sqrtf(x.y)); }

// Jiang-Shu smoothness indicator 13/12 a^2 + 1/4 b^2
__device__ __forceinline__ float2 pk_beta(float2 a, float2 b) {
    return pk_fma(pk_mul(pk(float(13.0 / 12.0)), a), a, pk_mul(pk_mul(pk(0.25f), b), b));
}

__device__ __forceinline__ float2 weno_left_f32x2(float2 v0, float2 v1, float2 v2, float2 v3, float2 v4) {
    const float2 q0 = pk_fma(pk(2.0f), v0, pk_fma(pk(-7.0f), v1, pk_mul(pk(11.0f), v2)));   // 6 p0
    const float2 q1 = pk_fma(pk(-1.0f), v1, pk_fma(pk(5.0f), v2, pk_mul(pk(2.0f), v3)));    // 6 p1
    const float2 q2 = pk_fma(pk(-1.0f), v4, pk_fma(pk(2.0f), v2, pk_mul(pk(5.0f), v3)));    // 6 p2
    const float2 beta0 = pk_beta(pk_add(pk_fma(pk(-2.0f), v1, v0), v2),
                                 pk_fma(pk(3.0f), v2, pk_fma(pk(-4.0f), v1, v0)));
    const float2 beta1 = pk_beta(pk_add(pk_fma(pk(-2.0f), v2, v1), v3), pk_fma(pk(-1.0f), v3, v1));
    const float2 beta2 = pk_beta(pk_add(pk_fma(pk(-2.0f), v3, v2), v4),
                                 pk_fma(pk(-4.0f), v3, pk_fma(pk(3.0f), v2, v4)));
    const float2 d = pk_fma(pk(-1.0f), beta0, beta2);
    const float2 tau5 = make_float2(fabsf(d.x), fabsf(d.y));
    const float2 eps = pk(float(kWenoEps));
    float2 r0 = pk_mul(tau5, pk_rcp(pk_add(beta0, eps)));
    float2 r1 = pk_mul(tau5, pk_rcp(pk_add(beta1, eps)));
    float2 r2 = pk_mul(tau5, pk_rcp(pk_add(beta2, eps)));
    r0 = make_float2(fminf(r0.x, 1e30f), fminf(r0.y, 1e30f));
    r1 = make_float2(fminf(r1.x, 1e30f), fminf(r1.y, 1e30f));
    r2 = make_float2(fminf(r2.x, 1e30f), fminf(r2.y, 1e30f));
    // alpha_k / s^2 = d_k (s^-2 + (r_k / s)^2) with s = max r where r^2 could overflow, else s = 1
    float2 sc = pk(1.0f);
    const float mx = fmaxf(r0.x, fmaxf(r1.x, r2.x)), my = fmaxf(r0.y, fmaxf(r1.y, r2.y));
    if (mx > 1e15f || my > 1e15f) {
        if (mx > 1e15f) sc.x = __fdividef(1.0f, mx);
        if (my > 1e15f) sc.y = __fdividef(1.0f, my);
    }
    const float2 e = pk_mul(sc, sc);
    const float2 t0 = pk_mul(r0, sc), t1 = pk_mul(r1, sc), t2 = pk_mul(r2, sc);
    const float2 al0 = pk_mul(pk(0.1f), pk_fma(t0, t0, e));
    const float2 al1 = pk_mul(pk(0.6f), pk_fma(t1, t1, e));
    const float2 al2 = pk_mul(pk(0.3f), pk_fma(t2, t2, e));
    const float2 inv = pk_rcp(pk_mul(pk(6.0f), pk_add(pk_add(al0, al1), al2)));
    return pk_fma(pk_mul(al2, inv), q2, pk_fma(pk_mul(al1, inv), q1, pk_mul(pk_mul(al0, inv), q0)));
}
#endif

// ---------------------------------------------------------------------------
// WENO3-Z left reconstruction (p = 2), reconstruction_methods/weno3.py:15-62
// ---------------------------------------------------------------------------
template <typename T>
PDM1_HD T weno3_left(T v0, T v1, T v2) {
    T p0 = T(-0.5) * v0 + T(1.5) * v1;
    T p1 = T(0.5) * v1 + T(0.5) * v2;
    T beta0 = (v1 - v0) * (v1 - v0);
    T beta1 = (v2 - v1) * (v2 - v1);
    T tau3 = fabs(beta1 - beta0);
    T r0 = tau3 / (beta0 + T(kWenoEps));
    T r1 = tau3 / (beta1 + T(kWenoEps));
    T alpha0 = T(1.0 / 3.0) * (T(1) + r0 * r0);
    T alpha1 = T(2.0 / 3.0) * (T(1) + r1 * r1);
    if (sizeof(T) < sizeof(double) && !(alpha0 < T(1e30) && alpha1 < T(1e30))) {
        // single precision: r^2 overflows; the weights are those of r0^2 : 2 r1^2
        T m = fmax(r0, r1), q0 = r0 / m, q1 = r1 / m;
        alpha0 = q0 * q0;
        alpha1 = T(2) * q1 * q1;
    }
    T s = alpha0 + alpha1;
    T w0 = alpha0 / s, w1 = alpha1 / s;
    return w0 * p0 + w1 * p1;
}

// Minmod-limited faces of a cell, reconstruction_methods/muscl.py:22-44.
template <typename T>
PDM1_HD void muscl_faces(T vm, T v0, T vp, T &minus, T &plus) {
    T a = v0 - vm, b = vp - v0, slope = T(0);
    if (a * b > T(0)) slope = (a > T(0) ? T(1) : T(-1)) * fmin(fabs(a), fabs(b));
    minus = v0 - T(0.5) * slope;
    plus = v0 + T(0.5) * slope;
}

// ---------------------------------------------------------------------------
// Realizability projection, numerics/realizability.py:132-176
// ---------------------------------------------------------------------------
template <typename T>
PDM1_HD void project(T &phi, T &jx, T &jy, T &jz) {
    if (phi < T(0)) phi = T(0);
    T jn = sqrt(jx * jx + jy * jy + jz * jz);
    T jmax = T(1.0 - kRealEps) * phi;
    if (jn > jmax) {
        T s = jmax / jn;
        jx *= s; jy *= s; jz *= s;
    }
}

// ---------------------------------------------------------------------------
// Exact M1 eigenvalues along an axis: numerics/flux.py:63-135
// (== numerics/wave_speeds.py:36-103)
// ---------------------------------------------------------------------------
template <typename T>
PDM1_HD void eigen(T phi, T jx, T jy, T jz, T jn, int axis, T &lmin, T &lmax) {
    const T iso = T(1) / sqrt(T(3));
    if (phi < T(kEigEps)) phi = T(kEigEps);
    if (jn < T(kEigEps)) { lmin = -iso; lmax = iso; return; }
    T f = jn / phi;
    if (f < T(0)) f = T(0);
    else if (f > T(1.0 - kEigEps)) f = T(1.0 - kEigEps);
    T jnormal = axis == 0 ? jx : (axis == 1 ? jy : jz);
    T mu = jnormal / jn;
    T chi = (T(5) - T(2) * sqrt(T(4) - T(3) * f * f)) / T(3);
    T den = T(5) - T(3) * chi;
    T disc = T(4) * f * f * mu * mu - den * (mu * mu * (T(3) * chi - T(1)) - T(2) * (T(1) - chi));
    if (disc < T(0)) disc = T(0);
    T root = sqrt(disc);
    lmin = (T(2) * f * mu - root) / den;
    lmax = (T(2) * f * mu + root) / den;
}

// max(|lambda_min|, |lambda_max|) along x, y and z at once: |J|, f, chi and
// 5 - 3 chi are formed once per cell instead of once per axis, each with the
// expressions and order of eigen(), so the speeds are eigen()'s bit for bit.
template <typename T>
PDM1_HD void max_abs_speeds3(T phi, T jx, T jy, T jz, T a[3]) {
    const T iso = T(1) / sqrt(T(3));
    const T jn = sqrt(jx * jx + jy * jy + jz * jz);
    if (phi < T(kEigEps)) phi = T(kEigEps);
    if (jn < T(kEigEps)) {
        a[0] = a[1] = a[2] = iso;
        return;
    }
    T f = jn / phi;
    if (f < T(0)) f = T(0);
    else if (f > T(1.0 - kEigEps)) f = T(1.0 - kEigEps);
    const T chi = (T(5) - T(2) * sqrt(T(4) - T(3) * f * f)) / T(3);
    const T den = T(5) - T(3) * chi;
    const T j[3] = {jx, jy, jz};
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        T mu = j[ax] / jn;
        T disc = T(4) * f * f * mu * mu - den * (mu * mu * (T(3) * chi - T(1)) - T(2) * (T(1) - chi));
        if (disc < T(0)) disc = T(0);
        T root = sqrt(disc);
        T lo = fabs((T(2) * f * mu - root) / den), hi = fabs((T(2) * f * mu + root) / den);
        a[ax] = lo > hi ? lo : hi;
    }
}

template <typename T>
PDM1_HD T max_abs_speed(T phi, T jx, T jy, T jz, int axis) {
    T jn = sqrt(jx * jx + jy * jy + jz * jz);
    T lo, hi;
    eigen(phi, jx, jy, jz, jn, axis, lo, hi);
    T alo = fabs(lo), ahi = fabs(hi);
    return alo > ahi ? alo : ahi;
}

// ---------------------------------------------------------------------------
// M1 closure and HLL flux, numerics/flux.py:10-61 and 137-386
// ---------------------------------------------------------------------------
template <typename T>
struct Closure { T jn, nx, ny, nz, iso, dir; };

template <typename T>
PDM1_HD Closure<T> closure(T phi, T jx, T jy, T jz) {
    Closure<T> c;
    c.jn = sqrt(jx * jx + jy * jy + jz * jz);
    T f;
    if (phi > T(0)) {
        f = c.jn / phi;
        if (f < T(0)) f = T(0);
        else if (f > T(1)) f = T(1);
    } else {
        f = T(0);
    }
    if (c.jn > T(0)) {
        c.nx = jx / c.jn; c.ny = jy / c.jn; c.nz = jz / c.jn;
    } else {
        c.nx = c.ny = c.nz = T(0);
    }
    if (sizeof(T) < sizeof(double)) {
        // single precision: 0.5*(1 - chi) cancels as f -> 1; the same quantity
        // without the cancellation is (1 - f^2) / (sqrt(4 - 3 f^2) + 1)
        T root = sqrt(T(4) - T(3) * f * f);
        c.iso = (T(1) - f) * (T(1) + f) / (root + T(1));
        c.dir = T(2) - root;
    } else {
        T chi = (T(5) - T(2) * sqrt(T(4) - T(3) * f * f)) / T(3);
        c.iso = T(0.5) * (T(1) - chi);
        c.dir = T(0.5) * (T(3) * chi - T(1));
    }
    return c;
}

template <typename T>
PDM1_HD void physical_flux(const T u[4], const Closure<T> &c, int axis, T F[4]) {
    T phi = u[0];
    if (axis == 0) {
        F[0] = u[1];
        F[1] = phi * (c.iso + c.dir * c.nx * c.nx);
        F[2] = phi * c.dir * c.nx * c.ny;
        F[3] = phi * c.dir * c.nx * c.nz;
    } else if (axis == 1) {
        F[0] = u[2];
        F[1] = phi * c.dir * c.nx * c.ny;
        F[2] = phi * (c.iso + c.dir * c.ny * c.ny);
        F[3] = phi * c.dir * c.ny * c.nz;
    } else {
        F[0] = u[3];
        F[1] = phi * c.dir * c.nx * c.nz;
        F[2] = phi * c.dir * c.ny * c.nz;
        F[3] = phi * (c.iso + c.dir * c.nz * c.nz);
    }
}

template <typename T>
PDM1_HD void hll_flux(const T L[4], const T R[4], int axis, bool unit_speeds, T F[4]) {
    Closure<T> cl = closure(L[0], L[1], L[2], L[3]);
    Closure<T> cr = closure(R[0], R[1], R[2], R[3]);
    T FL[4], FR[4];
    physical_flux(L, cl, axis, FL);
    physical_flux(R, cr, axis, FR);
    T sl, sr;
    if (!unit_speeds) {
        T lminl, lmaxl, lminr, lmaxr;
        eigen(L[0], L[1], L[2], L[3], cl.jn, axis, lminl, lmaxl);
        eigen(R[0], R[1], R[2], R[3], cr.jn, axis, lminr, lmaxr);
        sl = lminr < lminl ? lminr : lminl;
        sr = lmaxr > lmaxl ? lmaxr : lmaxl;
        if (sl > T(0)) sl = T(0);
        if (sr < T(0)) sr = T(0);
    } else {
        sl = T(-1);
        sr = T(1);
    }
    T den = sr - sl;
    T sp = sl * sr;
    if (sizeof(T) < sizeof(double) && !(den > T(0))) {
        // single precision only: |J|/phi rounds to 1 for an exactly directed
        // state, both speeds normal to J are then 0 and the fan collapses;
        // the HLL flux tends to the central flux as the fan closes
#pragma unroll
        for (int c = 0; c < 4; ++c) F[c] = T(0.5) * (FL[c] + FR[c]);
        return;
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) F[c] = (sr * FL[c] - sl * FR[c] + sp * (R[c] - L[c])) / den;
}

// ---------------------------------------------------------------------------
// Single-precision interface flux: the two realizability projections, the two
// closures, the exact wave speeds and the HLL combination of one face, with
// each shared quantity formed once.  The algebra is that of project, closure,
// eigen and hll_flux above; with q = (1 - f)(1 + f) and r = sqrt(1 + 3q)
// (= sqrt(4 - 3f^2)):
//   1 - chi = 2q / (r + 1) = 2 iso,   3 chi - 1 = 2 dir = 2 (2 - r),
//   5 - 3 chi = 2 + 6 iso,
// so the wave speeds reuse the closure's iso and dir, and |J| after the
// projection is the closure's |J|.  No factor carries the cancellation of
// 1 - chi as f -> 1.  One reciprocal serves each common denominator.
// ---------------------------------------------------------------------------
struct SideF32 { float phi, jx, jy, jz, jn, f, nx, ny, nz, iso, dir; };

PDM1_HD void closure_f32(float phi, float jn, float &f, float &iso, float &dir) {
    f = phi > 0.0f ? fminf(fast_div(jn, phi), 1.0f) : 0.0f;
    const float q = (1.0f - f) * (1.0f + f);
    const float r = sqrtf(1.0f + 3.0f * q);
    iso = fast_div(q, r + 1.0f);
    dir = 2.0f - r;
}

PDM1_HD SideF32 side_f32(const float u[4]) {
    SideF32 s;
    s.phi = u[0] < 0.0f ? 0.0f : u[0];
    s.jx = u[1]; s.jy = u[2]; s.jz = u[3];
    s.jn = sqrtf(s.jx * s.jx + s.jy * s.jy + s.jz * s.jz);
    const float jmax = float(1.0 - kRealEps) * s.phi;
    if (s.jn > jmax) {   // realizability projection onto |J| = jmax
        const float sc = fast_div(jmax, s.jn);
        s.jx *= sc; s.jy *= sc; s.jz *= sc;
        s.jn = jmax;
    }
    closure_f32(s.phi, s.jn, s.f, s.iso, s.dir);
    if (s.jn > 0.0f) {
        const float inv = fast_div(1.0f, s.jn);
        s.nx = s.jx * inv; s.ny = s.jy * inv; s.nz = s.jz * inv;
    } else {
        s.nx = s.ny = s.nz = 0.0f;
    }
    return s;
}

PDM1_HD void speeds_f32(const SideF32 &s, int axis, float &lmin, float &lmax) {
    if (s.jn < float(kEigEps)) {
        lmin = -0.57735026918962576f;   // -1/sqrt(3)
        lmax = 0.57735026918962576f;
        return;
    }
    float f = s.f, iso = s.iso, dir = s.dir;
    if (s.phi < float(kEigEps)) closure_f32(float(kEigEps), s.jn, f, iso, dir);   // phi floored
    f = fminf(f, float(1.0 - kEigEps));
    const float mu = axis == 0 ? s.nx : (axis == 1 ? s.ny : s.nz);
    const float den = 2.0f + 6.0f * iso;
    float disc = 4.0f * f * f * mu * mu - den * (2.0f * dir * mu * mu - 4.0f * iso);
    disc = fmaxf(disc, 0.0f);
    const float root = sqrtf(disc), inv = fast_div(1.0f, den), c = 2.0f * f * mu;
    lmin = (c - root) * inv;
    lmax = (c + root) * inv;
}

PDM1_HD void side_flux_f32(const SideF32 &s, int axis, float F[4]) {
    const float pd = s.phi * s.dir;
    if (axis == 0) {
        F[0] = s.jx;
        F[1] = s.phi * s.iso + pd * s.nx * s.nx;
        F[2] = pd * s.nx * s.ny;
        F[3] = pd * s.nx * s.nz;
    } else if (axis == 1) {
        F[0] = s.jy;
        F[1] = pd * s.nx * s.ny;
        F[2] = s.phi * s.iso + pd * s.ny * s.ny;
        F[3] = pd * s.ny * s.nz;
    } else {
        F[0] = s.jz;
        F[1] = pd * s.nx * s.nz;
        F[2] = pd * s.ny * s.nz;
        F[3] = s.phi * s.iso + pd * s.nz * s.nz;
    }
}

// L and R: the reconstructed (unprojected) face states; F: the HLL flux.
PDM1_HD void face_flux_f32(const float L[4], const float R[4], int axis, bool unit_speeds,
                                              float F[4]) {
    const SideF32 a = side_f32(L), b = side_f32(R);
    float FL[4], FR[4];
    side_flux_f32(a, axis, FL);
    side_flux_f32(b, axis, FR);
    float sl = -1.0f, sr = 1.0f;
    if (!unit_speeds) {
        float lminl, lmaxl, lminr, lmaxr;
        speeds_f32(a, axis, lminl, lmaxl);
        speeds_f32(b, axis, lminr, lmaxr);
        sl = fminf(fminf(lminl, lminr), 0.0f);
        sr = fmaxf(fmaxf(lmaxl, lmaxr), 0.0f);
    }
    const float den = sr - sl;
    if (!(den > 0.0f)) {
        // |J|/phi rounds to 1 for an exactly directed state: both speeds normal
        // to J are 0 and the fan collapses; the HLL flux tends to the central flux
#pragma unroll
        for (int c = 0; c < 4; ++c) F[c] = 0.5f * (FL[c] + FR[c]);
        return;
    }
    const float inv = fast_div(1.0f, den), sp = sl * sr;
    const float dl[4] = {b.phi - a.phi, b.jx - a.jx, b.jy - a.jy, b.jz - a.jz};
#pragma unroll
    for (int c = 0; c < 4; ++c) F[c] = (sr * FL[c] - sl * FR[c] + sp * dl[c]) * inv;
}

#if defined(__CUDACC__)
// ---------------------------------------------------------------------------
// The single-precision face flux with the two sides of the face in the two
// lanes of sm_100's packed f32x2 arithmetic (x = left state, y = right
// state).  Per lane the arithmetic is that of side_f32 / speeds_f32 /
// side_flux_f32 above: realizability projection, closure through
// iso = (1 - f)(1 + f) / (r + 1) and dir = 2 - r with r = sqrt(1 + 3(1 - f^2)),
// the exact wave speeds from iso and dir, the physical flux.  Square roots,
// reciprocals, comparisons and the HLL combination (which mixes the lanes)
// are per lane.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void face_flux_f32x2(const float L[4], const float R[4], int axis, bool unit_speeds,
                                                float F[4]) {
    const float2 one = pk(1.0f);
    float2 phi = make_float2(L[0] < 0.0f ? 0.0f : L[0], R[0] < 0.0f ? 0.0f : R[0]);
    float2 jx = make_float2(L[1], R[1]), jy = make_float2(L[2], R[2]), jz = make_float2(L[3], R[3]);
    float2 jn = pk_sqrt(pk_fma(jx, jx, pk_fma(jy, jy, pk_mul(jz, jz))));
    const float2 jmax = pk_mul(pk(float(1.0 - kRealEps)), phi);
    if (jn.x > jmax.x || jn.y > jmax.y) {   // realizability projection onto |J| = jmax
        float2 sc = one;
        if (jn.x > jmax.x) { sc.x = fast_div(jmax.x, jn.x); jn.x = jmax.x; }
        if (jn.y > jmax.y) { sc.y = fast_div(jmax.y, jn.y); jn.y = jmax.y; }
        jx = pk_mul(jx, sc); jy = pk_mul(jy, sc); jz = pk_mul(jz, sc);
    }
    // closure: f = |J| / phi (0 without fluence)
    float2 f = pk_mul(jn, pk_rcp(phi));
    f = make_float2(phi.x > 0.0f ? fminf(f.x, 1.0f) : 0.0f, phi.y > 0.0f ? fminf(f.y, 1.0f) : 0.0f);
    const float2 q = pk_mul(pk_fma(pk(-1.0f), f, one), pk_add(f, one));
    const float2 r = pk_sqrt(pk_fma(pk(3.0f), q, one));
    float2 iso = pk_mul(q, pk_rcp(pk_add(r, one)));
    float2 dir = pk_fma(pk(-1.0f), r, pk(2.0f));
    const float2 rjn = make_float2(jn.x > 0.0f ? __fdividef(1.0f, jn.x) : 0.0f,
                                   jn.y > 0.0f ? __fdividef(1.0f, jn.y) : 0.0f);
    const float2 nx = pk_mul(jx, rjn), ny = pk_mul(jy, rjn), nz = pk_mul(jz, rjn);
    const float2 na = axis == 0 ? nx : (axis == 1 ? ny : nz);
    const float2 ja = axis == 0 ? jx : (axis == 1 ? jy : jz);
    // physical fluxes of both sides
    const float2 pdn = pk_mul(pk_mul(phi, dir), na);
    const float2 pi = pk_mul(phi, iso);   // the isotropic pressure on the normal component
    float2 Fc[4];
    Fc[0] = ja;
    Fc[1] = axis == 0 ? pk_fma(pdn, nx, pi) : pk_mul(pdn, nx);
    Fc[2] = axis == 1 ? pk_fma(pdn, ny, pi) : pk_mul(pdn, ny);
    Fc[3] = axis == 2 ? pk_fma(pdn, nz, pi) : pk_mul(pdn, nz);
    float sl = -1.0f, sr = 1.0f;
    if (!unit_speeds) {
        // exact wave speeds; below the eigenvalue floor of phi the closure is
        // taken at phi = 1e-10 (wave_speeds.py:36-103), |J| below it: +-1/sqrt(3)
        if (phi.x < float(kEigEps) || phi.y < float(kEigEps)) {
            if (phi.x < float(kEigEps)) closure_f32(float(kEigEps), jn.x, f.x, iso.x, dir.x);
            if (phi.y < float(kEigEps)) closure_f32(float(kEigEps), jn.y, f.y, iso.y, dir.y);
        }
        f = make_float2(fminf(f.x, float(1.0 - kEigEps)), fminf(f.y, float(1.0 - kEigEps)));
        const float2 den = pk_fma(pk(6.0f), iso, pk(2.0f));
        const float2 mu2 = pk_mul(na, na), fm = pk_mul(f, na);
        const float2 t = pk_fma(pk_mul(pk(2.0f), dir), mu2, pk_mul(pk(-4.0f), iso));
        float2 disc = pk_fma(pk_mul(pk(-1.0f), den), t, pk_mul(pk_mul(pk(4.0f), fm), fm));
        disc = make_float2(fmaxf(disc.x, 0.0f), fmaxf(disc.y, 0.0f));
        const float2 root = pk_sqrt(disc), rden = pk_rcp(den), c = pk_mul(pk(2.0f), fm);
        float2 lmin = pk_mul(pk_fma(pk(-1.0f), root, c), rden);
        float2 lmax = pk_mul(pk_add(c, root), rden);
        const float iso3 = 0.57735026918962576f;   // 1/sqrt(3)
        if (jn.x < float(kEigEps)) { lmin.x = -iso3; lmax.x = iso3; }
        if (jn.y < float(kEigEps)) { lmin.y = -iso3; lmax.y = iso3; }
        sl = fminf(fminf(lmin.x, lmin.y), 0.0f);
        sr = fmaxf(fmaxf(lmax.x, lmax.y), 0.0f);
    }
    const float den = sr - sl;
    if (!(den > 0.0f)) {
        // |J|/phi rounds to 1 for an exactly directed state: both speeds normal
        // to J are 0 and the fan collapses; the HLL flux tends to the central flux
#pragma unroll
        for (int c = 0; c < 4; ++c) F[c] = 0.5f * (Fc[c].x + Fc[c].y);
        return;
    }
    const float inv = fast_div(1.0f, den), sp = sl * sr;
    const float dl[4] = {phi.y - phi.x, jx.y - jx.x, jy.y - jy.x, jz.y - jz.x};
#pragma unroll
    for (int c = 0; c < 4; ++c) F[c] = (sr * Fc[c].x - sl * Fc[c].y + sp * dl[c]) * inv;
}
#endif

// ---------------------------------------------------------------------------
// Coefficient tables (physics/stopping_power.py, coefficient_interpolation.py,
// numpy.interp).  A table is n nodes of (energy, value, PCHIP slope); the
// energies are log-spaced, which gives a first guess of the interval that
// is then corrected by comparisons, so the index is exactly
// numpy.searchsorted(energy, x, side="right") - 1.
// ---------------------------------------------------------------------------
struct TableView {
    const double *E, *v, *slope;
    int n;
    double log_e0, inv_log_step;   // inv_log_step == 0: no log guess
};

PDM1_HD int search_right(const TableView &t, double x) {
    int g;
    if (t.inv_log_step > 0.0 && x > 0.0) {
        double gf = (log(x) - t.log_e0) * t.inv_log_step;
        g = gf < 0.0 ? 0 : (gf > (double)(t.n - 1) ? t.n - 1 : (int)gf);
    } else {
        int lo = 0, hi = t.n;
        while (lo < hi) {
            int mid = (lo + hi) >> 1;
            if (t.E[mid] <= x) lo = mid + 1; else hi = mid;
        }
        return lo - 1;
    }
    while (g >= 0 && t.E[g] > x) --g;
    while (g + 1 < t.n && t.E[g + 1] <= x) ++g;
    return g;
}

PDM1_HD double pchip_eval(const TableView &t, double x) {
    int n = t.n;
    if (x >= t.E[n - 1]) return t.v[n - 1];
    int i = search_right(t, x);
    if (i < 0) i = 0;
    if (i > n - 2) i = n - 2;
    double h = t.E[i + 1] - t.E[i];
    double s = (x - t.E[i]) / h;
    double s2 = s * s;
    double s3 = s2 * s;
    double h00 = 2.0 * s3 - 3.0 * s2 + 1.0;
    double h10 = s3 - 2.0 * s2 + s;
    double h01 = -2.0 * s3 + 3.0 * s2;
    double h11 = s3 - s2;
    return h00 * t.v[i] + h10 * h * t.slope[i] + h01 * t.v[i + 1] + h11 * h * t.slope[i + 1];
}

PDM1_HD double linear_eval(const TableView &t, double x) {
    int n = t.n;
    if (x < t.E[0]) return t.v[0];
    if (x > t.E[n - 1]) return t.v[n - 1];
    int j = search_right(t, x);
    if (j >= n - 1) return t.v[n - 1];
    if (t.E[j] == x) return t.v[j];
    double slope = (t.v[j + 1] - t.v[j]) / (t.E[j + 1] - t.E[j]);
    double r = slope * (x - t.E[j]) + t.v[j];
    if (r != r) {
        r = slope * (x - t.E[j + 1]) + t.v[j + 1];
        if (r != r && t.v[j] == t.v[j + 1]) r = t.v[j];
    }
    return r;
}

// numpy.isclose(a, b) with rtol 1e-5, atol 1e-8; clip of stopping_power.py:151-170
PDM1_HD bool clip_energy(const TableView &t, double &x) {
    double lo = t.E[0], hi = t.E[t.n - 1];
    bool close_lo = fabs(x - lo) <= 1e-8 + 1e-5 * fabs(lo);
    bool close_hi = fabs(x - hi) <= 1e-8 + 1e-5 * fabs(hi);
    if ((x < lo && !close_lo) || (x > hi && !close_hi)) return false;
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return true;
}

}  // namespace pdm1
