/*
 * m1_oracle.c -- CPU restatement of the proton_solver M1 energy march.
 *
 * TEST INFRASTRUCTURE ONLY (see m1_oracle.h).  Every function cites the
 * reference file:line it restates (paths relative to the proton_solver
 * project).  Arithmetic is written in the reference's evaluation order and
 * compiled without FP contraction so that results track the reference's
 * FP64 path to a few ulp; the reference itself runs its WENO and HLL loops
 * under Numba fastmath, so bit equality with it is not expected.
 */
#include "m1_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define EIG_EPS 1.0e-10            /* numerics/wave_speeds.py:10 */
#define WENO_EPS 1.0e-12           /* reconstruction_methods/weno_z.py:8 */
#define REAL_EPS 1.0e-10           /* weno_z.py:10, realizability.py:110 */
#define MEV_TO_JOULE 1.602176634e-13   /* numerics/energy.py:37 */
#define EXP_CLAMP 700.0            /* numerics/energy.py:296-304 */
#define PROTON_REST_ENERGY_MEV 938.27208816   /* physics/scattering.py:21 */
#define ROSSI_ES_MEV 15.0                      /* physics/scattering.py:22 */

static __thread char g_err[256];

/* ======================================================================
 * exp in double-double arithmetic
 *
 * The reference calls math.exp / numpy.exp.  The oracle evaluates exp with
 * its own routine so that the CUDA path, which carries an identical routine,
 * reproduces every bit: Cody-Waite reduction x = k ln2 + r with ln2 held as
 * a double-double, exp(r / 2^10) by a degree-9 Taylor series in
 * double-double (Dekker/Knuth error-free sums and FMA products), ten
 * squarings, and a final scaling by 2^k.  The double-double result is good
 * to about 1e-29 relative, so the returned double is the correctly rounded
 * exp except in rare ties.
 * ==================================================================== */

typedef struct { double hi, lo; } dd_t;

static dd_t dd_quick(double a, double b) { dd_t r; r.hi = a + b; r.lo = b - (r.hi - a); return r; }

static dd_t dd_add(dd_t a, dd_t b)
{
    double s = a.hi + b.hi;
    double bb = s - a.hi;
    double e = (a.hi - (s - bb)) + (b.hi - bb);
    e += a.lo + b.lo;
    return dd_quick(s, e);
}

static dd_t dd_mul(dd_t a, dd_t b)
{
    double p = a.hi * b.hi;
    double e = fma(a.hi, b.hi, -p);
    e += a.hi * b.lo + a.lo * b.hi;
    return dd_quick(p, e);
}

static dd_t dd_div_d(double a, double b)
{
    double q1 = a / b;
    double p = q1 * b;
    double e = fma(q1, b, -p);
    double rem = (a - p) - e;
    return dd_quick(q1, rem / b);
}

static double dd_exp(double x)
{
    if (x != x) return x;
    if (x > 709.782712893384) return INFINITY;
    if (x < -745.2) return 0.0;
    const double ln2_hi = 0.6931471805599453094;      /* nearest double to ln 2 */
    const double ln2_lo = 2.3190468138462996e-17;     /* ln 2 - ln2_hi */
    double k = rint(x * 1.4426950408889634);
    double p = k * ln2_hi;
    double pe = fma(k, ln2_hi, -p);
    double s = x - p;                  /* exact: x and p are within a factor 2 */
    double t = -pe - k * ln2_lo;
    dd_t r = dd_quick(s, t);
    r.hi *= 0x1p-10;
    r.lo *= 0x1p-10;
    /* Horner: sum_{n=0..9} r^n / n! */
    double fact[10] = {1.0, 1.0, 2.0, 6.0, 24.0, 120.0, 720.0, 5040.0, 40320.0, 362880.0};
    dd_t acc = dd_div_d(1.0, fact[9]);
    for (int n = 8; n >= 0; --n) acc = dd_add(dd_mul(acc, r), dd_div_d(1.0, fact[n]));
    for (int q = 0; q < 10; ++q) acc = dd_mul(acc, acc);
    return ldexp(acc.hi + acc.lo, (int)k);
}

static int fail(int code, const char *msg)
{
    snprintf(g_err, sizeof g_err, "%s", msg);
    return code;
}

const char *orc_last_error(void) { return g_err; }

double orc_exp(double x) { return dd_exp(x); }

void orc_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ======================================================================
 * Tables
 * ==================================================================== */

typedef struct {
    int n;
    double *E, *v, *slope;
} table_t;

typedef struct {
    table_t sp, tr, nuc;
    double density, X0;
} mat_t;

enum { ORC_SCHEME_WENO_Z = 0, ORC_SCHEME_FIRST_ORDER = 1, ORC_SCHEME_MUSCL = 2, ORC_SCHEME_WENO3 = 3 };

struct orc_problem {
    orc_problem_desc d;
    double dx, dy, dz;
    int nm;
    mat_t *mats;
    int32_t *ids;
    double *spatial;     /* n_protons * normalised profile, (nx, ny) */
    double *schedule;    /* prescribed energies E_0 .. E_{n-1} (orc_set_schedule), or NULL */
    int n_schedule;
};

static double sign_of(double x) { return (x > 0.0) - (x < 0.0); }

/* physics/stopping_power.py:30-54 */
static double pchip_endpoint_slope(double h0, double h1, double d0, double d1)
{
    double slope = ((2.0 * h0 + h1) * d0 - h0 * d1) / (h0 + h1);
    if (sign_of(slope) != sign_of(d0)) return 0.0;
    if (sign_of(d0) != sign_of(d1) && fabs(slope) > 3.0 * fabs(d0)) return 3.0 * d0;
    return slope;
}

/* physics/stopping_power.py:94-138, coefficient_interpolation.py:19-48 */
static void pchip_slopes(table_t *t)
{
    int n = t->n;
    double *h = malloc(sizeof(double) * (n - 1));
    double *delta = malloc(sizeof(double) * (n - 1));
    for (int i = 0; i < n - 1; ++i) {
        h[i] = t->E[i + 1] - t->E[i];
        delta[i] = (t->v[i + 1] - t->v[i]) / h[i];
    }
    for (int i = 0; i < n; ++i) t->slope[i] = 0.0;
    if (n == 2) {
        t->slope[0] = t->slope[1] = delta[0];
    } else {
        for (int k = 1; k < n - 1; ++k) {
            if (delta[k - 1] * delta[k] > 0.0) {
                double w1 = 2.0 * h[k] + h[k - 1];
                double w2 = h[k] + 2.0 * h[k - 1];
                t->slope[k] = (w1 + w2) / (w1 / delta[k - 1] + w2 / delta[k]);
            }
        }
        t->slope[0] = pchip_endpoint_slope(h[0], h[1], delta[0], delta[1]);
        t->slope[n - 1] = pchip_endpoint_slope(h[n - 2], h[n - 3], delta[n - 2], delta[n - 3]);
    }
    free(h);
    free(delta);
}

/* numpy.searchsorted(E, x, side="right") - 1 */
static int search_right(const double *E, int n, double x)
{
    int lo = 0, hi = n;            /* first index with E[i] > x */
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (E[mid] <= x) lo = mid + 1; else hi = mid;
    }
    return lo - 1;
}

/* Cubic Hermite evaluation, physics/stopping_power.py:185-228
 * (same arithmetic as coefficient_interpolation.py:51-70). */
static double pchip_eval(const table_t *t, double x)
{
    int n = t->n;
    if (x >= t->E[n - 1]) return t->v[n - 1];
    int i = search_right(t->E, n, x);
    if (i < 0) i = 0;
    if (i > n - 2) i = n - 2;
    double h = t->E[i + 1] - t->E[i];
    double s = (x - t->E[i]) / h;
    double s2 = s * s;
    double s3 = s2 * s;
    double h00 = 2.0 * s3 - 3.0 * s2 + 1.0;
    double h10 = s3 - 2.0 * s2 + s;
    double h01 = -2.0 * s3 + 3.0 * s2;
    double h11 = s3 - s2;
    return h00 * t->v[i] + h10 * h * t->slope[i] + h01 * t->v[i + 1] + h11 * h * t->slope[i + 1];
}

/* numpy.interp for one abscissa (numpy core compiled_base.c arr_interp). */
static double linear_eval(const table_t *t, double x)
{
    int n = t->n;
    const double *E = t->E, *v = t->v;
    if (x < E[0]) return v[0];
    if (x > E[n - 1]) return v[n - 1];
    int j = search_right(E, n, x);
    if (j >= n - 1) return v[n - 1];
    if (E[j] == x) return v[j];
    double slope = (v[j + 1] - v[j]) / (E[j + 1] - E[j]);
    double r = slope * (x - E[j]) + v[j];
    if (isnan(r)) {
        r = slope * (x - E[j + 1]) + v[j + 1];
        if (isnan(r) && v[j] == v[j + 1]) r = v[j];
    }
    return r;
}

/* numpy.isclose(a, b) with rtol=1e-5, atol=1e-8 */
static int np_isclose(double a, double b) { return fabs(a - b) <= 1e-8 + 1e-5 * fabs(b); }

/* Range check + clip of physics/stopping_power.py:151-170 (and the same
 * block in scattering.py:75-97, nuclear.py:103-121). */
static int clip_energy(const table_t *t, double *x)
{
    double lo = t->E[0], hi = t->E[t->n - 1];
    if ((*x < lo && !np_isclose(*x, lo)) || (*x > hi && !np_isclose(*x, hi)))
        return fail(ORC_ERR_RANGE, "energy outside coefficient table range");
    if (*x < lo) *x = lo;
    if (*x > hi) *x = hi;
    return ORC_OK;
}

/* physics/stopping_power.py:141-228 */
static int stopping_power(const mat_t *m, double E, double *out)
{
    int rc = clip_energy(&m->sp, &E);
    if (rc) return rc;
    if (E == m->sp.E[m->sp.n - 1]) { *out = m->sp.v[m->sp.n - 1]; return ORC_OK; }
    *out = pchip_eval(&m->sp, E);
    return ORC_OK;
}

/* physics/scattering.py:137-153 */
static double rossi_coefficient(const mat_t *m, double E)
{
    double e = E > 1.0e-8 ? E : 1.0e-8;
    double M = PROTON_REST_ENERGY_MEV;
    double pv = e * (e + 2.0 * M) / (e + M);
    double r = ROSSI_ES_MEV / pv;
    return r * r / m->X0;
}

/* physics/scattering.py:65-116 (Wentzel) and 155-185 (model dispatch) */
static int transport_coefficient(const orc_problem *p, const mat_t *m, double E, double *out)
{
    if (p->d.scattering == ORC_SCATTER_OFF) { *out = 0.0; return ORC_OK; }
    if (p->d.scattering == ORC_SCATTER_ROSSI) { *out = rossi_coefficient(m, E); return ORC_OK; }
    int rc = clip_energy(&m->tr, &E);
    if (rc) return rc;
    *out = p->d.interpolation == ORC_INTERP_LINEAR ? linear_eval(&m->tr, E) : pchip_eval(&m->tr, E);
    return ORC_OK;
}

/* physics/nuclear.py:94-138 */
static int nuclear_coefficient(const orc_problem *p, const mat_t *m, double E, double *out)
{
    int rc = clip_energy(&m->nuc, &E);
    if (rc) return rc;
    *out = p->d.interpolation == ORC_INTERP_LINEAR ? linear_eval(&m->nuc, E) : pchip_eval(&m->nuc, E);
    return ORC_OK;
}

/* Two-point Gauss-Legendre optical depths over [E - dE, E]:
 * physics/scattering.py:267-306, physics/nuclear.py:202-233,
 * dispatch numerics/energy.py:234-270. */
static int optical_depths(const orc_problem *p, const mat_t *m, double E, double dE,
                          double *tau_s, double *tau_n)
{
    *tau_s = 0.0;
    *tau_n = 0.0;
    if (dE <= 0.0) return ORC_OK;
    double mid = E - 0.5 * dE;
    double half = 0.5 * dE;
    double off = half / sqrt(3.0);
    if (p->d.scattering != ORC_SCATTER_OFF) {
        double a, b, sa, sb;
        int rc;
        if ((rc = transport_coefficient(p, m, mid - off, &a))) return rc;
        if ((rc = stopping_power(m, mid - off, &sa))) return rc;
        if ((rc = transport_coefficient(p, m, mid + off, &b))) return rc;
        if ((rc = stopping_power(m, mid + off, &sb))) return rc;
        *tau_s = half * (a / sa + b / sb);
    }
    if (p->d.nuclear) {
        double a, b, sa, sb;
        int rc;
        if ((rc = nuclear_coefficient(p, m, mid - off, &a))) return rc;
        if ((rc = stopping_power(m, mid - off, &sa))) return rc;
        if ((rc = nuclear_coefficient(p, m, mid + off, &b))) return rc;
        if ((rc = stopping_power(m, mid + off, &sb))) return rc;
        *tau_n = half * (a / sa + b / sb);
    }
    return ORC_OK;
}

/* ======================================================================
 * Scalar kernels
 * ==================================================================== */

/* reconstruction_methods/weno_z.py:12-87 */
double orc_weno_left(const double v[5])
{
    double v0 = v[0], v1 = v[1], v2 = v[2], v3 = v[3], v4 = v[4];
    double p0 = v0 / 3.0 - 7.0 * v1 / 6.0 + 11.0 * v2 / 6.0;
    double p1 = -v1 / 6.0 + 5.0 * v2 / 6.0 + v3 / 3.0;
    double p2 = v2 / 3.0 + 5.0 * v3 / 6.0 - v4 / 6.0;
    double a, b;
    a = v0 - 2.0 * v1 + v2; b = v0 - 4.0 * v1 + 3.0 * v2;
    double beta0 = 13.0 / 12.0 * (a * a) + 0.25 * (b * b);
    a = v1 - 2.0 * v2 + v3; b = v1 - v3;
    double beta1 = 13.0 / 12.0 * (a * a) + 0.25 * (b * b);
    a = v2 - 2.0 * v3 + v4; b = 3.0 * v2 - 4.0 * v3 + v4;
    double beta2 = 13.0 / 12.0 * (a * a) + 0.25 * (b * b);
    double tau5 = fabs(beta2 - beta0);
    double r0 = tau5 / (beta0 + WENO_EPS);
    double r1 = tau5 / (beta1 + WENO_EPS);
    double r2 = tau5 / (beta2 + WENO_EPS);
    double al0 = 0.1 * (1.0 + r0 * r0);
    double al1 = 0.6 * (1.0 + r1 * r1);
    double al2 = 0.3 * (1.0 + r2 * r2);
    double s = al0 + al1 + al2;
    double w0 = al0 / s, w1 = al1 / s, w2 = al2 / s;
    return w0 * p0 + w1 * p1 + w2 * p2;
}

/* numerics/realizability.py:132-176 (same as weno_z.py:90-129) */
void orc_project(double u[4])
{
    double phi = u[0];
    if (phi < 0.0) phi = 0.0;
    double jx = u[1], jy = u[2], jz = u[3];
    double jn = sqrt(jx * jx + jy * jy + jz * jz);
    double jmax = (1.0 - REAL_EPS) * phi;
    if (jn > jmax) {
        double s = jmax / jn;
        jx *= s; jy *= s; jz *= s;
    }
    u[0] = phi; u[1] = jx; u[2] = jy; u[3] = jz;
}

/* numerics/flux.py:63-135 == numerics/wave_speeds.py:36-103 */
static void eigen_core(double phi, double jx, double jy, double jz, double jn, int axis,
                       double *lmin, double *lmax)
{
    double iso = 1.0 / sqrt(3.0);
    if (phi < EIG_EPS) phi = EIG_EPS;
    if (jn < EIG_EPS) { *lmin = -iso; *lmax = iso; return; }
    double f = jn / phi;
    if (f < 0.0) f = 0.0;
    else if (f > 1.0 - EIG_EPS) f = 1.0 - EIG_EPS;
    double jnormal = axis == 0 ? jx : (axis == 1 ? jy : jz);
    double mu = jnormal / jn;
    double chi = (5.0 - 2.0 * sqrt(4.0 - 3.0 * f * f)) / 3.0;
    double den = 5.0 - 3.0 * chi;
    double disc = 4.0 * f * f * mu * mu - den * (mu * mu * (3.0 * chi - 1.0) - 2.0 * (1.0 - chi));
    if (disc < 0.0) disc = 0.0;
    double root = sqrt(disc);
    *lmin = (2.0 * f * mu - root) / den;
    *lmax = (2.0 * f * mu + root) / den;
}

/* numerics/wave_speeds.py:12-105 */
void orc_eigenvalues(const double u[4], int axis, double *lmin, double *lmax)
{
    double jn = sqrt(u[1] * u[1] + u[2] * u[2] + u[3] * u[3]);
    eigen_core(u[0], u[1], u[2], u[3], jn, axis, lmin, lmax);
}

typedef struct { double jn, nx, ny, nz, iso, dir; } closure_t;

/* numerics/flux.py:10-61 */
static closure_t closure(double phi, double jx, double jy, double jz)
{
    closure_t c;
    c.jn = sqrt(jx * jx + jy * jy + jz * jz);
    double f;
    if (phi > 0.0) {
        f = c.jn / phi;
        if (f < 0.0) f = 0.0;
        else if (f > 1.0) f = 1.0;
    } else {
        f = 0.0;
    }
    double chi = (5.0 - 2.0 * sqrt(4.0 - 3.0 * f * f)) / 3.0;
    if (c.jn > 0.0) {
        c.nx = jx / c.jn; c.ny = jy / c.jn; c.nz = jz / c.jn;
    } else {
        c.nx = c.ny = c.nz = 0.0;
    }
    c.iso = 0.5 * (1.0 - chi);
    c.dir = 0.5 * (3.0 * chi - 1.0);
    return c;
}

/* numerics/flux.py:203-304: physical flux of one state along an axis */
static void physical_flux(const double u[4], const closure_t *c, int axis, double F[4])
{
    double phi = u[0];
    if (axis == 0) {
        F[0] = u[1];
        F[1] = phi * (c->iso + c->dir * c->nx * c->nx);
        F[2] = phi * c->dir * c->nx * c->ny;
        F[3] = phi * c->dir * c->nx * c->nz;
    } else if (axis == 1) {
        F[0] = u[2];
        F[1] = phi * c->dir * c->nx * c->ny;
        F[2] = phi * (c->iso + c->dir * c->ny * c->ny);
        F[3] = phi * c->dir * c->ny * c->nz;
    } else {
        F[0] = u[3];
        F[1] = phi * c->dir * c->nx * c->nz;
        F[2] = phi * c->dir * c->ny * c->nz;
        F[3] = phi * (c->iso + c->dir * c->nz * c->nz);
    }
}

/* numerics/flux.py:137-386 (fused closure, exact speeds, HLL) */
void orc_hll_flux(const double L[4], const double R[4], int axis, int wave_speeds, double F[4])
{
    closure_t cl = closure(L[0], L[1], L[2], L[3]);
    closure_t cr = closure(R[0], R[1], R[2], R[3]);
    double FL[4], FR[4];
    physical_flux(L, &cl, axis, FL);
    physical_flux(R, &cr, axis, FR);
    double sl, sr;
    if (wave_speeds == ORC_SPEEDS_EXACT) {
        double lminl, lmaxl, lminr, lmaxr;
        eigen_core(L[0], L[1], L[2], L[3], cl.jn, axis, &lminl, &lmaxl);
        eigen_core(R[0], R[1], R[2], R[3], cr.jn, axis, &lminr, &lmaxr);
        sl = lminr < lminl ? lminr : lminl;
        sr = lmaxr > lmaxl ? lmaxr : lmaxl;
        if (sl > 0.0) sl = 0.0;
        if (sr < 0.0) sr = 0.0;
    } else {
        sl = -1.0;
        sr = 1.0;
    }
    double den = sr - sl;
    double sp = sl * sr;
    for (int c = 0; c < 4; ++c)
        F[c] = (sr * FL[c] - sl * FR[c] + sp * (R[c] - L[c])) / den;
}

/* ======================================================================
 * Problem setup
 * ==================================================================== */

static int copy_table(table_t *t, int n, const double *E, const double *v)
{
    if (n < 2 || !E || !v) return fail(ORC_ERR_ARG, "coefficient table needs >= 2 nodes");
    t->n = n;
    t->E = malloc(sizeof(double) * n);
    t->v = malloc(sizeof(double) * n);
    t->slope = malloc(sizeof(double) * n);
    if (!t->E || !t->v || !t->slope) return fail(ORC_ERR_ALLOC, "out of memory");
    memcpy(t->E, E, sizeof(double) * n);
    memcpy(t->v, v, sizeof(double) * n);
    pchip_slopes(t);
    return ORC_OK;
}

/* numerics/boundary.py:11-27: exact cell averages of a 1-D Gaussian */
static void gaussian_cell_average(int n, double length, double mean, double sigma, double *g)
{
    double h = length / n;
    double scale = sqrt(2.0) * sigma;
    for (int i = 0; i < n; ++i) {
        double c = ((double)i + 0.5) * h - 0.5 * length;
        double lo = (c - 0.5 * h - mean) / scale;
        double hi = (c + 0.5 * h - mean) / scale;
        g[i] = 0.5 * (erf(hi) - erf(lo)) / h;
    }
}

/* numpy's pairwise summation (numpy/_core/src/umath/loops_utils.h.src),
 * used by ndarray.sum on the contiguous profile in boundary.py:50. */
static double pairwise_sum(const double *a, size_t n)
{
    if (n < 8) {
        double res = 0.0;
        for (size_t i = 0; i < n; ++i) res += a[i];
        return res;
    }
    if (n <= 128) {
        double r[8];
        for (int q = 0; q < 8; ++q) r[q] = a[q];
        size_t i;
        for (i = 8; i < n - (n % 8); i += 8)
            for (int q = 0; q < 8; ++q) r[q] += a[i + q];
        double res = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
        for (; i < n; ++i) res += a[i];
        return res;
    }
    size_t n2 = n / 2;
    n2 -= n2 % 8;
    return pairwise_sum(a, n2) + pairwise_sum(a + n2, n - n2);
}

/* numerics/boundary.py:30-60 and 68-80 */
static int build_inflow(orc_problem *p)
{
    const orc_problem_desc *d = &p->d;
    int nx = d->nx, ny = d->ny;
    double *gx = malloc(sizeof(double) * nx), *gy = malloc(sizeof(double) * ny);
    gaussian_cell_average(nx, d->lx, d->center_x, d->sigma_x, gx);
    gaussian_cell_average(ny, d->ly, d->center_y, d->sigma_y, gy);
    double cut2 = d->cutoff_sigma * d->cutoff_sigma;
    for (int i = 0; i < nx; ++i) {
        double x = ((double)i + 0.5) * p->dx - 0.5 * d->lx;
        double rx = (x - d->center_x) / d->sigma_x;
        for (int j = 0; j < ny; ++j) {
            double y = ((double)j + 0.5) * p->dy - 0.5 * d->ly;
            double ry = (y - d->center_y) / d->sigma_y;
            double r2 = rx * rx + ry * ry;
            double v = r2 <= cut2 ? gx[i] * gy[j] : 0.0;
            p->spatial[i * ny + j] = v;
        }
    }
    free(gx);
    free(gy);
    double mass = pairwise_sum(p->spatial, (size_t)nx * ny) * p->dx * p->dy;
    if (!isfinite(mass) || mass <= 0.0)
        return fail(ORC_ERR_NO_BEAM, "Beam profile has zero or non-finite mass on the domain.");
    for (int i = 0; i < nx * ny; ++i) p->spatial[i] = d->n_protons * (p->spatial[i] / mass);
    return ORC_OK;
}

int orc_set_schedule(orc_problem *p, const double *energies, int n)
{
    free(p->schedule);
    p->schedule = NULL;
    p->n_schedule = 0;
    if (n <= 0) return ORC_OK;
    p->schedule = malloc(sizeof(double) * n);
    if (!p->schedule) return fail(ORC_ERR_ARG, "schedule: out of memory");
    memcpy(p->schedule, energies, sizeof(double) * n);
    p->n_schedule = n;
    return ORC_OK;
}

void orc_problem_destroy(orc_problem *p)
{
    if (!p) return;
    if (p->mats) {
        for (int m = 0; m < p->nm; ++m) {
            table_t *ts[3] = {&p->mats[m].sp, &p->mats[m].tr, &p->mats[m].nuc};
            for (int t = 0; t < 3; ++t) { free(ts[t]->E); free(ts[t]->v); free(ts[t]->slope); }
        }
        free(p->mats);
    }
    free(p->ids);
    free(p->spatial);
    free(p->schedule);
    free(p);
}

int orc_problem_create(const orc_problem_desc *desc, orc_problem **out)
{
    *out = NULL;
    if (!desc || desc->nx <= 0 || desc->ny <= 0 || desc->nz <= 0 || desc->n_materials <= 0 ||
        !desc->materials || !desc->ids)
        return fail(ORC_ERR_ARG, "invalid problem description");
    orc_problem *p = calloc(1, sizeof *p);
    if (!p) return fail(ORC_ERR_ALLOC, "out of memory");
    p->d = *desc;
    p->d.materials = NULL;
    p->d.ids = NULL;
    p->dx = desc->lx / desc->nx;
    p->dy = desc->ly / desc->ny;
    p->dz = desc->lz / desc->nz;
    p->nm = desc->n_materials;
    p->mats = calloc(p->nm, sizeof(mat_t));
    size_t n = (size_t)desc->nx * desc->ny * desc->nz;
    p->ids = malloc(sizeof(int32_t) * n);
    p->spatial = malloc(sizeof(double) * desc->nx * desc->ny);
    if (!p->mats || !p->ids || !p->spatial) { orc_problem_destroy(p); return fail(ORC_ERR_ALLOC, "out of memory"); }
    for (size_t c = 0; c < n; ++c) {
        if (desc->ids[c] < 0 || desc->ids[c] >= p->nm) {
            orc_problem_destroy(p);
            return fail(ORC_ERR_ARG, "material id out of range");
        }
        p->ids[c] = desc->ids[c];
    }
    for (int m = 0; m < p->nm; ++m) {
        const orc_material_desc *md = &desc->materials[m];
        int rc;
        if ((rc = copy_table(&p->mats[m].sp, md->n_sp, md->sp_energy, md->sp_value)) ||
            (rc = copy_table(&p->mats[m].tr, md->n_tr, md->tr_energy, md->tr_value)) ||
            (rc = copy_table(&p->mats[m].nuc, md->n_nuc, md->nuc_energy, md->nuc_value))) {
            orc_problem_destroy(p);
            return rc;
        }
        p->mats[m].density = md->density;
        p->mats[m].X0 = md->radiation_length;
    }
    int rc = build_inflow(p);
    if (rc) { orc_problem_destroy(p); return rc; }
    *out = p;
    return ORC_OK;
}

/* ======================================================================
 * Public coefficient wrappers
 * ==================================================================== */

int orc_stopping_power(const orc_problem *p, int m, double E, double *out)
{
    if (m < 0 || m >= p->nm) return fail(ORC_ERR_ARG, "bad material");
    return stopping_power(&p->mats[m], E, out);
}

int orc_transport_coefficient(const orc_problem *p, int m, double E, double *out)
{
    if (m < 0 || m >= p->nm) return fail(ORC_ERR_ARG, "bad material");
    return transport_coefficient(p, &p->mats[m], E, out);
}

int orc_nuclear_coefficient(const orc_problem *p, int m, double E, double *out)
{
    if (m < 0 || m >= p->nm) return fail(ORC_ERR_ARG, "bad material");
    return nuclear_coefficient(p, &p->mats[m], E, out);
}

int orc_optical_depths(const orc_problem *p, int m, double E, double dE, double *ts, double *tn)
{
    if (m < 0 || m >= p->nm) return fail(ORC_ERR_ARG, "bad material");
    return optical_depths(p, &p->mats[m], E, dE, ts, tn);
}

/* numerics/boundary.py:82-114: energy density of the Gaussian spectrum */
static double energy_density(const orc_problem *p, double E)
{
    double de = E - p->d.energy;
    double s = p->d.energy_spread;
    return dd_exp(-(de * de) / (2.0 * (s * s))) / (sqrt(2.0 * M_PI) * s);
}

void orc_inflow_spatial(const orc_problem *p, double *spatial)
{
    memcpy(spatial, p->spatial, sizeof(double) * p->d.nx * p->d.ny);
}

/* ======================================================================
 * Domains: the full grid or a moving box (numerics/moving_active_domain.py)
 * ==================================================================== */

typedef struct {
    int nx, ny, nz;
    double dx, dy, dz;
    const int32_t *ids;     /* contiguous (nx, ny, nz) */
    const double *spatial;  /* inflow profile on this domain's z-min face, (nx, ny) */
} domain_t;

#define IDX(c, i, j, k) ((((size_t)(c) * nx + (i)) * ny + (j)) * nz + (k))

/* numerics/boundary.py:82-114 on a domain */
static void inflow_state(const orc_problem *p, const domain_t *dm, double E, double *st)
{
    double ed = energy_density(p, E);
    double rf = dd_exp(-(p->d.angular_spread * p->d.angular_spread));
    size_t n2 = (size_t)dm->nx * dm->ny;
    for (size_t c = 0; c < n2; ++c) {
        double phi = dm->spatial[c] * ed;
        st[c] = phi;
        st[n2 + c] = 0.0;
        st[2 * n2 + c] = 0.0;
        st[3 * n2 + c] = rf * phi;
    }
}

void orc_inflow_state(const orc_problem *p, double E, double *st)
{
    domain_t dm = {p->d.nx, p->d.ny, p->d.nz, p->dx, p->dy, p->dz, p->ids, p->spatial};
    inflow_state(p, &dm, E, st);
}

/* z-min ghost cells, numerics/boundary.py:117-320: the inflow state itself for
 * first order (ng = 1, 205-212); the quadratic through U_in and the first two
 * cell averages for MUSCL / WENO3 (ng = 2, 214-245); the quartic through U_in
 * and four cell averages for WENO-Z (ng = 3, 247-320).  Ghost g (0-based
 * from the face) is G[g]; unused ghosts are zero. */
static void zmin_ghosts(const domain_t *dm, int scheme, const double *U, const double *bc, double *G)
{
    int nx = dm->nx, ny = dm->ny, nz = dm->nz;
    size_t n2 = (size_t)nx * ny;
    memset(G, 0, sizeof(double) * 3 * 4 * n2);
    for (int c = 0; c < 4; ++c)
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) {
                double ui = bc[c * n2 + (size_t)i * ny + j];
                size_t o = c * n2 + (size_t)i * ny + j;
                if (scheme == ORC_SCHEME_FIRST_ORDER) {
                    G[o] = ui;
                } else if (scheme == ORC_SCHEME_MUSCL || scheme == ORC_SCHEME_WENO3) {
                    double u0 = U[IDX(c, i, j, 0)], u1 = U[IDX(c, i, j, 1)];
                    G[0 * 4 * n2 + o] = 3.0 * ui - 2.5 * u0 + 0.5 * u1;
                    G[1 * 4 * n2 + o] = 9.0 * ui - 10.5 * u0 + 2.5 * u1;
                } else {
                    double u0 = U[IDX(c, i, j, 0)], u1 = U[IDX(c, i, j, 1)];
                    double u2 = U[IDX(c, i, j, 2)], u3 = U[IDX(c, i, j, 3)];
                    G[0 * 4 * n2 + o] = 5.0 * ui - (77.0 / 12.0) * u0 + (43.0 / 12.0) * u1
                                        - (17.0 / 12.0) * u2 + 0.25 * u3;
                    G[1 * 4 * n2 + o] = 25.0 * ui - (505.0 / 12.0) * u0 + (335.0 / 12.0) * u1
                                        - (145.0 / 12.0) * u2 + (9.0 / 4.0) * u3;
                    G[2 * 4 * n2 + o] = 75.0 * ui - (545.0 / 4.0) * u0 + (395.0 / 4.0) * u1
                                        - (181.0 / 4.0) * u2 + (35.0 / 4.0) * u3;
                }
            }
}

/* reconstruction_methods/weno3.py:15-62 (WENO3-Z, p = 2) */
double orc_weno3_left(const double v[3])
{
    double p0 = -0.5 * v[0] + 1.5 * v[1];
    double p1 = 0.5 * v[1] + 0.5 * v[2];
    double beta0 = (v[1] - v[0]) * (v[1] - v[0]);
    double beta1 = (v[2] - v[1]) * (v[2] - v[1]);
    double tau3 = fabs(beta1 - beta0);
    double r0 = tau3 / (beta0 + 1.0e-12);
    double r1 = tau3 / (beta1 + 1.0e-12);
    double alpha0 = (1.0 / 3.0) * (1.0 + r0 * r0);
    double alpha1 = (2.0 / 3.0) * (1.0 + r1 * r1);
    double s = alpha0 + alpha1;
    double w0 = alpha0 / s, w1 = alpha1 / s;
    return w0 * p0 + w1 * p1;
}

/* reconstruction_methods/muscl.py:22-44: minmod-limited faces of the centre cell */
void orc_muscl_faces(double vm, double v0, double vp, double *minus, double *plus)
{
    double a = v0 - vm, b = vp - v0, slope = 0.0;
    if (a * b > 0.0) slope = (a > 0.0 ? 1.0 : -1.0) * (fabs(a) < fabs(b) ? fabs(a) : fabs(b));
    *minus = v0 - 0.5 * slope;
    *plus = v0 + 0.5 * slope;
}

/* Value of the ghost-extended state (numerics/boundary.py:117-399):
 * zero-gradient on x, y and z-max, extrapolated ghosts at z-min. */
static inline double ext_value(const domain_t *dm, const double *U, const double *G, int c, int i,
                               int j, int k)
{
    int nx = dm->nx, ny = dm->ny, nz = dm->nz;
    if (i < 0) i = 0;
    if (i >= nx) i = nx - 1;
    if (j < 0) j = 0;
    if (j >= ny) j = ny - 1;
    if (k >= nz) k = nz - 1;
    if (k < 0) {
        size_t n2 = (size_t)nx * ny;
        return G[(size_t)(-k - 1) * 4 * n2 + c * n2 + (size_t)i * ny + j];
    }
    return U[IDX(c, i, j, k)];
}

/* Reconstructed, projected left/right states at one interface and the HLL
 * flux through it (weno_z.py:131-321 + flux.py:137-386).  (i,j,k) is the
 * cell on the + side of the interface. */
static void face_flux(const domain_t *dm, int scheme, const double *U, const double *G, int axis, int i,
                      int j, int k, int wave_speeds, double F[4])
{
    double L[4], R[4];
    int di = axis == 0, dj = axis == 1, dk = axis == 2;
    for (int c = 0; c < 4; ++c) {
        /* w[s]: cells i-3 .. i+2 along the axis (the face lies between w[2] and w[3]) */
        double w[6];
        for (int s = 0; s < 6; ++s) {
            int o = s - 3;
            w[s] = ext_value(dm, U, G, c, i + o * di, j + o * dj, k + o * dk);
        }
        if (scheme == ORC_SCHEME_FIRST_ORDER) {          /* first_order.py:66-111 */
            L[c] = w[2];
            R[c] = w[3];
        } else if (scheme == ORC_SCHEME_MUSCL) {         /* muscl.py:86-145 */
            double lo, hi;
            orc_muscl_faces(w[1], w[2], w[3], &lo, &hi);
            L[c] = hi;
            orc_muscl_faces(w[2], w[3], w[4], &lo, &hi);
            R[c] = lo;
        } else if (scheme == ORC_SCHEME_WENO3) {         /* weno3.py:108-171 */
            double vl[3] = {w[1], w[2], w[3]};
            double vr[3] = {w[4], w[3], w[2]};
            L[c] = orc_weno3_left(vl);
            R[c] = orc_weno3_left(vr);
        } else {                                          /* weno_z.py:131-321 */
            double vl[5] = {w[0], w[1], w[2], w[3], w[4]};
            double vr[5] = {w[5], w[4], w[3], w[2], w[1]};
            L[c] = orc_weno_left(vl);
            R[c] = orc_weno_left(vr);
        }
    }
    orc_project(L);
    orc_project(R);
    orc_hll_flux(L, R, axis, wave_speeds, F);
}

/* numerics/spatial.py:104-252 (active_domain=False): rhs = -div F */
static int spatial_operator(const orc_problem *p, const domain_t *dm, const double *U,
                            const double *bc, double *rhs)
{
    int nx = dm->nx, ny = dm->ny, nz = dm->nz;
    const int scheme = p->d.spatial_scheme;
    if (scheme == ORC_SCHEME_WENO_Z && nz < 4)
        return fail(ORC_ERR_ARG, "WENO-Z inflow extrapolation requires at least four z cells.");
    if ((scheme == ORC_SCHEME_MUSCL || scheme == ORC_SCHEME_WENO3) && nz < 2)
        return fail(ORC_ERR_ARG, "WENO3 inflow extrapolation requires at least two z cells.");
    size_t n2 = (size_t)nx * ny;
    double *G = malloc(sizeof(double) * 3 * 4 * n2);
    double *Fx = malloc(sizeof(double) * 4 * (size_t)(nx + 1) * ny * nz);
    double *Fy = malloc(sizeof(double) * 4 * (size_t)nx * (ny + 1) * nz);
    double *Fz = malloc(sizeof(double) * 4 * n2 * (nz + 1));
    if (!G || !Fx || !Fy || !Fz) { free(G); free(Fx); free(Fy); free(Fz); return fail(ORC_ERR_ALLOC, "oom"); }
    zmin_ghosts(dm, scheme, U, bc, G);
    int ws = p->d.wave_speeds;
    size_t sx = (size_t)(nx + 1) * ny * nz, sy = (size_t)nx * (ny + 1) * nz, sz = n2 * (nz + 1);
#pragma omp parallel for schedule(static)
    for (int i = 0; i <= nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                double F[4];
                face_flux(dm, scheme, U, G, 0, i, j, k, ws, F);
                size_t o = ((size_t)i * ny + j) * nz + k;
                for (int c = 0; c < 4; ++c) Fx[c * sx + o] = F[c];
            }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j <= ny; ++j)
            for (int k = 0; k < nz; ++k) {
                double F[4];
                face_flux(dm, scheme, U, G, 1, i, j, k, ws, F);
                size_t o = ((size_t)i * (ny + 1) + j) * nz + k;
                for (int c = 0; c < 4; ++c) Fy[c * sy + o] = F[c];
            }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k <= nz; ++k) {
                double F[4];
                face_flux(dm, scheme, U, G, 2, i, j, k, ws, F);
                size_t o = ((size_t)i * ny + j) * (nz + 1) + k;
                for (int c = 0; c < 4; ++c) Fz[c * sz + o] = F[c];
            }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k)
                for (int c = 0; c < 4; ++c) {
                    size_t ox0 = ((size_t)i * ny + j) * nz + k, ox1 = ((size_t)(i + 1) * ny + j) * nz + k;
                    size_t oy0 = ((size_t)i * (ny + 1) + j) * nz + k, oy1 = ((size_t)i * (ny + 1) + j + 1) * nz + k;
                    size_t oz0 = ((size_t)i * ny + j) * (nz + 1) + k;
                    double gx = (Fx[c * sx + ox1] - Fx[c * sx + ox0]) / dm->dx;
                    double gy = (Fy[c * sy + oy1] - Fy[c * sy + oy0]) / dm->dy;
                    double gz = (Fz[c * sz + oz0 + 1] - Fz[c * sz + oz0]) / dm->dz;
                    rhs[IDX(c, i, j, k)] = -(gx + gy + gz);
                }
    free(G); free(Fx); free(Fy); free(Fz);
    return ORC_OK;
}

/* ======================================================================
 * Per-material step coefficients
 * ==================================================================== */

static int material_S(const orc_problem *p, double E, double *S)
{
    for (int m = 0; m < p->nm; ++m) {
        int rc = stopping_power(&p->mats[m], E, &S[m]);
        if (rc) return rc;
    }
    return ORC_OK;
}

/* numerics/energy.py:273-310: C(tau) (forward) and C(tau)^-1 (inverse),
 * phi factor exp(-+min(tau_n,700)), J factor exp(-+min(tau_n+tau_s,700)). */
typedef struct { double phi, cur; } factor_t;

static factor_t source_factor(double ts, double tn, int inverse)
{
    double sign = inverse ? 1.0 : -1.0;
    double a = tn < EXP_CLAMP ? tn : EXP_CLAMP;
    double tsum = tn + ts;
    double b = tsum < EXP_CLAMP ? tsum : EXP_CLAMP;
    factor_t f = {dd_exp(sign * a), dd_exp(sign * b)};
    return f;
}

/* ======================================================================
 * CFL step, numerics/energy.py:539-660 (+ vacuum-aware masks 459-537)
 * ==================================================================== */

static void dilate_axis(const domain_t *dm, unsigned char *mask, int axis, int radius)
{
    int nx = dm->nx, ny = dm->ny, nz = dm->nz;
    size_t n = (size_t)nx * ny * nz;
    unsigned char *old = malloc(n);
    for (int r = 0; r < radius; ++r) {
        memcpy(old, mask, n);
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j)
                for (int k = 0; k < nz; ++k) {
                    size_t o = IDX(0, i, j, k);
                    unsigned char v = old[o];
                    if (axis == 0) {
                        if (i > 0) v |= old[IDX(0, i - 1, j, k)];
                        if (i < nx - 1) v |= old[IDX(0, i + 1, j, k)];
                    } else if (axis == 1) {
                        if (j > 0) v |= old[IDX(0, i, j - 1, k)];
                        if (j < ny - 1) v |= old[IDX(0, i, j + 1, k)];
                    } else {
                        if (k > 0) v |= old[IDX(0, i, j, k - 1)];
                        if (k < nz - 1) v |= old[IDX(0, i, j, k + 1)];
                    }
                    mask[o] = v;
                }
    }
    free(old);
}

static int energy_step(const orc_problem *p, const domain_t *dm, const double *U, double E,
                       double vacuum_tol /* < 0: off */, double *dE_out)
{
    int nx = dm->nx, ny = dm->ny, nz = dm->nz;
    size_t n = (size_t)nx * ny * nz, n2 = (size_t)nx * ny;
    double S[64];
    if (p->nm > 64) return fail(ORC_ERR_ARG, "too many materials");
    int rc = material_S(p, E, S);
    if (rc) return rc;
    double maxinv = -INFINITY;
    if (p->d.wave_speeds == ORC_SPEEDS_UNIT) {
        for (size_t c = 0; c < n; ++c) {
            double s = S[dm->ids[c]];
            double inv = 1.0 / (s * dm->dx) + 1.0 / (s * dm->dy) + 1.0 / (s * dm->dz);
            if (inv > maxinv) maxinv = inv;
        }
    } else {
        double *st = malloc(sizeof(double) * 4 * n2);
        inflow_state(p, dm, E, st);
        unsigned char *mask[3] = {NULL, NULL, NULL};
        if (vacuum_tol >= 0.0) {
            double scale = -INFINITY;
            for (size_t c = 0; c < n; ++c) if (U[c] > scale) scale = U[c];
            for (size_t c = 0; c < n2; ++c) if (st[c] > scale) scale = st[c];
            if (scale != 0.0) {
                double thr = vacuum_tol * scale;
                unsigned char *act = malloc(n);
                for (size_t c = 0; c < n; ++c) act[c] = U[c] > thr;
                for (int i = 0; i < nx; ++i)
                    for (int j = 0; j < ny; ++j)
                        act[IDX(0, i, j, 0)] |= st[(size_t)i * ny + j] > thr;
                /* the reconstruction's ghost width, energy.py:611-622 */
                int sch = p->d.spatial_scheme;
                int radius = sch == ORC_SCHEME_FIRST_ORDER ? 1
                             : (sch == ORC_SCHEME_MUSCL || sch == ORC_SCHEME_WENO3) ? 2 : 3;
                for (int a = 0; a < 3; ++a) {
                    mask[a] = malloc(n);
                    memcpy(mask[a], act, n);
                    dilate_axis(dm, mask[a], a, radius);
                }
                free(act);
            }
        }
#pragma omp parallel for reduction(max : maxinv) schedule(static)
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j)
                for (int k = 0; k < nz; ++k) {
                    size_t o = IDX(0, i, j, k);
                    double u[4] = {U[o], U[n + o], U[2 * n + o], U[3 * n + o]};
                    double a[3];
                    for (int ax = 0; ax < 3; ++ax) {
                        double lo, hi;
                        orc_eigenvalues(u, ax, &lo, &hi);
                        double alo = fabs(lo), ahi = fabs(hi);
                        a[ax] = alo > ahi ? alo : ahi;
                    }
                    if (k == 0) {
                        size_t b = (size_t)i * ny + j;
                        double ui[4] = {st[b], st[n2 + b], st[2 * n2 + b], st[3 * n2 + b]};
                        double lo, hi;
                        orc_eigenvalues(ui, 2, &lo, &hi);
                        double alo = fabs(lo), ahi = fabs(hi);
                        double ain = alo > ahi ? alo : ahi;
                        if (ain > a[2]) a[2] = ain;
                    }
                    if (mask[0]) {
                        if (!mask[0][o]) a[0] = 0.0;
                        if (!mask[1][o]) a[1] = 0.0;
                        if (!mask[2][o]) a[2] = 0.0;
                    }
                    double s = S[dm->ids[o]];
                    double inv = a[0] / (s * dm->dx) + a[1] / (s * dm->dy) + a[2] / (s * dm->dz);
                    if (inv > maxinv) maxinv = inv;
                }
        for (int a = 0; a < 3; ++a) free(mask[a]);
        free(st);
    }
    double dE = p->d.cfl / maxinv;
    *dE_out = p->d.max_energy_step < dE ? p->d.max_energy_step : dE;
    return ORC_OK;
}

/* ======================================================================
 * Energy integrators
 * ==================================================================== */

typedef struct {
    double S0[64], S1[64], S2[64];   /* S(E), S(E-dE), S(E-dE/2) */
    factor_t c1[64], c1i[64];        /* C(tau over dE), inverse */
    factor_t c2[64], c2i[64];        /* C(tau over dE/2), inverse */
} rk_coeff_t;

/* Inflow traces for the two RK stages: numerics/energy.py:348-455
 * (integrating-factor form); with zero optical depths every factor is
 * exactly 1 and this reduces to numerics/energy.py:107-231. */
static int stage_inflow(const orc_problem *p, const domain_t *dm, double E, double dE,
                        int use_if, double *b1, double *b2)
{
    int nx = dm->nx, ny = dm->ny, nz = dm->nz;
    (void)nz;
    size_t n2 = (size_t)nx * ny;
    double taus[4] = {0.0, dE / 3.0, 2.0 * dE / 3.0, dE};
    double energies[4] = {E, E - dE / 3.0, E - 2.0 * dE / 3.0, E - dE};
    double *st = malloc(sizeof(double) * 4 * n2 * 4);
    int nm = p->nm;
    factor_t fi[4][64];
    double Sb[4][64];
    factor_t f1[64], f12[64];
    double S_1[64], S_12[64];
    for (int q = 0; q < 4; ++q) {
        inflow_state(p, dm, energies[q], st + q * 4 * n2);
        int rc = material_S(p, energies[q], Sb[q]);
        if (rc) { free(st); return rc; }
        for (int m = 0; m < nm; ++m) {
            double ts = 0.0, tn = 0.0;
            if (use_if && q > 0) {
                rc = optical_depths(p, &p->mats[m], E, taus[q], &ts, &tn);
                if (rc) { free(st); return rc; }
            }
            fi[q][m] = source_factor(ts, tn, 1);
        }
    }
    for (int m = 0; m < nm; ++m) {
        double ts = 0.0, tn = 0.0;
        int rc;
        if (use_if) {
            rc = optical_depths(p, &p->mats[m], E, dE, &ts, &tn);
            if (rc) { free(st); return rc; }
        }
        f1[m] = source_factor(ts, tn, 0);
        ts = tn = 0.0;
        if (use_if) {
            rc = optical_depths(p, &p->mats[m], E, 0.5 * dE, &ts, &tn);
            if (rc) { free(st); return rc; }
        }
        f12[m] = source_factor(ts, tn, 0);
    }
    int rc = material_S(p, E - dE, S_1);
    if (!rc) rc = material_S(p, E - 0.5 * dE, S_12);
    if (rc) { free(st); return rc; }
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) {
            int m = dm->ids[((size_t)i * ny + j) * nz];
            size_t b = (size_t)i * ny + j;
            for (int c = 0; c < 4; ++c) {
                double V[4];
                for (int q = 0; q < 4; ++q) {
                    double B = Sb[q][m] * st[q * 4 * n2 + c * n2 + b];
                    /* V_0 is not transformed (C(0) = I, energy.py:376-381) */
                    if (q > 0 && use_if) B *= (c == 0 ? fi[q][m].phi : fi[q][m].cur);
                    V[q] = B;
                }
                double vs1 = 0.5 * (-9.0 * V[0] + 18.0 * V[1] - 9.0 * V[2] + 2.0 * V[3]);
                double vs2 = 0.25 * (11.0 * V[0] - 27.0 * V[1] + 27.0 * V[2] - 7.0 * V[3]);
                if (use_if) {
                    vs1 *= (c == 0 ? f1[m].phi : f1[m].cur);
                    vs2 *= (c == 0 ? f12[m].phi : f12[m].cur);
                }
                b1[c * n2 + b] = vs1 / S_1[m];
                b2[c * n2 + b] = vs2 / S_12[m];
            }
        }
    free(st);
    return ORC_OK;
}

static void project_all(double *U, size_t n)
{
#pragma omp parallel for schedule(static)
    for (size_t c = 0; c < n; ++c) {
        double u[4] = {U[c], U[n + c], U[2 * n + c], U[3 * n + c]};
        orc_project(u);
        U[c] = u[0]; U[n + c] = u[1]; U[2 * n + c] = u[2]; U[3 * n + c] = u[3];
    }
}

/* SSPRK3 (numerics/energy.py:725-873) and IF-SSPRK3 (878-1130) on a domain.
 * use_if=0 gives SSPRK3: every integrating factor is the identity. */
static int rk3_step(const orc_problem *p, const domain_t *dm, double *U, double E, double dE,
                    int use_if, double *edep)
{
    int nx = dm->nx, ny = dm->ny, nz = dm->nz;
    size_t n = (size_t)nx * ny * nz, n2 = (size_t)nx * ny;
    int nm = p->nm, rc;
    if (dE <= 0.0) return fail(ORC_ERR_ARG, "dE must be positive.");
    rk_coeff_t k;
    if ((rc = material_S(p, E, k.S0)) || (rc = material_S(p, E - dE, k.S1)) ||
        (rc = material_S(p, E - 0.5 * dE, k.S2)))
        return rc;
    for (int m = 0; m < nm; ++m) {
        double ts1 = 0, tn1 = 0, ts2 = 0, tn2 = 0;
        if (use_if) {
            if ((rc = optical_depths(p, &p->mats[m], E, dE, &ts1, &tn1))) return rc;
            if ((rc = optical_depths(p, &p->mats[m], E, 0.5 * dE, &ts2, &tn2))) return rc;
        }
        k.c1[m] = source_factor(ts1, tn1, 0);
        k.c1i[m] = source_factor(ts1, tn1, 1);
        k.c2[m] = source_factor(ts2, tn2, 0);
        k.c2i[m] = source_factor(ts2, tn2, 1);
    }
    double *b0 = malloc(sizeof(double) * 4 * n2), *b1 = malloc(sizeof(double) * 4 * n2);
    double *b2 = malloc(sizeof(double) * 4 * n2);
    double *V0 = malloc(sizeof(double) * 4 * n), *V1 = malloc(sizeof(double) * 4 * n);
    double *V2 = malloc(sizeof(double) * 4 * n), *Us = malloc(sizeof(double) * 4 * n);
    double *L = malloc(sizeof(double) * 4 * n);
    double *q0 = malloc(sizeof(double) * n), *q1 = malloc(sizeof(double) * n);
    if (!b0 || !b1 || !b2 || !V0 || !V1 || !V2 || !Us || !L || !q0 || !q1) { rc = fail(ORC_ERR_ALLOC, "oom"); goto done; }
    inflow_state(p, dm, E, b0);
    if ((rc = stage_inflow(p, dm, E, dE, use_if, b1, b2))) goto done;

    /* stage 0 */
    for (size_t c = 0; c < n; ++c) {
        double s = k.S0[dm->ids[c]];
        for (int q = 0; q < 4; ++q) V0[q * n + c] = s * U[q * n + c];
        q0[c] = U[c] * s;
    }
    if ((rc = spatial_operator(p, dm, U, b0, L))) goto done;
    /* stage 1 */
    for (size_t c = 0; c < n; ++c) {
        int m = dm->ids[c];
        for (int q = 0; q < 4; ++q) {
            double v = L[q * n + c] * dE + V0[q * n + c];
            V1[q * n + c] = v;
            double w = v * (q == 0 ? k.c1[m].phi : k.c1[m].cur);
            Us[q * n + c] = w / k.S1[m];
        }
    }
    project_all(Us, n);
    for (size_t c = 0; c < n; ++c) q1[c] = Us[c] * k.S1[dm->ids[c]];
    if ((rc = spatial_operator(p, dm, Us, b1, L))) goto done;
    /* stage 2 */
    for (size_t c = 0; c < n; ++c) {
        int m = dm->ids[c];
        for (int q = 0; q < 4; ++q) {
            double r = L[q * n + c] * (q == 0 ? k.c1i[m].phi : k.c1i[m].cur);
            r = (r * dE + V1[q * n + c]) * 0.25;
            double v = 0.75 * V0[q * n + c] + r;
            V2[q * n + c] = v;
            double w = v * (q == 0 ? k.c2[m].phi : k.c2[m].cur);
            Us[q * n + c] = w / k.S2[m];
        }
    }
    project_all(Us, n);
    /* q2 and the quadrature, energy.py:1121-1128 */
    for (size_t c = 0; c < n; ++c) {
        double q2 = Us[c] * k.S2[dm->ids[c]];
        edep[c] = dE * (1.0 / 6.0 * q0[c] + 1.0 / 6.0 * q1[c] + 2.0 / 3.0 * q2);
    }
    if ((rc = spatial_operator(p, dm, Us, b2, L))) goto done;
    /* final stage */
    for (size_t c = 0; c < n; ++c) {
        int m = dm->ids[c];
        for (int q = 0; q < 4; ++q) {
            double r = L[q * n + c] * (q == 0 ? k.c2i[m].phi : k.c2i[m].cur);
            r = (r * dE + V2[q * n + c]) * (2.0 / 3.0);
            double v = 1.0 / 3.0 * V0[q * n + c] + r;
            double w = v * (q == 0 ? k.c1[m].phi : k.c1[m].cur);
            U[q * n + c] = w / k.S1[m];
        }
    }
    project_all(U, n);
    rc = ORC_OK;
done:
    free(b0); free(b1); free(b2); free(V0); free(V1); free(V2); free(Us); free(L); free(q0); free(q1);
    return rc;
}

/* numerics/energy.py:663-722 */
static int forward_euler_step(const orc_problem *p, const domain_t *dm, double *U, double E,
                              double dE, double *edep)
{
    int nx = dm->nx, ny = dm->ny, nz = dm->nz;
    size_t n = (size_t)nx * ny * nz, n2 = (size_t)nx * ny;
    double S0[64], S1[64];
    int rc;
    if ((rc = material_S(p, E, S0)) || (rc = material_S(p, E - dE, S1))) return rc;
    double *b0 = malloc(sizeof(double) * 4 * n2), *L = malloc(sizeof(double) * 4 * n);
    inflow_state(p, dm, E, b0);
    rc = spatial_operator(p, dm, U, b0, L);
    if (!rc) {
        for (size_t c = 0; c < n; ++c) {
            int m = dm->ids[c];
            edep[c] = dE * U[c] * S0[m];
            for (int q = 0; q < 4; ++q) {
                double w = L[q * n + c] * dE + S0[m] * U[q * n + c];
                U[q * n + c] = w / S1[m];
            }
        }
        project_all(U, n);
    }
    free(b0); free(L);
    return rc;
}

/* numerics/energy.py:1168-1191 */
static int half_source(const orc_problem *p, const domain_t *dm, double *U, const double *eta,
                       const double *taun)
{
    size_t n = (size_t)dm->nx * dm->ny * dm->nz;
    if (p->d.nuclear) {
        for (size_t c = 0; c < n; ++c) {
            double t = 0.5 * taun[dm->ids[c]];
            double f = dd_exp(-(t < EXP_CLAMP ? t : EXP_CLAMP));
            for (int q = 0; q < 4; ++q) U[q * n + c] *= f;
        }
    }
    if (p->d.scattering != ORC_SCATTER_OFF) {
        for (size_t c = 0; c < n; ++c) {
            double t = 0.5 * eta[dm->ids[c]];
            double f = dd_exp(-(t < EXP_CLAMP ? t : EXP_CLAMP));
            for (int q = 1; q < 4; ++q) U[q * n + c] *= f;
        }
    }
    return ORC_OK;
}

/* One accepted step, dispatched as numerics/energy.py:1580-1615 */
static int advance(const orc_problem *p, const domain_t *dm, double *U, double E, double dE,
                   double *edep)
{
    int sources = p->d.scattering != ORC_SCATTER_OFF || p->d.nuclear;
    int scheme = p->d.energy_scheme;
    if (scheme == ORC_SCHEME_IF_SSPRK3) return rk3_step(p, dm, U, E, dE, sources, edep);
    if (!sources) {
        if (scheme == ORC_SCHEME_FORWARD_EULER) return forward_euler_step(p, dm, U, E, dE, edep);
        return rk3_step(p, dm, U, E, dE, 0, edep);
    }
    /* Strang splitting, numerics/energy.py:1194-1260 */
    double eta[64], taun[64];
    for (int m = 0; m < p->nm; ++m) {
        double ts = 0.0, tn = 0.0;
        int rc = optical_depths(p, &p->mats[m], E, dE, &ts, &tn);
        if (rc) return rc;
        eta[m] = ts;
        taun[m] = tn;
    }
    half_source(p, dm, U, eta, taun);
    int rc = scheme == ORC_SCHEME_FORWARD_EULER ? forward_euler_step(p, dm, U, E, dE, edep)
                                                : rk3_step(p, dm, U, E, dE, 0, edep);
    if (rc) return rc;
    half_source(p, dm, U, eta, taun);
    return ORC_OK;
}

static domain_t full_domain(const orc_problem *p)
{
    domain_t dm = {p->d.nx, p->d.ny, p->d.nz, p->dx, p->dy, p->dz, p->ids, p->spatial};
    return dm;
}

int orc_spatial_operator(const orc_problem *p, const double *U, double E, const double *bc,
                         double *rhs)
{
    domain_t dm = full_domain(p);
    size_t n2 = (size_t)dm.nx * dm.ny;
    double *st = NULL;
    if (!bc) {
        st = malloc(sizeof(double) * 4 * n2);
        inflow_state(p, &dm, E, st);
        bc = st;
    }
    int rc = spatial_operator(p, &dm, U, bc, rhs);
    free(st);
    return rc;
}

int orc_energy_step(const orc_problem *p, const double *U, double E, double *dE)
{
    domain_t dm = full_domain(p);
    return energy_step(p, &dm, U, E, -1.0, dE);
}

int orc_advance(const orc_problem *p, double *U, double E, double dE, double *edep)
{
    domain_t dm = full_domain(p);
    return advance(p, &dm, U, E, dE, edep);
}

/* ======================================================================
 * The march, numerics/energy.py:1497-1643 and 1262-1494
 * ==================================================================== */

typedef struct { int i0, i1, j0, j1, k0, k1; } box_t;

static int box_eq(box_t a, box_t b)
{
    return a.i0 == b.i0 && a.i1 == b.i1 && a.j0 == b.j0 && a.j1 == b.j1 && a.k0 == b.k0 && a.k1 == b.k1;
}

/* numerics/moving_active_domain.py:35-60 */
static int initial_box(const orc_problem *p, int guard, box_t *b)
{
    int nx = p->d.nx, ny = p->d.ny;
    int ilo = -1, ihi = -1, jlo = -1, jhi = -1;
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            if (p->spatial[(size_t)i * ny + j] > 0.0) {
                if (ilo < 0 || i < ilo) ilo = i;
                if (i > ihi) ihi = i;
                if (jlo < 0 || j < jlo) jlo = j;
                if (j > jhi) jhi = j;
            }
    if (ilo < 0) return fail(ORC_ERR_NO_BEAM, "Beam inflow has empty transverse support.");
    b->i0 = ilo - guard > 0 ? ilo - guard : 0;
    b->i1 = ihi + 1 + guard < nx ? ihi + 1 + guard : nx;
    b->j0 = jlo - guard > 0 ? jlo - guard : 0;
    b->j1 = jhi + 1 + guard < ny ? jhi + 1 + guard : ny;
    b->k0 = 0;
    b->k1 = 1 + guard < p->d.nz ? 1 + guard : p->d.nz;
    return ORC_OK;
}

typedef struct {
    domain_t dm;
    int32_t *ids;
    double *spatial;
} local_t;

/* numerics/moving_active_domain.py:63-104 */
static void make_local(const orc_problem *p, box_t b, local_t *L)
{
    int bx = b.i1 - b.i0, by = b.j1 - b.j0, bz = b.k1 - b.k0;
    int ny = p->d.ny, nz = p->d.nz;
    L->ids = malloc(sizeof(int32_t) * (size_t)bx * by * bz);
    L->spatial = malloc(sizeof(double) * (size_t)bx * by);
    for (int i = 0; i < bx; ++i)
        for (int j = 0; j < by; ++j) {
            for (int k = 0; k < bz; ++k)
                L->ids[((size_t)i * by + j) * bz + k] =
                    p->ids[((size_t)(b.i0 + i) * ny + (b.j0 + j)) * nz + (b.k0 + k)];
            L->spatial[(size_t)i * by + j] = b.k0 == 0 ? p->spatial[(size_t)(b.i0 + i) * ny + (b.j0 + j)] : 0.0;
        }
    domain_t dm = {bx, by, bz, p->dx, p->dy, p->dz, L->ids, L->spatial};
    L->dm = dm;
}

static void free_local(local_t *L) { free(L->ids); free(L->spatial); }

/* numerics/moving_active_domain.py:107-193 */
static int desired_box(const orc_problem *p, const local_t *L, const double *U, box_t cur,
                       double E, double tol, int guard, box_t *next)
{
    const domain_t *dm = &L->dm;
    int nx = dm->nx, ny = dm->ny, nz = dm->nz;
    size_t n = (size_t)nx * ny * nz, n2 = (size_t)nx * ny;
    double *phi_in = NULL;
    double scale = -INFINITY;
    for (size_t c = 0; c < n; ++c) if (U[c] > scale) scale = U[c];
    if (cur.k0 == 0) {
        phi_in = malloc(sizeof(double) * 4 * n2);
        inflow_state(p, dm, E, phi_in);
        for (size_t c = 0; c < n2; ++c) if (phi_in[c] > scale) scale = phi_in[c];
    }
    int found = 0;
    box_t a = {0, 0, 0, 0, 0, 0};
    if (scale != 0.0) {
        double thr = tol * scale;
        int ilo = nx, ihi = -1, jlo = ny, jhi = -1, klo = nz, khi = -1;
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j)
                for (int k = 0; k < nz; ++k) {
                    int act = U[IDX(0, i, j, k)] > thr;
                    if (k == 0 && phi_in) act |= phi_in[(size_t)i * ny + j] > thr;
                    if (act) {
                        if (i < ilo) ilo = i;
                        if (i > ihi) ihi = i;
                        if (j < jlo) jlo = j;
                        if (j > jhi) jhi = j;
                        if (k < klo) klo = k;
                        if (k > khi) khi = k;
                    }
                }
        if (ihi >= 0) {
            found = 1;
            a.i0 = cur.i0 + ilo; a.i1 = cur.i0 + ihi + 1;
            a.j0 = cur.j0 + jlo; a.j1 = cur.j0 + jhi + 1;
            a.k0 = cur.k0 + klo; a.k1 = cur.k0 + khi + 1;
        }
    }
    free(phi_in);
    if (!found) return initial_box(p, guard, next);
    next->i0 = a.i0 - guard > 0 ? a.i0 - guard : 0;
    next->i1 = a.i1 + guard < p->d.nx ? a.i1 + guard : p->d.nx;
    next->j0 = a.j0 - guard > 0 ? a.j0 - guard : 0;
    next->j1 = a.j1 + guard < p->d.ny ? a.j1 + guard : p->d.ny;
    next->k0 = a.k0 - guard > 0 ? a.k0 - guard : 0;
    next->k1 = a.k1 + guard < p->d.nz ? a.k1 + guard : p->d.nz;
    return ORC_OK;
}

/* numerics/moving_active_domain.py:196-232 */
static double *rebox(const double *U, box_t o, box_t nb)
{
    int ox = o.i1 - o.i0, oy = o.j1 - o.j0, oz = o.k1 - o.k0;
    int bx = nb.i1 - nb.i0, by = nb.j1 - nb.j0, bz = nb.k1 - nb.k0;
    size_t on = (size_t)ox * oy * oz, nn = (size_t)bx * by * bz;
    double *Un = calloc(4 * nn, sizeof(double));
    int gi0 = o.i0 > nb.i0 ? o.i0 : nb.i0, gi1 = o.i1 < nb.i1 ? o.i1 : nb.i1;
    int gj0 = o.j0 > nb.j0 ? o.j0 : nb.j0, gj1 = o.j1 < nb.j1 ? o.j1 : nb.j1;
    int gk0 = o.k0 > nb.k0 ? o.k0 : nb.k0, gk1 = o.k1 < nb.k1 ? o.k1 : nb.k1;
    if (gi1 > gi0 && gj1 > gj0 && gk1 > gk0)
        for (int c = 0; c < 4; ++c)
            for (int i = gi0; i < gi1; ++i)
                for (int j = gj0; j < gj1; ++j)
                    for (int k = gk0; k < gk1; ++k)
                        Un[c * nn + ((size_t)(i - nb.i0) * by + (j - nb.j0)) * bz + (k - nb.k0)] =
                            U[c * on + ((size_t)(i - o.i0) * oy + (j - o.j0)) * oz + (k - o.k0)];
    return Un;
}

/* numerics/moving_active_domain.py:235-244 */
static void embed(const orc_problem *p, const double *U, box_t b, double *full)
{
    int ny = p->d.ny, nz = p->d.nz;
    size_t N = (size_t)p->d.nx * ny * nz;
    int bx = b.i1 - b.i0, by = b.j1 - b.j0, bz = b.k1 - b.k0;
    size_t bn = (size_t)bx * by * bz;
    memset(full, 0, sizeof(double) * 4 * N);
    for (int c = 0; c < 4; ++c)
        for (int i = 0; i < bx; ++i)
            for (int j = 0; j < by; ++j)
                for (int k = 0; k < bz; ++k)
                    full[c * N + ((size_t)(b.i0 + i) * ny + (b.j0 + j)) * nz + (b.k0 + k)] =
                        U[c * bn + ((size_t)i * by + j) * bz + k];
}

static int cmp_desc(const void *a, const void *b)
{
    double x = *(const double *)a, y = *(const double *)b;
    return (x < y) - (x > y);
}

static int march_impl(const orc_problem *p, double *U, double *dose, double *energies, int max_steps,
                      int *n_steps, const double *snap_targets, int n_snap, double *snap_out,
                      double *snap_E_out, int *n_taken, int *final_written, int step_limit)
{
    const orc_problem_desc *d = &p->d;
    size_t N = (size_t)d->nx * d->ny * d->nz;
    double E = d->energy + d->energy_window_sigma * d->energy_spread;
    double Emin = d->energy_min;
    int rc = ORC_OK;
    /* sorted unique targets in [Emin, E], descending (energy.py:1531-1538) */
    double *targets = malloc(sizeof(double) * (n_snap > 0 ? n_snap : 1));
    int nt = 0;
    for (int s = 0; s < n_snap; ++s) {
        double t = snap_targets[s];
        if (!(Emin <= t && t <= E)) continue;
        int dup = 0;
        for (int q = 0; q < nt; ++q) if (targets[q] == t) dup = 1;
        if (!dup) targets[nt++] = t;
    }
    qsort(targets, nt, sizeof(double), cmp_desc);
    int ti = 0, taken = 0, steps = 0;
    if (energies) energies[0] = E;
    memset(dose, 0, sizeof(double) * N);

    int moving = d->moving_active_domain;
    box_t box = {0, d->nx, 0, d->ny, 0, d->nz};
    double *Ua = U;
    double tol = exp(-0.5 * (d->active_truncation_sigma * d->active_truncation_sigma));   /* energy.py:1305-1307 */
    int guard = d->active_guard_cells;
    if (moving) {
        if ((rc = initial_box(p, guard, &box))) goto out;
        if (U) {
            box_t full = {0, d->nx, 0, d->ny, 0, d->nz};
            Ua = rebox(U, full, box);
        } else {
            Ua = calloc(4 * (size_t)(box.i1 - box.i0) * (box.j1 - box.j0) * (box.k1 - box.k0), sizeof(double));
        }
    } else if (!U) {
        rc = fail(ORC_ERR_ARG, "A full-grid initial state is required when moving_active_domain is disabled.");
        goto out;
    }
    while (E > Emin) {
        if (step_limit >= 0 && steps >= step_limit) break;
        if (steps >= max_steps) { rc = fail(ORC_ERR_MAX_STEPS, "energies buffer too short"); break; }
        local_t L;
        if (moving) {
            make_local(p, box, &L);
            box_t nb;
            rc = desired_box(p, &L, Ua, box, E, tol, guard, &nb);
            if (rc) { free_local(&L); break; }
            if (!box_eq(nb, box)) {
                double *Un = rebox(Ua, box, nb);
                free(Ua);
                Ua = Un;
                box = nb;
                free_local(&L);
                make_local(p, box, &L);
            }
        } else {
            L.dm = full_domain(p);
            L.ids = NULL;
            L.spatial = NULL;
        }
        double dE;
        rc = energy_step(p, &L.dm, Ua, E, (moving && d->vacuum_aware_cfl) ? tol : -1.0, &dE);
        if (rc) { free_local(&L); break; }
        /* a prescribed schedule replaces the CFL step (the fixed-schedule mode
           of the reference's harness: a patched compute_energy_step) */
        if (p->schedule) dE = steps + 1 < p->n_schedule ? E - p->schedule[steps + 1] : E - Emin;
        if (ti < nt) {
            double t = targets[ti];
            if (E > t && t >= E - dE) dE = E - t;
        }
        if (E - Emin < dE) dE = E - Emin;
        size_t bn = (size_t)L.dm.nx * L.dm.ny * L.dm.nz;
        double *edep = malloc(sizeof(double) * bn);
        rc = advance(p, &L.dm, Ua, E, dE, edep);
        if (rc) { free(edep); free_local(&L); break; }
        /* dose += edep * MEV_TO_JOULE / rho (energy.py:1617-1621, 1452-1457) */
        int bny = L.dm.ny, bnz = L.dm.nz;
        for (int i = 0; i < L.dm.nx; ++i)
            for (int j = 0; j < bny; ++j)
                for (int k = 0; k < bnz; ++k) {
                    size_t lo = ((size_t)i * bny + j) * bnz + k;
                    size_t go = ((size_t)(box.i0 + i) * d->ny + (box.j0 + j)) * d->nz + (box.k0 + k);
                    double rho = p->mats[L.dm.ids[lo]].density;
                    dose[go] += edep[lo] * MEV_TO_JOULE / rho;
                }
        free(edep);
        free_local(&L);
        E -= dE;
        if (p->schedule && steps + 1 < p->n_schedule) E = p->schedule[steps + 1];
        steps++;
        if (energies) energies[steps] = E;
        if (ti < nt && fabs(E - targets[ti]) <= 1e-12) {
            if (snap_out) {
                double *dst = snap_out + (size_t)taken * 4 * N;
                if (moving) embed(p, Ua, box, dst);
                else memcpy(dst, Ua, sizeof(double) * 4 * N);
            }
            if (snap_E_out) snap_E_out[taken] = targets[ti];
            taken++;
            ti++;
        }
    }
    if (moving) {
        int store = d->store_final_state;
        if (final_written) *final_written = store && U != NULL ? 1 : 0;
        if (store && U) embed(p, Ua, box, U);
        free(Ua);
    } else if (final_written) {
        *final_written = 1;
    }
out:
    if (n_steps) *n_steps = steps;
    if (n_taken) *n_taken = taken;
    free(targets);
    return rc;
}

int orc_march(const orc_problem *p, double *U, double *dose, double *energies, int max_steps,
              int *n_steps, const double *snap_targets, int n_snap, double *snap_out,
              double *snap_E_out, int *n_taken, int *final_written)
{
    return march_impl(p, U, dose, energies, max_steps, n_steps, snap_targets, n_snap, snap_out,
                      snap_E_out, n_taken, final_written, -1);
}

int orc_march_steps(const orc_problem *p, double *U, double *dose, int steps, int *n_done)
{
    return march_impl(p, U, dose, NULL, steps + 1, n_done, NULL, 0, NULL, NULL, NULL, NULL, steps);
}
