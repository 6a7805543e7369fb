/*
 * CPU oracle for the BIA pair step -- TEST INFRASTRUCTURE ONLY.
 *
 * This file restates, in plain C, the reference's CPU path of the Binary
 * Interaction Approximation (BIA) step so that the CUDA product can be checked
 * against it.  It is never linked into the product library; only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
 *
 * Every routine cites the reference file:line it follows.  Arithmetic order
 * follows the Fortran source (left-to-right evaluation, ** as repeated
 * multiplication) and the library is built with -ffp-contract=off so no FMA
 * contraction changes the rounding.  Deliberate deviations from the reference
 * are marked "DEVIATION" in the code; they are:
 *   - find_hyperbola leaves theta_stock uninitialised when the Newton loop never
 *     improves on the starting residual (bia/find_hyperbola.f90:93-119); here it
 *     starts as the starting iterate.
 *   - find_hyperbola returns without setting YN when an iterate leaves the
 *     (-theta_0, theta_0) bracket (bia/find_hyperbola.f90:98-101); here the loop
 *     stops and the best iterate so far is used.
 *   - pairs with zero relative velocity or zero angular momentum give NaN in the
 *     reference frame construction (bia/bia.f90:288-296), and near-parabolic pairs
 *     lose every digit in the reference's a = eps/W, b_0 = eps/W parametrisations
 *     (a barely bound pair can jump by 10^4 in one step); under ALG both go to a
 *     universal-variable (Stumpff) solver, which method 2 uses for every pair.
 *   - when the reference's hyperbola or ellipse iteration ends (iteration cap or
 *     bracket exit) without a small residual (bia/find_hyperbola.f90:94-118,
 *     bia/find_ellipse.f90:125-152: the ellipse Newton starts from xi_2 + delta_ini
 *     and can fail for high-eccentricity bound pairs), the same equation is
 *     re-solved by a bracketed Newton-bisection; pairs the reference converges are
 *     untouched.
 *   - find_parabola's diagnostic prints (bia/find_parabola.f90:40-103) are dropped.
 *   - the coupling may be per pair, eps_ij = eps_th * q_i * q_j, when a charge
 *     array is given (the reference has one global eps_th, bia/bia.f90:37).
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#include <quadmath.h>
#ifdef _OPENMP
#include <omp.h>
#endif


/* pair classes, also used by the per-pair statistics */
enum { OC_HYPERBOLA = 0, OC_PARABOLA = 1, OC_ELLIPSE = 2, OC_DEGENERATE = 3, OC_RKF = 4,
       OC_UNIVERSAL = 5 };

/* pairs with |e^2 - 1| = |E| L^2 / eps^2 below this go to the universal-variable solver */
#define NEAR_UNIT_ECC 0.1

typedef struct {
    int64_t count[6];      /* pairs per class */
    int64_t iterations;    /* Newton iterations summed over ALG pairs */
    int64_t rkf_steps;     /* accepted RKF steps summed over RKF pairs */
    int64_t nonconverged;  /* |error| > ERR (bia/bia.f90:151,167) */
    int64_t bracket_exits; /* hyperbola iterate left the bracket */
    int64_t fallbacks;     /* reference iteration ended unconverged; safeguarded re-solve */
    int64_t uv_iterations; /* Newton iterations of the universal-variable solver */
} oracle_stats;

/* Fortran SIGN(a,b) and the rest of the pair path are written once in
 * bia_oracle_core.inc over a scalar type REAL and instantiated twice:
 *   double      -- the reference's FP64 CPU path (names as written);
 *   __float128  -- the same algorithm evaluated in quad precision (names + "_q"),
 *                  i.e. the BIA step with rounding error removed, used to measure the
 *                  FP64 rounding noise of any implementation of the algorithm.
 * Record-level functions take and return FP64 arrays in both instantiations. */

#define REAL double
#define NAME(x) x
#define R_PI 3.14159265358979323846264338327950288419716939937510582097494
#define R_HUGE DBL_MAX
#define R_NAN NAN
#define R_SQRT sqrt
#define R_SINCOS sincos
#define R_SIN sin
#define R_COS cos
#define R_LOG log
#define R_ATAN2 atan2
#define R_ATAN atan
#define R_ACOS acos
#define R_POW pow
#define R_FABS fabs
#define R_FMIN fmin
#define R_FMAX fmax
#define R_EPS DBL_EPSILON
#define AL2 ((REAL)1 / 4)
#define AL3 ((REAL)3 / 8)
#define AL4 ((REAL)12 / 13)
#define AL5 ((REAL)1)
#define AL6 ((REAL)1 / 2)
#define B21 ((REAL)1 / 4)
#define B31 ((REAL)3 / 32)
#define B32 ((REAL)9 / 32)
#define B41 ((REAL)1932 / 2197)
#define B42 ((REAL)-7200 / 2197)
#define B43 ((REAL)7296 / 2197)
#define B51 ((REAL)439 / 216)
#define B52 ((REAL)-8)
#define B53 ((REAL)3680 / 513)
#define B54 ((REAL)-845 / 4104)
#define B61 ((REAL)-8 / 27)
#define B62 ((REAL)2)
#define B63 ((REAL)-3544 / 2565)
#define B64 ((REAL)1859 / 4104)
#define B65 ((REAL)-11 / 40)
#define GA1 ((REAL)16 / 135)
#define GA3 ((REAL)6656 / 12825)
#define GA4 ((REAL)28561 / 56430)
#define GA5 ((REAL)-9 / 50)
#define GA6 ((REAL)2 / 55)
#define DA1 ((REAL)1 / 360)
#define DA3 ((REAL)-128 / 4275)
#define DA4 ((REAL)-2197 / 75240)
#define DA5 ((REAL)1 / 50)
#define DA6 ((REAL)2 / 55)
#include "bia_oracle_core.inc"
#undef REAL
#undef NAME
#undef R_PI
#undef R_HUGE
#undef R_NAN
#undef R_SQRT
#undef R_SINCOS
#undef R_SIN
#undef R_COS
#undef R_LOG
#undef R_ATAN2
#undef R_ATAN
#undef R_ACOS
#undef R_POW
#undef R_FABS
#undef R_FMIN
#undef R_FMAX
#undef R_EPS

static void quad_sincos(__float128 x, __float128 *s, __float128 *c) { sincosq(x, s, c); }
#define REAL __float128
#define NAME(x) x##_q
#define R_PI M_PIq
#define R_HUGE ((__float128)DBL_MAX)
#define R_NAN ((__float128)NAN)
#define R_SQRT sqrtq
#define R_SINCOS quad_sincos
#define R_SIN sinq
#define R_COS cosq
#define R_LOG logq
#define R_ATAN2 atan2q
#define R_ATAN atanq
#define R_ACOS acosq
#define R_POW powq
#define R_FABS fabsq
#define R_FMIN fminq
#define R_FMAX fmaxq
#define R_EPS FLT128_EPSILON
#include "bia_oracle_core.inc"
#undef REAL
#undef NAME

/* ---------------------------------------------------------------------------
 * bia/Invariance_CPU.f90:1-19  Invariance_CPU (FP64, sequential sums).
 * out[11] = {KE, PE, Lx, Ly, Lz, Ua, Va, Wa, Xa, Ya, Za}
 * With a charge array the PE sum becomes sum q_i q_j / r_ij.
 * ------------------------------------------------------------------------- */
void oracle_invariance_cpu(int n, double eps_th, const double *q, const double *X,
                           const double *Y, const double *Z, const double *U, const double *V,
                           const double *W, double out[11])
{
    double Xa = 0, Ya = 0, Za = 0, Ua = 0, Va = 0, Wa = 0, Lx = 0, Ly = 0, Lz = 0, KE = 0;
    for (int i = 0; i < n; i++) Xa += X[i];
    for (int i = 0; i < n; i++) Ua += U[i];
    for (int i = 0; i < n; i++) Lx += Y[i] * W[i] - Z[i] * V[i];
    for (int i = 0; i < n; i++) Ya += Y[i];
    for (int i = 0; i < n; i++) Va += V[i];
    for (int i = 0; i < n; i++) Ly += Z[i] * U[i] - X[i] * W[i];
    for (int i = 0; i < n; i++) Za += Z[i];
    for (int i = 0; i < n; i++) Wa += W[i];
    for (int i = 0; i < n; i++) Lz += X[i] * V[i] - Y[i] * U[i];
    for (int i = 0; i < n; i++) KE += U[i] * U[i] + V[i] * V[i] + W[i] * W[i];
    double PE = 0;
    for (int i = 0; i < n - 1; i++) {
        double Xi = X[i], Yi = Y[i], Zi = Z[i];
        for (int j = i + 1; j < n; j++) {
            double dx = Xi - X[j], dy = Yi - Y[j], dz = Zi - Z[j];
            double w = 1 / sqrt(dx * dx + dy * dy + dz * dz);
            PE = PE + (q ? q[i] * q[j] * w : w);
        }
    }
    PE = eps_th * PE;
    double o[11] = {KE, PE, Lx, Ly, Lz, Ua, Va, Wa, Xa, Ya, Za};
    memcpy(out, o, sizeof o);
}

/* bia/Invariance_QPU.f90:1-19  Invariance_QPU: the same sums in __float128,
 * each result rounded to double on assignment. */
void oracle_invariance_qpu(int n, double eps_th, const double *q, const double *X,
                           const double *Y, const double *Z, const double *U, const double *V,
                           const double *W, double out[11])
{
    __float128 Xa = 0, Ya = 0, Za = 0, Ua = 0, Va = 0, Wa = 0, Lx = 0, Ly = 0, Lz = 0, KE = 0;
    for (int i = 0; i < n; i++) {
        __float128 x = X[i], y = Y[i], z = Z[i], u = U[i], v = V[i], w = W[i];
        Xa += x; Ya += y; Za += z; Ua += u; Va += v; Wa += w;
        Lx += y * w - z * v;
        Ly += z * u - x * w;
        Lz += x * v - y * u;
        KE += u * u + v * v + w * w;
    }
    __float128 QPE = 0;
    for (int i = 0; i < n - 1; i++) {
        __float128 xi = X[i], yi = Y[i], zi = Z[i];
        for (int j = i + 1; j < n; j++) {
            __float128 dx = xi - (__float128)X[j], dy = yi - (__float128)Y[j],
                       dz = zi - (__float128)Z[j];
            __float128 w = 1 / sqrtq(dx * dx + dy * dy + dz * dz);
            QPE += q ? (__float128)q[i] * (__float128)q[j] * w : w;
        }
    }
    double o[11] = {(double)KE, (double)((__float128)eps_th * QPE), (double)Lx, (double)Ly,
                    (double)Lz, (double)Ua, (double)Va, (double)Wa, (double)Xa, (double)Ya,
                    (double)Za};
    memcpy(out, o, sizeof o);
}

/* ---------------------------------------------------------------------------
 * dim/rkf_kernel.cu:55-73 moon (3-D direct sum, AoS y[6n], softening 1e-99)
 * and :161-188 fehl/flstep/fhstep with rkf_c_'s host control :237-483.
 * ------------------------------------------------------------------------- */
typedef struct { int np; double eps; } dim_ctx;

static void dim_moon(const void *vctx, double x, const double *y, double *f)
{
    (void)x;
    const dim_ctx *c = (const dim_ctx *)vctx;
    for (int ip = 0; ip < c->np; ip++) {
        int IP = 6 * ip;
        f[IP] = y[IP + 3]; f[IP + 1] = y[IP + 4]; f[IP + 2] = y[IP + 5];
        double Ex = 0, Ey = 0, Ez = 0;
        for (int jp = 0; jp < c->np; jp++) {
            int JP = 6 * jp;
            double xij = y[IP] - y[JP], yij = y[IP + 1] - y[JP + 1], zij = y[IP + 2] - y[JP + 2];
            double rsq = xij * xij + yij * yij + zij * zij + 1e-99;
            double eee = c->eps / (rsq * sqrt(rsq));
            Ex += xij * eee; Ey += yij * eee; Ez += zij * eee;
        }
        f[IP + 3] = Ex; f[IP + 4] = Ey; f[IP + 5] = Ez;
    }
}

/* dim/rkf_kernel.cu:194-495 rkf_c_ restated on the CPU for small n.
 * y0[6n] AoS state at x0, advanced to xe; result in yn.  Returns ier
 * (0 ok, 10000 too many iterations, 20000, 30000) and the accepted step count. */
int oracle_dim_rkf(int n, double eps_th, double x0, double xe, const double *y0, double relerr,
                   double abserr, double *yn, int *naccepted, int *nde)
{
    const double EPSMIN = 1e-15;
    const int ITEMAX = 10000;
    int neq = 6 * n;
    dim_ctx ctx = {n, eps_th};
    double *YH0 = calloc(neq, sizeof(double)), *YL0 = calloc(neq, sizeof(double));
    double *YLN = calloc(neq, sizeof(double)), *ERR = calloc(neq, sizeof(double));
    double *WRK = calloc((size_t)11 * neq, sizeof(double));
    for (int i = 0; i < neq; i++) { YH0[i] = y0[i]; YL0[i] = y0[i]; yn[i] = y0[i]; }
    dim_moon(&ctx, x0, YL0, WRK);
    double TOLDY = DBL_MAX;
    int changed = 0;
    for (int i = 0; i < neq; i++) {
        if (fabs(WRK[i]) > 0.0) {
            double TOL = relerr * fabs(YL0[i]) + abserr;
            TOLDY = fmin(TOLDY, fabs(TOL / WRK[i]));
            changed = 1;
        }
    }
    double H = changed ? fmin((xe - x0) / 100e0, pow(TOLDY, 0.2)) : EPSMIN * (xe - x0);
    int NDE = 1, acc = 0, ier = 10000;
    double X = x0;
    for (int ITER = 0; ITER < ITEMAX; ITER++) {
        double h = H;
        fehl_n(1, neq, dim_moon, &ctx, X, h, YL0, YLN, ERR, WRK);
        NDE += 6;
        double ERRET = 0;
        int bad = 0;
        for (int i = 0; i < neq; i++) {
            double ET = relerr * (fabs(YL0[i]) + fabs(YLN[i])) / 2 + abserr;
            if (ET == 0) { bad = 1; break; }
            ERRET = fmax(ERRET, fabs(ERR[i]) / ET);
        }
        if (bad) { ier = 20000; break; }
        if (ERRET > 1) {
            if (ERRET >= 59049) H *= 0.1;
            else H *= 0.9 / pow(ERRET, 0.2);
            if (H <= EPSMIN) { ier = 30000; break; }
        } else if (X + H < xe) {
            fhstep_n(neq, dim_moon, &ctx, X, H, YH0, yn, ERR, WRK);
            NDE += 12;
            X += H;
            for (int i = 0; i < neq; i++) { YL0[i] = YLN[i]; YH0[i] = yn[i]; }
            acc++;
            if (ERRET <= 1.889568e-4) H *= 5.0;
            else H *= 0.9 / pow(ERRET, 0.2);
        } else {
            h = H = xe - X;
            fehl_n(1, neq, dim_moon, &ctx, X, h, YL0, YLN, ERR, WRK);
            fhstep_n(neq, dim_moon, &ctx, X, h, YH0, yn, ERR, WRK);
            NDE += 18;
            acc++;
            ier = 0;
            break;
        }
    }
    if (naccepted) *naccepted = acc;
    if (nde) *nde = NDE;
    free(YH0); free(YL0); free(YLN); free(ERR); free(WRK);
    return ier;
}
