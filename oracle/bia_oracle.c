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
 * are marked "DEVIATION" and listed in DESIGN.md:
 *   - find_hyperbola leaves theta_stock uninitialised when the Newton loop never
 *     improves on the starting residual (bia/find_hyperbola.f90:93-119); here it
 *     starts as the starting iterate.
 *   - find_hyperbola returns without setting YN when an iterate leaves the
 *     (-theta_0, theta_0) bracket (bia/find_hyperbola.f90:98-101); here the loop
 *     stops and the best iterate so far is used.
 *   - pairs with zero relative velocity or zero angular momentum give NaN in the
 *     reference frame construction (bia/bia.f90:288-296); here they are advanced
 *     by the reference's own per-pair RKF45 along the line of motion.
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

#define ORACLE_PI 3.14159265358979323846264338327950288419716939937510582097494

/* pair classes, also used by the per-pair statistics */
enum { OC_HYPERBOLA = 0, OC_PARABOLA = 1, OC_ELLIPSE = 2, OC_DEGENERATE = 3, OC_RKF = 4 };

typedef struct {
    int64_t count[5];      /* pairs per class */
    int64_t iterations;    /* Newton iterations summed over ALG pairs */
    int64_t rkf_steps;     /* accepted RKF steps summed over RKF pairs */
    int64_t nonconverged;  /* |error| > ERR (bia/bia.f90:151,167) */
    int64_t bracket_exits; /* hyperbola iterate left the bracket */
} oracle_stats;

/* Fortran SIGN(a,b): |a| with the sign of b. */
static double f_sign(double a, double b) { return (b >= 0) ? fabs(a) : -fabs(a); }

/* ---------------------------------------------------------------------------
 * bia/bia.f90:284-314  xyz_to_xi_eta_zeta
 * e_eta = g/|g|, e_zeta = L/|L| with L = r x g, e_xi = e_eta x e_zeta,
 * Y = (r.e_xi, r.e_eta, 0, |g|).
 * Returns 0 on a regular pair, 1 when |g| == 0 or |L| == 0 (DEVIATION: the
 * reference divides by zero there; the caller then uses the radial frame).
 * ------------------------------------------------------------------------- */
int oracle_xyz_to_xi_eta_zeta(const double r[3], const double g[3], double e_xi[3],
                              double e_eta[3], double e_zeta[3], double Y[4])
{
    double gsq = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
    double gm = sqrt(gsq);
    double L[3];
    L[0] = r[1] * g[2] - r[2] * g[1];
    L[1] = r[2] * g[0] - r[0] * g[2];
    L[2] = r[0] * g[1] - r[1] * g[0];
    double Lsq = L[0] * L[0] + L[1] * L[1] + L[2] * L[2];
    if (gm == 0 || Lsq == 0) {
        /* radial frame: motion stays on one axis */
        if (gm == 0) {
            double rm = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
            for (int k = 0; k < 3; k++) { e_xi[k] = r[k] / rm; e_eta[k] = 0; e_zeta[k] = 0; }
            Y[0] = rm; Y[1] = 0; Y[2] = 0; Y[3] = 0;
        } else {
            for (int k = 0; k < 3; k++) { e_eta[k] = g[k] / gm; e_xi[k] = 0; e_zeta[k] = 0; }
            Y[0] = 0;
            Y[1] = r[0] * e_eta[0] + r[1] * e_eta[1] + r[2] * e_eta[2];
            Y[2] = 0;
            Y[3] = gm;
        }
        return 1;
    }
    double Lm = sqrt(Lsq);
    for (int k = 0; k < 3; k++) { e_eta[k] = g[k] / gm; e_zeta[k] = L[k] / Lm; }
    e_xi[0] = e_eta[1] * e_zeta[2] - e_eta[2] * e_zeta[1];
    e_xi[1] = e_eta[2] * e_zeta[0] - e_eta[0] * e_zeta[2];
    e_xi[2] = e_eta[0] * e_zeta[1] - e_eta[1] * e_zeta[0];
    Y[0] = r[0] * e_xi[0] + r[1] * e_xi[1] + r[2] * e_xi[2];
    Y[2] = 0;
    Y[1] = r[0] * e_eta[0] + r[1] * e_eta[1] + r[2] * e_eta[2];
    Y[3] = gm;
    return 0;
}

/* ---------------------------------------------------------------------------
 * bia/find_hyperbola.f90:1-166  find_hyperbola (+ contained find_theta :149-165)
 * Returns the number of Newton iterations taken in the main loop.
 * ------------------------------------------------------------------------- */
typedef struct {
    double theta_0, tn_0, cs_0, sn_0, time_end_;
} hyp_common;

/* bia/find_hyperbola.f90:149-165 */
static void hyp_find_theta(const hyp_common *c, double theta_now, double *theta_end,
                           double *dfdth_, double *error_)
{
    double sn_p = sin((c->theta_0 + theta_now) / 2);
    double sn_m = sin((c->theta_0 - theta_now) / 2);
    double sn_now, cs_now;
    sincos(theta_now, &sn_now, &cs_now);
    double D_inv = 1 / (cs_now - c->cs_0);
    *error_ = c->tn_0 * sn_now * D_inv - c->time_end_ + log(sn_p / sn_m);
    if (*error_ == 0) {
        *theta_end = theta_now;
    } else {
        *dfdth_ = c->tn_0 * (1 - c->cs_0 * cs_now) * (D_inv * D_inv) + c->sn_0 / (2 * sn_p * sn_m);
        *theta_end = theta_now - *error_ / *dfdth_;
    }
}

int oracle_find_hyperbola(double eps_th, double dt, const double YZ[4], double YN[4],
                          double *error_end, int ITR, int *bracket_exit)
{
    double X_ini = YZ[0], Y_ini = YZ[1], U_ini = YZ[2], V_ini = YZ[3];
    double r_g = X_ini * U_ini + Y_ini * V_ini;
    double Lz = X_ini * V_ini - Y_ini * U_ini;
    double r = sqrt(X_ini * X_ini + Y_ini * Y_ini);
    double g2 = U_ini * U_ini + V_ini * V_ini;
    double W = g2 + 2 * eps_th / r;
    double g_0 = sqrt(W);
    double b_0 = eps_th / W;
    double b = fabs(Lz) / g_0;
    hyp_common c;
    c.theta_0 = atan2(fabs(Lz), b_0 * g_0);
    double den0 = sqrt(b_0 * b_0 * (g_0 * g_0) + Lz * Lz);
    c.cs_0 = b_0 * g_0 / den0;
    c.sn_0 = fabs(Lz) / den0;
    c.tn_0 = fabs(Lz) / (b_0 * g_0);
    double theta_ini;
    if (fabs(c.cs_0 + b * c.sn_0 / r) > 1)
        theta_ini = 1e-30;
    else
        theta_ini = acos(c.cs_0 + b * c.sn_0 / r);
    if (Lz * r_g < 0) theta_ini = -theta_ini;
    double sn, cs;
    sincos(theta_ini, &sn, &cs);
    double x = r * cs, y = r * sn;
    double g0_sn0 = (Lz > 0) ? g_0 / c.sn_0 : -g_0 / c.sn_0;
    double u = g0_sn0 * (c.cs_0 * sn);
    double v = g0_sn0 * (1 - c.cs_0 * cs);
    double den_a = sqrt((X_ini * X_ini + Y_ini * Y_ini) * (x * x + y * y));
    double cs_a = (x * X_ini + y * Y_ini) / den_a;
    double sn_a = (x * Y_ini - y * X_ini) / den_a;
    double time_ini = (c.tn_0 * sn / (cs - c.cs_0)
                       + log(sin((c.theta_0 + theta_ini) / 2) / sin((c.theta_0 - theta_ini) / 2)))
                      * b_0 / g_0;
    double time_end = (Lz > 0) ? time_ini + dt : time_ini - dt;
    c.time_end_ = time_end * g_0 / b_0;
    double theta_gss = 2 / ORACLE_PI * c.theta_0 * atan(c.time_end_ / c.tn_0);

    double theta_ini_end, dfdth_ini_ = 0, error_ini_;
    double theta_gss_end, dfdth_gss_ = 0, error_gss_;
    hyp_find_theta(&c, theta_ini, &theta_ini_end, &dfdth_ini_, &error_ini_);
    hyp_find_theta(&c, theta_gss, &theta_gss_end, &dfdth_gss_, &error_gss_);
    double theta_end, error_, dfdth_ = 0;
    if (fabs(error_gss_) > 10 * fabs(error_ini_)) {
        theta_end = theta_ini_end;
        error_ = error_ini_;
    } else {
        theta_end = theta_gss_end;
        error_ = error_gss_;
    }
    double err_stock = error_;
    double theta_stock = theta_end; /* DEVIATION: defined start value */
    double error_restore_[64];
    if (ITR > 62) ITR = 62; /* restore buffer bound */
    int IR = 0;
    if (bracket_exit) *bracket_exit = 0;
    while (IR < ITR) {
        double theta_now = theta_end;
        double sn_p = sin((c.theta_0 + theta_now) / 2);
        double sn_m = sin((c.theta_0 - theta_now) / 2);
        if (sn_p * sn_m < 0) { /* DEVIATION: keep the best iterate so far */
            if (bracket_exit) *bracket_exit = 1;
            break;
        }
        hyp_find_theta(&c, theta_now, &theta_end, &dfdth_, &error_);
        IR = IR + 1;
        int cycle = 0;
        for (int num = IR - 1; num >= 1; num--)
            if (error_restore_[num] == error_) { cycle = 1; break; }
        if (cycle) break;
        error_restore_[IR] = error_;
        if (fabs(error_) < fabs(err_stock)) {
            err_stock = error_ * b_0 / g_0;
            theta_stock = theta_end;
            if (fabs(err_stock) < 2e-16) break;
        }
    }
    theta_end = theta_stock;
    *error_end = error_ * b_0 / g_0;

    double sn_end, cs_end;
    sincos(theta_end, &sn_end, &cs_end);
    double u_end = g0_sn0 * c.cs_0 * sn_end;
    double du_end = u_end - u;
    double v_end = g0_sn0 * (1 - c.cs_0 * cs_end);
    double dv_end = v_end - v;
    double r_end = b * c.sn_0 / (cs_end - c.cs_0);
    double r1end = r_end * (cs_end * cs_a - sn_end * sn_a);
    double r2end = r_end * (cs_end * sn_a + sn_end * cs_a);
    double dg1end = du_end * cs_a - dv_end * sn_a;
    double dg2end = du_end * sn_a + dv_end * cs_a;
    YN[0] = r1end;
    YN[1] = r2end;
    YN[2] = YZ[2] + dg1end;
    YN[3] = YZ[3] + dg2end;
    return IR;
}

/* ---------------------------------------------------------------------------
 * bia/find_ellipse.f90:1-157  FIND_ELLIPSE (+ contained Newton :106-157)
 * Returns the Newton iteration counter ir.
 * ------------------------------------------------------------------------- */
int oracle_find_ellipse(double eps_th, double dt, const double YZ[4], double YN[4],
                        double *error, int ITR)
{
    const double pi = ORACLE_PI;
    double X_ini = YZ[0], Y_ini = YZ[1], U_ini = YZ[2], V_ini = YZ[3];
    double g2_ini = U_ini * U_ini + V_ini * V_ini;
    double r_ini = sqrt(X_ini * X_ini + Y_ini * Y_ini);
    double W = g2_ini + 2 * eps_th / r_ini;
    double L = X_ini * V_ini - Y_ini * U_ini;
    double r_g_ini = X_ini * U_ini + Y_ini * V_ini;
    double g_a = f_sign(sqrt(-W), L);
    double a = eps_th / W;
    double b = L / g_a;
    double omega_a = g_a / a;
    double ecc = sqrt((a * g_a) * (a * g_a) - L * L) / (a * g_a);
    double xi_ini;
    if (r_g_ini == 0) {
        if (r_ini < a) {
            xi_ini = 0;
        } else if (r_ini == a) {
            xi_ini = atan2(Y_ini, X_ini);
            ecc = 0;
        } else {
            xi_ini = f_sign(pi, L);
        }
    } else {
        xi_ini = atan2(r_g_ini / g_a, a - r_ini);
    }
    double alpha = atan2(Y_ini, X_ini) - atan2(b * sin(xi_ini), a * (cos(xi_ini) - ecc));
    double tau_ini = xi_ini - ecc * sin(xi_ini);
    double time_ini = tau_ini / omega_a;
    double time_end = time_ini + dt;
    double tau_end = omega_a * time_end;
    *error = 0;
    if (dt == 0) {
        for (int k = 0; k < 4; k++) YN[k] = YZ[k];
        return 0;
    }
    /* contained subroutine Newton, bia/find_ellipse.f90:106-157 */
    int ir = 0;
    double error_ini = tau_end - xi_ini + ecc * sin(xi_ini);
    double delta_ini = error_ini * (1 - ecc * cos(xi_ini));
    double xi_2;
    if (cos(tau_end) < 0.9)
        xi_2 = tau_end;
    else
        xi_2 = f_sign(pi / 2, sin(tau_end));
    double error_tm2 = tau_end - xi_2 + ecc * sin(xi_2);
    double delta_xi2 = error_tm2 / (1 - ecc * cos(xi_2));
    double xi;
    if (fabs(error_ini) < fabs(error_tm2))
        xi = xi_2 + delta_ini;
    else
        xi = xi_2 + delta_xi2;
    double xi_1 = NAN; /* uninitialised in the reference; compares unequal */
    double error_tm1;
    while (xi_1 != xi_2 && ir <= ITR) {
        ir = ir + 1;
        xi_1 = xi;
        error_tm1 = tau_end - xi_1 + ecc * sin(xi_1);
        double delta_xi1 = error_tm1 / (1 - ecc * cos(xi_1));
        xi = xi_1 + delta_xi1;
        if (error_tm1 == 0 || error_tm1 == error_tm2 || error_tm1 + error_tm2 == 0) {
            *error = error_tm1;
            break;
        }
        ir = ir + 1;
        xi_2 = xi;
        error_tm2 = tau_end - xi_2 + ecc * sin(xi_2);
        delta_xi2 = error_tm2 / (1 - ecc * cos(xi_2));
        xi = xi_2 + delta_xi2;
        if (error_tm2 == 0 || error_tm1 == error_tm2 || error_tm1 + error_tm2 == 0) {
            *error = error_tm2;
            break;
        }
    }
    double xi_end = xi;
    double cs_end = cos(xi_end);
    double sn_end = sin(xi_end);
    double xx_end = a * (cs_end - ecc);
    double yy_end = b * sn_end;
    double rr_end = a * (1 - ecc * cs_end);
    double uu_end = -a * g_a * sn_end / rr_end;
    double vv_end = b * g_a * cs_end / rr_end;
    double cs_alp = cos(alpha);
    double sn_alp = sin(alpha);
    YN[0] = xx_end * cs_alp - yy_end * sn_alp;
    YN[1] = xx_end * sn_alp + yy_end * cs_alp;
    YN[2] = uu_end * cs_alp - vv_end * sn_alp;
    YN[3] = uu_end * sn_alp + vv_end * cs_alp;
    return ir;
}

/* ---------------------------------------------------------------------------
 * bia/find_parabola.f90:1-143  find_parabola (diagnostic prints dropped)
 * ------------------------------------------------------------------------- */
typedef struct { double r_min, g_max; } par_common;

/* bia/find_parabola.f90:119-123 */
static double par_time(const par_common *c, double theta)
{
    double sn, cs;
    sincos(theta, &sn, &cs);
    return (2 + cs) * sn / ((1 + cs) * (1 + cs)) * 4 * c->r_min / (3 * c->g_max);
}
/* bia/find_parabola.f90:125-128 */
static double par_dt_dtheta(const par_common *c, double theta)
{
    double ch = cos(theta / 2);
    double ch2 = ch * ch;
    return c->r_min / (c->g_max * (ch2 * ch2));
}
/* bia/find_parabola.f90:108-118 */
static double par_F(double t)
{
    double s = sqrt(1 + t * t);
    return pow(s + t, 1.0 / 3) - pow(s - t, 1.0 / 3);
}

int oracle_find_parabola(double eps_th, double DT, const double YZ[4], double YN[4],
                         double *error_time)
{
    enum { NI = 99 };
    double theta_Newton[NI + 1], error_Newton[NI + 1];
    double r_ini = sqrt(YZ[0] * YZ[0] + YZ[1] * YZ[1]);
    double r_dot_g = YZ[0] * YZ[2] + YZ[1] * YZ[3];
    double r_crs_g = YZ[0] * YZ[3] - YZ[1] * YZ[2];
    par_common c;
    c.g_max = -2 * eps_th / r_crs_g;
    c.r_min = r_crs_g / c.g_max;
    double x_ini = 2 * c.r_min - r_ini;
    double y_ini = f_sign(2 * c.r_min * sqrt(r_ini / c.r_min - 1), r_dot_g);
    double theta_ini = atan2(y_ini, x_ini);
    double time_ini = par_time(&c, theta_ini);
    double time_end = time_ini + DT;
    double time_end_ = 3 * c.g_max / (4 * c.r_min) * time_end;
    double theta_gss = 2 * atan(par_F(time_end_));
    double theta = theta_gss;
    double err_tm_min = 1e99, thetamin = theta;
    int i_min = 1, i;
    for (i = 1; i <= NI; i++) {
        double err_tm = par_time(&c, theta) - time_end;
        error_Newton[i] = err_tm;
        double dtheta = -err_tm / par_dt_dtheta(&c, theta);
        if (fabs(err_tm) < err_tm_min) {
            err_tm_min = fabs(err_tm);
            thetamin = theta;
            i_min = i;
        }
        theta = theta + dtheta;
        theta_Newton[i] = theta;
        if (dtheta == 0) break;
        if (theta - dtheta == theta) break;
        int cyc = 0;
        for (int j = 1; j <= i - 1; j++)
            if (error_Newton[i] == error_Newton[j]) { cyc = 1; break; }
        if (cyc) { theta = theta_Newton[i_min]; break; }
    }
    if (i == NI + 1) theta = thetamin;
    double theta_end = theta;
    double beta_end = theta_end / 2;
    double sn_b, cs_b;
    sincos(beta_end, &sn_b, &cs_b);
    double r_end = c.r_min / (cs_b * cs_b);
    double g_end = c.g_max * cs_b;
    double x_end = r_end * cos(theta_end);
    double y_end = r_end * sin(theta_end);
    double u_end = -g_end * sn_b;
    double v_end = g_end * cs_b;
    double s1 = x_ini * YZ[1] - y_ini * YZ[0];
    double c1 = x_ini * YZ[0] + y_ini * YZ[1];
    double tmp = 1 / sqrt(s1 * s1 + c1 * c1);
    double sn_gamma = s1 * tmp, cs_gamma = c1 * tmp;
    YN[0] = x_end * cs_gamma - y_end * sn_gamma;
    YN[1] = x_end * sn_gamma + y_end * cs_gamma;
    YN[2] = u_end * cs_gamma - v_end * sn_gamma;
    YN[3] = u_end * sn_gamma + v_end * cs_gamma;
    *error_time = time_end - par_time(&c, theta_end);
    return (i > NI) ? NI : i;
}

/* ---------------------------------------------------------------------------
 * bia/find_dXYUV_RKF.f90:1-170  find_dXYUV_RKF / moon_2D / rkf / flstep /
 * fhstep / fehl: per-pair adaptive RKF4(5) with step doubling.
 * ------------------------------------------------------------------------- */
/* bia/find_dXYUV_RKF.f90:161-165 (Fehlberg coefficients) */
#define AL2 (1.0 / 4)
#define AL3 (3.0 / 8)
#define AL4 (12.0 / 13)
#define AL5 (1.0)
#define AL6 (1.0 / 2)
#define B21 (1.0 / 4)
#define B31 (3.0 / 32)
#define B32 (9.0 / 32)
#define B41 (1932.0 / 2197)
#define B42 (-7200.0 / 2197)
#define B43 (7296.0 / 2197)
#define B51 (439.0 / 216)
#define B52 (-8.0)
#define B53 (3680.0 / 513)
#define B54 (-845.0 / 4104)
#define B61 (-8.0 / 27)
#define B62 (2.0)
#define B63 (-3544.0 / 2565)
#define B64 (1859.0 / 4104)
#define B65 (-11.0 / 40)
#define GA1 (16.0 / 135)
#define GA3 (6656.0 / 12825)
#define GA4 (28561.0 / 56430)
#define GA5 (-9.0 / 50)
#define GA6 (2.0 / 55)
#define DA1 (1.0 / 360)
#define DA3 (-128.0 / 4275)
#define DA4 (-2197.0 / 75240)
#define DA5 (1.0 / 50)
#define DA6 (2.0 / 55)

typedef void (*rhs_fn)(const void *ctx, double x, const double *y, double *f);

/* bia/find_dXYUV_RKF.f90:150-157 fehl, generic over neq */
static void fehl_n(int lindex, int neq, rhs_fn f, const void *ctx, double x, double h,
                   const double *y0, double *yn, double *er, double *wk)
{
    double *ak1 = wk, *ak2 = wk + neq, *ak3 = wk + 2 * neq, *ak4 = wk + 3 * neq;
    double *ak5 = wk + 4 * neq, *ak6 = wk + 5 * neq, *w2 = wk + 6 * neq, *w3 = wk + 7 * neq;
    double *w4 = wk + 8 * neq, *w5 = wk + 9 * neq, *w6 = wk + 10 * neq;
    int i;
    f(ctx, x, y0, ak1);
    for (i = 0; i < neq; i++) w2[i] = y0[i] + h * B21 * ak1[i];
    f(ctx, x + AL2 * h, w2, ak2);
    for (i = 0; i < neq; i++) w3[i] = y0[i] + h * (B31 * ak1[i] + B32 * ak2[i]);
    f(ctx, x + AL3 * h, w3, ak3);
    for (i = 0; i < neq; i++) w4[i] = y0[i] + h * (B41 * ak1[i] + B42 * ak2[i] + B43 * ak3[i]);
    f(ctx, x + AL4 * h, w4, ak4);
    for (i = 0; i < neq; i++)
        w5[i] = y0[i] + h * (B51 * ak1[i] + B52 * ak2[i] + B53 * ak3[i] + B54 * ak4[i]);
    f(ctx, x + AL5 * h, w5, ak5);
    for (i = 0; i < neq; i++)
        w6[i] = y0[i] + h * (B61 * ak1[i] + B62 * ak2[i] + B63 * ak3[i] + B64 * ak4[i] + B65 * ak5[i]);
    f(ctx, x + AL6 * h, w6, ak6);
    for (i = 0; i < neq; i++)
        yn[i] = y0[i] + h * (GA1 * ak1[i] + GA3 * ak3[i] + GA4 * ak4[i] + GA5 * ak5[i] + GA6 * ak6[i]);
    if (lindex == 1)
        for (i = 0; i < neq; i++)
            er[i] = h * (DA1 * ak1[i] + DA3 * ak3[i] + DA4 * ak4[i] + DA5 * ak5[i] + DA6 * ak6[i]);
}

/* bia/find_dXYUV_RKF.f90:136-148 fhstep: two half steps; y0 is overwritten by the midpoint */
static void fhstep_n(int neq, rhs_fn f, const void *ctx, double x, double h, double *y0,
                     double *yn, double *er, double *wk)
{
    double h1 = h / 2;
    fehl_n(0, neq, f, ctx, x, h1, y0, yn, er, wk);
    double x1 = x + h1;
    for (int i = 0; i < neq; i++) y0[i] = yn[i];
    fehl_n(0, neq, f, ctx, x1, h1, y0, yn, er, wk);
}

/* bia/find_dXYUV_RKF.f90:15-23 moon_2D */
static void moon_2d(const void *ctx, double x, const double *Y, double *F)
{
    (void)x;
    double eps_th = *(const double *)ctx;
    double rsq = Y[0] * Y[0] + Y[1] * Y[1];
    double aaa = eps_th / (rsq * sqrt(rsq));
    F[0] = Y[2];
    F[2] = Y[0] * aaa;
    F[1] = Y[3];
    F[3] = Y[1] * aaa;
}

/* bia/find_dXYUV_RKF.f90:25-117 rkf (init == 1 path).  On return yhn holds
 * the step-doubled solution.  Returns ier (0, 20000 or 30000; 10000 when the
 * iteration limit is reached). */
static int rkf_n(int neq, rhs_fn f, const void *ctx, double x0, double xe, double *yh0,
                 double relerr, double abserr, double *yhn, double *esterr, int *nacc,
                 double *yl0, double *yln, double *er, double *wk)
{
    const int itemax = 100000;
    const double epsmin = 1e-15;
    for (int i = 0; i < neq; i++) yl0[i] = yh0[i];
    f(ctx, x0, yl0, wk);
    double toldy = DBL_MAX;
    for (int i = 0; i < neq; i++) {
        if (wk[i] != 0) {
            double tol = relerr * fabs(yl0[i]) + abserr;
            double q = fabs(tol / wk[i]);
            if (q < toldy) toldy = q;
        }
    }
    double hmin = epsmin * (xe - x0);
    double h = (toldy == DBL_MAX) ? hmin : fmin((xe - x0) / 100, pow(toldy, 0.2));
    double x = x0;
    *nacc = 0;
    for (int iter = 1; iter <= itemax; iter++) {
        fehl_n(1, neq, f, ctx, x, h, yl0, yln, er, wk);
        double erret = 0;
        for (int i = 0; i < neq; i++) {
            double et = relerr / 2 * (fabs(yl0[i]) + fabs(yln[i])) + abserr;
            if (et == 0) return 20000;
            double q = fabs(er[i]) / et;
            if (q > erret) erret = q;
        }
        if (erret > 1) {
            if (erret >= 59049)
                h = 0.1 * h;
            else
                h = 0.9 * h / pow(erret, 0.2);
            if (h <= epsmin) return 30000;
        } else if (x + h < xe) {
            fhstep_n(neq, f, ctx, x, h, yh0, yhn, er, wk);
            x = x + h;
            for (int i = 0; i < neq; i++) { yl0[i] = yln[i]; yh0[i] = yhn[i]; }
            (*nacc)++;
            if (erret <= 1.889568e-4)
                h = 5 * h;
            else
                h = 0.9 * h / pow(erret, 0.2);
        } else {
            h = xe - x;
            fehl_n(1, neq, f, ctx, x, h, yl0, yln, er, wk);
            fhstep_n(neq, f, ctx, x, h, yh0, yhn, er, wk);
            for (int i = 0; i < neq; i++) esterr[i] = (yln[i] - yhn[i]) / 31;
            for (int i = 0; i < neq; i++) { yl0[i] = yln[i]; yh0[i] = yhn[i]; }
            (*nacc)++;
            return 0;
        }
    }
    return 10000;
}

/* bia/find_dXYUV_RKF.f90:1-13 find_dXYUV_RKF: relerr = 0, abserr = 1e-16 by default */
int oracle_find_dxyuv_rkf(double eps_th, double xe, const double YZ[4], double YN[4],
                          double *error, double relerr, double abserr, int *nacc)
{
    double y0[4], esterr[4] = {0, 0, 0, 0}, yl0[4], yln[4], er[4], wk[44];
    for (int i = 0; i < 4; i++) { y0[i] = YZ[i]; YN[i] = YZ[i]; }
    int n = 0;
    int ier = rkf_n(4, moon_2d, &eps_th, 0.0, xe, y0, relerr, abserr, YN, esterr, &n, yl0, yln, er, wk);
    double m = esterr[0];
    for (int i = 1; i < 4; i++) if (esterr[i] > m) m = esterr[i];
    *error = m;
    if (nacc) *nacc = n;
    return ier;
}

/* ---------------------------------------------------------------------------
 * bia/bia.f90:141-196  one pair (i, j): frame, classification, solver and the
 * half-displacements (dXXXh..dWijh) that bia.f90 adds to i and subtracts from j.
 * method: 1 = ALG, 0 = RKF.  h[0..5] receives (dXXXh, dYYYh, dZZZh, dUijh, dVijh, dWijh).
 * ------------------------------------------------------------------------- */
typedef struct {
    int method, ITR;
    double ERR, dt, relerr, abserr;
} pair_cfg;

static void oracle_pair(const pair_cfg *cfg, double eps_th, const double r[3], const double g[3],
                        double h[6], oracle_stats *st)
{
    double e_xi[3], e_eta[3], e_zeta[3], YZ[4], YN[4], error = 0;
    int degenerate = oracle_xyz_to_xi_eta_zeta(r, g, e_xi, e_eta, e_zeta, YZ);
    if (degenerate || cfg->method == 0) {
        int nacc = 0;
        oracle_find_dxyuv_rkf(eps_th, cfg->dt, YZ, YN, &error, cfg->relerr, cfg->abserr, &nacc);
        if (st) {
            st->count[degenerate ? OC_DEGENERATE : OC_RKF]++;
            st->rkf_steps += nacc;
            if (fabs(error) > cfg->ERR) st->nonconverged++;
        }
    } else {
        double r_ij = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
        double E_ij = g[0] * g[0] + g[1] * g[1] + g[2] * g[2] + 2 * eps_th / r_ij;
        int it, cls, bx = 0;
        if (E_ij > 0) {
            it = oracle_find_hyperbola(eps_th, cfg->dt, YZ, YN, &error, cfg->ITR, &bx);
            cls = OC_HYPERBOLA;
        } else if (E_ij == 0) {
            it = oracle_find_parabola(eps_th, cfg->dt, YZ, YN, &error);
            cls = OC_PARABOLA;
        } else {
            it = oracle_find_ellipse(eps_th, cfg->dt, YZ, YN, &error, cfg->ITR);
            cls = OC_ELLIPSE;
        }
        if (st) {
            st->count[cls]++;
            st->iterations += it;
            st->bracket_exits += bx;
            if (fabs(error) > cfg->ERR) st->nonconverged++;
        }
    }
    double dr_xi = YN[0] - YZ[0], dr_eta = YN[1] - YZ[1];
    double dX_ij = dr_xi * e_xi[0] + dr_eta * e_eta[0];
    double dY_ij = dr_xi * e_xi[1] + dr_eta * e_eta[1];
    double dZ_ij = dr_xi * e_xi[2] + dr_eta * e_eta[2];
    double dg_xi = YN[2] - YZ[2], dg_eta = YN[3] - YZ[3];
    h[3] = (dg_xi * e_xi[0] + dg_eta * e_eta[0]) / 2;
    h[4] = (dg_xi * e_xi[1] + dg_eta * e_eta[1]) / 2;
    h[5] = (dg_xi * e_xi[2] + dg_eta * e_eta[2]) / 2;
    h[0] = (dX_ij - g[0] * cfg->dt) / 2;
    h[1] = (dY_ij - g[1] * cfg->dt) / 2;
    h[2] = (dZ_ij - g[2] * cfg->dt) / 2;
}

/* Public single-pair entry: relative state r = x_i - x_j, g = v_i - v_j. */
void oracle_pair_halfdisp(int method, double eps_th, double dt, int ITR, double relerr,
                          double abserr, const double r[3], const double g[3], double h[6],
                          int64_t *stats /* 10 int64 or NULL */)
{
    pair_cfg cfg = {method, ITR, 1e-12, dt, relerr, abserr};
    oracle_stats st;
    memset(&st, 0, sizeof st);
    oracle_pair(&cfg, eps_th, r, g, h, &st);
    if (stats) memcpy(stats, &st, sizeof st);
}

static double pair_eps(double eps_th, const double *q, int i, int j)
{
    return q ? eps_th * q[i] * q[j] : eps_th;
}

/* ---------------------------------------------------------------------------
 * bia/bia.f90:126-204 (CPU branch): one BIA step over all pairs, in the
 * reference's order (i ascending, j = i+1..N), then drift and the update
 * X += dX, U += dU.  Arrays are SoA of length n.  dX..dW receive the step's
 * displacements (as written to the .BIA record, bia/bia.f90:206).
 * ------------------------------------------------------------------------- */
void oracle_bia_step(int method, int n, double eps_th, const double *q, double dt, int ITR,
                     double relerr, double abserr, double *X, double *Y, double *Z, double *U,
                     double *V, double *W, double *dX, double *dY, double *dZ, double *dU,
                     double *dV, double *dW, int64_t *stats)
{
    pair_cfg cfg = {method, ITR, 1e-12, dt, relerr, abserr};
    oracle_stats st;
    memset(&st, 0, sizeof st);
    for (int i = 0; i < n; i++) { dX[i] = dY[i] = dZ[i] = dU[i] = dV[i] = dW[i] = 0; }
    for (int i = 0; i < n; i++) {
        for (int j = i + 1; j < n; j++) {
            double r[3] = {X[i] - X[j], Y[i] - Y[j], Z[i] - Z[j]};
            double g[3] = {U[i] - U[j], V[i] - V[j], W[i] - W[j]};
            double h[6];
            oracle_pair(&cfg, pair_eps(eps_th, q, i, j), r, g, h, &st);
            dX[i] = dX[i] + h[0]; dY[i] = dY[i] + h[1]; dZ[i] = dZ[i] + h[2];
            dX[j] = dX[j] - h[0]; dY[j] = dY[j] - h[1]; dZ[j] = dZ[j] - h[2];
            dU[i] = dU[i] + h[3]; dV[i] = dV[i] + h[4]; dW[i] = dW[i] + h[5];
            dU[j] = dU[j] - h[3]; dV[j] = dV[j] - h[4]; dW[j] = dW[j] - h[5];
        }
        dX[i] = dX[i] + U[i] * dt;
        dY[i] = dY[i] + V[i] * dt;
        dZ[i] = dZ[i] + W[i] * dt;
    }
    for (int i = 0; i < n; i++) {
        X[i] = X[i] + dX[i]; Y[i] = Y[i] + dY[i]; Z[i] = Z[i] + dZ[i];
        U[i] = U[i] + dU[i]; V[i] = V[i] + dV[i]; W[i] = W[i] + dW[i];
    }
    if (stats) memcpy(stats, &st, sizeof st);
}

/* Row-sampled step for the CPU baseline: processes rows i in rows[0..nrows)
 * (all j > i) with OpenMP, accumulating into per-thread buffers.  Returns the
 * number of pairs processed.  Used only to time the CPU path on a bounded
 * sample; the displacement sums land in dX..dW (zeroed first, no drift). */
int64_t oracle_bia_rows_omp(int method, int n, double eps_th, const double *q, double dt, int ITR,
                            double relerr, double abserr, const double *X, const double *Y,
                            const double *Z, const double *U, const double *V, const double *W,
                            const int *rows, int nrows, double *dX, double *dY, double *dZ,
                            double *dU, double *dV, double *dW, int nthreads, int64_t *stats)
{
    pair_cfg cfg = {method, ITR, 1e-12, dt, relerr, abserr};
    int64_t pairs = 0;
    for (int k = 0; k < nrows; k++) pairs += n - 1 - rows[k];
    for (int i = 0; i < n; i++) { dX[i] = dY[i] = dZ[i] = dU[i] = dV[i] = dW[i] = 0; }
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#else
    nthreads = 1;
#endif
    double *acc = (double *)calloc((size_t)nthreads * 6 * n, sizeof(double));
    oracle_stats *sts = (oracle_stats *)calloc((size_t)nthreads, sizeof(oracle_stats));
#pragma omp parallel num_threads(nthreads)
    {
        int t = 0;
#ifdef _OPENMP
        t = omp_get_thread_num();
#endif
        double *a = acc + (size_t)t * 6 * n;
#pragma omp for schedule(dynamic, 1)
        for (int k = 0; k < nrows; k++) {
            int i = rows[k];
            for (int j = i + 1; j < n; j++) {
                double r[3] = {X[i] - X[j], Y[i] - Y[j], Z[i] - Z[j]};
                double g[3] = {U[i] - U[j], V[i] - V[j], W[i] - W[j]};
                double h[6];
                oracle_pair(&cfg, pair_eps(eps_th, q, i, j), r, g, h, &sts[t]);
                for (int c = 0; c < 6; c++) {
                    a[(size_t)c * n + i] += h[c];
                    a[(size_t)c * n + j] -= h[c];
                }
            }
        }
    }
    double *outs[6] = {dX, dY, dZ, dU, dV, dW};
    for (int t = 0; t < nthreads; t++)
        for (int c = 0; c < 6; c++)
            for (int i = 0; i < n; i++) outs[c][i] += acc[((size_t)t * 6 + c) * n + i];
    if (stats) {
        oracle_stats tot;
        memset(&tot, 0, sizeof tot);
        for (int t = 0; t < nthreads; t++) {
            for (int c = 0; c < 5; c++) tot.count[c] += sts[t].count[c];
            tot.iterations += sts[t].iterations;
            tot.rkf_steps += sts[t].rkf_steps;
            tot.nonconverged += sts[t].nonconverged;
            tot.bracket_exits += sts[t].bracket_exits;
        }
        memcpy(stats, &tot, sizeof tot);
    }
    free(acc);
    free(sts);
    return pairs;
}

/* Full displacement of selected particles p (all pairs j != p, drift included), for
 * parity checks at sizes where a whole oracle step is too slow.  The pair (p, j) with
 * j < p is evaluated as r = x_p - x_j, which by the exact antisymmetry of the pair
 * formulas equals minus the reference's h(j, p).  out: [nsel][6]. */
void oracle_particle_disp(int method, int n, double eps_th, const double *q, double dt, int ITR,
                          double relerr, double abserr, const double *X, const double *Y,
                          const double *Z, const double *U, const double *V, const double *W,
                          const int *sel, int nsel, double *out, int nthreads)
{
    pair_cfg cfg = {method, ITR, 1e-12, dt, relerr, abserr};
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#else
    nthreads = 1;
#endif
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
    for (int k = 0; k < nsel; k++) {
        int p = sel[k];
        double acc[6] = {0, 0, 0, 0, 0, 0};
        for (int j = 0; j < n; j++) {
            if (j == p) continue;
            double r[3] = {X[p] - X[j], Y[p] - Y[j], Z[p] - Z[j]};
            double g[3] = {U[p] - U[j], V[p] - V[j], W[p] - W[j]};
            double h[6];
            oracle_pair(&cfg, pair_eps(eps_th, q, p, j), r, g, h, NULL);
            for (int c = 0; c < 6; c++) acc[c] += h[c];
        }
        acc[0] += U[p] * dt;
        acc[1] += V[p] * dt;
        acc[2] += W[p] * dt;
        for (int c = 0; c < 6; c++) out[(size_t)k * 6 + c] = acc[c];
    }
}

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
