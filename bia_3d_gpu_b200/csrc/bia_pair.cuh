// bia_pair.cuh -- per-pair BIA solvers in FP64 for sm_100a.
//
// One unordered pair (i, j) with relative state r = x_i - x_j, g = v_i - v_j is
// reduced to a planar two-body problem (bia/bia.f90:284-314), classified by its
// energy (bia/bia.f90:156-166) and advanced over dt by the hyperbola, parabola or
// ellipse solver (bia/find_hyperbola.f90, find_parabola.f90, find_ellipse.f90) or by
// the per-pair RKF4(5) (bia/find_dXYUV_RKF.f90).  The result is the pair's
// half-displacement h (bia/bia.f90:173-185): i receives +h, j receives -h.
//
// The formulas follow the reference's CPU path; CUDA's double-precision math
// functions replace glibc's, and nvcc's FMA contraction is left on, so results agree
// with the CPU oracle to rounding, not bit for bit.  The same deviations as the
// oracle are taken where the reference is undefined or fails in FP64: uninitialised
// theta_stock, bracket exit without a result, iterations that end unconverged
// (bracketed re-solve), and pairs with zero |g| or |L| or with |e^2 - 1| < 0.1 (the
// classical parametrisations lose up to every digit there), which are advanced by a
// universal-variable (Stumpff function) solver.
#pragma once
#include <cstdint>

namespace bia {

constexpr double kPi = 3.14159265358979323846264338327950288419716939937510582097494;

// Optional out-of-line FP64 math: each libm call site expands to a long instruction
// sequence; routing the calls through one copy shrinks the code.  Measured on B200
// (n = 32768, 3 CTAs/SM): out-of-line math and hyp_eval 204 ms (Coulomb, mixed orbit
// classes) / 88 ms (Plummer, hyperbolae only) per step, everything inline 213 / 73 ms;
// inline is the default.
#ifndef BIA_NOINLINE_MATH
#define BIA_NOINLINE_MATH 0
#endif
#if BIA_NOINLINE_MATH
static __device__ __noinline__ void d_sincos(double x, double *s, double *c) { sincos(x, s, c); }
static __device__ __noinline__ double d_log(double x) { return log(x); }
static __device__ __noinline__ double d_atan2(double y, double x) { return atan2(y, x); }
static __device__ __noinline__ double d_acos(double x) { return acos(x); }
static __device__ __noinline__ double d_atan(double x) { return atan(x); }
#else
__device__ __forceinline__ void d_sincos(double x, double *s, double *c) { sincos(x, s, c); }
__device__ __forceinline__ double d_log(double x) { return log(x); }
__device__ __forceinline__ double d_atan2(double y, double x) { return atan2(y, x); }
__device__ __forceinline__ double d_acos(double x) { return acos(x); }
__device__ __forceinline__ double d_atan(double x) { return atan(x); }
#endif
#ifndef BIA_NOINLINE_HYPEVAL
#define BIA_NOINLINE_HYPEVAL 0
#endif
#if BIA_NOINLINE_HYPEVAL
#define BIA_HYPEVAL_INLINE static __device__ __noinline__
#else
#define BIA_HYPEVAL_INLINE __device__ __forceinline__
#endif

enum PairClass { kHyperbola = 0, kParabola = 1, kEllipse = 2, kDegenerate = 3, kRkf = 4, kUniversal = 5 };

// |e^2 - 1| below which ALG pairs use the universal-variable solver
constexpr double kNearUnitEcc = 0.1;

struct PairParams {
    double dt;
    double err;      // ERR, residual threshold for the not-converged count
    double relerr;   // RKF tolerances
    double abserr;
    int itr;         // Newton cap ITR
    int method;      // 0 RKF, 1 ALG, 2 universal variables for every pair
};

// Per-thread counters, reduced per warp before one atomic per counter.
struct PairCounters {
    int cls[6];
    int it_hyp, it_ell, it_par, it_uv;
    int rkf_steps;
    int nonconverged;
    int bracket_exits;
    int fallbacks;
    int nonfinite;
    int learned, learned_fallbacks, learned_coarse;  // BIA_METHOD_LEARNED
    int timeouts;
    int learned_fp32;  // FP32 Newton steps of the learned pairs' first correction
};

__device__ __forceinline__ void counters_zero(PairCounters &c)
{
#pragma unroll
    for (int k = 0; k < 6; k++) c.cls[k] = 0;
    c.it_hyp = c.it_ell = c.it_par = c.it_uv = 0;
    c.rkf_steps = c.nonconverged = c.bracket_exits = c.fallbacks = c.nonfinite = 0;
    c.learned = c.learned_fallbacks = c.learned_coarse = c.timeouts = c.learned_fp32 = 0;
}

#ifndef BIA_DIRECT_HALF_SINES
#define BIA_DIRECT_HALF_SINES 0
#endif
#ifndef BIA_STRICT_SETUP
#define BIA_STRICT_SETUP 0
#endif
#ifndef BIA_REF_END_STATE
#define BIA_REF_END_STATE 1
#endif
// Uncontracted IEEE operations, in the oracle's (the reference's) order: the frame and the
// hyperbola's start angle acos(cs_0 + b sn_0 / r) are ill-conditioned near pericentre
// (d theta / d arg ~ 1 / sqrt(1 - arg)), so an ulp of difference in the argument becomes
// up to ~1e-10 of displacement; these values are formed exactly as the CPU path forms
// them (no fused multiply-add, divisions instead of reciprocals).
__device__ __forceinline__ double m_(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double a_(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double s_(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double d_(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ double dot3_(const double a[3], const double b[3])
{
    return a_(a_(m_(a[0], b[0]), m_(a[1], b[1])), m_(a[2], b[2]));
}

// bia/bia.f90:284-314.  Returns true for a degenerate pair (|g| == 0 or |L| == 0):
// then the frame is the line of motion and Y has a single nonzero position axis.
__device__ __forceinline__ bool frame_xi_eta(const double r[3], const double g[3], double e_xi[3],
                                             double e_eta[3], double Y[4])
{
    const double gsq = dot3_(g, g);
    const double gm = __dsqrt_rn(gsq);
    double L[3];
    L[0] = s_(m_(r[1], g[2]), m_(r[2], g[1]));
    L[1] = s_(m_(r[2], g[0]), m_(r[0], g[2]));
    L[2] = s_(m_(r[0], g[1]), m_(r[1], g[0]));
    const double Lsq = dot3_(L, L);
    if (gm == 0.0 || Lsq == 0.0) {
        if (gm == 0.0) {
            const double rm = __dsqrt_rn(dot3_(r, r));
#pragma unroll
            for (int k = 0; k < 3; k++) { e_xi[k] = d_(r[k], rm); e_eta[k] = 0.0; }
            Y[0] = rm; Y[1] = 0.0; Y[2] = 0.0; Y[3] = 0.0;
        } else {
#pragma unroll
            for (int k = 0; k < 3; k++) { e_eta[k] = d_(g[k], gm); e_xi[k] = 0.0; }
            Y[0] = 0.0;
            Y[1] = dot3_(r, e_eta);
            Y[2] = 0.0;
            Y[3] = gm;
        }
        return true;
    }
    double ez[3];
#if BIA_STRICT_SETUP
    const double Lm = __dsqrt_rn(Lsq);
#pragma unroll
    for (int k = 0; k < 3; k++) {
        e_eta[k] = d_(g[k], gm);
        ez[k] = d_(L[k], Lm);
    }
#else
    const double iL = 1.0 / sqrt(Lsq), ig = 1.0 / gm;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        e_eta[k] = g[k] * ig;
        ez[k] = L[k] * iL;
    }
#endif
    e_xi[0] = s_(m_(e_eta[1], ez[2]), m_(e_eta[2], ez[1]));
    e_xi[1] = s_(m_(e_eta[2], ez[0]), m_(e_eta[0], ez[2]));
    e_xi[2] = s_(m_(e_eta[0], ez[1]), m_(e_eta[1], ez[0]));
    Y[0] = dot3_(r, e_xi);
    Y[2] = 0.0;
    Y[1] = dot3_(r, e_eta);
    Y[3] = gm;
    return false;
}

// ---------------------------------------------------------------------------
// bia/find_hyperbola.f90:1-166.  Returns the main-loop iteration count.
//
// The reference's time equation and Newton iteration in theta, evaluated through the
// half angle: with (sh, ch) = sincos(theta/2) and (s0h, c0h) = sincos(theta_0/2),
//   sin((theta_0 +- theta)/2) = s0h ch +- c0h sh,  sin theta = 2 sh ch,
//   cos theta = 1 - 2 sh^2,  cos theta - cos theta_0 = 2 sin((theta_0+theta)/2) sin((theta_0-theta)/2),
// so one sincos replaces the reference's sin, sin and sincos per evaluation, and the
// denominator cos theta - cos theta_0 is a product instead of a difference.
// ---------------------------------------------------------------------------
struct HypConsts {
    double theta_0, tn_0, cs_0, sn_0, s0h, c0h, time_end_;
};

// sin((theta_0 +- theta)/2) from the half angles.  Near theta = +-theta_0 (far along an
// asymptote) the difference of products cancels, so below 0.25 the sine of the small half
// angle is taken directly, as the reference computes it (bia/find_hyperbola.f90:157-158).
__device__ __forceinline__ void half_sines(const HypConsts &c, double theta, double sh, double ch, double &sp,
                                          double &sm)
{
    sp = c.s0h * ch + c.c0h * sh;
    sm = c.s0h * ch - c.c0h * sh;
#if BIA_DIRECT_HALF_SINES
    if (fabs(sm) < 0.25) sm = sin(0.5 * (c.theta_0 - theta));
    if (fabs(sp) < 0.25) sp = sin(0.5 * (c.theta_0 + theta));
#endif
}

// find_theta (bia/find_hyperbola.f90:149-165): residual e and derivative d at theta;
// sp, sm = sin((theta_0 +- theta)/2) for the bracket test.
BIA_HYPEVAL_INLINE void hyp_eval(const HypConsts &c, double theta, double &e, double &d,
                                         double &sp, double &sm)
{
    double sh, ch;
    d_sincos(0.5 * theta, &sh, &ch);
    half_sines(c, theta, sh, ch, sp, sm);
    const double Dinv = 1.0 / (2.0 * sp * sm);
    const double sn = 2.0 * sh * ch;
    const double cs = 1.0 - 2.0 * sh * sh;
    e = c.tn_0 * sn * Dinv - c.time_end_ + d_log(sp / sm);
    d = c.tn_0 * (1.0 - c.cs_0 * cs) * (Dinv * Dinv) + c.sn_0 * Dinv;
}

// Bracketed Newton-bisection on the same time equation, used only when the reference's
// loop ends without a small residual.  The equation is monotonic on (-theta_0, theta_0):
// increasing for repulsive pairs (tn_0 > 0), decreasing for attractive ones.
static __device__ __noinline__ double hyp_safe(const HypConsts c, double x)
{
    double lo = -c.theta_0, hi = c.theta_0;
    const double dir = (c.tn_0 > 0.0) ? 1.0 : -1.0;
    if (!(x > lo && x < hi)) x = 0.0;
    for (int it = 0; it < 400; it++) {
        double f, d, sp, sm;
        hyp_eval(c, x, f, d, sp, sm);
        if (f == 0.0) break;
        if (f * dir < 0.0) lo = x; else hi = x;
        double xn = x - f / d;
        if (!(xn > lo && xn < hi)) xn = 0.5 * (lo + hi);
        if (xn == x) break;
        x = xn;
    }
    return x;
}

__device__ __forceinline__ int hyperbola(double eps_th, double dt, int ITR, const double YZ[4],
                                         double YN[4], double *error_end, int *bracket_exit,
                                         int *fallback)
{
    const double X_ini = YZ[0], Y_ini = YZ[1], U_ini = YZ[2], V_ini = YZ[3];
#if BIA_STRICT_SETUP
    // up to the start angle: the oracle's operations and order (see m_ above)
    const double r_g = a_(m_(X_ini, U_ini), m_(Y_ini, V_ini));
    const double Lz = s_(m_(X_ini, V_ini), m_(Y_ini, U_ini));
    const double r = __dsqrt_rn(a_(m_(X_ini, X_ini), m_(Y_ini, Y_ini)));
    const double g2 = a_(m_(U_ini, U_ini), m_(V_ini, V_ini));
    const double W = a_(g2, d_(m_(2.0, eps_th), r));
    const double g_0 = __dsqrt_rn(W);
    const double b_0 = d_(eps_th, W);
    const double b = d_(fabs(Lz), g_0);
    HypConsts c;
    const double bg = m_(b_0, g_0);
    c.theta_0 = d_atan2(fabs(Lz), bg);
    const double den0 = __dsqrt_rn(a_(m_(m_(b_0, b_0), m_(g_0, g_0)), m_(Lz, Lz)));
    c.cs_0 = d_(bg, den0);
    c.sn_0 = d_(fabs(Lz), den0);
    c.tn_0 = d_(fabs(Lz), bg);
    d_sincos(0.5 * c.theta_0, &c.s0h, &c.c0h);
    const double arg = a_(c.cs_0, d_(m_(b, c.sn_0), r));
#else
    const double r_g = X_ini * U_ini + Y_ini * V_ini;
    const double Lz = X_ini * V_ini - Y_ini * U_ini;
    const double r = sqrt(X_ini * X_ini + Y_ini * Y_ini);
    const double g2 = U_ini * U_ini + V_ini * V_ini;
    const double W = g2 + 2.0 * eps_th / r;
    const double g_0 = sqrt(W);
    const double b_0 = eps_th / W;
    const double b = fabs(Lz) / g_0;
    HypConsts c;
    const double bg = b_0 * g_0;
    c.theta_0 = d_atan2(fabs(Lz), bg);
    const double den0 = sqrt(b_0 * b_0 * (g_0 * g_0) + Lz * Lz);
    c.cs_0 = bg / den0;
    c.sn_0 = fabs(Lz) / den0;
    c.tn_0 = fabs(Lz) / bg;
    d_sincos(0.5 * c.theta_0, &c.s0h, &c.c0h);
    const double arg = c.cs_0 + b * c.sn_0 / r;
#endif
    double theta_ini = (fabs(arg) > 1.0) ? 1e-30 : d_acos(arg);
    if (Lz * r_g < 0.0) theta_ini = -theta_ini;
    // state and dimensionless time at theta_ini (bia/find_hyperbola.f90:46-64)
    double sh, ch;
    d_sincos(0.5 * theta_ini, &sh, &ch);
    double sp_i, sm_i;
    half_sines(c, theta_ini, sh, ch, sp_i, sm_i);
    const double Dinv_i = 1.0 / (2.0 * sp_i * sm_i);
#if BIA_REF_END_STATE
    // the start position and the end state take sin and cos of the full angle, as the
    // reference does: the end position is a difference of two positions of magnitude r,
    // and only the same formula at both ends keeps their rounding from adding a bias
    double sn, cs;
    d_sincos(theta_ini, &sn, &cs);
    const double x = r * cs, y = r * sn;
    const double g0_sn0 = (Lz > 0.0) ? g_0 / c.sn_0 : -g_0 / c.sn_0;
    const double u = g0_sn0 * (c.cs_0 * sn);
    const double v = g0_sn0 * (1.0 - c.cs_0 * cs);
    const double den_a = sqrt((X_ini * X_ini + Y_ini * Y_ini) * (x * x + y * y));
    const double cs_a = (x * X_ini + y * Y_ini) / den_a;
    const double sn_a = (x * Y_ini - y * X_ini) / den_a;
#else
    const double sn = 2.0 * sh * ch, cs = 1.0 - 2.0 * sh * sh;
    const double x = r * cs, y = r * sn;
    const double g0_sn0 = (Lz > 0.0) ? g_0 / c.sn_0 : -g_0 / c.sn_0;
    const double u = g0_sn0 * (c.cs_0 * sn);
    const double v = g0_sn0 * (1.0 - c.cs_0 * cs);
    const double den_a = 1.0 / sqrt((X_ini * X_ini + Y_ini * Y_ini) * (x * x + y * y));
    const double cs_a = (x * X_ini + y * Y_ini) * den_a;
    const double sn_a = (x * Y_ini - y * X_ini) * den_a;
#endif
    const double tau_ini = c.tn_0 * sn * Dinv_i + d_log(sp_i / sm_i);
    const double time_ini = tau_ini * b_0 / g_0;
    const double time_end = (Lz > 0.0) ? time_ini + dt : time_ini - dt;
    c.time_end_ = time_end * g_0 / b_0;

    // two candidate starts (bia/find_hyperbola.f90:71-89): one Newton step from theta_ini
    // (its residual is known already) and one from the atan guess
    const double error_ini_ = tau_ini - c.time_end_;
    const double d_ini = c.tn_0 * (1.0 - c.cs_0 * cs) * (Dinv_i * Dinv_i) + c.sn_0 * Dinv_i;
    const double th_ini_end = (error_ini_ == 0.0) ? theta_ini : theta_ini - error_ini_ / d_ini;
    const double theta_gss = 2.0 / kPi * c.theta_0 * d_atan(c.time_end_ / c.tn_0);
    double error_gss_, d_gss, spg, smg;
    hyp_eval(c, theta_gss, error_gss_, d_gss, spg, smg);
    const double th_gss_end = (error_gss_ == 0.0) ? theta_gss : theta_gss - error_gss_ / d_gss;
    double theta_end, error_;
    if (fabs(error_gss_) > 10.0 * fabs(error_ini_)) {
        theta_end = th_ini_end;
        error_ = error_ini_;
    } else {
        theta_end = th_gss_end;
        error_ = error_gss_;
    }
    // minimum-residual Newton loop with cycle detection (bia/find_hyperbola.f90:93-120).
    // The reference compares each residual with every earlier one (error_restore_); here
    // the last four are kept in registers (h0 newest): an indexed history array lives in
    // local memory, whose write-back was most of the ALG kernel's DRAM traffic.  A cycle
    // only arises once the iteration sits at the rounding floor, where the iterates that
    // repeat are a few ulps apart; cycles of period 1-4 stop at the same iteration as in
    // the reference, a longer one runs on to the ITR cap with the same stock update rule.
    double err_stock = error_;
    double theta_stock = theta_end;
    double best_res = fabs(error_);
    const double kNoResidual = __longlong_as_double(0x7ff8000000000000LL);  // compares unequal
    double h0 = kNoResidual, h1 = kNoResidual, h2 = kNoResidual, h3 = kNoResidual;
    int IR = 0;
    *bracket_exit = 0;
    while (IR < ITR) {
        const double theta_now = theta_end;
        double e, d, sp, sm;
        hyp_eval(c, theta_now, e, d, sp, sm);
        if (sp * sm < 0.0) {
            *bracket_exit = 1;
            break;
        }
        error_ = e;
        theta_end = (e == 0.0) ? theta_now : theta_now - e / d;
        IR++;
        if (error_ == h0 || error_ == h1 || error_ == h2 || error_ == h3) break;
        h3 = h2;
        h2 = h1;
        h1 = h0;
        h0 = error_;
        best_res = fmin(best_res, fabs(error_));
        if (fabs(error_) < fabs(err_stock)) {
            err_stock = error_ * b_0 / g_0;
            theta_stock = theta_end;
            if (fabs(err_stock) < 2e-16) break;
        }
    }
    *error_end = error_ * b_0 / g_0;
    *fallback = 0;
    if (!(best_res <= 1e-8 * (1.0 + fabs(c.time_end_)))) {  // the reference loop did not converge
        theta_stock = hyp_safe(c, theta_stock);
        *fallback = 1;
    }
    // end state (bia/find_hyperbola.f90:126-142)
#if BIA_REF_END_STATE
    double sn_end, cs_end;
    d_sincos(theta_stock, &sn_end, &cs_end);
    const double r_end = b * c.sn_0 / (cs_end - c.cs_0);
#else
    d_sincos(0.5 * theta_stock, &sh, &ch);
    const double sn_end = 2.0 * sh * ch, cs_end = 1.0 - 2.0 * sh * sh;
    double sp_e, sm_e;
    half_sines(c, theta_stock, sh, ch, sp_e, sm_e);
    const double r_end = b * c.sn_0 / (2.0 * sp_e * sm_e);
#endif
    const double u_end = g0_sn0 * c.cs_0 * sn_end;
    const double du_end = u_end - u;
    const double v_end = g0_sn0 * (1.0 - c.cs_0 * cs_end);
    const double dv_end = v_end - v;
    YN[0] = r_end * (cs_end * cs_a - sn_end * sn_a);
    YN[1] = r_end * (cs_end * sn_a + sn_end * cs_a);
    YN[2] = YZ[2] + (du_end * cs_a - dv_end * sn_a);
    YN[3] = YZ[3] + (du_end * sn_a + dv_end * cs_a);
    return IR;
}

// ---------------------------------------------------------------------------
// bia/find_ellipse.f90:1-157 (with its contained Newton).  Returns ir.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double f_sign(double a, double b) { return (b >= 0.0) ? fabs(a) : -fabs(a); }

// Bracketed Newton-bisection for Kepler's equation xi - e sin(xi) = M (root in
// [M - |e|, M + |e|]), used only when the reference's iteration ends unconverged.
static __device__ __noinline__ double kepler_safe(double M, double e, double x)
{
    const double ae = fabs(e);
    double lo = M - ae, hi = M + ae;
    if (!(x >= lo && x <= hi)) x = M;
    for (int it = 0; it < 400; it++) {
        double sx, cx;
        d_sincos(x, &sx, &cx);
        const double f = x - e * sx - M;
        if (f == 0.0) break;
        if (f < 0.0) lo = x; else hi = x;
        double xn = x - f / (1.0 - e * cx);
        if (!(xn > lo && xn < hi)) xn = 0.5 * (lo + hi);
        if (xn == x) break;
        x = xn;
    }
    return x;
}

#ifndef BIA_INLINE_ELLIPSE
#define BIA_INLINE_ELLIPSE 0
#endif
#if BIA_INLINE_ELLIPSE
#define BIA_ELLIPSE_LINKAGE __device__ __forceinline__
#else
#define BIA_ELLIPSE_LINKAGE static __device__ __noinline__
#endif
BIA_ELLIPSE_LINKAGE int ellipse(double eps_th, double dt, int ITR, const double YZ[4], double YN[4],
                                double *error, int *fallback)
{
    const double X_ini = YZ[0], Y_ini = YZ[1], U_ini = YZ[2], V_ini = YZ[3];
    const double g2_ini = U_ini * U_ini + V_ini * V_ini;
    const double r_ini = sqrt(X_ini * X_ini + Y_ini * Y_ini);
    const double W = g2_ini + 2.0 * eps_th / r_ini;
    const double L = X_ini * V_ini - Y_ini * U_ini;
    const double r_g_ini = X_ini * U_ini + Y_ini * V_ini;
    const double g_a = f_sign(sqrt(-W), L);
    const double a = eps_th / W;
    const double b = L / g_a;
    const double omega_a = g_a / a;
    double ecc = sqrt((a * g_a) * (a * g_a) - L * L) / (a * g_a);
    double xi_ini;
    if (r_g_ini == 0.0) {
        if (r_ini < a) {
            xi_ini = 0.0;
        } else if (r_ini == a) {
            xi_ini = d_atan2(Y_ini, X_ini);
            ecc = 0.0;
        } else {
            xi_ini = f_sign(kPi, L);
        }
    } else {
        xi_ini = d_atan2(r_g_ini / g_a, a - r_ini);
    }
    double s_ini, c_ini;
    d_sincos(xi_ini, &s_ini, &c_ini);
    const double alpha = d_atan2(Y_ini, X_ini) - d_atan2(b * s_ini, a * (c_ini - ecc));
    const double tau_ini = xi_ini - ecc * s_ini;
    const double time_ini = tau_ini / omega_a;
    const double time_end = time_ini + dt;
    const double tau_end = omega_a * time_end;
    *error = 0.0;
    if (dt == 0.0) {
#pragma unroll
        for (int k = 0; k < 4; k++) YN[k] = YZ[k];
        return 0;
    }
    // Kepler's equation tau_end = xi - e sin(xi) by the reference's Newton loop
    // (bia/find_ellipse.f90:106-157).  Start: one Newton step from the initial anomaly
    // xi_ini, whose residual is omega dt, instead of the reference's start from the mean
    // anomaly (xi_2 + delta_ini, bia/find_ellipse.f90:116-129), which needs ~8 steps on
    // average and fails outright for e near 1; the root is the same.
    int ir = 0;
    const double error_ini = tau_end - xi_ini + ecc * s_ini;
    double xi_2 = xi_ini;
    double error_tm2 = error_ini;
    double s2, c2, delta_xi2;
    double xi = xi_ini + error_ini / (1.0 - ecc * c_ini);
    double xi_1 = __longlong_as_double(0x7ff8000000000000LL);  // unset: compares unequal
    double error_tm1 = error_tm2;
    bool conv = false;
    while (xi_1 != xi_2 && ir <= ITR) {
        ir++;
        xi_1 = xi;
        double s1, c1;
        d_sincos(xi_1, &s1, &c1);
        error_tm1 = tau_end - xi_1 + ecc * s1;
        xi = xi_1 + error_tm1 / (1.0 - ecc * c1);
        if (error_tm1 == 0.0 || error_tm1 == error_tm2 || error_tm1 + error_tm2 == 0.0) {
            *error = error_tm1;
            conv = true;
            break;
        }
        ir++;
        xi_2 = xi;
        d_sincos(xi_2, &s2, &c2);
        error_tm2 = tau_end - xi_2 + ecc * s2;
        delta_xi2 = error_tm2 / (1.0 - ecc * c2);
        xi = xi_2 + delta_xi2;
        if (error_tm2 == 0.0 || error_tm1 == error_tm2 || error_tm1 + error_tm2 == 0.0) {
            *error = error_tm2;
            conv = true;
            break;
        }
    }
    if (xi_1 == xi_2) conv = true;
    *fallback = 0;
    if (!conv && !(fmin(fabs(error_tm1), fabs(error_tm2)) <= 1e-8 * (1.0 + fabs(tau_end)))) {
        xi = kepler_safe(tau_end, ecc, xi);
        *fallback = 1;
    }
    double sn_end, cs_end;
    d_sincos(xi, &sn_end, &cs_end);
    const double xx_end = a * (cs_end - ecc);
    const double yy_end = b * sn_end;
    const double rr_end = a * (1.0 - ecc * cs_end);
    const double uu_end = -a * g_a * sn_end / rr_end;
    const double vv_end = b * g_a * cs_end / rr_end;
    double sn_alp, cs_alp;
    d_sincos(alpha, &sn_alp, &cs_alp);
    YN[0] = xx_end * cs_alp - yy_end * sn_alp;
    YN[1] = xx_end * sn_alp + yy_end * cs_alp;
    YN[2] = uu_end * cs_alp - vv_end * sn_alp;
    YN[3] = uu_end * sn_alp + vv_end * cs_alp;
    return ir;
}

// ---------------------------------------------------------------------------
// bia/find_parabola.f90:1-143 (diagnostic prints dropped).  Returns iterations.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double par_time(double r_min, double g_max, double theta)
{
    double sn, cs;
    sincos(theta, &sn, &cs);
    return (2.0 + cs) * sn / ((1.0 + cs) * (1.0 + cs)) * 4.0 * r_min / (3.0 * g_max);
}

static __device__ __noinline__ int parabola(double eps_th, double DT, const double YZ[4], double YN[4],
                                     double *error_time)
{
    constexpr int NI = 99;
    double theta_Newton[NI + 1], error_Newton[NI + 1];
    const double r_ini = sqrt(YZ[0] * YZ[0] + YZ[1] * YZ[1]);
    const double r_dot_g = YZ[0] * YZ[2] + YZ[1] * YZ[3];
    const double r_crs_g = YZ[0] * YZ[3] - YZ[1] * YZ[2];
    const double g_max = -2.0 * eps_th / r_crs_g;
    const double r_min = r_crs_g / g_max;
    const double x_ini = 2.0 * r_min - r_ini;
    const double y_ini = f_sign(2.0 * r_min * sqrt(r_ini / r_min - 1.0), r_dot_g);
    const double theta_ini = atan2(y_ini, x_ini);
    const double time_ini = par_time(r_min, g_max, theta_ini);
    const double time_end = time_ini + DT;
    const double t_ = 3.0 * g_max / (4.0 * r_min) * time_end;
    const double sq = sqrt(1.0 + t_ * t_);
    const double theta_gss = 2.0 * atan(pow(sq + t_, 1.0 / 3) - pow(sq - t_, 1.0 / 3));
    double theta = theta_gss, err_tm_min = 1e99, thetamin = theta;
    int i_min = 1, i;
    for (i = 1; i <= NI; i++) {
        const double err_tm = par_time(r_min, g_max, theta) - time_end;
        error_Newton[i] = err_tm;
        const double ch = cos(theta * 0.5);
        const double ch2 = ch * ch;
        const double dtheta = -err_tm / (r_min / (g_max * (ch2 * ch2)));
        if (fabs(err_tm) < err_tm_min) {
            err_tm_min = fabs(err_tm);
            thetamin = theta;
            i_min = i;
        }
        theta = theta + dtheta;
        theta_Newton[i] = theta;
        if (dtheta == 0.0) break;
        if (theta - dtheta == theta) break;
        bool cyc = false;
        for (int j = 1; j <= i - 1; j++)
            if (error_Newton[i] == error_Newton[j]) { cyc = true; break; }
        if (cyc) { theta = theta_Newton[i_min]; break; }
    }
    if (i == NI + 1) theta = thetamin;
    const double theta_end = theta;
    double sn_b, cs_b;
    sincos(theta_end * 0.5, &sn_b, &cs_b);
    const double r_end = r_min / (cs_b * cs_b);
    const double g_end = g_max * cs_b;
    double st, ct;
    sincos(theta_end, &st, &ct);
    const double x_end = r_end * ct, y_end = r_end * st;
    const double u_end = -g_end * sn_b, v_end = g_end * cs_b;
    const double s1 = x_ini * YZ[1] - y_ini * YZ[0];
    const double c1 = x_ini * YZ[0] + y_ini * YZ[1];
    const double tmp = 1.0 / sqrt(s1 * s1 + c1 * c1);
    const double sn_g = s1 * tmp, cs_g = c1 * tmp;
    YN[0] = x_end * cs_g - y_end * sn_g;
    YN[1] = x_end * sn_g + y_end * cs_g;
    YN[2] = u_end * cs_g - v_end * sn_g;
    YN[3] = u_end * sn_g + v_end * cs_g;
    *error_time = time_end - par_time(r_min, g_max, theta_end);
    return (i > NI) ? NI : i;
}

// ---------------------------------------------------------------------------
// bia/find_dXYUV_RKF.f90:1-170: per-pair RKF4(5) with step doubling on the planar
// relative equation r'' = eps r/|r|^3 (moon_2D).  Returns ier; YN = step-doubled
// solution, *error = max of (yln - yhn)/31.
// ---------------------------------------------------------------------------
struct Fehlberg {
    static constexpr double AL2 = 1.0 / 4, AL3 = 3.0 / 8, AL4 = 12.0 / 13, AL5 = 1.0, AL6 = 1.0 / 2;
    static constexpr double B21 = 1.0 / 4;
    static constexpr double B31 = 3.0 / 32, B32 = 9.0 / 32;
    static constexpr double B41 = 1932.0 / 2197, B42 = -7200.0 / 2197, B43 = 7296.0 / 2197;
    static constexpr double B51 = 439.0 / 216, B52 = -8.0, B53 = 3680.0 / 513, B54 = -845.0 / 4104;
    static constexpr double B61 = -8.0 / 27, B62 = 2.0, B63 = -3544.0 / 2565, B64 = 1859.0 / 4104,
                            B65 = -11.0 / 40;
    static constexpr double GA1 = 16.0 / 135, GA3 = 6656.0 / 12825, GA4 = 28561.0 / 56430,
                            GA5 = -9.0 / 50, GA6 = 2.0 / 55;
    static constexpr double DA1 = 1.0 / 360, DA3 = -128.0 / 4275, DA4 = -2197.0 / 75240,
                            DA5 = 1.0 / 50, DA6 = 2.0 / 55;
};

__device__ __forceinline__ void moon2d(double eps_th, const double Y[4], double F[4])
{
    const double rsq = Y[0] * Y[0] + Y[1] * Y[1];
    const double aaa = eps_th / (rsq * sqrt(rsq));
    F[0] = Y[2];
    F[1] = Y[3];
    F[2] = Y[0] * aaa;
    F[3] = Y[1] * aaa;
}

// bia/find_dXYUV_RKF.f90:150-157 fehl on 4 equations; er written when want_er.
__device__ __forceinline__ void fehl4(double eps_th, double h, const double y0[4], double yn[4],
                                      double er[4], bool want_er)
{
    using F = Fehlberg;
    double k1[4], k2[4], k3[4], k4[4], k5[4], k6[4], w[4];
    moon2d(eps_th, y0, k1);
#pragma unroll
    for (int i = 0; i < 4; i++) w[i] = y0[i] + h * F::B21 * k1[i];
    moon2d(eps_th, w, k2);
#pragma unroll
    for (int i = 0; i < 4; i++) w[i] = y0[i] + h * (F::B31 * k1[i] + F::B32 * k2[i]);
    moon2d(eps_th, w, k3);
#pragma unroll
    for (int i = 0; i < 4; i++) w[i] = y0[i] + h * (F::B41 * k1[i] + F::B42 * k2[i] + F::B43 * k3[i]);
    moon2d(eps_th, w, k4);
#pragma unroll
    for (int i = 0; i < 4; i++)
        w[i] = y0[i] + h * (F::B51 * k1[i] + F::B52 * k2[i] + F::B53 * k3[i] + F::B54 * k4[i]);
    moon2d(eps_th, w, k5);
#pragma unroll
    for (int i = 0; i < 4; i++)
        w[i] = y0[i] + h * (F::B61 * k1[i] + F::B62 * k2[i] + F::B63 * k3[i] + F::B64 * k4[i] +
                            F::B65 * k5[i]);
    moon2d(eps_th, w, k6);
#pragma unroll
    for (int i = 0; i < 4; i++)
        yn[i] = y0[i] + h * (F::GA1 * k1[i] + F::GA3 * k3[i] + F::GA4 * k4[i] + F::GA5 * k5[i] +
                             F::GA6 * k6[i]);
    if (want_er) {
#pragma unroll
        for (int i = 0; i < 4; i++)
            er[i] = h * (F::DA1 * k1[i] + F::DA3 * k3[i] + F::DA4 * k4[i] + F::DA5 * k5[i] +
                         F::DA6 * k6[i]);
    }
}

static __device__ __noinline__ int rkf_pair(double eps_th, double xe, double relerr, double abserr,
                                     const double YZ[4], double YN[4], double *error, int *nacc)
{
    const int itemax = 100000;
    const double epsmin = 1e-15;
    double yh0[4], yl0[4], yln[4], yhn[4], er[4], ymid[4];
#pragma unroll
    for (int i = 0; i < 4; i++) { yh0[i] = YZ[i]; yl0[i] = YZ[i]; yhn[i] = YZ[i]; }
    double f0[4];
    moon2d(eps_th, yl0, f0);
    double toldy = 1.7976931348623157e308;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        if (f0[i] != 0.0) {
            const double tol = relerr * fabs(yl0[i]) + abserr;
            toldy = fmin(toldy, fabs(tol / f0[i]));
        }
    }
    double h = (toldy == 1.7976931348623157e308) ? epsmin * xe : fmin(xe / 100.0, pow(toldy, 0.2));
    double x = 0.0;
    int ier = 10000, n = 0;
    *error = 0.0;
    for (int iter = 1; iter <= itemax; iter++) {
        fehl4(eps_th, h, yl0, yln, er, true);
        double erret = 0.0;
        bool bad = false;
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const double et = relerr / 2.0 * (fabs(yl0[i]) + fabs(yln[i])) + abserr;
            if (et == 0.0) bad = true;
            erret = fmax(erret, fabs(er[i]) / et);
        }
        if (bad) { ier = 20000; break; }
        if (erret > 1.0) {
            h = (erret >= 59049.0) ? 0.1 * h : 0.9 * h / pow(erret, 0.2);
            if (h <= epsmin) { ier = 30000; break; }
        } else if (x + h < xe) {
            fehl4(eps_th, h * 0.5, yh0, ymid, er, false);
            fehl4(eps_th, h * 0.5, ymid, yhn, er, false);
            x = x + h;
#pragma unroll
            for (int i = 0; i < 4; i++) { yl0[i] = yln[i]; yh0[i] = yhn[i]; }
            n++;
            h = (erret <= 1.889568e-4) ? 5.0 * h : 0.9 * h / pow(erret, 0.2);
        } else {
            h = xe - x;
            fehl4(eps_th, h, yl0, yln, er, true);
            fehl4(eps_th, h * 0.5, yh0, ymid, er, false);
            fehl4(eps_th, h * 0.5, ymid, yhn, er, false);
            double m = (yln[0] - yhn[0]) / 31.0;
#pragma unroll
            for (int i = 1; i < 4; i++) m = fmax(m, (yln[i] - yhn[i]) / 31.0);
            *error = m;
            n++;
            ier = 0;
            break;
        }
    }
#pragma unroll
    for (int i = 0; i < 4; i++) YN[i] = yhn[i];
    *nacc = n;
    return ier;
}

// ---------------------------------------------------------------------------
// Universal-variable propagation of r'' = eps r/|r|^3 (mu = -eps) with Stumpff
// functions (Danby, Fundamentals of Celestial Mechanics, 2nd ed., 6.7-6.9).  Uniformly
// well conditioned for every conic and for radial or zero-velocity pairs; the
// displacement from free motion is formed without cancellation:
//   r(t) - r0 - v0 dt = -(mu/r0) s^2 c2 r0vec - mu s^3 c3 v0vec
//   v(t) - v0         = -(mu/(r r0)) s c1 r0vec - (mu/r) s^2 c2 v0vec
// with s the root of r0 s c1 + sigma0 s^2 c2 + mu s^3 c3 = dt (bracketed Newton).
// No transcendental function is called: the Stumpff functions come from a series at
// |x| <= 0.1 and the duplication formulas c0(4x) = 2c0^2 - 1, c1(4x) = c0 c1,
// c2(4x) = c1^2/2, c3(4x) = (c2 + c0 c3)/4.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void stumpff(double x, double c[4])
{
    if (fabs(x) <= 1e-6) {
        // three terms: the next ones, x^3/8! and x^3/9!, are below 3e-23
        const double c2 = 0.5 - x * (1.0 / 24 - x * (1.0 / 720));
        const double c3 = 1.0 / 6 - x * (1.0 / 120 - x * (1.0 / 5040));
        c[0] = 1.0 - x * c2;
        c[1] = 1.0 - x * c3;
        c[2] = c2;
        c[3] = c3;
        return;
    }
    if (fabs(x) <= 1e-2) {
        // the first five terms: the next ones, x^5/12! and x^5/13!, are below 2e-19
        const double c2 = 0.5 - x * (1.0 / 24 - x * (1.0 / 720 - x * (1.0 / 40320 - x * (1.0 / 3628800))));
        const double c3 = 1.0 / 6 - x * (1.0 / 120 - x * (1.0 / 5040 - x * (1.0 / 362880 - x * (1.0 / 39916800))));
        c[0] = 1.0 - x * c2;
        c[1] = 1.0 - x * c3;
        c[2] = c2;
        c[3] = c3;
        return;
    }
    int n = 0;
    while (fabs(x) > 0.1 && n < 200) { x *= 0.25; n++; }
    // c2 = sum (-x)^j / (2+2j)!, c3 = sum (-x)^j / (3+2j)!, j = 0..10 (|x| <= 0.1)
    double c2 = 1.0 / 620448401733239439360000.0;    // 1/24!
    double c3 = 1.0 / 15511210043330985984000000.0;  // 1/25!
    c2 = 1.0 / 20922789888000.0 - x * (1.0 / 6402373705728000.0 - x * (1.0 / 2432902008176640000.0 - x * (1.0 / 1124000727777607680000.0 - x * c2)));
    c3 = 1.0 / 355687428096000.0 - x * (1.0 / 121645100408832000.0 - x * (1.0 / 51090942171709440000.0 - x * (1.0 / 25852016738884976640000.0 - x * c3)));
    c2 = 0.5 - x * (1.0 / 24 - x * (1.0 / 720 - x * (1.0 / 40320 - x * (1.0 / 3628800 - x * (1.0 / 479001600 - x * (1.0 / 87178291200.0 - x * c2))))));
    c3 = 1.0 / 6 - x * (1.0 / 120 - x * (1.0 / 5040 - x * (1.0 / 362880 - x * (1.0 / 39916800 - x * (1.0 / 6227020800.0 - x * (1.0 / 1307674368000.0 - x * c3))))));
    double c1 = 1.0 - x * c3;
    double c0 = 1.0 - x * c2;
    for (; n > 0; n--) {
        const double c3n = (c2 + c0 * c3) * 0.25;
        const double c2n = c1 * c1 * 0.5;
        const double c1n = c0 * c1;
        const double c0n = 2.0 * c0 * c0 - 1.0;
        c0 = c0n; c1 = c1n; c2 = c2n; c3 = c3n;
    }
    c[0] = c0; c[1] = c1; c[2] = c2; c[3] = c3;
}

// iteration cap of the universal-variable solver; a pair that reaches it is counted as
// not converged
constexpr int kUvItMax = 200;

// The universal-variable pair in pieces (prepare, start, iterate, compose) so that other
// solvers can supply their own start; uv_halfdisp chains them.
struct UvPair {
    double mu, r0, sig, beta;
    double ir0;  // 1 / r0, so that start and composition need one division fewer each
};

__device__ __forceinline__ UvPair uv_prepare(double eps_th, const double r[3], const double g[3])
{
    UvPair p;
    p.mu = -eps_th;
    // one reciprocal square root for both r0 and 1/r0 (rsqrt: within 1 ulp)
    const double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
    p.ir0 = rsqrt(r2);
    p.r0 = (r2 > 0.0) ? r2 * p.ir0 : 0.0;
    p.sig = r[0] * g[0] + r[1] * g[1] + r[2] * g[2];
    const double v2 = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
    p.beta = 2.0 * p.mu * p.ir0 - v2;
    return p;
}

// Third-order start: the reversion of t = r0 s + (sig/2) s^2 + ((mu - beta r0)/6) s^3 + O(s^4),
//   s = x - (sig / (2 r0)) x^2 + (sig^2/2 - r0 (mu - beta r0)/6) x^3 / r0^2,  x = dt / r0,
// leaves a relative error O((dt/T)^3), so at small steps the first Newton correction is
// already below the 1e-10 acceptance of uv_iterate (the second-order start needed two).
__device__ __forceinline__ double uv_start(const UvPair &p, double dt)
{
    const double x = dt * p.ir0;
    const double a2 = -0.5 * p.sig * p.ir0;
    const double a3 = (0.5 * p.sig * p.sig - p.r0 * (p.mu - p.beta * p.r0) * (1.0 / 6.0)) * (p.ir0 * p.ir0);
    const double s = x + x * x * (a2 + x * a3);
    return (s > 0.0) ? s : x;
}

// Fifth-order start of the universal-variable method and the split learned step's plain
// pairs, in dimensionless form.  The universal Kepler equation
//   t = b1 s + b2 s^2 + b3 s^3 + b4 s^4 + b5 s^5 + O(s^6),
//   b1 = r0, b2 = sig/2, b3 = (mu - beta r0)/6, b4 = -sig beta/24, b5 = beta (beta r0 - mu)/120
// (the Stumpff series of r0 s c1 + sig s^2 c2 + mu s^3 c3) is inverted with the Lagrange
// reversion coefficients (Abramowitz and Stegun 3.6.25):
//   a1 = 1/b1, a2 = -b2/b1^3, a3 = (2 b2^2 - b1 b3)/b1^5, a4 = (5 b1 b2 b3 - b1^2 b4 - 5 b2^3)/b1^7,
//   a5 = (6 b1^2 b2 b4 + 3 b1^2 b3^2 + 14 b2^4 - b1^3 b5 - 21 b1 b2^2 b3)/b1^9,
//   s = a1 t + a2 t^2 + a3 t^3 + a4 t^4 + a5 t^5 + O(t^6).
// With x = dt/r0, y = sig dt/(2 r0^2), m = mu/r0, z = (m - beta) x^2/6 and w = beta x^2 the
// relative terms c_k = a_(k+1) dt^k / a1 are
//   c1 = -y, c2 = 2y^2 - z, c3 = y (5z + w/12 - 5y^2),
//   c4 = y^2 (14y^2 - 21z - w/2) + z (3z + w/20),
// and s = x S with S = 1 + c1 + c2 + c3 + c4 (about 25 FP64 operations instead of 65 for the
// same sum from the a_k).  When every |c_k| <= Q^k with Q = 3e-4 (the step is that small
// against the pair's time scales) the sum is exact: its truncation is below 1.1e-17
// relative, a tenth of an FP64 ulp (checked in extended precision against the solved equation
// on 12000 attractive and repulsive pairs drawn around that boundary), so no Newton
// correction runs and uv_compose_series composes the half-displacement from S.  Otherwise
// uv_series_start gives the third-order sum x (1 + c1 + c2) (error O((dt/T)^3), one Newton
// correction below the 1e-10 acceptance at small steps).  The ALG kernels keep uv_start:
// changing the code they inline changes how the compiler contracts their own FP64
// expressions.  Every product and sum is written out (fma, __dmul_rn) so that each kernel
// that inlines this computes the same bits and takes the same branch: the ensemble's systems
// equal their own steps bit for bit.
struct UvSeries {
    double x, y, x2, w, c2;
    double mh;  // -m/2
    double S;   // s = x S where exact
    bool exact;
};

__device__ __forceinline__ UvSeries uv_series(const UvPair &p, double dt)
{
    UvSeries q;
    q.x = __dmul_rn(dt, p.ir0);
    const double m = __dmul_rn(p.mu, p.ir0);
    q.mh = -0.5 * m;
    q.y = __dmul_rn(__dmul_rn(0.5 * p.sig, p.ir0), q.x);
    q.x2 = __dmul_rn(q.x, q.x);
    q.w = __dmul_rn(p.beta, q.x2);
    const double y = q.y, w = q.w;
    const double z = __dmul_rn(__dsub_rn(m, p.beta), __dmul_rn(q.x2, 1.0 / 6.0));
    const double y2 = __dmul_rn(y, y);
    q.c2 = fma(2.0 * y, y, -z);
    const double c3 = __dmul_rn(y, fma(-5.0, y2, fma(w, 1.0 / 12.0, 5.0 * z)));
    const double c4 = fma(z, fma(3.0, z, __dmul_rn(w, 0.05)), __dmul_rn(y2, fma(14.0, y2, fma(-21.0, z, -0.5 * w))));
    constexpr double Q = 3e-4;
    const bool small = fabs(y) <= Q && fabs(q.c2) <= Q * Q && fabs(c3) <= Q * Q * Q && fabs(c4) <= Q * Q * Q * Q;
    q.S = 1.0 + (q.c2 - y + (c3 + c4));
    q.exact = small && q.S > 0.0 && dt > 0.0;  // s = x S > 0
    return q;
}

// The third-order start for a pair whose series is not exact (uv_iterate corrects it).
__device__ __forceinline__ double uv_series_start(const UvSeries &q)
{
    const double s3 = __dmul_rn(q.x, 1.0 + (q.c2 - q.y));
    return (s3 > 0.0) ? s3 : q.x;
}

// Half-displacement of an exact series pair: the coefficients of uv_compose in the series'
// variables.  With K = -m x^2/2 (= -mu dt^2/(2 r0^3)), A = S^2 c2(w S^2), B = S^3 c3(w S^2)
// and rho = r0/r(s):
//   (f - 1)/2 = K A,  (g - dt)/2 = K dt B,  (g' - 1)/2 = K A rho,  f'/2 = -(m/2)(x/r0) S c1 rho,
// and r(s)/r0 = 1 + d with d = -w S^2 c2 + 2 y S c1 - 2 K A (r(s) = r0 c0 + sig s c1 +
// mu s^2 c2 and c0 = 1 - beta s^2 c2), formed without cancellation.  rho is the alternating
// series of 1/(1 + d) to d^5 where |d| <= 1e-3 (truncation below 1e-18), else a division.
// f'/2 is formed as (K/dt) S c1 rho (K/dt = -(m/2) x/r0; 1/dt is the same for every pair).
// The factor 1/2 of the half-displacement is inside K (a power of two: the same bits).
__device__ __forceinline__ void uv_compose_series(const UvPair &p, const UvSeries &q, double dt, const double r[3],
                                                  const double g[3], double h[6])
{
    const double S = q.S;
    const double S2 = __dmul_rn(S, S);
    const double arg = __dmul_rn(q.w, S2);
    double c[4];
    stumpff(arg, c);
    const double A = __dmul_rn(S2, c[2]);
    const double B = __dmul_rn(__dmul_rn(S2, S), c[3]);
    const double K = __dmul_rn(q.mh, q.x2);
    const double fm1 = __dmul_rn(K, A);
    const double gmdt = __dmul_rn(__dmul_rn(K, dt), B);
    const double d = fma(-arg, c[2], fma(__dmul_rn(2.0 * q.y, S), c[1], -2.0 * fm1));
    double rho;
    if (fabs(d) <= 1e-3) {
        const double nd = -d;
        rho = fma(nd, fma(nd, fma(nd, fma(nd, fma(nd, 1.0, 1.0), 1.0), 1.0), 1.0), 1.0);
    } else {
        rho = 1.0 / (1.0 + d);
    }
    const double gdm1 = __dmul_rn(fm1, rho);
    const double fdot = __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(K, 1.0 / dt), S), c[1]), rho);
#pragma unroll
    for (int k = 0; k < 3; k++) {
        h[k] = fma(fm1, r[k], __dmul_rn(gmdt, g[k]));
        h[3 + k] = fma(fdot, r[k], __dmul_rn(gdm1, g[k]));
    }
}

// Safeguarded Newton on F(s) = t(s) - dt, F' = r(s) > 0, with the bracket [lo, hi]
// (F(0) = -dt < 0; hi < 0 until an upper bound is seen).  A Newton step that leaves the
// bracket, or is not below half the step before last, is replaced by bisection, so the
// bracket at least halves every two iterations: on hyperbolic branches Newton from far
// above the root moves only ~1/sqrt(-beta) per step.  Returns the iterations
// (kUvItMax + 1 when the cap was reached).
// ifp (optional): 1 / F' at the last evaluation, for uv_compose (F' = r(s)).
__device__ __forceinline__ int uv_iterate(const UvPair &p, double dt, double &s_io, double *ifp = nullptr)
{
    double c[4];
    double s = s_io;
    double lo = 0.0, hi = -1.0, dx = 1e300, dxold = 1e300;
    double ifp_last = 0.0;
    int it;
    for (it = 1; it <= kUvItMax; it++) {
        stumpff(p.beta * s * s, c);
        const double F = p.r0 * s * c[1] + p.sig * s * s * c[2] + p.mu * s * s * s * c[3] - dt;
        const double Fp = p.r0 * c[0] + p.sig * s * c[1] + p.mu * s * s * c[2];
        if (F == 0.0) break;
        ifp_last = 1.0 / Fp;
        const double step = F * ifp_last;
        if (Fp > 0.0 && fabs(step) <= 4.0 * 2.220446049250313e-16 * fabs(s)) {
            s = s - step;  // converged: the remaining correction is a few ulps
            break;
        }
        if (F < 0.0) lo = s; else hi = s;  // a NaN F (overflow far above the root) lowers hi
        double sn = s - step;
        const bool newton = (Fp > 0.0) && (sn > lo) && (hi < 0.0 || sn < hi) &&
                            (hi < 0.0 || fabs(step) <= 0.5 * dxold);
        if (!newton) sn = (hi > 0.0) ? 0.5 * (lo + hi) : 2.0 * s;
        dxold = dx;
        dx = fabs(sn - s);
        s = sn;
        if (dx <= 4.0 * 2.220446049250313e-16 * fabs(s)) break;  // bracket collapsed
        // Newton converges quadratically: after a step of relative size 1e-10 the next
        // one would be below rounding, so s is final without another evaluation
        if (newton && dx <= 1e-10 * fabs(s)) break;
    }
    s_io = s;
    if (ifp) *ifp = ifp_last;
    return it;
}

// One Halley step on the same equation from s: returns the step ds (s_new = s - ds).
// F'' = dr/ds = sig c0 + (mu - beta r0) s c1.
__device__ __forceinline__ double uv_halley_step(const UvPair &p, double dt, double s)
{
    double c[4];
    stumpff(p.beta * s * s, c);
    const double F = p.r0 * s * c[1] + p.sig * s * s * c[2] + p.mu * s * s * s * c[3] - dt;
    const double Fp = p.r0 * c[0] + p.sig * s * c[1] + p.mu * s * s * c[2];
    const double Fpp = p.sig * c[0] + (p.mu - p.beta * p.r0) * s * c[1];
    return F * Fp / (Fp * Fp - 0.5 * F * Fpp);
}

// Half-displacement from the solved s: f - 1, g - dt, f', g' - 1 from the Stumpff
// functions (no cancellation at small s).  irr_hint (optional, 0: none): an approximation
// of 1/r(s), such as uv_iterate's last 1/F'; within 1e-8 of it one Newton-Raphson step for
// the reciprocal (x + x (1 - r x)) gives 1/r(s) to ~1e-16, else 1/r(s) is divided out.
// kTwoSteps (the universal-variable method and the split step's plain pairs after Newton
// iterations, the learned finish): two Newton-Raphson steps from a hint within 1e-4
// (error e^4 <= 1e-16); the ALG kernels keep the one-step form.
template <bool kTwoSteps = false>
__device__ __forceinline__ void uv_compose(const UvPair &p, double s, const double r[3], const double g[3],
                                           double h[6], double irr_hint = 0.0)
{
    double c[4];
    stumpff(p.beta * s * s, c);
    const double s2c2 = s * s * c[2], s3c3 = s * s * s * c[3];
    const double rr = p.r0 * c[0] + p.sig * s * c[1] + p.mu * s2c2;
    const double e = fma(-rr, irr_hint, 1.0);
    double irr;
    if (kTwoSteps) {
        if (irr_hint != 0.0 && fabs(e) <= 1e-4) {
            const double x1 = fma(irr_hint, e, irr_hint);
            irr = fma(x1, fma(-rr, x1, 1.0), x1);
        } else {
            irr = 1.0 / rr;
        }
    } else {
        irr = (irr_hint != 0.0 && fabs(e) <= 1e-8) ? fma(irr_hint, e, irr_hint) : 1.0 / rr;
    }
    // the half-displacement's factor 1/2 is taken into the coefficients: scaling by a power of
    // two is exact, so h is the same as (f - 1) r + (g - dt) v halved afterwards, at four
    // multiplications instead of six
    const double fm1 = -0.5 * p.mu * s2c2 * p.ir0;
    const double gmdt = -0.5 * p.mu * s3c3;
    const double fdot = -0.5 * p.mu * s * c[1] * (irr * p.ir0);
    const double gdm1 = -0.5 * p.mu * s2c2 * irr;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        h[k] = fm1 * r[k] + gmdt * g[k];
        h[3 + k] = fdot * r[k] + gdm1 * g[k];
    }
}

__device__ __forceinline__ int uv_halfdisp(double eps_th, double dt, const double r[3], const double g[3],
                                           double h[6])
{
#pragma unroll
    for (int k = 0; k < 6; k++) h[k] = 0.0;
    if (dt == 0.0) return 0;
    const UvPair p = uv_prepare(eps_th, r, g);
    double s = uv_start(p, dt);
    double ifp;
    const int it = uv_iterate(p, dt, s, &ifp);
    uv_compose(p, s, r, g, h, ifp);
    return it;
}

// uv_halfdisp from the fifth-order start: no Newton correction where the series alone is
// exact (returns 0 iterations for those pairs).  The ALG kernels keep uv_halfdisp.
__device__ __forceinline__ int uv_halfdisp_fast(double eps_th, double dt, const double r[3], const double g[3],
                                                double h[6])
{
#pragma unroll
    for (int k = 0; k < 6; k++) h[k] = 0.0;
    if (dt == 0.0) return 0;
    const UvPair p = uv_prepare(eps_th, r, g);
    const UvSeries q = uv_series(p, dt);
    if (q.exact) {
        uv_compose_series(p, q, dt, r, g, h);
        return 0;
    }
    double s = uv_series_start(q);
    double ifp = 0.0;
    const int it = uv_iterate(p, dt, s, &ifp);
    uv_compose<true>(p, s, r, g, h, ifp);
    return it;
}

// ---------------------------------------------------------------------------
// One pair: frame, classification, solve, half-displacement (bia/bia.f90:141-191).
// Returns the half-displacement in h[6] = (dX, dY, dZ, dU, dV, dW)/2 terms.
// ---------------------------------------------------------------------------
// ALG pair classes (bia/bia.f90:156-166 plus the guards): the branch each pair takes.
enum AlgClass { kClsHyp = 0, kClsEll = 1, kClsUv = 2, kClsPar = 3, kClsDeg = 4 };

// Branch of an ALG pair: E == 0 exactly keeps the reference's parabola branch; zero |g| or
// |L| (degenerate) and |e^2 - 1| = |E| L^2 / eps^2 < 0.1 go to the universal-variable
// solver; otherwise hyperbola (E > 0) or ellipse (E < 0).
__device__ __forceinline__ int alg_classify(double eps_ij, const double r[3], const double g[3], double &E_out,
                                            double &Lsq_out)
{
    const double gsq = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
    const double L0 = r[1] * g[2] - r[2] * g[1];
    const double L1 = r[2] * g[0] - r[0] * g[2];
    const double L2 = r[0] * g[1] - r[1] * g[0];
    const double Lsq = L0 * L0 + L1 * L1 + L2 * L2;
    const double r_ij = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    const double E_ij = gsq + 2.0 * eps_ij / r_ij;
    E_out = E_ij;
    Lsq_out = Lsq;
    if (E_ij == 0.0) return kClsPar;
    if (gsq == 0.0 || Lsq == 0.0) return kClsDeg;
    if (fabs(E_ij) * Lsq < kNearUnitEcc * (eps_ij * eps_ij)) return kClsUv;
    return (E_ij > 0.0) ? kClsHyp : kClsEll;
}

__device__ __forceinline__ int alg_classify(double eps_ij, const double r[3], const double g[3])
{
    double E, Lsq;
    return alg_classify(eps_ij, r, g, E, Lsq);
}

// |g| == 0 or |L| == 0: the pair's frame is degenerate (counted apart from the other
// universal-variable pairs)
__device__ __forceinline__ bool pair_degenerate(const double r[3], const double g[3])
{
    const double gsq = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
    const double L0 = r[1] * g[2] - r[2] * g[1];
    const double L1 = r[2] * g[0] - r[0] * g[2];
    const double L2 = r[0] * g[1] - r[1] * g[0];
    return gsq == 0.0 || (L0 * L0 + L1 * L1 + L2 * L2) == 0.0;
}

// M: the compiled method (kMethodRkf, kMethodAlg, kMethodUniversal); each kernel is
// instantiated per method so it carries only that method's code and registers.
constexpr int kMethodRkf = 0, kMethodAlg = 1, kMethodUniversal = 2, kMethodLearned = 3;

__device__ __forceinline__ void count_nonfinite(const double h[6], PairCounters &cnt)
{
    bool finite = true;
#pragma unroll
    for (int k = 0; k < 6; k++) finite = finite && isfinite(h[k]);
    if (!finite) cnt.nonfinite++;
}

// Half-displacement from the in-plane solution: h = ((dr . e - g dt) / 2, (dg . e) / 2)
// (bia/bia.f90:170-191).
__device__ __forceinline__ void compose_halfdisp(const PairParams &P, const double g[3], const double e_xi[3],
                                                 const double e_eta[3], const double YZ[4],
                                                 const double YN[4], double h[6])
{
    const double dr_xi = YN[0] - YZ[0], dr_eta = YN[1] - YZ[1];
    const double dg_xi = YN[2] - YZ[2], dg_eta = YN[3] - YZ[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        h[k] = (dr_xi * e_xi[k] + dr_eta * e_eta[k] - g[k] * P.dt) * 0.5;
        h[3 + k] = (dg_xi * e_xi[k] + dg_eta * e_eta[k]) * 0.5;
    }
}

// ALG pair whose class C is known (kClsHyp, kClsEll or kClsPar): frame, conic solver,
// half-displacement (bia/bia.f90:141-191).
template <int C>
__device__ __forceinline__ void alg_conic_pair(const PairParams &P, double eps_ij, const double r[3],
                                               const double g[3], double h[6], PairCounters &cnt)
{
    double e_xi[3], e_eta[3], YZ[4], YN[4];
    double error = 0.0;
    frame_xi_eta(r, g, e_xi, e_eta, YZ);
    if (C == kClsHyp) {
        int bx = 0, fb = 0;
        cnt.it_hyp += hyperbola(eps_ij, P.dt, P.itr, YZ, YN, &error, &bx, &fb);
        cnt.bracket_exits += bx;
        cnt.fallbacks += fb;
        cnt.cls[kHyperbola]++;
    } else if (C == kClsEll) {
        int fb = 0;
        cnt.it_ell += ellipse(eps_ij, P.dt, P.itr, YZ, YN, &error, &fb);
        cnt.fallbacks += fb;
        cnt.cls[kEllipse]++;
    } else {
        cnt.it_par += parabola(eps_ij, P.dt, YZ, YN, &error);
        cnt.cls[kParabola]++;
    }
    if (fabs(error) > P.err) cnt.nonconverged++;
    compose_halfdisp(P, g, e_xi, e_eta, YZ, YN, h);
    count_nonfinite(h, cnt);
}

// ALG pair of the rare classes (parabola, degenerate, near-unit eccentricity): c is
// alg_classify's answer for it.
__device__ __forceinline__ void alg_rare_pair(const PairParams &P, double eps_ij, const double r[3],
                                              const double g[3], double h[6], PairCounters &cnt, int c)
{
    if (c == kClsPar) {
        alg_conic_pair<kClsPar>(P, eps_ij, r, g, h, cnt);
    } else {
        const int it = uv_halfdisp(eps_ij, P.dt, r, g, h);
        cnt.it_uv += it;
        if (it > kUvItMax) cnt.nonconverged++;
        cnt.cls[c == kClsDeg ? kDegenerate : kUniversal]++;
        count_nonfinite(h, cnt);
    }
}

// kCountNonfinite false (universal variables and RKF45 only): the caller counts the
// non-finite half-displacements itself (once per warp-block from its sums, see
// warp_block_solve_uv).
template <int M, bool kCountNonfinite = true>
__device__ __forceinline__ void pair_halfdisp(const PairParams &P, double eps_ij, const double r[3],
                                              const double g[3], double h[6], PairCounters &cnt)
{
    if (M == kMethodUniversal) {
        const int it = uv_halfdisp_fast(eps_ij, P.dt, r, g, h);
        cnt.it_uv += it;
        if (it > kUvItMax) cnt.nonconverged++;
        cnt.cls[kUniversal]++;
        if (kCountNonfinite) count_nonfinite(h, cnt);
    } else if (M == kMethodAlg) {
        const int c = alg_classify(eps_ij, r, g);
        if (c == kClsUv || c == kClsDeg) {
            alg_rare_pair(P, eps_ij, r, g, h, cnt, c);
        } else {
            // one copy of the frame and composition for the three conic branches
            double e_xi[3], e_eta[3], YZ[4], YN[4];
            double error = 0.0;
            frame_xi_eta(r, g, e_xi, e_eta, YZ);
            if (c == kClsHyp) {
                int bx = 0, fb = 0;
                cnt.it_hyp += hyperbola(eps_ij, P.dt, P.itr, YZ, YN, &error, &bx, &fb);
                cnt.bracket_exits += bx;
                cnt.fallbacks += fb;
                cnt.cls[kHyperbola]++;
            } else if (c == kClsEll) {
                int fb = 0;
                cnt.it_ell += ellipse(eps_ij, P.dt, P.itr, YZ, YN, &error, &fb);
                cnt.fallbacks += fb;
                cnt.cls[kEllipse]++;
            } else {
                cnt.it_par += parabola(eps_ij, P.dt, YZ, YN, &error);
                cnt.cls[kParabola]++;
            }
            if (fabs(error) > P.err) cnt.nonconverged++;
            compose_halfdisp(P, g, e_xi, e_eta, YZ, YN, h);
            count_nonfinite(h, cnt);
        }
    } else {
        double e_xi[3], e_eta[3], YZ[4], YN[4];
        double error = 0.0;
        const bool degenerate = frame_xi_eta(r, g, e_xi, e_eta, YZ);
        int nacc = 0;
        rkf_pair(eps_ij, P.dt, P.relerr, P.abserr, YZ, YN, &error, &nacc);
        cnt.cls[degenerate ? kDegenerate : kRkf]++;
        cnt.rkf_steps += nacc;
        if (fabs(error) > P.err) cnt.nonconverged++;
        compose_halfdisp(P, g, e_xi, e_eta, YZ, YN, h);
        if (kCountNonfinite) count_nonfinite(h, cnt);
    }
}

// A warp-block's sums are finite exactly when every half-displacement added into them is (a
// NaN stays NaN and an infinity stays infinite or turns NaN), so the walks test the lane's
// row and column sums once per block instead of each pair.
__device__ __forceinline__ bool sums_finite(const double racc[6], const double cacc[6])
{
    bool ok = true;
#pragma unroll
    for (int c = 0; c < 6; c++) ok = ok && isfinite(racc[c]) && isfinite(cacc[c]);
    return ok;
}

}  // namespace bia
