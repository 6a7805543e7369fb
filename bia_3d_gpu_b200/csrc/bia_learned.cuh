// bia_learned.cuh -- the learned mixed-precision form of one pair (BIA_METHOD_LEARNED).
//
// An attractive conic pair is written in orbital elements, its mean anomaly after dt goes
// through a learned head (mlp_tc.cuh) for a starting guess of the anomaly, one Newton
// correction runs in FP32, one Halley step in FP64 finishes it, and the half-displacement
// is composed in FP64 from the Stumpff functions (no cancellation).  Everything else, and
// any pair whose FP64 step does not settle, takes the plain universal-variable solver.
//
// Elements from the pair (mu = -eps_ij > 0, beta = 2 mu / r0 - |g|^2, sig = r . g):
//   ellipse (beta > 0):    e cos E0 = C0 = 1 - r0 beta / mu,  e sin E0 = S0 = sig sqrt(beta) / mu,
//                          n = beta^{3/2} / mu,  M = E - e sin E;
//   hyperbola (beta < 0):  e cosh H0 = C0 = 1 - r0 beta / mu, e sinh H0 = S0 = sig sqrt(-beta) / mu,
//                          n = (-beta)^{3/2} / mu, M = e sinh H - H.
// The anomaly increment D = A1 - A0 solves the difference form of Kepler's equation,
//   ellipse:   (1 - C0) D + C0 (D - sin D) + S0 (1 - cos D) - n dt = 0,
//   hyperbola: (C0 - 1) sinh D + S0 (cosh D - 1) + (sinh D - D) - n dt = 0,
// and D = sqrt(|beta|) s where s is the universal variable of uv_halfdisp, so the FP64
// step and the composition are the universal-variable ones.
#pragma once
#include "bia_pair.cuh"

namespace bia {

constexpr int kLearnedPlain = 0, kLearnedEll = 1, kLearnedHyp = 2;
constexpr int kHeadEll = 0, kHeadHyp = 1;

// Head domains and input scaling (the same numbers as bia_3d_gpu_b200/train_heads.py).
constexpr float kEllEMax = 0.99f;
constexpr float kHypEMin = 1.001f, kHypEMax = 50.0f, kHypMMax = 100.0f;
constexpr float kHypOut = 6.0f;
constexpr float kTwoPiF = 6.283185307179586f;
constexpr float kPiF = 3.141592653589793f;

// The pair in elements, FP64 parts and the FP32 inputs of its head.
struct LearnedPair {
    UvPair p;
    double sqb, isqb;      // sqrt(|beta|) and its reciprocal
    float C0m, S0, C0;     // C0m = |1 - C0| = r0 |beta| / mu (no cancellation)
    float dM, A0;          // n dt, initial anomaly
    float x0, x1;          // head inputs
    float unfold_sign, unfold_shift;  // A = sign * A_head + shift
    int kind;              // kLearnedPlain / kLearnedEll / kLearnedHyp
};

// Cheap first test: can the pair be in a head's domain?  ellipses (all of them: the
// universal-variable guard leaves e^2 <= 0.9), and attractive hyperbolae with
// e^2 - 1 = E L^2 / eps^2 <= 50^2 - 1.  learned_prepare makes the final decision.
__device__ __forceinline__ bool learned_candidate(double eps_ij, double dt, const double r[3], const double g[3])
{
    double E, Lsq;
    const int c = alg_classify(eps_ij, r, g, E, Lsq);
    if (!(dt > 0.0) || !(eps_ij < 0.0)) return false;
    if (c == kClsEll) return true;
    return c == kClsHyp && E * Lsq <= (double)(kHypEMax * kHypEMax - 1.0f) * (eps_ij * eps_ij);
}

// The heads' eccentricity bands on the universal-variable quantities of the pair: with
// t = mu - r0 beta, e^2 mu^2 = t^2 + sig^2 beta for ellipses and hyperbolae alike (no
// division, no root).  Ellipses with e^2 < 0.9 and attractive hyperbolae with
// 1.1 < e^2 <= 2500 (the universal-variable band of alg_classify, |e^2 - 1| < 0.1, and the
// hyperbolic head's e <= 50); radial (L = 0), zero-velocity and parabolic pairs have e = 1.
// Returns kLearnedEll, kLearnedHyp or kLearnedPlain; e2m = e^2 mu^2.
__device__ __forceinline__ int learned_band(const UvPair &p, double dt, double &e2m)
{
    e2m = 0.0;
    if (!(dt > 0.0) || !(p.mu > 0.0)) return kLearnedPlain;
    const double t = fma(-p.r0, p.beta, p.mu);
    e2m = fma(p.sig * p.sig, p.beta, t * t);
    const double mu2 = p.mu * p.mu;
    if (p.beta > 0.0) return e2m < 0.9 * mu2 ? kLearnedEll : kLearnedPlain;
    if (p.beta < 0.0 && e2m > 1.1 * mu2 && e2m <= (double)(kHypEMax * kHypEMax) * mu2) return kLearnedHyp;
    return kLearnedPlain;
}

// known_kind (kLearnedEll or kLearnedHyp): the pair was accepted before with that kind, so
// the classification, the domain tests and the head inputs are skipped; every field the
// finishing step reads comes out as in the full call.
__device__ __forceinline__ void learned_prepare(double eps_ij, double dt, const double r[3], const double g[3],
                                                LearnedPair &L, int known_kind = kLearnedPlain)
{
    L.p = uv_prepare(eps_ij, r, g);
    L.kind = kLearnedPlain;
    L.x0 = L.x1 = 0.0f;
    int c;
    if (known_kind == kLearnedPlain) {
        double e2m;
        const int band = learned_band(L.p, dt, e2m);
        if (band == kLearnedPlain) return;
        c = (band == kLearnedEll) ? kClsEll : kClsHyp;
    } else {
        c = (known_kind == kLearnedEll) ? kClsEll : kClsHyp;
    }
    // one rsqrt and one reciprocal for the elements (|beta| > 0 inside the bands)
    const double ab = fabs(L.p.beta);
    L.isqb = rsqrt(ab);
    L.sqb = ab * L.isqb;
    const double imu = 1.0 / L.p.mu;
    const double c0m = L.p.r0 * ab * imu;
    const double s0 = L.p.sig * L.sqb * imu;
    const double n_dt = ab * L.sqb * imu * dt;
    L.C0m = (float)c0m;
    L.S0 = (float)s0;
    L.dM = (float)n_dt;
    if (c == kClsEll) {
        const double c0 = 1.0 - c0m;
        L.C0 = (float)c0;
        L.A0 = atan2f(L.S0, L.C0);
        const float M1 = L.A0 - L.S0 + L.dM;
        const float k = rintf(M1 / kTwoPiF);
        const float Mr = M1 - kTwoPiF * k;
        L.unfold_sign = (Mr < 0.0f) ? -1.0f : 1.0f;
        L.unfold_shift = kTwoPiF * k;
        if (known_kind == kLearnedPlain) {
            const float e = sqrtf((float)fma(c0, c0, s0 * s0));  // a head input only
            if (!(e <= kEllEMax)) return;
            L.x0 = 2.0f * e / kEllEMax - 1.0f;
            L.x1 = 2.0f * fabsf(Mr) / kPiF - 1.0f;
        }
        L.kind = kLearnedEll;
    } else {
        const double c0 = 1.0 + c0m;
        const float e = sqrtf((float)((c0 - s0) * (c0 + s0)));  // head input and A0 only
        if (known_kind == kLearnedPlain && !(e >= kHypEMin && e <= kHypEMax)) return;
        L.C0 = (float)c0;
        L.A0 = asinhf(L.S0 / e);
        const float M1 = L.S0 - L.A0 + L.dM;
        if (known_kind == kLearnedPlain) {
            if (!(fabsf(M1) <= kHypMMax)) return;
            L.x0 = 2.0f * logf(e) / logf(kHypEMax) - 1.0f;
            L.x1 = 2.0f * log1pf(fabsf(M1)) / log1pf(kHypMMax) - 1.0f;
        }
        L.unfold_sign = (M1 < 0.0f) ? -1.0f : 1.0f;
        L.unfold_shift = 0.0f;
        L.kind = kLearnedHyp;
    }
}

// The heads' domain as a cheap test on the universal-variable quantities of the pair (the
// split step's filter that sends a pair to the learned kernel): learned_band, then for the
// hyperbolae in the band |M1| <= 100 in FP32.  The learned kernel decides again with
// learned_prepare (the same band, |M1| from its own elements) and solves a pair outside
// its domain with the plain solver, so this test only chooses the kernel.
__device__ __forceinline__ bool learned_filter(const UvPair &p, double dt)
{
    double e2m;
    const int band = learned_band(p, dt, e2m);
    if (band != kLearnedHyp) return band == kLearnedEll;
    const float mu = (float)p.mu, ab = (float)(-p.beta), sqb = sqrtf(ab);
    const float s0 = (float)p.sig * sqb / mu;
    const float e = sqrtf((float)e2m) / mu;
    const float M1 = s0 - asinhf(s0 / e) + ab * sqb / mu * (float)dt;
    return fabsf(M1) <= kHypMMax;
}

// x - sin x and sinh x - x without cancellation (FP32): series below 0.5
__device__ __forceinline__ float xmsin_f(float x)
{
    const float x2 = x * x;
    if (fabsf(x) < 0.5f) return x * x2 * (1.0f / 6.0f) * (1.0f - x2 * (1.0f / 20.0f) * (1.0f - x2 * (1.0f / 42.0f)));
    return x - sinf(x);
}
__device__ __forceinline__ float sinhmx_f(float x)
{
    const float x2 = x * x;
    if (fabsf(x) < 0.5f) return x * x2 * (1.0f / 6.0f) * (1.0f + x2 * (1.0f / 20.0f) * (1.0f + x2 * (1.0f / 42.0f)));
    return sinhf(x) - x;
}
// sin x and 1 - cos x (FP32); below 0.5 from the series (no libm call, full relative
// accuracy at the tiny increments of small time steps)
__device__ __forceinline__ void sin_omc_f(float x, float &sn, float &omc)
{
    if (fabsf(x) < 0.5f) {
        sn = x - xmsin_f(x);
        const float h = 0.5f * x, h2 = h * h;
        const float sh = h * (1.0f - h2 * (1.0f / 6.0f) * (1.0f - h2 * (1.0f / 20.0f)));
        omc = 2.0f * sh * sh;
    } else {
        float c;
        sincosf(x, &sn, &c);
        omc = 1.0f - c;
    }
}
// sinh x and cosh x - 1 (FP32), series below 0.5
__device__ __forceinline__ void sinh_chm1_f(float x, float &sh, float &chm1)
{
    if (fabsf(x) < 0.5f) {
        sh = x + sinhmx_f(x);
        const float h = 0.5f * x, h2 = h * h;
        const float s2 = h * (1.0f + h2 * (1.0f / 6.0f) * (1.0f + h2 * (1.0f / 20.0f)));
        chm1 = 2.0f * s2 * s2;
    } else {
        const float e = expf(x), ei = 1.0f / e;
        sh = 0.5f * (e - ei);
        chm1 = 0.5f * (e + ei) - 1.0f;
    }
}

// Anomaly guess of the head output y, then the FP32 correction: Newton on the difference
// form, at most kLearnedFp32Steps steps, until a step is below 1e-6 of D.  (At small dt the
// increment D is much smaller than the head's error in the absolute anomaly, so the first
// step alone does not reach the FP64 step's basin.)
constexpr int kLearnedFp32Steps = 4;

__device__ __forceinline__ float learned_first_correction(const LearnedPair &L, float y, int &steps)
{
    float D;
    if (L.kind == kLearnedEll) D = L.unfold_sign * (y * kPiF) + L.unfold_shift - L.A0;
    else D = L.unfold_sign * (y * kHypOut) - L.A0;
    for (steps = 1; steps <= kLearnedFp32Steps; steps++) {
        float F, Fp;
        if (L.kind == kLearnedEll) {
            float sn, omc;  // sin D, 1 - cos D
            sin_omc_f(D, sn, omc);
            F = L.C0m * D + L.C0 * xmsin_f(D) + L.S0 * omc - L.dM;
            Fp = L.C0m + L.C0 * omc + L.S0 * sn;
        } else {
            float sh, chm1;  // sinh D, cosh D - 1
            sinh_chm1_f(D, sh, chm1);
            F = L.C0m * sh + L.S0 * chm1 + sinhmx_f(D) - L.dM;
            Fp = L.C0m * (chm1 + 1.0f) + L.S0 * sh + chm1;
        }
        const float step = __fdividef(F, Fp);  // a guess for the FP64 step: 2 ulp suffice
        D = D - step;
        if (!(fabsf(step) > 1e-6f * fabsf(D))) break;
    }
    if (steps > kLearnedFp32Steps) steps = kLearnedFp32Steps;  // the loop ran out: that many steps
    return D;
}

// The learned pair from the head output y: FP32 correction, FP64 Halley step, composition.
// Returns false (nothing written to h) when the FP64 step did not settle: the caller then
// runs the plain solver.  coarse: the head's guess was more than 1e-2 off in anomaly.
__device__ __forceinline__ bool learned_finish(const LearnedPair &L, double dt, float y, const double r[3],
                                               const double g[3], double h[6], bool &coarse, int &fp32_steps)
{
    const float D = learned_first_correction(L, y, fp32_steps);
    const float Aguess = (L.kind == kLearnedEll) ? L.unfold_sign * (y * kPiF) + L.unfold_shift
                                                 : L.unfold_sign * (y * kHypOut);
    double s = (double)D * L.isqb;
    if (!(s > 0.0) || !isfinite(s)) {
        coarse = true;
        return false;
    }
    const double ds = uv_halley_step(L.p, dt, s);
    const double sn = s - ds;
    coarse = fabsf(Aguess - (L.A0 + (float)(sn * L.sqb))) > 1e-2f;
    if (!(sn > 0.0) || !(fabs(ds) <= 1e-5 * sn)) return false;
    uv_compose(L.p, sn, r, g, h);
    return true;
}

}  // namespace bia
