"""The universal-variable start and the heads' eccentricity bands, restated in numpy and
checked in extended precision (CPU).

uv_series (csrc/bia_pair.cuh) inverts the universal Kepler equation
    t = r0 s c1(beta s^2) + sig s^2 c2(beta s^2) + mu s^3 c3(beta s^2)
to fifth order with the Lagrange reversion coefficients (Abramowitz and Stegun 3.6.25),
written in the dimensionless variables x = dt/r0, y = sig dt/(2 r0^2), m = mu/r0,
z = (m - beta) x^2/6, w = beta x^2, and skips the Newton correction when every
|a_k t^(k-1)| <= Q^(k-1) a1 with Q = 3e-4; the truncation must then be below a tenth of an
FP64 ulp.  uv_compose_series composes the half-displacement from the same variables.  learned_band (csrc/bia_learned.cuh)
decides the heads' domain from e^2 mu^2 = (mu - r0 beta)^2 + sig^2 beta, which must be the
eccentricity of e^2 = 1 + E L^2 / mu^2 with E = |g|^2 - 2 mu / r0.
"""
import math

import numpy as np

L = np.longdouble
Q = 3e-4
FACT = [L(1)]
for _k in range(1, 50):
    FACT.append(FACT[-1] * _k)


def _time_of_flight(s, r0, sig, mu, beta):
    z = beta * s * s
    c = [sum((-z) ** j / FACT[2 * j + m] for j in range(16)) for m in range(4)]
    return r0 * s * c[1] + sig * s * s * c[2] + mu * s ** 3 * c[3], r0 * c[0] + sig * s * c[1] + mu * s * s * c[2]


def _reversion(r0, sig, mu, beta, t):
    ir0 = 1 / r0
    h = sig / 2
    b3 = (mu - r0 * beta) / 6
    b4 = -h * beta / 12
    b5 = beta * (r0 * beta - mu) / 120
    a = [ir0, -h * ir0 ** 3, (2 * h * h - r0 * b3) * ir0 ** 5,
         (5 * r0 * h * b3 - r0 * r0 * b4 - 5 * h ** 3) * ir0 ** 7,
         (6 * r0 * r0 * h * b4 + 3 * r0 * r0 * b3 * b3 + 14 * h ** 4 - r0 ** 3 * b5 - 21 * r0 * h * h * b3) * ir0 ** 9]
    small = all(abs(a[k] * t ** k) <= L(Q) ** k * a[0] for k in range(1, 5))
    s5 = t * (a[0] + t * (a[1] + t * (a[2] + t * (a[3] + t * a[4]))))
    return s5, small


def test_fifth_order_start_is_exact_where_newton_is_skipped():
    rng = np.random.default_rng(3)
    worst, skipped = 0.0, 0
    for _ in range(1500):
        r0 = L(10 ** rng.uniform(-3, 0.5))
        v = L(10 ** rng.uniform(-2, 1))
        sig = r0 * v * L(rng.uniform(-1, 1))
        mu = L(10 ** rng.uniform(-7, 0)) * (1 if rng.uniform() < 0.8 else -1)   # repulsive pairs too
        beta = 2 * mu / r0 - v * v
        T = min(r0 / v, L(math.sqrt(float(r0 ** 3 / abs(mu)))))
        dt = T * L(10 ** rng.uniform(-4.5, -2.8))                               # around the bound
        s = dt / r0
        for _ in range(40):                                                      # the solved s
            F, Fp = _time_of_flight(s, r0, sig, mu, beta)
            s = s - (F - dt) / Fp
        s5, small = _reversion(r0, sig, mu, beta, dt)
        if small and s5 > 0:
            skipped += 1
            worst = max(worst, float(abs(s5 - s) / s))
    assert skipped > 500
    assert worst <= 2e-17, worst


def _dimensionless(r0, sig, mu, beta, dt):
    """uv_series' variables and relative terms c1..c4 (c_k = a_(k+1) dt^k / a1)."""
    x = dt / r0
    y = sig / r0 * x / 2
    m = mu / r0
    x2 = x * x
    z = (m - beta) * x2 / 6
    w = beta * x2
    c = [-y, 2 * y * y - z, y * (5 * z + w / 12 - 5 * y * y),
         y * y * (14 * y * y - 21 * z - w / 2) + z * (3 * z + w / 20)]
    return x, y, m, x2, w, c


def _pairs(rng, count):
    for _ in range(count):
        r0 = L(10 ** rng.uniform(-3, 0.5))
        v = L(10 ** rng.uniform(-2, 1))
        sig = r0 * v * L(rng.uniform(-1, 1))
        mu = L(10 ** rng.uniform(-7, 0)) * (1 if rng.uniform() < 0.8 else -1)
        beta = 2 * mu / r0 - v * v
        T = min(r0 / v, L(math.sqrt(float(r0 ** 3 / abs(mu)))))
        yield r0, sig, mu, beta, T * L(10 ** rng.uniform(-5, -2.5))


def test_dimensionless_terms_are_the_reversion_coefficients():
    rng = np.random.default_rng(5)
    agree = 0
    for r0, sig, mu, beta, dt in _pairs(rng, 1500):
        ir0 = 1 / r0
        h = sig / 2
        b3 = (mu - r0 * beta) / 6
        b4 = -h * beta / 12
        b5 = beta * (r0 * beta - mu) / 120
        a = [ir0, -h * ir0 ** 3, (2 * h * h - r0 * b3) * ir0 ** 5,
             (5 * r0 * h * b3 - r0 * r0 * b4 - 5 * h ** 3) * ir0 ** 7,
             (6 * r0 * r0 * h * b4 + 3 * r0 * r0 * b3 * b3 + 14 * h ** 4 - r0 ** 3 * b5 - 21 * r0 * h * h * b3) * ir0 ** 9]
        x, _, _, _, _, c = _dimensionless(r0, sig, mu, beta, dt)
        for k in range(1, 5):
            ref = a[k] * dt ** k / a[0]
            # both forms sum terms that cancel; compare on the scale of the largest term of c_k
            scale = max(abs(ref), L(Q) ** (k + 2))
            assert abs(c[k - 1] - ref) <= 1e-15 * scale
        # the same exactness decision and the same fifth-order sum
        small_a = all(abs(a[k] * dt ** k) <= L(Q) ** k * a[0] for k in range(1, 5))
        small_c = all(abs(c[k - 1]) <= L(Q) ** k for k in range(1, 5))
        s5 = dt * (a[0] + dt * (a[1] + dt * (a[2] + dt * (a[3] + dt * a[4]))))
        assert abs(x * (1 + sum(c)) - s5) <= 1e-17 * abs(s5)
        agree += small_a == small_c
    assert agree >= 1495


def test_series_composition_matches_the_lagrange_coefficients():
    """(f - 1)/2 = K A, (g - dt)/2 = K dt B, f'/2 = -(m/2)(x/r0) S c1 rho, (g' - 1)/2 = K A rho
    with rho = 1/(1 + d), d = -w S^2 c2 + 2 y S c1 - 2 K A, at the solved s = x S."""
    rng = np.random.default_rng(6)
    worst = 0.0
    for r0, sig, mu, beta, dt in _pairs(rng, 400):
        s = dt / r0
        for _ in range(40):
            F, Fp = _time_of_flight(s, r0, sig, mu, beta)
            s = s - (F - dt) / Fp
        z = beta * s * s
        st = [sum((-z) ** j / FACT[2 * j + m] for j in range(16)) for m in range(4)]
        rr = r0 * st[0] + sig * s * st[1] + mu * s * s * st[2]
        ref = [-mu * s * s * st[2] / r0, -mu * s ** 3 * st[3], -mu * s * st[1] / (rr * r0), -mu * s * s * st[2] / rr]
        x, y, m, x2, w, _ = _dimensionless(r0, sig, mu, beta, dt)
        S = s / x
        arg = w * S * S
        c = [sum((-arg) ** j / FACT[2 * j + k] for j in range(16)) for k in range(4)]
        K = -m * x2 / 2
        A, B = S * S * c[2], S ** 3 * c[3]
        d = -arg * c[2] + 2 * y * S * c[1] - 2 * K * A
        rho = 1 / (1 + d)
        got = [2 * K * A, 2 * K * dt * B, -m * x / r0 * S * c[1] * rho, 2 * K * A * rho]
        worst = max(worst, max(float(abs(g - f) / abs(f)) for g, f in zip(got, ref)))
    assert worst <= 1e-17, worst


def test_eccentricity_bands_identity():
    rng = np.random.default_rng(4)
    r = rng.standard_normal((3, 2000))
    g = rng.standard_normal((3, 2000)) * rng.uniform(0.1, 3.0, 2000)
    mu = rng.uniform(0.1, 5.0, 2000)
    r0 = np.sqrt((r * r).sum(0))
    sig = (r * g).sum(0)
    v2 = (g * g).sum(0)
    beta = 2 * mu / r0 - v2
    e2m = (mu - r0 * beta) ** 2 + sig * sig * beta
    Lsq = (np.cross(r.T, g.T) ** 2).sum(1)
    E = v2 - 2 * mu / r0
    e2 = 1 + E * Lsq / mu ** 2
    assert np.allclose(e2m / mu ** 2, e2, rtol=1e-9, atol=1e-9)
