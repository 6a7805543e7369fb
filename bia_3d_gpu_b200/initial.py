"""Seeded initial conditions for the BIA workloads.

All generators use numpy.random.default_rng(seed) and return SoA float64 arrays of
shape (6, n) (x, y, z, u, v, w), plus the pair coupling.  The coupling follows the
reference's convention: the relative equation of motion is r'' = eps_ij r / |r|^3
(bia/find_dXYUV_RKF.f90:15-23), so gravity with G = 1 and masses m_i gives
eps_ij = -(m_i + m_j) and Coulomb with unit masses gives eps_ij = +2 q_i q_j.

Workloads (name: n, coupling, positions, velocities, dt x steps):
  gravity_ball_1332   1332, -2/n, uniform unit ball, Gaussian sigma 0.3, 1e-4 x 100
  coulomb_cube_32768  32768, 2 q_i q_j (q = +-1 balanced, shuffled), unit cube with
                      minimum separation 1e-3, Maxwellian sigma 1, 1e-5 x 50
  plummer_32768       32768, -2/n, Plummer sphere (a = 1, G = M = 1), 1e-4 x 100
  cold_ball_131072    131072, -2/n, uniform unit ball, zero velocity, 5e-5 x 50
  lattice             (2 NL + 1)^3 + 1 particles on a jittered cubic lattice with
                      uniform velocities in [-1/2, 1/2), particle 1 at rest at the
                      origin, ordered shell by shell (IC/bbb_maker_REV.f90:10-71;
                      numpy's generator replaces gfortran's random_number)
"""
import numpy as np


def uniform_ball(n, rng):
    v = rng.standard_normal((3, n))
    v /= np.linalg.norm(v, axis=0)
    r = rng.random(n) ** (1.0 / 3.0)
    return v * r


def _remove_bulk(s):
    s = s.copy()
    s[:3] -= s[:3].mean(axis=1, keepdims=True)
    s[3:] -= s[3:].mean(axis=1, keepdims=True)
    return s


def gravity_ball(n=1332, sigma=0.3, seed=1):
    rng = np.random.default_rng(seed)
    pos = uniform_ball(n, rng)
    vel = rng.standard_normal((3, n)) * sigma
    return np.ascontiguousarray(np.vstack([pos, vel])), -2.0 / n


def _enforce_min_separation(pos, dmin, rng, lo=0.0, hi=1.0, max_rounds=100):
    from scipy.spatial import cKDTree
    for _ in range(max_rounds):
        pairs = cKDTree(pos.T).query_pairs(dmin, output_type="ndarray")
        if len(pairs) == 0:
            return pos
        bad = np.unique(pairs[:, 1])
        pos[:, bad] = lo + (hi - lo) * rng.random((3, bad.size))
    raise RuntimeError("could not reach the minimum separation")


def coulomb_cube(n=32768, sigma=1.0, dmin=1e-3, seed=2):
    """Returns (state, eps_th, q): pair coupling eps_th * q_i * q_j with eps_th = 2."""
    rng = np.random.default_rng(seed)
    pos = _enforce_min_separation(rng.random((3, n)), dmin, rng)
    vel = rng.standard_normal((3, n)) * sigma
    q = np.ones(n)
    q[: n // 2] = -1.0
    rng.shuffle(q)
    return np.ascontiguousarray(np.vstack([pos, vel])), 2.0, q


def plummer(n=32768, seed=3, rmax=None):
    """Plummer sphere, scale radius 1, G = M = 1 (Aarseth, Henon & Wielen 1974)."""
    rng = np.random.default_rng(seed)
    x1 = rng.random(n)
    r = 1.0 / np.sqrt(x1 ** (-2.0 / 3.0) - 1.0)
    if rmax is not None:
        while np.any(r > rmax):
            bad = r > rmax
            x1b = rng.random(bad.sum())
            r[bad] = 1.0 / np.sqrt(x1b ** (-2.0 / 3.0) - 1.0)
    dirs = rng.standard_normal((3, n))
    dirs /= np.linalg.norm(dirs, axis=0)
    pos = dirs * r
    # speed fraction q of the escape speed from g(q) = q^2 (1 - q^2)^{7/2} by rejection
    q = np.empty(n)
    todo = np.arange(n)
    while todo.size:
        a = rng.random(todo.size)
        b = rng.random(todo.size) * 0.1
        ok = b < a * a * (1.0 - a * a) ** 3.5
        q[todo[ok]] = a[ok]
        todo = todo[~ok]
    vesc = np.sqrt(2.0) * (1.0 + r * r) ** -0.25
    vd = rng.standard_normal((3, n))
    vd /= np.linalg.norm(vd, axis=0)
    vel = vd * (q * vesc)
    s = _remove_bulk(np.vstack([pos, vel]))
    return np.ascontiguousarray(s), -2.0 / n


def cold_ball(n=131072, seed=5):
    rng = np.random.default_rng(seed)
    pos = uniform_ball(n, rng)
    vel = np.zeros((3, n))
    return np.ascontiguousarray(np.vstack([pos, vel])), -2.0 / n


def lattice(NL=5, seed=0):
    """Jittered cubic lattice of IC/bbb_maker_REV.f90 (shell-by-shell order)."""
    rng = np.random.default_rng(seed)
    n = (2 * NL + 1) ** 3 + 1
    dd = rng.random((n, 6)) - 0.5
    out = np.zeros((n, 6))
    out[1] = dd[1]
    k = 2
    for L in range(1, NL + 1):
        cells = []
        for iz in (-L, L):
            for iy in range(-L, L + 1):
                for ix in range(-L, L + 1):
                    cells.append((ix, iy, iz))
        for iy in (-L, L):
            for iz in range(1 - L, L):
                for ix in range(-L, L + 1):
                    cells.append((ix, iy, iz))
        for ix in (-L, L):
            for iz in range(1 - L, L):
                for iy in range(1 - L, L):
                    cells.append((ix, iy, iz))
        for ix, iy, iz in cells:
            out[k, :3] = dd[k, :3] + (ix, iy, iz)
            out[k, 3:] = dd[k, 3:]
            k += 1
    assert k == n
    return np.ascontiguousarray(out.T), None


def ensemble_sizes(systems=4096, nmin=32, nmax=1024, seed=4):
    rng = np.random.default_rng(seed)
    return rng.integers(nmin, nmax + 1, size=systems)


WORKLOADS = {
    "gravity_ball_1332": dict(gen=gravity_ball, n=1332, dt=1e-4, steps=100),
    "coulomb_cube_32768": dict(gen=coulomb_cube, n=32768, dt=1e-5, steps=50),
    "plummer_32768": dict(gen=plummer, n=32768, dt=1e-4, steps=100),
    "cold_ball_131072": dict(gen=cold_ball, n=131072, dt=5e-5, steps=50),
}


def make(name, n=None, seed=None):
    """(state, eps_th, q, dt, steps) of a named workload, optionally at another n."""
    w = WORKLOADS[name]
    kw = {}
    if n is not None:
        kw["n"] = n
    if seed is not None:
        kw["seed"] = seed
    out = w["gen"](**kw)
    if len(out) == 3:
        s, eps, q = out
    else:
        (s, eps), q = out, None
    return s, eps, q, w["dt"], w["steps"]
