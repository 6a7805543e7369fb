"""ctypes binding of the CPU oracle (test infrastructure only).

The oracle restates the reference's CPU path of the BIA step in plain C
(``oracle/bia_oracle.c``).  Only the test-suite, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline leg import this module; the product library never
does.  Arrays are numpy float64, structure-of-arrays: ``state`` has shape
``(6, n)`` holding x, y, z, u, v, w.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libbia_oracle.so")
_lib = None

_D = ctypes.c_double
_I = ctypes.c_int
_PD = ctypes.POINTER(ctypes.c_double)
_PI = ctypes.POINTER(ctypes.c_int)
_PL = ctypes.POINTER(ctypes.c_int64)

STAT_NAMES = ("hyperbola", "parabola", "ellipse", "degenerate", "rkf", "universal",
              "iterations", "rkf_steps", "nonconverged", "bracket_exits", "fallbacks",
              "uv_iterations")


def build():
    """Compile the oracle library (gcc, no FMA contraction)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.oracle_bia_step.argtypes = [_I, _I, _D, _PD, _D, _I, _D, _D] + [_PD] * 12 + [_PL]
        L.oracle_bia_rows_omp.argtypes = ([_I, _I, _D, _PD, _D, _I, _D, _D] + [_PD] * 6 +
                                          [_PI, _I] + [_PD] * 6 + [_I, _PL])
        L.oracle_bia_rows_omp.restype = ctypes.c_int64
        L.oracle_particle_disp.argtypes = ([_I, _I, _D, _PD, _D, _I, _D, _D] + [_PD] * 6 +
                                           [_PI, _I, _PD, _I])
        L.oracle_pair_halfdisp.argtypes = [_I, _D, _D, _I, _D, _D, _PD, _PD, _PD, _PL]
        L.oracle_pair_halfdisp_q.argtypes = L.oracle_pair_halfdisp.argtypes
        L.oracle_bia_step_q.argtypes = L.oracle_bia_step.argtypes
        L.oracle_particle_disp_q.argtypes = L.oracle_particle_disp.argtypes
        L.oracle_bia_rows_omp_q.argtypes = L.oracle_bia_rows_omp.argtypes
        L.oracle_bia_rows_omp_q.restype = ctypes.c_int64
        L.oracle_find_hyperbola.argtypes = [_D, _D, _PD, _PD, _PD, _I, _PI, _PI]
        L.oracle_find_hyperbola.restype = _I
        L.oracle_find_ellipse.argtypes = [_D, _D, _PD, _PD, _PD, _I, _PI]
        L.oracle_find_ellipse.restype = _I
        L.oracle_find_parabola.argtypes = [_D, _D, _PD, _PD, _PD]
        L.oracle_find_parabola.restype = _I
        L.oracle_find_dxyuv_rkf.argtypes = [_D, _D, _PD, _PD, _PD, _D, _D, _PI]
        L.oracle_find_dxyuv_rkf.restype = _I
        L.oracle_xyz_to_xi_eta_zeta.argtypes = [_PD] * 6
        L.oracle_xyz_to_xi_eta_zeta.restype = _I
        L.oracle_invariance_cpu.argtypes = [_I, _D, _PD] + [_PD] * 6 + [_PD]
        L.oracle_invariance_qpu.argtypes = [_I, _D, _PD] + [_PD] * 6 + [_PD]
        L.oracle_dim_rkf.argtypes = [_I, _D, _D, _D, _PD, _D, _D, _PD, _PI, _PI]
        L.oracle_dim_rkf.restype = _I
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(_PD) if a is not None else None


def _c(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def bia_step(state, eps_th, dt, method=1, q=None, itr=18, relerr=0.0, abserr=1e-16, quad=False):
    """One BIA step in the reference's pair order (bia/bia.f90:126-204).

    Returns (new_state, disp, stats) where disp = (dX..dW) including drift.
    quad=True evaluates the same algorithm in __float128 (state stored in FP64 between
    steps): the step without rounding noise.
    """
    s = np.array(state, dtype=np.float64, copy=True)
    n = s.shape[1]
    d = np.zeros((6, n))
    qq = _c(q) if q is not None else None
    st = np.zeros(12, dtype=np.int64)
    rows = [np.ascontiguousarray(s[k]) for k in range(6)]
    f = lib().oracle_bia_step_q if quad else lib().oracle_bia_step
    f(method, n, eps_th, _p(qq), dt, itr, relerr, abserr,
                          *[_p(r) for r in rows], *[_p(d[k]) for k in range(6)],
                          st.ctypes.data_as(_PL))
    return np.stack(rows), d, dict(zip(STAT_NAMES, st.tolist()))


def bia_rows(state, eps_th, dt, rows, method=1, q=None, itr=18, relerr=0.0, abserr=1e-16,
             nthreads=0):
    """Pair sums for the given rows i (all j > i), OpenMP; no drift.  Returns
    (pair_sums (6, n), pairs, stats)."""
    s = _c(state)
    n = s.shape[1]
    r = np.ascontiguousarray(rows, dtype=np.int32)
    d = np.zeros((6, n))
    qq = _c(q) if q is not None else None
    st = np.zeros(12, dtype=np.int64)
    cols = [np.ascontiguousarray(s[k]) for k in range(6)]
    pairs = lib().oracle_bia_rows_omp(method, n, eps_th, _p(qq), dt, itr, relerr, abserr,
                                      *[_p(c) for c in cols], r.ctypes.data_as(_PI), len(r),
                                      *[_p(d[k]) for k in range(6)], nthreads,
                                      st.ctypes.data_as(_PL))
    return d, int(pairs), dict(zip(STAT_NAMES, st.tolist()))


def particle_disp(state, eps_th, dt, sel, method=1, q=None, itr=18, relerr=0.0, abserr=1e-16,
                  nthreads=0, quad=False):
    """Full step displacement (dX..dW, drift included) of the particles in sel,
    summed over every other particle.  Returns (len(sel), 6)."""
    s = _c(state)
    n = s.shape[1]
    sl = np.ascontiguousarray(sel, dtype=np.int32)
    out = np.zeros((len(sl), 6))
    qq = _c(q) if q is not None else None
    cols = [np.ascontiguousarray(s[k]) for k in range(6)]
    f = lib().oracle_particle_disp_q if quad else lib().oracle_particle_disp
    f(method, n, eps_th, _p(qq), dt, itr, relerr, abserr,
                               *[_p(c) for c in cols], sl.ctypes.data_as(_PI), len(sl), _p(out),
                               nthreads)
    return out


def pair_halfdisp(r, g, eps_th, dt, method=1, itr=18, relerr=0.0, abserr=1e-16, quad=False):
    """Half-displacement h (6,) that bia.f90 adds to i and subtracts from j."""
    rr, gg, h = _c(r), _c(g), np.zeros(6)
    st = np.zeros(12, dtype=np.int64)
    f = lib().oracle_pair_halfdisp_q if quad else lib().oracle_pair_halfdisp
    f(method, eps_th, dt, itr, relerr, abserr, _p(rr), _p(gg), _p(h),
                               st.ctypes.data_as(_PL))
    return h, dict(zip(STAT_NAMES, st.tolist()))


def frame(r, g):
    rr, gg = _c(r), _c(g)
    exi, eeta, ezeta, Y = np.zeros(3), np.zeros(3), np.zeros(3), np.zeros(4)
    deg = lib().oracle_xyz_to_xi_eta_zeta(_p(rr), _p(gg), _p(exi), _p(eeta), _p(ezeta), _p(Y))
    return exi, eeta, ezeta, Y, bool(deg)


def find_hyperbola(eps_th, dt, YZ, itr=18, return_fallback=False):
    yz, yn, err, bx, fb = _c(YZ), np.zeros(4), _D(0), _I(0), _I(0)
    it = lib().oracle_find_hyperbola(eps_th, dt, _p(yz), _p(yn), ctypes.byref(err), itr,
                                     ctypes.byref(bx), ctypes.byref(fb))
    if return_fallback:
        return yn, err.value, it, fb.value
    return yn, err.value, it


def find_ellipse(eps_th, dt, YZ, itr=18, return_fallback=False):
    yz, yn, err, fb = _c(YZ), np.zeros(4), _D(0), _I(0)
    it = lib().oracle_find_ellipse(eps_th, dt, _p(yz), _p(yn), ctypes.byref(err), itr,
                                   ctypes.byref(fb))
    if return_fallback:
        return yn, err.value, it, fb.value
    return yn, err.value, it


def find_parabola(eps_th, dt, YZ):
    yz, yn, err = _c(YZ), np.zeros(4), _D(0)
    it = lib().oracle_find_parabola(eps_th, dt, _p(yz), _p(yn), ctypes.byref(err))
    return yn, err.value, it


def find_dxyuv_rkf(eps_th, dt, YZ, relerr=0.0, abserr=1e-16):
    yz, yn, err, nacc = _c(YZ), np.zeros(4), _D(0), _I(0)
    ier = lib().oracle_find_dxyuv_rkf(eps_th, dt, _p(yz), _p(yn), ctypes.byref(err), relerr,
                                      abserr, ctypes.byref(nacc))
    return yn, err.value, ier, nacc.value


INV_NAMES = ("KE", "PE", "Lx", "Ly", "Lz", "Ua", "Va", "Wa", "Xa", "Ya", "Za")


def invariance(state, eps_th, q=None, quad=False):
    """bia/Invariance_CPU.f90 (FP64) or bia/Invariance_QPU.f90 (__float128)."""
    s = _c(state)
    qq = _c(q) if q is not None else None
    out = np.zeros(11)
    f = lib().oracle_invariance_qpu if quad else lib().oracle_invariance_cpu
    f(s.shape[1], eps_th, _p(qq), *[_p(np.ascontiguousarray(s[k])) for k in range(6)], _p(out))
    return dict(zip(INV_NAMES, out.tolist()))


def dim_rkf(y0_aos, eps_th, x0, xe, relerr=0.0, abserr=1e-16):
    """dim/rkf_kernel.cu rkf_c_ restated on the CPU.  y0_aos: (6n,) AoS."""
    y0 = _c(y0_aos)
    n = y0.size // 6
    yn = np.zeros_like(y0)
    nacc, nde = _I(0), _I(0)
    ier = lib().oracle_dim_rkf(n, eps_th, x0, xe, _p(y0), relerr, abserr, _p(yn),
                               ctypes.byref(nacc), ctypes.byref(nde))
    return yn, ier, nacc.value, nde.value


# ---- the reference's own GPU code, built from its sources by oracle/build_ref.sh ----------
_REF_PATH = os.path.join(_HERE, "_ref", "libref_bia.so")
_ref = None


def ref_gpu_available():
    return os.path.exists(_REF_PATH)


def ref_gpu_lib():
    """The reference's find_dxyuv_kernel_ / invariance_gpu_ compiled for sm_100a."""
    global _ref
    if _ref is None:
        L = ctypes.CDLL(_REF_PATH)
        L.find_dxyuv_kernel_.argtypes = [_I, _I, _I, _D, _D, _I] + [_PD] * 8
        L.find_dxyuv_kernel_.restype = None
        _ref = L
    return _ref


def ref_gpu_rows(state, eps_th, dt, rows, itr=18):
    """The reference's GPU branch of bia/bia.f90:128-140 for the given 1-based rows I
    (ALG method only): returns the accumulated pair sums (6, n), no drift."""
    L = ref_gpu_lib()
    s = _c(state)
    n = s.shape[1]
    acc = [np.zeros(n) for _ in range(6)]
    rel = np.zeros(6 * n)
    out = np.zeros(6 * n)
    for I in rows:
        i = I - 1
        for k in range(6):
            rel[k::6] = s[k, i] - s[k]
        L.find_dxyuv_kernel_(1, n, int(I), eps_th, dt, itr, *[_p(a) for a in acc], _p(rel), _p(out))
    return np.stack(acc)
