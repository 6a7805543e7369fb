"""bia_3d_gpu_b200 -- the BIA pair step of bia_3d_gpu, rebuilt for B200 (sm_100a).

Two layers, both backed only by libbia_b200.so (CUDA kernels; no CPU fallback):

* the reference's Fortran-facing interface, same names and argument meaning:
    find_dxyuv_kernel(METHOD, N, I, EPS, DT, ITR, dX, dY, dZ, dU, dV, dW, RXYZUVW, dXYZUVW)
        bia/find_dXYUV_kernel.cu:526-561, as called from bia/bia.f90:135,138
    invariance_gpu(N, eps_th, X, Y, Z, U, V, W) -> (KE, PE, Lx, Ly, Lz, Ua, Va, Wa, Xa, Ya, Za)
        bia/invariance.cu:50-110, as called from bia/bia.f90:67-68
  operating in place on host numpy float64 arrays;

* BIASolver: whole steps on device-resident state (a (6, n) float64 CUDA tensor),
  multi-step runs captured in a CUDA graph, host-buffer runs, device invariants.
"""
import ctypes
import os

import numpy as np

from . import capi
from .capi import (BIA_ERR_NONFINITE, BIA_OK, METHOD_ALG, METHOD_LEARNED, METHOD_RKF,
                   METHOD_UNIVERSAL, BiaConfig, BiaError, BiaStats, default_config)

__all__ = ["find_dxyuv_kernel", "invariance_gpu", "BIASolver", "default_config", "BiaConfig",
           "BiaError", "METHOD_ALG", "METHOD_RKF", "METHOD_UNIVERSAL", "METHOD_LEARNED",
           "INVARIANT_NAMES", "measure_fp64_peak", "HEADS_PATH", "HeadTrainer"]

# the trained heads of BIA_METHOD_LEARNED (bia_3d_gpu_b200/train_heads.py writes them)
HEADS_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "learned_heads.bin")

INVARIANT_NAMES = ("KE", "PE", "Lx", "Ly", "Lz", "Ua", "Va", "Wa", "Xa", "Ya", "Za")

_PD = ctypes.POINTER(ctypes.c_double)


def _host_f64(a, n, name):
    if not isinstance(a, np.ndarray) or a.dtype != np.float64 or not a.flags.c_contiguous:
        raise TypeError(f"{name} must be a C-contiguous float64 numpy array")
    if a.size < n:
        raise ValueError(f"{name} has {a.size} elements, need {n}")
    return a.ctypes.data_as(_PD)


def find_dxyuv_kernel(METHOD, N, I, EPS, DT, ITR, dX, dY, dZ, dU, dV, dW, RXYZUVW, dXYZUVW):
    """Pair solve of particle I (1-based) against every j > I, on the GPU.

    Mirrors find_dxyuv_kernel_ (bia/find_dXYUV_kernel.cu:526-561): RXYZUVW holds the
    AoS relative state x_I - x_j, ..., w_I - w_j for all j (6N doubles); dXYZUVW
    (6N doubles) receives the half-displacements; dX..dW are accumulated in place
    (dX[I] += h_j, dX[j] -= h_j).  No drift is added.  Returns the status code
    (0 ok, 2 when a pair gave a non-finite result); other failures raise BiaError.
    """
    L = capi.lib()
    ptrs = [_host_f64(a, N, nm) for a, nm in ((dX, "dX"), (dY, "dY"), (dZ, "dZ"), (dU, "dU"),
                                              (dV, "dV"), (dW, "dW"))]
    p_rel = _host_f64(RXYZUVW, 6 * N, "RXYZUVW")
    p_out = _host_f64(dXYZUVW, 6 * N, "dXYZUVW")
    L.find_dxyuv_kernel_(int(METHOD), int(N), int(I), float(EPS), float(DT), int(ITR), *ptrs,
                         p_rel, p_out)
    st = L.bia_last_error()
    if st not in (BIA_OK, BIA_ERR_NONFINITE):
        raise BiaError(st, "find_dxyuv_kernel")
    return st


def invariance_gpu(N, eps_th, X, Y, Z, U, V, W):
    """Invariants on the GPU (bia/invariance.cu:50-110): returns the tuple
    (KE, PE, Lx, Ly, Lz, Ua, Va, Wa, Xa, Ya, Za) that the reference returns through
    its scalar pointer arguments.  KE = sum |v|^2, PE = eps_th * sum_{i<j} 1/r_ij."""
    L = capi.lib()
    ins = [_host_f64(a, N, nm) for a, nm in ((X, "X"), (Y, "Y"), (Z, "Z"), (U, "U"), (V, "V"),
                                             (W, "W"))]
    outs = [ctypes.c_double(0.0) for _ in range(11)]
    L.invariance_gpu_(int(N), float(eps_th), *ins, *[ctypes.byref(o) for o in outs])
    st = L.bia_last_error()
    if st != BIA_OK:
        raise BiaError(st, "invariance_gpu")
    return tuple(o.value for o in outs)


def rkf_c(neq, eps_th, X0, XE, YH0, INIT, RELERR, ABSERR, H=0.0):
    """Direct-integration run on the GPU, mirroring rkf_c_ (dim/rkf_kernel.cu:194-495) as
    called from dim/dim_3D.f90:30.  YH0: host AoS state (neq = 6n float64), updated to
    the final state; H: the step size to start from when INIT != 1 (the previous call's).
    Returns a dict with YHN, ESE, NDE, IER, H, X0 (= XE), INIT."""
    L = capi.lib()
    n = int(neq)
    x0 = ctypes.c_double(X0)
    xe = ctypes.c_double(XE)
    init = ctypes.c_int(INIT)
    rel = ctypes.c_double(RELERR)
    abs_ = ctypes.c_double(ABSERR)
    nde = ctypes.c_int(0)
    ier = ctypes.c_int(0)
    h = ctypes.c_double(H)
    yh0 = np.ascontiguousarray(YH0, dtype=np.float64)
    outs = {k: np.zeros(n) for k in ("YHN", "ESE", "YL0", "YLN", "ERR")}
    _host_f64(yh0, n, "YH0")
    L.rkf_c_(n, float(eps_th), ctypes.byref(x0), ctypes.byref(xe), yh0.ctypes.data_as(_PD),
             ctypes.byref(init), ctypes.byref(rel), ctypes.byref(abs_),
             outs["YHN"].ctypes.data_as(_PD), outs["ESE"].ctypes.data_as(_PD), ctypes.byref(nde),
             ctypes.byref(ier), ctypes.byref(h), outs["YL0"].ctypes.data_as(_PD),
             outs["YLN"].ctypes.data_as(_PD), outs["ERR"].ctypes.data_as(_PD), None)
    st = L.bia_last_error()
    if st not in (BIA_OK, capi.BIA_ERR_NOT_CONVERGED):
        raise BiaError(st, "rkf_c")
    return dict(outs, NDE=nde.value, IER=ier.value, H=h.value, X0=x0.value, INIT=init.value,
                YH0=yh0)


def measure_fp64_peak(device=0):
    """Measured FP64 FMA throughput of the device in TFLOP/s."""
    out = ctypes.c_double(0.0)
    capi.check(capi.lib().bia_measure_fp64_peak(int(device), ctypes.byref(out)),
               "bia_measure_fp64_peak")
    return out.value


class BIASolver:
    """Device-resident BIA steps through libbia_b200.so.

    state: a (6, n) contiguous float64 CUDA tensor (x, y, z, u, v, w rows), updated in
    place.  q: optional (n,) float64 CUDA tensor of charges (pair coupling
    eps_th * q_i * q_j).  The solver launches on `stream` (a torch.cuda.Stream; default:
    a new non-default stream, which allows CUDA-graph replay in run()).
    """

    def __init__(self, device=0, stream=None):
        import torch
        self._torch = torch
        self.device = torch.device("cuda", device)
        if stream is None:
            stream = torch.cuda.Stream(device=self.device)
        self.stream = stream
        self._ctx = ctypes.c_void_p()
        capi.check(capi.lib().bia_context_create(ctypes.byref(self._ctx), int(device),
                                                 ctypes.c_void_p(stream.cuda_stream)),
                   "bia_context_create")

    def close(self):
        if self._ctx:
            capi.lib().bia_context_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- helpers ----------------------------------------------------------------------
    def _check_state(self, state):
        t = self._torch
        if not (isinstance(state, t.Tensor) and state.is_cuda and state.dtype == t.float64 and
                state.dim() == 2 and state.shape[0] == 6 and state.is_contiguous()):
            raise TypeError("state must be a contiguous (6, n) float64 CUDA tensor")
        return state.shape[1]

    def _ptrs(self, state):
        n = state.shape[1]
        base = state.data_ptr()
        return [ctypes.c_void_p(base + k * n * 8) for k in range(6)]

    def _qptr(self, q, n):
        if q is None:
            return ctypes.c_void_p(None)
        t = self._torch
        if not (isinstance(q, t.Tensor) and q.is_cuda and q.dtype == t.float64 and
                q.numel() == n and q.is_contiguous()):
            raise TypeError("q must be a contiguous float64 CUDA tensor of n charges")
        return ctypes.c_void_p(q.data_ptr())

    def _enter(self):
        """Order the solver's stream after work already queued on torch's current stream."""
        cur = self._torch.cuda.current_stream(self.device)
        if cur.cuda_stream != self.stream.cuda_stream:
            self.stream.wait_stream(cur)
        return cur

    def _leave(self, cur):
        """Make torch's current stream wait for the solver's launches."""
        if cur.cuda_stream != self.stream.cuda_stream:
            cur.wait_stream(self.stream)

    @staticmethod
    def _finish(st, stats, what):
        if st not in (BIA_OK, BIA_ERR_NONFINITE):
            raise BiaError(st, what)
        return stats.as_dict()

    # -- API --------------------------------------------------------------------------
    def step(self, state, cfg, q=None, disp=None, stats=True):
        """One BIA step (all pairs, reduction, drift, update).  disp: optional (6, n)
        float64 CUDA tensor receiving dX..dW.  Returns the step's counters (this
        synchronises) or None with stats=False."""
        n = self._check_state(state)
        dp = ctypes.c_void_p(disp.data_ptr()) if disp is not None else ctypes.c_void_p(None)
        s = BiaStats()
        cur = self._enter()
        st = capi.lib().bia_step(self._ctx, ctypes.byref(cfg), n, *self._ptrs(state),
                                 self._qptr(q, n), dp, ctypes.byref(s) if stats else None)
        self._leave(cur)
        if not stats:
            capi.check(st, "bia_step")
            return None
        return self._finish(st, s, "bia_step")

    def step_shard(self, state, cfg, shard, nshards, sums, q=None, stats=False):
        """Shard `shard` of `nshards` of one step (bia_step_shard): its pairs' sums into
        sums ((6, n) float64 CUDA tensor); the state is unchanged."""
        n = self._check_state(state)
        if sums.shape != (6, n) or not sums.is_contiguous():
            raise ValueError("sums must be a contiguous (6, n) float64 tensor")
        st_ = BiaStats()
        cur = self._enter()
        st = capi.lib().bia_step_shard(self._ctx, ctypes.byref(cfg), n, *self._ptrs(state), self._qptr(q, n),
                                       int(shard), int(nshards), ctypes.c_void_p(sums.data_ptr()),
                                       ctypes.byref(st_) if stats else None)
        self._leave(cur)
        if not stats:
            capi.check(st, "bia_step_shard")
            return None
        return self._finish(st, st_, "bia_step_shard")

    def apply_update(self, state, dt, sums):
        """Drift and update from the summed shard sums (bia_apply_update)."""
        n = self._check_state(state)
        cur = self._enter()
        st = capi.lib().bia_apply_update(self._ctx, n, float(dt), *self._ptrs(state),
                                         ctypes.c_void_p(sums.data_ptr()))
        self._leave(cur)
        capi.check(st, "bia_apply_update")

    def step_distributed(self, state, cfg, q=None, group=None):
        """One step of a system split over the ranks of a torch.distributed process group
        (NCCL over NVLink on GPUs): every rank holds the whole state, solves its shard of the
        pairs, the shard sums are all-reduced (6n FP64) and every rank applies the same
        update."""
        import torch.distributed as dist
        rank, world = dist.get_rank(group), dist.get_world_size(group)
        sums = self._torch.empty_like(state)
        self.step_shard(state, cfg, rank, world, sums, q=q)
        dist.all_reduce(sums, group=group)
        self.apply_update(state, cfg.dt, sums)

    def run(self, state, cfg, nsteps, q=None, graph=True, stats=True):
        """nsteps steps; the step sequence is captured once in a CUDA graph and replayed."""
        n = self._check_state(state)
        s = BiaStats()
        cur = self._enter()
        st = capi.lib().bia_run(self._ctx, ctypes.byref(cfg), n, *self._ptrs(state),
                                self._qptr(q, n), int(nsteps), int(bool(graph)),
                                ctypes.byref(s) if stats else None)
        self._leave(cur)
        if not stats:
            capi.check(st, "bia_run")
            return None
        return self._finish(st, s, "bia_run")

    def run_host(self, state, cfg, nsteps, q=None):
        """nsteps steps on a host (6, n) float64 numpy state, updated in place (the
        host-to-device and device-to-host copies are part of the call)."""
        if not (isinstance(state, np.ndarray) and state.dtype == np.float64 and
                state.flags.c_contiguous and state.ndim == 2 and state.shape[0] == 6):
            raise TypeError("state must be a C-contiguous (6, n) float64 numpy array")
        n = state.shape[1]
        base = state.ctypes.data
        ptrs = [ctypes.c_void_p(base + k * n * 8) for k in range(6)]
        qp = ctypes.c_void_p(None)
        if q is not None:
            q = np.ascontiguousarray(q, dtype=np.float64)
            qp = ctypes.c_void_p(q.ctypes.data)
        s = BiaStats()
        st = capi.lib().bia_run_host(self._ctx, ctypes.byref(cfg), n, *ptrs, qp, int(nsteps),
                                     ctypes.byref(s))
        return self._finish(st, s, "bia_run_host")

    def invariance(self, state, eps_th, q=None):
        """Invariants of the device state (FP64, fixed-order reductions)."""
        n = self._check_state(state)
        out = (ctypes.c_double * 11)()
        cur = self._enter()
        st = capi.lib().bia_invariance(self._ctx, n, float(eps_th), *self._ptrs(state),
                                       self._qptr(q, n), out)
        self._leave(cur)
        capi.check(st, "bia_invariance")
        return dict(zip(INVARIANT_NAMES, list(out)))

    def counters(self, reset=True):
        """Counters summed over every step run with stats=False since the last reset."""
        s = BiaStats()
        st = capi.lib().bia_context_stats(self._ctx, ctypes.byref(s), int(bool(reset)))
        return self._finish(st, s, "bia_context_stats")

    def dim_integrate(self, state, eps_th, x0, xe, relerr=0.0, abserr=1e-16):
        """Direct-integration reference solver (dim/rkf_kernel.cu) on the device state,
        advanced in place from x0 to xe.  eps_th is the per-particle coupling of
        dim/dim_3D.f90 (half the BIA pair coupling).  Returns the step counters."""
        n = self._check_state(state)
        st_ = capi.BiaDimStats()
        cur = self._enter()
        st = capi.lib().bia_dim_integrate(self._ctx, n, float(eps_th), ctypes.c_void_p(state.data_ptr()),
                                          float(x0), float(xe), float(relerr), float(abserr),
                                          ctypes.byref(st_))
        self._leave(cur)
        if st not in (BIA_OK, capi.BIA_ERR_NOT_CONVERGED):
            raise BiaError(st, "bia_dim_integrate")
        return st_.as_dict()

    def autotune(self, state, cfg, q=None):
        """Time the pair-kernel shapes of cfg's method on this state (unchanged) and keep
        the fastest for this size; returns (variant, {shape: ms})."""
        n = self._check_state(state)
        var = ctypes.c_int(-1)
        ms = (ctypes.c_float * 3)()
        cur = self._enter()
        st = capi.lib().bia_context_autotune(self._ctx, ctypes.byref(cfg), n, *self._ptrs(state),
                                             self._qptr(q, n), ctypes.byref(var), ms)
        self._leave(cur)
        capi.check(st, "bia_context_autotune")
        names = (("one_kernel", "split", "-") if cfg.method == capi.METHOD_LEARNED
                 else ("tiles8", "phase32_lane", "phase32"))
        return var.value, {names[k]: float(ms[k]) for k in range(3) if ms[k] >= 0}

    def set_shape(self, method, n, shape, deterministic=True):
        """Pin the pair-kernel shape of `method` (ALG: "tiles8", "phase32_lane", "phase32";
        learned: "one_kernel", "split"; None: the default rule) for sizes in n's
        floor(log2 n) bucket, as autotune would store it."""
        names = (("one_kernel", "split") if method == capi.METHOD_LEARNED
                 else ("tiles8", "phase32_lane", "phase32"))
        var = -1 if shape is None else names.index(shape)
        capi.check(capi.lib().bia_context_set_shape(self._ctx, int(method), int(bool(deterministic)), int(n), var),
                   "bia_context_set_shape")

    def load_heads(self, path=None):
        """Load the learned heads (learned_heads.bin) for METHOD_LEARNED steps."""
        blob = open(path or HEADS_PATH, "rb").read()
        capi.check(capi.lib().bia_context_set_heads(self._ctx, blob, len(blob)), "bia_context_set_heads")

    def head_eval(self, head, inputs, out):
        """Evaluate learned head `head` (0 elliptic, 1 hyperbolic) on the tensor cores:
        inputs (n, 2) float32 CUDA tensor -> out (n,) float32 CUDA tensor."""
        t = self._torch
        if inputs.dtype != t.float32 or out.dtype != t.float32 or not inputs.is_contiguous():
            raise ValueError("inputs and out must be contiguous float32 CUDA tensors")
        n = inputs.shape[0]
        if inputs.shape != (n, 2) or out.shape != (n,):
            raise ValueError("inputs must be (n, 2) and out (n,)")
        cur = self._enter()
        st = capi.lib().bia_learned_head_eval(self._ctx, int(head), int(n), ctypes.c_void_p(inputs.data_ptr()),
                                              ctypes.c_void_p(out.data_ptr()))
        self._leave(cur)
        capi.check(st, "bia_learned_head_eval")

    def trainer(self, head, nsamples=1 << 22, seed=0):
        """A device trainer of learned head `head` (0 elliptic, 1 hyperbolic) on this
        solver's device and stream (bia_trainer_*)."""
        return HeadTrainer(self, head, nsamples, seed)

    def ensemble(self, sizes, eps):
        """An ensemble of independent systems (sizes[s] particles, pair coupling eps[s])
        stored back to back; returns an Ensemble bound to this solver."""
        return Ensemble(self, sizes, eps)

    def set_timing(self, on):
        capi.check(capi.lib().bia_context_set_timing(self._ctx, int(bool(on))))

    def kernel_ms(self):
        """(summed duration in ms, launches) of the pair kernel since the last call."""
        ms = ctypes.c_double(0.0)
        cnt = ctypes.c_longlong(0)
        capi.check(capi.lib().bia_context_kernel_ms(self._ctx, ctypes.byref(ms), ctypes.byref(cnt)))
        return ms.value, cnt.value


class Ensemble:
    """Independent systems of uneven size advanced together (bia_ensemble_*).  The state
    is one (6, sum(sizes)) float64 CUDA tensor with the systems back to back."""

    def __init__(self, solver, sizes, eps):
        self.solver = solver
        self.sizes = np.ascontiguousarray(sizes, dtype=np.int32)
        self.eps = np.ascontiguousarray(eps, dtype=np.float64)
        if self.sizes.shape != self.eps.shape:
            raise ValueError("sizes and eps must have one entry per system")
        self.nsys = int(self.sizes.size)
        self.offsets = np.concatenate([[0], np.cumsum(self.sizes)])
        self._ens = ctypes.c_void_p()
        capi.check(capi.lib().bia_ensemble_create(
            solver._ctx, self.nsys, self.sizes.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
            self.eps.ctypes.data_as(_PD), ctypes.byref(self._ens)), "bia_ensemble_create")

    def close(self):
        if self._ens:
            capi.lib().bia_ensemble_destroy(self._ens)
            self._ens = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step_shard(self, state, cfg, shard, nshards, sums, q=None, stats=False):
        """Shard `shard` of `nshards` of one step (bia_step_shard): its pairs' sums into
        sums ((6, n) float64 CUDA tensor); the state is unchanged."""
        n = self._check_state(state)
        if sums.shape != (6, n) or not sums.is_contiguous():
            raise ValueError("sums must be a contiguous (6, n) float64 tensor")
        st_ = BiaStats()
        cur = self._enter()
        st = capi.lib().bia_step_shard(self._ctx, ctypes.byref(cfg), n, *self._ptrs(state), self._qptr(q, n),
                                       int(shard), int(nshards), ctypes.c_void_p(sums.data_ptr()),
                                       ctypes.byref(st_) if stats else None)
        self._leave(cur)
        if not stats:
            capi.check(st, "bia_step_shard")
            return None
        return self._finish(st, st_, "bia_step_shard")

    def apply_update(self, state, dt, sums):
        """Drift and update from the summed shard sums (bia_apply_update)."""
        n = self._check_state(state)
        cur = self._enter()
        st = capi.lib().bia_apply_update(self._ctx, n, float(dt), *self._ptrs(state),
                                         ctypes.c_void_p(sums.data_ptr()))
        self._leave(cur)
        capi.check(st, "bia_apply_update")

    def step_distributed(self, state, cfg, q=None, group=None):
        """One step of a system split over the ranks of a torch.distributed process group
        (NCCL over NVLink on GPUs): every rank holds the whole state, solves its shard of the
        pairs, the shard sums are all-reduced (6n FP64) and every rank applies the same
        update."""
        import torch.distributed as dist
        rank, world = dist.get_rank(group), dist.get_world_size(group)
        sums = self._torch.empty_like(state)
        self.step_shard(state, cfg, rank, world, sums, q=q)
        dist.all_reduce(sums, group=group)
        self.apply_update(state, cfg.dt, sums)

    def run(self, state, cfg, nsteps, q=None, graph=True, stats=True):
        s = self.solver
        n = s._check_state(state)
        if n != int(self.offsets[-1]):
            raise ValueError("state does not hold sum(sizes) particles")
        st_ = BiaStats()
        cur = s._enter()
        st = capi.lib().bia_ensemble_run(s._ctx, self._ens, ctypes.byref(cfg), *s._ptrs(state),
                                         s._qptr(q, n), int(nsteps), int(bool(graph)),
                                         ctypes.byref(st_) if stats else None)
        s._leave(cur)
        if not stats:
            capi.check(st, "bia_ensemble_run")
            return None
        return s._finish(st, st_, "bia_ensemble_run")

    SHAPES = {1: ("tiles8", "phase32_lane", "phase32"), 2: ("item_per_warp", "persistent"),
              3: ("head_1_cta_per_sm", "head_2_ctas_per_sm")}

    def autotune(self, state, cfg, q=None):
        """Time the launch shapes of cfg.method's pair kernels on these systems and keep the
        fastest (bia_ensemble_autotune); returns (shape name or None, {shape: ms})."""
        s = self.solver
        n = s._check_state(state)
        var = ctypes.c_int(-1)
        ms = (ctypes.c_float * 3)()
        cur = s._enter()
        st = capi.lib().bia_ensemble_autotune(s._ctx, self._ens, ctypes.byref(cfg), *s._ptrs(state),
                                              s._qptr(q, n), ctypes.byref(var), ms)
        s._leave(cur)
        capi.check(st, "bia_ensemble_autotune")
        names = self.SHAPES.get(cfg.method)
        if names is None:
            return None, {}
        return names[var.value], {names[k]: float(ms[k]) for k in range(len(names)) if ms[k] >= 0}

    def energy(self, state, q=None):
        """(KE, PE) arrays per system: KE = sum |v|^2, PE = eps_s sum_{i<j} (q_i q_j)/r_ij."""
        s = self.solver
        n = s._check_state(state)
        out = np.zeros(2 * self.nsys)
        cur = s._enter()
        st = capi.lib().bia_ensemble_energy(s._ctx, self._ens, *s._ptrs(state), s._qptr(q, n),
                                            out.ctypes.data_as(_PD))
        s._leave(cur)
        capi.check(st, "bia_ensemble_energy")
        return out[0::2].copy(), out[1::2].copy()


class HeadTrainer:
    """Training of one learned head on the GPU (bia_trainer_*): samples from the FP64 Kepler
    solver on the device, forward and backward passes on the tensor cores (BF16 operands,
    FP32 accumulation), Adam on FP32 master parameters."""

    def __init__(self, solver, head, nsamples, seed):
        self._solver = solver
        self._t = ctypes.c_void_p()
        cur = solver._enter()
        st = capi.lib().bia_trainer_create(solver._ctx, int(head), int(nsamples), int(seed), ctypes.byref(self._t))
        solver._leave(cur)
        capi.check(st, "bia_trainer_create")
        self.head = head
        self.nparams = capi.lib().bia_trainer_param_count()

    def close(self):
        if self._t:
            capi.lib().bia_trainer_destroy(self._t)
            self._t = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _fp(self, a):
        return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))

    def params(self):
        out = np.zeros(self.nparams, np.float32)
        capi.check(capi.lib().bia_trainer_get_params(self._t, self._fp(out)), "bia_trainer_get_params")
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        capi.check(capi.lib().bia_trainer_set_params(self._t, self._fp(p)), "bia_trainer_set_params")

    def samples(self):
        """(x, y, n): device pointers of the samples' inputs [n][2] and targets [n]."""
        x, y, n = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_longlong()
        capi.check(capi.lib().bia_trainer_samples(self._t, ctypes.byref(x), ctypes.byref(y), ctypes.byref(n)))
        return x.value, y.value, n.value

    def copy_samples(self, first, count):
        """Host copies (x float32[count][2], y float32[count]) of samples first .. + count."""
        x = np.zeros((count, 2), np.float32)
        y = np.zeros(count, np.float32)
        capi.check(capi.lib().bia_trainer_copy_samples(self._t, int(first), int(count), self._fp(x), self._fp(y)),
                   "bia_trainer_copy_samples")
        return x, y

    def gradient(self, x_ptr, y_ptr, rows):
        """Gradient of the mean squared error on device rows (pointers) at the current
        parameters: (grad float32[nparams], loss)."""
        g = np.zeros(self.nparams, np.float32)
        loss = ctypes.c_float(0.0)
        cur = self._solver._enter()
        st = capi.lib().bia_trainer_gradient(self._t, ctypes.c_void_p(x_ptr), ctypes.c_void_p(y_ptr), int(rows),
                                             self._fp(g), ctypes.byref(loss))
        self._solver._leave(cur)
        capi.check(st, "bia_trainer_gradient")
        return g, loss.value

    def train(self, epochs, batch=4096, lr=2e-3):
        """Adam over the samples; returns the mean squared error of each epoch."""
        losses = np.zeros(epochs, np.float32)
        cur = self._solver._enter()
        st = capi.lib().bia_trainer_train(self._t, int(epochs), int(batch), float(lr), self._fp(losses))
        self._solver._leave(cur)
        capi.check(st, "bia_trainer_train")
        return losses

    def export(self):
        """The head as a learned_heads.bin record (bytes)."""
        buf = ctypes.create_string_buffer(19472)
        capi.check(capi.lib().bia_trainer_export(self._t, buf), "bia_trainer_export")
        return buf.raw
