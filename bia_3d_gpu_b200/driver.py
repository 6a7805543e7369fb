"""The reference's two programs, run on this library.

    python -m bia_3d_gpu_b200.driver bia OUT/0001332_10^0.bbb OUT/0001332_10^0.BIA OUT/BIA_10^0.0001332
    python -m bia_3d_gpu_b200.driver dim OUT/0001332_10^0.bbb OUT/0001332_10^0.DIM OUT/DIM_10^0.0001332

run_bia follows bia/bia.f90: for every realisation of the .bbb file (one unformatted record
of x, y, z, u, v, w per particle, :64) one BIA step of length time_end (the GPU branch of
:126-204, here the whole step on the device), then one .BIA record of time_end and
dX, dY, dZ, dU, dV, dW per particle (:206) and particle 1's final state as a text line
(:207, format es23.16, 6es24.16).  The invariants of the first realisation before the
step (:67-68) are returned with the stats.

run_dim follows dim/dim_3D.f90: for every realisation, N_time calls of the direct-
integration solver rkf_c_ from 0 to time_end (INIT = 1 on the first call, then the solver's
own step size carries over), particle 1's line after each call (:31) and one .DIM record of
time_end and the final state (:32).
"""
import argparse
import os

import numpy as np

from . import records


def fortran_line(t, values):
    """Fortran '(es23.16,6es24.16)' of t and the six values (exponent with two digits,
    as gfortran writes it for |exponent| < 100)."""
    def es(x, w):
        s = format(float(x), f".16E")
        mant, exp = s.split("E")
        e = int(exp)
        s = f"{mant}E{'+' if e >= 0 else '-'}{abs(e):02d}"
        return s.rjust(w)
    return es(t, 23) + "".join(es(v, 24) for v in values)


def run_bia(bbb_path, bia_path, text_path, eps_th=-6e-7, time_end=1.0, method=1, itr=18, device=0,
            heads=None):
    """bia/bia.f90 on the GPU.  Returns (per-realisation step stats, invariants of the first
    realisation before its step)."""
    import torch

    from . import BIASolver, default_config
    states = records.read_bbb(bbb_path)
    cfg = default_config(eps_th=eps_th, dt=time_end, method=method, itr=itr)
    out_stats = []
    inv0 = None
    with open(bia_path, "wb") as fb, open(text_path, "w") as ft, BIASolver(device=device) as solver:
        if method == 3:
            solver.load_heads(heads)
        for k, s in enumerate(states):
            t = torch.tensor(s, device=solver.device)
            if k == 0:
                inv0 = solver.invariance(t, eps_th)
            d = torch.zeros_like(t)
            st = solver.step(t, cfg, disp=d)
            solver.stream.synchronize()
            disp = d.cpu().numpy()
            new = t.cpu().numpy()
            records.write_record(fb, np.concatenate([[time_end], records.soa_to_aos(disp)]).astype("<f8").tobytes())
            ft.write(fortran_line(time_end, new[:, 0]) + "\n")
            out_stats.append(st)
    return out_stats, inv0


def run_dim(bbb_path, dim_path, text_path, eps_th=-3e-7, time_end=1.0, n_time=1, relerr=0.0, abserr=1e-16):
    """dim/dim_3D.f90 with the rkf_c_ drop-in.  Returns per-realisation (IER, NDE)."""
    from . import rkf_c
    states = records.read_bbb(bbb_path)
    th = time_end / n_time
    out = []
    with open(dim_path, "wb") as fd, open(text_path, "w") as ft:
        for s in states:
            y = records.soa_to_aos(s).copy()
            x0, init, h = 0.0, 1, 0.0
            res = None
            for i in range(1, n_time + 1):
                xe = th * i
                res = rkf_c(y.size, eps_th, x0, xe, y, init, relerr, abserr, H=h)
                x0, init, h = res["X0"], res["INIT"], res["H"]
                y = res["YHN"].copy()
                ft.write(fortran_line(xe, y[:6]) + "\n")
            records.write_record(fd, np.concatenate([[th * n_time], y]).astype("<f8").tobytes())
            out.append((res["IER"], res["NDE"]))
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("program", choices=("bia", "dim"))
    ap.add_argument("bbb")
    ap.add_argument("out")
    ap.add_argument("text")
    ap.add_argument("--eps-th", type=float, default=None)
    ap.add_argument("--time-end", type=float, default=1.0)
    ap.add_argument("--method", choices=("alg", "rkf", "universal", "learned"), default="alg")
    a = ap.parse_args(argv)
    if a.program == "bia":
        m = {"rkf": 0, "alg": 1, "universal": 2, "learned": 3}[a.method]
        st, _ = run_bia(a.bbb, a.out, a.text, eps_th=-6e-7 if a.eps_th is None else a.eps_th,
                        time_end=a.time_end, method=m)
        print(f"{len(st)} realisation(s) -> {os.path.basename(a.out)}")
    else:
        r = run_dim(a.bbb, a.out, a.text, eps_th=-3e-7 if a.eps_th is None else a.eps_th, time_end=a.time_end)
        print(f"{len(r)} realisation(s) -> {os.path.basename(a.out)}, IER/NDE {r}")


if __name__ == "__main__":
    main()
