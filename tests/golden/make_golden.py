"""Convert the reference's committed output files into the test fixture
``tests/golden/ref_0001332.npz``.

Run once in a checkout that has the reference next to it:

    python tests/golden/make_golden.py /path/to/bia_3d_gpu

Sources (all under the reference's ``OUT/``):
  0001332_10^0.bbb   IC record, 1332 particles, AoS x,y,z,u,v,w (bbb_maker output)
  0001332_10^0.BIA   record (t, dX,dY,dZ,dU,dV,dW per particle) from bia.f90:206,
                     ALG method, GPU platform (the defaults at bia/bia.f90:5,7),
                     eps_th = -6e-7, time_end = 1, ITR = 18
  0001332_10^0.DIM   record (t, final state) from dim/dim_3D.f90:32, eps_th = -3e-7
  BIA_10^0.0001332   text: t and the final state of particle 1 (bia/bia.f90:207)
  DIM_10^0.0001332   text: the same from DIM (dim/dim_3D.f90:31)
  0001332.DIM        text: DIM's adaptive-step trajectory of particle 1
                     (dim/rkf_kernel.cu:207-219,375-383)

All three binary files are Fortran sequential-unformatted: a 4-byte record
length before and after each record.
"""
import os
import struct
import sys

import numpy as np


def fortran_records(path):
    data = open(path, "rb").read()
    out, p = [], 0
    while p < len(data):
        (n,) = struct.unpack("<i", data[p:p + 4])
        body = data[p + 4:p + 4 + n]
        (m,) = struct.unpack("<i", data[p + 4 + n:p + 8 + n])
        if n != m:
            raise ValueError(f"{path}: record markers differ ({n} != {m})")
        out.append(body)
        p += 8 + n
    return out


def main(ref_root):
    out_dir = os.path.join(ref_root, "OUT")
    ic = np.frombuffer(fortran_records(os.path.join(out_dir, "0001332_10^0.bbb"))[0], "<f8")
    bia = np.frombuffer(fortran_records(os.path.join(out_dir, "0001332_10^0.BIA"))[0], "<f8")
    dim = np.frombuffer(fortran_records(os.path.join(out_dir, "0001332_10^0.DIM"))[0], "<f8")
    bia_txt = np.loadtxt(os.path.join(out_dir, "BIA_10^0.0001332"))
    dim_txt = np.loadtxt(os.path.join(out_dir, "DIM_10^0.0001332"))
    traj = np.loadtxt(os.path.join(out_dir, "0001332.DIM"), skiprows=1)
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_0001332.npz")
    np.savez_compressed(dst, ic_aos=ic, bia_t=bia[0], bia_disp_aos=bia[1:], dim_t=dim[0],
                        dim_final_aos=dim[1:], bia_p1=bia_txt, dim_p1=dim_txt,
                        dim_p1_traj=traj, eps_bia=-6e-7, eps_dim=-3e-7, time_end=1.0, itr=18)
    print("wrote", dst, "n =", ic.size // 6)


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("BIA_REFERENCE_DIR")
    if not root:
        sys.exit("usage: make_golden.py <reference checkout> (or set BIA_REFERENCE_DIR)")
    main(root)
