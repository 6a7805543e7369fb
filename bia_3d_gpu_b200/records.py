"""Fortran sequential-unformatted record I/O for the BIA state files.

The reference reads and writes its state with gfortran unformatted sequential
records: a 4-byte little-endian length, the payload, the same length again.
  *.bbb  one record per realisation: x,y,z,u,v,w per particle (AoS), written by
         IC/bbb_maker_REV.f90:71 and read by bia/bia.f90:64
  *.BIA  one record per realisation: t, then dX,dY,dZ,dU,dV,dW per particle
         (bia/bia.f90:206)
  *.DIM  one record per realisation: t, then the final state (dim/dim_3D.f90:32)
Arrays returned here are SoA numpy float64 of shape (6, n).
"""
import struct

import numpy as np


def read_records(path):
    """All records of a file as bytes objects; raises on malformed markers."""
    with open(path, "rb") as f:
        data = f.read()
    out, p = [], 0
    while p < len(data):
        if p + 4 > len(data):
            raise ValueError(f"{path}: truncated record marker at byte {p}")
        (n,) = struct.unpack("<i", data[p:p + 4])
        if n < 0 or p + 8 + n > len(data):
            raise ValueError(f"{path}: record length {n} at byte {p} runs past the end")
        (m,) = struct.unpack("<i", data[p + 4 + n:p + 8 + n])
        if m != n:
            raise ValueError(f"{path}: record markers differ ({n} != {m}) at byte {p}")
        out.append(data[p + 4:p + 4 + n])
        p += 8 + n
    return out


def write_record(f, payload):
    payload = bytes(payload)
    n = struct.pack("<i", len(payload))
    f.write(n)
    f.write(payload)
    f.write(n)


def aos_to_soa(a):
    a = np.asarray(a, dtype=np.float64)
    if a.size % 6:
        raise ValueError("AoS state length is not a multiple of 6")
    return np.ascontiguousarray(a.reshape(-1, 6).T)


def soa_to_aos(s):
    return np.ascontiguousarray(np.asarray(s, dtype=np.float64).T).reshape(-1)


def read_bbb(path):
    """List of (6, n) initial states, one per realisation."""
    return [aos_to_soa(np.frombuffer(r, "<f8")) for r in read_records(path)]


def read_timed(path):
    """List of (t, (6, n) array) for .BIA / .DIM files."""
    out = []
    for r in read_records(path):
        a = np.frombuffer(r, "<f8")
        out.append((float(a[0]), aos_to_soa(a[1:])))
    return out


def write_bbb(path, states):
    with open(path, "wb") as f:
        for s in states:
            write_record(f, soa_to_aos(s).astype("<f8").tobytes())


def write_timed(path, items):
    with open(path, "wb") as f:
        for t, s in items:
            write_record(f, np.concatenate([[t], soa_to_aos(s)]).astype("<f8").tobytes())
