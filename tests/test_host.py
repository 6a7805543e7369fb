"""Host-side logic on the CPU: record I/O, initial conditions, the C-ABI symbol table."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from bia_3d_gpu_b200 import capi, initial, records
from conftest import ROOT


def test_record_roundtrip(tmp_path):
    rng = np.random.default_rng(0)
    states = [rng.standard_normal((6, 10)), rng.standard_normal((6, 10))]
    p = tmp_path / "x.bbb"
    records.write_bbb(p, states)
    back = records.read_bbb(p)
    assert len(back) == 2 and all(np.array_equal(a, b) for a, b in zip(states, back))
    q = tmp_path / "x.BIA"
    records.write_timed(q, [(1.0, states[0])])
    (t, s), = records.read_timed(q)
    assert t == 1.0 and np.array_equal(s, states[0])


def test_reads_reference_layout(golden):
    """The fixture arrays are the payload of the reference's records."""
    ic = golden["ic_aos"]
    s = records.aos_to_soa(ic)
    assert s.shape == (6, 1332)
    assert np.array_equal(s[:, 0], np.zeros(6))  # particle 1 at rest at the origin
    assert np.array_equal(records.soa_to_aos(s), ic)


@pytest.mark.parametrize("damage", ["truncated", "mismatch", "negative"])
def test_malformed_records_raise(tmp_path, damage):
    p = tmp_path / "bad.bbb"
    body = np.arange(12, dtype="<f8").tobytes()
    if damage == "truncated":
        data = (len(body)).to_bytes(4, "little", signed=True) + body[:40]
    elif damage == "mismatch":
        data = (len(body)).to_bytes(4, "little") + body + (len(body) - 8).to_bytes(4, "little")
    else:
        data = (-8).to_bytes(4, "little", signed=True) + body
    p.write_bytes(data)
    with pytest.raises(ValueError):
        records.read_records(p)


def test_initial_conditions_shapes_and_seeds():
    s1, eps1 = initial.gravity_ball(200, seed=7)
    s2, _ = initial.gravity_ball(200, seed=7)
    assert s1.shape == (6, 200) and np.array_equal(s1, s2) and eps1 == -2.0 / 200
    assert np.linalg.norm(s1[:3], axis=0).max() <= 1.0
    s, eps, q = initial.coulomb_cube(512, seed=3, dmin=1e-2)
    assert eps == 2.0 and q.sum() == 0 and set(np.unique(q)) == {-1.0, 1.0}
    assert s[:3].min() >= 0 and s[:3].max() <= 1
    from scipy.spatial.distance import pdist
    assert pdist(s[:3].T).min() >= 1e-2
    sp, epsp = initial.plummer(4096, seed=1)
    assert np.abs(sp[:3].mean(axis=1)).max() < 1e-12 and np.abs(sp[3:].mean(axis=1)).max() < 1e-12
    # half-mass radius of a Plummer sphere with a = 1 is ~1.305
    rh = np.median(np.linalg.norm(sp[:3], axis=0))
    assert 1.15 < rh < 1.45
    sc, _ = initial.cold_ball(100)
    assert np.all(sc[3:] == 0)


def test_lattice_layout():
    s, _ = initial.lattice(NL=2, seed=1)
    n = 5 ** 3 + 1
    assert s.shape == (6, n)
    assert np.all(s[:, 0] == 0)
    # every particle sits within 1/2 of an integer lattice point in [-2, 2]^3
    off = s[:3, 1:] - np.round(s[:3, 1:])
    assert np.abs(off).max() <= 0.5 and np.abs(np.round(s[:3, 1:])).max() <= 2
    # shell order: the first 27 (after the origin block) are the |cell|_inf <= 1 cells
    cells = np.abs(np.round(s[:3, 2:])).max(axis=0)
    assert np.all(np.diff(cells) >= 0)


def _declared_functions():
    text = open(os.path.join(ROOT, "include", "bia_capi.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?(?:void|int|char)\s*\*?\s*(\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    """libbia_b200.so loads on a CPU-only machine and exports every function that
    include/bia_capi.h declares (no compute call is made)."""
    declared = _declared_functions()
    assert "find_dxyuv_kernel_" in declared and "invariance_gpu_" in declared
    L = capi.lib()
    for name in declared:
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", capi.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert set(declared) <= exported
    assert set(capi.EXPORTED_SYMBOLS) <= exported


def test_config_defaults_are_the_references():
    cfg = capi.default_config()
    assert cfg.method == capi.METHOD_ALG and cfg.itr == 18
    assert cfg.eps_th == -6e-7 and cfg.dt == 1.0 and cfg.err == 1e-12
    assert cfg.rkf_relerr == 0.0 and cfg.rkf_abserr == 1e-16 and cfg.deterministic == 1
    for st in range(8):
        assert capi.status_string(st)


def test_context_without_device_reports_no_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    ctx = ctypes.c_void_p()
    st = capi.lib().bia_context_create(ctypes.byref(ctx), 0, None)
    assert st == capi.BIA_ERR_NO_DEVICE and not ctx.value


def test_bench_reference_arm_prints_the_contract_line():
    """`bench.py --impl reference` (the reference's CPU ALG path, restated in C, on the
    host cores) prints one JSON line with the contract's keys, on the same metric and
    workload as the default line; it needs no GPU."""
    import json
    import os
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference",
                          "--steps", "1", "--warmup", "0"], capture_output=True, text=True,
                         check=True, cwd=root, timeout=600).stdout
    lines = [l for l in out.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "pair-updates/s" and d["value"] > 0
    assert d["metric"].startswith("BIA pair-updates/s: learned-guess form vs plain FP64")
    assert d["config"]["workload"] == "plummer_32768" and d["higher_is_better"] is True
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]


def test_fortran_text_line_format():
    """driver.fortran_line writes bia/bia.f90:207's '(es23.16,6es24.16)': widths 23 and 24,
    16 digits after the point, a two-digit exponent; the values read back exactly."""
    from bia_3d_gpu_b200.driver import fortran_line
    vals = [-1.2345678901234567e-3, 2.0, 0.0, 3.141592653589793e7, -4.5e-10, 1e-5]
    line = fortran_line(1.0, vals)
    assert len(line) == 23 + 6 * 24
    assert line[:23] == " 1.0000000000000000E+00"
    back = [float(line[23 + 24 * k:23 + 24 * (k + 1)]) for k in range(6)]
    assert back == vals
    assert "-1.2345678901234567E-03" in line
