"""The C++ drop-in layer (include/fdtd_b200.hpp): tests/cpp/drop_in.cpp writes
the reference's time loop with the reference's functor names, runs it on the
GPU, and its fields are compared with the CPU oracle on the same problem."""
import math
import os
import subprocess

import numpy as np
import pytest

import scenarios
from helpers import rel_l2

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def drop_in(fdtd, tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("cpp") / "drop_in")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "drop_in.cpp"), "-L" + os.path.dirname(fdtd.LIB_PATH),
                    "-lfdtd_b200", "-Wl,-rpath," + os.path.dirname(fdtd.LIB_PATH), "-o", exe], check=True)
    return exe


def run(exe, which, tmp_path, nfields, shape):
    out = str(tmp_path / f"{which}.bin")
    subprocess.run([exe, which, out], check=True)
    return np.fromfile(out, dtype=np.float64).reshape(nfields, *shape)


def test_tm_plain_through_templates(drop_in, oracle, tmp_path):
    from fdtd_b200.problem import TM, Problem, Source, courant_dt
    p = Problem(TM, (40, 36, 1), 1e-6, courant_dt(1e-6, 0.99 / math.sqrt(2.0)))
    for a in (0, 1):
        for s in (0, 1):
            p.pml[(a, s)] = 6
    n = np.arange(80, dtype=np.float64)
    p.sources.append(Source(2, (20, 18, 0), np.exp(-(((n - 20.0) / 6.0) ** 2)), "E"))
    o = oracle.run_oracle(p, 80)
    got = run(drop_in, "tm", tmp_path, 3, (1, 36, 40))
    for q, name in enumerate(["Ez", "Hx", "Hy"]):
        assert rel_l2(got[q], o.get(name)) <= 1e-12, name


def test_forward_material_updates_through_templates(drop_in, oracle, tmp_path):
    """grid.apply_forward_materials(FieldType::Electric / Magnetic) after the
    tm loop: D and B from the fields, as the oracle's forward updates (which
    reproduce the reference's XUpdate<Mode, ft, true>) give them (FP64,
    <= 1e-12; the loop's source values come from the C++ signal)."""
    from fdtd_b200.problem import TM, Problem, Source, courant_dt
    p = Problem(TM, (40, 36, 1), 1e-6, courant_dt(1e-6, 0.99 / math.sqrt(2.0)))
    for a in (0, 1):
        for s in (0, 1):
            p.pml[(a, s)] = 6
    n = np.arange(80, dtype=np.float64)
    p.sources.append(Source(2, (20, 18, 0), np.exp(-(((n - 20.0) / 6.0) ** 2)), "E"))
    o = oracle.run_oracle(p, 80)
    o.material_explicit(0)
    o.material_explicit(1)
    got = run(drop_in, "fw", tmp_path, 3, (1, 36, 40))
    for q, name in enumerate(["Dz", "Bx", "By"]):
        ref = o.get(name)
        assert np.any(ref), name
        assert rel_l2(got[q], ref) <= 1e-12, name


def test_tm_custom_cpml_model_through_templates(drop_in, oracle, tmp_path):
    """grid.set_pml(d, o, n, PMLParameterModel(m, ma, sMax, kMax, aMax)):
    the user's grading reaches the GPU profiles (FP64 <= 1e-12)."""
    from fdtd_b200.problem import IMP0, TM, Problem, Source, courant_dt
    p = Problem(TM, (40, 36, 1), 1e-6, courant_dt(1e-6, 0.99 / math.sqrt(2.0)))
    for a in (0, 1):
        for s in (0, 1):
            p.pml[(a, s)] = 6
    s0 = 0.8 * 4 / (IMP0 * 1e-6)
    p.pml_models[(0, 0)] = (4.0, 2.0, 1.3 * s0, 8.0, 0.1)
    p.pml_models[(1, 1)] = (3.5, 1.5, 2.0 * s0, 3.0, 0.2)
    n = np.arange(80, dtype=np.float64)
    p.sources.append(Source(2, (20, 18, 0), np.exp(-(((n - 20.0) / 6.0) ** 2)), "E"))
    o = oracle.run_oracle(p, 80)
    got = run(drop_in, "pm", tmp_path, 3, (1, 36, 40))
    for q, name in enumerate(["Ez", "Hx", "Hy"]):
        assert rel_l2(got[q], o.get(name)) <= 1e-12, name
    # and the grading is not the default one
    p.pml_models = {}
    assert rel_l2(got[0], oracle.run_oracle(p, 80).get("Ez")) > 1e-9


def test_3d_fused_material_map_tfsf_through_templates(drop_in, oracle, tmp_path):
    p = scenarios.td_tfsf_box()
    o = oracle.run_oracle(p)
    got = run(drop_in, "td", tmp_path, 6, (24, 24, 24))
    for q, name in enumerate(["Ex", "Ey", "Ez", "Hx", "Hy", "Hz"]):
        assert rel_l2(got[q], o.get(name)) <= 1e-4, name


def test_tm_bd3_boundaries_through_templates(drop_in, oracle, tmp_path):
    """YeeUpdate<TM, F, BD3> and make_pec/periodic_boundary through the C++
    layer equal the oracle's BD3 step with the same faces."""
    from fdtd_b200.problem import TM, Problem, Source, courant_dt
    p = Problem(TM, (36, 30, 1), 1e-6, courant_dt(1e-6, 0.5 / math.sqrt(2.0)))
    p.pml[(0, 1)] = 6
    p.boundaries = {(0, 0): "pec", (1, 0): "periodic", (1, 1): "periodic"}
    p.time_scheme = 3
    n = np.arange(90, dtype=np.float64)
    p.sources.append(Source(2, (10, 8, 0), np.exp(-(((n - 20.0) / 6.0) ** 2)), "E"))
    from fdtd_b200.problem import DFTRegion
    p.dfts.append(DFTRegion(8, (2, 2, 0), (33, 27, 0), [0.03, 0.05]))
    o = oracle.run_oracle(p, 90)
    out = str(tmp_path / "bd.bin")
    subprocess.run([drop_in, "bd", out], check=True)
    raw = np.fromfile(out, dtype=np.float64)
    n = 30 * 36
    for q, name in enumerate(["Ez", "Hx", "Hy"]):
        assert rel_l2(raw[q * n:(q + 1) * n].reshape(1, 30, 36), o.get(name)) <= 1e-12, name
    jh = raw[3 * n:3 * n + 34 * 28]
    assert rel_l2(jh, o.read_quantity(9, (1, 1, 0), (34, 28, 0)).ravel()) <= 1e-12
    spec = raw[3 * n + 34 * 28:]
    ref = o.dft(0).ravel()
    got = spec[0::2] + 1j * spec[1::2]
    assert rel_l2(got, ref) <= 1e-12
