"""bench.py host logic: the workload variants and the algorithmic-bytes model
behind the roofline fractions."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
from fdtd_b200 import problem as P  # noqa: E402


def test_variants_change_only_what_they_name():
    base = bench.make_problem("drude384", 10, 64)
    pec = bench.make_problem("drude384", 10, 64, "pec_backed")
    assert pec.boundaries == {(a, s): "pec" for a in range(3) for s in (0, 1)}
    assert pec.pml == base.pml and pec.dt == base.dt
    sd = bench.make_problem("drude384", 10, 64, "surface_dft")
    for r0, r1 in zip(base.dfts, sd.dfts):
        assert r1.comp == (r0.comp + 9 if r0.comp < 3 else r0.comp + 3)
        assert P.quantity_in_mode(sd.mode, r1.comp)
        assert all(1 <= lo and hi <= n - 2 for lo, hi, n in zip(r1.lo, r1.hi, sd.shape))
    b3 = bench.make_problem("drude384", 10, 64, "bd3")
    assert b3.time_scheme == 1 and b3.dt == base.dt  # the FP32 leg keeps the leapfrog
    b3p = bench.make_problem("drude384", 10, 64, "bd3", fp64=True)
    assert b3p.time_scheme == 3 and b3p.dt == pytest.approx(base.dt * 0.5 / 0.99)


def test_plain_bytes_count_the_flux_history():
    p1 = bench.make_problem("drude384", 10, 32, fp64=True)
    p3 = bench.make_problem("drude384", 10, 32, "bd3", fp64=True)
    p4 = bench.make_problem("drude384", 10, 32, "bd4", fp64=True)
    a1, a3, a4 = (bench.alg_bytes(p, 8) for p in (p1, p3, p4))
    cells = p1.interior_cells
    # 3 flux components, 2 (BD3) or 3 (BD4) past values, read and written
    assert a3["e_sweep"] - a1["e_sweep"] == pytest.approx(cells * 8 * 3 * 4)
    assert a4["h_sweep"] - a1["h_sweep"] == pytest.approx(cells * 8 * 3 * 6)
    # FP32 bytes ignore the scheme (the fused method is leapfrog only)
    assert bench.alg_bytes(p1, 4) == bench.alg_bytes(bench.make_problem("drude384", 10, 32), 4)


def test_reference_arm_copies_run_at_once():
    """The reference arm's sample runs as concurrent single-thread copies:
    the reported cores are the copies, the rate their combined cell-updates."""
    one = bench.cpu_baseline("drude384", budget_s=0.3)
    two = bench.cpu_baseline("drude384", budget_s=0.3, replicas=2)
    assert one["cores"] == 1 and two["cores"] == 2
    assert two["kind"] == one["kind"] and two["value"] > 0
    assert "2 copies at once" in two["sample"]
