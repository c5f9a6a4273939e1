"""The CPU oracle (oracle/fdtd_oracle.c) against the reference.

* golden fixtures (tests/golden/*.npz, produced from the reference's own
  functors by tests/golden/make_golden.py) must be reproduced bit for bit;
* where the reference runner can be built (the reference tree is present),
  the oracle must match it bit for bit on the same scenarios live;
* known-answer checks for the parts the reference does not implement (the
  DFT capture, multi-pole Lorentz) and the constants the reference pins
  (tests/testConstants.cpp prints them).
"""
import copy
import math
import os

import numpy as np
import pytest

import pyoracle

import scenarios
from helpers import rel_l2

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("make", scenarios.REFERENCE_SCENARIOS, ids=lambda f: f.__name__)
def test_oracle_matches_golden_bitwise(oracle, make):
    p = make()
    gold = np.load(os.path.join(GOLDEN, p.name + ".npz"))
    assert int(gold["steps"]) == p.steps
    g = oracle.run_oracle(p)
    names = [n for n in gold.files if n != "steps"]
    assert len(names) >= 6
    for n in names:
        got = g.get(n)
        assert np.array_equal(got, gold[n]), f"{p.name}:{n} differs (rel {rel_l2(got, gold[n]):.2e})"
    # every field the fixture omits is identically zero in the oracle too
    for n in oracle.NAMES + oracle.PSI_NAMES:
        if n not in names:
            assert not np.any(g.get(n)), f"{p.name}:{n} should be zero"


@pytest.mark.skipif(not pyoracle.reference_tree_present(), reason="reference tree not present")
def test_oracle_matches_reference_runner_live(oracle):
    import subprocess
    subprocess.run(["make", "-s", "-C", os.path.dirname(oracle.__file__), "_ref/ref_runner"], check=True)
    for make in scenarios.REFERENCE_SCENARIOS:
        p = make()
        p.steps = p.steps // 2 + 3  # a different step count than the fixtures
        ref = oracle.run_reference(p)
        g = oracle.run_oracle(p)
        for n in oracle.ALL_NAMES:
            assert np.array_equal(g.get(n), ref[n]), f"{p.name}:{n}"


@pytest.mark.parametrize("make", scenarios.FORWARD_SCENARIOS, ids=lambda f: f.__name__)
def test_forward_material_updates_match_golden(oracle, make):
    """The steps, then the forward (explicit) material updates of E and of H:
    bit for bit the reference's XUpdate<Mode, ft, true> (<name>_fwd.npz)."""
    p = scenarios.forward_materials(make)
    gold = np.load(os.path.join(GOLDEN, p.name + ".npz"))
    g = oracle.run_oracle(p)
    g.material_explicit(0)
    g.material_explicit(1)
    for n in oracle.NAMES + oracle.PSI_NAMES:
        want = gold[n] if n in gold.files else np.zeros_like(g.get(n))
        assert np.array_equal(g.get(n), want), f"{p.name}:{n}"


def test_forward_lorentz_update_is_refused(oracle):
    g = oracle.run_oracle(scenarios.td_drude_lorentz(), 2)
    with pytest.raises(ValueError):
        g.material_explicit(0)
    g.material_explicit(1)  # the magnetic side has no Lorentz material


@pytest.mark.skipif(not pyoracle.reference_tree_present(), reason="reference tree not present")
def test_forward_material_updates_match_reference_runner_live(oracle):
    for make in scenarios.FORWARD_SCENARIOS:
        p = scenarios.forward_materials(make)
        p.steps = p.steps // 2 + 5
        ref = oracle.run_reference(p, explicit=True)
        g = oracle.run_oracle(p)
        g.material_explicit(0)
        g.material_explicit(1)
        for n in oracle.NAMES + oracle.PSI_NAMES:
            assert np.array_equal(g.get(n), ref[n]), f"{p.name}:{n}"


def test_constants_match_reference():
    from fdtd_b200 import problem as P
    assert P.EPS0 == 8.854e-12
    assert P.MU0 == 3.14159265358979323846264338327950288 * 4.0e-7
    assert P.C0 == 2.99792458e8
    # imp0 uses the reference's Newton sqrt; it agrees with sqrt to an ulp
    assert abs(P.IMP0 - math.sqrt(P.MU0 / P.EPS0)) <= 1e-13 * P.IMP0


def test_levi_civita_and_offsets_pinned():
    """Facts tests/testConstants.cpp prints (FDTDConstants.hpp:602-637, :680-744)."""
    from fdtd_b200.problem import TM
    # the oracle's curl signs are exercised by the golden tests; check the
    # staggering convention the TFSF helper relies on: E at -0.5 off-axis,
    # H at -0.5 on-axis
    import fdtd_b200.problem as P
    planes = P.tfsf_box_planes(TM, (10, 12), (20, 22))
    assert [(q.axis, q.orient, q.lo, q.hi) for q in planes] == [
        (0, 0, (9, 12, 0), (9, 22, 0)), (0, 1, (20, 12, 0), (20, 22, 0)),
        (1, 0, (10, 11, 0), (20, 11, 0)), (1, 1, (10, 22, 0), (20, 22, 0))]


def test_dft_known_answer(oracle):
    """A soft source drives Ez at a cell whose neighbours see nothing yet on
    step 1: the DFT of Ez at the source cell over one step is known."""
    from fdtd_b200.problem import TM, Problem, Source, DFTRegion
    p = Problem(TM, (9, 9, 1), 1e-6, 1e-15)
    v = np.array([0.7])
    p.sources.append(Source(2, (4, 4, 0), v, "E"))
    f = 0.125
    p.dfts.append(DFTRegion(2, (4, 4, 0), (4, 4, 0), [f]))
    g = oracle.run_oracle(p, 1)
    X = g.dft(0)[0, 0]
    assert abs(X - 0.7 * np.exp(-2j * np.pi * f * 1.0)) < 1e-15


def test_dft_of_sinusoid(oracle):
    """A sinusoidal E source sampled over N steps: the running DFT at its
    frequency equals the direct sum of the recorded samples."""
    from fdtd_b200.problem import TM, Problem, Source, DFTRegion, courant_dt
    n = 31
    dt = courant_dt(1e-6, 0.99 / math.sqrt(2))
    p = Problem(TM, (n, n, 1), 1e-6, dt)
    for a in (0, 1):
        for s in (0, 1):
            p.pml[(a, s)] = 5
    steps = 120
    f0 = 0.05
    vals = np.sin(2 * np.pi * f0 * np.arange(steps)) * np.tanh(np.arange(steps) / 20)
    p.sources.append(Source(2, (15, 15, 0), vals, "E"))
    p.dfts.append(DFTRegion(2, (13, 15, 0), (17, 15, 0), [f0, 2 * f0]))
    g = oracle.OracleGrid(p)
    samples = []
    for t in range(steps):
        g.step(1)
        samples.append(g.get("Ez")[0, 15, 13:18].copy())
    samples = np.array(samples)
    nvec = np.arange(1, steps + 1)
    for q, f in enumerate([f0, 2 * f0]):
        direct = (samples * np.exp(-2j * np.pi * f * nvec)[:, None]).sum(0)
        assert rel_l2(g.dft(0)[q], direct) < 1e-13


def test_lorentz_two_pole_reduces_to_reference(oracle):
    """The multi-pole Lorentz update at one pole with delta_eps = 1 is the
    reference's LorentzUpdate: a second pole of zero strength and zero
    frequency leaves the fields bit-identical."""
    from fdtd_b200.problem import Material
    p1 = scenarios.te_materials()
    p2 = scenarios.te_materials()
    m = p2.materials[3]
    p2.materials[3] = Material.lorentz(m.eps_inf, [m.poles[0], (0.0, 0.0, 0.0)])
    g1 = oracle.run_oracle(p1)
    g2 = oracle.run_oracle(p2)
    for n in ["Ex", "Ey", "Hz", "Px", "Jx"]:
        assert np.array_equal(g1.get(n), g2.get(n))


def test_tfsf_confines_the_incident_wave(oracle):
    """With the consistent H polarisation and tfsf_box_planes, the scattered
    field region stays empty in vacuum (leakage at round-off level)."""
    from fdtd_b200.problem import TM, TFSF, Problem, courant_dt, gaussian_pulse, tfsf_box_planes
    n = 70
    p = Problem(TM, (n, n, 1), 1e-6, courant_dt(1e-6, 0.99 / math.sqrt(2)))
    for a in (0, 1):
        for s in (0, 1):
            p.pml[(a, s)] = 8
    lo, hi = 22, 47
    p.tfsf = TFSF(aux_ncells=n, aux_values=gaussian_pulse(160, 40, 10, offset=1.0), origin=(n / 2, n / 2, 0),
                  k=(1.0, 0.0, 0.0), pol_e=(0, 0, 1), pol_h=(0, 1, 0), planes=tfsf_box_planes(TM, (lo, lo), (hi, hi)))
    g = oracle.OracleGrid(p)
    inside = outside = 0.0
    for _ in range(4):
        g.step(40)
        ez = g.get("Ez")[0]
        mask = np.ones_like(ez, bool)
        mask[lo - 1:hi + 2, lo - 1:hi + 2] = False
        inside = max(inside, np.abs(ez[lo:hi + 1, lo:hi + 1]).max())
        outside = max(outside, np.abs(ez[mask]).max())
    assert inside > 1e-3
    assert outside < 1e-12 * inside


def test_reference_tm_polarisation_leaks(oracle):
    """The reference's default TM H polarisation (ky, -kx, 0)
    (include/Source.hpp:577-579) injects H with the opposite sign to the aux
    grid's Hy, so the box does not confine the wave. Pinned as a finding."""
    from fdtd_b200.problem import TM, TFSF, Problem, courant_dt, gaussian_pulse, tfsf_box_planes, ref_tm_polarisation
    n = 70
    p = Problem(TM, (n, n, 1), 1e-6, courant_dt(1e-6, 0.99 / math.sqrt(2)))
    for a in (0, 1):
        for s in (0, 1):
            p.pml[(a, s)] = 8
    lo, hi = 22, 47
    pe, ph = ref_tm_polarisation((1.0, 0.0, 0.0))
    p.tfsf = TFSF(aux_ncells=n, aux_values=gaussian_pulse(160, 40, 10, offset=1.0), origin=(n / 2, n / 2, 0),
                  k=(1.0, 0.0, 0.0), pol_e=pe, pol_h=ph, planes=tfsf_box_planes(TM, (lo, lo), (hi, hi)))
    g = oracle.run_oracle(p, 120)
    ez = g.get("Ez")[0]
    mask = np.ones_like(ez, bool)
    mask[lo - 1:hi + 2, lo - 1:hi + 2] = False
    assert np.abs(ez[mask]).max() > 0.1 * np.abs(ez).max()


def test_eps_map_equals_per_cell_constant_materials(oracle):
    """oracle_set_eps_map is a ConstantUpdate(K) per cell: bit-identical to
    the same permittivities given as one material per value."""
    from fdtd_b200.problem import Material
    p = scenarios.tm_cpml_sources()
    nx, ny, nz = p.shape
    rng = np.random.default_rng(5)
    levels = 1.0 + 5.0 * rng.random(6)
    pick = rng.integers(0, 6, (nz, ny, nx))
    q = copy.deepcopy(p)
    q.materials = [Material.vacuum()] + [Material.constant(float(v)) for v in levels]
    q.ids = (1 + pick).astype(np.uint8)
    p.eps_map = levels[pick]
    a, b = oracle.run_oracle(p), oracle.run_oracle(q)
    for n in ["Ez", "Dz", "Hx", "Hy"]:
        assert np.array_equal(a.get(n), b.get(n)), n


def _objective(oracle, p, spec):
    g = oracle.run_oracle(scenarios.objective_problem(p, spec))
    X = g.dft(0)
    return float(np.sum(np.abs(X) ** 2))


def test_cpu_adjoint_matches_central_differences(oracle):
    """The FP64 adjoint of the oracle's own TM step against central finite
    differences (h = 1e-4 in eps_r) of the oracle forward, at six design
    cells; and its J against a plain forward run."""
    p, spec = scenarios.tm_adjoint_small()
    J, grad = oracle.adjoint_tm(p, p.steps, spec.probe_lo[:2], spec.probe_hi[:2], spec.freq, spec.design_lo[:2],
                                spec.design_hi[:2])
    assert J > 0
    assert abs(J - _objective(oracle, p, spec)) <= 1e-12 * J
    rng = np.random.default_rng(2)
    d0 = spec.design_lo
    h = 1e-4
    for _ in range(6):
        jj, ii = (int(v) for v in rng.integers(0, grad.shape[0], size=2))
        c = (0, d0[1] + jj, d0[0] + ii)
        vals = []
        for sgn in (1, -1):
            q = copy.deepcopy(p)
            q.eps_map = p.eps_map.copy()
            q.eps_map[c] += sgn * h
            vals.append(_objective(oracle, q, spec))
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(grad[jj, ii] - fd) <= 1e-5 * np.abs(grad).max(), (c, grad[jj, ii], fd)
