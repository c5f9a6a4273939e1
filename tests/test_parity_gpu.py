"""GPU parity: the CUDA library, called through the C ABI, against the CPU
oracle on the same seeded inputs.

* FP64 plain method: <= 1e-12 relative L2 on every stored field, CPML
  integrator, polarisation state and DFT accumulator (the kernels follow the
  reference's operation order without FMA contraction, so in practice the
  fields come out bit-identical; the tolerance is the stated bar).
* FP32 fused method: <= 1e-4 relative L2 on E, H, P, J and the DFTs.
* Surface quantities (rho, Je, Jh of include/SurfaceQuantities.hpp, read
  with fdtd_read_quantity): bit-identical in FP64; in FP32 they are
  differences of neighbouring fields, so the bar is 1e-3 relative L2.
"""
import numpy as np
import pytest

import scenarios
from helpers import mode_fields, rel_l2

pytestmark = pytest.mark.gpu

PLAIN_TOL = 1e-12
FUSED_TOL = 1e-4
SURFACE_F32_TOL = 1e-3


def _compare(p, g, o, names, tol):
    worst = {}
    for n in names:
        ref = o.get(n)
        if not np.any(ref):
            continue
        worst[n] = rel_l2(g.get(n), ref)
    for q in range(len(p.dfts)):
        worst[f"dft{q}"] = rel_l2(g.dft(q), o.dft(q))
    bad = {k: v for k, v in worst.items() if not v <= tol}
    assert not bad, f"{p.name}: {bad}"
    return worst


@pytest.mark.parametrize("make", scenarios.ALL_SCENARIOS, ids=lambda f: f.__name__)
def test_plain_f64_matches_oracle(fdtd, oracle, make):
    p = make()
    o = oracle.run_oracle(p)
    g = fdtd.Grid.from_problem(p, "f64")
    g.step(p.steps)
    g.synchronize()
    E, H, D, B = mode_fields(p.mode)
    names = E + H + D + B + oracle.PSI_NAMES + ["Px", "Py", "Pz", "Jx", "Jy", "Jz"]
    _compare(p, g, o, names, PLAIN_TOL)
    npoles = max(len(m.poles) for m in p.materials)
    for pole in range(1, npoles):
        for n in ["Px", "Py", "Pz", "Jx", "Jy", "Jz"]:
            ref = o.get_pole(pole, n)
            assert rel_l2(g.get_pole(pole, n), ref) <= PLAIN_TOL


@pytest.mark.parametrize("make", scenarios.ALL_SCENARIOS, ids=lambda f: f.__name__)
def test_plain_f64_bitwise_fields(fdtd, oracle, make):
    """Stronger than the bar: E and H are bit-identical to the oracle."""
    p = make()
    o = oracle.run_oracle(p)
    g = fdtd.Grid.from_problem(p, "f64")
    g.step(p.steps)
    E, H, _, _ = mode_fields(p.mode)
    for n in E + H + oracle.SURFACE_NAMES:
        assert np.array_equal(g.get(n), o.get(n)), n


@pytest.mark.parametrize("make", scenarios.LEAPFROG_SCENARIOS, ids=lambda f: f.__name__)
def test_fused_f32_matches_oracle(fdtd, oracle, make):
    p = make()
    o = oracle.run_oracle(p)
    g = fdtd.Grid.from_problem(p, "f32")
    g.step(p.steps)
    g.synchronize()
    E, H, _, _ = mode_fields(p.mode)
    _compare(p, g, o, E + H, FUSED_TOL)
    for n in oracle.SURFACE_NAMES:
        ref = o.get(n)
        if np.any(ref):
            assert rel_l2(g.get(n), ref) <= SURFACE_F32_TOL, n


PSI_F32_TOL = 1e-3


@pytest.mark.parametrize("make", [scenarios.td_tfsf_box, scenarios.td_drude_lorentz, scenarios.te_materials,
                                  scenarios.tm_cpml_sources], ids=lambda f: f.__name__)
def test_fused_f32_cpml_integrators_read_back(fdtd, oracle, make):
    """The FP32 method's CPML integrators, read through fdtd_download (the x
    slab in its group-aligned rows, the y and z slabs in field rows), hold the
    oracle's values at the oracle's cells: <= 1e-3 relative L2 for each
    integrator the scenario drives."""
    p = make()
    o = oracle.run_oracle(p)
    g = fdtd.Grid.from_problem(p, "f32")
    g.step(p.steps)
    g.synchronize()
    seen = 0
    for n in oracle.PSI_NAMES:
        ref, got = o.get(n), g.get(n)
        if np.any(ref):
            assert rel_l2(got, ref) <= PSI_F32_TOL, n
            seen += 1
    assert seen >= 2


@pytest.mark.parametrize("pml", [{(0, 0): 5}, {(0, 1): 7}, {(0, 0): 2, (0, 1): 6, (1, 1): 4}, {(1, 0): 3, (2, 1): 4}],
                         ids=["x_low", "x_high", "x_both_y_high", "y_low_z_high"])
@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_one_sided_cpml(fdtd, oracle, pml, prec):
    """CPML on some faces only (the x slab's aligned rows with one side, or
    with ends of different widths): fields and integrators as the oracle's."""
    p = scenarios.td_drude_lorentz()
    p.pml = dict(pml)
    p.name += "_" + "_".join(f"{a}{s}{n}" for (a, s), n in sorted(pml.items()))
    o = oracle.run_oracle(p)
    g = fdtd.Grid.from_problem(p, prec)
    g.step(p.steps)
    g.synchronize()
    E, H, _, _ = mode_fields(p.mode)
    _compare(p, g, o, E + H, FUSED_TOL if prec == "f32" else PLAIN_TOL)
    for n in oracle.PSI_NAMES:
        ref = o.get(n)
        if np.any(ref):
            assert rel_l2(g.get(n), ref) <= (PSI_F32_TOL if prec == "f32" else PLAIN_TOL), n


def test_read_quantity_boxes_and_errors(fdtd, oracle):
    """fdtd_read_quantity on sub-boxes equals the oracle's, and refuses
    quantities outside the mode and boxes that leave the interior."""
    p = scenarios.td_drude_lorentz()
    o = oracle.OracleGrid(p)
    o.step(p.steps)
    g = fdtd.Grid.from_problem(p, "f64")
    g.step(p.steps)
    for q, lo, hi in [(12, (1, 2, 3), (12, 9, 14)), (6, (4, 1, 1), (9, 13, 5)), (11, (2, 2, 2), (2, 13, 14)),
                      (2, (0, 0, 0), (13, 14, 15)), (4, (3, 3, 3), (8, 8, 8))]:
        assert np.array_equal(g.read_quantity(q, lo, hi), o.read_quantity(q, lo, hi)), q
    with pytest.raises(fdtd.FdtdError):
        g.read_quantity(6, (0, 1, 1), (5, 5, 5))
    t = scenarios.tm_cpml_sources()
    gt = fdtd.Grid.from_problem(t, "f32")
    with pytest.raises(fdtd.FdtdError):
        gt.read_quantity(12, (1, 1, 0), (5, 5, 0))  # rho: the TM functor does nothing
    with pytest.raises(fdtd.FdtdError):
        gt.read_quantity(6, (1, 1, 0), (5, 5, 0))  # Je_x: no Ex in TM


@pytest.mark.parametrize("sweep", ["regs", "tma", "flat", "staged"])
@pytest.mark.parametrize("make", [m for m in scenarios.LEAPFROG_SCENARIOS if m().mode == 3], ids=lambda f: f.__name__)
def test_fused_3d_sweep_kernels(fdtd, oracle, make, sweep):
    """Every 3D FP32 sweep implementation (register prefetch, TMA pipeline,
    flat) meets the bar and reports no device-side error."""
    p = make()
    o = oracle.run_oracle(p)
    g = fdtd.Grid.from_problem(p, "f32")
    g.set_sweep_kernel(sweep)
    g.step(p.steps)
    g.synchronize()
    assert g.error_flags() == 0
    E, H, _, _ = mode_fields(p.mode)
    _compare(p, g, o, E + H, FUSED_TOL)


def _all_dispersive(kind):
    """td_drude_lorentz with a material table that holds dispersive
    materials only (the sweeps then stage the ADE state with the fields)."""
    from fdtd_b200.problem import Material
    p = scenarios.td_drude_lorentz()
    dt = p.dt
    drude = Material.drude(1.0, 0.3 / dt, 0.01 / dt)
    if kind == "drude":
        p.materials, p.ids = [drude], None
    elif kind == "drude_lorentz1":
        p.materials = [drude, Material.lorentz(2.0, [(1.0, 0.1 / dt, 0.005 / dt)])]
        p.ids = (p.ids == 2).astype(np.uint8)
    else:
        p.materials = [Material.lorentz(2.0, [(1.5, 0.1 / dt, 0.005 / dt), (0.8, 0.25 / dt, 0.02 / dt)]),
                       Material.lorentz(3.0, [(1.0, 0.12 / dt, 0.01 / dt), (0.5, 0.2 / dt, 0.03 / dt)])]
        p.ids = (p.ids == 1).astype(np.uint8)
    p.name = f"td_all_{kind}"
    return p


@pytest.mark.parametrize("sweep", ["regs", "tma", "flat", "staged"])
@pytest.mark.parametrize("kind", ["drude", "drude_lorentz1", "lorentz2"])
def test_all_dispersive_tables_every_sweep(fdtd, oracle, kind, sweep):
    p = _all_dispersive(kind)
    o = oracle.run_oracle(p)
    g = fdtd.Grid.from_problem(p, "f32")
    g.set_sweep_kernel(sweep)
    g.step(p.steps)
    g.synchronize()
    assert g.error_flags() == 0
    E, H, _, _ = mode_fields(p.mode)
    _compare(p, g, o, E + H, FUSED_TOL)


@pytest.mark.parametrize("kind", ["drude", "drude_lorentz1", "lorentz2"])
def test_all_dispersive_tables_f64_bitwise(fdtd, oracle, kind):
    """The FP64 sweeps that stage P and J with the fields (one pole: 256
    threads per CTA; two poles: 128) give the oracle's every stored array bit
    for bit, the grid's z extent not a multiple of their 8 planes per thread."""
    p = _all_dispersive(kind)
    o = oracle.run_oracle(p)
    g = fdtd.Grid.from_problem(p, "f64")
    g.step(p.steps)
    g.synchronize()
    assert (p.shape[2] - 2) % 8 != 0
    for n in oracle.NAMES + oracle.PSI_NAMES:
        assert np.array_equal(g.get(n), o.get(n)), n
    for pole in range(1, max(len(m.poles) for m in p.materials)):
        for n in ["Px", "Py", "Pz", "Jx", "Jy", "Jz"]:
            assert np.array_equal(g.get_pole(pole, n), o.get_pole(pole, n)), (pole, n)


def test_multistep_schemes_are_fp64_only(fdtd):
    p = scenarios.tm_bd3_tfsf()
    with pytest.raises(fdtd.FdtdError):
        fdtd.Grid.from_problem(p, "f32")
    g = fdtd.Grid(p.mode, p.shape, p.dx, p.dt, "f32")
    g.set_time_scheme(1)
    with pytest.raises(fdtd.FdtdError):
        g.set_time_scheme(2)


def test_multistep_split_steps_and_reset(fdtd, oracle):
    """BD4 history survives split fdtd_step calls and graph chunks; setting
    the scheme again clears it, as on the oracle."""
    p = scenarios.td_bd4_boundaries()
    g1 = fdtd.Grid.from_problem(p, "f64")
    g1.step(p.steps)
    g2 = fdtd.Grid.from_problem(p, "f64")
    g2.step(13)
    g2.step(p.steps - 13)
    for n in ["Ex", "Ey", "Ez", "Hx", "Hy", "Hz"]:
        assert np.array_equal(g1.get(n), g2.get(n)), n
    o = oracle.OracleGrid(p)
    o.step(9)
    g3 = fdtd.Grid.from_problem(p, "f64")
    g3.step(9)
    o.set_time_scheme(3)
    g3.set_time_scheme(3)
    o.step(11)
    g3.step(11)
    for n in ["Ex", "Ey", "Ez", "Hx", "Hy", "Hz"]:
        assert np.array_equal(g3.get(n), o.get(n)), n


def test_split_steps_equal_one_call(fdtd, oracle):
    """fdtd_step(a) then fdtd_step(b) == fdtd_step(a+b), TFSF aux included."""
    p = scenarios.tm_tfsf_reference_polarisation()
    g1 = fdtd.Grid.from_problem(p, "f64")
    g1.step(p.steps)
    g2 = fdtd.Grid.from_problem(p, "f64")
    g2.step(37)
    g2.step(p.steps - 37)
    for n in ["Ez", "Hx", "Hy", "Dz"]:
        assert np.array_equal(g1.get(n), g2.get(n))
    assert g2.step_count == p.steps


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_graph_replay_equals_eager(fdtd, prec):
    """150 steps as two 64-step graph replays plus 22 eager steps give the
    same fields and spectra as 150 eagerly launched steps."""
    p = scenarios.td_tfsf_box()
    p.tfsf.aux_values = np.concatenate([p.tfsf.aux_values, np.zeros(200)])
    out = []
    for graphs in (True, False):
        g = fdtd.Grid.from_problem(p, prec)
        g.use_graphs(graphs)
        g.step(150)
        out.append((g.get("Ez"), g.get("Hy"), g.dft(0)))
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)


def test_deterministic(fdtd):
    p = scenarios.td_tfsf_box()
    outs = []
    for _ in range(2):
        g = fdtd.Grid.from_problem(p, "f32")
        g.step(p.steps)
        outs.append(g.get("Ez"))
    assert np.array_equal(outs[0], outs[1])


def test_errors_are_reported(fdtd):
    from fdtd_b200.problem import TM, THREED
    with pytest.raises(fdtd.FdtdError) as e:
        fdtd.Grid(TM, (8, 8, 2), 1e-6, 1e-15)
    assert e.value.code == -1
    g = fdtd.Grid(TM, (16, 16, 1), 1e-6, 1e-15)
    with pytest.raises(fdtd.FdtdError):
        g.set_pml(0, 0, 20)  # wider than the grid
    with pytest.raises(fdtd.FdtdError):
        g.add_source(0, (5, 5, 0), [1.0])  # Ex is not a TM component
    with pytest.raises(fdtd.FdtdError):
        g.add_source(2, (0, 5, 0), [1.0])  # ring cell
    with pytest.raises(fdtd.FdtdError):
        # the plane projects far outside a 51-cell aux grid
        g.add_tfsf_plane(0, 0, (5, 5, 0), (5, 10, 0), (-100, 8, 0), (1, 0, 0), (0, 0, 1), (0, 1, 0), 1, [1.0])
    f = fdtd.Grid(THREED, (8, 8, 8), 1e-6, 1e-15, "f32")
    with pytest.raises(fdtd.FdtdError) as e:
        f.get("Dx")  # the fused method stores no D
    assert e.value.code == -3


def test_check_finite_flags_nan(fdtd):
    from fdtd_b200.problem import TM
    g = fdtd.Grid(TM, (16, 16, 1), 1e-6, 1e-15)
    g.check_finite()
    a = np.zeros((1, 16, 16))
    a[0, 5, 5] = np.nan
    g.set("Ez", a)
    with pytest.raises(fdtd.FdtdError) as e:
        g.check_finite()
    assert e.value.code == -5


def _with_eps_map(p, seed):
    """A per-cell permittivity map over the vacuum cells of `p`, and the same
    problem restated for the oracle as one ConstantUpdate material per value."""
    import copy
    from fdtd_b200.problem import VACUUM, Material
    nx, ny, nz = p.shape
    rng = np.random.default_rng(seed)
    levels = 1.0 + 3.0 * rng.random(8)
    pick = rng.integers(0, len(levels), (nz, ny, nx))
    base = p.cell_ids()
    base = np.zeros((nz, ny, nx), np.uint8) if base is None else base
    mats = list(p.materials) if p.materials else [Material.vacuum()]
    vac = np.array([m.kind == VACUUM for m in mats])[base]
    eps = np.where(vac, levels[pick], 0.0)
    q = copy.deepcopy(p)
    q.materials = mats + [Material.constant(float(v)) for v in levels]
    q.ids = np.where(vac, len(mats) + pick, base).astype(np.uint8)
    q.block_ids = None
    return eps, q


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("make", [scenarios.tm_cpml_sources, scenarios.te_materials, scenarios.td_drude_lorentz,
                                  scenarios.td_tfsf_box, scenarios.tm_line_source], ids=lambda f: f.__name__)
def test_eps_map_matches_per_cell_materials(fdtd, oracle, make, prec):
    """fdtd_set_eps_map gives the same fields as one constant material per
    cell (bit-identical E and H for the FP64 plain method)."""
    p = make()
    eps, q = _with_eps_map(p, 7)
    o = oracle.run_oracle(q)
    g = fdtd.Grid.from_problem(p, prec)
    g.set_eps_map(eps)
    g.step(p.steps)
    g.synchronize()
    E, H, _, _ = mode_fields(p.mode)
    _compare(p, g, o, E + H, PLAIN_TOL if prec == "f64" else FUSED_TOL)
    if prec == "f64":
        for n in E + H:
            assert np.array_equal(g.get(n), o.get(n)), n


@pytest.mark.parametrize("make", [scenarios.tm_cpml_sources, scenarios.td_surface_dft, scenarios.td_tfsf_box],
                         ids=lambda f: f.__name__)
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_dft_regions_added_mid_run(fdtd, oracle, make, precision):
    """DFT regions added after steps were taken sample from the next step on,
    as the reference's running DFT does: the first half of the regions after
    70 whole steps (one captured graph and a remainder), the rest after three
    half-step pairs that left samples in the buffers of the old layout."""
    p = make()
    regions, p.dfts = p.dfts, []
    first, rest = regions[: max(1, len(regions) // 2)], regions[max(1, len(regions) // 2):]
    o = oracle.OracleGrid(p)
    g = fdtd.Grid.from_problem(p, precision)
    o.step(70)
    g.step(70)
    for r in first:
        o.add_dft(r.comp, r.lo, r.hi, r.freqs)
        g.add_dft(r.comp, r.lo, r.hi, r.freqs)
    o.step(75)
    g.step(75)
    for _ in range(3):
        for ph in (0, 1):
            o.step_half(ph)
            g.step_half(ph)
    g.step_half(0)
    with pytest.raises(fdtd.FdtdError):
        g.add_dft(regions[0].comp, regions[0].lo, regions[0].hi, regions[0].freqs)
    g.step_half(1)
    o.step(1)
    for r in rest:
        o.add_dft(r.comp, r.lo, r.hi, r.freqs)
        g.add_dft(r.comp, r.lo, r.hi, r.freqs)
    o.step(40)
    g.step(40)
    tol = PLAIN_TOL if precision == "f64" else FUSED_TOL
    for q in range(len(regions)):
        assert rel_l2(g.dft(q), o.dft(q)) <= tol, (q, regions[q].comp)


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_large_spectrum_read_equals_its_parts(fdtd, precision):
    """A spectrum of more than 8 MB is read through pinned staging chunks and
    several host threads; it must equal, bit for bit, the same points taken
    as four smaller regions (read with one plain copy each)."""
    from fdtd_b200 import problem as P
    n = 38
    p = P.Problem(P.THREED, (n, n, n), 1e-6, P.courant_dt(1e-6, 0.99 / np.sqrt(3.0)), name="large_spectrum")
    for a in range(3):
        for s in (0, 1):
            p.pml[(a, s)] = 4
    p.sources.append(P.Source(1, (n // 2, n // 2, n // 2), P.gaussian_pulse(30, 12, 4), "E"))
    p.steps = 30
    nx, ny, nz = p.shape
    lo, hi = (1, 1, 1), (nx - 2, ny - 2, nz - 2)
    freqs = [0.01 * (q + 1) for q in range(32)]
    g = fdtd.Grid.from_problem(p, precision)
    whole = g.add_dft(1, lo, hi, freqs)
    cuts = np.linspace(lo[2], hi[2] + 1, 5).astype(int)
    parts = [g.add_dft(1, (lo[0], lo[1], int(a)), (hi[0], hi[1], int(b) - 1), freqs) for a, b in zip(cuts, cuts[1:])]
    g.step(p.steps)
    w = g.dft(whole)
    assert w.nbytes > 8 << 20
    ex, ey = hi[0] - lo[0] + 1, hi[1] - lo[1] + 1
    got = np.concatenate([g.dft(h).reshape(len(freqs), -1, ey, ex) for h in parts], axis=1)
    assert np.any(w != 0)
    assert np.array_equal(got.reshape(w.shape), w)


@pytest.mark.parametrize("make", scenarios.FORWARD_SCENARIOS, ids=lambda f: f.__name__)
def test_forward_material_updates_match_oracle(fdtd, oracle, make):
    """fdtd_material_explicit (the reference's XUpdate<Mode, ft, true>) after
    the steps: every stored array bit for bit the oracle's, which reproduces
    the reference's <name>_fwd fixtures."""
    p = scenarios.forward_materials(make)
    o = oracle.run_oracle(p)
    o.material_explicit(0)
    o.material_explicit(1)
    g = fdtd.Grid.from_problem(p, "f64")
    g.step(p.steps)
    g.material_explicit(0)
    g.material_explicit(1)
    g.synchronize()
    for n in oracle.NAMES + oracle.PSI_NAMES:
        assert np.array_equal(g.get(n), o.get(n)), f"{p.name}:{n}"


def test_forward_material_updates_refusals(fdtd):
    g = fdtd.Grid.from_problem(scenarios.td_drude_lorentz(), "f64")
    with pytest.raises(fdtd.FdtdError) as e:
        g.material_explicit(0)  # a Lorentz material: no explicit update in the reference
    assert e.value.code == -3
    g.material_explicit(1)
    f32 = fdtd.Grid.from_problem(scenarios.forward_materials(scenarios.te_materials), "f32")
    with pytest.raises(fdtd.FdtdError) as e:
        f32.material_explicit(1)  # the FP32 method stores no D or B
    assert e.value.code == -3
    with pytest.raises(fdtd.FdtdError):
        g.material_explicit(2)


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_step_graph_follows_new_tfsf_tables(fdtd, prec):
    """Calls of growing length: a call of more steps than the TFSF tables hold
    gets new tables, and the step graph captured before (whose launches hold
    the old tables' addresses) is captured again. Graph-replayed calls give
    the eager steps' fields bit for bit; so does a grid whose graph
    fdtd_prepare captured."""
    p = scenarios.td_tfsf_box()
    a = fdtd.Grid.from_problem(p, prec)
    b = fdtd.Grid.from_problem(p, prec)
    b.use_graphs(False)
    c = fdtd.Grid.from_problem(p, prec)
    c.prepare()
    for n in (64, 300, 70, 520):
        for g in (a, b, c):
            g.step(n)
    for n in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
        ref = b.get(n)
        assert np.array_equal(a.get(n), ref), n
        assert np.array_equal(c.get(n), ref), n
    for q in range(len(p.dfts)):
        assert np.any(b.dft(q)), q
        assert np.array_equal(a.dft(q), b.dft(q)), q
        assert np.array_equal(c.dft(q), b.dft(q)), q
