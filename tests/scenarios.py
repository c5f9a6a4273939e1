"""Small seeded scenarios shared by the golden-fixture generator and the
parity tests. Each exercises one slice of the hot path at a size the CPU
oracle finishes in well under a second."""
from __future__ import annotations

import math

import numpy as np

from fdtd_b200.problem import (CONSTANT, DRUDE, IMP0, LORENTZ, TE, TM, THREED, TFSF, Material, Problem, Source, DFTRegion,
                               courant_dt, gaussian_pulse, ref_te_polarisation, ref_tm_polarisation, sinusoid,
                               tfsf_box_planes)

DX = 1e-6
DT2 = courant_dt(DX, 0.99 / math.sqrt(2.0))
DT3 = courant_dt(DX, 0.99 / math.sqrt(3.0))


def tm_cpml_sources() -> Problem:
    p = Problem(TM, (40, 36, 1), DX, DT2, name="tm_cpml_sources")
    for a in (0, 1):
        for s in (0, 1):
            p.pml[(a, s)] = 6
    p.sources.append(Source(2, (20, 18, 0), gaussian_pulse(80, 20, 6), "E"))
    p.sources.append(Source(2, (12, 10, 0), 1e-12 * gaussian_pulse(80, 25, 6), "D"))
    p.dfts.append(DFTRegion(2, (0, 18, 0), (39, 18, 0), [0.02, 0.05]))
    p.dfts.append(DFTRegion(3, (5, 5, 0), (9, 8, 0), [0.03]))
    # surface current Je_z and Jh_x (SurfaceQuantities.hpp) on boxes
    p.dfts.append(DFTRegion(8, (8, 6, 0), (31, 28, 0), [0.03]))
    p.dfts.append(DFTRegion(9, (1, 1, 0), (38, 34, 0), [0.02, 0.05]))
    p.steps = 80
    return p


def te_materials() -> Problem:
    p = Problem(TE, (33, 41, 1), DX, DT2, name="te_materials")
    for a in (0, 1):
        for s in (0, 1):
            p.pml[(a, s)] = 5 + s
    dt = DT2
    p.materials = [Material.vacuum(), Material.constant(4.0), Material.drude(2.0, 0.3 / dt, 0.01 / dt),
                   Material.lorentz(1.5, [(1.0, 0.1 / dt, 0.005 / dt)])]
    ids = np.zeros((1, 41, 33), np.uint8)
    ids[0, 10:20, 8:14] = 1
    ids[0, 22:30, 10:25] = 2
    ids[0, 5:9, 15:28] = 3
    p.ids = ids
    p.sources.append(Source(0, (16, 20, 0), gaussian_pulse(60, 20, 6), "E"))
    p.sources.append(Source(1, (16, 21, 0), gaussian_pulse(60, 20, 6), "E"))
    p.dfts.append(DFTRegion(5, (3, 3, 0), (29, 37, 0), [0.04]))
    # surface charge density and currents (SurfaceQuantities.hpp)
    p.dfts.append(DFTRegion(12, (2, 2, 0), (30, 38, 0), [0.04]))
    p.dfts.append(DFTRegion(7, (6, 6, 0), (26, 34, 0), [0.03]))
    p.dfts.append(DFTRegion(11, (1, 1, 0), (31, 39, 0), [0.04]))
    p.steps = 60
    return p


def td_drude_lorentz() -> Problem:
    nx, ny, nz = 14, 15, 16
    p = Problem(THREED, (nx, ny, nz), DX, DT3, name="td_drude_lorentz")
    for a in range(3):
        for s in (0, 1):
            p.pml[(a, s)] = 3
    dt = DT3
    p.materials = [Material.vacuum(), Material.drude(1.0, 0.3 / dt, 0.01 / dt),
                   Material.lorentz(2.0, [(1.0, 0.1 / dt, 0.005 / dt)])]
    ids = np.zeros((nz, ny, nx), np.uint8)
    ids[6:10, 6:9, 5:9] = 1
    ids[3:6, 8:12, 4:7] = 2
    p.ids = ids
    p.sources.append(Source(2, (7, 7, 8), gaussian_pulse(40, 15, 5), "E"))
    p.sources.append(Source(0, (6, 8, 7), gaussian_pulse(40, 18, 5), "E"))
    p.dfts.append(DFTRegion(2, (1, 1, 8), (12, 13, 8), [0.02, 0.05]))
    p.dfts.append(DFTRegion(4, (2, 7, 2), (11, 7, 13), [0.04]))
    p.steps = 40
    return p


def tm_tfsf_reference_polarisation() -> Problem:
    n = 60
    p = Problem(TM, (n, n, 1), DX, DT2, name="tm_tfsf_refpol")
    for a in (0, 1):
        for s in (0, 1):
            p.pml[(a, s)] = 8
    k = (1.0, 0.0, 0.0)
    pe, ph = ref_tm_polarisation(k)
    p.tfsf = TFSF(aux_ncells=n, aux_values=gaussian_pulse(100, 40, 10, offset=1.0), origin=(n / 2, n / 2, 0), k=k,
                  pol_e=pe, pol_h=ph, planes=tfsf_box_planes(TM, (18, 18), (41, 41)))
    p.steps = 100
    return p


def te_tfsf_oblique() -> Problem:
    n = 56
    p = Problem(TE, (n, n, 1), DX, DT2, name="te_tfsf_oblique")
    for a in (0, 1):
        for s in (0, 1):
            p.pml[(a, s)] = 7
    k = (math.cos(0.4), math.sin(0.4), 0.0)
    pe, ph = ref_te_polarisation(k)
    p.tfsf = TFSF(aux_ncells=2 * n, aux_values=gaussian_pulse(90, 35, 9, offset=1.0), origin=(n / 2, n / 2, 0), k=k,
                  pol_e=pe, pol_h=ph, planes=tfsf_box_planes(TE, (16, 16), (39, 39)))
    p.steps = 90
    return p


def td_tfsf_box() -> Problem:
    n = 24
    p = Problem(THREED, (n, n, n), DX, DT3, name="td_tfsf_box")
    for a in range(3):
        for s in (0, 1):
            p.pml[(a, s)] = 4
    dt = DT3
    p.materials = [Material.vacuum(), Material.drude(1.0, 0.3 / dt, 0.01 / dt)]
    ids = np.zeros((n, n, n), np.uint8)
    ids[10:14, 10:14, 10:14] = 1
    p.ids = ids
    k = (1.0, 0.0, 0.0)
    c = n // 2
    p.tfsf = TFSF(aux_ncells=n, aux_values=gaussian_pulse(50, 20, 6, offset=1.0), origin=(c, c, c), k=k,
                  pol_e=(0.0, 0.0, 1.0), pol_h=(0.0, 1.0, 0.0), planes=tfsf_box_planes(THREED, (7, 7, 7), (16, 16, 16)))
    for a in range(3):
        lo, hi = [6, 6, 6], [17, 17, 17]
        lo[a] = hi[a] = 6
        p.dfts.append(DFTRegion((a + 1) % 3, tuple(lo), tuple(hi), [0.03, 0.06]))
        p.dfts.append(DFTRegion(3 + (a + 2) % 3, tuple(lo), tuple(hi), [0.03, 0.06]))
    p.steps = 50
    return p


def td_surface_dft() -> Problem:
    """3D running DFTs of every surface quantity (rho, Je, Jh of
    SurfaceQuantities.hpp) on boxes through a Drude cube and a Lorentz slab."""
    p = td_drude_lorentz()
    p.name = "td_surface_dft"
    nx, ny, nz = p.shape
    for q in range(6, 13):
        lo = (1 + q % 2, 2, 1 + q % 3)
        hi = (nx - 2, ny - 3 + q % 2, nz - 2 - q % 2)
        p.dfts.append(DFTRegion(q, lo, hi, [0.03, 0.05]))
    return p


def tm_magnetic_tfsf() -> Problem:
    """TM TFSF box around magnetic cells: a constant block (eps 2, mu 1.7)
    and a Drude block with mu 1.3 (ConstantUpdate<Mode, Magnetic>), with a
    B-target source inside the magnetic block."""
    p = tm_tfsf_reference_polarisation()
    p.name = "tm_magnetic_tfsf"
    n = p.shape[0]
    dt = p.dt
    p.materials = [Material.vacuum(), Material(CONSTANT, 2.0, 1.7, []),
                   Material(DRUDE, 1.0, 1.3, [(1.0, 0.3 / dt, 0.01 / dt)])]
    ids = np.zeros((1, n, n), np.uint8)
    ids[0, 24:32, 22:30] = 1
    ids[0, 30:38, 33:40] = 2
    p.ids = ids
    p.sources.append(Source(0, (25, 27, 0), 1e-9 * gaussian_pulse(100, 30, 8), "B"))
    p.dfts.append(DFTRegion(4, (20, 30, 0), (39, 30, 0), [0.03]))
    return p


def td_magnetic_tfsf() -> Problem:
    """3D TFSF box with a magnetic cube (eps 1.5, mu 2.2), a magnetic Drude
    slab (mu 1.4) and H- and B-target sources in them."""
    p = td_tfsf_box()
    p.name = "td_magnetic_tfsf"
    n = p.shape[0]
    dt = p.dt
    p.materials = [Material.vacuum(), Material(CONSTANT, 1.5, 2.2, []),
                   Material(DRUDE, 1.0, 1.4, [(1.0, 0.3 / dt, 0.01 / dt)])]
    ids = np.zeros((n, n, n), np.uint8)
    ids[9:13, 10:14, 9:15] = 1
    ids[13:16, 8:16, 11:13] = 2
    p.ids = ids
    p.sources.append(Source(1, (11, 12, 10), 1e-3 * gaussian_pulse(50, 15, 5), "H"))
    p.sources.append(Source(2, (12, 10, 14), 1e-9 * gaussian_pulse(50, 18, 5), "B"))
    return p


def td_lorentz_two_pole_blocks() -> Problem:
    """Two-pole Lorentz on a per-block eps_inf map (an extension: the
    reference holds one pole; at one pole with delta_eps = 1 it reduces to
    LorentzUpdate)."""
    n = 20
    p = Problem(THREED, (n, n, n), DX, DT3, name="td_lorentz2_blocks")
    for a in range(3):
        for s in (0, 1):
            p.pml[(a, s)] = 3
    dt = DT3
    rng = np.random.default_rng(0)
    nb = (n + 7) // 8
    eps = rng.uniform(1.0, 6.0, size=nb ** 3)
    poles = [(1.5, 0.1 / dt, 0.005 / dt), (0.8, 0.25 / dt, 0.02 / dt)]
    p.materials = [Material.lorentz(float(e), poles) for e in eps]
    p.block_ids = np.arange(nb ** 3, dtype=np.uint16).reshape(nb, nb, nb)
    p.block_shift = 3
    p.sources.append(Source(2, (10, 10, 10), gaussian_pulse(40, 15, 5), "E"))
    p.dfts.append(DFTRegion(2, (0, 0, 10), (n - 1, n - 1, 10), [0.02, 0.04]))
    p.steps = 40
    return p


def te_h_sources() -> Problem:
    """TE with soft sources on Hz after the magnetic update (H target, as
    make_soft_source<Hz>) and on Bz before the magnetic CPML pass (B target)."""
    p = Problem(TE, (44, 38, 1), DX, DT2, name="te_h_sources")
    for a in (0, 1):
        for s in (0, 1):
            p.pml[(a, s)] = 6
    p.sources.append(Source(2, (21, 19, 0), gaussian_pulse(70, 20, 6), "H"))
    p.sources.append(Source(2, (12, 25, 0), 1e-6 * gaussian_pulse(70, 25, 6), "B"))
    p.dfts.append(DFTRegion(5, (2, 19, 0), (41, 19, 0), [0.03]))
    p.steps = 70
    return p


def td_h_sources() -> Problem:
    nx, ny, nz = 16, 14, 15
    p = Problem(THREED, (nx, ny, nz), DX, DT3, name="td_h_sources")
    for a in range(3):
        for s in (0, 1):
            p.pml[(a, s)] = 3
    p.sources.append(Source(0, (8, 7, 7), gaussian_pulse(40, 15, 5), "H"))
    p.sources.append(Source(1, (6, 7, 8), 1e-6 * gaussian_pulse(40, 12, 5), "B"))
    p.steps = 40
    return p


def tm_line_source() -> Problem:
    """TM with a line source (one Sinusoid-driven soft source per cell of a
    column, E target), a point source on a cell of that line (point sources
    apply first), and a box of soft sources on Hy (H target)."""
    nx, ny = 42, 38
    p = Problem(TM, (nx, ny, 1), DX, DT2, name="tm_line_source")
    for a in (0, 1):
        for s in (0, 1):
            p.pml[(a, s)] = 6
    p.sources.append(Source(2, (10, 18, 0), 0.5 * gaussian_pulse(90, 20, 6), "E"))
    p.sources.append(Source(2, (10, 1, 0), sinusoid(90, 0.05), "E", hi=(10, ny - 2, 0)))
    p.sources.append(Source(1, (20, 15, 0), 1e-3 * gaussian_pulse(90, 30, 8), "H", hi=(22, 17, 0)))
    p.dfts.append(DFTRegion(2, (30, 1, 0), (30, ny - 2, 0), [0.05]))
    p.steps = 90
    return p


def td_box_sources() -> Problem:
    """3D box sources on Ez (E target) through a Drude block, and on Hx (H
    target)."""
    nx, ny, nz = 14, 15, 16
    p = Problem(THREED, (nx, ny, nz), DX, DT3, name="td_box_sources")
    for a in range(3):
        for s in (0, 1):
            p.pml[(a, s)] = 3
    dt = DT3
    p.materials = [Material.vacuum(), Material.drude(1.5, 0.3 / dt, 0.01 / dt)]
    ids = np.zeros((nz, ny, nx), np.uint8)
    ids[6:11, 5:10, 4:9] = 1
    p.ids = ids
    p.sources.append(Source(2, (6, 4, 5), gaussian_pulse(40, 15, 5), "E", hi=(6, 9, 8)))
    p.sources.append(Source(0, (8, 7, 9), 1e-3 * gaussian_pulse(40, 12, 5), "H", hi=(9, 8, 9)))
    p.dfts.append(DFTRegion(2, (1, 1, 8), (nx - 2, ny - 2, 8), [0.03]))
    p.steps = 40
    return p


def tm_boundaries() -> Problem:
    """TM with a PEC face (x min), a CPML face (x max) and periodic faces in y."""
    nx, ny = 36, 30
    p = Problem(TM, (nx, ny, 1), DX, DT2, name="tm_boundaries")
    p.pml[(0, 1)] = 6
    p.boundaries = {(0, 0): "pec", (1, 0): "periodic", (1, 1): "periodic"}
    p.sources.append(Source(2, (10, 8, 0), gaussian_pulse(90, 20, 6), "E"))
    p.sources.append(Source(0, (20, 22, 0), 1e-3 * gaussian_pulse(90, 25, 6), "H"))
    p.dfts.append(DFTRegion(2, (1, 15, 0), (nx - 2, 15, 0), [0.04]))
    p.steps = 90
    return p


def te_boundaries() -> Problem:
    """TE with symmetric (x min), antisymmetric (y max) and PMC (y min)
    faces and a CPML face (x max), through a constant-eps block."""
    nx, ny = 34, 38
    p = Problem(TE, (nx, ny, 1), DX, DT2, name="te_boundaries")
    p.pml[(0, 1)] = 5
    p.boundaries = {(0, 0): "symmetric", (1, 1): "antisymmetric", (1, 0): "pmc"}
    p.materials = [Material.vacuum(), Material.constant(3.0)]
    ids = np.zeros((1, ny, nx), np.uint8)
    ids[0, 12:20, 6:14] = 1
    p.ids = ids
    p.sources.append(Source(2, (9, 18, 0), gaussian_pulse(80, 20, 6), "H"))
    p.sources.append(Source(0, (15, 25, 0), gaussian_pulse(80, 25, 6), "E"))
    p.dfts.append(DFTRegion(5, (1, 1, 0), (nx - 2, ny - 2, 0), [0.03]))
    p.steps = 80
    return p


def td_boundaries() -> Problem:
    """3D: periodic x, symmetric y min, PMC z min, PEC z max, CPML y max,
    with a Drude block."""
    nx, ny, nz = 14, 16, 15
    p = Problem(THREED, (nx, ny, nz), DX, DT3, name="td_boundaries")
    p.pml[(1, 1)] = 3
    p.boundaries = {(0, 0): "periodic", (0, 1): "periodic", (1, 0): "symmetric", (2, 0): "pmc", (2, 1): "pec"}
    dt = DT3
    p.materials = [Material.vacuum(), Material.drude(1.0, 0.3 / dt, 0.01 / dt)]
    ids = np.zeros((nz, ny, nx), np.uint8)
    ids[5:9, 4:8, 3:7] = 1
    p.ids = ids
    p.sources.append(Source(2, (7, 8, 7), gaussian_pulse(40, 15, 5), "E"))
    p.sources.append(Source(0, (4, 10, 9), 1e-3 * gaussian_pulse(40, 12, 5), "H"))
    p.dfts.append(DFTRegion(1, (1, 1, 7), (nx - 2, ny - 2, 7), [0.03]))
    p.steps = 40
    return p


def _time_scheme(p: Problem, scheme: int, name: str) -> Problem:
    """`p` stepped with the BD3/BD4 time policy at half the Courant limit
    (both diverge near the limit); materials keep their rates."""
    p.time_scheme = scheme
    p.dt = courant_dt(p.dx, 0.5 / math.sqrt(p.dim))
    p.name = name
    return p


def tm_bd3_tfsf() -> Problem:
    """BD3 with a TFSF box, CPML and the reference's TM polarisation."""
    return _time_scheme(tm_tfsf_reference_polarisation(), 3, "tm_bd3_tfsf")


def te_bd4_materials() -> Problem:
    """BD4 through constant, Drude and Lorentz cells with CPML."""
    return _time_scheme(te_materials(), 4, "te_bd4_materials")


def td_bd3_tfsf() -> Problem:
    """3D BD3 with a TFSF box around a Drude cube."""
    return _time_scheme(td_tfsf_box(), 3, "td_bd3_tfsf")


def td_bd4_boundaries() -> Problem:
    """3D BD4 with periodic, symmetric, PMC and PEC faces and H sources."""
    return _time_scheme(td_boundaries(), 4, "td_bd4_boundaries")


def tm_adjoint_small(n: int = 40, steps: int = 260, design: int = 8, seed: int = 1):
    """The adjoint workload at a size the CPU oracle runs in well under a
    second: TM, 6-cell CPML, a central design box of random eps_r in [1, 12],
    an Ez line source (Sinusoid at 0.05 cycles/step), 4 probe cells on the
    right. Returns (Problem, AdjointSpec)."""
    from fdtd_b200.problem import AdjointSpec
    p = Problem(TM, (n, n, 1), DX, DT2, name=f"tm{n}_adjoint_small")
    for a in (0, 1):
        for s in (0, 1):
            p.pml[(a, s)] = 6
    rng = np.random.default_rng(seed)
    d0 = (n - design) // 2
    eps = np.zeros((1, n, n))
    eps[0, d0:d0 + design, d0:d0 + design] = rng.uniform(1.0, 12.0, size=(design, design))
    p.eps_map = eps
    p.sources.append(Source(2, (8, 1, 0), sinusoid(steps, 0.05), "E", hi=(8, n - 2, 0)))
    pc, j0 = n - 9, n // 2 - 2
    spec = AdjointSpec((pc, j0, 0), (pc, j0 + 3, 0), 0.05, (d0, d0, 0), (d0 + design - 1, d0 + design - 1, 0), 32)
    p.steps = steps
    return p, spec


def objective_problem(p, spec):
    """`p` with the objective's DFT region as its only DFT region."""
    import copy
    q = copy.deepcopy(p)
    q.dfts = [DFTRegion(2, spec.probe_lo, spec.probe_hi, [spec.freq])]
    return q


def tm_cpml_model() -> Problem:
    """TM with CPML sides graded by their own PMLParameterModel(m, ma, sMax,
    kMax, aMax) (include/PML.hpp:376-377): a steeper, stronger layer, a
    kappa-free quadratic one, a third shape, and one default side."""
    p = tm_cpml_sources()
    p.name = "tm_cpml_model"
    s0 = 0.8 * 4 / (IMP0 * DX)
    p.pml_models[(0, 0)] = (4.0, 2.0, 1.3 * s0, 8.0, 0.1)
    p.pml_models[(0, 1)] = (2.0, 1.0, 0.6 * s0, 1.0, 0.0)
    p.pml_models[(1, 1)] = (3.5, 1.5, 2.0 * s0, 3.0, 0.2)
    return p


def td_cpml_model() -> Problem:
    """3D dispersive cells with the z and x-max CPML sides graded by
    PMLParameterModel(m, ma, sMax, kMax, aMax)."""
    p = td_drude_lorentz()
    p.name = "td_cpml_model"
    s0 = 0.8 * 4 / (IMP0 * DX)
    p.pml_models[(2, 0)] = (2.5, 1.0, 1.5 * s0, 6.0, 0.08)
    p.pml_models[(2, 1)] = (4.0, 3.0, 0.9 * s0, 2.0, 0.01)
    p.pml_models[(0, 1)] = (3.0, 2.0, 1.1 * s0, 11.0, 0.15)
    return p


# scenarios the reference itself can run (one pole per cell)
REFERENCE_SCENARIOS = [tm_cpml_sources, te_materials, td_drude_lorentz, tm_tfsf_reference_polarisation,
                       te_tfsf_oblique, td_tfsf_box, te_h_sources, td_h_sources, tm_line_source, td_box_sources,
                       tm_boundaries, te_boundaries, td_boundaries, tm_bd3_tfsf, te_bd4_materials, td_bd3_tfsf,
                       td_bd4_boundaries, tm_magnetic_tfsf, td_magnetic_tfsf, tm_cpml_model, td_cpml_model]
# scenarios whose every material has a forward (explicit) update in the
# reference, run with those updates applied after the steps
# (forward_materials): each Lorentz material becomes a magnetic constant one
FORWARD_SCENARIOS = [te_materials, td_drude_lorentz, tm_cpml_sources]


def forward_materials(make) -> Problem:
    """Scenario `make` with each Lorentz material replaced by a constant one of
    the same eps_inf and mu_r 1.6 (the reference's explicit Lorentz update is a
    static_assert), named <name>_fwd."""
    p = make()
    p.materials = [Material.constant(m.eps_inf, 1.6) if m.kind == LORENTZ else m for m in p.materials]
    p.name += "_fwd"
    return p


# scenarios on the BD3/BD4 time policies (FP64 plain method only)
MULTISTEP_SCENARIOS = [tm_bd3_tfsf, te_bd4_materials, td_bd3_tfsf, td_bd4_boundaries]
ALL_SCENARIOS = REFERENCE_SCENARIOS + [td_lorentz_two_pole_blocks, td_surface_dft]
# scenarios the FP32 fused method runs (it steps with the leapfrog only)
LEAPFROG_SCENARIOS = [m for m in ALL_SCENARIOS if m not in MULTISTEP_SCENARIOS]
