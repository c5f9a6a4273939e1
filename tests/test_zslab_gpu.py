"""Z-slab decomposition on the GPU: every slab of the grid in this process on
one device (ZSlabDomain: fdtd_step_half_part for the halves, the ghost planes
copied plane to plane with fdtd_copy_plane_between on a second stream while the interior parts of
the sweeps run; events order them, no kernel ever waits on another). The
assembled fields and spectra must equal those of the single grid stepped with
fdtd_step, bit for bit, for both methods; so must a single grid stepped in
split half steps."""
import numpy as np
import pytest

import scenarios
from fdtd_b200.zslab import ZSlabDomain

pytestmark = pytest.mark.gpu

CASES = [scenarios.td_tfsf_box, scenarios.td_drude_lorentz, scenarios.td_box_sources, scenarios.td_h_sources,
         scenarios.td_lorentz_two_pole_blocks, scenarios.td_boundaries, scenarios.td_bd4_boundaries]


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("make", CASES, ids=lambda f: f.__name__)
def test_slabs_reproduce_the_single_grid(fdtd, make, world, prec):
    if make is scenarios.td_lorentz_two_pole_blocks and world == 3:
        pytest.skip("no block-aligned 3-way partition of this grid")
    if make in scenarios.MULTISTEP_SCENARIOS and prec == "f32":
        pytest.skip("the FP32 fused method steps with the leapfrog only")
    p = make()
    ref = fdtd.Grid.from_problem(p, prec)
    ref.step(p.steps)
    dom = ZSlabDomain(p, world, prec)
    dom.step(p.steps)
    for n in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
        assert np.array_equal(dom.get(n), ref.get(n)[1:-1]), n
    for q in range(len(p.dfts)):
        assert np.array_equal(dom.dft(q), ref.dft(q)), q


def test_half_steps_must_alternate(fdtd):
    p = scenarios.td_tfsf_box()
    g = fdtd.Grid.from_problem(p, "f32")
    with pytest.raises(fdtd.FdtdError):
        g.step_half(1)
    g.step_half(0)
    with pytest.raises(fdtd.FdtdError):
        g.step(1)  # a full step between the halves
    g.step_half(1)
    g.step(3)
    assert g.step_count == 4


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("make", [scenarios.td_tfsf_box, scenarios.td_box_sources, scenarios.td_boundaries,
                                  scenarios.td_lorentz_two_pole_blocks], ids=lambda f: f.__name__)
def test_split_half_steps_equal_the_step(fdtd, make, prec):
    """fdtd_step_half_part: part 0 (planes that read no ghost plane) then
    part 1 (the plane next to it, and the rest of the half step) of both
    halves give fdtd_step's fields and spectra bit for bit."""
    p = make()
    ref = fdtd.Grid.from_problem(p, prec)
    ref.step(p.steps)
    g = fdtd.Grid.from_problem(p, prec)
    for _ in range(p.steps):
        for phase in (0, 1):
            g.step_half_part(phase, 0)
            g.step_half_part(phase, 1)
    assert g.step_count == p.steps
    for n in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
        assert np.array_equal(g.get(n), ref.get(n)), n
    for q in range(len(p.dfts)):
        assert np.array_equal(g.dft(q), ref.dft(q)), q


def test_split_half_steps_are_ordered(fdtd):
    p = scenarios.td_tfsf_box()
    g = fdtd.Grid.from_problem(p, "f32")
    with pytest.raises(fdtd.FdtdError):
        g.step_half_part(0, 1)  # part 1 before part 0
    g.step_half_part(0, 0)
    for bad in (lambda: g.step_half(0), lambda: g.step(1), lambda: g.step_half_part(0, 0),
                lambda: g.step_half_part(1, 0)):
        with pytest.raises(fdtd.FdtdError):
            bad()
    g.step_half_part(0, 1)
    g.step_half(1)
    assert g.step_count == 1
    tm = fdtd.Grid.from_problem(scenarios.tm_cpml_sources(), "f32")
    with pytest.raises(fdtd.FdtdError) as e:
        tm.step_half_part(0, 0)  # 2D grids have no z planes to split
    assert e.value.code == -3


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_plane_copy_between_grids(fdtd, prec):
    """fdtd_copy_plane_between moves exactly one z plane of one component."""
    p = scenarios.td_tfsf_box()
    a = fdtd.Grid.from_problem(p, prec)
    b = fdtd.Grid.from_problem(p, prec)
    a.step(7)
    a.synchronize()
    a.copy_plane_to("Hy", 5, b, 9)
    b.synchronize()
    got, src = b.get("Hy"), a.get("Hy")
    assert np.array_equal(got[9], src[5])
    got[9] = 0.0
    assert not np.any(got)
    assert not np.any(b.get("Hx"))
    c = fdtd.Grid.from_problem(scenarios.td_drude_lorentz(), prec)  # another x-y extent
    with pytest.raises(fdtd.FdtdError):
        a.copy_plane_to("Hy", 5, c, 3)
    with pytest.raises(fdtd.FdtdError):
        a.copy_plane_to("Hy", 99, b, 3)
