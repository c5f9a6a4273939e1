"""Z-slab decomposition on the GPU: every slab of the grid in this process on
one device (ZSlabDomain: fdtd_step_half for the halves, fdtd_copy_plane for
the ghost planes, all in one stream, so no kernel ever waits on another). The
assembled fields and spectra must equal those of the single grid stepped with
fdtd_step, bit for bit, for both methods."""
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
