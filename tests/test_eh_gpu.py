"""The one-launch step (FDTD_SWEEP_EH: the staged E and H updates of a
whole step in one persistent launch, H tiles following the E tiles they read)
against the two staged sweeps.

Each cell's update is the same code with the same operands in both, so the
results must be bit-identical -- fields, CPML integrators, ADE state and DFT
spectra -- on grids whose tiles (128 cells x 8 rows, as two 4-row halves)
and lag cover the schedule's cases: one tile per plane, many x and y tiles,
a last tile with one half or a partly filled half, a lag equal to the plane
count (all E before all H) and a lag of a few planes; graph replay (64-step
chunks) and eager launches. Grids the one-launch step does not
take (TFSF planes, boundary conditions, box sources) are refused.
"""
import numpy as np
import pytest

import scenarios
from fdtd_b200 import problem as P

pytestmark = pytest.mark.gpu

FIELDS = ["Ex", "Ey", "Ez", "Hx", "Hy", "Hz", "Px", "Py", "Pz", "Jx", "Jy", "Jz"]
PSI = [f"psi{'EH'[f]}{'xyz'[i]}{'xyz'[j]}" for f in range(2) for i in range(3) for j in range(3)]


def _pair(fdtd, p, steps, graphs=True):
    ref = fdtd.Grid.from_problem(p, "f32")
    ref.set_sweep_kernel("staged")
    new = fdtd.Grid.from_problem(p, "f32")
    new.set_sweep_kernel("eh")
    for g in (ref, new):
        g.use_graphs(graphs)
        g.step(steps)
        g.synchronize()
    return ref, new


def _assert_identical(p, ref, new):
    assert new.error_flags() == 0
    for n in FIELDS + PSI:
        a, b = new.get(n), ref.get(n)
        assert np.array_equal(a, b), n
    npoles = max((len(m.poles) for m in p.materials), default=0)
    for pole in range(1, npoles):
        for n in ["Px", "Py", "Pz", "Jx", "Jy", "Jz"]:
            assert np.array_equal(new.get_pole(pole, n), ref.get_pole(pole, n)), (pole, n)
    for q in range(len(p.dfts)):
        assert np.array_equal(new.dft(q), ref.dft(q)), q


@pytest.mark.parametrize("make", [scenarios.td_drude_lorentz, scenarios.td_surface_dft,
                                  scenarios.td_lorentz_two_pole_blocks, scenarios.td_h_sources],
                         ids=lambda f: f.__name__)
def test_eh_step_identical_to_sweeps_scenarios(fdtd, make):
    p = make()
    ref, new = _pair(fdtd, p, p.steps)
    _assert_identical(p, ref, new)


def _drude_no_tfsf(shape, steps):
    p = P.config2(steps=steps, shape=shape)
    p.tfsf = None
    p.sources.append(P.Source(2, tuple(v // 2 + 3 for v in shape), P.gaussian_pulse(steps), "E"))
    return p


@pytest.mark.parametrize("graphs", [True, False])
@pytest.mark.parametrize("case", ["lorentz_4x11", "drude_3x9", "lorentz_1x2_deep"])
def test_eh_step_identical_to_sweeps_many_tiles(fdtd, case, graphs):
    """Several x and y tiles per plane and H a few planes behind E (about
    resident CTAs / tiles per plane + 1: 15 planes of 62 for the two-pole
    grid, 23 of 48 for the Drude grid, at 4 CTAs per SM), or the lag capped
    at the plane count (all E tiles before all H tiles); the Drude grid's
    last tile has one 4-row half, the deep grid's a half with 2 of 4 rows;
    70 steps = one replayed 64-step graph plus eager steps when graphs are
    on."""
    if case == "lorentz_4x11":
        p = P.config5(steps=70, shape=(512, 90, 64), block=16, npml=8)
    elif case == "drude_3x9":
        p = _drude_no_tfsf((384, 70, 50), 70)
    else:
        p = P.config5(steps=70, shape=(100, 12, 120), block=8, npml=3)
    ref, new = _pair(fdtd, p, 70, graphs)
    _assert_identical(p, ref, new)


def test_eh_step_mixes_with_half_steps_and_sweeps(fdtd):
    """Steps of the one-launch kernel, half steps and staged sweeps on one
    grid give the staged sweeps' result (the epoch of the tile flags only
    advances with one-launch steps)."""
    p = P.config5(steps=40, shape=(140, 30, 24), block=8, npml=5)
    ref, new = _pair(fdtd, p, 10)
    # the same calls on both grids, so that the DFT samples are folded into
    # the spectra in the same groups
    for g in (ref, new):
        g.step_half(0)
        g.step_half(1)
    new.set_sweep_kernel("staged")
    for g in (ref, new):
        g.step(5)
    new.set_sweep_kernel("eh")
    for g in (ref, new):
        g.step(9)
    _assert_identical(p, ref, new)


@pytest.mark.parametrize("make", [scenarios.td_tfsf_box, scenarios.td_boundaries, scenarios.td_box_sources],
                         ids=lambda f: f.__name__)
def test_eh_step_refuses_grids_with_extra_kernels(fdtd, make):
    p = make()
    p.time_scheme = 1
    g = fdtd.Grid.from_problem(p, "f32")
    g.set_sweep_kernel("eh")
    with pytest.raises(fdtd.FdtdError) as e:
        g.step(2)
    assert e.value.code == -3
