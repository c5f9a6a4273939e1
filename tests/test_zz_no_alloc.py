"""fdtd_step_static_scratch (the step that allocates no device memory)
against fdtd_step. Collected last on purpose: the entry point's fixed device
array is shared by every grid of the device, so this file also checks that it
still gives fdtd_step's results after all other tests have run."""
import numpy as np
import pytest

import scenarios
from helpers import mode_fields, rel_l2

pytestmark = pytest.mark.gpu

TOL = {"f64": 1e-12, "f32": 1e-4}


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("make", [scenarios.tm_tfsf_reference_polarisation, scenarios.td_tfsf_box],
                         ids=lambda f: f.__name__)
def test_static_scratch_step_matches_step(fdtd, make, prec):
    """Two calls in a row of each entry point give the same fields and spectra."""
    p = make()
    ref = fdtd.Grid.from_problem(p, prec)
    new = fdtd.Grid.from_problem(p, prec)
    # lay out what set-up deferred (CPML slabs, DFT buffers) before the
    # first no-allocation step
    new.prepare()
    E, H, _, _ = mode_fields(p.mode)
    n = p.steps // 2
    for _ in range(2):
        ref.step(n)
        new.step_static_scratch(n)
        assert new.step_count == ref.step_count
        for name in E + H:
            a, b = new.get(name), ref.get(name)
            if np.any(b):
                assert rel_l2(a, b) <= TOL[prec], name
        for q in range(len(p.dfts)):
            assert rel_l2(new.dft(q), ref.dft(q)) <= TOL[prec]
    assert new.error_flags() == 0


def test_static_scratch_step_refuses_oversize_calls(fdtd):
    p = scenarios.td_tfsf_box()
    p.dfts = []
    g = fdtd.Grid.from_problem(p, "f32")
    with pytest.raises(fdtd.FdtdError) as e:
        g.step_static_scratch(1 << 20)
    assert e.value.code == -1
    assert "steps per call" in str(e.value)
    assert g.step_count == 0


def test_static_scratch_step_needs_dft_layout(fdtd):
    p = scenarios.td_tfsf_box()
    assert p.dfts
    g = fdtd.Grid.from_problem(p, "f32")
    with pytest.raises(fdtd.FdtdError) as e:
        g.step_static_scratch(4)
    assert e.value.code == -1
    g.step(1)
    g.step_static_scratch(4)
    assert g.step_count == 5


def test_static_scratch_step_after_prepare(fdtd):
    """fdtd_prepare lays out the CPML slabs and DFT buffers, after which the
    no-allocation step runs on a grid that never took an ordinary step."""
    p = scenarios.td_tfsf_box()
    ref = fdtd.Grid.from_problem(p, "f32")
    new = fdtd.Grid.from_problem(p, "f32")
    with pytest.raises(fdtd.FdtdError):
        new.step_static_scratch(4)  # CPML and DFT layout pending
    new.prepare()
    ref.step(20)
    new.step_static_scratch(20)
    for name in ("Ex", "Ez", "Hy"):
        assert rel_l2(new.get(name), ref.get(name)) <= TOL["f32"], name
    assert rel_l2(new.dft(0), ref.dft(0)) <= TOL["f32"]


def test_static_scratch_step_on_caller_stream(fdtd):
    """A stream of the caller (not the grid's own) gives fdtd_step's results;
    the grid's set-up work is ordered before it."""
    import torch
    p = scenarios.td_tfsf_box()
    ref = fdtd.Grid.from_problem(p, "f32")
    new = fdtd.Grid.from_problem(p, "f32")
    new.prepare()
    s = torch.cuda.Stream()
    n = p.steps // 2
    for _ in range(2):
        ref.step(n)
        new.step_static_scratch(n, stream=s.cuda_stream)
    s.synchronize()
    for name in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
        assert rel_l2(new.get(name), ref.get(name)) <= TOL["f32"], name
    for q in range(len(p.dfts)):
        assert rel_l2(new.dft(q), ref.dft(q)) <= TOL["f32"]


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_static_scratch_step_refuses_between_halves(fdtd, prec):
    p = scenarios.td_tfsf_box()
    g = fdtd.Grid.from_problem(p, prec)
    g.prepare()
    g.step_half(0)
    with pytest.raises(fdtd.FdtdError) as e:
        g.step_static_scratch(2)
    assert e.value.code == -1
    assert "half" in str(e.value)
    g.step_half(1)
    g.step_static_scratch(2)
    assert g.step_count == 3


def test_static_scratch_step_refuses_oversize_calls_f64(fdtd):
    p = scenarios.td_tfsf_box()
    p.dfts = []
    g = fdtd.Grid.from_problem(p, "f64")
    with pytest.raises(fdtd.FdtdError) as e:
        g.step_static_scratch(1 << 20)
    assert e.value.code == -1
    assert "steps per call" in str(e.value)
    assert g.step_count == 0


def test_static_scratch_step_allocates_nothing(fdtd):
    """Free device memory (cudaMemGetInfo) is the same before and after a
    call that takes more steps than any call before it (fdtd_step would grow
    its TFSF table with cudaMalloc there)."""
    import torch
    p = scenarios.td_tfsf_box()
    g = fdtd.Grid.from_problem(p, "f32")
    g.prepare()
    # the first call on a device looks up the array's address, and the
    # runtime may load kernels on their first use: one call of every kernel
    # this test runs comes first
    g.step_static_scratch(p.steps)
    g.synchronize()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    g.step_static_scratch(p.steps + 8)
    g.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
