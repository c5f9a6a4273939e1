"""GPU adjoint (fdtd_adjoint_*, FP32 fused 2D TM) against
* the FP64 CPU adjoint of the oracle's TM step (oracle_adjoint_tm, itself
  checked against central differences in tests/test_oracle_cpu.py), at a size
  the CPU runs in a fraction of a second: <= 1e-3 relative L2;
* the same at 128^2 over 1000 steps, cell by cell;
* central finite differences (h = 1e-4 in eps_r) of the FP64 plain GPU method
  on the full inverse-design workload (512^2, 4000 steps, 128^2 design box,
  checkpoints every 64 steps) at 32 random design cells: <= 1e-3 relative L2
  over the 32 and <= 1e-3 relative error at each of them.
"""
import copy

import numpy as np
import pytest

import scenarios
from helpers import rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-3


def _gpu_gradient(fdtd, p, spec, ckpt_every=None):
    g = fdtd.Grid.from_problem(p, "f32")
    adj = fdtd.Adjoint(g, spec.probe_lo[:2], spec.probe_hi[:2], spec.freq, spec.design_lo[:2], spec.design_hi[:2],
                       ckpt_every or spec.ckpt_every)
    J = adj.forward(p.steps)
    grad = adj.backward()
    return J, grad, g, adj


def test_gpu_adjoint_matches_fp64_cpu_adjoint(fdtd, oracle):
    p, spec = scenarios.tm_adjoint_small()
    Jc, gc = oracle.adjoint_tm(p, p.steps, spec.probe_lo[:2], spec.probe_hi[:2], spec.freq, spec.design_lo[:2],
                               spec.design_hi[:2])
    Jg, gg, _, _ = _gpu_gradient(fdtd, p, spec)
    assert abs(Jg - Jc) <= 1e-4 * Jc
    assert rel_l2(gg, gc) <= TOL


def test_gpu_adjoint_matches_fp64_cpu_adjoint_128(fdtd, oracle):
    """128^2 grid, 1000 steps, 32^2 design box: every design cell's gradient
    within 1e-3 of the FP64 CPU adjoint, relative to the largest |dJ/deps|
    (cells where the gradient passes through zero have no relative error of
    their own), and <= 1e-3 relative L2 over the box."""
    p, spec = scenarios.tm_adjoint_small(n=128, steps=1000, design=32)
    Jc, gc = oracle.adjoint_tm(p, p.steps, spec.probe_lo[:2], spec.probe_hi[:2], spec.freq, spec.design_lo[:2],
                               spec.design_hi[:2])
    Jg, gg, _, _ = _gpu_gradient(fdtd, p, spec)
    assert abs(Jg - Jc) <= 1e-4 * Jc
    assert rel_l2(gg, gc) <= TOL
    worst = float(np.max(np.abs(gg - gc)) / np.max(np.abs(gc)))
    print("128^2 adjoint: rel L2", rel_l2(gg, gc), "max cell error / max |grad|", worst)
    assert worst <= TOL


def test_checkpoint_spacing_does_not_change_the_gradient(fdtd):
    p, spec = scenarios.tm_adjoint_small()
    _, a, _, _ = _gpu_gradient(fdtd, p, spec, 7)
    _, b, _, _ = _gpu_gradient(fdtd, p, spec, 64)
    assert np.array_equal(a, b)


def test_graph_replayed_backward_equals_eager(fdtd):
    p, spec = scenarios.tm_adjoint_small()
    _, a, _, _ = _gpu_gradient(fdtd, p, spec)
    g = fdtd.Grid.from_problem(p, "f32")
    g.use_graphs(False)
    adj = fdtd.Adjoint(g, spec.probe_lo[:2], spec.probe_hi[:2], spec.freq, spec.design_lo[:2], spec.design_hi[:2],
                       spec.ckpt_every)
    adj.forward(p.steps)
    assert np.array_equal(adj.backward(), a)


def test_backward_leaves_the_post_forward_state(fdtd):
    p, spec = scenarios.tm_adjoint_small()
    g = fdtd.Grid.from_problem(p, "f32")
    adj = fdtd.Adjoint(g, spec.probe_lo[:2], spec.probe_hi[:2], spec.freq, spec.design_lo[:2], spec.design_hi[:2], 32)
    adj.forward(p.steps)
    after = [g.get(n) for n in ("Ez", "Hx", "Hy")]
    adj.backward()
    for a, n in zip(after, ("Ez", "Hx", "Hy")):
        assert np.array_equal(g.get(n), a), n
    assert g.step_count == p.steps
    # the grid steps on from there as if the backward had not run
    g.step(5)
    ref = fdtd.Grid.from_problem(p, "f32")
    ref.step(p.steps + 5)
    assert np.array_equal(g.get("Ez"), ref.get("Ez"))


def test_adjoint_rejects_unsupported_grids(fdtd):
    p, spec = scenarios.tm_adjoint_small()
    args = (spec.probe_lo[:2], spec.probe_hi[:2], spec.freq, spec.design_lo[:2], spec.design_hi[:2], 16)
    with pytest.raises(fdtd.FdtdError) as e:
        fdtd.Adjoint(fdtd.Grid.from_problem(p, "f64"), *args)
    assert e.value.code == -3
    g = fdtd.Grid.from_problem(p, "f32")
    g.step(1)
    with pytest.raises(fdtd.FdtdError):
        fdtd.Adjoint(g, *args)
    g = fdtd.Grid.from_problem(p, "f32")
    with pytest.raises(fdtd.FdtdError) as e:
        fdtd.Adjoint(g, spec.probe_lo[:2], spec.probe_hi[:2], spec.freq, (2, 2), (10, 10), 16)  # inside the CPML
    assert e.value.code == -3
    adj = fdtd.Adjoint(g, *args)
    with pytest.raises(fdtd.FdtdError):
        adj.backward()  # before forward


def _fp64_objective(fdtd, p, spec):
    g = fdtd.Grid.from_problem(scenarios.objective_problem(p, spec), "f64")
    g.step(p.steps)
    X = g.dft(0)
    return float(np.sum(np.abs(X) ** 2))


def test_inverse_design_gradient_matches_fp64_finite_differences(fdtd):
    from fdtd_b200.problem import config4
    p, spec = config4()
    J, grad, _, _ = _gpu_gradient(fdtd, p, spec)
    assert J > 0
    rng = np.random.default_rng(4)
    h = 1e-4
    picks = rng.integers(0, grad.shape[0], size=(32, 2))
    fd = np.empty(32)
    for q, (jj, ii) in enumerate(picks):
        c = (0, spec.design_lo[1] + int(jj), spec.design_lo[0] + int(ii))
        vals = []
        for sgn in (1, -1):
            pp = copy.copy(p)
            pp.eps_map = p.eps_map.copy()
            pp.eps_map[c] += sgn * h
            vals.append(_fp64_objective(fdtd, pp, spec))
        fd[q] = (vals[0] - vals[1]) / (2 * h)
    adj = np.array([grad[int(jj), int(ii)] for jj, ii in picks])
    assert rel_l2(adj, fd) <= TOL, (adj, fd)
    # and cell by cell: each of the 32 within 1e-3 of its own difference quotient
    per_cell = np.abs(adj - fd) / np.abs(fd)
    print("FD check: rel L2", rel_l2(adj, fd), "max per-cell relative error", float(per_cell.max()),
          "smallest |fd| / largest", float(np.abs(fd).min() / np.abs(fd).max()))
    assert float(per_cell.max()) <= TOL, (per_cell, adj, fd)
