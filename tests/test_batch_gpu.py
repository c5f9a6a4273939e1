"""Batched 2D grids (fdtd_batch_*): one graph launch (a persistent kernel, or
one kernel per half step) advances many independent grids of uneven sizes; each must match the oracle as if stepped
alone, tuning must leave the state untouched, and the bounded grid barrier
must never report an expiry in a normal run."""
import numpy as np
import pytest

from fdtd_b200 import problem as P
from helpers import mode_fields, rel_l2

pytestmark = pytest.mark.gpu


def small_te_batch(steps=60):
    return P.config3(nproblems=5, steps=steps, seed=3, nmin=40, nmax=150, npml=6, nrect=4)


def small_tm_batch(steps=50):
    rng = np.random.default_rng(7)
    out = []
    for q in range(4):
        nx, ny = (int(v) for v in rng.integers(36, 140, size=2))
        dt = P.courant_dt(1e-6, 0.99 / np.sqrt(2.0))
        p = P.Problem(P.TM, (nx, ny, 1), 1e-6, dt, name=f"tm{q}")
        for a in (0, 1):
            for s in (0, 1):
                p.pml[(a, s)] = 5
        p.materials = [P.Material.vacuum(), P.Material.drude(1.0, 0.3 / dt, 0.01 / dt),
                       P.Material.lorentz(2.0, [(1.2, 0.1 / dt, 0.005 / dt), (0.5, 0.2 / dt, 0.01 / dt)])]
        ids = np.zeros((1, ny, nx), np.uint8)
        ids[0, 10:20, 12:22] = 1
        ids[0, ny - 22:ny - 12, nx - 25:nx - 14] = 2
        p.ids = ids
        p.sources.append(P.Source(2, (nx // 2, ny // 2, 0), P.gaussian_pulse(steps, 20, 6), "E"))
        p.sources.append(P.Source(0, (nx // 3, ny // 3, 0), 1e-3 * P.gaussian_pulse(steps, 25, 6), "H"))
        p.steps = steps
        out.append(p)
    return out


@pytest.mark.parametrize("make", [small_te_batch, small_tm_batch], ids=["te", "tm"])
def test_batch_matches_oracle(fdtd, oracle, make):
    probs = make()
    grids = [fdtd.Grid.from_problem(p, "f32") for p in probs]
    b = fdtd.Batch(grids)
    b.step(probs[0].steps - 7)
    b.step(7)
    assert b.error_flags() == 0
    for p, g in zip(probs, grids):
        o = oracle.run_oracle(p)
        E, H, _, _ = mode_fields(p.mode)
        for n in E + H:
            r = rel_l2(g.get(n), o.get(n))
            assert r <= 1e-4, (p.name, n, r)
        assert g.step_count == p.steps


def test_batch_tuning_preserves_state_and_results(fdtd):
    probs = small_te_batch(40)
    out = []
    for tune in (False, True):
        grids = [fdtd.Grid.from_problem(p, "f32") for p in probs]
        b = fdtd.Batch(grids)
        if tune:
            b.step(10)
            b.tune(3)
            info = b.info()
            assert info["rows"] in (1, 2, 4, 8) and all(v > 0 for v in info["tune_ms_per_step"].values())
            # work-item heights per size class: 1, 2, 4 or 8 tiles, one height per class
            ir = b.item_rows()
            assert ir["tuned_ms_per_step"] > 0
            assert set(ir["size_class"]) == set(range(min(4, len(grids))))
            for r, c in zip(ir["rows"], ir["size_class"]):
                assert r in (info["rows"], 2 * info["rows"], 4 * info["rows"], 8 * info["rows"])
                assert len({r2 for r2, c2 in zip(ir["rows"], ir["size_class"]) if c2 == c}) == 1
            b.step(30)
        else:
            b.step(10)
            b.step(30)
        out.append([g.get("Hz") for g in grids])
    for a, c in zip(out[0], out[1]):
        assert np.array_equal(a, c)


@pytest.mark.parametrize("persistent", [True, False])
def test_batch_item_heights_per_grid_agree(fdtd, persistent):
    """Work items 1, 2, 4 and 8 tiles high, mixed per grid (as the tuner sets
    them per size class), give the one-tile result bit for bit."""
    probs = small_te_batch(30)
    out = []
    for mixed in (False, True):
        grids = [fdtd.Grid.from_problem(p, "f32") for p in probs]
        b = fdtd.Batch(grids)
        b.configure(persistent, 2)
        if mixed:
            b.set_item_rows([2 * (1 << (q % 4)) for q in range(len(grids))])
            assert b.item_rows()["rows"] == [2 * (1 << (q % 4)) for q in range(len(grids))]
        b.step(30)
        assert b.error_flags() == 0
        out.append([g.get("Hz") for g in grids] + [g.get("Ex") for g in grids])
        b.close()
    for a, c in zip(out[0], out[1]):
        assert np.array_equal(a, c)
    grids = [fdtd.Grid.from_problem(p, "f32") for p in probs]
    b = fdtd.Batch(grids)
    b.configure(True, 2)
    with pytest.raises(fdtd.FdtdError):
        b.set_item_rows([3] * len(grids))


@pytest.mark.parametrize("make", [small_te_batch, small_tm_batch], ids=["te", "tm"])
def test_batch_launch_modes_and_tiles_agree(fdtd, make):
    """The persistent kernel and the per-half-step launches, with every tile
    height, run the same update: bit-identical fields."""
    probs = make()
    ref = None
    for persistent in (True, False):
        for rows in (1, 2, 4, 8):
            grids = [fdtd.Grid.from_problem(p, "f32") for p in probs]
            b = fdtd.Batch(grids)
            b.configure(persistent, rows)
            b.step(probs[0].steps)
            assert b.error_flags() == 0
            assert b.info()["launch"] == ("persistent" if persistent else "per_phase")
            E, H, _, _ = mode_fields(probs[0].mode)
            out = [g.get(n) for g in grids for n in E + H]
            if ref is None:
                ref = out
            else:
                for a, c in zip(ref, out):
                    assert np.array_equal(a, c), (persistent, rows)
            b.close()


def test_batch_rejects_unsupported_grids(fdtd):
    p = small_te_batch(10)[0]
    g64 = fdtd.Grid.from_problem(p, "f64")
    with pytest.raises(fdtd.FdtdError):
        fdtd.Batch([g64])
    g3 = fdtd.Grid(P.THREED, (16, 16, 16), 1e-6, 1e-15, "f32")
    with pytest.raises(fdtd.FdtdError):
        fdtd.Batch([g3])
    g = fdtd.Grid.from_problem(p, "f32")
    g.add_dft(5, (2, 2, 0), (5, 5, 0), [0.1])
    with pytest.raises(fdtd.FdtdError):
        fdtd.Batch([g])


def _single_vs_batch_problems():
    import scenarios
    tm, _ = scenarios.tm_adjoint_small(n=56, steps=90)
    tm.sources = [P.Source(2, (9, 20, 0), P.sinusoid(90, 0.05), "E"),
                  P.Source(2, (30, 33, 0), 1e-2 * P.gaussian_pulse(90, 30, 8), "D")]
    te = small_te_batch(90)[1]
    return [tm, te]


@pytest.mark.parametrize("which", [0, 1], ids=["tm_eps_map", "te_rects"])
def test_batch_of_one_matches_the_single_grid(fdtd, which):
    """A grid advanced in a batch equals the same grid advanced alone up to
    float rounding (the batch's 128-bit group updates and the single-grid
    sweeps may contract different products into FMAs); the adjoint's
    persistent recompute is built on the same group updates."""
    p = _single_vs_batch_problems()[which]
    a = fdtd.Grid.from_problem(p, "f32")
    a.step(p.steps)
    g = fdtd.Grid.from_problem(p, "f32")
    b = fdtd.Batch([g])
    b.step(p.steps)
    assert b.error_flags() == 0
    E, H, _, _ = mode_fields(p.mode)
    for n in E + H:
        assert rel_l2(g.get(n), a.get(n)) <= 1e-6, n


def small_tm_dielectric_batch(steps=50):
    """TM grids without poles: dielectric blocks, an eps map on one grid,
    sources of all four targets, CPML on some faces only."""
    import scenarios
    rng = np.random.default_rng(11)
    dt = P.courant_dt(1e-6, 0.99 / np.sqrt(2.0))
    out = []
    for q in range(3):
        nx, ny = (int(v) for v in rng.integers(40, 150, size=2))
        p = P.Problem(P.TM, (nx, ny, 1), 1e-6, dt, name=f"tmd{q}")
        for a in (0, 1):
            for s in (0, 1):
                if not (q == 1 and s == 1):
                    p.pml[(a, s)] = 5 + q
        p.materials = [P.Material.vacuum(), P.Material.constant(4.0), P.Material.constant(2.5)]
        ids = np.zeros((1, ny, nx), np.uint8)
        ids[0, 12:24, 10:21] = 1
        ids[0, ny - 20:ny - 9, nx - 23:nx - 12] = 2
        p.ids = ids
        p.sources += [P.Source(2, (nx // 2, ny // 2, 0), P.gaussian_pulse(steps, 20, 6), "E"),
                      P.Source(0, (nx // 3, ny // 3, 0), 1e-3 * P.gaussian_pulse(steps, 25, 6), "H"),
                      P.Source(2, (2 * nx // 3, ny // 4, 0), 1e-12 * P.gaussian_pulse(steps, 15, 5), "D"),
                      P.Source(1, (nx // 4, 2 * ny // 3, 0), 1e-9 * P.gaussian_pulse(steps, 18, 5), "B"),
                      P.Source(2, (nx // 2, ny // 2, 0), 0.5 * P.gaussian_pulse(steps, 30, 6), "E")]
        p.steps = steps
        out.append(p)
    tm, _ = scenarios.tm_adjoint_small(n=56, steps=steps)
    tm.sources = [P.Source(2, (9, 20, 0), P.sinusoid(steps, 0.05), "E")]
    out.append(tm)
    return out


@pytest.mark.parametrize("make", [small_te_batch, small_tm_dielectric_batch], ids=["te", "tm"])
@pytest.mark.parametrize("depth", [2, 3, 4])
def test_batch_temporal_blocking_matches_per_phase(fdtd, make, depth):
    """Temporal blocking (depth steps per launch from shared memory, the
    windows reading one copy of the state and writing the other) gives the
    per-half-step launches' fields bit for bit, over calls that end inside a
    pair of launches and calls of whole pairs."""
    probs = make()
    E, H, _, _ = mode_fields(probs[0].mode)
    out = []
    for tb in (0, depth):
        grids = [fdtd.Grid.from_problem(p, "f32") for p in probs]
        b = fdtd.Batch(grids)
        b.configure(False, 2)
        if tb:
            b.set_temporal(tb)
            assert b.temporal()["depth"] == tb
        b.step(7)
        b.step(4 * depth)
        b.step(probs[0].steps - 7 - 4 * depth)
        assert b.error_flags() == 0
        assert all(g.step_count == probs[0].steps for g in grids)
        out.append([g.get(n) for g in grids for n in E + H])
        b.close()
    for q, (a, c) in enumerate(zip(*out)):
        assert np.array_equal(a, c), (q, float(np.abs(a - c).max()))


def test_batch_temporal_blocking_matches_oracle(fdtd, oracle):
    probs = small_tm_dielectric_batch(60)
    grids = [fdtd.Grid.from_problem(p, "f32") for p in probs]
    b = fdtd.Batch(grids)
    b.set_temporal(3)
    b.step(60)
    for p, g in zip(probs, grids):
        o = oracle.run_oracle(p)
        E, H, _, _ = mode_fields(p.mode)
        for n in E + H:
            r = rel_l2(g.get(n), o.get(n))
            assert r <= 1e-4, (p.name, n, r)


def test_batch_temporal_blocking_refusals(fdtd):
    grids = [fdtd.Grid.from_problem(p, "f32") for p in small_tm_batch(10)]
    b = fdtd.Batch(grids)
    with pytest.raises(fdtd.FdtdError):
        b.set_temporal(2)  # dispersive materials
    b = fdtd.Batch([fdtd.Grid.from_problem(small_te_batch(10)[0], "f32")])
    for bad in (1, 5, -1):
        with pytest.raises(fdtd.FdtdError):
            b.set_temporal(bad)
    b.set_temporal(4)
    b.configure(False, 2)
    assert b.temporal()["depth"] == 0


def test_batch_tuner_times_temporal_blocking(fdtd):
    probs = small_te_batch(48)
    out = []
    for tune in (False, True):
        grids = [fdtd.Grid.from_problem(p, "f32") for p in probs]
        b = fdtd.Batch(grids)
        if tune:
            b.tune(6)
            tm = b.temporal()
            assert all(v > 0 for v in tm["tune_ms_per_step"].values())
            assert tm["depth"] in (0, 2, 3, 4)
        b.step(48)
        out.append([g.get("Hz") for g in grids])
    for a, c in zip(out[0], out[1]):
        assert np.array_equal(a, c)
