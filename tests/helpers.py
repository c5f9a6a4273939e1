import numpy as np


def rel_l2(a: np.ndarray, ref: np.ndarray) -> float:
    """||a - ref||_2 / ||ref||_2 (0 when both are zero)."""
    den = float(np.sqrt(np.sum(np.abs(ref) ** 2)))
    num = float(np.sqrt(np.sum(np.abs(a - ref) ** 2)))
    if den == 0.0:
        return 0.0 if num == 0.0 else float("inf")
    return num / den


def mode_fields(mode: int):
    """(E names, H names, D names, B names) carried by a mode."""
    from fdtd_b200.problem import TE, TM
    if mode == TM:
        return ["Ez"], ["Hx", "Hy"], ["Dz"], ["Bx", "By"]
    if mode == TE:
        return ["Ex", "Ey"], ["Hz"], ["Dx", "Dy"], ["Bz"]
    return ["Ex", "Ey", "Ez"], ["Hx", "Hy", "Hz"], ["Dx", "Dy", "Dz"], ["Bx", "By", "Bz"]


# ---------------------------------------------------------------- long runs
# Problems of the configurations' own lengths, built by name so that a
# worker process (spawned, no CUDA) can run the CPU oracle on them while the
# GPU tests run in the parent.
def long_problem(name: str):
    from fdtd_b200 import problem as P
    if name == "tm256_2000":
        return P.config1(256, steps=2000)
    if name == "drude132x44x44_1000":
        return P.config2(steps=1000, shape=(132, 44, 44))
    if name == "lorentz132x48x48_500":
        return P.config5(steps=500, shape=(132, 48, 48), block=16, npml=12)
    if name.startswith("batch3000_"):
        q = int(name.split("_")[1])
        return batch_subset()[q]
    raise KeyError(name)


def batch_subset():
    """The four smallest of the 64 batched 2D TE problems (seed 0), each of
    its own size, at their full 3000 steps."""
    from fdtd_b200 import problem as P
    allp = P.config3(64, steps=3000)
    order = sorted(range(len(allp)), key=lambda q: allp[q].interior_cells)
    return [allp[q] for q in order[:4]]


def oracle_job(job):
    """(problem name, field names) -> ({name: array}, [spectra], seconds,
    {name: largest L2 norm over the run}) of the CPU oracle after the
    problem's steps; the norms are sampled every 50 steps (runs in a worker
    process)."""
    import time
    import pyoracle
    name, names = job
    p = long_problem(name)
    t0 = time.perf_counter()
    o = pyoracle.OracleGrid(p)
    peak = {n: 0.0 for n in names}
    done = 0
    while done < p.steps:
        n_ = min(50, p.steps - done)
        o.step(n_)
        done += n_
        for n in names:
            peak[n] = max(peak[n], float(np.linalg.norm(o.get(n))))
    fields = {n: o.get(n) for n in names}
    dfts = [o.dft(q) for q in range(len(p.dfts))]
    return fields, dfts, time.perf_counter() - t0, peak
