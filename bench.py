"""Benchmark of the FDTD time-step hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload drude384|lorentz768|tm256|batch64|adjoint512]

Workload (default, lorentz768): the 3D FP32 two-pole Lorentz grid -- 768^3
cells, 16-cell CPML, two Lorentz poles in every cell (delta_eps 1.5, w0*dt
0.1, delta*dt 0.005 and 0.8, 0.25, 0.02), eps_inf per 32^3 block uniform in
[1,6] from seed 0, soft Ez Gaussian dipole at the centre, 4-frequency DFT of
Ez on the central z plane; 500 steps in the configuration. drude384 is the
384^3 Drude-sphere grid with a TFSF box and face DFTs (1000 steps), tm256 the
2D TM FP64 vacuum grid (2000 steps). A "step" is one full FDTD time step (E
half + H half) over the whole grid. Metric: Gcell-updates/s over interior
cells (the outer ring is never updated, as in the reference). Synthetic
inputs; the state (32.6 GB of FP32 state at 768^3) is far larger than L2, so
no flush is needed between steps.

The line also carries: the FP64 plain method on the same grid (the metric's
comparison); `error_vs_fp64`, the FP32 method's relative L2 error of every E
and H component and of the DFT spectra against the FP64 plain grid after the
configuration's number of steps (both grids on the GPU; the FP64 plain method
is bit-identical to the CPU oracle at test sizes); `roofline`, the whole step
against the minimal formulation's algorithmic bytes per cell-step, with each
sweep's own figure beside it; `e2e`, the configuration's whole job through
the public API from host buffers (grid creation, uploads, its own number of
steps -- 500 at 768^3 -- and D2H of the spectra).

Multi-GPU (torchrun, one process per GPU): for the single-grid workloads
every rank runs its own grid of the same size (independent replicas: the
workload is one grid; sharding it by z slabs needs a halo exchange). For
batch64, 64 problems per GPU are drawn from one seed and partitioned across
the ranks by cost (fdtd_b200/shard.py); each rank steps only its share, with
no exchange on the data path. value = cells of all ranks / max rank time;
scaling "weak".

--impl reference times the reference's own functors (oracle/_ref/ref_runner,
compiled from the reference headers) on the host cores, on a reduced grid of
the same physics, and prints its line; ranks other than 0 exit at once. The
reference steps a grid on one thread, so the arm runs one copy of the sample
per host core at once and reports their combined rate ("cores").
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Gcell-updates/s (FP32 fused; FP64 plain alongside)"
ADJ_METRIC = "inverse-design gradient: Gcell-updates/s of forward + adjoint (FP32 fused)"


# steps of each workload's configuration (the bench times --steps of them)
P_STEPS = {"drude384": 1000, "lorentz768": 500, "tm256": 2000}

# DRAM bytes per interior cell of one sweep launch, from ncu captures at 256^3 (profiles/)
MEASURED_TRAFFIC = {
    ("drude384", "staged"): {"e": 669.810688e6 / 16387064, "h": 634.496512e6 / 16387064,
                             "source": "ncu capture at 256^3 scaled by interior cells "
                                       "(profiles/staged_sweeps_drude256.md)"},
    ("lorentz768", "staged"): {"e": 7597.061e6 / 55742968, "h": 2221.944e6 / 55742968,
                               "source": "ncu capture at 384^3 scaled by interior cells "
                                         "(profiles/staged_sweeps_lorentz384.md)"},
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="lorentz768", choices=["drude384", "lorentz768", "tm256", "batch64",
                                                                     "adjoint512"])
    ap.add_argument("--n", type=int, default=0, help="override the grid size (same physics, scaled): for profiling")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-f64", action="store_true")
    ap.add_argument("--accuracy-steps", type=int, default=-1,
                    help="steps at which the FP32 error against FP64 is measured (-1: the configuration's length, "
                         "0: skip)")
    ap.add_argument("--sweep", default="auto", choices=["auto", "regs", "tma", "flat", "staged", "eh"],
                    help="3D FP32 sweep kernels (fdtd_set_sweep_kernel)")
    ap.add_argument("--batch-mode", default="tune", choices=["tune", "persistent", "per_phase"],
                    help="batch64: autotune, or force a launch mode (with --batch-rows)")
    ap.add_argument("--batch-rows", type=int, default=4, choices=[1, 2, 4, 8])
    ap.add_argument("--batch-temporal", type=int, default=0, choices=[0, 2, 3, 4],
                    help="batch64 with a forced launch mode: steps per launch of temporal blocking (0: off)")
    ap.add_argument("--decompose", default="replicas", choices=["replicas", "zslab"],
                    help="single-grid workloads on N GPUs: independent replicas (weak scaling), or one grid cut "
                         "into z slabs, one per rank, ghost planes over NCCL overlapped with the interior sweep "
                         "(strong scaling)")
    ap.add_argument("--variant", default="none", choices=list(VARIANTS),
                    help="3D/2D grid workloads: measure a feature beside the hot path (see VARIANTS)")
    return ap.parse_args()


# Variants of the grid workloads that exercise the features around the hot
# path; each keeps the workload's grid, materials and sources.
VARIANTS = {
    "none": "the workload as configured",
    "pec_backed": "a PEC boundary condition on all six faces behind the CPML (boundary image kernel each half step)",
    "surface_dft": "the face DFTs capture the surface currents instead of the fields: Jh in place of each E "
                   "component, Je in place of each H component",
    "bd3": "the FP64 plain leg steps with the BD3 time policy (flux history) at Courant 0.5",
    "bd4": "the FP64 plain leg steps with the BD4 time policy (flux history) at Courant 0.5",
}


def apply_variant(p, variant: str, fp64: bool = False):
    """The problem p changed for `variant` (in place); bd3/bd4 change only the
    FP64 plain problem (the FP32 method steps with the leapfrog)."""
    if variant == "pec_backed":
        for a in range(p.dim):
            for s in (0, 1):
                p.boundaries[(a, s)] = "pec"
    elif variant == "surface_dft":
        for r in p.dfts:
            r.comp = r.comp + 9 if r.comp < 3 else r.comp + 3
    elif variant in ("bd3", "bd4") and fp64:
        p.time_scheme = 3 if variant == "bd3" else 4
        p.dt = p.dt * 0.5 / 0.99
    return p


def make_problem(workload: str, steps: int, n: int = 0, variant: str = "none", fp64: bool = False):
    from fdtd_b200 import problem as P
    if workload == "drude384":
        p = P.config2(n=n or 384, steps=steps)
    elif workload == "lorentz768":
        p = P.config5(n=n or 768, steps=steps)
    else:
        p = P.config1(n=n or 256, steps=steps)
    return apply_variant(p, variant, fp64)


def small_problem(workload: str, steps: int, variant: str = "none"):
    """Same physics on a grid the CPU finishes in seconds (the CPU path is
    the FP64 one: bd3/bd4 apply)."""
    from fdtd_b200 import problem as P
    if workload == "drude384":
        p, d = P.config2(n=64, steps=steps), "64^3 grid (sphere, CPML, insets scaled by 64/384)"
    elif workload == "lorentz768":
        p, d = P.config5(n=64, steps=steps, block=16), "64^3 grid, 16^3 eps blocks"
    else:
        p, d = P.config1(n=256, steps=steps), "256^2 grid"
    if variant != "none":
        d += f", variant {variant}"
    return apply_variant(p, variant, fp64=True), d


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """SM clock and throttle reasons of the GPU sampled every 10 ms by a
    thread through NVML while the timed region runs (falls back to
    nvidia-smi at its 200 ms floor where NVML is unavailable). Reading
    clocks changes no GPU setting."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
               "sw_power_cap": 0x4, "hw_power_brake_slowdown": 0x80}
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int, period_s: float = 0.01):
        self.device = device
        self.period = period_s
        self.samples = []  # (sm_mhz, max_mhz, reason_bits)
        self.proc = None
        self.nvml = None
        self.stop = threading.Event()
        self.thread = None

    def _handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(self.device).uuid)
            uuid = uuid if uuid.startswith("GPU-") else "GPU-" + uuid
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(uuid)
        except Exception:
            vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
            idx = self.device
            if vis and vis.split(",")[0].strip().isdigit():
                idx = int(vis.split(",")[self.device])
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(idx)

    def __enter__(self):
        try:
            nv, h = self._handle()
            self.nvml = (nv, h)
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _poll(self):
        nv, h = self.nvml
        get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            nv.nvmlDeviceGetCurrentClocksThrottleReasons
        mx = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
        while not self.stop.is_set():
            try:
                self.samples.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)), mx, int(get_reasons(h))))
            except Exception:
                pass
            time.sleep(self.period)

    def _read(self):
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.proc.stdout:
            parts = [x.strip() for x in ln.strip().split(",")]
            if len(parts) < 9:
                continue
            try:
                bits = 0
                for nm, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        bits |= self.REASONS[nm]
                self.samples.append((float(parts[1]), float(parts[2]), bits))
            except ValueError:
                continue

    def __exit__(self, *a):
        self.stop.set()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=2)

    def summary(self):
        sm = [x[0] for x in self.samples]
        mx = self.samples[-1][1] if self.samples else None
        reasons = sorted({nm for x in self.samples for nm, bit in self.REASONS.items() if x[2] & bit})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(sm), "sampler": "nvml 10 ms" if self.nvml else "nvidia-smi 200 ms"}


# ------------------------------------------------------------------ bytes model
def alg_bytes(p, word: int):
    """Algorithmic bytes of one E sweep and one H sweep launch, and of one
    cell-step of the minimal formulation (each persistent state word read
    once and written once per step, per-cell parameters read once, CPML psi
    over the slab cells only, ADE state over dispersive cells only)."""
    from fdtd_b200.problem import THREED, DRUDE, LORENTZ
    nx, ny, nz = p.shape
    cells = p.interior_cells
    ne = 3 if p.mode == THREED else (1 if p.mode == 2 else 2)
    nh = 3 if p.mode == THREED else (2 if p.mode == 2 else 1)
    dim = 3 if p.mode == THREED else 2
    # psi: for every axis with CPML, the cells of its slabs carry one psi per
    # transverse component (E sweep: components != axis; H sweep likewise)
    ext = [nx - 2, ny - 2, nz - 2 if dim == 3 else 1]
    slab_cells = 0
    for a in range(dim):
        w = sum(p.pml.get((a, s), 0) + 1 for s in (0, 1) if p.pml.get((a, s), 0) > 0)
        others = np.prod([ext[b] for b in range(dim) if b != a])
        slab_cells += min(w, ext[a]) * others
    psi_e = slab_cells * 2 * 2 * word  # 2 components, read + write
    psi_h = psi_e
    # dispersive state
    ids = p.cell_ids()
    disp_words = 0
    if ids is not None:
        counts = np.bincount(ids.ravel(), minlength=len(p.materials))
    else:
        counts = np.zeros(len(p.materials))
        counts[0] = p.ncell
    for m, cnt in zip(p.materials, counts):
        if m.kind == DRUDE:
            disp_words += cnt * ne * 2 * (1 if word == 4 else 2)  # J (and P in the plain form)
        elif m.kind == LORENTZ:
            disp_words += cnt * ne * 2 * 2 * len(m.poles)  # P and J per pole, read + write
    disp = disp_words * word
    id_bytes = cells * (1 if p.ids is not None else 0)
    if word == 4:
        e_sweep = cells * word * (ne * 2 + nh) + psi_e + disp + id_bytes
        h_sweep = cells * word * (nh * 2 + ne) + psi_h
        step_min = cells * word * (ne + nh) * 2 + psi_e + psi_h + disp + id_bytes
    else:  # plain FP64 keeps D, E, B, H: flux read+write, field write, curl read
        # BD3/BD4 keep 2/3 past fluxes per component, each read and written
        hist = {3: 2, 4: 3}.get(getattr(p, "time_scheme", 1), 0) * 2
        e_sweep = cells * word * (ne * (3 + hist) + nh) + psi_e + disp + id_bytes
        h_sweep = cells * word * (nh * (3 + hist) + ne) + psi_h + id_bytes
        step_min = e_sweep + h_sweep
    return {"e_sweep": float(e_sweep), "h_sweep": float(h_sweep), "step": float(step_min),
            "per_cell_step": float(step_min) / cells}


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ------------------------------------------------------------------ CPU legs
def cpu_rate(problem, steps: int, kind: str):
    """Cell-updates/s of the reference runner (kind 'reference') or of the C
    restatement ('port') on a bounded sample."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    if kind == "reference":
        dt = pyoracle.run_reference(problem, steps)["loop_seconds"]
    else:
        dt = pyoracle.run_oracle(problem, steps).loop_seconds
    return problem.interior_cells * steps / dt, dt


def host_cores() -> int:
    """The CPUs this process may run on."""
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_baseline(workload: str, budget_s: float = 15.0, variant: str = "none", replicas: int = 1):
    """The reference's functors (or the C restatement) on a bounded sample of
    the workload. The reference steps one grid on one thread (it has no
    threading of its own), so with replicas > 1 that many copies of the
    sample run at once, one process each, and the rate is their combined
    cell-updates over the slowest copy's time loop."""
    import concurrent.futures as cf
    import multiprocessing as mp
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    kind = "reference" if pyoracle.reference_available() else "port"
    p, desc = small_problem(workload, 10, variant)
    if kind == "reference" and p.materials and max(len(m.poles) for m in p.materials) > 1:
        kind = "port"  # the reference holds one pole per cell
    # calibrate on a few steps, then run a sample of about budget_s
    rate0, _ = cpu_rate(small_problem(workload, 4, variant)[0], 4, kind)
    steps = max(4, int(budget_s * rate0 / p.interior_cells))
    p, desc = small_problem(workload, steps, variant)
    if replicas <= 1:
        rate, dt = cpu_rate(p, steps, kind)
        return {"value": rate / 1e9, "unit": "Gcell-updates/s", "cores": 1, "kind": kind,
                "sample": f"{desc}, {steps} steps, {dt:.1f} s, single thread"}
    with cf.ProcessPoolExecutor(max_workers=replicas, mp_context=mp.get_context("spawn")) as ex:
        loops = list(ex.map(_cpu_one, [(p, steps, kind)] * replicas))
    slow = max(loops)
    return {"value": p.interior_cells * steps * replicas / slow / 1e9, "unit": "Gcell-updates/s", "cores": replicas,
            "kind": kind,
            "sample": f"{desc}, {steps} steps, {replicas} copies at once (one process and thread each: the "
                      f"reference steps a grid on one thread), slowest time loop {slow:.1f} s; rate = copies x "
                      f"cells x steps / slowest time loop"}


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if args.workload == "batch64":
        from fdtd_b200 import problem as P
        cb = cpu_batch_baseline(P.config3(64, steps=args.steps + 16), budget_s=20.0)
    elif args.workload == "adjoint512":
        cb = cpu_adjoint_baseline(budget_s=20.0, replicas=min(128, host_cores()))
    else:
        cb = cpu_baseline(args.workload, budget_s=max(5.0, min(30.0, 3.0 * max(1, args.steps) / 100)),
                          variant=args.variant, replicas=min(128, host_cores()))
    metric = ADJ_METRIC if args.workload == "adjoint512" else METRIC
    line = {"impl": "reference", "metric": metric, "value": cb["value"], "unit": "Gcell-updates/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "dtype": "f64", "data": "synthetic", "scaling": "weak",
            "config": {"workload": args.workload, "reference_sample": cb["sample"]},
            "cpu_baseline": cb, "e2e": {"value": cb["value"], "unit": "Gcell-updates/s",
                                        "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "vs_baseline": None}
    print(json.dumps(line), flush=True)


def _adjoint_problem(n: int, steps: int):
    from fdtd_b200 import problem as P
    scale = n / 512
    return P.config4(n=n, steps=steps, npml=max(6, int(16 * scale)), design=max(8, int(128 * scale)),
                     nprobe=max(4, int(16 * scale)))


def _adjoint_one(job):
    n, steps = job
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    p, s = _adjoint_problem(n, steps)
    t0 = time.perf_counter()
    pyoracle.adjoint_tm(p, steps, s.probe_lo[:2], s.probe_hi[:2], s.freq, s.design_lo[:2], s.design_hi[:2])
    return time.perf_counter() - t0, p.interior_cells


def cpu_adjoint_baseline(budget_s: float = 20.0, replicas: int = 1):
    """The FP64 CPU adjoint (the oracle's restatement: the reference has no
    adjoint) on a reduced inverse-design grid; value = gradient cell-steps/s
    (forward + backward). One thread per gradient; with replicas > 1 that many
    gradients run at once, one process each, and the rate is their combined
    cell-steps over the slowest."""
    import concurrent.futures as cf
    import multiprocessing as mp
    n = 128
    dt0, cells = _adjoint_one((n, 40))
    steps = max(40, int(budget_s / dt0 * 40))
    if replicas <= 1:
        dt, cells = _adjoint_one((n, steps))
        return {"value": cells * steps / dt / 1e9, "unit": "Gcell-updates/s", "cores": 1, "kind": "port",
                "sample": f"{n}^2 inverse-design grid, {steps} steps forward + adjoint, {dt:.1f} s, single thread"}
    with cf.ProcessPoolExecutor(max_workers=replicas, mp_context=mp.get_context("spawn")) as ex:
        runs = list(ex.map(_adjoint_one, [(n, steps)] * replicas))
    slow = max(r[0] for r in runs)
    return {"value": cells * steps * replicas / slow / 1e9, "unit": "Gcell-updates/s", "cores": replicas,
            "kind": "port",
            "sample": f"{n}^2 inverse-design grid, {steps} steps forward + adjoint, {replicas} gradients at once "
                      f"(one process and thread each), slowest {slow:.1f} s; rate = copies x cells x steps / slowest"}


def run_adjoint(args, torch, world, rank, local):
    """Inverse-design gradient, 2D TM FP32: one forward (checkpoints every 64
    steps) and one backward of `steps` time steps on the 512^2 grid; value =
    interior cells x steps / gradient time. Host clock around the synchronous
    forward and backward calls (both end with a device synchronize)."""
    import torch.distributed as dist
    from fdtd_b200 import grid as G
    steps = args.steps
    p, spec = _adjoint_problem(args.n or 512, steps)
    for _ in range(max(1, args.warmup // 10)):
        pw, sw = _adjoint_problem(args.n or 512, 64)
        gw = G.Grid.from_problem(pw, "f32", device=local)
        aw = G.Adjoint(gw, sw.probe_lo[:2], sw.probe_hi[:2], sw.freq, sw.design_lo[:2], sw.design_hi[:2], 64)
        aw.forward(64)
        aw.backward()
        aw.close()
        gw.close()
    g = G.Grid.from_problem(p, "f32", device=local)
    adj = G.Adjoint(g, spec.probe_lo[:2], spec.probe_hi[:2], spec.freq, spec.design_lo[:2], spec.design_hi[:2],
                    spec.ckpt_every)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = g.launch_count
    with ClockSampler(local) as clk:
        t0 = time.perf_counter()
        J = adj.forward(steps)
        t1 = time.perf_counter()
        grad = adj.backward()
        t2 = time.perf_counter()
    launches = g.launch_count - l0
    tt = torch.tensor([t2 - t0], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    wall = float(tt.item())
    cells = p.interior_cells
    cpu = cpu_adjoint_baseline() if (rank == 0 and world == 1 and not args.no_cpu_baseline) else None
    return {
        "metric": ADJ_METRIC, "value":
            cells * steps * world / wall / 1e9, "unit": "Gcell-updates/s", "n_gpus": world, "steps": steps,
        "warmup": args.warmup, "ms_per_step": wall * 1e3 / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "adjoint512_tm_design128", "grid": list(p.shape), "interior_cells": cells,
                   "design_box": [spec.design_lo[:2], spec.design_hi[:2]], "probes": 16, "freq": spec.freq,
                   "ckpt_every": spec.ckpt_every, "l2": "512^2 state fits L2 (launch-bound)",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "gradient_s": wall, "forward_s": t1 - t0, "backward_s": t2 - t1, "J": J,
        "grad_abs_max": float(np.abs(grad).max()),
        "e2e": {"value": cells * steps * world / wall / 1e9, "unit": "Gcell-updates/s",
                "h2d_bytes_per_step": float(p.eps_map.nbytes) / steps, "d2h_bytes_per_step": float(grad.nbytes) / steps,
                "note": "the forward and backward calls are the public API; eps map uploaded at grid creation"},
        "cpu_baseline": cpu, "gpu_launches": launches, "clocks": clk.summary(),
    }


def batch_alg_bytes(problems):
    """Algorithmic bytes of one step of a batch of 2D TE grids: E (2 words)
    and H (1 word) read and written once, material ids once, CPML psi over
    the slab cells."""
    total = 0.0
    for p in problems:
        nx, ny, _ = p.shape
        cells = (nx - 2) * (ny - 2)
        slab = 0
        for a, ext, other in ((0, nx - 2, ny - 2), (1, ny - 2, nx - 2)):
            w = sum(p.pml.get((a, s), 0) + 1 for s in (0, 1) if p.pml.get((a, s), 0) > 0)
            slab += min(w, ext) * other
        total += cells * (4 * 6 + 1) + slab * 4 * 2 * 2
    return total


def cpu_batch_baseline(problems, budget_s: float = 20.0):
    """The reference's functors on the batch's problems, one process per
    problem spread over all host cores, on a bounded number of steps."""
    import concurrent.futures as cf
    import multiprocessing as mp
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    kind = "reference" if pyoracle.reference_available() else "port"
    cores = host_cores()
    cells = sum(p.interior_cells for p in problems)
    ctx = mp.get_context("spawn")

    def run(nsteps):
        # time-loop seconds of every problem, run concurrently on the cores;
        # the aggregate rate assumes perfect packing of the loops on the cores
        with cf.ProcessPoolExecutor(max_workers=cores, mp_context=ctx) as ex:
            return sum(ex.map(_cpu_one, [(p, nsteps, kind) for p in problems]))
    steps = 2
    loops = run(steps)
    steps = max(2, int(steps * budget_s * cores / max(loops, 1e-3)))
    loops = run(steps)
    return {"value": cells * steps / (loops / cores) / 1e9, "unit": "Gcell-updates/s", "cores": cores, "kind": kind,
            "sample": f"all {len(problems)} problems, {steps} steps each, one process per problem over {cores} cores; "
                      f"rate = cells*steps / (sum of time-loop seconds / cores)"}


def _cpu_one(job):
    p, nsteps, kind = job
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    if kind == "reference":
        return pyoracle.run_reference(p, nsteps)["loop_seconds"]
    return pyoracle.run_oracle(p, nsteps).loop_seconds


def run_batch(args, torch, world, rank, local, stream):
    import torch.distributed as dist
    from fdtd_b200 import grid as G, problem as P
    from fdtd_b200.shard import imbalance, partition_by_cost, problem_cost

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # 64 problems per GPU, drawn from one seed and partitioned by cost: each
    # rank steps only its own share (no exchange on the data path)
    allp = P.config3(64 * world, steps=args.steps + args.warmup + 16)
    shares = partition_by_cost([problem_cost(p) for p in allp], world)
    probs = [allp[q] for q in shares[rank]]
    grids = [G.Grid.from_problem(p, "f32", device=local) for p in probs]
    batch = G.Batch(grids)
    if args.batch_mode == "tune":
        batch.tune(4)
    else:
        batch.configure(args.batch_mode, args.batch_rows)
        if args.batch_temporal:
            batch.set_temporal(args.batch_temporal)
    batch.step(args.warmup, stream=stream.cuda_stream)
    barrier()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        with torch.cuda.stream(stream):
            start.record(stream)
            batch.step(args.steps, stream=stream.cuda_stream)
            end.record(stream)
        barrier()
    ms = max_over_ranks(start.elapsed_time(end))
    assert batch.error_flags() == 0
    cells = sum(p.interior_cells for p in probs)
    total_cells = sum(p.interior_cells for p in allp)
    value = total_cells * args.steps / (ms / 1e3) / 1e9
    ab = batch_alg_bytes(probs)
    peak, peak_kind = peaks()
    ach = ab * args.steps / (ms / 1e3) / 1e9
    info = batch.info()
    ir = batch.item_rows()
    tbi = batch.temporal()
    tb = tbi["depth"]
    classes = {}
    for p_, r_, c_ in zip(probs, ir["rows"], ir["size_class"]):
        e = classes.setdefault(str(c_), {"problems": 0, "cells_min": None, "cells_max": 0, "item_rows": set()})
        e["problems"] += 1
        e["cells_min"] = p_.interior_cells if e["cells_min"] is None else min(e["cells_min"], p_.interior_cells)
        e["cells_max"] = max(e["cells_max"], p_.interior_cells)
        e["item_rows"].add(r_)
    for e in classes.values():
        e["item_rows"] = sorted(e["item_rows"])
    batch.close()
    for g in grids:
        g.close()
    # FP64 plain, one grid at a time (no batch kernel for the plain method)
    f64 = None
    if not args.no_f64:
        n64 = max(3, min(50, args.steps))
        g64 = [G.Grid.from_problem(p, "f64", device=local) for p in probs]
        for g in g64:
            g.step(2, stream=stream.cuda_stream)
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            start.record(stream)
            for g in g64:
                g.step(n64, stream=stream.cuda_stream)
            end.record(stream)
        torch.cuda.synchronize()
        ms64 = start.elapsed_time(end)
        for g in g64:
            g.close()
        f64 = {"value": cells * n64 / (ms64 / 1e3) / 1e9, "steps": n64, "note": "grids stepped one by one"}
    # end to end: create this rank's grids from host arrays, run, read every Hz back
    e2e = None
    if not args.no_e2e:
        barrier()
        t0 = time.perf_counter()
        ge = [G.Grid.from_problem(p, "f32", device=local) for p in probs]
        be = G.Batch(ge)
        if tb:
            be.set_temporal(tb)
        be.step(args.steps)
        out = [g.get("Hz") for g in ge]
        t_e2e = max_over_ranks(time.perf_counter() - t0)
        h2d = sum(p.ids.nbytes + sum(s.values.nbytes for s in p.sources) for p in probs)
        d2h = sum(o.size * 8 for o in out)
        be.close()
        for g in ge:
            g.close()
        e2e = {"value": total_cells * args.steps / t_e2e / 1e9, "unit": "Gcell-updates/s",
               "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps, "wall_s": t_e2e,
               "note": "grid creation from host arrays, the steps without tuning (the tuned temporal-blocking "
                       "depth kept), D2H of every Hz; host clock"}
    cpu = cpu_batch_baseline(probs) if (rank == 0 and world == 1 and not args.no_cpu_baseline) else None
    return {
        "metric": METRIC, "value": value, "unit": "Gcell-updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "batch64_te_rects", "problems": len(allp), "problems_per_gpu": 64,
                   "interior_cells": total_cells, "seed": 0, "shard_imbalance": imbalance(
                       [problem_cost(p) for p in allp], shares),
                   "cpml": 10, "steps_in_config": 3000, "tile_rows": info["rows"], "ctas": info["blocks"],
                   "launch": f"temporal blocking, {tb} steps per launch" if tb else info["launch"],
                   "tune_ms_per_step": info["tune_ms_per_step"],
                   "temporal_depth": tb, "tune_ms_per_step_temporal": tbi["tune_ms_per_step"],
                   "size_classes": classes, "tuned_ms_per_step": ir["tuned_ms_per_step"],
                   "l2": "state ~290 MB > L2; no flush", "parallelism": f"problems sharded by cost over {world} GPUs" if world > 1 else "single GPU"},
        "roofline": {"bound": "hbm", "kernel": (f"batch_tb_kernel ({tb} steps per launch from shared memory; the "
                                                "fraction counts the one-sweep bytes of every step and can exceed 1)"
                                                if tb else "batch_kernel (persistent, all steps)"
                                                if info["launch"] == "persistent"
                                                else "batch_phase_kernel (E and H launches of one step)"),
                     "achieved": ach, "peak": peak,
                     "unit": "GB/s", "frac": ach / peak, "peak_kind": peak_kind, "alg_bytes_per_step": ab,
                     "traffic": None},
        "fp64_plain": f64,
        "e2e": e2e,
        "cpu_baseline": cpu,
        "gpu_launches": (args.steps // (2 * tb) * 2 + 2 * (args.steps % (2 * tb)) + 1) if tb
        else 2 if info["launch"] == "persistent" else 2 * args.steps + 1,
        "clocks": clk.summary(),
    }


# ------------------------------------------------------------------ GPU arm
def main():
    args = parse()
    if args.impl == "reference":
        run_reference_arm(args)
        return
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))

    from fdtd_b200 import grid as G

    stream = torch.cuda.Stream()
    if args.workload in ("batch64", "adjoint512"):
        if args.workload == "batch64":
            line = run_batch(args, torch, world, rank, local, stream)
        else:
            line = run_adjoint(args, torch, world, rank, local)
        if rank == 0:
            print(json.dumps(line), flush=True)
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return
    line = run_zslab(args, torch, world, rank, local) if args.decompose == "zslab" else \
        run_grid(args, torch, world, rank, local, stream)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def accuracy(g, g64, p, steps: int) -> dict:
    """Advance the FP32 grid g and the FP64 plain grid g64 (same problem) to
    `steps` steps, then the relative L2 error of every E and H component
    (over all cells, on the device) and of every DFT spectrum of g against
    g64. The FP64 plain method is bit-identical to the CPU oracle at test
    sizes and stands in for it at full size."""
    for gr in (g, g64):
        left = steps - gr.step_count
        if left > 0:
            gr.step(left)
        gr.synchronize()
    from fdtd_b200.problem import THREED
    comps = ["Ex", "Ey", "Ez", "Hx", "Hy", "Hz"] if p.mode == THREED else (
        ["Ez", "Hx", "Hy"] if p.mode == 2 else ["Ex", "Ey", "Hz"])
    fields = {c: g.field_error(g64, c) for c in comps}
    dfts = []
    for q in range(len(p.dfts)):
        a, b = g.dft(q), g64.dft(q)
        nb = float(np.linalg.norm(b))
        dfts.append(float(np.linalg.norm(a - b)) / nb if nb > 0 else float(np.linalg.norm(a)))
    worst = max(list(fields.values()) + dfts)
    return {"steps": steps, "vs": "FP64 plain method on the same GPU (bit-identical to the CPU oracle at test sizes)",
            "fields_rel_l2": fields, "dft_rel_l2_max": max(dfts) if dfts else None,
            "dft_rel_l2": dfts if len(dfts) <= 8 else None, "worst": worst, "bound": 1e-4,
            "within_bound": bool(worst <= 1e-4)}


def run_zslab(args, torch, world, rank, local):
    """One grid of the workload cut into `world` z slabs, one per rank
    (fdtd_b200/zslab.py): each half step sends the ghost planes over NCCL
    while the interior part of the sweep runs (fdtd_step_half_part). value =
    the global grid's interior cell-updates / max rank time; scaling strong."""
    import torch.distributed as dist
    from fdtd_b200.zslab import GpuSlab, ZSlabRank, local_problem, partition_z
    p = make_problem(args.workload, args.steps + args.warmup, args.n, args.variant)
    z0, z1 = partition_z(p, world)[rank]
    q = local_problem(p, z0, z1)
    slab = GpuSlab(q, "f32", device=local)
    drv = ZSlabRank(slab, q.shape[2], rank, world)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    drv.step(args.warmup)
    slab.synchronize()
    barrier()
    launches0 = slab.grid.launch_count
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        start.record(slab.stream)
        drv.step(args.steps)
        end.record(slab.stream)
        slab.synchronize()
        barrier()
    ms = start.elapsed_time(end)
    t = torch.tensor([ms], device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    cells = p.interior_cells
    ab = alg_bytes(p, 4)
    peak, peak_kind = peaks()
    step_ach = ab["step"] * args.steps / (ms_max / 1e3) / 1e9
    return {
        "metric": METRIC, "value": cells * args.steps / (ms_max / 1e3) / 1e9, "unit": "Gcell-updates/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": p.name, "grid": list(p.shape), "interior_cells": cells,
                   "parallelism": f"z slabs x{world}", "slab_planes": [list(r) for r in partition_z(p, world)],
                   "l2": "state larger than L2, no flush"},
        "roofline": {"bound": "hbm", "scope": "whole step, all GPUs", "achieved": step_ach, "peak": peak * world,
                     "unit": "GB/s", "frac": step_ach / (peak * world), "peak_kind": peak_kind,
                     "alg_bytes_per_cell_step": ab["per_cell_step"], "traffic": None},
        "e2e": None, "cpu_baseline": None, "gpu_launches": slab.grid.launch_count - launches0,
        "clocks": clk.summary(),
    }


def run_grid(args, torch, world, rank, local, stream):
    """One 3D (or 2D) grid per GPU: the FP32 fused method timed over --steps
    steps; the FP64 plain method on the same grid; the FP32 error against it
    at the configuration's length; end to end through the public API."""
    import torch.distributed as dist
    from fdtd_b200 import grid as G

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    nprof = min(20, max(3, args.steps // 10))
    acc_steps = P_STEPS.get(args.workload, 0) if args.accuracy_steps < 0 else args.accuracy_steps
    if args.variant in ("bd3", "bd4") or args.no_f64:
        acc_steps = 0  # the FP64 leg steps other physics (or does not run)
    nsig = max(args.warmup + args.steps + nprof + 1, acc_steps)
    p = make_problem(args.workload, nsig, args.n, args.variant)
    g = G.Grid.from_problem(p, "f32", device=local)
    if args.sweep != "auto":
        g.set_sweep_kernel(args.sweep)
    g.prepare()  # set-up: CPML slabs, DFT buffers, TFSF tables and the captured step graph
    g.step(args.warmup, stream=stream.cuda_stream)
    torch.cuda.synchronize()
    launches0 = g.launch_count
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    with ClockSampler(local) as clk:
        with torch.cuda.stream(stream):
            start.record(stream)
            g.step(args.steps, stream=stream.cuda_stream)
            end.record(stream)
        barrier()
    ms = start.elapsed_time(end)
    launches = g.launch_count - launches0
    t = torch.tensor([ms], device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    cells = p.interior_cells
    value = cells * args.steps * world / (ms_max / 1e3) / 1e9

    # per-kernel CUDA-event times on the launching stream (separate pass)
    prof = g.profile_step(nprof, stream=stream.cuda_stream)
    ab = alg_bytes(p, 4)
    peak, peak_kind = peaks()
    state_gb = g.memory_bytes / 1e9
    three_d = p.mode == 3
    kind = {"auto": "staged"}.get(args.sweep, args.sweep)
    one_launch = kind == "eh" and three_d
    if one_launch:
        # E and H of the whole step in one launch: its bytes are the step's
        ab = dict(ab, e_sweep=ab["step"], h_sweep=0.0)
    e_ach = ab["e_sweep"] / (prof["e_sweep"] / 1e3) / 1e9
    h_ach = ab["h_sweep"] / (prof["h_sweep"] / 1e3) / 1e9 if prof["h_sweep"] > 0 else None
    step_ach = ab["step"] * args.steps / (ms / 1e3) / 1e9
    if one_launch:
        e_name, h_name = "staged_eh_kernel (E and H sweeps of a step, one launch)", None
    else:
        e_name = f"{kind}_e_kernel (E sweep)" if three_d else "fused_e_kernel (E sweep)"
        h_name = f"{kind}_h_kernel (H sweep)" if three_d else "fused_h_kernel (H sweep)"
    # DRAM traffic per launch: dram__bytes_read.sum + dram__bytes_write.sum of
    # one ncu capture of the same kernel on the same physics at a smaller size,
    # scaled by interior cells (traffic grows with the cells swept)
    tr = MEASURED_TRAFFIC.get((args.workload, kind))
    traffic_e = tr["e"] * cells if tr else None
    traffic_h = tr["h"] * cells if tr else None

    # end to end through the public API with host buffers: upload the problem
    # (material ids, source and aux tables), run, read every DFT spectrum back
    e2e = None
    if not args.no_e2e:
        # the whole job of the configuration (its own number of steps) from
        # host arrays to spectra on the host
        n_e2e = P_STEPS.get(args.workload, args.steps) if args.n == 0 else args.steps
        pe = make_problem(args.workload, n_e2e, args.n, args.variant)  # the user's host-side description
        barrier()
        t0 = time.perf_counter()
        ge = G.Grid.from_problem(pe, "f32", device=local)
        ge.synchronize()
        t1 = time.perf_counter()
        ge.step(n_e2e)
        ge.synchronize()
        t2 = time.perf_counter()
        spectra = [ge.dft(q) for q in range(len(pe.dfts))]
        ge.synchronize()
        t_e2e = time.perf_counter() - t0
        parts = {"create_s": t1 - t0, "steps_s": t2 - t1, "read_s": t_e2e - (t2 - t0)}
        h2d = (pe.ids.nbytes if pe.ids is not None else 0) + sum(s.values.nbytes for s in pe.sources)
        if pe.block_ids is not None:
            h2d += pe.block_ids.nbytes
        if pe.tfsf is not None:
            h2d += pe.tfsf.aux_values.nbytes
        d2h = sum(s.size * 16 for s in spectra)
        tt = torch.tensor([t_e2e], device="cuda")
        if world > 1:
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e = {"value": cells * n_e2e * world / float(tt.item()) / 1e9, "unit": "Gcell-updates/s",
               "steps": n_e2e, "h2d_bytes_per_step": h2d / n_e2e, "d2h_bytes_per_step": d2h / n_e2e,
               "wall_s": float(tt.item()), "parts": parts,
               "note": "the configuration's whole job through the C ABI: grid creation, H2D of material ids/"
                       "blocks/source/aux tables, its steps and D2H of every DFT spectrum, timed by the host clock "
                       "(the synthetic problem is built before)"}
        ge.close()
        del ge

    # FP64 plain on the same grid and GPU (the metric's comparison)
    f64 = None
    acc = None
    if not args.no_f64:
        p64 = make_problem(args.workload, nsig, args.n, args.variant, fp64=True)
        g64 = G.Grid.from_problem(p64, "f64", device=local)
        n64 = max(3, min(args.steps, 200))
        g64.prepare()
        g64.step(args.warmup, stream=stream.cuda_stream)
        barrier()
        with torch.cuda.stream(stream):
            start.record(stream)
            g64.step(n64, stream=stream.cuda_stream)
            end.record(stream)
        barrier()
        ms64 = start.elapsed_time(end)
        prof64 = g64.profile_step(min(10, n64), stream=stream.cuda_stream)
        ab64 = alg_bytes(p64, 8)
        e64 = ab64["e_sweep"] / (prof64["e_sweep"] / 1e3) / 1e9
        h64 = ab64["h_sweep"] / (prof64["h_sweep"] / 1e3) / 1e9
        f64 = {"value": cells * n64 / (ms64 / 1e3) / 1e9, "steps": n64, "ms_per_step": ms64 / n64,
               "time_scheme": p64.time_scheme, "kernel_ms": prof64,
               "roofline": {"bound": "hbm", "kernel": "plain_e_kernel (E sweep)", "achieved": e64, "peak": peak,
                            "unit": "GB/s", "frac": e64 / peak, "alg_bytes_per_launch": ab64["e_sweep"],
                            "launch_ms": prof64["e_sweep"]},
               "roofline_h": {"kernel": "plain_h_kernel (H sweep)", "achieved": h64, "frac": h64 / peak,
                              "alg_bytes_per_launch": ab64["h_sweep"], "launch_ms": prof64["h_sweep"]},
               "roofline_step": {"alg_bytes_per_cell_step": ab64["per_cell_step"],
                                 "achieved": ab64["step"] * n64 / (ms64 / 1e3) / 1e9,
                                 "frac": ab64["step"] * n64 / (ms64 / 1e3) / 1e9 / peak}}
        if acc_steps > 0:
            acc = accuracy(g, g64, p, max(acc_steps, g.step_count, g64.step_count))
        g64.close()
        del g64
    g.close()
    del g

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args.workload, variant=args.variant)

    step_ms = ms_max / args.steps
    return {
        "metric": METRIC, "value": value, "unit": "Gcell-updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": p.name, "variant": args.variant, "grid": list(p.shape), "interior_cells": cells,
                   "cpml": max(p.pml.values()) if p.pml else 0, "steps_in_config": P_STEPS.get(args.workload),
                   "l2": f"state {state_gb:.2f} GB on the device; "
                         + ("larger than L2, no flush" if state_gb > 0.126 else "fits L2"),
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        # the whole step against the minimal formulation's bytes per cell-step
        "roofline": {"bound": "hbm", "scope": "whole step (all kernels of a step)",
                     "kernel": f"{e_name} + extras" if h_name is None else f"{e_name} + {h_name} + extras",
                     "achieved": step_ach, "peak": peak, "unit": "GB/s", "frac": step_ach / peak,
                     "peak_kind": peak_kind, "alg_bytes_per_cell_step": ab["per_cell_step"],
                     "alg_bytes_per_step": ab["step"], "step_ms": ms / args.steps,
                     "traffic": (traffic_e + traffic_h) if tr else None,
                     "traffic_source": tr["source"] if tr else None},
        "roofline_e": {"kernel": e_name, "achieved": e_ach, "frac": e_ach / peak,
                       "alg_bytes_per_launch": ab["e_sweep"], "launch_ms": prof["e_sweep"], "traffic": traffic_e},
        "roofline_h": None if h_name is None else {
            "kernel": h_name, "achieved": h_ach, "frac": h_ach / peak, "alg_bytes_per_launch": ab["h_sweep"],
            "launch_ms": prof["h_sweep"], "traffic": traffic_h},
        "kernel_ms": prof,
        "fp64_plain": f64,
        "fp32_over_fp64": (value / world / f64["value"]) if f64 else None,
        "error_vs_fp64": acc,
        "e2e": e2e, "cpu_baseline": cpu, "gpu_launches": launches,
        "clocks": clk.summary(),
    }


if __name__ == "__main__":
    main()
