"""Python driver for the CPU checkers (TEST INFRASTRUCTURE ONLY).

Runs a ``fdtd_b200.problem.Problem`` through
  * ``run_oracle``: the plain-C restatement (oracle/liboracle.so), or
  * ``run_reference``: the reference's own functors (oracle/_ref/ref_runner,
    compiled from the reference headers by oracle/Makefile).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import tempfile
from typing import Dict, List, Optional

import numpy as np

SOURCE_TARGETS = {"E": 0, "D": 1, "H": 2, "B": 3}
BOUNDARY_KINDS = {"pec": 1, "pmc": 2, "symmetric": 3, "antisymmetric": 4, "periodic": 5}

HERE = os.path.dirname(os.path.abspath(__file__))
# Where the reference tree (pederson/fdtd) lies: FDTD_REFERENCE_DIR, or the
# container's read-only copy. The reference runner and the XML writers are
# compiled from its headers there; without it the golden fixtures stand in.
REFERENCE_DIR = os.environ.get("FDTD_REFERENCE_DIR") or "/root/reference"


def reference_tree_present() -> bool:
    return os.path.isfile(os.path.join(REFERENCE_DIR, "include", "YeeUpdates.hpp"))
LIB_PATH = os.path.join(HERE, "liboracle.so")
RUNNER_PATH = os.path.join(HERE, "_ref", "ref_runner")

# output order of oracle_get / ref_runner
NAMES = ["Dx", "Dy", "Dz", "Ex", "Ey", "Ez", "Bx", "By", "Bz", "Hx", "Hy", "Hz",
         "Px", "Py", "Pz", "Jx", "Jy", "Jz"]
PSI_NAMES = [f"psi{'EH'[f]}{'xyz'[i]}{'xyz'[j]}" for f in range(2) for i in range(3) for j in range(3)]
# surface quantities (include/SurfaceQuantities.hpp) on every interior cell,
# by quantity code (oracle_read_quantity): rho 12, Je 6..8, Jh 9..11
SURFACE_NAMES = ["rho", "Jex", "Jey", "Jez", "Jhx", "Jhy", "Jhz"]
SURFACE_CODES = {"rho": 12, "Jex": 6, "Jey": 7, "Jez": 8, "Jhx": 9, "Jhy": 10, "Jhz": 11}
ALL_NAMES = NAMES + PSI_NAMES + SURFACE_NAMES


class OracleMaterial(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("npoles", ctypes.c_int), ("eps_inf", ctypes.c_double),
                ("mu_r", ctypes.c_double), ("delta_eps", ctypes.c_double * 4),
                ("freq", ctypes.c_double * 4), ("gamma", ctypes.c_double * 4)]


_lib = None


def build(quiet: bool = True) -> None:
    """Compile liboracle.so (and the reference runner when the reference tree
    is present)."""
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)
    if reference_tree_present():
        subprocess.run(["make", "-s", "-C", HERE, f"REF={REFERENCE_DIR}", "_ref/ref_runner"], check=True,
                       stdout=subprocess.DEVNULL if quiet else None)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        vp, ip, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
        L.oracle_create.restype = vp
        L.oracle_create.argtypes = [ctypes.c_int] * 4 + [ctypes.c_double] * 2
        L.oracle_destroy.argtypes = [vp]
        L.oracle_set_pml.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.oracle_set_pml_model.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int] + [ctypes.c_double] * 5
        L.oracle_set_materials.argtypes = [vp, ctypes.POINTER(OracleMaterial), ctypes.c_int]
        L.oracle_set_material_ids.argtypes = [vp, ctypes.c_void_p]
        L.oracle_add_source.argtypes = [vp] + [ctypes.c_int] * 5 + [dp, ctypes.c_int]
        L.oracle_add_tfsf_plane.argtypes = [vp, ctypes.c_int, ctypes.c_int, ip, ip, dp, dp, dp, dp,
                                            ctypes.c_int, dp, ctypes.c_int]
        L.oracle_add_dft.argtypes = [vp, ctypes.c_int, ip, ip, dp, ctypes.c_int]
        L.oracle_step.argtypes = [vp, ctypes.c_int]
        L.oracle_step_half.argtypes = [vp, ctypes.c_int]
        L.oracle_material_explicit.argtypes = [vp, ctypes.c_int]
        L.oracle_set_boundary.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.oracle_set_time_scheme.argtypes = [vp, ctypes.c_int]
        L.oracle_get.argtypes = [vp, ctypes.c_int, dp]
        L.oracle_set.argtypes = [vp, ctypes.c_int, dp]
        L.oracle_dft_get.argtypes = [vp, ctypes.c_int, dp]
        L.oracle_dft_npoints.argtypes = [vp, ctypes.c_int]
        L.oracle_pml_profile.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp]
        L.oracle_imp0.restype = ctypes.c_double
        L.oracle_add_source_box.argtypes = [vp, ctypes.c_int, ctypes.c_int, ip, ip, dp, ctypes.c_int]
        L.oracle_set_eps_map.argtypes = [vp, dp]
        L.oracle_adjoint_tm.argtypes = [vp, ctypes.c_int, ip, ip, ctypes.c_double, ip, ip, dp, dp]
        L.oracle_read_quantity.argtypes = [vp, ctypes.c_int, ip, ip, dp]
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(seq):
    arr = (ctypes.c_int * len(seq))(*seq)
    return arr


def _mat_struct(m) -> OracleMaterial:
    s = OracleMaterial()
    s.kind = m.kind
    s.npoles = len(m.poles)
    s.eps_inf = m.eps_inf
    s.mu_r = m.mu_r
    for q, (de, f, g) in enumerate(m.poles):
        s.delta_eps[q] = de
        s.freq[q] = f
        s.gamma[q] = g
    return s


class OracleGrid:
    """The C restatement, set up from a Problem."""

    def __init__(self, p):
        L = lib()
        nx, ny, nz = p.shape
        self.p = p
        self.h = L.oracle_create(p.mode, nx, ny, nz, p.dx, p.dt)
        if not self.h:
            raise ValueError("oracle_create rejected the grid")
        for (a, s), n in sorted(p.pml.items()):
            if (a, s) in getattr(p, "pml_models", {}):
                assert L.oracle_set_pml_model(self.h, a, s, n, *[float(v) for v in p.pml_models[(a, s)]]) == 0
            else:
                assert L.oracle_set_pml(self.h, a, s, n) == 0
        for (a, s), kind in sorted(p.boundaries.items()):
            assert L.oracle_set_boundary(self.h, a, s, BOUNDARY_KINDS[kind]) == 0
        if p.time_scheme != 1:
            assert L.oracle_set_time_scheme(self.h, p.time_scheme) == 0
        if len(p.materials) > 256:
            raise ValueError("the oracle takes at most 256 materials")
        mats = (OracleMaterial * len(p.materials))(*[_mat_struct(m) for m in p.materials])
        assert L.oracle_set_materials(self.h, mats, len(p.materials)) == 0
        ids = p.cell_ids()
        if ids is not None:
            ids8 = np.ascontiguousarray(ids.astype(np.uint8))
            assert L.oracle_set_material_ids(self.h, ids8.ctypes.data) == 0
        self._keep = []
        for s in p.sources:
            v = np.ascontiguousarray(s.values, dtype=np.float64)
            if s.hi is None:
                assert L.oracle_add_source(self.h, s.comp, SOURCE_TARGETS[s.target], *s.pos, _dp(v), len(v)) == 0
            else:
                assert L.oracle_add_source_box(self.h, s.comp, SOURCE_TARGETS[s.target], _ip(s.pos), _ip(s.hi),
                                               _dp(v), len(v)) == 0
        if p.eps_map is not None:
            self._eps = np.ascontiguousarray(p.eps_map, dtype=np.float64)
            assert self._eps.size == nx * ny * nz
            assert L.oracle_set_eps_map(self.h, _dp(self._eps)) == 0
        if p.tfsf is not None:
            t = p.tfsf
            av = np.ascontiguousarray(t.aux_values, dtype=np.float64)
            for pl in t.planes:
                rc = L.oracle_add_tfsf_plane(self.h, pl.axis, pl.orient, _ip(pl.lo), _ip(pl.hi),
                                             _dp(np.array(t.origin, float)), _dp(np.array(t.k, float)),
                                             _dp(np.array(t.pol_e, float)), _dp(np.array(t.pol_h, float)),
                                             t.aux_ncells, _dp(av), len(av))
                assert rc == 0
        self.dft_handles, self.dft_nf = [], []
        for r in p.dfts:
            self.add_dft(r.comp, r.lo, r.hi, r.freqs)

    def add_dft(self, comp: int, lo, hi, freqs) -> int:
        """A running DFT region (also after steps were taken: its samples
        start with the next step); returns its index for dft()."""
        fr = np.array(freqs, dtype=np.float64)
        hnd = lib().oracle_add_dft(self.h, comp, _ip(lo), _ip(hi), _dp(fr), len(fr))
        assert hnd >= 0
        self.dft_handles.append(hnd)
        self.dft_nf.append(len(fr))
        return len(self.dft_handles) - 1

    def set_time_scheme(self, scheme: int) -> None:
        assert lib().oracle_set_time_scheme(self.h, int(scheme)) == 0

    def step(self, n: int) -> None:
        lib().oracle_step(self.h, n)

    def step_half(self, phase: int) -> None:
        assert lib().oracle_step_half(self.h, phase) == 0

    def material_explicit(self, ft: int) -> None:
        """The forward material updates (flux from field) of field type ft."""
        rc = lib().oracle_material_explicit(self.h, int(ft))
        if rc != 0:
            raise ValueError("no forward material update for this grid (a Lorentz material)")

    def get_plane(self, name: str, k: int) -> np.ndarray:
        return self.get(name)[k].copy()

    def set_plane(self, name: str, k: int, plane: np.ndarray) -> None:
        a = self.get(name)
        a[k] = plane
        self.set(name, a)

    def read_quantity(self, code: int, lo, hi) -> np.ndarray:
        """A quantity (0..5 E/H, 6..8 Je, 9..11 Jh, 12 rho) over an inclusive
        box, shape (nz_b, ny_b, nx_b)."""
        n = [h - l + 1 for l, h in zip(lo, hi)]
        out = np.empty(n[0] * n[1] * n[2], dtype=np.float64)
        rc = lib().oracle_read_quantity(self.h, int(code), _ip(lo), _ip(hi), _dp(out))
        if rc != 0:
            raise ValueError("quantity not in this mode or box outside the interior")
        return out.reshape(n[2], n[1], n[0])

    def surface(self, name: str) -> np.ndarray:
        """A surface quantity on every interior cell (zero elsewhere, and
        zero where the mode has none), as the reference runner dumps it."""
        nx, ny, nz = self.p.shape
        out = np.zeros((nz, ny, nx))
        code = SURFACE_CODES[name]
        three = self.p.mode == 3
        lo, hi = (1, 1, 1 if three else 0), (nx - 2, ny - 2, nz - 2 if three else 0)
        try:
            out[lo[2]:hi[2] + 1, 1:ny - 1, 1:nx - 1] = self.read_quantity(code, lo, hi)
        except ValueError:
            pass
        return out

    def get(self, name: str) -> np.ndarray:
        if name in SURFACE_CODES:
            return self.surface(name)
        which = ALL_NAMES.index(name) if name in ALL_NAMES else int(name)
        nx, ny, nz = self.p.shape
        out = np.empty(nx * ny * nz, dtype=np.float64)
        assert lib().oracle_get(self.h, which, _dp(out)) == 0
        return out.reshape(nz, ny, nx)

    def get_pole(self, pole: int, name: str) -> np.ndarray:
        if pole == 0:
            return self.get(name)
        r = ["Px", "Py", "Pz", "Jx", "Jy", "Jz"].index(name)
        return self.get(str(36 + (pole - 1) * 6 + r))

    def set(self, name: str, arr: np.ndarray) -> None:
        which = ALL_NAMES.index(name)
        a = np.ascontiguousarray(arr, dtype=np.float64).ravel()
        assert lib().oracle_set(self.h, which, _dp(a)) == 0

    def dft(self, q: int) -> np.ndarray:
        """[nf][npoints] complex"""
        L = lib()
        n = L.oracle_dft_npoints(self.h, self.dft_handles[q])
        nf = self.dft_nf[q]
        out = np.empty(nf * n * 2, dtype=np.float64)
        assert L.oracle_dft_get(self.h, self.dft_handles[q], _dp(out)) == 0
        out = out.reshape(nf, n, 2)
        return out[..., 0] + 1j * out[..., 1]

    def pml_profile(self, ft: int, axis: int) -> np.ndarray:
        n = self.p.shape[axis]
        out = np.empty(4 * n, dtype=np.float64)
        assert lib().oracle_pml_profile(self.h, ft, axis, _dp(out)) == 0
        return out.reshape(4, n)

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().oracle_destroy(self.h)
                self.h = None
        except Exception:
            pass


def run_oracle(p, steps: Optional[int] = None) -> OracleGrid:
    import time
    g = OracleGrid(p)
    t0 = time.perf_counter()
    g.step(p.steps if steps is None else steps)
    g.loop_seconds = time.perf_counter() - t0
    return g


def reference_available() -> bool:
    return os.path.exists(RUNNER_PATH)


def run_reference(p, steps: Optional[int] = None, explicit: bool = False) -> Dict[str, np.ndarray]:
    """Run the reference's own functors on the same Problem; returns every
    output array by name (shape (nz, ny, nx)). explicit: after the steps, the
    reference's forward material updates (XUpdate<Mode, ft, true>) of the
    electric and then the magnetic field on every interior cell."""
    if not reference_available():
        raise RuntimeError("oracle/_ref/ref_runner is not built")
    steps = p.steps if steps is None else steps
    nx, ny, nz = p.shape
    with tempfile.TemporaryDirectory() as td:
        lines = [f"mode {p.mode}", f"dims {nx} {ny} {nz}", f"dxdt {p.dx!r} {p.dt!r}"]
        pm = [p.pml.get((a, s), 0) for a in range(3) for s in range(2)]
        lines.append("pml " + " ".join(str(x) for x in pm))
        for (a, sd), mp in sorted(getattr(p, "pml_models", {}).items()):
            lines.append(f"pmlmodel {a} {sd} " + " ".join(repr(float(v)) for v in mp))
        lines.append(f"nmat {len(p.materials)}")
        for m in p.materials:
            if len(m.poles) > 1:
                raise ValueError("the reference holds one pole per cell")
            de, f, g = m.poles[0] if m.poles else (1.0, 0.0, 0.0)
            lines.append(f"{m.kind} {m.eps_inf!r} {de!r} {f!r} {g!r} {m.mu_r!r}")
        ids = p.cell_ids()
        if ids is not None:
            ip = os.path.join(td, "ids.bin")
            np.ascontiguousarray(ids.astype(np.uint8)).tofile(ip)
            lines.append(f"matids {ip}")
        else:
            lines.append("matids none")
        if p.eps_map is not None:
            raise ValueError("the reference runner takes per-cell material ids, not a permittivity map")
        # a box source is one SoftSource per cell, applied after the point sources
        pts = [(s, s.pos) for s in p.sources if s.hi is None]
        for s in p.sources:
            if s.hi is not None:
                pts += [(s, (i, j, k)) for k in range(s.pos[2], s.hi[2] + 1) for j in range(s.pos[1], s.hi[1] + 1)
                        for i in range(s.pos[0], s.hi[0] + 1)]
        lines.append(f"nsrc {len(pts)}")
        files = {}
        for q, (s, pos) in enumerate(pts):
            if id(s) not in files:
                files[id(s)] = os.path.join(td, f"src{len(files)}.bin")
                np.ascontiguousarray(s.values, dtype=np.float64).tofile(files[id(s)])
            lines.append(f"{s.comp} {SOURCE_TARGETS[s.target]} {pos[0]} {pos[1]} {pos[2]} {files[id(s)]}")
        if p.tfsf is not None:
            t = p.tfsf
            ap = os.path.join(td, "aux.bin")
            np.ascontiguousarray(t.aux_values, dtype=np.float64).tofile(ap)
            lines.append(f"ntfsf {len(t.planes)} {t.aux_ncells} {ap} {t.origin[0]!r} {t.origin[1]!r} {t.origin[2]!r} "
                         f"{t.k[0]!r} {t.k[1]!r} {t.k[2]!r} 1 {t.pol_e[0]!r} {t.pol_e[1]!r} {t.pol_e[2]!r} "
                         f"{t.pol_h[0]!r} {t.pol_h[1]!r} {t.pol_h[2]!r}")
            for pl in t.planes:
                lines.append(f"{pl.axis} {pl.orient} {pl.lo[0]} {pl.hi[0]} {pl.lo[1]} {pl.hi[1]} {pl.lo[2]} {pl.hi[2]}")
        if p.boundaries:
            lines.append(f"nbc {len(p.boundaries)}")
            for (a, sd), kind in sorted(p.boundaries.items()):
                lines.append(f"{a} {sd} {BOUNDARY_KINDS[kind]}")
        if p.time_scheme != 1:
            lines.append(f"scheme {p.time_scheme}")
        if explicit:
            lines.append("explicit 1")
        lines.append(f"steps {steps}")
        op = os.path.join(td, "out.bin")
        lines.append(f"out {op}")
        sc = os.path.join(td, "scenario.txt")
        with open(sc, "w") as f:
            f.write("\n".join(lines) + "\n")
        res = subprocess.run([RUNNER_PATH, sc], check=True, capture_output=True, text=True)
        raw = np.fromfile(op, dtype=np.float64).reshape(len(ALL_NAMES), nz, ny, nx)
    out = {n: raw[q] for q, n in enumerate(ALL_NAMES)}
    for line in res.stdout.splitlines():
        if line.startswith("loop_seconds"):
            out["loop_seconds"] = float(line.split()[1])
    return out


def adjoint_tm(p, steps: int, probe_lo, probe_hi, freq: float, design_lo, design_hi):
    """FP64 CPU adjoint (oracle_adjoint_tm) of a TM Problem from t = 0:
    returns (J, dJ/deps_r over the design box as [ny_d, nx_d])."""
    g = OracleGrid(p)
    nd = (design_hi[0] - design_lo[0] + 1) * (design_hi[1] - design_lo[1] + 1)
    grad = np.zeros(nd)
    J = ctypes.c_double()
    rc = lib().oracle_adjoint_tm(g.h, steps, _ip(probe_lo), _ip(probe_hi), freq, _ip(design_lo), _ip(design_hi),
                                 ctypes.byref(J), _dp(grad))
    if rc != 0:
        raise ValueError("oracle_adjoint_tm rejected the problem")
    return J.value, grad.reshape(design_hi[1] - design_lo[1] + 1, design_hi[0] - design_lo[0] + 1)
