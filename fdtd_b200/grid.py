"""ctypes binding of the fdtd_b200 C ABI (include/fdtd_b200.h).

``Grid`` owns one fdtd_grid handle. Every call goes through the CUDA library
libfdtd_b200.so built in-tree by ``fdtd_b200.build_lib``; there is no CPU path:
if the library or a GPU is missing, construction raises.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence

import numpy as np

from . import problem as P

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfdtd_b200.so")

PLAIN_F64 = 0
FUSED_F32 = 1
PRECISIONS = {"f64": PLAIN_F64, "plain": PLAIN_F64, "f32": FUSED_F32, "fused": FUSED_F32}

FIELD_NAMES = ["Dx", "Dy", "Dz", "Ex", "Ey", "Ez", "Bx", "By", "Bz", "Hx", "Hy", "Hz",
               "Px", "Py", "Pz", "Jx", "Jy", "Jz"]
PSI_NAMES = [f"psi{'EH'[f]}{'xyz'[i]}{'xyz'[j]}" for f in range(2) for i in range(3) for j in range(3)]
ALL_NAMES = FIELD_NAMES + PSI_NAMES

STATUS = {0: "FDTD_OK", -1: "FDTD_ERR_INVALID", -2: "FDTD_ERR_CUDA", -3: "FDTD_ERR_UNSUPPORTED",
          -4: "FDTD_ERR_NOMEM", -5: "FDTD_ERR_NONFINITE", -6: "FDTD_ERR_TIMEOUT"}

# every symbol include/fdtd_b200.h declares
EXPORTS = ["fdtd_grid_create", "fdtd_grid_destroy", "fdtd_set_pml", "fdtd_set_pml_model", "fdtd_set_materials", "fdtd_set_material_ids",
           "fdtd_set_material_blocks", "fdtd_set_eps_map", "fdtd_set_boundary", "fdtd_set_time_scheme", "fdtd_add_source", "fdtd_add_source_box", "fdtd_add_tfsf_plane", "fdtd_add_dft",
           "fdtd_dft_npoints", "fdtd_dft_read", "fdtd_read_quantity", "fdtd_step", "fdtd_prepare", "fdtd_step_static_scratch", "fdtd_step_half", "fdtd_step_half_part", "fdtd_copy_plane", "fdtd_copy_plane_between", "fdtd_material_explicit", "fdtd_profile_step", "fdtd_set_sweep_kernel", "fdtd_use_graphs", "fdtd_error_flags", "fdtd_synchronize", "fdtd_download", "fdtd_upload",
           "fdtd_check_finite", "fdtd_field_error", "fdtd_get_step", "fdtd_launch_count", "fdtd_memory_bytes",
           "fdtd_batch_create", "fdtd_batch_destroy", "fdtd_batch_tune", "fdtd_batch_configure", "fdtd_batch_step",
           "fdtd_batch_info", "fdtd_batch_item_rows", "fdtd_batch_set_item_rows", "fdtd_batch_set_temporal",
           "fdtd_batch_temporal",
           "fdtd_batch_error_flags", "fdtd_adjoint_create", "fdtd_adjoint_forward", "fdtd_adjoint_backward",
           "fdtd_adjoint_destroy", "fdtd_last_error_string"]


class FdtdError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class GridDesc(ctypes.Structure):
    _fields_ = [("mode", ctypes.c_int), ("precision", ctypes.c_int), ("nx", ctypes.c_int), ("ny", ctypes.c_int),
                ("nz", ctypes.c_int), ("dx", ctypes.c_double), ("dt", ctypes.c_double), ("device", ctypes.c_int)]


class MaterialC(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("npoles", ctypes.c_int), ("eps_inf", ctypes.c_double),
                ("mu_r", ctypes.c_double), ("delta_eps", ctypes.c_double * 4),
                ("freq", ctypes.c_double * 4), ("gamma", ctypes.c_double * 4)]


_lib = None


def load_library(path: str = LIB_PATH):
    """Load libfdtd_b200.so and declare its signatures. Raises if missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is not built: run `python -m fdtd_b200.build_lib` (there is no CPU fallback)")
    L = ctypes.CDLL(path)
    vp, ip, dp, i = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double), ctypes.c_int
    llp = ctypes.POINTER(ctypes.c_longlong)
    sig = {
        "fdtd_grid_create": [ctypes.POINTER(GridDesc), ctypes.POINTER(vp)],
        "fdtd_grid_destroy": [vp],
        "fdtd_set_pml": [vp, i, i, i],
        "fdtd_set_pml_model": [vp, i, i, i] + [ctypes.c_double] * 5,
        "fdtd_set_materials": [vp, ctypes.POINTER(MaterialC), i],
        "fdtd_set_material_ids": [vp, vp],
        "fdtd_set_material_blocks": [vp, i, vp, i, i, i],
        "fdtd_set_eps_map": [vp, dp],
        "fdtd_set_boundary": [vp, i, i, i],
        "fdtd_set_time_scheme": [vp, i],
        "fdtd_prepare": [vp],
        "fdtd_step_static_scratch": [vp, i, vp],
        "fdtd_step_half": [vp, i, vp],
        "fdtd_step_half_part": [vp, i, i, vp],
        "fdtd_copy_plane": [vp, i, i, vp, i, vp],
        "fdtd_copy_plane_between": [vp, i, i, vp, i, vp],
        "fdtd_material_explicit": [vp, i, vp],
        "fdtd_add_source": [vp, i, i, i, i, i, dp, i],
        "fdtd_add_source_box": [vp, i, i, ip, ip, dp, i],
        "fdtd_add_tfsf_plane": [vp, i, i, ip, ip, dp, dp, dp, dp, i, dp, i],
        "fdtd_add_dft": [vp, i, ip, ip, dp, i, ip],
        "fdtd_dft_npoints": [vp, i, llp],
        "fdtd_dft_read": [vp, i, dp],
        "fdtd_read_quantity": [vp, i, ip, ip, dp],
        "fdtd_step": [vp, i, vp],
        "fdtd_profile_step": [vp, i, vp, dp],
        "fdtd_set_sweep_kernel": [vp, i],
        "fdtd_use_graphs": [vp, i],
        "fdtd_error_flags": [vp, ip],
        "fdtd_synchronize": [vp],
        "fdtd_download": [vp, i, dp],
        "fdtd_upload": [vp, i, dp],
        "fdtd_check_finite": [vp],
        "fdtd_field_error": [vp, vp, i, dp, dp],
        "fdtd_get_step": [vp, llp],
        "fdtd_launch_count": [vp, llp],
        "fdtd_memory_bytes": [vp, llp],
        "fdtd_batch_create": [i, ctypes.POINTER(vp), ctypes.POINTER(vp)],
        "fdtd_batch_destroy": [vp],
        "fdtd_batch_tune": [vp, i],
        "fdtd_batch_step": [vp, i, vp],
        "fdtd_batch_info": [vp, ip, ip, ip, ip, ctypes.POINTER(ctypes.c_float)],
        "fdtd_batch_item_rows": [vp, ip, ip, ctypes.POINTER(ctypes.c_float)],
        "fdtd_batch_set_item_rows": [vp, ip],
        "fdtd_batch_configure": [vp, i, i],
        "fdtd_batch_set_temporal": [vp, i],
        "fdtd_batch_temporal": [vp, ip, ctypes.POINTER(ctypes.c_float)],
        "fdtd_batch_error_flags": [vp, ip],
        "fdtd_adjoint_create": [vp, ip, ip, ctypes.c_double, ip, ip, i, ctypes.POINTER(vp)],
        "fdtd_adjoint_forward": [vp, i, dp],
        "fdtd_adjoint_backward": [vp, dp],
        "fdtd_adjoint_destroy": [vp],
    }
    for name, args in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = ctypes.c_int
    L.fdtd_last_error_string.restype = ctypes.c_char_p
    L.fdtd_last_error_string.argtypes = []
    _lib = L
    return L


def _check(rc: int) -> None:
    if rc != 0:
        raise FdtdError(rc, load_library().fdtd_last_error_string().decode())


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(seq):
    return (ctypes.c_int * len(seq))(*[int(x) for x in seq])


def material_struct(m: P.Material) -> MaterialC:
    s = MaterialC()
    s.kind = m.kind
    s.npoles = len(m.poles)
    s.eps_inf = m.eps_inf
    s.mu_r = m.mu_r
    for q, (de, f, g) in enumerate(m.poles):
        s.delta_eps[q] = de
        s.freq[q] = f
        s.gamma[q] = g
    return s


class Grid:
    """One grid on one GPU, driven through the C ABI."""

    def __init__(self, mode: int, shape: Sequence[int], dx: float, dt: float, precision="f64", device: int = 0):
        L = load_library()
        prec = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        nx, ny, nz = shape
        d = GridDesc(mode, prec, nx, ny, nz, dx, dt, device)
        h = ctypes.c_void_p()
        _check(L.fdtd_grid_create(ctypes.byref(d), ctypes.byref(h)))
        self.h = h
        self.mode, self.shape, self.dx, self.dt, self.precision = mode, (nx, ny, nz), dx, dt, prec
        self.dft_meta = []

    # ------------------------------------------------------------ set-up
    def set_pml(self, axis: int, side: int, ncells: int) -> None:
        _check(load_library().fdtd_set_pml(self.h, axis, side, ncells))

    def set_pml_model(self, axis: int, side: int, ncells: int, m: float, ma: float, sigma_max: float,
                      kappa_max: float, alpha_max: float) -> None:
        """CPML graded with PMLParameterModel(m, ma, sMax, kMax, aMax)."""
        _check(load_library().fdtd_set_pml_model(self.h, axis, side, ncells, float(m), float(ma), float(sigma_max),
                                                 float(kappa_max), float(alpha_max)))

    def set_materials(self, mats) -> None:
        arr = (MaterialC * len(mats))(*[material_struct(m) for m in mats])
        _check(load_library().fdtd_set_materials(self.h, arr, len(mats)))

    def set_material_ids(self, ids: np.ndarray) -> None:
        a = np.ascontiguousarray(ids, dtype=np.uint8)
        assert a.size == self.shape[0] * self.shape[1] * self.shape[2]
        _check(load_library().fdtd_set_material_ids(self.h, a.ctypes.data))

    def set_material_blocks(self, shift: int, bids: np.ndarray) -> None:
        a = np.ascontiguousarray(bids, dtype=np.uint16)
        nbz, nby, nbx = a.shape
        _check(load_library().fdtd_set_material_blocks(self.h, shift, a.ctypes.data, nbx, nby, nbz))

    def set_boundary(self, axis: int, side: int, kind: str) -> None:
        """kind: 'none', 'pec', 'pmc', 'symmetric', 'antisymmetric' or 'periodic'."""
        code = 0 if kind == "none" else P.BOUNDARY_KINDS[kind]
        _check(load_library().fdtd_set_boundary(self.h, int(axis), int(side), code))

    def prepare(self) -> None:
        """Lay out the deferred device state (CPML slabs, DFT buffers, TFSF
        tables) and capture the step graph now."""
        _check(load_library().fdtd_prepare(self.h))

    def set_time_scheme(self, scheme: int) -> None:
        """1 (BD1, leapfrog), 3 (BD3) or 4 (BD4): the TimePolicy of every
        curl update and TFSF correction; FP64 grids only for 3 and 4."""
        _check(load_library().fdtd_set_time_scheme(self.h, int(scheme)))

    def set_eps_map(self, eps: Optional[np.ndarray]) -> None:
        if eps is None:
            _check(load_library().fdtd_set_eps_map(self.h, None))
            return
        a = np.ascontiguousarray(eps, dtype=np.float64)
        assert a.size == self.shape[0] * self.shape[1] * self.shape[2]
        _check(load_library().fdtd_set_eps_map(self.h, _dp(a)))

    def add_source_box(self, comp: int, lo, hi, values, target: str = "E") -> None:
        v = np.ascontiguousarray(values, dtype=np.float64)
        _check(load_library().fdtd_add_source_box(self.h, comp, P.SOURCE_TARGETS[target], _ip(lo), _ip(hi), _dp(v),
                                                  len(v)))

    def add_source(self, comp: int, pos, values, target: str = "E") -> None:
        v = np.ascontiguousarray(values, dtype=np.float64)
        _check(load_library().fdtd_add_source(self.h, comp, P.SOURCE_TARGETS[target], *pos, _dp(v), len(v)))

    def add_tfsf_plane(self, axis, orient, lo, hi, origin, k, pol_e, pol_h, aux_ncells, aux_values) -> None:
        av = np.ascontiguousarray(aux_values, dtype=np.float64)
        f = lambda x: np.ascontiguousarray(x, dtype=np.float64)
        _check(load_library().fdtd_add_tfsf_plane(self.h, axis, orient, _ip(lo), _ip(hi), _dp(f(origin)), _dp(f(k)),
                                                  _dp(f(pol_e)), _dp(f(pol_h)), aux_ncells, _dp(av), len(av)))

    def add_dft(self, comp: int, lo, hi, freqs) -> int:
        fr = np.ascontiguousarray(freqs, dtype=np.float64)
        h = ctypes.c_int()
        _check(load_library().fdtd_add_dft(self.h, comp, _ip(lo), _ip(hi), _dp(fr), len(fr), ctypes.byref(h)))
        self.dft_meta.append(len(fr))
        return h.value

    @classmethod
    def from_problem(cls, p: P.Problem, precision="f64", device: int = 0) -> "Grid":
        g = cls(p.mode, p.shape, p.dx, p.dt, precision, device)
        for (a, s), n in sorted(p.pml.items()):
            if (a, s) in p.pml_models:
                g.set_pml_model(a, s, n, *p.pml_models[(a, s)])
            else:
                g.set_pml(a, s, n)
        for (a, s), kind in sorted(p.boundaries.items()):
            g.set_boundary(a, s, kind)
        if p.time_scheme != 1:
            g.set_time_scheme(p.time_scheme)
        g.set_materials(p.materials)
        if p.ids is not None:
            g.set_material_ids(p.ids)
        elif p.block_ids is not None:
            g.set_material_blocks(p.block_shift, p.block_ids)
        if p.eps_map is not None:
            g.set_eps_map(p.eps_map)
        for s in p.sources:
            if s.hi is None:
                g.add_source(s.comp, s.pos, s.values, s.target)
            else:
                g.add_source_box(s.comp, s.pos, s.hi, s.values, s.target)
        if p.tfsf is not None:
            t = p.tfsf
            for pl in t.planes:
                g.add_tfsf_plane(pl.axis, pl.orient, pl.lo, pl.hi, t.origin, t.k, t.pol_e, t.pol_h,
                                 t.aux_ncells, t.aux_values)
        g.dft_handles = [g.add_dft(r.comp, r.lo, r.hi, r.freqs) for r in p.dfts]
        return g

    # ------------------------------------------------------------ run
    def step(self, n: int, stream: Optional[int] = None) -> None:
        _check(load_library().fdtd_step(self.h, int(n), ctypes.c_void_p(stream) if stream else None))

    def step_half(self, phase: int, stream: Optional[int] = None) -> None:
        _check(load_library().fdtd_step_half(self.h, int(phase), ctypes.c_void_p(stream) if stream else None))

    def step_half_part(self, phase: int, part: int, stream: Optional[int] = None) -> None:
        """Part 0 or 1 of half step `phase`: the planes that read no ghost
        plane, then the ghost-adjacent plane and the rest of the half step."""
        _check(load_library().fdtd_step_half_part(self.h, int(phase), int(part),
                                                  ctypes.c_void_p(stream) if stream else None))

    def copy_plane(self, name: str, k: int, dev_ptr: int, to_grid: bool, stream: Optional[int] = None) -> None:
        """Copy z plane k of component `name` ('Ex'..'Hz') between the grid and
        a compact device buffer at address dev_ptr (nx*ny values)."""
        which = FIELD_NAMES.index(name)
        _check(load_library().fdtd_copy_plane(self.h, which, int(k), ctypes.c_void_p(dev_ptr), 1 if to_grid else 0,
                                              ctypes.c_void_p(stream) if stream else None))

    def copy_plane_to(self, name: str, k: int, dst: "Grid", k_dst: int, stream: Optional[int] = None) -> None:
        """Copy z plane k of component `name` into z plane k_dst of grid dst."""
        which = FIELD_NAMES.index(name)
        _check(load_library().fdtd_copy_plane_between(self.h, which, int(k), dst.h, int(k_dst),
                                                      ctypes.c_void_p(stream) if stream else None))

    def material_explicit(self, ft: int, stream: Optional[int] = None) -> None:
        """The forward material updates of field type ft (0 electric: D, and
        the Drude P and J, from E; 1 magnetic: B from H). FP64 grids."""
        _check(load_library().fdtd_material_explicit(self.h, int(ft), ctypes.c_void_p(stream) if stream else None))

    def step_static_scratch(self, n: int, stream: Optional[int] = None) -> None:
        """step() that allocates no device memory: the TFSF table of the call
        lives in a fixed 4 MiB device array shared by all grids of the device
        (at most 4 MiB / (16 B x sum of the planes' aux lengths) - 1 steps per
        call; calls that overlap on the GPU race on the array)."""
        _check(load_library().fdtd_step_static_scratch(self.h, int(n), ctypes.c_void_p(stream) if stream else None))

    def profile_step(self, n: int, stream: Optional[int] = None) -> dict:
        """Mean per-step kernel times (ms) over n steps, from CUDA events
        recorded around each kernel on its launching stream."""
        ms = np.zeros(5, dtype=np.float64)
        _check(load_library().fdtd_profile_step(self.h, int(n), ctypes.c_void_p(stream) if stream else None, _dp(ms)))
        return dict(zip(["e_sweep", "e_extra", "h_sweep", "h_extra", "advance_flush"], ms.tolist()))

    SWEEP_KINDS = {"auto": 0, "regs": 1, "tma": 2, "flat": 3, "staged": 4, "eh": 5}

    def set_sweep_kernel(self, kind: str) -> None:
        _check(load_library().fdtd_set_sweep_kernel(self.h, self.SWEEP_KINDS[kind]))

    def use_graphs(self, enable: bool) -> None:
        _check(load_library().fdtd_use_graphs(self.h, 1 if enable else 0))

    def error_flags(self) -> int:
        v = ctypes.c_int()
        _check(load_library().fdtd_error_flags(self.h, ctypes.byref(v)))
        return v.value

    def synchronize(self) -> None:
        _check(load_library().fdtd_synchronize(self.h))

    # ------------------------------------------------------------ read back
    def read_quantity(self, q: int, lo, hi) -> np.ndarray:
        """Quantity q (P.QUANTITIES: E, H, the surface currents Je, Jh and the
        surface charge density rho) over the inclusive box lo..hi from the
        current fields, shape (nz_b, ny_b, nx_b)."""
        n = [h - l + 1 for l, h in zip(lo, hi)]
        out = np.empty(n[0] * n[1] * n[2], dtype=np.float64)
        _check(load_library().fdtd_read_quantity(self.h, int(q), _ip(lo), _ip(hi), _dp(out)))
        return out.reshape(n[2], n[1], n[0])

    def surface(self, name: str) -> np.ndarray:
        """Surface quantity `name` (rho, Jex, .., Jhz) on every interior cell,
        zero elsewhere and where the mode has none."""
        nx, ny, nz = self.shape
        out = np.zeros((nz, ny, nx))
        q = P.QUANTITIES[name]
        three = self.mode == P.THREED
        lo, hi = (1, 1, 1 if three else 0), (nx - 2, ny - 2, nz - 2 if three else 0)
        if P.quantity_in_mode(self.mode, q):
            out[lo[2]:hi[2] + 1, 1:ny - 1, 1:nx - 1] = self.read_quantity(q, lo, hi)
        return out

    def get(self, name: str) -> np.ndarray:
        if isinstance(name, str) and name in P.SURFACE_NAMES:
            return self.surface(name)
        which = ALL_NAMES.index(name) if isinstance(name, str) and name in ALL_NAMES else int(name)
        nx, ny, nz = self.shape
        out = np.empty(nx * ny * nz, dtype=np.float64)
        _check(load_library().fdtd_download(self.h, which, _dp(out)))
        return out.reshape(nz, ny, nx)

    def get_pole(self, pole: int, name: str) -> np.ndarray:
        if pole == 0:
            return self.get(name)
        r = ["Px", "Py", "Pz", "Jx", "Jy", "Jz"].index(name)
        return self.get(str(36 + (pole - 1) * 6 + r))

    def set(self, name: str, arr: np.ndarray) -> None:
        which = ALL_NAMES.index(name)
        a = np.ascontiguousarray(arr, dtype=np.float64).ravel()
        _check(load_library().fdtd_upload(self.h, which, _dp(a)))

    def dft(self, handle: int) -> np.ndarray:
        """[nf][npoints] complex"""
        L = load_library()
        n = ctypes.c_longlong()
        _check(L.fdtd_dft_npoints(self.h, handle, ctypes.byref(n)))
        nf = self.dft_meta[handle]
        # (re, im) pairs as written by the C ABI are complex128 in memory
        out = np.empty((nf, n.value), dtype=np.complex128)
        _check(L.fdtd_dft_read(self.h, handle, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return out

    def check_finite(self) -> None:
        _check(load_library().fdtd_check_finite(self.h))

    def field_error(self, ref: "Grid", name: str) -> float:
        """Relative L2 error of field `name` of this grid against the same
        field of grid `ref` (same shape and device), computed on the device
        in FP64 over every cell (fdtd_field_error)."""
        which = ALL_NAMES.index(name)
        e2, r2 = ctypes.c_double(), ctypes.c_double()
        _check(load_library().fdtd_field_error(self.h, ref.h, which, ctypes.byref(e2), ctypes.byref(r2)))
        return float(np.sqrt(e2.value / r2.value)) if r2.value > 0 else float(np.sqrt(e2.value))

    @property
    def step_count(self) -> int:
        v = ctypes.c_longlong()
        _check(load_library().fdtd_get_step(self.h, ctypes.byref(v)))
        return v.value

    @property
    def launch_count(self) -> int:
        v = ctypes.c_longlong()
        _check(load_library().fdtd_launch_count(self.h, ctypes.byref(v)))
        return v.value

    @property
    def memory_bytes(self) -> int:
        v = ctypes.c_longlong()
        _check(load_library().fdtd_memory_bytes(self.h, ctypes.byref(v)))
        return v.value

    def close(self) -> None:
        if getattr(self, "h", None):
            load_library().fdtd_grid_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Independent FP32 2D grids advanced together by one persistent kernel
    launch per step() call (fdtd_batch_*)."""

    def __init__(self, grids):
        L = load_library()
        self.grids = list(grids)
        arr = (ctypes.c_void_p * len(self.grids))(*[g.h.value for g in self.grids])
        h = ctypes.c_void_p()
        _check(L.fdtd_batch_create(len(self.grids), arr, ctypes.byref(h)))
        self.h = h

    def tune(self, steps: int = 4) -> None:
        _check(load_library().fdtd_batch_tune(self.h, steps))

    def step(self, n: int, stream: Optional[int] = None) -> None:
        _check(load_library().fdtd_batch_step(self.h, int(n), ctypes.c_void_p(stream) if stream else None))
        for g in self.grids:
            g._stepped_in_batch = True

    def configure(self, persistent, rows: int) -> None:
        """persistent: True or 'persistent' for the cooperative kernel,
        False or 'per_phase' for one launch per half step."""
        if isinstance(persistent, str):
            persistent = persistent == "persistent"
        _check(load_library().fdtd_batch_configure(self.h, 1 if persistent else 0, int(rows)))

    def info(self) -> dict:
        rows, blocks, items, pers = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        ms = (ctypes.c_float * 8)()
        _check(load_library().fdtd_batch_info(self.h, ctypes.byref(rows), ctypes.byref(blocks), ctypes.byref(items),
                                              ctypes.byref(pers), ms))
        keys = [f"persistent_rows{r}" for r in (1, 2, 4, 8)] + [f"per_phase_rows{r}" for r in (1, 2, 4, 8)]
        return {"rows": rows.value, "blocks": blocks.value, "items": items.value,
                "launch": "persistent" if pers.value else "per_phase",
                "tune_ms_per_step": {k: float(m) for k, m in zip(keys, ms)}}

    def item_rows(self) -> dict:
        """Per grid: the rows of its work items and its size class; and the
        tuner's ms per step with them."""
        n = len(self.grids)
        rows, cls, ms = (ctypes.c_int * n)(), (ctypes.c_int * n)(), ctypes.c_float()
        _check(load_library().fdtd_batch_item_rows(self.h, rows, cls, ctypes.byref(ms)))
        return {"rows": list(rows), "size_class": list(cls), "tuned_ms_per_step": float(ms.value)}

    def set_item_rows(self, rows_per_grid) -> None:
        _check(load_library().fdtd_batch_set_item_rows(self.h, _ip(rows_per_grid)))

    def set_temporal(self, depth: int) -> None:
        """Temporal blocking: `depth` (2, 3 or 4) steps per launch from shared
        memory, or 0 for off (fdtd_batch_set_temporal)."""
        _check(load_library().fdtd_batch_set_temporal(self.h, int(depth)))

    def temporal(self) -> dict:
        """The temporal-blocking depth in use (0: off) and the tuner's ms per
        step with depths 2, 3 and 4 (0: not timed)."""
        d, ms = ctypes.c_int(), (ctypes.c_float * 3)()
        _check(load_library().fdtd_batch_temporal(self.h, ctypes.byref(d), ms))
        return {"depth": d.value, "tune_ms_per_step": {str(k): float(m) for k, m in zip((2, 3, 4), ms)}}

    def error_flags(self) -> int:
        v = ctypes.c_int()
        _check(load_library().fdtd_batch_error_flags(self.h, ctypes.byref(v)))
        return v.value

    def close(self) -> None:
        if getattr(self, "h", None):
            load_library().fdtd_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Adjoint:
    """d(objective)/d(eps_r) of a 2D TM FP32 grid by the discrete adjoint
    (fdtd_adjoint_*): J = sum over the probe box of |DFT_freq(Ez)|^2. The
    grid must be unstepped; forward() steps it and returns J, backward()
    returns dJ/deps_r over the design box as [ny_d, nx_d]."""

    def __init__(self, grid: Grid, probe_lo, probe_hi, freq: float, design_lo, design_hi, ckpt_every: int = 64):
        self.grid = grid
        self.design = (tuple(design_lo), tuple(design_hi))
        h = ctypes.c_void_p()
        _check(load_library().fdtd_adjoint_create(grid.h, _ip(probe_lo), _ip(probe_hi), float(freq), _ip(design_lo),
                                                  _ip(design_hi), int(ckpt_every), ctypes.byref(h)))
        self.h = h

    def forward(self, nsteps: int) -> float:
        J = ctypes.c_double()
        _check(load_library().fdtd_adjoint_forward(self.h, int(nsteps), ctypes.byref(J)))
        return J.value

    def backward(self) -> np.ndarray:
        (x0, y0), (x1, y1) = self.design[0][:2], self.design[1][:2]
        out = np.zeros((y1 - y0 + 1, x1 - x0 + 1))
        _check(load_library().fdtd_adjoint_backward(self.h, _dp(out)))
        return out

    def close(self) -> None:
        if self.h:
            load_library().fdtd_adjoint_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
