"""Problem descriptions for the FDTD hot path.

A ``Problem`` is a plain description of one grid and what acts on it during a
time step: CPML widths, the material table and per-cell (or per-block) ids,
soft sources, TFSF planes and DFT capture regions. The same description
drives the GPU library (``fdtd_b200.grid.Grid.from_problem``) and the CPU
checkers under ``oracle/`` in the tests, so both see identical inputs.

Units are SI as in the reference (include/FDTDConstants.hpp:394-398). The
configs below are written in "grid units" (one cell = dx, one step = dt) and
converted here: frequencies in cycles/step become rad/s via 2*pi*f/dt for the
DFT only; material rates given "in grid units" (w*dt) become w = value/dt.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

# include/FDTDConstants.hpp:394-398
PI = 3.14159265358979323846264338327950288
EPS0 = 8.854e-12
MU0 = PI * 4.0e-7
C0 = 2.99792458e8

# Detail::EMMode order (include/FDTDConstants.hpp:410-415)
TEM, TE, TM, THREED = 0, 1, 2, 3
MODE_NAMES = {"TEM": TEM, "TE": TE, "TM": TM, "ThreeD": THREED, "3D": THREED}

VACUUM, CONSTANT, DRUDE, LORENTZ = 0, 1, 2, 3
SOURCE_TARGETS = {"E": 0, "D": 1, "H": 2, "B": 3}
# boundary conditions of a face (include/BoundaryUpdates.hpp:18-27, 528-760):
# the outer cell beyond the face takes a sign-masked image of the interior
# cell next to the face, or (periodic) of the interior cell at the other end
BOUNDARY_KINDS = {"pec": 1, "pmc": 2, "symmetric": 3, "antisymmetric": 4, "periodic": 5}
MAX_POLES = 4


def ref_sqrt(x: float) -> float:
    """The reference's constexpr Newton sqrt (include/FDTDConstants.hpp:136-156)."""
    curr, prev = x, 0.0
    while curr != prev:
        curr, prev = 0.5 * (curr + x / curr), curr
    return curr


IMP0 = ref_sqrt(MU0 / EPS0)


@dataclass
class Material:
    """One row of the material table.

    kind: VACUUM / CONSTANT (eps_inf) / DRUDE (one pole: plasma freq, gamma) /
    LORENTZ (poles of (delta_eps, resonance freq, gamma)). Frequencies in
    rad/s and gamma in 1/s as the reference's storages take them
    (include/DispersiveMaterials.hpp:778-789, :1078-1088). The reference's
    Lorentz ignores its Delta argument, i.e. delta_eps = 1 reproduces it.
    """

    kind: int = VACUUM
    eps_inf: float = 1.0
    mu_r: float = 1.0
    poles: List[Tuple[float, float, float]] = field(default_factory=list)

    @staticmethod
    def vacuum() -> "Material":
        return Material(VACUUM, 1.0, 1.0, [])

    @staticmethod
    def constant(eps_r: float, mu_r: float = 1.0) -> "Material":
        return Material(CONSTANT, eps_r, mu_r, [])

    @staticmethod
    def drude(eps_inf: float, wp: float, gamma: float) -> "Material":
        return Material(DRUDE, eps_inf, 1.0, [(1.0, wp, gamma)])

    @staticmethod
    def lorentz(eps_inf: float, poles: Sequence[Tuple[float, float, float]]) -> "Material":
        return Material(LORENTZ, eps_inf, 1.0, [tuple(p) for p in poles])


@dataclass
class Source:
    """Soft source (include/Source.hpp:183-261): values[t] added at step t to
    component ``comp`` (0..2) of E (target 'E', after the constitutive
    update), D ('D', before the CPML pass), H ('H', after the magnetic
    constitutive update) or B ('B', before the magnetic CPML pass)."""

    comp: int
    pos: Tuple[int, int, int]
    values: np.ndarray
    target: str = "E"
    # with `hi`, the same source on every cell of the inclusive box pos..hi
    # (a line source); E and H targets only
    hi: Optional[Tuple[int, int, int]] = None


@dataclass
class TFSFPlaneSpec:
    axis: int
    orient: int  # 0 = MIN (normal -axis), 1 = MAX (normal +axis)
    lo: Tuple[int, int, int]
    hi: Tuple[int, int, int]


@dataclass
class TFSF:
    """Plane-wave injection: TFSF planes (include/Source.hpp:472-634), each
    with its own Aux1D grid of ``aux_ncells`` (+50) cells whose source at aux
    step s is aux_values[s-1]. ``origin`` (cells) is where the location
    functor puts 0; cell (i,j,k) sits at ((i,j,k) - origin) * dx."""

    aux_ncells: int
    aux_values: np.ndarray
    origin: Tuple[float, float, float]
    k: Tuple[float, float, float]
    pol_e: Tuple[float, float, float]
    pol_h: Tuple[float, float, float]
    planes: List[TFSFPlaneSpec] = field(default_factory=list)


@dataclass
class DFTRegion:
    """Running DFT of quantity comp (QUANTITIES: 0..2 E, 3..5 H, 6..8 Je,
    9..11 Jh, 12 rho) over the inclusive box lo..hi at frequencies freqs
    (cycles/step). The quantities of E (E, Jh, rho), sampled at the end of
    the E half of step t, carry time index t+1; those of H (H, Je) t+1.5;
    X_f = sum_n x[n] * exp(-2*pi*i*f*n). Boxes of surface quantities lie in
    the interior."""

    comp: int
    lo: Tuple[int, int, int]
    hi: Tuple[int, int, int]
    freqs: Sequence[float]


# quantity codes of the C ABI (FDTD_Q_*): fields, then the surface quantities
# of include/SurfaceQuantities.hpp (Je from H, Jh from E, rho from E)
QUANTITIES = {"Ex": 0, "Ey": 1, "Ez": 2, "Hx": 3, "Hy": 4, "Hz": 5, "Jex": 6, "Jey": 7, "Jez": 8,
              "Jhx": 9, "Jhy": 10, "Jhz": 11, "rho": 12}
SURFACE_NAMES = ["rho", "Jex", "Jey", "Jez", "Jhx", "Jhy", "Jhz"]


def quantity_in_mode(mode: int, q: int) -> bool:
    """Whether quantity q exists in `mode` (rho: TE and ThreeD)."""
    has_e = [mode == THREED or (mode == TE and c < 2) or (mode == TM and c == 2) for c in range(3)]
    has_h = [mode == THREED or (mode == TE and c == 2) or (mode == TM and c < 2) for c in range(3)]
    if q < 3:
        return has_e[q]
    if q < 6:
        return has_h[q - 3]
    if q < 9:
        return has_e[q - 6]
    if q < 12:
        return has_h[q - 9]
    return q == 12 and mode != TM


@dataclass
class Problem:
    mode: int
    shape: Tuple[int, int, int]  # (nx, ny, nz); nz = 1 for 2D
    dx: float
    dt: float
    pml: dict = field(default_factory=dict)  # {(axis, side): ncells}
    # {(axis, side): (m, ma, sigma_max, kappa_max, alpha_max)}: sides graded
    # with PMLParameterModel(m, ma, sMax, kMax, aMax) instead of (dx)
    pml_models: dict = field(default_factory=dict)
    boundaries: dict = field(default_factory=dict)  # {(axis, side): kind in BOUNDARY_KINDS}
    # time policy of the curl updates and TFSF corrections: 1 BD1 (leapfrog),
    # 3 BD3, 4 BD4 (include/YeeUpdates.hpp:182-294)
    time_scheme: int = 1
    materials: List[Material] = field(default_factory=lambda: [Material.vacuum()])
    ids: Optional[np.ndarray] = None  # uint8, shape (nz, ny, nx)
    # per-cell relative permittivity of vacuum/constant cells (> 0 replaces
    # the material's eps_inf), float64, shape (nz, ny, nx)
    eps_map: Optional[np.ndarray] = None
    block_ids: Optional[np.ndarray] = None  # uint16, shape (nbz, nby, nbx)
    block_shift: int = 0
    sources: List[Source] = field(default_factory=list)
    tfsf: Optional[TFSF] = None
    dfts: List[DFTRegion] = field(default_factory=list)
    steps: int = 0
    name: str = ""

    @property
    def dim(self) -> int:
        return 3 if self.mode == THREED else (1 if self.mode == TEM else 2)

    @property
    def ncell(self) -> int:
        nx, ny, nz = self.shape
        return nx * ny * nz

    @property
    def interior_cells(self) -> int:
        nx, ny, nz = self.shape
        n = (nx - 2) * (ny - 2)
        return n * (nz - 2) if self.mode == THREED else n

    def cell_ids(self) -> Optional[np.ndarray]:
        """Per-cell material ids (expanding a block map if one is set)."""
        if self.ids is not None:
            return self.ids
        if self.block_ids is None:
            return None
        nx, ny, nz = self.shape
        s = self.block_shift
        k = np.arange(nz)[:, None, None] >> s
        j = np.arange(ny)[None, :, None] >> s
        i = np.arange(nx)[None, None, :] >> s
        return self.block_ids[k, j, i]


def courant_dt(dx: float, courant: float) -> float:
    return courant * dx / C0


def gaussian_pulse(nsteps: int, t0: float = 60.0, spread: float = 20.0, offset: float = 0.0) -> np.ndarray:
    """g(n) = exp(-((n + offset - t0)/spread)^2) for n = 0..nsteps-1."""
    n = np.arange(nsteps, dtype=np.float64) + offset
    return np.exp(-(((n - t0) / spread) ** 2))


def sinusoid(nsteps: int, freq: float, phase: float = 0.0) -> np.ndarray:
    """The reference's SinData / Sinusoid signal (include/Source.hpp:100-129)
    sampled at t = n dt, with freq in cycles per step: angular frequency
    w = 2 pi freq / dt, s(t) = tanh(t / tau) sin(w t + phase), tau = (10 / w)(pi / 2);
    in steps, tau = 2.5 / freq."""
    n = np.arange(nsteps, dtype=np.float64)
    w = 2.0 * math.pi * freq
    tau = 10.0 / w * math.pi / 2.0
    return np.tanh(n / tau) * np.sin(w * n + phase)


@dataclass
class AdjointSpec:
    """Objective J = sum over the probe box of |DFT_freq(Ez)|^2, gradient over
    the design box (inclusive boxes, z = 0)."""
    probe_lo: Tuple[int, int, int]
    probe_hi: Tuple[int, int, int]
    freq: float
    design_lo: Tuple[int, int, int]
    design_hi: Tuple[int, int, int]
    ckpt_every: int = 64


def ref_tm_polarisation(k):
    """Default TM polarisation of TFSFPlane (include/Source.hpp:577-579)."""
    return (0.0, 0.0, 1.0), (k[1], -k[0], 0.0)


def ref_te_polarisation(k):
    """Default TE polarisation of TFSFPlane (include/Source.hpp:573-576)."""
    return (k[1], -k[0], 0.0), (0.0, 0.0, 1.0)


def tfsf_box_planes(mode: int, lo: Sequence[int], hi: Sequence[int]) -> List[TFSFPlaneSpec]:
    """TFSF planes around the total-field box whose E cells are lo..hi.

    The MIN face of an axis is the plane of cells just outside the box
    (index lo-1) and the MAX face is the box's last plane (index hi), with the
    tangential extent of the box. With the reference's per-cell correction
    (include/Source.hpp:506-531) this is the placement where the D correction
    of a face and the B correction of the same face use the incident field at
    the staggered positions the curl actually reads.
    """
    dim = 3 if mode == THREED else 2
    planes = []
    for a in range(dim):
        for orient in (0, 1):
            plo = list(lo) + [0] * (3 - len(lo))
            phi = list(hi) + [0] * (3 - len(hi))
            idx = lo[a] - 1 if orient == 0 else hi[a]
            plo[a] = idx
            phi[a] = idx
            planes.append(TFSFPlaneSpec(a, orient, tuple(plo), tuple(phi)))
    return planes


# ---------------------------------------------------------------- configs

def config1(n: int = 256, steps: int = 2000, npml: int = 16) -> Problem:
    """2D TM FP64 vacuum, 16-cell CPML, soft Ez Gaussian at the centre, DFT of
    Ez along the centre row at 0.02/0.04/0.06 cycles/step."""
    dx = 1e-6
    dt = courant_dt(dx, 0.99 / math.sqrt(2.0))
    p = Problem(TM, (n, n, 1), dx, dt, name=f"tm{n}_vacuum_cpml{npml}")
    for a in (0, 1):
        for s in (0, 1):
            p.pml[(a, s)] = npml
    c = n // 2
    p.sources.append(Source(2, (c, c, 0), gaussian_pulse(steps), "E"))
    p.dfts.append(DFTRegion(2, (0, c, 0), (n - 1, c, 0), [0.02, 0.04, 0.06]))
    p.steps = steps
    return p


def config2(n: int = 384, steps: int = 1000, npml: int = 12, radius: Optional[int] = None,
            tfsf_inset: Optional[int] = None, dft_inset: Optional[int] = None, nfreq: int = 8,
            shape: Optional[Tuple[int, int, int]] = None) -> Problem:
    """3D, 12-cell CPML, Courant 0.98/sqrt(3), Drude sphere (eps_inf 1, wp*dt
    0.3, gamma*dt 0.01) of radius 64 at the centre, TFSF box inset 24 with an x-propagating
    z-polarised Gaussian plane wave, DFT at 8 frequencies of the 4 tangential
    components on the 6 faces of the box inset 20. Smaller n scales radius
    and insets by n/384. `shape` (nx, ny, nz) replaces the cube n^3; the
    radius and insets then scale with its smallest extent."""
    shape = tuple(shape) if shape is not None else (n, n, n)
    nmin = min(shape)
    scale = nmin / 384.0
    radius = radius if radius is not None else max(2, int(round(64 * scale)))
    tfsf_inset = tfsf_inset if tfsf_inset is not None else max(npml + 3, int(round(24 * scale)))
    dft_inset = dft_inset if dft_inset is not None else max(npml + 2, tfsf_inset - max(1, int(round(4 * scale))))
    dx = 1e-6
    # Courant 0.98/sqrt(3): the reference's Drude update (DispersiveMaterials.hpp
    # :979-998) with wp*dt = 0.3 is stable only while 4 S^2 + (wp dt)^2 <= 4,
    # S = c dt sqrt(3)/dx, i.e. S <= 0.9887; at 0.99 the highest Yee mode in
    # the sphere grows by ~1.1 per step (tests/test_stability_cpu.py)
    dt = courant_dt(dx, 0.98 / math.sqrt(3.0))
    name = f"3d{n}_drude_sphere_tfsf_dft" if shape == (n, n, n) else \
        f"3d{shape[0]}x{shape[1]}x{shape[2]}_drude_sphere_tfsf_dft"
    p = Problem(THREED, shape, dx, dt, name=name)
    for a in range(3):
        for s in (0, 1):
            p.pml[(a, s)] = npml
    p.materials = [Material.vacuum(), Material.drude(1.0, 0.3 / dt, 0.01 / dt)]
    cx, cy, cz = (v // 2 for v in shape)
    r2 = ((np.arange(shape[2]) - cz)[:, None, None] ** 2 + (np.arange(shape[1]) - cy)[None, :, None] ** 2
          + (np.arange(shape[0]) - cx)[None, None, :] ** 2)
    p.ids = (r2 <= radius * radius).astype(np.uint8)
    lo = (tfsf_inset,) * 3
    hi = tuple(v - 1 - tfsf_inset for v in shape)
    k = (1.0, 0.0, 0.0)
    # E along z, H along y: the aux Hy already carries the sign of the
    # incident Hy, so the H polarisation multiplying it is +y.
    p.tfsf = TFSF(aux_ncells=max(shape), aux_values=gaussian_pulse(steps, offset=1.0), origin=(cx, cy, cz), k=k,
                  pol_e=(0.0, 0.0, 1.0), pol_h=(0.0, 1.0, 0.0), planes=tfsf_box_planes(THREED, lo, hi))
    freqs = [0.01 * (q + 1) for q in range(nfreq)]
    for a in range(3):
        for side in (0, 1):
            plo = [dft_inset] * 3
            phi = [v - 1 - dft_inset for v in shape]
            plo[a] = phi[a] = dft_inset if side == 0 else shape[a] - 1 - dft_inset
            tang = [b for b in range(3) if b != a]
            for b in tang:
                p.dfts.append(DFTRegion(b, tuple(plo), tuple(phi), freqs))
                p.dfts.append(DFTRegion(3 + b, tuple(plo), tuple(phi), freqs))
    p.steps = steps
    return p


def config3(nproblems: int = 64, steps: int = 3000, seed: int = 0, nmin: int = 128, nmax: int = 1024,
            npml: int = 10, nrect: int = 10) -> List[Problem]:
    """Batched 2D TE: `nproblems` grids with Nx, Ny uniform in [nmin, nmax]
    from `seed`; each with `nrect` axis-aligned dielectric rectangles (eps_r
    uniform in [1, 12], sides uniform in [8, 64]) placed inside the CPML-free
    interior, a 10-cell CPML, and a Gaussian soft Hz source at a random
    interior cell."""
    dx = 1e-6
    dt = courant_dt(dx, 0.99 / math.sqrt(2.0))
    rng = np.random.default_rng(seed)
    out = []
    for q in range(nproblems):
        nx, ny = (int(v) for v in rng.integers(nmin, nmax + 1, size=2))
        p = Problem(TE, (nx, ny, 1), dx, dt, name=f"te{nx}x{ny}_rects")
        for a in (0, 1):
            for s in (0, 1):
                p.pml[(a, s)] = npml
        lo = npml + 2
        ids = np.zeros((1, ny, nx), np.uint8)
        mats = [Material.vacuum()]
        for r in range(nrect):
            w, h = (int(v) for v in rng.integers(8, 65, size=2))
            w = min(w, nx - 2 * lo - 1)
            h = min(h, ny - 2 * lo - 1)
            x0 = int(rng.integers(lo, nx - lo - w))
            y0 = int(rng.integers(lo, ny - lo - h))
            mats.append(Material.constant(float(rng.uniform(1.0, 12.0))))
            ids[0, y0:y0 + h, x0:x0 + w] = len(mats) - 1
        p.materials = mats
        p.ids = ids
        si, sj = int(rng.integers(lo, nx - lo)), int(rng.integers(lo, ny - lo))
        p.sources.append(Source(2, (si, sj, 0), gaussian_pulse(steps), "H"))
        p.steps = steps
        out.append(p)
    return out


def config4(n: int = 512, steps: int = 4000, npml: int = 16, design: int = 128, seed: int = 0, nprobe: int = 16,
            freq: float = 0.05, ckpt_every: int = 64):
    """Adjoint inverse design, 2D TM: 16-cell CPML, a central design box of
    design^2 cells with eps_r uniform in [1, 12] from `seed`, a line source of
    Ez (the Sinusoid signal at `freq` cycles per step) on column npml + 8
    over every interior row, and the objective sum |DFT_freq(Ez)|^2 over
    `nprobe` cells of column n - 1 - (npml + 8), centred. Returns (Problem,
    AdjointSpec)."""
    dx = 1e-6
    dt = courant_dt(dx, 0.99 / math.sqrt(2.0))
    p = Problem(TM, (n, n, 1), dx, dt, name=f"tm{n}_adjoint_design{design}")
    for a in (0, 1):
        for s in (0, 1):
            p.pml[(a, s)] = npml
    rng = np.random.default_rng(seed)
    d0 = (n - design) // 2
    eps = np.zeros((1, n, n))
    eps[0, d0:d0 + design, d0:d0 + design] = rng.uniform(1.0, 12.0, size=(design, design))
    p.eps_map = eps
    col = npml + 8
    p.sources.append(Source(2, (col, 1, 0), sinusoid(steps, freq), "E", hi=(col, n - 2, 0)))
    pc = n - 1 - (npml + 8)
    j0 = n // 2 - nprobe // 2
    spec = AdjointSpec((pc, j0, 0), (pc, j0 + nprobe - 1, 0), freq, (d0, d0, 0), (d0 + design - 1, d0 + design - 1, 0),
                       ckpt_every)
    p.steps = steps
    return p, spec


def config5(n: int = 768, steps: int = 500, npml: int = 16, block: int = 32, seed: int = 0,
            nfreq: int = 4, shape: Optional[Tuple[int, int, int]] = None) -> Problem:
    """3D, 16-cell CPML, two-pole Lorentz everywhere (delta_eps 1.5, w0*dt
    0.1, delta*dt 0.005 and 0.8, 0.25, 0.02), eps_inf per 32^3 block uniform
    in [1,6] from `seed`, soft Ez dipole at the centre, DFT of Ez at 4
    frequencies on the central z plane. `shape` (nx, ny, nz) replaces the
    cube n^3."""
    shape = tuple(shape) if shape is not None else (n, n, n)
    dx = 1e-6
    dt = courant_dt(dx, 0.99 / math.sqrt(3.0))
    name = f"3d{n}_lorentz2_blocks{block}" if shape == (n, n, n) else \
        f"3d{shape[0]}x{shape[1]}x{shape[2]}_lorentz2_blocks{block}"
    p = Problem(THREED, shape, dx, dt, name=name)
    for a in range(3):
        for s in (0, 1):
            p.pml[(a, s)] = npml
    shift = int(round(math.log2(block)))
    assert 1 << shift == block
    nb = [(v + block - 1) // block for v in shape]
    rng = np.random.default_rng(seed)
    eps = rng.uniform(1.0, 6.0, size=nb[0] * nb[1] * nb[2])
    poles = [(1.5, 0.1 / dt, 0.005 / dt), (0.8, 0.25 / dt, 0.02 / dt)]
    p.materials = [Material.lorentz(float(e), poles) for e in eps]
    p.block_ids = np.arange(eps.size, dtype=np.uint16).reshape(nb[2], nb[1], nb[0])
    p.block_shift = shift
    cx, cy, cz = (v // 2 for v in shape)
    p.sources.append(Source(2, (cx, cy, cz), gaussian_pulse(steps), "E"))
    freqs = [0.01 * (q + 1) for q in range(nfreq)]
    p.dfts.append(DFTRegion(2, (0, 0, cz), (shape[0] - 1, shape[1] - 1, cz), freqs))
    p.steps = steps
    return p
