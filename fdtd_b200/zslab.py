"""Z-slab decomposition of one 3D grid across ranks.

Each rank owns a contiguous range of interior z planes [z0, z1) of the global
grid and holds it as an ordinary grid of (z1 - z0) + 2 planes: local plane 0
is global plane z0 - 1 and local plane nz_l - 1 is global plane z1. Where those
are the global outer ring they stay untouched, as in a single grid; between
ranks they are ghost planes, refilled every half step:

* before the E half, a rank's ghost plane 0 takes Hx, Hy of the plane below
  its range (the top plane of the rank below), since the E update at its
  first plane differences H along z;
* before the H half, its top ghost plane takes Ex, Ey of the plane above its
  range (the first plane of the rank above).

This is the exchange of the reference's MPI boundary (BoundaryUpdates.hpp:
919-1051), restated for SoA planes. Everything else is cut along z: material
ids and the permittivity map are sliced; the z CPML and z-face boundary
conditions stay with the first and last rank (range boundaries are kept out of the CPML slabs, and out of the
middle of material blocks); sources, TFSF planes (each rank replays the same
aux grid) and DFT regions are clipped to each range and moved to local
coordinates. Per cell the arithmetic is that of the single grid, so the
decomposed run reproduces it to the last bit.

Two drivers share the slicing: `ZSlabDomain` keeps every range in one process
(on one device; no kernel ever waits on another), and `ZSlabRank` is one range
per process, with the ghost planes sent over torch.distributed (NCCL between
GPUs, gloo on CPU).

Both overlap the transfer of a ghost plane with the sweep, through the split
half step of the C ABI (fdtd_step_half_part): part 0 of a half step sweeps
every plane whose update reads no ghost plane while the planes travel; once
they have landed, part 1 sweeps the plane next to the ghost and finishes the
half step. Per cell the arithmetic is unchanged.
"""
from __future__ import annotations

import copy
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import problem as P

H_HALO = ("Hx", "Hy")  # read by the E half from the plane below
E_HALO = ("Ex", "Ey")  # read by the H half from the plane above


def _slab_planes(nz: int, p: P.Problem) -> Tuple[int, int]:
    """Last global plane of the low z CPML slab and first plane of the high one."""
    lo = p.pml.get((2, 0), 0)
    hi = p.pml.get((2, 1), 0)
    last_lo = lo + 1 if lo > 0 else 0
    first_hi = nz - 2 - hi if hi > 0 else nz - 1
    return last_lo, first_hi


def partition_z(p: P.Problem, world: int) -> List[Tuple[int, int]]:
    """Owned interior plane ranges [z0, z1) of `world` ranks, as even as the
    constraints allow: boundaries outside the z CPML slabs and, with a block
    material map, on block edges."""
    nz = p.shape[2]
    if p.mode != P.THREED:
        raise ValueError("z-slab decomposition is for 3D grids")
    interior = nz - 2
    if world < 1 or world > interior:
        raise ValueError("world must be 1..nz-2")
    if world > 1 and "periodic" in (p.boundaries.get((2, 0)), p.boundaries.get((2, 1))):
        raise ValueError("a periodic z boundary joins the first and last rank: not decomposed along z")
    last_lo, first_hi = _slab_planes(nz, p)
    align = (1 << p.block_shift) if (p.block_ids is not None and p.ids is None) else 1
    bounds = [1]
    for r in range(1, world):
        b = 1 + round(r * interior / world)
        b = max(b, last_lo + 1)
        b = min(b, first_hi)
        b = 1 + ((b - 1) // align) * align  # z0 - 1 on a block edge
        if b <= bounds[-1] or b > first_hi or b <= last_lo:
            raise ValueError("the grid is too thin in z for this many ranks around its CPML and blocks")
        bounds.append(b)
    bounds.append(nz - 1)
    return [(bounds[r], bounds[r + 1]) for r in range(world)]


def _clip_box(lo, hi, z0, z1):
    zl, zh = max(lo[2], z0), min(hi[2], z1 - 1)
    if zl > zh:
        return None
    off = z0 - 1
    return (lo[0], lo[1], zl - off), (hi[0], hi[1], zh - off)


def local_problem(p: P.Problem, z0: int, z1: int) -> P.Problem:
    """The problem of the rank that owns global planes [z0, z1)."""
    nx, ny, nz = p.shape
    off = z0 - 1
    nzl = z1 - z0 + 2
    q = copy.copy(p)
    q.shape = (nx, ny, nzl)
    q.name = f"{p.name}_z{z0}-{z1}"
    q.pml = {k: v for k, v in p.pml.items() if k[0] != 2}
    if z0 == 1 and p.pml.get((2, 0), 0) > 0:
        q.pml[(2, 0)] = p.pml[(2, 0)]
    if z1 == nz - 1 and p.pml.get((2, 1), 0) > 0:
        q.pml[(2, 1)] = p.pml[(2, 1)]
    q.boundaries = {k: v for k, v in p.boundaries.items() if k[0] != 2}
    if z0 == 1 and (2, 0) in p.boundaries:
        q.boundaries[(2, 0)] = p.boundaries[(2, 0)]
    if z1 == nz - 1 and (2, 1) in p.boundaries:
        q.boundaries[(2, 1)] = p.boundaries[(2, 1)]
    q.ids = None if p.ids is None else np.ascontiguousarray(p.ids[off:off + nzl])
    q.block_ids = None
    if p.block_ids is not None and p.ids is None:
        s = p.block_shift
        nb = ((nzl - 1) >> s) + 1
        q.block_ids = np.ascontiguousarray(p.block_ids[(off >> s):(off >> s) + nb])
        if q.block_ids.shape[0] < nb:
            raise ValueError("block map does not cover the slab")
    q.eps_map = None if p.eps_map is None else np.ascontiguousarray(p.eps_map[off:off + nzl])
    q.sources = []
    for s in p.sources:
        if s.hi is None:
            if z0 <= s.pos[2] < z1:
                q.sources.append(P.Source(s.comp, (s.pos[0], s.pos[1], s.pos[2] - off), s.values, s.target))
        else:
            c = _clip_box(s.pos, s.hi, z0, z1)
            if c is not None:
                q.sources.append(P.Source(s.comp, c[0], s.values, s.target, hi=c[1]))
    if p.tfsf is not None:
        t = copy.copy(p.tfsf)
        planes = []
        for pl in p.tfsf.planes:
            c = _clip_box(pl.lo, pl.hi, z0, z1)
            if c is not None:
                pq = copy.copy(pl)
                pq.lo, pq.hi = c
                planes.append(pq)
        t.planes = planes
        t.origin = (t.origin[0], t.origin[1], t.origin[2] - off)
        q.tfsf = t if planes else None
    q.dfts = []
    q.dft_map = []  # local region index -> global region index
    for gi, r in enumerate(p.dfts):
        c = _clip_box(r.lo, r.hi, z0, z1)
        if c is not None:
            # Je_x, Je_y and rho read the plane below, Jh_x and Jh_y the plane
            # above; at a slab boundary that plane is a ghost whose exchange
            # comes after the half step's DFT sample
            lo_z, hi_z = c[0][2] + off, c[1][2] + off
            if r.comp in (6, 7, 12) and z0 > 1 and lo_z == z0:
                raise ValueError(f"DFT region {gi} of quantity {r.comp} reads the plane below slab boundary {z0}")
            if r.comp in (9, 10) and z1 < nz - 1 and hi_z == z1 - 1:
                raise ValueError(f"DFT region {gi} of quantity {r.comp} reads the plane above slab boundary {z1}")
            q.dfts.append(P.DFTRegion(r.comp, c[0], c[1], list(r.freqs)))
            q.dft_map.append(gi)
    return q


def merge_dfts(p: P.Problem, parts: Sequence[Tuple[List[int], List[np.ndarray]]]) -> List[np.ndarray]:
    """Global DFT spectra [nf][npoints] from the ranks' (dft_map, spectra) in
    rank order: a region's points run x fastest and z slowest, so the ranks'
    pieces follow one another."""
    out = []
    for gi in range(len(p.dfts)):
        pieces = [spec[li] for dmap, spec in parts for li, g in enumerate(dmap) if g == gi]
        out.append(np.concatenate(pieces, axis=1))
    return out


class ZSlabDomain:
    """Every z range of one grid in this process, on one device: the
    decomposed run on a single GPU (or as a check of the decomposition). The
    sweeps run on one stream and the ghost-plane copies on a second one, so
    that each half step's copies overlap the slabs' interior sweeps (part 0);
    events order the copies after the half step that produced their planes
    and the ghost-adjacent sweeps (part 1) after the copies."""

    def __init__(self, p: P.Problem, world: int, precision: str = "f32", device: int = 0):
        import torch
        from .grid import Grid
        self.p = p
        self.ranges = partition_z(p, world)
        self.parts = [local_problem(p, z0, z1) for z0, z1 in self.ranges]
        self.grids = [Grid.from_problem(q, precision, device=device) for q in self.parts]
        self.torch = torch
        self.stream_obj = torch.cuda.Stream(device)
        self.copy_obj = torch.cuda.Stream(device)
        self.stream = self.stream_obj.cuda_stream
        self.copy_stream = self.copy_obj.cuda_stream
        self.stream_obj.wait_stream(torch.cuda.current_stream(device))
        self.copy_obj.wait_stream(torch.cuda.current_stream(device))

    def _halo(self, names, up: bool):
        """The ghost-plane copies of one half step on the copy stream, plane
        to plane (fdtd_copy_plane_between)."""
        n = len(self.grids)
        for r in range(n - 1):
            lower, upper = self.grids[r], self.grids[r + 1]
            for name in names:
                if up:  # lower's top owned plane -> upper's ghost plane 0
                    lower.copy_plane_to(name, lower.shape[2] - 2, upper, 0, self.copy_stream)
                else:  # upper's first owned plane -> lower's top ghost plane
                    upper.copy_plane_to(name, 1, lower, lower.shape[2] - 1, self.copy_stream)

    def _half(self, phase: int, names, up: bool):
        # the planes to send are final once the previous half step has run
        self.copy_obj.wait_stream(self.stream_obj)
        self._halo(names, up)
        for g in self.grids:
            g.step_half_part(phase, 0, self.stream)
        self.stream_obj.wait_stream(self.copy_obj)
        for g in self.grids:
            g.step_half_part(phase, 1, self.stream)

    def step(self, n: int) -> None:
        for _ in range(n):
            self._half(0, H_HALO, up=True)
            self._half(1, E_HALO, up=False)

    def get(self, name: str) -> np.ndarray:
        """The global field assembled from the ranges' owned planes."""
        self.stream_obj.synchronize()
        return np.concatenate([g.get(name)[1:-1] for g in self.grids], axis=0)

    def dft(self, q: int) -> np.ndarray:
        self.stream_obj.synchronize()
        parts = [(lp.dft_map, [g.dft(li) for li in range(len(lp.dfts))]) for lp, g in zip(self.parts, self.grids)]
        return merge_dfts(self.p, parts)[q]


class ZSlabRank:
    """One z range per process (one process per GPU): this rank's grid and
    the exchange of its ghost planes with the ranks above and below over
    torch.distributed (NCCL between GPUs; gloo with CPU tensors). Each half
    step posts the plane transfers, runs the interior part of the sweep,
    waits for the transfers, writes the ghost plane and runs the rest. `grid`
    is anything with step_half_part(phase, part), read_plane(name, k) ->
    tensor, write_plane(name, k, tensor) and empty_plane()."""

    def __init__(self, grid, nz_local: int, rank: int, world: int, group=None):
        self.g = grid
        self.nzl = nz_local
        self.rank, self.world, self.group = rank, world, group

    def _post(self, names, up: bool):
        """Send this rank's planes of `names` and request the neighbour's:
        the transfers run while the interior sweep does."""
        import torch.distributed as dist
        peer_send = self.rank + 1 if up else self.rank - 1
        peer_recv = self.rank - 1 if up else self.rank + 1
        k_send = self.nzl - 2 if up else 1
        k_recv = 0 if up else self.nzl - 1
        reqs, recvd = [], []
        for name in names:
            if 0 <= peer_send < self.world:
                reqs.append(dist.isend(self.g.read_plane(name, k_send), peer_send, group=self.group))
            if 0 <= peer_recv < self.world:
                buf = self.g.empty_plane()
                reqs.append(dist.irecv(buf, peer_recv, group=self.group))
                recvd.append((name, buf))
        return reqs, recvd, k_recv

    def _land(self, pending):
        """Wait for the transfers and write the received planes into the
        ghost plane."""
        reqs, recvd, k_recv = pending
        for r in reqs:
            r.wait()
        for name, buf in recvd:
            self.g.write_plane(name, k_recv, buf)

    def _half(self, phase: int, names, up: bool):
        pending = self._post(names, up)
        self.g.step_half_part(phase, 0)
        self._land(pending)
        self.g.step_half_part(phase, 1)

    def step(self, n: int) -> None:
        import contextlib
        ctx = self.g.stream_context() if hasattr(self.g, "stream_context") else contextlib.nullcontext()
        with ctx:
            for _ in range(n):
                self._half(0, H_HALO, up=True)
                self._half(1, E_HALO, up=False)


class GpuSlab:
    """The grid of one rank, with plane access through torch CUDA tensors. The
    grid's kernels, the plane copies and (inside stream_context) the NCCL
    transfers all run on one stream of this object, in the order issued."""

    def __init__(self, q: P.Problem, precision: str = "f32", device: int = 0):
        import torch
        from .grid import Grid
        self.torch = torch
        self.q = q
        self.grid = Grid.from_problem(q, precision, device=device)
        self.dtype = torch.float32 if precision in ("f32", "fused") else torch.float64
        self.device = device
        self.n = q.shape[0] * q.shape[1]
        self.stream = torch.cuda.Stream(device)

    def stream_context(self):
        return self.torch.cuda.stream(self.stream)

    def synchronize(self):
        self.stream.synchronize()

    def _stream(self):
        return self.stream.cuda_stream

    def empty_plane(self):
        return self.torch.empty(self.n, dtype=self.dtype, device=f"cuda:{self.device}")

    def read_plane(self, name, k):
        t = self.empty_plane()
        self.grid.copy_plane(name, k, t.data_ptr(), False, self._stream())
        return t

    def write_plane(self, name, k, t):
        self.grid.copy_plane(name, k, t.data_ptr(), True, self._stream())

    def step_half(self, phase):
        self.grid.step_half(phase, self._stream())

    def step_half_part(self, phase, part):
        self.grid.step_half_part(phase, part, self._stream())
