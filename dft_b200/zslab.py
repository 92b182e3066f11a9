"""Z-slab domain decomposition of the 3D grid over ranks (one process per GPU).

The reference solves on one grid in one thread.  Here the grid is split along z into
contiguous runs of owned planes, one per rank, and each rank holds its planes plus halo
planes copied from its neighbours:

* Jacobi Poisson (`calculateHartreePotential`, HartreePotentialMolecule.cpp:99-324): T halo
  planes per side let a rank run T sweeps between exchanges.  The stop measure max|dV| of
  every sweep is folded over the rank's own planes, the T values are reduced with MAX over
  ranks, and the first sweep that meets the stop rule (max|dV| < tol, or the cap) ends the
  solve.  When it falls inside a block the block is replayed from its start up to that sweep.
  Values and sweep count are bit-identical to `dft_hartree_dev` on the whole grid.
* H psi (`applyMolecularKohnShamHamiltonian`, KohnShamHamiltonianMolecule.cpp:78-177): one
  halo plane per side; the owned planes are bit-identical to the whole-grid result.

Transport: `torch.distributed` point-to-point (NCCL over NVLink / NVSwitch between GPUs, gloo
on the CPU); every halo plane lands in the receiving rank's own memory before a kernel reads
it.  `LocalSlabs` holds all ranks' slabs in one process and exchanges by copies, which runs
the same decomposition on one device.

* XC (ExchangeCorrelationMolecule.cpp:576-842): two halo planes per side; potentials
  bit-identical on the owned planes, E_xc summed over ranks.
* Gram products (the block eigensolver's dV A^T B): per-rank products over the owned planes,
  summed over ranks.

The compute goes through `CudaSlabOps` (the slab kernels of libdft_b200); the driver takes
any object with the same methods.
"""
from __future__ import annotations

from typing import Dict, List, Optional, Sequence, Tuple

import ctypes as C

import torch
import torch.distributed as dist


def owned_planes(nz: int, world: int) -> List[Tuple[int, int]]:
    """Contiguous runs [a, b) of the planes 0..nz-1, one per rank, sizes differing by at most
    one (the first nz % world ranks take one more).  The faces z = 0 and z = nz-1 belong to the
    first and the last rank."""
    if world < 1:
        raise ValueError("world size must be at least 1")
    if nz < world:
        raise ValueError(f"{nz} planes cannot give each of {world} ranks a plane")
    base, extra = divmod(nz, world)
    runs, a = [], 0
    for r in range(world):
        b = a + base + (1 if r < extra else 0)
        runs.append((a, b))
        a = b
    return runs


class SlabLayout:
    """Owned planes and slab extents of an (nx, ny, nz) grid split over `world` ranks with
    `halo` halo planes per side.  The halo is capped by the smallest owned run, so that every
    halo plane is an owned plane of the adjacent rank."""

    def __init__(self, shape: Sequence[int], world: int, halo: int):
        self.nx, self.ny, self.nz = (int(s) for s in shape)
        self.world = int(world)
        if halo < 1:
            raise ValueError("halo must be at least 1")
        self.own = owned_planes(self.nz, self.world)
        self.halo = int(min(halo, min(b - a for a, b in self.own)))

    @property
    def plane_points(self) -> int:
        return self.nx * self.ny

    def extent(self, r: int) -> Tuple[int, int]:
        a, b = self.own[r]
        return max(0, a - self.halo), min(self.nz, b + self.halo)

    def planes(self, r: int) -> int:
        lo, hi = self.extent(r)
        return hi - lo

    def points(self, r: int) -> int:
        return self.planes(r) * self.plane_points

    def owned_rows(self, r: int) -> slice:
        """The owned planes as rows of the slab's (planes, nx*ny) view."""
        lo, _ = self.extent(r)
        a, b = self.own[r]
        return slice(a - lo, b - lo)

    def scatter(self, field: torch.Tensor, r: int) -> torch.Tensor:
        """Rank r's slab (owned + halo planes) of a whole-grid field whose last dimension is
        nz*ny*nx (x fastest); a leading band dimension is kept.  Returns a contiguous copy."""
        lo, hi = self.extent(r)
        n = self.plane_points
        return field[..., lo * n:hi * n].contiguous()

    def gather(self, slabs: Dict[int, torch.Tensor]) -> torch.Tensor:
        """The whole-grid field from every rank's slab (owned planes only)."""
        n = self.plane_points
        parts = []
        for r in range(self.world):
            s = slabs[r]
            rows = self.owned_rows(r)
            parts.append(s[..., rows.start * n:rows.stop * n])
        return torch.cat(parts, dim=-1)


def _check_width(layout: SlabLayout, width: int) -> None:
    if layout.world > 1 and not 1 <= width <= layout.halo:
        raise ValueError(f"a halo exchange of {width} planes needs a layout with at least that many halo planes "
                         f"(this one has {layout.halo})")


def _rows(t: torch.Tensor, n: int) -> torch.Tensor:
    """(bands, planes, nx*ny) view of a slab field (one band when the field is flat)."""
    return t.view(-1, t.shape[-1] // n, n)


class LocalSlabs:
    """Every rank's slab held by this process: halos move by copies between the slabs and the
    reductions run over the held values.  Runs the decomposition on one device."""

    def __init__(self, world: int):
        self.world = int(world)
        self.ranks = list(range(self.world))

    def exchange(self, layout: SlabLayout, fields: Dict[int, torch.Tensor], width: int) -> None:
        _check_width(layout, width)
        n = layout.plane_points
        for r in self.ranks:
            lo, _ = layout.extent(r)
            a, b = layout.own[r]
            dst = _rows(fields[r], n)
            if r > 0:
                plo, _ = layout.extent(r - 1)
                dst[:, a - width - lo:a - lo].copy_(_rows(fields[r - 1], n)[:, a - width - plo:a - plo])
            if r + 1 < self.world:
                nlo, _ = layout.extent(r + 1)
                dst[:, b - lo:b + width - lo].copy_(_rows(fields[r + 1], n)[:, b - nlo:b + width - nlo])

    def allreduce_max(self, values: Dict[int, torch.Tensor]) -> torch.Tensor:
        return torch.stack([values[r] for r in self.ranks]).amax(dim=0)

    def allreduce_sum(self, values: Dict[int, torch.Tensor]) -> torch.Tensor:
        out = values[self.ranks[0]].clone()
        for r in self.ranks[1:]:
            out += values[r]
        return out


class ProcessGroupSlabs:
    """This process holds its own rank's slab; halos move by torch.distributed point-to-point
    sends and receives (batched), the reductions are all-reduces.  `group` defaults to the
    world group."""

    def __init__(self, group=None):
        if not (dist.is_available() and dist.is_initialized()):
            raise RuntimeError("ProcessGroupSlabs needs an initialised torch.distributed process group")
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.ranks = [self.rank]

    def _peer(self, r: int) -> int:
        return r if self.group is None else dist.get_global_rank(self.group, r)

    def exchange(self, layout: SlabLayout, fields: Dict[int, torch.Tensor], width: int) -> None:
        _check_width(layout, width)
        r = self.rank
        n = layout.plane_points
        lo, _ = layout.extent(r)
        a, b = layout.own[r]
        view = _rows(fields[r], n)
        ops, landing = [], []
        if r > 0:
            ops.append(dist.P2POp(dist.isend, view[:, a - lo:a + width - lo].contiguous(), self._peer(r - 1),
                                  self.group))
            buf = torch.empty((view.shape[0], width, n), dtype=view.dtype, device=view.device)
            ops.append(dist.P2POp(dist.irecv, buf, self._peer(r - 1), self.group))
            landing.append((slice(a - width - lo, a - lo), buf))
        if r + 1 < self.world:
            ops.append(dist.P2POp(dist.isend, view[:, b - width - lo:b - lo].contiguous(), self._peer(r + 1),
                                  self.group))
            buf = torch.empty((view.shape[0], width, n), dtype=view.dtype, device=view.device)
            ops.append(dist.P2POp(dist.irecv, buf, self._peer(r + 1), self.group))
            landing.append((slice(b - lo, b + width - lo), buf))
        if not ops:
            return
        for w in dist.batch_isend_irecv(ops):
            w.wait()
        for rows, buf in landing:
            view[:, rows].copy_(buf)

    def allreduce_max(self, values: Dict[int, torch.Tensor]) -> torch.Tensor:
        t = values[self.rank].clone()
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=self.group)
        return t

    def allreduce_sum(self, values: Dict[int, torch.Tensor]) -> torch.Tensor:
        t = values[self.rank].clone()
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)
        return t


class CudaSlabOps:
    """The slab kernels of libdft_b200 (`dft_zslab_*_dev`) on torch CUDA tensors of the
    engine's device.  Each call waits for torch's current stream first (the halo copies and
    receives land there) and returns with the engine's stream drained."""

    def __init__(self, engine):
        from . import load
        self.engine = engine
        self.lib = load()

    def _ready(self, t: torch.Tensor) -> None:
        if not t.is_cuda:
            raise TypeError("CudaSlabOps works on CUDA tensors")
        torch.cuda.current_stream(t.device).synchronize()

    def jacobi_init(self, grid, z_lo: int, z_hi: int, Q: float, v: torch.Tensor,
                    guess: Optional[torch.Tensor] = None) -> None:
        from . import _check
        self._ready(v)
        g = grid.c()
        _check(self.lib.dft_zslab_jacobi_init_dev(self.engine.ctx, C.byref(g), int(z_lo), int(z_hi), C.c_double(Q),
                                                  C.c_void_p(guess.data_ptr() if guess is not None else None),
                                                  C.c_void_p(v.data_ptr())))

    def jacobi_sweeps(self, grid, z_lo: int, z_hi: int, own_lo: int, own_hi: int, rho: torch.Tensor,
                      v_in: torch.Tensor, v_out: torch.Tensor, scratch: torch.Tensor, sweeps: int,
                      diffs: torch.Tensor) -> None:
        from . import _check
        self._ready(v_in)
        g = grid.c()
        _check(self.lib.dft_zslab_jacobi_sweeps_dev(self.engine.ctx, C.byref(g), int(z_lo), int(z_hi), int(own_lo),
                                                    int(own_hi), C.c_void_p(rho.data_ptr()),
                                                    C.c_void_p(v_in.data_ptr()), C.c_void_p(v_out.data_ptr()),
                                                    C.c_void_p(scratch.data_ptr()), int(sweeps),
                                                    C.c_void_p(diffs.data_ptr())))

    def hamiltonian(self, grid, z_lo: int, z_hi: int, V: torch.Tensor, psi: torch.Tensor, hpsi: torch.Tensor,
                    nbands: int) -> None:
        from . import _check
        self._ready(psi)
        g = grid.c()
        ld = psi.shape[-1]
        _check(self.lib.dft_zslab_hamiltonian_dev(self.engine.ctx, C.byref(g), int(z_lo), int(z_hi),
                                                  C.c_void_p(V.data_ptr()), C.c_void_p(psi.data_ptr()),
                                                  C.c_void_p(hpsi.data_ptr()), int(nbands), C.c_long(ld)))
        self.engine.synchronize()


    def xc(self, grid, z_lo: int, z_hi: int, own_lo: int, own_hi: int, kind: int, na: torch.Tensor,
           nb: torch.Tensor, va: Optional[torch.Tensor], vb: Optional[torch.Tensor]) -> float:
        from . import _check
        self._ready(na)
        g = grid.c()
        e = C.c_double()
        ptr = lambda t: C.c_void_p(t.data_ptr() if t is not None else None)  # noqa: E731
        _check(self.lib.dft_zslab_xc_dev(self.engine.ctx, C.byref(g), int(z_lo), int(z_hi), int(own_lo), int(own_hi),
                                         int(kind), ptr(na), ptr(nb), ptr(va), ptr(vb), C.byref(e)))
        return e.value

    def gram(self, grid, z_lo: int, z_hi: int, own_lo: int, own_hi: int, A: torch.Tensor, ka: int, B: torch.Tensor,
             kb: int, precision: int = 0) -> torch.Tensor:
        import numpy as np

        from . import _check
        self._ready(A)
        g = grid.c()
        out = np.zeros((ka, kb))
        _check(self.lib.dft_zslab_gram_dev(self.engine.ctx, C.byref(g), int(z_lo), int(z_hi), int(own_lo),
                                           int(own_hi), C.c_void_p(A.data_ptr()), C.c_long(A.shape[-1]), int(ka),
                                           C.c_void_p(B.data_ptr()), C.c_long(B.shape[-1]), int(kb), int(precision),
                                           out.ctypes.data_as(C.POINTER(C.c_double))))
        return torch.from_numpy(out).to(A.device)


def _faces_exact(grid) -> bool:
    """Whether every face's last node lands exactly on its bound (the reference's face values
    are then all zero and the total charge is unused)."""
    def one(n, lo, hi):
        d = (hi - lo) / float(n - 1)
        return lo + float(n - 1) * d == hi
    xmin, xmax, ymin, ymax, zmin, zmax = grid.bounds
    return one(grid.nx, xmin, xmax) and one(grid.ny, ymin, ymax) and one(grid.nz, zmin, zmax)


def hartree_zslab(comm, layout: SlabLayout, grid, rho: Dict[int, torch.Tensor], ops, tol: float = 1e-8,
                  max_sweeps: int = 10000, guess: Optional[Dict[int, torch.Tensor]] = None):
    """`calculateHartreePotential` over z-slabs: returns ({rank: V slab}, sweeps, last max|dV|)
    for the slabs this process holds.  rho (and guess, for a warm interior start) are slabs in
    `layout`; every rank takes the same steps in the same order.

    The stop rule is the reference's (HartreePotentialMolecule.cpp:207-321): sweep s ends the
    solve when its max|dV| over the whole interior is below tol or s reaches max_sweeps.  With
    max_sweeps = 0 the result is the initial state; a grid without interior points reports one
    sweep, as the reference's loop does.  On grids whose faces miss their bounds by rounding the
    face values need the total charge, which is summed over ranks in a different order than the
    reference's sequential sum."""
    if max_sweeps < 0:
        raise ValueError("max_sweeps must be >= 0")
    if (layout.nx, layout.ny, layout.nz) != (grid.nx, grid.ny, grid.nz) or layout.world != comm.world:
        raise ValueError("layout does not match the grid or the number of ranks")
    n = layout.plane_points
    Q = 0.0
    if not _faces_exact(grid):
        part = {}
        for r in comm.ranks:
            rows = layout.owned_rows(r)
            part[r] = rho[r][rows.start * n:rows.stop * n].sum().reshape(1)
        Q = float(comm.allreduce_sum(part).item()) * (grid.getDx() * grid.getDy() * grid.getDz())
    # three buffers per slab: the block's start (read only), the block's result, and scratch
    v, out, scratch, diffs = {}, {}, {}, {}
    for r in comm.ranks:
        lo, hi = layout.extent(r)
        v[r] = torch.empty(layout.points(r), dtype=torch.float64, device=rho[r].device)
        ops.jacobi_init(grid, lo, hi, Q, v[r], None if guess is None else guess[r])
    if max_sweeps == 0:
        return v, 0, 0.0
    if grid.nx < 3 or grid.ny < 3 or grid.nz < 3:
        return v, 1, 0.0
    T = layout.halo
    for r in comm.ranks:
        out[r] = torch.empty_like(v[r])
        scratch[r] = torch.empty_like(v[r])
        diffs[r] = torch.zeros(T, dtype=torch.float64, device=v[r].device)
    done = 0
    while True:
        comm.exchange(layout, v, T)
        nb = min(T, max_sweeps - done)
        for r in comm.ranks:
            lo, hi = layout.extent(r)
            a, b = layout.own[r]
            ops.jacobi_sweeps(grid, lo, hi, a, b, rho[r], v[r], out[r], scratch[r], nb, diffs[r])
        d = comm.allreduce_max({r: diffs[r][:nb] for r in comm.ranks}).cpu().tolist()
        stop = None
        for s in range(nb):
            if d[s] < tol or done + s + 1 >= max_sweeps:
                stop = s + 1
                break
        if stop is not None and stop < nb:
            # the block passed the stop: rerun its first `stop` sweeps from the untouched start
            for r in comm.ranks:
                lo, hi = layout.extent(r)
                a, b = layout.own[r]
                ops.jacobi_sweeps(grid, lo, hi, a, b, rho[r], v[r], out[r], scratch[r], stop, diffs[r])
        v, out = out, v
        if stop is not None:
            return v, done + stop, d[stop - 1]
        done += nb


def hamiltonian_zslab(comm, layout: SlabLayout, grid, V: Dict[int, torch.Tensor], psi: Dict[int, torch.Tensor],
                      nbands: int, ops) -> Dict[int, torch.Tensor]:
    """`applyMolecularKohnShamHamiltonian` over z-slabs for a block of bands: psi slabs are
    (nbands, points) in `layout` (one halo plane is enough and is what is exchanged); the owned
    planes of each returned slab are bit-identical to the whole-grid H psi.  The halo planes of
    psi are overwritten by the exchange."""
    if (layout.nx, layout.ny, layout.nz) != (grid.nx, grid.ny, grid.nz) or layout.world != comm.world:
        raise ValueError("layout does not match the grid or the number of ranks")
    comm.exchange(layout, psi, 1)
    out = {}
    for r in comm.ranks:
        lo, hi = layout.extent(r)
        out[r] = torch.empty_like(psi[r])
        ops.hamiltonian(grid, lo, hi, V[r], psi[r], out[r], nbands)
    return out


def xc_zslab(comm, layout: SlabLayout, grid, kind: int, na: Dict[int, torch.Tensor], nb: Dict[int, torch.Tensor],
             ops, potentials: bool = True):
    """`calculateMolecularSpinExchangeCorrelationPotential` for both spins and
    `calculateMolecularExchangeCorrelationEnergy` (ExchangeCorrelationMolecule.cpp:576-842)
    over z-slabs: returns ({rank: v_alpha}, {rank: v_beta}, E_xc), the potentials' owned planes
    bit-identical to the whole grid's, E_xc the sum of the ranks' parts (a different summation
    order).  The layout needs two halo planes (every rank owns at least two planes); the halo
    planes of na and nb are overwritten by the exchange."""
    if (layout.nx, layout.ny, layout.nz) != (grid.nx, grid.ny, grid.nz) or layout.world != comm.world:
        raise ValueError("layout does not match the grid or the number of ranks")
    if comm.world > 1:
        if layout.halo < 2:
            raise ValueError("XC on slabs needs two halo planes per side")
        comm.exchange(layout, na, 2)
        comm.exchange(layout, nb, 2)
    va, vb, part = {}, {}, {}
    for r in comm.ranks:
        lo, hi = layout.extent(r)
        a, b = layout.own[r]
        va[r] = torch.empty_like(na[r]) if potentials else None
        vb[r] = torch.empty_like(nb[r]) if potentials else None
        e = ops.xc(grid, lo, hi, a, b, kind, na[r], nb[r], va[r], vb[r])
        part[r] = torch.tensor([e], dtype=torch.float64, device=na[r].device)
    return va, vb, float(comm.allreduce_sum(part).item())


def gram_zslab(comm, layout: SlabLayout, grid, A: Dict[int, torch.Tensor], ka: int, B: Dict[int, torch.Tensor],
               kb: int, ops, precision: int = 0) -> torch.Tensor:
    """The block eigensolver's Gram product dV A^T B over z-slabs: each rank's product over its
    owned planes, summed over ranks (an all-reduce of ka x kb values).  A and B are (bands,
    points) slabs in `layout`; their halo planes are not read."""
    if (layout.nx, layout.ny, layout.nz) != (grid.nx, grid.ny, grid.nz) or layout.world != comm.world:
        raise ValueError("layout does not match the grid or the number of ranks")
    part = {}
    for r in comm.ranks:
        lo, hi = layout.extent(r)
        a, b = layout.own[r]
        part[r] = ops.gram(grid, lo, hi, a, b, A[r], ka, B[r], kb, precision)
    return comm.allreduce_sum(part)
