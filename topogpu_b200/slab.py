"""x-slab decomposition of the state solve over ranks (one process per GPU).

The structured mesh is cut along x into contiguous element slabs, one per
rank. Rank r owns elements [e0, e1) and stores the node planes x = e0 .. e1
of every vector, so each interface plane x = e1 between ranks r and r+1 is
stored twice. Vectors are kept *consistent*: both copies hold the full value.

One matvec is the slab's local K u (its own elements only, so interface
planes hold partial sums) followed by an exchange of the two interface
planes with the neighbours (``interface_sum``): one node plane, 3 (ny+1)
(nz+1) values, per direction per matvec. Dot products sum over the planes a
rank owns (an interface plane belongs to the rank on its left) and are
all-reduced. The preconditioner is additive Schwarz with minimal overlap:
rank r applies a V-cycle of the Dirichlet problem on its node planes (the
principal submatrix of the global K on planes e0 .. e1, assembled from the
elements e0-1 .. e1, the planes e0-1 and e1+1 held fixed), and the two
contributions on each interface plane are summed. The sum of the ranks'
symmetric positive definite pieces is symmetric positive definite, so PCG
applies unchanged (the global problem of src/gpu_fem/solver_v4.py:146-267
solved by _cupy_pcg, solver_v2.py:552-624, on a partitioned mesh).

The per-rank arithmetic is behind ``SlabLocalOps``: ``CudaSlabOps`` runs it
through libtopo_b200 (a context on the slab for K u, a context on the
extended slab for the V-cycle); any other implementation with the same two
methods (the tests use one on the CPU) plugs into ``SlabPCG`` unchanged.
Communication goes through ``torch.distributed`` point-to-point calls and
all-reduces: NCCL on GPUs, gloo on CPU.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Protocol

import numpy as np
import torch


def partition(nelx: int, world: int) -> list[tuple[int, int]]:
    """Balanced element ranges [e0, e1) along x, one per rank."""
    if world < 1 or world > nelx:
        raise ValueError(f"cannot cut {nelx} element layers into {world} slabs")
    base, extra = divmod(nelx, world)
    out, e = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        out.append((e, e + n))
        e += n
    return out


@dataclass(frozen=True)
class Slab:
    """Rank ``rank``'s share of an (nelx, nely, nelz) mesh."""

    nel: tuple[int, int, int]
    rank: int
    world: int
    e0: int
    e1: int

    @staticmethod
    def of(nel, rank: int, world: int) -> "Slab":
        nel = tuple(int(v) for v in nel)
        e0, e1 = partition(nel[0], world)[rank]
        return Slab(nel, rank, world, e0, e1)

    @property
    def plane_dofs(self) -> int:
        return 3 * (self.nel[1] + 1) * (self.nel[2] + 1)

    @property
    def n_planes(self) -> int:
        return self.e1 - self.e0 + 1

    @property
    def ndof(self) -> int:
        return self.n_planes * self.plane_dofs

    @property
    def has_left(self) -> bool:
        return self.e0 > 0

    @property
    def has_right(self) -> bool:
        return self.e1 < self.nel[0]

    # extended slab of the preconditioner: elements [x_lo, x_hi)
    @property
    def x_lo(self) -> int:
        return self.e0 - 1 if self.has_left else 0

    @property
    def x_hi(self) -> int:
        return self.e1 + 1 if self.has_right else self.nel[0]

    @property
    def local_nel(self) -> tuple[int, int, int]:
        return (self.e1 - self.e0, self.nel[1], self.nel[2])

    @property
    def ext_nel(self) -> tuple[int, int, int]:
        return (self.x_hi - self.x_lo, self.nel[1], self.nel[2])

    def dof_range(self) -> tuple[int, int]:
        """Global DoF range of planes e0 .. e1 (planes are contiguous, x slowest)."""
        return self.e0 * self.plane_dofs, (self.e1 + 1) * self.plane_dofs

    def ext_dof_range(self) -> tuple[int, int]:
        return self.x_lo * self.plane_dofs, (self.x_hi + 1) * self.plane_dofs

    def element_range(self, lo: int, hi: int) -> tuple[int, int]:
        per = self.nel[1] * self.nel[2]
        return lo * per, hi * per

    def owned_mask(self, dtype=torch.float64, device="cpu") -> torch.Tensor:
        """1 on the planes this rank owns (its left interface plane belongs to
        the left neighbour), 0 elsewhere: dot products count every DoF once."""
        w = torch.ones(self.ndof, dtype=dtype, device=device)
        if self.has_left:
            w[: self.plane_dofs] = 0
        return w

    def local_free_mask(self, free_mask_global: np.ndarray) -> np.ndarray:
        a, b = self.dof_range()
        return np.ascontiguousarray(free_mask_global[a:b])

    def ext_free_mask(self, free_mask_global: np.ndarray) -> np.ndarray:
        """Free mask of the extended slab: the global mask with the planes
        outside e0 .. e1 fixed (the Dirichlet ring of the Schwarz piece)."""
        a, b = self.ext_dof_range()
        m = np.array(free_mask_global[a:b], dtype=np.uint8, copy=True)
        pd = self.plane_dofs
        if self.has_left:
            m[:pd] = 0
        if self.has_right:
            m[-pd:] = 0
        return m

    def ext_offset(self) -> int:
        """Offset of plane e0 inside an extended-slab vector."""
        return (self.e0 - self.x_lo) * self.plane_dofs


def interface_sum(y: torch.Tensor, slab: Slab, dist) -> torch.Tensor:
    """Add the neighbours' partial sums on the two interface planes, in place,
    so both copies of every interface plane hold the full value."""
    if slab.world == 1:
        return y
    pd = slab.plane_dofs
    ops, recv = [], {}
    if slab.has_left:
        recv["l"] = torch.empty(pd, dtype=y.dtype, device=y.device)
        ops += [dist.P2POp(dist.isend, y[:pd].contiguous(), slab.rank - 1),
                dist.P2POp(dist.irecv, recv["l"], slab.rank - 1)]
    if slab.has_right:
        recv["r"] = torch.empty(pd, dtype=y.dtype, device=y.device)
        ops += [dist.P2POp(dist.isend, y[-pd:].contiguous(), slab.rank + 1),
                dist.P2POp(dist.irecv, recv["r"], slab.rank + 1)]
    for req in dist.batch_isend_irecv(ops):
        req.wait()
    if "l" in recv:
        y[:pd] += recv["l"]
    if "r" in recv:
        y[-pd:] += recv["r"]
    return y


def all_dots(pairs, w: torch.Tensor, dist, world: int) -> list[float]:
    """Global dot products of several (a, b) pairs in one all-reduce."""
    v = torch.stack([torch.dot(a * w, b) for a, b in pairs])
    if world > 1:
        dist.all_reduce(v)
    return [float(x) for x in v.cpu()]


class SlabLocalOps(Protocol):
    def matvec(self, u: torch.Tensor) -> torch.Tensor:
        """K_slab u on planes e0 .. e1 (partial sums on interface planes;
        fixed DoFs zero)."""

    def precondition(self, r: torch.Tensor) -> torch.Tensor:
        """The rank's Schwarz piece applied to r (planes e0 .. e1)."""


class SlabPCG:
    """Preconditioned CG over the slabs of all ranks (every rank calls
    ``solve`` with its own slab of b; all take the same steps)."""

    def __init__(self, slab: Slab, ops: SlabLocalOps, dist, device="cpu"):
        self.slab, self.ops, self.dist = slab, ops, dist
        self.w = slab.owned_mask(device=device)

    def apply_K(self, u: torch.Tensor) -> torch.Tensor:
        return interface_sum(self.ops.matvec(u), self.slab, self.dist)

    def apply_M(self, r: torch.Tensor) -> torch.Tensor:
        return interface_sum(self.ops.precondition(r), self.slab, self.dist)

    def solve(self, b: torch.Tensor, x: torch.Tensor | None = None, tol=1e-8, maxiter=500):
        """Returns (x, iterations, relative residual, converged); b and x are
        consistent slab vectors (FP64). Every rank must pass an initial x, or
        every rank none."""
        world = self.slab.world
        # the branch depends only on the call (every rank passes x or none),
        # never on this rank's data, so all ranks take the same exchanges
        if x is None:
            x = torch.zeros_like(b)
            r = b.clone()
        else:
            r = b - self.apply_K(x)
        (bb,) = all_dots([(b, b)], self.w, self.dist, world)
        bn = max(np.sqrt(bb), 1e-300)
        z = self.apply_M(r)
        p = z.clone()
        rz, rr = all_dots([(r, z), (r, r)], self.w, self.dist, world)
        if np.sqrt(rr) / bn <= tol:
            return x, 0, np.sqrt(rr) / bn, True
        for it in range(1, maxiter + 1):
            q = self.apply_K(p)
            (pq,) = all_dots([(p, q)], self.w, self.dist, world)
            alpha = rz / pq
            x.add_(p, alpha=alpha)
            r.add_(q, alpha=-alpha)
            z = self.apply_M(r)
            rz_new, rr = all_dots([(r, z), (r, r)], self.w, self.dist, world)
            if np.sqrt(rr) / bn <= tol:
                return x, it, np.sqrt(rr) / bn, True
            p.mul_(rz_new / rz).add_(z)
            rz = rz_new
        return x, maxiter, np.sqrt(rr) / bn, False


class CudaSlabOps:
    """``SlabLocalOps`` on the GPU through libtopo_b200: the slab's K u by a
    one-level context on elements [e0, e1), the Schwarz piece by a GMG
    V-cycle (FP64) of a context on the extended slab [x_lo, x_hi) whose
    outer planes are fixed. Not run on more than one GPU here (one GPU per
    test box); with one rank it is the plain solve on the whole mesh."""

    def __init__(self, slab: Slab, free_mask_global: np.ndarray, E_global: torch.Tensor, n_levels=3,
                 smoother="chebyshev"):
        from .context import TopoContext

        self.slab = slab
        dev = E_global.device
        if dev.type != "cuda":
            raise TypeError("CudaSlabOps needs the moduli on a CUDA device")
        zeros = torch.zeros(slab.ndof, dtype=torch.float64, device=dev)
        self.op = TopoContext(slab.local_nel, n_levels=1, mode="fp64", smoother=smoother)
        self.op.set_problem(torch.as_tensor(slab.local_free_mask(free_mask_global), device=dev), zeros)
        a, b = slab.element_range(slab.e0, slab.e1)
        self.E_op = E_global[a:b].contiguous()
        self.pre = TopoContext(slab.ext_nel, n_levels=n_levels, mode="fp64", smoother=smoother)
        ext_mask = slab.ext_free_mask(free_mask_global)
        self.pre.set_problem(torch.as_tensor(ext_mask, device=dev),
                             torch.zeros(len(ext_mask), dtype=torch.float64, device=dev))
        a, b = slab.element_range(slab.x_lo, slab.x_hi)
        self.pre.gmg_setup(E_global[a:b].contiguous())
        self.off = slab.ext_offset()
        self.ext = torch.zeros(len(ext_mask), dtype=torch.float64, device=dev)

    def matvec(self, u):
        return self.op.matvec(u, self.E_op)

    def precondition(self, r):
        self.ext.zero_()
        self.ext[self.off:self.off + self.slab.ndof] = r
        z = self.pre.gmg_apply(self.ext)
        return z[self.off:self.off + self.slab.ndof].clone()
