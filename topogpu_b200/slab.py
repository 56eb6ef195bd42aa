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

The pieces may overlap by more planes (``Slab.overlap``: the residual's
overlap planes are fetched from the neighbours before the local solve and
the overlap results sent back and summed after it), and a replicated coarse
level (``SlabCoarse``: the Galerkin operator of a coarser grid of the whole
mesh, summed from every rank's elements and factored on every rank) makes
it a two-level method, in additive or balanced form, so the iteration count
stays nearly flat as the slab count grows.

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
    """Rank ``rank``'s share of an (nelx, nely, nelz) mesh. ``overlap`` is the
    number of node planes the rank's Schwarz piece reaches past its own
    planes on each side (0: neighbouring pieces share only the interface
    plane)."""

    nel: tuple[int, int, int]
    rank: int
    world: int
    e0: int
    e1: int
    overlap: int = 0

    @staticmethod
    def of(nel, rank: int, world: int, overlap: int = 0) -> "Slab":
        nel = tuple(int(v) for v in nel)
        parts = partition(nel[0], world)
        if overlap < 0 or (world > 1 and overlap >= min(b - a for a, b in parts)):
            raise ValueError("overlap must be >= 0 and smaller than every slab")
        e0, e1 = parts[rank]
        return Slab(nel, rank, world, e0, e1, int(overlap))

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

    # free planes of the Schwarz piece: [p_lo, p_hi]
    @property
    def p_lo(self) -> int:
        return max(self.e0 - self.overlap, 0)

    @property
    def p_hi(self) -> int:
        return min(self.e1 + self.overlap, self.nel[0])

    # extended slab of the preconditioner: elements [x_lo, x_hi), the planes
    # just outside [p_lo, p_hi] held fixed
    @property
    def x_lo(self) -> int:
        return self.p_lo - 1 if self.p_lo > 0 else 0

    @property
    def x_hi(self) -> int:
        return self.p_hi + 1 if self.p_hi < self.nel[0] else self.nel[0]

    @property
    def local_nel(self) -> tuple[int, int, int]:
        return (self.e1 - self.e0, self.nel[1], self.nel[2])

    @property
    def ext_nel(self) -> tuple[int, int, int]:
        return (self.x_hi - self.x_lo, self.nel[1], self.nel[2])

    @property
    def piece_ndof(self) -> int:
        """DoFs of the piece's free planes p_lo .. p_hi."""
        return (self.p_hi - self.p_lo + 1) * self.plane_dofs

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
        outside p_lo .. p_hi fixed (the Dirichlet ring of the Schwarz piece)."""
        a, b = self.ext_dof_range()
        m = np.array(free_mask_global[a:b], dtype=np.uint8, copy=True)
        pd = self.plane_dofs
        if self.p_lo > 0:
            m[:pd] = 0
        if self.p_hi < self.nel[0]:
            m[-pd:] = 0
        return m

    def ext_offset(self) -> int:
        """Offset of plane p_lo inside an extended-slab vector."""
        return (self.p_lo - self.x_lo) * self.plane_dofs


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


def _exchange(slab: Slab, dist, send_left, send_right, n_left: int, n_right: int, like: torch.Tensor):
    """Send tensors to the left/right neighbours and receive n_left/n_right
    values from them (None where there is no neighbour)."""
    ops, recv = [], {}
    if slab.has_left:
        recv["l"] = torch.empty(n_left, dtype=like.dtype, device=like.device)
        ops += [dist.P2POp(dist.isend, send_left.contiguous(), slab.rank - 1),
                dist.P2POp(dist.irecv, recv["l"], slab.rank - 1)]
    if slab.has_right:
        recv["r"] = torch.empty(n_right, dtype=like.dtype, device=like.device)
        ops += [dist.P2POp(dist.isend, send_right.contiguous(), slab.rank + 1),
                dist.P2POp(dist.irecv, recv["r"], slab.rank + 1)]
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()
    return recv.get("l"), recv.get("r")


def halo_gather(r: torch.Tensor, slab: Slab, dist) -> torch.Tensor:
    """Consistent r on planes e0 .. e1 -> r on the piece's planes p_lo .. p_hi
    (the overlap planes come from the neighbours, who store them)."""
    ov = slab.overlap
    if ov == 0 or slab.world == 1:
        return r
    pd = slab.plane_dofs
    nl = (slab.e0 - slab.p_lo) * pd
    nr = (slab.p_hi - slab.e1) * pd
    # the left neighbour needs my planes e0+1 .. e0+ov, the right one e1-ov .. e1-1
    got_l, got_r = _exchange(slab, dist, r[pd:(1 + ov) * pd], r[-(1 + ov) * pd:-pd], nl, nr, r)
    parts = ([got_l] if got_l is not None else []) + [r] + ([got_r] if got_r is not None else [])
    return torch.cat(parts)


def halo_scatter_add(z: torch.Tensor, slab: Slab, dist) -> torch.Tensor:
    """A piece's result on planes p_lo .. p_hi -> consistent z on planes
    e0 .. e1: every plane gets the sum of all pieces covering it (with no
    overlap this is the interface sum)."""
    if slab.world == 1:
        return z
    pd, ov = slab.plane_dofs, slab.overlap
    nl = (slab.e0 - slab.p_lo) * pd
    own = z[nl:nl + slab.ndof].clone()
    # to the left neighbour my planes p_lo .. e0 (its e1' - ov .. e1'), to the
    # right one e1 .. p_hi
    got_l, got_r = _exchange(slab, dist, z[:nl + pd], z[nl + slab.ndof - pd:], (ov + 1) * pd, (ov + 1) * pd, z)
    if got_l is not None:
        own[:(ov + 1) * pd] += got_l
    if got_r is not None:
        own[-(ov + 1) * pd:] += got_r
    return own


def all_dots(pairs, w: torch.Tensor, dist, world: int) -> list[float]:
    """Global dot products of several (a, b) pairs in one all-reduce."""
    v = torch.stack([torch.dot(a * w, b) for a, b in pairs])
    if world > 1:
        dist.all_reduce(v)
    return [float(x) for x in v.cpu()]


def _weights_1d(nf: int, nc: int):
    """Row-normalised 1-D trilinear parent weights of fine nodes 0..nf on a
    grid of nc coarse elements: even i -> parent i/2 (1); odd i -> parents
    i>>1 and (i>>1)+1 (1/2 each), renormalised when the second lies past nc
    (the transfer rule of src/gpu_fem/solver_v2.py:62-149)."""
    out = []
    for i in range(nf + 1):
        cand = [(i >> 1, 1.0)] if (i & 1) == 0 else [(i >> 1, 0.5), ((i >> 1) + 1, 0.5)]
        cand = [(c, w) for c, w in cand if c <= nc]
        t = sum(w for _, w in cand)
        out.append([(c, w / t) for c, w in cand])
    return out


def coarse_prolongation(nel, free_mask: np.ndarray, levels: int):
    """P0 of the slab coarse space: `levels` factor-2 trilinear prolongations
    chained (all fine DoFs x free coarse DoFs, scipy CSR). Rows of fixed fine
    DoFs are zero; the coarse free set of every level follows the multigrid
    hierarchy's injection rule (coarse node (I,J,K) is free in component d
    iff fine node (2I,2J,2K) is; src/gpu_fem/solver_v2.py:717-764)."""
    import scipy.sparse as sp

    dims = [tuple(int(v) for v in nel)]
    for _ in range(levels):
        dims.append(tuple(max(1, d // 2) for d in dims[-1]))
    mask = np.asarray(free_mask, dtype=bool)
    P0 = sp.diags(mask.astype(np.float64), format="csr")
    cols = np.arange(len(mask))  # the columns of P0, as DoFs of the current level
    for fine, coarse in zip(dims[:-1], dims[1:]):
        w = [_weights_1d(f, c) for f, c in zip(fine, coarse)]
        nyf, nzf = fine[1] + 1, fine[2] + 1
        nyc, nzc = coarse[1] + 1, coarse[2] + 1
        ri, cj, vals = [], [], []
        for i, px in enumerate(w[0]):
            for j, py in enumerate(w[1]):
                for k, pz in enumerate(w[2]):
                    r = (i * nyf + j) * nzf + k
                    for a0, a in px:
                        for b0, b in py:
                            for c0, c in pz:
                                ri.append(r)
                                cj.append((a0 * nyc + b0) * nzc + c0)
                                vals.append(a * b * c)
        nf = (fine[0] + 1) * nyf * nzf
        nc = (coarse[0] + 1) * nyc * nzc
        Pv = sp.kron(sp.csr_matrix((vals, (ri, cj)), shape=(nf, nc)), sp.eye(3), format="csr")
        I, J, K = np.meshgrid(*(np.arange(c + 1) for c in coarse), indexing="ij")
        fn = ((2 * I * nyf + 2 * J) * nzf + 2 * K).ravel()
        cmask = np.zeros(3 * nc, dtype=bool)
        for d in range(3):
            fd = 3 * fn + d
            ok = fd < len(mask)
            cmask[(3 * np.arange(len(fn)) + d)[ok]] = mask[fd[ok]]
        cfree = np.flatnonzero(cmask)
        P0 = (P0 @ Pv[cols, :][:, cfree]).tocsr()
        mask, cols = cmask, cfree
    return P0.tocsr()


class SlabLocalOps(Protocol):
    def matvec(self, u: torch.Tensor) -> torch.Tensor:
        """K_slab u on planes e0 .. e1 (partial sums on interface planes;
        fixed DoFs zero)."""

    def precondition(self, r: torch.Tensor) -> torch.Tensor:
        """The rank's Schwarz piece applied to r on the piece's planes
        p_lo .. p_hi (e0 .. e1 without overlap); result on the same planes."""


class SlabCoarse:
    """Replicated coarse space of the slab preconditioner. P holds this
    rank's rows of the global prolongation P0 (the rank's node planes x free
    coarse DoFs); A0 = P0^T K P0 is the Galerkin coarse operator, the same on
    every rank, factorised once by Cholesky. The correction of a consistent
    residual r is P (A0^-1 sum_ranks P^T w r): the coarse residual sums each
    rank's owned planes (w) in one all-reduce, every rank solves the small
    system itself, and the prolongation onto the rank's planes gives both
    copies of an interface plane the same value."""

    def __init__(self, slab: Slab, P: torch.Tensor, A0: torch.Tensor, dist):
        self.slab, self.dist = slab, dist
        self.P = P
        self.L = torch.linalg.cholesky(A0)

    @staticmethod
    def galerkin(slab: Slab, P: torch.Tensor, local_matvec, dist) -> torch.Tensor:
        """A0 = sum over ranks of P^T K_slab P, K_slab u being the rank's
        element-local product (partial sums on interface planes, as
        SlabLocalOps.matvec returns): summed over ranks this is P0^T K P0.
        Costs one local product per coarse DoF."""
        cols = [local_matvec(P[:, j].contiguous()) for j in range(P.shape[1])]
        KP = torch.stack(cols, dim=1) if cols else torch.zeros_like(P)
        A0 = P.T @ KP
        if slab.world > 1:
            dist.all_reduce(A0)
        return 0.5 * (A0 + A0.T)

    def apply(self, r: torch.Tensor, w: torch.Tensor) -> torch.Tensor:
        r0 = self.P.T @ (w * r)
        if self.slab.world > 1:
            self.dist.all_reduce(r0)
        z0 = torch.cholesky_solve(r0[:, None], self.L)[:, 0]
        return self.P @ z0


class SlabPCG:
    """Preconditioned CG over the slabs of all ranks (every rank calls
    ``solve`` with its own slab of b; all take the same steps).

    Without ``coarse`` the preconditioner is one-level additive Schwarz (the
    ranks' pieces, overlapping by slab.overlap planes, summed). With it,
    ``balanced=False`` adds the coarse correction Q = P0 A0^-1 P0^T, and
    ``balanced=True`` applies the balanced two-level form
    Q + (I - Q K) M1 (I - K Q), symmetric and exact on the coarse space, at
    two more operator products per application."""

    def __init__(self, slab: Slab, ops: SlabLocalOps, dist, device="cpu", coarse: SlabCoarse | None = None,
                 balanced: bool = False):
        self.slab, self.ops, self.dist = slab, ops, dist
        self.w = slab.owned_mask(device=device)
        self.coarse = coarse
        self.balanced = balanced and coarse is not None

    def apply_K(self, u: torch.Tensor) -> torch.Tensor:
        return interface_sum(self.ops.matvec(u), self.slab, self.dist)

    def _local(self, r: torch.Tensor) -> torch.Tensor:
        return halo_scatter_add(self.ops.precondition(halo_gather(r, self.slab, self.dist)), self.slab, self.dist)

    def apply_M(self, r: torch.Tensor) -> torch.Tensor:
        if self.coarse is None:
            return self._local(r)
        if not self.balanced:
            return self._local(r) + self.coarse.apply(r, self.w)
        t = self.coarse.apply(r, self.w)
        v = self._local(r - self.apply_K(t))
        return t + v - self.coarse.apply(self.apply_K(v), self.w)

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


# ----------------------------------------------------- design update on slabs
def element_halo(x: torch.Tensor, slab: Slab, h: int, dist) -> torch.Tensor:
    """Element field of the rank's layers [e0, e1) -> layers
    [max(e0-h, 0), min(e1+h, nelx)) with the neighbours' layers (h must not
    exceed any slab's layer count)."""
    if slab.world == 1 or h == 0:
        return x
    per = slab.nel[1] * slab.nel[2]
    hl = min(h, slab.e0) * per
    hr = min(h, slab.nel[0] - slab.e1) * per
    got_l, got_r = _exchange(slab, dist, x[:h * per], x[-h * per:], hl, hr, x)
    parts = ([got_l] if got_l is not None else []) + [x] + ([got_r] if got_r is not None else [])
    return torch.cat(parts)


class SlabFilter:
    """The linear-hat density filter of run_simp (neighbours at centre
    distance <= rmin - 1e-10, weight rmin - d, the element itself weight rmin,
    rows normalised; src/gpu_fem/pub_simp_solver.py:215-243) on one rank's
    element layers. H x needs floor(rmin) halo layers of x from each
    neighbour; H^T x needs the same halo of x / Hs. The row sums Hs depend on
    the global position only, so every rank computes them itself."""

    def __init__(self, slab: Slab, rmin: float, dist, device="cpu"):
        import math

        self.slab, self.dist, self.rmin = slab, dist, float(rmin)
        self.h = R = int(math.floor(rmin))
        if slab.world > 1 and R > min(b - a for a, b in partition(slab.nel[0], slab.world)):
            raise ValueError("filter radius larger than a slab")
        self.offsets = []
        for dx in range(-R, R + 1):
            for dy in range(-R, R + 1):
                for dz in range(-R, R + 1):
                    d = math.sqrt(float(dx * dx + dy * dy + dz * dz))
                    if dx == dy == dz == 0:
                        self.offsets.append((0, 0, 0, rmin))
                    elif d <= rmin - 1e-10:
                        self.offsets.append((dx, dy, dz, rmin - d))
        nx, ny, nz = slab.nel
        ones = torch.ones(nx, ny, nz, dtype=torch.float64, device=device)
        lo = max(slab.e0 - R, 0)
        self.Hs = self._stencil(ones[lo:min(slab.e1 + R, nx)], lo)

    def _stencil(self, xe: torch.Tensor, g_lo: int) -> torch.Tensor:
        """sum over the offsets of w * x[e + offset] for the rank's elements
        e, neighbours outside the mesh left out; xe holds the global layers
        g_lo .. (layers, ny, nz), covering every source layer."""
        R = self.h
        nx = self.slab.nel[0]
        pad = torch.nn.functional.pad(xe, (R, R, R, R))  # zero y/z padding (outside the mesh)
        e0, e1 = self.slab.e0, self.slab.e1
        out = torch.zeros(e1 - e0, xe.shape[1], xe.shape[2], dtype=xe.dtype, device=xe.device)
        ny, nz = xe.shape[1], xe.shape[2]
        for dx, dy, dz, w in self.offsets:
            a, b = e0 + dx, e1 + dx  # source layers for the owned outputs
            lo, hi = max(a, 0), min(b, nx)
            if lo >= hi:
                continue
            src = pad[lo - g_lo:hi - g_lo, R + dy:R + dy + ny, R + dz:R + dz + nz]
            out[lo - a:hi - a] += w * src
        return out

    def _ext(self, x: torch.Tensor) -> tuple[torch.Tensor, int]:
        ny, nz = self.slab.nel[1], self.slab.nel[2]
        xe = element_halo(x, self.slab, self.h, self.dist)
        return xe.view(-1, ny, nz), max(self.slab.e0 - self.h, 0)

    def apply(self, x: torch.Tensor) -> torch.Tensor:
        """(H x) on the rank's elements."""
        xe, g_lo = self._ext(x)
        return (self._stencil(xe, g_lo) / self.Hs).reshape(-1)

    def apply_transpose(self, x: torch.Tensor) -> torch.Tensor:
        """(H^T x) on the rank's elements: sum_i w_ij x_i / Hs_i (the weights
        are symmetric, and the neighbours' x / Hs arrive in the halo)."""
        xe, g_lo = self._ext((x.view_as(self.Hs) / self.Hs).reshape(-1))
        return self._stencil(xe, g_lo).reshape(-1)


def slab_oc_filtered(rho, dc, dv, colsum, volfrac, move, slab: Slab, dist, rho_min=1e-3):
    """The filtered-volume OC bisection of run_simp (pub_simp_solver.py:
    319-340: l1 = 0, l2 = 1e9, at most 100 steps, stop when l2 - l1 < 1e-9,
    volume measured on H * candidate) on the rank's elements: the volume
    sum_i (H rn)_i = sum_j rn_j colsum_j (colsum = H^T 1) is all-reduced once
    per bisection step, so every rank takes the same steps. Returns
    (candidate, number of evaluations)."""
    n = float(np.prod(slab.nel))
    dcs = torch.clamp(dc, max=-1e-12)
    dvs = torch.clamp(dv, min=1e-12)
    l1, l2 = 0.0, 1e9
    rn = rho
    k = 0
    for k in range(100):
        lm = 0.5 * (l1 + l2)
        rn = rho * torch.sqrt(-dcs / (lm * dvs))
        rn = torch.minimum(torch.maximum(rn, rho - move), rho + move)
        rn = torch.clamp(rn, min=rho_min, max=1.0)
        vol = (rn * colsum).sum().reshape(1)
        if slab.world > 1:
            dist.all_reduce(vol)
        if float(vol) / n > volfrac:
            l1 = lm
        else:
            l2 = lm
        if l2 - l1 < 1e-9:
            break
    return rn, k + 1


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
        n = self.slab.piece_ndof
        self.ext.zero_()
        self.ext[self.off:self.off + n] = r
        z = self.pre.gmg_apply(self.ext)
        return z[self.off:self.off + n].clone()
