"""ProblemSpec -> (fixed DoFs, free DoFs, load vector) for 3-D structured grids.

Host-side, once per run. Follows the reference's ``generate_bc``
(src/gpu_fem/bc_generator.py:381-447): face supports fix the requested
components of every face node, point supports and point loads snap to the
nearest node (first index on ties), distributed loads use trapezoidal
tributary areas, loads on fixed DoFs are zeroed, and an all-zero free load is
an error. Face node order (and hence F) matches the reference's loops.

Everything is closed form over the structured grid, so the cost is linear in
the DoF count with no Python loop over nodes: the nearest node is searched
among the (up to) 8 grid nodes around the point with the same distance
arithmetic as a search over all nodes, and the free set is the complement of
a boolean mask (at 8M elements the setup takes a fraction of a second).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .problem_spec import DistributedLoad, EdgeSupport, PointLoad, PointSupport, ProblemSpec


@dataclass
class BCResult:
    fixed_dofs: np.ndarray
    free_dofs: np.ndarray
    F: np.ndarray
    ndof: int
    node_coords: np.ndarray

    def free_mask(self) -> np.ndarray:
        m = np.zeros(self.ndof, dtype=np.uint8)
        m[self.free_dofs] = 1
        return m


def node_coords(spec: ProblemSpec) -> np.ndarray:
    nx, ny, nz = spec.nelx, spec.nely, spec.nelz
    c = np.empty((nx + 1, ny + 1, nz + 1, 3))
    c[..., 0] = (np.arange(nx + 1) * (spec.Lx / nx))[:, None, None]
    c[..., 1] = (np.arange(ny + 1) * (spec.Ly / ny))[None, :, None]
    c[..., 2] = (np.arange(nz + 1) * (spec.Lz / nz))[None, None, :]
    return c.reshape(-1, 3)


def face_nodes(face: str, nel) -> np.ndarray:
    nx, ny, nz = nel
    nid = lambda i, j, k: (i * (ny + 1) + j) * (nz + 1) + k  # noqa: E731
    r = {"x": np.arange(nx + 1), "y": np.arange(ny + 1), "z": np.arange(nz + 1)}
    if face in ("left", "right"):
        a, b = np.meshgrid(r["y"], r["z"], indexing="ij")
        return nid(0 if face == "left" else nx, a, b).ravel()
    if face in ("bottom", "top"):
        a, b = np.meshgrid(r["x"], r["z"], indexing="ij")
        return nid(a, 0 if face == "bottom" else ny, b).ravel()
    if face in ("front", "back"):
        a, b = np.meshgrid(r["x"], r["y"], indexing="ij")
        return nid(a, b, 0 if face == "front" else nz).ravel()
    raise ValueError(f"Unknown 3D face: {face}")


def _nearest_bruteforce(coords: np.ndarray, p) -> int:
    """Reference rule: argmin of the Euclidean distance over all nodes, the
    first node on ties (bc_generator.py:108-111)."""
    return int(np.argmin(np.linalg.norm(coords - np.asarray(p, dtype=float)[None, :], axis=1)))


def _nearest(spec: ProblemSpec, coords: np.ndarray, p) -> int:
    """Same node as ``_nearest_bruteforce``: the nearest grid node is one of
    the 8 nodes of the cell around p (clamped to the grid), and those are
    compared with the same distance arithmetic, in increasing node order, so
    ties resolve to the first node as argmin does."""
    n = (spec.nelx, spec.nely, spec.nelz)
    L = (spec.Lx, spec.Ly, spec.Lz)
    p = np.asarray(p, dtype=float)
    cand = []
    for ax in range(3):
        h = L[ax] / n[ax]
        f = int(np.floor(p[ax] / h)) if np.isfinite(p[ax]) else 0
        cand.append(sorted({min(max(f + d, 0), n[ax]) for d in (-1, 0, 1, 2)}))
    ny1, nz1 = n[1] + 1, n[2] + 1
    ids = np.array(sorted((i * ny1 + j) * nz1 + k for i in cand[0] for j in cand[1] for k in cand[2]))
    return int(ids[np.argmin(np.linalg.norm(coords[ids] - p[None, :], axis=1))])


def _tributary(spec: ProblemSpec, face: str, xyz: np.ndarray) -> np.ndarray:
    if len(xyz) <= 1:
        return np.ones(len(xyz))
    axes = {"left": (1, 2), "right": (1, 2), "bottom": (0, 2), "top": (0, 2), "front": (0, 1), "back": (0, 1)}[face]
    h = [spec.Lx / spec.nelx, spec.Ly / spec.nely, spec.Lz / spec.nelz]
    w = np.ones(len(xyz))
    for ax in axes:
        hh = h[ax]
        c = xyz[:, ax]
        wa = np.full(len(xyz), hh)
        wa[np.abs(c - c.min()) < 0.01 * hh] = hh / 2
        wa[np.abs(c - c.max()) < 0.01 * hh] = hh / 2
        w *= wa
    return w


def generate_bc(spec: ProblemSpec) -> BCResult:
    errors = spec.validate()
    if errors:
        raise ValueError("ProblemSpec validation failed:\n" + "\n".join(f"  - {e}" for e in errors))
    if not spec.is_3d:
        raise ValueError("the B200 SolverV4 path handles 3-D problems only")
    nel = (spec.nelx, spec.nely, spec.nelz)
    coords = node_coords(spec)
    ndof = 3 * len(coords)
    fixed_parts = []
    for sup in spec.supports:
        nodes = face_nodes(sup.edge, nel) if isinstance(sup, EdgeSupport) else np.array(
            [_nearest(spec, coords, (sup.x, sup.y, sup.z))])
        offs = np.asarray(list(sup.dof_mask(3)), dtype=np.int64)
        if offs.size:
            fixed_parts.append((3 * np.asarray(nodes, dtype=np.int64)[:, None] + offs[None, :]).ravel())
    fixed = np.unique(np.concatenate(fixed_parts)) if fixed_parts else np.zeros(0, dtype=np.int64)
    is_free = np.ones(ndof, dtype=bool)
    is_free[fixed] = False
    free = np.flatnonzero(is_free).astype(np.int64)
    F = np.zeros(ndof)
    for ld in spec.loads:
        if isinstance(ld, PointLoad):
            n = _nearest(spec, coords, (ld.x, ld.y, ld.z))
            F[3 * n] += ld.fx
            F[3 * n + 1] += ld.fy
            F[3 * n + 2] += ld.fz
        elif isinstance(ld, DistributedLoad):
            nodes = face_nodes(ld.edge, nel)
            w = _tributary(spec, ld.edge, coords[nodes])
            comp, sign = {"left": (0, -1.0), "right": (0, 1.0), "bottom": (1, -1.0), "top": (1, 1.0),
                          "front": (2, -1.0), "back": (2, 1.0)}[ld.edge]
            # face nodes are distinct, so the scatter-add has no repeated index
            F[3 * nodes + comp] += ld.magnitude * sign * w
    F[fixed] = 0.0
    if np.max(np.abs(F[free])) < 1e-30:
        raise ValueError("Force vector is zero on all free DOFs. "
                         "Check that loads are not placed on fully-fixed supports.")
    return BCResult(fixed, free, F, ndof, coords)


def cantilever_edge_load(nel, total: float = -1.0):
    """Benchmark cantilever: x=0 face clamped; a total load `total` in z split
    evenly over the nodes of the x=nelx, z=0 edge. Returns (free_mask uint8, F)."""
    nx, ny, nz = nel
    ndof = 3 * (nx + 1) * (ny + 1) * (nz + 1)
    mask = np.ones(ndof, dtype=np.uint8)
    face = face_nodes("left", nel)
    for c in range(3):
        mask[3 * face + c] = 0
    F = np.zeros(ndof)
    edge = (nx * (ny + 1) + np.arange(ny + 1)) * (nz + 1)
    F[3 * edge + 2] = total / len(edge)
    return mask, F


def face_point_loads(nel, k, seed):
    """k unit point loads at distinct random nodes of the x = nelx face, in
    random unit directions (seeded): the load cases of the multi-load
    benchmark. Returns a (k, ndof) float64 array."""
    nx, ny, nz = (int(v) for v in nel)
    rng = np.random.default_rng(seed)
    face = ((nx * (ny + 1) + np.arange(ny + 1)[:, None]) * (nz + 1) + np.arange(nz + 1)[None, :]).ravel()
    nodes = rng.choice(face, k, replace=False)
    dirs = rng.normal(size=(k, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    B = np.zeros((k, 3 * (nx + 1) * (ny + 1) * (nz + 1)))
    for j in range(k):
        B[j, 3 * nodes[j]:3 * nodes[j] + 3] = dirs[j]
    return B

