"""Oracle: hex8 element, DoF numbering, boundary conditions and matrix-free K.u.

Test infrastructure only (see ``oracle/__init__.py``).

Numbering (reference ``src/gpu_fem/pub_simp_solver.py:196-207``):
node (ix, iy, iz) -> ix*(ny+1)*(nz+1) + iy*(nz+1) + iz, DoF = 3*node + comp,
element (ex, ey, ez) -> ex*ny*nz + ey*nz + ez.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

# Corner order of the reference hex8 (pub_simp_solver.py:159-161): bit pattern
# (x, y, z) = (0,0,0) (1,0,0) (1,1,0) (0,1,0) (0,0,1) (1,0,1) (1,1,1) (0,1,1).
CORNERS = np.array(
    [[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]],
    dtype=np.int64,
)


def hex8_stiffness(nu: float = 0.3, E: float = 1.0) -> np.ndarray:
    """24x24 unit-cube hex8 stiffness with 2x2x2 Gauss quadrature.

    Follows ``_build_ke_unit_3d`` (pub_simp_solver.py:157-183): isotropic D
    from Lame constants, B from shape-function derivatives at the Gauss points
    of the reference cube [-1,1]^3 with the physical cube also [-1,1]^3
    (Jacobian = identity), KE = sum B^T D B |J|.
    """
    g = 1.0 / math.sqrt(3.0)
    sgn = (2 * CORNERS - 1).astype(np.float64)  # +-1 corner signs
    lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    mu = E / (2.0 * (1.0 + nu))
    D = np.zeros((6, 6))
    D[:3, :3] = lam
    D[0, 0] = D[1, 1] = D[2, 2] = lam + 2.0 * mu
    D[3, 3] = D[4, 4] = D[5, 5] = mu
    KE = np.zeros((24, 24))
    for gp in sgn * g:
        r, s, t = gp
        # dN_a/d(r,s,t) = 1/8 * sa*(1+s sa... ) for trilinear N_a = 1/8 (1+ra r)(1+sa s)(1+ta t)
        dN = np.empty((8, 3))
        for a in range(8):
            ra, sa, ta = sgn[a]
            dN[a, 0] = 0.125 * ra * (1 + sa * s) * (1 + ta * t)
            dN[a, 1] = 0.125 * sa * (1 + ra * r) * (1 + ta * t)
            dN[a, 2] = 0.125 * ta * (1 + ra * r) * (1 + sa * s)
        J = dN.T @ sgn
        dxyz = dN @ np.linalg.inv(J).T
        B = np.zeros((6, 24))
        for a in range(8):
            dx, dy, dz = dxyz[a]
            B[0, 3 * a] = dx
            B[1, 3 * a + 1] = dy
            B[2, 3 * a + 2] = dz
            B[3, 3 * a] = dy
            B[3, 3 * a + 1] = dx
            B[4, 3 * a + 1] = dz
            B[4, 3 * a + 2] = dy
            B[5, 3 * a] = dz
            B[5, 3 * a + 2] = dx
        KE += B.T @ D @ B * abs(np.linalg.det(J))
    return KE


KE_UNIT = hex8_stiffness()


def n_dof(nel) -> int:
    nx, ny, nz = nel
    return 3 * (nx + 1) * (ny + 1) * (nz + 1)


def edof_table(nel) -> np.ndarray:
    """Element -> 24 DoFs, int32 (pub_simp_solver.py:196-207)."""
    nx, ny, nz = nel
    ex, ey, ez = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    ex, ey, ez = ex.ravel(), ey.ravel(), ez.ravel()
    nyz = (ny + 1) * (nz + 1)
    nodes = np.stack(
        [(ex + c[0]) * nyz + (ey + c[1]) * (nz + 1) + (ez + c[2]) for c in CORNERS], axis=1
    )
    return (3 * nodes[:, :, None] + np.arange(3)[None, None, :]).reshape(-1, 24).astype(np.int32)


# ---------------------------------------------------------------------------
# Boundary conditions (restates bc_generator.py:381-447 for the cases used here)
# ---------------------------------------------------------------------------

@dataclass
class BC:
    fixed: np.ndarray  # int64 sorted
    free: np.ndarray   # int64 sorted
    F: np.ndarray      # float64 [ndof]
    ndof: int


def node_coords(nel, L) -> np.ndarray:
    """bc_generator.py:_node_coords_3d (55-63)."""
    nx, ny, nz = nel
    ix, iy, iz = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    return np.column_stack([ix.ravel() * (L[0] / nx), iy.ravel() * (L[1] / ny), iz.ravel() * (L[2] / nz)])


def face_nodes(face: str, nel) -> np.ndarray:
    """bc_generator.py:_face_nodes_3d (136-166): loop order is outer-first-axis."""
    nx, ny, nz = nel
    I, J, K = np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1)
    nid = lambda i, j, k: (i * (ny + 1) + j) * (nz + 1) + k  # noqa: E731
    if face == "left":
        a, b = np.meshgrid(J, K, indexing="ij")
        return nid(0, a, b).ravel()
    if face == "right":
        a, b = np.meshgrid(J, K, indexing="ij")
        return nid(nx, a, b).ravel()
    if face == "bottom":
        a, b = np.meshgrid(I, K, indexing="ij")
        return nid(a, 0, b).ravel()
    if face == "top":
        a, b = np.meshgrid(I, K, indexing="ij")
        return nid(a, ny, b).ravel()
    if face == "front":
        a, b = np.meshgrid(I, J, indexing="ij")
        return nid(a, b, 0).ravel()
    if face == "back":
        a, b = np.meshgrid(I, J, indexing="ij")
        return nid(a, b, nz).ravel()
    raise ValueError(face)


def nearest_node(coords: np.ndarray, p) -> int:
    """bc_generator.py:_nearest_node (107-110): first index of the minimum."""
    return int(np.argmin(np.linalg.norm(coords - np.asarray(p, dtype=float)[None, :], axis=1)))


def cantilever_bc(nel) -> BC:
    """Config-style cantilever: x=0 face clamped, unit total -z load spread
    evenly over the nodes of the x=nelx, z=0 edge (the synthetic BC of the
    benchmark configurations)."""
    nx, ny, nz = nel
    nd = n_dof(nel)
    face = face_nodes("left", nel)
    fixed = np.unique(np.concatenate([3 * face, 3 * face + 1, 3 * face + 2])).astype(np.int64)
    free = np.setdiff1d(np.arange(nd), fixed)
    F = np.zeros(nd)
    edge = (nx * (ny + 1) + np.arange(ny + 1)) * (nz + 1)
    F[3 * edge + 2] = -1.0 / len(edge)
    F[fixed] = 0.0
    return BC(fixed, free, F, nd)


# ---------------------------------------------------------------------------
# Precision helpers
# ---------------------------------------------------------------------------

def bf16_round(x) -> np.ndarray:
    """FP32 -> BF16 (returned as FP32 values), round to nearest even.

    Same rule as the reference's KE packing (cuda_fused_matvec.py:316-330) and
    ``__float2bfloat16`` for finite inputs.
    """
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    bits = a.view(np.uint32).astype(np.uint64)
    bits = (bits + 0x7FFF + ((bits >> 16) & 1)) >> 16
    return (bits.astype(np.uint32) << 16).view(np.float32).reshape(a.shape)


# ---------------------------------------------------------------------------
# Matrix-free operator (solver_v2.py:1122-1252; cuda_fused_matvec.py:41-246)
# ---------------------------------------------------------------------------

def simp_modulus(rho, penal: float = 3.0, E0: float = 1.0, Emin: float = 1e-9) -> np.ndarray:
    """E_e = Emin + (E0-Emin) rho^p (solver_v4.py:168; defaults fem_gpu.py:183-184)."""
    return Emin + (E0 - Emin) * np.asarray(rho, dtype=np.float64) ** penal


def matvec_full(u_full, E, nel, precision: str = "fp64", KE: np.ndarray = KE_UNIT) -> np.ndarray:
    """y = sum_e E_e KE u_e scattered to all DoFs (no Dirichlet restriction).

    precision:
      fp64  - MatrixFreeKff.matvec in FP64 (solver_v2.py:1183-1223)
      fp32  - same in FP32 (u, E, KE cast; per-element GEMM in FP32)
      bf16  - BF16-input / FP32-accumulate: u and KE rounded to BF16, E FP32
              (semantics of fused_matvec_bf16, cuda_fused_matvec.py:112-246)
    """
    edof = edof_table(nel)
    nd = n_dof(nel)
    if precision == "fp64":
        ue = np.asarray(u_full, dtype=np.float64)[edof]
        fe = (ue @ KE.T) * np.asarray(E, dtype=np.float64)[:, None]
        return np.bincount(edof.ravel(), weights=fe.ravel(), minlength=nd)
    if precision == "fp32":
        ue = np.asarray(u_full, dtype=np.float32)[edof]
        fe = (ue @ KE.astype(np.float32).T) * np.asarray(E, dtype=np.float32)[:, None]
        return np.bincount(edof.ravel(), weights=fe.ravel().astype(np.float64), minlength=nd).astype(np.float32)
    if precision == "bf16":
        ue = bf16_round(u_full)[edof].astype(np.float64)
        ke = bf16_round(KE).astype(np.float64)
        fe = ((ue @ ke.T).astype(np.float32) * np.asarray(E, dtype=np.float32)[:, None]).astype(np.float64)
        return np.bincount(edof.ravel(), weights=fe.ravel(), minlength=nd).astype(np.float32)
    raise ValueError(precision)


def matvec_free(u_free, E, nel, free, precision: str = "fp64") -> np.ndarray:
    """K_ff . u_free on compact free vectors (solver_v2.py:1183-1223)."""
    nd = n_dof(nel)
    dt = np.float64 if precision == "fp64" else np.float32
    u_full = np.zeros(nd, dtype=dt)
    u_full[free] = u_free
    return matvec_full(u_full, E, nel, precision)[free]


def diagonal_full(E, nel, KE: np.ndarray = KE_UNIT) -> np.ndarray:
    """diag(K) on all DoFs (solver_v2.py:1229-1252)."""
    edof = edof_table(nel)
    w = np.asarray(E, dtype=np.float64)[:, None] * np.diag(KE)[None, :]
    return np.bincount(edof.ravel(), weights=w.ravel(), minlength=n_dof(nel))


def element_energy(u_full, nel, KE: np.ndarray = KE_UNIT) -> np.ndarray:
    """ce_e = u_e^T KE u_e (solver_v4.py:246-250)."""
    ue = np.asarray(u_full, dtype=np.float64)[edof_table(nel)]
    return np.einsum("ei,ei->e", ue @ KE, ue)


def sensitivity(u_full, rho, nel, penal: float = 3.0, E0: float = 1.0, Emin: float = 1e-9) -> np.ndarray:
    """dc = -p (E0-Emin) rho^(p-1) ce (solver_v4.py:251)."""
    return -penal * (E0 - Emin) * np.asarray(rho, dtype=np.float64) ** (penal - 1) * element_energy(u_full, nel)


def assemble_K(E, nel, KE: np.ndarray = KE_UNIT):
    """Assembled CSR stiffness (used only for direct-solve ground truth)."""
    import scipy.sparse as sp

    edof = edof_table(nel).astype(np.int64)
    rows = np.repeat(edof, 24, axis=1).ravel()
    cols = np.tile(edof, (1, 24)).ravel()
    vals = (np.asarray(E, dtype=np.float64)[:, None] * KE.ravel()[None, :]).ravel()
    nd = n_dof(nel)
    return sp.csr_matrix((vals, (rows, cols)), shape=(nd, nd))


def direct_solve(E, nel, bc: BC) -> np.ndarray:
    """SciPy sparse direct solve of K_ff u = F_f; returns the full u."""
    from scipy.sparse.linalg import spsolve

    K = assemble_K(E, nel).tocsc()
    u = np.zeros(bc.ndof)
    u[bc.free] = spsolve(K[bc.free][:, bc.free], bc.F[bc.free])
    return u
