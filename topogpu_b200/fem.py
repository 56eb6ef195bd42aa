"""Host-side constants of the hex8 discretisation.

``KE_UNIT`` is the 24x24 stiffness of a unit cube with E=1, nu=0.3 under 2x2x2
Gauss quadrature and the corner order (0,0,0) (1,0,0) (1,1,0) (0,1,0) (0,0,1)
(1,0,1) (1,1,1) (0,1,1); it matches KE_UNIT_3D of the reference
(src/gpu_fem/pub_simp_solver.py:157-186) and is uploaded once to the
device's constant memory by each context.
"""

from __future__ import annotations

import numpy as np

_CORNER_BITS = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                         [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]])


def unit_hex_stiffness(nu: float = 0.3, E: float = 1.0) -> np.ndarray:
    s = (2.0 * _CORNER_BITS - 1.0)                     # corner signs, shape (8,3)
    lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    mu = E / (2.0 * (1.0 + nu))
    D = np.full((3, 3), lam) + 2.0 * mu * np.eye(3)
    D = np.block([[D, np.zeros((3, 3))], [np.zeros((3, 3)), mu * np.eye(3)]])
    g = s / np.sqrt(3.0)                               # Gauss points
    KE = np.zeros((24, 24))
    for p in g:
        # d/d(xi_k) of N_a = prod_j (1 + s_aj p_j)/2 ; the cube [-1,1]^3 maps to itself (J = I)
        f = 0.5 * (1.0 + s * p[None, :])                # (8,3) factors
        grad = np.empty((8, 3))
        for k in range(3):
            others = [j for j in range(3) if j != k]
            grad[:, k] = 0.5 * s[:, k] * f[:, others[0]] * f[:, others[1]]
        B = np.zeros((6, 24))
        B[0, 0::3], B[1, 1::3], B[2, 2::3] = grad[:, 0], grad[:, 1], grad[:, 2]
        B[3, 0::3], B[3, 1::3] = grad[:, 1], grad[:, 0]
        B[4, 1::3], B[4, 2::3] = grad[:, 2], grad[:, 1]
        B[5, 0::3], B[5, 2::3] = grad[:, 2], grad[:, 0]
        KE += B.T @ D @ B
    return KE


KE_UNIT = unit_hex_stiffness()


def n_dof(nel) -> int:
    nx, ny, nz = nel
    return 3 * (nx + 1) * (ny + 1) * (nz + 1)
