"""run_simp checkpoint format: ``<path>.npz`` (arrays) + ``<path>.json`` (scalars).

Same files, keys and types as the reference's ``_save_checkpoint`` /
``_load_checkpoint`` (src/gpu_fem/pub_simp_solver.py:397-410) and its call
sites (495-514, 597-603): arrays rho, best_rho, compliance_hist; scalars
best_compliance (JSON ``Infinity`` before a valid best exists),
best_iteration, best_is_valid (0/1), best_grayness, penal, rmin, move, beta,
iteration. The file name is ``ckpt_<nelx>x<nely>x<nelz>_<problem>`` inside
the checkpoint directory. A checkpoint written here resumes in the reference
and the other way round.

The arrays are written to ``<path>.tmp.npz`` and renamed into place, as the
reference does; the JSON file is written the same way here (the reference
writes it in place), so a crash never leaves a torn scalar file.
"""

from __future__ import annotations

import json
import os
from typing import Any

import numpy as np

ARRAY_KEYS = ("rho", "best_rho", "compliance_hist")
SCALAR_KEYS = ("best_compliance", "best_iteration", "best_is_valid", "best_grayness", "penal", "rmin", "move",
               "beta", "iteration")


def checkpoint_path(directory: str, nel, problem: str = "cantilever") -> str:
    """``<dir>/ckpt_<tag>`` without extension (pub_simp_solver.py:495-498)."""
    nelx, nely, nelz = (int(v) for v in nel)
    tag = f"{nelx}x{nely}" + (f"x{nelz}" if nelz > 0 else "") + f"_{problem}"
    return os.path.join(directory, f"ckpt_{tag}")


def save_checkpoint(path: str, state: dict[str, Any]) -> None:
    arrays = {k: np.asarray(v) for k, v in state.items() if isinstance(v, np.ndarray)}
    scalars = {k: (v.tolist() if isinstance(v, np.ndarray) else v) for k, v in state.items()
               if not isinstance(v, np.ndarray)}
    np.savez_compressed(path + ".tmp", **arrays)
    os.replace(path + ".tmp.npz", path + ".npz")
    with open(path + ".json.tmp", "w") as f:
        json.dump(scalars, f)
    os.replace(path + ".json.tmp", path + ".json")


def load_checkpoint(path: str) -> dict[str, Any] | None:
    """The merged arrays and scalars, or None when either file is missing."""
    if not (os.path.exists(path + ".npz") and os.path.exists(path + ".json")):
        return None
    with np.load(path + ".npz") as z:
        data: dict[str, Any] = {k: z[k] for k in z.files}
    with open(path + ".json") as f:
        data.update(json.load(f))
    return data


def grayness(rho: np.ndarray) -> float:
    """4 mean(rho (1 - rho)) (pub_simp_solver.py:255)."""
    rho = np.asarray(rho, dtype=np.float64)
    return float(4.0 * np.mean(rho * (1.0 - rho)))
