"""Problem schema of the public API (host side, once per run).

Same names, fields, defaults and validation messages as the reference's
``ProblemSpec`` family (src/gpu_fem/problem_spec.py:31-313), so a TopoGPU
problem definition runs unchanged here. Coordinates: x in [0,Lx], y in
[0,Ly], z in [0,Lz]; a 3-D problem has Lz > 0 and nelz > 0.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Optional

_DOF_MASK_3D = {
    "fixed": [0, 1, 2], "pin_x": [0], "pin_y": [1], "pin_z": [2],
    "roller_x": [1, 2], "roller_y": [0, 2], "roller_z": [0, 1],
}
_DOF_MASK_2D = {
    "fixed": [0, 1], "pin_x": [0], "pin_y": [1], "pin_z": [],
    "roller_x": [1], "roller_y": [0], "roller_z": [0, 1],
}


def _dof_mask(constraint: str, ndim: int) -> list[int]:
    table = _DOF_MASK_3D if ndim == 3 else _DOF_MASK_2D
    return list(table.get(constraint, range(ndim)))


@dataclass
class PointSupport:
    """Constrain the node nearest to (x, y, z)."""
    x: float
    y: float
    z: float = 0.0
    constraint: str = "fixed"

    def dof_mask(self, ndim: int) -> list[int]:
        return _dof_mask(self.constraint, ndim)


@dataclass
class EdgeSupport:
    """Constrain every node of a named face (left/right/bottom/top/front/back)."""
    edge: str
    constraint: str = "fixed"

    def dof_mask(self, ndim: int) -> list[int]:
        return _dof_mask(self.constraint, ndim)


@dataclass
class PointLoad:
    """Force applied at the node nearest to (x, y, z)."""
    x: float
    y: float
    z: float = 0.0
    fx: float = 0.0
    fy: float = 0.0
    fz: float = 0.0

    @property
    def magnitude(self) -> float:
        return math.sqrt(self.fx ** 2 + self.fy ** 2 + self.fz ** 2)


@dataclass
class DistributedLoad:
    """Uniform normal pressure on a named face (trapezoidal tributary areas)."""
    edge: str
    magnitude: float = -1.0


@dataclass
class CircularRegion:
    cx: float
    cy: float
    radius: float
    kind: str = "void"


@dataclass
class RectangularRegion:
    x0: float
    y0: float
    x1: float
    y1: float
    kind: str = "void"


@dataclass
class ProblemSpec:
    Lx: float = 2.0
    Ly: float = 1.0
    Lz: float = 0.0
    nelx: int = 60
    nely: int = 30
    nelz: int = 0
    E: float = 1.0
    nu: float = 0.3
    volfrac: float = 0.5
    supports: list = field(default_factory=list)
    loads: list = field(default_factory=list)
    passive_regions: list = field(default_factory=list)
    max_iter: Optional[int] = None
    rmin: Optional[float] = None

    @property
    def is_3d(self) -> bool:
        return self.Lz > 0 and self.nelz > 0

    @property
    def ndim(self) -> int:
        return 3 if self.is_3d else 2

    def validate(self) -> list[str]:
        """Physical-plausibility checks; an empty list means valid."""
        errs: list[str] = []
        if self.Lx <= 0 or self.Ly <= 0:
            errs.append("Domain dimensions Lx, Ly must be positive.")
        if self.Lz < 0:
            errs.append("Lz must be >= 0 (0 for 2D).")
        if self.nelx < 2 or self.nely < 2:
            errs.append("Mesh must have at least 2 elements in x and y.")
        if self.Lz > 0 and self.nelz < 2:
            errs.append("3D domain requires nelz >= 2.")
        if self.E <= 0:
            errs.append("Young's modulus E must be positive.")
        if not (-1.0 < self.nu < 0.5):
            errs.append("Poisson's ratio must be in (-1, 0.5).")
        if not (0.01 <= self.volfrac <= 0.99):
            errs.append("Volume fraction must be in [0.01, 0.99].")
        if not self.supports:
            errs.append("At least one support (fixed DOF) is required.")
        if not self.loads:
            errs.append("At least one load is required.")
        for i, ld in enumerate(self.loads):
            if isinstance(ld, PointLoad) and ld.magnitude < 1e-30:
                errs.append(f"Load[{i}] has zero magnitude.")
        h = max(self.Lx / max(self.nelx, 1), self.Ly / max(self.nely, 1))
        for ld in self.loads:
            if not isinstance(ld, PointLoad):
                continue
            for sup in self.supports:
                if isinstance(sup, PointSupport) and sup.constraint == "fixed":
                    d = math.sqrt((ld.x - sup.x) ** 2 + (ld.y - sup.y) ** 2 + (ld.z - sup.z) ** 2)
                    if d < 0.5 * h:
                        errs.append(f"Point load at ({ld.x},{ld.y}) coincides with "
                                    f"a fixed support — load will be zeroed out.")
        for i, pr in enumerate(self.passive_regions):
            if isinstance(pr, CircularRegion) and pr.radius <= 0:
                errs.append(f"Passive region [{i}] radius must be > 0.")
            elif isinstance(pr, RectangularRegion) and (pr.x0 >= pr.x1 or pr.y0 >= pr.y1):
                errs.append(f"Passive region [{i}] has inverted bounds.")
        return errs

    def to_dict(self) -> dict:
        d = {"Lx": self.Lx, "Ly": self.Ly, "Lz": self.Lz, "nelx": self.nelx, "nely": self.nely,
             "nelz": self.nelz, "E": self.E, "nu": self.nu, "volfrac": self.volfrac,
             "max_iter": self.max_iter, "rmin": self.rmin, "supports": [], "loads": [], "passive_regions": []}
        for s in self.supports:
            if isinstance(s, EdgeSupport):
                d["supports"].append({"type": "edge", "edge": s.edge, "constraint": s.constraint})
            else:
                d["supports"].append({"type": "point", "x": s.x, "y": s.y, "z": s.z, "constraint": s.constraint})
        for ld in self.loads:
            if isinstance(ld, DistributedLoad):
                d["loads"].append({"type": "distributed", "edge": ld.edge, "magnitude": ld.magnitude})
            else:
                d["loads"].append({"type": "point", "x": ld.x, "y": ld.y, "z": ld.z,
                                   "fx": ld.fx, "fy": ld.fy, "fz": ld.fz})
        for pr in self.passive_regions:
            if isinstance(pr, CircularRegion):
                d["passive_regions"].append({"type": "circle", "cx": pr.cx, "cy": pr.cy,
                                             "radius": pr.radius, "kind": pr.kind})
            else:
                d["passive_regions"].append({"type": "rect", "x0": pr.x0, "y0": pr.y0,
                                             "x1": pr.x1, "y1": pr.y1, "kind": pr.kind})
        return d

    @classmethod
    def from_dict(cls, d: dict) -> "ProblemSpec":
        sup = [EdgeSupport(s["edge"], s.get("constraint", "fixed")) if s["type"] == "edge"
               else PointSupport(s["x"], s["y"], s.get("z", 0.0), s.get("constraint", "fixed"))
               for s in d.get("supports", [])]
        lds = [DistributedLoad(l["edge"], l.get("magnitude", -1.0)) if l["type"] == "distributed"
               else PointLoad(l["x"], l["y"], l.get("z", 0.0), l.get("fx", 0.0), l.get("fy", 0.0), l.get("fz", 0.0))
               for l in d.get("loads", [])]
        prs = [CircularRegion(p["cx"], p["cy"], p["radius"], p.get("kind", "void")) if p["type"] == "circle"
               else RectangularRegion(p["x0"], p["y0"], p["x1"], p["y1"], p.get("kind", "void"))
               for p in d.get("passive_regions", [])]
        return cls(Lx=d.get("Lx", 2.0), Ly=d.get("Ly", 1.0), Lz=d.get("Lz", 0.0), nelx=d.get("nelx", 60),
                   nely=d.get("nely", 30), nelz=d.get("nelz", 0), E=d.get("E", 1.0), nu=d.get("nu", 0.3),
                   volfrac=d.get("volfrac", 0.5), supports=sup, loads=lds, passive_regions=prs,
                   max_iter=d.get("max_iter"), rmin=d.get("rmin"))
