"""Problem definitions and the case gallery of the public interface.

``TopologyProblem`` and the gallery constructors keep the names and fields of
the reference (src/topogpu/problem.py:13-58, src/topogpu/gallery.py:10-94).
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Any

import numpy as np

from .problem_spec import EdgeSupport, PointLoad, ProblemSpec


@dataclass
class TopologyProblem:
    name: str
    spec: ProblemSpec
    filter_radius: float | None = None
    force_override: np.ndarray | None = None
    role: str = "user_case"
    metadata: dict[str, Any] = field(default_factory=dict)

    @property
    def nel(self) -> tuple[int, int, int]:
        return (self.spec.nelx, self.spec.nely, self.spec.nelz)

    @property
    def volfrac(self) -> float:
        return float(self.spec.volfrac)

    @property
    def is_3d(self) -> bool:
        return self.spec.is_3d

    def validate(self) -> None:
        errors = self.spec.validate()
        if errors:
            raise ValueError(f"Invalid TopoGPU problem {self.name!r}: {'; '.join(errors)}")

    def to_dict(self) -> dict[str, Any]:
        d = self.spec.to_dict()
        d.update({"name": self.name, "filter_radius": self.filter_radius, "role": self.role,
                  "metadata": dict(self.metadata), "has_force_override": self.force_override is not None})
        return d


def cantilever_3d(nel=(24, 12, 6), volfrac=0.30, filter_radius=1.5, support="xmin", load="tip_patch_z"):
    """Left-face-clamped 3-D cantilever with a downward (z) or sideways (y)
    unit load at the node nearest (2.0, 0.5, 0.25)."""
    if support != "xmin":
        raise ValueError("Only support='xmin' is currently implemented.")
    if load not in {"tip_patch_z", "tip_point_y"}:
        raise ValueError("Supported loads are 'tip_patch_z' and 'tip_point_y'.")
    force = {"tip_patch_z": {"fz": -1.0}, "tip_point_y": {"fy": -1.0}}[load]
    spec = ProblemSpec(Lx=2.0, Ly=1.0, Lz=0.5, nelx=nel[0], nely=nel[1], nelz=nel[2], volfrac=volfrac,
                       supports=[EdgeSupport(edge="left", constraint="fixed")],
                       loads=[PointLoad(x=2.0, y=0.5, z=0.25, **force)], rmin=filter_radius)
    return TopologyProblem(name="cantilever_3d", spec=spec, filter_radius=filter_radius, role="example",
                           metadata={"support": support, "load": load})


def side_load_cantilever(nel=(56, 36, 28), volfrac=0.24, filter_radius=2.3):
    return cantilever_3d(nel=nel, volfrac=volfrac, filter_radius=filter_radius, load="tip_point_y")


def benchmark_cantilever(nel, volfrac=0.30, filter_radius=None, name="benchmark_cantilever"):
    """Cantilever of the benchmark configurations: x=0 face clamped, total unit
    load in -z spread evenly over the nodes of the x=nelx, z=0 edge (passed as
    ``force_override``)."""
    from .bc import cantilever_edge_load

    nx, ny, nz = nel
    spec = ProblemSpec(Lx=float(nx), Ly=float(ny), Lz=float(nz), nelx=nx, nely=ny, nelz=nz, volfrac=volfrac,
                       supports=[EdgeSupport(edge="left", constraint="fixed")],
                       loads=[PointLoad(x=float(nx), y=0.0, z=0.0, fz=-1.0)], rmin=filter_radius)
    _, F = cantilever_edge_load(nel)
    return TopologyProblem(name=name, spec=spec, filter_radius=filter_radius, force_override=F, role="benchmark",
                           metadata={"load": "x_max_z0_edge_unit_total"})


def tool_case(name: str, dims: str | None = None):
    raise NotImplementedError(
        "tool_case builds problems with the reference's experiment drivers, which are outside this package; "
        "construct a TopologyProblem from a ProblemSpec instead")


class CaseGallery:
    cantilever_3d = staticmethod(cantilever_3d)
    side_load_cantilever = staticmethod(side_load_cantilever)
    benchmark_cantilever = staticmethod(benchmark_cantilever)
    tool_case = staticmethod(tool_case)
