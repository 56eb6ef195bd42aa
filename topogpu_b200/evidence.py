"""Evidence bundle writer with a SHA-256 manifest.

Same files and manifest columns as the reference's ``EvidenceBundle``
(src/topogpu/evidence.py:23-90): history.csv (sorted union of row keys),
rho_final.npy, render_metadata.json, summary.json, ARTIFACT_MANIFEST.csv.
"""

from __future__ import annotations

import csv
import hashlib
import json
from dataclasses import dataclass, field
from pathlib import Path
from typing import Any

import numpy as np


def sha256_file(path: Path) -> str:
    h = hashlib.sha256()
    with path.open("rb") as f:
        for chunk in iter(lambda: f.read(1 << 20), b""):
            h.update(chunk)
    return h.hexdigest()


@dataclass
class EvidenceBundle:
    root: Path
    rows: list = field(default_factory=list)

    def __post_init__(self):
        self.root = Path(self.root)

    def _prep(self, name: str) -> Path:
        self.root.mkdir(parents=True, exist_ok=True)
        return self.root / name

    def write_summary(self, summary: dict[str, Any]) -> Path:
        p = self._prep("summary.json")
        p.write_text(json.dumps(summary, indent=2), encoding="utf-8")
        self.add(p, role="summary")
        return p

    def write_history(self, rows: list[dict[str, Any]]) -> Path:
        p = self._prep("history.csv")
        keys = sorted({k for r in rows for k in r})
        with p.open("w", newline="", encoding="utf-8") as f:
            w = csv.DictWriter(f, fieldnames=keys)
            w.writeheader()
            w.writerows(rows)
        self.add(p, role="history")
        return p

    def write_density(self, rho: np.ndarray) -> Path:
        p = self._prep("rho_final.npy")
        np.save(p, rho)
        self.add(p, role="density")
        return p

    def write_array(self, name: str, values: np.ndarray, role: str) -> Path:
        if not name.endswith(".npy"):
            raise ValueError("Evidence arrays must use a .npy filename.")
        p = self._prep(name)
        np.save(p, values)
        self.add(p, role=role)
        return p

    def write_render_metadata(self, metadata: dict[str, Any]) -> Path:
        p = self._prep("render_metadata.json")
        p.write_text(json.dumps(metadata, indent=2), encoding="utf-8")
        self.add(p, role="render_metadata")
        return p

    def add(self, path: Path, role: str) -> None:
        r = Path(path).resolve()
        self.rows.append({"path": str(r.relative_to(self.root.resolve())), "role": role,
                          "bytes": r.stat().st_size, "sha256": sha256_file(r)})

    def write_manifest(self) -> Path:
        p = self._prep("ARTIFACT_MANIFEST.csv")
        with p.open("w", newline="", encoding="utf-8") as f:
            w = csv.DictWriter(f, fieldnames=["path", "role", "bytes", "sha256"])
            w.writeheader()
            w.writerows(self.rows)
        return p
