"""bench.py's host-side helpers (no GPU): the committed DRAM-traffic figures
are reported only while the sources of their kernel are unchanged, and the
CPU baseline's sample is carried to the 160x80x80 mesh linearly."""

import hashlib
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402


def _fake_tree(tmp_path, src_text, recorded_from=None):
    (tmp_path / "profiles").mkdir()
    (tmp_path / "k.cu").write_text(src_text)
    h = hashlib.sha256((recorded_from if recorded_from is not None else src_text).encode()).hexdigest()
    d = {"kernel": "k", "bytes_per_launch": 1234, "sources": ["k.cu"], "src_sha256": h}
    (tmp_path / "profiles" / "k_traffic.json").write_text(json.dumps(d))


def test_traffic_reported_while_sources_match(tmp_path, monkeypatch):
    _fake_tree(tmp_path, "__global__ void k() {}\n")
    monkeypatch.setattr(bench, "ROOT", tmp_path)
    assert bench.traffic_for("k") == 1234


def test_traffic_dropped_when_a_source_changed(tmp_path, monkeypatch):
    _fake_tree(tmp_path, "__global__ void k() { /* edited */ }\n", recorded_from="__global__ void k() {}\n")
    monkeypatch.setattr(bench, "ROOT", tmp_path)
    assert bench.traffic_for("k") is None


def test_traffic_absent_or_source_missing(tmp_path, monkeypatch):
    monkeypatch.setattr(bench, "ROOT", tmp_path)
    assert bench.traffic_for("nothing") is None
    _fake_tree(tmp_path, "x")
    (tmp_path / "k.cu").unlink()
    assert bench.traffic_for("k") is None


def test_committed_traffic_files_name_existing_sources():
    for f in (ROOT / "profiles").glob("*_traffic.json"):
        d = json.loads(f.read_text())
        assert d["sources"] and all((ROOT / p).exists() for p in d["sources"]), f.name
        assert d["bytes_per_launch"] == d["dram_read"] + d["dram_write"], f.name


def test_cpu_sample_scales_linearly_in_elements():
    n_full, n_sample = np.prod(bench.NEL), np.prod(bench.REF_SAMPLE)
    assert bench.scale_to_full(2.0) == 2.0 * n_full / n_sample
    # the sample is the same cantilever shape (2:1:1), only smaller
    assert n_sample < n_full
    assert np.allclose(np.array(bench.REF_SAMPLE) / bench.REF_SAMPLE[1], np.array(bench.NEL) / bench.NEL[1])
