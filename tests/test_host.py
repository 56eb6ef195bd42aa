"""Host-side logic and the C ABI library, without a GPU."""

from __future__ import annotations

import csv
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from conftest import ROOT, load_golden


def test_library_loads_and_exports_every_declared_symbol():
    from topogpu_b200 import _lib, build

    build.build()
    lib = _lib.load()
    header = (ROOT / "include" / "topo_b200.h").read_text()
    declared = set(re.findall(r"^\s*(?:int|long long)\s+(topo_\w+)\s*\(", header, flags=re.M))
    assert declared, "no declarations found in include/topo_b200.h"
    for name in declared:
        assert hasattr(lib, name), name
    assert declared <= set(_lib.SIGNATURES), declared - set(_lib.SIGNATURES)
    assert lib.topo_version() == 100


def test_library_reports_errors_without_gpu_work():
    from topogpu_b200 import _lib

    lib = _lib.load()
    h = ctypes.c_void_p()
    ke = np.zeros(576)
    rc = lib.topo_ctx_create(0, 1, 1, 1, 0, 2, 2, 1 / 30, 100, ke.ctypes.data_as(ctypes.c_void_p), ctypes.byref(h))
    assert rc < 0
    assert "grid dims" in _lib.last_error(None)


def test_entries_reject_a_null_context_without_gpu_work():
    """Every context entry validates its arguments before touching the device:
    a NULL context is an error status naming the entry (the byte-count query
    answers 0)."""
    from topogpu_b200 import _lib

    lib = _lib.load()
    no_ctx = {"topo_version", "topo_last_error", "topo_ctx_destroy", "topo_launch_count", "topo_ctx_create",
              "topo_oc_noalloc", "topo_debug_tc_wait"}
    checked = 0
    for name, (restype, argtypes) in sorted(_lib.SIGNATURES.items()):
        if name in no_ctx:
            continue
        args = [t() if t is not ctypes.c_void_p else None for t in argtypes]
        rc = getattr(lib, name)(*args)
        if name == "topo_workspace_bytes":
            assert rc == 0
            continue
        assert rc < 0, name
        assert name in _lib.last_error(None), (name, _lib.last_error(None))
        checked += 1
    assert checked >= 25


def test_product_stiffness_matches_reference():
    from topogpu_b200.fem import KE_UNIT

    np.testing.assert_allclose(KE_UNIT, load_golden("ke_edof")["KE"], rtol=0, atol=1e-14)


@pytest.mark.parametrize("tag,nel", [("4x3x2", (4, 3, 2)), ("24x12x6", (24, 12, 6)), ("7x5x3", (7, 5, 3))])
def test_generate_bc_matches_reference(tag, nel):
    import topogpu_b200 as tg
    from topogpu_b200.bc import generate_bc

    g = load_golden("bc")
    bc = generate_bc(tg.gallery.cantilever_3d(nel=nel, volfrac=0.3).spec)
    assert np.array_equal(bc.free_dofs, g[f"free_{tag}"])
    assert np.array_equal(bc.F, g[f"F_{tag}"])
    bc2 = generate_bc(tg.gallery.side_load_cantilever(nel=nel).spec)
    assert np.array_equal(bc2.free_dofs, g[f"side_free_{tag}"])
    assert np.array_equal(bc2.F, g[f"side_F_{tag}"])


def test_nearest_node_closed_form_matches_bruteforce():
    """The 8-neighbour nearest-node search picks the node the reference's
    argmin over all nodes picks, ties (cell midpoints, faces) and points
    outside the box included."""
    from topogpu_b200.bc import _nearest, _nearest_bruteforce, node_coords
    from topogpu_b200.problem_spec import ProblemSpec

    rng = np.random.default_rng(3)
    for nel, L in [((4, 3, 2), (4.0, 3.0, 2.0)), ((7, 5, 3), (1.0, 0.7, 0.3)), ((10, 4, 6), (2.5, 1.0, 1.5))]:
        spec = ProblemSpec(nelx=nel[0], nely=nel[1], nelz=nel[2], Lx=L[0], Ly=L[1], Lz=L[2])
        c = node_coords(spec)
        h = np.array(L) / np.array(nel)
        pts = list(rng.uniform(-0.3, 1.3, (200, 3)) * np.array(L))
        pts += list((rng.integers(0, 2 * np.array(nel) + 1, (200, 3)) * 0.5) * h)  # nodes, midpoints
        pts += [np.array(L), np.zeros(3), np.array(L) / 2]
        for p in pts:
            assert _nearest(spec, c, p) == _nearest_bruteforce(c, p), (nel, p)


def test_problem_validation_errors():
    import topogpu_b200 as tg

    p = tg.gallery.cantilever_3d(nel=(4, 3, 2), volfrac=0.30)
    p.validate()
    assert p.nel == (4, 3, 2) and p.volfrac == 0.30 and p.metadata["support"] == "xmin"
    p.spec.volfrac = 2.0
    with pytest.raises(ValueError, match="Volume fraction"):
        p.validate()
    with pytest.raises(ValueError):
        tg.gallery.cantilever_3d(support="ymin")


def test_spec_round_trip():
    import topogpu_b200 as tg
    from topogpu_b200.problem_spec import ProblemSpec

    spec = tg.gallery.cantilever_3d().spec
    assert ProblemSpec.from_dict(spec.to_dict()).to_dict() == spec.to_dict()


def test_density_filter_host_api():
    import topogpu_b200 as tg

    f = tg.DensityFilter((4, 3, 2), radius=1.5)
    assert np.allclose(f.apply(np.ones(24)), 1.0, atol=1e-12)
    np.testing.assert_allclose(tg.DensityFilter((4, 3, 2), 1.5).matrix(), load_golden("filter")["dense_432_r1.5"],
                               rtol=1e-15)
    w = tg.DensityFilter((3, 2, 2), radius=1.5).matrix()
    assert np.allclose(w.sum(axis=1), 1.0, atol=1e-12)
    # the energy form of the reference's tests/test_energy_consistency.py
    rho = np.linspace(0.1, 1.0, w.shape[0])
    assert float(rho @ (w @ rho)) > 0.0


def test_evidence_bundle_manifest(tmp_path):
    from topogpu_b200.evidence import EvidenceBundle

    b = EvidenceBundle(tmp_path)
    b.write_history([{"iteration": 1, "compliance": 1.0}, {"iteration": 2, "compliance": 0.5, "wall_s": 0.1}])
    b.write_summary({"status": "ok"})
    b.write_density(np.ones(3))
    b.write_render_metadata({"density_threshold": 0.5})
    m = b.write_manifest()
    rows = list(csv.DictReader(m.open()))
    assert {r["path"] for r in rows} >= {"history.csv", "summary.json", "rho_final.npy", "render_metadata.json"}
    assert all(len(r["sha256"]) == 64 for r in rows)
    head = (tmp_path / "history.csv").read_text().splitlines()[0]
    assert head == "compliance,iteration,wall_s"


def test_backend_and_optimizer_checks():
    import topogpu_b200 as tg

    assert tg.SIMPSolver(backend="cpu").backend == "cpu"  # run_simp, physics on the GPU
    with pytest.raises(ValueError, match="Unknown backend"):
        tg.SIMPSolver(backend="tpu")
    with pytest.raises(ValueError, match="optimizer"):
        tg.SIMPSolver(optimizer="mma")


def test_benchmark_problem_load():
    import topogpu_b200 as tg

    p = tg.gallery.benchmark_cantilever((24, 12, 6))
    F = p.force_override
    assert abs(F.sum() + 1.0) < 1e-14 and np.count_nonzero(F) == 13


def test_autograd_compliance_plumbing_without_gpu():
    """The autograd wrapper returns the state solver's sensitivity as the
    gradient (checked with a stand-in solver whose 'compliance' is sum rho^3)."""
    import torch

    from topogpu_b200.autograd import compliance

    class _Stand:
        def solve(self, rho, penal):
            return float((rho ** 3).sum()), 3.0 * rho ** 2

    rho = torch.linspace(0.1, 1.0, 17, dtype=torch.float64, requires_grad=True)
    c = compliance(rho, _Stand())
    (2.0 * c).backward()
    assert torch.allclose(rho.grad, 6.0 * rho.detach() ** 2)
    assert abs(float(c) - float((rho.detach() ** 3).sum())) < 1e-12


def test_checkpoint_format_matches_reference(tmp_path):
    """A run_simp checkpoint (written by the reference after iteration 2 of
    config 0) loads here with every key, and writing it back gives files the
    reference's loader reads to the same values (pub_simp_solver.py:397-410)."""
    import json
    import shutil

    from conftest import GOLDEN
    from topogpu_b200.checkpoint import ARRAY_KEYS, SCALAR_KEYS, checkpoint_path, load_checkpoint, save_checkpoint

    assert checkpoint_path(str(tmp_path), (24, 12, 6)) == str(tmp_path / "ckpt_24x12x6_cantilever")
    src = str(GOLDEN / "ckpt_24x12x6_cantilever")
    ck = load_checkpoint(src)
    assert set(ck) == set(ARRAY_KEYS) | set(SCALAR_KEYS)
    assert ck["iteration"] == 2 and ck["best_compliance"] == float("inf") and ck["best_is_valid"] == 0
    assert ck["rho"].shape == (1728,) and len(ck["compliance_hist"]) == 2
    out = str(tmp_path / "ckpt_24x12x6_cantilever")
    save_checkpoint(out, {k: ck[k] for k in ck})
    back = load_checkpoint(out)
    for k in ARRAY_KEYS:
        assert np.array_equal(back[k], ck[k]), k
    for k in SCALAR_KEYS:
        assert back[k] == ck[k], k
    with open(out + ".json") as f, open(src + ".json") as g:
        assert json.load(f) == json.load(g)
    with np.load(out + ".npz") as a, np.load(src + ".npz") as b:
        assert sorted(a.files) == sorted(b.files)
    assert not (tmp_path / "ckpt_24x12x6_cantilever.tmp.npz").exists()
    # a missing half means no checkpoint, as in the reference
    shutil.copy(src + ".npz", tmp_path / "only.npz")
    assert load_checkpoint(str(tmp_path / "only")) is None


def test_range_checked_build_compiles_and_exports_every_symbol():
    """The TOPO_DEBUG_BOUNDS variant (libtopo_b200_dbg.so) builds and exports
    the same entry points; the normal build reports that it has no checks."""
    import subprocess
    import sys

    from topogpu_b200 import _lib, build

    path = build.build(debug_bounds=True)
    assert path.name == "libtopo_b200_dbg.so"
    header = (ROOT / "include" / "topo_b200.h").read_text()
    declared = set(re.findall(r"^\s*(?:int|long long)\s+(topo_\w+)\s*\(", header, flags=re.M))
    dbg = ctypes.CDLL(str(path))
    for name in declared:
        assert hasattr(dbg, name), name
    lib = _lib.load()
    t = ctypes.c_int(7)
    assert lib.topo_debug_bounds(ctypes.byref(t)) == 1 and t.value == 0
    code = "from topogpu_b200 import _lib; print(_lib.lib_path().name)"
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env={**__import__("os").environ, "TOPO_B200_LIB": "dbg"},
                         capture_output=True, text=True, check=True)
    assert out.stdout.strip() == "libtopo_b200_dbg.so"
