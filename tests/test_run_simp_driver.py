"""The run_simp driver (topogpu_b200.run_simp) against the reference's run_simp.

The fixture ``run_simp_control.npz`` is the reference run on its 3-D
cantilever preset with a scripted controller (tests/golden/make_golden.py
``ScriptedController``: an initial move change, beta and penal raised at
iteration 2, a restart from the best design at 4, a stop at 6, a two-step
tail at a new radius). On the CPU the driver runs with the oracle's physics
(direct solves, as the reference), so the control flow itself is checked:
the same iterations, parameter changes, best-design record, tail and
compliances to 1e-9. The GPU test runs the same script with the device
physics (FP64 GMG-PCG to 1e-11) and holds the compliances to 1e-6.
"""

from __future__ import annotations

import importlib.util
from pathlib import Path

import numpy as np
import pytest

from conftest import load_golden
from oracle import design, fem

ROOT = Path(__file__).resolve().parents[1]


def _controller():
    spec = importlib.util.spec_from_file_location("make_golden", ROOT / "tests" / "golden" / "make_golden.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.ScriptedController()


def _params():
    from topogpu_b200.run_simp import SIMPParams

    return SIMPParams(nelx=16, nely=8, nelz=4, volfrac=0.3, rmin=1.5, move=0.2, max_iter=10, min_iter=3,
                      use_heaviside=True, beta_init=1.0, max_gray_for_best=0.9)


class OracleFEA:
    """The physics of one run_simp iteration from the oracle (CPU)."""

    def __init__(self, nel, free, F):
        self.nel = tuple(nel)
        ndof = len(F)
        is_free = np.zeros(ndof, dtype=bool)
        is_free[free] = True
        self.bc = fem.BC(np.flatnonzero(~is_free), np.flatnonzero(is_free), np.asarray(F, dtype=np.float64), ndof)
        self.n = int(np.prod(nel))
        self._H = {}

    def set_volfrac(self, v):
        self.volfrac = float(v)

    def uniform(self, v):
        return np.full(self.n, float(v))

    from_host = staticmethod(lambda a: np.array(a, dtype=np.float64))
    to_host = staticmethod(lambda x: x)
    copy = staticmethod(lambda x: x.copy())
    clip = staticmethod(np.clip)

    @staticmethod
    def grayness(x):
        return float(4.0 * np.mean(x * (1.0 - x)))

    def step(self, rho, penal, rmin, move, beta, eta, use_heaviside):
        if rmin not in self._H:
            self._H[rmin] = design.filter_matrix(self.nel, rmin)
        H = self._H[rmin]
        rf = H @ rho
        project = use_heaviside and beta > 1e-6
        rp = design.heaviside(rf, beta, eta) if project else rf
        U = fem.direct_solve(1e-9 + (1 - 1e-9) * rp**penal, self.nel, self.bc)
        c = float(self.bc.F @ U)
        dcp = -penal * (1 - 1e-9) * rp ** (penal - 1) * fem.element_energy(U, self.nel)
        dh = design.heaviside_deriv(rf, beta, eta) if project else np.ones_like(rf)
        dc, dv = H.T @ (dcp * dh), H.T @ dh
        if project:
            rn, _ = design.oc_update_projected(rho, dc, dv, self.volfrac, move, H, beta, eta)
        else:
            rn, _ = design.oc_update_filtered(rho, dc, dv, self.volfrac, move, H)
        return c, rn, float(np.max(np.abs(rn - rho))), rp

    def close(self):
        pass


def _check(res, g, rtol):
    np.testing.assert_allclose(res["compliance_history"], g["compliance"], rtol=rtol)
    assert res["n_iter"] == int(g["n_iter"]) and res["best_iteration"] == int(g["best_iteration"])
    assert bool(res["best_is_valid"]) == bool(g["best_is_valid"])
    np.testing.assert_allclose(res["best_compliance"], float(g["best_compliance"]), rtol=rtol)
    log = res["params_log"]
    assert [r["iter"] for r in log] == list(g["log_iter"])
    assert [r["phase"] == "tail" for r in log] == list(g["log_tail"])
    for key, col in (("penal", "log_penal"), ("rmin", "log_rmin"), ("move", "log_move"), ("beta", "log_beta")):
        assert [r[key] for r in log] == list(g[col]), key
    np.testing.assert_allclose([r["grayness"] for r in log], g["log_gray"], rtol=100 * rtol, atol=1e-10)
    np.testing.assert_allclose([r["volume_fraction"] for r in log], g["log_vf"], rtol=100 * rtol, atol=1e-10)


def test_driver_control_flow_matches_reference_with_oracle_physics():
    from topogpu_b200.run_simp import cantilever_bc_3d, run_simp

    g = load_golden("run_simp_control")
    p = _params()
    _, free, F = cantilever_bc_3d(p.nelx, p.nely, p.nelz)
    res = run_simp(p, callback=_controller(), fea=OracleFEA((p.nelx, p.nely, p.nelz), free, F))
    _check(res, g, 1e-9)
    np.testing.assert_allclose(res["rho_final"], g["rho_final"], rtol=1e-7, atol=1e-9)
    np.testing.assert_allclose(res["final_compliance"], float(g["final_compliance"]), rtol=1e-8)


def test_driver_helpers_match_reference_rules():
    from topogpu_b200.run_simp import SIMPParams, apply_action, cantilever_bc_3d, tail_defaults

    r = np.zeros(3)
    best = np.ones(3)
    pen, rm, mv, bt, rn = apply_action({"penal": 9, "rmin": 0.5, "move": 1.0, "beta": 100, "restart": True},
                                       3.0, 1.5, 0.2, 1.0, r, best, True, np.copy)
    assert (pen, rm, mv, bt) == (5.0, 1.1, 0.4, 64.0) and np.array_equal(rn, best)
    _, _, _, _, rn = apply_action({"restart": True}, 3.0, 1.5, 0.2, 1.0, r, best, False, np.copy)
    assert rn is r  # no valid best: the candidate stays
    t = tail_defaults(None, SIMPParams(beta_max=16.0))
    assert t["enabled"] is False and t["beta"] == 16.0 and t["tail_iters"] == 18
    fixed, free, F = cantilever_bc_3d(4, 2, 2)
    assert len(fixed) == 3 * 3 * 3 and F.sum() == -1.0 and len(free) + len(fixed) == 3 * 5 * 3 * 3
    with pytest.raises(ValueError):
        from topogpu_b200.run_simp import run_simp

        run_simp(SIMPParams(nelz=0), fea=object())


@pytest.mark.gpu
def test_driver_on_device_matches_reference(cuda_dev):
    from topogpu_b200.run_simp import run_simp

    g = load_golden("run_simp_control")
    res = run_simp(_params(), callback=_controller(), krylov_tol=1e-11)
    _check(res, g, 1e-6)


class _MildController:
    def __call__(self, state, rho_new):
        if state.iteration == 2:
            return {"beta": 2.0}
        if state.iteration == 4:
            return {"move": 0.1, "penal": 3.2}
        return None


@pytest.mark.gpu
def test_driver_device_physics_matches_oracle_physics(cuda_dev):
    """The same driver and script with the device physics and with the
    oracle's: compliances to 1e-6 along a run with beta and penal changes."""
    from topogpu_b200.run_simp import SIMPParams, cantilever_bc_3d, run_simp

    p = SIMPParams(nelx=16, nely=8, nelz=4, volfrac=0.3, rmin=1.5, move=0.2, max_iter=6, min_iter=3,
                   use_heaviside=True, beta_init=1.0)
    _, free, F = cantilever_bc_3d(p.nelx, p.nely, p.nelz)
    ref = run_simp(p, callback=_MildController(), fea=OracleFEA((p.nelx, p.nely, p.nelz), free, F))
    res = run_simp(p, callback=_MildController(), krylov_tol=1e-11)
    np.testing.assert_allclose(res["compliance_history"], ref["compliance_history"], rtol=1e-6)
    assert res["n_iter"] == ref["n_iter"]
    assert [r["beta"] for r in res["params_log"]] == [r["beta"] for r in ref["params_log"]]
    np.testing.assert_allclose(res["rho_final"], ref["rho_final"], atol=1e-5)


@pytest.mark.gpu
def test_simpsolver_cpu_backend_runs_run_simp_on_device(cuda_dev):
    """SIMPSolver(backend="cpu") is the reference's run_simp path
    (src/topogpu/solver.py:156-184) with the problem's own BCs: against the
    driver with the oracle physics on the same parameters."""
    import topogpu_b200 as tg
    from topogpu_b200.bc import generate_bc
    from topogpu_b200.run_simp import SIMPParams, run_simp

    p = tg.gallery.benchmark_cantilever((16, 8, 4), volfrac=0.3, filter_radius=1.5)
    res = tg.SIMPSolver(backend="cpu", max_iter=3, move=0.2).solve(p)
    bc = generate_bc(p.spec)
    F = p.force_override if p.force_override is not None else bc.F  # the loads SIMPSolver uses
    params = SIMPParams(nelx=16, nely=8, nelz=4, volfrac=0.3, rmin=1.5, max_iter=3, min_iter=2, move=0.2, tol=1e-3)
    ref = run_simp(params, fea=OracleFEA((16, 8, 4), bc.free_dofs, F))
    np.testing.assert_allclose([r["compliance"] for r in res.history], ref["compliance_history"], rtol=1e-6)
    assert res.summary["backend"] == "cpu" and res.summary["n_iter"] == ref["n_iter"]
    np.testing.assert_allclose(res.rho_final, ref["rho_final"], atol=1e-5)


def test_driver_checkpoint_resume_matches_reference(tmp_path):
    """Interrupted after 4 of 7 iterations (checkpoint_every 2) and resumed,
    as the reference run_simp did for ``run_simp_resume.npz``: both legs with
    the oracle physics, and the second leg really starts from the checkpoint."""
    from topogpu_b200.run_simp import SIMPParams, cantilever_bc_3d, run_simp

    g = load_golden("run_simp_resume")
    _, free, F = cantilever_bc_3d(16, 8, 4)
    for leg, max_iter in (("a", 4), ("b", 7)):
        fea = OracleFEA((16, 8, 4), free, F)
        calls = []
        step = fea.step
        fea.step = lambda *a, _s=step, _c=calls: (_c.append(1), _s(*a))[1]
        p = SIMPParams(nelx=16, nely=8, nelz=4, volfrac=0.3, rmin=1.5, move=0.2, max_iter=max_iter,
                       min_iter=max_iter, use_heaviside=True, beta_init=2.0, checkpoint_dir=str(tmp_path),
                       checkpoint_every=2)
        res = run_simp(p, fea=fea)
        np.testing.assert_allclose(res["compliance_history"], g[f"compliance_{leg}"], rtol=1e-9)
        np.testing.assert_allclose(res["rho_final"], g[f"rho_final_{leg}"], rtol=1e-7, atol=1e-9)
        assert res["n_iter"] == int(g[f"n_iter_{leg}"])
        assert len(calls) == (4 if leg == "a" else 3) + 1  # iterations run here + the final evaluation
