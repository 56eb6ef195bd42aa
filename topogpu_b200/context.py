"""Torch-facing wrapper of one ``topo_ctx`` (grid + multigrid hierarchy).

Every method takes CUDA tensors (contiguous, dtype checked here), passes raw
device pointers and the current torch stream to the C ABI, and raises on a
negative status. Vectors are full length (all DoFs, reference numbering) with
fixed DoFs held at zero.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .fem import KE_UNIT

_DT = {torch.float64: _lib.F64, torch.float32: _lib.F32, torch.bfloat16: _lib.BF16}


def _ptr(t: torch.Tensor, dtype=None, n=None, name="tensor") -> int:
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError(f"{name} must be a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    if dtype is not None and t.dtype not in (dtype if isinstance(dtype, tuple) else (dtype,)):
        raise TypeError(f"{name} has dtype {t.dtype}, expected {dtype}")
    if n is not None and t.numel() != n:
        raise ValueError(f"{name} has {t.numel()} entries, expected {n}")
    return t.data_ptr()


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


class TopoContext:
    """Structured hex8 grid ``nel=(nelx, nely, nelz)`` with its GMG hierarchy.

    mode: "fp64" | "fp32" | "mixed" (see include/topo_b200.h).
    """

    SMOOTHERS = {"reference": 0, "chebyshev": 1}

    def __init__(self, nel, n_levels=4, mode="mixed", fine_degree=2, coarse_degree=2,
                 cheb_lower=1.0 / 30.0, dense_max=16384, KE=None, smoother="chebyshev", lam_safety=None):
        self._lib = _lib.load()
        if mode not in _lib.MODES:
            raise ValueError(f"mode must be one of {sorted(_lib.MODES)}, got {mode!r}")
        self.nel = tuple(int(v) for v in nel)
        nx, ny, nz = self.nel
        self.n_elem = nx * ny * nz
        self.n_nodes = (nx + 1) * (ny + 1) * (nz + 1)
        self.ndof = 3 * self.n_nodes
        self.n_levels = int(n_levels)
        self.mode = mode
        self.vec_dtype = torch.float64 if mode == "fp64" else torch.float32
        ke = np.ascontiguousarray(KE if KE is not None else KE_UNIT, dtype=np.float64)
        h = C.c_void_p()
        rc = self._lib.topo_ctx_create(nx, ny, nz, self.n_levels, _lib.MODES[mode], int(fine_degree),
                                       int(coarse_degree), float(cheb_lower), int(dense_max),
                                       ke.ctypes.data_as(C.c_void_p), C.byref(h))
        _lib.check(rc, None, "topo_ctx_create")
        self._h = h
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.set_smoother(smoother, lam_safety)

    def set_smoother(self, smoother="chebyshev", lam_safety=None):
        """"reference" reproduces the reference V-cycle (safety 1.0 by
        default); "chebyshev" is the first-kind Chebyshev iteration (safety
        1.25 by default)."""
        if smoother not in self.SMOOTHERS:
            raise ValueError(f"smoother must be one of {sorted(self.SMOOTHERS)}")
        if lam_safety is None:
            lam_safety = 1.0 if smoother == "reference" else 1.25
        self._chk(self._lib.topo_set_smoother(self._h, self.SMOOTHERS[smoother], float(lam_safety)), "set_smoother")
        self.smoother, self.lam_safety = smoother, float(lam_safety)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.topo_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, rc, what):
        return _lib.check(rc, self._h, what)

    # -- problem -----------------------------------------------------------
    def set_problem(self, free_mask: torch.Tensor, F: torch.Tensor):
        self._chk(self._lib.topo_set_problem(self._h, _ptr(free_mask, torch.uint8, self.ndof, "free_mask"),
                                             _ptr(F, torch.float64, self.ndof, "F"), _stream()), "set_problem")

    def modulus(self, rho, penal=3.0, E0=1.0, Emin=1e-9, out=None):
        out = torch.empty_like(rho) if out is None else out
        self._chk(self._lib.topo_modulus(self._h, _ptr(rho, torch.float64, self.n_elem, "rho"), penal, E0, Emin,
                                         _ptr(out, torch.float64, self.n_elem, "E"), _stream()), "modulus")
        return out

    # -- operators ---------------------------------------------------------
    def matvec(self, u: torch.Tensor, E: torch.Tensor, out=None):
        """y = K(E) u (fixed rows zero). u: f64 / f32 / bf16; E and y follow
        u's precision (f32 for bf16)."""
        dt = _DT.get(u.dtype)
        if dt is None:
            raise TypeError(f"unsupported dtype {u.dtype}")
        ydt = torch.float64 if u.dtype == torch.float64 else torch.float32
        out = torch.empty(self.ndof, dtype=ydt, device=u.device) if out is None else out
        self._chk(self._lib.topo_matvec(self._h, dt, _ptr(u, None, self.ndof, "u"), _ptr(out, ydt, self.ndof, "y"),
                                        _ptr(E, ydt, self.n_elem, "E"), _stream()), "matvec")
        return out

    EPILOGUES = {"store": _lib.EPI_STORE, "residual": _lib.EPI_RESIDUAL, "rupd": _lib.EPI_RUPD,
                 "cheb": _lib.EPI_CHEB}

    def wait_status(self):
        """Synchronise and raise if a wait of an earlier level-0 launch timed
        out (asynchronous entries report it only at their next call)."""
        self._chk(self._lib.topo_wait_status(self._h, _stream()), "wait_status")

    def level0_apply(self, u, E, epi="store", *, y=None, b=None, r=None, x=None, d_out=None, dinv=None, s=1.0,
                     c1=0.0, c2=0.0, ax=0.0, u_fp32_to_bf16=False):
        """One level-0 operator application with its fused epilogue (see
        topo_level0_apply): "store" y = K u, "residual" y = b - K u, "rupd"
        r -= s K u, "cheb" r -= s K u; d_out = c1 u + c2 dinv r; x += ax d_out.
        u's dtype picks the arithmetic (f64, f32, bf16); u_fp32_to_bf16 runs
        an f32 u through the BF16 tensor-core operator (the smoother's form).
        The other vectors are f64 for an f64 u and f32 otherwise. Returns y
        for "store"/"residual", else None (r, x, d_out are updated)."""
        if epi not in self.EPILOGUES:
            raise ValueError(f"epi must be one of {sorted(self.EPILOGUES)}")
        if u_fp32_to_bf16:
            if u.dtype != torch.float32:
                raise TypeError("u_fp32_to_bf16 needs an f32 u")
            dt = _lib.BF16_F32IN
        else:
            dt = _DT.get(u.dtype)
            if dt is None:
                raise TypeError(f"unsupported dtype {u.dtype}")
        vdt = torch.float64 if u.dtype == torch.float64 else torch.float32
        if epi in ("store", "residual") and y is None:
            y = torch.empty(self.ndof, dtype=vdt, device=u.device)

        def opt(t, name, n=self.ndof):
            return None if t is None else _ptr(t, vdt, n, name)

        self._chk(self._lib.topo_level0_apply(self._h, dt, self.EPILOGUES[epi], _ptr(u, None, self.ndof, "u"),
                                              _ptr(E, vdt, self.n_elem, "E"), opt(y, "y"), opt(b, "b"), opt(r, "r"),
                                              opt(x, "x"), opt(d_out, "d_out"), opt(dinv, "dinv"), float(s), float(c1),
                                              float(c2), float(ax), _stream()), "level0_apply")
        return y if epi in ("store", "residual") else None

    def diag(self, E, out=None):
        out = torch.empty(self.ndof, dtype=torch.float64, device=E.device) if out is None else out
        self._chk(self._lib.topo_diag(self._h, _ptr(E, torch.float64, self.n_elem, "E"),
                                      _ptr(out, torch.float64, self.ndof, "diag"), _stream()), "diag")
        return out

    def gmg_setup(self, E):
        self._chk(self._lib.topo_gmg_setup(self._h, _ptr(E, torch.float64, self.n_elem, "E"), _stream()),
                  "gmg_setup")

    def gmg_apply(self, r, out=None):
        out = torch.empty_like(r) if out is None else out
        self._chk(self._lib.topo_gmg_apply(self._h, _ptr(r, self.vec_dtype, self.ndof, "r"),
                                           _ptr(out, self.vec_dtype, self.ndof, "z"), _stream()), "gmg_apply")
        return out

    def pcg(self, b, x, tol=1e-5, maxiter=800):
        """Solve in place into x (holds the initial guess). Returns
        (iterations, true relative residual, converged)."""
        it, rr = C.c_int(0), C.c_double(0.0)
        rc = self._chk(self._lib.topo_pcg(self._h, _ptr(b, torch.float64, self.ndof, "b"),
                                          _ptr(x, torch.float64, self.ndof, "x"), float(tol), int(maxiter),
                                          C.byref(it), C.byref(rr), _stream()), "pcg")
        return it.value, rr.value, rc == 0

    def fgmres(self, b, x, tol=1e-5, maxiter=800, restart=32):
        it, rr = C.c_int(0), C.c_double(0.0)
        rc = self._chk(self._lib.topo_fgmres(self._h, _ptr(b, torch.float64, self.ndof, "b"),
                                             _ptr(x, torch.float64, self.ndof, "x"), float(tol), int(maxiter),
                                             int(restart), C.byref(it), C.byref(rr), _stream()), "fgmres")
        return it.value, rr.value, rc == 0

    def set_coarse_lag(self, on: bool):
        """Apply the previous setup's coarsest factor while the new one builds
        in the background (see topo_set_coarse_lag)."""
        self._chk(self._lib.topo_set_coarse_lag(self._h, int(bool(on))), "set_coarse_lag")

    def set_cycle(self, cycle_type: str):
        """"v" (one coarse correction per level) or "w" (two)
        (multigrid_v4.py:986-1042)."""
        if cycle_type not in ("v", "w"):
            raise ValueError(f"cycle_type must be 'v' or 'w'; got {cycle_type!r}")
        self._chk(self._lib.topo_set_cycle(self._h, 1 if cycle_type == "v" else 2), "set_cycle")

    def set_tensor_cores(self, on: bool):
        """BF16 level-0 K.u on tcgen05 (True) or on the CUDA cores (False)."""
        self._chk(self._lib.topo_set_tc(self._h, int(bool(on))), "set_tc")

    def block_pcg(self, B, X, tol=1e-5, maxiter=800):
        """Block PCG over the rows of B (nrhs x ndof, float64); X (same shape)
        holds initial guesses and receives the solutions. Returns
        (iterations, [relres per column], all_converged)."""
        if B.dim() != 2 or B.shape != X.shape or B.shape[1] != self.ndof:
            raise ValueError("block_pcg: B and X must be (nrhs, ndof)")
        nrhs = int(B.shape[0])
        it = C.c_int(0)
        rr = (C.c_double * nrhs)()
        rc = self._chk(self._lib.topo_block_pcg(self._h, _ptr(B, torch.float64, nrhs * self.ndof, "B"),
                                                _ptr(X, torch.float64, nrhs * self.ndof, "X"), nrhs, float(tol),
                                                int(maxiter), C.byref(it), rr, _stream()), "block_pcg")
        return it.value, list(rr), rc == 0

    # -- design ------------------------------------------------------------
    def sensitivity(self, u, rho, penal=3.0, E0=1.0, Emin=1e-9, out=None):
        dt = _DT.get(u.dtype)
        if dt not in (_lib.F64, _lib.F32):
            raise TypeError("u must be float64 or float32")
        out = torch.empty(self.n_elem, dtype=torch.float64, device=u.device) if out is None else out
        self._chk(self._lib.topo_sensitivity(self._h, _ptr(u, None, self.ndof, "u"), dt,
                                             _ptr(rho, torch.float64, self.n_elem, "rho"), penal, E0, Emin,
                                             _ptr(out, torch.float64, self.n_elem, "dc"), _stream()), "sensitivity")
        return out

    def sensitivity_adjoint(self, u, lam, rho, penal=3.0, E0=1.0, Emin=1e-9, out=None):
        """dJ/drho for J = L^T u given the adjoint lam (K lam = L)."""
        dt = _DT.get(u.dtype)
        if dt not in (_lib.F64, _lib.F32) or lam.dtype != u.dtype:
            raise TypeError("u and lam must both be float64 or both float32")
        out = torch.empty(self.n_elem, dtype=torch.float64, device=u.device) if out is None else out
        self._chk(self._lib.topo_sensitivity_adjoint(self._h, _ptr(u, None, self.ndof, "u"),
                                                     _ptr(lam, None, self.ndof, "lam"), dt,
                                                     _ptr(rho, torch.float64, self.n_elem, "rho"), penal, E0, Emin,
                                                     _ptr(out, torch.float64, self.n_elem, "dc"), _stream()),
                  "sensitivity_adjoint")
        return out

    def dot(self, a, b) -> float:
        if a.dtype != b.dtype or a.numel() != b.numel():
            raise ValueError("dot: operands must match in dtype and size")
        out = C.c_double(0.0)
        self._chk(self._lib.topo_dot(self._h, _DT[a.dtype], _ptr(a, None, None, "a"), _ptr(b, None, None, "b"),
                                     a.numel(), C.byref(out), _stream()), "dot")
        return out.value

    def filter(self, rmin, x, transpose=False, out=None):
        out = torch.empty_like(x) if out is None else out
        self._chk(self._lib.topo_filter(self._h, float(rmin), _ptr(x, torch.float64, self.n_elem, "in"),
                                        _ptr(out, torch.float64, self.n_elem, "out"), int(bool(transpose)),
                                        _stream()), "filter")
        return out

    def oc(self, rho, dc, volfrac, move=0.10, rho_min=1e-3, out=None):
        out = torch.empty_like(rho) if out is None else out
        ev = C.c_int(0)
        self._chk(self._lib.topo_oc(self._h, _ptr(rho, torch.float64, self.n_elem, "rho"),
                                    _ptr(dc, torch.float64, self.n_elem, "dc"), float(volfrac), float(move),
                                    float(rho_min), _ptr(out, torch.float64, self.n_elem, "out"), C.byref(ev),
                                    _stream()), "oc")
        return out, ev.value

    def oc_filtered(self, rho, dc, dv, colsum, volfrac, move=0.2, rho_min=1e-3, out=None):
        out = torch.empty_like(rho) if out is None else out
        ev = C.c_int(0)
        n = self.n_elem
        self._chk(self._lib.topo_oc_filtered(self._h, _ptr(rho, torch.float64, n, "rho"), _ptr(dc, torch.float64, n, "dc"),
                                             _ptr(dv, torch.float64, n, "dv"), _ptr(colsum, torch.float64, n, "colsum"),
                                             float(volfrac), float(move), float(rho_min),
                                             _ptr(out, torch.float64, n, "out"), C.byref(ev), _stream()),
                  "oc_filtered")
        return out, ev.value

    def heaviside(self, rho_f, beta, eta=0.5, phys=None, dh=None, want_deriv=True):
        """Projection h(rho_f) and, with ``want_deriv``, h'(rho_f)
        (pub_simp_solver.py:245-253)."""
        n = self.n_elem
        phys = torch.empty_like(rho_f) if phys is None else phys
        if want_deriv and dh is None:
            dh = torch.empty_like(rho_f)
        self._chk(self._lib.topo_heaviside(self._h, _ptr(rho_f, torch.float64, n, "rho_f"), float(beta), float(eta),
                                           _ptr(phys, torch.float64, n, "phys"),
                                           _ptr(dh, torch.float64, n, "dh") if want_deriv else None, _stream()),
                  "heaviside")
        return (phys, dh) if want_deriv else phys

    def oc_projected(self, rmin, rho, dc, dv, beta, eta=0.5, volfrac=0.3, move=0.2, rho_min=1e-3, out=None):
        """run_simp's OC with the volume measured after filter and projection
        (pub_simp_solver.py:319-340)."""
        out = torch.empty_like(rho) if out is None else out
        ev = C.c_int(0)
        n = self.n_elem
        self._chk(self._lib.topo_oc_projected(self._h, float(rmin), _ptr(rho, torch.float64, n, "rho"),
                                              _ptr(dc, torch.float64, n, "dc"), _ptr(dv, torch.float64, n, "dv"),
                                              float(beta), float(eta), float(volfrac), float(move), float(rho_min),
                                              _ptr(out, torch.float64, n, "out"), C.byref(ev), _stream()),
                  "oc_projected")
        return out, ev.value

    def field_stats(self, x):
        out = (C.c_double * 4)()
        self._chk(self._lib.topo_field_stats(self._h, _ptr(x, torch.float64, None, "x"), x.numel(), out, _stream()),
                  "field_stats")
        return {"mean": out[0], "min": out[1], "max": out[2], "grayness": out[3]}

    def gmg_info(self):
        nf = (C.c_longlong * self.n_levels)()
        lam = (C.c_double * self.n_levels)()
        kind = C.c_int(0)
        self._chk(self._lib.topo_gmg_info(self._h, nf, lam, C.byref(kind)), "gmg_info")
        return {"n_free": list(nf), "lambda_max": list(lam),
                "coarse_solve": {0: "none", 1: "dense_cholesky", 2: "regularised_cholesky"}.get(kind.value, "?")}

    def setup_phases(self) -> dict:
        """Device milliseconds of the phases of the last gmg_setup."""
        ms = (C.c_double * 5)()
        self._chk(self._lib.topo_setup_phases(self._h, ms), "setup_phases")
        return dict(zip(("fine_diag_lambda", "coarse_stencils", "coarsest_copy", "coarsest_factor", "pivot_check"),
                        list(ms)))

    def level_operator(self, level: int) -> torch.Tensor:
        """FP64 stencil of coarse level ``level`` as a (27, 3, 3, nnodes) tensor."""
        nx, ny, nz = self.nel
        for _ in range(level):
            nx, ny, nz = max(1, nx // 2), max(1, ny // 2), max(1, nz // 2)
        nn = (nx + 1) * (ny + 1) * (nz + 1)
        out = torch.empty(243 * nn, dtype=torch.float64, device=self.device)
        self._chk(self._lib.topo_gmg_level_operator(self._h, int(level), out.data_ptr(), _stream()), "level_operator")
        return out.view(27, 3, 3, nn)

    def workspace_bytes(self) -> int:
        return int(self._lib.topo_workspace_bytes(self._h))
