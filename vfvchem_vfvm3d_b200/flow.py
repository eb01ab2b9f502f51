"""Steady coupled Navier-Stokes (the reference's SteadyFlow) on the device.

``SteadyFlowGpu`` holds the field-major [u | v | w | p] system of ``SteadyFlow::assemble_matrix``
(src/steady/core/steady_flow.rs:255-303) for a :class:`~vfvchem_vfvm3d_b200.problems.FlowProblem`:
velocity boundaries on every face and the pressure fixed at one vertex. ``assemble`` forms A(x)
and b(x) on the GPU (Rhie-Chow flow data of flow_helper.rs, then every operator's triplets summed
in push order); ``picard`` runs the damped Picard loop of ``SteadyBase::solve``
(src/steady/steady_base.rs:70-112) with the GMRES of :class:`~vfvchem_vfvm3d_b200.Pattern`
(GMRES(100) + 4x4 block-Jacobi by default) as the linear solver.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .core import Context, GmresOptions, Pattern, SolveInfo, _check, default_context  # noqa: F401


def pattern_host(mesh, pref_vid: int):
    """CSR pattern (rowptr, colind) of the NS system, computed on the host only."""
    nnz, nt = C.c_int64(), C.c_int64()
    _check(None, L.load().vfv_flow_pattern_host(mesh.handle, int(pref_vid), C.byref(nnz), C.byref(nt), None, None))
    rp = np.empty(4 * mesh.n_tot + 1, np.int32)
    ci = np.empty(nnz.value, np.int32)
    _check(None, L.load().vfv_flow_pattern_host(mesh.handle, int(pref_vid), None, None, L.ptr(rp, C.c_int32), L.ptr(ci, C.c_int32)))
    return rp, ci, nt.value


@dataclass
class PicardResult:
    x: np.ndarray
    residuals: np.ndarray
    lin_iters: np.ndarray
    iterations: int
    solve_seconds: float
    status: int


def flow_options(precision: int = L.FP64, tol: float = 1e-8, restart: int = 100, max_outer: int = 200) -> GmresOptions:
    """GMRES(100) + 4x4 block-Jacobi, FP64 or FP32-inner / FP64-refinement."""
    return GmresOptions(tol=tol, restart=restart, max_outer=max_outer, precond=L.PRECOND_BJ4, precision=precision, inner_rtol=1e-6)


class SteadyFlowGpu:
    def __init__(self, prob, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        self.prob = prob
        n = prob.n
        self.n = n
        rho = np.ascontiguousarray(np.broadcast_to(prob.rho, (n,)), dtype=np.float64)
        mu = np.ascontiguousarray(np.broadcast_to(prob.mu, (n,)), dtype=np.float64)
        fce = np.ascontiguousarray(prob.fce, dtype=np.float64).reshape(3, n)
        bcv = np.ascontiguousarray(prob.bc_vel, dtype=np.float64).reshape(3, n)
        h = C.c_void_p()
        _check(self.ctx.handle, L.load().vfv_flow_create(self.ctx.handle, prob.mesh.handle, L.dptr(rho), L.dptr(mu), L.dptr(fce),
                                                        L.dptr(bcv), int(prob.pref_vid), float(prob.pref), C.byref(h)))
        self._h = h
        nu, nnz, nt = C.c_int64(), C.c_int64(), C.c_int64()
        _check(self.ctx.handle, L.load().vfv_flow_info(h, C.byref(nu), C.byref(nnz), C.byref(nt)))
        self.n_unknowns, self.nnz, self.ntrip = nu.value, nnz.value, nt.value
        self.pattern = Pattern(self.ctx, L.load().vfv_flow_pattern(h), owned=False)

    def assemble(self, x) -> np.ndarray:
        """A(x) into ``pattern`` and returns b(x)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        b = np.empty(4 * self.n)
        _check(self.ctx.handle, L.load().vfv_flow_assemble(self.ctx.handle, self._h, L.dptr(x), L.dptr(b)))
        return b

    def assemble_device(self, x_ptr: int, b_ptr: int = 0) -> None:
        _check(self.ctx.handle, L.load().vfv_flow_assemble_device(self.ctx.handle, self._h, C.c_void_p(x_ptr), C.c_void_p(b_ptr or None)))

    def picard(self, x0=None, max_iter: int = 20, tol: float = 1e-3, damp: float = 0.8, opts: GmresOptions | None = None,
               raise_on_error: bool = True) -> PicardResult:
        opts = opts or flow_options()
        x = np.ascontiguousarray(self.prob.initial_state() if x0 is None else x0, dtype=np.float64).copy()
        res = np.zeros(max_iter)
        its = np.zeros(max_iter, np.int32)
        done = C.c_int32()
        ts = C.c_double()
        o = opts.to_c()
        code = L.load().vfv_flow_picard(self.ctx.handle, self._h, L.dptr(x), int(max_iter), float(tol), float(damp), C.byref(o), L.dptr(res),
                                        L.ptr(its, C.c_int32), C.byref(done), C.byref(ts))
        if code != 0 and (raise_on_error or code != L.VFV_NOT_CONVERGED):
            _check(self.ctx.handle, code)
        k = done.value
        return PicardResult(x, res[:k], its[:k], k, ts.value, code)

    def close(self) -> None:
        if getattr(self, "_h", None):
            self.pattern = None
            L.load().vfv_flow_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
