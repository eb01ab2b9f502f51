"""Device assembly of the steady heat operator (``SteadyHeat`` with one domain).

Reference: ``SteadyHeat::initial_operator`` / ``assemble_matrix`` (src/steady/core/steady_heat.rs:80-171):
domain diffusion + production + source on points, Dirichlet rows on temperature boundaries,
boundary diffusion + production + source + Neumann on flux boundaries. Gradients of the
coefficients and of the unknown come from ``ScalarDomain::update_grad`` (src/base/scl_dom.rs:146-164).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .core import Context, Pattern, _check, default_context
from .mesh import Mesh


class SteadyHeatGpu:
    def __init__(self, mesh: Mesh, bnd_kind, ctx: Context | None = None):
        """bnd_kind[b] is ``_lib.BC_TEMP`` or ``_lib.BC_FLUX`` for boundary id b (0..5 on cube meshes)."""
        self.ctx = ctx or default_context()
        self.mesh = mesh
        kinds = np.ascontiguousarray(bnd_kind, dtype=np.int32)
        h = C.c_void_p()
        _check(self.ctx.handle, L.load().vfv_heat_create(self.ctx.handle, mesh.handle, kinds.size, L.ptr(kinds, C.c_int32),
                                                        C.byref(h)))
        self._h = h
        self.bnd_kind = kinds
        self.n = mesh.n_tot
        self.pattern = Pattern(self.ctx, L.load().vfv_heat_pattern(h), owned=False)

    def assemble(self, k, q, s, T, bc_val, return_b: bool = True):
        """Assemble A (kept on the device in ``self.pattern``) and b; host arrays of n_tot doubles."""
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (k, q, s, T, bc_val)]
        for a in arrs:
            if a.size != self.n:
                raise ValueError("field arrays must have n_tot entries")
        b = np.empty(self.n) if return_b else None
        _check(self.ctx.handle, L.load().vfv_heat_assemble(self.ctx.handle, self._h, *[a.ctypes.data_as(C.c_void_p) for a in arrs],
                                                          0, L.dptr(b) if b is not None else None))
        return b

    def assemble_device(self, k_ptr, q_ptr, s_ptr, T_ptr, bc_ptr) -> None:
        """Assemble from device arrays; b stays on the device (``rhs_device_ptr``)."""
        _check(self.ctx.handle, L.load().vfv_heat_assemble(self.ctx.handle, self._h, *[C.c_void_p(p) for p in
                                                                                        (k_ptr, q_ptr, s_ptr, T_ptr, bc_ptr)], 1, None))

    @property
    def rhs_device_ptr(self) -> int:
        return L.load().vfv_heat_rhs_device(self._h) or 0

    def adjoint(self, T, dJdT, opts=None):
        """backward(): (lambda, dJ/dlog k, dJ/dq) for an objective J(T) with gradient dJdT at the state T."""
        from .core import GmresOptions, SolveInfo
        opts = opts or GmresOptions(tol=1e-12, restart=50, max_outer=2000, precond=L.PRECOND_ILU0)
        T = np.ascontiguousarray(T, dtype=np.float64)
        g = np.ascontiguousarray(dJdT, dtype=np.float64)
        lam, dk, dq = np.empty(self.n), np.empty(self.n), np.empty(self.n)
        info = L.SolveInfo()
        o = opts.to_c()
        _check(self.ctx.handle, L.load().vfv_heat_adjoint(self.ctx.handle, self._h, L.dptr(T), L.dptr(g), C.byref(o), L.dptr(lam),
                                                         L.dptr(dk), L.dptr(dq), C.byref(info)))
        return lam, dk, dq, SolveInfo.from_c(info)

    def grad(self, f) -> np.ndarray:
        f = np.ascontiguousarray(f, dtype=np.float64)
        g = np.empty((3, self.n))
        _check(self.ctx.handle, L.load().vfv_update_grad(self.ctx.handle, self._h, L.dptr(f), L.dptr(g)))
        return g

    def close(self) -> None:
        if getattr(self, "_h", None):
            self.pattern = None
            L.load().vfv_heat_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
