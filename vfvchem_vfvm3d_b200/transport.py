"""Batched transient advection-diffusion over many independent meshes.

The meshes are concatenated into one block-diagonal system (``vfv_transport``); every kernel of
the assembly and of the GMRES runs over all meshes at once, while every mesh keeps its own Krylov
recurrence (dot products, Hessenberg matrix, Givens rotations, stopping test), so each mesh is
solved as if alone — the reference solves each system by itself (src/transient/transient_base.rs:83-109);
a time step's solve ends when every mesh meets its own relative-residual tolerance. Operators per row, in push order:
``OpSclDomTimeUnity`` (src/operator/core/opscl_dom_timeunity.rs:32-58), ``OpSclDomDiffusion``
(opscl_dom_diff.rs:40-91), ``OpSclDomAdvection`` (power law, opscl_dom_adv.rs:49-125) with the face
mass flux of ``flow_helper::update_flux`` (flow_helper.rs:72-179) at zero pressure/body force.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .core import Context, GmresOptions, Pattern, _check, default_context
from .mesh import Mesh


class TransientTransportGpu:
    def __init__(self, meshes: list[Mesh], dt: float, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        self.meshes = meshes
        arr = (C.c_void_p * len(meshes))(*[m.handle.value if hasattr(m.handle, "value") else m.handle for m in meshes])
        h = C.c_void_p()
        _check(self.ctx.handle, L.load().vfv_transport_create(self.ctx.handle, len(meshes), arr, float(dt), C.byref(h)))
        self._h = h
        self.dt = dt
        n, nnz, nm = C.c_int64(), C.c_int64(), C.c_int32()
        _check(self.ctx.handle, L.load().vfv_transport_info(h, C.byref(n), C.byref(nnz), C.byref(nm), None))
        self.n, self.nnz, self.nmesh = n.value, nnz.value, nm.value
        self.row_ptr = np.empty(self.nmesh + 1, np.int64)
        _check(self.ctx.handle, L.load().vfv_transport_info(h, None, None, None, L.ptr(self.row_ptr, C.c_int64)))
        self.pattern = Pattern(self.ctx, L.load().vfv_transport_pattern(h), owned=False)

    def assemble(self, D, vel) -> None:
        D = np.ascontiguousarray(np.broadcast_to(D, (self.n,)), dtype=np.float64)
        vel = np.ascontiguousarray(vel, dtype=np.float64).reshape(3, self.n)
        _check(self.ctx.handle, L.load().vfv_transport_assemble(self.ctx.handle, self._h, D.ctypes.data_as(C.c_void_p),
                                                               vel.ctypes.data_as(C.c_void_p), 0))

    def run(self, c0, nsteps: int, opts: GmresOptions | None = None):
        opts = opts or GmresOptions(tol=1e-10, restart=30, max_outer=200, precond=L.PRECOND_ILU0, precision=L.MIXED,
                                    inner_rtol=1e-6)
        c0 = np.ascontiguousarray(c0, dtype=np.float64)
        out = np.empty(self.n)
        its = np.zeros(max(nsteps, 1), np.int32)
        o = opts.to_c()
        _check(self.ctx.handle, L.load().vfv_transport_run(self.ctx.handle, self._h, L.dptr(c0), int(nsteps), C.byref(o), L.dptr(out),
                                                          L.ptr(its, C.c_int32)))
        return out, its[:nsteps]

    def mesh_steps(self) -> np.ndarray:
        """Arnoldi steps of every mesh summed over the time steps of the last :meth:`run`."""
        out = np.empty(self.nmesh, np.int64)
        _check(self.ctx.handle, L.load().vfv_transport_mesh_steps(self._h, L.ptr(out, C.c_int64)))
        return out

    def adjoint_D(self, c0, nsteps: int, target, every: int = 10, opts: GmresOptions | None = None, return_iters: bool = False):
        """(J, dJ/dD) for J = 0.5 ||c_nsteps - target||^2, checkpointing every `every` steps; with
        return_iters also the GMRES iterations of each transposed solve ([k] gives lambda_{k+1})."""
        opts = opts or GmresOptions(tol=1e-12, restart=30, max_outer=500, precond=L.PRECOND_ILU0)
        c0 = np.ascontiguousarray(c0, dtype=np.float64)
        target = np.ascontiguousarray(target, dtype=np.float64)
        J, g = C.c_double(), C.c_double()
        its = np.zeros(max(nsteps, 1), np.int32)
        o = opts.to_c()
        _check(self.ctx.handle, L.load().vfv_transport_adjoint_D(self.ctx.handle, self._h, L.dptr(c0), int(nsteps), int(every),
                                                                L.dptr(target), C.byref(o), C.byref(J), C.byref(g),
                                                                L.ptr(its, C.c_int32)))
        return (J.value, g.value, its[:nsteps]) if return_iters else (J.value, g.value)

    def close(self) -> None:
        if getattr(self, "_h", None):
            self.pattern = None
            L.load().vfv_transport_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
