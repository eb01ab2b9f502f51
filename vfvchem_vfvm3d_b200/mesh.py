"""Seeded jittered-cube meshes with their Voronoi dual (host, C++ in csrc/host/mesh.cpp)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .errors import raise_for

BOUNDARIES = ("bnd_l", "bnd_r", "bnd_f", "bnd_k", "bnd_b", "bnd_t")  # x=0, x=1, y=0, y=1, z=0, z=1


def _check(code: int) -> None:
    if code != 0:
        msg = L.load().vfv_last_error(None)
        raise_for(code, msg.decode() if msg else f"status {code}")


class Mesh:
    """Vertices (points first, then boundary nodes), Delaunay tetrahedra and the Voronoi dual.

    ``jitter_cube(n, seed)`` builds the n^3 jittered grid on the unit cube: interior grid points
    jittered by up to +-jitter*h on each axis, surface nodes jittered in-plane only (edges along
    the edge, corners fixed), one boundary per node (x faces win over y, y over z).
    """

    def __init__(self, handle):
        self._h = handle
        a = [C.c_int64() for _ in range(5)]
        _check(L.load().vfv_mesh_info(handle, *[C.byref(x) for x in a]))
        self.n_pts, self.n_nds, self.n_tet, self.n_dir, self.n_bsub = (x.value for x in a)
        self.n_tot = self.n_pts + self.n_nds
        self._dual = None

    @classmethod
    def jitter_cube(cls, n: int, seed: int = 42, jitter: float = 0.25) -> "Mesh":
        h = C.c_void_p()
        _check(L.load().vfv_mesh_jitter_cube(int(n), int(seed) & 0xFFFFFFFFFFFFFFFF, float(jitter), C.byref(h)))
        return cls(h)

    @classmethod
    def jitter_cubes(cls, ns, seeds, jitter: float = 0.25) -> list["Mesh"]:
        """Many jittered cubes at once, built in parallel on the host."""
        ns = np.ascontiguousarray(ns, dtype=np.int32)
        seeds = np.ascontiguousarray(seeds, dtype=np.uint64)
        out = (C.c_void_p * ns.size)()
        _check(L.load().vfv_mesh_jitter_cubes(int(ns.size), L.ptr(ns, C.c_int32), L.ptr(seeds, C.c_uint64), float(jitter), out))
        return [cls(C.c_void_p(out[i])) for i in range(ns.size)]

    @classmethod
    def jitter_cubes_device_dual(cls, ctx, ns, seeds, jitter: float = 0.25) -> list["Mesh"]:
        """As :meth:`jitter_cubes`, with the Voronoi duals built on the device of ``ctx`` (same bits)."""
        ns = np.ascontiguousarray(ns, dtype=np.int32)
        seeds = np.ascontiguousarray(seeds, dtype=np.uint64)
        out = (C.c_void_p * ns.size)()
        code = L.load().vfv_mesh_jitter_cubes_device_dual(ctx.handle, int(ns.size), L.ptr(ns, C.c_int32), L.ptr(seeds, C.c_uint64),
                                                           float(jitter), out)
        if code != 0:
            msg = L.load().vfv_last_error(ctx.handle)
            raise_for(code, msg.decode() if msg else f"status {code}")
        return [cls(C.c_void_p(out[i])) for i in range(ns.size)]

    def build_dual_device(self, ctx) -> None:
        """Recompute this mesh's dual on the device of ``ctx`` (replaces the host-built one; same bits)."""
        code = L.load().vfv_mesh_dual_device(ctx.handle, self._h)
        if code != 0:
            msg = L.load().vfv_last_error(ctx.handle)
            raise_for(code, msg.decode() if msg else f"status {code}")
        self._dual = None

    @classmethod
    def from_vertices(cls, pos: np.ndarray, n_pts: int, node_bnd: np.ndarray) -> "Mesh":
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        node_bnd = np.ascontiguousarray(node_bnd, dtype=np.int32)
        h = C.c_void_p()
        _check(L.load().vfv_mesh_from_vertices(int(n_pts), int(node_bnd.size), L.dptr(pos), L.ptr(node_bnd, C.c_int32),
                                              C.byref(h)))
        return cls(h)

    @property
    def handle(self):
        return self._h

    def export(self):
        """(pos[n_tot,3], node_bnd[n_nds], tets[n_tet,4])"""
        pos = np.empty((self.n_tot, 3))
        nb = np.empty(self.n_nds, np.int32)
        tets = np.empty((self.n_tet, 4), np.int32)
        _check(L.load().vfv_mesh_export(self._h, L.dptr(pos), L.ptr(nb, C.c_int32), L.ptr(tets, C.c_int32)))
        return pos, nb, tets

    def dual(self) -> dict:
        """Flattened Tetrahedron arrays (geom_tet.rs:5-46); vectors are [3][count]."""
        if self._dual is not None:
            return self._dual
        N, D, B = self.n_tot, self.n_dir, self.n_bsub
        d = dict(
            nbr_ptr=np.empty(N + 1, np.int64), nbr_idx=np.empty(D, np.int32), dist=np.empty(D), area=np.empty(D),
            norm=np.empty((3, D)), skew=np.empty((3, D)), grad_wgt=np.empty((3, D)), cvol=np.empty(N),
            cskew=np.empty((3, N)), bnd_ptr=np.empty(N + 1, np.int64), bnd_j=np.empty(B, np.int32),
            bnd_k=np.empty(B, np.int32), bnd_area=np.empty(B), bnd_norm=np.empty((3, B)), bnd_wgt=np.empty((3, B)),
        )
        order = ["nbr_ptr", "nbr_idx", "dist", "area", "norm", "skew", "grad_wgt", "cvol", "cskew", "bnd_ptr", "bnd_j",
                 "bnd_k", "bnd_area", "bnd_norm", "bnd_wgt"]
        args = []
        for k in order:
            a = d[k]
            ct = {np.dtype(np.int64): C.c_int64, np.dtype(np.int32): C.c_int32, np.dtype(np.float64): C.c_double}[a.dtype]
            args.append(a.ctypes.data_as(C.POINTER(ct)))
        _check(L.load().vfv_mesh_export_dual(self._h, *args))
        self._dual = d
        return d

    def close(self) -> None:
        if getattr(self, "_h", None):
            L.load().vfv_mesh_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
