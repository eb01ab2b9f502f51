"""Mesh-stage oracle — TEST INFRASTRUCTURE (the checker, and the input builder of the CPU
baseline). C restatements in mesh_oracle.c, independent of the product's mesh code:

* ``jitter_cube(n, seed, jitter)``: the seeded jittered-cube vertex set (points first, then the
  nodes of boundaries 0..5), on the 2^-18 lattice;
* ``delaunay(pos)``: Bowyer-Watson as src/base/delaunay.rs:6-170 performs it, exact predicates;
* ``dual(pos, tets, n_pts)``: the Voronoi dual of Tetrahedron::update_tet (src/base/geom_tet.rs:101-293)
  in the layout of the product's dual export (component-major vectors).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import lib as _oracle_lib


class _DualOut(C.Structure):
    _fields_ = [("n", C.c_int64), ("n_dir", C.c_int64), ("n_bsub", C.c_int64)] + [
        (name, C.c_void_p) for name in ("nbr_ptr", "nbr_idx", "dist", "area", "norm", "skew", "grad_wgt", "cvol", "cskew", "bnd_ptr",
                                        "bnd_j", "bnd_k", "bnd_area", "bnd_norm", "bnd_wgt")]


def _lib():
    L = _oracle_lib()
    L.orc_jitter_cube.restype = C.c_int64
    L.orc_delaunay.restype = C.c_int64
    L.orc_dual.restype = C.c_int
    return L


def jitter_cube(n: int, seed: int = 42, jitter: float = 0.25):
    """(pos [N, 3], node_bnd [N] (-1 for points), n_pts) of the n^3 jittered cube."""
    N = n ** 3
    pos = np.empty((N, 3))
    bnd = np.empty(N, np.int32)
    npts = _lib().orc_jitter_cube(C.c_int(n), C.c_uint64(seed & 0xFFFFFFFFFFFFFFFF), C.c_double(jitter), C.c_void_p(pos.ctypes.data),
                                  C.c_void_p(bnd.ctypes.data))
    return pos, bnd, int(npts)


def delaunay(pos: np.ndarray) -> np.ndarray:
    """Tetrahedra [T, 4] (positively oriented) of the convex hull of pos [N, 3]."""
    pos = np.ascontiguousarray(pos, np.float64)
    out = C.c_void_p()
    L = _lib()
    nt = L.orc_delaunay(C.c_int64(pos.shape[0]), C.c_void_p(pos.ctypes.data), C.byref(out))
    if nt < 0:
        raise ValueError("oracle Delaunay: degenerate input (duplicate points, no volume)")
    tets = np.ctypeslib.as_array(C.cast(out, C.POINTER(C.c_int32)), shape=(nt * 4,)).reshape(nt, 4).copy()
    L.orc_free(out)
    return tets


def dual(pos: np.ndarray, tets: np.ndarray, n_pts: int) -> dict:
    pos = np.ascontiguousarray(pos, np.float64)
    tets = np.ascontiguousarray(tets, np.int32)
    d = _DualOut()
    L = _lib()
    rc = L.orc_dual(C.c_int64(pos.shape[0]), C.c_int64(n_pts), C.c_void_p(pos.ctypes.data), C.c_int64(tets.shape[0]),
                    C.c_void_p(tets.ctypes.data), C.byref(d))
    if rc != 0:
        L.orc_dual_free(C.byref(d))
        raise ValueError({1: "a boundary face joins an interior point", 2: "singular gradient", 3: "size out of range"}[rc])
    n, D, B = d.n, d.n_dir, d.n_bsub

    def arr(ptr, ctype, shape):
        size = int(np.prod(shape))
        if size == 0:
            return np.zeros(shape, np.ctypeslib.as_ctypes_type(ctype) if False else None)
        return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ctype)), shape=(size,)).reshape(shape).copy()

    out = {"nbr_ptr": arr(d.nbr_ptr, C.c_int64, (n + 1,)), "nbr_idx": arr(d.nbr_idx, C.c_int32, (D,)),
           "dist": arr(d.dist, C.c_double, (D,)), "area": arr(d.area, C.c_double, (D,)), "norm": arr(d.norm, C.c_double, (3, D)),
           "skew": arr(d.skew, C.c_double, (3, D)), "grad_wgt": arr(d.grad_wgt, C.c_double, (3, D)),
           "cvol": arr(d.cvol, C.c_double, (n,)), "cskew": arr(d.cskew, C.c_double, (3, n)),
           "bnd_ptr": arr(d.bnd_ptr, C.c_int64, (n + 1,)), "bnd_j": arr(d.bnd_j, C.c_int32, (B,)), "bnd_k": arr(d.bnd_k, C.c_int32, (B,)),
           "bnd_area": arr(d.bnd_area, C.c_double, (B,)), "bnd_norm": arr(d.bnd_norm, C.c_double, (3, B)),
           "bnd_wgt": arr(d.bnd_wgt, C.c_double, (3, B))}
    L.orc_dual_free(C.byref(d))
    return out
