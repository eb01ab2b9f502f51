"""Field output in the reference's VTU and CSV formats (host, C++ in csrc/host/write_out.cpp).

An output path is split at its last dot into a name and a type, as ``ScalarDomain::new_*`` does
(src/base/scl_dom.rs:55-62); a time step ``ts`` is written to ``<name>_<ts:04>.<type>``
(src/base/write_vtu.rs:7, write_csv.rs:7). ``write_*`` dispatch on the type as
``ScalarDomain::write`` does (scl_dom.rs:132-139): an empty path writes nothing, "csv" and "vtu"
write that format, any other type raises :class:`OutputTypeError`.

Domain fields live on the mesh's vertices, points first and then nodes (the reference's vertex
numbering); boundary and interface fields on a set of nodes whose positions the caller passes.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _lib as L
from .errors import OutputTypeError, raise_for


def _check(code: int) -> None:
    if code != 0:
        msg = L.load().vfv_last_error(None)
        raise_for(code, msg.decode() if msg else f"status {code}")


def split_output_path(file_path: str, geom: str = "Domain", kind: str = "Scalar") -> tuple[str, str]:
    """(name, type) of an output path; ("", "") for no output (scl_dom.rs:55-62)."""
    if file_path == "":
        return "", ""
    name, dot, ftype = file_path.rpartition(".")
    if not dot:
        raise OutputTypeError(f"{kind}{geom}: Cannot deduce output file type from path: {file_path}.")
    return name, ftype


def output_file(file_path: str, ts: int, geom: str = "Domain", kind: str = "Scalar") -> str | None:
    """The file a time step writes, or None when the path is empty or its type is not csv/vtu
    (the latter raises, as the reference's write() does)."""
    name, ftype = split_output_path(file_path, geom, kind)
    if ftype == "":
        return None
    if ftype not in ("csv", "vtu"):
        raise OutputTypeError(f"{kind}{geom}: Output file must be CSV or VTU. Found {ftype}.")
    return f"{name}_{int(ts):04d}.{ftype}"


def _values(values, n: int) -> tuple[np.ndarray, int]:
    v = np.ascontiguousarray(values, dtype=np.float64)
    if v.shape == (n,):
        return v, 1
    if v.shape == (n, 3):
        return v, 3
    raise ValueError(f"values must have shape ({n},) or ({n}, 3), got {v.shape}")


def write_domain(mesh, values, file_path: str, ts: int) -> str | None:
    """A scalar ([n_tot]) or vector ([n_tot, 3]) field over the mesh's vertices with its tetrahedra
    (write_scldom_vtu/csv, write_vecdom_vtu/csv); returns the file written, or None."""
    v, ncomp = _values(values, mesh.n_tot)
    path = output_file(file_path, ts, "Domain", "Scalar" if ncomp == 1 else "Vector")
    if path is None:
        return None
    fn = L.load().vfv_mesh_write_vtu if path.endswith(".vtu") else L.load().vfv_mesh_write_csv
    _check(fn(mesh.handle, L.dptr(v), ncomp, os.fsencode(path)))
    return path


def write_nodes(pos, values, file_path: str, ts: int, geom: str = "Boundary") -> str | None:
    """A field on a boundary's or interface's nodes at pos [n, 3], one vertex cell each
    (write_sclbnd_*, write_vecbnd_*, write_vecitf_*). values None writes write_sclitf_vtu's empty
    value array (VTU only)."""
    p = np.ascontiguousarray(pos, dtype=np.float64)
    if p.ndim != 2 or p.shape[1] != 3:
        raise ValueError("pos must have shape (n, 3)")
    n = p.shape[0]
    if values is None:
        v, ncomp = None, 1
    else:
        v, ncomp = _values(values, n)
    path = output_file(file_path, ts, geom, "Scalar" if ncomp == 1 else "Vector")
    if path is None:
        return None
    if path.endswith(".vtu"):
        fn = L.load().vfv_points_write_vtu
    else:
        if v is None:
            raise ValueError("CSV output needs values")
        fn = L.load().vfv_points_write_csv
    _check(fn(C.c_int64(n), L.dptr(p), L.dptr(v) if v is not None else None, ncomp, os.fsencode(path)))
    return path
