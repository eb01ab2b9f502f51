"""Pure-Python restatement of the reference's VTU and CSV writers — TEST INFRASTRUCTURE ONLY.

The bytes of src/base/write_vtu.rs and src/base/write_csv.rs, line by line, for checking the
library's writers. Numbers are Rust's ``{:.9}`` of an f64: fixed notation with 9 decimals,
rounded exactly with ties to even (Python's ``%.9f``), and ``NaN``, ``inf``, ``-inf``.
"""
from __future__ import annotations

import math


def num(x: float) -> str:
    x = float(x)
    if math.isnan(x):
        return "NaN"
    if math.isinf(x):
        return "inf" if x > 0 else "-inf"
    return "%.9f" % x


def _head(npts: int, ncells: int, pos) -> list[str]:
    # the opening of every writer in write_vtu.rs: XML header, piece sizes, point coordinates
    out = ['<?xml version="1.0"?>', '<VTKFile type="UnstructuredGrid" version="0.1" byte_order="LittleEndian">', "<UnstructuredGrid>",
           f'<Piece NumberOfPoints="{npts}" NumberOfCells="{ncells}">', "<Points>",
           '<DataArray type="Float64" NumberOfComponents="3" format="ascii">']
    out += [f"{num(p[0])} {num(p[1])} {num(p[2])}" for p in pos]
    out += ["</DataArray>", "</Points>"]
    return out


def _tail(values, ncomp: int) -> list[str]:
    # the closing of every writer: point data (none for write_sclitf_vtu, write_vtu.rs:133), empty cell data
    out = ['<PointData Scalars="value">']
    if ncomp == 3:
        out.append('<DataArray type="Float64" Name="value" NumberOfComponents="3" format="ascii">')
        if values is not None:
            out += [f"{num(v[0])} {num(v[1])} {num(v[2])}" for v in values]
    else:
        out.append('<DataArray type="Float64" Name="value" format="ascii">')
        if values is not None:
            out += [num(v) for v in values]
    out += ["</DataArray>", "</PointData>", "<CellData>", "</CellData>", "</Piece>", "</UnstructuredGrid>", "</VTKFile>"]
    return out


def vtu_tets(pos, tets, values, ncomp: int) -> str:
    """write_scldom_vtu / write_vecdom_vtu (write_vtu.rs:5, :192)."""
    out = _head(len(pos), len(tets), pos)
    out += ["<Cells>", '<DataArray type="Int32" Name="connectivity" format="ascii">']
    out += [f"{t[0]} {t[1]} {t[2]} {t[3]}" for t in tets]
    out += ["</DataArray>", '<DataArray type="Int32" Name="offsets" format="ascii">']
    out += [str(4 * (k + 1)) for k in range(len(tets))]
    out += ["</DataArray>", '<DataArray type="Int32" Name="types" format="ascii">']
    out += ["10"] * len(tets)
    out += ["</DataArray>", "</Cells>"]
    out += _tail(values, ncomp)
    return "\n".join(out) + "\n"


def vtu_points(pos, values, ncomp: int) -> str:
    """write_sclbnd_vtu, write_sclitf_vtu, write_vecbnd_vtu, write_vecitf_vtu (write_vtu.rs:71, :133, :259,
    :322): one vertex cell each."""
    n = len(pos)
    out = _head(n, n, pos)
    out += ["<Cells>", '<DataArray type="Int32" Name="connectivity" format="ascii">']
    out += [str(i) for i in range(n)]
    out += ["</DataArray>", '<DataArray type="Int32" Name="offsets" format="ascii">']
    out += [str(i + 1) for i in range(n)]
    out += ["</DataArray>", '<DataArray type="Int32" Name="types" format="ascii">']
    out += ["1"] * n
    out += ["</DataArray>", "</Cells>"]
    out += _tail(values, ncomp)
    return "\n".join(out) + "\n"


def csv(pos, values, ncomp: int) -> str:
    """write_scldom_csv / write_vecdom_csv and the boundary / interface twins (write_csv.rs:5, :68; :30, :49,
    :93, :112)."""
    out = ["x,y,z,value" if ncomp == 1 else "x,y,z,value_x,value_y,value_z"]
    for p, v in zip(pos, values):
        vs = [v] if ncomp == 1 else list(v)
        out.append(",".join(num(a) for a in list(p) + vs))
    return "\n".join(out) + "\n"
