"""VTU and CSV output (host, no GPU): the library's files equal, byte for byte, the oracle's
restatement of the reference's writers (src/base/write_vtu.rs, src/base/write_csv.rs), including
Rust's spelling of non-finite numbers and exact ties in the 9-decimal rounding."""
import numpy as np
import pytest

from oracle import output as orc

SPECIALS = [np.nan, np.inf, -np.inf, -0.0, 0.0, 1e300, -1e300, 1e-12, -1e-12, 1 / 1024, 3 / 1024, -5 / 1024, 0.5e-9, 2.5e-9,
            123456789.123456789, 5e-324]


@pytest.fixture(scope="module")
def mesh(lib_built):
    from vfvchem_vfvm3d_b200 import Mesh
    return Mesh.jitter_cube(6, seed=3)


def _read(path):
    with open(path, "rb") as f:
        return f.read().decode()


def _field(n, ncomp, seed):
    v = np.random.default_rng(seed).standard_normal((n, ncomp) if ncomp == 3 else n) * 10.0
    flat = v.reshape(-1)
    flat[: len(SPECIALS)] = SPECIALS
    return v


@pytest.mark.parametrize("ncomp", [1, 3])
@pytest.mark.parametrize("ext", ["vtu", "csv"])
def test_domain_field_matches_reference_format(mesh, tmp_path, ncomp, ext):
    from vfvchem_vfvm3d_b200 import output
    pos, _, tets = mesh.export()
    v = _field(mesh.n_tot, ncomp, 1 + ncomp)
    path = output.write_domain(mesh, v, str(tmp_path / f"T.{ext}"), 7)
    assert path == str(tmp_path / f"T_0007.{ext}")
    want = orc.vtu_tets(pos, tets, v, ncomp) if ext == "vtu" else orc.csv(pos, v, ncomp)
    assert _read(path) == want


@pytest.mark.parametrize("ncomp", [1, 3])
@pytest.mark.parametrize("ext", ["vtu", "csv"])
def test_node_field_matches_reference_format(mesh, tmp_path, ncomp, ext):
    from vfvchem_vfvm3d_b200 import output
    pos, node_bnd, _ = mesh.export()
    nodes = pos[mesh.n_pts:][node_bnd == 2]  # one boundary's nodes
    v = _field(len(nodes), ncomp, 5 + ncomp)
    path = output.write_nodes(nodes, v, str(tmp_path / f"bnd.{ext}"), 12)
    assert path == str(tmp_path / f"bnd_0012.{ext}")
    want = orc.vtu_points(nodes, v, ncomp) if ext == "vtu" else orc.csv(nodes, v, ncomp)
    assert _read(path) == want


def test_interface_scalar_vtu_has_an_empty_value_array(mesh, tmp_path):
    """write_sclitf_vtu writes the value DataArray without values."""
    from vfvchem_vfvm3d_b200 import output
    pos, _, _ = mesh.export()
    nodes = pos[mesh.n_pts: mesh.n_pts + 9]
    path = output.write_nodes(nodes, None, str(tmp_path / "itf.vtu"), 0, geom="Interface")
    text = _read(path)
    assert text == orc.vtu_points(nodes, None, 1)
    assert '<DataArray type="Float64" Name="value" format="ascii">\n</DataArray>' in text


def test_large_field_spans_parallel_chunks(lib_built, tmp_path):
    """64,000 vertices and ~390,000 tetrahedra: the parallel formatter's chunks are written in order."""
    from vfvchem_vfvm3d_b200 import Mesh, output
    m = Mesh.jitter_cube(40, seed=5)
    pos, _, tets = m.export()
    v = np.random.default_rng(8).standard_normal(m.n_tot)
    path = output.write_domain(m, v, str(tmp_path / "big.vtu"), 1)
    assert _read(path) == orc.vtu_tets(pos, tets, v, 1)
    path = output.write_domain(m, np.stack([v, -v, 2 * v], 1), str(tmp_path / "big.csv"), 1)
    assert _read(path) == orc.csv(pos, np.stack([v, -v, 2 * v], 1), 3)


def test_output_paths_and_errors(mesh, tmp_path):
    from vfvchem_vfvm3d_b200 import OutputTypeError, OutputWriteError, output
    v = np.zeros(mesh.n_tot)
    assert output.output_file("run/T.vtu", 3) == "run/T_0003.vtu"
    assert output.output_file("a.b.csv", 12345) == "a.b_12345.csv"
    assert output.write_domain(mesh, v, "", 0) is None  # a blank path writes nothing
    with pytest.raises(OutputTypeError, match="Cannot deduce output file type"):
        output.write_domain(mesh, v, "noext", 0)
    with pytest.raises(OutputTypeError, match="must be CSV or VTU. Found txt"):
        output.write_domain(mesh, v, str(tmp_path / "T.txt"), 0)
    with pytest.raises(OutputWriteError, match="cannot write file"):
        output.write_domain(mesh, v, str(tmp_path / "missing_dir" / "T.vtu"), 0)
    with pytest.raises(ValueError):
        output.write_domain(mesh, np.zeros(mesh.n_tot + 1), str(tmp_path / "T.vtu"), 0)


def test_number_spelling_matches_rust():
    """Rust's {:.9} of an f64, as the oracle spells it: fixed notation, ties to even, NaN/inf."""
    assert orc.num(1 / 1024) == "0.000976562"  # exact tie ...5 at the 10th decimal: to even
    assert orc.num(3 / 1024) == "0.002929688"  # 0.0029296875: to even
    assert orc.num(-0.0) == "-0.000000000"
    assert orc.num(-1e-12) == "-0.000000000"
    assert orc.num(float("nan")) == "NaN" and orc.num(float("inf")) == "inf" and orc.num(float("-inf")) == "-inf"
    assert orc.num(1e21) == "1000000000000000000000.000000000"
