"""The mesh-stage oracle (oracle/mesh_oracle.c) against the product's host mesh code and against
independent facts (CPU only).

The oracle restates the reference's Bowyer-Watson insertion (src/base/delaunay.rs:6-170) and the
dual of Tetrahedron::update_tet (src/base/geom_tet.rs:101-293) in C with exact predicates. The
product builds the same tetrahedra (the Delaunay tetrahedralisation of points in general position
is unique) in a different order (its insertion order and tetrahedron storage differ), so sums over
tetrahedra agree to round-off, not bit for bit, and per-vertex boundary sub-faces agree as sets.
"""
import numpy as np
import pytest
from scipy.spatial import Delaunay

from oracle import geom_tet
from oracle import mesh as om


def _tetset(t):
    return set(map(tuple, np.sort(np.asarray(t), axis=1)))


def test_jitter_cube_equals_product_vertices(lib_built):
    from vfvchem_vfvm3d_b200 import Mesh
    pos, bnd, npts = om.jitter_cube(9, 42, 0.25)
    m = Mesh.jitter_cube(9, 42, 0.25)
    ppos, pnb, _ = m.export()
    assert npts == m.n_pts
    assert np.array_equal(pos, ppos) and np.array_equal(bnd[npts:], pnb) and np.all(bnd[:npts] == -1)
    assert np.array_equal(np.ldexp(pos, 18), np.rint(np.ldexp(pos, 18)))  # on the 2^-18 lattice


@pytest.mark.parametrize("n", [5, 8, 12])
def test_delaunay_equals_qhull_and_product(lib_built, n):
    from vfvchem_vfvm3d_b200 import Mesh
    pos, _, _ = om.jitter_cube(n, 100 + n, 0.25)
    tets = om.delaunay(pos)
    p = [pos[tets[:, i]] for i in range(4)]
    det = np.einsum("ij,ij->i", p[0] - p[3], np.cross(p[1] - p[3], p[2] - p[3]))
    assert np.all(det > 0) and abs(det.sum() / 6.0 - 1.0) < 1e-12
    st = np.sort(Delaunay(pos).simplices, axis=1)
    a, b, c, d = (pos[st[:, i]] for i in range(4))
    st = st[np.abs(np.einsum("ij,ij->i", a - d, np.cross(b - d, c - d))) > 1e-15]
    assert _tetset(tets) == _tetset(st)
    _, _, ptets = Mesh.jitter_cube(n, 100 + n, 0.25).export()
    assert _tetset(tets) == _tetset(ptets)


def test_delaunay_rejects_duplicates():
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 0, 0]], float)
    with pytest.raises(ValueError):
        om.delaunay(pos)


@pytest.mark.parametrize("n", [6, 10])
def test_dual_agrees_with_product_and_numpy_restatement(lib_built, n):
    from vfvchem_vfvm3d_b200 import Mesh
    pos, _, npts = om.jitter_cube(n, 42, 0.25)
    tets = om.delaunay(pos)
    d = om.dual(pos, tets, npts)
    nd = geom_tet.build_dual(pos, tets, npts)  # numpy restatement on the oracle's own tetrahedra and order
    for k in ["nbr_ptr", "nbr_idx", "bnd_ptr", "bnd_j", "bnd_k"]:
        assert np.array_equal(d[k].astype(np.int64), np.asarray(nd[k]).astype(np.int64)), k
    for k in ["dist", "area", "norm", "skew", "grad_wgt", "cvol", "cskew", "bnd_area", "bnd_norm", "bnd_wgt"]:
        scale = max(np.max(np.abs(nd[k])), 1e-300)
        assert np.max(np.abs(d[k] - nd[k])) <= 1e-12 * scale, k
    pd = Mesh.jitter_cube(n, 42, 0.25).dual()
    for k in ["nbr_ptr", "nbr_idx", "bnd_ptr"]:
        assert np.array_equal(d[k].astype(np.int64), pd[k].astype(np.int64)), k
    for k in ["dist", "norm", "grad_wgt", "area", "cvol", "cskew"]:
        assert np.max(np.abs(d[k] - pd[k])) <= 1e-12 * np.max(np.abs(pd[k])), k
    # skew is a ratio with the face area: compare it on faces that carry area
    big = np.abs(pd["area"]) > 1e-6 * pd["dist"] ** 2
    assert np.max(np.abs(d["skew"][:, big] - pd["skew"][:, big])) <= 1e-10 * np.max(np.abs(pd["skew"]))
    # boundary sub-faces: the same (j, k, area) per vertex, listed in each code's triangle order
    for v in range(n ** 3):
        a0, a1, b0, b1 = d["bnd_ptr"][v], d["bnd_ptr"][v + 1], pd["bnd_ptr"][v], pd["bnd_ptr"][v + 1]
        sa = sorted(zip(d["bnd_j"][a0:a1], d["bnd_k"][a0:a1]))
        sb = sorted(zip(pd["bnd_j"][b0:b1], pd["bnd_k"][b0:b1]))
        assert sa == sb
    # control volumes tile the unit cube and close: sum over faces of A n = 0 for interior points
    assert abs(d["cvol"].sum() - 1.0) < 1e-12
    v = np.repeat(np.arange(n ** 3), np.diff(d["nbr_ptr"]))
    an = np.zeros((3, n ** 3))
    for c in range(3):
        np.add.at(an[c], v, d["area"] * d["norm"][c])
    assert np.max(np.abs(an[:, :npts])) < 1e-12


def _box_jitter(n, seed, scale=1.0, shift=0.0):
    """A jittered n^3 grid in raw doubles (no lattice), faces jittered in plane, corners fixed, then
    scaled and shifted: the hull is the box, the vertices are in general position."""
    rng = np.random.default_rng(seed)
    g = np.linspace(0.0, 1.0, n)
    x, y, z = np.meshgrid(g, g, g, indexing="ij")
    p = np.stack([x.ravel(), y.ravel(), z.ravel()], 1)
    h = 1.0 / (n - 1)
    inner = (p > 0) & (p < 1)
    p = p + inner * rng.uniform(-0.3, 0.3, p.shape) * h
    return p * scale + shift


def _points_and_nodes(pos):
    """Interior vertices first, then the hull's with one boundary id each (x faces over y over z),
    the vertex order and boundary rule of the generated cubes; returns (pos, n_pts, node_bnd)."""
    lo, hi = pos.min(0), pos.max(0)
    bid = np.full(len(pos), -1)
    for c in (2, 1, 0):  # x faces win: assigned last
        bid[pos[:, c] == lo[c]] = 2 * c
        bid[pos[:, c] == hi[c]] = 2 * c + 1
    inner = bid < 0
    return np.concatenate([pos[inner], pos[~inner]]), int(inner.sum()), bid[~inner].astype(np.int32)


def _exact_checks(pos, tets):
    """Exact rational checks of a tetrahedralisation: positive orientation, volumes summing to the
    box, and no vertex strictly inside any circumsphere."""
    from fractions import Fraction as F
    P = [[F(float(c)) for c in q] for q in pos]

    def sub(a, b):
        return [a[0] - b[0], a[1] - b[1], a[2] - b[2]]

    def det3(a, b, c):
        return a[0] * (b[1] * c[2] - b[2] * c[1]) - a[1] * (b[0] * c[2] - b[2] * c[0]) + a[2] * (b[0] * c[1] - b[1] * c[0])

    vol = F(0)
    for t in tets:
        a, b, c, d = (P[i] for i in t)
        o = det3(sub(a, d), sub(b, d), sub(c, d))
        assert o > 0
        vol += o / 6
        for j, e in enumerate(P):
            if j in t:
                continue
            q = [sub(a, e), sub(b, e), sub(c, e), sub(d, e)]
            lf = [v[0] * v[0] + v[1] * v[1] + v[2] * v[2] for v in q]
            r = (lf[1] * det3(q[0], q[2], q[3]) - lf[0] * det3(q[1], q[2], q[3]) + lf[3] * det3(q[0], q[1], q[2])
                 - lf[2] * det3(q[0], q[1], q[3]))
            assert r <= 0  # not strictly inside
    lo = [min(q[i] for q in P) for i in range(3)]
    hi = [max(q[i] for q in P) for i in range(3)]
    assert vol == (hi[0] - lo[0]) * (hi[1] - lo[1]) * (hi[2] - lo[2])


@pytest.mark.parametrize("scale,shift", [(1.0, 0.0), (3.7, 0.0), (1e-3, 123.456), (250.0, -1e4)])
def test_delaunay_of_raw_doubles_equals_qhull(lib_built, scale, shift):
    """Vertices off the 2^-18 lattice and far outside the unit box (a domain in metres, offset):
    the double predicates with their exact fallback give Qhull's tetrahedra."""
    from vfvchem_vfvm3d_b200 import Mesh
    pos, n_pts, bnd = _points_and_nodes(_box_jitter(6, 11, scale, shift))
    m = Mesh.from_vertices(pos, n_pts, bnd)
    _, _, tets = m.export()
    # Qhull rounds in doubles, so it gets the exactly translated copy (each difference of two
    # coordinates within a factor of two is exact); the Delaunay tetrahedra do not change
    rel = pos - pos.min(0)
    assert np.array_equal(rel + pos.min(0), pos)
    st = np.sort(Delaunay(rel).simplices, axis=1)
    a, b, c, d = (rel[st[:, i]] for i in range(4))
    vol = np.abs(np.einsum("ij,ij->i", a - d, np.cross(b - d, c - d)))
    st = st[vol > 1e-12 * vol.max()]
    assert _tetset(tets) == _tetset(st)
    d = m.dual()  # the Voronoi dual builds on it: control volumes fill the box
    assert d["nbr_ptr"][-1] == m.n_dir
    box = np.prod(pos.max(0) - pos.min(0))
    assert abs(d["cvol"].sum() - box) <= 1e-9 * box


def test_delaunay_of_cospherical_doubles_is_exact(lib_built):
    """A regular grid of spacing 0.1 (off the lattice; every cell's 8 corners cospherical): the exact
    fallback settles every tie; the result is a valid Delaunay tetrahedralisation, checked in
    rationals."""
    from vfvchem_vfvm3d_b200 import Mesh
    g = np.arange(4) * 0.1
    x, y, z = np.meshgrid(g, g, g, indexing="ij")
    pos, n_pts, bnd = _points_and_nodes(np.stack([x.ravel(), y.ravel(), z.ravel()], 1))
    m = Mesh.from_vertices(pos, n_pts, bnd)
    _, _, tets = m.export()
    _exact_checks(pos, tets)


def test_delaunay_of_ulp_perturbed_grid_is_exact(lib_built):
    """Interior vertices of a 0.1-spaced grid moved by one ulp (the hull stays the box): every
    circumsphere test is within rounding of zero, so the big-integer fallback decides nearly all of
    them; the result is checked in rationals."""
    from vfvchem_vfvm3d_b200 import Mesh
    g = np.arange(5) * 0.1
    x, y, z = np.meshgrid(g, g, g, indexing="ij")
    p = np.stack([x.ravel(), y.ravel(), z.ravel()], 1)
    rng = np.random.default_rng(21)
    inner = np.all((p > 0) & (p < g[-1]), axis=1)
    steps = rng.integers(-1, 2, size=(int(inner.sum()), 3))
    q = p[inner]
    q = np.where(steps > 0, np.nextafter(q, np.inf), np.where(steps < 0, np.nextafter(q, -np.inf), q))
    p[inner] = q
    pos, n_pts, bnd = _points_and_nodes(p)
    m = Mesh.from_vertices(pos, n_pts, bnd)
    _, _, tets = m.export()
    _exact_checks(pos, tets)
