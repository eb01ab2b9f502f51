"""Known-answer tests that pin the CPU oracle (and the product's host-side dual) on the CPU.

The reference ships no golden vectors for this path, so the oracle is pinned to facts its
algorithms must satisfy: an independent Delaunay (Qhull) and an independent dual restatement,
closed control volumes, exact least-squares gradients and two-point fluxes for linear fields,
symmetry and zero row sums of the diffusion block, the FP64 LU solution and the 1-D slab profile
of examples/heat/heat_analytic.rs:9.
"""
import numpy as np
import scipy.sparse as sp
import pytest
from scipy.spatial import Delaunay

import oracle
from oracle import geom_tet, ordering
from oracle.lu import lu_solve
from tests.conftest import oracle_system


def _mesh(n, seed=42):
    from vfvchem_vfvm3d_b200 import Mesh
    return Mesh.jitter_cube(n, seed, 0.25)


@pytest.mark.parametrize("n", [5, 9])
def test_delaunay_matches_qhull(lib_built, n):
    m = _mesh(n, seed=3 + n)
    pos, _, tets = m.export()
    dl = Delaunay(pos)
    st = np.sort(dl.simplices, axis=1)
    a, b, c, d = (pos[st[:, i]] for i in range(4))
    vol = np.einsum("ij,ij->i", a - d, np.cross(b - d, c - d))
    st = st[np.abs(vol) > 1e-15]
    assert set(map(tuple, st)) == set(map(tuple, np.sort(tets, axis=1)))
    # every tetrahedron positively oriented (orient3d > 0), volumes fill the cube
    p = [pos[tets[:, i]] for i in range(4)]
    det = np.einsum("ij,ij->i", p[0] - p[3], np.cross(p[1] - p[3], p[2] - p[3]))
    assert np.all(det > 0)
    assert abs(det.sum() / 6.0 - 1.0) < 1e-12


@pytest.mark.parametrize("n", [6, 11])
def test_dual_matches_numpy_restatement(lib_built, n):
    m = _mesh(n)
    pos, _, tets = m.export()
    d = m.dual()
    od = geom_tet.build_dual(pos, tets, m.n_pts)
    for k in ["nbr_ptr", "nbr_idx", "bnd_ptr", "bnd_j", "bnd_k"]:
        assert np.array_equal(d[k], od[k]), k
    for k in ["dist", "area", "norm", "skew", "grad_wgt", "cvol", "cskew", "bnd_area", "bnd_norm", "bnd_wgt"]:
        scale = max(np.max(np.abs(od[k])), 1e-300)
        assert np.max(np.abs(d[k] - od[k])) <= 1e-12 * scale, k


def test_dual_from_qhull_tets_agrees(lib_built):
    """Same dual from Qhull's tetrahedra in Qhull's order (different accumulation order)."""
    m = _mesh(7)
    pos, _, tets = m.export()
    dl = Delaunay(pos)
    st = dl.simplices
    p = [pos[st[:, i]] for i in range(4)]
    vol = np.einsum("ij,ij->i", p[0] - p[3], np.cross(p[1] - p[3], p[2] - p[3]))
    od = geom_tet.build_dual(pos, st[np.abs(vol) > 1e-15], m.n_pts)
    d = m.dual()
    assert np.array_equal(d["nbr_idx"], od["nbr_idx"])
    for k in ["area", "cvol", "skew", "grad_wgt"]:
        scale = np.max(np.abs(od[k]))
        assert np.max(np.abs(d[k] - od[k])) <= 1e-10 * scale, k


def test_control_volumes_closed(lib_built):
    m = _mesh(10)
    d = m.dual()
    pos, _, _ = m.export()
    N = m.n_tot
    assert abs(d["cvol"].sum() - 1.0) < 1e-12
    owner = np.repeat(np.arange(N), np.diff(d["nbr_ptr"]))
    flux = np.zeros((N, 3))
    for c in range(3):
        np.add.at(flux[:, c], owner, d["area"] * d["norm"][c])
    bown = np.repeat(np.arange(N), np.diff(d["bnd_ptr"]))
    for c in range(3):
        np.add.at(flux[:, c], bown, d["bnd_area"] * d["bnd_norm"][c])
    scale = np.abs(d["area"]).max()
    assert np.max(np.abs(flux)) < 1e-12 * scale * 30
    # boundary sub-face normals point out of the cube
    nb_pos = pos[bown]
    out = np.where(nb_pos[:, 0] == 0.0, -1.0, np.where(nb_pos[:, 0] == 1.0, 1.0, 0.0))
    sel = (nb_pos[:, 0] == 0.0) & (nb_pos[:, 1] > 0) & (nb_pos[:, 1] < 1) & (nb_pos[:, 2] > 0) & (nb_pos[:, 2] < 1)
    assert np.allclose(d["bnd_norm"][0][sel], out[sel])


def test_unjittered_grid_degenerate_delaunay(lib_built):
    """A regular grid (jitter 0): the eight corners of every cell are cospherical, so every cell is
    split by the tie rule and every in-sphere decision there is an exact zero. The result must
    still be a positively oriented tetrahedralisation of the cube whose dual equals the numpy
    restatement on the same tetrahedra and whose control volumes close."""
    from vfvchem_vfvm3d_b200 import Mesh
    m = Mesh.jitter_cube(6, 1, 0.0)
    pos, _, tets = m.export()
    p = [pos[tets[:, i]] for i in range(4)]
    det = np.einsum("ij,ij->i", p[0] - p[3], np.cross(p[1] - p[3], p[2] - p[3]))
    assert np.all(det > 0)
    assert abs(det.sum() / 6.0 - 1.0) < 1e-12
    d = m.dual()
    od = geom_tet.build_dual(pos, tets, m.n_pts)
    for k in ["nbr_ptr", "nbr_idx", "bnd_ptr", "bnd_j", "bnd_k"]:
        assert np.array_equal(d[k], od[k]), k
    for k in ["dist", "area", "norm", "skew", "cvol", "bnd_area", "bnd_norm"]:
        scale = max(np.max(np.abs(od[k])), 1e-300)
        assert np.max(np.abs(d[k] - od[k])) <= 1e-12 * scale, k
    assert abs(d["cvol"].sum() - 1.0) < 1e-12
    # every interior control volume is the cell cube h^3, up to the 2^-18 rounding of the vertices
    h = 1.0 / 5.0
    assert np.allclose(d["cvol"][:m.n_pts], h ** 3, rtol=1e-4)


def test_lsq_gradient_exact_for_linear(lib_built):
    m = _mesh(9)
    pos, _, _ = m.export()
    d = m.dual()
    a = np.array([0.3, -1.7, 2.5])
    f = pos @ a + 4.0
    g = oracle.grad(d, f)
    assert np.max(np.abs(g - a[:, None])) < 1e-10


def test_linear_field_exactness(c1, c1_system):
    """k const, q = s = 0, zero-flux y/z walls: the two-point flux on a Voronoi dual reproduces T = x."""
    (rp, ci, va), b, _ = c1_system
    pos, _, _ = c1.mesh.export()
    x = pos[:, 0]
    r = oracle.spmv(rp, ci, va, x) - b
    assert np.max(np.abs(r)) < 1e-12
    xs = lu_solve(rp, ci, va, b)
    assert np.max(np.abs(xs - x)) < 1e-11


def test_point_block_symmetric_and_row_sums(c1_hetero, c1h_system):
    (rp, ci, va), b, _ = c1h_system
    npts = c1_hetero.mesh.n_pts
    import scipy.sparse as sp
    A = sp.csr_matrix((va, ci, rp), shape=(c1_hetero.n, c1_hetero.n))
    P = A[:npts, :npts]
    asym = abs(P - P.T).max()
    assert asym <= 1e-14 * abs(P).max()
    # row sums of the diffusion part vanish: A 1 = production diagonal only
    s_c = c1_hetero.s  # constant production, so its gradient is zero
    rowsum = np.asarray(A.sum(axis=1)).ravel()[:npts]
    assert np.allclose(rowsum, s_c[:npts] * c1_hetero.mesh.dual()["cvol"][:npts], atol=1e-13)


def test_csr_from_triplets_sums_duplicates_in_order(lib_built):
    rows = np.array([2, 0, 2, 1, 0, 2], np.uint64)
    cols = np.array([1, 0, 1, 2, 0, 0], np.uint64)
    vals = np.array([1e16, 1.0, -1e16, 3.0, 2.0, 5.0])
    rp, ci, va = oracle.csr_from_triplets(3, rows, cols, vals)
    assert rp.tolist() == [0, 1, 2, 4]
    assert ci.tolist() == [0, 2, 0, 1]
    assert va.tolist() == [3.0, 3.0, 5.0, 0.0]  # (1e16 + -1e16) kept as an explicit zero


def test_oracle_gmres_matches_lu(c1, c1_system):
    (rp, ci, va), b, _ = c1_system
    xl = lu_solve(rp, ci, va, b)
    x, ok, its, rel = oracle.gmres(rp, ci, va, b, c1.T0, tol=1e-10, restart=30, max_outer=500, precond=1)
    assert ok and rel <= 1e-10
    assert np.linalg.norm(x - xl) / np.linalg.norm(xl) < 1e-7  # condition number ~ 1e2..1e3
    x, ok, its, rel = oracle.gmres(rp, ci, va, b, c1.T0, tol=1e-13, restart=30, max_outer=2000, precond=1)
    assert ok and np.linalg.norm(x - xl) / np.linalg.norm(xl) < 1e-10


def test_oracle_ilu0_is_exact_on_pattern(c1_hetero, c1h_system):
    (rp, ci, va), _, _ = c1h_system
    for fn in (ordering.natural, ordering.multicolor):
        perm, lev = fn(rp, ci)
        # no two coupled rows share a level; lower neighbours have lower levels
        rows = np.repeat(np.arange(rp.size - 1), np.diff(rp))
        off = rows != ci
        assert np.all(lev[rows[off]] != lev[ci[off]])
        ilu = oracle.Ilu0(rp, ci, va, perm)
        n = rp.size - 1
        L = np.zeros((n, n))
        U = np.zeros((n, n))
        r2 = np.repeat(np.arange(n), np.diff(ilu.rp))
        for k in range(ilu.ci.size):
            i, j = r2[k], ilu.ci[k]
            if j < i:
                L[i, j] = ilu.lu[k]
            else:
                U[i, j] = ilu.lu[k]
        L += np.eye(n)
        LU = L @ U
        iperm = np.empty(n, np.int64)
        iperm[perm] = np.arange(n)
        pr, pc = iperm[rows], iperm[ci]
        assert np.allclose(LU[pr, pc], va, rtol=1e-12, atol=1e-12 * np.abs(va).max())


def test_oracle_ilu0_sweeps(c1h_system):
    """The Jacobi-sweep apply of the ILU(0) factors: as many sweeps as the ordering has levels
    solve both triangles exactly (N and S are nilpotent over the levels); two sweeps equal the
    recurrences written with dense factors; the iterates do not depend on the numbering."""
    (rp, ci, va), _, _ = c1h_system
    n = rp.size - 1
    r = np.random.default_rng(5).standard_normal(n)
    perm, lev = ordering.multicolor(rp, ci)
    ilu = oracle.Ilu0(rp, ci, va, perm)
    nlev = int(lev.max()) + 1
    zx = ilu.apply(r)
    assert np.linalg.norm(ilu.sweep_apply(r, nlev) - zx) <= 1e-12 * np.linalg.norm(zx)
    assert np.linalg.norm(ilu.sweep_apply(r, 1) - zx) > 1e-3 * np.linalg.norm(zx)
    rows = np.repeat(np.arange(n), np.diff(ilu.rp))
    N = np.zeros((n, n))
    S = np.zeros((n, n))
    low, up = ilu.ci < rows, ilu.ci > rows
    N[rows[low], ilu.ci[low]] = ilu.lu[low]
    S[rows[up], ilu.ci[up]] = ilu.lu[up]
    d = ilu.lu[ilu.dg]
    y = r[perm]
    u = y - N @ (y - N @ y)
    w = u / d
    w = (u - S @ ((u - S @ w) / d)) / d
    z = np.empty(n)
    z[perm] = w
    assert np.linalg.norm(ilu.sweep_apply(r, 2) - z) <= 1e-13 * np.linalg.norm(z)
    zh = ilu.sweep_apply(r, 2, half=True)  # half-precision copies: close to, but not, the float sweeps
    assert 1e-7 < np.linalg.norm(zh - z) / np.linalg.norm(z) < 1e-2
    pn, _ = ordering.natural(rp, ci)
    za = oracle.Ilu0(rp, ci, va, pn).sweep_apply(r, 3)
    zb = oracle.Ilu0(rp, ci, va, np.arange(n, dtype=np.int32)).sweep_apply(r, 3)
    assert np.linalg.norm(za - zb) <= 1e-12 * np.linalg.norm(zb)


def test_heat_slab_profile(lib_built):
    """T(x) = x + q x (1 - x) / (2 k) for a uniform source (heat_analytic.rs:9 with L = 1)."""
    from vfvchem_vfvm3d_b200.problems import steady_heat
    prob = steady_heat(16)
    prob.q[:] = 1.0
    (rp, ci, va), b, _ = oracle_system(prob)
    x = lu_solve(rp, ci, va, b)
    pos, _, _ = prob.mesh.export()
    exact = pos[:, 0] + pos[:, 0] * (1.0 - pos[:, 0]) / 2.0
    assert np.max(np.abs(x - exact)) < 5e-3


def test_oracle_adjoint_matches_finite_differences(lib_built):
    """Heat adjoint check at small size: the oracle's adjoint gradient against central differences
    (step 1e-6) of the oracle's own forward model, on random unit directions in (log k, q)."""
    from oracle import adjoint
    from vfvchem_vfvm3d_b200.problems import steady_heat
    prob = steady_heat(9, hetero=True)
    rng = np.random.default_rng(11)
    sensors = rng.choice(prob.n, size=40, replace=False)
    target = rng.uniform(0.0, 1.0, sensors.size)
    logk = np.log(prob.k)
    J, gk, gq, _ = adjoint.gradient(prob, logk, prob.q, sensors, target)
    worst = 0.0
    for _ in range(6):
        dk = rng.standard_normal(prob.n)
        dq = rng.standard_normal(prob.n)
        nrm = np.sqrt(dk @ dk + dq @ dq)
        dk, dq = dk / nrm, dq / nrm
        fd = adjoint.fd_directional(prob, logk, prob.q, sensors, target, dk, dq)
        ad = gk @ dk + gq @ dq
        worst = max(worst, abs(fd - ad) / max(abs(ad), 1e-30))
    assert worst < 1e-6


def test_transport_operator_preserves_uniform_fields(lib_built):
    """Transport oracle (time + diffusion + power-law advection, zero-flux walls): every spatial
    row sums to zero (diffusion pairs c, -c; the non-conservative advection pairs coeff, -coeff),
    so A 1 = -vol/dt and a uniform field is a fixed point of the implicit step; with zero velocity
    the diffusion block is symmetric."""
    from vfvchem_vfvm3d_b200 import Mesh
    from vfvchem_vfvm3d_b200.problems import transport_fields
    m = Mesh.jitter_cubes([6], [31])[0]
    vel, _ = transport_fields([m])
    d = m.dual()
    _, nb, _ = m.export()
    node_bnd = np.full(m.n_tot, -1, np.int32)
    node_bnd[m.n_pts:] = nb
    dt = 1e-2
    for v in (vel, np.zeros_like(vel)):
        r, c, val = oracle.transport_triplets(d, m.n_pts, node_bnd, 1e-3, v, dt)
        rp, ci, va = oracle.csr_from_triplets(m.n_tot, r, c, val)
        A = sp.csr_matrix((va, ci, rp), shape=(m.n_tot, m.n_tot))
        rows = np.asarray(A.sum(axis=1)).ravel()
        scale = np.max(np.abs(va))
        assert np.max(np.abs(rows + d["cvol"] / dt)) <= 1e-12 * scale
    asym = A - A.T  # zero velocity: pure time + diffusion
    assert abs(asym).max() <= 1e-14 * scale
