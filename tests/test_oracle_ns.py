"""Known answers for the Navier-Stokes oracle (CPU only)."""
import numpy as np
import pytest

import oracle
from oracle.lu import lu_solve


@pytest.fixture(scope="module")
def cavity(lib_built):
    from vfvchem_vfvm3d_b200.problems import lid_cavity
    return lid_cavity(7)


@pytest.fixture(scope="module")
def geom(cavity):
    return oracle.NsGeom(cavity.mesh.dual(), cavity.mesh.n_pts)


def _ns_system(geom, prob, x):
    n = prob.n
    vel, p = x[:3 * n].reshape(3, n), x[3 * n:]
    r, c, v, b = geom.triplets(prob.node_bnd, prob.bnd_order, prob.bc_vel, prob.pref_vid, prob.pref, vel, p, prob.rho, prob.mu, prob.fce)
    rp, ci, va = oracle.csr_from_triplets(4 * n, r, c, v)
    return rp, ci, va, b, (r, c, v)


def test_grad_coeff_zero_for_constants_exact_for_linear(geom, cavity):
    """sum_m c_m = 0 (closed control volume) and sum_m c_m p_m = V grad p for linear p."""
    pos, _, _ = cavity.mesh.export()
    a = np.array([0.3, -1.7, 2.2])
    p = pos @ a + 0.4
    vol = cavity.mesh.dual()["cvol"]
    for v in range(cavity.n):
        s, e = geom.gcp[v], geom.gcp[v + 1]
        c = geom.gcc[:, s:e]
        scale = np.abs(c).sum()
        assert np.all(np.abs(c.sum(axis=1)) <= 1e-13 * scale)
        g = c @ p[geom.gcv[s:e]]
        assert np.allclose(g, vol[v] * a, rtol=0, atol=1e-12 * scale)


def test_grad_coeff_rows_are_sorted_and_unique(geom):
    for v in range(geom.n):
        m = geom.gcv[geom.gcp[v]:geom.gcp[v + 1]]
        assert np.all(np.diff(m) > 0)


def test_hydrostatic_state_is_exact(geom, lib_built):
    """Closed box, no slip everywhere, body force (0, 0, -rho g): u = 0 and p = -rho g (z - z_ref)
    solve the assembled system to round-off (Rhie-Chow face flux and momentum balance both vanish)."""
    from vfvchem_vfvm3d_b200.problems import lid_cavity
    prob = lid_cavity(7, lid=(0.0, 0.0, 0.0), gravity=9.81)
    n = prob.n
    x0 = prob.initial_state()
    rp, ci, va, b, _ = _ns_system(geom, prob, x0)
    x = lu_solve(rp, ci, va, b)
    pos, _, _ = prob.mesh.export()
    p_exact = -9.81 * (pos[:, 2] - pos[prob.pref_vid, 2])
    assert np.max(np.abs(x[:3 * n])) <= 1e-10
    assert np.max(np.abs(x[3 * n:] - p_exact)) <= 1e-10 * 9.81
    # and the flow data at that state: zero face mass flux
    _, flux = geom.flow(x[:3 * n], x[3 * n:], prob.rho, prob.mu, prob.fce)
    assert np.max(np.abs(flux)) <= 1e-12


def test_pattern_properties(geom, cavity):
    n = cavity.n
    rp, ci, va, b, (r, c, v) = _ns_system(geom, cavity, cavity.initial_state())
    assert rp.size == 4 * n + 1
    xid = 3 * n + cavity.pref_vid
    assert rp[xid + 1] - rp[xid] == 1 and ci[rp[xid]] == xid and va[rp[xid]] == 1.0
    nodes = np.arange(cavity.mesh.n_pts, n)
    for q in range(3):  # Dirichlet momentum rows of the nodes: the identity
        rows = q * n + nodes
        assert np.all(rp[rows + 1] - rp[rows] == 1)
        assert np.array_equal(ci[rp[rows]], rows)
    lid_rows = nodes[cavity.node_bnd[nodes] == 5]
    assert np.all(b[lid_rows] == 1.0)
    # every pressure row of a point reaches the two-ring of velocity unknowns
    assert (rp[3 * n + 1] - rp[3 * n]) > 60


def test_picard_lid_cavity_converges_with_lu(geom, cavity):
    """Damped Picard (steady_base.rs:70-112) with the LU as the linear solver: the scaled change
    falls below 1e-3 within 30 iterations on the 7^3 cavity."""
    n = cavity.n
    x = cavity.initial_state()
    res = []
    for _ in range(30):
        rp, ci, va, b, _ = _ns_system(geom, cavity, x)
        xu = lu_solve(rp, ci, va, b)
        xd = 0.2 * x + 0.8 * xu
        du = np.sqrt(np.mean((xd[:3 * n] - x[:3 * n]) ** 2) * 3) / max(np.max(np.linalg.norm(xd[:3 * n].reshape(3, n), axis=0)), 1e-30)
        res.append(du)
        x = xd
        if du < 1e-3:
            break
    assert res[-1] < 1e-3


def test_host_pattern_matches_oracle(geom, cavity):
    """The library's host-side symbolic setup gives the oracle's de-duplicated pattern bit-exactly
    (no device needed)."""
    from vfvchem_vfvm3d_b200.flow import pattern_host
    rp, ci, va, b, (r, c, v) = _ns_system(geom, cavity, cavity.initial_state())
    hrp, hci, ntrip = pattern_host(cavity.mesh, cavity.pref_vid)
    assert np.array_equal(hrp.astype(np.int64), rp)
    assert np.array_equal(hci, ci)
    assert ntrip == r.size
