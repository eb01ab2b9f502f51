"""Coupled Navier-Stokes on the GPU against the oracle (lid-driven cavity, run with -m gpu)."""
import numpy as np
import pytest

import oracle
from oracle.lu import lu_solve

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cavity(lib_built):
    from vfvchem_vfvm3d_b200.problems import lid_cavity
    return lid_cavity(7)


@pytest.fixture(scope="module")
def geom(cavity):
    return oracle.NsGeom(cavity.mesh.dual(), cavity.mesh.n_pts)


@pytest.fixture(scope="module")
def flow(gpu_ctx, cavity):
    from vfvchem_vfvm3d_b200 import SteadyFlowGpu
    return SteadyFlowGpu(cavity, ctx=gpu_ctx)


def _state(prob, seed=3):
    """A non-trivial state: smooth velocity field plus noise, boundary velocities loaded, and a
    smooth pressure."""
    n = prob.n
    pos, _, _ = prob.mesh.export()
    x, y, z = pos.T
    rng = np.random.default_rng(seed)
    u = np.stack([np.sin(np.pi * x) * np.cos(np.pi * z), 0.3 * np.sin(np.pi * y), -0.5 * np.cos(np.pi * x) * z])
    u += 0.05 * rng.standard_normal(u.shape)
    nodes = prob.node_bnd >= 0
    u[:, nodes] = prob.bc_vel[:, nodes]
    p = 0.2 * np.cos(np.pi * x) * np.sin(np.pi * y) + 0.1 * z
    return np.concatenate([u.reshape(-1), p])


def _oracle_system(geom, prob, x):
    n = prob.n
    r, c, v, b = geom.triplets(prob.node_bnd, prob.bnd_order, prob.bc_vel, prob.pref_vid, prob.pref, x[:3 * n].reshape(3, n), x[3 * n:],
                               prob.rho, prob.mu, prob.fce)
    rp, ci, va = oracle.csr_from_triplets(4 * n, r, c, v)
    return rp, ci, va, b


@pytest.mark.parametrize("which", ["initial", "perturbed"])
def test_flow_assembly_matches_oracle(flow, geom, cavity, which):
    x = cavity.initial_state() if which == "initial" else _state(cavity)
    rp, ci, va, b_o = _oracle_system(geom, cavity, x)
    b = flow.assemble(x)
    grp, gci, gva = flow.pattern.export()
    assert np.array_equal(grp.astype(np.int64), rp) and np.array_equal(gci, ci)
    assert np.max(np.abs(gva - va)) <= 1e-12 * np.max(np.abs(va))
    assert np.max(np.abs(b - b_o)) <= 1e-12 * max(np.max(np.abs(b_o)), 1e-300)


@pytest.mark.parametrize("precision", [0, 1])
def test_gmres_bj4_matches_lu(flow, geom, cavity, precision):
    """GMRES(100) + 4x4 block-Jacobi, FP64 and FP32-inner / FP64-refinement, against the LU."""
    from vfvchem_vfvm3d_b200.flow import flow_options
    x = _state(cavity)
    rp, ci, va, b_o = _oracle_system(geom, cavity, x)
    xl = lu_solve(rp, ci, va, b_o)
    b = flow.assemble(x)
    xs, info = flow.pattern.solve(b, x0=x, opts=flow_options(precision=precision, tol=1e-12, max_outer=400))
    assert info.status == 0
    assert np.linalg.norm(xs - xl) / np.linalg.norm(xl) <= 1e-8


def test_picard_matches_oracle_lu_picard(flow, geom, cavity):
    """Five damped Picard iterations on the GPU (GMRES to 1e-12) against the same loop with the
    oracle's assembly and the LU."""
    from vfvchem_vfvm3d_b200.flow import flow_options
    n = cavity.n
    res = flow.picard(max_iter=5, tol=1e-300, damp=0.8, opts=flow_options(tol=1e-12, max_outer=400), raise_on_error=False)
    assert res.iterations == 5
    x = cavity.initial_state()
    for _ in range(5):
        rp, ci, va, b = _oracle_system(geom, cavity, x)
        x = 0.2 * x + 0.8 * lu_solve(rp, ci, va, b)
    assert np.linalg.norm(res.x - x) / np.linalg.norm(x) <= 1e-8
    assert np.all(np.diff(res.residuals) < 0)  # the change shrinks every iteration on this cavity
    assert abs(res.x[3 * n + cavity.pref_vid]) == 0.0


def test_picard_mixed_tracks_fp64(flow):
    from vfvchem_vfvm3d_b200 import _lib as L
    from vfvchem_vfvm3d_b200.flow import flow_options
    # both linear solvers to relres 1e-12, so the two Picard trajectories differ only by that
    r64 = flow.picard(max_iter=6, tol=1e-300, opts=flow_options(L.FP64, tol=1e-12, max_outer=400), raise_on_error=False)
    rmx = flow.picard(max_iter=6, tol=1e-300, opts=flow_options(L.MIXED, tol=1e-12, max_outer=400), raise_on_error=False)
    assert np.linalg.norm(rmx.x - r64.x) / np.linalg.norm(r64.x) <= 1e-8


def test_picard_errors(flow):
    from vfvchem_vfvm3d_b200 import VFVChemError
    for kw in [dict(damp=0.0), dict(damp=1.5), dict(max_iter=0), dict(tol=0.0)]:
        with pytest.raises(VFVChemError):
            flow.picard(**kw)
