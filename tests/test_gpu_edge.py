"""Edge cases of the device path: tiny and ragged systems, a batch of one mesh, rows without
off-diagonals, happy breakdown of the Arnoldi process (run with -m gpu)."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg  # noqa: F401  (sp.linalg)

pytestmark = pytest.mark.gpu

ENGINES = [(1, 2), (2, 2), (1, 1), (1, 0), (0, 2)]  # (engine, precond)


def _solve(ctx, A, b, engine, precond, precision, restart=50):
    from vfvchem_vfvm3d_b200 import GmresOptions, Pattern
    A = sp.csr_matrix(A)
    A.sort_indices()
    p = Pattern.from_csr(ctx, A.indptr.astype(np.int32), A.indices.astype(np.int32))
    p.set_values(A.data.astype(np.float64))
    return p.solve(b, opts=GmresOptions(tol=1e-12, restart=restart, max_outer=200, precond=precond, precision=precision,
                                        inner_rtol=1e-6 if precision else 0.0, engine=engine))


@pytest.mark.parametrize("engine,precond", ENGINES)
@pytest.mark.parametrize("precision", [0, 1])
def test_one_by_one_system(gpu_ctx, engine, precond, precision):
    x, info = _solve(gpu_ctx, np.array([[2.5]]), np.array([5.0]), engine, precond, precision)
    assert info.status == 0 and abs(x[0] - 2.0) <= 1e-12


@pytest.mark.parametrize("engine,precond", ENGINES)
def test_diagonal_system_breaks_down_happily(gpu_ctx, engine, precond):
    """A diagonal matrix with Jacobi or ILU(0) is solved exactly in one step: the Krylov space
    closes (next basis norm 0) and the cycle must stop cleanly."""
    d = np.linspace(1.0, 3.0, 37)
    b = np.arange(1.0, 38.0)
    x, info = _solve(gpu_ctx, np.diag(d), b, engine, precond, 0)
    assert info.status == 0 and np.all(np.isfinite(x))
    assert np.max(np.abs(x - b / d)) <= 1e-12 * np.max(np.abs(b / d))


@pytest.mark.parametrize("engine,precond", ENGINES)
def test_restart_longer_than_the_system(gpu_ctx, engine, precond):
    rng = np.random.default_rng(2)
    n = 9
    A = np.diag(4.0 + rng.uniform(0, 1, n)) + np.diag(-1.0 * np.ones(n - 1), 1) + np.diag(-1.2 * np.ones(n - 1), -1)
    b = rng.standard_normal(n)
    x, info = _solve(gpu_ctx, A, b, engine, precond, 0, restart=50)
    assert info.status == 0
    assert np.linalg.norm(x - np.linalg.solve(A, b)) <= 1e-10 * np.linalg.norm(np.linalg.solve(A, b))


def test_transport_batch_of_one_mesh(gpu_ctx):
    from vfvchem_vfvm3d_b200 import GmresOptions, Mesh, TransientTransportGpu
    from vfvchem_vfvm3d_b200 import _lib as L
    from vfvchem_vfvm3d_b200.problems import transport_fields
    m = Mesh.jitter_cubes([6], [21])
    vel, c0 = transport_fields(m)
    tr = TransientTransportGpu(m, 1e-2, ctx=gpu_ctx)
    tr.assemble(1e-3, vel)
    c, its = tr.run(c0, 3, GmresOptions(tol=1e-12, restart=30, max_outer=100, precond=L.PRECOND_ILU0))
    rp, ci, va = tr.pattern.export()
    A = sp.csr_matrix((va, ci, rp), shape=(tr.n, tr.n))
    vol = m[0].dual()["cvol"]
    x = c0.copy()
    for _ in range(3):
        x = sp.linalg.spsolve(A.tocsc(), -x * vol / 1e-2)
    assert np.linalg.norm(c - x) / np.linalg.norm(x) <= 1e-9


def test_ilu_needs_every_diagonal(gpu_ctx):
    from vfvchem_vfvm3d_b200 import GmresOptions, Pattern, VFVChemError
    p = Pattern.from_csr(gpu_ctx, np.array([0, 1, 2], np.int32), np.array([1, 0], np.int32))
    p.set_values(np.array([1.0, 1.0]))
    with pytest.raises(VFVChemError):
        p.solve(np.ones(2), opts=GmresOptions(precond=2))
    x, info = p.solve(np.array([3.0, 5.0]), opts=GmresOptions(tol=1e-12, precond=0))  # the permutation itself
    assert info.status == 0 and np.allclose(x, [5.0, 3.0], rtol=0, atol=1e-12)
