"""Bounded device waits, the single-launch ILU(0) sweeps and the dataflow ILU(0) factorisation
(run with -m gpu on a B200).

The persistent engine's grid barriers, the single-launch ILU(0) sweeps (VFV_ILU_CHAIN=1) and the
dataflow factorisation of orderings with many levels (a warp per row waiting for its pivot rows)
wait on other CTAs through memory; every such wait has a poll limit (vfv_gmres_opts.wait_limit). A
limit of one poll makes the waits give up in practice (a barrier needs every CTA to arrive; a
natural-order ILU(0) row needs rows of the level before it): the solve must then end with status 5
(DeviceWaitTimeout) instead of hanging, and the same context must solve correctly right
afterwards.
"""
import numpy as np
import pytest

from oracle.lu import lu_solve

pytestmark = pytest.mark.gpu

SOL_RTOL = 1e-8


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def _pattern(ctx, system):
    from vfvchem_vfvm3d_b200 import Pattern
    (rp, ci, va), b, _ = system
    p = Pattern.from_csr(ctx, rp.astype(np.int32), ci)
    p.set_values(va)
    return p


@pytest.mark.parametrize("engine,order", [(0, 0), (1, 1)])
def test_wait_that_gives_up_reports_timeout_and_context_recovers(gpu_ctx, c1h_system, c1_hetero, engine, order, monkeypatch):
    from vfvchem_vfvm3d_b200 import DeviceWaitTimeout, GmresOptions
    (rp, ci, va), b, _ = c1h_system
    if engine == 1:
        monkeypatch.setenv("VFV_ILU_CHAIN", "1")  # the graph engine waits only inside the single-launch sweeps
    p = _pattern(gpu_ctx, c1h_system)
    kw = dict(tol=1e-12, restart=30, max_outer=500, precond=2, ilu_order=order, engine=engine)
    with pytest.raises(DeviceWaitTimeout):
        p.solve(b, c1_hetero.T0, GmresOptions(wait_limit=1, **kw))
    x, info = p.solve(b, c1_hetero.T0, GmresOptions(**kw))
    assert info.status == 0 and info.relres <= 1e-12
    assert _rel(x, lu_solve(rp, ci, va, b)) <= SOL_RTOL
    # and once more: the recovered state stays consistent over repeated solves
    x2, info2 = p.solve(b, c1_hetero.T0, GmresOptions(**kw))
    assert info2.iters == info.iters and np.array_equal(x, x2)


def test_negative_wait_limit_is_rejected(gpu_ctx, c1h_system, c1_hetero):
    from vfvchem_vfvm3d_b200 import GmresOptions, LinearGmresBadInput
    _, b, _ = c1h_system
    p = _pattern(gpu_ctx, c1h_system)
    with pytest.raises(LinearGmresBadInput):
        p.solve(b, None, GmresOptions(wait_limit=-1, precond=2))


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("order", [0, 1])
def test_chain_and_level_sweeps_agree(gpu_ctx, c1h_system, c1_hetero, precision, order, monkeypatch):
    """The single-launch sweeps sum every row in the order of the per-level kernels: identical
    iterates (VFV_ILU_CHAIN=1 selects the single-launch sweeps for a new solver)."""
    from vfvchem_vfvm3d_b200 import GmresOptions
    _, b, _ = c1h_system
    out = []
    for chain in (True, False):
        if chain:
            monkeypatch.setenv("VFV_ILU_CHAIN", "1")
        else:
            monkeypatch.delenv("VFV_ILU_CHAIN", raising=False)
        p = _pattern(gpu_ctx, c1h_system)  # a new pattern builds new solvers
        out.append(p.solve(b, c1_hetero.T0, GmresOptions(tol=1e-11, restart=30, max_outer=500, precond=2, ilu_order=order,
                                                         precision=precision, inner_rtol=1e-6 if precision else 0.0)))
    monkeypatch.delenv("VFV_ILU_CHAIN", raising=False)
    assert out[0][1].iters == out[1][1].iters
    assert np.array_equal(out[0][0], out[1][0])


def test_ilu_apply_repeats_bit_identically(gpu_ctx, c1h_system, c1_hetero):
    """Many applies in a row give the same bits (the sweeps are deterministic)."""
    import torch
    p = _pattern(gpu_ctx, c1h_system)
    r = torch.tensor(np.random.default_rng(3).standard_normal(c1_hetero.n), device="cuda")
    zs = [torch.empty_like(r) for _ in range(5)]
    torch.cuda.synchronize()
    for z in zs:
        p.ilu0_apply_device(r.data_ptr(), z.data_ptr(), 1)
    for z in zs[1:]:
        assert torch.equal(z, zs[0])


@pytest.fixture(scope="module")
def heat40(lib_built):
    """The 64,000-vertex heterogeneous heat system (natural ordering: several hundred levels)."""
    from tests.conftest import oracle_system
    from vfvchem_vfvm3d_b200.problems import steady_heat
    prob = steady_heat(40, hetero=True)
    return prob, oracle_system(prob)


@pytest.mark.parametrize("which", ["c1", "heat40"])
def test_dataflow_factorisation_matches_levels(gpu_ctx, c1h_system, c1_hetero, heat40, which, monkeypatch):
    """The natural ordering has many narrow levels, so its factor is computed by the dataflow kernel;
    VFV_ILU_FACTOR=levels selects the level-by-level launches. Each row's arithmetic is the same, so
    the factors, and the applies and solves built on them, are bit-identical."""
    import torch
    from vfvchem_vfvm3d_b200 import GmresOptions
    prob, system = (c1_hetero, c1h_system) if which == "c1" else heat40
    _, b, _ = system
    r = torch.tensor(np.random.default_rng(5).standard_normal(prob.n), device="cuda")
    zs, sols = [], []
    for levels in (False, True):
        if levels:
            monkeypatch.setenv("VFV_ILU_FACTOR", "levels")
        else:
            monkeypatch.delenv("VFV_ILU_FACTOR", raising=False)
        p = _pattern(gpu_ctx, system)
        _, lev_ptr = p.ilu0_ordering(1)
        assert len(lev_ptr) - 1 >= 32  # enough levels for the dataflow kernel
        z = torch.empty_like(r)
        p.ilu0_apply_device(r.data_ptr(), z.data_ptr(), 1)
        torch.cuda.synchronize()
        zs.append(z)
        sols.append(p.solve(b, prob.T0, GmresOptions(tol=1e-11, restart=30, max_outer=500, precond=2, ilu_order=1, ilu_sweeps=3,
                                                     precision=1, inner_rtol=1e-6, engine=2)))
    monkeypatch.delenv("VFV_ILU_FACTOR", raising=False)
    assert torch.equal(zs[0], zs[1])
    assert sols[0][1].iters == sols[1][1].iters and np.array_equal(sols[0][0], sols[1][0])


def test_dataflow_factorisation_wait_gives_up_and_recovers(gpu_ctx, heat40, monkeypatch):
    """A one-poll limit makes the dataflow factorisation's waits give up: DeviceWaitTimeout, then the
    same pattern factors and solves correctly with the default limit (new values on every solve, so
    every solve factors again)."""
    from vfvchem_vfvm3d_b200 import DeviceWaitTimeout, GmresOptions
    monkeypatch.delenv("VFV_ILU_FACTOR", raising=False)
    prob, system = heat40
    (rp, ci, va), b, _ = system
    p = _pattern(gpu_ctx, system)
    kw = dict(tol=1e-12, restart=50, max_outer=500, precond=2, ilu_order=1, ilu_sweeps=4, engine=2, precision=1, inner_rtol=1e-6)
    with pytest.raises(DeviceWaitTimeout):
        p.solve(b, prob.T0, GmresOptions(wait_limit=1, **kw))
    x_ref = lu_solve(rp, ci, va, b)
    for _ in range(2):
        p.set_values(va)
        x, info = p.solve(b, prob.T0, GmresOptions(**kw))
        assert info.status == 0 and info.relres <= 1e-12
        assert _rel(x, x_ref) <= SOL_RTOL


def _long_row_system(n=1500, seed=2):
    """A diagonally dominant M-matrix: tridiagonal, plus every 29th row coupled symmetrically to the
    40 rows before it and every 97th to the 30 rows after it. Natural ordering: one level per row (the
    tridiagonal chain); rows with 40 lower entries, and rows whose pivot row has 30 upper entries
    (more than the warp staging holds), take the serial path of the factorisation."""
    rng = np.random.default_rng(seed)
    pairs = {(i, i - 1) for i in range(1, n)}
    for i in range(40, n, 29):
        pairs.update((i, j) for j in range(i - 40, i))
    for i in range(0, n - 30, 97):
        pairs.update((j, i) for j in range(i + 1, i + 31))
    pairs |= {(j, i) for i, j in pairs}
    rows = np.array([p[0] for p in pairs] + list(range(n)))
    cols = np.array([p[1] for p in pairs] + list(range(n)))
    vals = np.concatenate([-rng.uniform(0.1, 1.0, len(pairs)), np.zeros(n)])
    off = np.bincount(rows[: len(pairs)], weights=-vals[: len(pairs)], minlength=n)
    vals[len(pairs):] = off + 1.0
    o = np.lexsort((cols, rows))
    rp = np.zeros(n + 1, np.int64)
    np.add.at(rp, rows + 1, 1)
    return np.cumsum(rp), cols[o].astype(np.int32), vals[o]


def test_dataflow_factorisation_serial_rows(gpu_ctx, monkeypatch):
    """Rows longer than a warp in the dataflow factorisation (lane 0 waits for each pivot row in
    turn): bit-identical to the level-by-level factor and the oracle's ILU(0) to 1e-12."""
    import torch
    import oracle
    from vfvchem_vfvm3d_b200 import Pattern
    rp, ci, va = _long_row_system()
    n = rp.size - 1
    r = torch.tensor(np.random.default_rng(4).standard_normal(n), device="cuda")
    zs = []
    for levels in (False, True):
        if levels:
            monkeypatch.setenv("VFV_ILU_FACTOR", "levels")
        else:
            monkeypatch.delenv("VFV_ILU_FACTOR", raising=False)
        p = Pattern.from_csr(gpu_ctx, rp.astype(np.int32), ci)
        p.set_values(va)
        z = torch.empty_like(r)
        nlev = p.ilu0_apply_device(r.data_ptr(), z.data_ptr(), 1)
        torch.cuda.synchronize()
        assert nlev == n
        zs.append(z)
    monkeypatch.delenv("VFV_ILU_FACTOR", raising=False)
    assert torch.equal(zs[0], zs[1])
    perm, _ = p.ilu0_ordering(1)
    zo = oracle.Ilu0(rp, ci, va, perm).apply(r.cpu().numpy())
    assert _rel(zs[0].cpu().numpy(), zo) <= 1e-12
