"""Bounded device waits and the single-launch ILU(0) sweeps (run with -m gpu on a B200).

The persistent engine's grid barriers and the single-launch ILU(0) sweeps (VFV_ILU_CHAIN=1) wait
on other CTAs through memory; every such wait has a poll limit (vfv_gmres_opts.wait_limit). A
limit of one poll makes the waits give up in practice (a barrier needs every CTA to arrive; a
natural-order ILU(0) level needs the level before it): the solve must then end with status 5
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
