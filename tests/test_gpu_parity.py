"""GPU parity against the CPU oracle, through the C ABI (run with -m gpu on a B200).

Bars (from the task's parity criteria): CSR pattern bit-exact; FP64 coefficients and b within
1e-12 relative (the assembly kernels are compiled without FMA contraction and reproduce the
oracle's push-order sums, so they are in fact bit-identical); solutions within 1e-8 relative
2-norm error of the FP64 LU solution.
"""
import numpy as np
import pytest

import oracle
from oracle import ordering
from oracle.lu import lu_solve
from tests.conftest import oracle_system

pytestmark = pytest.mark.gpu

COEF_RTOL = 1e-12
SOL_RTOL = 1e-8


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def _gpu_heat(ctx, prob, T=None):
    from vfvchem_vfvm3d_b200 import SteadyHeatGpu
    h = SteadyHeatGpu(prob.mesh, prob.bnd_kind, ctx=ctx)
    b = h.assemble(prob.k, prob.q, prob.s, prob.T0 if T is None else T, prob.bc_val)
    return h, b


@pytest.mark.parametrize("which", ["c1", "c1_hetero"])
def test_gradient_matches_oracle(gpu_ctx, which, request):
    prob = request.getfixturevalue(which)
    h, _ = _gpu_heat(gpu_ctx, prob)
    d = prob.mesh.dual()
    rng = np.random.default_rng(3)
    f = rng.standard_normal(prob.n)
    g = h.grad(f)
    go = oracle.grad(d, f)
    assert np.array_equal(g, go) or np.max(np.abs(g - go)) <= COEF_RTOL * np.max(np.abs(go))


@pytest.mark.parametrize("which", ["c1", "c1_hetero"])
def test_heat_assembly_matches_oracle(gpu_ctx, which, request):
    prob = request.getfixturevalue(which)
    (rp, ci, va), b_o, _ = oracle_system(prob)
    h, b = _gpu_heat(gpu_ctx, prob)
    grp, gci, gva = h.pattern.export()
    assert np.array_equal(grp.astype(np.int64), rp)
    assert np.array_equal(gci, ci)
    assert np.max(np.abs(gva - va)) <= COEF_RTOL * np.max(np.abs(va))
    assert np.max(np.abs(b - b_o)) <= COEF_RTOL * max(np.max(np.abs(b_o)), 1e-300)


def test_heat_assembly_with_nonzero_unknown(gpu_ctx, c1_hetero):
    """The production operator's lagged skew term reads grad(T): assemble at a non-trivial T."""
    prob = c1_hetero
    pos, _, _ = prob.mesh.export()
    T = np.sin(3 * pos[:, 0]) + pos[:, 1] * pos[:, 2]
    (rp, ci, va), b_o, _ = oracle_system(prob, T)
    h, b = _gpu_heat(gpu_ctx, prob, T)
    _, _, gva = h.pattern.export()
    assert np.max(np.abs(gva - va)) <= COEF_RTOL * np.max(np.abs(va))
    assert np.max(np.abs(b - b_o)) <= COEF_RTOL * np.max(np.abs(b_o))


def test_assembly_is_deterministic(gpu_ctx, c1_hetero):
    h, b1 = _gpu_heat(gpu_ctx, c1_hetero)
    _, _, v1 = h.pattern.export()
    b2 = h.assemble(c1_hetero.k, c1_hetero.q, c1_hetero.s, c1_hetero.T0, c1_hetero.bc_val)
    _, _, v2 = h.pattern.export()
    assert np.array_equal(v1, v2) and np.array_equal(b1, b2)


def test_triplet_pattern_and_values(gpu_ctx, c1h_system, c1_hetero):
    """update_sparse + build_matrix from the oracle's push-order triplets."""
    from vfvchem_vfvm3d_b200 import Pattern
    (rp, ci, va), _, (r, c, v) = c1h_system
    p = Pattern.from_triplets(gpu_ctx, c1_hetero.n, r, c)
    assert p.ntrip == r.size and p.nnz == ci.size
    p.values_from_triplets(v)
    grp, gci, gva = p.export()
    assert np.array_equal(grp.astype(np.int64), rp) and np.array_equal(gci, ci)
    assert np.array_equal(gva, va)  # same push-order summation


def test_triplet_index_out_of_range_is_reported(gpu_ctx, c1h_system, c1_hetero):
    """A row or column >= n is rejected before any device work, naming the first bad triplet
    (the keys are built in parallel, the reported index is still the smallest)."""
    from vfvchem_vfvm3d_b200 import Pattern, VFVChemError
    _, _, (r, c, _) = c1h_system
    r = r.astype(np.uint64).copy()
    c = c.astype(np.uint64).copy()
    last = r.size - 5
    r[last] = c1_hetero.n
    c[r.size // 2] = c1_hetero.n + 7
    with pytest.raises(VFVChemError, match=rf"out of range at {r.size // 2}$"):
        Pattern.from_triplets(gpu_ctx, c1_hetero.n, r, c)


def test_spmv_matches_oracle(gpu_ctx, c1h_system, c1_hetero):
    import torch
    from vfvchem_vfvm3d_b200 import Pattern
    (rp, ci, va), _, _ = c1h_system
    p = Pattern.from_csr(gpu_ctx, rp.astype(np.int32), ci)
    p.set_values(va)
    x = np.random.default_rng(5).standard_normal(c1_hetero.n)
    xd = torch.tensor(x, device="cuda")
    yd = torch.empty_like(xd)
    torch.cuda.synchronize()
    p.spmv_device(xd.data_ptr(), yd.data_ptr())
    gpu_ctx.synchronize()
    y = yd.cpu().numpy()
    yo = oracle.spmv(rp, ci, va, x)
    assert np.max(np.abs(y - yo)) <= 1e-13 * np.max(np.abs(yo))
    xf = xd.float()
    yf = torch.empty_like(xf)
    torch.cuda.synchronize()
    p.spmv_device_f32(xf.data_ptr(), yf.data_ptr())
    gpu_ctx.synchronize()
    assert np.max(np.abs(yf.cpu().numpy() - yo)) <= 1e-5 * np.max(np.abs(yo))


@pytest.mark.parametrize("lanes", [2, 4, 8, 16, 32])
def test_spmv_lanes_variants_match_oracle(gpu_ctx, c1h_system, c1_hetero, lanes):
    """Every lanes-per-row variant the autotuner may pick gives the oracle's product, and a solve
    through it still converges to the LU solution."""
    import torch
    from vfvchem_vfvm3d_b200 import GmresOptions, Pattern, VFVChemError
    from vfvchem_vfvm3d_b200 import _lib as L
    (rp, ci, va), b, _ = c1h_system
    xlu = lu_solve(rp, ci, va, b)
    p = Pattern.from_csr(gpu_ctx, rp.astype(np.int32), ci)
    p.set_values(va)
    p.set_spmv_lanes(lanes, lanes)
    x = np.random.default_rng(6).standard_normal(c1_hetero.n)
    xd = torch.tensor(x, device="cuda")
    yd = torch.empty_like(xd)
    torch.cuda.synchronize()
    p.spmv_device(xd.data_ptr(), yd.data_ptr())
    gpu_ctx.synchronize()
    yo = oracle.spmv(rp, ci, va, x)
    assert np.max(np.abs(yd.cpu().numpy() - yo)) <= 1e-13 * np.max(np.abs(yo))
    xs, info = p.solve(b, opts=GmresOptions(tol=1e-12, restart=40, max_outer=100, precond=L.PRECOND_ILU0, precision=L.MIXED))
    assert info.status == 0
    assert np.max(np.abs(xs - xlu)) <= 1e-8 * np.max(np.abs(xlu))
    with pytest.raises(VFVChemError):
        p.set_spmv_lanes(3, 4)


def test_autotune_picks_a_variant(gpu_ctx, c1h_system):
    from vfvchem_vfvm3d_b200 import Pattern
    (rp, ci, va), b, _ = c1h_system
    p = Pattern.from_csr(gpu_ctx, rp.astype(np.int32), ci)
    p.set_values(va)
    a, f = p.autotune()
    assert a in (2, 4, 8, 16, 32) and f in (2, 4, 8, 16, 32)
    x, info = p.solve(b)
    assert info.status == 0


def _check_ordering(rp, ci, perm, lev_ptr):
    """The permutation groups rows into levels no two coupled rows share, and every coupling
    points from a later level to an earlier one in the lower factor (true of any ordering)."""
    n = rp.size - 1
    assert np.array_equal(np.sort(perm), np.arange(n))
    level = np.empty(n, np.int64)
    for l in range(lev_ptr.size - 1):
        level[perm[lev_ptr[l]:lev_ptr[l + 1]]] = l
    rows = np.repeat(np.arange(n), np.diff(rp))
    off = rows != ci
    assert np.all(level[rows[off]] != level[ci[off]])


@pytest.mark.parametrize("order", [0, 1])
def test_ilu0_apply_matches_oracle(gpu_ctx, c1h_system, c1_hetero, order):
    """ILU(0) on the product's ordering, restated by the oracle on the same permutation."""
    import torch
    from vfvchem_vfvm3d_b200 import Pattern
    (rp, ci, va), _, _ = c1h_system
    p = Pattern.from_csr(gpu_ctx, rp.astype(np.int32), ci)
    p.set_values(va)
    r = np.random.default_rng(9).standard_normal(c1_hetero.n)
    rd = torch.tensor(r, device="cuda")
    zd = torch.empty_like(rd)
    torch.cuda.synchronize()
    nlev = p.ilu0_apply_device(rd.data_ptr(), zd.data_ptr(), order)
    perm, lev_ptr = p.ilu0_ordering(order)
    assert lev_ptr.size == nlev + 1
    _check_ordering(rp, ci, perm, lev_ptr)
    if order == 1:  # the natural ordering is fully determined: level = longest lower chain
        perm_o, lev_o = ordering.natural(rp, ci)
        assert np.array_equal(perm, perm_o) and nlev == int(lev_o.max()) + 1
    else:  # at most as many colours as plain greedy colouring
        _, col = ordering.multicolor(rp, ci)
        assert nlev <= int(col.max()) + 1
    zo = oracle.Ilu0(rp, ci, va, perm).apply(r)
    assert _rel(zd.cpu().numpy(), zo) <= 1e-12


def test_ilu0_apply_f32_matches_oracle(gpu_ctx, c1h_system, c1_hetero):
    """The float sweeps of the mixed-precision solver: same levels as the double apply, the
    oracle's ILU(0) on the same permutation to float accuracy, identical bits on a repeat call,
    and a work vector that aliases r or z is rejected."""
    import torch
    from vfvchem_vfvm3d_b200 import Pattern, VFVChemError
    (rp, ci, va), _, _ = c1h_system
    p = Pattern.from_csr(gpu_ctx, rp.astype(np.int32), ci)
    p.set_values(va)
    r = np.random.default_rng(11).standard_normal(c1_hetero.n)
    rd = torch.tensor(r, device="cuda", dtype=torch.float32)
    td = torch.empty_like(rd)
    zd = torch.empty_like(rd)
    z2 = torch.empty_like(rd)
    torch.cuda.synchronize()
    nlev = p.ilu0_apply_device_f32(rd.data_ptr(), td.data_ptr(), zd.data_ptr())
    assert p.ilu0_apply_device_f32(rd.data_ptr(), td.data_ptr(), z2.data_ptr()) == nlev
    gpu_ctx.synchronize()
    perm, lev_ptr = p.ilu0_ordering(0)
    assert lev_ptr.size == nlev + 1
    zo = oracle.Ilu0(rp, ci, va, perm).apply(r.astype(np.float32).astype(np.float64))
    assert _rel(zd.cpu().numpy().astype(np.float64), zo) <= 1e-4
    assert torch.equal(zd, z2)
    with pytest.raises(VFVChemError):
        p.ilu0_apply_device_f32(rd.data_ptr(), rd.data_ptr(), zd.data_ptr())


@pytest.mark.parametrize("sweeps", [1, 3])
@pytest.mark.parametrize("order", [0, 1])
def test_ilu0_sweep_apply_matches_oracle(gpu_ctx, c1h_system, c1_hetero, order, sweeps):
    """Jacobi sweeps of the ILU(0) factors (double and float), against the oracle's restatement on
    the same factor; the natural ordering runs in A's numbering, the multicolour one permuted.
    Repeat calls give identical bits; r and z may alias."""
    import torch
    from vfvchem_vfvm3d_b200 import Pattern
    (rp, ci, va), _, _ = c1h_system
    p = Pattern.from_csr(gpu_ctx, rp.astype(np.int32), ci)
    p.set_values(va)
    r = np.random.default_rng(13).standard_normal(c1_hetero.n)
    perm, _ = p.ilu0_ordering(order) if order == 0 else (np.arange(c1_hetero.n, dtype=np.int32), None)
    ilu = oracle.Ilu0(rp, ci, va, perm)
    zo = ilu.sweep_apply(r, sweeps)
    rd = torch.tensor(r, device="cuda")
    zd, z2 = torch.empty_like(rd), torch.empty_like(rd)
    p.ilu0_sweep_apply_device(rd.data_ptr(), zd.data_ptr(), sweeps, order)
    p.ilu0_sweep_apply_device(rd.data_ptr(), z2.data_ptr(), sweeps, order)
    gpu_ctx.synchronize()
    assert p.ilu0_sweep_layout(order) == 2  # the 2,744-row pattern fits 16-bit column offsets
    assert _rel(zd.cpu().numpy(), zo) <= 1e-12
    assert torch.equal(zd, z2)
    za = rd.clone()
    p.ilu0_sweep_apply_device(za.data_ptr(), za.data_ptr(), sweeps, order)
    gpu_ctx.synchronize()
    assert torch.equal(za, zd)
    r32 = r.astype(np.float32)
    rf = torch.tensor(r32, device="cuda")
    zf = torch.empty_like(rf)
    p.ilu0_sweep_apply_device(rf.data_ptr(), zf.data_ptr(), sweeps, order, f32=True)
    gpu_ctx.synchronize()
    assert _rel(zf.cpu().numpy().astype(np.float64), ilu.sweep_apply(r32.astype(np.float64), sweeps)) <= 1e-5
    zh = torch.empty_like(rf)  # the row-scaled half-precision values
    p.ilu0_sweep_apply_device(rf.data_ptr(), zh.data_ptr(), sweeps, order, half=True)
    gpu_ctx.synchronize()
    assert _rel(zh.cpu().numpy().astype(np.float64), ilu.sweep_apply(r32.astype(np.float64), sweeps, half=True)) <= 1e-5


@pytest.fixture(scope="module")
def heat40_system(lib_built):
    """The 64,000-vertex heterogeneous heat system (boundary vertices numbered after the interior,
    so A's own bandwidth exceeds 16-bit column offsets)."""
    from vfvchem_vfvm3d_b200.problems import steady_heat
    prob = steady_heat(40, hetero=True)
    return prob, oracle_system(prob)


@pytest.mark.parametrize("order", [0, 1])
def test_ilu0_sweeps_wide_pattern_match_oracle(gpu_ctx, heat40_system, order):
    """A factor whose bandwidth is too wide for 16-bit column offsets is swept with 32-bit columns:
    same iterates as the oracle's sweeps (double 1e-12, float 1e-5)."""
    import torch
    from vfvchem_vfvm3d_b200 import Pattern
    prob, ((rp, ci, va), _, _) = heat40_system
    p = Pattern.from_csr(gpu_ctx, rp.astype(np.int32), ci)
    p.set_values(va)
    perm = p.ilu0_ordering(0)[0] if order == 0 else np.arange(prob.n, dtype=np.int32)
    ilu = oracle.Ilu0(rp, ci, va, perm)
    r = np.random.default_rng(21).standard_normal(prob.n)
    rd = torch.tensor(r, device="cuda")
    zd = torch.empty_like(rd)
    p.ilu0_sweep_apply_device(rd.data_ptr(), zd.data_ptr(), 2, order)
    gpu_ctx.synchronize()
    assert p.ilu0_sweep_layout(order) == 4
    assert _rel(zd.cpu().numpy(), ilu.sweep_apply(r, 2)) <= 1e-12
    rf = rd.float()
    zf = torch.empty_like(rf)
    p.ilu0_sweep_apply_device(rf.data_ptr(), zf.data_ptr(), 2, order, f32=True)
    gpu_ctx.synchronize()
    assert _rel(zf.cpu().numpy().astype(np.float64), ilu.sweep_apply(rf.cpu().numpy().astype(np.float64), 2)) <= 1e-5


@pytest.mark.parametrize("upper", [0, 5])
@pytest.mark.parametrize("engine", [1, 2])
@pytest.mark.parametrize("order", [0, 1])
@pytest.mark.parametrize("precision", [0, 1])
def test_gmres_ilu_sweeps_matches_lu(gpu_ctx, c1h_system, c1_hetero, precision, order, engine, upper):
    """GMRES preconditioned by ILU(0) with 3 Jacobi sweeps of the lower factor and 3 (or 5) of the
    upper one: the same bars against LU; the persistent engine refuses the sweeps."""
    from vfvchem_vfvm3d_b200 import GmresOptions, Pattern, VFVChemError
    (rp, ci, va), b, _ = c1h_system
    p = Pattern.from_csr(gpu_ctx, rp.astype(np.int32), ci)
    p.set_values(va)
    xl = lu_solve(rp, ci, va, b)
    opts = GmresOptions(tol=1e-12, restart=30, max_outer=2000, precond=2, precision=precision, ilu_order=order, ilu_sweeps=3,
                        ilu_sweeps_upper=upper, inner_rtol=1e-6 if precision == 1 else 0.0, engine=engine)
    x, info = p.solve(b, c1_hetero.T0, opts)
    assert info.status == 0 and info.relres <= 1e-12
    assert _rel(x, xl) <= SOL_RTOL
    with pytest.raises(VFVChemError):
        p.solve(b, None, GmresOptions(precond=2, ilu_sweeps=3, engine=0))
    with pytest.raises(VFVChemError):
        p.solve(b, None, GmresOptions(precond=2, ilu_sweeps=17))
    with pytest.raises(VFVChemError):
        p.solve(b, None, GmresOptions(precond=2, ilu_sweeps=3, ilu_sweeps_upper=-1))


@pytest.mark.parametrize("engine", [0, 1])
@pytest.mark.parametrize("precond", [0, 1, 2])
@pytest.mark.parametrize("precision", [0, 1])
def test_gmres_matches_lu(gpu_ctx, c1h_system, c1_hetero, precond, precision, engine):
    from vfvchem_vfvm3d_b200 import GmresOptions, Pattern
    (rp, ci, va), b, _ = c1h_system
    p = Pattern.from_csr(gpu_ctx, rp.astype(np.int32), ci)
    p.set_values(va)
    xl = lu_solve(rp, ci, va, b)
    opts = GmresOptions(tol=1e-12, restart=30, max_outer=2000, precond=precond, precision=precision,
                        inner_rtol=1e-6 if precision == 1 else 0.0, engine=engine)
    x, info = p.solve(b, c1_hetero.T0, opts)
    assert info.status == 0 and info.relres <= 1e-12
    assert _rel(x, xl) <= SOL_RTOL


@pytest.mark.parametrize("engine", [1, 2])
@pytest.mark.parametrize("order", [0, 1])
def test_gmres_ilu_sweeps_half_matches_lu(gpu_ctx, c1h_system, c1_hetero, order, engine):
    """The mixed solver with the swept factors in row-scaled half precision: the same bars against LU
    (the FP64 refinement keeps the answer exact); refused outside that combination."""
    from vfvchem_vfvm3d_b200 import GmresOptions, Pattern, VFVChemError
    (rp, ci, va), b, _ = c1h_system
    p = Pattern.from_csr(gpu_ctx, rp.astype(np.int32), ci)
    p.set_values(va)
    xl = lu_solve(rp, ci, va, b)
    opts = GmresOptions(tol=1e-12, restart=30, max_outer=2000, precond=2, precision=1, ilu_order=order, ilu_sweeps=3, ilu_sweep_half=1,
                        inner_rtol=1e-6, engine=engine)
    x, info = p.solve(b, c1_hetero.T0, opts)
    assert info.status == 0 and info.relres <= 1e-12
    assert _rel(x, xl) <= SOL_RTOL
    with pytest.raises(VFVChemError):
        p.solve(b, None, GmresOptions(precond=2, ilu_sweeps=3, ilu_sweep_half=1))  # FP64
    with pytest.raises(VFVChemError):
        p.solve(b, None, GmresOptions(precond=2, precision=1, ilu_sweep_half=1))  # exact ILU(0)


@pytest.mark.parametrize("ortho", [1, 2])
@pytest.mark.parametrize("engine", [1, 2])
@pytest.mark.parametrize("precision", [0, 1])
def test_gram_schmidt_variants_match_lu(gpu_ctx, c1h_system, c1_hetero, precision, engine, ortho):
    """Classical Gram-Schmidt with a second pass only when needed (DGKS test) and with one pass: the
    same bars against LU, and within a few iterations of two passes; the persistent engine refuses
    them."""
    from vfvchem_vfvm3d_b200 import GmresOptions, Pattern, VFVChemError
    (rp, ci, va), b, _ = c1h_system
    p = Pattern.from_csr(gpu_ctx, rp.astype(np.int32), ci)
    p.set_values(va)
    xl = lu_solve(rp, ci, va, b)
    kw = dict(tol=1e-12, restart=30, max_outer=2000, precond=2, precision=precision, engine=engine,
              inner_rtol=1e-6 if precision == 1 else 0.0)
    x, info = p.solve(b, c1_hetero.T0, GmresOptions(ortho=ortho, **kw))
    assert info.status == 0 and info.relres <= 1e-12
    assert _rel(x, xl) <= SOL_RTOL
    _, ref = p.solve(b, c1_hetero.T0, GmresOptions(**kw))
    assert abs(info.iters - ref.iters) <= max(3, ref.iters // 10)
    with pytest.raises(VFVChemError):
        p.solve(b, None, GmresOptions(precond=2, ortho=ortho, engine=0))
    with pytest.raises(VFVChemError):
        p.solve(b, None, GmresOptions(precond=2, ortho=3))


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("order", [0, 1])
def test_overlap_engine_matches_lu(gpu_ctx, c1h_system, c1_hetero, precision, order):
    """Flexible GMRES with the ILU(0) sweeps overlapped with the orthogonalisation: same bars,
    and within a few iterations of the plain right-preconditioned GMRES."""
    from vfvchem_vfvm3d_b200 import GmresOptions, Pattern, VFVChemError
    (rp, ci, va), b, _ = c1h_system
    p = Pattern.from_csr(gpu_ctx, rp.astype(np.int32), ci)
    p.set_values(va)
    xl = lu_solve(rp, ci, va, b)
    kw = dict(tol=1e-12, restart=30, max_outer=2000, precond=2, precision=precision, ilu_order=order,
              inner_rtol=1e-6 if precision == 1 else 0.0)
    x, info = p.solve(b, c1_hetero.T0, GmresOptions(engine=2, **kw))
    assert info.status == 0 and info.relres <= 1e-12
    assert _rel(x, xl) <= SOL_RTOL
    _, ref = p.solve(b, c1_hetero.T0, GmresOptions(engine=1, **kw))
    assert abs(info.iters - ref.iters) <= max(3, ref.iters // 10)
    with pytest.raises(VFVChemError):
        p.solve(b, None, GmresOptions(engine=2, precond=1))


@pytest.mark.parametrize("engine", [1, 2])
def test_conditional_and_straight_cycle_graphs_agree(gpu_ctx, c1h_system, c1_hetero, engine, monkeypatch):
    """The cycle graph with IF nodes over groups of steps and the straight graph (VFV_STRAIGHT_GRAPH)
    run the same kernels in the same order: identical iterates."""
    from vfvchem_vfvm3d_b200 import GmresOptions, Pattern
    (rp, ci, va), b, _ = c1h_system
    out = []
    for straight in (False, True):
        if straight:
            monkeypatch.setenv("VFV_STRAIGHT_GRAPH", "1")
        else:
            monkeypatch.delenv("VFV_STRAIGHT_GRAPH", raising=False)
        p = Pattern.from_csr(gpu_ctx, rp.astype(np.int32), ci)  # a new pattern builds its own graph
        p.set_values(va)
        out.append(p.solve(b, c1_hetero.T0, GmresOptions(tol=1e-11, restart=30, max_outer=500, precond=2, engine=engine)))
    monkeypatch.delenv("VFV_STRAIGHT_GRAPH", raising=False)
    assert out[0][1].iters == out[1][1].iters
    assert np.array_equal(out[0][0], out[1][0])


def test_engines_agree(gpu_ctx, c1h_system, c1_hetero):
    """The persistent cycle kernel and the graph of per-phase kernels run the same arithmetic."""
    from vfvchem_vfvm3d_b200 import GmresOptions, Pattern
    (rp, ci, va), b, _ = c1h_system
    p = Pattern.from_csr(gpu_ctx, rp.astype(np.int32), ci)
    p.set_values(va)
    res = []
    for engine in (0, 1):
        x, info = p.solve(b, c1_hetero.T0, GmresOptions(tol=1e-11, restart=20, max_outer=500, precond=2, engine=engine))
        res.append((x, info))
    assert res[0][1].iters == res[1][1].iters
    assert _rel(res[0][0], res[1][0]) <= 1e-12


def test_uniform_heat_gmres30_jacobi(gpu_ctx, c1, c1_system):
    """Uniform heat slab (n=20): GMRES(30) + Jacobi to 1e-10 relative residual against the FP64 LU solution."""
    from vfvchem_vfvm3d_b200 import GmresOptions, Pattern
    (rp, ci, va), b, _ = c1_system
    p = Pattern.from_csr(gpu_ctx, rp.astype(np.int32), ci)
    p.set_values(va)
    x, info = p.solve(b, c1.T0, GmresOptions(tol=1e-10, restart=30, max_outer=500))
    xo, ok, its_o, _ = oracle.gmres(rp, ci, va, b, c1.T0, tol=1e-10, restart=30, max_outer=500, precond=1)
    xl = lu_solve(rp, ci, va, b)
    assert info.relres <= 1e-10
    assert _rel(x, xl) <= 1e-7 and _rel(x, xo) <= 1e-7
    # same algorithm (right-preconditioned Jacobi GMRES(30)): iteration counts agree closely
    assert abs(info.iters - its_o) <= max(3, 0.1 * its_o)


def test_gmres_errors(gpu_ctx, c1h_system, c1_hetero):
    from vfvchem_vfvm3d_b200 import GmresOptions, LinearGmresDidNotConverge, LinearGmresNonFinite, Pattern
    (rp, ci, va), b, _ = c1h_system
    p = Pattern.from_csr(gpu_ctx, rp.astype(np.int32), ci)
    p.set_values(va)
    with pytest.raises(LinearGmresDidNotConverge):
        p.solve(b, None, GmresOptions(tol=1e-14, restart=2, max_outer=1))
    bad = b.copy()
    bad[3] = np.nan
    with pytest.raises(LinearGmresNonFinite):
        p.solve(bad, None, GmresOptions())
    x, info = p.solve(np.zeros_like(b), np.ones_like(b), GmresOptions())
    assert info.status == 0 and np.all(x == 0.0)
    # the context stays usable after the failures
    x, info = p.solve(b, None, GmresOptions(tol=1e-10))
    assert info.relres <= 1e-10


def test_linear_gmres_drop_in(gpu_ctx, c1, c1_system):
    """LinearBase call sequence of SteadyBase::solve (steady_base.rs:65-78) on the GPU."""
    from vfvchem_vfvm3d_b200 import LinearGmres
    (rp, ci, va), b, (r, c, v) = c1_system
    lin = LinearGmres.new_with_options(1, 1e-10, 50, 200, ctx=gpu_ctx)
    lin.update_sparse((r, c, v), c1.n)
    a_mat = lin.build_matrix((r, c, v))
    x = lin.solve_matrix(a_mat, b, c1.T0, c1.n)
    pos, _, _ = c1.mesh.export()
    assert np.max(np.abs(x - pos[:, 0])) < 1e-7  # linear-field exactness through the GPU path
    key = lin._key
    lin.update_sparse((r, c, v), c1.n)  # unchanged pattern is recognised
    assert lin._key == key


def test_larger_mesh_properties(gpu_ctx):
    """n=40 (64,000 vertices): GPU-assembled system solved on the GPU; residual and linear exactness."""
    from vfvchem_vfvm3d_b200 import GmresOptions, SteadyHeatGpu
    from vfvchem_vfvm3d_b200.problems import steady_heat
    prob = steady_heat(40)
    h = SteadyHeatGpu(prob.mesh, prob.bnd_kind, ctx=gpu_ctx)
    b = h.assemble(prob.k, prob.q, prob.s, prob.T0, prob.bc_val)
    x, info = h.pattern.solve(b, prob.T0, GmresOptions(tol=1e-12, restart=50, max_outer=400, precond=2))
    pos, _, _ = prob.mesh.export()
    assert np.max(np.abs(x - pos[:, 0])) < 1e-8
    rp, ci, va = h.pattern.export()
    assert np.linalg.norm(oracle.spmv(rp.astype(np.int64), ci, va, x) - b) <= 1e-10 * np.linalg.norm(b)


def test_host_solve_into_given_array(gpu_ctx, c1h_system, c1_hetero):
    """Pattern.solve(..., out=) writes x into the caller's array (pinned memory here) with the same
    bits as a new array; a wrong array is refused."""
    import torch
    from vfvchem_vfvm3d_b200 import GmresOptions, Pattern
    (rp, ci, va), b, _ = c1h_system
    p = Pattern.from_csr(gpu_ctx, rp.astype(np.int32), ci)
    p.set_values(va)
    o = GmresOptions(tol=1e-12, restart=30, max_outer=500, precond=2, precision=1, inner_rtol=1e-6)
    x, _ = p.solve(b, c1_hetero.T0, o)
    buf = torch.empty(c1_hetero.n, dtype=torch.float64).pin_memory().numpy()
    x2, _ = p.solve(b, c1_hetero.T0, o, out=buf)
    assert x2 is buf and np.array_equal(x, buf)
    with pytest.raises(ValueError):
        p.solve(b, c1_hetero.T0, o, out=np.empty(c1_hetero.n, np.float32))
