"""Adjoint gradient of the steady heat solution on the GPU through the C ABI: vfv_heat_adjoint against the oracle's
independently built adjoint and against central finite differences (step 1e-6) of the oracle's
forward model on 64 random unit directions in (log k, q)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def adj_case(lib_built):
    from vfvchem_vfvm3d_b200.problems import steady_heat
    prob = steady_heat(12, hetero=True)
    rng = np.random.default_rng(5)
    sensors = rng.choice(prob.n, size=100, replace=False)
    target = rng.uniform(0.0, 1.0, sensors.size)
    return prob, sensors, target


def _gpu_gradient(ctx, prob, sensors, target):
    from vfvchem_vfvm3d_b200 import GmresOptions, SteadyHeatGpu
    from vfvchem_vfvm3d_b200 import _lib as L
    heat = SteadyHeatGpu(prob.mesh, prob.bnd_kind, ctx=ctx)
    b = heat.assemble(prob.k, prob.q, prob.s, prob.T0, prob.bc_val)
    opts = GmresOptions(tol=1e-14, restart=50, max_outer=4000, precond=L.PRECOND_ILU0)
    T, _ = heat.pattern.solve(b, prob.T0, opts)
    g = np.zeros(prob.n)
    g[sensors] = T[sensors] - target
    lam, dk, dq, info = heat.adjoint(T, g, opts)
    return T, lam, dk, dq, info


def test_adjoint_matches_oracle_adjoint(gpu_ctx, adj_case):
    from oracle import adjoint
    prob, sensors, target = adj_case
    T, lam, dk, dq, info = _gpu_gradient(gpu_ctx, prob, sensors, target)
    J, ok, oq, olam = adjoint.gradient(prob, np.log(prob.k), prob.q, sensors, target)
    assert np.linalg.norm(lam - olam) <= 1e-9 * np.linalg.norm(olam)
    assert np.linalg.norm(dk - ok) <= 1e-9 * np.linalg.norm(ok)
    assert np.linalg.norm(dq - oq) <= 1e-9 * np.linalg.norm(oq)


def test_adjoint_matches_finite_differences_64_directions(gpu_ctx, adj_case):
    from oracle import adjoint
    prob, sensors, target = adj_case
    _, _, dk, dq, _ = _gpu_gradient(gpu_ctx, prob, sensors, target)
    rng = np.random.default_rng(64)
    logk = np.log(prob.k)
    gnorm = np.sqrt(dk @ dk + dq @ dq)
    errs, nerrs = [], []
    for _ in range(64):
        ek = rng.standard_normal(prob.n)
        eq = rng.standard_normal(prob.n)
        nrm = np.sqrt(ek @ ek + eq @ eq)
        ek, eq = ek / nrm, eq / nrm
        fd = adjoint.fd_directional(prob, logk, prob.q, sensors, target, ek, eq, h=1e-6)
        ad = dk @ ek + dq @ eq
        errs.append(abs(fd - ad) / abs(ad))
        nerrs.append(abs(fd - ad) / gnorm)
        if len(errs) <= 8:  # a larger step separates the adjoint's error from the difference quotient's round-off
            fd4 = adjoint.fd_directional(prob, logk, prob.q, sensors, target, ek, eq, h=1e-4)
            assert abs(fd4 - ad) / abs(ad) < 1e-6
    # At h = 1e-6 the difference quotient carries ~1e-8 |grad J| of round-off from re-assembling
    # A(p +- h delta): relative to the directional derivative that is ~1e-6 typically (more for
    # directions nearly orthogonal to the gradient), relative to |grad J| it is ~1e-8.
    assert np.median(errs) < 1e-6
    assert max(nerrs) < 1e-7
