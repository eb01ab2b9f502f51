"""Committed golden vectors (tests/golden/golden_small.npz, made by tests/golden/make_golden.py).

CPU: the oracle and the mesh generator still reproduce them (patterns and values exactly, LU
solutions to 1e-12). GPU: the device assembly and solvers reproduce them through the C ABI
within the parity bars (coefficients 1e-12 relative, solutions 1e-8 relative)."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "golden_small.npz")


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(GOLD))


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def test_oracle_reproduces_golden(gold, lib_built):
    sys.path.insert(0, os.path.join(HERE, "golden"))
    import make_golden
    new = make_golden.build()
    assert set(new) == set(gold)
    for k, v in new.items():
        if k in ("heat_x", "flow_x1"):  # LU solutions: round-off of the sparse factorisation
            assert _rel(v, gold[k]) <= 1e-12, k
        else:
            assert v.dtype == gold[k].dtype and np.array_equal(v, gold[k]), k


@pytest.mark.gpu
def test_gpu_heat_matches_golden(gold, gpu_ctx):
    from vfvchem_vfvm3d_b200 import GmresOptions, SteadyHeatGpu
    from vfvchem_vfvm3d_b200 import _lib as L
    from vfvchem_vfvm3d_b200.problems import steady_heat
    prob = steady_heat(6, hetero=True, flux_top=0.3, prod=-0.5)
    pos, _, _ = prob.mesh.export()
    assert np.array_equal(pos, gold["heat_pos"])
    h = SteadyHeatGpu(prob.mesh, prob.bnd_kind, ctx=gpu_ctx)
    b = h.assemble(prob.k, prob.q, prob.s, prob.T0, prob.bc_val)
    rp, ci, va = h.pattern.export()
    assert np.array_equal(rp.astype(np.int64), gold["heat_rp"]) and np.array_equal(ci, gold["heat_ci"])
    assert np.max(np.abs(va - gold["heat_va"])) <= 1e-12 * np.max(np.abs(gold["heat_va"]))
    assert np.max(np.abs(b - gold["heat_b"])) <= 1e-12 * np.max(np.abs(gold["heat_b"]))
    x, info = h.pattern.solve(b, opts=GmresOptions(tol=1e-13, restart=50, max_outer=200, precond=L.PRECOND_ILU0, precision=L.MIXED))
    assert _rel(x, gold["heat_x"]) <= 1e-8


@pytest.mark.gpu
def test_gpu_transport_matches_golden(gold, gpu_ctx):
    from vfvchem_vfvm3d_b200 import Mesh, TransientTransportGpu
    from vfvchem_vfvm3d_b200.problems import transport_fields
    m = Mesh.jitter_cubes([5], [11])
    vel, _ = transport_fields(m)
    tr = TransientTransportGpu(m, 1e-2, ctx=gpu_ctx)
    tr.assemble(1e-3, vel)
    rp, ci, va = tr.pattern.export()
    assert np.array_equal(rp.astype(np.int64), gold["trans_rp"]) and np.array_equal(ci, gold["trans_ci"])
    assert np.max(np.abs(va - gold["trans_va"])) <= 1e-12 * np.max(np.abs(gold["trans_va"]))


@pytest.mark.gpu
def test_gpu_flow_matches_golden(gold, gpu_ctx):
    from vfvchem_vfvm3d_b200 import SteadyFlowGpu
    from vfvchem_vfvm3d_b200.flow import flow_options
    from vfvchem_vfvm3d_b200.problems import lid_cavity
    prob = lid_cavity(5)
    fl = SteadyFlowGpu(prob, ctx=gpu_ctx)
    b = fl.assemble(prob.initial_state())
    rp, ci, va = fl.pattern.export()
    assert np.array_equal(rp.astype(np.int64), gold["flow_rp"]) and np.array_equal(ci, gold["flow_ci"])
    assert np.max(np.abs(va - gold["flow_va"])) <= 1e-12 * np.max(np.abs(gold["flow_va"]))
    assert np.max(np.abs(b - gold["flow_b"])) <= 1e-12 * np.max(np.abs(gold["flow_b"]))
    r = fl.picard(max_iter=1, tol=1e-300, damp=0.8, opts=flow_options(tol=1e-13, max_outer=400), raise_on_error=False)
    assert r.iterations == 1
    assert _rel(r.x, gold["flow_x1"]) <= 1e-8
