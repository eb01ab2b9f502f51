"""Batched transient advection-diffusion on the GPU through the C ABI, against the
oracle's restatement of the same operator composition and SuperLU time stepping."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import oracle

pytestmark = pytest.mark.gpu

DT = 1e-2


@pytest.fixture(scope="module")
def batch(lib_built):
    from vfvchem_vfvm3d_b200 import Mesh
    from vfvchem_vfvm3d_b200.problems import transport_fields
    meshes = Mesh.jitter_cubes([5, 8, 6], [11, 12, 13])
    vel, c0 = transport_fields(meshes)
    return meshes, vel, c0


def _oracle_blocks(meshes, vel, D):
    out, off = [], 0
    for m in meshes:
        d = m.dual()
        _, nb, _ = m.export()
        node_bnd = np.full(m.n_tot, -1, np.int32)
        node_bnd[m.n_pts:] = nb
        r, c, v = oracle.transport_triplets(d, m.n_pts, node_bnd, D, vel[:, off:off + m.n_tot], DT)
        out.append(oracle.csr_from_triplets(m.n_tot, r, c, v))
        off += m.n_tot
    return out


def test_transport_assembly_matches_oracle(gpu_ctx, batch):
    from vfvchem_vfvm3d_b200 import TransientTransportGpu
    meshes, vel, _ = batch
    tr = TransientTransportGpu(meshes, DT, ctx=gpu_ctx)
    tr.assemble(1e-3, vel)
    rp, ci, va = tr.pattern.export()
    for i, (orp, oci, ova) in enumerate(_oracle_blocks(meshes, vel, 1e-3)):
        r0, r1 = tr.row_ptr[i], tr.row_ptr[i + 1]
        brp = rp[r0:r1 + 1].astype(np.int64) - rp[r0]
        assert np.array_equal(brp, orp)
        assert np.array_equal(ci[rp[r0]:rp[r1]] - r0, oci)
        assert np.max(np.abs(va[rp[r0]:rp[r1]] - ova)) <= 1e-12 * np.max(np.abs(ova))


@pytest.mark.parametrize("sweeps", [0, 3])
def test_transport_steps_match_lu(gpu_ctx, batch, sweeps):
    """Per-mesh batched GMRES with exact ILU(0) or with Jacobi sweeps of the natural-order factors
    (one swept factor for the whole block-diagonal batch) against LU time stepping."""
    from vfvchem_vfvm3d_b200 import GmresOptions, TransientTransportGpu
    from vfvchem_vfvm3d_b200 import _lib as L
    meshes, vel, c0 = batch
    tr = TransientTransportGpu(meshes, DT, ctx=gpu_ctx)
    tr.assemble(1e-3, vel)
    opts = GmresOptions(tol=1e-12, restart=30, max_outer=500, precond=L.PRECOND_ILU0, precision=L.MIXED, inner_rtol=1e-6,
                        ilu_order=L.ILU_NATURAL if sweeps else L.ILU_MULTICOLOR, ilu_sweeps=sweeps)
    c_gpu, its = tr.run(c0, 5, opts)
    assert np.all(its > 0)
    off = 0
    for m, (orp, oci, ova) in zip(meshes, _oracle_blocks(meshes, vel, 1e-3)):
        A = sp.csr_matrix((ova, oci, orp), shape=(m.n_tot, m.n_tot)).tocsc()
        lu = spla.splu(A)
        c = c0[off:off + m.n_tot].copy()
        vol = m.dual()["cvol"]
        for _ in range(5):
            c = lu.solve(-c * vol / DT)
        g = c_gpu[off:off + m.n_tot]
        assert np.linalg.norm(g - c) <= 1e-9 * np.linalg.norm(c)
        off += m.n_tot


def test_uniform_field_is_preserved(gpu_ctx, batch):
    """Non-conservative advection keeps a uniform field uniform (opscl_dom_adv.rs: 'uniform c is preserved')."""
    from vfvchem_vfvm3d_b200 import GmresOptions, TransientTransportGpu
    from vfvchem_vfvm3d_b200 import _lib as L
    meshes, vel, _ = batch
    tr = TransientTransportGpu(meshes, DT, ctx=gpu_ctx)
    tr.assemble(1e-3, vel)
    c, _ = tr.run(np.full(tr.n, 2.5), 3, GmresOptions(tol=1e-12, restart=30, max_outer=500, precond=L.PRECOND_ILU0))
    assert np.max(np.abs(c - 2.5)) < 1e-9


def _oracle_J(meshes, vel, c0, target, D, nsteps):
    J, off = 0.0, 0
    for m, (orp, oci, ova) in zip(meshes, _oracle_blocks(meshes, vel, D)):
        lu = spla.splu(sp.csr_matrix((ova, oci, orp), shape=(m.n_tot, m.n_tot)).tocsc())
        c = c0[off:off + m.n_tot].copy()
        vol = m.dual()["cvol"]
        for _ in range(nsteps):
            c = lu.solve(-c * vol / DT)
        r = c - target[off:off + m.n_tot]
        J += 0.5 * float(r @ r)
        off += m.n_tot
    return J


def test_transient_adjoint_dJdD_matches_finite_differences(gpu_ctx, batch):
    """dJ/dD with checkpoints every 10 steps over 25 steps (a partial last segment) against central
    differences of the oracle's LU time stepping."""
    from vfvchem_vfvm3d_b200 import GmresOptions, TransientTransportGpu
    from vfvchem_vfvm3d_b200 import _lib as L
    meshes, vel, c0 = batch
    D = 1e-3
    target = 0.9 * c0 + 0.05
    tr = TransientTransportGpu(meshes, DT, ctx=gpu_ctx)
    tr.assemble(D, vel)
    opts = GmresOptions(tol=1e-13, restart=30, max_outer=2000, precond=L.PRECOND_ILU0)
    J, g = tr.adjoint_D(c0, 25, target, every=10, opts=opts)
    Jo = _oracle_J(meshes, vel, c0, target, D, 25)
    assert abs(J - Jo) <= 1e-10 * abs(Jo)
    h = 1e-7
    fd = (_oracle_J(meshes, vel, c0, target, D + h, 25) - _oracle_J(meshes, vel, c0, target, D - h, 25)) / (2 * h)
    assert abs(fd - g) <= 1e-6 * abs(fd)
    # the checkpoint interval changes only the schedule, not the result
    _, g2 = tr.adjoint_D(c0, 25, target, every=7, opts=opts)
    assert abs(g2 - g) <= 1e-9 * abs(g)


@pytest.mark.parametrize("precision", [0, 1])
def test_mesh_in_a_batch_iterates_as_if_alone(gpu_ctx, precision):
    """Every mesh of a batch has its own Krylov recurrence: a mesh solved inside a 16-mesh batch
    gives the iterate of the same mesh solved alone (to 1e-12; the arithmetic is the same), and
    its Arnoldi steps are its own."""
    from vfvchem_vfvm3d_b200 import GmresOptions, Mesh, TransientTransportGpu
    from vfvchem_vfvm3d_b200 import _lib as L
    from vfvchem_vfvm3d_b200.problems import transport_fields
    ns = [5, 9, 6, 7, 5, 8, 6, 10, 5, 7, 9, 6, 8, 5, 7, 6]
    meshes = Mesh.jitter_cubes(ns, [101 + i for i in range(16)])
    vel, c0 = transport_fields(meshes)
    opts = GmresOptions(tol=1e-10, restart=20, max_outer=200, precond=L.PRECOND_ILU0, precision=precision,
                        inner_rtol=1e-6 if precision else 0.0)
    tr = TransientTransportGpu(meshes, DT, ctx=gpu_ctx)
    tr.assemble(1e-3, vel)
    c_b, _ = tr.run(c0, 3, opts)
    steps_b = tr.mesh_steps()
    assert steps_b.shape == (16,) and np.all(steps_b > 0)
    for i in (0, 7, 13):
        r0, r1 = tr.row_ptr[i], tr.row_ptr[i + 1]
        alone = TransientTransportGpu([meshes[i]], DT, ctx=gpu_ctx)
        alone.assemble(1e-3, vel[:, r0:r1])
        c_a, its_a = alone.run(c0[r0:r1], 3, opts)
        assert np.linalg.norm(c_b[r0:r1] - c_a) <= 1e-12 * np.linalg.norm(c_a)
        assert steps_b[i] == alone.mesh_steps()[0] == int(np.sum(its_a))
