"""The Voronoi dual built on the device (csrc/kernels/dual.cu) against the host dual
(csrc/host/mesh.cpp), which the CPU suite pins to the numpy and C restatements of
Tetrahedron::update_tet (src/base/geom_tet.rs:122-293): every array equal bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KEYS = ["nbr_ptr", "nbr_idx", "dist", "area", "norm", "skew", "grad_wgt", "cvol", "cskew", "bnd_ptr", "bnd_j", "bnd_k", "bnd_area",
        "bnd_norm", "bnd_wgt"]


def _same(a, b):
    for k in KEYS:
        assert a[k].shape == b[k].shape, k
        assert np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize("n", [6, 13, 30])
def test_device_dual_equals_host_dual(gpu_ctx, n):
    from vfvchem_vfvm3d_b200 import Mesh
    m = Mesh.jitter_cube(n, 42 + n, 0.25)
    host = {k: v.copy() for k, v in m.dual().items()}
    m.build_dual_device(gpu_ctx)
    _same(m.dual(), host)


def test_device_dual_batch_equals_host_batch(gpu_ctx):
    from vfvchem_vfvm3d_b200 import Mesh
    ns, seeds = [5, 11, 8, 14], [7, 8, 9, 10]
    host = Mesh.jitter_cubes(ns, seeds)
    dev = Mesh.jitter_cubes_device_dual(gpu_ctx, ns, seeds)
    for a, b in zip(dev, host):
        _same(a.dual(), b.dual())
