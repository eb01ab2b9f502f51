import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def lib_built():
    """libvfvgpu.so and the oracle library, built in-tree."""
    from vfvchem_vfvm3d_b200 import _lib
    import oracle
    if not os.path.exists(_lib.LIB_PATH):
        import subprocess
        subprocess.run(["make", "-s", "-C", os.path.dirname(_lib.LIB_PATH)], check=True)
    oracle.lib()
    return _lib.load()


@pytest.fixture(scope="session")
def c1(lib_built):
    """Uniform heat slab: n=20 cube (8,000 vertices), k=1, q=s=0, T=0/1 on x=0/1, zero flux elsewhere."""
    from vfvchem_vfvm3d_b200.problems import steady_heat
    return steady_heat(20)


@pytest.fixture(scope="session")
def c1_hetero(lib_built):
    """n=14 cube with log-normal k, uniform q, a production term and an outward flux on z=1."""
    from vfvchem_vfvm3d_b200.problems import steady_heat
    return steady_heat(14, hetero=True, flux_top=0.3, prod=-0.5)


def oracle_system(prob, T=None):
    """Oracle CSR (rp, ci, va), b and triplets for a HeatProblem."""
    import oracle
    d = prob.mesh.dual()
    T = prob.T0 if T is None else T
    r, c, v, b = oracle.heat_triplets(d, prob.mesh.n_pts, prob.node_bnd, prob.bnd_order, prob.bnd_kind, prob.k, prob.q, prob.s, T,
                                      prob.bc_val)
    rp, ci, va = oracle.csr_from_triplets(prob.n, r, c, v)
    return (rp, ci, va), b, (r, c, v)


@pytest.fixture(scope="session")
def c1_system(c1):
    return oracle_system(c1)


@pytest.fixture(scope="session")
def c1h_system(c1_hetero):
    return oracle_system(c1_hetero)


@pytest.fixture(scope="session")
def gpu_ctx(lib_built):
    from vfvchem_vfvm3d_b200 import Context
    return Context(0)
