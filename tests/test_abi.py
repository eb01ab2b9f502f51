"""C ABI surface: the library loads, exports every symbol include/*.h declares, host-only entry
points work without a GPU, and device entry points fail loudly (no CPU fallback)."""
import ctypes as C
import glob
import os
import re

import numpy as np
import pytest

from tests.conftest import ROOT


def _declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(vfv_[a-z0-9_]+)\s*\(", src):
            names.add(m.group(1))
    return names


def test_every_declared_symbol_is_exported(lib_built):
    from vfvchem_vfvm3d_b200 import _lib
    names = _declared_symbols()
    assert len(names) >= 25
    lib = C.CDLL(_lib.LIB_PATH)
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing
    bound = {s[0] for s in _lib.SIGNATURES}
    assert names <= bound, sorted(names - bound)


def test_default_opts_are_the_reference_defaults(lib_built):
    from vfvchem_vfvm3d_b200 import _lib
    o = _lib.GmresOpts()
    _lib.load().vfv_gmres_default_opts(C.byref(o))
    assert (o.tol, o.restart, o.max_outer, o.precond, o.precision) == (1e-6, 50, 200, _lib.PRECOND_JACOBI, _lib.FP64)


def test_host_mesh_entry_points_without_gpu(lib_built):
    from vfvchem_vfvm3d_b200 import Mesh
    m = Mesh.jitter_cube(6, 1, 0.25)
    assert (m.n_pts, m.n_nds) == (64, 152)
    pos, nb, tets = m.export()
    assert pos.shape == (216, 3) and nb.shape == (152,) and tets.shape[1] == 4
    assert set(np.unique(nb)) == set(range(6))
    # x faces own their edges and corners
    assert np.all(pos[64:][nb == 0][:, 0] == 0.0) and np.all(pos[64:][nb == 1][:, 0] == 1.0)
    d = m.dual()
    assert d["nbr_ptr"][-1] == m.n_dir
    m2 = Mesh.from_vertices(pos, m.n_pts, nb)
    assert m2.n_tet == m.n_tet


def test_mesh_rejects_bad_input(lib_built):
    from vfvchem_vfvm3d_b200 import Mesh, VFVChemError
    with pytest.raises(VFVChemError):
        Mesh.jitter_cube(2, 1, 0.25)
    with pytest.raises(VFVChemError):
        Mesh.jitter_cube(5, 1, 0.7)
    pos = np.zeros((4, 3))
    with pytest.raises(VFVChemError):  # coincident vertices
        Mesh.from_vertices(pos, 0, np.zeros(4, np.int32))
    ref = Mesh.jitter_cube(4, 5, 0.25)
    vpos, vbnd, _ = ref.export()
    m = Mesh.from_vertices(vpos, ref.n_pts, vbnd)  # on the 2^-18 lattice, inside the exact range
    assert m.n_tet == ref.n_tet
    bad = vpos.copy()
    bad[3, 1] = np.nan
    with pytest.raises(VFVChemError, match="finite"):
        Mesh.from_vertices(bad, ref.n_pts, vbnd)
    bad[3, 1] = 1e60
    with pytest.raises(VFVChemError, match="finite"):
        Mesh.from_vertices(bad, ref.n_pts, vbnd)


def test_linear_gmres_constructor_checks():
    from vfvchem_vfvm3d_b200 import (LinearGmres, LinearGmresNonPositiveMaxOuter, LinearGmresNonPositiveRestart,
                                     LinearGmresNonPositiveThreads, LinearGmresNonPositiveTolerance)
    with pytest.raises(LinearGmresNonPositiveThreads):
        LinearGmres.new_with_options(0, 1e-6, 50, 200)
    with pytest.raises(LinearGmresNonPositiveTolerance):
        LinearGmres.new_with_options(1, 0.0, 50, 200)
    with pytest.raises(LinearGmresNonPositiveTolerance):
        LinearGmres.new_with_options(1, float("nan"), 50, 200)
    with pytest.raises(LinearGmresNonPositiveRestart):
        LinearGmres.new_with_options(1, 1e-6, 0, 200)
    with pytest.raises(LinearGmresNonPositiveMaxOuter):
        LinearGmres.new_with_options(1, 1e-6, 50, 0)


def test_no_cpu_fallback_without_device(lib_built):
    """Without a usable CUDA device the context cannot be created: nothing silently runs on the CPU."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from vfvchem_vfvm3d_b200 import Context, VFVChemError
    with pytest.raises(VFVChemError):
        Context(0)


_DUAL_DIGEST = """
import hashlib, numpy as np
from vfvchem_vfvm3d_b200 import Mesh
m = Mesh.jitter_cube(14, 5, 0.25)
h = hashlib.sha256()
for k, a in sorted(m.dual().items()):
    h.update(k.encode()); h.update(np.ascontiguousarray(a).tobytes())
print(h.hexdigest())
"""


def test_dual_does_not_depend_on_thread_count(lib_built):
    """The Voronoi dual is built by parallel passes whose sums run in a fixed order (tetrahedron,
    edge, side), so one thread and several give the same bits; so do stored and recomputed face
    pieces (VFV_DUAL_PIECE_STORE_MB=0 forces the recomputation large meshes use)."""
    import subprocess
    import sys
    digests = []
    for threads, store_mb in (("1", None), ("3", None), ("3", "0")):
        env = dict(os.environ, OMP_NUM_THREADS=threads)
        env.pop("VFV_DUAL_PIECE_STORE_MB", None)
        if store_mb is not None:
            env["VFV_DUAL_PIECE_STORE_MB"] = store_mb
        out = subprocess.run([sys.executable, "-c", _DUAL_DIGEST], cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
        assert out.returncode == 0, out.stderr
        digests.append(out.stdout.strip().splitlines()[-1])
    assert digests[0] == digests[1] == digests[2]
