"""The multi-process path on CPU: two gloo ranks (no GPU involved)."""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    from vfvchem_vfvm3d_b200 import replicas
    R = replicas.init_from_env(backend="gloo", timeout_s=60)
    m = replicas.max_over_ranks(R, [1.5 + rank, 10.0 - rank])
    replicas.finalize(R)
    out.put((rank, m))


def test_max_over_ranks_gloo_world2():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    got = dict(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got[0] == got[1] == [2.5, 10.0]


def test_single_process_needs_no_group():
    from vfvchem_vfvm3d_b200 import replicas
    R = replicas.Ranks()
    assert not R.active
    assert replicas.max_over_ranks(R, [3.0]) == [3.0]


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_shard_meshes_is_a_balanced_partition(world):
    from vfvchem_vfvm3d_b200 import replicas
    rng = np.random.default_rng(4)
    sizes = np.exp(rng.uniform(np.log(2000), np.log(50000), 256)).astype(np.int64)
    parts = [replicas.shard_meshes(sizes, r, world) for r in range(world)]
    allidx = np.concatenate(parts)
    assert np.array_equal(np.sort(allidx), np.arange(sizes.size))
    loads = np.array([sizes[p].sum() for p in parts])
    assert loads.max() - loads.min() <= sizes.max()


def test_reference_arm_under_torchrun_two_ranks(lib_built):
    """bench.py --impl reference launched under two-rank torchrun, with gloo: rank 0 prints one
    JSON line, rank 1 exits without work, both exit 0."""
    env = dict(os.environ, VFV_DIST_BACKEND="gloo", OMP_NUM_THREADS="2")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr", "127.0.0.1",
           "--master-port", str(_free_port()), os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1",
           "--warmup", "1", "--grid", "8"]
    p = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    rec = json.loads(lines[0])
    assert rec["impl"] == "reference" and rec["n_gpus"] == 2 and rec["value"] > 0
    assert rec["e2e"]["h2d_bytes_per_step"] == 0
