"""The multi-GPU plumbing of bench.py on CPU: two gloo ranks. The path shards
with no data-path collective (every rank traces its own rays); the ranks only
meet at the barriers around the timed region and in the max over ranks of the
step time, which is what the job's rate is computed from."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist
    import bench
    r, w, local = bench.dist_env()
    assert (r, w, local) == (rank, world, rank)
    on = bench.init_dist(w, local)
    assert on and dist.get_backend() == "gloo"
    bench.barrier(on)
    ms = 3.0 + rank  # this rank's step time
    worst = bench.max_over_ranks(ms, on)
    # the job rate: every rank's rays over the slowest rank's time
    rate = 4_194_304 * w / (worst * 1e-3) / 1e6
    out.put((rank, worst, rate))
    dist.destroy_process_group()


def test_two_rank_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=5) for _ in range(2))
    assert [x[1] for x in res] == [4.0, 4.0]
    assert res[0][2] == pytest.approx(4_194_304 * 2 / 4e-3 / 1e6)


def test_reference_arm_nonzero_ranks_exit_quietly():
    import subprocess
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "1"], env=env, capture_output=True,
                       text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""
