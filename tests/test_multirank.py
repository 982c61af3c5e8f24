"""The N > 1 host path of bench.py on CPU: gloo ranks as the bench's torchrun
launch makes them (one process per rank, 127.0.0.1 rendezvous): the barriers
around the timed region and the max over ranks of the device time. The strips'
own exchanges and sums over gloo are tested in test_strips.py."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench

    w, r, local, pg = bench.dist_setup()
    bench.barrier(pg)
    t = bench.allreduce_max(pg, 1.0 + 2.0 * rank)  # rank 1 is the slower one
    bench.barrier(pg)
    q.put((w, r, local, t))
    pg.destroy_process_group()


def test_max_over_ranks_with_gloo():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[:3] for o in out] == [(2, 0, 0), (2, 1, 1)]
    assert all(o[3] == 3.0 for o in out)  # every rank sees the slowest rank's time


@pytest.mark.timeout(300)
def test_reference_arm_under_torchrun():
    """bench.py --impl reference launched under torchrun with 2 ranks (one process per GPU):
    rank 0 alone runs the CPU reference and prints one JSON line; the other
    rank exits 0 without work."""
    env = dict(os.environ, LBFEM_CPU_BUDGET_S="1", OMP_NUM_THREADS="2")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "2", "--warmup", "1", "--cells", "8", "--degree", "1"]
    res = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=280)
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [ln for ln in res.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, res.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["e2e"]["h2d_bytes_per_step"] == 0
