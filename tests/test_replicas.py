"""Multi-process host logic of the replica runs (no GPU): one process per
rank over gloo, as bench.py runs under torchrun with one independent box per
GPU and no data-path collective."""
import json
import os
import socket
import subprocess
import sys

import pytest

torch = pytest.importorskip("torch")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(WORLD_SIZE=str(world), RANK=str(rank), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    w, r, _ = bench.dist_init()
    bench.barrier(w)
    mx = bench.allmax(w, 1.5 + r)          # per-rank device times -> the max over ranks
    sm = bench.allsum(w, 1000 * (r + 1))   # per-rank particle-steps -> the job total
    out.put((r, w, mx, sm))
    import torch.distributed as dist
    dist.destroy_process_group()


def test_replica_reductions_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    assert [r for r, *_ in res] == [0, 1]
    for _, w, mx, sm in res:
        assert w == 2 and mx == 2.5 and sm == 3000


def test_reference_arm_two_ranks():
    """bench.py --impl reference under torchrun: rank 0 alone runs the CPU
    path and prints one JSON line; the other rank exits 0 without work."""
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes", "1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0", "--config", "c1"]
    p = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600,
                       env=dict(os.environ, OMP_NUM_THREADS="2"))
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["e2e"]["h2d_bytes_per_step"] == 0
