"""The multi-GPU path on the CPU: two gloo ranks (127.0.0.1) check the frame
sharding and the slowest-rank timing of goav1_b200.dist, and bench.py's
reference arm under torchrun with two ranks prints one line from rank 0
while rank 1 exits 0 without work."""

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


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import torch.distributed as td

    from goav1_b200 import dist

    dist.init("gloo", timeout_s=60)
    r, w, _ = dist.env()
    mine = list(dist.shard(5, r))
    every = [None] * w
    td.all_gather_object(every, mine)
    slowest = dist.max_over_ranks(10.0 + r, w)
    dist.barrier(w)
    td.destroy_process_group()
    q.put((r, every, slowest))


def test_two_gloo_ranks_shard_and_take_the_slowest_time():
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, every, slowest in out:
        assert slowest == 11.0
        flat = [i for shard in every for i in shard]
        assert sorted(flat) == list(range(10)) and len(set(flat)) == 10


@pytest.mark.timeout(300)
def test_bench_reference_arm_two_ranks():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(port), "bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1",
           "--warmup", "0", "--frames", "2"]
    p = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=280)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, p.stdout
    rec = json.loads(lines[0])
    assert rec["impl"] == "reference" and rec["n_gpus"] == 2 and rec["value"] > 0
    assert rec["cpu_baseline"]["kind"] == "port" and rec["e2e"]["h2d_bytes_per_step"] == 0
