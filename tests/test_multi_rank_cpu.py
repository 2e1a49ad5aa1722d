"""The N > 1 path of bench.py on CPU, world size 2 over gloo (no GPU).

The step does not shard (one simulation per GPU, replicas only), so the
multi-rank logic is host-side: the rendezvous, the barrier around the timed
region, the max over ranks of the timings, one JSON line from rank 0, and
the reference arm run by rank 0 alone.
"""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench

    w, r, local, pg = bench.dist_setup()
    assert (w, r, local) == (world, rank, rank) and pg is not None
    bench.barrier(pg)
    # each rank's own time; every rank gets the slowest
    out[rank] = bench.allreduce_max(pg, 1.5 + rank)
    bench.barrier(pg)
    pg.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        assert dict(out) == {0: 2.5, 1: 2.5}


@pytest.mark.timeout(300)
def test_reference_arm_under_torchrun_two_ranks():
    """`bench.py --impl reference` launched as the driver launches N > 1:
    rank 0 runs the CPU reference and prints one line, rank 1 exits 0."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--config", "discs", "--gpus", "2", "--steps", "2", "--warmup", "3"]
    env = dict(os.environ, OMP_NUM_THREADS="1")
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=280)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    # the reference arm times at most --ref-steps (2) steps after --ref-warmup (1)
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["steps"] == 2 and d["warmup"] == 1
    sys.path.insert(0, ROOT)
    import bench

    assert d["config"] == bench.static_config("discs", 2)
    assert d["value"] > 0 and d["cpu_baseline"]["kind"] == "port"
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]
