"""The multi-rank plumbing of `bench.py --gpus N` (cpu-renderer_b200/replicas.py), run as two
gloo ranks on the CPU: per-rank sample streams, the max over ranks of each rank's time, the
whole-job rate, a rank that never arrives ending the others' collective with an error, and
the reference arm's ranks other than 0 leaving without work."""
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


def _env(rank, world, port):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, os.path.join(ROOT, "cpu-renderer_b200"))


def _rates(rank, world, port, out):
    _env(rank, world, port)
    from replicas import Replicas
    r = Replicas("gloo", timeout_s=30)
    r.barrier()
    result = {
        "rank": r.rank, "world": r.world, "seed": r.seed(42),
        "slowest": r.max_over_ranks(1.5 + rank),       # rank 1 is the slower one
        "rate": r.whole_job_rate(1_000_000, 1.0 + 3 * rank),
    }
    r.close()
    out.put(result)


def test_two_ranks_max_time_and_whole_job_rate():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rates, args=(k, 2, port, q)) for k in range(2)]
    for p in procs:
        p.start()
    results = sorted((q.get(timeout=120) for _ in procs), key=lambda d: d["rank"])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [d["seed"] for d in results] == [42, 43]          # each replica its own streams
    assert all(d["world"] == 2 for d in results)
    assert all(d["slowest"] == 2.5 for d in results)         # every rank sees the same max
    # 2 ranks x 1 M units over the slowest rank's 4 s = 0.5 M units/s
    assert all(d["rate"] == pytest.approx(0.5) for d in results)


def _absent_peer(rank, world, port, out):
    _env(rank, world, port)
    from replicas import Replicas
    r = Replicas("gloo", timeout_s=5)
    if rank == 1:
        os._exit(0)  # leaves between steps, without joining the next collective
    try:
        r.barrier()
        out.put("returned")
    except Exception as e:  # the group's timeout or the lost connection ends the wait
        out.put("error: " + type(e).__name__)


def test_a_rank_that_never_arrives_ends_the_collective_with_an_error():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_absent_peer, args=(k, 2, port, q)) for k in range(2)]
    for p in procs:
        p.start()
    outcome = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    assert outcome.startswith("error"), outcome


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1", MASTER_ADDR="127.0.0.1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       capture_output=True, text=True, timeout=120, env=env)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
