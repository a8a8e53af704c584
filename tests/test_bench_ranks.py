"""bench.py's multi-rank plumbing on the CPU (gloo, two ranks).

With N GPUs the bench runs one process per GPU: every rank times its own
replica and the reported time is the maximum over ranks; the reference arm
runs on rank 0 alone.  These tests start two real processes on 127.0.0.1.
"""
import os
import socket
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

WORKER = """
import os, sys
sys.path.insert(0, {root!r})
import torch.distributed as dist
import bench
dist.init_process_group("gloo", init_method="env://")
rank, world = dist.get_rank(), dist.get_world_size()
v = bench.max_over_ranks(1.5 + 10.0 * rank, world)
dist.barrier()
dist.destroy_process_group()
print("RESULT", rank, v, flush=True)
"""


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env(rank: int, world: int, port: int) -> dict:
    env = dict(os.environ)
    env.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
               MASTER_PORT=str(port))
    return env


def test_max_over_ranks_two_gloo_ranks():
    port = _free_port()
    code = WORKER.format(root=ROOT)
    procs = [subprocess.Popen([sys.executable, "-c", code], env=_env(r, 2, port), stdout=subprocess.PIPE,
                              stderr=subprocess.PIPE, text=True) for r in range(2)]
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=120)
        assert p.returncode == 0, err
        outs.append(out)
    got = sorted(line.split()[1:] for o in outs for line in o.splitlines() if line.startswith("RESULT"))
    assert got == [["0", "11.5"], ["1", "11.5"]]


def test_max_over_ranks_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.25, 1) == 3.25


def test_reference_arm_runs_on_rank_zero_only():
    # a non-zero rank of the reference arm exits at once, printing nothing
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0"], env=_env(1, 2, _free_port()), capture_output=True,
                       text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
