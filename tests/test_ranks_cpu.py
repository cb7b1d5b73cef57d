"""The multi-rank plumbing of bench.py (one process per GPU, launched by
torch.distributed.run) on the CPU: world size 2 over gloo, 127.0.0.1.

bench.py --gpus N runs N independent replicas of the single-GPU step (the
hot path has no exchange step: no data-path collective).  What crosses ranks
is the timing protocol: a barrier on both sides of the timed region and the
maximum of the per-rank device times, which rank 0 reports.  The reference
arm is run by rank 0 alone; the other ranks exit 0 without work.
"""
import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import json, sys
sys.path.insert(0, {root!r})
import bench
rank, world, local = bench.dist_init(None)
bench.barrier(world)
# each rank's 'device time'; the job's time is the slowest rank's
t = bench.max_over_ranks(1.5 * (rank + 1), world)
bench.barrier(world)
import torch.distributed as dist
print(json.dumps({{"rank": rank, "world": world, "backend": dist.get_backend(), "max": t}}))
dist.destroy_process_group()
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env(rank, world, port):
    env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world),
               MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
    return env


def test_barrier_and_max_over_ranks_world_2():
    port = _free_port()
    code = CHILD.format(root=ROOT)
    procs = [subprocess.Popen([sys.executable, "-c", code], env=_env(r, 2, port),
                              stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)
             for r in range(2)]
    outs = []
    try:
        for p in procs:
            out, err = p.communicate(timeout=120)
            assert p.returncode == 0, err[-2000:]
            outs.append(json.loads(out.strip().splitlines()[-1]))
    finally:
        for p in procs:
            if p.poll() is None:
                p.kill()
    assert sorted(o["rank"] for o in outs) == [0, 1]
    for o in outs:
        assert o["world"] == 2 and o["backend"] == "gloo"
        assert o["max"] == 3.0


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    os.environ.pop("WORLD_SIZE", None)
    rank, world, _ = bench.dist_init(None)
    assert (rank, world) == (int(os.environ.get("RANK", "0")), 1)
    bench.barrier(world)
    assert bench.max_over_ranks(2.5, world) == 2.5


def test_reference_arm_runs_on_rank_0_only():
    env = _env(1, 2, _free_port())
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2"], env=env, capture_output=True, text=True, timeout=120,
                       cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""
