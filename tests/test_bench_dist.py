"""The N>1 plumbing of bench.py on the CPU, world size 2 over gloo.

`bench.py --gpus N` runs one independent replica per rank (the step does not
shard); the ranks share only a barrier before each timed region and the max
over ranks of its device time.  Here two CPU processes run those helpers, and
a torchrun launch of the reference arm checks that rank 0 alone prints its
line while the other rank exits 0 without work."""
import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


CHILD = r"""
import sys
sys.path.insert(0, {root!r})
import bench
world, rank, local, dist = bench.dist_setup(None)
assert world == 2 and dist is not None, (world, dist)
assert dist.get_backend() == "gloo"
bench.barrier(dist)
v = bench.reduce_max(dist, 1.0 + 2.5 * rank)
assert v == 3.5, v
bench.barrier(dist)
dist.destroy_process_group()
print("rank", rank, "ok", v)
"""


def test_replica_helpers_two_ranks():
    port = free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2",
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", CHILD.format(root=ROOT)], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        try:
            o, e = p.communicate(timeout=240)
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            raise
        outs.append((p.returncode, o, e))
    for rank, (rc, o, e) in enumerate(outs):
        assert rc == 0, e[-2000:]
        assert f"rank {rank} ok 3.5" in o


def test_reference_arm_prints_on_rank0_only():
    port = free_port()
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--grid", "16", "--steps", "1", "--warmup", "3"]
    r = subprocess.run(cmd, env=env, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = lines[0]
    assert line["impl"] == "reference"
    if "unavailable" not in line:
        assert line["n_gpus"] == 2 and line["value"] > 0
        assert line["cpu_baseline"]["kind"] == "reference"
