"""The N>1 path of bench.py on CPU: world_size-2 `gloo` ranks.

Multi-GPU here is replicas only (each rank solves its own copy; no data-path
collective), so what the ranks share is the timing protocol: a barrier before and after
the timed region and the maximum of the ranks' times. These tests run that protocol
(bench.Dist) between two CPU processes, and the reference arm under torch.distributed.run
with two ranks (rank 0 alone measures and prints one line; the other exits 0)."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update({"WORLD_SIZE": str(world), "RANK": str(rank), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "CUDA_VISIBLE_DEVICES": ""})
    sys.path.insert(0, ROOT)
    import bench

    d = bench.Dist(world)
    d.barrier()
    m = d.max(10.0 + rank)  # each rank's own "time"
    d.barrier()
    d.close()
    out.put((rank, d.world, m))


def test_two_gloo_ranks_agree_on_the_max_time():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=5) for _ in range(2))
    assert got == [(0, 2, 11.0), (1, 2, 11.0)]


def test_reference_arm_under_two_ranks_prints_one_line():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()), "bench.py", "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "1", "--scale", "0.0005"]
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="", PYTHONPATH=ROOT)
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = lines[0]
    assert line["impl"] == "reference" and line["value"] > 0 and line["n_gpus"] == 2
    assert line["cpu_baseline"]["kind"] == "port" and line["e2e"]["value"] == line["value"]


def test_reference_arm_never_loads_the_library():
    """The reference arm builds its LP with the oracle's copy of the generators and times the
    oracle: the CUDA library is never mapped into its process."""
    code = ("import runpy, sys; sys.argv = ['bench.py', '--impl', 'reference', '--scale', '0.0005', '--steps', '1', "
            "'--warmup', '1']; runpy.run_path('bench.py', run_name='__main__'); "
            "m = open('/proc/self/maps').read(); print('MAPS', 'libsaddlepoint_b200' in m, 'libsp_oracle' in m)")
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="", PYTHONPATH=ROOT)
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    maps = [l for l in r.stdout.splitlines() if l.startswith("MAPS")]
    assert maps == ["MAPS False True"], r.stdout
    line = json.loads([l for l in r.stdout.splitlines() if l.startswith("{")][0])
    assert line["config"]["workload"] == "single large LP, power-law columns" and "parallelism" not in line["config"]
