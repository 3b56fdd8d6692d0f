"""The multi-rank host logic of bench.py on CPU: gloo ranks, world size 2."""
import json
import os
import subprocess
import sys

import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = 2.0 + rank                                   # rank 1 is the slower one
        bench.dist_barrier(world)
        m = bench.dist_max(ms, world, "cpu")
        out[rank] = (m, bench.job_rate(world, 1000, m))
        bench.dist_barrier(world)
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_job_rate_with_gloo():
    world = 2
    out = mp.Manager().dict()
    mp.start_processes(_rank, args=(world, 29517, out), nprocs=world, start_method="spawn")
    assert out[0] == out[1]
    m, rate = out[0]
    assert m == 3.0
    assert abs(rate - 2 * 1000 / 3.0e-3 / 1e9) < 1e-15


def test_reference_arm_prints_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--n", "8", "--steps", "1", "--warmup", "0",
                        ], cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == ""
    env = dict(os.environ, RANK="0", WORLD_SIZE="1", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--n", "8", "--steps", "1", "--warmup", "0",
                        ], cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["cpu_baseline"]["kind"] == "port"
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["unit"] == "GElem/s"
