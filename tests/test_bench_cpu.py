"""Host logic of bench.py without a GPU: the max-over-ranks timing of a
multi-replica run (two gloo ranks), the reference arm's rank handling, and
the argument contract."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, q):
    import torch.distributed as D
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    D.init_process_group("gloo", rank=rank, world_size=world)
    sys.path.insert(0, ROOT)
    import bench
    got = bench.max_over_ranks(1.5 + rank * 2.0, "cpu")
    D.barrier()
    D.destroy_process_group()
    q.put((rank, got))


def test_max_over_ranks_two_gloo_ranks():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29000 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == {0: 3.5, 1: 3.5}


def _run_bench(args, env_extra):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + args,
                          capture_output=True, text=True, env=env, timeout=600)


def test_reference_arm_other_ranks_print_nothing():
    r = _run_bench(["--impl", "reference", "--steps", "1", "--warmup", "3"],
                   {"RANK": "1", "WORLD_SIZE": "2"})
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


def test_reference_arm_rank0_line():
    r = _run_bench(["--impl", "reference", "--workload", "scan_u32", "--steps", "1",
                    "--warmup", "3"], {"RANK": "0", "WORLD_SIZE": "1"})
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] == 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["warmup"] >= 3


def test_reference_arm_serving_unavailable():
    r = _run_bench(["--impl", "reference", "--workload", "serving"], {"RANK": "0"})
    assert r.returncode == 0
    assert "unavailable" in json.loads(r.stdout.strip().splitlines()[-1])
