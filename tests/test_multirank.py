"""The N > 1 host logic of bench.py with two `gloo` ranks on the CPU: the
barrier, the max-over-ranks step time, weak-scaling rows (each rank its own
seeded polynomials) and the whole-job value; and the reference arm under a
launcher, where only rank 0 works and prints."""
import json
import os
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank_main(rank, ws, port, q):
    os.environ.update(WORLD_SIZE=str(ws), RANK=str(rank), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist
    w, r, _ = bench.dist_init(None, backend="gloo")
    bench.barrier(w)
    step_ms = 100.0 + 50.0 * r  # rank 1 is the slow one
    total = bench.max_over_ranks(step_ms, w)
    seeds = bench.rank_rows_seed(r)
    value = bench.job_value(w, 262144, 1, total)
    q.put((r, total, seeds, value))
    dist.destroy_process_group()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [x[1] for x in res] == [150.0, 150.0]          # every rank sees the slowest time
    assert res[0][2] != res[1][2]                           # distinct rows per rank
    assert res[0][3] == pytest.approx(2 * 262144 / 0.150)  # whole-job proofs/s


def test_reference_arm_only_rank0_prints():
    env = dict(os.environ, WORLD_SIZE="2", RANK="1", LOCAL_RANK="1")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                         env=env, capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.strip() == ""
    env = dict(os.environ, WORLD_SIZE="1", RANK="0", LOCAL_RANK="0")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--n", "1024",
                          "--cpu-rows", "2", "--steps", "1", "--warmup", "0"],
                         env=env, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["cpu_baseline"]["kind"] == "port"
    assert line["e2e"]["h2d_bytes_per_step"] == 0
