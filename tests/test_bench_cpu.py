"""bench.py pieces that run without a GPU: the reference (CPU) arm's JSON line and
the multi-rank aggregation, the latter over gloo with two ranks."""
import json
import os
import subprocess
import sys

import pytest

import _libs

sys.path.insert(0, _libs.REPO)
import bench  # noqa: E402


def test_reference_arm_prints_contract_line():
    r = subprocess.run([sys.executable, os.path.join(_libs.REPO, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1", "--cpu-sample", "48"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e", "impl"):
        assert k in line, k
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "port"


def test_rank_seeds_are_disjoint():
    seen = set()
    for r in range(8):
        s = set(bench.rank_seeds(r))
        assert not (s & seen)
        seen |= s


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    rate, ms = bench.job_rate(1000000, 100.0 * (rank + 1), dist, "cpu")
    q.put((rank, rate, ms))
    dist.destroy_process_group()


def test_job_rate_takes_slowest_rank_over_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29511 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
    for rank, rate, ms in res:
        assert ms == pytest.approx(200.0)
        assert rate == pytest.approx(2 * 1000000 / 0.2 / 1e6)
