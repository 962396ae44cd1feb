"""Multi-rank host logic on CPU: world_size-2 `gloo` process groups and a 2-process torchrun.

What runs across GPUs is sharding, not a data-path collective: an ensemble is split over ranks by
greedy LPT (`lbm_b200.shard.lpt_assign`) and every timing is the max over ranks
(`lbm_b200.shard.max_over_ranks`).  These tests exercise both with real process groups on the host.
"""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "lbm-arrayfire_b200"))
sys.path.insert(0, str(ROOT))

from lbm_b200.shard import lpt_assign, rank_loads  # noqa: E402


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_lpt_assign_covers_disjointly_and_balances():
    rng = np.random.default_rng(0)
    costs = rng.integers(1, 1000, size=64).astype(float)
    for n in (1, 2, 3, 8):
        parts = lpt_assign(costs, n)
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(len(costs)))
        loads = rank_loads(costs, parts)
        lower = max(costs.sum() / n, costs.max())
        assert max(loads) <= 4.0 / 3.0 * lower + 1e-9  # Graham's LPT bound
        assert parts == lpt_assign(costs, n)  # deterministic
    with pytest.raises(ValueError):
        lpt_assign(costs, 0)


def test_lpt_assign_more_ranks_than_members():
    parts = lpt_assign([5.0, 3.0], 4)
    assert sorted(len(p) for p in parts) == [0, 0, 1, 1]


def _ranks_body(rank, world, port, out_dir):
    import torch.distributed as dist

    import lbm_b200 as lb
    from bench import ensemble_members
    from lbm_b200.shard import max_over_ranks, sum_over_ranks

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t_max = max_over_ranks(1.5 + rank)
        t_sum = sum_over_ranks(1.5 + rank)
        # the config-5 ensemble, sharded as bench.py shards it (descriptors and masks only: host code)
        members = ensemble_members(lb, lb.F16S)
        costs = [2 * d.q * 2 * d.cells for d, _, _ in members]
        parts = lpt_assign(costs, world)
        shares = [None] * world
        dist.all_gather_object(shares, parts[rank])
        (Path(out_dir) / f"rank{rank}.json").write_text(json.dumps(
            {"max": t_max, "sum": t_sum, "shares": shares, "costs": costs, "n": len(members)}))
    finally:
        dist.destroy_process_group()


def test_gloo_two_ranks_max_over_ranks_and_ensemble_shards(tmp_path):
    world = 2
    mp.start_processes(_ranks_body, args=(world, free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    res = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in range(world)]
    for r in res:
        assert r["max"] == 2.5 and r["sum"] == 4.0
        assert r["shares"] == res[0]["shares"]  # every rank agrees on the split
    shares = res[0]["shares"]
    flat = sorted(k for s in shares for k in s)
    assert flat == list(range(res[0]["n"])) and res[0]["n"] == 64
    costs = res[0]["costs"]
    loads = [sum(costs[k] for k in s) for s in shares]
    assert max(loads) <= 4.0 / 3.0 * max(sum(costs) / world, max(costs))


def test_reference_arm_under_torchrun_prints_one_line_from_rank_zero():
    env = dict(os.environ)
    env.pop("CUDA_VISIBLE_DEVICES", None)
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes", "1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()),
           str(ROOT / "bench.py"), "--impl", "reference", "--workload", "d2q9_lid_128",
           "--steps", "3", "--warmup", "0", "--ref-seconds", "2", "--gpus", "2"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=240, env=env, cwd=str(ROOT))
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    rec = json.loads(lines[0])
    assert rec["impl"] == "reference" and rec["n_gpus"] == 2 and rec["value"] > 0
    assert rec["e2e"]["h2d_bytes_per_step"] == 0 and rec["cpu_baseline"]["kind"] == "port"


_REF_ARM_PROBE = r"""
import json, sys
sys.argv = ["bench.py", "--impl", "reference", "--workload", WORKLOAD, "--steps", "2", "--warmup", "0",
            "--ref-seconds", "1"]
sys.path.insert(0, ROOT)
import bench
bench.main()
maps = open("/proc/self/maps").read()
print(json.dumps({"engine_loaded": "liblbm_b200" in maps, "oracle_loaded": "liblbm_oracle" in maps,
                  "engine_module": "lbm_b200" in sys.modules, "tests_module": "helpers" in sys.modules}))
"""


@pytest.mark.parametrize("workload", ["d2q9_lid_128", "d3q27_mrt_gs_lid_256", "ensemble_config5"])
def test_reference_arm_loads_only_the_oracle(workload):
    code = f"WORKLOAD = {workload!r}\nROOT = {str(ROOT)!r}\n" + _REF_ARM_PROBE
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300, cwd=str(ROOT))
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [json.loads(ln) for ln in out.stdout.splitlines() if ln.startswith("{")]
    rec, probe = lines[0], lines[-1]
    assert rec["impl"] == "reference" and rec["value"] > 0
    assert probe == {"engine_loaded": False, "oracle_loaded": True, "engine_module": False, "tests_module": False}
