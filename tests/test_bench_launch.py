"""bench.py's multi-rank plumbing on the CPU: ``--gpus 2`` outside torchrun starts two ranks
itself (torch.distributed.run on 127.0.0.1), the ranks shard the 512-case ensemble by estimated
work and combine their totals over gloo, and rank 0 alone prints the JSON line."""

import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_bench_gpus_2_launches_two_ranks():
    env = dict(os.environ)
    env.pop("WORLD_SIZE", None)
    res = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--dry-run"],
                         capture_output=True, text=True, timeout=300, env=env)
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [json.loads(x) for x in res.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1  # rank 0 only
    line = lines[0]
    assert line["n_gpus"] == 2
    sh = line["batched"]["sharding"]
    assert sh["ranks"] == 2
    assert sum(sh["cases_per_rank"]) == 512
    assert sh["estimated_imbalance"] < 1.01
    # the summed cells of both shards are the whole ensemble's
    from schemi_b200 import cases

    assert line["batched"]["cells"] == sum(cases.richtmyer_meshkov_draws(i)[0] ** 2 for i in range(512))


def test_bench_refuses_mismatched_world_size():
    env = dict(os.environ, WORLD_SIZE="1", RANK="0", LOCAL_RANK="0")
    res = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--dry-run"],
                         capture_output=True, text=True, timeout=120, env=env)
    assert res.returncode != 0
    assert "WORLD_SIZE" in res.stderr


def test_conserved_errors_scales():
    import numpy as np

    sys.path.insert(0, ROOT)
    import bench

    want = {"rho1": np.array([1.0, 2.0]), "rho2": np.array([1.0, 1.0]), "rho": np.array([2.0, 3.0]),
            "mx": np.array([3.0, 0.0]), "my": np.array([0.0, 4.0]), "mz": np.zeros(2), "E": np.array([5.0, 5.0])}
    got = {k: v.copy() for k, v in want.items()}
    assert bench.conserved_errors(got, want, 2)["l1"] == 0.0
    got["my"] = np.array([0.0, 4.4])
    e = bench.conserved_errors(got, want, 2)
    # momentum as a vector: |0.4| over |3| + |4| summed over the cells
    assert abs(e["fields"]["m"]["l1"] - 0.4 / 7.0) < 1e-15
    assert abs(e["fields"]["m"]["linf"] - 0.4 / 4.0) < 1e-15
    assert "mz" not in e["fields"]
