"""bench.py's multi-rank path on CPU: `--gpus 2` without torchrun starts two
ranks itself (torch.distributed.run), and the ranks run bench.py's own
dist_setup / barrier / max-and-sum reduction sequence over gloo. The dry run
stands in a step time of 1 + rank ms and counters (rank, 1) per rank, so the
line must report 2 ranks, the max time (2 ms) and the summed counters."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_bench_launches_two_gloo_ranks():
    env = dict(os.environ)
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT"):
        env.pop(k, None)
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--dry-run",
                          "--backend", "gloo", "--steps", "2"], capture_output=True, text=True, timeout=300,
                         env=env, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout          # rank 0 alone prints
    line = json.loads(lines[0])
    assert line["n_gpus"] == 2 and line["dry_run"] is True
    assert line["ms_per_step"] == 2.0            # max over ranks of 1 + rank
    assert line["counters"] == {"frame_errors": 1.0, "ranks": 2.0}   # sums over ranks


def test_bench_refuses_more_gpus_than_visible():
    env = dict(os.environ)
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        env.pop(k, None)
    env["CUDA_VISIBLE_DEVICES"] = ""
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--steps", "1"],
                         capture_output=True, text=True, timeout=300, env=env, cwd=ROOT)
    assert out.returncode == 2
    assert "only 0 CUDA device(s) are visible" in out.stderr
