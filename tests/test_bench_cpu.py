"""bench.py's reference arm on the CPU: the JSON line of the contract, and silence on ranks > 0.

The reference arm times the restatement of the reference's ThreadedBackend on the host cores; it
needs no GPU, so its output contract is checked here: one JSON line with the metric, a positive value,
the CPU-baseline description and an end-to-end entry without host-device copies.
"""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_bench(args, env_extra=None):
    env = dict(os.environ)
    env.update(env_extra or {})
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + args, cwd=ROOT, env=env,
                       capture_output=True, text=True, timeout=600)
    return p


def test_reference_arm_prints_one_contract_line():
    p = run_bench(["--impl", "reference", "--config", "c0", "--steps", "2", "--warmup", "3"])
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.strip().startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["value"] > 0 and d["unit"] == "pair-evals/s" and d["higher_is_better"] is True
    assert d["steps"] == 2 and d["warmup"] == 3
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["cores"] >= 1 and cb["kind"] in ("port", "reference") and cb["sample"]
    assert d["e2e"]["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0


def test_reference_arm_without_cpu_restatement_says_so():
    """The serving loop has no CPU restatement: one `unavailable` line, exit 0."""
    p = run_bench(["--impl", "reference", "--config", "c4", "--steps", "1", "--warmup", "3"])
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.strip().startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and "c4" in d["unavailable"]


@pytest.mark.parametrize("config", ["rsp1d", "rsp2d"])
def test_reference_arm_single_pass_shapes(config):
    """The single-pass shapes time the oracle's restatement of the reference's own passes (the 1D fused
    four-operator loop; the 2D loop with its six row updates per pair)."""
    p = run_bench(["--impl", "reference", "--config", config, "--steps", "1", "--warmup", "3"])
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.strip().startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and config in d["config"]["workload"]


def test_reference_arm_is_silent_on_other_ranks():
    p = run_bench(["--impl", "reference", "--config", "c0", "--steps", "2", "--warmup", "3"],
                  {"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert p.returncode == 0, p.stderr[-2000:]
    assert not [l for l in p.stdout.splitlines() if l.strip().startswith("{")]


def test_gpus_flag_launches_one_rank_per_gpu():
    """`bench.py --gpus 2` without a launcher starts two ranks itself (torch.distributed.run with
    RANK / LOCAL_RANK / WORLD_SIZE set); rank 0 alone prints the line, which names both ranks."""
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--impl", "reference",
                        "--config", "c0", "--steps", "1", "--warmup", "3"], cwd=ROOT, env=env,
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.strip().startswith("{")]
    assert len(lines) == 1
    assert json.loads(lines[0])["n_gpus"] == 2
