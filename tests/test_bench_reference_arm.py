"""CPU: the benchmark's reference arm (`bench.py --impl reference`): one JSON
line with the contract's keys, timed by the oracle port on the host cores, and
under a multi-rank launch only rank 0 runs and prints (the other ranks exit 0
without work).  Run at 18 qubits to stay small."""
import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def run(rank, world):
    env = dict(os.environ, RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    return subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference",
                           "--qubits", "18", "--steps", "1", "--warmup", "0", "--gpus",
                           str(world)], capture_output=True, text=True, env=env, timeout=300,
                          cwd=ROOT)


def test_reference_arm_prints_the_contract_line():
    p = run(0, 1)
    assert p.returncode == 0, p.stderr
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == "18q gate-layer GB/s"
    assert d["unit"] == "GB/s" and d["higher_is_better"] is True and d["value"] > 0
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "GB/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


def test_other_ranks_exit_without_work():
    p = run(1, 2)
    assert p.returncode == 0, p.stderr
    assert not [l for l in p.stdout.splitlines() if l.startswith("{")]
