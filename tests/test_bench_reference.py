"""The reference arm of bench.py on the CPU: one JSON line with the GPU
arm's metric, unit and workload, its own start / barostat / arithmetic
stated in the config, a cpu_baseline describing the run and an e2e block
without transfers; rank 0 alone prints it."""

import json
import os
import subprocess
import sys
from pathlib import Path
from types import SimpleNamespace

ROOT = Path(__file__).resolve().parents[1]


def run_arm(env_extra):
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    env.update(env_extra)
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1",
                          "--warmup", "0", "--molecules", "512"],
                         cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    return [l for l in out.stdout.splitlines() if l.startswith("{")]


def test_reference_line_matches_the_gpu_arm_contract():
    sys.path.insert(0, str(ROOT))
    import bench
    from heddle_b200 import systems as S

    lines = run_arm({})
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert (d["metric"], d["unit"], d["higher_is_better"]) == (bench.METRIC, bench.UNIT, True)
    assert d["value"] > 0 and d["cpu_baseline"]["value"] == d["value"]
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": bench.UNIT, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    args = SimpleNamespace(molecules=512, equilibrate=300, barostat=1)
    spec = S.spc_water(512)
    gpu = bench.workload_config(args, spec, 1)
    for key in ("workload", "atoms", "grid", "parallelism"):
        assert d["config"][key] == gpu[key]
    # what this arm does differently is said, not inherited from the GPU arm
    assert d["config"]["barostat"].startswith("none")
    assert d["config"]["start"] == "lattice start, no relaxation"
    assert "FP64" in d["config"]["arithmetic"]


def test_reference_arm_prints_on_rank_zero_only():
    assert run_arm({"RANK": "1", "WORLD_SIZE": "2"}) == []
    d = json.loads(run_arm({"RANK": "0", "WORLD_SIZE": "2"})[0])
    assert d["config"]["parallelism"] == "replicas x2"
