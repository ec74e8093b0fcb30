"""bench.py's reference arm (the reference algorithm's pair loop on the host cores, through the
oracle) keeps the benchmark's JSON contract, and under a multi-rank launch only rank 0 works."""
import json
import os
import subprocess
import sys

from conftest import ROOT


def _run(args, env=None, timeout=600):
    e = dict(os.environ)
    e.update(env or {})
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + args, cwd=ROOT,
                          capture_output=True, text=True, env=e, timeout=timeout)


def test_reference_arm_json_contract():
    r = _run(["--impl", "reference", "--steps", "1", "--warmup", "0", "--ref-budget", "1"])
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "higher_is_better",
              "scaling", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["metric"] == "s/solve" and line["higher_is_better"] is False
    cb = line["cpu_baseline"]
    assert cb["value"] == line["value"] and cb["kind"] in ("port", "reference") and cb["cores"] >= 1
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"],
                           "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert line["value"] > 0


def test_reference_arm_nonzero_rank_exits_without_work():
    r = _run(["--impl", "reference", "--steps", "1", "--warmup", "0", "--ref-budget", "1"],
             env={"RANK": "1", "LOCAL_RANK": "1", "WORLD_SIZE": "2"}, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""
