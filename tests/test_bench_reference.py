"""The reference arm of bench.py on the CPU: the oracle (the C restatement of
the reference step) timed on the host cores, one JSON line with the bench
contract's keys, printed by rank 0 only."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(env_extra):
    env = dict(os.environ, OMP_NUM_THREADS="2", **env_extra)
    return subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", "elastic_cube",
                           "--ref-steps", "1", "--ref-warmup", "0"], cwd=ROOT, env=env, capture_output=True,
                          text=True, timeout=600)


def test_reference_arm_prints_the_contract_line(oracle_built):
    r = _run({})
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["unit"] == "particle-steps/s"
    assert line["higher_is_better"] is True and line["steps"] == 1
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] == 2 and cb["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["config"]["workload"] == "elastic_cube"


def test_reference_arm_other_ranks_do_no_work(oracle_built):
    r = _run({"RANK": "1", "WORLD_SIZE": "2"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""
