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
                           "--steps", "1", "--warmup", "0"], cwd=ROOT, env=env, capture_output=True,
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


def _bench_module():
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_both_arms_emit_the_same_config(oracle_built):
    from nexus_b200 import scenes
    r = _run({})
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    bench = _bench_module()
    assert line["config"] == json.loads(json.dumps(bench.workload_config(scenes.elastic_cube(), 1)))


def test_traffic_figure_is_tied_to_the_kernel_sources(tmp_path):
    """The roofline's traffic comes from a profile that names the hash of the
    kernel sources it was captured on, and is reported only while they match."""
    bench = _bench_module()
    prof = tmp_path / "traffic.md"
    bench.TRAFFIC_PROFILE = str(prof)
    assert bench.load_traffic("sand_water")[0] is None  # no capture
    current = bench.kernel_sources_hash()
    prof.write_text(f"traffic_bytes_per_step: 7.5e8 sources: {current}\n")
    got, info = bench.load_traffic("sand_water")
    assert got == 7.5e8 and info["stale"] is False
    prof.write_text("traffic_bytes_per_step: 7.5e8 sources: 0123456789abcdef\n")
    got, info = bench.load_traffic("sand_water")
    assert got is None and info["stale"] is True and info["last_capture_bytes"] == 7.5e8
