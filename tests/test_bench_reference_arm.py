"""bench.py's reference arm on the CPU: it times complete solves of the
oracle's restatement of the reference solver on the host cores and prints
one JSON line with the keys the bench contract asks for; it never maps this
repository's libpgc.so; under torchrun only rank 0 works."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ARGS = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", "plain_642_60_k2",
        "--steps", "1", "--warmup", "3"]


# runs bench.py as __main__, then reports whether the process mapped the product library
_MAPS_PROBE = ("import runpy, sys; sys.argv = sys.argv[1:]; runpy.run_path(sys.argv[0], run_name='__main__'); "
               "maps = open('/proc/self/maps').read(); print('LIBPGC_MAPPED', 'libpgc.so' in maps)")


def _run(env_extra, probe=False):
    env = dict(os.environ, **env_extra)
    args = [sys.executable, "-c", _MAPS_PROBE] + ARGS[1:] if probe else ARGS
    return subprocess.run(args, capture_output=True, text=True, timeout=600, cwd=ROOT, env=env)


def test_reference_arm_prints_one_contract_line():
    r = _run({}, probe=True)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["value"] > 0 and d["unit"] == "solves/s" and d["higher_is_better"] is True
    # complete solves are timed: at most the requested steps, after one warm-up step
    assert (d["steps"], d["warmup"], d["steps_requested"], d["warmup_requested"]) == (1, 1, 1, 3)
    assert len(d["step_s"]) == 1 and abs(d["ms_per_step"] - 1000.0 * d["step_s"][0]) < 1e-6
    assert d["config"]["workload"] == "plain_642_60_k2"
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert cb["cpu"]["usable_cores"] == cb["cores"] and cb["cpu"]["model"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    # the arm never loads the product library (it imports only the synthetic data module)
    assert "LIBPGC_MAPPED False" in r.stdout


def test_reference_arm_other_ranks_exit_without_work():
    r = _run({"RANK": "1", "LOCAL_RANK": "1", "WORLD_SIZE": "2"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert not [l for l in r.stdout.splitlines() if l.startswith("{")]
