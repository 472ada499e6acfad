"""The benchmark's CPU side, without a GPU: the reference arm's JSON line
(the FP64 restatement of the reference's algorithm on the host cores) and
its launch contract.  The arm must not load the product library, and under
torchrun ranks other than 0 exit 0 without printing a line."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ARGS = ["--impl", "reference", "--steps", "1", "--warmup", "1", "--pairs", "64", "--cpu-seconds", "1"]


def _run(args, env_extra=None):
    env = dict(os.environ, **(env_extra or {}))
    code = ("import runpy, sys\n"
            f"sys.argv = ['bench.py'] + {args!r}\n"
            "runpy.run_path('bench.py', run_name='__main__')\n"
            "maps = open('/proc/self/maps').read()\n"
            "print('SO_MAPPED' if 'libphotonprop_b200' in maps else 'SO_NOT_MAPPED')\n"
            "print('PKG_IMPORTED' if 'photonprop_b200' in sys.modules else 'PKG_NOT_IMPORTED')\n")
    return subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True, text=True,
                          timeout=600)


def test_reference_arm_line():
    r = _run(ARGS)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "photons/s" and d["value"] > 0
    assert d["higher_is_better"] is True and d["steps"] == 1 and d["warmup"] == 1
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"]
    assert cb["value"] == d["value"]
    assert d["config"]["workload"]
    # the product is neither imported nor mapped in the reference arm
    assert "SO_NOT_MAPPED" in r.stdout and "PKG_NOT_IMPORTED" in r.stdout


def test_reference_arm_other_ranks_print_nothing():
    r = _run(ARGS, {"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert not any(ln.startswith("{") for ln in r.stdout.splitlines())
