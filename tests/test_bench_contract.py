"""The bench's reference arm runs the reference's host perft on the CPU, so
its JSON line can be checked here: the keys the bench contract names, a
bounded sample, and the same metric and workload names as the GPU arm."""
import json
import os
import subprocess
import sys

from tests._oracle import ROOT

KEYS = {"impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "higher_is_better", "scaling",
        "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"}


def _run(*args):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", *args],
                       capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    return lines[0]


def test_reference_arm_line():
    d = _run("--steps", "1", "--warmup", "0", "--cpu-seconds", "1")
    assert KEYS <= set(d)
    assert d["impl"] == "reference" and d["metric"] == "perft leaf nodes/s (bit-exact)"
    assert d["unit"] == "leaf nodes/s" and d["higher_is_better"] is True and d["value"] > 0
    assert d["config"]["workload"].startswith("batch4096")
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_other_workload():
    d = _run("--workload", "start", "--steps", "2", "--warmup", "1", "--cpu-seconds", "1")
    assert d["config"]["workload"].startswith("initial position, depth 5")
    assert d["steps"] == 2 and d["value"] > 0


def test_reference_arm_other_ranks_exit_quietly():
    """Under torchrun only rank 0 runs the reference arm and prints; the
    other ranks exit 0 without work or output."""
    env = dict(os.environ, WORLD_SIZE="2", RANK="1", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0"], capture_output=True, text=True, timeout=120, cwd=ROOT,
                       env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    assert not [x for x in r.stdout.splitlines() if x.startswith("{")]
    env.update(RANK="0", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0", "--cpu-seconds", "1"], capture_output=True, text=True,
                       timeout=300, cwd=ROOT, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1 and lines[0]["n_gpus"] == 2 and lines[0]["impl"] == "reference"


def test_reference_arm_loads_no_engine_library():
    """The reference arm reads its workload from the stored numpy file and runs
    only the reference's host perft: with the engine library made unloadable it
    still succeeds, and its process never maps libperft_b200."""
    code = ("import runpy, sys\n"
            "sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '0', '--cpu-seconds', '1']\n"
            "try:\n"
            "    runpy.run_path('bench.py', run_name='__main__')\n"
            "except SystemExit as e:\n"
            "    assert not e.code, e.code\n"
            "maps = open('/proc/self/maps').read()\n"
            "print('ENGINE_MAPPED' if 'libperft_b200' in maps else 'ENGINE_NOT_MAPPED')\n")
    env = dict(os.environ, PERFT_B200_LIB=os.path.join(ROOT, "no-such-dir", "libperft_b200.so"))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300, cwd=ROOT,
                       env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "ENGINE_NOT_MAPPED" in r.stdout
    line = json.loads(next(x for x in r.stdout.splitlines() if x.startswith("{")))
    assert line["cpu_baseline"]["library"].startswith("oracle/")
