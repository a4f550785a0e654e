"""bench.py's reference arm times only the reference engine: its process loads
no library of this package, builds the same scene as the b200 arm and prints
the same workload description (CPU)."""
import json
import os
import subprocess
import sys

import numpy as np

import velox_b200

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_PROBE = r"""
import runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--size", "600", "--steps", "1", "--warmup", "1"] + sys.argv[1:]
try:
    runpy.run_path("bench.py", run_name="__main__")
except SystemExit:
    pass
maps = open("/proc/self/maps").read()
print("LOADED " + json.dumps(sorted({l.split()[-1] for l in maps.splitlines() if l.endswith(".so")})))
"""


def _run(extra=()):
    env = dict(os.environ, VXB_REFERENCE_BUDGET_S="30")
    out = subprocess.run([sys.executable, "-c", "import json\n" + _PROBE] + list(extra), cwd=ROOT, env=env,
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = out.stdout.strip().splitlines()
    line = json.loads(next(l for l in lines if l.startswith("{")))
    loaded = json.loads(next(l for l in lines if l.startswith("LOADED "))[7:])
    return line, loaded


def test_reference_arm_loads_no_library_of_this_package(ref):
    line, loaded = _run()
    assert line["impl"] == "reference"
    assert not any("libvelox_b200" in p for p in loaded), loaded
    assert any("libvelox_ref_fast" in p for p in loaded), loaded
    assert line["cpu_baseline"]["single_worker"]["cores"] == 1


def test_reference_arm_prints_the_b200_arms_workload(ref):
    import bench
    line, _ = _run()
    assert line["config"] == bench.single_config(line["config"]["bodies"], 1)


def test_reference_build_generates_the_librarys_scenes(ref):
    for config, size in [(1, 4), (2, 800), (3, 2), (4, 12), (5, 6)]:
        a, pa = ref.generate_scene(config, seed=config, size=size)
        b, pb = velox_b200.generate_scene(config, seed=config, size=size)
        assert a.tobytes() == b.tobytes()
        assert np.array_equal(pa, pb)
