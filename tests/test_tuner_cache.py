"""The launch-shape cache file of the tuner (velox_b200/csrc/tuner.cpp), host
logic only: a decision replaces its own (device, site, bucket) line and keeps
every other line, other devices' and this device's other buckets alike; the
file is rewritten whole with its header. Built with g++ against the CUDA
runtime; without a GPU the device key is the empty name."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    if not shutil.which("g++") or not os.path.exists(os.path.join(CUDA, "include", "cuda_runtime.h")):
        pytest.skip("g++ or the CUDA headers are missing")
    out = str(tmp_path_factory.mktemp("tuner") / "tuner_cache_check")
    subprocess.run(["g++", "-std=c++17", "-I", os.path.join(ROOT, "velox_b200", "csrc"), "-I",
                    os.path.join(CUDA, "include"), os.path.join(ROOT, "tests", "tuner_cache_check.cpp"),
                    os.path.join(ROOT, "velox_b200", "csrc", "tuner.cpp"), "-L", os.path.join(CUDA, "lib64"),
                    "-lcudart", "-Wl,-rpath," + os.path.join(CUDA, "lib64"), "-o", out], check=True)
    return out


def _lines(path):
    return [ln.split() for ln in open(path).read().splitlines() if ln and not ln.startswith("#")]


def test_a_decision_replaces_its_line_and_keeps_the_others(checker, tmp_path):
    cache = tmp_path / "shapes.txt"
    subprocess.run([checker, str(tmp_path / "probe.txt")], check=True)
    key = _lines(tmp_path / "probe.txt")[0][0]  # this machine's device key
    cache.write_text(f"other:132:9.0 collide_convex 14 64 32\n"
                     f"{key} rewind_probe 12 32 8\n"
                     f"{key} collide_convex 14 32 64\n")
    subprocess.run([checker, str(cache)], check=True)
    text = cache.read_text()
    assert text.startswith("# velox_b200 launch shapes")
    lines = sorted(map(tuple, _lines(cache)))
    assert lines == sorted([
        ("other:132:9.0", "collide_convex", "14", "64", "32"),   # another device: kept
        (key, "rewind_probe", "12", "32", "8"),                  # this device, another bucket: kept
        (key, "collide_convex", "14", "128", "16"),              # replaced by this run's decision
        (key, "collide_plane", "16", "128", "16"),               # new
    ])


def test_a_missing_cache_directory_is_created(checker, tmp_path):
    cache = tmp_path / "a" / "b" / "shapes.txt"
    subprocess.run([checker, str(cache)], check=True)
    assert {ln[1] for ln in _lines(cache)} == {"collide_convex", "collide_plane"}
