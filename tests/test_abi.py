"""C-ABI surface and host-side scene construction (no GPU needed)."""
import ctypes
import os
import re

import numpy as np

import velox_b200
from velox_b200 import binding

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for header in os.listdir(os.path.join(ROOT, "include")):
        if not header.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", header)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[a-z_ A-Z0-9\*]*?\b(vxb_[a-z0-9_]+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(binding.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 25
    for name in names:
        assert hasattr(lib, name), name


def test_status_strings_and_version():
    L = velox_b200.lib()
    assert b"sm_100a" in L.vxb_version()
    for s in range(8):
        assert L.vxb_status_string(s)


def test_context_without_device_reports_no_device():
    import torch
    if torch.cuda.is_available():
        return
    L = velox_b200.lib()
    h = ctypes.c_void_p()
    assert L.vxb_context_create(0, ctypes.byref(h)) == 2  # VXB_ERR_NO_DEVICE


def test_record_sizes_match_reference_layout():
    assert binding.BODY.itemsize == 320
    assert binding.CONTACT.itemsize == 128
    assert binding.SPEC.itemsize == 116
    assert ctypes.sizeof(binding.SolverOptions) == 24


def test_records_restore_the_struct_layout():
    # np.concatenate of padded records drops the padding: the binding re-lays
    # such arrays field by field, and refuses them where the library writes back
    a = np.zeros(3, binding.BODY)
    a["position"] = np.arange(9, dtype=np.float32).reshape(3, 3)
    a["motionType"] = [0, 2, 0]
    both = np.concatenate([a, a])
    assert both.dtype.itemsize != binding.BODY.itemsize
    fixed = binding.records(both, binding.BODY)
    assert fixed.dtype == binding.BODY and fixed.flags["C_CONTIGUOUS"]
    assert np.array_equal(fixed["position"], both["position"])
    assert list(fixed["motionType"]) == [0, 2, 0, 0, 2, 0]
    assert binding.records(a, binding.BODY) is a
    try:
        binding.records(both, binding.BODY, inout=True)
    except ValueError:
        pass
    else:
        raise AssertionError("an in/out array in another layout was accepted")


def test_scene_generation_is_seeded_and_sized():
    a, pa = velox_b200.generate_scene(2, size=500)
    b, pb = velox_b200.generate_scene(2, size=500)
    assert len(a) == 501 and np.array_equal(a.view(np.uint8), b.view(np.uint8))
    assert np.array_equal(pa, pb)
    shapes = np.bincount(a["shape"][1:], minlength=8)
    assert shapes[0] > 0 and shapes[2] > 0 and shapes[3] > 0 and shapes[5] > 0 and shapes[7] > 0
    c, _ = velox_b200.generate_scene(3, size=2)
    assert len(c) == 1 + 2 * 210
    d, _ = velox_b200.generate_scene(4, size=16)
    assert d["world"].max() == 15 and (d["shape"] == 1).sum() == 16
    e, _ = velox_b200.generate_scene(5, size=4)
    assert len(e) == 4 * 7


def test_hull_construction_is_closed_and_outward():
    specs, pool = velox_b200.generate_scene(2, size=200)
    bodies, hull, faces = velox_b200.bodies_from_specs(specs, pool)
    for b in bodies[bodies["shape"] == 5][:20]:
        pts = hull[b["hullFirst"]:b["hullFirst"] + b["hullCount"]]
        tri = faces[b["hullFaceFirst"]:b["hullFaceFirst"] + 3 * b["hullFaceCount"]].reshape(-1, 3)
        assert len(tri) == 2 * len(pts) - 4  # closed triangulated sphere: F = 2V - 4
        centroid = pts.mean(0)
        for t in tri:
            n = np.cross(pts[t[1]] - pts[t[0]], pts[t[2]] - pts[t[0]])
            assert np.dot(n, pts[t[0]] - centroid) > 0
        assert abs(np.linalg.norm(pts, axis=1).max() - b["radius"]) < 1e-6
