"""The allocation-free broad-phase entry point (vxb_stage_pairs_noalloc).

It serves callers that must not allocate device memory during a call (fixed
memory budgets, plugin hosts that own device memory, nearly full devices):
all its device memory is one library-owned array. Its pairs must equal those
of the allocating entry point (vxb_stage_pairs) exactly — pairs are integers —
on two calls in a row, since every call reuses the same array.
"""
import ctypes

import numpy as np
import pytest

import velox_b200
from velox_b200 import binding
from scenes import scene

pytestmark = pytest.mark.gpu
DT = 1.0 / 60.0
CAP = 32768 + 8192


def _noalloc(bodies, cap=CAP):
    L = velox_b200.lib()
    count = ctypes.c_uint32()
    out = np.zeros(max(cap, 1), np.uint64)
    status = L.vxb_stage_pairs_noalloc(binding.ptr(bodies), len(bodies), DT, binding.ptr(out), cap,
                                       ctypes.byref(count), None)
    return status, out[:min(count.value, cap)], count.value


@pytest.mark.parametrize("kind,size", [(1, 0), ("dense", 800), (2, 3000)])
def test_noalloc_pairs_equal_allocating_entry_point(kind, size):
    specs, pool = scene(kind, size)
    bodies, _, _ = velox_b200.bodies_from_specs(specs, pool)
    ctx = velox_b200.Context(0)
    expected = ctx.pairs(bodies, DT)
    ctx.close()
    assert len(expected) > 0
    # the scenes stand on a plane: body-plane pairs are part of the output
    planes = np.flatnonzero(bodies["shape"] == binding.SHAPE["plane"])
    assert np.isin(expected & 0xffffffff, planes).any() or np.isin(expected >> 32, planes).any()
    for call in range(2):
        status, pairs, _ = _noalloc(bodies)
        assert status == 0, (call, status)
        assert np.array_equal(pairs, expected), call


def test_noalloc_reports_the_needed_size_when_the_output_is_too_small():
    specs, pool = scene("dense", 800)
    bodies, _, _ = velox_b200.bodies_from_specs(specs, pool)
    status, _, needed = _noalloc(bodies)
    assert status == 0 and needed > 1
    status, _, count = _noalloc(bodies, cap=1)
    assert status == 5 and count == needed  # VXB_ERR_CAPACITY, *count = pairs found
    status, pairs, _ = _noalloc(bodies, cap=count)
    assert status == 0
    ctx = velox_b200.Context(0)
    expected = ctx.pairs(bodies, DT)
    ctx.close()
    assert np.array_equal(pairs, expected)


def test_noalloc_rejects_more_bodies_than_its_limit():
    specs, pool = scene(2, 5000)
    bodies, _, _ = velox_b200.bodies_from_specs(specs, pool)
    status, pairs, _ = _noalloc(bodies)
    assert status == 5  # VXB_ERR_CAPACITY
    assert len(pairs) == 0


def test_noalloc_rejects_more_body_pairs_than_its_limit():
    # 4,000 spheres of radius 0.5 on a 0.4 m lattice: every sphere overlaps its
    # 26 lattice neighbours, far beyond 32,768 body-body candidate pairs.
    specs, pool = scene(2, 4000)
    side = 16
    k = np.arange(len(specs))
    dyn = specs["shape"] != binding.SHAPE["plane"]
    specs["shape"][dyn] = binding.SHAPE["sphere"]
    specs["radius"][dyn] = 0.5
    specs["position"][:, 0] = 0.4 * (k % side)
    specs["position"][:, 1] = 2.0 + 0.4 * ((k // side) % side)
    specs["position"][:, 2] = 0.4 * (k // (side * side))
    specs["velocity"] = 0.0
    bodies, _, _ = velox_b200.bodies_from_specs(specs, pool)
    status, pairs, count = _noalloc(bodies)
    assert status == 5  # VXB_ERR_CAPACITY
    assert count > 32768
