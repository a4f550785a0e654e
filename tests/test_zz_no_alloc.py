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


def _noalloc(bodies):
    L = velox_b200.lib()
    count = ctypes.c_uint32()
    out = np.zeros(CAP, np.uint64)
    status = L.vxb_stage_pairs_noalloc(binding.ptr(bodies), len(bodies), DT, binding.ptr(out), CAP,
                                       ctypes.byref(count), None)
    return status, out[:count.value]


@pytest.mark.parametrize("kind,size", [(1, 0), ("dense", 800), (2, 3000)])
def test_noalloc_pairs_equal_allocating_entry_point(kind, size):
    specs, pool = scene(kind, size)
    bodies, _, _ = velox_b200.bodies_from_specs(specs, pool)
    ctx = velox_b200.Context(0)
    expected = ctx.pairs(bodies, DT)
    ctx.close()
    assert len(expected) > 0
    for call in range(2):
        status, pairs = _noalloc(bodies)
        assert status == 0, (call, status)
        assert np.array_equal(pairs, expected), call


def test_noalloc_rejects_more_bodies_than_its_limit():
    specs, pool = scene(2, 5000)
    bodies, _, _ = velox_b200.bodies_from_specs(specs, pool)
    status, pairs = _noalloc(bodies)
    assert status == 5  # VXB_ERR_CAPACITY
    assert len(pairs) == 0
