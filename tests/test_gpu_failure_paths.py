"""Failure detection on the GPU without a fault.

* Host-side injection: VELOX_CUDA_TEST_FAIL=oom|device-loss makes
  Backend::integrate fail before any device work (the reference's own test
  hook, src/backend_cuda.cu:69-78); the reference World running on the
  library then restarts the frame on its CPU backend
  (src/world.cpp:3807-3828).
* Bounded device waits: with the context's wait limit cut to one poll, the
  grid barriers and dataflow waits of the cooperative solve give up, the call
  reports VXB_ERR_TIMEOUT, the World falls back to the CPU, and the context
  stays usable (a later call with the default limit succeeds).
"""
import numpy as np
import pytest

import velox_b200

pytestmark = pytest.mark.gpu
DT = 1.0 / 60.0


def _state(b):
    return np.concatenate([b["position"], b["orientation"], b["velocity"], b["angularVelocity"]], 1)


@pytest.fixture(scope="module")
def pile(ref):
    # 3,000 mixed shapes settled on the plane: giant islands (cooperative solve)
    specs, pool = velox_b200.generate_scene(2, size=3000)
    w = ref.RefWorld(specs, pool)
    start = w.bodies()
    pts, faces = w.soup()
    w.close()
    soup = velox_b200.make_soup(pts, faces)
    ctx = velox_b200.Context(0)
    ctx.load(start, soup)
    ctx.configure(dt=DT, substeps=4)
    ctx.step(250)
    state = ctx.read_bodies()
    ctx.close()
    return specs, pool, state, soup


def _dropin(ref):
    if not ref.available("dropin"):
        pytest.skip("drop-in build missing")


@pytest.mark.parametrize("mode", ["oom", "device-loss"])
def test_injected_failure_falls_back_to_the_cpu(ref, monkeypatch, mode):
    _dropin(ref)
    from scenes import scene
    specs, pool = scene("dense", 400)
    dev = ref.RefWorld(specs, pool, backend=ref.BACKEND_CUDA_EMULATED, strict="dropin")
    cpu = ref.RefWorld(specs, pool, backend=ref.BACKEND_CPU, strict=True)
    for w in (dev, cpu):
        w.configure(substeps=4, workers=1)
    assert dev.L.ref_world_backend_name(dev.h) == b"cuda"
    # the first frame fails on the device and is re-run on the CPU, so it
    # equals a CPU world's first frame (no warm-start history on either side)
    monkeypatch.setenv("VELOX_CUDA_TEST_FAIL", mode)
    dev.step(DT, 1)
    monkeypatch.delenv("VELOX_CUDA_TEST_FAIL")
    assert dev.L.ref_world_backend_name(dev.h) == b"cpu"
    cpu.step(DT, 1)
    err = np.abs(_state(dev.bodies()) - _state(cpu.bodies())) / np.maximum(1.0, np.abs(_state(cpu.bodies())))
    assert err.max() <= 1e-4


def test_timed_out_wait_falls_back_to_the_cpu(ref, monkeypatch, pile):
    _dropin(ref)
    specs, pool, state, _ = pile
    monkeypatch.setenv("VXB_WAIT_LIMIT", "1")  # read when the World creates its backend
    dev = ref.RefWorld(specs, pool, backend=ref.BACKEND_CUDA_EMULATED, strict="dropin")
    monkeypatch.delenv("VXB_WAIT_LIMIT")
    cpu = ref.RefWorld(specs, pool, backend=ref.BACKEND_CPU, strict=True)
    for w in (dev, cpu):
        w.configure(substeps=4, workers=1)
        w.set_bodies(state)
    assert dev.L.ref_world_backend_name(dev.h) == b"cuda"
    dev.step(DT, 1)
    cpu.step(DT, 1)
    assert dev.L.ref_world_backend_name(dev.h) == b"cpu"
    err = np.abs(_state(dev.bodies()) - _state(cpu.bodies())) / np.maximum(1.0, np.abs(_state(cpu.bodies())))
    assert err.max() <= 1e-4


def test_timed_out_wait_leaves_the_context_usable(pile):
    _, _, state, soup = pile
    ctx = velox_b200.Context(0)
    ctx.load(state, soup)
    ctx.configure(dt=DT, substeps=4)
    ctx.set_wait_limit(1)
    with pytest.raises(velox_b200.VeloxError) as info:
        ctx.step(1)
    assert info.value.status == 7  # VXB_ERR_TIMEOUT
    ctx.set_wait_limit(0)  # the default limit again
    ctx.load(state, soup)
    ctx.step(1)
    st = ctx.stats()
    assert st["giantIslands"] >= 1
    assert np.isfinite(_state(ctx.read_bodies())).all()
    ctx.close()
