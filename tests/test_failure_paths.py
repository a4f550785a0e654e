"""Failure detection and recovery through the drop-in adapter, on the CPU.

The reference engine's World runs on velox_b200/dropin/b200_backend.cpp
linked against a fake of the library's Backend entry points
(oracle/fake_vxb.c) whose Backend::integrate returns a chosen status. The
adapter must map the status onto the reference's error model
(src/backend_cuda.cu:24-40): recoverable failures (allocation failure, device
loss, a timed-out device wait) throw BackendFailure, which World::step answers
by restarting the frame on the CPU backend (src/world.cpp:3807-3828); the
others surface as exceptions. No GPU is involved."""
import os

import numpy as np
import pytest

from scenes import scene

DT = 1.0 / 60.0
VXB_ERR_OOM, VXB_ERR_DEVICE_LOST, VXB_ERR_CAPACITY, VXB_ERR_TIMEOUT, VXB_ERR_INTERNAL = 3, 4, 5, 7, 8


@pytest.fixture()
def fake(ref, monkeypatch):
    if not ref.available("dropin_fake"):
        pytest.skip("fake drop-in build missing (make -C oracle fake)")
    monkeypatch.delenv("VXB_FAKE_STATUS", raising=False)
    return ref


def _state(b):
    return np.concatenate([b["position"], b["orientation"], b["velocity"], b["angularVelocity"]], 1)


@pytest.mark.parametrize("status", [VXB_ERR_OOM, VXB_ERR_DEVICE_LOST, VXB_ERR_TIMEOUT])
def test_recoverable_failure_restarts_the_frame_on_the_cpu(fake, monkeypatch, status):
    specs, pool = scene("dense", 300)
    dev = fake.RefWorld(specs, pool, backend=fake.BACKEND_CUDA_EMULATED, strict="dropin_fake")
    cpu = fake.RefWorld(specs, pool, backend=fake.BACKEND_CPU, strict=True)
    assert dev.L.ref_world_backend_name(dev.h) == b"cuda"
    for w in (dev, cpu):
        w.configure(substeps=4, workers=1)
    monkeypatch.setenv("VXB_FAKE_STATUS", str(status))
    dev.step(DT, 1)
    cpu.step(DT, 1)
    assert dev.L.ref_world_backend_name(dev.h) == b"cpu"
    # the frame was rolled back and re-run on the CPU backend: the same state
    assert np.array_equal(_state(dev.bodies()), _state(cpu.bodies()))
    dev.step(DT, 2)
    cpu.step(DT, 2)
    assert np.array_equal(_state(dev.bodies()), _state(cpu.bodies()))


@pytest.mark.parametrize("status,needle", [(VXB_ERR_CAPACITY, "caller buffer too small"),
                                           (VXB_ERR_INTERNAL, "consistency check failed")])
def test_unrecoverable_failure_surfaces_as_an_exception(fake, monkeypatch, status, needle):
    specs, pool = scene("dense", 200)
    dev = fake.RefWorld(specs, pool, backend=fake.BACKEND_CUDA_EMULATED, strict="dropin_fake")
    dev.configure(substeps=4, workers=1)
    monkeypatch.setenv("VXB_FAKE_STATUS", str(status))
    with pytest.raises(RuntimeError, match=needle):
        dev.step(DT, 1)
    assert dev.L.ref_world_backend_name(dev.h) == b"cuda"


def test_fake_passes_through_when_nothing_is_injected(fake):
    # With no injected status the fake's later entry points refuse work: the
    # step fails loudly rather than silently succeeding on the fake.
    specs, pool = scene("dense", 200)
    dev = fake.RefWorld(specs, pool, backend=fake.BACKEND_CUDA_EMULATED, strict="dropin_fake")
    dev.configure(substeps=4, workers=1)
    with pytest.raises(RuntimeError, match="velox_b200"):
        dev.step(DT, 1)
    assert os.environ.get("VXB_FAKE_STATUS") is None
