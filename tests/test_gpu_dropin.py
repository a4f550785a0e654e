"""The reference engine's own World::step running on the B200 library as its
CUDA backend (velox_b200/dropin/b200_backend.cpp), against the same World
with the CPU emulation of the reference CUDA backend."""
import numpy as np
import pytest

from scenes import scene

pytestmark = pytest.mark.gpu
DT = 1.0 / 60.0


def _state(b):
    return np.concatenate([b["position"], b["orientation"], b["velocity"], b["angularVelocity"]], 1)


@pytest.mark.parametrize("kind,size,substeps", [(3, 2, 8), ("dense", 600, 4)])
def test_reference_world_on_b200_backend(ref, kind, size, substeps):
    if not ref.available("dropin"):
        pytest.skip("drop-in build missing")
    specs, pool = scene(kind, size)
    emu = ref.RefWorld(specs, pool, backend=ref.BACKEND_CUDA_EMULATED, strict=True)
    dev = ref.RefWorld(specs, pool, backend=ref.BACKEND_CUDA_EMULATED, strict="dropin")
    assert dev.L.ref_world_backend_name(dev.h) == b"cuda"
    for w in (emu, dev):
        w.configure(substeps=substeps, workers=1)
    for step in range(3):
        emu.step(DT, 1)
        dev.step(DT, 1)
        a, b = emu.bodies(), dev.bodies()
        err = np.abs(_state(a) - _state(b)) / np.maximum(1.0, np.abs(_state(a)))
        assert err.max() <= 1e-4, (step, float(err.max()))
    st = dev.stats()
    assert st["deviceSubsteps"] == 1 and st["generated"] > 0
