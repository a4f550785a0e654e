"""Joints on the device: the reference World (src/world.cpp:4196-4207) stepping
on this library through its Backend interface, whose advanceSubsteps takes
64 or more joints to the device joint pass (velox_b200/csrc/joints.cu; the
reference CUDA backend's algorithm, src/backend_cuda.cu:691-760), against
the same World on the oracle's CPU emulation of that backend, and against
the reference's own CUDA backend on this GPU. The joint rows themselves are
pinned bit for bit on the CPU (tests/test_joint_rows.py)."""
import numpy as np
import pytest

import joint_scenes as js

pytestmark = pytest.mark.gpu
DT = 1.0 / 60.0


def _state(b):
    return np.concatenate([b["position"], b["orientation"], b["velocity"], b["angularVelocity"]], 1)


def _rel(mine, theirs):
    return float((np.abs(_state(mine) - _state(theirs)) / np.maximum(1.0, np.abs(_state(theirs)))).max())


def _need(ref, build):
    if not ref.available(build):
        pytest.skip(f"{build} build missing")


def test_jointed_world_on_b200_backend_matches_the_emulated_reference(ref):
    _need(ref, "dropin")
    emu = js.jointed_world(ref)
    dev = js.jointed_world(ref, strict="dropin")
    assert dev.L.ref_world_backend_name(dev.h) == b"cuda" and len(dev.joints()) == 80
    for w in (emu, dev):
        w.configure(substeps=4, workers=1)
    contacts = 0
    # 25 steps: beyond them the chains' ulp-level differences (CUDA's atan2f /
    # acosf in the hinge, cone-twist and frame rows against the host's) grow
    # past 1e-4 in the swinging links
    for step in range(25):
        emu.step(DT, 1)
        dev.step(DT, 1)
        assert dev.stats()["deviceSubsteps"] == 1 and emu.stats()["deviceSubsteps"] == 1
        assert _rel(dev.bodies(), emu.bodies()) <= 1e-4, step
        contacts = max(contacts, dev.stats()["generated"])
        je, jd = emu.joints(), dev.joints()
        for f in ("reactionLinearImpulse", "reactionAngularImpulse", "motorImpulse", "limitImpulse"):
            assert np.allclose(jd[f], je[f], rtol=1e-3, atol=1e-4), (step, f)
    assert contacts > 0  # contacts and joints share bodies
    emu.close()
    dev.close()


def test_jointed_world_matches_the_reference_cuda_backend(ref):
    _need(ref, "dropin")
    _need(ref, "cuda")
    theirs = js.jointed_world(ref, strict="cuda")
    mine = js.jointed_world(ref, strict="dropin")
    for w in (theirs, mine):
        w.configure(substeps=4, workers=1)
    for step in range(20):
        theirs.step(DT, 1)
        mine.step(DT, 1)
        assert theirs.stats()["deviceSubsteps"] == 1 and mine.stats()["deviceSubsteps"] == 1
        assert _rel(mine.bodies(), theirs.bodies()) <= 1e-4, step
    theirs.close()
    mine.close()


def test_breaking_joints_match_the_emulated_reference(ref):
    _need(ref, "dropin")
    emu = js.jointed_world(ref, break_force=60.0)
    dev = js.jointed_world(ref, strict="dropin", break_force=60.0)
    for w in (emu, dev):
        w.configure(substeps=4, workers=1)
    for step in range(20):
        emu.step(DT, 1)
        dev.step(DT, 1)
        assert len(dev.joints()) == len(emu.joints()), step
        assert _rel(dev.bodies(), emu.bodies()) <= 1e-4, step
    assert len(emu.joints()) < 80  # some joints broke and the World removed them
    emu.close()
    dev.close()


def test_fewer_than_64_joints_stay_on_the_host_path(ref):
    _need(ref, "dropin")
    emu = js.jointed_world(ref, chains=4)
    dev = js.jointed_world(ref, chains=4, strict="dropin")
    for w in (emu, dev):
        w.configure(substeps=4, workers=1)
    for step in range(10):
        emu.step(DT, 1)
        dev.step(DT, 1)
        assert dev.stats()["deviceSubsteps"] == 0
        assert _rel(dev.bodies(), emu.bodies()) <= 1e-4, step
    emu.close()
    dev.close()


def _kinematic_world(ref, strict):
    """Spheres on a plane swept by a kinematic box paddle (moving and
    spinning at a set velocity) and resting on a kinematic platform."""
    from velox_b200 import binding
    specs = np.zeros(2 + 2 + 40, binding.SPEC)
    specs["orientation"] = (0, 0, 0, 1)
    specs["friction"] = 0.5
    specs[0]["shape"], specs[0]["planeNormal"] = 1, (0, 1, 0)
    specs[1]["shape"], specs[1]["mass"], specs[1]["halfExtents"] = 2, 1.0, (0.2, 0.4, 1.5)
    specs[1]["position"] = (-2.0, 0.45, 0.0)
    specs[2]["shape"], specs[2]["mass"], specs[2]["halfExtents"] = 2, 1.0, (1.0, 0.1, 1.0)
    specs[2]["position"] = (3.0, 1.0, 0.0)
    specs[3]["shape"], specs[3]["mass"], specs[3]["radius"] = 0, 1.0, 0.2
    specs[3]["position"] = (3.0, 1.35, 0.0)
    rng = np.random.default_rng(3)
    for k in range(4, len(specs)):
        specs[k]["shape"], specs[k]["mass"], specs[k]["radius"] = 0, 0.5, 0.18
        specs[k]["position"] = (rng.uniform(-1.0, 2.0), 0.2 + 0.4 * (k % 3), rng.uniform(-1.2, 1.2))
    w = ref.RefWorld(specs, np.zeros((0, 3), np.float32), strict=strict)
    b = w.bodies()
    for k, v, om in ((1, (2.0, 0.0, 0.0), (0.0, 1.0, 0.0)), (2, (0.0, 0.5, 0.0), (0.0, 0.0, 0.0))):
        b["motionType"][k] = 1  # Kinematic
        b["invMass"][k] = 0.0
        b["invInertia"][k] = (0.0, 0.0, 0.0)
        b["velocity"][k], b["angularVelocity"][k] = v, om
    w.set_bodies(b)
    return w


def test_kinematic_bodies_on_the_b200_backend_match_the_emulated_reference(ref):
    _need(ref, "dropin")
    emu, dev = _kinematic_world(ref, True), _kinematic_world(ref, "dropin")
    for w in (emu, dev):
        w.configure(substeps=4, workers=1)
    for step in range(30):
        emu.step(DT, 1)
        dev.step(DT, 1)
        assert dev.stats()["deviceSubsteps"] == 1
        assert _rel(dev.bodies(), emu.bodies()) <= 1e-4, step
    b = dev.bodies()
    assert abs(b["position"][1][0] - (-2.0 + 2.0 * 30 * DT)) < 1e-3  # the paddle moved at its set speed
    assert dev.stats()["generated"] > 0
    emu.close()
    dev.close()
