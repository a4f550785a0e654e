"""Island sleeping, the wake pass and contact events of the device world
against the reference World (its own SleepManager::update, src/sleep.cpp:52-237;
wake pass src/world.cpp:4106-4128; events :4398-4488; resting pairs' cached
contacts :4496-4521) on a scene that comes to rest, turns drowsy, falls asleep,
is struck by a projectile (waking one stack) and falls asleep again; one box
that may not sleep holds its island awake.

Per step for 150 steps: body state (including asleep and sleepTimer) within
1e-4 relative, and the same events (pairs, types, sensor flags; impulses to
1e-4 relative; point and normal of the representative contact when its
impulse is positive: with all impulses zero the reference's pick follows a
contact order it leaves unspecified)."""
import numpy as np
import pytest

import velox_b200
from velox_b200 import binding
from sleep_scenes import resting_scene

pytestmark = pytest.mark.gpu
DT = 1.0 / 60.0
REL_TOL = 1e-4


def _state(b):
    return np.concatenate([b["position"], b["orientation"], b["velocity"], b["angularVelocity"]], 1)


def _same_events(mine, theirs, step):
    assert len(mine) == len(theirs), (step, len(mine), len(theirs))
    assert np.array_equal(mine["a"], theirs["a"]) and np.array_equal(mine["b"], theirs["b"]), step
    assert np.array_equal(mine["type"], theirs["type"]), step
    assert np.array_equal(mine["sensor"], theirs["sensor"]), step
    imp_err = np.abs(mine["impulse"] - theirs["impulse"]) / np.maximum(1.0, np.abs(theirs["impulse"]))
    assert imp_err.max(initial=0.0) <= REL_TOL, (step, imp_err.max())
    pos = theirs["impulse"] > 0
    for f in ("point", "normal"):
        err = np.abs(mine[f][pos] - theirs[f][pos]).max(initial=0.0)
        assert err <= 1e-4, (step, f, err)


def test_sleeping_waking_and_events_follow_the_reference(ref):
    specs, pool, bodies, soup = resting_scene()
    w = ref.RefWorld(specs, pool)
    w.configure(substeps=4, workers=1)
    ctx = velox_b200.Context(0)
    ctx.load(w.bodies(), soup)
    ctx.configure(dt=DT, substeps=4)
    ctx.enable_events(True)
    seen = {"drowsy": 0, "asleep": 0, "woken": 0, "end": 0}
    prev_asleep = None
    for step in range(150):
        w.step(DT, 1)
        ctx.step(1)
        theirs, mine = w.bodies(), ctx.read_bodies()
        err = np.abs(_state(mine) - _state(theirs)) / np.maximum(1.0, np.abs(_state(theirs)))
        assert err.max() <= REL_TOL, (step, float(err.max()))
        assert np.array_equal(mine["asleep"], theirs["asleep"]), (step, np.flatnonzero(mine["asleep"] != theirs["asleep"]))
        assert np.abs(mine["sleepTimer"] - theirs["sleepTimer"]).max() <= 1e-6, step
        _same_events(ctx.read_events(), w.events(), step)
        asleep = theirs["asleep"] == 1
        seen["drowsy"] += int((theirs["asleep"] == 2).any())
        seen["asleep"] += int(asleep.any())
        if prev_asleep is not None:
            seen["woken"] += int((prev_asleep & ~asleep).any())
        seen["end"] += int((w.events()["type"] == 2).any())
        prev_asleep = asleep
    assert all(v > 0 for v in seen.values()), seen
    ctx.close()
    w.close()


def test_sleep_thresholds_are_configurable(ref):
    specs, pool, bodies, soup = resting_scene(projectile=False, non_sleeper=False)
    cfg = binding.SleepConfig.default(timeToSleep=0.25, enableGradualSleep=0, contactStabilityFrames=4)
    w = ref.RefWorld(specs, pool)
    w.configure(substeps=4, workers=1)
    w.sleep_config(cfg)
    ctx = velox_b200.Context(0)
    ctx.load(w.bodies(), soup)
    ctx.configure(dt=DT, substeps=4)
    ctx.configure_sleep(cfg)
    first = None
    for step in range(60):
        w.step(DT, 1)
        ctx.step(1)
        theirs, mine = w.bodies(), ctx.read_bodies()
        assert np.array_equal(mine["asleep"], theirs["asleep"]), step
        assert not (theirs["asleep"] == 2).any()
        if first is None and (theirs["asleep"] == 1).any():
            first = step
    assert first is not None and first < 35
    ctx.close()
    w.close()


def test_batched_sleeping_worlds_equal_the_worlds_alone():
    parts = [resting_scene(seed=s) for s in range(3)]
    bodies = binding.records(np.concatenate([p[2] for p in parts]), binding.BODY)
    world_of = np.concatenate([np.full(len(p[2]), k, np.uint32) for k, p in enumerate(parts)])
    batch = velox_b200.Context(0)
    batch.load(bodies, parts[0][3], world_of=world_of)
    batch.configure(dt=DT, substeps=4)
    alone = []
    for p in parts:
        c = velox_b200.Context(0)
        c.load(p[2], p[3])
        c.configure(dt=DT, substeps=4)
        alone.append(c)
    for _ in range(100):
        batch.step(1)
        for c in alone:
            c.step(1)
    got = batch.read_bodies()
    want = binding.records(np.concatenate([c.read_bodies() for c in alone]), binding.BODY)
    assert np.array_equal(_state(got), _state(want))
    assert np.array_equal(got["asleep"], want["asleep"]) and (got["asleep"] == 1).any()
    batch.close()
    for c in alone:
        c.close()


def test_snapshot_keeps_the_sleep_state():
    specs, pool, bodies, soup = resting_scene()
    ctx = velox_b200.Context(0)
    ctx.load(bodies, soup)
    ctx.configure(dt=DT, substeps=4)
    ctx.step(45)  # a stack asleep, the projectile in flight
    assert (ctx.read_bodies()["asleep"] == 1).any()
    ctx.snapshot_save(0)
    ctx.step(30)
    first = ctx.read_bodies()
    ctx.snapshot_restore(0)
    ctx.step(30)
    again = ctx.read_bodies()
    assert first.tobytes() == again.tobytes()
    ctx.close()
