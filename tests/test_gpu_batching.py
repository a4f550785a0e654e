"""Batched worlds (world id in the cell-key high bits, per-world planes,
islands that never cross worlds) step exactly like the same worlds stepped one
at a time, and match the reference step for each world."""
import numpy as np
import pytest

import velox_b200

pytestmark = pytest.mark.gpu
DT = 1.0 / 60.0


def _state(b):
    return np.concatenate([b["position"], b["orientation"], b["velocity"], b["angularVelocity"]], 1)


@pytest.mark.parametrize("config,worlds,steps", [(4, 12, 20), (5, 8, 30)])
def test_batched_worlds_equal_individual_worlds(config, worlds, steps):
    specs, pool = velox_b200.generate_scene(config, size=worlds)
    bodies, hull, faces = velox_b200.bodies_from_specs(specs, pool)
    soup = velox_b200.make_soup(hull, faces)
    batched = velox_b200.Context(0)
    batched.load(bodies, soup, world_of=specs["world"])
    batched.configure(dt=DT, substeps=4)
    batched.step(steps)
    together = batched.read_bodies()
    assert batched.stats()["contacts"] > 0
    batched.close()
    for w in range(worlds):
        sel = np.where(specs["world"] == w)[0]
        sub = np.ascontiguousarray(bodies[sel])
        one = velox_b200.Context(0)
        one.load(sub, soup)
        one.configure(dt=DT, substeps=4)
        one.step(steps)
        alone = one.read_bodies()
        one.close()
        assert np.array_equal(_state(alone), _state(together[sel])), w


def test_batched_world_matches_reference(ref):
    # two worlds of the batching scene; world 1 compared with the reference world
    specs, pool = velox_b200.generate_scene(4, size=2)
    w = ref.RefWorld(specs[specs["world"] == 1], pool)
    pts, faces = w.soup()
    all_bodies, _, _ = velox_b200.bodies_from_specs(specs, pool)
    sel = np.where(specs["world"] == 1)[0]
    all_bodies[sel] = w.bodies()  # world 1 exactly as the reference built it
    ctx = velox_b200.Context(0)
    ctx.load(all_bodies, velox_b200.make_soup(pts, faces), world_of=specs["world"])
    ctx.configure(dt=DT, substeps=4)
    w.configure(substeps=4, workers=1)
    for step in range(3):
        w.step(DT, 1)
        ctx.step(1)
        mine = ctx.read_bodies()[sel]
        theirs = w.bodies()
        err = np.abs(_state(mine) - _state(theirs)) / np.maximum(1.0, np.abs(_state(theirs)))
        assert err.max() <= 1e-4, (step, float(err.max()))
    ctx.close()
