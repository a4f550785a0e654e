"""A settled pile: one island of thousands of contacts (solved by the whole
grid, coloured by the parallel fixed point) with many conservative-advancement
rewinds. Starting from the same pile state, one device step equals one
reference step (the reference's CUDA-backend algorithm run on the CPU)."""
import numpy as np
import pytest

import velox_b200

pytestmark = pytest.mark.gpu
DT = 1.0 / 60.0


def _state(b):
    return np.concatenate([b["position"], b["orientation"], b["velocity"], b["angularVelocity"]], 1)


def test_pile_step_matches_reference(ref):
    # 3000 mixed shapes dropped for 250 steps settle into a pile on the plane
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
    pile = ctx.read_bodies()
    ctx.close()

    w = ref.RefWorld(specs, pool)
    w.configure(substeps=4, workers=1)
    w.set_bodies(pile)
    ctx = velox_b200.Context(0)
    ctx.load(pile, soup)
    ctx.configure(dt=DT, substeps=4)
    for step in range(2):
        w.step(DT, 1)
        ctx.step(1)
        stats = ctx.stats()
        mine, theirs = _state(ctx.read_bodies()), _state(w.bodies())
        err = np.abs(mine - theirs) / np.maximum(1.0, np.abs(theirs))
        assert err.max() <= 1e-4, (step, float(err.max()))
        assert stats["contacts"] == w.stats()["generated"]
    ctx.close()
    w.close()
    # the paths this test exists for were taken
    assert stats["giantIslands"] >= 1
    assert stats["colorRounds"] > 0
    assert stats["rewinds"] > 0


def test_two_piles_in_two_worlds_match_reference(ref):
    # the same 2,500-body scene in two worlds: two giant islands at once (the
    # clustered solve over several islands), each world equal to the reference
    specs, pool = velox_b200.generate_scene(2, size=2500)
    w = ref.RefWorld(specs, pool)
    start = w.bodies()
    pts, faces = w.soup()
    w.close()
    soup = velox_b200.make_soup(pts, faces)
    n = len(start)
    both = np.concatenate([start, start])
    world_of = np.repeat(np.arange(2, dtype=np.uint32), n)
    ctx = velox_b200.Context(0)
    ctx.load(both, soup, world_of=world_of)
    ctx.configure(dt=DT, substeps=4)
    ctx.step(220)
    piles = ctx.read_bodies()
    ctx.close()
    assert np.array_equal(_state(piles[:n]), _state(piles[n:]))
    # one step from the piles on both engines (fresh contact caches on both)
    w = ref.RefWorld(specs, pool)
    w.configure(substeps=4, workers=1)
    w.set_bodies(piles[:n])
    w.step(DT, 1)
    ctx = velox_b200.Context(0)
    ctx.load(piles, soup, world_of=world_of)
    ctx.configure(dt=DT, substeps=4)
    ctx.step(1)
    stats = ctx.stats()
    out = ctx.read_bodies()
    ctx.close()
    theirs = _state(w.bodies())
    w.close()
    assert stats["giantIslands"] >= 2
    for half in (out[:n], out[n:]):
        err = np.abs(_state(half) - theirs) / np.maximum(1.0, np.abs(theirs))
        assert err.max() <= 1e-4, float(err.max())
