"""Launch-shape autotuning of the narrow phase and the rewind probe
(vxb_context_set_tuning): the first launch in a size bucket runs the six
candidate shapes twice on the same inputs and keeps the fastest; the trials
leave the contacts and body state bit-identical to the fixed default shape,
the decision reaches the cache file, and a new context starts from the cached
shape."""
import numpy as np
import pytest

import velox_b200
from scenes import scene

pytestmark = pytest.mark.gpu
DT = 1.0 / 60.0
CANDIDATES = 6
SAMPLES = 2


def _dense(size=600):
    specs, pool = scene("dense", size)
    bodies, hull, faces = velox_b200.bodies_from_specs(specs, pool)
    return bodies, velox_b200.make_soup(hull, faces)


def _same(got, want, what):
    if got.tobytes() == want.tobytes():
        return
    assert len(got) == len(want), (what, len(got), len(want))
    fields = [f for f in want.dtype.names if got[f].tobytes() != want[f].tobytes()]
    raise AssertionError(f"{what}: differs in {fields or 'padding bytes'}")


def test_explored_shapes_give_the_default_contacts_and_the_decision_is_cached(tmp_path, monkeypatch):
    cache = tmp_path / "launch_shapes.txt"
    monkeypatch.setenv("VXB_TUNE_CACHE", str(cache))
    bodies, soup = _dense()
    fixed = velox_b200.Context(0)
    fixed.set_tuning(False)
    pairs = fixed.pairs(bodies, DT, soup)
    assert len(pairs) > 100
    want, want_counts = fixed.collide(bodies, soup, pairs, DT)
    assert len(want) > 0
    assert fixed.tuned_shape("collide_any", len(pairs)) == (128, 16, True)
    fixed.close()

    tuned = velox_b200.Context(0)
    assert tuned.tuned_shape("collide_any", len(pairs)) == (128, 16, False)
    launches = tuned.launches
    for call in range(3):
        got, counts = tuned.collide(bodies, soup, pairs, DT)
        _same(got, want, f"contacts, call {call}")
        assert np.array_equal(counts, want_counts)
        if call == 0:  # the trials: every candidate twice, then the real launch
            trial_launches = tuned.launches - launches
        launches = tuned.launches
    chosen = tuned.tuned_shape("collide_any", len(pairs))
    assert chosen[2]
    assert (chosen[0], chosen[1]) in {(128, 16), (64, 32), (32, 64), (128, 2), (64, 4), (32, 8)}
    fixed_launches = velox_b200.Context(0)
    fixed_launches.set_tuning(False)
    before = fixed_launches.launches
    fixed_launches.collide(bodies, soup, pairs, DT)
    assert trial_launches - (fixed_launches.launches - before) == CANDIDATES * SAMPLES
    fixed_launches.close()
    tuned.close()  # writes the decisions

    lines = [ln.split() for ln in cache.read_text().splitlines() if not ln.startswith("#")]
    bucket = int(np.floor(np.log2(len(pairs))))
    assert [ln[1:] for ln in lines if ln[1] == "collide_any"] == [
        ["collide_any", str(bucket), str(chosen[0]), str(chosen[1])]]
    again = velox_b200.Context(0)
    assert again.tuned_shape("collide_any", len(pairs)) == chosen
    got, _ = again.collide(bodies, soup, pairs, DT)
    _same(got, want, "contacts from the cached shape")
    again.close()


def test_world_steps_are_identical_with_the_tuner_trials(tmp_path, monkeypatch):
    monkeypatch.setenv("VXB_TUNE_CACHE", str(tmp_path / "launch_shapes.txt"))
    bodies, soup = _dense(600)
    worlds = []
    for on in (False, True):
        ctx = velox_b200.Context(0)
        ctx.set_tuning(on)
        ctx.load(bodies, soup)
        ctx.configure(dt=DT, substeps=4)
        worlds.append(ctx)
    fixed, tuned = worlds
    probes = 0
    for step in range(30):
        for ctx in worlds:
            ctx.step(1)
        st = fixed.stats()
        probes += st["contacts"] > 0
        if step % 5 == 4:
            _same(tuned.read_bodies(), fixed.read_bodies(), f"bodies after step {step + 1}")
            _same(tuned.read_contacts(), fixed.read_contacts(), f"contacts after step {step + 1}")
    assert probes > CANDIDATES
    # each decided bucket adds one wait per trial
    extra = tuned.host_syncs - fixed.host_syncs
    assert fixed.host_syncs > 0 and extra > 0 and extra % (CANDIDATES * SAMPLES) == 0
    for ctx in worlds:
        ctx.close()
