"""Launch-shape autotuning of the narrow phase and the rewind probe
(vxb_context_set_tuning): every shape the tuner explores gives the same
contacts and body state as the fixed default shape, a size bucket is decided
after two timings of each of its six candidates, the decision reaches the
cache file, and a new context starts from the cached shape."""
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
    shapes = set()
    # the timing of call k is folded in at call k + 1: one call more than the samples
    for call in range(CANDIDATES * SAMPLES + 1):
        t, b, decided = tuned.tuned_shape("collide_any", len(pairs))
        assert not decided
        shapes.add((t, b))
        got, counts = tuned.collide(bodies, soup, pairs, DT)
        _same(got, want, f"contacts, call {call} with {t} threads x {b} blocks/SM")
        assert np.array_equal(counts, want_counts)
    assert len(shapes) == CANDIDATES
    chosen = tuned.tuned_shape("collide_any", len(pairs))
    assert chosen[2]
    assert (chosen[0], chosen[1]) in shapes
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


def test_world_steps_are_identical_while_the_tuner_explores(tmp_path, monkeypatch):
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
    assert tuned.host_syncs > 0 and tuned.host_syncs == fixed.host_syncs
    for ctx in worlds:
        ctx.close()
