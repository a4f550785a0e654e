"""Snapshots of the device world (World::saveSnapshot / restoreSnapshot,
src/world.cpp:2038-2128): after a restore, stepping repeats the original
steps bit for bit — body state and the contacts with their warm-start
impulses — from a device slot and from a byte image in another context."""
import numpy as np
import pytest

import velox_b200
from scenes import scene

pytestmark = pytest.mark.gpu
DT = 1.0 / 60.0


def _setup(kind="dense", size=600, world_of=None):
    specs, pool = scene(kind, size)
    bodies, hull, faces = velox_b200.bodies_from_specs(specs, pool)
    soup = velox_b200.make_soup(hull, faces)
    ctx = velox_b200.Context(0)
    ctx.load(bodies, soup, world_of=world_of if world_of is not None else None)
    ctx.configure(dt=DT, substeps=4)
    return ctx, bodies, soup


def _state(ctx):
    return ctx.read_bodies(), ctx.read_contacts()


def _same(x, y):
    """Bit-identical body and contact images; on a mismatch, names the fields."""
    for got, want in zip(x, y):
        if got.tobytes() == want.tobytes():
            continue
        assert len(got) == len(want), (len(got), len(want))
        fields = [f for f in want.dtype.names if got[f].tobytes() != want[f].tobytes()]
        raise AssertionError(f"differs in {fields or 'padding bytes'}")


def test_device_slot_rollback_repeats_the_steps():
    ctx, _, _ = _setup()
    ctx.step(5)
    ctx.snapshot_save(0)
    ctx.step(10)
    first = _state(ctx)
    assert ctx.stats()["contacts"] > 0
    ctx.snapshot_restore(0)
    ctx.step(10)
    _same(_state(ctx), first)
    ctx.snapshot_restore(0)  # a slot survives a restore
    ctx.step(10)
    _same(_state(ctx), first)
    ctx.close()


def test_byte_image_restores_into_another_context():
    ctx, bodies, soup = _setup("dense", 500)
    ctx.step(7)
    image = ctx.snapshot_bytes()
    other = velox_b200.Context(0)
    other.load(bodies, soup)
    other.configure(dt=DT, substeps=8)  # replaced by the image's configuration
    other.snapshot_load(image)
    ctx.step(6)
    other.step(6)
    _same(_state(other), _state(ctx))
    ctx.close()
    other.close()


def test_incompatible_image_is_rejected():
    ctx, _, _ = _setup("dense", 300)
    ctx.step(2)
    image = ctx.snapshot_bytes()
    other, _, _ = _setup("dense", 400)
    with pytest.raises(velox_b200.VeloxError) as info:
        other.snapshot_load(image)
    assert info.value.status == 1
    with pytest.raises(velox_b200.VeloxError):
        other.snapshot_load(image[:16])
    with pytest.raises(velox_b200.VeloxError):
        other.snapshot_restore(3)  # empty slot
    ctx.close()
    other.close()
