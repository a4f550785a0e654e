"""Parity of the CUDA pipeline (through the C ABI) against the reference
engine compiled from its sources (strict floating point), stage by stage and
for whole steps."""
import numpy as np
import pytest

import velox_b200
from velox_b200 import binding
from scenes import reference_scene

pytestmark = pytest.mark.gpu
DT = 1.0 / 60.0

# Geometry tolerances of the parity bar: positions/depths 1e-5 m, normals 1e-4 rad.
POS_TOL = 1e-5
ANGLE_TOL = 1e-4


@pytest.mark.parametrize("kind,size", [(1, 0), (2, 3000), (3, 2), (4, 8), ("dense", 800)])
def test_broadphase_pairs_bit_exact(ctx, ref, kind, size):
    w, specs, pool, bodies, soup = reference_scene(ref, kind, size)
    mine = ctx.pairs(bodies, DT)
    theirs = ref.candidate_pairs(bodies, DT)
    assert len(theirs) > 0
    assert np.array_equal(mine, theirs)


def _compare_contacts(mine, theirs):
    assert len(mine) == len(theirs)
    if len(mine) == 0:
        return
    assert np.array_equal(mine["a"], theirs["a"])
    assert np.array_equal(mine["b"], theirs["b"])
    assert np.array_equal(mine["featureKey"], theirs["featureKey"])
    for f in ("point", "localAnchorA", "localAnchorB"):
        assert np.abs(mine[f] - theirs[f]).max() <= POS_TOL, f
    for f in ("gap", "bias0"):
        assert np.abs(mine[f] - theirs[f]).max() <= POS_TOL, f
    a = mine["normal"].astype(np.float64)
    b = theirs["normal"].astype(np.float64)
    angle = np.arctan2(np.linalg.norm(np.cross(a, b), axis=1), np.sum(a * b, 1))
    assert angle.max() <= ANGLE_TOL
    for f in ("vn0", "restitution", "friction1", "friction2"):
        assert np.allclose(mine[f], theirs[f], rtol=1e-5, atol=1e-5), f


@pytest.mark.parametrize("kind,size", [(1, 0), (3, 2), ("dense", 800), ("dense", 2000)])
def test_narrowphase_matches_reference(ctx, ref, kind, size):
    w, specs, pool, bodies, soup = reference_scene(ref, kind, size)
    pairs = ref.candidate_pairs(bodies, DT)
    theirs, tcounts = ref.collide_pairs(bodies, soup, pairs, DT)
    mine, mcounts = ctx.collide(bodies, soup, pairs, DT)
    assert len(theirs) > 0
    assert np.array_equal(mcounts, tcounts)
    _compare_contacts(mine, theirs)


@pytest.mark.parametrize("kind,size", [(3, 3), ("dense", 2000), (1, 0)])
def test_coloring_bit_exact_given_contact_order(ctx, ref, kind, size):
    w, specs, pool, bodies, soup = reference_scene(ref, kind, size)
    pairs = ref.candidate_pairs(bodies, DT)
    contacts, _ = ref.collide_pairs(bodies, soup, pairs, DT)
    contacts = ref.sort_contacts(contacts)
    theirs, tn = ref.color_contacts(bodies, contacts)
    mine, mn = ctx.color(bodies, contacts)
    assert len(contacts) > 0
    assert mn == tn
    assert np.array_equal(mine, theirs)


def _state(b):
    return np.concatenate([b["position"], b["orientation"], b["velocity"], b["angularVelocity"]], 1)


@pytest.mark.parametrize("kind,size,substeps", [(3, 2, 8), ("dense", 600, 4), (1, 4, 4)])
def test_world_step_matches_reference_cuda_semantics(ref, kind, size, substeps):
    w, specs, pool, bodies, soup = reference_scene(ref, kind, size)
    w.configure(substeps=substeps, workers=1)
    ctx = velox_b200.Context(0)
    ctx.load(bodies, soup)
    ctx.configure(dt=DT, substeps=substeps)
    for step in range(3):
        w.step(DT, 1)
        ctx.step(1)
        rb, mb = w.bodies(), ctx.read_bodies()
        scale = np.maximum(1.0, np.abs(_state(rb)))
        err = np.abs(_state(mb) - _state(rb)) / scale
        assert err.max() <= 1e-4, (step, float(err.max()))
    st = ctx.stats()
    assert st["contacts"] > 0
    ctx.close()


def test_coloring_past_64_colours_in_a_large_island(ctx, ref):
    # 50 overlapping big spheres in a row, each crowded by 90 small ones: one
    # island of more than 4096 contacts (parallel colouring) needing > 64 colours
    rng = np.random.default_rng(5)
    spec = velox_b200.binding.SPEC
    specs = np.zeros(50 + 50 * 90, spec)
    specs["orientation"] = (0, 0, 0, 1)
    specs["mass"] = 1.0
    specs["friction"] = 0.5
    specs["planeNormal"] = (0, 1, 0)
    specs["radius"][:50] = 2.0
    specs["position"][:50, 0] = 3.5 * np.arange(50)
    d = rng.normal(size=(50 * 90, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    centres = np.repeat(specs["position"][:50], 90, axis=0)
    specs["radius"][50:] = 0.3
    specs["position"][50:] = centres + 2.0 * d
    bodies, _, _ = velox_b200.bodies_from_specs(specs, np.zeros((1, 3), np.float32))
    soup = velox_b200.make_soup(np.zeros((1, 3), np.float32), np.zeros(1, np.uint32))
    pairs = ref.candidate_pairs(bodies, DT)
    contacts, _ = ref.collide_pairs(bodies, soup, pairs, DT)
    contacts = ref.sort_contacts(contacts)
    theirs, tn = ref.color_contacts(bodies, contacts)
    mine, mn = ctx.color(bodies, contacts)
    assert len(contacts) > 4096 and tn > 64
    assert mn == tn
    assert np.array_equal(mine, theirs)


@pytest.mark.parametrize("seed", [0, 1])
def test_pairs_and_colours_under_filters_static_and_sleeping_bodies(ctx, ref, seed):
    # collision groups, category/mask bits, static and sleeping bodies: the
    # device pair filter and the colouring's endpoints against the reference
    w, specs, pool, bodies, soup = reference_scene(ref, "dense", 800)
    rng = np.random.default_rng(seed)
    b = bodies.copy()
    dyn = np.flatnonzero(b["shape"] != 1)
    b["groupIndex"][dyn] = rng.choice([0, 0, 0, 1, -1, 2, -2], len(dyn))
    b["categoryBits"][dyn] = rng.choice([1, 2, 4, 0xffff], len(dyn))
    b["maskBits"][dyn] = rng.choice([0xffff, 0xffff, 1 | 4, 2, 0], len(dyn))
    b["motionType"][rng.choice(dyn, len(dyn) // 10, replace=False)] = 0  # static
    b["asleep"][rng.choice(dyn, len(dyn) // 10, replace=False)] = 1
    theirs = ref.candidate_pairs(b, DT)
    assert len(theirs) > 0
    assert np.array_equal(ctx.pairs(b, DT), theirs)
    contacts, _ = ref.collide_pairs(b, soup, theirs, DT)
    contacts = ref.sort_contacts(contacts)
    tc, tn = ref.color_contacts(b, contacts)
    mc, mn = ctx.color(b, contacts)
    assert len(contacts) > 0 and mn == tn
    assert np.array_equal(mc, tc)
