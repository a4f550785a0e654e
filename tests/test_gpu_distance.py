"""The rewind's distance query. The register-resident GJK (Normal-quality
pairs, separated) must return bit for bit what the general GJK/EPA returns,
and both must match the reference's gjkDistance (include/velox/gjk.h:751-777)
on separated, touching and overlapping pairs of every convex shape (to 1e-5;
same overlap decisions)."""
import numpy as np
import pytest

import velox_b200
from scenes import reference_scene

pytestmark = pytest.mark.gpu


def _pairs(bodies, rng, count):
    dyn = np.where(bodies["shape"] != 1)[0]
    a = rng.choice(dyn, count)
    b = rng.choice(dyn, count)
    keep = a != b
    return (a[keep].astype(np.uint64) << np.uint64(32)) | b[keep].astype(np.uint64)


@pytest.mark.parametrize("kind,size,spread", [("dense", 600, 1.0), (2, 2000, 0.05), (3, 4, 1.0)])
def test_distance_paths_match_reference_gjk(ctx, ref, kind, size, spread):
    w, specs, pool, bodies, soup = reference_scene(ref, kind, size)
    w.close()
    rng = np.random.default_rng(11)
    bodies = bodies.copy()
    if spread != 1.0:  # pull bodies together so that many pairs are close or overlapping
        dyn = bodies["shape"] != 1
        bodies["position"][dyn] *= spread
    pairs = _pairs(bodies, rng, 3000)
    theirs = ref.gjk_distances(bodies, soup, pairs)
    fast = ctx.distance(bodies, soup, pairs, path=0)
    general = ctx.distance(bodies, soup, pairs, path=1)
    assert (theirs[:, 10] == 0).any() and (theirs[:, 10] == 1).any() or kind == 3
    assert np.array_equal(fast.view(np.uint32), general.view(np.uint32))
    assert np.array_equal(general[:, 10], theirs[:, 10])
    assert np.allclose(general[:, :10], theirs[:, :10], rtol=0.0, atol=1e-5)


def test_curved_and_rounded_shapes_match_reference_gjk(ctx, ref):
    # cones, rounded boxes and ellipsoids (absent from the generated scenes)
    # against every other convex shape, separated and overlapping
    w, specs, pool, bodies, soup = reference_scene(ref, "dense", 600)
    w.close()
    rng = np.random.default_rng(3)
    bodies = bodies.copy()
    dyn = np.flatnonzero(bodies["shape"] != 1)
    pick = rng.choice(dyn, len(dyn) // 2, replace=False)
    kinds = rng.choice([8, 9, 10], len(pick))
    bodies["shape"][pick] = kinds
    bodies["halfExtents"][pick] = rng.uniform(0.08, 0.3, (len(pick), 3))
    bodies["radius"][pick] = rng.uniform(0.03, 0.2, len(pick))
    bodies["capsuleHalfHeight"][pick] = rng.uniform(0.08, 0.3, len(pick))
    pairs = _pairs(bodies, rng, 4000)
    theirs = ref.gjk_distances(bodies, soup, pairs)
    fast = ctx.distance(bodies, soup, pairs, path=0)
    general = ctx.distance(bodies, soup, pairs, path=1)
    a = bodies["shape"][(pairs >> np.uint64(32)).astype(np.int64)]
    b = bodies["shape"][(pairs & np.uint64(0xffffffff)).astype(np.int64)]
    curved = np.isin(a, [8, 9, 10]) | np.isin(b, [8, 9, 10])
    assert curved.sum() > 1000 and (theirs[curved, 10] == 1).any() and (theirs[curved, 10] == 0).any()
    assert np.array_equal(fast.view(np.uint32), general.view(np.uint32))
    assert np.array_equal(general[:, 10], theirs[:, 10])
    bad = np.flatnonzero(np.abs(general[:, :10] - theirs[:, :10]).max(1) > 1e-5)
    assert len(bad) == 0, [(int(a[k]), int(b[k]), general[k].tolist(), theirs[k].tolist()) for k in bad[:3]]
