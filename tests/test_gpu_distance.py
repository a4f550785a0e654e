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
