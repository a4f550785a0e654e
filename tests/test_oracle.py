"""The C restatement of the integer stages (oracle/velox_oracle.c) against the
reference engine compiled from its sources, on seeded workloads (CPU)."""
import numpy as np
import pytest

import ref as refmod
from scenes import reference_scene

DT = 1.0 / 60.0


@pytest.mark.parametrize("kind,size", [(1, 0), (2, 3000), (3, 2), (4, 8), ("dense", 800)])
def test_oracle_pair_set_matches_reference(ref, kind, size):
    w, specs, pool, bodies, soup = reference_scene(ref, kind, size)
    assert np.array_equal(ref.oracle_pairs(bodies, DT), ref.candidate_pairs(bodies, DT))


def test_oracle_pair_set_after_motion(ref):
    w, specs, pool, bodies, soup = reference_scene(ref, "dense", 600)
    w.configure(workers=1)
    w.step(DT, 5)
    b = w.bodies()
    assert np.array_equal(ref.oracle_pairs(b, DT), ref.candidate_pairs(b, DT))


@pytest.mark.parametrize("kind,size", [(3, 2), ("dense", 1500), (1, 0)])
def test_oracle_sort_and_coloring_match_reference(ref, kind, size):
    w, specs, pool, bodies, soup = reference_scene(ref, kind, size)
    contacts, _ = ref.collide_pairs(bodies, soup, ref.candidate_pairs(bodies, DT), DT)
    shuffled = contacts[np.random.default_rng(1).permutation(len(contacts))]
    mine = ref.oracle_sort(shuffled)
    theirs = ref.sort_contacts(shuffled)
    # payload bytes (the trailing 8 bytes of each 128-byte record are padding)
    assert np.array_equal(mine.view(np.uint8).reshape(-1, 128)[:, :120],
                          theirs.view(np.uint8).reshape(-1, 128)[:, :120])
    c1, n1 = ref.oracle_color(bodies, mine)
    c2, n2 = ref.color_contacts(bodies, theirs)
    assert n1 == n2 and np.array_equal(c1, c2)
    order, starts = ref.oracle_color_order(c1, n1)
    assert np.all(np.diff(c1[order]) >= 0)
    assert starts[-1] == len(c1)


def test_coloring_spill_rule_over_64_colours(ref):
    # 80 coincident spheres: every pair touches (the reference's dense-capacity
    # case), forcing the >64-colour spill path.
    import velox_b200
    specs, pool = velox_b200.generate_scene(2, size=80)
    specs["position"][1:] = (0.0, 1.0, 0.0)
    specs["shape"][1:] = 0
    specs["radius"][1:] = 0.5
    specs["mass"][1:] = 1.0
    w = ref.RefWorld(specs, pool)
    bodies = w.bodies()
    pts, faces = w.soup()
    soup = velox_b200.make_soup(pts, faces)
    contacts, _ = ref.collide_pairs(bodies, soup, ref.candidate_pairs(bodies, DT), DT)
    contacts = ref.sort_contacts(contacts)
    c1, n1 = ref.oracle_color(bodies, contacts)
    c2, n2 = ref.color_contacts(bodies, contacts)
    assert n1 > 64 and n1 == n2 and np.array_equal(c1, c2)


def test_oracle_warm_start_match_semantics(ref):
    w, specs, pool, bodies, soup = reference_scene(ref, 3, 1)
    contacts, _ = ref.collide_pairs(bodies, soup, ref.candidate_pairs(bodies, DT), DT)
    prev = ref.oracle_sort(contacts)
    prev["normalImpulse"] = np.arange(len(prev), dtype=np.float32) + 1
    cur = prev.copy()
    cur["normalImpulse"] = 0
    out, warm = ref.oracle_warm_start(cur, prev)
    assert warm == len(cur)
    assert np.array_equal(out["normalImpulse"], prev["normalImpulse"])
    # feature keys cleared -> proximity match within 5 cm picks the same point
    cur2 = cur.copy()
    cur2["featureKey"] = 0
    out2, warm2 = ref.oracle_warm_start(cur2, prev)
    assert warm2 == len(cur)
    # a far-away point does not inherit
    cur3 = cur2.copy()
    cur3["point"][:, 1] += 10.0
    out3, warm3 = ref.oracle_warm_start(cur3, prev)
    assert warm3 == 0 and np.all(out3["normalImpulse"] == 0)


def test_oracle_pairs_on_empty_and_single_body_inputs(ref):
    w, specs, pool, bodies, soup = reference_scene(ref, "dense", 200)
    plane = bodies[bodies["shape"] == 1]
    one = bodies[bodies["shape"] != 1][:1]
    for b in (bodies[:0], plane, one, np.concatenate([plane, one])):
        b = np.ascontiguousarray(b)
        mine, theirs = ref.oracle_pairs(b, DT), ref.candidate_pairs(b, DT)
        assert np.array_equal(mine, theirs)
    # one body resting on the plane pairs with it
    assert len(ref.candidate_pairs(np.ascontiguousarray(np.concatenate([plane, one])), DT)) <= 1


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_oracle_pairs_under_filters_static_and_sleeping_bodies(ref, seed):
    # collision groups, category/mask bits, static and sleeping bodies: the
    # pair filter (Body::canCollideWith and the inert-pair rule) on both sides
    w, specs, pool, bodies, soup = reference_scene(ref, "dense", 800)
    rng = np.random.default_rng(seed)
    b = bodies.copy()
    dyn = np.flatnonzero(b["shape"] != 1)
    b["groupIndex"][dyn] = rng.choice([0, 0, 0, 1, -1, 2, -2], len(dyn))
    b["categoryBits"][dyn] = rng.choice([1, 2, 4, 0xffff], len(dyn))
    b["maskBits"][dyn] = rng.choice([0xffff, 0xffff, 1 | 4, 2, 0], len(dyn))
    b["motionType"][rng.choice(dyn, len(dyn) // 10, replace=False)] = 0  # static
    b["asleep"][rng.choice(dyn, len(dyn) // 10, replace=False)] = 1
    mine, theirs = ref.oracle_pairs(b, DT), ref.candidate_pairs(b, DT)
    assert len(theirs) > 0 and np.array_equal(mine, theirs)
    assert len(theirs) < len(ref.candidate_pairs(bodies, DT))  # the filters removed pairs


def test_oracle_coloring_with_static_endpoints(ref):
    # contacts against static bodies do not constrain colours; the restatement
    # and the reference agree on which endpoints count
    w, specs, pool, bodies, soup = reference_scene(ref, "dense", 1200)
    contacts, _ = ref.collide_pairs(bodies, soup, ref.candidate_pairs(bodies, DT), DT)
    contacts = ref.sort_contacts(contacts)
    b = bodies.copy()
    dyn = np.flatnonzero(b["shape"] != 1)
    b["motionType"][np.random.default_rng(3).choice(dyn, len(dyn) // 4, replace=False)] = 0
    c1, n1 = ref.oracle_color(b, contacts)
    c2, n2 = ref.color_contacts(b, contacts)
    assert n1 == n2 and np.array_equal(c1, c2)
    full, nfull = ref.color_contacts(bodies, contacts)
    assert n2 <= nfull
