"""Solver and geometry branches beyond the reference's defaults, and long
runs, against the reference engine compiled from its sources (strict floating
point, its CUDA backend's coloured algorithm run on the CPU):

* rolling and spinning friction (src/narrowphase.h:324-359),
* the cone-block friction model (src/narrowphase.h:260-319),
* anisotropic friction scale (src/narrowphase.h:68-75),
* Robust and Paranoid geometry quality (GJK re-seeding, include/velox/gjk.h:751-777),
* 30-step whole runs of the dense and pyramid scenes,
* one step of the 100,001-body benchmark scene from a settled device state.

Per-step body state must stay within 1e-4 relative (the whole-step bar)."""
import numpy as np
import pytest

import velox_b200
from velox_b200 import binding
from scenes import reference_scene

pytestmark = pytest.mark.gpu
DT = 1.0 / 60.0
REL_TOL = 1e-4


def _state(b):
    return np.concatenate([b["position"], b["orientation"], b["velocity"], b["angularVelocity"]], 1)


def _rel_err(mine, theirs):
    a, b = _state(mine), _state(theirs)
    return float((np.abs(a - b) / np.maximum(1.0, np.abs(b))).max())


def _run_both(ref, bodies, soup, specs, pool, steps, substeps=4, solver=None, check_every=1):
    w = ref.RefWorld(specs, pool)
    w.configure(substeps=substeps, workers=1, solver=solver)
    w.set_bodies(bodies)
    ctx = velox_b200.Context(0)
    ctx.load(bodies, soup)
    ctx.configure(dt=DT, substeps=substeps, solver=solver)
    worst, contacts = 0.0, 0
    for step in range(steps):
        w.step(DT, 1)
        ctx.step(1)
        contacts = max(contacts, ctx.stats()["contacts"])
        if (step + 1) % check_every == 0 or step == steps - 1:
            err = _rel_err(ctx.read_bodies(), w.bodies())
            worst = max(worst, err)
            assert err <= REL_TOL, (step, err)
    ctx.close()
    w.close()
    return worst, contacts


def _with(bodies, **fields):
    b = bodies.copy()
    dyn = b["shape"] != binding.SHAPE["plane"]
    for name, value in fields.items():
        col = b[name]
        if callable(value):
            col[dyn] = value(int(dyn.sum()))
        else:
            col[dyn] = value
    return b


@pytest.mark.parametrize("rolling,spinning", [(0.05, 0.0), (0.0, 0.04), (0.03, 0.02)])
def test_rolling_and_spinning_friction(ref, rolling, spinning):
    w, specs, pool, bodies, soup = reference_scene(ref, "dense", 600)
    w.close()
    b = _with(bodies, rollingFriction=rolling, spinningFriction=spinning)
    _, contacts = _run_both(ref, b, soup, specs, pool, steps=6)
    assert contacts > 0


@pytest.mark.parametrize("kind,size", [("dense", 600), (3, 2)])
def test_cone_block_friction_model(ref, kind, size):
    w, specs, pool, bodies, soup = reference_scene(ref, kind, size)
    w.close()
    solver = binding.SolverOptions.default(frictionModel=1)  # FrictionModel::ConeBlockSolver
    _, contacts = _run_both(ref, bodies, soup, specs, pool, steps=6, solver=solver)
    assert contacts > 0


def test_cone_block_with_rolling_and_spinning(ref):
    w, specs, pool, bodies, soup = reference_scene(ref, "dense", 500)
    w.close()
    b = _with(bodies, rollingFriction=0.02, spinningFriction=0.02)
    solver = binding.SolverOptions.default(frictionModel=1)
    _run_both(ref, b, soup, specs, pool, steps=5, solver=solver)


def test_anisotropic_friction_scale(ref):
    w, specs, pool, bodies, soup = reference_scene(ref, "dense", 600)
    w.close()
    rng = np.random.default_rng(3)
    b = _with(bodies, frictionScale=lambda k: rng.uniform(0.3, 2.0, (k, 3)).astype(np.float32))
    _, contacts = _run_both(ref, b, soup, specs, pool, steps=6)
    assert contacts > 0


@pytest.mark.parametrize("quality", [1, 2])  # GeometryQuality::Robust, ::Paranoid
def test_robust_and_paranoid_geometry_quality(ctx, ref, quality):
    w, specs, pool, bodies, soup = reference_scene(ref, "dense", 600)
    w.close()
    b = _with(bodies, geometryQuality=quality)
    # the narrow phase with re-seeded GJK against the reference's, pair by pair
    pairs = ref.candidate_pairs(b, DT)
    theirs, tcounts = ref.collide_pairs(b, soup, pairs, DT)
    mine, mcounts = ctx.collide(b, soup, pairs, DT)
    assert len(theirs) > 0
    assert np.array_equal(mcounts, tcounts)
    assert np.array_equal(mine["featureKey"], theirs["featureKey"])
    for f in ("point", "localAnchorA", "localAnchorB", "gap", "bias0"):
        assert np.abs(mine[f] - theirs[f]).max() <= 1e-5, f
    # the distance query itself (the rewind's path and the general path)
    keys = pairs[:400]
    want = ref.gjk_distances(b, soup, keys)
    for path in (0, 1):
        got = ctx.distance(b, soup, keys, path=path)
        assert np.array_equal(got[:, 10], want[:, 10])
        assert np.abs(got[:, :10] - want[:, :10]).max() <= 1e-5
    # and whole steps
    _run_both(ref, b, soup, specs, pool, steps=4)


@pytest.mark.parametrize("kind,size,substeps", [("dense", 600, 4), (3, 2, 8)])
def test_thirty_step_runs(ref, kind, size, substeps):
    w, specs, pool, bodies, soup = reference_scene(ref, kind, size)
    w.close()
    _, contacts = _run_both(ref, bodies, soup, specs, pool, steps=30, substeps=substeps)
    assert contacts > 0


def test_benchmark_scene_step_from_a_settled_state(ref):
    # The 100,001-body benchmark scene after 200 device steps (a pile on the
    # plane): one more step from that state equals the reference's step.
    specs, pool = velox_b200.generate_scene(2)
    w = ref.RefWorld(specs, pool)
    start = w.bodies()
    pts, faces = w.soup()
    soup = velox_b200.make_soup(pts, faces)
    ctx = velox_b200.Context(0)
    ctx.load(start, soup)
    ctx.configure(dt=DT, substeps=4)
    ctx.step(200)
    state = ctx.read_bodies()
    ctx.close()
    w.configure(substeps=4, workers=1)
    w.set_bodies(state)
    ctx = velox_b200.Context(0)
    ctx.load(state, soup)
    ctx.configure(dt=DT, substeps=4)
    w.step(DT, 1)
    ctx.step(1)
    stats = ctx.stats()
    err = _rel_err(ctx.read_bodies(), w.bodies())
    assert stats["contacts"] == w.stats()["generated"]
    ctx.close()
    w.close()
    assert stats["contacts"] > 100000
    assert err <= REL_TOL, err
