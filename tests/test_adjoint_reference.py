"""The FP64 restatement of the frozen-contact step and its hand-derived
adjoint (oracle/adjoint_ref.c) against FP64 central finite differences, on the
CPU. Contacts are the reference narrow phase's (ref.collide_pairs) for a small
stack hit by a sphere, frozen over the rollout (each contact warm-starts from
its own previous impulses)."""
import numpy as np
import pytest

import velox_b200
from velox_b200 import binding

DT = 1.0 / 60.0


def _scene(seed=0):
    spec = binding.SPEC
    specs = np.zeros(6, spec)
    specs["orientation"] = (0, 0, 0, 1)
    specs["friction"] = 0.5
    specs["restitution"] = 0.3
    specs["planeNormal"] = (0, 1, 0)
    specs["shape"][0] = binding.SHAPE["plane"]
    rng = np.random.default_rng(seed)
    for k in range(1, 5):
        specs["shape"][k] = binding.SHAPE["box"]
        specs["halfExtents"][k] = 0.5
        specs["mass"][k] = 1.0
        # slight overlaps (position corrections) and small generic velocities: a
        # stack exactly at rest sits on the clamp's kink (zero impulse, zero
        # approach speed), where the step has no derivative
        specs["position"][k] = (0.01 * k, 0.4985 + (k - 1) * 1.0 - 0.002 * (k - 1), -0.005 * k)
        specs["velocity"][k] = rng.normal(scale=0.02, size=3)
        specs["angularVelocity"][k] = rng.normal(scale=0.02, size=3)
    specs["shape"][5] = binding.SHAPE["sphere"]
    specs["radius"][5] = 0.3
    specs["mass"][5] = 2.0
    specs["position"][5] = (-0.83, 1.4, 0.05)
    specs["velocity"][5] = (3.0, 0.5, 0.2)
    specs["angularVelocity"][5] = (0.1, -0.4, 0.3)
    bodies, hull, faces = velox_b200.bodies_from_specs(specs, np.zeros((1, 3), np.float32))
    return bodies, velox_b200.make_soup(hull, faces)


def _frozen_rollout_inputs(ref, steps):
    bodies, soup = _scene()
    pairs = ref.candidate_pairs(bodies, DT)
    contacts, _ = ref.collide_pairs(bodies, soup, pairs, DT)
    contacts = ref.sort_contacts(contacts)
    colors, _ = ref.color_contacts(bodies, contacts)
    m = len(contacts)
    allc = np.concatenate([contacts] * steps)
    step_start = np.arange(steps + 1, dtype=np.uint32) * m
    src = np.full((steps * m, 2), 0xffffffff, np.uint32)
    src[m:, 0] = np.tile(np.arange(m, dtype=np.uint32), steps - 1)  # warm start from the same contact
    color = np.tile(colors, steps).astype(np.int32)
    state0 = np.concatenate([bodies["position"], bodies["orientation"], bodies["velocity"],
                             bodies["angularVelocity"]], 1).astype(np.float64)
    return bodies, allc, step_start, src, color, state0


def _loss(ref, cfg, bodies, state0, im, ii, c, ss, src, col, seed):
    out, h = ref.adjoint_reference(cfg, bodies, state0, im, ii, c, ss, src, col)
    return float(np.sum(out * seed)), h


def test_adjoint_restatement_matches_central_differences(ref):
    steps = 12
    bodies, c, ss, src, col, state0 = _frozen_rollout_inputs(ref, steps)
    assert len(c) > 0
    cfg = ref.AdjConfig.make()
    im = bodies["invMass"].astype(np.float64)
    ii = bodies["invInertia"][:, 0].astype(np.float64)
    rng = np.random.default_rng(1)
    seed = rng.normal(size=state0.shape)
    dyn = bodies["motionType"] == 2
    seed[~dyn] = 0.0
    _, h0, grad, gim, gii = ref.adjoint_reference(cfg, bodies, state0, im, ii, c, ss, src, col, seed=seed)
    assert np.isfinite(grad).all()
    checked = 0
    for trial in range(16):
        ds = rng.normal(size=state0.shape)
        ds[~dyn] = 0.0
        ds[:, 3:7] = 0.0 if trial % 2 == 0 else ds[:, 3:7]
        dim = rng.normal(size=im.shape) * dyn * 0.1
        dii = rng.normal(size=ii.shape) * dyn * 0.1
        predicted = np.sum(grad * ds) + np.sum(gim * dim) + np.sum(gii * dii)
        # Near-sliding contacts put the friction ellipse's projection at its
        # boundary (E == 1), a kink of the step: stencils that straddle a kink
        # change the branch hash and are not smooth points. A tight stencil
        # (1e-7) checks the algebra; the 1e-4 stencil is the FD bar.
        for eps, tol in [(1e-7, 1e-5), (1e-4, 1e-3)]:
            lp, hp = _loss(ref, cfg, bodies, state0 + eps * ds, im + eps * dim, ii + eps * dii, c, ss, src, col, seed)
            lm, hm = _loss(ref, cfg, bodies, state0 - eps * ds, im - eps * dim, ii - eps * dii, c, ss, src, col, seed)
            if hp != h0 or hm != h0:
                continue  # an active set changed inside the stencil: not a smooth point
            fd = (lp - lm) / (2 * eps)
            assert abs(fd - predicted) <= tol * max(1.0, abs(fd)), (trial, eps, fd, predicted)
            checked += 1
    assert checked >= 6


def test_adjoint_restatement_per_parameter(ref):
    # dL/d(sphere velocity) and dL/d(masses) one coordinate at a time
    steps = 10
    bodies, c, ss, src, col, state0 = _frozen_rollout_inputs(ref, steps)
    cfg = ref.AdjConfig.make()
    im = bodies["invMass"].astype(np.float64)
    ii = bodies["invInertia"][:, 0].astype(np.float64)
    seed = np.zeros_like(state0)
    seed[1:5, 0:3] = np.random.default_rng(2).normal(size=(4, 3))  # box positions
    _, h0, grad, gim, gii = ref.adjoint_reference(cfg, bodies, state0, im, ii, c, ss, src, col, seed=seed)
    eps = 1e-7
    checked = 0
    for (i, j) in [(5, 7), (5, 8), (5, 9), (5, 10), (5, 11), (5, 12), (2, 8), (4, 1)]:
        d = np.zeros_like(state0)
        d[i, j] = 1.0
        lp, hp = _loss(ref, cfg, bodies, state0 + eps * d, im, ii, c, ss, src, col, seed)
        lm, hm = _loss(ref, cfg, bodies, state0 - eps * d, im, ii, c, ss, src, col, seed)
        if hp == h0 and hm == h0:
            fd = (lp - lm) / (2 * eps)
            assert abs(fd - grad[i, j]) <= 1e-5 * max(1.0, abs(fd)), (i, j, fd, grad[i, j])
            checked += 1
    for i in range(1, 6):
        d = np.zeros_like(im)
        d[i] = 1.0
        lp, hp = _loss(ref, cfg, bodies, state0, im + eps * d, ii, c, ss, src, col, seed)
        lm, hm = _loss(ref, cfg, bodies, state0, im - eps * d, ii, c, ss, src, col, seed)
        if hp == h0 and hm == h0:
            fd = (lp - lm) / (2 * eps)
            assert abs(fd - gim[i]) <= 1e-5 * max(1.0, abs(fd)), (i, fd, gim[i])
            checked += 1
    assert checked >= 10


def _branch_blocks(cfg):
    return cfg.substeps * (1 + cfg.sweeps) + 1 + cfg.positionIterations


def test_forced_branches_reproduce_the_run_and_make_the_piece_smooth(ref):
    # The decisions a run takes, fed back, reproduce it bit for bit; with the
    # decisions held, central differences of the piece match the adjoint even
    # where the free model sits on a kink (an exactly resting stack).
    steps = 8
    bodies, c, ss, src, col, state0 = _frozen_rollout_inputs(ref, steps)
    cfg = ref.AdjConfig.make()
    im = bodies["invMass"].astype(np.float64)
    ii = bodies["invInertia"][:, 0].astype(np.float64)
    rows = int(np.diff(ss).max())
    rec = np.zeros((steps, _branch_blocks(cfg), rows), np.uint8)
    seed = np.random.default_rng(4).normal(size=state0.shape)
    seed[bodies["motionType"] != 2] = 0.0
    out, h, grad, gim, gii = ref.adjoint_reference(cfg, bodies, state0, im, ii, c, ss, src, col, seed=seed,
                                                   record=rec)
    assert rec.any()
    out2, h2, grad2, gim2, gii2 = ref.adjoint_reference(cfg, bodies, state0, im, ii, c, ss, src, col, seed=seed,
                                                        branches=rec)
    assert np.array_equal(out, out2) and np.array_equal(grad, grad2) and np.array_equal(gim, gim2)
    # the stack at exact rest: the free model's hash changes under any perturbation
    rest = state0.copy()
    rest[1:5, 0:3] = np.round(rest[1:5, 0:3] * 2) / 2  # exact half-unit lattice: corners at zero gap
    rest[1:5, 7:13] = 0.0
    rest[1:5, 3:7] = (0.0, 0.0, 0.0, 1.0)
    rec[:] = 0
    _, h0, g0, _, _ = ref.adjoint_reference(cfg, bodies, rest, im, ii, c, ss, src, col, seed=seed, record=rec)
    rng = np.random.default_rng(6)
    eps = 1e-7  # the held piece bends sharply away from its own decisions: a tight stencil
    for trial in range(6):
        d = rng.normal(size=rest.shape)
        d[bodies["motionType"] != 2] = 0.0
        d[:, 3:7] = 0.0
        lp, _ = ref.adjoint_reference(cfg, bodies, rest + eps * d, im, ii, c, ss, src, col, branches=rec)
        lm, _ = ref.adjoint_reference(cfg, bodies, rest - eps * d, im, ii, c, ss, src, col, branches=rec)
        fd = np.sum((lp - lm) * seed) / (2 * eps)
        predicted = np.sum(g0 * d)
        assert abs(fd - predicted) <= 1e-5 * max(1.0, abs(fd)), (trial, fd, predicted)
