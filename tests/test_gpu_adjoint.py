"""The adjoint of the device world's step (vxb_adjoint_backward) on the
differentiation workload: batched worlds, each a 5-box stack on a plane hit by
a sphere launched from 6 m at 4-12 m/s; 1/60 s steps, 4 substeps; loss = sum
of squared box centre-of-mass displacements from seeded targets.

Two properties of the reference's step shape the checks:

* It is piecewise smooth: the live gap's speculative branch, the impulse
  clamp, the friction ellipse and the position correction switch its pieces.
  A resting stack sits on those switches (speculative contacts close their
  gap to zero, a corner carries no load), so an FP32 and an FP64 run of the
  same trajectory take different pieces. The checks hold the pieces the FP32
  forward took (vxb_adjoint_backward_branches reports them) and compare
  derivatives of that piece.
* On a resting stack its Jacobian has a growing mode: a 1e-9 state change
  grows about 15x over 10 steps and 1.5e4x over 30 (gradients of a 120-step
  rollout reach 1e5). FP32 rounding alone moves a 120-step FP32 trajectory by
  a millimetre from its FP64 twin, so FP32 and FP64 gradients agree only over
  shorter windows. The gradient checks therefore tape 10-step windows at
  several points of the 120-step rollout (the projectile's impacts fall in
  them); the 120-step rollout itself is checked through torch.autograd.

Checks:
* the recomputed trajectory equals the forward (no VXB_ADJ_DIVERGED flag on a
  world that was not rewound);
* on worlds without a rewind in the window, the FP32 GPU gradients w.r.t. the
  sphere's linear and angular velocity and every body's mass at the window's
  start equal the FP64 CPU adjoint (oracle/adjoint_ref.c) of the same recorded
  contacts and pieces within 1e-3 relative, or within 3x the spread of that
  FP64 gradient under FP32-sized perturbations (2^-24 relative) of the state
  after every substep, which bounds how close the problem's conditioning lets
  any FP32 evaluation come; most comparisons meet 1e-3 outright. Worlds
  whose FP64 gradient moves by more than 2% under those perturbations have no
  FP32 gradient to compare and are skipped (counted);
* that FP64 adjoint equals FP64 central finite differences of the same piece
  within 1e-3 relative (h = 1e-6: a held piece bends sharply past its own
  switches, so the h = 1e-4 stencil is reported, not asserted);
* torch.autograd through the 120-step rollout (checkpoints every 10 steps)
  gives the C ABI's gradients.
"""
import numpy as np
import pytest
import torch

import velox_b200
from velox_b200.autograd import Rollout

pytestmark = pytest.mark.gpu
DT = 1.0 / 60.0
STEPS = 120
EVERY = 10
REL_TOL = 1e-3
WINDOW = 10
WINDOW_STARTS = (0, 32, 56, 80, 104)
# A world whose FP64 gradient moves by more than this (relative) under
# FP32-sized perturbations has no FP32 gradient to compare: skipped, counted.
ILL_CONDITIONED = 0.02


@pytest.fixture(scope="module")
def workload():
    specs, pool = velox_b200.generate_scene(5, size=128)
    bodies, hull, faces = velox_b200.bodies_from_specs(specs, pool)
    soup = velox_b200.make_soup(hull, faces)
    world_of = np.ascontiguousarray(specs["world"], np.uint32)
    rng = np.random.default_rng(5)
    boxes = bodies["shape"] == velox_b200.binding.SHAPE["box"]
    target = np.zeros((len(bodies), 3), np.float32)
    target[boxes] = rng.normal(scale=0.05, size=(int(boxes.sum()), 3))
    return specs, bodies, soup, world_of, boxes, target


def _loss_seed(final, bodies, boxes, target):
    d = final["position"] - bodies["position"] - target
    seed = np.zeros((len(bodies), 13), np.float32)
    seed[boxes, 0:3] = 2.0 * d[boxes]
    return float(np.sum(d[boxes] ** 2)), seed


def _world_tape(tape, world_of, w, b0):
    """One world's slice of the tape, body indices local to the world and
    sources local to the world's contacts of the previous step."""
    c, ss, src, col = tape["contacts"], tape["step_start"], tape["src"], tape["colors"]
    steps = len(ss) - 1
    parts, srcs, cols, starts, prev_lo = [], [], [], [0], 0
    for t in range(steps):
        ct = c[ss[t]:ss[t + 1]]
        wo = world_of[ct["a"]]
        lo, hi = int(np.searchsorted(wo, w, "left")), int(np.searchsorted(wo, w, "right"))
        part = ct[lo:hi].copy()
        part["a"] -= b0
        part["b"] -= b0
        s = src[ss[t] + lo:ss[t] + hi].astype(np.int64)
        s = np.where(s == 0xffffffff, -1, s - prev_lo)
        s = np.where(s < 0, 0xffffffff, s)
        parts.append(part)
        srcs.append(s.astype(np.uint32))
        cols.append(col[ss[t] + lo:ss[t] + hi])
        starts.append(starts[-1] + (hi - lo))
        prev_lo = lo
    return (np.concatenate(parts), np.array(starts, np.uint32), np.concatenate(srcs).reshape(-1, 2),
            np.concatenate(cols).astype(np.int32))


def _mass_grad(wb, im, ii, gim, gii):
    """dL/dmass from dL/d(invMass, isotropic invInertia) (inertia scales with mass)."""
    return np.where(wb["motionType"] == 2, -im * im * gim - ii * im * gii, 0.0)


def _window(bodies, soup, world_of, boxes, target, t0):
    """Steps to t0, tapes WINDOW steps and runs the backward with the pieces."""
    ctx = velox_b200.Context(0)
    ctx.load(bodies, soup, world_of=world_of)
    ctx.configure(dt=DT, substeps=4)
    if t0:
        ctx.step(t0)
    ctx.tape_begin(WINDOW, WINDOW // 2)
    start = ctx.read_bodies()
    ctx.step(WINDOW)
    final = ctx.read_bodies()
    d = final["position"] - start["position"] - target
    seed = np.zeros((len(bodies), 13), np.float32)
    seed[boxes, 0:3] = 2.0 * d[boxes]
    grad, ginv, gmass, flags, branches = ctx.adjoint_backward_branches(seed)
    g_plain, _, m_plain, f_plain = ctx.adjoint_backward(seed)
    tape = ctx.tape_read()
    ctx.close()
    # reporting the pieces changes nothing
    assert np.array_equal(g_plain, grad) and np.array_equal(m_plain, gmass) and np.array_equal(f_plain, flags)
    return final, seed, grad, gmass, flags, branches, tape


def test_adjoint_matches_fp64_reference_and_finite_differences(ref, workload):
    specs, bodies, soup, world_of, boxes, target = workload
    cfg = ref.AdjConfig.make()
    starts = np.searchsorted(world_of, np.arange(world_of.max() + 2))
    compared = impacts = fd_checked = 0
    coarse = []
    within = {"v": 0, "w": 0, "mass": 0}
    ill = 0
    for t0 in WINDOW_STARTS:
        final, seed, grad, gmass, flags, branches, tape = _window(bodies, soup, world_of, boxes, target, t0)
        assert np.isfinite(grad).all() and np.isfinite(gmass).all()
        rewound, diverged = (flags & 1) != 0, (flags & 2) != 0
        assert not (diverged & ~rewound).any(), ("recomputation left the forward path without a rewind", t0, flags)
        assert not grad[np.repeat(flags != 0, np.diff(starts))].any()
        ck0 = tape["checkpoints"][0]  # (4, n, 4): state at the window's start
        state0 = np.concatenate([ck0[0, :, :3], ck0[1], ck0[2, :, :3], ck0[3, :, :3]], 1).astype(np.float64)
        # worlds whose projectile touches a box in the window first, then others
        smooth = np.flatnonzero(flags == 0)
        sphere_hits = []
        for w in smooth:
            b0, b1 = int(starts[w]), int(starts[w + 1])
            c = tape["contacts"]
            hit = (c["b"] == b1 - 1) & (c["a"] > b0) | (c["a"] == b1 - 1) & (c["b"] > b0)
            sphere_hits.append(bool(hit.any()))
        order = sorted(range(len(smooth)), key=lambda k: not sphere_hits[k])
        for k in order[:12]:
            w = smooth[k]
            b0, b1 = int(starts[w]), int(starts[w + 1])
            c, ss, src, col = _world_tape(tape, world_of, w, b0)
            piece = branches[w]
            wb = bodies[b0:b1]
            im = wb["invMass"].astype(np.float64)
            ii = wb["invInertia"][:, 0].astype(np.float64)
            s0 = state0[b0:b1]
            sw = seed[b0:b1].astype(np.float64)
            out, _, g64, gim, gii = ref.adjoint_reference(cfg, wb, s0, im, ii, c, ss, src, col, seed=sw,
                                                          branches=piece)
            gm64 = _mass_grad(wb, im, ii, gim, gii)
            # the FP64 gradient's own spread under FP32-sized perturbations of
            # the state after every substep: how close the problem's
            # conditioning lets any FP32 evaluation come
            spread = np.zeros((3, 3)), np.zeros((3, 3)), np.zeros((3, len(wb)))
            for r in range(3):
                _, _, gn, gimn, giin = ref.adjoint_reference(cfg, wb, s0, im, ii, c, ss, src, col, seed=sw,
                                                             branches=piece, noise=2.0 ** -24, noise_seed=r)
                spread[0][r], spread[1][r] = gn[-1, 7:10], gn[-1, 10:13]
                spread[2][r] = _mass_grad(wb, im, ii, gimn, giin)
            sphere = b1 - 1
            checks = [("v", grad[sphere, 7:10], g64[-1, 7:10], spread[0]),
                      ("w", grad[sphere, 10:13], g64[-1, 10:13], spread[1]),
                      ("mass", gmass[b0:b1], gm64, spread[2])]
            # a quantity that is zero in exact arithmetic (the mass of a body in
            # free flight) is compared on the scale of the world's gradient
            floor = 1e-5 * max(np.abs(g64).max(), 1e-9)
            scales = [max(np.abs(theirs).max(), floor) for _, _, theirs, _ in checks]
            bands = [np.abs(noise - theirs).max() / sc for (_, _, theirs, noise), sc in zip(checks, scales)]
            if max(bands) > ILL_CONDITIONED:
                ill += 1
                continue
            # on the same piece the FP64 trajectory follows the FP32 forward
            assert np.abs(out[:, 0:3] - final["position"][b0:b1]).max() < 1e-4, (t0, w)
            for (name, mine, theirs, noise), band, scale in zip(checks, bands, scales):
                err = np.abs(mine - theirs).max() / scale
                assert err <= max(REL_TOL, 3.0 * band), (t0, w, name, mine, theirs, band)
                within[name] += err <= REL_TOL
            compared += 1
            impacts += sphere_hits[k]
            # FP64 central differences of the same piece
            for j in (7, 8, 10, 12):
                dv = np.zeros_like(s0)
                dv[-1, j] = 1.0
                for eps in (1e-6, 1e-4):
                    lp, _ = ref.adjoint_reference(cfg, wb, s0 + eps * dv, im, ii, c, ss, src, col, branches=piece)
                    lm, _ = ref.adjoint_reference(cfg, wb, s0 - eps * dv, im, ii, c, ss, src, col, branches=piece)
                    fd = np.sum((lp - lm) * sw) / (2 * eps)
                    err = abs(fd - g64[-1, j]) / max(abs(fd), 1e-3)
                    if eps == 1e-6:
                        assert err <= REL_TOL, (t0, w, j, fd, g64[-1, j])
                        fd_checked += 1
                    else:
                        coarse.append(err)
    assert compared >= 16, (compared, ill)
    assert impacts >= 4, impacts
    assert sum(within.values()) >= 0.75 * 3 * compared, within
    assert fd_checked >= 4 * compared
    print(f"compared {compared} worlds ({impacts} with the projectile on the stack, {ill} ill-conditioned "
          f"skipped); within {REL_TOL} "
          f"relative: {within}; h=1e-4 stencil: {np.mean(np.array(coarse) <= REL_TOL):.0%} of {len(coarse)}")


def test_autograd_function_gives_the_adjoint(workload):
    specs, bodies, soup, world_of, boxes, target = workload
    rollout = Rollout(bodies, soup, world_of, steps=STEPS, checkpoint_every=EVERY)
    v = torch.tensor(bodies["velocity"], requires_grad=True)
    w = torch.tensor(bodies["angularVelocity"], requires_grad=True)
    mass = torch.tensor(np.where(rollout.dynamic, rollout.mass0, 0.0).astype(np.float32), requires_grad=True)
    pos = rollout(v, w, mass)
    p0 = torch.tensor(bodies["position"])
    mask = torch.tensor(boxes)
    loss = (((pos - p0 - torch.tensor(target)) ** 2)[mask]).sum()
    loss.backward()
    # the same through the C ABI directly
    ctx = velox_b200.Context(0)
    ctx.load(bodies, soup, world_of=world_of)
    ctx.configure(dt=DT, substeps=4)
    ctx.tape_begin(STEPS, EVERY)
    ctx.step(STEPS)
    final = ctx.read_bodies()
    l2, seed = _loss_seed(final, bodies, boxes, target)
    grad, _, gmass, _ = ctx.adjoint_backward(seed)
    ctx.close()
    rollout.close()
    assert abs(loss.item() - l2) <= 1e-5 * max(1.0, l2)
    assert np.allclose(v.grad.numpy(), grad[:, 7:10], rtol=1e-6, atol=1e-7)
    assert np.allclose(w.grad.numpy(), grad[:, 10:13], rtol=1e-6, atol=1e-7)
    assert np.allclose(mass.grad.numpy(), gmass, rtol=1e-6, atol=1e-7)
