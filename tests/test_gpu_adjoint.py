"""The adjoint of the device world's step (vxb_adjoint_backward) on the
differentiation workload: batched worlds, each a 5-box stack on a plane hit by
a sphere launched from 6 m at 4-12 m/s; 120 steps of 1/60 s, 4 substeps,
checkpoints every 10 steps; loss = sum of squared box centre-of-mass
displacements from seeded targets.

Checks, on smooth worlds (no rewind, recomputation on the forward's path):
* the recomputed trajectory equals the forward (no VXB_ADJ_DIVERGED flag);
* the FP32 GPU gradients w.r.t. the sphere's initial linear and angular
  velocity and every body's mass equal the FP64 CPU adjoint
  (oracle/adjoint_ref.c) of the same recorded contacts within 1e-3 relative;
* that FP64 adjoint equals FP64 central finite differences (h = 1e-4) of the
  same frozen-contact step within 1e-3 relative;
* torch.autograd through the rollout gives the same gradients.
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


def test_adjoint_matches_fp64_reference_and_finite_differences(ref, workload):
    specs, bodies, soup, world_of, boxes, target = workload
    ctx = velox_b200.Context(0)
    ctx.load(bodies, soup, world_of=world_of)
    ctx.configure(dt=DT, substeps=4)
    ctx.tape_begin(STEPS, EVERY)
    ctx.step(STEPS)
    final = ctx.read_bodies()
    loss, seed = _loss_seed(final, bodies, boxes, target)
    grad, ginv, gmass, flags = ctx.adjoint_backward(seed)
    tape = ctx.tape_read()
    ctx.close()
    assert np.isfinite(grad).all() and np.isfinite(gmass).all()
    rewound = (flags & 1) != 0
    diverged = (flags & 2) != 0
    assert not (diverged & ~rewound).any(), ("recomputation left the forward path without a rewind", flags)
    # Most projectiles strike hard enough for a conservative-advancement rewind
    # (a discrete time-of-impact event, not differentiated: zero gradients);
    # the rest are the smooth trajectories the bar applies to.
    smooth = np.flatnonzero(flags == 0)
    assert len(smooth) >= 8, flags
    assert not grad[np.repeat(flags != 0, np.diff(np.searchsorted(world_of, np.arange(len(flags) + 1))))].any()
    cfg = ref.AdjConfig.make()
    starts = np.searchsorted(world_of, np.arange(len(flags) + 1))
    ck0 = tape["checkpoints"][0]  # (4, n, 4): state at the first taped step
    state0 = np.concatenate([ck0[0, :, :3], ck0[1], ck0[2, :, :3], ck0[3, :, :3]], 1).astype(np.float64)
    compared = fd_checked = 0
    for w in smooth[:16]:
        b0, b1 = int(starts[w]), int(starts[w + 1])
        c, ss, src, col = _world_tape(tape, world_of, w, b0)
        wb = bodies[b0:b1]
        im = wb["invMass"].astype(np.float64)
        ii = wb["invInertia"][:, 0].astype(np.float64)
        s0 = state0[b0:b1]
        out, h0, g64, gim, gii = ref.adjoint_reference(cfg, wb, s0, im, ii, c, ss, src, col,
                                                       seed=seed[b0:b1].astype(np.float64))
        # the FP64 model's trajectory follows the FP32 forward
        assert np.abs(out[:, 0:3] - final["position"][b0:b1]).max() < 5e-3, w
        gm64 = np.where(wb["motionType"] == 2, -im * im * gim - ii * im * gii, 0.0)
        sphere = b1 - 1
        for name, mine, theirs in [("v0", grad[sphere, 7:10], g64[-1, 7:10]),
                                   ("w0", grad[sphere, 10:13], g64[-1, 10:13]),
                                   ("mass", gmass[b0:b1], gm64)]:
            scale = max(np.abs(theirs).max(), 1e-6)
            assert np.abs(mine - theirs).max() <= REL_TOL * scale, (w, name, mine, theirs)
        compared += 1
        # FP64 central differences of the same frozen-contact step (h = 1e-4)
        eps = 1e-4
        for j in (7, 8, 10, 12):
            d = np.zeros_like(s0)
            d[-1, j] = 1.0
            lp, hp = ref.adjoint_reference(cfg, wb, s0 + eps * d, im, ii, c, ss, src, col)
            lm, hm = ref.adjoint_reference(cfg, wb, s0 - eps * d, im, ii, c, ss, src, col)
            if hp != h0 or hm != h0:
                continue
            fd = np.sum((lp - lm) * seed[b0:b1]) / (2 * eps)
            assert abs(fd - g64[-1, j]) <= REL_TOL * max(abs(fd), 1e-3), (w, j, fd, g64[-1, j])
            fd_checked += 1
    assert compared >= 8
    assert fd_checked >= 8


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
