"""torch.autograd over the device world: a batch of worlds stepped from given
initial velocities and masses, differentiated by the library's adjoint
(vxb_tape_begin / vxb_adjoint_backward through ctypes).

    rollout = Rollout(bodies, soup, world_of, steps=120)
    pos = rollout(velocity, angular_velocity, mass)   # final positions (n x 3)
    loss = ((pos - pos0 - target) ** 2).sum()
    loss.backward()                                   # grads of velocity, angular velocity, mass

Masses scale each dynamic body's inverse mass and (isotropic) inverse inertia
together, as a change of density would. The gradient is the adjoint of the
step with each step's contact set and active sets frozen (see
include/velox_b200.h); worlds outside its scope are listed in
Rollout.last_flags.
"""
import numpy as np
import torch

from .binding import BODY, Context, records

DYNAMIC = 2


class Rollout:
    def __init__(self, bodies, soup, world_of=None, steps=120, dt=1.0 / 60.0, substeps=4, checkpoint_every=10,
                 solver=None, device=0, gravity=(0.0, -9.81, 0.0)):
        self.bodies = records(bodies, BODY).copy()
        self.soup = soup
        self.world_of = None if world_of is None else np.ascontiguousarray(world_of, np.uint32)
        self.steps = steps
        self.dt = dt
        self.substeps = substeps
        self.every = checkpoint_every
        self.solver = solver
        self.gravity = gravity
        self.ctx = Context(device)
        dyn = self.bodies["motionType"] == DYNAMIC
        self.dynamic = dyn
        self.mass0 = np.where(dyn & (self.bodies["invMass"] > 0), 1.0 / np.maximum(self.bodies["invMass"], 1e-30), 0.0)
        self.last_flags = None
        self.final = None

    def close(self):
        self.ctx.close()

    def bodies_for(self, velocity, angular_velocity, mass):
        b = self.bodies.copy()
        b["velocity"] = np.asarray(velocity, np.float32)
        b["angularVelocity"] = np.asarray(angular_velocity, np.float32)
        m = np.asarray(mass, np.float64)
        d = self.dynamic & (m > 0)
        b["invMass"][d] = (1.0 / m[d]).astype(np.float32)
        scale = (self.mass0[d] / m[d]).astype(np.float32)
        b["invInertia"][d] = self.bodies["invInertia"][d] * scale[:, None]
        return b

    def __call__(self, velocity, angular_velocity, mass):
        return RolloutFunction.apply(velocity, angular_velocity, mass, self)


class RolloutFunction(torch.autograd.Function):
    @staticmethod
    def forward(fctx, velocity, angular_velocity, mass, rollout):
        b = rollout.bodies_for(velocity.detach().cpu().numpy(), angular_velocity.detach().cpu().numpy(),
                               mass.detach().cpu().numpy())
        ctx = rollout.ctx
        ctx.load(b, rollout.soup, world_of=rollout.world_of)
        ctx.configure(dt=rollout.dt, substeps=rollout.substeps, gravity=rollout.gravity, solver=rollout.solver)
        ctx.tape_begin(rollout.steps, rollout.every)
        ctx.step(rollout.steps)
        rollout.final = ctx.read_bodies()
        fctx.rollout = rollout
        fctx.dtype = velocity.dtype
        fctx.device = velocity.device
        return torch.from_numpy(rollout.final["position"].copy()).to(velocity.device, velocity.dtype)

    @staticmethod
    def backward(fctx, grad_position):
        rollout = fctx.rollout
        n = len(rollout.bodies)
        seed = np.zeros((n, 13), np.float32)
        seed[:, 0:3] = grad_position.detach().cpu().numpy()
        grad, _, gmass, flags = rollout.ctx.adjoint_backward(seed)
        rollout.last_flags = flags

        def as_t(a):
            return torch.from_numpy(np.ascontiguousarray(a)).to(fctx.device, fctx.dtype)

        return as_t(grad[:, 7:10]), as_t(grad[:, 10:13]), as_t(gmass), None
