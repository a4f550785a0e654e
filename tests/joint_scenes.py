"""Seeded jointed scenes built through the reference's World joint adders
(addBallJoint ... addGearJoint, include/velox/world.h:617-670): hanging
chains whose links cycle through all thirteen joint types with limits,
motors, springs and soft welds switched on, and spheres dropped onto them so
that contacts and joints share bodies. 8 chains of 10 links give 80 joints:
above the 64 at which the reference CUDA backend solves joints on the device."""
import numpy as np

from velox_b200 import binding

IDENTITY = (0.0, 0.0, 0.0, 1.0)
LINK = 0.42  # link spacing along x


def jointed_world(ref, chains=8, links=10, drops=12, seed=0, strict=True, backend=None, break_force=None,
                  kinds=tuple(range(13)), soft_weld=0.0, steering=True):
    rng = np.random.default_rng(seed)
    n = 1 + chains * (1 + links) + drops
    specs = np.zeros(n, binding.SPEC)
    specs["orientation"] = IDENTITY
    specs["friction"] = 0.5
    specs[0]["shape"] = 1
    specs[0]["planeNormal"] = (0, 1, 0)
    k = 1
    anchors, first_link = [], []
    for c in range(chains):
        z = 1.5 * (c - chains / 2)
        s = specs[k]
        s["shape"], s["halfExtents"], s["position"] = 2, (0.2, 0.2, 0.2), (0.0, 6.0, z)
        anchors.append(k)
        k += 1
        first_link.append(k)
        for i in range(links):
            s = specs[k]
            s["shape"] = 2 if i % 3 else 0
            s["mass"] = 1.0 + 0.2 * (i % 4)
            s["halfExtents"] = (0.14, 0.09, 0.1)
            s["radius"] = 0.12
            s["position"] = (LINK * (i + 1), 6.0 + 0.02 * rng.normal(), z + 0.02 * rng.normal())
            s["angularVelocity"] = rng.normal(scale=0.2, size=3)
            k += 1
    for d in range(drops):
        s = specs[k]
        s["shape"], s["mass"], s["radius"] = 0, 0.6, 0.15
        s["position"] = (rng.uniform(0.5, 4.0), rng.uniform(7.0, 9.0), 1.5 * (rng.integers(chains) - chains / 2))
        s["velocity"] = (0.0, -3.0, 0.0)
        k += 1
    kw = {"strict": strict}
    if backend is not None:
        kw["backend"] = backend
    w = ref.RefWorld(specs, np.zeros((0, 3), np.float32), **kw)
    t = 0
    for c in range(chains):
        z = 1.5 * (c - chains / 2)
        prev, prev_x = anchors[c], 0.0
        for i in range(links):
            me = first_link[c] + i
            x = LINK * (i + 1)
            mid = ((prev_x + x) / 2, 6.0, z)
            kind = kinds[t % len(kinds)]
            t += 1
            args = dict(p0=mid)
            if kind == 1:  # distance (every other one a spring)
                args = dict(p0=(prev_x, 6.0, z), p1=(x, 6.0, z), x=(2.0 if i % 2 else 0.0, 0.4, 0.0))
            elif kind in (2, 3, 5, 9):  # hinge, cone twist, prismatic, wheel
                args = dict(p0=mid, axis0=(0.0, 0.0, 1.0) if kind == 2 else (1.0, 0.0, 0.0))
            elif kind == 7:  # motor
                args = dict(p0=(prev_x, 6.0, z), p1=(x, 6.0, z), x=(40.0, 40.0, 0.0))
            elif kind == 8:  # weld
                args = dict(p0=mid, x=(3.4e38, 3.4e38, 0.0))
            elif kind == 10:  # rope
                args = dict(p0=(prev_x, 6.0, z), p1=(x, 6.0, z), x=(LINK * 1.05, 0.0, 0.0))
            elif kind == 11:  # pulley
                args = dict(p0=(prev_x, 6.0, z), p1=(x, 6.0, z), ground0=(prev_x, 7.0, z), ground1=(x, 7.0, z),
                            x=(1.5, 0.0, 0.0))
            elif kind == 12:  # gear
                args = dict(axis0=(0.0, 0.0, 1.0), axis1=(0.0, 0.0, 1.0), x=(-1.0, 0.0, 0.0))
            j = w.add_joint(kind, prev, me, **args)
            rec = w.joint(j)
            if kind == 2:
                rec["enableLimit"], rec["lowerLimit"], rec["upperLimit"] = 1, -0.4, 0.5
                rec["enableMotor"], rec["motorSpeed"], rec["maxMotorTorque"] = 1, 0.8, 2.0
            elif kind == 3:
                rec["enableSwingLimit"], rec["swingLimit"] = 1, 0.3
                rec["enableTwistLimit"], rec["lowerTwistLimit"], rec["upperTwistLimit"] = 1, -0.2, 0.2
            elif kind == 5:
                rec["enableLimit"], rec["lowerLimit"], rec["upperLimit"] = 1, -0.05, 0.1
                rec["enableMotor"], rec["motorSpeed"], rec["maxMotorForce"] = 1, 0.3, 5.0
            elif kind == 6:
                rec["linearLimitMask"], rec["angularLimitMask"] = 7, 5
                rec["upperAngularLimit"] = (0.0, 0.6, 0.0)
                rec["lowerAngularLimit"] = (0.0, -0.6, 0.0)
                rec["angularMotorMask"], rec["angularMotorSpeed"] = 2, (0.0, 0.5, 0.0)
                rec["maxAngularMotorTorque"] = (0.0, 3.0, 0.0)
            elif kind == 8 and soft_weld:
                rec["weldFrequencyHz"], rec["weldDampingRatio"] = soft_weld, 1.0
            elif kind == 9 and steering:
                rec["enableSteering"], rec["steeringAngle"] = 1, 0.2
                rec["enableMotor"], rec["motorSpeed"], rec["maxMotorTorque"] = 1, 3.0, 1.0
            if break_force is not None and kind in (0, 4):
                rec["breakForce"] = break_force
            w.set_joint(j, rec)
            prev, prev_x = me, x
    return w
