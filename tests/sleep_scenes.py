"""Scenes for the sleeping and contact-event tests: bodies that come to rest
within a few dozen steps, and a projectile that strikes one resting group
later (the wake pass)."""
import numpy as np

import velox_b200
from velox_b200 import binding


def resting_scene(seed=0, projectile=True, non_sleeper=True):
    """A plane; a 3x3 grid of unit boxes resting on it; two 3-box stacks; a
    sphere launched at one stack after a delay (it starts high and far);
    optionally one box that may not sleep, resting on another box."""
    rng = np.random.default_rng(seed)
    rows = []

    def add(shape, pos, half=0.5, radius=0.3, mass=1.0, vel=(0, 0, 0), sleep=1):
        r = np.zeros(1, binding.SPEC)
        r["shape"] = binding.SHAPE[shape]
        r["orientation"] = (0, 0, 0, 1)
        r["friction"] = 0.5
        r["restitution"] = 0.1
        r["enableSleep"] = sleep
        r["position"] = pos
        r["velocity"] = vel
        r["mass"] = mass
        if shape == "box":
            r["halfExtents"] = half
        elif shape == "sphere":
            r["radius"] = radius
        elif shape == "plane":
            r["planeNormal"] = (0, 1, 0)
            r["mass"] = 0.0
        rows.append(r)

    add("plane", (0, 0, 0), sleep=0)
    for i in range(3):
        for j in range(3):
            jitter = rng.uniform(-0.01, 0.01, 2)
            add("box", (i * 1.2 + jitter[0], 0.5 + 1e-3, j * 1.2 + jitter[1]))
    for x in (6.0, 9.0):
        for level in range(3):
            add("box", (x + 0.01 * level, 0.5 + level * 1.0 + 2e-3 * (level + 1), 0.0))
    if non_sleeper:
        add("box", (-3.0, 0.5 + 1e-3, 0.0))
        add("box", (-3.0, 1.5 + 3e-3, 0.0), sleep=0)
    if projectile:
        # reaches the stack at x = 9 after about a second
        add("sphere", (9.0, 7.0, -6.0), radius=0.3, mass=2.0, vel=(0.0, 0.5, 6.0))
    specs = binding.records(np.concatenate(rows), binding.SPEC)  # concatenate drops the padding
    bodies, hull, faces = velox_b200.bodies_from_specs(specs, np.zeros((1, 3), np.float32))
    return specs, np.zeros((1, 3), np.float32), bodies, velox_b200.make_soup(hull, faces)
