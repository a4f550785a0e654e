"""Seeded scenes for parity tests, built through the reference's World::add*
so both engines consume identical bodies and hull soup."""
import numpy as np

import velox_b200


def dense_mixed(size=800, squeeze=0.3, seed=7):
    """Mixed shapes (spheres, boxes, capsules, cylinders, hulls) packed so that
    many pairs touch or overlap: config-2 positions squeezed toward the origin."""
    specs, pool = velox_b200.generate_scene(2, seed=seed, size=size)
    dyn = specs["shape"] != 1
    specs["position"][dyn, 0] *= squeeze
    specs["position"][dyn, 2] *= squeeze
    specs["position"][dyn, 1] = 0.6 + (specs["position"][dyn, 1] - 1.0) * squeeze * 0.25
    return specs, pool


def scene(kind, size=0):
    if kind == "dense":
        return dense_mixed(size or 800)
    return velox_b200.generate_scene(kind, size=size)


def reference_scene(ref, kind, size=0, backend=2):
    specs, pool = scene(kind, size)
    w = ref.RefWorld(specs, pool, backend=backend)
    bodies = w.bodies()
    pts, faces = w.soup()
    return w, specs, pool, bodies, velox_b200.make_soup(pts, faces)


def world_of(specs):
    return np.ascontiguousarray(specs["world"], np.uint32)
