"""Scene construction agrees with the reference's World::add* (CPU)."""
import numpy as np

import velox_b200


def test_non_hull_bodies_are_byte_identical_to_reference(ref):
    specs, pool = velox_b200.generate_scene(2, size=1500)
    w = ref.RefWorld(specs, pool)
    rb = w.bodies()
    mb, _, _ = velox_b200.bodies_from_specs(specs, pool)
    nonhull = specs["shape"] != 5
    a = rb.view(np.uint8).reshape(-1, 320)[nonhull]
    b = mb.view(np.uint8).reshape(-1, 320)[nonhull]
    assert np.array_equal(a, b)


def test_hull_mass_properties_match_reference(ref):
    specs, pool = velox_b200.generate_scene(2, size=400)
    w = ref.RefWorld(specs, pool)
    rb = w.bodies()
    mb, _, _ = velox_b200.bodies_from_specs(specs, pool)
    h = specs["shape"] == 5
    assert np.allclose(rb["position"][h], mb["position"][h], atol=1e-5)
    assert np.allclose(rb["radius"][h], mb["radius"][h], atol=1e-5)
    # principal moments agree as a set (axis order is a convention)
    assert np.allclose(np.sort(1.0 / rb["invInertia"][h], 1), np.sort(1.0 / mb["invInertia"][h], 1), rtol=1e-4)


def test_reference_soup_export_matches_what_world_step_sees(ref):
    specs, pool = velox_b200.generate_scene(2, size=300)
    w = ref.RefWorld(specs, pool)
    pts, faces = w.soup()
    w.configure(workers=1)
    w.step(1.0 / 60.0, 1)
    import ctypes
    nf = ctypes.c_uint32()
    n = w.L.ref_world_captured_soup(w.h, None, None, ctypes.byref(nf))
    cp = np.zeros((n, 3), np.float32)
    cf = np.zeros(nf.value, np.uint32)
    w.L.ref_world_captured_soup(w.h, ref._p(cp), ref._p(cf), ctypes.byref(nf))
    assert np.array_equal(cp, pts) and np.array_equal(cf, faces)
