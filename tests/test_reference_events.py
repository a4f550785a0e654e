"""The reference's contact events at a sleep transition, on the CPU: the
step in which a group falls asleep also reports End for pairs that are
active in it (src/world.cpp:4458-4482 looks prevPairKeys_ up with
std::binary_search in pairKeys_ after appending resting pairs to it, so the
array it searches is no longer sorted). The device world reproduces this
(tests/test_gpu_sleep.py); this pins it on the reference itself."""
import numpy as np

from sleep_scenes import resting_scene

DT = 1.0 / 60.0


def test_a_sleep_transition_ends_active_pairs(ref):
    specs, pool, bodies, soup = resting_scene(projectile=False)
    w = ref.RefWorld(specs, pool)
    w.configure(substeps=4, workers=1)
    found = False
    for _ in range(60):
        w.step(DT, 1)
        e = w.events()
        keys = e["a"].astype(np.uint64) << np.uint64(32) | e["b"].astype(np.uint64)
        ended = set(keys[e["type"] == 2].tolist())
        live = set(keys[e["type"] != 2].tolist())
        if ended & live:
            found = True
            break
    w.close()
    assert found
