"""Invalid public state is rejected before it reaches the device world, with
the reference's rules (World::stepImpl validation, src/world.cpp:3855-3931):
non-finite body state, bad shape parameters, bad solver options, non-finite
gravity or forces. The context stays usable afterwards."""
import numpy as np
import pytest

import velox_b200
from velox_b200 import binding
from scenes import scene

pytestmark = pytest.mark.gpu


def _world():
    specs, pool = scene("dense", 200)
    bodies, hull, faces = velox_b200.bodies_from_specs(specs, pool)
    return bodies, velox_b200.make_soup(hull, faces)


@pytest.mark.parametrize("field,index,value,needle", [
    ("position", 3, np.nan, "body 3: body contains invalid or non-finite state"),
    ("velocity", 5, np.inf, "body 5: body contains invalid or non-finite state"),
    ("friction", 7, -1.0, "body 7: body contains invalid or non-finite state"),
    ("orientation", 2, 0.0, "body 2: body orientation must be a finite non-zero quaternion"),
])
def test_invalid_bodies_are_rejected(field, index, value, needle):
    bodies, soup = _world()
    bad = bodies.copy()
    bad[field][index] = value
    ctx = velox_b200.Context(0)
    with pytest.raises(velox_b200.VeloxError) as info:
        ctx.load(bad, soup)
    assert info.value.status == 1 and needle in str(info.value)
    ctx.load(bodies, soup)  # still usable
    ctx.configure()
    ctx.step(1)
    ctx.close()


def test_invalid_shape_parameters_are_rejected():
    bodies, soup = _world()
    spheres = np.flatnonzero(bodies["shape"] == binding.SHAPE["sphere"])
    bad = bodies.copy()
    bad["radius"][spheres[0]] = 0.0
    ctx = velox_b200.Context(0)
    with pytest.raises(velox_b200.VeloxError, match="sphere body has an invalid radius"):
        ctx.load(bad, soup)
    ctx.close()


def test_invalid_configuration_and_forces_are_rejected():
    bodies, soup = _world()
    ctx = velox_b200.Context(0)
    ctx.load(bodies, soup)
    with pytest.raises(velox_b200.VeloxError, match="gravity must be finite"):
        ctx.configure(gravity=(0.0, np.nan, 0.0))
    with pytest.raises(velox_b200.VeloxError, match="solver options are invalid"):
        ctx.configure(solver=binding.SolverOptions.default(velocityIterations=0))
    ctx.configure()
    forces = np.zeros((len(bodies), 6), np.float32)
    forces[4, 1] = np.inf
    with pytest.raises(velox_b200.VeloxError, match="forces and torques must be finite"):
        ctx.write_forces(forces)
    forces[4, 1] = 0.0
    ctx.write_forces(forces)
    ctx.step(1)
    assert np.isfinite(ctx.read_bodies()["position"]).all()
    ctx.close()
