"""The device joint rows (velox_b200/csrc/joints.cuh) against the reference's
joint_solver::solve (src/joint_solver.h), on the CPU: the same header
compiled for the host (oracle/joint_check.cu) and run beside the reference
on random joints of all thirteen types (limits, motors, springs, soft welds,
steering; dynamic, static, locked and fixed-rotation endpoints; anisotropic
inertia in rotated frames). Velocities and every joint field must agree bit
for bit after eight sweeps, as must reset and the break test."""
import ctypes
import os

import numpy as np
import pytest

from velox_b200 import binding

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_ref", "libjoint_check.so")

JOINT = binding.JOINT


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB):
        pytest.skip("joint harness not built (make -C oracle joints)")
    L = ctypes.CDLL(LIB)
    vp = ctypes.c_void_p
    L.joint_check.argtypes = [vp, vp, ctypes.c_int, ctypes.c_float, ctypes.c_int, vp, vp, vp, vp]
    L.joint_check_reset_break.argtypes = [vp, vp, ctypes.c_float, ctypes.c_int]
    return L


def _unit(rng, n):
    v = rng.normal(size=(n, 3))
    return (v / np.linalg.norm(v, axis=1, keepdims=True)).astype(np.float32)


def _quat(rng, n):
    q = rng.normal(size=(n, 4))
    return (q / np.linalg.norm(q, axis=1, keepdims=True)).astype(np.float32)


def _bodies(rng, n):
    b = np.zeros(n, binding.BODY)
    b["position"] = rng.uniform(-2, 2, (n, 3))
    b["orientation"] = _quat(rng, n)
    b["velocity"] = rng.normal(scale=2.0, size=(n, 3))
    b["angularVelocity"] = rng.normal(scale=3.0, size=(n, 3))
    b["invMass"] = rng.uniform(0.2, 2.0, n)
    b["invInertia"] = rng.uniform(0.5, 8.0, (n, 3))
    iso = rng.random(n) < 0.3
    b["invInertia"][iso] = b["invInertia"][iso][:, :1]
    b["inertiaOrientation"] = _quat(rng, n)
    b["inertiaOrientation"][rng.random(n) < 0.4] = (0, 0, 0, 1)
    b["motionType"] = rng.choice([0, 1, 2, 2, 2, 2], n)
    b["ccdTuning"]["quality"] = rng.choice([1, 1, 1, 2, 3], n)  # some Locked
    b["fixedRotation"] = rng.random(n) < 0.1
    b["shape"] = 2
    return b


def _joints(rng, count):
    j = np.zeros(count, JOINT)
    j["type"] = np.arange(count) % 13
    j["a"] = 2 * np.arange(count)
    j["b"] = 2 * np.arange(count) + 1
    for f in ("localAnchorA", "localAnchorB"):
        j[f] = rng.uniform(-0.5, 0.5, (count, 3))
    for f in ("localAxisA", "localAxisB", "localRefA", "localRefB"):
        j[f] = _unit(rng, count)
    par = rng.random(count) < 0.1  # reference parallel to the axis: the fallback frames
    j["localRefA"][par] = j["localAxisA"][par]
    j["restLength"] = rng.uniform(0.2, 1.5, count)
    j["enableSpring"] = rng.random(count) < 0.5
    j["springFrequencyHz"] = rng.uniform(0.5, 5.0, count)
    j["springDampingRatio"] = rng.uniform(0.0, 1.5, count)
    j["breakForce"] = np.where(rng.random(count) < 0.5, 3.4e38, rng.uniform(1.0, 500.0, count))
    j["breakTorque"] = np.where(rng.random(count) < 0.5, 3.4e38, rng.uniform(1.0, 500.0, count))
    j["enableMotor"] = rng.random(count) < 0.5
    j["motorSpeed"] = rng.normal(scale=2.0, size=count)
    j["maxMotorTorque"] = rng.uniform(0.0, 20.0, count)
    j["maxMotorForce"] = rng.uniform(0.0, 20.0, count)
    j["enableLimit"] = rng.random(count) < 0.6
    lo = rng.uniform(-1.0, 0.3, count)
    j["lowerLimit"] = lo
    j["upperLimit"] = lo + rng.uniform(0.0, 1.0, count)
    j["enableSwingLimit"] = rng.random(count) < 0.6
    j["swingLimit"] = rng.uniform(0.05, 1.5, count)
    j["enableTwistLimit"] = rng.random(count) < 0.6
    tl = rng.uniform(-1.0, 0.2, count)
    j["lowerTwistLimit"] = tl
    j["upperTwistLimit"] = tl + rng.uniform(0.0, 1.0, count)
    for f in ("linearLimitMask", "angularLimitMask", "linearMotorMask", "angularMotorMask"):
        j[f] = rng.integers(0, 8, count)
    ll = rng.uniform(-0.5, 0.2, (count, 3))
    locked = rng.random((count, 3)) < 0.3
    j["lowerLinearLimit"] = ll
    j["upperLinearLimit"] = np.where(locked, ll, ll + rng.uniform(0.0, 0.5, (count, 3)))
    al = rng.uniform(-0.8, 0.2, (count, 3))
    j["lowerAngularLimit"] = al
    j["upperAngularLimit"] = np.where(locked, al, al + rng.uniform(0.0, 0.8, (count, 3)))
    j["linearMotorSpeed"] = rng.normal(size=(count, 3))
    j["angularMotorSpeed"] = rng.normal(size=(count, 3))
    j["maxLinearMotorForce"] = rng.uniform(0.0, 10.0, (count, 3))
    j["maxAngularMotorTorque"] = rng.uniform(0.0, 10.0, (count, 3))
    j["weldFrequencyHz"] = np.where(rng.random(count) < 0.5, 0.0, rng.uniform(0.5, 5.0, count))
    j["weldDampingRatio"] = rng.uniform(0.0, 1.5, count)
    j["suspensionFrequencyHz"] = np.where(rng.random(count) < 0.2, 0.0, rng.uniform(0.5, 5.0, count))
    j["suspensionDampingRatio"] = rng.uniform(0.0, 1.5, count)
    j["wheelRadius"] = 0.5
    j["enableSteering"] = rng.random(count) < 0.5
    j["steeringAngle"] = rng.uniform(-0.5, 0.5, count)
    j["maxSteeringAngle"] = 0.6
    j["maxLength"] = rng.uniform(0.0, 2.0, count)
    j["pulleyAnchorA"] = rng.uniform(-3, 3, (count, 3))
    j["pulleyAnchorB"] = rng.uniform(-3, 3, (count, 3))
    j["pulleyRatio"] = rng.uniform(0.5, 2.0, count)
    j["gearRatio"] = rng.uniform(-2.0, 2.0, count)
    return j


def _same(x, y):
    return np.array_equal(np.ascontiguousarray(x).view(np.uint8), np.ascontiguousarray(y).view(np.uint8))


def _rows(records, sel):
    """Raw bytes of the selected records (fancy indexing of a structured
    array with padding would not copy the padding bytes)."""
    return records.view(np.uint8).reshape(len(records), -1)[sel]


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_joint_rows_equal_the_reference_bit_for_bit(lib, seed):
    rng = np.random.default_rng(seed)
    count = 13 * 60
    bodies = _bodies(rng, 2 * count)
    joints = _joints(rng, count)
    ref_b, my_b = np.zeros_like(bodies), np.zeros_like(bodies)
    ref_j, my_j = np.zeros_like(joints), np.zeros_like(joints)
    p = lambda a: ctypes.c_void_p(a.ctypes.data)
    lib.joint_check(p(bodies), p(joints), count, 1.0 / 240.0, 8, p(ref_b), p(ref_j), p(my_b), p(my_j))
    moved = np.abs(ref_b["velocity"] - bodies["velocity"]).max(1) > 0
    assert moved.sum() > count // 2  # the rows act
    for k in range(13):
        sel = np.flatnonzero(joints["type"] == k)
        bs = np.sort(np.concatenate([2 * sel, 2 * sel + 1]))
        assert _same(my_b[bs]["velocity"], ref_b[bs]["velocity"]), k
        assert _same(my_b[bs]["angularVelocity"], ref_b[bs]["angularVelocity"]), k
        assert _same(_rows(my_j, sel), _rows(ref_j, sel)), k


def test_reset_and_break_test_equal_the_reference(lib):
    rng = np.random.default_rng(5)
    count = 13 * 20
    bodies = _bodies(rng, 2 * count)
    joints = _joints(rng, count)
    ref_b, my_b = np.zeros_like(bodies), np.zeros_like(bodies)
    ref_j, my_j = np.zeros_like(joints), np.zeros_like(joints)
    p = lambda a: ctypes.c_void_p(a.ctypes.data)
    lib.joint_check(p(bodies), p(joints), count, 1.0 / 240.0, 8, p(ref_b), p(ref_j), p(my_b), p(my_j))
    broken = 0
    for k in range(count):
        r, m = ref_j[k:k + 1], my_j[k:k + 1]  # views: the padding bytes are the records' own
        lib.joint_check_reset_break(p(r), p(m), 1.0 / 240.0, 0)
        assert _same(_rows(r, [0]), _rows(m, [0]))
        broken += int(r["broken"][0])
        lib.joint_check_reset_break(p(r), p(m), 1.0 / 240.0, 1)
        assert _same(_rows(r, [0]), _rows(m, [0])) and r["broken"][0] == 0
    assert 0 < broken < count
