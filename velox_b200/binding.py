"""ctypes binding of libvelox_b200.so and numpy views of its records.

The records mirror include/velox_b200_types.h (and through it the reference
engine's velox::Body / velox::Contact host layouts).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libvelox_b200.so")

VXB_OK = 0
VXB_ERR_INVALID = 1
STATUS = {0: "ok", 1: "invalid", 2: "no device", 3: "out of memory", 4: "device lost",
          5: "capacity", 6: "unsupported", 7: "timeout"}

SHAPE = dict(sphere=0, plane=1, box=2, capsule=3, mesh=4, hull=5, compound=6, cylinder=7,
             cone=8, rounded_box=9, ellipsoid=10)

_v3 = (np.float32, 3)
_q4 = (np.float32, 4)

CCD_SETTINGS = np.dtype({
    "names": ["quality", "maxAdvancementIterations", "maxRootFindIterations", "distanceTolerance",
              "timeTolerance", "enableRotationalCcd", "enableCompoundCcd", "useBrentRootFinder",
              "meshBvhMaxDepth", "speculativeMargin"],
    "formats": [np.uint8, np.uint32, np.uint32, np.float32, np.float32, np.uint8, np.uint8, np.uint8,
                np.uint32, np.float32],
    "offsets": [0, 4, 8, 12, 16, 20, 21, 22, 24, 28],
    "itemsize": 32})

CCD_TUNING = np.dtype({
    "names": ["quality", "collisionMargin", "speculativeDistance", "enableContinuous",
              "minVelocityForCCD", "ccdSettings"],
    "formats": [np.uint8, np.float32, np.float32, np.uint8, np.float32, CCD_SETTINGS],
    "offsets": [0, 4, 8, 12, 16, 20],
    "itemsize": 52})

BODY = np.dtype({
    "names": ["position", "orientation", "velocity", "angularVelocity", "force", "torque", "invMass",
              "invInertia", "inertiaOrientation", "restitution", "friction", "frictionScale",
              "rollingFriction", "spinningFriction", "frictionCombine", "restitutionCombine",
              "linearDamping", "angularDamping", "gravityScale", "motionType", "ccdTuning",
              "geometryQuality", "categoryBits", "maskBits", "groupIndex", "sensor", "enableSleep",
              "fixedRotation", "asleep", "sleepTimer", "shape", "radius", "halfExtents",
              "capsuleHalfHeight", "planeNormal", "planeOffset", "meshIndex", "hullFirst", "hullCount",
              "hullFaceFirst", "hullFaceCount", "compoundFirst", "compoundCount"],
    "formats": [_v3, _q4, _v3, _v3, _v3, _v3, np.float32, _v3, _q4, np.float32, np.float32, _v3,
                np.float32, np.float32, np.uint8, np.uint8, np.float32, np.float32, np.float32, np.uint8,
                CCD_TUNING, np.uint8, np.uint32, np.uint32, np.int32, np.uint8, np.uint8, np.uint8,
                np.uint8, np.float32, np.uint8, np.float32, _v3, np.float32, _v3, np.float32, np.uint32,
                np.uint32, np.uint32, np.uint32, np.uint32, np.uint32, np.uint32],
    "offsets": [0, 12, 28, 40, 52, 64, 76, 80, 92, 108, 112, 116, 128, 132, 136, 137, 140, 144, 148,
                152, 156, 208, 212, 216, 220, 224, 225, 226, 227, 228, 232, 236, 240, 252, 256, 268,
                272, 276, 280, 284, 288, 292, 296],
    "itemsize": 320})

CONTACT = np.dtype({
    "names": ["a", "b", "featureKey", "normal", "point", "localAnchorA", "localAnchorB", "gap", "bias0",
              "vn0", "restitution", "friction1", "friction2", "rollingFriction", "spinningFriction",
              "normalImpulse", "tangentImpulse1", "tangentImpulse2", "rollingImpulse1",
              "rollingImpulse2", "spinningImpulse"],
    "formats": [np.uint32, np.uint32, np.uint64, _v3, _v3, _v3, _v3] + [np.float32] * 14,
    "offsets": [0, 4, 8, 16, 28, 40, 52] + [64 + 4 * k for k in range(14)],
    "itemsize": 128})

SPEC = np.dtype({
    "names": ["shape", "enableSleep", "world", "mass", "radius", "halfHeight", "halfExtents",
              "position", "orientation", "velocity", "angularVelocity", "friction", "restitution",
              "planeNormal", "planeOffset", "hullFirst", "hullCount"],
    "formats": [np.uint8, np.uint8, np.uint32, np.float32, np.float32, np.float32, _v3, _v3, _q4, _v3,
                _v3, np.float32, np.float32, _v3, np.float32, np.uint32, np.uint32],
    "offsets": [0, 1, 4, 8, 12, 16, 20, 32, 44, 60, 72, 84, 88, 92, 104, 108, 112],
    "itemsize": 116})

EVENT = np.dtype({
    "names": ["a", "b", "point", "normal", "impulse", "type", "sensor"],
    "formats": [np.uint32, np.uint32, _v3, _v3, np.float32, np.uint8, np.uint8],
    "offsets": [0, 4, 8, 20, 32, 36, 37],
    "itemsize": 40})
EVENT_TYPES = {0: "begin", 1: "persist", 2: "end"}

# Contact fields that carry physics (padding bytes excluded).
CONTACT_FLOAT_FIELDS = ["normal", "point", "localAnchorA", "localAnchorB", "gap", "bias0", "vn0",
                        "restitution", "friction1", "friction2", "rollingFriction", "spinningFriction",
                        "normalImpulse", "tangentImpulse1", "tangentImpulse2", "rollingImpulse1",
                        "rollingImpulse2", "spinningImpulse"]


class SleepConfig(ctypes.Structure):
    """vxb_sleep_config (velox::SleepConfig's thresholds)."""
    _fields_ = [("linearVelocityThreshold", ctypes.c_float), ("angularVelocityThreshold", ctypes.c_float),
                ("accelerationThreshold", ctypes.c_float), ("timeToSleep", ctypes.c_float),
                ("timeToDrowsy", ctypes.c_float), ("contactStabilityThreshold", ctypes.c_float),
                ("contactStabilityFrames", ctypes.c_int32), ("enableGradualSleep", ctypes.c_uint8),
                ("enableContactStability", ctypes.c_uint8), ("pad", ctypes.c_uint8 * 2)]

    @classmethod
    def default(cls, **kw):
        c = cls()
        lib().vxb_sleep_config_default(ctypes.byref(c))
        for k, v in kw.items():
            setattr(c, k, v)
        return c


class SolverOptions(ctypes.Structure):
    _fields_ = [("impulseThreshold", ctypes.c_float), ("stackStiffness", ctypes.c_float),
                ("stackDamping", ctypes.c_float), ("velocityIterations", ctypes.c_int32),
                ("positionIterations", ctypes.c_int32), ("frictionModel", ctypes.c_uint8),
                ("iterationPolicy", ctypes.c_uint8), ("enableStackStabilization", ctypes.c_uint8),
                ("reserved", ctypes.c_uint8)]

    @classmethod
    def default(cls, **kw):
        o = cls(1e-5, 1000.0, 10.0, 8, 3, 0, 0, 0, 0)
        for k, v in kw.items():
            setattr(o, k, v)
        return o


class Vec3(ctypes.Structure):
    _fields_ = [("x", ctypes.c_float), ("y", ctypes.c_float), ("z", ctypes.c_float)]


class Soup(ctypes.Structure):
    _fields_ = [("hullPoints", ctypes.c_void_p), ("hullPointCount", ctypes.c_uint32),
                ("hullFaceIndices", ctypes.c_void_p), ("hullFaceIndexCount", ctypes.c_uint32),
                ("vertices", ctypes.c_void_p), ("vertexCount", ctypes.c_uint32),
                ("indices", ctypes.c_void_p), ("indexCount", ctypes.c_uint32),
                ("meshes", ctypes.c_void_p), ("meshCount", ctypes.c_uint32),
                ("bvhNodes", ctypes.c_void_p), ("bvhNodeCount", ctypes.c_uint32),
                ("bvhTriRefs", ctypes.c_void_p), ("bvhTriRefCount", ctypes.c_uint32),
                ("compoundChildren", ctypes.c_void_p), ("compoundChildCount", ctypes.c_uint32)]


# velox::Mesh, velox::BvhNode and velox::CompoundChild records (vx_mesh,
# vx_bvh_node, vx_compound_child in include/velox_b200_types.h).
MESH = np.dtype([("firstVertex", "<u4"), ("vertexCount", "<u4"), ("firstIndex", "<u4"), ("indexCount", "<u4"),
                 ("firstNode", "<u4"), ("nodeCount", "<u4"), ("firstTriRef", "<u4"),
                 ("aabbMin", "<f4", 3), ("aabbMax", "<f4", 3)])
BVH_NODE = np.dtype([("aabbMin", "<f4", 3), ("aabbMax", "<f4", 3), ("leftFirst", "<u4"), ("triCount", "<u4")])
COMPOUND_CHILD = np.dtype({"names": ["shape", "localPosition", "localOrientation", "radius", "halfExtents",
                                     "capsuleHalfHeight", "hullFirst", "hullCount", "hullFaceFirst",
                                     "hullFaceCount"],
                           "formats": ["u1", ("<f4", 3), ("<f4", 4), "<f4", ("<f4", 3), "<f4", "<u4", "<u4",
                                       "<u4", "<u4"],
                           "offsets": [0, 4, 16, 32, 36, 48, 52, 56, 60, 64], "itemsize": 68})
assert MESH.itemsize == 52 and BVH_NODE.itemsize == 32

# velox::Joint (vx_joint in include/velox_b200_types.h, 420 bytes).
JOINT = np.dtype({
    "names": ["type", "a", "b", "localAnchorA", "localAnchorB", "localAxisA", "localAxisB", "localRefA",
              "localRefB", "restLength", "collideConnected", "enableSpring", "springFrequencyHz",
              "springDampingRatio", "breakForce", "breakTorque", "enableMotor", "motorSpeed", "maxMotorTorque",
              "maxMotorForce", "enableLimit", "lowerLimit", "upperLimit", "enableSwingLimit", "swingLimit",
              "enableTwistLimit", "lowerTwistLimit", "upperTwistLimit", "linearLimitMask", "angularLimitMask",
              "linearMotorMask", "angularMotorMask", "lowerLinearLimit", "upperLinearLimit", "lowerAngularLimit",
              "upperAngularLimit", "linearMotorSpeed", "angularMotorSpeed", "maxLinearMotorForce",
              "maxAngularMotorTorque", "weldFrequencyHz", "weldDampingRatio", "suspensionFrequencyHz",
              "suspensionDampingRatio", "wheelRadius", "enableSteering", "steeringAngle", "maxSteeringAngle",
              "maxLength", "pulleyAnchorA", "pulleyAnchorB", "pulleyRatio", "gearRatio", "motorImpulse",
              "limitImpulse", "swingImpulse", "twistImpulse", "springImpulse", "linearMotorImpulse",
              "angularMotorImpulse", "linearLimitImpulse", "angularLimitImpulse", "reactionLinearImpulse",
              "reactionAngularImpulse", "broken"],
    "formats": ["u1", "<u4", "<u4"] + [("<f4", 3)] * 6 + ["<f4", "u1", "u1", "<f4", "<f4", "<f4", "<f4", "u1",
                "<f4", "<f4", "<f4", "u1", "<f4", "<f4", "u1", "<f4", "u1", "<f4", "<f4", "u1", "u1", "u1", "u1"]
               + [("<f4", 3)] * 8 + ["<f4"] * 5 + ["u1", "<f4", "<f4", "<f4", ("<f4", 3), ("<f4", 3), "<f4", "<f4",
                "<f4", "<f4", "<f4", "<f4", "<f4"] + [("<f4", 3)] * 6 + ["u1"],
    "offsets": [0, 4, 8, 12, 24, 36, 48, 60, 72, 84, 88, 89, 92, 96, 100, 104, 108, 112, 116, 120, 124, 128, 132,
                136, 140, 144, 148, 152, 156, 157, 158, 159, 160, 172, 184, 196, 208, 220, 232, 244, 256, 260, 264,
                268, 272, 276, 280, 284, 288, 292, 304, 316, 320, 324, 328, 332, 336, 340, 344, 356, 368, 380, 392,
                404, 416],
    "itemsize": 420})


class StepConfig(ctypes.Structure):
    _fields_ = [("dt", ctypes.c_float), ("gravity", Vec3), ("substeps", ctypes.c_int32),
                ("solver", SolverOptions)]


class StepStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in ("candidatePairs", "contacts", "colors", "islands",
                                               "largestIsland", "rewinds", "velocityIterations",
                                               "warmStarted", "colorRounds", "giantIslands",
                                               "rewindRounds", "rewindReplays", "rewindGapQueries",
                                               "rewindCriticalMicros", "rewindSpeculateMicros")]


def ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None and a.size else ctypes.c_void_p(0)


def records(a, dtype, inout=False):
    """`a` as contiguous records in the C struct layout `dtype`. A structured
    array with the same fields but another layout (np.concatenate of padded
    records drops the padding) is copied field by field; an array the library
    writes into must already be in the layout, else ValueError."""
    if a.dtype == dtype and a.flags["C_CONTIGUOUS"]:
        return a
    if inout or a.dtype.names is None or set(a.dtype.names) != set(dtype.names):
        raise ValueError(f"expected a C-contiguous array of {len(dtype.names)}-field records, itemsize {dtype.itemsize}")
    out = np.zeros(len(a), dtype)
    for name in dtype.names:
        out[name] = a[name]
    return out


_lib = None


def lib(path=LIB_PATH):
    """Loads the library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"velox_b200: {path} is missing; run `python -m velox_b200.build`")
    L = ctypes.CDLL(path)
    vp, u32, i32, f32 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int, ctypes.c_float
    p_u32 = ctypes.POINTER(ctypes.c_uint32)
    sig = {
        "vxb_version": ([], ctypes.c_char_p),
        "vxb_status_string": ([i32], ctypes.c_char_p),
        "vxb_context_create": ([i32, ctypes.POINTER(vp)], i32),
        "vxb_context_destroy": ([vp], None),
        "vxb_context_last_error": ([vp], ctypes.c_char_p),
        "vxb_context_set_stream": ([vp, vp], i32),
        "vxb_context_launch_count": ([vp], ctypes.c_uint64),
        "vxb_context_set_wait_limit": ([vp, u32], i32),
        "vxb_context_host_syncs": ([vp], ctypes.c_uint64),
        "vxb_context_set_tuning": ([vp, i32], i32),
        "vxb_context_tuned_shape": ([vp, i32, u32, p_u32, p_u32, ctypes.POINTER(ctypes.c_int)], i32),
        "vxb_context_tuning_save": ([vp], i32),
        "vxb_context_enable_timing": ([vp, i32], i32),
        "vxb_context_stage_times": ([vp, vp, vp, u32], i32),
        "vxb_backend_integrate": ([vp, vp, u32, Vec3, f32], i32),
        "vxb_backend_find_contacts": ([vp, vp, u32, ctypes.POINTER(Soup), f32, p_u32], i32),
        "vxb_backend_copy_contacts": ([vp, vp, u32], i32),
        "vxb_backend_solve_velocities": ([vp, vp, u32, vp, u32, f32, i32, ctypes.POINTER(SolverOptions),
                                          p_u32], i32),
        "vxb_backend_advance_substeps": ([vp, vp, u32, vp, u32, Vec3, f32, i32,
                                          ctypes.POINTER(SolverOptions), ctypes.POINTER(ctypes.c_int),
                                          p_u32], i32),
        "vxb_backend_fetch_impulses": ([vp, vp, u32], i32),
        "vxb_backend_invalidate": ([vp], i32),
        "vxb_world_load": ([vp, vp, u32, ctypes.POINTER(Soup), vp], i32),
        "vxb_world_configure": ([vp, ctypes.POINTER(StepConfig)], i32),
        "vxb_world_step": ([vp, i32], i32),
        "vxb_world_read_bodies": ([vp, vp, u32], i32),
        "vxb_world_read_poses": ([vp, vp, u32], i32),
        "vxb_world_write_forces": ([vp, vp, u32], i32),
        "vxb_world_read_contacts": ([vp, vp, u32, p_u32], i32),
        "vxb_world_write_contacts": ([vp, vp, u32], i32),
        "vxb_sleep_config_default": ([vp], None),
        "vxb_world_configure_sleep": ([vp, vp], i32),
        "vxb_world_enable_events": ([vp, i32], i32),
        "vxb_world_read_events": ([vp, vp, u32, p_u32], i32),
        "vxb_world_stats": ([vp, ctypes.POINTER(StepStats)], i32),
        "vxb_stage_pairs": ([vp, vp, u32, f32, vp, u32, p_u32], i32),
        "vxb_stage_collide": ([vp, vp, u32, ctypes.POINTER(Soup), vp, u32, f32, vp, u32, vp, p_u32], i32),
        "vxb_stage_pairs_soup": ([vp, vp, u32, ctypes.POINTER(Soup), f32, vp, u32, p_u32], i32),
        "vxb_stage_distance": ([vp, vp, u32, ctypes.POINTER(Soup), vp, u32, i32, vp], i32),
        "vxb_stage_color": ([vp, vp, u32, vp, u32, vp, p_u32], i32),
        "vxb_stage_pairs_noalloc": ([vp, u32, f32, vp, u32, p_u32, vp], i32),
        "vxb_world_snapshot_save": ([vp, u32], i32),
        "vxb_world_snapshot_restore": ([vp, u32], i32),
        "vxb_world_snapshot_bytes": ([vp, ctypes.POINTER(ctypes.c_uint64)], i32),
        "vxb_world_snapshot_read": ([vp, vp, ctypes.c_uint64], i32),
        "vxb_world_snapshot_write": ([vp, vp, ctypes.c_uint64], i32),
        "vxb_tape_begin": ([vp, u32, u32], i32),
        "vxb_tape_info": ([vp, p_u32, p_u32, p_u32], i32),
        "vxb_tape_read": ([vp, vp, vp, vp, vp, vp, vp], i32),
        "vxb_adjoint_backward": ([vp, vp, vp, vp, vp, vp], i32),
        "vxb_adjoint_backward_branches": ([vp, vp, vp, vp, vp, vp, vp, ctypes.c_size_t, vp, vp], i32),
        "vxb_tape_end": ([vp], i32),
        "vxb_scene_generate": ([i32, ctypes.c_uint64, u32, vp, u32, p_u32, vp, u32, p_u32], i32),
        "vxb_bodies_from_specs": ([vp, u32, vp, vp, vp, u32, p_u32, vp, u32, p_u32], i32),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _lib = L
    return L


class VeloxError(RuntimeError):
    def __init__(self, status, message=""):
        super().__init__(f"velox_b200 status {status} ({STATUS.get(status, '?')}): {message}")
        self.status = status


def check(status, ctx=None):
    if status != VXB_OK:
        msg = lib().vxb_context_last_error(ctx).decode() if ctx else ""
        raise VeloxError(status, msg)


def generate_scene(config, seed=None, size=0):
    """Specs + raw hull point pool of a benchmark workload (1..5)."""
    L = lib()
    seed = config if seed is None else seed
    count, pool = ctypes.c_uint32(), ctypes.c_uint32()
    check(L.vxb_scene_generate(config, seed, size, None, 0, ctypes.byref(count), None, 0, ctypes.byref(pool)))
    specs = np.zeros(count.value, SPEC)
    pts = np.zeros((max(pool.value, 1), 3), np.float32)
    check(L.vxb_scene_generate(config, seed, size, ptr(specs), count.value, ctypes.byref(count), ptr(pts),
                               pool.value, ctypes.byref(pool)))
    return specs, pts[:pool.value]


def bodies_from_specs(specs, pool):
    L = lib()
    n = len(specs)
    hc, fc = ctypes.c_uint32(), ctypes.c_uint32()
    check(L.vxb_bodies_from_specs(ptr(specs), n, ptr(pool), None, None, 0, ctypes.byref(hc), None, 0,
                                  ctypes.byref(fc)))
    bodies = np.zeros(n, BODY)
    hull = np.zeros((max(hc.value, 1), 3), np.float32)
    faces = np.zeros(max(fc.value, 1), np.uint32)
    check(L.vxb_bodies_from_specs(ptr(specs), n, ptr(pool), ptr(bodies), ptr(hull), hc.value,
                                  ctypes.byref(hc), ptr(faces), fc.value, ctypes.byref(fc)))
    return bodies, hull[:hc.value], faces[:fc.value]


def make_soup(hull, faces, vertices=None, indices=None, meshes=None, nodes=None, tri_refs=None, children=None):
    """A vx_soup over numpy arrays (kept alive by the returned object)."""
    hull = np.ascontiguousarray(hull, np.float32).reshape(-1, 3)
    faces = np.ascontiguousarray(faces, np.uint32).reshape(-1)
    vertices = np.ascontiguousarray(np.zeros((0, 3)) if vertices is None else vertices, np.float32).reshape(-1, 3)
    indices = np.ascontiguousarray(np.zeros(0) if indices is None else indices, np.uint32).reshape(-1)
    meshes = records(np.zeros(0, MESH) if meshes is None else meshes, MESH)
    nodes = records(np.zeros(0, BVH_NODE) if nodes is None else nodes, BVH_NODE)
    tri_refs = np.ascontiguousarray(np.zeros(0) if tri_refs is None else tri_refs, np.uint32).reshape(-1)
    children = records(np.zeros(0, COMPOUND_CHILD) if children is None else children, COMPOUND_CHILD)
    keep = (hull, faces, vertices, indices, meshes, nodes, tri_refs, children)
    s = Soup(*[x for a in keep for x in (ptr(a) if len(a) else None, len(a))])
    s._keep = keep
    return s


class Context:
    """One pipeline instance (one CUDA stream on one device)."""

    def __init__(self, device=0):
        self.L = lib()
        h = ctypes.c_void_p()
        check(self.L.vxb_context_create(device, ctypes.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            self.L.vxb_context_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, status):
        check(status, self.h)

    def set_wait_limit(self, polls):
        """Polls before a device-side wait gives up (0 = the default)."""
        self._check(self.L.vxb_context_set_wait_limit(self.h, polls))

    @property
    def launches(self):
        return int(self.L.vxb_context_launch_count(self.h))

    @property
    def host_syncs(self):
        """Blocking reads of device counts since the context was created."""
        return int(self.L.vxb_context_host_syncs(self.h))

    TUNE_SITES = {"collide_convex": 0, "collide_complex": 1, "collide_plane": 2, "collide_any": 3,
                  "rewind_probe": 4}

    def set_tuning(self, on=True):
        """Launch-shape autotuning on (the default) or the fixed default shapes."""
        self._check(self.L.vxb_context_set_tuning(self.h, 1 if on else 0))

    def tuned_shape(self, site, items):
        """(threads, blocks per SM, decided) the next launch of `site` over
        `items` items would use."""
        t, b, d = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_int()
        self._check(self.L.vxb_context_tuned_shape(self.h, self.TUNE_SITES.get(site, site), items, ctypes.byref(t),
                                                   ctypes.byref(b), ctypes.byref(d)))
        return t.value, b.value, bool(d.value)

    def tuning_save(self):
        self._check(self.L.vxb_context_tuning_save(self.h))

    STAGES = ["prepare", "broadphase", "cell_sort", "narrowphase", "placement", "warm_start",
              "islands", "solve", "rewind", "positions"]

    def enable_timing(self, on=True):
        self._check(self.L.vxb_context_enable_timing(self.h, int(on)))

    def stage_times(self):
        ms = np.zeros(10, np.float64)
        calls = np.zeros(10, np.uint64)
        self._check(self.L.vxb_context_stage_times(self.h, ptr(ms), ptr(calls), 10))
        return {n: (float(ms[i]), int(calls[i])) for i, n in enumerate(self.STAGES)}

    def set_stream(self, stream_handle):
        self._check(self.L.vxb_context_set_stream(self.h, ctypes.c_void_p(stream_handle)))

    # ---- device world
    def load(self, bodies, soup, world_of=None):
        bodies = records(bodies, BODY)
        self.bodies_n = len(bodies)
        wo = None if world_of is None else np.ascontiguousarray(world_of, np.uint32)
        self.worlds = 1 if wo is None or len(wo) == 0 else int(wo.max()) + 1
        self._check(self.L.vxb_world_load(self.h, ptr(bodies), len(bodies), ctypes.byref(soup), ptr(wo)))

    def configure(self, dt=1.0 / 60.0, substeps=4, gravity=(0.0, -9.81, 0.0), solver=None):
        cfg = StepConfig(dt, Vec3(*gravity), substeps, solver or SolverOptions.default())
        self._check(self.L.vxb_world_configure(self.h, ctypes.byref(cfg)))

    def step(self, steps=1):
        self._check(self.L.vxb_world_step(self.h, steps))

    def read_bodies(self):
        out = np.zeros(self.bodies_n, BODY)
        self._check(self.L.vxb_world_read_bodies(self.h, ptr(out), self.bodies_n))
        return out

    def read_poses(self, out=None):
        if out is None:
            out = np.zeros((self.bodies_n, 7), np.float32)
        self._check(self.L.vxb_world_read_poses(self.h, ptr(out), self.bodies_n))
        return out

    def write_forces(self, ft):
        self._check(self.L.vxb_world_write_forces(self.h, ptr(ft), self.bodies_n))

    def read_contacts(self):
        cnt = ctypes.c_uint32()
        self._check(self.L.vxb_world_read_contacts(self.h, None, 0, ctypes.byref(cnt)))
        out = np.zeros(cnt.value, CONTACT)
        self._check(self.L.vxb_world_read_contacts(self.h, ptr(out), cnt.value, ctypes.byref(cnt)))
        return out

    def configure_sleep(self, config=None, **kw):
        """Sleeping thresholds (SleepConfig.default(**kw) when config is None)."""
        config = config or SleepConfig.default(**kw)
        self._check(self.L.vxb_world_configure_sleep(self.h, ctypes.byref(config)))

    def enable_events(self, on=True):
        self._check(self.L.vxb_world_enable_events(self.h, 1 if on else 0))

    def read_events(self):
        cnt = ctypes.c_uint32()
        self._check(self.L.vxb_world_read_events(self.h, None, 0, ctypes.byref(cnt)))
        out = np.zeros(cnt.value, EVENT)
        self._check(self.L.vxb_world_read_events(self.h, ptr(out), cnt.value, ctypes.byref(cnt)))
        return out

    def write_contacts(self, contacts):
        """Replaces the warm-start cache with `contacts` (sorted by (a, b))."""
        contacts = records(contacts, CONTACT)
        self._check(self.L.vxb_world_write_contacts(self.h, ptr(contacts), len(contacts)))

    def stats(self):
        s = StepStats()
        self._check(self.L.vxb_world_stats(self.h, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in StepStats._fields_}

    # ---- snapshots
    def snapshot_save(self, slot=0):
        self._check(self.L.vxb_world_snapshot_save(self.h, slot))

    def snapshot_restore(self, slot=0):
        self._check(self.L.vxb_world_snapshot_restore(self.h, slot))

    def snapshot_bytes(self):
        """The world's state as a byte image (numpy uint8)."""
        size = ctypes.c_uint64()
        self._check(self.L.vxb_world_snapshot_bytes(self.h, ctypes.byref(size)))
        out = np.zeros(size.value, np.uint8)
        self._check(self.L.vxb_world_snapshot_read(self.h, ptr(out), size.value))
        return out

    def snapshot_load(self, image):
        image = np.ascontiguousarray(image, np.uint8)
        self._check(self.L.vxb_world_snapshot_write(self.h, ptr(image), image.size))

    # ---- adjoint
    def tape_begin(self, steps, checkpoint_every=10):
        """Record the next `steps` steps for vxb_adjoint_backward."""
        self._check(self.L.vxb_tape_begin(self.h, steps, checkpoint_every))

    def tape_info(self):
        r, c, k = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        self._check(self.L.vxb_tape_info(self.h, ctypes.byref(r), ctypes.byref(c), ctypes.byref(k)))
        return {"recorded": r.value, "contacts": c.value, "checkpoints": k.value}

    def tape_read(self):
        """The recorded tape: contacts (after matching), step starts, sources
        (impulse, vn0; 0xffffffff = none), colours, checkpoints (slots x 4 x n
        x 4 floats: position, orientation, velocity, angular velocity), world flags."""
        info = self.tape_info()
        total, slots, n = info["contacts"], info["checkpoints"], self.bodies_n
        contacts = np.zeros(max(total, 1), CONTACT)
        starts = np.zeros(info["recorded"] + 1, np.uint32)
        src = np.zeros((max(total, 1), 2), np.uint32)
        colors = np.zeros(max(total, 1), np.int32)
        ckpt = np.zeros((slots, 4, n, 4), np.float32)
        flags = np.zeros(self.worlds, np.uint32)
        self._check(self.L.vxb_tape_read(self.h, ptr(contacts), ptr(starts), ptr(src), ptr(colors), ptr(ckpt),
                                         ptr(flags)))
        return {"contacts": contacts[:total], "step_start": starts, "src": src[:total], "colors": colors[:total],
                "checkpoints": ckpt, "flags": flags}

    def adjoint_backward(self, seed=None):
        """dL/d(state at the tape's first step) from dL/d(state after its last
        step) (n x 13: position, orientation, velocity, angular velocity).
        Returns (grad n x 13, dL/d(invMass, invInertia) n x 2, dL/dmass n,
        world flags)."""
        n = self.bodies_n
        seed = None if seed is None else np.ascontiguousarray(seed, np.float32).reshape(n, 13)
        grad = np.zeros((n, 13), np.float32)
        ginv = np.zeros((n, 2), np.float32)
        gmass = np.zeros(n, np.float32)
        flags = np.zeros(self.worlds, np.uint32)
        self._check(self.L.vxb_adjoint_backward(self.h, ptr(seed), ptr(grad), ptr(ginv), ptr(gmass), ptr(flags)))
        return grad, ginv, gmass, flags

    def adjoint_backward_branches(self, seed=None):
        """adjoint_backward plus the branch decisions the reverse
        differentiated: uint8 array (worlds, steps, blocks, rows) with blocks
        [substeps live-gap signs, warm start, substeps x sweeps row bits,
        position passes push activity] (vxb_adjoint_backward_branches)."""
        n = self.bodies_n
        seed = None if seed is None else np.ascontiguousarray(seed, np.float32).reshape(n, 13)
        grad = np.zeros((n, 13), np.float32)
        ginv = np.zeros((n, 2), np.float32)
        gmass = np.zeros(n, np.float32)
        flags = np.zeros(self.worlds, np.uint32)
        need, rows = ctypes.c_size_t(), ctypes.c_uint32()
        st = self.L.vxb_adjoint_backward_branches(self.h, ptr(seed), None, None, None, None, None, 0,
                                                   ctypes.byref(need), ctypes.byref(rows))
        if st != 5:  # VXB_ERR_CAPACITY: the size query
            self._check(st)
        bits = np.zeros(need.value, np.uint8)
        self._check(self.L.vxb_adjoint_backward_branches(self.h, ptr(seed), ptr(grad), ptr(ginv), ptr(gmass),
                                                         ptr(flags), ptr(bits), need.value, ctypes.byref(need),
                                                         ctypes.byref(rows)))
        steps = self.tape_info()["recorded"]
        blocks = need.value // max(1, self.worlds * steps * rows.value)
        return grad, ginv, gmass, flags, bits.reshape(self.worlds, steps, blocks, rows.value)

    def tape_end(self):
        self._check(self.L.vxb_tape_end(self.h))

    # ---- stages
    def pairs(self, bodies, dt, soup=None):
        bodies = records(bodies, BODY)
        cnt = ctypes.c_uint32()
        if soup is None:
            call = lambda out, cap: self.L.vxb_stage_pairs(self.h, ptr(bodies), len(bodies), dt, out, cap,
                                                           ctypes.byref(cnt))
        else:
            call = lambda out, cap: self.L.vxb_stage_pairs_soup(self.h, ptr(bodies), len(bodies),
                                                                ctypes.byref(soup), dt, out, cap, ctypes.byref(cnt))
        self._check(call(None, 0))
        out = np.zeros(max(cnt.value, 1), np.uint64)
        self._check(call(ptr(out), cnt.value))
        return out[:cnt.value]

    def collide(self, bodies, soup, pairs, dt, cap=None):
        bodies = records(bodies, BODY)
        pairs = np.ascontiguousarray(pairs, np.uint64)
        cap = cap or max(12 * len(pairs), 1)
        out = np.zeros(cap, CONTACT)
        counts = np.zeros(max(len(pairs), 1), np.uint32)
        total = ctypes.c_uint32()
        self._check(self.L.vxb_stage_collide(self.h, ptr(bodies), len(bodies), ctypes.byref(soup), ptr(pairs),
                                             len(pairs), dt, ptr(out), cap, ptr(counts), ctypes.byref(total)))
        return out[:total.value], counts[:len(pairs)]

    def distance(self, bodies, soup, pairs, path=0):
        """gjkDistance per pair: (npairs, 11) float32 rows (distance, normal,
        pointA, pointB, overlapping)."""
        bodies = records(bodies, BODY)
        pairs = np.ascontiguousarray(pairs, np.uint64)
        out = np.zeros((max(len(pairs), 1), 11), np.float32)
        self._check(self.L.vxb_stage_distance(self.h, ptr(bodies), len(bodies), ctypes.byref(soup), ptr(pairs),
                                              len(pairs), path, ptr(out)))
        return out[:len(pairs)]

    def color(self, bodies, contacts):
        bodies, contacts = records(bodies, BODY), records(contacts, CONTACT)
        colors = np.zeros(max(len(contacts), 1), np.int32)
        nc = ctypes.c_uint32()
        self._check(self.L.vxb_stage_color(self.h, ptr(bodies), len(bodies), ptr(contacts), len(contacts),
                                           ptr(colors), ctypes.byref(nc)))
        return colors[:len(contacts)], nc.value

    # ---- Backend interface
    def backend_integrate(self, bodies, gravity, dt):
        bodies = records(bodies, BODY, inout=True)
        self._check(self.L.vxb_backend_integrate(self.h, ptr(bodies), len(bodies), Vec3(*gravity), dt))

    def backend_find_contacts(self, bodies, soup, dt):
        bodies = records(bodies, BODY)
        cnt = ctypes.c_uint32()
        self._check(self.L.vxb_backend_find_contacts(self.h, ptr(bodies), len(bodies), ctypes.byref(soup), dt,
                                                     ctypes.byref(cnt)))
        out = np.zeros(cnt.value, CONTACT)
        self._check(self.L.vxb_backend_copy_contacts(self.h, ptr(out), cnt.value))
        return out

    def backend_advance_substeps(self, bodies, contacts, gravity, h, substeps, solver=None):
        bodies = records(bodies, BODY, inout=True)
        contacts = records(contacts, CONTACT, inout=True)
        adv = ctypes.c_int()
        it = ctypes.c_uint32()
        opts = solver or SolverOptions.default()
        self._check(self.L.vxb_backend_advance_substeps(self.h, ptr(bodies), len(bodies), ptr(contacts),
                                                        len(contacts), Vec3(*gravity), h, substeps,
                                                        ctypes.byref(opts), ctypes.byref(adv), ctypes.byref(it)))
        return bool(adv.value), it.value

    def backend_fetch_impulses(self, contacts):
        contacts = records(contacts, CONTACT, inout=True)
        self._check(self.L.vxb_backend_fetch_impulses(self.h, ptr(contacts), len(contacts)))
