"""Test infrastructure: ctypes binding of the reference engine built from its
sources by oracle/Makefile (oracle/_ref/libvelox_ref_*.so, see ref_shim.cpp).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, as the checker / baseline — never as the product path.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
STRICT = os.path.join(REF_DIR, "libvelox_ref_strict.so")
FAST = os.path.join(REF_DIR, "libvelox_ref_fast.so")
# The reference engine whose CUDA backend is velox_b200/dropin/b200_backend.cpp.
DROPIN = os.path.join(REF_DIR, "libvelox_ref_dropin.so")
# The same engine over a fake of the library's Backend entry points (no GPU).
DROPIN_FAKE = os.path.join(REF_DIR, "libvelox_ref_dropin_fake.so")
# The reference engine with its own CUDA backend (src/backend_cuda.cu, sm_100a):
# strict floating point (the GPU solver oracle) and the default build (timed).
CUDA_STRICT = os.path.join(REF_DIR, "libvelox_ref_cuda_strict.so")
CUDA_FAST = os.path.join(REF_DIR, "libvelox_ref_cuda_fast.so")

BACKEND_CPU = 1
BACKEND_CUDA_EMULATED = 2


def _path(strict):
    if strict == "dropin":
        return DROPIN
    if strict == "dropin_fake":
        return DROPIN_FAKE
    if strict == "cuda":
        return CUDA_STRICT
    if strict == "cuda_fast":
        return CUDA_FAST
    return STRICT if strict else FAST


def available(strict=True):
    return os.path.exists(_path(strict))


_libs = {}


def lib(strict=True):
    """strict=True: strict-FP build; False: default Release build; "dropin":
    strict build whose CUDA backend is the B200 library."""
    path = _path(strict)
    if path in _libs:
        return _libs[path]
    if not os.path.exists(path):
        raise RuntimeError(f"reference build missing: {path} (run `make -C oracle ref`)")
    L = ctypes.CDLL(path)
    vp, u32, i32, f32 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int, ctypes.c_float
    sig = {
        "ref_last_error": ([], ctypes.c_char_p),
        "ref_is_strict": ([], i32),
        "ref_world_new": ([i32], vp),
        "ref_world_free": ([vp], None),
        "ref_world_backend_name": ([vp], ctypes.c_char_p),
        "ref_world_build": ([vp, vp, u32, vp], i32),
        "ref_world_body_count": ([vp], u32),
        "ref_world_get_bodies": ([vp, vp], None),
        "ref_world_set_bodies": ([vp, vp], None),
        "ref_world_soup": ([vp, vp, vp, ctypes.POINTER(u32)], u32),
        "ref_world_captured_soup": ([vp, vp, vp, ctypes.POINTER(u32)], u32),
        "ref_world_configure": ([vp, f32, f32, f32, i32, vp, i32], None),
        "ref_world_worker_count": ([vp], u32),
        "ref_world_step": ([vp, f32, i32], i32),
        "ref_world_last_call_ms": ([vp], ctypes.c_double),
        "ref_world_stats": ([vp, vp], None),
        "ref_world_contacts": ([vp, vp, u32], u32),
        "ref_world_prev_contacts": ([vp, vp, u32], u32),
        "ref_world_events": ([vp, vp, u32], u32),
        "ref_world_sleep_config": ([vp, f32, f32, f32, f32, f32, f32, i32, i32, i32], None),
        "ref_world_fix_tie_order": ([vp, i32], None),
        "ref_world_found_contacts": ([vp, vp, u32], u32),
        "ref_candidate_pairs": ([vp, u32, f32, vp, u32, vp], u32),
        "ref_world_add_compound": ([vp, vp, vp, u32, vp], i32),
        "ref_world_add_static_mesh": ([vp, vp, u32, vp, u32], i32),
        "ref_world_add_heightfield": ([vp, u32, u32, f32, vp, vp], i32),
        "ref_world_soup_part": ([vp, i32, vp, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)], u32),
        "ref_world_add_joint": ([vp, i32, u32, u32, vp, vp], i32),
        "ref_world_joint_count": ([vp], u32),
        "ref_world_joint_get": ([vp, u32, vp], None),
        "ref_world_joint_set": ([vp, u32, vp], None),
        "ref_world_joints": ([vp, vp, u32], u32),
        "ref_body_aabb": ([vp, f32, vp], None),
        "ref_collide_pairs": ([vp, vp, vp, u32, f32, vp, u32, vp], u32),
        "ref_gjk": ([vp, vp, vp, vp], None),
        "ref_sort_contacts": ([vp, u32], None),
        "ref_color_contacts": ([vp, u32, vp, u32, vp], u32),
        "ref_solve_sequence": ([vp, vp, u32, f32, vp, i32, i32], None),
        "ref_integrate_velocities": ([vp, u32, f32, f32, f32, f32], None),
        "ref_integrate_transforms": ([vp, u32, f32], None),
        "ref_scene_generate": ([i32, ctypes.c_uint64, u32, vp, u32, ctypes.POINTER(u32), vp, u32,
                                ctypes.POINTER(u32)], i32),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _libs[path] = L
    return L


def _p(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None and a.size else ctypes.c_void_p(0)


def generate_scene(config, seed=None, size=0, strict=False):
    """Specs + hull point pool of a benchmark workload, from the scene
    generator compiled into the reference build (the same source and seeds as
    the library's vxb_scene_generate). A process that only times the reference
    builds its scene through this and loads no library of this package."""
    from velox_b200.binding import SPEC  # record layout only (no library load)
    L = lib(strict)
    seed = config if seed is None else seed
    count, npool = ctypes.c_uint32(), ctypes.c_uint32()
    if L.ref_scene_generate(config, seed, size, None, 0, ctypes.byref(count), None, 0, ctypes.byref(npool)) != 0:
        raise RuntimeError("scene generation failed")
    specs = np.zeros(count.value, SPEC)
    pts = np.zeros((max(npool.value, 1), 3), np.float32)
    if L.ref_scene_generate(config, seed, size, _p(specs), count.value, ctypes.byref(count), _p(pts), npool.value,
                            ctypes.byref(npool)) != 0:
        raise RuntimeError("scene generation failed")
    return specs, pts[:npool.value]


class RefWorld:
    """A reference World built from shape specs (dense index == spec index)."""

    def __init__(self, specs, pool, backend=BACKEND_CUDA_EMULATED, strict=True, fix_tie_order=True,
                 reverse_ties=False):
        from velox_b200.binding import BODY  # record layout only
        self._BODY = BODY
        self.L = lib(strict)
        self.h = self.L.ref_world_new(backend)
        if not self.h:
            raise RuntimeError(self.L.ref_last_error().decode())
        pool = np.ascontiguousarray(pool, np.float32)
        if self.L.ref_world_build(self.h, _p(specs), len(specs), _p(pool)) != 0:
            raise RuntimeError(self.L.ref_last_error().decode())
        self.n = len(specs)
        # the emulated backend's worlds fix the reference's unspecified
        # within-pair order of the warm-start cache (no effect elsewhere)
        self.fix_tie_order(fix_tie_order, reverse_ties)

    def close(self):
        if self.h:
            self.L.ref_world_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def configure(self, gravity=(0.0, -9.81, 0.0), substeps=4, solver=None, workers=1):
        self.L.ref_world_configure(self.h, gravity[0], gravity[1], gravity[2], substeps,
                                   ctypes.byref(solver) if solver is not None else None, workers)

    def bodies(self):
        out = np.zeros(self.n, self._BODY)
        self.L.ref_world_get_bodies(self.h, _p(out))
        return out

    def set_bodies(self, b):
        self.L.ref_world_set_bodies(self.h, _p(np.ascontiguousarray(b)))

    def soup(self):
        nf = ctypes.c_uint32()
        npts = self.L.ref_world_soup(self.h, None, None, ctypes.byref(nf))
        pts = np.zeros((max(npts, 1), 3), np.float32)
        faces = np.zeros(max(nf.value, 1), np.uint32)
        self.L.ref_world_soup(self.h, _p(pts), _p(faces), ctypes.byref(nf))
        return pts[:npts], faces[:nf.value]

    def _added(self, index):
        if index < 0:
            raise RuntimeError(self.L.ref_last_error().decode())
        self.n += 1
        return index

    def add_compound(self, spec, children, pool=None):
        """World::addCompound at spec's position with spec's mass, then the
        spec's orientation, velocities, friction, restitution and enableSleep.
        children: velox_b200 COMPOUND_CHILD records (hull children index
        `pool`). Returns the body's dense index."""
        from velox_b200.binding import COMPOUND_CHILD, SPEC, records
        spec = records(np.atleast_1d(spec), SPEC)
        children = records(np.atleast_1d(children), COMPOUND_CHILD)
        pool = np.ascontiguousarray(np.zeros((0, 3)) if pool is None else pool, np.float32)
        return self._added(self.L.ref_world_add_compound(self.h, _p(spec), _p(children), len(children), _p(pool)))

    def add_static_mesh(self, vertices, indices):
        v = np.ascontiguousarray(vertices, np.float32).reshape(-1, 3)
        i = np.ascontiguousarray(indices, np.uint32).reshape(-1)
        return self._added(self.L.ref_world_add_static_mesh(self.h, _p(v), len(v), _p(i), len(i)))

    def add_heightfield(self, heights, cell_size, origin=(0.0, 0.0, 0.0)):
        """heights: (depth, width) samples (World::addStaticHeightfield)."""
        h = np.ascontiguousarray(heights, np.float32)
        o = np.asarray(origin, np.float32)
        return self._added(self.L.ref_world_add_heightfield(self.h, h.shape[1], h.shape[0], cell_size, _p(h), _p(o)))

    def add_joint(self, kind, a, b, p0=(0, 0, 0), p1=(0, 0, 0), axis0=(0, 1, 0), axis1=(0, 1, 0),
                  ground0=(0, 0, 0), ground1=(0, 0, 0), x=(0.0, 0.0, 0.0)):
        """A joint of `kind` (velox_b200.binding JOINT_* / VX_JOINT_*) between
        dense bodies a and b through the World's typed adder; returns its
        creation index. Which arguments a kind reads: ref_shim.cpp."""
        v = np.array([*p0, *p1, *axis0, *axis1, *ground0, *ground1], np.float32)
        xs = np.array(x, np.float32)
        k = self.L.ref_world_add_joint(self.h, kind, a, b, _p(v), _p(xs))
        if k < 0:
            raise RuntimeError(self.L.ref_last_error().decode())
        return k

    def joint(self, k):
        from velox_b200.binding import JOINT
        out = np.zeros(1, JOINT)
        self.L.ref_world_joint_get(self.h, k, _p(out))
        return out

    def set_joint(self, k, record):
        from velox_b200.binding import JOINT, records
        self.L.ref_world_joint_set(self.h, k, _p(records(np.atleast_1d(record), JOINT)))

    def joints(self):
        """World::joints_ in dense order (what the backend receives)."""
        from velox_b200.binding import JOINT
        n = self.L.ref_world_joints(self.h, None, 0)
        if n == 0xffffffff:
            raise RuntimeError("the reference's snapshot layout did not parse")
        out = np.zeros(n, JOINT)
        self.L.ref_world_joints(self.h, _p(out), n)
        return out

    def mesh_soup(self):
        """The world's whole MeshSoup: dict of numpy arrays (record layouts of
        velox_b200.binding)."""
        from velox_b200.binding import BVH_NODE, COMPOUND_CHILD, MESH
        kinds = [("vertices", (np.float32, 3)), ("indices", np.uint32), ("meshes", MESH), ("nodes", BVH_NODE),
                 ("tri_refs", np.uint32), ("hull", (np.float32, 3)), ("faces", np.uint32),
                 ("children", COMPOUND_CHILD)]
        out = {}
        for part, (name, kind) in enumerate(kinds):
            elem = ctypes.c_uint64()
            n = self.L.ref_world_soup_part(self.h, part, None, 0, ctypes.byref(elem))
            if n == 0xffffffff:
                raise RuntimeError("the reference's snapshot layout did not parse")
            if isinstance(kind, tuple):
                arr = np.zeros((n, kind[1]), kind[0])
            else:
                arr = np.zeros(n, kind)
            if n:
                assert elem.value == arr.nbytes // n, (name, elem.value)
                self.L.ref_world_soup_part(self.h, part, _p(arr), arr.nbytes, ctypes.byref(elem))
            out[name] = arr
        return out

    def vx_soup(self):
        """mesh_soup() as a velox_b200 Soup."""
        from velox_b200.binding import make_soup
        s = self.mesh_soup()
        return make_soup(s["hull"], s["faces"], s["vertices"], s["indices"], s["meshes"], s["nodes"], s["tri_refs"],
                         s["children"])

    def step(self, dt=1.0 / 60.0, steps=1):
        if self.L.ref_world_step(self.h, dt, steps) != 0:
            raise RuntimeError(self.L.ref_last_error().decode())
        return self.L.ref_world_last_call_ms(self.h)

    def stats(self):
        out = np.zeros(5, np.uint64)
        self.L.ref_world_stats(self.h, _p(out))
        return dict(zip(["generated", "solved", "iterations", "deviceSubsteps", "awake"], out.tolist()))

    def contacts(self):
        from velox_b200.binding import CONTACT
        m = self.L.ref_world_contacts(self.h, None, 0)
        out = np.zeros(m, CONTACT)
        self.L.ref_world_contacts(self.h, _p(out), m)
        return out

    def fix_tie_order(self, on=True, reverse=False):
        """Before each step, order the warm-start cache within a pair by
        (point, emission order): the reference leaves that order to an
        unstable sort (emulated backend only). reverse: ties in reverse
        emission order there and in the contact sort (another order the
        reference allows)."""
        self.L.ref_world_fix_tie_order(self.h, (2 if reverse else 1) if on else 0)

    def found_contacts(self):
        """The emulated backend's narrow-phase output of the last step (pair
        order, emission order within a pair, before warm-start matching)."""
        from velox_b200.binding import CONTACT
        m = self.L.ref_world_found_contacts(self.h, None, 0)
        out = np.zeros(m, CONTACT)
        self.L.ref_world_found_contacts(self.h, _p(out), m)
        return out

    def events(self):
        """The last step's contact events (dense indices; velox_b200 EVENT layout)."""
        from velox_b200.binding import EVENT
        k = self.L.ref_world_events(self.h, None, 0)
        out = np.zeros(k, EVENT)
        self.L.ref_world_events(self.h, _p(out), k)
        return out

    def sleep_config(self, cfg):
        """World::sleepConfig() from a velox_b200 SleepConfig."""
        self.L.ref_world_sleep_config(self.h, cfg.linearVelocityThreshold, cfg.angularVelocityThreshold,
                                      cfg.accelerationThreshold, cfg.timeToSleep, cfg.timeToDrowsy,
                                      cfg.contactStabilityThreshold, cfg.contactStabilityFrames,
                                      cfg.enableGradualSleep, cfg.enableContactStability)

    def prev_contacts(self):
        """The world's warm-start cache (World::prevContacts_) in its order."""
        from velox_b200.binding import CONTACT
        m = self.L.ref_world_prev_contacts(self.h, None, 0)
        if m == 0xffffffff:
            raise RuntimeError("the reference's snapshot layout did not parse")
        out = np.zeros(m, CONTACT)
        self.L.ref_world_prev_contacts(self.h, _p(out), m)
        return out


def candidate_pairs(bodies, dt, strict=True, soup=None):
    """soup: a velox_b200 Soup (needed when the bodies include meshes)."""
    L = lib(strict)
    sp = ctypes.byref(soup) if soup is not None else None
    n = L.ref_candidate_pairs(_p(bodies), len(bodies), dt, None, 0, sp)
    out = np.zeros(max(n, 1), np.uint64)
    L.ref_candidate_pairs(_p(bodies), len(bodies), dt, _p(out), n, sp)
    return out[:n]


def collide_pairs(bodies, soup, pairs, dt, strict=True):
    from velox_b200.binding import CONTACT
    L = lib(strict)
    pairs = np.ascontiguousarray(pairs, np.uint64)
    cap = 12 * max(len(pairs), 1)
    out = np.zeros(cap, CONTACT)
    counts = np.zeros(max(len(pairs), 1), np.uint32)
    total = L.ref_collide_pairs(_p(bodies), ctypes.byref(soup), _p(pairs), len(pairs), dt, _p(out), cap,
                                _p(counts))
    return out[:total], counts[:len(pairs)]


def gjk_distances(bodies, soup, pairs, strict=True):
    """gjkDistance(makeConvex(a), makeConvex(b)) per pair, rows of 11 floats
    (distance, normal, pointA, pointB, overlapping) like vxb_stage_distance."""
    L = lib(strict)
    pairs = np.ascontiguousarray(pairs, np.uint64)
    out = np.zeros((max(len(pairs), 1), 11), np.float32)
    row = np.zeros(11, np.float32)
    for k, key in enumerate(pairs.tolist()):
        a, b = key >> 32, key & 0xffffffff
        L.ref_gjk(_p(bodies[a:a + 1]), _p(bodies[b:b + 1]), ctypes.byref(soup), _p(row))
        out[k] = row
    return out[:len(pairs)]


def sort_contacts(contacts, strict=True):
    c = np.ascontiguousarray(contacts).copy()
    lib(strict).ref_sort_contacts(_p(c), len(c))
    return c


def color_contacts(bodies, contacts, strict=True):
    colors = np.zeros(max(len(contacts), 1), np.int32)
    nc = lib(strict).ref_color_contacts(_p(bodies), len(bodies), _p(contacts), len(contacts), _p(colors))
    return colors[:len(contacts)], nc


def solve_sequence(bodies, contacts, dt, solver, warm_start=True, sweeps=16, strict=True):
    b = np.ascontiguousarray(bodies).copy()
    c = np.ascontiguousarray(contacts).copy()
    lib(strict).ref_solve_sequence(_p(b), _p(c), len(c), dt, ctypes.byref(solver), int(warm_start), sweeps)
    return b, c


# ---- the C restatement (oracle/velox_oracle.c) -------------------------------

ORACLE = os.path.join(HERE, "_build", "libvelox_oracle.so")
_oracle = None


def oracle():
    global _oracle
    if _oracle is not None:
        return _oracle
    if not os.path.exists(ORACLE):
        raise RuntimeError(f"oracle restatement missing: {ORACLE} (run `make -C oracle oracle`)")
    L = ctypes.CDLL(ORACLE)
    vp, u32 = ctypes.c_void_p, ctypes.c_uint32
    for name, args, res in [
        ("vxo_candidate_pairs", [vp, u32, ctypes.c_float, vp, u32], u32),
        ("vxo_sort_contacts", [vp, u32], None),
        ("vxo_color_contacts", [vp, u32, vp, u32, vp], u32),
        ("vxo_color_order", [vp, u32, u32, vp, vp], None),
        ("vxo_warm_start_match", [vp, u32, vp, u32], u32),
        ("vxo_body_aabb", [vp, ctypes.c_float, vp, vp], None),
    ]:
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _oracle = L
    return L


def oracle_pairs(bodies, dt):
    L = oracle()
    n = L.vxo_candidate_pairs(_p(bodies), len(bodies), dt, None, 0)
    out = np.zeros(max(n, 1), np.uint64)
    L.vxo_candidate_pairs(_p(bodies), len(bodies), dt, _p(out), n)
    return out[:n]


def oracle_sort(contacts):
    c = np.ascontiguousarray(contacts).copy()
    oracle().vxo_sort_contacts(_p(c), len(c))
    return c


def oracle_color(bodies, contacts):
    colors = np.zeros(max(len(contacts), 1), np.int32)
    nc = oracle().vxo_color_contacts(_p(bodies), len(bodies), _p(contacts), len(contacts), _p(colors))
    return colors[:len(contacts)], nc


def oracle_color_order(colors, num_colors):
    colors = np.ascontiguousarray(colors, np.int32)
    order = np.zeros(max(len(colors), 1), np.uint32)
    starts = np.zeros(num_colors + 1, np.uint32)
    oracle().vxo_color_order(_p(colors), len(colors), num_colors, _p(order), _p(starts))
    return order[:len(colors)], starts


def oracle_warm_start(cur, prev):
    c = np.ascontiguousarray(cur).copy()
    p = np.ascontiguousarray(prev)
    warm = oracle().vxo_warm_start_match(_p(c), len(c), _p(p), len(p))
    return c, warm


# ---- the FP64 frozen-contact step and its adjoint (oracle/adjoint_ref.c) ------

ADJREF = os.path.join(HERE, "_build", "libvelox_adjref.so")
_adjref = None


class AdjConfig(ctypes.Structure):
    _fields_ = [("dt", ctypes.c_double), ("gx", ctypes.c_double), ("gy", ctypes.c_double), ("gz", ctypes.c_double),
                ("substeps", ctypes.c_int), ("sweeps", ctypes.c_int), ("positionIterations", ctypes.c_int),
                ("stackStabilization", ctypes.c_int), ("stackStiffness", ctypes.c_double),
                ("stackDamping", ctypes.c_double)]

    @classmethod
    def make(cls, dt=1.0 / 60.0, gravity=(0.0, -9.81, 0.0), substeps=4, velocity_iterations=8,
             position_iterations=3, stack_stabilization=0, stack_stiffness=1000.0, stack_damping=10.0):
        return cls(dt, gravity[0], gravity[1], gravity[2], substeps, 2 * velocity_iterations, position_iterations,
                   stack_stabilization, stack_stiffness, stack_damping)


def adjref():
    global _adjref
    if _adjref is not None:
        return _adjref
    if not os.path.exists(ADJREF):
        raise RuntimeError(f"adjoint restatement missing: {ADJREF} (run `make -C oracle oracle`)")
    L = ctypes.CDLL(ADJREF)
    vp = ctypes.c_void_p
    L.adjref_run.argtypes = [ctypes.POINTER(AdjConfig), vp, ctypes.c_uint32, vp, vp, vp, vp, vp, vp, vp,
                             ctypes.c_uint32, vp, vp, vp, vp, vp, ctypes.POINTER(ctypes.c_uint64)]
    L.adjref_run.restype = ctypes.c_int
    L.adjref_force_branches.argtypes = [vp, ctypes.c_uint32]
    L.adjref_force_branches.restype = None
    L.adjref_record_branches.argtypes = [vp, ctypes.c_uint32]
    L.adjref_record_branches.restype = None
    L.adjref_set_state_noise.argtypes = [ctypes.c_double, ctypes.c_uint64]
    L.adjref_set_state_noise.restype = None
    _adjref = L
    return L


def adjoint_reference(cfg, bodies, state0, inv_mass, inv_inertia, contacts, step_start, src, color, seed=None,
                      branches=None, record=None, noise=0.0, noise_seed=0):
    """FP64 frozen-contact rollout from state0 (n x 13: p, q, v, w) over the
    recorded contacts of each step. Returns (final state, branch hash) and, with
    a seed (dL/d final state), also (dL/d state0, dL/d invMass, dL/d invInertia).
    `branches` (steps x blocks x rows uint8, one world's slice of
    Context.adjoint_backward_branches): follow those branch decisions instead
    of deciding them. `record` (an array of that shape): receives the
    decisions the run takes. `noise` > 0: perturb the state by up to that
    relative amount after every substep (seeded by `noise_seed`), an FP32-like
    evaluation for estimating the problem's conditioning."""
    from velox_b200.binding import BODY, CONTACT, records  # record layouts only (no library load)
    L = adjref()
    n = len(bodies)
    bodies = records(bodies, BODY)
    contacts = records(contacts, CONTACT)
    state0 = np.ascontiguousarray(state0, np.float64)
    inv_mass = np.ascontiguousarray(inv_mass, np.float64)
    inv_inertia = np.ascontiguousarray(inv_inertia, np.float64)
    step_start = np.ascontiguousarray(step_start, np.uint32)
    src = np.ascontiguousarray(src, np.uint32)
    color = np.ascontiguousarray(color, np.int32)
    out = np.zeros((n, 13), np.float64)
    h = ctypes.c_uint64()
    grad = gim = gii = None
    if seed is not None:
        seed = np.ascontiguousarray(seed, np.float64)
        grad = np.zeros((n, 13), np.float64)
        gim = np.zeros(n, np.float64)
        gii = np.zeros(n, np.float64)
    if branches is not None:
        branches = np.ascontiguousarray(branches, np.uint8)
        L.adjref_force_branches(_p(branches), branches.shape[-1])
    if record is not None:
        assert record.dtype == np.uint8 and record.flags["C_CONTIGUOUS"]
        L.adjref_record_branches(_p(record), record.shape[-1])
    L.adjref_set_state_noise(float(noise), int(noise_seed))
    try:
        rc = L.adjref_run(ctypes.byref(cfg), _p(bodies), n, _p(state0), _p(inv_mass),
                          _p(inv_inertia), _p(contacts), _p(step_start), _p(src), _p(color), len(step_start) - 1,
                          _p(out), _p(seed), _p(grad), _p(gim), _p(gii), ctypes.byref(h))
    finally:
        L.adjref_force_branches(None, 0)
        L.adjref_record_branches(None, 0)
        L.adjref_set_state_noise(0.0, 0)
    if rc != 0:
        raise ValueError("adjoint restatement: anisotropic inverse inertia")
    if seed is None:
        return out, h.value
    return out, h.value, grad, gim, gii
