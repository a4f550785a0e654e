"""Seeded scenes with compound bodies, a heightfield and a triangle mesh,
built through the reference's World (addCompound, addStaticHeightfield,
addStaticMesh, src/world.cpp:987-1477), so both engines consume the same
bodies and the same MeshSoup (BVHs included, read back from the world)."""
import numpy as np

import velox_b200
from velox_b200 import binding

IDENTITY = (0.0, 0.0, 0.0, 1.0)


def _quat(rng):
    q = rng.normal(size=4)
    return q / np.linalg.norm(q)


def _child(shape, pos, q=IDENTITY, radius=0.5, half=(0.5, 0.5, 0.5), hh=0.5, hull=(0, 0)):
    c = np.zeros(1, binding.COMPOUND_CHILD)
    c["shape"] = shape
    c["localPosition"] = pos
    c["localOrientation"] = q
    c["radius"] = radius
    c["halfExtents"] = half
    c["capsuleHalfHeight"] = hh
    c["hullFirst"], c["hullCount"] = hull
    return c


def _blob(rng, count=10, scale=0.25):
    d = rng.normal(size=(count, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return (d * scale * rng.uniform(0.8, 1.2, size=(count, 1))).astype(np.float32)


def compound_kinds(rng, pool):
    """Child lists of the compound families: dumbbell, L block, hull + box,
    cylinder + cone, rounded box + ellipsoid, capsule cross. Hull children
    append their points to `pool` (a list of arrays)."""
    def hull_child(pos):
        pts = _blob(rng)
        first = sum(len(p) for p in pool)
        pool.append(pts)
        return _child(5, pos, tuple(_quat(rng)), hull=(first, len(pts)))

    return [
        np.concatenate([_child(0, (-0.45, 0, 0), radius=0.22), _child(0, (0.45, 0, 0), radius=0.22),
                        _child(3, (0, 0, 0), (0.0, 0.0, 0.7071068, 0.7071068), radius=0.08, hh=0.35)]),
        np.concatenate([_child(2, (-0.25, 0, 0), half=(0.35, 0.12, 0.15)),
                        _child(2, (0.0, 0.3, 0), half=(0.1, 0.3, 0.15))]),
        np.concatenate([hull_child((0.2, 0, 0)), _child(2, (-0.25, 0, 0), tuple(_quat(rng)), half=(0.15, 0.2, 0.1))]),
        np.concatenate([_child(7, (0, -0.2, 0), radius=0.2, hh=0.15), _child(8, (0, 0.2, 0), radius=0.2, hh=0.15)]),
        np.concatenate([_child(9, (0.2, 0, 0), radius=0.05, half=(0.15, 0.1, 0.1)),
                        _child(10, (-0.25, 0, 0), half=(0.2, 0.12, 0.15))]),
        np.concatenate([_child(3, (0, 0, 0), radius=0.09, hh=0.3),
                        _child(3, (0, 0, 0), (0.7071068, 0.0, 0.0, 0.7071068), radius=0.09, hh=0.3),
                        _child(0, (0, 0.3, 0), radius=0.12)]),
    ]


def heightfield(width=12, depth=12, seed=0):
    rng = np.random.default_rng(seed)
    x = np.arange(width)[None, :]
    z = np.arange(depth)[:, None]
    h = 0.35 * np.sin(0.8 * x + 0.3) * np.cos(0.6 * z) + 0.05 * rng.normal(size=(depth, width))
    return h.astype(np.float32)


def ramp_mesh(nx=4, nz=4, origin=(0.5, 0.0, -3.0), size=(5.0, 6.0), slope=0.25):
    """A tilted quad grid (two triangles per cell), a static triangle mesh."""
    xs = np.linspace(0.0, size[0], nx + 1)
    zs = np.linspace(0.0, size[1], nz + 1)
    v = np.array([(origin[0] + x, origin[1] + slope * x + 0.05 * np.sin(3.0 * z), origin[2] + z)
                  for z in zs for x in xs], np.float32)
    idx = []
    for j in range(nz):
        for i in range(nx):
            a = j * (nx + 1) + i
            b, c = a + 1, a + nx + 1
            idx += [a, c, b, b, c, c + 1]
    return v, np.array(idx, np.uint32)


def mesh_compound_world(ref, seed=0, compounds=24, convex=16, projectile=True, fix_tie_order=True,
                        reverse_ties=False, backend=None, strict=True, mesh_rows=4):
    """A RefWorld: a plane at y = -2, a 12 x 12 heightfield (cell 0.6) on
    x in [-7, -0.4], a ramp mesh on x in [0.5, 5.5], `compounds` compound
    bodies (six families), `convex` spheres / boxes / capsules / hulls above
    them, and optionally a fast sphere falling onto the heightfield (the
    rewind's mesh path). Dense indices: specs (plane, convex bodies,
    projectile), heightfield, ramp, compounds."""
    rng = np.random.default_rng(seed)
    spec = binding.SPEC
    specs = np.zeros(1 + convex + (1 if projectile else 0), spec)
    specs["orientation"] = IDENTITY
    specs["friction"] = 0.5
    specs[0]["shape"] = 1
    specs[0]["planeNormal"] = (0, 1, 0)
    specs[0]["planeOffset"] = -2.0
    pool = [np.zeros((0, 3), np.float32)]
    for k in range(convex):
        s = specs[1 + k]
        s["shape"] = (0, 2, 3, 5)[k % 4]
        s["mass"] = 1.0
        s["radius"] = 0.2
        s["halfHeight"] = 0.2
        s["halfExtents"] = (0.2, 0.15, 0.25)
        s["position"] = (rng.uniform(-6.5, 5.0), rng.uniform(2.2, 3.2), rng.uniform(-2.5, 2.5))
        s["orientation"] = _quat(rng)
        s["velocity"] = rng.normal(scale=0.3, size=3)
        if s["shape"] == 5:
            pts = _blob(rng, 12, 0.22)
            s["hullFirst"] = sum(len(p) for p in pool)
            s["hullCount"] = len(pts)
            pool.append(pts)
    if projectile:
        s = specs[-1]
        s["shape"] = 0
        s["mass"] = 0.5
        s["radius"] = 0.15
        s["position"] = (-3.7, 1.6, 0.2)
        s["velocity"] = (0.0, -55.0, 0.0)
    kw = dict(fix_tie_order=fix_tie_order, reverse_ties=reverse_ties, strict=strict)
    if backend is not None:
        kw["backend"] = backend
    hull_pool = np.concatenate(pool).astype(np.float32)
    w = ref.RefWorld(specs, hull_pool, **kw)
    w.add_heightfield(heightfield(seed=seed), 0.6, (-7.0, -0.5, -3.3))
    v, i = ramp_mesh(nx=mesh_rows, nz=mesh_rows)
    w.add_static_mesh(v, i)
    cpool = []
    kinds = compound_kinds(rng, cpool)
    cpool = np.concatenate(cpool) if cpool else np.zeros((0, 3), np.float32)
    for k in range(compounds):
        s = np.zeros(1, spec)
        s["mass"] = 2.0
        s["friction"] = 0.6
        s["restitution"] = 0.1
        s["position"] = (rng.uniform(-6.5, 5.0), rng.uniform(0.9, 2.0), rng.uniform(-2.5, 2.5))
        s["orientation"] = _quat(rng)
        s["velocity"] = rng.normal(scale=0.3, size=3)
        s["angularVelocity"] = rng.normal(scale=0.5, size=3)
        w.add_compound(s, kinds[k % len(kinds)], cpool)
    return w


def load_pair(ref, **kw):
    """(reference world, its bodies, its soup as a velox_b200 Soup)."""
    w = mesh_compound_world(ref, **kw)
    return w, w.bodies(), w.vx_soup()


def device_world(bodies, soup, substeps=4, dt=1.0 / 60.0):
    ctx = velox_b200.Context(0)
    ctx.load(bodies, soup)
    ctx.configure(dt=dt, substeps=substeps)
    return ctx


SOUP_KEYS = ("hull", "faces", "vertices", "indices", "meshes", "nodes", "tri_refs", "children")


def make_soup(s):
    return velox_b200.make_soup(s["hull"], s["faces"], s["vertices"], s["indices"], s["meshes"], s["nodes"],
                                s["tri_refs"], s["children"])


def merge_worlds(parts):
    """Independent worlds [(bodies, mesh_soup dict), ...] as one batch: the
    bodies concatenated (world ids ascending), the soups concatenated with
    every reference into them offset (hull point and face ranges of bodies
    and hull children, mesh indices, compound child ranges, mesh vertex /
    index / node / triangle-reference ranges, and the BVH's node and leaf
    links). Returns (bodies, world_of, soup dict)."""
    bodies, world, acc = [], [], {k: [] for k in SOUP_KEYS}
    off = {k: 0 for k in SOUP_KEYS}
    for w, (b, s) in enumerate(parts):
        b = b.copy()
        hull = b["shape"] == 5
        b["hullFirst"][hull] += off["hull"]
        b["hullFaceFirst"][hull] += off["faces"]
        b["meshIndex"][b["shape"] == 4] += off["meshes"]
        b["compoundFirst"][b["shape"] == 6] += off["children"]
        m = s["meshes"].copy()
        m["firstVertex"] += off["vertices"]
        m["firstIndex"] += off["indices"]
        m["firstNode"] += off["nodes"]
        m["firstTriRef"] += off["tri_refs"]
        nodes = s["nodes"].copy()
        inner = nodes["triCount"] == 0
        nodes["leftFirst"][inner] += off["nodes"]
        nodes["leftFirst"][~inner] += off["tri_refs"]
        ch = s["children"].copy()
        hc = ch["shape"] == 5
        ch["hullFirst"][hc] += off["hull"]
        ch["hullFaceFirst"][hc] += off["faces"]
        shifted = dict(s, meshes=m, nodes=nodes, children=ch)
        for k in SOUP_KEYS:
            acc[k].append(shifted[k])
            off[k] += len(s[k])
        bodies.append(b)
        world.append(np.full(len(b), w, np.uint32))
    return (np.concatenate(bodies), np.concatenate(world),
            {k: np.concatenate(v) for k, v in acc.items()})
