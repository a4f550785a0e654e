// Test infrastructure: a C adapter over the reference engine, compiled from the
// reference sources by oracle/Makefile into oracle/_ref/. Nothing in the
// product links or loads it; only tests and bench.py's CPU-baseline leg do.
//
// It provides
//   * createCudaBackend(): a CPU emulation of the reference CUDA backend's
//     algorithm (src/backend_cuda.cu:390-768) built from the reference's own
//     VELOX_HD routines — all-pairs/grid candidate set, collidePair, host
//     contact sort, greedy first-free-bit colouring, counting sort into colour
//     order, per-colour warm start and 2*velocityIterations coloured sweeps,
//     the advanceSubsteps loop and fetchImpulses. Running World(BackendType::Cuda)
//     against it reproduces the reference CUDA backend's step on the CPU
//     (colour order makes the parallel solve equal to this sequential one).
//   * extern "C" entry points for scene building, stepping and the
//     individual stages (pair set, narrow phase, colouring, coloured solve).
#include "velox/world.h"
#include "velox/backend.h"
#include "velox/sleep.h"
#include "velox/serialization.h"
#include "narrowphase.h"
#include "joint_solver.h"
#include "mass_properties.h"
#include "velox_b200_types.h"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

static_assert(sizeof(velox::Body) == sizeof(vx_body), "Body layout");
static_assert(offsetof(velox::Body, ccdTuning) == offsetof(vx_body, ccdTuning), "Body.ccdTuning");
static_assert(offsetof(velox::Body, shape) == offsetof(vx_body, shape), "Body.shape");
static_assert(offsetof(velox::Body, hullFaceCount) == offsetof(vx_body, hullFaceCount), "Body.hullFaceCount");
static_assert(offsetof(velox::Body, sleepTimer) == offsetof(vx_body, sleepTimer), "Body.sleepTimer");
static_assert(sizeof(velox::Contact) == sizeof(vx_contact), "Contact layout");
static_assert(offsetof(velox::Contact, spinningImpulse) == offsetof(vx_contact, spinningImpulse), "Contact tail");
static_assert(sizeof(velox::SolverOptions) == sizeof(vx_solver_options), "SolverOptions layout");
static_assert(sizeof(velox::Mesh) == sizeof(vx_mesh), "Mesh layout");
static_assert(sizeof(velox::Joint) == sizeof(vx_joint), "Joint layout");
static_assert(offsetof(velox::Joint, broken) == offsetof(vx_joint, broken), "Joint tail");
static_assert(sizeof(velox::BvhNode) == sizeof(vx_bvh_node), "BvhNode layout");
static_assert(sizeof(velox::CompoundChild) == sizeof(vx_compound_child), "CompoundChild layout");
static_assert(offsetof(velox::CompoundChild, localOrientation) == offsetof(vx_compound_child, localOrientation),
              "CompoundChild.localOrientation");
static_assert(offsetof(velox::CompoundChild, hullFaceCount) == offsetof(vx_compound_child, hullFaceCount),
              "CompoundChild tail");

namespace velox {
namespace {

thread_local std::string g_error;

inline bool inert(const Body& b) { return b.isStatic() || isFullyAsleep(b.asleep); }

struct BoxLH { Vec3 lo, hi; };

// Candidate pair set of the reference CUDA backend: allPairsContactsKernel
// (backend_cuda.cu:272-299) below 4096 bodies, the grid (:174-250) above. Both
// enumerate exactly the pairs i<j whose compact AABBs overlap (planes are
// unbounded, meshes take their root bounds, :100-129), that are not both
// inert and that pass canCollideWith. Returned sorted ascending as (i<<32)|j.
std::vector<uint64_t> candidatePairs(const std::vector<Body>& bodies, float dt, const Mesh* meshes) {
    const size_t n = bodies.size();
    std::vector<BoxLH> boxes(n);
    std::vector<uint32_t> order;
    std::vector<uint32_t> planes;
    for (uint32_t i = 0; i < n; ++i) {
        const Body& b = bodies[i];
        if (b.shape == ShapeType::Plane) {
            boxes[i] = {{-1e30f, -1e30f, -1e30f}, {1e30f, 1e30f, 1e30f}};
            planes.push_back(i);
        } else if (b.shape == ShapeType::Mesh) {
            boxes[i] = {meshes[b.meshIndex].aabbMin, meshes[b.meshIndex].aabbMax};
            order.push_back(i);
        } else {
            bodyAabb(b, dt, boxes[i].lo, boxes[i].hi);
            order.push_back(i);
        }
    }
    std::vector<uint64_t> pairs;
    auto consider = [&](uint32_t i, uint32_t j) {
        uint32_t lo = i < j ? i : j, hi = i < j ? j : i;
        if (!aabbOverlap(boxes[lo].lo, boxes[lo].hi, boxes[hi].lo, boxes[hi].hi)) return;
        if (inert(bodies[lo]) && inert(bodies[hi])) return;
        if (!bodies[lo].canCollideWith(bodies[hi])) return;
        pairs.push_back((uint64_t(lo) << 32) | hi);
    };
    for (size_t p = 0; p < planes.size(); ++p) {
        for (uint32_t i : order) consider(planes[p], i);
        for (size_t q = p + 1; q < planes.size(); ++q) consider(planes[p], planes[q]);
    }
    std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
        return boxes[a].lo.x < boxes[b].lo.x || (boxes[a].lo.x == boxes[b].lo.x && a < b);
    });
    for (size_t s = 0; s < order.size(); ++s) {
        uint32_t i = order[s];
        for (size_t t = s + 1; t < order.size(); ++t) {
            uint32_t j = order[t];
            if (boxes[j].lo.x > boxes[i].hi.x) break;
            consider(i, j);
        }
    }
    std::sort(pairs.begin(), pairs.end());
    return pairs;
}

bool contactLess(const Contact& x, const Contact& y) {
    uint64_t kx = (uint64_t)x.a << 32 | x.b;
    uint64_t ky = (uint64_t)y.a << 32 | y.b;
    if (kx != ky) return kx < ky;
    if (x.point.x != y.point.x) return x.point.x < y.point.x;
    if (x.point.y != y.point.y) return x.point.y < y.point.y;
    return x.point.z < y.point.z;
}

// Greedy first-free-bit colouring exactly as backend_cuda.cu:603-630.
int greedyColor(const std::vector<Body>& bodies, const Contact* contacts, int m,
                int* colorOf) {
    const size_t n = bodies.size();
    std::vector<uint64_t> mask(n, 0);
    std::vector<int> nextColor(n, 64);
    int numColors = 0;
    for (int k = 0; k < m; ++k) {
        const Contact& c = contacts[k];
        bool sensor = bodies[c.a].isSensor() || bodies[c.b].isSensor();
        bool sa = sensor || !bodies[c.a].isDynamic();
        bool sb = sensor || !bodies[c.b].isDynamic();
        uint64_t used = (sa ? 0 : mask[c.a]) | (sb ? 0 : mask[c.b]);
        int color;
        if (~used) {
            color = 0;
            while (used & (1ull << color)) ++color;
        } else {
            int na = sa ? 64 : nextColor[c.a];
            int nb = sb ? 64 : nextColor[c.b];
            color = na > nb ? na : nb;
            if (!sa) nextColor[c.a] = color + 1;
            if (!sb) nextColor[c.b] = color + 1;
        }
        if (color < 64) {
            if (!sa) mask[c.a] |= 1ull << color;
            if (!sb) mask[c.b] |= 1ull << color;
        }
        colorOf[k] = color;
        if (color + 1 > numColors) numColors = color + 1;
    }
    return numColors;
}

void integrateVelocities(std::vector<Body>& bodies, const Vec3& gravity, float dt) {
    for (Body& b : bodies) {  // integrateKernel, backend_cuda.cu:80-89
        if (!b.isDynamic() || b.isLocked() || isFullyAsleep(b.asleep)) continue;
        b.velocity += (gravity * b.gravityScale + b.force * b.solverInvMass()) * dt;
        b.angularVelocity += b.invInertiaMul(b.torque) * dt;
        b.velocity *= 1.0f / (1.0f + b.linearDamping * dt);
        b.angularVelocity *= 1.0f / (1.0f + b.angularDamping * dt);
    }
}

void integrateTransforms(std::vector<Body>& bodies, float dt) {
    for (Body& b : bodies) {  // integrateTransformsKernel, backend_cuda.cu:91-97
        if (b.isStatic() || b.isLocked() || isFullyAsleep(b.asleep)) continue;
        b.advanceTransform(dt);
    }
}

class ColoredCpuBackend final : public Backend {
public:
    const char* name() const override { return "cuda"; }
    uint32_t lastVelocityIterations() const override { return lastIterations_; }

    void integrate(std::vector<Body>& bodies, const Vec3& gravity, float dt) override {
        integrateVelocities(bodies, gravity, dt);
    }

    void findContacts(const std::vector<Body>& bodies, const MeshSoup& meshes, float dt,
                      const std::vector<uint64_t>*, std::vector<Contact>& out) override {
        out.clear();
        soupPoints = meshes.hullPoints;
        soupFaces = meshes.hullFaceIndices;
        if (bodies.size() < 2) return;
        const MeshSoupView soup = view(meshes);
        lastPairs = candidatePairs(bodies, dt, meshes.meshes.data());
        Contact buf[kMaxContactsPerPair];
        for (uint64_t p : lastPairs) {
            BodyIndex i = BodyIndex(p >> 32), j = BodyIndex(p);
            int count = collidePair(bodies[i], bodies[j], i, j, soup, dt, buf,
                                    kMaxContactsPerPair);
            out.insert(out.end(), buf, buf + count);
        }
        lastFound = out;
    }

    void solveVelocities(std::vector<Body>& bodies, std::vector<Contact>& contacts,
                         float dt, bool warmStart, const SolverOptions& options) override {
        lastIterations_ = 0;
        const int m = (int)contacts.size();
        if (m == 0) return;
        if (warmStart) {
            // backend_cuda.cu:587-595 std::sorts contacts that its kernel
            // appended in atomic arrival order, so contacts that tie on
            // (a, b, point) (a box vertex on another box's edge emits the same
            // point under two feature keys) end in an unspecified order. The
            // emulation fixes that order: pair order, then emission order.
            if (reverseTies) std::reverse(contacts.begin(), contacts.end());
            std::stable_sort(contacts.begin(), contacts.end(), contactLess);
            colorOf_.resize(m);
            numColors_ = greedyColor(bodies, contacts.data(), m, colorOf_.data());
            colorStart_.assign(numColors_ + 1, 0);
            for (int k = 0; k < m; ++k) ++colorStart_[colorOf_[k] + 1];
            for (int c = 0; c < numColors_; ++c) colorStart_[c + 1] += colorStart_[c];
            std::vector<int> fill = colorStart_;
            solve_.resize(m);
            for (int k = 0; k < m; ++k) solve_[fill[colorOf_[k]]++] = contacts[k];
            contacts = solve_;
            for (Contact& c : solve_)
                if (!bodies[c.a].isSensor() && !bodies[c.b].isSensor())
                    warmStartContact(bodies[c.a], bodies[c.b], c);
        }
        sweeps_ = 2 * options.velocityIterations;
        lastIterations_ = (uint32_t)sweeps_;
        runSweeps(bodies, dt, options);
    }

    // The joint path (backend_cuda.cu:691-760, prepareJoints :800-880): 64 or
    // more supported joints are coloured greedily over their dynamic
    // endpoints and, every substep after the contact sweeps, reset (broken
    // ones kept from the second substep on), swept kIterations times colour
    // by colour and break-tested. Solving a colour's joints one after another
    // equals the device's parallel pass: they share no dynamic body.
    bool advanceSubsteps(std::vector<Body>& bodies, std::vector<Contact>& contacts,
                         std::vector<Joint>& joints, const Vec3& gravity, float dt,
                         int substeps, const SolverOptions& options) override {
        if (!joints.empty() && joints.size() < 64) return false;
        for (const Joint& joint : joints)
            if (!joint_solver::supported(joint)) return false;
        for (const Joint& joint : joints) {
            if (bodies[joint.a].asleep == bodies[joint.b].asleep) continue;
            bodies[joint.a].asleep = bodies[joint.b].asleep = 0;
            bodies[joint.a].sleepTimer = bodies[joint.b].sleepTimer = 0.0f;
        }
        if (options.iterationPolicy == IterationPolicy::Adaptive) return false;
        const bool hasContacts = !contacts.empty();
        solveVelocities(bodies, contacts, dt, true, options);
        std::vector<int> colorStart, order;
        std::vector<Joint> sorted;
        if (!joints.empty()) colorJoints(bodies, joints, colorStart, order, sorted);
        for (int s = 0; s < substeps; ++s) {
            if (s > 0) {
                integrateVelocities(bodies, gravity, dt);
                if (hasContacts) runSweeps(bodies, dt, options);
            }
            if (!sorted.empty()) {
                for (Joint& joint : sorted)
                    if (!(s > 0 && joint.broken)) joint_solver::reset(joint);
                for (int it = 0; it < joint_solver::kIterations; ++it)
                    for (size_t c = 0; c + 1 < colorStart.size(); ++c)
                        for (int k = colorStart[c]; k < colorStart[c + 1]; ++k) {
                            Joint& joint = sorted[k];
                            if (joint.broken) continue;
                            joint_solver::solve(joint, bodies[joint.a], bodies[joint.b], dt);
                        }
                for (Joint& joint : sorted) {
                    if (joint.broken) continue;
                    float force = length(joint.reactionLinearImpulse) / dt;
                    float torque = length(joint.reactionAngularImpulse) / dt;
                    joint.broken = force > joint.breakForce || torque > joint.breakTorque;
                }
            }
            integrateTransforms(bodies, dt);
        }
        for (size_t k = 0; k < sorted.size(); ++k) joints[order[k]] = sorted[k];
        lastIterations_ *= (uint32_t)substeps;
        return true;
    }

    static void colorJoints(const std::vector<Body>& bodies, const std::vector<Joint>& joints,
                            std::vector<int>& colorStart, std::vector<int>& order, std::vector<Joint>& sorted) {
        const size_t count = joints.size();
        std::vector<uint64_t> mask(bodies.size(), 0);
        std::vector<int> next(bodies.size(), 64), colorOf(count);
        int colors = 0;
        for (size_t k = 0; k < count; ++k) {
            const Joint& joint = joints[k];
            const bool staticA = !bodies[joint.a].isDynamic(), staticB = !bodies[joint.b].isDynamic();
            const uint64_t used = (staticA ? 0 : mask[joint.a]) | (staticB ? 0 : mask[joint.b]);
            int color;
            if (~used) {
                color = 0;
                while (used & (1ull << color)) ++color;
            } else {
                color = std::max(staticA ? 64 : next[joint.a], staticB ? 64 : next[joint.b]);
                if (!staticA) next[joint.a] = color + 1;
                if (!staticB) next[joint.b] = color + 1;
            }
            if (color < 64) {
                if (!staticA) mask[joint.a] |= 1ull << color;
                if (!staticB) mask[joint.b] |= 1ull << color;
            }
            colorOf[k] = color;
            colors = std::max(colors, color + 1);
        }
        colorStart.assign(colors + 1, 0);
        for (int color : colorOf) ++colorStart[color + 1];
        for (int c = 0; c < colors; ++c) colorStart[c + 1] += colorStart[c];
        std::vector<int> fill(colorStart.begin(), colorStart.end() - 1);
        order.assign(count, 0);
        sorted.resize(count);
        for (size_t k = 0; k < count; ++k) {
            const int at = fill[colorOf[k]]++;
            order[at] = (int)k;
            sorted[at] = joints[k];
        }
    }

    void fetchImpulses(std::vector<Contact>& contacts) override {
        if (solve_.empty() || contacts.size() != solve_.size()) return;
        contacts = solve_;
    }

    void invalidateCaches() override { solve_.clear(); }

    std::vector<Contact> solve_;
    std::vector<Contact> lastFound;
    bool reverseTies = false;  // ties in reverse emission order (a second valid realisation)
    std::vector<uint64_t> lastPairs;
    std::vector<Vec3> soupPoints;
    std::vector<uint32_t> soupFaces;

private:
    void runSweeps(std::vector<Body>& bodies, float dt, const SolverOptions& options) {
        for (int it = 0; it < sweeps_; ++it)
            for (Contact& c : solve_)
                if (!bodies[c.a].isSensor() && !bodies[c.b].isSensor())
                    solveContact(bodies[c.a], bodies[c.b], c, dt, options);
    }
    std::vector<int> colorOf_, colorStart_;
    int numColors_ = 0;
    int sweeps_ = 0;
    uint32_t lastIterations_ = 0;
};

thread_local ColoredCpuBackend* g_lastEmulated = nullptr;

}  // namespace

// The drop-in build links velox_b200/dropin/b200_backend.cpp instead, whose
// createCudaBackend() serves World(BackendType::Cuda) from libvelox_b200.so;
// the CUDA build links the reference's own src/backend_cuda.cu.
#if !defined(REF_SHIM_DROPIN) && !defined(REF_SHIM_CUDA)
Backend* createCudaBackend() {
    auto* backend = new ColoredCpuBackend();
    g_lastEmulated = backend;
    return backend;
}
#endif

}  // namespace velox

using namespace velox;

namespace {

struct RefWorld {
    std::unique_ptr<World> world;
    ColoredCpuBackend* emulated = nullptr;
    std::vector<BodyId> ids;
    std::vector<JointId> jointIds;
    std::vector<Vec3> soupPoints;
    std::vector<uint32_t> soupFaces;
    double lastStepMs = 0.0;
    int fixTieOrder = 0;  // 0 left to std::sort, 1 emission order, 2 reverse emission order
};

// Offset and count of World::prevContacts_ inside the world's serialized
// snapshot (SerializationAccess::encode, src/serialization.cpp:263-300: five
// fixed-size fields, then vectors stored as element size, count and
// elements; the sixth vector is prevContacts_). False when it does not parse.
bool locatePrevContacts(const std::vector<uint8_t>& bytes, size_t* offset, uint64_t* count) {
    size_t at = sizeof(Vec3) + sizeof(int) + sizeof(WorldCcdDefaults) + sizeof(WorldMultiToiSettings) +
                sizeof(SolverOptions);
    for (int v = 0; v < 6; ++v) {
        uint64_t elem = 0, n = 0;
        if (at + 16 > bytes.size()) return false;
        std::memcpy(&elem, bytes.data() + at, 8);
        std::memcpy(&n, bytes.data() + at + 8, 8);
        at += 16;
        if (at + elem * n > bytes.size()) return false;
        if (v == 5) {
            if (elem != sizeof(Contact)) return false;
            *offset = at;
            *count = n;
            return true;
        }
        at += elem * n;
    }
    return false;
}

// World::prevContacts_ is std::sorted on the pair key alone
// (src/world.cpp:4517-4520), which leaves the order of one pair's contacts
// unspecified; the nearest-point warm-start fallback (src/world.cpp:4170-4181)
// takes the first of equally near cached contacts, so contacts that share a
// point under two feature keys make the result depend on that order. This
// fixes it to (a, b, point, narrow-phase emission order) by rewriting the
// cache through the world's own snapshot round trip.
void fixPrevContactOrder(RefWorld* w) {
    SerializedScene scene = serializeWorld(*w->world);
    size_t off = 0;
    uint64_t m = 0;
    if (!locatePrevContacts(scene.data, &off, &m)) throw std::runtime_error("snapshot layout did not parse");
    if (m < 2) return;
    std::vector<Contact> prev(m);
    std::memcpy(prev.data(), scene.data.data() + off, m * sizeof(Contact));
    std::vector<std::pair<uint64_t, uint64_t>> emitted;  // (pair and feature key mix, emission index)
    const std::vector<Contact>& found = w->emulated->lastFound;
    auto tag = [](const Contact& c) {
        return ((uint64_t)c.a << 32 | c.b) * 0x9e3779b97f4a7c15ull ^ c.featureKey;
    };
    emitted.reserve(found.size());
    for (size_t k = 0; k < found.size(); ++k) emitted.push_back({tag(found[k]), (uint64_t)k});
    std::sort(emitted.begin(), emitted.end());
    auto rank = [&](const Contact& c) -> uint64_t {
        auto it = std::lower_bound(emitted.begin(), emitted.end(), std::pair<uint64_t, uint64_t>(tag(c), 0));
        return it != emitted.end() && it->first == tag(c) ? it->second : ~0ull;
    };
    std::vector<std::pair<uint64_t, size_t>> order(m);
    const bool reverse = w->fixTieOrder == 2;
    for (size_t k = 0; k < m; ++k) {
        const uint64_t r = rank(prev[k]);
        order[k] = {reverse && r != ~0ull ? ~0ull - 1 - r : r, k};
    }
    std::stable_sort(order.begin(), order.end(), [&](const auto& x, const auto& y) {
        const Contact& cx = prev[x.second];
        const Contact& cy = prev[y.second];
        if (contactLess(cx, cy)) return true;
        if (contactLess(cy, cx)) return false;
        return x.first < y.first;
    });
    std::vector<Contact> sorted(m);
    for (size_t k = 0; k < m; ++k) sorted[k] = prev[order[k].second];
    std::memcpy(scene.data.data() + off, sorted.data(), m * sizeof(Contact));
    deserializeWorld(*w->world, scene);
}

Vec3 V(const vx_vec3& v) { return {v.x, v.y, v.z}; }
Quat Q(const vx_quat& q) { return {q.x, q.y, q.z, q.w}; }

MeshSoupView soupView(const vx_soup* s) {
    MeshSoupView v{};
    if (s) {
        v.hullPoints = reinterpret_cast<const Vec3*>(s->hullPoints);
        v.hullFaceIndices = s->hullFaceIndices;
        v.vertices = reinterpret_cast<const Vec3*>(s->vertices);
        v.indices = s->indices;
        v.meshes = reinterpret_cast<const Mesh*>(s->meshes);
        v.bvhNodes = reinterpret_cast<const BvhNode*>(s->bvhNodes);
        v.bvhTriRefs = s->bvhTriRefs;
        v.compoundChildren = reinterpret_cast<const CompoundChild*>(s->compoundChildren);
    }
    return v;
}

}  // namespace

extern "C" {

const char* ref_last_error(void) { return g_error.c_str(); }

int ref_is_strict(void) { return VELOX_STRICT_FLOATING_POINT ? 1 : 0; }

// backend: 1 = the reference CPU backend, 2 = World(BackendType::Cuda) served
// by the CPU emulation of the CUDA backend above.
void* ref_world_new(int backend) {
    try {
        auto* w = new RefWorld();
        g_lastEmulated = nullptr;
        w->world.reset(new World(backend == 2 ? BackendType::Cuda : BackendType::Cpu));
        if (backend == 2) w->emulated = g_lastEmulated;
        return w;
    } catch (const std::exception& e) {
        g_error = e.what();
        return nullptr;
    }
}

void ref_world_free(void* handle) { delete static_cast<RefWorld*>(handle); }

const char* ref_world_backend_name(void* handle) {
    return static_cast<RefWorld*>(handle)->world->backendName();
}

// Adds the bodies of a scene through World::add* in spec order, so dense
// index == spec index. Hull points are centred exactly as addConvexHull does
// (src/world.cpp:909-985); the resulting hull soup is mirrored for export.
int ref_world_build(void* handle, const vx_shape_spec* specs, uint32_t n,
                    const vx_vec3* pool) {
    auto* w = static_cast<RefWorld*>(handle);
    try {
        for (uint32_t k = 0; k < n; ++k) {
            const vx_shape_spec& s = specs[k];
            BodyId id;
            switch (s.shape) {
            case VX_SHAPE_SPHERE: id = w->world->addSphere(V(s.position), s.radius, s.mass); break;
            case VX_SHAPE_BOX: id = w->world->addBox(V(s.position), V(s.halfExtents), s.mass); break;
            case VX_SHAPE_CAPSULE:
                id = w->world->addCapsule(V(s.position), s.radius, s.halfHeight, s.mass); break;
            case VX_SHAPE_CYLINDER:
                id = w->world->addCylinder(V(s.position), s.radius, s.halfHeight, s.mass); break;
            case VX_SHAPE_PLANE:
                id = w->world->addStaticPlane(V(s.planeNormal), s.planeOffset); break;
            case VX_SHAPE_HULL: {
                std::vector<Vec3> pts;
                for (uint32_t i = 0; i < s.hullCount; ++i) pts.push_back(V(pool[s.hullFirst + i]));
                id = w->world->addConvexHull(V(s.position), pts, s.mass);
                mass_properties::ConvexMassProperties props = mass_properties::convex(pts);
                if (s.mass > 0.0f)
                    for (Vec3& p : pts) p -= props.center;
                w->soupPoints.insert(w->soupPoints.end(), pts.begin(), pts.end());
                for (const auto& t : props.triangles)
                    w->soupFaces.insert(w->soupFaces.end(), t.begin(), t.end());
                break;
            }
            default:
                g_error = "unsupported shape in spec";
                return -1;
            }
            w->ids.push_back(id);
            if (s.shape != VX_SHAPE_PLANE) {
                Body& b = w->world->body(id);
                b.orientation = Q(s.orientation);
                b.velocity = V(s.velocity);
                b.angularVelocity = V(s.angularVelocity);
                b.friction = s.friction;
                b.restitution = s.restitution;
                b.enableSleep = s.enableSleep;
            }
        }
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}

// The state a spec gives a body after World::add* (as ref_world_build does).
static void applySpecState(RefWorld* w, BodyId id, const vx_shape_spec& s) {
    Body& b = w->world->body(id);
    b.orientation = Q(s.orientation);
    b.velocity = V(s.velocity);
    b.angularVelocity = V(s.angularVelocity);
    b.friction = s.friction;
    b.restitution = s.restitution;
    b.enableSleep = s.enableSleep;
}

// World::addCompound (src/world.cpp:987-1301) at spec->position with
// spec->mass; children as vx_compound_child records whose hull children give
// their points as [hullFirst, +hullCount) of `pool`. Returns the dense index
// or -1 (ref_last_error).
int ref_world_add_compound(void* handle, const vx_shape_spec* spec, const vx_compound_child* children,
                           uint32_t count, const vx_vec3* pool) {
    auto* w = static_cast<RefWorld*>(handle);
    try {
        std::vector<CompoundShape> shapes(count);
        for (uint32_t k = 0; k < count; ++k) {
            const vx_compound_child& c = children[k];
            CompoundShape& sh = shapes[k];
            sh.shape = (ShapeType)c.shape;
            sh.localPosition = V(c.localPosition);
            sh.localOrientation = Q(c.localOrientation);
            sh.radius = c.radius;
            sh.halfExtents = V(c.halfExtents);
            sh.capsuleHalfHeight = c.capsuleHalfHeight;
            for (uint32_t i = 0; i < c.hullCount; ++i) sh.hullPoints.push_back(V(pool[c.hullFirst + i]));
        }
        BodyId id = w->world->addCompound(V(spec->position), shapes, spec->mass);
        w->ids.push_back(id);
        applySpecState(w, id, *spec);
        return (int)w->ids.size() - 1;
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}

// World::addStaticMesh (src/world.cpp:1379-1440). Returns the dense index or -1.
int ref_world_add_static_mesh(void* handle, const vx_vec3* vertices, uint32_t vertexCount, const uint32_t* indices,
                              uint32_t indexCount) {
    auto* w = static_cast<RefWorld*>(handle);
    try {
        std::vector<Vec3> v(vertexCount);
        for (uint32_t i = 0; i < vertexCount; ++i) v[i] = V(vertices[i]);
        std::vector<uint32_t> ix(indices, indices + indexCount);
        w->ids.push_back(w->world->addStaticMesh(v, ix));
        return (int)w->ids.size() - 1;
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}

// World::addStaticHeightfield (src/world.cpp:1442-1477). Returns the dense index or -1.
int ref_world_add_heightfield(void* handle, uint32_t width, uint32_t depth, float cellSize, const float* heights,
                              const vx_vec3* origin) {
    auto* w = static_cast<RefWorld*>(handle);
    try {
        std::vector<float> h(heights, heights + (size_t)width * depth);
        w->ids.push_back(w->world->addStaticHeightfield(width, depth, cellSize, h, V(*origin)));
        return (int)w->ids.size() - 1;
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}

// One array of the world's MeshSoup, read from its snapshot (the soup is
// serialised after the 17 state vectors that follow the fixed header):
// part 0 vertices, 1 indices, 2 meshes, 3 bvhNodes, 4 bvhTriRefs, 5 hullPoints,
// 6 hullFaceIndices, 7 compoundChildren. Copies up to capBytes into out and
// returns the element count (element size in *elemSize); ~0u on a layout error.
uint32_t ref_world_soup_part(void* handle, int part, void* out, uint64_t capBytes, uint64_t* elemSize) {
    auto* w = static_cast<RefWorld*>(handle);
    SerializedScene scene = serializeWorld(*w->world);
    const std::vector<uint8_t>& bytes = scene.data;
    size_t at = sizeof(Vec3) + sizeof(int) + sizeof(WorldCcdDefaults) + sizeof(WorldMultiToiSettings) +
                sizeof(SolverOptions);
    for (int v = 0; v <= 17 + part; ++v) {
        uint64_t elem = 0, n = 0;
        if (at + 16 > bytes.size()) return ~0u;
        std::memcpy(&elem, bytes.data() + at, 8);
        std::memcpy(&n, bytes.data() + at + 8, 8);
        at += 16;
        if (at + elem * n > bytes.size()) return ~0u;
        if (v == 17 + part) {
            if (elemSize) *elemSize = elem;
            if (out) std::memcpy(out, bytes.data() + at, std::min<uint64_t>(elem * n, capBytes));
            return (uint32_t)n;
        }
        at += elem * n;
    }
    return ~0u;
}

// A joint between dense bodies a and b through the World's typed adder for
// `type` (include/velox/world.h:617-670). v: six points / axes (p0, p1, axis0,
// axis1, ground0, ground1), x: three scalars; which ones a type reads:
//   Ball, Fixed, SixDof: p0            Distance: p0, p1 (x0 > 0: a spring of
//   x0 Hz and damping x1)              Hinge, ConeTwist, Prismatic, Wheel: p0, axis0
//   Motor: p0, p1, x0 force, x1 torque Weld: p0, x0 / x1 break force / torque
//   Rope: p0, p1, x0 length            Pulley: p0, p1, ground0, ground1, x0 ratio
//   Gear: axis0, axis1, x0 ratio
// Returns the joint's index (creation order) or -1 (ref_last_error).
int ref_world_add_joint(void* handle, int type, uint32_t a, uint32_t b, const float* v, const float* x) {
    auto* w = static_cast<RefWorld*>(handle);
    try {
        World& W = *w->world;
        const BodyId A = w->ids.at(a), B = w->ids.at(b);
        const Vec3 p0{v[0], v[1], v[2]}, p1{v[3], v[4], v[5]}, ax0{v[6], v[7], v[8]}, ax1{v[9], v[10], v[11]};
        const Vec3 g0{v[12], v[13], v[14]}, g1{v[15], v[16], v[17]};
        JointId id;
        switch ((JointType)type) {
        case JointType::Ball: id = W.addBallJoint(A, B, p0); break;
        case JointType::Distance:
            id = x[0] > 0.0f ? W.addSpringJoint(A, B, p0, p1, x[0], x[1]) : W.addDistanceJoint(A, B, p0, p1);
            break;
        case JointType::Hinge: id = W.addHingeJoint(A, B, p0, ax0); break;
        case JointType::ConeTwist: id = W.addConeTwistJoint(A, B, p0, ax0); break;
        case JointType::Fixed: id = W.addFixedJoint(A, B, p0); break;
        case JointType::Prismatic: id = W.addPrismaticJoint(A, B, p0, ax0); break;
        case JointType::SixDof: id = W.addSixDofJoint(A, B, p0); break;
        case JointType::Motor: id = W.addMotorJoint(A, B, p0, p1, x[0], x[1]); break;
        case JointType::Weld: id = W.addWeldJoint(A, B, p0, x[0], x[1]); break;
        case JointType::Wheel: id = W.addWheelJoint(A, B, p0, ax0); break;
        case JointType::Rope: id = W.addRopeJoint(A, B, p0, p1, x[0]); break;
        case JointType::Pulley: id = W.addPulleyJoint(A, B, p0, p1, g0, g1, x[0]); break;
        case JointType::Gear: id = W.addGearJoint(A, B, ax0, ax1, x[0]); break;
        default: g_error = "unknown joint type"; return -1;
        }
        w->jointIds.push_back(id);
        return (int)w->jointIds.size() - 1;
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}

// The world's joints in dense order (World::joints_, the sixth state vector
// of its snapshot after prevContacts_), as the backend receives them; broken
// joints are removed by the World after a step. Returns the count (~0u on a
// layout error).
uint32_t ref_world_joints(void* handle, vx_joint* out, uint32_t cap) {
    auto* w = static_cast<RefWorld*>(handle);
    SerializedScene scene = serializeWorld(*w->world);
    const std::vector<uint8_t>& bytes = scene.data;
    size_t at = sizeof(Vec3) + sizeof(int) + sizeof(WorldCcdDefaults) + sizeof(WorldMultiToiSettings) +
                sizeof(SolverOptions);
    for (int v = 0; v <= 6; ++v) {
        uint64_t elem = 0, n = 0;
        if (at + 16 > bytes.size()) return ~0u;
        std::memcpy(&elem, bytes.data() + at, 8);
        std::memcpy(&n, bytes.data() + at + 8, 8);
        at += 16;
        if (at + elem * n > bytes.size()) return ~0u;
        if (v == 6) {
            if (elem != sizeof(Joint)) return ~0u;
            if (out) std::memcpy(out, bytes.data() + at, std::min<uint64_t>(n, cap) * sizeof(Joint));
            return (uint32_t)n;
        }
        at += elem * n;
    }
    return ~0u;
}

// Reads / overwrites joint k (creation order) as the vx_joint record.
uint32_t ref_world_joint_count(void* handle) { return (uint32_t)static_cast<RefWorld*>(handle)->jointIds.size(); }
void ref_world_joint_get(void* handle, uint32_t k, vx_joint* out) {
    auto* w = static_cast<RefWorld*>(handle);
    const Joint& j = w->world->joint(w->jointIds.at(k));
    std::memcpy(out, &j, sizeof(Joint));
}
void ref_world_joint_set(void* handle, uint32_t k, const vx_joint* in) {
    auto* w = static_cast<RefWorld*>(handle);
    Joint& j = w->world->joint(w->jointIds.at(k));
    std::memcpy(&j, in, sizeof(Joint));
}

uint32_t ref_world_body_count(void* handle) {
    return (uint32_t)static_cast<RefWorld*>(handle)->ids.size();
}

void ref_world_get_bodies(void* handle, vx_body* out) {
    auto* w = static_cast<RefWorld*>(handle);
    for (size_t i = 0; i < w->ids.size(); ++i) {
        Body b = w->world->bodyState(w->ids[i]);
        std::memcpy(&out[i], &b, sizeof(Body));
    }
}

void ref_world_set_bodies(void* handle, const vx_body* in) {
    auto* w = static_cast<RefWorld*>(handle);
    for (size_t i = 0; i < w->ids.size(); ++i)
        std::memcpy(&w->world->body(w->ids[i]), &in[i], sizeof(Body));
}

// The last step's contact events (World::contactEvents) with dense body
// indices, in the record layout of vxb_contact_event (a, b, point, normal,
// impulse, type, sensor, 2 pad bytes: 40 bytes). Returns the count.
struct RefEvent {
    uint32_t a, b;
    float point[3], normal[3];
    float impulse;
    uint8_t type, sensor, pad[2];
};
static_assert(sizeof(RefEvent) == 40, "event record");

uint32_t ref_world_events(void* handle, void* out, uint32_t cap) {
    auto* w = static_cast<RefWorld*>(handle);
    const std::vector<ContactEvent>& ev = w->world->contactEvents();
    if (out) {
        std::vector<std::pair<uint64_t, uint32_t>> index(w->ids.size());
        for (size_t i = 0; i < w->ids.size(); ++i) index[i] = {w->ids[i].value, (uint32_t)i};
        std::sort(index.begin(), index.end());
        auto dense = [&](BodyId id) {
            auto it = std::lower_bound(index.begin(), index.end(), std::make_pair(id.value, 0u));
            return it != index.end() && it->first == id.value ? it->second : ~0u;
        };
        RefEvent* o = static_cast<RefEvent*>(out);
        for (size_t k = 0; k < ev.size() && k < cap; ++k) {
            RefEvent r;
            std::memset(&r, 0, sizeof(r));
            r.a = dense(ev[k].a);
            r.b = dense(ev[k].b);
            r.point[0] = ev[k].point.x; r.point[1] = ev[k].point.y; r.point[2] = ev[k].point.z;
            r.normal[0] = ev[k].normal.x; r.normal[1] = ev[k].normal.y; r.normal[2] = ev[k].normal.z;
            r.impulse = ev[k].impulse;
            r.type = (uint8_t)ev[k].type;
            r.sensor = ev[k].sensor ? 1 : 0;
            o[k] = r;
        }
    }
    return (uint32_t)ev.size();
}

// World::sleepConfig(): the thresholds the device library takes as
// vxb_sleep_config, in its field order.
void ref_world_sleep_config(void* handle, float linear, float angular, float acceleration, float timeToSleep,
                            float timeToDrowsy, float stabilityThreshold, int stabilityFrames, int gradual,
                            int stability) {
    SleepConfig& c = static_cast<RefWorld*>(handle)->world->sleepConfig();
    c.linearVelocityThreshold = linear;
    c.angularVelocityThreshold = angular;
    c.accelerationThreshold = acceleration;
    c.timeToSleep = timeToSleep;
    c.timeToDrowsy = timeToDrowsy;
    c.contactStabilityThreshold = stabilityThreshold;
    c.contactStabilityFrames = stabilityFrames;
    c.enableGradualSleep = gradual != 0;
    c.enableContactStability = stability != 0;
}

// Copies the hull soup; returns the number of points, writes the number of
// face indices to *faceIndexCount. Pass null buffers to query sizes.
uint32_t ref_world_soup(void* handle, vx_vec3* points, uint32_t* faces,
                        uint32_t* faceIndexCount) {
    auto* w = static_cast<RefWorld*>(handle);
    if (points) std::memcpy(points, w->soupPoints.data(), w->soupPoints.size() * sizeof(Vec3));
    if (faces) std::memcpy(faces, w->soupFaces.data(), w->soupFaces.size() * sizeof(uint32_t));
    if (faceIndexCount) *faceIndexCount = (uint32_t)w->soupFaces.size();
    return (uint32_t)w->soupPoints.size();
}

// Hull soup as the emulated backend last received it from World::step.
uint32_t ref_world_captured_soup(void* handle, vx_vec3* points, uint32_t* faces,
                                 uint32_t* faceIndexCount) {
    auto* w = static_cast<RefWorld*>(handle);
    if (!w->emulated) return 0;
    const auto& P = w->emulated->soupPoints;
    const auto& F = w->emulated->soupFaces;
    if (points) std::memcpy(points, P.data(), P.size() * sizeof(Vec3));
    if (faces) std::memcpy(faces, F.data(), F.size() * sizeof(uint32_t));
    if (faceIndexCount) *faceIndexCount = (uint32_t)F.size();
    return (uint32_t)P.size();
}

void ref_world_configure(void* handle, float gx, float gy, float gz, int substeps,
                         const vx_solver_options* options, int workers) {
    auto* w = static_cast<RefWorld*>(handle);
    w->world->gravity = {gx, gy, gz};
    w->world->substeps = substeps;
    if (options) {
        SolverOptions o;
        std::memcpy(&o, options, sizeof(o));
        w->world->setSolverOptions(o);
    }
    if (workers >= 0) w->world->setWorkerCount((uint32_t)workers);
}

uint32_t ref_world_worker_count(void* handle) {
    return static_cast<RefWorld*>(handle)->world->workerCount();
}

int ref_world_step(void* handle, float dt, int steps) {
    auto* w = static_cast<RefWorld*>(handle);
    try {
        double ms = 0.0;
        for (int s = 0; s < steps; ++s) {
            if (w->fixTieOrder && w->emulated) fixPrevContactOrder(w);
            auto t0 = std::chrono::steady_clock::now();
            w->world->step(dt);
            auto t1 = std::chrono::steady_clock::now();
            ms += std::chrono::duration<double, std::milli>(t1 - t0).count();
        }
        w->lastStepMs = ms;
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}

double ref_world_last_call_ms(void* handle) { return static_cast<RefWorld*>(handle)->lastStepMs; }

// StepStats subset: [generatedContacts, solvedContacts, velocityIterations,
// deviceSubsteps, awakeDynamicBodies].
void ref_world_stats(void* handle, uint64_t* out5) {
    const StepStats& s = static_cast<RefWorld*>(handle)->world->lastStepStats();
    out5[0] = s.generatedContacts;
    out5[1] = s.solvedContacts;
    out5[2] = s.velocityIterations;
    out5[3] = s.deviceSubsteps ? 1 : 0;
    out5[4] = s.awakeDynamicBodies;
}

// Contacts held by the emulated CUDA backend after the last step: colour order,
// impulses and points as fetchImpulses returns them (World::contacts_).
uint32_t ref_world_contacts(void* handle, vx_contact* out, uint32_t cap) {
    auto* w = static_cast<RefWorld*>(handle);
    if (!w->emulated) return 0;
    const auto& c = w->emulated->solve_;
    uint32_t m = (uint32_t)c.size();
    if (out) std::memcpy(out, c.data(), std::min(m, cap) * sizeof(Contact));
    return m;
}

// The world's warm-start cache (World::prevContacts_, in the world's order:
// sorted by (a, b) by src/world.cpp:4517-4520, within a pair as std::sort left
// it), read from the world's own serialized snapshot. Returns the count, or
// ~0u when the layout does not parse.
uint32_t ref_world_prev_contacts(void* handle, vx_contact* out, uint32_t cap) {
    auto* w = static_cast<RefWorld*>(handle);
    const std::vector<uint8_t> bytes = serializeWorld(*w->world).data;
    size_t off = 0;
    uint64_t m = 0;
    if (!locatePrevContacts(bytes, &off, &m)) return ~0u;
    if (out) std::memcpy(out, bytes.data() + off, std::min<uint64_t>(m, cap) * sizeof(Contact));
    return (uint32_t)m;
}

// Test switch (default 0, off): before each step of an emulated-backend world,
// fix the within-pair order of its warm-start cache (fixPrevContactOrder);
// 1 = emission order (the order the device keeps), 2 = reverse emission order
// for ties both there and in the backend's contact sort (another order the
// reference allows, to find the steps that depend on it).
void ref_world_fix_tie_order(void* handle, int mode) {
    auto* w = static_cast<RefWorld*>(handle);
    w->fixTieOrder = mode;
    if (w->emulated) w->emulated->reverseTies = mode == 2;
}

// Contacts as the emulated backend's findContacts produced them in the last
// step (pair order, before warm-start matching).
uint32_t ref_world_found_contacts(void* handle, vx_contact* out, uint32_t cap) {
    auto* w = static_cast<RefWorld*>(handle);
    if (!w->emulated) return 0;
    const auto& c = w->emulated->lastFound;
    uint32_t m = (uint32_t)c.size();
    if (out) std::memcpy(out, c.data(), std::min(m, cap) * sizeof(Contact));
    return m;
}

// ---- stage-level entry points over raw arrays ---------------------------

uint32_t ref_candidate_pairs(const vx_body* bodies, uint32_t n, float dt, uint64_t* out,
                             uint32_t cap, const vx_soup* soup) {
    std::vector<Body> v(reinterpret_cast<const Body*>(bodies),
                        reinterpret_cast<const Body*>(bodies) + n);
    std::vector<uint64_t> pairs = candidatePairs(v, dt, soup ? reinterpret_cast<const Mesh*>(soup->meshes) : nullptr);
    if (out) std::memcpy(out, pairs.data(), std::min<size_t>(pairs.size(), cap) * 8);
    return (uint32_t)pairs.size();
}

void ref_body_aabb(const vx_body* body, float dt, float* out6) {
    Vec3 lo, hi;
    bodyAabb(*reinterpret_cast<const Body*>(body), dt, lo, hi);
    out6[0] = lo.x; out6[1] = lo.y; out6[2] = lo.z;
    out6[3] = hi.x; out6[4] = hi.y; out6[5] = hi.z;
}

// collidePair over a list of pairs; contacts are appended in pair order and
// counts[p] receives each pair's count. Returns the total (may exceed cap).
uint32_t ref_collide_pairs(const vx_body* bodies, const vx_soup* soup, const uint64_t* pairs,
                           uint32_t npairs, float dt, vx_contact* out, uint32_t cap,
                           uint32_t* counts) {
    const Body* b = reinterpret_cast<const Body*>(bodies);
    MeshSoupView sv = soupView(soup);
    Contact buf[kMaxContactsPerPair];
    uint32_t total = 0;
    for (uint32_t p = 0; p < npairs; ++p) {
        BodyIndex i = BodyIndex(pairs[p] >> 32), j = BodyIndex(pairs[p]);
        int count = collidePair(b[i], b[j], i, j, sv, dt, buf, kMaxContactsPerPair);
        if (counts) counts[p] = (uint32_t)count;
        for (int c = 0; c < count; ++c) {
            if (total < cap) std::memcpy(&out[total], &buf[c], sizeof(Contact));
            ++total;
        }
    }
    return total;
}

// gjkDistance(makeConvex(a), makeConvex(b)); out = distance, normal[3],
// pointA[3], pointB[3], overlapping.
void ref_gjk(const vx_body* a, const vx_body* b, const vx_soup* soup, float* out11) {
    MeshSoupView sv = soupView(soup);
    GjkResult r = gjkDistance(makeConvex(*reinterpret_cast<const Body*>(a), sv),
                              makeConvex(*reinterpret_cast<const Body*>(b), sv));
    out11[0] = r.distance;
    out11[1] = r.normal.x; out11[2] = r.normal.y; out11[3] = r.normal.z;
    out11[4] = r.pointA.x; out11[5] = r.pointA.y; out11[6] = r.pointA.z;
    out11[7] = r.pointB.x; out11[8] = r.pointB.y; out11[9] = r.pointB.z;
    out11[10] = r.overlapping ? 1.0f : 0.0f;
}

void ref_sort_contacts(vx_contact* contacts, uint32_t m) {
    Contact* c = reinterpret_cast<Contact*>(contacts);
    std::stable_sort(c, c + m, contactLess);
}

uint32_t ref_color_contacts(const vx_body* bodies, uint32_t n, const vx_contact* contacts,
                            uint32_t m, int32_t* colorOf) {
    std::vector<Body> v(reinterpret_cast<const Body*>(bodies),
                        reinterpret_cast<const Body*>(bodies) + n);
    return (uint32_t)greedyColor(v, reinterpret_cast<const Contact*>(contacts), (int)m,
                                 colorOf);
}

// Warm start (optional) then `sweeps` passes of solveContact over the contacts
// in the given order (colour order reproduces the coloured parallel solve).
void ref_solve_sequence(vx_body* bodies, vx_contact* contacts, uint32_t m, float dt,
                        const vx_solver_options* options, int warmStart, int sweeps) {
    Body* b = reinterpret_cast<Body*>(bodies);
    Contact* c = reinterpret_cast<Contact*>(contacts);
    SolverOptions o;
    std::memcpy(&o, options, sizeof(o));
    if (warmStart)
        for (uint32_t k = 0; k < m; ++k)
            if (!b[c[k].a].isSensor() && !b[c[k].b].isSensor())
                warmStartContact(b[c[k].a], b[c[k].b], c[k]);
    for (int it = 0; it < sweeps; ++it)
        for (uint32_t k = 0; k < m; ++k)
            if (!b[c[k].a].isSensor() && !b[c[k].b].isSensor())
                solveContact(b[c[k].a], b[c[k].b], c[k], dt, o);
}

void ref_integrate_velocities(vx_body* bodies, uint32_t n, float gx, float gy, float gz,
                              float dt) {
    std::vector<Body> v(reinterpret_cast<Body*>(bodies), reinterpret_cast<Body*>(bodies) + n);
    integrateVelocities(v, {gx, gy, gz}, dt);
    std::memcpy(bodies, v.data(), n * sizeof(Body));
}

void ref_integrate_transforms(vx_body* bodies, uint32_t n, float dt) {
    std::vector<Body> v(reinterpret_cast<Body*>(bodies), reinterpret_cast<Body*>(bodies) + n);
    integrateTransforms(v, dt);
    std::memcpy(bodies, v.data(), n * sizeof(Body));
}

}  // extern "C"
