// Device narrow phase and contact solver rows.
//
// Algorithms and their constants follow the reference's shared host/device
// code so that contacts, impulses and body state agree with it to rounding:
//   Convex support mapping / GJK / EPA   src/gjk.h:13-777
//   face clipping manifolds              src/manifold.h:1-371
//   plane contacts, emit, collidePair    src/narrowphase.h:369-714
//   warm start and the TGS contact row   src/narrowphase.h:80-366
// The data layout is this library's own: bodies are read from SoA arrays
// into a compact view (BodyView), hull points come from a pointer that may
// address global or shared memory, and the scratch of EPA and clipping lives
// in per-thread local arrays sized to the reference's limits.
#pragma once
#include "vmath.cuh"
#include "velox_b200_types.h"

namespace vxb {

constexpr int kMaxContactsPerPair = 12;
constexpr uint32_t kNoFeature = 0xffffffffu;
constexpr uint32_t kFaceFeature = 0x40000000u;
constexpr uint32_t kImplicitFeature = 0x80000000u;
constexpr uint32_t kTriangleFeature = 0xc0000000u;
constexpr uint32_t kEdgeTag = 0x20000000u;
constexpr uint32_t kFaceTag = 0x40000000u;

// Device body arrays (structure of arrays, one entry per body).
struct BodyArrays {
    float4* pos;     // position xyz
    float4* rot;     // orientation quaternion
    float4* vel;     // linear velocity xyz
    float4* ang;     // angular velocity xyz
    float4* inertia; // invInertia xyz, invMass
    float4* iq;      // inertiaOrientation
    float4* dims;    // halfExtents xyz, radius
    float4* extra;   // capsuleHalfHeight, gravityScale, linearDamping, angularDamping
    float4* mat;     // friction, restitution, rollingFriction, spinningFriction
    float4* fscale;  // frictionScale xyz, ccd speculativeDistance
    float4* ccd;     // ccd collisionMargin, minVelocityForCCD, -, -
    float4* plane;   // planeNormal xyz, planeOffset
    uint4* hull;     // hullFirst, hullCount, hullFaceFirst, hullFaceCount
    uint4* filt;     // flags, categoryBits, maskBits, groupIndex
    float4* force;   // force xyz
    float4* torque;  // torque xyz
};

struct Soup {
    const float* points;   // hull points, xyz triples
    const uint32_t* faces; // hull faces, index triples local to a hull's points
    const float* vertices;             // mesh vertices, xyz triples
    const uint32_t* indices;           // mesh index triples, relative to a mesh's firstVertex
    const vx_mesh* meshes;
    const vx_bvh_node* nodes;          // all meshes' BVH nodes
    const uint32_t* triRefs;           // leaf triangle numbers
    const vx_compound_child* children; // compound children
};

// Everything the narrow phase reads of one body.
struct BodyView {
    V3 p; Q4 q; V3 v; V3 w;
    uint32_t flags;
    V3 half; float radius; float hh;
    V3 planeN; float planeOff;
    float friction, restitution, rolling, spinning;
    V3 fscale; float specDist; float margin;
    uint32_t hullFirst, hullCount, faceFirst, faceCount;
    uint32_t category, mask; int32_t group;
};

VXD BodyView loadView(const BodyArrays& B, uint32_t i) {
    BodyView b;
    float4 t = B.pos[i]; b.p = f3(t);
    b.q = q4(B.rot[i]);
    t = B.vel[i]; b.v = f3(t);
    t = B.ang[i]; b.w = f3(t);
    uint4 f = B.filt[i];
    b.flags = f.x; b.category = f.y; b.mask = f.z; b.group = (int32_t)f.w;
    t = B.dims[i]; b.half = f3(t); b.radius = t.w;
    t = B.extra[i]; b.hh = t.x;
    t = B.plane[i]; b.planeN = f3(t); b.planeOff = t.w;
    t = B.mat[i]; b.friction = t.x; b.restitution = t.y; b.rolling = t.z; b.spinning = t.w;
    t = B.fscale[i]; b.fscale = f3(t); b.specDist = t.w;
    t = B.ccd[i]; b.margin = t.x;
    uint4 h = B.hull[i];
    b.hullFirst = h.x; b.hullCount = h.y; b.faceFirst = h.z; b.faceCount = h.w;
    return b;
}

// loadView with the mutable state (pose, velocities) read through L2: for
// kernels where other SMs move bodies between this thread's reads.
VXD BodyView loadViewCoherent(const BodyArrays& B, uint32_t i) {
    BodyView b = loadView(B, i);
    b.p = f3(__ldcg(B.pos + i));
    b.q = q4(__ldcg(B.rot + i));
    b.v = f3(__ldcg(B.vel + i));
    b.w = f3(__ldcg(B.ang + i));
    return b;
}

// Body::maxPointSpeed (body.h:329-344).
VXD float maxPointSpeedOf(uint32_t shape, const V3& half, float radius, float hh, const V3& v,
                          const V3& w) {
    float r = radius;
    if (shape == kBox) r = length(half);
    else if (shape == kRoundedBox) r = length(half) + radius;
    else if (shape == kEllipsoid) r = vmax(half.x, vmax(half.y, half.z));
    else if (shape == kCapsule) r = hh + radius;
    else if (shape == kCylinder) r = sqrtf(hh * hh + radius * radius);
    else if (shape == kCone) {
        const float top = 1.5f * hh;
        r = vmax(top, sqrtf(radius * radius + 0.25f * hh * hh));
    } else if (shape == kCompound) r = radius;
    return length(v) + length(w) * r;
}
VXD float maxPointSpeed(const BodyView& b) {
    return maxPointSpeedOf(shapeOf(b.flags), b.half, b.radius, b.hh, b.v, b.w);
}

// Bound on the distance from a body's position to any point of the surface
// that gjkDistance measures for it (support point plus inflation radius).
// This is the `ext` term of bodyAabb (narrowphase.h:371-390) except where the
// distance query's shape reaches further: a rounded box's support already
// adds its radius and the query inflates by it again (gjk.h:112-127, :208-213),
// and an ellipsoid's support points have unit length (gjk.h:128-143 divides
// by |(a^2 d.x, b^2 d.y, c^2 d.z)|). Compounds return a negative value: no
// bound (their aggregate radius inherits the children's nominal extents).
VXD float coreExtent(uint32_t shape, const V3& half, float radius, float hh) {
    switch (shape) {
    case kBox: return length(half);
    case kRoundedBox: return length(half) + 2.0f * radius;
    case kEllipsoid: return vmax(1.0f, vmax(half.x, vmax(half.y, half.z)));
    case kCapsule: return hh + radius;
    case kSphere: case kHull: return radius;
    case kCylinder: return sqrtf(radius * radius + hh * hh);
    case kCone: return vmax(1.5f * hh, sqrtf(radius * radius + 0.25f * hh * hh));
    default: return -1.0f;
    }
}

// Swept AABB half width of bodyAabb (narrowphase.h:369-398) minus position.
VXD float aabbReach(uint32_t flags, const V3& half, float radius, float hh, float margin,
                    const V3& v, const V3& w, float dt) {
    const uint32_t shape = shapeOf(flags);
    float ext;
    switch (shape) {
    case kBox: ext = length(half); break;
    case kRoundedBox: ext = length(half) + radius; break;
    case kEllipsoid: ext = vmax(half.x, vmax(half.y, half.z)); break;
    case kCapsule: ext = hh + radius; break;
    case kSphere: ext = radius; break;
    case kHull: ext = radius; break;
    case kCompound: ext = radius; break;
    case kCylinder: ext = sqrtf(radius * radius + hh * hh); break;
    case kCone: {
        const float top = 1.5f * hh;
        ext = vmax(top, sqrtf(radius * radius + 0.25f * hh * hh));
        break;
    }
    default: ext = 0.0f; break;
    }
    const float sweep = sweeps(flags) ? maxPointSpeedOf(shape, half, radius, hh, v, w) * dt : 0.0f;
    return ext + sweep + margin + 1e-2f;
}

VXD bool aabbOverlap(const V3& lo1, const V3& hi1, const V3& lo2, const V3& hi2) {
    return hi1.x >= lo2.x && lo1.x <= hi2.x && hi1.y >= lo2.y && lo1.y <= hi2.y &&
           hi1.z >= lo2.z && lo1.z <= hi2.z;
}

// Body::canCollideWith (body.h:196-202).
VXD bool canCollide(uint32_t catA, uint32_t maskA, int32_t groupA, uint32_t catB, uint32_t maskB,
                    int32_t groupB) {
    if (groupA != 0 && groupA == groupB) return groupA > 0;
    return (maskA & catB) != 0 && (maskB & catA) != 0;
}

// ---- convex support mapping (gjk.h:13-226) --------------------------------

enum ConvexKind : uint8_t { cPoint, cSegment, cBox, cTriangle, cHull, cCylinder, cCone, cRoundedBox,
                            cEllipsoid };

struct Convex {
    uint8_t kind;
    uint8_t quality;   // GeometryQuality
    V3 position;
    Q4 orientation;
    V3 halfExtents;
    V3 segA, segB;
    const float* hullPts;      // local points, xyz triples
    uint32_t hullCount;
    const uint32_t* hullFaces; // index triples, local to hullPts
    uint32_t hullFaceCount;
    float radius;
    float geomRadius;
    float boundingRadius;
};

VXD V3 hullPoint(const float* pts, uint32_t i) {
    return V3{pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]};
}

VXD V3 supportOffsetBody(const Convex& c, const V3& dir) {
    switch (c.kind) {
    case cPoint: return V3{0.0f, 0.0f, 0.0f};
    case cSegment: {
        const V3 a = c.segA - c.position, b = c.segB - c.position;
        return dot(dir, a) > dot(dir, b) ? a : b;
    }
    case cBox: {
        const V3 d = rotateInv(c.orientation, dir);
        const V3 l{d.x >= 0 ? c.halfExtents.x : -c.halfExtents.x,
                   d.y >= 0 ? c.halfExtents.y : -c.halfExtents.y,
                   d.z >= 0 ? c.halfExtents.z : -c.halfExtents.z};
        return rotate(c.orientation, l);
    }
    case cHull: {
        const V3 d = rotateInv(c.orientation, dir);
        uint32_t best = 0;
        float bestDot = dot(d, hullPoint(c.hullPts, 0));
        for (uint32_t i = 1; i < c.hullCount; ++i) {
            const float t = dot(d, hullPoint(c.hullPts, i));
            if (t > bestDot) { bestDot = t; best = i; }
        }
        return rotate(c.orientation, hullPoint(c.hullPts, best));
    }
    case cCylinder: {
        const V3 d = rotateInv(c.orientation, dir);
        const float radial = sqrtf(d.x * d.x + d.z * d.z);
        const V3 l{radial > 1e-9f ? c.geomRadius * d.x / radial : 0.0f,
                   d.y >= 0.0f ? c.halfExtents.y : -c.halfExtents.y,
                   radial > 1e-9f ? c.geomRadius * d.z / radial : 0.0f};
        return rotate(c.orientation, l);
    }
    case cCone: {
        const V3 d = rotateInv(c.orientation, dir);
        const float radial = sqrtf(d.x * d.x + d.z * d.z);
        const float hh = c.halfExtents.y;
        const V3 base{radial > 1e-9f ? c.geomRadius * d.x / radial : 0.0f, -0.5f * hh,
                      radial > 1e-9f ? c.geomRadius * d.z / radial : 0.0f};
        const V3 tip{0.0f, 1.5f * hh, 0.0f};
        return rotate(c.orientation, dot(d, tip) > dot(d, base) ? tip : base);
    }
    case cRoundedBox: {
        const V3 d = rotateInv(c.orientation, dir);
        const V3 core{d.x >= 0 ? c.halfExtents.x : -c.halfExtents.x,
                      d.y >= 0 ? c.halfExtents.y : -c.halfExtents.y,
                      d.z >= 0 ? c.halfExtents.z : -c.halfExtents.z};
        const V3 n = normalize(d);
        return rotate(c.orientation, core + n * c.radius);
    }
    case cEllipsoid: {
        const V3 d = rotateInv(c.orientation, dir);
        const V3 s{c.halfExtents.x * c.halfExtents.x * d.x, c.halfExtents.y * c.halfExtents.y * d.y,
                   c.halfExtents.z * c.halfExtents.z * d.z};
        const float len = length(s);
        const V3 l = len > 1e-9f ? s * (1.0f / len) : V3{0.0f, 0.0f, 0.0f};
        return rotate(c.orientation, l);
    }
    case cTriangle: {  // corners segA, segB and triC (kept in halfExtents)
        V3 best = c.segA - c.position;
        const V3 b = c.segB - c.position, t = c.halfExtents - c.position;
        if (dot(dir, b) > dot(dir, best)) best = b;
        if (dot(dir, t) > dot(dir, best)) best = t;
        return best;
    }
    default: return V3{0.0f, 0.0f, 0.0f};
    }
}
// Out-of-line copy for the general GJK/EPA paths (keeps their code size down).
static __device__ __noinline__ V3 supportOffset(const Convex& c, const V3& dir) { return supportOffsetBody(c, dir); }
VXD V3 support(const Convex& c, const V3& dir) { return c.position + supportOffset(c, dir); }

// makeConvex (gjk.h:155-226).
VXD Convex makeConvex(const BodyView& b, const Soup& soup) {
    Convex c;
    c.position = b.p;
    c.orientation = b.q;
    c.quality = (uint8_t)((b.flags >> kGeomQualityShift) & 3u);
    c.halfExtents = V3{0.0f, 0.0f, 0.0f};
    c.segA = c.segB = V3{0.0f, 0.0f, 0.0f};
    c.hullPts = nullptr; c.hullCount = 0; c.hullFaces = nullptr; c.hullFaceCount = 0;
    c.radius = 0.0f; c.geomRadius = 0.0f; c.boundingRadius = 0.0f;
    switch (shapeOf(b.flags)) {
    case kSphere:
        c.kind = cPoint; c.radius = b.radius; c.boundingRadius = 0.0f; break;
    case kCapsule: {
        c.kind = cSegment;
        const V3 axis = rotate(b.q, V3{0.0f, b.hh, 0.0f});
        c.segA = b.p + axis;
        c.segB = b.p - axis;
        c.radius = b.radius;
        c.boundingRadius = b.hh;
        break;
    }
    case kBox:
        c.kind = cBox; c.halfExtents = b.half; c.radius = 0.0f; c.boundingRadius = length(b.half); break;
    case kHull:
        c.kind = cHull;
        c.hullPts = soup.points + 3 * (size_t)b.hullFirst;
        c.hullCount = b.hullCount;
        c.hullFaces = b.faceCount ? soup.faces + b.faceFirst : nullptr;
        c.hullFaceCount = b.faceCount;
        c.radius = 0.0f;
        c.boundingRadius = b.radius;
        break;
    case kCylinder:
        c.kind = cCylinder;
        c.halfExtents.y = b.hh;
        c.geomRadius = b.radius;
        c.boundingRadius = sqrtf(b.hh * b.hh + b.radius * b.radius);
        break;
    case kCone:
        c.kind = cCone;
        c.halfExtents.y = b.hh;
        c.geomRadius = b.radius;
        c.boundingRadius = vmax(1.5f * b.hh, sqrtf(b.radius * b.radius + 0.25f * b.hh * b.hh));
        break;
    case kRoundedBox:
        c.kind = cRoundedBox; c.halfExtents = b.half; c.radius = b.radius;
        c.boundingRadius = length(b.half) + b.radius;
        break;
    case kEllipsoid:
        c.kind = cEllipsoid; c.halfExtents = b.half;
        c.boundingRadius = vmax(b.half.x, vmax(b.half.y, b.half.z));
        break;
    default:
        c.kind = cPoint; break;
    }
    return c;
}

// makeTriangle (gjk.h:228-239): a triangle of a static mesh, centred on its
// centroid, corners in world space (the third corner in halfExtents).
VXD Convex makeTriangle(const V3& a, const V3& b, const V3& c) {
    Convex t;
    t.kind = cTriangle;
    t.quality = 0;
    t.position = a + ((b - a) + (c - a)) * (1.0f / 3.0f);
    t.orientation = Q4{0.0f, 0.0f, 0.0f, 1.0f};
    t.segA = a;
    t.segB = b;
    t.halfExtents = c;
    t.hullPts = nullptr; t.hullCount = 0; t.hullFaces = nullptr; t.hullFaceCount = 0;
    t.radius = 0.0f;
    t.geomRadius = 0.0f;
    t.boundingRadius = vmax(length(a - t.position), vmax(length(b - t.position), length(c - t.position)));
    return t;
}

// ---- GJK / EPA (gjk.h:241-777) --------------------------------------------

struct GjkResult {
    float distance;
    V3 normal;   // from B towards A
    V3 pointA, pointB;
    bool overlapping;
};

struct SupportVert { V3 p, a, b; };
struct Simplex { SupportVert v[4]; float bary[4]; int count; };

VXD uint8_t pairQuality(const Convex& A, const Convex& B) {
    return A.quality >= B.quality ? A.quality : B.quality;
}
VXD float convexScale(const Convex& c) {
    if (c.boundingRadius > 0.0f) return c.boundingRadius + c.radius;
    if (c.kind == cBox) return length(c.halfExtents) + c.radius;
    if (c.kind == cSegment) return 0.5f * length(c.segA - c.segB) + c.radius;
    if (c.kind == cTriangle)
        return vmax(length(c.segA - c.position), vmax(length(c.segB - c.position), length(c.halfExtents - c.position)));
    return c.radius;
}
VXD float pairScale(const Convex& A, const Convex& B) {
    return vmax(1e-8f, convexScale(A) + convexScale(B));
}
VXD float relativeTolerance(const Convex& A, const Convex& B) {
    const uint8_t q = pairQuality(A, B);
    return q == 0 ? 1e-7f : q == 1 ? 3e-7f : 1e-6f;
}
VXD float duplicateDistanceSq(const Convex& A, const Convex& B) {
    if (pairQuality(A, B) == 0) return 1e-12f;
    const float e = pairScale(A, B) * relativeTolerance(A, B);
    return vmax(1e-30f, e * e);
}
VXD float witnessResidual(const Convex& A, const Convex& B, const GjkResult& r) {
    if (r.overlapping || lengthSq(r.normal) < 0.25f) return 1e30f;
    const float aPlane = dot(-r.normal, support(A, -r.normal)) - A.radius;
    const float bPlane = dot(r.normal, support(B, r.normal)) + B.radius;
    return fabsf(dot(-r.normal, r.pointA) - aPlane) + fabsf(dot(r.normal, r.pointB) - bPlane);
}
VXD SupportVert supportVertex(const Convex& A, const Convex& B, const V3& dir) {
    SupportVert s;
    const V3 oa = supportOffset(A, dir);
    const V3 ob = supportOffset(B, -dir);
    s.a = A.position + oa;
    s.b = B.position + ob;
    s.p = (A.position - B.position) + (oa - ob);
    return s;
}

// Closest point of a segment / triangle simplex to the origin (gjk.h:301-380)
// on named vertices, so the register-resident GJK below and the general one
// run the same arithmetic.
VXD void solveSegmentV(SupportVert& v0, const SupportVert& v1, float& b0, float& b1, int& count) {
    const V3 a = v0.p, b = v1.p;
    const V3 ab = b - a;
    float t = -dot(a, ab);
    if (t <= 0.0f) { count = 1; b0 = 1.0f; return; }
    const float denom = dot(ab, ab);
    if (t >= denom) { v0 = v1; count = 1; b0 = 1.0f; return; }
    t /= denom;
    count = 2; b0 = 1.0f - t; b1 = t;
}

VXD void solveTriangleV(SupportVert& v0, SupportVert& v1, const SupportVert& v2, float& b0, float& b1, float& b2,
                        int& count) {
    const V3 a = v0.p, b = v1.p, c = v2.p;
    const V3 ab = b - a, ac = c - a, ap = -a;
    const float d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.0f && d2 <= 0.0f) { count = 1; b0 = 1.0f; return; }
    const V3 bp = -b;
    const float d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0.0f && d4 <= d3) { v0 = v1; count = 1; b0 = 1.0f; return; }
    const float vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
        const float t = d1 / (d1 - d3);
        count = 2; b0 = 1.0f - t; b1 = t; return;
    }
    const V3 cp = -c;
    const float d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0.0f && d5 <= d6) { v0 = v2; count = 1; b0 = 1.0f; return; }
    const float vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
        const float t = d2 / (d2 - d6);
        v1 = v2;
        count = 2; b0 = 1.0f - t; b1 = t; return;
    }
    const float va = d3 * d6 - d5 * d4;
    if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f) {
        const float t = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        v0 = v1; v1 = v2;
        count = 2; b0 = 1.0f - t; b1 = t; return;
    }
    const float sum = va + vb + vc;
    if (sum < 1e-20f) {  // degenerate triangle: keep the vertex nearest the origin
        int best = 0;
        if (lengthSq(v1.p) < lengthSq(v0.p)) best = 1;
        if (lengthSq(v2.p) < lengthSq((best == 0 ? v0 : v1).p)) best = 2;
        if (best == 1) v0 = v1;
        else if (best == 2) v0 = v2;
        count = 1; b0 = 1.0f;
        return;
    }
    const float inv = 1.0f / sum;
    count = 3; b0 = va * inv; b1 = vb * inv; b2 = vc * inv;
}

VXD void solveSegment(Simplex& s) { solveSegmentV(s.v[0], s.v[1], s.bary[0], s.bary[1], s.count); }

static __device__ __noinline__ void solveTriangle(Simplex& s) {
    solveTriangleV(s.v[0], s.v[1], s.v[2], s.bary[0], s.bary[1], s.bary[2], s.count);
}

static __constant__ int kTetFaces[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};

VXD V3 simplexClosest(const Simplex& s) {
    V3 c{0.0f, 0.0f, 0.0f};
    for (int i = 0; i < s.count; ++i) c += s.v[i].p * s.bary[i];
    return c;
}

// Returns true if the origin is inside the tetrahedron (gjk.h:382-445).
static __device__ __noinline__ bool solveTetrahedron(Simplex& s, float scale) {
    const float volume = dot(s.v[1].p - s.v[0].p, cross(s.v[2].p - s.v[0].p, s.v[3].p - s.v[0].p));
    const float floorVol = 1e-10f * scale * scale * scale;
    Simplex best;
    best.count = 0;
    float bestDist = 1e30f;
    if (fabsf(volume) < floorVol) {
        for (int f = 0; f < 4; ++f) {
            Simplex tri;
            tri.count = 3;
            tri.v[0] = s.v[kTetFaces[f][0]]; tri.v[1] = s.v[kTetFaces[f][1]]; tri.v[2] = s.v[kTetFaces[f][2]];
            solveTriangle(tri);
            const float d = lengthSq(simplexClosest(tri));
            if (d < bestDist) { bestDist = d; best = tri; }
        }
        s = best;
        return false;
    }
    bool inside = true;
    const float boundary = 3e-6f * scale;
    for (int f = 0; f < 4; ++f) {
        const int i0 = kTetFaces[f][0], i1 = kTetFaces[f][1], i2 = kTetFaces[f][2];
        const V3 a = s.v[i0].p, b = s.v[i1].p, c = s.v[i2].p;
        const V3 n = cross(b - a, c - a);
        const float nLen = length(n);
        if (nLen < 1e-20f) continue;
        const V3 opposite = s.v[6 - i0 - i1 - i2].p;
        const float originDist = dot(n, -a) / nLen;
        const float oppositeDist = dot(n, opposite - a) / nLen;
        if (originDist * oppositeDist < 0.0f || fabsf(originDist) <= boundary) {
            inside = false;
            Simplex tri;
            tri.count = 3;
            tri.v[0] = s.v[i0]; tri.v[1] = s.v[i1]; tri.v[2] = s.v[i2];
            solveTriangle(tri);
            const float d = lengthSq(simplexClosest(tri));
            if (d < bestDist) { bestDist = d; best = tri; }
        }
    }
    if (!inside) s = best;
    return inside;
}

VXD bool originInsideTetrahedron(const V3& p0, const V3& p1, const V3& p2, const V3& p3,
                                 float scale) {
    const V3 v[4] = {p0, p1, p2, p3};
    const float volume = dot(v[1] - v[0], cross(v[2] - v[0], v[3] - v[0]));
    const float floorVol = 1e-10f * scale * scale * scale;
    if (fabsf(volume) < floorVol) return false;
    for (int f = 0; f < 4; ++f) {
        const int i0 = kTetFaces[f][0], i1 = kTetFaces[f][1], i2 = kTetFaces[f][2];
        const int opp = 6 - i0 - i1 - i2;
        const V3 n = cross(v[i1] - v[i0], v[i2] - v[i0]);
        const float originSide = dot(n, -v[i0]);
        const float oppositeSide = dot(n, v[opp] - v[i0]);
        if (originSide * oppositeSide <= floorVol * floorVol) return false;
    }
    return true;
}

static __constant__ float kExpandDirs[14][3] = {
    {1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}, {1, 1, 1},
    {-1, 1, 1}, {1, -1, 1}, {1, 1, -1}, {-1, -1, 1}, {-1, 1, -1}, {1, -1, -1}, {-1, -1, -1}};

// Seeds EPA with a tetrahedron containing the origin (gjk.h:474-502).
static __device__ __noinline__ bool expandOverlapSimplex(const Convex& A, const Convex& B, Simplex& s) {
    SupportVert cand[18];
    int count = 0;
    for (int i = 0; i < s.count; ++i) cand[count++] = s.v[i];
    const float dupSq = duplicateDistanceSq(A, B);
    for (int d = 0; d < 14 && count < 18; ++d) {
        const SupportVert w = supportVertex(A, B, V3{kExpandDirs[d][0], kExpandDirs[d][1], kExpandDirs[d][2]});
        bool duplicate = false;
        for (int i = 0; i < count; ++i)
            if (lengthSq(w.p - cand[i].p) < dupSq) duplicate = true;
        if (!duplicate) cand[count++] = w;
    }
    const float scale = pairScale(A, B);
    for (int i = 0; i < count - 3; ++i)
        for (int j = i + 1; j < count - 2; ++j)
            for (int k = j + 1; k < count - 1; ++k)
                for (int l = k + 1; l < count; ++l)
                    if (originInsideTetrahedron(cand[i].p, cand[j].p, cand[k].p, cand[l].p, scale)) {
                        s.count = 4;
                        s.v[0] = cand[i]; s.v[1] = cand[j]; s.v[2] = cand[k]; s.v[3] = cand[l];
                        return true;
                    }
    return false;
}

struct EpaFace { int a, b, c; V3 normal; float distance; bool valid; };

VXD bool makeEpaFace(const SupportVert* verts, int ia, int ib, int ic, float minAreaSq, EpaFace& face) {
    const V3 a = verts[ia].p, b = verts[ib].p, c = verts[ic].p;
    V3 n = cross(b - a, c - a);
    const float n2 = lengthSq(n);
    if (n2 < minAreaSq) return false;
    n *= 1.0f / sqrtf(n2);
    float distance = dot(n, a);
    if (distance < 0.0f) {
        const int t = ib; ib = ic; ic = t;
        n = -n;
        distance = -distance;
    }
    face.a = ia; face.b = ib; face.c = ic; face.normal = n; face.distance = distance; face.valid = true;
    return true;
}

VXD void epaWitness(const SupportVert* verts, const EpaFace& f, V3& pa, V3& pb) {
    Simplex tri;
    tri.count = 3;
    tri.v[0] = verts[f.a]; tri.v[1] = verts[f.b]; tri.v[2] = verts[f.c];
    solveTriangle(tri);
    pa = V3{0.0f, 0.0f, 0.0f};
    pb = V3{0.0f, 0.0f, 0.0f};
    for (int i = 0; i < tri.count; ++i) {
        pa += tri.v[i].a * tri.bary[i];
        pb += tri.v[i].b * tri.bary[i];
    }
}

static __constant__ int kEpaInitial[4][3] = {{0, 1, 2}, {0, 3, 1}, {0, 2, 3}, {1, 3, 2}};

// Expanding polytope penetration (gjk.h:546-657): at most 64 vertices, 128
// faces, 192 horizon edges, 48 iterations at Normal quality.
static __device__ __noinline__ bool epaPenetration(const Convex& A, const Convex& B, const Simplex& simplex,
                                            GjkResult& result) {
    constexpr int kMaxVertices = 64, kMaxFaces = 128, kMaxEdges = 192;
    SupportVert verts[kMaxVertices];
    EpaFace faces[kMaxFaces];
    int vertexCount = 4, faceCount = 0;
    for (int i = 0; i < 4; ++i) verts[i] = simplex.v[i];
    float maxInitialAreaSq = 0.0f;
    for (int i = 0; i < 4; ++i) {
        const V3 a = verts[kEpaInitial[i][0]].p, b = verts[kEpaInitial[i][1]].p, c = verts[kEpaInitial[i][2]].p;
        maxInitialAreaSq = vmax(maxInitialAreaSq, lengthSq(cross(b - a, c - a)));
    }
    const float scale = pairScale(A, B);
    const uint8_t quality = pairQuality(A, B);
    const float areaFloorSq = quality == 0 ? 1e-16f
        : vmax(maxInitialAreaSq * 1e-16f, 1e-20f * scale * scale * scale * scale);
    for (int i = 0; i < 4; ++i) {
        EpaFace f;
        if (makeEpaFace(verts, kEpaInitial[i][0], kEpaInitial[i][1], kEpaInitial[i][2],
                        quality == 0 ? 1e-16f : 0.0f, f))
            faces[faceCount++] = f;
    }
    if (faceCount < 4) return false;
    const float dupSq = duplicateDistanceSq(A, B);
    int bestFace = 0;
    const int maxIterations = quality == 0 ? 48 : 64;
    for (int it = 0; it < maxIterations; ++it) {
        bestFace = -1;
        float bestDistance = 1e30f;
        for (int i = 0; i < faceCount; ++i)
            if (faces[i].valid && faces[i].distance < bestDistance) {
                bestDistance = faces[i].distance;
                bestFace = i;
            }
        if (bestFace < 0) return false;
        const EpaFace closest = faces[bestFace];
        const SupportVert w = supportVertex(A, B, closest.normal);
        const float supportDistance = dot(closest.normal, w.p);
        const float tolerance = quality == 0 ? 1e-4f * vmax(1.0f, supportDistance)
                                             : 1e-4f * vmax(scale, fabsf(supportDistance));
        bool duplicate = false;
        for (int i = 0; i < vertexCount; ++i)
            if (lengthSq(w.p - verts[i].p) < dupSq) duplicate = true;
        if (supportDistance - closest.distance <= tolerance || duplicate) {
            V3 ca, cb;
            epaWitness(verts, closest, ca, cb);
            result.normal = -closest.normal;
            result.distance = -(closest.distance + A.radius + B.radius);
            result.pointA = ca - result.normal * A.radius;
            result.pointB = cb + result.normal * B.radius;
            result.overlapping = true;
            return true;
        }
        if (vertexCount >= kMaxVertices) break;
        const int nv = vertexCount++;
        verts[nv] = w;
        int2 edges[kMaxEdges];
        int edgeCount = 0;
        for (int i = 0; i < faceCount; ++i) {
            if (!faces[i].valid) continue;
            const EpaFace f = faces[i];
            if (dot(f.normal, w.p - verts[f.a].p) <= tolerance) continue;
            faces[i].valid = false;
            const int fe[3][2] = {{f.a, f.b}, {f.b, f.c}, {f.c, f.a}};
            for (int e = 0; e < 3; ++e) {
                int reverse = -1;
                for (int k = 0; k < edgeCount; ++k)
                    if (edges[k].x == fe[e][1] && edges[k].y == fe[e][0]) { reverse = k; break; }
                if (reverse >= 0) edges[reverse] = edges[--edgeCount];
                else if (edgeCount < kMaxEdges) edges[edgeCount++] = make_int2(fe[e][0], fe[e][1]);
            }
        }
        for (int e = 0; e < edgeCount; ++e) {
            EpaFace f;
            if (!makeEpaFace(verts, edges[e].x, edges[e].y, nv, areaFloorSq, f)) continue;
            int slot = -1;
            for (int i = 0; i < faceCount; ++i)
                if (!faces[i].valid) { slot = i; break; }
            if (slot >= 0) faces[slot] = f;
            else if (faceCount < kMaxFaces) faces[faceCount++] = f;
            else return false;
        }
    }
    if (bestFace >= 0 && faces[bestFace].valid) {
        V3 ca, cb;
        epaWitness(verts, faces[bestFace], ca, cb);
        result.normal = -faces[bestFace].normal;
        result.distance = -(faces[bestFace].distance + A.radius + B.radius);
        result.pointA = ca - result.normal * A.radius;
        result.pointB = cb + result.normal * B.radius;
        result.overlapping = true;
        return true;
    }
    return false;
}

// The overlap branch of gjkSeeded: expand the simplex when the loop stopped
// on a vanishing distance (not inside a tetrahedron), then EPA, else the
// centre-line estimate.
static __device__ __noinline__ GjkResult gjkOverlapTail(const Convex& A, const Convex& B, Simplex& s, bool expand) {
    const float scale = pairScale(A, B);
    const float scaleSq = scale * scale;
    const bool robust = pairQuality(A, B) != 0;
    if (expand && s.count < 4) expandOverlapSimplex(A, B, s);
    GjkResult r;
    r.distance = 0.0f;
    r.normal = r.pointA = r.pointB = V3{0.0f, 0.0f, 0.0f};
    r.overlapping = true;
    if (s.count == 4 && epaPenetration(A, B, s, r)) return r;
    V3 n = A.position - B.position;
    n = lengthSq(n) > (robust ? scaleSq * 1e-14f : 1e-12f) ? normalize(n) : V3{0.0f, 1.0f, 0.0f};
    const float depth = dot(n, support(B, n) - support(A, -n));
    r.normal = n;
    r.distance = -depth - A.radius - B.radius;
    r.pointA = support(A, -n);
    r.pointB = support(B, n);
    return r;
}

static __device__ __noinline__ GjkResult gjkSeeded(const Convex& A, const Convex& B, V3 dir) {
    Simplex s;
    const float scale = pairScale(A, B);
    const float scaleSq = scale * scale;
    const uint8_t quality = pairQuality(A, B);
    const bool robust = quality != 0;
    if (lengthSq(dir) < (robust ? scaleSq * 1e-14f : 1e-12f)) dir = A.position - B.position;
    if (lengthSq(dir) < (robust ? scaleSq * 1e-14f : 1e-12f)) dir = V3{1.0f, 0.0f, 0.0f};
    s.v[0] = supportVertex(A, B, dir);
    s.count = 1;
    s.bary[0] = 1.0f;
    GjkResult r;
    r.distance = 0.0f;
    r.normal = r.pointA = r.pointB = V3{0.0f, 0.0f, 0.0f};
    r.overlapping = false;
    const int maxIterations = quality == 0 ? 32 : quality == 1 ? 64 : 96;
    const float rel = relativeTolerance(A, B);
    const float dupSq = duplicateDistanceSq(A, B);
    for (int it = 0; it < maxIterations; ++it) {
        const V3 closest = simplexClosest(s);
        const float distSq = lengthSq(closest);
        if (distSq < (robust ? scaleSq * 1e-10f : 1e-10f)) return gjkOverlapTail(A, B, s, true);
        const V3 d = -closest;
        const SupportVert w = supportVertex(A, B, d);
        const float progress = dot(w.p, d) - dot(closest, d);
        const float progressFloor = robust ? rel * scale * sqrtf(distSq) + rel * rel * scaleSq
                                           : 1e-6f * sqrtf(distSq) + 1e-9f;
        if (progress < progressFloor) break;
        bool duplicate = false;
        for (int i = 0; i < s.count; ++i)
            if (lengthSq(w.p - s.v[i].p) < dupSq) { duplicate = true; break; }
        if (duplicate) break;
        s.v[s.count++] = w;
        if (s.count == 2) solveSegment(s);
        else if (s.count == 3) solveTriangle(s);
        else if (solveTetrahedron(s, scale)) return gjkOverlapTail(A, B, s, false);
    }
    V3 pa{0.0f, 0.0f, 0.0f}, pb{0.0f, 0.0f, 0.0f};
    for (int i = 0; i < s.count; ++i) {
        pa += s.v[i].a * s.bary[i];
        pb += s.v[i].b * s.bary[i];
    }
    const V3 delta = pa - pb;
    const float coreDist = length(delta);
    r.normal = coreDist > (robust ? scale * 1e-7f : 1e-8f) ? delta * (1.0f / coreDist) : V3{0.0f, 1.0f, 0.0f};
    r.distance = coreDist - A.radius - B.radius;
    r.pointA = pa - r.normal * A.radius;
    r.pointB = pb + r.normal * B.radius;
    return r;
}

static __constant__ float kRobustDirs[14][3] = {
    {1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}, {1, 1, 1},
    {-1, 1, 1}, {1, -1, 1}, {1, 1, -1}, {-1, -1, 1}, {-1, 1, -1}, {1, -1, -1}, {-1, -1, -1}};

// gjkDistance (gjk.h:751-777): Robust/Paranoid geometry re-seeds from fixed
// directions and keeps the best-supported witness.
VXD GjkResult gjkDistance(const Convex& A, const Convex& B) {
    GjkResult best = gjkSeeded(A, B, A.position - B.position);
    const uint8_t quality = pairQuality(A, B);
    if (quality == 0 || best.overlapping) return best;
    const int directions = quality == 1 ? 6 : 14;
    float bestResidual = witnessResidual(A, B, best);
    const float tol = pairScale(A, B) * 1e-6f;
    for (int i = 0; i < directions; ++i) {
        const GjkResult cand = gjkSeeded(A, B, V3{kRobustDirs[i][0], kRobustDirs[i][1], kRobustDirs[i][2]});
        if (cand.overlapping) return cand;
        const float res = witnessResidual(A, B, cand);
        if (res + tol < bestResidual || (res <= bestResidual + tol && cand.distance < best.distance)) {
            best = cand;
            bestResidual = res;
        }
    }
    return best;
}

// ---- register-resident GJK distance --------------------------------------
//
// gjkSeeded for Normal-quality pairs (quality 0: 32 iterations, no re-seeding)
// with the same arithmetic in the same order, the simplex in named registers
// instead of an indexed array, and the support mappings inlined: a single
// thread runs it at register latency rather than local-memory latency, which
// is what the rewind pass's chains of dependent queries wait on. When the
// general routine would report an overlap (and go on to EPA) this one hands
// the simplex to gjkOverlapTail, the branch gjkSeeded itself would take.

VXD SupportVert supportVertexInline(const Convex& A, const Convex& B, const V3& dir) {
    SupportVert s;
    const V3 oa = supportOffsetBody(A, dir);
    const V3 ob = supportOffsetBody(B, -dir);
    s.a = A.position + oa;
    s.b = B.position + ob;
    s.p = (A.position - B.position) + (oa - ob);
    return s;
}

// One face of solveTetrahedron: solve the triangle (x, y, z) and keep it when
// its closest point is nearer than the best so far (strictly).
VXD void tetFaceCandidate(const SupportVert& x, const SupportVert& y, const SupportVert& z, SupportVert& t0,
                          SupportVert& t1, SupportVert& t2, float& c0, float& c1, float& c2, int& bc,
                          float& bestDist) {
    SupportVert u0 = x, u1 = y, u2 = z;
    float e0 = 0.0f, e1 = 0.0f, e2 = 0.0f;
    int n = 3;
    solveTriangleV(u0, u1, u2, e0, e1, e2, n);
    V3 c{0.0f, 0.0f, 0.0f};
    c += u0.p * e0;
    if (n > 1) c += u1.p * e1;
    if (n > 2) c += u2.p * e2;
    const float d = lengthSq(c);
    if (d < bestDist) {
        bestDist = d;
        t0 = u0; t1 = u1; t2 = u2;
        c0 = e0; c1 = e1; c2 = e2;
        bc = n;
    }
}

// solveTetrahedron (gjk.h:382-445) on named vertices; true = origin inside.
VXD bool solveTetrahedronV(SupportVert& v0, SupportVert& v1, SupportVert& v2, const SupportVert& v3, float& b0,
                           float& b1, float& b2, int& count, float scale) {
    const float volume = dot(v1.p - v0.p, cross(v2.p - v0.p, v3.p - v0.p));
    const float floorVol = 1e-10f * scale * scale * scale;
    SupportVert t0 = v0, t1 = v0, t2 = v0;
    float c0 = 0.0f, c1 = 0.0f, c2 = 0.0f;
    int bc = 0;
    float bestDist = 1e30f;
    if (fabsf(volume) < floorVol) {
        tetFaceCandidate(v0, v1, v2, t0, t1, t2, c0, c1, c2, bc, bestDist);
        tetFaceCandidate(v0, v1, v3, t0, t1, t2, c0, c1, c2, bc, bestDist);
        tetFaceCandidate(v0, v2, v3, t0, t1, t2, c0, c1, c2, bc, bestDist);
        tetFaceCandidate(v1, v2, v3, t0, t1, t2, c0, c1, c2, bc, bestDist);
        v0 = t0; v1 = t1; v2 = t2; b0 = c0; b1 = c1; b2 = c2; count = bc;
        return false;
    }
    bool inside = true;
    const float boundary = 3e-6f * scale;
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        const SupportVert& x = f == 3 ? v1 : v0;
        const SupportVert& y = f == 0 || f == 1 ? v1 : v2;
        const SupportVert& z = f == 0 ? v2 : v3;
        const SupportVert& o = f == 0 ? v3 : f == 1 ? v2 : f == 2 ? v1 : v0;
        const V3 a = x.p, b = y.p, c = z.p;
        const V3 n = cross(b - a, c - a);
        const float nLen = length(n);
        if (nLen < 1e-20f) continue;
        const float originDist = dot(n, -a) / nLen;
        const float oppositeDist = dot(n, o.p - a) / nLen;
        if (originDist * oppositeDist < 0.0f || fabsf(originDist) <= boundary) {
            inside = false;
            tetFaceCandidate(x, y, z, t0, t1, t2, c0, c1, c2, bc, bestDist);
        }
    }
    if (!inside) { v0 = t0; v1 = t1; v2 = t2; b0 = c0; b1 = c1; b2 = c2; count = bc; }
    return inside;
}

enum : int { kGjkSeparated = 0, kGjkOverlapExpand = 1, kGjkOverlapInside = 2, kGjkGeneral = 3 };

VXD void toSimplex(const SupportVert& v0, const SupportVert& v1, const SupportVert& v2, const SupportVert& v3,
                   float b0, float b1, float b2, int count, Simplex& s) {
    s.v[0] = v0; s.v[1] = v1; s.v[2] = v2; s.v[3] = v3;
    s.bary[0] = b0; s.bary[1] = b1; s.bary[2] = b2; s.bary[3] = 0.0f;
    s.count = count;
}

// kGjkSeparated: r holds the result. kGjkOverlap*: gjkSeeded would take its
// overlap branch with simplex s (kGjkOverlapExpand: after expanding it).
// kGjkGeneral: not a Normal-quality pair.
VXD int gjkDistanceFast(const Convex& A, const Convex& B, GjkResult& r, Simplex& s) {
    if (pairQuality(A, B) != 0) return kGjkGeneral;
    const float scale = pairScale(A, B);
    V3 dir = A.position - B.position;
    if (lengthSq(dir) < 1e-12f) dir = V3{1.0f, 0.0f, 0.0f};
    SupportVert v0 = supportVertexInline(A, B, dir), v1 = v0, v2 = v0, v3 = v0;
    float b0 = 1.0f, b1 = 0.0f, b2 = 0.0f;
    int count = 1;
    for (int it = 0; it < 32; ++it) {
        V3 closest{0.0f, 0.0f, 0.0f};
        if (count > 0) closest += v0.p * b0;
        if (count > 1) closest += v1.p * b1;
        if (count > 2) closest += v2.p * b2;
        const float distSq = lengthSq(closest);
        if (distSq < 1e-10f) {  // overlap
            toSimplex(v0, v1, v2, v3, b0, b1, b2, count, s);
            return kGjkOverlapExpand;
        }
        const V3 d = -closest;
        const SupportVert w = supportVertexInline(A, B, d);
        const float progress = dot(w.p, d) - dot(closest, d);
        const float progressFloor = 1e-6f * sqrtf(distSq) + 1e-9f;
        if (progress < progressFloor) break;
        bool duplicate = count > 0 && lengthSq(w.p - v0.p) < 1e-12f;
        if (!duplicate && count > 1) duplicate = lengthSq(w.p - v1.p) < 1e-12f;
        if (!duplicate && count > 2) duplicate = lengthSq(w.p - v2.p) < 1e-12f;
        if (duplicate) break;
        if (count == 0) {
            v0 = w; count = 1;  // appended to an emptied simplex: no solve step (gjkSeeded does none)
        } else if (count == 1) {
            v1 = w; count = 2;
            solveSegmentV(v0, v1, b0, b1, count);
        } else if (count == 2) {
            v2 = w; count = 3;
            solveTriangleV(v0, v1, v2, b0, b1, b2, count);
        } else {
            v3 = w; count = 4;
            if (solveTetrahedronV(v0, v1, v2, v3, b0, b1, b2, count, scale)) {
                toSimplex(v0, v1, v2, v3, b0, b1, b2, 4, s);
                return kGjkOverlapInside;
            }
        }
    }
    V3 pa{0.0f, 0.0f, 0.0f}, pb{0.0f, 0.0f, 0.0f};
    if (count > 0) { pa += v0.a * b0; pb += v0.b * b0; }
    if (count > 1) { pa += v1.a * b1; pb += v1.b * b1; }
    if (count > 2) { pa += v2.a * b2; pb += v2.b * b2; }
    const V3 delta = pa - pb;
    const float coreDist = length(delta);
    r.normal = coreDist > 1e-8f ? delta * (1.0f / coreDist) : V3{0.0f, 1.0f, 0.0f};
    r.distance = coreDist - A.radius - B.radius;
    r.pointA = pa - r.normal * A.radius;
    r.pointB = pb + r.normal * B.radius;
    r.overlapping = false;
    return kGjkSeparated;
}

// gjkDistance with the register-resident loop for Normal-quality pairs; an
// overlap continues into gjkSeeded's overlap branch from the same simplex.
static __device__ __noinline__ GjkResult gjkDistanceQuick(const Convex& A, const Convex& B) {
    GjkResult r;
    Simplex s;
    const int status = gjkDistanceFast(A, B, r, s);
    if (status == kGjkSeparated) return r;
    if (status == kGjkGeneral) return gjkDistance(A, B);
    return gjkOverlapTail(A, B, s, status == kGjkOverlapExpand);
}

// ---- face clipping manifolds (manifold.h:38-367) ---------------------------

constexpr int kMaxFaceVerts = 64;
constexpr int kMaxManifoldPoints = 8;

struct ClipVertex { V3 p; uint32_t id; };
struct FacePolygon { ClipVertex v[kMaxFaceVerts]; int count; uint32_t faceId; float plane; };
struct ClipVertex2D { float u, v; uint32_t featureA, featureB; };
struct ManifoldPoint { V3 pointA, pointB; float gap; uint32_t featureA, featureB; };

VXD uint32_t edgeFeature(uint32_t a, uint32_t b) {
    const uint32_t lo = a < b ? a : b, hi = a < b ? b : a;
    return kEdgeTag | (((lo * 0x1f123bb5u) ^ (hi * 0x5f356495u)) & 0x1fffffffu);
}
VXD uint32_t faceFeature(const uint32_t* ids, int count) {
    uint32_t sorted[kMaxFaceVerts];
    for (int i = 0; i < count; ++i) sorted[i] = ids[i];
    for (int i = 1; i < count; ++i) {
        const uint32_t key = sorted[i];
        int j = i - 1;
        while (j >= 0 && sorted[j] > key) { sorted[j + 1] = sorted[j]; --j; }
        sorted[j + 1] = key;
    }
    uint32_t h = 2166136261u;
    for (int i = 0; i < count; ++i) h = (h ^ sorted[i]) * 16777619u;
    return kFaceTag | (h & 0x1fffffffu);
}
VXD void planeBasis(const V3& n, V3& u, V3& v) {
    const V3 ref = fabsf(n.x) < 0.9f ? V3{1.0f, 0.0f, 0.0f} : V3{0.0f, 1.0f, 0.0f};
    u = normalize(cross(n, ref));
    v = cross(n, u);
}
static __device__ __noinline__ void orderCounterClockwise(ClipVertex* vs, int count, const V3& u, const V3& v) {
    if (count < 2) return;
    V3 center{0.0f, 0.0f, 0.0f};
    for (int i = 0; i < count; ++i) center += vs[i].p;
    center *= 1.0f / float(count);
    for (int i = 1; i < count; ++i) {
        const ClipVertex key = vs[i];
        const float keyAngle = atan2f(dot(key.p - center, v), dot(key.p - center, u));
        int j = i - 1;
        while (j >= 0) {
            const float angle = atan2f(dot(vs[j].p - center, v), dot(vs[j].p - center, u));
            if (angle <= keyAngle) break;
            vs[j + 1] = vs[j];
            --j;
        }
        vs[j + 1] = key;
    }
}

VXD int boxFace(const Convex& c, const V3& direction, FacePolygon& out) {
    const V3 d = rotateInv(c.orientation, direction);
    const float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    const int axis = ax >= ay && ax >= az ? 0 : (ay >= az ? 1 : 2);
    const bool positive = (axis == 0 ? d.x : axis == 1 ? d.y : d.z) >= 0.0f;
    const int o0 = axis == 0 ? 1 : 0;
    const int o1 = axis == 2 ? 1 : 2;
    const float ext[3] = {c.halfExtents.x, c.halfExtents.y, c.halfExtents.z};
    out.count = 0;
    for (int bits = 0; bits < 4; ++bits) {
        float val[3] = {-ext[0], -ext[1], -ext[2]};
        val[axis] = positive ? ext[axis] : -ext[axis];
        val[o0] = (bits & 1) ? ext[o0] : -ext[o0];
        val[o1] = (bits & 2) ? ext[o1] : -ext[o1];
        const int vertex = (val[0] > 0.0f ? 1 : 0) | (val[1] > 0.0f ? 2 : 0) | (val[2] > 0.0f ? 4 : 0);
        out.v[out.count].p = c.position + rotate(c.orientation, V3{val[0], val[1], val[2]});
        out.v[out.count].id = (uint32_t)vertex;
        ++out.count;
    }
    out.faceId = kFaceTag | uint32_t(axis * 2 + (positive ? 1 : 0));
    return out.count;
}

static __device__ __noinline__ int hullFace(const Convex& c, const V3& direction, FacePolygon& out) {
    if (!c.hullPts || c.hullCount == 0) return 0;
    uint32_t ids[kMaxFaceVerts];
    if (c.hullFaces && c.hullFaceCount > 0) {
        int seed = -1;
        V3 seedNormal{0.0f, 0.0f, 0.0f};
        float bestAlignment = -1e30f;
        for (uint32_t f = 0; f < c.hullFaceCount; ++f) {
            const uint32_t* ix = c.hullFaces + f * 3;
            if (ix[0] >= c.hullCount || ix[1] >= c.hullCount || ix[2] >= c.hullCount) return 0;
            const V3 p0 = hullPoint(c.hullPts, ix[0]);
            const V3 ln = cross(hullPoint(c.hullPts, ix[1]) - p0, hullPoint(c.hullPts, ix[2]) - p0);
            if (lengthSq(ln) < 1e-16f) return 0;
            const V3 wn = rotate(c.orientation, normalize(ln));
            const float al = dot(direction, wn);
            if (al > bestAlignment) { bestAlignment = al; seed = (int)f; seedNormal = wn; }
        }
        if (seed < 0 || bestAlignment < 0.95f) return 0;
        const uint32_t* si = c.hullFaces + seed * 3;
        const V3 seedPoint = c.position + rotate(c.orientation, hullPoint(c.hullPts, si[0]));
        float scale = 1.0f;
        for (uint32_t i = 0; i < c.hullCount; ++i) scale = vmax(scale, length(hullPoint(c.hullPts, i)));
        const float planeTol = 1e-5f + 1e-4f * scale;
        out.count = 0;
        for (uint32_t f = 0; f < c.hullFaceCount; ++f) {
            const uint32_t* ix = c.hullFaces + f * 3;
            const V3 p0 = hullPoint(c.hullPts, ix[0]);
            const V3 ln = cross(hullPoint(c.hullPts, ix[1]) - p0, hullPoint(c.hullPts, ix[2]) - p0);
            if (lengthSq(ln) < 1e-16f) return 0;
            const V3 wn = rotate(c.orientation, normalize(ln));
            const V3 point = c.position + rotate(c.orientation, p0);
            if (dot(seedNormal, wn) < 1.0f - 1e-4f || fabsf(dot(seedNormal, point - seedPoint)) > planeTol)
                continue;
            for (int corner = 0; corner < 3; ++corner) {
                const uint32_t id = ix[corner];
                bool present = false;
                for (int i = 0; i < out.count; ++i)
                    if (out.v[i].id == id) present = true;
                if (!present) {
                    if (out.count >= kMaxFaceVerts) return 0;
                    out.v[out.count].p = c.position + rotate(c.orientation, hullPoint(c.hullPts, id));
                    out.v[out.count].id = id;
                    ids[out.count++] = id;
                }
            }
        }
        if (out.count < 3) return 0;
        out.faceId = faceFeature(ids, out.count);
        return out.count;
    }
    // Point cloud without topology (manifold.h:193-217).
    float sup = -1e30f, minSup = 1e30f;
    const int total = c.hullCount < 64u ? (int)c.hullCount : 64;
    for (int i = 0; i < total; ++i) {
        const V3 wp = c.position + rotate(c.orientation, hullPoint(c.hullPts, i));
        const float pr = dot(direction, wp);
        sup = vmax(sup, pr);
        minSup = vmin(minSup, pr);
    }
    const float tol = 1e-5f + 1e-4f * vmax(1.0f, sup - minSup);
    out.count = 0;
    for (int i = 0; i < total; ++i) {
        const V3 wp = c.position + rotate(c.orientation, hullPoint(c.hullPts, i));
        if (dot(direction, wp) >= sup - tol) {
            out.v[out.count].p = wp;
            out.v[out.count].id = (uint32_t)i;
            ids[out.count++] = (uint32_t)i;
        }
    }
    if (out.count < 3) return 0;
    out.faceId = faceFeature(ids, out.count);
    return out.count;
}

VXD int supportFace(const Convex& c, const V3& direction, FacePolygon& out) {
    if (c.kind == cBox) return boxFace(c, direction, out);
    if (c.kind == cHull) return hullFace(c, direction, out);
    return 0;
}

VXD int clipAgainstEdge(const ClipVertex2D* in, int inCount, const ClipVertex2D& ea,
                        const ClipVertex2D& eb, ClipVertex2D* out) {
    if (inCount == 0) return 0;
    const float eu = eb.u - ea.u, ev = eb.v - ea.v;
    int outCount = 0;
    for (int i = 0; i < inCount; ++i) {
        const ClipVertex2D& prev = in[(i + inCount - 1) % inCount];
        const ClipVertex2D& cur = in[i];
        const float ps = eu * (prev.v - ea.v) - ev * (prev.u - ea.u);
        const float cs = eu * (cur.v - ea.v) - ev * (cur.u - ea.u);
        const bool pin = ps >= -1e-6f, cin = cs >= -1e-6f;
        if (pin != cin && outCount < 64) {
            const float den = ps - cs;
            float t = fabsf(den) > 1e-12f ? ps / den : 0.0f;
            t = vclamp(t, 0.0f, 1.0f);
            out[outCount].u = prev.u + (cur.u - prev.u) * t;
            out[outCount].v = prev.v + (cur.v - prev.v) * t;
            out[outCount].featureA = edgeFeature(prev.featureA, cur.featureA);
            out[outCount].featureB = edgeFeature(ea.featureB, eb.featureB);
            ++outCount;
        }
        if (cin && outCount < 64) out[outCount++] = cur;
    }
    return outCount;
}

// Clipped manifold between A's face facing -normal and B's face facing
// +normal (manifold.h:323-367), reduced to at most 8 points (:281-317).
static __device__ __noinline__ int clipFaceManifold(const Convex& A, const Convex& B, const V3& normal,
                                             ManifoldPoint* outPts) {
    FacePolygon faceA, faceB;
    faceA.count = faceB.count = 0;
    if (supportFace(A, -normal, faceA) < 3 || supportFace(B, normal, faceB) < 3) return 0;
    V3 u, v;
    planeBasis(normal, u, v);
    orderCounterClockwise(faceA.v, faceA.count, u, v);
    orderCounterClockwise(faceB.v, faceB.count, u, v);
    faceA.plane = dot(normal, faceA.v[0].p);
    faceB.plane = dot(normal, faceB.v[0].p);
    // clipFaces (manifold.h:253-279): subject = A, clip = B.
    planeBasis(normal, u, v);
    const V3 origin = faceB.v[0].p;
    ClipVertex2D cur[64], scratch[64], clip2d[kMaxFaceVerts];
    for (int i = 0; i < faceA.count; ++i) {
        const V3 d = faceA.v[i].p - origin;
        cur[i].u = dot(d, u); cur[i].v = dot(d, v);
        cur[i].featureA = faceA.v[i].id; cur[i].featureB = faceB.faceId;
    }
    for (int i = 0; i < faceB.count; ++i) {
        const V3 d = faceB.v[i].p - origin;
        clip2d[i].u = dot(d, u); clip2d[i].v = dot(d, v);
        clip2d[i].featureA = 0; clip2d[i].featureB = faceB.v[i].id;
    }
    int count = faceA.count;
    for (int i = 0; i < faceB.count && count > 0; ++i) {
        count = clipAgainstEdge(cur, count, clip2d[i], clip2d[(i + 1) % faceB.count], scratch);
        for (int j = 0; j < count; ++j) cur[j] = scratch[j];
    }
    if (count == 0) return 0;
    const float originPlane = dot(normal, origin);
    const float gap = faceA.plane - faceB.plane;
    const int pc = count < 64 ? count : 64;
    // Candidates (pointA, pointB, ids) are rebuilt on demand from cur[] to
    // keep the scratch small; reducePoints selects by pointA and feature ids.
    auto pointA = [&](int i) {
        const V3 tp = origin + u * cur[i].u + v * cur[i].v;
        return tp + normal * (faceA.plane - originPlane);
    };
    auto pointB = [&](int i) {
        const V3 tp = origin + u * cur[i].u + v * cur[i].v;
        return tp + normal * (faceB.plane - originPlane);
    };
    if (pc <= kMaxManifoldPoints) {
        for (int i = 0; i < pc; ++i) {
            outPts[i].pointA = pointA(i);
            outPts[i].pointB = pointB(i);
            outPts[i].gap = gap;
            outPts[i].featureA = cur[i].featureA;
            outPts[i].featureB = cur[i].featureB;
        }
        return pc;
    }
    // reducePoints: deepest first (all share one gap, so the lowest feature
    // pair wins ties), then farthest-point selection on pointA.
    bool used[64];
    for (int i = 0; i < pc; ++i) used[i] = false;
    int deepest = 0;
    for (int i = 1; i < pc; ++i)
        if (cur[i].featureA < cur[deepest].featureA ||
            (cur[i].featureA == cur[deepest].featureA && cur[i].featureB < cur[deepest].featureB))
            deepest = i;
    int sel[kMaxManifoldPoints];
    V3 selA[kMaxManifoldPoints];
    sel[0] = deepest;
    selA[0] = pointA(deepest);
    used[deepest] = true;
    int outN = 1;
    for (int o = 1; o < kMaxManifoldPoints; ++o) {
        int best = -1;
        float bestDistance = -1.0f;
        for (int i = 0; i < pc; ++i) {
            if (used[i]) continue;
            const V3 pa = pointA(i);
            float nearest = 1e30f;
            for (int j = 0; j < o; ++j) nearest = vmin(nearest, lengthSq(pa - selA[j]));
            if (nearest > bestDistance ||
                (nearest == bestDistance && best >= 0 &&
                 (cur[i].featureA < cur[best].featureA ||
                  (cur[i].featureA == cur[best].featureA && cur[i].featureB < cur[best].featureB)))) {
                best = i;
                bestDistance = nearest;
            }
        }
        if (best < 0) break;
        sel[o] = best;
        selA[o] = pointA(best);
        used[best] = true;
        outN = o + 1;
    }
    for (int i = 0; i < outN; ++i) {
        outPts[i].pointA = selA[i];
        outPts[i].pointB = pointB(sel[i]);
        outPts[i].gap = gap;
        outPts[i].featureA = cur[sel[i]].featureA;
        outPts[i].featureB = cur[sel[i]].featureB;
    }
    return kMaxManifoldPoints;
}

// ---- contact records (narrowphase.h:22-75, :414-463) ----------------------

VXD V3 pointVelocity(const V3& p, const V3& v, const V3& w, const V3& at) {
    return v + cross(w, at - p);
}
VXD V3 anchorWorld(bool sphere, const V3& p, const Q4& q, const V3& local) {
    return p + (sphere ? local : rotate(q, local));
}
VXD V3 anchorLocal(bool sphere, const V3& p, const Q4& q, const V3& world) {
    const V3 off = world - p;
    return sphere ? off : rotateInv(q, off);
}
VXD void contactTangents(const V3& n, V3& t1, V3& t2) {
    const V3 an{fabsf(n.x), fabsf(n.y), fabsf(n.z)};
    const V3 ref = an.x < an.y ? (an.x < an.z ? V3{1.0f, 0.0f, 0.0f} : V3{0.0f, 0.0f, 1.0f})
                               : (an.y < an.z ? V3{0.0f, 1.0f, 0.0f} : V3{0.0f, 0.0f, 1.0f});
    t1 = normalize(cross(n, ref));
    t2 = cross(n, t1);
}
VXD float combineMaterial(float a, float b, uint32_t modeA, uint32_t modeB) {
    const uint32_t mode = modeA >= modeB ? modeA : modeB;
    switch (mode) {
    case 0: return 0.5f * a + 0.5f * b;
    case 1: return sqrtf(a) * sqrtf(b);
    case 2: return vmin(a, b);
    case 3: return b > 0.0f && a > 3.402823466e+38F / b ? 3.402823466e+38F : a * b;
    case 4: return vmax(a, b);
    }
    return 0.0f;
}
VXD float directionalFrictionScale(const BodyView& b, const V3& dir) {
    const V3 l = rotateInv(b.q, dir);
    return length(V3{l.x * b.fscale.x, l.y * b.fscale.y, l.z * b.fscale.z});
}
VXD uint64_t contactFeatureKey(uint32_t fa, uint32_t fb) {
    const uint64_t a = fa == kNoFeature ? 0 : (uint64_t)fa + 1;
    const uint64_t b = fb == kNoFeature ? 0 : (uint64_t)fb + 1;
    return (a << 32) | b;
}
VXD uint64_t manifoldFeatureKey(uint32_t a, uint32_t b) {
    return ((uint64_t(a) + 1) << 32) | (uint64_t(b) + 1);
}

// Appends a speculative contact when the pair can touch within dt
// (narrowphase.h:425-463).
static __device__ __noinline__ void emitContact(const BodyView& a, const BodyView& b, uint32_t ia, uint32_t ib,
                                         const V3& normal, const V3& point, float gap, float dt,
                                         vx_contact* out, int cap, int& n, uint64_t featureKey) {
    if (n >= cap) return;
    const float slop = 1e-3f;
    const float reach = (sweeps(a.flags) ? maxPointSpeed(a) : 0.0f) * dt +
                        (sweeps(b.flags) ? maxPointSpeed(b) : 0.0f) * dt + a.specDist + b.specDist + slop;
    if (gap > reach) return;
    const float vn = dot(pointVelocity(a.p, a.v, a.w, point) - pointVelocity(b.p, b.v, b.w, point), normal);
    const V3 la = anchorLocal(shapeOf(a.flags) == kSphere, a.p, a.q, point);
    const V3 lb = anchorLocal(shapeOf(b.flags) == kSphere, b.p, b.q, point);
    V3 t1, t2;
    contactTangents(normal, t1, t2);
    const uint32_t fca = (a.flags >> kFrictionCombineShift) & 7u, fcb = (b.flags >> kFrictionCombineShift) & 7u;
    const uint32_t rca = (a.flags >> kRestitutionCombineShift) & 7u, rcb = (b.flags >> kRestitutionCombineShift) & 7u;
    const float friction = combineMaterial(a.friction, b.friction, fca, fcb);
    const float s1 = sqrtf(directionalFrictionScale(a, t1) * directionalFrictionScale(b, t1));
    const float s2 = sqrtf(directionalFrictionScale(a, t2) * directionalFrictionScale(b, t2));
    const float restitution = combineMaterial(a.restitution, b.restitution, rca, rcb);
    const float rolling = combineMaterial(a.rolling, b.rolling, fca, fcb);
    const float spinning = combineMaterial(a.spinning, b.spinning, fca, fcb);
    vx_contact& c = out[n++];
    c.a = ia; c.b = ib; c.featureKey = featureKey;
    c.normal = vx_vec3{normal.x, normal.y, normal.z};
    c.point = vx_vec3{point.x, point.y, point.z};
    c.localAnchorA = vx_vec3{la.x, la.y, la.z};
    c.localAnchorB = vx_vec3{lb.x, lb.y, lb.z};
    c.gap = gap; c.bias0 = gap; c.vn0 = vn; c.restitution = restitution;
    c.friction1 = friction * s1; c.friction2 = friction * s2;
    c.rollingFriction = rolling; c.spinningFriction = spinning;
    c.normalImpulse = c.tangentImpulse1 = c.tangentImpulse2 = 0.0f;
    c.rollingImpulse1 = c.rollingImpulse2 = c.spinningImpulse = 0.0f;
}

// Plane contacts (narrowphase.h:465-546).
static __device__ __noinline__ void planeConvex(const BodyView& conv, const BodyView& plane, uint32_t ic, uint32_t ip,
                                         const Soup& soup, float dt, vx_contact* out, int cap, int& n) {
    const V3 pn = plane.planeN;
    switch (shapeOf(conv.flags)) {
    case kHull: {
        const float* pts = soup.points + 3 * (size_t)conv.hullFirst;
        uint32_t selected[4] = {0, 0, 0, 0};
        int selectedCount = 0;
        for (int pick = 0; pick < 4 && pick < (int)conv.hullCount; ++pick) {
            float bestGap = 1e30f;
            V3 bestP{0.0f, 0.0f, 0.0f};
            uint32_t bestIndex = 0;
            for (uint32_t i = 0; i < conv.hullCount; ++i) {
                const V3 p = conv.p + rotate(conv.q, hullPoint(pts, i));
                const float g = dot(pn, p) - plane.planeOff;
                bool taken = false;
                for (int k = 0; k < selectedCount; ++k)
                    if (selected[k] == i) taken = true;
                if (!taken && g < bestGap) { bestGap = g; bestP = p; bestIndex = i; }
            }
            selected[selectedCount++] = bestIndex;
            emitContact(conv, plane, ic, ip, pn, bestP, bestGap, dt, out, cap, n,
                        contactFeatureKey(bestIndex, kFaceFeature));
        }
        break;
    }
    case kSphere:
        emitContact(conv, plane, ic, ip, pn, conv.p - pn * conv.radius,
                    dot(pn, conv.p) - plane.planeOff - conv.radius, dt, out, cap, n,
                    contactFeatureKey(kImplicitFeature, kFaceFeature));
        break;
    case kCapsule: {
        const V3 axis = rotate(conv.q, V3{0.0f, conv.hh, 0.0f});
        const V3 ends[2] = {conv.p + axis, conv.p - axis};
        for (int e = 0; e < 2; ++e)
            emitContact(conv, plane, ic, ip, pn, ends[e] - pn * conv.radius,
                        dot(pn, ends[e]) - plane.planeOff - conv.radius, dt, out, cap, n,
                        contactFeatureKey(kImplicitFeature | (uint32_t)e, kFaceFeature));
        break;
    }
    case kBox: {
        V3 pts[8];
        float gaps[8];
        uint32_t feats[8];
        for (int i = 0; i < 8; ++i) {
            const V3 l{(i & 1) ? conv.half.x : -conv.half.x, (i & 2) ? conv.half.y : -conv.half.y,
                       (i & 4) ? conv.half.z : -conv.half.z};
            pts[i] = conv.p + rotate(conv.q, l);
            gaps[i] = dot(pn, pts[i]) - plane.planeOff;
            feats[i] = (uint32_t)i;
        }
        for (int pick = 0; pick < 4; ++pick) {
            int best = pick;
            for (int i = pick + 1; i < 8; ++i)
                if (gaps[i] < gaps[best]) best = i;
            { const float t = gaps[pick]; gaps[pick] = gaps[best]; gaps[best] = t; }
            { const V3 t = pts[pick]; pts[pick] = pts[best]; pts[best] = t; }
            { const uint32_t t = feats[pick]; feats[pick] = feats[best]; feats[best] = t; }
            emitContact(conv, plane, ic, ip, pn, pts[pick], gaps[pick], dt, out, cap, n,
                        contactFeatureKey(feats[pick], kFaceFeature));
        }
        break;
    }
    case kCylinder:
    case kCone: {
        const Convex shape = makeConvex(conv, soup);
        const V3 deepest = support(shape, -pn);
        emitContact(conv, plane, ic, ip, pn, deepest, dot(pn, deepest) - plane.planeOff, dt, out, cap, n,
                    contactFeatureKey(kImplicitFeature, kFaceFeature));
        break;
    }
    default: break;
    }
}

VXD bool isConvexVolume(uint32_t s) {
    return s == kSphere || s == kBox || s == kCapsule || s == kHull || s == kCylinder || s == kCone ||
           s == kRoundedBox || s == kEllipsoid;
}

// Convex pair (narrowphase.h:555-607): GJK/EPA, then face clipping for
// Box/Hull pairs closer than 5 cm (boxes snap to the best separating face
// axis first), else one GJK witness contact.
static __device__ __noinline__ void convexConvex(const BodyView& a, const BodyView& b, uint32_t ia, uint32_t ib,
                                          const Soup& soup, float dt, vx_contact* out, int cap, int& n) {
    const Convex ca = makeConvex(a, soup), cb = makeConvex(b, soup);
    const GjkResult r = gjkDistanceQuick(ca, cb);  // gjkDistance's result
    const uint32_t sa = shapeOf(a.flags), sb = shapeOf(b.flags);
    if (r.distance < 0.05f && (sa == kBox || sa == kHull) && (sb == kBox || sb == kHull)) {
        V3 manifoldNormal = r.normal;
        if (sa == kBox && sb == kBox) {
            float best = -1e30f;
            for (int side = 0; side < 2; ++side) {
                const Q4 q = side ? b.q : a.q;
                for (int axis = 0; axis < 3; ++axis) {
                    V3 cand = rotate(q, V3{axis == 0 ? 1.0f : 0.0f, axis == 1 ? 1.0f : 0.0f,
                                           axis == 2 ? 1.0f : 0.0f});
                    if (dot(cand, a.p - b.p) < 0.0f) cand = -cand;
                    const float sep = dot(cand, support(ca, -cand) - support(cb, cand));
                    if (sep > best) { best = sep; manifoldNormal = cand; }
                }
            }
        }
        ManifoldPoint mp[kMaxManifoldPoints];
        const int pc = clipFaceManifold(ca, cb, manifoldNormal, mp);
        if (pc > 0) {
            bool emitted = false;
            for (int i = 0; i < pc && n < cap; ++i) {
                emitContact(a, b, ia, ib, manifoldNormal, (mp[i].pointA + mp[i].pointB) * 0.5f, mp[i].gap, dt,
                            out, cap, n, manifoldFeatureKey(mp[i].featureA, mp[i].featureB));
                emitted = true;
            }
            if (emitted) return;
        }
    }
    emitContact(a, b, ia, ib, r.normal, (r.pointA + r.pointB) * 0.5f, r.distance, dt, out, cap, n, 0);
}

// ---- static triangle meshes and compounds (narrowphase.h:609-714) ---------
//
// A mesh body keeps its mesh index in the hull word (hullFirst); a compound
// keeps compoundFirst / compoundCount there (hullFirst / hullCount). Neither
// shape has hull points of its own.

VXD V3 v3(const vx_vec3& v) { return V3{v.x, v.y, v.z}; }

VXD V3 meshVertex(const Soup& soup, uint32_t i) {
    return V3{soup.vertices[3 * (size_t)i], soup.vertices[3 * (size_t)i + 1], soup.vertices[3 * (size_t)i + 2]};
}

// Triangle `tri` of mesh `m` as a convex (makeTriangle of its three corners).
VXD Convex meshTriangle(const Soup& soup, const vx_mesh& m, uint32_t tri) {
    const uint32_t base = m.firstIndex + tri * 3;
    return makeTriangle(meshVertex(soup, m.firstVertex + soup.indices[base]),
                        meshVertex(soup, m.firstVertex + soup.indices[base + 1]),
                        meshVertex(soup, m.firstVertex + soup.indices[base + 2]));
}

// compoundChildBody (backend.h:42-57): child `ch` of `parent` posed in world
// space, with the parent's motion, materials, filters and CCD tuning.
VXD BodyView compoundChildView(const BodyView& parent, const vx_compound_child& ch) {
    BodyView r = parent;
    r.flags = (parent.flags & ~kShapeMask) | ((uint32_t)ch.shape & kShapeMask);
    r.p = parent.p + rotate(parent.q, v3(ch.localPosition));
    r.q = qmul(parent.q, Q4{ch.localOrientation.x, ch.localOrientation.y, ch.localOrientation.z,
                            ch.localOrientation.w});
    r.radius = ch.radius;
    r.half = v3(ch.halfExtents);
    r.hh = ch.capsuleHalfHeight;
    r.hullFirst = ch.hullFirst;
    r.hullCount = ch.hullCount;
    r.faceFirst = ch.hullFaceFirst;
    r.faceCount = ch.hullFaceCount;
    return r;
}

// Bounding-volume descent of one mesh's BVH (the explicit 48-entry stack of
// narrowphase.h:617-636: children that do not fit are dropped, as there),
// calling visit(tri) for each triangle of a leaf whose box overlaps [lo, hi].
// visit returns false to stop the walk early.
template <class Visit>
VXD void meshVisit(const Soup& soup, const vx_mesh& m, const V3& lo, const V3& hi, Visit visit) {
    uint32_t stack[48];
    int sp = 0;
    stack[sp++] = m.firstNode;
    while (sp > 0) {
        const vx_bvh_node& node = soup.nodes[stack[--sp]];
        if (!aabbOverlap(lo, hi, v3(node.aabbMin), v3(node.aabbMax))) continue;
        if (node.triCount == 0) {
            if (sp + 2 <= 48) {
                stack[sp++] = node.leftFirst;
                stack[sp++] = node.leftFirst + 1;
            }
            continue;
        }
        for (uint32_t k = 0; k < node.triCount; ++k)
            if (!visit(soup.triRefs[node.leftFirst + k])) return;
    }
}

// meshConvex (narrowphase.h:609-643): one GJK witness contact per triangle
// whose BVH leaf overlaps the convex's swept AABB, feature key
// (implicit, triangle | tri). Contacts: a = the convex, b = the mesh.
static __device__ __noinline__ void meshConvex(const BodyView& conv, const BodyView& mesh, uint32_t ic, uint32_t im,
                                               const Soup& soup, float dt, vx_contact* out, int cap, int& n) {
    const vx_mesh& m = soup.meshes[mesh.hullFirst];
    const float reach = aabbReach(conv.flags, conv.half, conv.radius, conv.hh, conv.margin, conv.v, conv.w, dt);
    const V3 lo = conv.p - V3{reach, reach, reach}, hi = conv.p + V3{reach, reach, reach};
    const Convex cc = makeConvex(conv, soup);
    meshVisit(soup, m, lo, hi, [&](uint32_t tri) {
        const GjkResult r = gjkDistanceQuick(cc, meshTriangle(soup, m, tri));  // gjkDistance's result
        emitContact(conv, mesh, ic, im, r.normal, (r.pointA + r.pointB) * 0.5f, r.distance, dt, out, cap, n,
                    contactFeatureKey(kImplicitFeature, kTriangleFeature | tri));
        return n < cap;  // later triangles could emit nothing more
    });
}

// collideSimplePair (narrowphase.h:656-673).
VXD int collideSimplePair(const BodyView& a, const BodyView& b, uint32_t ia, uint32_t ib, const Soup& soup,
                          float dt, vx_contact* out, int cap) {
    int n = 0;
    const uint32_t sa = shapeOf(a.flags), sb = shapeOf(b.flags);
    if (isConvexVolume(sa) && isConvexVolume(sb)) convexConvex(a, b, ia, ib, soup, dt, out, cap, n);
    else if (isConvexVolume(sa) && sb == kPlane) planeConvex(a, b, ia, ib, soup, dt, out, cap, n);
    else if (sa == kPlane && isConvexVolume(sb)) planeConvex(b, a, ib, ia, soup, dt, out, cap, n);
    else if (isConvexVolume(sa) && sb == kMesh) meshConvex(a, b, ia, ib, soup, dt, out, cap, n);
    else if (sa == kMesh && isConvexVolume(sb)) meshConvex(b, a, ib, ia, soup, dt, out, cap, n);
    return n;
}

VXD bool isComplexShape(uint32_t s) { return s == kMesh || s == kCompound; }

// Compound dispatch of collidePair (narrowphase.h:678-714): every child pair
// through collideSimplePair, contacts owned by the parents: anchors in the
// parents' frames, vn0 from the parents' point velocities, feature keys
// tagged with the child numbers.
static __device__ __noinline__ int collideCompound(const BodyView& a, const BodyView& b, uint32_t ia, uint32_t ib,
                                                   const Soup& soup, float dt, vx_contact* out, int cap) {
    const bool ca = shapeOf(a.flags) == kCompound, cb = shapeOf(b.flags) == kCompound;
    const int countA = ca ? (int)a.hullCount : 1;
    const int countB = cb ? (int)b.hullCount : 1;
    int total = 0;
    for (int x = 0; x < countA && total < cap; ++x) {
        const BodyView ga = ca ? compoundChildView(a, soup.children[a.hullFirst + x]) : a;
        for (int y = 0; y < countB && total < cap; ++y) {
            const BodyView gb = cb ? compoundChildView(b, soup.children[b.hullFirst + y]) : b;
            const int added = collideSimplePair(ga, gb, ia, ib, soup, dt, out + total, cap - total);
            const uint64_t tag = (uint64_t)(x + 1) * 0x9e3779b185ebca87ull ^ (uint64_t)(y + 1) * 0xc2b2ae3d27d4eb4full;
            for (int k = 0; k < added; ++k) {
                vx_contact& c = out[total + k];
                const BodyView& ownerA = c.a == ia ? a : b;
                const BodyView& ownerB = c.b == ib ? b : a;
                const V3 point = v3(c.point), normal = v3(c.normal);
                const V3 la = rotateInv(ownerA.q, point - ownerA.p);
                const V3 lb = rotateInv(ownerB.q, point - ownerB.p);
                c.localAnchorA = vx_vec3{la.x, la.y, la.z};
                c.localAnchorB = vx_vec3{lb.x, lb.y, lb.z};
                c.vn0 = dot(pointVelocity(ownerA.p, ownerA.v, ownerA.w, point) -
                                pointVelocity(ownerB.p, ownerB.v, ownerB.w, point),
                            normal);
                c.featureKey ^= tag;
            }
            total += added;
        }
    }
    return total;
}

// collidePair (narrowphase.h:678-714).
VXD int collidePair(const BodyView& a, const BodyView& b, uint32_t ia, uint32_t ib, const Soup& soup,
                    float dt, vx_contact* out, int cap) {
    if (shapeOf(a.flags) == kCompound || shapeOf(b.flags) == kCompound)
        return collideCompound(a, b, ia, ib, soup, dt, out, cap);
    return collideSimplePair(a, b, ia, ib, soup, dt, out, cap);
}

// ---- solver rows (narrowphase.h:80-366) -----------------------------------

// Mutable state of one body inside the solver.
struct SolverBody {
    V3 p; Q4 q; V3 v; V3 w;
    Mass m;
    bool sphere;
    Q4 frame;  // inertiaFrameAt(q): constant while q is (one substep's sweeps)
};

VXD V3 invI(const SolverBody& b, const V3& v) { return invInertiaMulAt(b.m, v, b.q); }

VXD void cacheFrame(SolverBody& b) { b.frame = inertiaFrameAt(b.m, b.q); }

// invInertiaMulAt(b.m, v, b.q) with the frame cached by cacheFrame (same arithmetic).
VXD V3 invIF(const SolverBody& b, const V3& v) {
    if (!isDynamic(b.m.flags) || isRotationLocked(b.m.flags)) return V3{0.0f, 0.0f, 0.0f};
    const V3 l = rotateInv(b.frame, v);
    return rotate(b.frame, V3{l.x * b.m.invI.x, l.y * b.m.invI.y, l.z * b.m.invI.z});
}

// The contact fields the solver reads and writes.
struct RowContact {
    V3 normal, point, la, lb;
    float bias0, vn0, restitution, friction1, friction2, rolling, spinning;
    float nImp, t1Imp, t2Imp, r1Imp, r2Imp, sImp;
};

VXD void warmStartRow(SolverBody& a, SolverBody& b, RowContact& c) {
    if (c.nImp <= 0.0f && c.t1Imp == 0.0f && c.t2Imp == 0.0f && c.r1Imp == 0.0f && c.r2Imp == 0.0f &&
        c.sImp == 0.0f)
        return;
    const V3 pa = anchorWorld(a.sphere, a.p, a.q, c.la);
    const V3 pb = anchorWorld(b.sphere, b.p, b.q, c.lb);
    c.point = (pa + pb) * 0.5f;
    V3 t1, t2;
    contactTangents(c.normal, t1, t2);
    const V3 impulse = c.normal * c.nImp + t1 * c.t1Imp + t2 * c.t2Imp;
    const V3 angular = t1 * c.r1Imp + t2 * c.r2Imp + c.normal * c.sImp;
    if (isDynamic(a.m.flags)) {
        a.v += impulse * solverInvMass(a.m);
        a.w += invI(a, cross(pa - a.p, impulse));
        a.w += invI(a, angular);
    }
    if (isDynamic(b.m.flags)) {
        b.v -= impulse * solverInvMass(b.m);
        b.w -= invI(b, cross(pb - b.p, impulse));
        b.w -= invI(b, angular);
    }
}

// One sequential-impulse pass over one contact: normal row against the live
// gap with restitution, then two-axis elliptic Coulomb friction (or the
// coupled cone block), then rolling and spinning resistance.
static __device__ __forceinline__ void solveRow(SolverBody& a, SolverBody& b, RowContact& c, float dt, bool coneBlock) {
    const V3 pa = anchorWorld(a.sphere, a.p, a.q, c.la);
    const V3 pb = anchorWorld(b.sphere, b.p, b.q, c.lb);
    c.point = (pa + pb) * 0.5f;
    const V3 ra = pa - a.p;
    const V3 rb = pb - b.p;
    const float ima = solverInvMass(a.m), imb = solverInvMass(b.m);
    const V3 raxn = cross(ra, c.normal);
    const V3 rbxn = cross(rb, c.normal);
    const float kNormal = ima + imb + dot(raxn, invI(a, raxn)) + dot(rbxn, invI(b, rbxn));
    if (kNormal <= 0.0f) return;
    const float vn = dot(pointVelocity(a.p, a.v, a.w, pa) - pointVelocity(b.p, b.v, b.w, pb), c.normal);
    const float liveGap = c.bias0 + dot(c.normal, pa - pb);
    float target = liveGap > 0.0f ? -liveGap / dt : 0.0f;
    if (c.vn0 < -1.0f && (liveGap <= 0.0f || vn > 0.0f)) target = vmax(target, -c.restitution * c.vn0);
    V3 t1, t2;
    contactTangents(c.normal, t1, t2);
    const V3 raxt1 = cross(ra, t1), rbxt1 = cross(rb, t1);
    const V3 raxt2 = cross(ra, t2), rbxt2 = cross(rb, t2);
    const float k1 = ima + imb + dot(raxt1, invI(a, raxt1)) + dot(rbxt1, invI(b, rbxt1));
    const float k2 = ima + imb + dot(raxt2, invI(a, raxt2)) + dot(rbxt2, invI(b, rbxt2));
    const float kN1 = dot(raxn, invI(a, raxt1)) + dot(rbxn, invI(b, rbxt1));
    const float kN2 = dot(raxn, invI(a, raxt2)) + dot(rbxn, invI(b, rbxt2));
    const bool dynA = isDynamic(a.m.flags), dynB = isDynamic(b.m.flags);
    if (!coneBlock) {
        float jn = (target - vn) / kNormal;
        const float nextNormal = vmax(c.nImp + jn, 0.0f);
        jn = nextNormal - c.nImp;
        c.nImp = nextNormal;
        const V3 ni = c.normal * jn;
        if (dynA) { a.v += ni * ima; a.w += invI(a, cross(ra, ni)); }
        if (dynB) { b.v -= ni * imb; b.w -= invI(b, cross(rb, ni)); }
        if (k1 > 0.0f && k2 > 0.0f) {
            const V3 rv = pointVelocity(a.p, a.v, a.w, pa) - pointVelocity(b.p, b.v, b.w, pb);
            const float old1 = c.t1Imp, old2 = c.t2Imp;
            float next1 = old1 - dot(rv, t1) / k1;
            float next2 = old2 - dot(rv, t2) / k2;
            const float max1 = c.friction1 * c.nImp;
            const float max2 = c.friction2 * c.nImp;
            if (max1 <= 0.0f) next1 = 0.0f;
            if (max2 <= 0.0f) next2 = 0.0f;
            const float ellipse = (max1 > 0.0f ? next1 * next1 / (max1 * max1) : 0.0f) +
                                  (max2 > 0.0f ? next2 * next2 / (max2 * max2) : 0.0f);
            if (ellipse > 1.0f) {
                const float s = 1.0f / sqrtf(ellipse);
                next1 *= s;
                next2 *= s;
            }
            c.t1Imp = next1;
            c.t2Imp = next2;
            const V3 fi = t1 * (next1 - old1) + t2 * (next2 - old2);
            if (dynA) { a.v += fi * ima; a.w += invI(a, cross(ra, fi)); }
            if (dynB) { b.v -= fi * imb; b.w -= invI(b, cross(rb, fi)); }
        }
    } else {
        const float oldNormal = c.nImp;
        const float old1 = c.t1Imp, old2 = c.t2Imp;
        float nextNormal = oldNormal, next1 = old1, next2 = old2;
        if (k1 > 0.0f && k2 > 0.0f) {
            const float k12 = dot(raxt1, invI(a, raxt2)) + dot(rbxt1, invI(b, rbxt2));
            const float det = kNormal * (k1 * k2 - k12 * k12) - kN1 * (kN1 * k2 - kN2 * k12) +
                              kN2 * (kN1 * k12 - kN2 * k1);
            if (fabsf(det) > 1e-12f) {
                const V3 rv = pointVelocity(a.p, a.v, a.w, pa) - pointVelocity(b.p, b.v, b.w, pb);
                const float bN = target - dot(rv, c.normal);
                const float b1 = -dot(rv, t1);
                const float b2 = -dot(rv, t2);
                const float dN = (bN * (k1 * k2 - k12 * k12) + b1 * (kN2 * k12 - kN1 * k2) +
                                  b2 * (kN1 * k12 - kN2 * k1)) / det;
                const float d1 = (bN * (kN2 * k12 - kN1 * k2) + b1 * (kNormal * k2 - kN2 * kN2) +
                                  b2 * (kN1 * kN2 - kNormal * k12)) / det;
                const float d2 = (bN * (kN1 * k12 - kN2 * k1) + b1 * (kN1 * kN2 - kNormal * k12) +
                                  b2 * (kNormal * k1 - kN1 * kN1)) / det;
                nextNormal = vmax(oldNormal + dN, 0.0f);
                next1 = old1 + d1;
                next2 = old2 + d2;
            }
        }
        const float max1 = c.friction1 * nextNormal;
        const float max2 = c.friction2 * nextNormal;
        if (max1 <= 0.0f) next1 = 0.0f;
        if (max2 <= 0.0f) next2 = 0.0f;
        const float ellipse = (max1 > 0.0f ? next1 * next1 / (max1 * max1) : 0.0f) +
                              (max2 > 0.0f ? next2 * next2 / (max2 * max2) : 0.0f);
        if (ellipse > 1.0f) {
            const float s = 1.0f / sqrtf(ellipse);
            next1 *= s;
            next2 *= s;
        }
        c.nImp = nextNormal;
        c.t1Imp = next1;
        c.t2Imp = next2;
        const V3 imp = c.normal * (nextNormal - oldNormal) + t1 * (next1 - old1) + t2 * (next2 - old2);
        if (dynA) { a.v += imp * ima; a.w += invI(a, cross(ra, imp)); }
        if (dynB) { b.v -= imp * imb; b.w -= invI(b, cross(rb, imp)); }
    }
    V3 wr = a.w - b.w;
    const float kr1 = dot(t1, invI(a, t1)) + dot(t1, invI(b, t1));
    const float kr2 = dot(t2, invI(a, t2)) + dot(t2, invI(b, t2));
    if (c.rolling > 0.0f && kr1 > 0.0f && kr2 > 0.0f) {
        const float o1 = c.r1Imp, o2 = c.r2Imp;
        float n1 = o1 - dot(wr, t1) / kr1;
        float n2 = o2 - dot(wr, t2) / kr2;
        const float limit = c.rolling * c.nImp;
        const float mag = sqrtf(n1 * n1 + n2 * n2);
        if (mag > limit && mag > 1e-9f) {
            const float s = limit / mag;
            n1 *= s;
            n2 *= s;
        }
        c.r1Imp = n1;
        c.r2Imp = n2;
        const V3 tq = t1 * (n1 - o1) + t2 * (n2 - o2);
        if (dynA) a.w += invI(a, tq);
        if (dynB) b.w -= invI(b, tq);
    }
    wr = a.w - b.w;
    const float ks = dot(c.normal, invI(a, c.normal)) + dot(c.normal, invI(b, c.normal));
    if (c.spinning > 0.0f && ks > 0.0f) {
        const float old = c.sImp;
        float next = old - dot(wr, c.normal) / ks;
        const float limit = c.spinning * c.nImp;
        next = vclamp(next, -limit, limit);
        c.sImp = next;
        const V3 tq = c.normal * (next - old);
        if (dynA) a.w += invI(a, tq);
        if (dynB) b.w -= invI(b, tq);
    }
}

// ---- solver rows split by what changes -------------------------------------
//
// Within one substep's warm start and sweeps only velocities and impulses
// change; poses are fixed. Every pose-dependent quantity of solveRow (anchors,
// arms, tangents, effective masses, the live gap) is therefore the same value
// in every sweep. prepRow evaluates them once per substep with exactly the
// expressions of solveRow, and sweepRow / warmPrepRow consume them, so the
// results equal solveRow / warmStartRow bit for bit.

struct RowPrep {
    V3 ra, rb, point;
    V3 raxn, rbxn, t1, t2, raxt1, rbxt1, raxt2, rbxt2;
    float kNormal, liveGap, targetBase, k1, k2, kN1, kN2, k12, kr1, kr2, ks;
};

// Bodies must have their frames cached (cacheFrame) for the current poses.
VXD void prepRow(const SolverBody& a, const SolverBody& b, const RowContact& c, float dt, bool coneBlock,
                 RowPrep& P) {
    const V3 pa = anchorWorld(a.sphere, a.p, a.q, c.la);
    const V3 pb = anchorWorld(b.sphere, b.p, b.q, c.lb);
    P.point = (pa + pb) * 0.5f;
    P.ra = pa - a.p;
    P.rb = pb - b.p;
    const float ima = solverInvMass(a.m), imb = solverInvMass(b.m);
    P.raxn = cross(P.ra, c.normal);
    P.rbxn = cross(P.rb, c.normal);
    P.kNormal = ima + imb + dot(P.raxn, invIF(a, P.raxn)) + dot(P.rbxn, invIF(b, P.rbxn));
    P.liveGap = c.bias0 + dot(c.normal, pa - pb);
    P.targetBase = P.liveGap > 0.0f ? -P.liveGap / dt : 0.0f;
    contactTangents(c.normal, P.t1, P.t2);
    P.raxt1 = cross(P.ra, P.t1); P.rbxt1 = cross(P.rb, P.t1);
    P.raxt2 = cross(P.ra, P.t2); P.rbxt2 = cross(P.rb, P.t2);
    P.k1 = ima + imb + dot(P.raxt1, invIF(a, P.raxt1)) + dot(P.rbxt1, invIF(b, P.rbxt1));
    P.k2 = ima + imb + dot(P.raxt2, invIF(a, P.raxt2)) + dot(P.rbxt2, invIF(b, P.rbxt2));
    P.kN1 = dot(P.raxn, invIF(a, P.raxt1)) + dot(P.rbxn, invIF(b, P.rbxt1));
    P.kN2 = dot(P.raxn, invIF(a, P.raxt2)) + dot(P.rbxn, invIF(b, P.rbxt2));
    P.k12 = coneBlock ? dot(P.raxt1, invIF(a, P.raxt2)) + dot(P.rbxt1, invIF(b, P.rbxt2)) : 0.0f;
    P.kr1 = c.rolling > 0.0f ? dot(P.t1, invIF(a, P.t1)) + dot(P.t1, invIF(b, P.t1)) : 0.0f;
    P.kr2 = c.rolling > 0.0f ? dot(P.t2, invIF(a, P.t2)) + dot(P.t2, invIF(b, P.t2)) : 0.0f;
    P.ks = c.spinning > 0.0f ? dot(c.normal, invIF(a, c.normal)) + dot(c.normal, invIF(b, c.normal)) : 0.0f;
}

// warmStartContact with prepared arms (narrowphase.h:80-124).
VXD void warmPrepRow(SolverBody& a, SolverBody& b, RowContact& c, const RowPrep& P) {
    if (c.nImp <= 0.0f && c.t1Imp == 0.0f && c.t2Imp == 0.0f && c.r1Imp == 0.0f && c.r2Imp == 0.0f &&
        c.sImp == 0.0f)
        return;
    c.point = P.point;
    const V3 impulse = c.normal * c.nImp + P.t1 * c.t1Imp + P.t2 * c.t2Imp;
    const V3 angular = P.t1 * c.r1Imp + P.t2 * c.r2Imp + c.normal * c.sImp;
    if (isDynamic(a.m.flags)) {
        a.v += impulse * solverInvMass(a.m);
        a.w += invIF(a, cross(P.ra, impulse));
        a.w += invIF(a, angular);
    }
    if (isDynamic(b.m.flags)) {
        b.v -= impulse * solverInvMass(b.m);
        b.w -= invIF(b, cross(P.rb, impulse));
        b.w -= invIF(b, angular);
    }
}

// One sweep of solveContact (narrowphase.h:130-366) with prepared pose terms.
VXD void sweepRow(SolverBody& a, SolverBody& b, RowContact& c, const RowPrep& P, bool coneBlock) {
    c.point = P.point;
    if (P.kNormal <= 0.0f) return;
    const float ima = solverInvMass(a.m), imb = solverInvMass(b.m);
    const bool dynA = isDynamic(a.m.flags), dynB = isDynamic(b.m.flags);
    const float vn = dot((a.v + cross(a.w, P.ra)) - (b.v + cross(b.w, P.rb)), c.normal);
    float target = P.targetBase;
    if (c.vn0 < -1.0f && (P.liveGap <= 0.0f || vn > 0.0f)) target = vmax(target, -c.restitution * c.vn0);
    if (!coneBlock) {
        float jn = (target - vn) / P.kNormal;
        const float nextNormal = vmax(c.nImp + jn, 0.0f);
        jn = nextNormal - c.nImp;
        c.nImp = nextNormal;
        const V3 ni = c.normal * jn;
        if (dynA) { a.v += ni * ima; a.w += invIF(a, cross(P.ra, ni)); }
        if (dynB) { b.v -= ni * imb; b.w -= invIF(b, cross(P.rb, ni)); }
        if (P.k1 > 0.0f && P.k2 > 0.0f) {
            const V3 rv = (a.v + cross(a.w, P.ra)) - (b.v + cross(b.w, P.rb));
            const float old1 = c.t1Imp, old2 = c.t2Imp;
            float next1 = old1 - dot(rv, P.t1) / P.k1;
            float next2 = old2 - dot(rv, P.t2) / P.k2;
            const float max1 = c.friction1 * c.nImp;
            const float max2 = c.friction2 * c.nImp;
            if (max1 <= 0.0f) next1 = 0.0f;
            if (max2 <= 0.0f) next2 = 0.0f;
            const float ellipse = (max1 > 0.0f ? next1 * next1 / (max1 * max1) : 0.0f) +
                                  (max2 > 0.0f ? next2 * next2 / (max2 * max2) : 0.0f);
            if (ellipse > 1.0f) {
                const float sc = 1.0f / sqrtf(ellipse);
                next1 *= sc;
                next2 *= sc;
            }
            c.t1Imp = next1;
            c.t2Imp = next2;
            const V3 fi = P.t1 * (next1 - old1) + P.t2 * (next2 - old2);
            if (dynA) { a.v += fi * ima; a.w += invIF(a, cross(P.ra, fi)); }
            if (dynB) { b.v -= fi * imb; b.w -= invIF(b, cross(P.rb, fi)); }
        }
    } else {
        const float oldNormal = c.nImp;
        const float old1 = c.t1Imp, old2 = c.t2Imp;
        float nextNormal = oldNormal, next1 = old1, next2 = old2;
        if (P.k1 > 0.0f && P.k2 > 0.0f) {
            const float kNormal = P.kNormal, k1 = P.k1, k2 = P.k2, kN1 = P.kN1, kN2 = P.kN2, k12 = P.k12;
            const float det = kNormal * (k1 * k2 - k12 * k12) - kN1 * (kN1 * k2 - kN2 * k12) +
                              kN2 * (kN1 * k12 - kN2 * k1);
            if (fabsf(det) > 1e-12f) {
                const V3 rv = (a.v + cross(a.w, P.ra)) - (b.v + cross(b.w, P.rb));
                const float bN = target - dot(rv, c.normal);
                const float b1 = -dot(rv, P.t1);
                const float b2 = -dot(rv, P.t2);
                const float dN = (bN * (k1 * k2 - k12 * k12) + b1 * (kN2 * k12 - kN1 * k2) +
                                  b2 * (kN1 * k12 - kN2 * k1)) / det;
                const float d1 = (bN * (kN2 * k12 - kN1 * k2) + b1 * (kNormal * k2 - kN2 * kN2) +
                                  b2 * (kN1 * kN2 - kNormal * k12)) / det;
                const float d2 = (bN * (kN1 * k12 - kN2 * k1) + b1 * (kN1 * kN2 - kNormal * k12) +
                                  b2 * (kNormal * k1 - kN1 * kN1)) / det;
                nextNormal = vmax(oldNormal + dN, 0.0f);
                next1 = old1 + d1;
                next2 = old2 + d2;
            }
        }
        const float max1 = c.friction1 * nextNormal;
        const float max2 = c.friction2 * nextNormal;
        if (max1 <= 0.0f) next1 = 0.0f;
        if (max2 <= 0.0f) next2 = 0.0f;
        const float ellipse = (max1 > 0.0f ? next1 * next1 / (max1 * max1) : 0.0f) +
                              (max2 > 0.0f ? next2 * next2 / (max2 * max2) : 0.0f);
        if (ellipse > 1.0f) {
            const float sc = 1.0f / sqrtf(ellipse);
            next1 *= sc;
            next2 *= sc;
        }
        c.nImp = nextNormal;
        c.t1Imp = next1;
        c.t2Imp = next2;
        const V3 imp = c.normal * (nextNormal - oldNormal) + P.t1 * (next1 - old1) + P.t2 * (next2 - old2);
        if (dynA) { a.v += imp * ima; a.w += invIF(a, cross(P.ra, imp)); }
        if (dynB) { b.v -= imp * imb; b.w -= invIF(b, cross(P.rb, imp)); }
    }
    if (c.rolling > 0.0f && P.kr1 > 0.0f && P.kr2 > 0.0f) {
        const V3 wr = a.w - b.w;
        const float o1 = c.r1Imp, o2 = c.r2Imp;
        float n1 = o1 - dot(wr, P.t1) / P.kr1;
        float n2 = o2 - dot(wr, P.t2) / P.kr2;
        const float limit = c.rolling * c.nImp;
        const float mag = sqrtf(n1 * n1 + n2 * n2);
        if (mag > limit && mag > 1e-9f) {
            const float sc = limit / mag;
            n1 *= sc;
            n2 *= sc;
        }
        c.r1Imp = n1;
        c.r2Imp = n2;
        const V3 tq = P.t1 * (n1 - o1) + P.t2 * (n2 - o2);
        if (dynA) a.w += invIF(a, tq);
        if (dynB) b.w -= invIF(b, tq);
    }
    if (c.spinning > 0.0f && P.ks > 0.0f) {
        const V3 wr = a.w - b.w;
        const float old = c.sImp;
        float next = old - dot(wr, c.normal) / P.ks;
        const float limit = c.spinning * c.nImp;
        next = vclamp(next, -limit, limit);
        c.sImp = next;
        const V3 tq = c.normal * (next - old);
        if (dynA) a.w += invIF(a, tq);
        if (dynB) b.w -= invIF(b, tq);
    }
}

}  // namespace vxb
