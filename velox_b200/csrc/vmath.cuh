// Device vector / quaternion arithmetic and the rigid-body kinematics of the
// contact pipeline.
//
// Evaluation order follows the reference's VELOX_HD math
// (include/velox/math.h, include/velox/body.h) operation for operation, and
// the library is compiled with --fmad=false, so results agree bit for bit
// with the reference built with VELOX_STRICT_FLOATING_POINT. The rules that
// make orientation state canonical are reproduced exactly:
//   * cross products give zero components a sign chosen by the lexicographic
//     order of the operands (math.h:34-47);
//   * unit-quaternion products are rounded to a 2^-22 grid (math.h:64-86);
//   * quaternion normalisation rescales only outside [1e-16, FLT_MAX]
//     (math.h:88-112).
#pragma once
#include <cfloat>
#include <cstdint>

namespace vxb {

// A host-side parity check of code written on this header may define VXD as
// __host__ __device__ before including it.
#ifndef VXD
#define VXD __device__ __forceinline__
#endif

struct V3 { float x, y, z; };
struct Q4 { float x, y, z, w; };

VXD V3 mk(float x, float y, float z) { return V3{x, y, z}; }
VXD V3 operator+(const V3& a, const V3& b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
VXD V3 operator-(const V3& a, const V3& b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
VXD V3 operator*(const V3& a, float s) { return V3{a.x * s, a.y * s, a.z * s}; }
VXD V3 operator-(const V3& a) { return V3{-a.x, -a.y, -a.z}; }
VXD V3& operator+=(V3& a, const V3& b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
VXD V3& operator-=(V3& a, const V3& b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; return a; }
VXD V3& operator*=(V3& a, float s) { a.x *= s; a.y *= s; a.z *= s; return a; }

VXD float dot(const V3& a, const V3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
VXD float signedZero(float value, int order) {
    return value != 0.0f ? value : (order > 0 ? 0.0f : -0.0f);
}
VXD V3 cross(const V3& a, const V3& b) {
    const int order = a.x != b.x ? (a.x > b.x ? 1 : -1)
                    : a.y != b.y ? (a.y > b.y ? 1 : -1)
                    : a.z != b.z ? (a.z > b.z ? 1 : -1) : 1;
    return V3{signedZero(a.y * b.z - a.z * b.y, order),
              signedZero(a.z * b.x - a.x * b.z, order),
              signedZero(a.x * b.y - a.y * b.x, order)};
}
VXD float lengthSq(const V3& v) { return dot(v, v); }
VXD float length(const V3& v) { return sqrtf(lengthSq(v)); }
VXD V3 normalize(const V3& v) {
    float len = length(v);
    return len > 1e-8f ? v * (1.0f / len) : V3{0.0f, 0.0f, 0.0f};
}
VXD float vmin(float a, float b) { return a < b ? a : b; }
VXD float vmax(float a, float b) { return a > b ? a : b; }
VXD float vclamp(float v, float lo, float hi) { return vmin(vmax(v, lo), hi); }

VXD float gridRound(float value) {
    const float kGrid = 4194304.0f;  // 2^22
    const float scaled = value * kGrid;
    const float rounded = scaled >= 0.0f ? floorf(scaled + 0.5f) : ceilf(scaled - 0.5f);
    return rounded / kGrid;
}

VXD Q4 qmul(const Q4& a, const Q4& b) {
    Q4 r{a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
         a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
         a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w,
         a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z};
    const float la = a.x * a.x + a.y * a.y + a.z * a.z + a.w * a.w;
    const float lb = b.x * b.x + b.y * b.y + b.z * b.z + b.w * b.w;
    if (la < 0.999f || la > 1.001f || lb < 0.999f || lb > 1.001f) return r;
    return Q4{gridRound(r.x), gridRound(r.y), gridRound(r.z), gridRound(r.w)};
}

VXD Q4 qnormalize(const Q4& q) {
    const float ls = q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w;
    if (ls >= 1e-16f && ls <= FLT_MAX) {
        const float inv = 1.0f / sqrtf(ls);
        return Q4{q.x * inv, q.y * inv, q.z * inv, q.w * inv};
    }
    const float s = vmax(vmax(fabsf(q.x), fabsf(q.y)), vmax(fabsf(q.z), fabsf(q.w)));
    if (!(s >= 1e-8f)) return Q4{0.0f, 0.0f, 0.0f, 1.0f};
    const float x = q.x / s, y = q.y / s, z = q.z / s, w = q.w / s;
    const float l = sqrtf(x * x + y * y + z * z + w * w);
    if (!(l >= 1e-8f)) return Q4{0.0f, 0.0f, 0.0f, 1.0f};
    const float inv = 1.0f / l;
    return Q4{x * inv, y * inv, z * inv, w * inv};
}

VXD V3 rotate(const Q4& q, const V3& v) {
    const V3 u{q.x, q.y, q.z};
    const V3 t = cross(u, cross(u, v) + v * q.w);
    return v + t * 2.0f;
}
VXD V3 rotateInv(const Q4& q, const V3& v) { return rotate(Q4{-q.x, -q.y, -q.z, q.w}, v); }

VXD Q4 qintegrate(const Q4& q, const V3& omega, float dt) {
    const Q4 dq = qmul(Q4{omega.x * 0.5f * dt, omega.y * 0.5f * dt, omega.z * 0.5f * dt, 0.0f}, q);
    return qnormalize(Q4{q.x + dq.x, q.y + dq.y, q.z + dq.z, q.w + dq.w});
}

VXD V3 f3(const float4& v) { return V3{v.x, v.y, v.z}; }
VXD Q4 q4(const float4& v) { return Q4{v.x, v.y, v.z, v.w}; }
VXD float4 pack(const V3& v, float w) { return make_float4(v.x, v.y, v.z, w); }
VXD float4 pack(const Q4& q) { return make_float4(q.x, q.y, q.z, q.w); }

// ---- packed per-body flags (built from vx_body by the pack kernel) -------

enum : uint32_t {
    kShapeMask = 0xFu,            // bits 0-3 ShapeType
    kMotionShift = 4,             // bits 4-5 MotionType
    kQualityShift = 6,            // bits 6-7 MotionQuality
    kContinuousBit = 1u << 8,     // ccdTuning.enableContinuous
    kSensorBit = 1u << 9,
    kFixedRotationBit = 1u << 10,
    kAsleepBit = 1u << 11,        // asleep == 1 (isFullyAsleep)
    kFrictionCombineShift = 12,   // bits 12-14
    kRestitutionCombineShift = 15,// bits 15-17
    kGeomQualityShift = 18,       // bits 18-19
};
enum : uint32_t { kSphere = 0, kPlane = 1, kBox = 2, kCapsule = 3, kMesh = 4, kHull = 5,
                  kCompound = 6, kCylinder = 7, kCone = 8, kRoundedBox = 9, kEllipsoid = 10 };
enum : uint32_t { kStatic = 0, kKinematic = 1, kDynamic = 2 };
enum : uint32_t { kQualityLow = 0, kQualityMedium = 1, kQualityHigh = 2, kQualityLocked = 3 };

VXD uint32_t shapeOf(uint32_t f) { return f & kShapeMask; }
VXD uint32_t motionOf(uint32_t f) { return (f >> kMotionShift) & 3u; }
VXD uint32_t qualityOf(uint32_t f) { return (f >> kQualityShift) & 3u; }
VXD bool isDynamic(uint32_t f) { return motionOf(f) == kDynamic; }
VXD bool isStaticBody(uint32_t f) { return motionOf(f) == kStatic; }
VXD bool isSensor(uint32_t f) { return (f & kSensorBit) != 0; }
VXD bool isAsleep(uint32_t f) { return (f & kAsleepBit) != 0; }
VXD bool isLocked(uint32_t f) { return qualityOf(f) == kQualityLocked; }
VXD bool isRotationLocked(uint32_t f) { return isLocked(f) || (f & kFixedRotationBit) != 0; }
VXD bool sweeps(uint32_t f) {  // continuous sweep enabled (narrowphase.h:391-394, :431-436)
    return (f & kContinuousBit) && qualityOf(f) != kQualityLow && qualityOf(f) != kQualityLocked;
}
VXD bool inert(uint32_t f) { return isStaticBody(f) || isAsleep(f); }

// Mass properties needed by the solver and the integrator.
struct Mass {
    V3 invI;        // invInertia
    float invMass;  // raw Body::invMass
    Q4 iq;          // inertiaOrientation
    uint32_t flags;
};

VXD float solverInvMass(const Mass& m) {
    return isDynamic(m.flags) && !isLocked(m.flags) ? m.invMass : 0.0f;
}
VXD Q4 inertiaFrameAt(const Mass& m, const Q4& at) {
    if (m.iq.x == 0.0f && m.iq.y == 0.0f && m.iq.z == 0.0f && m.iq.w == 1.0f) return at;
    return qmul(at, m.iq);
}
// World-space inverse inertia times v at orientation `at` (body.h:219-226).
VXD V3 invInertiaMulAt(const Mass& m, const V3& v, const Q4& at) {
    if (!isDynamic(m.flags) || isRotationLocked(m.flags)) return V3{0.0f, 0.0f, 0.0f};
    const Q4 frame = inertiaFrameAt(m, at);
    const V3 l = rotateInv(frame, v);
    return rotate(frame, V3{l.x * m.invI.x, l.y * m.invI.y, l.z * m.invI.z});
}
// Inertia (not inverse) times v at orientation `at` (body.h:233-243).
VXD V3 inertiaMulAt(const Mass& m, const V3& v, const Q4& at) {
    if (isRotationLocked(m.flags)) return V3{0.0f, 0.0f, 0.0f};
    const Q4 frame = inertiaFrameAt(m, at);
    const V3 l = rotateInv(frame, v);
    const V3 w{m.invI.x > 0.0f ? l.x / m.invI.x : 0.0f, m.invI.y > 0.0f ? l.y / m.invI.y : 0.0f,
               m.invI.z > 0.0f ? l.z / m.invI.z : 0.0f};
    return rotate(frame, w);
}

// Body::advanceOrientation (body.h:266-300): implicit-midpoint gyroscopic
// update for anisotropic dynamic bodies, plain integration otherwise.
VXD void advanceOrientation(const Mass& m, Q4& q, V3& w, float dt) {
    if (isRotationLocked(m.flags)) { w = V3{0.0f, 0.0f, 0.0f}; return; }
    const bool anisotropic = m.invI.x != m.invI.y || m.invI.y != m.invI.z;
    const float lo = vmin(m.invI.x, vmin(m.invI.y, m.invI.z));
    const float hi = vmax(m.invI.x, vmax(m.invI.y, m.invI.z));
    const bool stable = lo > 0.0f && hi / lo <= 1.0e6f;
    if (isDynamic(m.flags) && anisotropic && stable) {
        const V3 L = inertiaMulAt(m, w, q);
        const Q4 start = q;
        const V3 w0 = w;
        Q4 next = qintegrate(start, w0, dt);
        for (int it = 0; it < 3; ++it) {
            const V3 w1 = invInertiaMulAt(m, L, next);
            const V3 mid = (w0 + w1) * 0.5f;
            next = qintegrate(start, mid, dt);
        }
        q = next;
        w = invInertiaMulAt(m, L, q);
    } else {
        q = qintegrate(q, w, dt);
    }
}

// Body::advanceTransform (body.h:306-321).
VXD void advanceTransform(const Mass& m, V3& p, Q4& q, const V3& v, V3& w, float dt) {
    if (isLocked(m.flags)) return;
    const V3 prev = p;
    const V3 d = v * dt;
    p += d;
    if (d.x != 0.0f && p.x == prev.x) p.x = nextafterf(prev.x, d.x > 0.0f ? FLT_MAX : -FLT_MAX);
    if (d.y != 0.0f && p.y == prev.y) p.y = nextafterf(prev.y, d.y > 0.0f ? FLT_MAX : -FLT_MAX);
    if (d.z != 0.0f && p.z == prev.z) p.z = nextafterf(prev.z, d.z > 0.0f ? FLT_MAX : -FLT_MAX);
    advanceOrientation(m, q, w, dt);
}

}  // namespace vxb
