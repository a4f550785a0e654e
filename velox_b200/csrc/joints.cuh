// Joint constraints of the reference's device joint pass (src/joint_solver.h,
// run by src/backend_cuda.cu:691-760 once per substep after the contact
// sweeps): the velocity-level impulse solve of the thirteen joint types,
// with Baumgarte position bias. Written on this library's vector types and
// mass records; every expression keeps the reference's evaluation order so
// that, compiled with --fmad=false, results equal the reference's strict
// build to rounding (atan2f / acosf are CUDA's on the device).
//
// The functions are VXD (device; a host-side parity check may redefine VXD
// as __host__ __device__) and touch only the joint record and two bodies.
#pragma once
#include "vmath.cuh"
#include "velox_b200_types.h"

namespace vxb {
namespace joint {

constexpr int kIterations = 8;          // joint sweeps per substep
constexpr float kBeta = 0.2f;           // Baumgarte factor
constexpr float kMaxPositionBias = 10.0f;

// One body as the joint rows see it (pose, velocities, mass record).
struct JBody {
    V3 p;
    Q4 q;
    V3 v;
    V3 w;
    Mass m;
};

struct M3 {
    V3 c0, c1, c2;
};

VXD V3 v3of(const vx_vec3& v) { return V3{v.x, v.y, v.z}; }
VXD vx_vec3 vxOf(const V3& v) { return vx_vec3{v.x, v.y, v.z}; }
VXD void addTo(vx_vec3& acc, const V3& d) { acc = vxOf(v3of(acc) + d); }

VXD bool movable(const JBody& b) { return isDynamic(b.m.flags) && !isLocked(b.m.flags); }
VXD float invMassOf(const JBody& b) { return solverInvMass(b.m); }
VXD V3 invI(const JBody& b, const V3& v) { return invInertiaMulAt(b.m, v, b.q); }

VXD V3 clampPositionBias(const V3& bias) {
    const float magnitudeSq = lengthSq(bias);
    if (magnitudeSq <= kMaxPositionBias * kMaxPositionBias) return bias;
    return bias * (kMaxPositionBias / sqrtf(magnitudeSq));
}

VXD V3 mul(const M3& m, const V3& v) { return m.c0 * v.x + m.c1 * v.y + m.c2 * v.z; }

VXD M3 inverse(const M3& m) {
    const V3 r0 = cross(m.c1, m.c2);
    const V3 r1 = cross(m.c2, m.c0);
    const V3 r2 = cross(m.c0, m.c1);
    const float det = dot(m.c0, r0);
    const float inv = fabsf(det) > 1e-12f ? 1.0f / det : 0.0f;
    return M3{V3{r0.x * inv, r1.x * inv, r2.x * inv}, V3{r0.y * inv, r1.y * inv, r2.y * inv},
              V3{r0.z * inv, r1.z * inv, r2.z * inv}};
}

// Point-to-point effective-mass matrix of two anchors, column by column.
VXD V3 pointMassColumn(const JBody& a, const JBody& b, const V3& ra, const V3& rb, const V3& e) {
    V3 k = e * (invMassOf(a) + invMassOf(b));
    k += cross(invI(a, cross(ra, e)), ra);
    k += cross(invI(b, cross(rb, e)), rb);
    return k;
}
VXD M3 pointMass(const JBody& a, const JBody& b, const V3& ra, const V3& rb) {
    return M3{pointMassColumn(a, b, ra, rb, V3{1.0f, 0.0f, 0.0f}),
              pointMassColumn(a, b, ra, rb, V3{0.0f, 1.0f, 0.0f}),
              pointMassColumn(a, b, ra, rb, V3{0.0f, 0.0f, 1.0f})};
}

VXD M3 angularMass(const JBody& a, const JBody& b) {
    return M3{invI(a, V3{1.0f, 0.0f, 0.0f}) + invI(b, V3{1.0f, 0.0f, 0.0f}),
              invI(a, V3{0.0f, 1.0f, 0.0f}) + invI(b, V3{0.0f, 1.0f, 0.0f}),
              invI(a, V3{0.0f, 0.0f, 1.0f}) + invI(b, V3{0.0f, 0.0f, 1.0f})};
}

VXD V3 anchorVelocity(const JBody& body, const V3& r) { return body.v + cross(body.w, r); }

VXD void applyImpulse(JBody& body, const V3& r, const V3& impulse, float sign) {
    if (!movable(body)) return;
    body.v += impulse * (sign * invMassOf(body));
    body.w += invI(body, cross(r, impulse)) * sign;
}

VXD void applyLinear(vx_joint& j, JBody& a, JBody& b, const V3& ra, const V3& rb, const V3& impulse, float signA) {
    applyImpulse(a, ra, impulse, signA);
    applyImpulse(b, rb, impulse, -signA);
    addTo(j.reactionLinearImpulse, impulse * signA);
}

VXD void applyAngular(vx_joint& j, JBody& a, JBody& b, const V3& impulse, float signA = 1.0f) {
    if (movable(a)) a.w += invI(a, impulse) * signA;
    if (movable(b)) b.w -= invI(b, impulse) * signA;
    addTo(j.reactionAngularImpulse, impulse * signA);
}

// Orthonormal joint frames of both bodies (axis, reference, their cross).
VXD void frames(const vx_joint& j, const JBody& a, const JBody& b, V3& xA, V3& yA, V3& zA, V3& xB, V3& yB,
                V3& zB) {
    xA = normalize(rotate(a.q, v3of(j.localAxisA)));
    yA = normalize(rotate(a.q, v3of(j.localRefA)));
    zA = normalize(cross(xA, yA));
    yA = cross(zA, xA);
    xB = normalize(rotate(b.q, v3of(j.localAxisB)));
    yB = normalize(rotate(b.q, v3of(j.localRefB)));
    zB = normalize(cross(xB, yB));
    yB = cross(zB, xB);
}

// Rotation matrix to unit quaternion (the branch on the largest diagonal term).
VXD Q4 matrixQuaternion(float m00, float m01, float m02, float m10, float m11, float m12, float m20, float m21,
                        float m22) {
    Q4 q;
    const float trace = m00 + m11 + m22;
    if (trace > 0.0f) {
        const float s = sqrtf(trace + 1.0f) * 2.0f;
        q = Q4{(m21 - m12) / s, (m02 - m20) / s, (m10 - m01) / s, 0.25f * s};
    } else if (m00 > m11 && m00 > m22) {
        const float s = sqrtf(1.0f + m00 - m11 - m22) * 2.0f;
        q = Q4{0.25f * s, (m01 + m10) / s, (m02 + m20) / s, (m21 - m12) / s};
    } else if (m11 > m22) {
        const float s = sqrtf(1.0f + m11 - m00 - m22) * 2.0f;
        q = Q4{(m01 + m10) / s, 0.25f * s, (m12 + m21) / s, (m02 - m20) / s};
    } else {
        const float s = sqrtf(1.0f + m22 - m00 - m11) * 2.0f;
        q = Q4{(m02 + m20) / s, (m12 + m21) / s, 0.25f * s, (m10 - m01) / s};
    }
    return qnormalize(q);
}

// Relative rotation of B's frame in A's frame as a rotation vector.
VXD V3 rotationVector(const vx_joint& j, const JBody& a, const JBody& b) {
    V3 xA, yA, zA, xB, yB, zB;
    frames(j, a, b, xA, yA, zA, xB, yB, zB);
    Q4 q = matrixQuaternion(dot(xA, xB), dot(xA, yB), dot(xA, zB), dot(yA, xB), dot(yA, yB), dot(yA, zB),
                            dot(zA, xB), dot(zA, yB), dot(zA, zB));
    if (q.w < 0.0f) q = Q4{-q.x, -q.y, -q.z, -q.w};
    const V3 v{q.x, q.y, q.z};
    const float sinHalf = length(v);
    if (sinHalf < 1e-7f) return v * 2.0f;
    const float angle = 2.0f * atan2f(sinHalf, vclamp(q.w, 0.0f, 1.0f));
    return v * (angle / sinHalf);
}

VXD float comp(const V3& v, int axis) { return axis == 0 ? v.x : (axis == 1 ? v.y : v.z); }
VXD float comp(const vx_vec3& v, int axis) { return axis == 0 ? v.x : (axis == 1 ? v.y : v.z); }
VXD float& compRef(vx_vec3& v, int axis) { return axis == 0 ? v.x : (axis == 1 ? v.y : v.z); }

// Clears a joint's per-substep scratch and its broken flag.
VXD void reset(vx_joint& j) {
    j.motorImpulse = 0.0f;
    j.limitImpulse = 0.0f;
    j.swingImpulse = 0.0f;
    j.twistImpulse = 0.0f;
    j.springImpulse = 0.0f;
    const vx_vec3 z{0.0f, 0.0f, 0.0f};
    j.linearMotorImpulse = z;
    j.angularMotorImpulse = z;
    j.linearLimitImpulse = z;
    j.angularLimitImpulse = z;
    j.reactionLinearImpulse = z;
    j.reactionAngularImpulse = z;
    j.broken = 0;
}

// Locks the relative orientation (frames aligned) in one 3x3 solve.
VXD void solveAngularFrame(vx_joint& j, JBody& a, JBody& b, float biasScale) {
    V3 xA, yA, zA, xB, yB, zB;
    frames(j, a, b, xA, yA, zA, xB, yB, zB);
    const V3 error = (cross(xB, xA) + cross(yB, yA) + cross(zB, zA)) * 0.5f;
    const V3 relativeW = a.w - b.w;
    const V3 impulse = mul(inverse(angularMass(a, b)), -(relativeW + error * biasScale));
    applyAngular(j, a, b, impulse);
}


// Per-axis linear and angular limits and motors in A's joint frame
// (joint_solver.h:171-257).
VXD void solveSixDof(vx_joint& j, JBody& a, JBody& b, const V3& ra, const V3& rb, const V3& pa, const V3& pb,
                     float dt) {
    V3 xA, yA, zA, xB, yB, zB;
    frames(j, a, b, xA, yA, zA, xB, yB, zB);
    const V3 axes[3] = {xA, yA, zA};
    const V3 d = pb - pa;
    const M3 pointK = pointMass(a, b, ra, rb);
    for (int i = 0; i < 3; ++i) {
        const uint8_t bit = (uint8_t)(1u << i);
        const V3 axis = axes[i];
        const float k = dot(axis, mul(pointK, axis));
        if (k <= 0.0f) continue;
        float speed = dot(anchorVelocity(b, rb) - anchorVelocity(a, ra), axis);
        if (j.linearMotorMask & bit) {
            float lambda = (comp(j.linearMotorSpeed, i) - speed) / k;
            const float maxImpulse = comp(j.maxLinearMotorForce, i) * dt;
            float& sum = compRef(j.linearMotorImpulse, i);
            const float old = sum;
            sum = vclamp(old + lambda, -maxImpulse, maxImpulse);
            lambda = sum - old;
            applyLinear(j, a, b, ra, rb, axis * lambda, -1.0f);
            speed = dot(anchorVelocity(b, rb) - anchorVelocity(a, ra), axis);
        }
        if (!(j.linearLimitMask & bit)) continue;
        const float position = dot(d, axis);
        const float lower = comp(j.lowerLinearLimit, i);
        const float upper = comp(j.upperLinearLimit, i);
        float lambda = 0.0f;
        float& sum = compRef(j.linearLimitImpulse, i);
        const float old = sum;
        if (lower == upper) {
            lambda = -(speed + (position - lower) * (kBeta / dt)) / k;
            sum += lambda;
        } else if (position < lower) {
            lambda = -(speed + (position - lower) * (kBeta / dt)) / k;
            sum = vmax(0.0f, old + lambda);
            lambda = sum - old;
        } else if (position > upper) {
            lambda = -(speed + (position - upper) * (kBeta / dt)) / k;
            sum = vmin(0.0f, old + lambda);
            lambda = sum - old;
        }
        if (lambda != 0.0f) applyLinear(j, a, b, ra, rb, axis * lambda, -1.0f);
    }
    const V3 rotation = rotationVector(j, a, b);
    for (int i = 0; i < 3; ++i) {
        const uint8_t bit = (uint8_t)(1u << i);
        const V3 axis = axes[i];
        const float k = dot(axis, invI(a, axis)) + dot(axis, invI(b, axis));
        if (k <= 0.0f) continue;
        float speed = dot(b.w - a.w, axis);
        if (j.angularMotorMask & bit) {
            float lambda = (speed - comp(j.angularMotorSpeed, i)) / k;
            const float maxImpulse = comp(j.maxAngularMotorTorque, i) * dt;
            float& sum = compRef(j.angularMotorImpulse, i);
            const float old = sum;
            sum = vclamp(old + lambda, -maxImpulse, maxImpulse);
            lambda = sum - old;
            applyAngular(j, a, b, axis * lambda);
            speed = dot(b.w - a.w, axis);
        }
        if (!(j.angularLimitMask & bit)) continue;
        const float angle = comp(rotation, i);
        const float lower = comp(j.lowerAngularLimit, i);
        const float upper = comp(j.upperAngularLimit, i);
        float lambda = 0.0f;
        float& sum = compRef(j.angularLimitImpulse, i);
        const float old = sum;
        if (lower == upper) {
            lambda = (speed + (angle - lower) * (kBeta / dt)) / k;
            sum += lambda;
        } else if (angle < lower) {
            lambda = (speed + (angle - lower) * (kBeta / dt)) / k;
            sum = vmin(0.0f, old + lambda);
            lambda = sum - old;
        } else if (angle > upper) {
            lambda = (speed + (angle - upper) * (kBeta / dt)) / k;
            sum = vmax(0.0f, old + lambda);
            lambda = sum - old;
        }
        if (lambda != 0.0f) applyAngular(j, a, b, axis * lambda);
    }
}

// Two lateral directions perpendicular to `axis`, from the reference vector
// `ref` (or a fixed world axis when `ref` is parallel to `axis`).
VXD void lateralPair(const V3& axis, V3 ref, V3& t0, V3& t1) {
    V3 t = normalize(ref - axis * dot(ref, axis));
    if (lengthSq(t) < 1e-12f) {
        ref = fabsf(axis.x) < 0.9f ? V3{1.0f, 0.0f, 0.0f} : V3{0.0f, 1.0f, 0.0f};
        t = normalize(cross(axis, ref));
    }
    t0 = t;
    t1 = cross(axis, t);
}

// Slider: lateral lock, locked frame, motor and travel limits along the axis
// (joint_solver.h:259-315).
VXD void solvePrismatic(vx_joint& j, JBody& a, JBody& b, const V3& ra, const V3& rb, const V3& pa, const V3& pb,
                        float dt) {
    const V3 axis = normalize(rotate(a.q, v3of(j.localAxisA)));
    V3 tangents[2];
    lateralPair(axis, rotate(a.q, v3of(j.localRefA)), tangents[0], tangents[1]);
    const M3 pointK = pointMass(a, b, ra, rb);
    const V3 error = pa - pb;
    V3 velocity = anchorVelocity(a, ra) - anchorVelocity(b, rb);
    for (int i = 0; i < 2; ++i) {
        const V3 tangent = tangents[i];
        const float k = dot(tangent, mul(pointK, tangent));
        if (k <= 0.0f) continue;
        const float lambda = -(dot(velocity, tangent) + dot(error, tangent) * (kBeta / dt)) / k;
        applyLinear(j, a, b, ra, rb, tangent * lambda, 1.0f);
        velocity = anchorVelocity(a, ra) - anchorVelocity(b, rb);
    }
    solveAngularFrame(j, a, b, kBeta / dt);
    const float kAxis = dot(axis, mul(pointK, axis));
    if (kAxis <= 0.0f) return;
    float axisSpeed = dot(anchorVelocity(b, rb) - anchorVelocity(a, ra), axis);
    if (j.enableMotor) {
        float lambda = (j.motorSpeed - axisSpeed) / kAxis;
        const float maxImpulse = j.maxMotorForce * dt;
        const float old = j.motorImpulse;
        j.motorImpulse = vclamp(old + lambda, -maxImpulse, maxImpulse);
        lambda = j.motorImpulse - old;
        applyLinear(j, a, b, ra, rb, axis * lambda, -1.0f);
        axisSpeed = dot(anchorVelocity(b, rb) - anchorVelocity(a, ra), axis);
    }
    if (!j.enableLimit) return;
    const float translation = dot(pb - pa, axis);
    float lambda = 0.0f;
    const float old = j.limitImpulse;
    if (translation < j.lowerLimit) {
        const float bias = (translation - j.lowerLimit) * (kBeta / dt);
        lambda = -(axisSpeed + bias) / kAxis;
        j.limitImpulse = vmax(0.0f, old + lambda);
        lambda = j.limitImpulse - old;
    } else if (translation > j.upperLimit) {
        const float bias = (translation - j.upperLimit) * (kBeta / dt);
        lambda = -(axisSpeed + bias) / kAxis;
        j.limitImpulse = vmin(0.0f, old + lambda);
        lambda = j.limitImpulse - old;
    }
    if (lambda != 0.0f) applyLinear(j, a, b, ra, rb, axis * lambda, -1.0f);
}

// Point lock with the clamped bias, then an angular limit-or-motor about a
// single axis (the hinge's head, joint_solver.h:320-324).
VXD void lockPointClamped(vx_joint& j, JBody& a, JBody& b, const V3& ra, const V3& rb, const V3& pa, const V3& pb,
                          float dt) {
    const V3 velocity = anchorVelocity(a, ra) - anchorVelocity(b, rb);
    const V3 bias = clampPositionBias((pa - pb) * (kBeta / dt));
    const V3 impulse = mul(inverse(pointMass(a, b, ra, rb)), -(velocity + bias));
    applyLinear(j, a, b, ra, rb, impulse, 1.0f);
}

// Hinge: point lock, two angular rows keeping the axes aligned, motor and
// angle limits about A's axis (joint_solver.h:317-375).
VXD void solveHinge(vx_joint& j, JBody& a, JBody& b, const V3& ra, const V3& rb, const V3& pa, const V3& pb,
                    float dt) {
    lockPointClamped(j, a, b, ra, rb, pa, pb, dt);
    const V3 axisA = rotate(a.q, v3of(j.localAxisA));
    const V3 axisB = rotate(b.q, v3of(j.localAxisB));
    const V3 error = cross(axisB, axisA);
    const V3 ref = fabsf(axisA.x) < 0.9f ? V3{1.0f, 0.0f, 0.0f} : V3{0.0f, 1.0f, 0.0f};
    V3 tangents[2];
    tangents[0] = normalize(cross(axisA, ref));
    tangents[1] = cross(axisA, tangents[0]);
    V3 relativeW = a.w - b.w;
    for (int i = 0; i < 2; ++i) {
        const V3 tangent = tangents[i];
        const float k = dot(tangent, invI(a, tangent)) + dot(tangent, invI(b, tangent));
        if (k <= 0.0f) continue;
        const float lambda = -(dot(relativeW, tangent) + dot(error, tangent) * (kBeta / dt)) / k;
        applyAngular(j, a, b, tangent * lambda);
        relativeW = a.w - b.w;
    }
    const float kAxis = dot(axisA, invI(a, axisA)) + dot(axisA, invI(b, axisA));
    if (kAxis <= 0.0f) return;
    if (j.enableMotor) {
        const float wAxis = dot(a.w - b.w, axisA);
        float lambda = (j.motorSpeed - wAxis) / kAxis;
        const float maxImpulse = j.maxMotorTorque * dt;
        const float old = j.motorImpulse;
        j.motorImpulse = vclamp(old + lambda, -maxImpulse, maxImpulse);
        lambda = j.motorImpulse - old;
        applyAngular(j, a, b, axisA * lambda);
    }
    if (!j.enableLimit) return;
    const V3 refA = rotate(a.q, v3of(j.localRefA));
    const V3 refB = rotate(b.q, v3of(j.localRefB));
    const float angle = atan2f(dot(cross(refA, refB), axisA), dot(refA, refB));
    const float wAxis = dot(a.w - b.w, axisA);
    float lambda = 0.0f;
    const float old = j.limitImpulse;
    if (angle < j.lowerLimit) {
        const float target = (angle - j.lowerLimit) * (kBeta / dt);
        lambda = (target - wAxis) / kAxis;
        j.limitImpulse = vmin(0.0f, old + lambda);
        lambda = j.limitImpulse - old;
    } else if (angle > j.upperLimit) {
        const float target = (angle - j.upperLimit) * (kBeta / dt);
        lambda = (target - wAxis) / kAxis;
        j.limitImpulse = vmax(0.0f, old + lambda);
        lambda = j.limitImpulse - old;
    }
    if (lambda != 0.0f) applyAngular(j, a, b, axisA * lambda);
}

// Unclamped point lock (ball, cone-twist, fixed and motor heads).
VXD V3 pointLockImpulse(const JBody& a, const JBody& b, const V3& ra, const V3& rb, const V3& pa, const V3& pb,
                        float dt) {
    const V3 velocity = anchorVelocity(a, ra) - anchorVelocity(b, rb);
    const V3 bias = (pa - pb) * (kBeta / dt);
    return mul(inverse(pointMass(a, b, ra, rb)), -(velocity + bias));
}

// Ball joint with a cone swing limit and a twist limit (joint_solver.h:377-437).
VXD void solveConeTwist(vx_joint& j, JBody& a, JBody& b, const V3& ra, const V3& rb, const V3& pa, const V3& pb,
                        float dt) {
    applyLinear(j, a, b, ra, rb, pointLockImpulse(a, b, ra, rb, pa, pb, dt), 1.0f);
    const V3 axisA = normalize(rotate(a.q, v3of(j.localAxisA)));
    const V3 axisB = normalize(rotate(b.q, v3of(j.localAxisB)));
    V3 relativeW = a.w - b.w;
    if (j.enableSwingLimit) {
        const float angle = acosf(vclamp(dot(axisA, axisB), -1.0f, 1.0f));
        if (angle > j.swingLimit) {
            V3 n = cross(axisB, axisA);
            if (lengthSq(n) < 1e-10f) n = cross(axisA, rotate(a.q, v3of(j.localRefA)));
            n = normalize(n);
            const float k = dot(n, invI(a, n)) + dot(n, invI(b, n));
            if (k > 0.0f) {
                const float error = angle - j.swingLimit;
                float lambda = -(dot(relativeW, n) + error * (kBeta / dt)) / k;
                const float old = j.swingImpulse;
                j.swingImpulse = vmin(0.0f, old + lambda);
                lambda = j.swingImpulse - old;
                applyAngular(j, a, b, n * lambda);
                relativeW = a.w - b.w;
            }
        }
    }
    if (!j.enableTwistLimit) return;
    V3 refA = rotate(a.q, v3of(j.localRefA));
    V3 refB = rotate(b.q, v3of(j.localRefB));
    refA = normalize(refA - axisA * dot(refA, axisA));
    refB = normalize(refB - axisA * dot(refB, axisA));
    if (lengthSq(refA) < 1e-10f || lengthSq(refB) < 1e-10f) return;
    const float angle = atan2f(dot(cross(refA, refB), axisA), dot(refA, refB));
    const float k = dot(axisA, invI(a, axisA)) + dot(axisA, invI(b, axisA));
    if (k <= 0.0f) return;
    const float wAxis = dot(a.w - b.w, axisA);
    float lambda = 0.0f;
    const float old = j.twistImpulse;
    if (angle < j.lowerTwistLimit) {
        const float target = (angle - j.lowerTwistLimit) * (kBeta / dt);
        lambda = (target - wAxis) / k;
        j.twistImpulse = vmin(0.0f, old + lambda);
        lambda = j.twistImpulse - old;
    } else if (angle > j.upperTwistLimit) {
        const float target = (angle - j.upperTwistLimit) * (kBeta / dt);
        lambda = (target - wAxis) / k;
        j.twistImpulse = vmax(0.0f, old + lambda);
        lambda = j.twistImpulse - old;
    }
    if (lambda != 0.0f) applyAngular(j, a, b, axisA * lambda);
}

// Rigid lock with an optionally soft angular part (joint_solver.h:439-474).
VXD void solveWeld(vx_joint& j, JBody& a, JBody& b, const V3& ra, const V3& rb, const V3& pa, const V3& pb,
                   float dt) {
    lockPointClamped(j, a, b, ra, rb, pa, pb, dt);
    if (j.weldFrequencyHz > 0.0f) {
        const V3 rotation = rotationVector(j, a, b);
        const V3 relativeW = a.w - b.w;
        const float tau = 6.28318530718f;
        const float omega = tau * j.weldFrequencyHz;
        const M3 angK = angularMass(a, b);
        const V3 ex{1.0f, 0.0f, 0.0f};
        const float mass = 1.0f / (dot(ex, invI(a, ex)) + dot(ex, invI(b, ex)) + 1e-12f);
        const float stiffness = mass * omega * omega;
        const float damping = 2.0f * mass * j.weldDampingRatio * omega;
        const float denom = vmax(dt * (damping + dt * stiffness), 1e-12f);
        const float softness = 1.0f / denom;
        const V3 angularBias = rotation * (dt * stiffness * softness);
        const V3 lambda = mul(inverse(angK), -(relativeW + angularBias + v3of(j.angularMotorImpulse) * softness));
        addTo(j.angularMotorImpulse, lambda);
        applyAngular(j, a, b, lambda);
    } else {
        solveAngularFrame(j, a, b, kBeta / dt);
    }
}

// Wheel on a suspension axis: lateral lock, spring along the axis, two
// locked angular directions, steering and an axle motor
// (joint_solver.h:476-583).
VXD void solveWheel(vx_joint& j, JBody& a, JBody& b, const V3& ra, const V3& rb, const V3& pa, const V3& pb,
                    float dt) {
    const V3 axisA = normalize(rotate(a.q, v3of(j.localAxisA)));
    V3 tangents[2];
    lateralPair(axisA, rotate(a.q, v3of(j.localRefA)), tangents[0], tangents[1]);
    const M3 pointK = pointMass(a, b, ra, rb);
    const V3 error = pa - pb;
    V3 vel = anchorVelocity(a, ra) - anchorVelocity(b, rb);
    for (int i = 0; i < 2; ++i) {
        const V3 tangent = tangents[i];
        const float k = dot(tangent, mul(pointK, tangent));
        if (k <= 0.0f) continue;
        const float lambda = -(dot(vel, tangent) + dot(error, tangent) * (kBeta / dt)) / k;
        applyLinear(j, a, b, ra, rb, tangent * lambda, 1.0f);
        vel = anchorVelocity(a, ra) - anchorVelocity(b, rb);
    }
    const float kAxis = dot(axisA, mul(pointK, axisA));
    if (kAxis > 0.0f) {
        const float axisSpeed = dot(anchorVelocity(b, rb) - anchorVelocity(a, ra), axisA);
        const float displacement = dot(pb - pa, axisA);
        const float tau = 6.28318530718f;
        const float mass = 1.0f / kAxis;
        const float omega = tau * j.suspensionFrequencyHz;
        const float stiffness = mass * omega * omega;
        const float damping = 2.0f * mass * j.suspensionDampingRatio * omega;
        const float softness = (damping + dt * stiffness) > 1e-10f ? 1.0f / (dt * (damping + dt * stiffness)) : 0.0f;
        const float bias = displacement * dt * stiffness * softness;
        const float lambda = -(axisSpeed + bias + softness * j.springImpulse) / (kAxis + softness);
        j.springImpulse += lambda;
        applyLinear(j, a, b, ra, rb, axisA * lambda, -1.0f);
    }
    V3 relativeW = a.w - b.w;
    for (int i = 0; i < 2; ++i) {
        const V3 tangent = tangents[i];
        const float k = dot(tangent, invI(a, tangent)) + dot(tangent, invI(b, tangent));
        if (k <= 0.0f) continue;
        const V3 refA = rotate(a.q, v3of(j.localRefA));
        const V3 refB = rotate(b.q, v3of(j.localRefB));
        const V3 frameError = cross(refB, refA);
        const float lambda = -(dot(relativeW, tangent) + dot(frameError, tangent) * (kBeta / dt)) / k;
        applyAngular(j, a, b, tangent * lambda);
        relativeW = a.w - b.w;
    }
    if (j.enableSteering) {
        const V3 steerAxis = normalize(rotate(a.q, v3of(j.localRefA)));
        const float kSteer = dot(steerAxis, invI(a, steerAxis)) + dot(steerAxis, invI(b, steerAxis));
        if (kSteer > 0.0f) {
            const V3 refA = rotate(a.q, v3of(j.localRefA));
            const V3 refB = rotate(b.q, v3of(j.localRefB));
            const V3 axle = axisA;
            const V3 pA = normalize(refA - axle * dot(refA, axle));
            const V3 pB = normalize(refB - axle * dot(refB, axle));
            const float currentAngle = atan2f(dot(cross(pA, pB), steerAxis), dot(pA, pB));
            const float angleError = j.steeringAngle - currentAngle;
            const float wSteer = dot(b.w - a.w, steerAxis);
            const float lambda = (wSteer - angleError * (kBeta / dt)) / kSteer;
            applyAngular(j, a, b, steerAxis * lambda);
        }
    }
    if (j.enableMotor) {
        const float kAxle = dot(axisA, invI(a, axisA)) + dot(axisA, invI(b, axisA));
        if (kAxle > 0.0f) {
            const float wAxle = dot(b.w - a.w, axisA);
            float lambda = (wAxle - j.motorSpeed) / kAxle;
            const float maxImpulse = j.maxMotorTorque * dt;
            const float old = j.motorImpulse;
            j.motorImpulse = vclamp(old + lambda, -maxImpulse, maxImpulse);
            lambda = j.motorImpulse - old;
            applyAngular(j, a, b, axisA * lambda);
        }
    }
}

// Maximum distance; slack is free (joint_solver.h:585-607).
VXD void solveRope(vx_joint& j, JBody& a, JBody& b, const V3& ra, const V3& rb, const V3& pa, const V3& pb,
                   float dt) {
    const V3 d = pa - pb;
    const float len = length(d);
    if (len < 1e-8f || len <= j.maxLength) return;
    const V3 n = d * (1.0f / len);
    const V3 velocity = anchorVelocity(a, ra) - anchorVelocity(b, rb);
    const V3 raxn = cross(ra, n), rbxn = cross(rb, n);
    const float k = invMassOf(a) + invMassOf(b) + dot(raxn, invI(a, raxn)) + dot(rbxn, invI(b, rbxn));
    if (k <= 0.0f) return;
    const float overshoot = len - j.maxLength;
    const float bias = overshoot * (kBeta / dt);
    float lambda = -(dot(velocity, n) + bias) / k;
    const float old = j.limitImpulse;
    j.limitImpulse = vmin(0.0f, old + lambda);
    lambda = j.limitImpulse - old;
    applyLinear(j, a, b, ra, rb, n * lambda, 1.0f);
}

// lengthA + ratio * lengthB held at restLength through two fixed pulley
// anchors (joint_solver.h:609-651).
VXD void solvePulley(vx_joint& j, JBody& a, JBody& b, const V3& ra, const V3& rb, const V3& pa, const V3& pb,
                     float dt) {
    const V3 dA = pa - v3of(j.pulleyAnchorA);
    const V3 dB = pb - v3of(j.pulleyAnchorB);
    const float lenA = length(dA);
    const float lenB = length(dB);
    if (lenA < 1e-8f || lenB < 1e-8f) return;
    const V3 nA = dA * (1.0f / lenA);
    const V3 nB = dB * (1.0f / lenB);
    const V3 raxnA = cross(ra, nA);
    const V3 rbxnB = cross(rb, nB);
    const float kA = invMassOf(a) + dot(raxnA, invI(a, raxnA));
    const float kB = invMassOf(b) + dot(rbxnB, invI(b, rbxnB));
    const float ratio = j.pulleyRatio;
    const float k = kA + ratio * ratio * kB;
    if (k <= 0.0f) return;
    const float restTotal = j.restLength;
    const float C = lenA + ratio * lenB - restTotal;
    const float bias = C * (kBeta / dt);
    const float speedA = dot(anchorVelocity(a, ra), nA);
    const float speedB = dot(anchorVelocity(b, rb), nB);
    const float cdot = speedA + ratio * speedB;
    float lambda = -(cdot + bias) / k;
    const float old = j.limitImpulse;
    j.limitImpulse += lambda;
    lambda = j.limitImpulse - old;
    applyImpulse(a, ra, nA * lambda, 1.0f);
    applyImpulse(b, rb, nB * (lambda * ratio), 1.0f);
    addTo(j.reactionLinearImpulse, nA * lambda);
}

// Angular velocities about the two axes coupled at gearRatio
// (joint_solver.h:653-680).
VXD void solveGear(vx_joint& j, JBody& a, JBody& b) {
    const V3 axisA = normalize(rotate(a.q, v3of(j.localAxisA)));
    const V3 axisB = normalize(rotate(b.q, v3of(j.localAxisB)));
    const float ratio = j.gearRatio;
    const float kA = dot(axisA, invI(a, axisA));
    const float kB = dot(axisB, invI(b, axisB));
    const float k = kA + ratio * ratio * kB;
    if (k <= 0.0f) return;
    const float wA = dot(a.w, axisA);
    const float wB = dot(b.w, axisB);
    const float cdot = wA + ratio * wB;
    float lambda = -cdot / k;
    const float old = j.motorImpulse;
    j.motorImpulse += lambda;
    lambda = j.motorImpulse - old;
    if (movable(a)) a.w += invI(a, axisA * lambda);
    if (movable(b)) b.w += invI(b, axisB * (lambda * ratio));
    addTo(j.reactionAngularImpulse, axisA * lambda);
}

// One joint row (joint_solver.h:682-775).
VXD void solve(vx_joint& j, JBody& a, JBody& b, float dt) {
    const V3 ra = rotate(a.q, v3of(j.localAnchorA));
    const V3 rb = rotate(b.q, v3of(j.localAnchorB));
    const V3 pa = a.p + ra;
    const V3 pb = b.p + rb;
    const V3 velocity = anchorVelocity(a, ra) - anchorVelocity(b, rb);
    switch (j.type) {
    case VX_JOINT_BALL:
        applyLinear(j, a, b, ra, rb, pointLockImpulse(a, b, ra, rb, pa, pb, dt), 1.0f);
        break;
    case VX_JOINT_DISTANCE: {
        const V3 d = pa - pb;
        const float len = length(d);
        if (len < 1e-8f) break;
        const V3 n = d * (1.0f / len);
        const V3 raxn = cross(ra, n), rbxn = cross(rb, n);
        const float k = invMassOf(a) + invMassOf(b) + dot(raxn, invI(a, raxn)) + dot(rbxn, invI(b, rbxn));
        if (k <= 0.0f) break;
        float lambda;
        if (j.enableSpring) {
            const float tau = 6.28318530718f;
            const float mass = 1.0f / k;
            const float omega = tau * j.springFrequencyHz;
            const float stiffness = mass * omega * omega;
            const float damping = 2.0f * mass * j.springDampingRatio * omega;
            const float softness = 1.0f / (dt * (damping + dt * stiffness));
            const float bias = (len - j.restLength) * dt * stiffness * softness;
            lambda = -(dot(velocity, n) + bias + softness * j.springImpulse) / (k + softness);
            j.springImpulse += lambda;
        } else {
            const float bias = (len - j.restLength) * (kBeta / dt);
            lambda = -(dot(velocity, n) + bias) / k;
        }
        applyLinear(j, a, b, ra, rb, n * lambda, 1.0f);
        break;
    }
    case VX_JOINT_FIXED:
        applyLinear(j, a, b, ra, rb, pointLockImpulse(a, b, ra, rb, pa, pb, dt), 1.0f);
        solveAngularFrame(j, a, b, kBeta / dt);
        break;
    case VX_JOINT_MOTOR: {
        V3 impulse = pointLockImpulse(a, b, ra, rb, pa, pb, dt);
        const float maxImpulse = j.maxMotorForce * dt;
        const float mag = length(impulse);
        if (mag > maxImpulse && mag > 1e-9f) impulse = impulse * (maxImpulse / mag);
        applyLinear(j, a, b, ra, rb, impulse, 1.0f);
        solveAngularFrame(j, a, b, kBeta / dt);
        break;
    }
    case VX_JOINT_WELD: solveWeld(j, a, b, ra, rb, pa, pb, dt); break;
    case VX_JOINT_WHEEL: solveWheel(j, a, b, ra, rb, pa, pb, dt); break;
    case VX_JOINT_ROPE: solveRope(j, a, b, ra, rb, pa, pb, dt); break;
    case VX_JOINT_PULLEY: solvePulley(j, a, b, ra, rb, pa, pb, dt); break;
    case VX_JOINT_GEAR: solveGear(j, a, b); break;
    case VX_JOINT_SIX_DOF: solveSixDof(j, a, b, ra, rb, pa, pb, dt); break;
    case VX_JOINT_PRISMATIC: solvePrismatic(j, a, b, ra, rb, pa, pb, dt); break;
    case VX_JOINT_HINGE: solveHinge(j, a, b, ra, rb, pa, pb, dt); break;
    case VX_JOINT_CONE_TWIST: solveConeTwist(j, a, b, ra, rb, pa, pb, dt); break;
    default: break;
    }
}

// The device pass handles every type up to the gear joint.
VXD bool supported(const vx_joint& j) { return j.type <= VX_JOINT_GEAR; }

// Break test after a substep's joint sweeps (src/backend_cuda.cu:341-348).
VXD void markBroken(vx_joint& j, float dt) {
    if (j.broken) return;
    const float force = length(v3of(j.reactionLinearImpulse)) / dt;
    const float torque = length(v3of(j.reactionAngularImpulse)) / dt;
    j.broken = (force > j.breakForce || torque > j.breakTorque) ? 1 : 0;
}

}  // namespace joint
}  // namespace vxb
