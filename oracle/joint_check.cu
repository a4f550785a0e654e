// Test infrastructure: the library's joint rows (velox_b200/csrc/joints.cuh,
// compiled here for the host) beside the reference's joint_solver::solve
// (src/joint_solver.h) on the same inputs, so that their parity is checked
// on the CPU. Built by oracle/Makefile into oracle/_ref/; nothing in the
// product links or loads it.
#define VXD __host__ __device__ __forceinline__
#include "vmath.cuh"
#include "joints.cuh"

#include "velox/body.h"
#include "joint_solver.h"

#include <cstring>

static_assert(sizeof(velox::Joint) == sizeof(vx_joint), "Joint layout");
static_assert(sizeof(velox::Body) == sizeof(vx_body), "Body layout");

namespace {

// The packed flags the device keeps for a body (motion type, quality,
// fixed rotation: what the joint rows read).
uint32_t flagsOf(const vx_body& b) {
    return (uint32_t)(b.shape & 15u) | ((uint32_t)(b.motionType & 3u) << vxb::kMotionShift) |
           ((uint32_t)(b.ccdTuning.quality & 3u) << vxb::kQualityShift) |
           (b.fixedRotation ? vxb::kFixedRotationBit : 0u);
}

vxb::joint::JBody jbody(const vx_body& b) {
    vxb::joint::JBody j;
    j.p = vxb::V3{b.position.x, b.position.y, b.position.z};
    j.q = vxb::Q4{b.orientation.x, b.orientation.y, b.orientation.z, b.orientation.w};
    j.v = vxb::V3{b.velocity.x, b.velocity.y, b.velocity.z};
    j.w = vxb::V3{b.angularVelocity.x, b.angularVelocity.y, b.angularVelocity.z};
    j.m.invI = vxb::V3{b.invInertia.x, b.invInertia.y, b.invInertia.z};
    j.m.invMass = b.invMass;
    j.m.iq = vxb::Q4{b.inertiaOrientation.x, b.inertiaOrientation.y, b.inertiaOrientation.z,
                     b.inertiaOrientation.w};
    j.m.flags = flagsOf(b);
    return j;
}

}  // namespace

extern "C" {

// For joint k, bodies[2k] and bodies[2k+1] are its a and b. Runs `sweeps`
// solves of every joint with dt on both implementations; writes each side's
// bodies (velocities changed) and joints (scratch changed).
void joint_check(const vx_body* bodies, const vx_joint* joints, int count, float dt, int sweeps,
                 vx_body* refBodies, vx_joint* refJoints, vx_body* myBodies, vx_joint* myJoints) {
    for (int k = 0; k < count; ++k) {
        velox::Body a, b;
        std::memcpy(&a, &bodies[2 * k], sizeof(a));
        std::memcpy(&b, &bodies[2 * k + 1], sizeof(b));
        velox::Joint j;
        std::memcpy(&j, &joints[k], sizeof(j));
        for (int s = 0; s < sweeps; ++s) velox::joint_solver::solve(j, a, b, dt);
        std::memcpy(&refBodies[2 * k], &a, sizeof(a));
        std::memcpy(&refBodies[2 * k + 1], &b, sizeof(b));
        std::memcpy(&refJoints[k], &j, sizeof(j));

        vxb::joint::JBody ma = jbody(bodies[2 * k]), mb = jbody(bodies[2 * k + 1]);
        vx_joint mj = joints[k];
        for (int s = 0; s < sweeps; ++s) vxb::joint::solve(mj, ma, mb, dt);
        myBodies[2 * k] = bodies[2 * k];
        myBodies[2 * k + 1] = bodies[2 * k + 1];
        myBodies[2 * k].velocity = vx_vec3{ma.v.x, ma.v.y, ma.v.z};
        myBodies[2 * k].angularVelocity = vx_vec3{ma.w.x, ma.w.y, ma.w.z};
        myBodies[2 * k + 1].velocity = vx_vec3{mb.v.x, mb.v.y, mb.v.z};
        myBodies[2 * k + 1].angularVelocity = vx_vec3{mb.w.x, mb.w.y, mb.w.z};
        myJoints[k] = mj;
    }
}

// reset / markBroken of both sides (joint_solver.h reset, backend_cuda.cu:341-348).
void joint_check_reset_break(vx_joint* refJoint, vx_joint* myJoint, float dt, int reset) {
    velox::Joint j;
    std::memcpy(&j, refJoint, sizeof(j));
    if (reset) {
        velox::joint_solver::reset(j);
        vxb::joint::reset(*myJoint);
    } else {
        if (!j.broken) {
            float force = velox::length(j.reactionLinearImpulse) / dt;
            float torque = velox::length(j.reactionAngularImpulse) / dt;
            j.broken = force > j.breakForce || torque > j.breakTorque;
        }
        vxb::joint::markBroken(*myJoint, dt);
    }
    std::memcpy(refJoint, &j, sizeof(j));
}

}  // extern "C"
