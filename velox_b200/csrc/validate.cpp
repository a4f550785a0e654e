// Host-side validation of what enters the device world, following the
// reference's per-step validation of public state (World::stepImpl,
// src/world.cpp:3855-3931; validateRuntimeBody :219-247, validateCcdTuning
// :42-48, validateSolverOptions :69-79). The device world's state changes
// only through vxb_world_load, vxb_world_write_forces and its own steps, so
// validating those inputs once gives every step the reference's guarantees
// without a host round trip per step.
#include <cmath>
#include <string>

#include "velox_b200.h"

namespace vxb {

namespace {

bool fin(float v) { return std::isfinite(v); }
bool fin3(const vx_vec3& v) { return fin(v.x) && fin(v.y) && fin(v.z); }
bool finq(const vx_quat& q) { return fin(q.x) && fin(q.y) && fin(q.z) && fin(q.w); }
bool positive(float v) { return fin(v) && v > 0.0f; }
bool nonNegative(float v) { return fin(v) && v >= 0.0f; }
bool positive3(const vx_vec3& v) { return fin3(v) && v.x > 0.0f && v.y > 0.0f && v.z > 0.0f; }

bool bad(std::string& why, const char* what) {
    why = what;
    return false;
}

}  // namespace

bool convexShape(uint8_t s) {
    return s == VX_SHAPE_SPHERE || s == VX_SHAPE_BOX || s == VX_SHAPE_CAPSULE || s == VX_SHAPE_HULL ||
           s == VX_SHAPE_CYLINDER || s == VX_SHAPE_CONE || s == VX_SHAPE_ROUNDED_BOX || s == VX_SHAPE_ELLIPSOID;
}

// References of a mesh or compound body into the soup (src/world.cpp:3901-3927).
bool validComplexRefs(const vx_body& b, const vx_soup* soup, std::string& why) {
    if (b.shape == VX_SHAPE_MESH) {
        if (!soup || b.meshIndex >= soup->meshCount) return bad(why, "mesh body references an invalid mesh");
    } else if (b.shape == VX_SHAPE_COMPOUND) {
        if (!soup || b.compoundCount == 0 || (size_t)b.compoundFirst + b.compoundCount > soup->compoundChildCount)
            return bad(why, "compound body references invalid child storage");
    }
    return true;
}

// Structure of the soup's meshes, BVHs and compound children, checked once
// when it is loaded so that the device walks stay inside their arrays and
// every BVH descent ends (an inner node's children follow it).
bool validSoup(const vx_soup* soup, std::string& why) {
    if (!soup) return true;
    const vx_soup& s = *soup;
    if ((s.hullPointCount && !s.hullPoints) || (s.hullFaceIndexCount && !s.hullFaceIndices) ||
        (s.vertexCount && !s.vertices) || (s.indexCount && !s.indices) || (s.meshCount && !s.meshes) ||
        (s.bvhNodeCount && !s.bvhNodes) || (s.bvhTriRefCount && !s.bvhTriRefs) ||
        (s.compoundChildCount && !s.compoundChildren))
        return bad(why, "mesh soup has a null array with a non-zero count");
    for (uint32_t k = 0; k < s.meshCount; ++k) {
        const vx_mesh& m = s.meshes[k];
        const size_t tris = m.indexCount / 3;
        if ((size_t)m.firstVertex + m.vertexCount > s.vertexCount || (size_t)m.firstIndex + m.indexCount > s.indexCount ||
            m.indexCount % 3 != 0 || m.nodeCount == 0 || (size_t)m.firstNode + m.nodeCount > s.bvhNodeCount)
            return bad(why, "mesh references invalid vertex, index or node storage");
        for (uint32_t x = 0; x < m.indexCount; ++x)
            if (s.indices[m.firstIndex + x] >= m.vertexCount) return bad(why, "mesh index is outside the vertex array");
        const size_t nodeEnd = (size_t)m.firstNode + m.nodeCount;
        for (size_t v = m.firstNode; v < nodeEnd; ++v) {
            const vx_bvh_node& node = s.bvhNodes[v];
            if (node.triCount == 0) {
                if (node.leftFirst <= v || (size_t)node.leftFirst + 1 >= nodeEnd)
                    return bad(why, "mesh BVH has an invalid inner node");
            } else {
                if ((size_t)node.leftFirst + node.triCount > s.bvhTriRefCount)
                    return bad(why, "mesh BVH leaf references invalid triangle storage");
                for (uint32_t t = 0; t < node.triCount; ++t)
                    if (s.bvhTriRefs[node.leftFirst + t] >= tris)
                        return bad(why, "mesh BVH leaf references an invalid triangle");
            }
        }
    }
    for (uint32_t k = 0; k < s.compoundChildCount; ++k) {
        const vx_compound_child& c = s.compoundChildren[k];
        if (!fin3(c.localPosition) || !finq(c.localOrientation) || !convexShape(c.shape))
            return bad(why, "compound child contains invalid state");
        if (c.shape == VX_SHAPE_HULL) {
            if (c.hullCount == 0 || (size_t)c.hullFirst + c.hullCount > s.hullPointCount ||
                (size_t)c.hullFaceFirst + (size_t)c.hullFaceCount * 3 > s.hullFaceIndexCount)
                return bad(why, "compound child references invalid hull storage");
            for (size_t f = 0; f < (size_t)c.hullFaceCount * 3; ++f)
                if (s.hullFaceIndices[c.hullFaceFirst + f] >= c.hullCount)
                    return bad(why, "compound child references invalid hull storage");
        }
    }
    return true;
}

bool validBody(const vx_body& b, const vx_soup* soup, std::string& why) {
    const size_t hullPoints = soup ? soup->hullPointCount : 0, faceIndices = soup ? soup->hullFaceIndexCount : 0;
    if (!fin3(b.position) || !finq(b.orientation) || !finq(b.inertiaOrientation) || !fin3(b.velocity) ||
        !fin3(b.angularVelocity) || !fin3(b.force) || !fin3(b.torque) || !nonNegative(b.invMass) ||
        !fin3(b.invInertia) || b.invInertia.x < 0.0f || b.invInertia.y < 0.0f || b.invInertia.z < 0.0f ||
        !nonNegative(b.restitution) || !nonNegative(b.friction) || !fin3(b.frictionScale) ||
        b.frictionScale.x < 0.0f || b.frictionScale.y < 0.0f || b.frictionScale.z < 0.0f ||
        !nonNegative(b.rollingFriction) || !nonNegative(b.spinningFriction) ||
        b.frictionCombine > VX_COMBINE_MAXIMUM || b.restitutionCombine > VX_COMBINE_MAXIMUM ||
        !nonNegative(b.linearDamping) || !nonNegative(b.angularDamping) || !fin(b.gravityScale))
        return bad(why, "body contains invalid or non-finite state");
    if (b.ccdTuning.quality > VX_QUALITY_LOCKED || !nonNegative(b.ccdTuning.collisionMargin) ||
        !nonNegative(b.ccdTuning.speculativeDistance) || !nonNegative(b.ccdTuning.minVelocityForCCD))
        return bad(why, "body CCD tuning is invalid");
    const vx_quat& q = b.orientation;
    const float q2 = q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w;
    if (!fin(q2) || q2 < 1e-12f) return bad(why, "body orientation must be a finite non-zero quaternion");
    const vx_quat& iq = b.inertiaOrientation;
    const float iq2 = iq.x * iq.x + iq.y * iq.y + iq.z * iq.z + iq.w * iq.w;
    if (!fin(iq2) || iq2 < 1e-12f) return bad(why, "inertia orientation must be a finite non-zero quaternion");
    switch (b.shape) {
    case VX_SHAPE_SPHERE:
        if (!positive(b.radius)) return bad(why, "sphere body has an invalid radius");
        break;
    case VX_SHAPE_BOX:
        if (!positive3(b.halfExtents)) return bad(why, "box body has invalid half extents");
        break;
    case VX_SHAPE_CAPSULE:
        if (!positive(b.radius)) return bad(why, "capsule body has an invalid radius");
        if (!nonNegative(b.capsuleHalfHeight)) return bad(why, "capsule body has an invalid half height");
        break;
    case VX_SHAPE_CYLINDER:
    case VX_SHAPE_CONE:
        if (!positive(b.radius) || !positive(b.capsuleHalfHeight))
            return bad(why, "cylinder or cone body has an invalid radius or half height");
        break;
    case VX_SHAPE_ROUNDED_BOX:
        if (!positive3(b.halfExtents) || !positive(b.radius))
            return bad(why, "rounded box body has invalid half extents or radius");
        break;
    case VX_SHAPE_ELLIPSOID:
        if (!positive3(b.halfExtents)) return bad(why, "ellipsoid body has invalid radii");
        break;
    case VX_SHAPE_PLANE: {
        const vx_vec3& n = b.planeNormal;
        if (!fin3(n) || n.x * n.x + n.y * n.y + n.z * n.z < 1e-12f || !fin(b.planeOffset))
            return bad(why, "plane body has invalid geometry");
        break;
    }
    case VX_SHAPE_HULL:
        if (b.hullCount < 4 || (size_t)b.hullFirst + b.hullCount > hullPoints || b.hullFaceCount == 0 ||
            (size_t)b.hullFaceFirst + (size_t)b.hullFaceCount * 3 > faceIndices)
            return bad(why, "hull body references invalid point storage");
        break;
    case VX_SHAPE_MESH:
    case VX_SHAPE_COMPOUND:
        if (!validComplexRefs(b, soup, why)) return false;
        break;
    default:
        return bad(why, "body has an unknown shape");
    }
    return true;
}

bool validSolverOptions(const vx_solver_options& o, std::string& why) {
    if ((o.frictionModel != VX_FRICTION_TWO_AXIS && o.frictionModel != VX_FRICTION_CONE_BLOCK) ||
        o.iterationPolicy > 1 || o.velocityIterations <= 0 || o.positionIterations <= 0 ||
        !positive(o.impulseThreshold) || !nonNegative(o.stackStiffness) || !nonNegative(o.stackDamping))
        return bad(why, "solver options are invalid");
    return true;
}

bool finiteValues(const float* v, size_t count) {
    for (size_t k = 0; k < count; ++k)
        if (!std::isfinite(v[k])) return false;
    return true;
}

}  // namespace vxb
