/*
 * velox_b200_types.h — plain-C data layouts shared by the B200 contact
 * pipeline's C ABI, its CPU oracle and its tests.
 *
 * The records are byte-compatible with the reference engine's host arrays so
 * a `std::vector<velox::Body>` / `std::vector<velox::Contact>` can be handed
 * across the ABI as a raw pointer without repacking:
 *
 *   vx_body     <-> velox::Body     include/velox/body.h:128-345   (320 B, align 64)
 *   vx_contact  <-> velox::Contact  include/velox/backend.h:63-83  (128 B, align 64)
 *   vx_solver_options <-> velox::SolverOptions include/velox/solver.h:23-35 (24 B)
 *   vx_ccd_tuning <-> velox::BodyCcdTuning include/velox/ccd.h:89-96 (52 B)
 *
 * Field order, widths and padding follow the reference exactly (the offsets
 * are asserted at compile time below and against the reference headers by
 * the reference-side adapter).
 */
#ifndef VELOX_B200_TYPES_H
#define VELOX_B200_TYPES_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VX_ALIGN64 __attribute__((aligned(64)))

typedef struct vx_vec3 { float x, y, z; } vx_vec3;
typedef struct vx_quat { float x, y, z, w; } vx_quat;

/* velox::ShapeType (include/velox/body.h:59-62) */
enum {
    VX_SHAPE_SPHERE = 0, VX_SHAPE_PLANE = 1, VX_SHAPE_BOX = 2, VX_SHAPE_CAPSULE = 3,
    VX_SHAPE_MESH = 4, VX_SHAPE_HULL = 5, VX_SHAPE_COMPOUND = 6, VX_SHAPE_CYLINDER = 7,
    VX_SHAPE_CONE = 8, VX_SHAPE_ROUNDED_BOX = 9, VX_SHAPE_ELLIPSOID = 10
};
/* velox::MotionType (body.h:65-69) */
enum { VX_MOTION_STATIC = 0, VX_MOTION_KINEMATIC = 1, VX_MOTION_DYNAMIC = 2 };
/* velox::MotionQuality (ccd.h) */
enum { VX_QUALITY_LOW = 0, VX_QUALITY_MEDIUM = 1, VX_QUALITY_HIGH = 2, VX_QUALITY_LOCKED = 3 };
/* velox::GeometryQuality (body.h:77) */
enum { VX_GEOM_NORMAL = 0, VX_GEOM_ROBUST = 1, VX_GEOM_PARANOID = 2 };
/* velox::MaterialCombineMode (body.h:84-86) */
enum { VX_COMBINE_AVERAGE = 0, VX_COMBINE_GEOMETRIC_MEAN = 1, VX_COMBINE_MINIMUM = 2,
       VX_COMBINE_MULTIPLY = 3, VX_COMBINE_MAXIMUM = 4 };
/* velox::FrictionModel (solver.h:11-14) */
enum { VX_FRICTION_TWO_AXIS = 0, VX_FRICTION_CONE_BLOCK = 1 };

typedef struct vx_ccd_settings {
    uint8_t quality;
    uint8_t pad0[3];
    uint32_t maxAdvancementIterations;
    uint32_t maxRootFindIterations;
    float distanceTolerance;
    float timeTolerance;
    uint8_t enableRotationalCcd;
    uint8_t enableCompoundCcd;
    uint8_t useBrentRootFinder;
    uint8_t pad1;
    uint32_t meshBvhMaxDepth;
    float speculativeMargin;
} vx_ccd_settings;

typedef struct vx_ccd_tuning {
    uint8_t quality;
    uint8_t pad0[3];
    float collisionMargin;
    float speculativeDistance;
    uint8_t enableContinuous;
    uint8_t pad1[3];
    float minVelocityForCCD;
    vx_ccd_settings ccdSettings;
} vx_ccd_tuning;

typedef struct VX_ALIGN64 vx_body {
    vx_vec3 position;
    vx_quat orientation;
    vx_vec3 velocity;
    vx_vec3 angularVelocity;
    vx_vec3 force;
    vx_vec3 torque;
    float invMass;
    vx_vec3 invInertia;
    vx_quat inertiaOrientation;
    float restitution;
    float friction;
    vx_vec3 frictionScale;
    float rollingFriction;
    float spinningFriction;
    uint8_t frictionCombine;
    uint8_t restitutionCombine;
    uint8_t pad0[2];
    float linearDamping;
    float angularDamping;
    float gravityScale;
    uint8_t motionType;
    uint8_t pad1[3];
    vx_ccd_tuning ccdTuning;
    uint8_t geometryQuality;
    uint8_t pad2[3];
    uint32_t categoryBits;
    uint32_t maskBits;
    int32_t groupIndex;
    uint8_t sensor;
    uint8_t enableSleep;
    uint8_t fixedRotation;
    uint8_t asleep;
    float sleepTimer;
    uint8_t shape;
    uint8_t pad3[3];
    float radius;
    vx_vec3 halfExtents;
    float capsuleHalfHeight;
    vx_vec3 planeNormal;
    float planeOffset;
    uint32_t meshIndex;
    uint32_t hullFirst, hullCount;
    uint32_t hullFaceFirst, hullFaceCount;
    uint32_t compoundFirst, compoundCount;
} vx_body;

typedef struct VX_ALIGN64 vx_contact {
    uint32_t a, b;
    uint64_t featureKey;
    vx_vec3 normal;        /* from b towards a */
    vx_vec3 point;
    vx_vec3 localAnchorA;
    vx_vec3 localAnchorB;
    float gap;
    float bias0;
    float vn0;
    float restitution;
    float friction1, friction2;
    float rollingFriction, spinningFriction;
    float normalImpulse;
    float tangentImpulse1;
    float tangentImpulse2;
    float rollingImpulse1, rollingImpulse2;
    float spinningImpulse;
} vx_contact;

typedef struct vx_solver_options {
    float impulseThreshold;
    float stackStiffness;
    float stackDamping;
    int32_t velocityIterations;
    int32_t positionIterations;
    uint8_t frictionModel;
    uint8_t iterationPolicy;
    uint8_t enableStackStabilization;
    uint8_t reserved;
} vx_solver_options;

/* velox::Mesh (include/velox/body.h:354-362, 52 B): one static triangle mesh
 * in the soup. Vertices [firstVertex, +vertexCount), index triples
 * [firstIndex, +indexCount) relative to firstVertex, BVH nodes
 * [firstNode, +nodeCount) (absolute node indices; the root is firstNode),
 * leaf triangle references from firstTriRef; aabb = root bounds. */
typedef struct vx_mesh {
    uint32_t firstVertex, vertexCount;
    uint32_t firstIndex, indexCount;
    uint32_t firstNode, nodeCount;
    uint32_t firstTriRef;
    vx_vec3 aabbMin, aabbMax;
} vx_mesh;

/* velox::BvhNode (body.h:370-374, 32 B). Inner node: triCount 0, children
 * leftFirst and leftFirst + 1 (absolute node indices). Leaf: triCount > 0
 * triangle references at bvhTriRefs[leftFirst ...], each a triangle number
 * within its mesh. */
typedef struct vx_bvh_node {
    vx_vec3 aabbMin, aabbMax;
    uint32_t leftFirst;
    uint32_t triCount;
} vx_bvh_node;

/* velox::CompoundChild (body.h:105-114, 68 B): one convex child of a
 * compound body, posed in the compound's frame (position relative to the
 * compound's centre of mass). Hull children index the soup's hull arrays. */
typedef struct vx_compound_child {
    uint8_t shape;        /* a convex VX_SHAPE_* */
    uint8_t pad[3];
    vx_vec3 localPosition;
    vx_quat localOrientation;
    float radius;
    vx_vec3 halfExtents;
    float capsuleHalfHeight;
    uint32_t hullFirst, hullCount;
    uint32_t hullFaceFirst, hullFaceCount;
} vx_compound_child;

/* Static geometry of a scene: velox::MeshSoup (include/velox/backend.h:13-22).
 * Hull bodies index hullPoints through hullFirst/hullCount and
 * hullFaceIndices through hullFaceFirst/hullFaceCount (triangles, three point
 * indices each, local to the body's point range). Mesh bodies index meshes
 * through meshIndex; compound bodies index compoundChildren through
 * compoundFirst/compoundCount. A caller without meshes or compounds leaves
 * the fields after hullFaceIndexCount zero. */
typedef struct vx_soup {
    const vx_vec3* hullPoints;
    uint32_t hullPointCount;
    const uint32_t* hullFaceIndices;
    uint32_t hullFaceIndexCount;
    const vx_vec3* vertices;
    uint32_t vertexCount;
    const uint32_t* indices;
    uint32_t indexCount;
    const vx_mesh* meshes;
    uint32_t meshCount;
    const vx_bvh_node* bvhNodes;
    uint32_t bvhNodeCount;
    const uint32_t* bvhTriRefs;
    uint32_t bvhTriRefCount;
    const vx_compound_child* compoundChildren;
    uint32_t compoundChildCount;
} vx_soup;

/* velox::JointType (include/velox/joint.h:46-60) */
enum {
    VX_JOINT_BALL = 0, VX_JOINT_DISTANCE = 1, VX_JOINT_HINGE = 2, VX_JOINT_CONE_TWIST = 3,
    VX_JOINT_FIXED = 4, VX_JOINT_PRISMATIC = 5, VX_JOINT_SIX_DOF = 6, VX_JOINT_MOTOR = 7,
    VX_JOINT_WELD = 8, VX_JOINT_WHEEL = 9, VX_JOINT_ROPE = 10, VX_JOINT_PULLEY = 11,
    VX_JOINT_GEAR = 12
};

/* velox::Joint (include/velox/joint.h:92-188): a two-body constraint with
 * its configuration and the solver's per-substep scratch (the impulses after
 * gearRatio, reset every substep) and the broken flag. a, b are dense body
 * indices. Byte-identical to the reference record (asserted by the
 * reference-side adapter). */
typedef struct vx_joint {
    uint8_t type;
    uint8_t pad0[3];
    uint32_t a, b;
    vx_vec3 localAnchorA, localAnchorB;
    vx_vec3 localAxisA, localAxisB;
    vx_vec3 localRefA, localRefB;
    float restLength;
    uint8_t collideConnected;
    uint8_t enableSpring;
    uint8_t pad1[2];
    float springFrequencyHz, springDampingRatio;
    float breakForce, breakTorque;
    uint8_t enableMotor;
    uint8_t pad2[3];
    float motorSpeed, maxMotorTorque, maxMotorForce;
    uint8_t enableLimit;
    uint8_t pad3[3];
    float lowerLimit, upperLimit;
    uint8_t enableSwingLimit;
    uint8_t pad4[3];
    float swingLimit;
    uint8_t enableTwistLimit;
    uint8_t pad5[3];
    float lowerTwistLimit, upperTwistLimit;
    uint8_t linearLimitMask, angularLimitMask, linearMotorMask, angularMotorMask;
    vx_vec3 lowerLinearLimit, upperLinearLimit;
    vx_vec3 lowerAngularLimit, upperAngularLimit;
    vx_vec3 linearMotorSpeed, angularMotorSpeed;
    vx_vec3 maxLinearMotorForce, maxAngularMotorTorque;
    float weldFrequencyHz, weldDampingRatio;
    float suspensionFrequencyHz, suspensionDampingRatio, wheelRadius;
    uint8_t enableSteering;
    uint8_t pad6[3];
    float steeringAngle, maxSteeringAngle;
    float maxLength;
    vx_vec3 pulleyAnchorA, pulleyAnchorB;
    float pulleyRatio;
    float gearRatio;
    float motorImpulse, limitImpulse, swingImpulse, twistImpulse, springImpulse;
    vx_vec3 linearMotorImpulse, angularMotorImpulse;
    vx_vec3 linearLimitImpulse, angularLimitImpulse;
    vx_vec3 reactionLinearImpulse, reactionAngularImpulse;
    uint8_t broken;
    uint8_t pad7[3];
} vx_joint;

/* One body of a synthetic scene, described at the level of the reference's
 * World::add* calls (include/velox/world.h:459-470: addSphere, addBox,
 * addCapsule, addCylinder, addConvexHull, addStaticPlane). Mass properties,
 * hull topology and centring are derived from it by whichever engine builds
 * the scene, so the same spec list drives the reference and this library. */
typedef struct vx_shape_spec {
    uint8_t shape;         /* VX_SHAPE_SPHERE/BOX/CAPSULE/CYLINDER/HULL/PLANE */
    uint8_t enableSleep;   /* copied into Body::enableSleep */
    uint8_t pad[2];
    uint32_t world;        /* batch world id; 0 for single-world scenes */
    float mass;            /* > 0 dynamic, 0 static */
    float radius;          /* sphere / capsule / cylinder radius */
    float halfHeight;      /* capsule / cylinder half height */
    vx_vec3 halfExtents;   /* box half extents */
    vx_vec3 position;      /* requested position (hulls: before centring) */
    vx_quat orientation;
    vx_vec3 velocity;
    vx_vec3 angularVelocity;
    float friction;
    float restitution;
    vx_vec3 planeNormal;   /* planes only */
    float planeOffset;     /* planes only */
    uint32_t hullFirst;    /* hulls: first raw point in the scene's point pool */
    uint32_t hullCount;    /* hulls: number of raw points */
} vx_shape_spec;

#ifdef __cplusplus
}  /* extern "C" */
#define VX_STATIC_ASSERT(c, m) static_assert(c, m)
#else
#define VX_STATIC_ASSERT(c, m) _Static_assert(c, m)
#endif

VX_STATIC_ASSERT(sizeof(vx_ccd_settings) == 32, "vx_ccd_settings layout");
VX_STATIC_ASSERT(sizeof(vx_ccd_tuning) == 52, "vx_ccd_tuning layout");
VX_STATIC_ASSERT(sizeof(vx_body) == 320, "vx_body must match velox::Body (320 B)");
VX_STATIC_ASSERT(offsetof(vx_body, ccdTuning) == 156, "vx_body.ccdTuning offset");
VX_STATIC_ASSERT(offsetof(vx_body, shape) == 232, "vx_body.shape offset");
VX_STATIC_ASSERT(offsetof(vx_body, compoundCount) == 296, "vx_body.compoundCount offset");
VX_STATIC_ASSERT(sizeof(vx_contact) == 128, "vx_contact must match velox::Contact (128 B)");
VX_STATIC_ASSERT(offsetof(vx_contact, normalImpulse) == 96, "vx_contact.normalImpulse offset");
VX_STATIC_ASSERT(sizeof(vx_solver_options) == 24, "vx_solver_options layout");
VX_STATIC_ASSERT(sizeof(vx_mesh) == 52, "vx_mesh must match velox::Mesh (52 B)");
VX_STATIC_ASSERT(sizeof(vx_bvh_node) == 32, "vx_bvh_node must match velox::BvhNode (32 B)");
VX_STATIC_ASSERT(sizeof(vx_compound_child) == 68, "vx_compound_child must match velox::CompoundChild (68 B)");
VX_STATIC_ASSERT(offsetof(vx_compound_child, hullFaceCount) == 64, "vx_compound_child.hullFaceCount offset");
VX_STATIC_ASSERT(offsetof(vx_joint, gearRatio) == 320, "vx_joint.gearRatio offset");
VX_STATIC_ASSERT(sizeof(vx_joint) == 420, "vx_joint must match velox::Joint (420 B)");

#endif /* VELOX_B200_TYPES_H */
