// Reference-side drop-in: a velox::Backend (include/velox/backend.h:111-172)
// served by libvelox_b200.so through its C ABI. A maintainer adds this file
// to the reference engine in place of src/backend_cuda.cu and links
// libvelox_b200.so; World(BackendType::Cuda | Auto) and
// velox_World_Create(VELOX_BACKEND_CUDA) then run the B200 pipeline.
//
// Status codes map onto the reference's error model (src/backend_cuda.cu:24-40):
// out-of-memory -> BackendFailure(MemoryAllocation); device lost or a timed
// out device wait -> BackendFailure(DeviceLost), which World::step turns into
// a CPU retry of the frame (src/world.cpp:3807-3828); a caller buffer too
// small -> VeloxCapacityExceeded(ContactCountOverflow); anything else ->
// VeloxRuntimeError(BackendUnavailable).
#include "velox/backend.h"
#include "velox/error.h"

#include <cstddef>
#include <cstring>
#include <string>
#include <vector>

#include "velox_b200.h"

static_assert(sizeof(velox::Body) == sizeof(vx_body), "velox::Body and vx_body must share one layout");
static_assert(sizeof(velox::Contact) == sizeof(vx_contact), "velox::Contact and vx_contact must share one layout");
static_assert(sizeof(velox::SolverOptions) == sizeof(vx_solver_options), "SolverOptions layout");
static_assert(sizeof(velox::Mesh) == sizeof(vx_mesh), "Mesh layout");
static_assert(sizeof(velox::Joint) == sizeof(vx_joint), "Joint layout");
static_assert(offsetof(velox::Joint, gearRatio) == offsetof(vx_joint, gearRatio), "Joint.gearRatio");
static_assert(offsetof(velox::Joint, broken) == offsetof(vx_joint, broken), "Joint tail");
static_assert(sizeof(velox::BvhNode) == sizeof(vx_bvh_node), "BvhNode layout");
static_assert(sizeof(velox::CompoundChild) == sizeof(vx_compound_child), "CompoundChild layout");
static_assert(offsetof(velox::CompoundChild, hullFaceCount) == offsetof(vx_compound_child, hullFaceCount),
              "CompoundChild tail");

namespace velox {
namespace {

class B200Backend final : public Backend {
public:
    explicit B200Backend(vxb_context* ctx) : ctx_(ctx) {}
    ~B200Backend() override { vxb_context_destroy(ctx_); }

    const char* name() const override { return "cuda"; }
    uint32_t lastVelocityIterations() const override { return lastIterations_; }

    void integrate(std::vector<Body>& bodies, const Vec3& gravity, float dt) override {
        check(vxb_backend_integrate(ctx_, asBodies(bodies), (uint32_t)bodies.size(), vec(gravity), dt));
    }

    void findContacts(const std::vector<Body>& bodies, const MeshSoup& meshes, float dt,
                      const std::vector<uint64_t>* /*hostPairs: the broad phase runs on the device*/,
                      std::vector<Contact>& out) override {
        out.clear();
        vx_soup soup{reinterpret_cast<const vx_vec3*>(meshes.hullPoints.data()),
                     (uint32_t)meshes.hullPoints.size(),
                     meshes.hullFaceIndices.data(),
                     (uint32_t)meshes.hullFaceIndices.size(),
                     reinterpret_cast<const vx_vec3*>(meshes.vertices.data()),
                     (uint32_t)meshes.vertices.size(),
                     meshes.indices.data(),
                     (uint32_t)meshes.indices.size(),
                     reinterpret_cast<const vx_mesh*>(meshes.meshes.data()),
                     (uint32_t)meshes.meshes.size(),
                     reinterpret_cast<const vx_bvh_node*>(meshes.bvhNodes.data()),
                     (uint32_t)meshes.bvhNodes.size(),
                     meshes.bvhTriRefs.data(),
                     (uint32_t)meshes.bvhTriRefs.size(),
                     reinterpret_cast<const vx_compound_child*>(meshes.compoundChildren.data()),
                     (uint32_t)meshes.compoundChildren.size()};
        uint32_t count = 0;
        check(vxb_backend_find_contacts(ctx_, reinterpret_cast<const vx_body*>(bodies.data()),
                                        (uint32_t)bodies.size(), &soup, dt, &count));
        out.resize(count);
        if (count) check(vxb_backend_copy_contacts(ctx_, asContacts(out), count));
    }

    void solveVelocities(std::vector<Body>& bodies, std::vector<Contact>& contacts, float dt, bool warmStart,
                         const SolverOptions& options) override {
        vx_solver_options o;
        std::memcpy(&o, &options, sizeof(o));
        check(vxb_backend_solve_velocities(ctx_, asBodies(bodies), (uint32_t)bodies.size(), asContacts(contacts),
                                           (uint32_t)contacts.size(), dt, warmStart ? 1 : 0, &o, &lastIterations_));
    }

    bool advanceSubsteps(std::vector<Body>& bodies, std::vector<Contact>& contacts, std::vector<Joint>& joints,
                         const Vec3& gravity, float h, int substeps, const SolverOptions& options) override {
        vx_solver_options o;
        std::memcpy(&o, &options, sizeof(o));
        int advanced = 0;
        check(vxb_backend_advance_substeps_joints(
            ctx_, asBodies(bodies), (uint32_t)bodies.size(), asContacts(contacts), (uint32_t)contacts.size(),
            reinterpret_cast<vx_joint*>(joints.data()), (uint32_t)joints.size(), vec(gravity), h, substeps, &o,
            &advanced, &lastIterations_));
        return advanced != 0;
    }

    void fetchImpulses(std::vector<Contact>& contacts) override {
        check(vxb_backend_fetch_impulses(ctx_, asContacts(contacts), (uint32_t)contacts.size()));
    }

    void invalidateCaches() override { check(vxb_backend_invalidate(ctx_)); }

private:
    static vx_body* asBodies(std::vector<Body>& b) { return reinterpret_cast<vx_body*>(b.data()); }
    static vx_contact* asContacts(std::vector<Contact>& c) { return reinterpret_cast<vx_contact*>(c.data()); }
    static vx_vec3 vec(const Vec3& v) { return vx_vec3{v.x, v.y, v.z}; }

    void check(int status) {
        if (status == VXB_OK) return;
        std::string message = std::string("velox_b200: ") + vxb_status_string(status) + ": " +
                              vxb_context_last_error(ctx_);
        switch (status) {
        case VXB_ERR_OOM: throw BackendFailure(BackendFailureKind::MemoryAllocation, message);
        case VXB_ERR_DEVICE_LOST:
        case VXB_ERR_TIMEOUT: throw BackendFailure(BackendFailureKind::DeviceLost, message);
        case VXB_ERR_CAPACITY: VELOX_THROW(VeloxCapacityExceeded, ErrorCode::ContactCountOverflow, message);
        default: VELOX_THROW(VeloxRuntimeError, ErrorCode::BackendUnavailable, message);
        }
    }

    vxb_context* ctx_;
    uint32_t lastIterations_ = 0;
};

}  // namespace

// Replaces the factory of src/backend_cuda.cu:1020: nullptr when no device.
Backend* createCudaBackend() {
    vxb_context* ctx = nullptr;
    if (vxb_context_create(0, &ctx) != VXB_OK) return nullptr;
    return new B200Backend(ctx);
}

}  // namespace velox
