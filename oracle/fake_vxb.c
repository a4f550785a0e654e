/*
 * Test infrastructure (not the product): a fake of libvelox_b200.so's Backend
 * entry points (include/velox_b200.h) that needs no GPU. Linked with the
 * reference engine and velox_b200/dropin/b200_backend.cpp into
 * oracle/_ref/libvelox_ref_dropin_fake.so, it lets CPU tests drive the
 * adapter's status-to-exception mapping and the reference World's CPU retry
 * (src/world.cpp:3807-3828) through real reference code.
 *
 * vxb_backend_integrate returns the status in the environment variable
 * VXB_FAKE_STATUS (0 when unset) and touches nothing; every other entry point
 * fails with VXB_ERR_INVALID, so a test that reaches them notices.
 */
#include <stdlib.h>
#include <string.h>

#include "velox_b200.h"

struct vxb_context {
    char message[128];
};

static struct vxb_context g_fake;

const char* vxb_status_string(int status) {
    switch (status) {
    case VXB_OK: return "ok";
    case VXB_ERR_OOM: return "device memory allocation failed";
    case VXB_ERR_DEVICE_LOST: return "device lost";
    case VXB_ERR_CAPACITY: return "caller buffer too small";
    case VXB_ERR_TIMEOUT: return "bounded device wait timed out";
    case VXB_ERR_INTERNAL: return "device-side consistency check failed";
    default: return "fake status";
    }
}

int vxb_context_create(int device, vxb_context** out) {
    (void)device;
    strcpy(g_fake.message, "fake backend");
    *out = &g_fake;
    return VXB_OK;
}

void vxb_context_destroy(vxb_context* ctx) { (void)ctx; }

const char* vxb_context_last_error(const vxb_context* ctx) { return ctx->message; }

int vxb_backend_integrate(vxb_context* ctx, vx_body* bodies, uint32_t n, vx_vec3 gravity, float dt) {
    (void)ctx; (void)bodies; (void)n; (void)gravity; (void)dt;
    const char* s = getenv("VXB_FAKE_STATUS");
    return s ? atoi(s) : VXB_OK;
}

int vxb_backend_find_contacts(vxb_context* ctx, const vx_body* bodies, uint32_t n, const vx_soup* soup, float dt,
                              uint32_t* count) {
    (void)ctx; (void)bodies; (void)n; (void)soup; (void)dt; (void)count;
    return VXB_ERR_INVALID;
}

int vxb_backend_copy_contacts(vxb_context* ctx, vx_contact* out, uint32_t cap) {
    (void)ctx; (void)out; (void)cap;
    return VXB_ERR_INVALID;
}

int vxb_backend_solve_velocities(vxb_context* ctx, vx_body* bodies, uint32_t n, vx_contact* contacts, uint32_t m,
                                 float dt, int warmStart, const vx_solver_options* options, uint32_t* iterations) {
    (void)ctx; (void)bodies; (void)n; (void)contacts; (void)m; (void)dt; (void)warmStart; (void)options;
    (void)iterations;
    return VXB_ERR_INVALID;
}

int vxb_backend_advance_substeps(vxb_context* ctx, vx_body* bodies, uint32_t n, vx_contact* contacts, uint32_t m,
                                 vx_vec3 gravity, float h, int substeps, const vx_solver_options* options,
                                 int* advanced, uint32_t* iterations) {
    (void)ctx; (void)bodies; (void)n; (void)contacts; (void)m; (void)gravity; (void)h; (void)substeps;
    (void)options; (void)advanced; (void)iterations;
    return VXB_ERR_INVALID;
}

int vxb_backend_advance_substeps_joints(vxb_context* ctx, vx_body* bodies, uint32_t n, vx_contact* contacts,
                                        uint32_t m, vx_joint* joints, uint32_t njoints, vx_vec3 gravity, float h,
                                        int substeps, const vx_solver_options* options, int* advanced,
                                        uint32_t* iterations) {
    (void)ctx; (void)bodies; (void)n; (void)contacts; (void)m; (void)joints; (void)njoints; (void)gravity; (void)h;
    (void)substeps; (void)options; (void)advanced; (void)iterations;
    return VXB_ERR_INVALID;
}

int vxb_backend_fetch_impulses(vxb_context* ctx, vx_contact* contacts, uint32_t m) {
    (void)ctx; (void)contacts; (void)m;
    return VXB_ERR_INVALID;
}

int vxb_backend_invalidate(vxb_context* ctx) {
    (void)ctx;
    return VXB_OK;
}
