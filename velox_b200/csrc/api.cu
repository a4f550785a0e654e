// extern "C" entry points (include/velox_b200.h). Every function validates
// its arguments, never throws, and maps failures to status codes.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>

#include "context.cuh"

using vxb::Context;

struct vxb_context {
    Context impl;
};

namespace {

int guardContext(vxb_context* ctx) {
    if (!ctx) return VXB_ERR_INVALID;
    cudaError_t e = cudaSetDevice(ctx->impl.device);
    if (e != cudaSuccess) return vxb::cudaStatus(ctx->impl, e, "cudaSetDevice");
    return VXB_OK;
}

#define GUARD(ctx)                          \
    do {                                    \
        int g_ = guardContext(ctx);         \
        if (g_ != VXB_OK) return g_;        \
    } while (0)

#define TRY(expr)                          \
    do {                                   \
        int s_ = (expr);                   \
        if (s_ != VXB_OK) return s_;       \
    } while (0)

// Failure injection for tests, read on every Backend::integrate call (the
// first backend call of each World::step) like the reference's
// injectCudaFailureForTesting (src/backend_cuda.cu:69-78, :394):
// VELOX_CUDA_TEST_FAIL=oom reports an allocation failure, =device-loss a lost
// device, before any device work. Nothing on the device is touched.
int injectedFailure(Context& c) {
    const char* mode = std::getenv("VELOX_CUDA_TEST_FAIL");
    if (!mode || mode[0] == '\0') return VXB_OK;
    if (std::strcmp(mode, "oom") == 0)
        return vxb::fail(c, VXB_ERR_OOM, "test injection: allocation failure");
    if (std::strcmp(mode, "device-loss") == 0)
        return vxb::fail(c, VXB_ERR_DEVICE_LOST, "test injection: device loss");
    return VXB_OK;
}

int ensureCounters(Context& c) {
    TRY(vxb::ensure(c, c.countersBuf, sizeof(vxb::Counters)));
    c.dCounters = reinterpret_cast<vxb::Counters*>(c.countersBuf.ptr);
    return VXB_OK;
}

}  // namespace

extern "C" {

const char* vxb_version(void) { return "velox_b200 0.1 (sm_100a)"; }

const char* vxb_status_string(int status) {
    switch (status) {
    case VXB_OK: return "ok";
    case VXB_ERR_INVALID: return "invalid argument or state";
    case VXB_ERR_NO_DEVICE: return "no CUDA device";
    case VXB_ERR_OOM: return "device memory allocation failed";
    case VXB_ERR_DEVICE_LOST: return "device lost";
    case VXB_ERR_CAPACITY: return "caller buffer too small";
    case VXB_ERR_UNSUPPORTED: return "unsupported input";
    case VXB_ERR_TIMEOUT: return "bounded device wait timed out";
    case VXB_ERR_INTERNAL: return "device-side consistency check failed";
    default: return "unknown status";
    }
}

int vxb_context_create(int device, vxb_context** out) {
    if (!out) return VXB_ERR_INVALID;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return VXB_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= count) return VXB_ERR_INVALID;
    if (cudaSetDevice(device) != cudaSuccess) return VXB_ERR_NO_DEVICE;
    auto* ctx = new (std::nothrow) vxb_context();
    if (!ctx) return VXB_ERR_OOM;
    Context& c = ctx->impl;
    c.device = device;
    vxb::sleepConfigDefault(&c.sleep.config);
    if (const char* limit = std::getenv("VXB_WAIT_LIMIT")) {  // polls; 0 or unset = the default
        const unsigned long v = std::strtoul(limit, nullptr, 10);
        if (v > 0 && v <= vxb::kSpinLimit) c.waitLimit = (uint32_t)v;
    }
    cudaDeviceGetAttribute(&c.smCount, cudaDevAttrMultiProcessorCount, device);
    cudaDeviceGetAttribute(&c.cooperative, cudaDevAttrCooperativeLaunch, device);
    if (cudaStreamCreateWithFlags(&c.ownStream, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        return VXB_ERR_DEVICE_LOST;
    }
    c.stream = c.ownStream;
    if (ensureCounters(c) != VXB_OK) {
        cudaStreamDestroy(c.ownStream);
        delete ctx;
        return VXB_ERR_OOM;
    }
    c.tuner.init(device, c.smCount);
    *out = ctx;
    return VXB_OK;
}

void vxb_context_destroy(vxb_context* ctx) {
    if (!ctx) return;
    Context& c = ctx->impl;
    cudaSetDevice(c.device);
    if (c.stream) cudaStreamSynchronize(c.stream);
    c.tuner.release();  // after the drain: its last samples have completed
    vxb::tapeEnd(c);
    for (auto& snap : c.snapshots)
        if (snap.buf.ptr) cudaFree(snap.buf.ptr);
    vxb::DevBuf* bufs[] = {&c.bodyBuf, &c.aosBuf, &c.worldOfBuf, &c.planeStartBuf, &c.planeListBuf, &c.prevPoseBuf,
                           &c.snapBuf, &c.hullPtsBuf, &c.facesBuf, &c.vertBuf, &c.indexBuf, &c.meshBuf, &c.nodeBuf,
                           &c.triRefBuf, &c.childBuf, &c.jointBuf, &c.aabbBuf, &c.cellKeyBuf, &c.cellValBuf,
                           &c.sortKeysAlt, &c.sortValsAlt, &c.sortHist, &c.hashKeyBuf, &c.hashValBuf, &c.pairBuf,
                           &c.contactTmpBuf, &c.recKeyBuf, &c.recValBuf, &c.recInfoBuf, &c.recCountBuf,
                           &c.contactBuf[0], &c.contactBuf[1], &c.prevKeyBuf, &c.pairKeyBuf, &c.recOffsetBuf,
                           &c.parentBuf, &c.islandOfBodyBuf, &c.islandKeyBuf, &c.islandValBuf, &c.colorBuf,
                           &c.colorKeyBuf, &c.maskBuf, &c.nextColorBuf, &c.islandStartBuf, &c.islandInfoBuf,
                           &c.flagBuf, &c.scanBuf, &c.scanTmp, &c.segStartBuf, &c.islandSegBuf, &c.bodyKeyBuf,
                           &c.bodyValBuf, &c.islandBodyStartBuf, &c.caFlagBuf, &c.caBodyMarkBuf, &c.caCandBuf, &c.caSpecBuf,
                           &c.localIdxBuf, &c.prepBuf, &c.frameBuf, &c.fpKeyBuf, &c.fpValBuf,
                           &c.fpSlotBuf, &c.fpColorBuf, &c.fpRunStartBuf, &c.fpIslandBuf, &c.coopBuf,
                           &c.giantBuf, &c.classKeyBuf, &c.classValBuf, &c.rowBodyBuf, &c.tinyBuf, &c.tinyKeyBuf, &c.clusterInfoBuf, &c.clusterKeyBuf,
                           &c.clusterValBuf, &c.clusterOfBuf, &c.clusterCountBuf, &c.clusterStartBuf,
                           &c.clusterRowsBuf, &c.clusterLinkBuf, &c.caInfoBuf, &c.tuneSaveBuf,
                           &c.countersBuf};
    for (vxb::DevBuf* b : bufs)
        if (b->ptr) cudaFree(b->ptr);
    if (c.ownStream) cudaStreamDestroy(c.ownStream);
    delete ctx;
}

const char* vxb_context_last_error(const vxb_context* ctx) {
    return ctx ? ctx->impl.lastError.c_str() : "null context";
}

int vxb_context_set_stream(vxb_context* ctx, void* stream) {
    GUARD(ctx);
    ctx->impl.stream = stream ? reinterpret_cast<cudaStream_t>(stream) : ctx->impl.ownStream;
    return VXB_OK;
}

uint64_t vxb_context_launch_count(const vxb_context* ctx) { return ctx ? ctx->impl.launches : 0; }

uint64_t vxb_context_host_syncs(const vxb_context* ctx) { return ctx ? ctx->impl.hostSyncs : 0; }

int vxb_context_set_tuning(vxb_context* ctx, int mode) {
    GUARD(ctx);
    if (mode != 0 && mode != 1) return VXB_ERR_INVALID;
    ctx->impl.tuner.setMode(mode);
    return VXB_OK;
}

int vxb_context_tuned_shape(const vxb_context* ctx, int site, uint32_t items, uint32_t* threads,
                            uint32_t* blocksPerSm, int* decided) {
    if (!ctx || site < 0 || site >= vxb::kTuneSiteCount || !threads || !blocksPerSm) return VXB_ERR_INVALID;
    bool d = false;
    const vxb::LaunchShape s = ctx->impl.tuner.shapeFor(site, items, &d);
    *threads = s.threads;
    *blocksPerSm = s.blocksPerSm;
    if (decided) *decided = d ? 1 : 0;
    return VXB_OK;
}

int vxb_context_tuning_save(vxb_context* ctx) {
    GUARD(ctx);
    return ctx->impl.tuner.save() ? VXB_OK : VXB_ERR_INVALID;
}

int vxb_context_set_wait_limit(vxb_context* ctx, uint32_t polls) {
    if (!ctx || polls > vxb::kSpinLimit) return VXB_ERR_INVALID;
    ctx->impl.waitLimit = polls ? polls : vxb::kSpinLimit;
    return VXB_OK;
}

int vxb_context_enable_timing(vxb_context* ctx, int enable) {
    GUARD(ctx);
    Context& c = ctx->impl;
    TRY(vxb::stageResolve(c));
    for (int s = 0; s < vxb::kStageCount; ++s) {
        c.timer.ms[s] = 0.0;
        c.timer.calls[s] = 0;
    }
    c.timing = enable != 0;
    return VXB_OK;
}

int vxb_context_stage_times(vxb_context* ctx, double* ms, uint64_t* calls, uint32_t count) {
    GUARD(ctx);
    if (!ms || !calls || count > (uint32_t)vxb::kStageCount) return VXB_ERR_INVALID;
    Context& c = ctx->impl;
    TRY(vxb::stageResolve(c));
    for (uint32_t s = 0; s < count; ++s) {
        ms[s] = c.timer.ms[s];
        calls[s] = c.timer.calls[s];
    }
    return VXB_OK;
}

// ---- Backend interface ---------------------------------------------------

int vxb_backend_integrate(vxb_context* ctx, vx_body* bodies, uint32_t n, vx_vec3 gravity, float dt) {
    GUARD(ctx);
    TRY(injectedFailure(ctx->impl));
    if (n == 0) return VXB_OK;
    if (!bodies) return VXB_ERR_INVALID;
    Context& c = ctx->impl;
    TRY(ensureCounters(c));
    TRY(vxb::loadBodies(c, bodies, n, nullptr));
    TRY(vxb::backendIntegrate(c, gravity, dt));
    return vxb::readBodies(c, bodies, n);
}

// The soup's structure and the mesh / compound bodies' references into it:
// what device reads depend on (the reference World validated the rest).
static int checkSoupRefs(Context& c, const vx_body* bodies, uint32_t n, const vx_soup* soup) {
    std::string why;
    if (!vxb::validSoup(soup, why)) return vxb::fail(c, VXB_ERR_INVALID, why);
    for (uint32_t i = 0; i < n; ++i)
        if (!vxb::validComplexRefs(bodies[i], soup, why))
            return vxb::fail(c, VXB_ERR_INVALID, "body " + std::to_string(i) + ": " + why);
    return VXB_OK;
}

int vxb_backend_find_contacts(vxb_context* ctx, const vx_body* bodies, uint32_t n, const vx_soup* soup, float dt,
                              uint32_t* count) {
    GUARD(ctx);
    if (!count) return VXB_ERR_INVALID;
    *count = 0;
    Context& c = ctx->impl;
    c.backendContacts = 0;
    if (n < 2) return VXB_OK;
    if (!bodies) return VXB_ERR_INVALID;
    TRY(checkSoupRefs(c, bodies, n, soup));
    TRY(ensureCounters(c));
    TRY(vxb::loadBodies(c, bodies, n, nullptr));
    TRY(vxb::loadSoup(c, soup));
    return vxb::backendFindContacts(c, dt, count);
}

int vxb_backend_copy_contacts(vxb_context* ctx, vx_contact* out, uint32_t cap) {
    GUARD(ctx);
    if (!out && ctx->impl.backendContacts) return VXB_ERR_INVALID;
    return vxb::backendCopyContacts(ctx->impl, out, cap);
}

int vxb_backend_solve_velocities(vxb_context* ctx, vx_body* bodies, uint32_t n, vx_contact* contacts, uint32_t m,
                                 float dt, int warmStart, const vx_solver_options* options, uint32_t* iterations) {
    GUARD(ctx);
    if (iterations) *iterations = 0;
    if (m == 0) return VXB_OK;
    if (!bodies || !contacts || !options || n == 0) return VXB_ERR_INVALID;
    Context& c = ctx->impl;
    if (!warmStart && (!c.backendColored || c.backendContacts != m))
        return vxb::fail(c, VXB_ERR_INVALID, "solve without warm start needs the resident coloured contacts");
    TRY(ensureCounters(c));
    TRY(vxb::loadBodies(c, bodies, n, nullptr));
    TRY(vxb::backendSolve(c, contacts, m, dt, warmStart != 0, *options, vx_vec3{0, 0, 0}, 1, false));
    if (iterations) *iterations = (uint32_t)(2 * options->velocityIterations);
    return vxb::readBodies(c, bodies, n);
}

int vxb_backend_advance_substeps(vxb_context* ctx, vx_body* bodies, uint32_t n, vx_contact* contacts, uint32_t m,
                                 vx_vec3 gravity, float h, int substeps, const vx_solver_options* options,
                                 int* advanced, uint32_t* iterations) {
    GUARD(ctx);
    if (!advanced || !options) return VXB_ERR_INVALID;
    *advanced = 0;
    if (iterations) *iterations = 0;
    if (options->iterationPolicy != 0) return VXB_OK;  // Adaptive: host path, like the reference
    if (n == 0) { *advanced = 1; return VXB_OK; }
    if (!bodies || (m && !contacts) || substeps <= 0) return VXB_ERR_INVALID;
    Context& c = ctx->impl;
    TRY(ensureCounters(c));
    TRY(vxb::loadBodies(c, bodies, n, nullptr));
    if (c.kinematic) {
        // kinematic bodies move every substep: the substep-wise order keeps
        // their poses current for the contact rows of every island
        TRY(vxb::backendStepwise(c, bodies, n, contacts, m, nullptr, 0, gravity, h, substeps, *options, iterations));
        *advanced = 1;
        return VXB_OK;
    }
    TRY(vxb::backendSolve(c, contacts, m, h, true, *options, gravity, substeps, true));
    TRY(vxb::readBodies(c, bodies, n));
    *advanced = 1;
    if (iterations) *iterations = m ? (uint32_t)(2 * options->velocityIterations * substeps) : 0u;
    return VXB_OK;
}

int vxb_backend_advance_substeps_joints(vxb_context* ctx, vx_body* bodies, uint32_t n, vx_contact* contacts,
                                        uint32_t m, vx_joint* joints, uint32_t njoints, vx_vec3 gravity, float h,
                                        int substeps, const vx_solver_options* options, int* advanced,
                                        uint32_t* iterations) {
    GUARD(ctx);
    if (!advanced || !options) return VXB_ERR_INVALID;
    *advanced = 0;
    if (iterations) *iterations = 0;
    if (njoints == 0)
        return vxb_backend_advance_substeps(ctx, bodies, n, contacts, m, gravity, h, substeps, options, advanced,
                                            iterations);
    if (!bodies || !joints || n == 0 || (m && !contacts) || substeps <= 0) return VXB_ERR_INVALID;
    Context& c = ctx->impl;
    TRY(ensureCounters(c));
    return vxb::backendAdvanceJoints(c, bodies, n, contacts, m, joints, njoints, gravity, h, substeps, *options,
                                     advanced, iterations);
}

int vxb_backend_fetch_impulses(vxb_context* ctx, vx_contact* contacts, uint32_t m) {
    GUARD(ctx);
    if (m && !contacts) return VXB_ERR_INVALID;
    return vxb::backendFetchImpulses(ctx->impl, contacts, m);
}

int vxb_backend_invalidate(vxb_context* ctx) {
    GUARD(ctx);
    ctx->impl.backendColored = false;
    ctx->impl.backendContacts = 0;
    ctx->impl.prevCount = 0;
    return VXB_OK;
}

// ---- device-resident world -------------------------------------------------

int vxb_world_load(vxb_context* ctx, const vx_body* bodies, uint32_t n, const vx_soup* soup,
                   const uint32_t* worldOfBody) {
    GUARD(ctx);
    if (!bodies || n == 0) return VXB_ERR_INVALID;
    Context& c = ctx->impl;
    {
        std::string why;
        if (!vxb::validSoup(soup, why)) return vxb::fail(c, VXB_ERR_INVALID, why);
        for (uint32_t i = 0; i < n; ++i)
            if (!vxb::validBody(bodies[i], soup, why))
                return vxb::fail(c, VXB_ERR_INVALID, "body " + std::to_string(i) + ": " + why);
    }
    TRY(ensureCounters(c));
    vxb::tapeEnd(c);  // a tape belongs to the world it recorded
    c.backendContacts = 0;  // a new world: no coloured Backend contacts
    c.backendColored = false;
    TRY(vxb::loadBodies(c, bodies, n, worldOfBody, true));
    TRY(vxb::loadSoup(c, soup));
    cudaError_t e = cudaStreamSynchronize(c.stream);
    return vxb::cudaStatus(c, e, "world load");
}

int vxb_world_configure(vxb_context* ctx, const vxb_step_config* config) {
    GUARD(ctx);
    if (!config || !(config->dt >= 0.0f) || !std::isfinite(config->dt) || config->substeps <= 0)
        return vxb::fail(ctx->impl, VXB_ERR_INVALID, "dt must be finite and >= 0, substeps > 0");
    if (!std::isfinite(config->gravity.x) || !std::isfinite(config->gravity.y) || !std::isfinite(config->gravity.z))
        return vxb::fail(ctx->impl, VXB_ERR_INVALID, "gravity must be finite");
    {
        std::string why;
        if (!vxb::validSolverOptions(config->solver, why)) return vxb::fail(ctx->impl, VXB_ERR_INVALID, why);
    }
    if (config->solver.iterationPolicy != 0)
        return vxb::fail(ctx->impl, VXB_ERR_UNSUPPORTED, "the adaptive iteration policy runs on the host");
    ctx->impl.config = *config;
    ctx->impl.configured = true;
    return VXB_OK;
}

int vxb_world_step(vxb_context* ctx, int steps) {
    GUARD(ctx);
    if (steps < 0) return VXB_ERR_INVALID;
    if (ctx->impl.config.dt == 0.0f) return VXB_OK;
    return vxb::worldStep(ctx->impl, steps);
}

int vxb_world_read_bodies(vxb_context* ctx, vx_body* out, uint32_t n) {
    GUARD(ctx);
    if (!out) return VXB_ERR_INVALID;
    return vxb::readBodies(ctx->impl, out, n);
}

int vxb_world_read_poses(vxb_context* ctx, float* out, uint32_t n) {
    GUARD(ctx);
    if (!out) return VXB_ERR_INVALID;
    return vxb::readPoses(ctx->impl, out, n);
}

int vxb_world_write_forces(vxb_context* ctx, const float* in, uint32_t n) {
    GUARD(ctx);
    if (!in) return VXB_ERR_INVALID;
    if (!vxb::finiteValues(in, (size_t)n * 6))
        return vxb::fail(ctx->impl, VXB_ERR_INVALID, "forces and torques must be finite");
    return vxb::writeForces(ctx->impl, in, n);
}

int vxb_world_read_contacts(vxb_context* ctx, vx_contact* out, uint32_t cap, uint32_t* count) {
    GUARD(ctx);
    return vxb::readContacts(ctx->impl, out, cap, count);
}

void vxb_sleep_config_default(vxb_sleep_config* out) {
    if (out) vxb::sleepConfigDefault(out);
}

int vxb_world_configure_sleep(vxb_context* ctx, const vxb_sleep_config* config) {
    GUARD(ctx);
    if (!config) return VXB_ERR_INVALID;
    const float v[] = {config->linearVelocityThreshold, config->angularVelocityThreshold,
                       config->accelerationThreshold, config->timeToSleep, config->timeToDrowsy,
                       config->contactStabilityThreshold};
    for (float x : v)
        if (!std::isfinite(x) || x < 0.0f)
            return vxb::fail(ctx->impl, VXB_ERR_INVALID, "sleep thresholds and times must be finite and >= 0");
    if (config->contactStabilityFrames < 0 || config->contactStabilityFrames > 65535)
        return vxb::fail(ctx->impl, VXB_ERR_INVALID, "contactStabilityFrames must be in [0, 65535]");
    ctx->impl.sleep.config = *config;
    return VXB_OK;
}

int vxb_world_enable_events(vxb_context* ctx, int enable) {
    GUARD(ctx);
    ctx->impl.sleep.events = enable != 0;
    if (!ctx->impl.sleep.events) ctx->impl.sleep.eventCount = 0;
    return VXB_OK;
}

int vxb_world_read_events(vxb_context* ctx, vxb_contact_event* out, uint32_t cap, uint32_t* count) {
    GUARD(ctx);
    return vxb::readEvents(ctx->impl, out, cap, count);
}

int vxb_world_write_contacts(vxb_context* ctx, const vx_contact* contacts, uint32_t m) {
    GUARD(ctx);
    vxb::Context& c = ctx->impl;
    if (m && !contacts) return VXB_ERR_INVALID;
    if (c.n == 0) return vxb::fail(c, VXB_ERR_INVALID, "no bodies loaded");
    for (uint32_t k = 0; k < m; ++k) {
        const vx_contact& x = contacts[k];
        if (x.a >= x.b || x.b >= c.n)
            return vxb::fail(c, VXB_ERR_INVALID, "contact " + std::to_string(k) + ": needs a < b < body count");
        if (k && (((uint64_t)x.a << 32) | x.b) < (((uint64_t)contacts[k - 1].a << 32) | contacts[k - 1].b))
            return vxb::fail(c, VXB_ERR_INVALID, "contacts must be sorted by (a, b)");
    }
    return vxb::writeContacts(c, contacts, m);
}

int vxb_world_stats(vxb_context* ctx, vxb_step_stats* out) {
    if (!ctx || !out) return VXB_ERR_INVALID;
    *out = ctx->impl.stats;
    return VXB_OK;
}

// ---- snapshots ---------------------------------------------------------------

int vxb_world_snapshot_save(vxb_context* ctx, uint32_t slot) {
    GUARD(ctx);
    return vxb::snapshotSave(ctx->impl, slot);
}

int vxb_world_snapshot_restore(vxb_context* ctx, uint32_t slot) {
    GUARD(ctx);
    return vxb::snapshotRestore(ctx->impl, slot);
}

int vxb_world_snapshot_bytes(vxb_context* ctx, uint64_t* bytes) {
    GUARD(ctx);
    if (!bytes) return VXB_ERR_INVALID;
    size_t b = 0;
    TRY(vxb::snapshotBytes(ctx->impl, &b));
    *bytes = b;
    return VXB_OK;
}

int vxb_world_snapshot_read(vxb_context* ctx, void* out, uint64_t capacity) {
    GUARD(ctx);
    if (!out) return VXB_ERR_INVALID;
    return vxb::snapshotRead(ctx->impl, out, (size_t)capacity);
}

int vxb_world_snapshot_write(vxb_context* ctx, const void* in, uint64_t size) {
    GUARD(ctx);
    if (!in) return VXB_ERR_INVALID;
    return vxb::snapshotWrite(ctx->impl, in, (size_t)size);
}

// ---- adjoint -----------------------------------------------------------------

int vxb_tape_begin(vxb_context* ctx, uint32_t steps, uint32_t checkpointEvery) {
    GUARD(ctx);
    Context& c = ctx->impl;
    if (!c.configured) return vxb::fail(c, VXB_ERR_INVALID, "vxb_world_configure was not called");
    TRY(vxb::tapeEnd(c));
    return vxb::tapeBegin(c, steps, checkpointEvery);
}

int vxb_tape_info(vxb_context* ctx, uint32_t* recordedSteps, uint32_t* contacts, uint32_t* checkpoints) {
    if (!ctx) return VXB_ERR_INVALID;
    const vxb::Tape& T = ctx->impl.tape;
    if (recordedSteps) *recordedSteps = T.active ? T.recorded : 0u;
    if (contacts) *contacts = T.active ? T.stepStart.back() : 0u;
    if (checkpoints) *checkpoints = T.active ? (T.steps + T.every - 1) / T.every + 1 : 0u;
    return VXB_OK;
}

int vxb_tape_read(vxb_context* ctx, vx_contact* contacts, uint32_t* stepStart, uint32_t* sources, int32_t* colors,
                  float* checkpoints, uint32_t* worldFlags) {
    GUARD(ctx);
    if (!ctx->impl.tape.active) return vxb::fail(ctx->impl, VXB_ERR_INVALID, "no tape");
    return vxb::tapeRead(ctx->impl, contacts, stepStart, sources, colors, checkpoints, worldFlags);
}

int vxb_adjoint_backward(vxb_context* ctx, const float* seed, float* grad, float* gradInverseMass, float* gradMass,
                         uint32_t* worldFlags) {
    GUARD(ctx);
    return vxb::adjointBackward(ctx->impl, seed, grad, gradInverseMass, gradMass, worldFlags);
}

int vxb_adjoint_backward_branches(vxb_context* ctx, const float* seed, float* grad, float* gradInverseMass,
                                  float* gradMass, uint32_t* worldFlags, uint8_t* branches, size_t capacity,
                                  size_t* branchBytes, uint32_t* branchRows) {
    GUARD(ctx);
    if (!branchBytes || !branchRows) return VXB_ERR_INVALID;
    return vxb::adjointBackward(ctx->impl, seed, grad, gradInverseMass, gradMass, worldFlags, branches, capacity,
                                branchBytes, branchRows);
}

int vxb_tape_end(vxb_context* ctx) {
    GUARD(ctx);
    return vxb::tapeEnd(ctx->impl);
}

// ---- stages ----------------------------------------------------------------

int vxb_stage_pairs(vxb_context* ctx, const vx_body* bodies, uint32_t n, float dt, uint64_t* out, uint32_t cap,
                    uint32_t* count) {
    GUARD(ctx);
    if (!bodies || !count || n == 0) return VXB_ERR_INVALID;
    Context& c = ctx->impl;
    for (uint32_t i = 0; i < n; ++i)
        if (bodies[i].shape == VX_SHAPE_MESH)
            return vxb::fail(c, VXB_ERR_INVALID, "mesh bodies need their soup: use vxb_stage_pairs_soup");
    TRY(ensureCounters(c));
    TRY(vxb::loadBodies(c, bodies, n, nullptr));
    return vxb::stagePairs(c, dt, out, cap, count);
}

int vxb_stage_pairs_soup(vxb_context* ctx, const vx_body* bodies, uint32_t n, const vx_soup* soup, float dt,
                         uint64_t* out, uint32_t cap, uint32_t* count) {
    GUARD(ctx);
    if (!bodies || !count || n == 0) return VXB_ERR_INVALID;
    Context& c = ctx->impl;
    TRY(checkSoupRefs(c, bodies, n, soup));
    TRY(ensureCounters(c));
    TRY(vxb::loadBodies(c, bodies, n, nullptr));
    TRY(vxb::loadSoup(c, soup));
    return vxb::stagePairs(c, dt, out, cap, count);
}

int vxb_stage_distance(vxb_context* ctx, const vx_body* bodies, uint32_t n, const vx_soup* soup,
                       const uint64_t* pairs, uint32_t npairs, int path, float* out) {
    GUARD(ctx);
    if (!bodies || n == 0 || (npairs && (!pairs || !out)) || (path != 0 && path != 1)) return VXB_ERR_INVALID;
    Context& c = ctx->impl;
    for (uint32_t p = 0; p < npairs; ++p)
        if ((uint32_t)(pairs[p] >> 32) >= n || (uint32_t)pairs[p] >= n) return VXB_ERR_INVALID;
    for (uint32_t i = 0; i < n; ++i)
        if (bodies[i].shape == VX_SHAPE_MESH || bodies[i].shape == VX_SHAPE_COMPOUND)
            return vxb::fail(c, VXB_ERR_UNSUPPORTED, "the distance stage takes convex bodies and planes");
    TRY(ensureCounters(c));
    TRY(vxb::loadBodies(c, bodies, n, nullptr));
    TRY(vxb::loadSoup(c, soup));
    return vxb::stageDistance(c, pairs, npairs, path, out);
}

int vxb_stage_collide(vxb_context* ctx, const vx_body* bodies, uint32_t n, const vx_soup* soup,
                      const uint64_t* pairs, uint32_t npairs, float dt, vx_contact* out, uint32_t cap,
                      uint32_t* counts, uint32_t* total) {
    GUARD(ctx);
    if (!bodies || !total || n == 0 || (npairs && !pairs)) return VXB_ERR_INVALID;
    Context& c = ctx->impl;
    for (uint32_t p = 0; p < npairs; ++p)
        if ((uint32_t)(pairs[p] >> 32) >= n || (uint32_t)pairs[p] >= n) return VXB_ERR_INVALID;
    TRY(checkSoupRefs(c, bodies, n, soup));
    TRY(ensureCounters(c));
    TRY(vxb::loadBodies(c, bodies, n, nullptr));
    TRY(vxb::loadSoup(c, soup));
    return vxb::stageCollide(c, pairs, npairs, dt, out, cap, counts, total);
}

int vxb_stage_color(vxb_context* ctx, const vx_body* bodies, uint32_t n, const vx_contact* contacts, uint32_t m,
                    int32_t* colorOf, uint32_t* numColors) {
    GUARD(ctx);
    if (!bodies || !numColors || n == 0 || (m && (!contacts || !colorOf))) return VXB_ERR_INVALID;
    Context& c = ctx->impl;
    for (uint32_t k = 0; k < m; ++k)
        if (contacts[k].a >= n || contacts[k].b >= n) return VXB_ERR_INVALID;
    TRY(ensureCounters(c));
    TRY(vxb::loadBodies(c, bodies, n, nullptr));
    return vxb::stageColor(c, contacts, m, colorOf, numColors);
}

}  // extern "C"
