/*
 * velox_b200.h — C ABI of the B200 (sm_100a) rigid-body contact pipeline.
 *
 * The library replaces the reference engine's CUDA backend
 * (src/backend_cuda.cu, class CudaBackend) behind its Backend interface
 * (include/velox/backend.h:111-172). Every entry point takes plain pointers
 * and sizes, returns a status code (never throws), and operates on one
 * vxb_context = one backend instance = one CUDA stream on one device.
 * Records crossing the ABI use the reference's host layouts
 * (velox_b200_types.h), so the reference-side adapter passes
 * `std::vector<Body>::data()` straight through.
 *
 * Status codes map onto the reference's error model
 * (src/backend_cuda.cu:24-40, include/velox/backend.h:95-106):
 *   VXB_ERR_OOM          -> BackendFailure(MemoryAllocation)
 *   VXB_ERR_DEVICE_LOST  -> BackendFailure(DeviceLost)
 *   VXB_ERR_TIMEOUT      -> BackendFailure(DeviceLost) (a bounded device wait gave up)
 *   VXB_ERR_CAPACITY     -> VeloxCapacityExceeded(ContactCountOverflow)
 *   VXB_ERR_INTERNAL     -> VeloxRuntimeError(BackendUnavailable)
 *   VXB_ERR_NO_DEVICE    -> createCudaBackend() returning nullptr
 *   others               -> VeloxRuntimeError(BackendUnavailable)
 * Threading matches the reference backend: one owner thread per context.
 */
#ifndef VELOX_B200_H
#define VELOX_B200_H

#include "velox_b200_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Every declaration below is exported from libvelox_b200.so (the library is
 * otherwise built with hidden visibility). */
#pragma GCC visibility push(default)

#define VXB_OK 0
#define VXB_ERR_INVALID 1
#define VXB_ERR_NO_DEVICE 2
#define VXB_ERR_OOM 3
#define VXB_ERR_DEVICE_LOST 4
#define VXB_ERR_CAPACITY 5
#define VXB_ERR_UNSUPPORTED 6
#define VXB_ERR_TIMEOUT 7
#define VXB_ERR_INTERNAL 8 /* a device-side consistency check failed; the step's results are void */

typedef struct vxb_context vxb_context;

/* Per-step configuration of the device-resident world (World::step's inputs:
 * include/velox/world.h:434-438 gravity/substeps, SolverOptions). */
typedef struct vxb_step_config {
    float dt;
    vx_vec3 gravity;
    int32_t substeps;
    vx_solver_options solver;
} vxb_step_config;

/* Sleeping thresholds (velox::SleepConfig, include/velox/sleep.h:98-140;
 * vxb_sleep_config_default gives the reference's defaults). */
typedef struct vxb_sleep_config {
    float linearVelocityThreshold;   /* 0.05 m/s */
    float angularVelocityThreshold;  /* 0.05 rad/s */
    float accelerationThreshold;     /* 0.01 m/s^2 */
    float timeToSleep;               /* 0.5 s */
    float timeToDrowsy;              /* 0.25 s */
    float contactStabilityThreshold; /* 0.02 m/s */
    int32_t contactStabilityFrames;  /* 10 */
    uint8_t enableGradualSleep;      /* 1 */
    uint8_t enableContactStability;  /* 1 */
    uint8_t pad[2];
} vxb_sleep_config;

/* A contact or sensor event of the last step (velox::ContactEvent,
 * include/velox/world.h:65-75, with dense body indices a < b instead of
 * handles). type: 0 Begin, 1 Persist, 2 End. */
typedef struct vxb_contact_event {
    uint32_t a, b;
    vx_vec3 point;
    vx_vec3 normal;  /* from a towards b */
    float impulse;
    uint8_t type;
    uint8_t sensor;
    uint8_t pad[2];
} vxb_contact_event;

/* Counters of the last device step (subset of velox::StepStats,
 * include/velox/world.h:175-208, plus pipeline internals). */
typedef struct vxb_step_stats {
    uint32_t candidatePairs;     /* broad-phase pairs (narrowPhaseTests) */
    uint32_t contacts;           /* generatedContacts */
    uint32_t colors;             /* largest colour count of any island */
    uint32_t islands;            /* contact islands solved */
    uint32_t largestIsland;      /* contacts in the largest island */
    uint32_t rewinds;            /* conservative-advancement rewinds */
    uint32_t velocityIterations; /* sweeps per step (2*velocityIterations*substeps) */
    uint32_t warmStarted;        /* contacts that inherited impulses */
    uint32_t colorRounds;        /* fixed-point rounds of the parallel colouring (0 = none) */
    uint32_t giantIslands;       /* islands solved by the whole grid (cooperative launch) */
    uint32_t rewindRounds;       /* dependency depth of the rewind passes (summed over passes) */
    uint32_t rewindReplays;      /* rewind passes replayed with a widened body set */
    uint32_t rewindGapQueries;   /* distance queries of the rewind passes */
    uint32_t rewindCriticalMicros; /* evaluation time along the longest rewind dependency chain */
    uint32_t rewindSpeculateMicros; /* the longest single pair's conservative advancement (speculated
                                       in parallel before the ordered pass; part of that chain) */
} vxb_step_stats;

/* ---- library / context ------------------------------------------------ */

const char* vxb_version(void);
const char* vxb_status_string(int status);

/* Creates a backend instance on `device` (createCudaBackend(),
 * src/backend_cuda.cu:352-356 and :1020). Returns VXB_ERR_NO_DEVICE when no
 * CUDA device is present (the reference returns nullptr). */
int vxb_context_create(int device, vxb_context** out);
/* Drains the stream and releases every device buffer (~CudaBackend,
 * src/backend_cuda.cu:358-388). Never fails. */
void vxb_context_destroy(vxb_context* ctx);
/* Message of the last failure on this context ("" when none). */
const char* vxb_context_last_error(const vxb_context* ctx);
/* Launch subsequent work on `stream` (a cudaStream_t); null restores the
 * context's own stream. */
int vxb_context_set_stream(vxb_context* ctx, void* stream);
/* Number of kernel launches this context issued since it was created. */
uint64_t vxb_context_launch_count(const vxb_context* ctx);
/* Polls after which any device-side wait of this context (grid barriers,
 * dataflow waits of the cooperative solve and rewind kernels) gives up; the
 * call then fails with VXB_ERR_TIMEOUT and the context stays usable. 0
 * restores the default (2^24 polls of at least 32 ns, over a second). The
 * environment variable VXB_WAIT_LIMIT sets it for contexts created after it.
 * No counterpart in the reference (its CUDA backend has no device-side
 * waits); it exists to bound and test the recovery path of
 * src/world.cpp:3807-3828. */
int vxb_context_set_wait_limit(vxb_context* ctx, uint32_t polls);

/* Blocking host reads of device counts this context made since it was
 * created (each drains the stream: a step sizes its later launches from the
 * counts of earlier kernels). No counterpart in the reference. */
uint64_t vxb_context_host_syncs(const vxb_context* ctx);

/* Launch-shape autotuning of the throughput kernels: the narrow phase's
 * per-pair kernels and the rewind's per-pair probe. Per site and size bucket
 * (floor(log2(items))) the first launch runs six shapes (block size 32/64/128
 * threads x grid cap of 2,048 threads per SM or one resident wave) twice each
 * on the same inputs, timed with CUDA events on the context's stream (a
 * one-time cost that waits for each trial); the fastest is kept and written to
 * a cache file that later contexts on the same device model read at creation.
 * Shapes change timing only: every result is identical under any shape.
 * mode 1 (the default; VXB_TUNE=0 in the environment makes it 0 for new
 * contexts) tunes; mode 0 launches the fixed default shape (128 threads,
 * 16 blocks per SM). The cache file is VXB_TUNE_CACHE, else
 * $XDG_CACHE_HOME/velox_b200/launch_shapes.txt, else
 * $HOME/.cache/velox_b200/launch_shapes.txt; VXB_TUNE_CACHE="" keeps the
 * decisions in memory. No counterpart in the reference, whose narrow phase
 * launches a fixed 256-thread block per 256 pairs (src/backend_cuda.cu:459,
 * :556-561). */
#define VXB_TUNE_COLLIDE_CONVEX 0
#define VXB_TUNE_COLLIDE_COMPLEX 1
#define VXB_TUNE_COLLIDE_PLANE 2
#define VXB_TUNE_COLLIDE_ANY 3
#define VXB_TUNE_REWIND_PROBE 4
int vxb_context_set_tuning(vxb_context* ctx, int mode);
/* The shape the next launch of `site` over `items` items would use, and
 * whether its size bucket is decided (1) or still has its trials ahead (0). */
int vxb_context_tuned_shape(const vxb_context* ctx, int site, uint32_t items, uint32_t* threads,
                            uint32_t* blocksPerSm, int* decided);
/* Writes this context's decisions to the cache file now (also done when a
 * bucket is decided and when the context is destroyed). VXB_ERR_INVALID when
 * no cache file is configured or it cannot be written. */
int vxb_context_tuning_save(vxb_context* ctx);

/* Per-stage device timing with CUDA events recorded on the context's stream
 * (stages: 0 prepare, 1 broad phase, 2 cell-key sort, 3 narrow phase,
 * 4 contact placement, 5 warm start, 6 islands + colouring, 7 substep solve,
 * 8 rewind, 9 position correction). Enabling resets the totals. */
int vxb_context_enable_timing(vxb_context* ctx, int enable);
/* Totals since timing was enabled: ms[stage] and calls[stage] for
 * `count` stages (<= 10). Synchronises the stream. */
int vxb_context_stage_times(vxb_context* ctx, double* ms, uint64_t* calls, uint32_t count);

/* ---- Backend interface over host arrays ------------------------------- */

/* Backend::integrate (backend.h:116; CudaBackend::integrate,
 * src/backend_cuda.cu:393-403): first-substep velocity integration. Honours
 * the reference's test injection VELOX_CUDA_TEST_FAIL=oom|device-loss
 * (src/backend_cuda.cu:69-78): VXB_ERR_OOM / VXB_ERR_DEVICE_LOST before any
 * device work. */
int vxb_backend_integrate(vxb_context* ctx, vx_body* bodies, uint32_t n, vx_vec3 gravity,
                          float dt);
/* Backend::findContacts (backend.h:125-127; src/backend_cuda.cu:405-567):
 * speculative contacts of every candidate pair for a step of `dt`. Contacts
 * stay device-resident; *count receives their number, copy them with
 * vxb_backend_copy_contacts. Hull geometry comes from `soup`. */
int vxb_backend_find_contacts(vxb_context* ctx, const vx_body* bodies, uint32_t n,
                              const vx_soup* soup, float dt, uint32_t* count);
/* Copies the contacts of the last find (sorted by (a, b, point)). */
int vxb_backend_copy_contacts(vxb_context* ctx, vx_contact* out, uint32_t cap);
/* Backend::solveVelocities (backend.h:132-135; src/backend_cuda.cu:569-689).
 * With warmStart != 0 the contacts are sorted, coloured and written back in
 * colour order, exactly as the reference writes back its colour-sorted copy. */
int vxb_backend_solve_velocities(vxb_context* ctx, vx_body* bodies, uint32_t n,
                                 vx_contact* contacts, uint32_t m, float dt, int warmStart,
                                 const vx_solver_options* options, uint32_t* iterations);
/* Backend::advanceSubsteps (backend.h:139-144; src/backend_cuda.cu:691-761).
 * *advanced = 0 when the request needs the host path (iteration policy
 * Adaptive), matching the reference's `return false`. */
int vxb_backend_advance_substeps(vxb_context* ctx, vx_body* bodies, uint32_t n,
                                 vx_contact* contacts, uint32_t m, vx_vec3 gravity, float h,
                                 int substeps, const vx_solver_options* options, int* advanced,
                                 uint32_t* iterations);
/* Backend::advanceSubsteps with joints (src/backend_cuda.cu:691-760): with
 * 64 or more joints, all of types up to VX_JOINT_GEAR, every substep runs
 * the contact sweeps (the first warm-started), the joints' reset, 8 sweeps
 * colour by colour and break test, and the position integration of every
 * body; joints (their scratch impulses and broken flags) and bodies are
 * written back. A joint whose endpoints differ in `asleep` wakes both first
 * (also when the call declines). *advanced = 0 (the host path) for fewer
 * joints, an unsupported type or the Adaptive iteration policy. */
int vxb_backend_advance_substeps_joints(vxb_context* ctx, vx_body* bodies, uint32_t n,
                                        vx_contact* contacts, uint32_t m, vx_joint* joints,
                                        uint32_t njoints, vx_vec3 gravity, float h, int substeps,
                                        const vx_solver_options* options, int* advanced,
                                        uint32_t* iterations);
/* Backend::fetchImpulses (backend.h:148; src/backend_cuda.cu:763-768). */
int vxb_backend_fetch_impulses(vxb_context* ctx, vx_contact* contacts, uint32_t m);
/* Backend::invalidateCaches (backend.h:150; src/backend_cuda.cu:770-784). */
int vxb_backend_invalidate(vxb_context* ctx);

/* ---- device-resident world: the whole World::step on the GPU --------------
 * One call runs src/world.cpp:3830-4521's contact pipeline for every world
 * of the batch without host round trips: orientation normalisation,
 * first-substep gravity, broad phase, narrow phase, warm-start matching,
 * colouring, the substep loop, the conservative-advancement rewind,
 * split-impulse position correction and the previous-contact cache.
 * Batches: `worldOfBody` (nullable = one world) assigns each body to a world;
 * bodies of one world must be contiguous and worlds never interact.
 * Inputs are validated with the reference's per-step rules for public state
 * (src/world.cpp:3855-3931): vxb_world_load rejects non-finite or out-of-range
 * body state and invalid shape parameters ("body <i>: <reason>"),
 * vxb_world_configure non-finite dt or gravity and invalid solver options,
 * vxb_world_write_forces non-finite values; each with VXB_ERR_INVALID. */
int vxb_world_load(vxb_context* ctx, const vx_body* bodies, uint32_t n, const vx_soup* soup,
                   const uint32_t* worldOfBody);
int vxb_world_configure(vxb_context* ctx, const vxb_step_config* config);
int vxb_world_step(vxb_context* ctx, int steps);
int vxb_world_read_bodies(vxb_context* ctx, vx_body* out, uint32_t n);
/* position xyz + orientation xyzw per body (7 floats). */
int vxb_world_read_poses(vxb_context* ctx, float* out, uint32_t n);
/* force xyz + torque xyz per body (6 floats), consumed and cleared by the
 * next step like Body::force/torque. */
int vxb_world_write_forces(vxb_context* ctx, const float* in, uint32_t n);
int vxb_world_read_contacts(vxb_context* ctx, vx_contact* out, uint32_t cap, uint32_t* count);
/* Replaces the warm-start cache (the previous step's contacts, what the next
 * step matches against: World::prevContacts_, src/world.cpp:4496-4520 and
 * 4133-4184). `contacts` must be sorted by (a, b) with a < b < n; within one
 * pair the given order is kept (it decides exact ties of the nearest-point
 * fallback). m = 0 empties the cache. Ends an adjoint tape. */
int vxb_world_write_contacts(vxb_context* ctx, const vx_contact* contacts, uint32_t m);
int vxb_world_stats(vxb_context* ctx, vxb_step_stats* out);

/* ---- sleeping and contact events of the device world -------------------------
 * Every step runs the reference's wake pass (src/world.cpp:4106-4128, after
 * detection, before warm starting), island sleeping (SleepManager::update,
 * src/sleep.cpp:52-237: union-find islands over dynamic-dynamic contacts,
 * contact stability, calm timers, the island minimum, drowsy / asleep
 * transitions) and keeps the cached contacts of resting pairs for warm
 * starting (src/world.cpp:4496-4521), whenever a loaded body may sleep
 * (enableSleep) or is asleep. Body read-back carries `asleep` and
 * `sleepTimer`. */
void vxb_sleep_config_default(vxb_sleep_config* out);
/* Replaces the sleeping thresholds (default: the reference's). */
int vxb_world_configure_sleep(vxb_context* ctx, const vxb_sleep_config* config);
/* Contact and sensor events (src/world.cpp:4398-4488): off by default (they
 * cost a sort and two small read-backs per step); when on, every step
 * records Begin / Persist / End events in the reference's order. */
int vxb_world_enable_events(vxb_context* ctx, int enable);
/* The last step's events; *count receives their number (out nullable). */
int vxb_world_read_events(vxb_context* ctx, vxb_contact_event* out, uint32_t cap, uint32_t* count);

/* ---- snapshots of the device world ------------------------------------------
 * World::saveSnapshot / restoreSnapshot (src/world.cpp:2038-2128) for the
 * state this library keeps on the device: all body state, the previous step's
 * contacts (the warm-start cache), the step configuration and the last step's
 * statistics. A snapshot restores only into a world with the same body count
 * and world partition (VXB_ERR_INVALID otherwise); restoring ends an adjoint
 * tape. Stepping after a restore repeats the original steps bit for bit. */

/* Device-memory snapshot slots 0..7 (copies stay on the device: rollback and
 * replay without host round trips). */
int vxb_world_snapshot_save(vxb_context* ctx, uint32_t slot);
int vxb_world_snapshot_restore(vxb_context* ctx, uint32_t slot);
/* The same state as a byte image in caller memory (files, other contexts):
 * size, copy out (VXB_ERR_CAPACITY if `capacity` is too small), copy in. */
int vxb_world_snapshot_bytes(vxb_context* ctx, uint64_t* bytes);
int vxb_world_snapshot_read(vxb_context* ctx, void* out, uint64_t capacity);
int vxb_world_snapshot_write(vxb_context* ctx, const void* in, uint64_t size);

/* ---- adjoint of the device world's step ---------------------------------------
 * No counterpart in the reference (it has no differentiation). The adjoint
 * differentiates the step as the device world runs it (src/world.cpp:4007-4397
 * with the coloured solve of src/backend_cuda.cu:569-761): the warm start and
 * solveContact sweeps (src/narrowphase.h:80-366), the integration
 * (include/velox/body.h:266-321) and the position correction
 * (src/world.cpp:4370-4397), with each step's contact set, feature matching,
 * colours and clamp / friction-ellipse / correction active sets frozen from
 * the forward pass. Scope: two-axis friction, isotropic inverse inertia, zero
 * rolling and spinning friction, no forces written during the taped steps.
 *
 * Use: vxb_world_load + vxb_world_configure, vxb_tape_begin(steps, k), then
 * vxb_world_step for those steps (they are recorded: contacts after matching,
 * body checkpoints every k steps), then vxb_adjoint_backward. The backward
 * pass recomputes each k-step segment from its checkpoint (bit-identical to
 * the forward) and runs the reverse; one warp per world. */

/* Per-world flags of a tape / backward pass. */
#define VXB_ADJ_REWOUND 1u     /* a conservative-advancement rewind moved a body: not smooth */
#define VXB_ADJ_DIVERGED 2u    /* the recomputed segment left the forward trajectory */
#define VXB_ADJ_UNSUPPORTED 4u /* outside the reverse's scope (see above) */

/* Starts recording the next `steps` steps of vxb_world_step, with a body
 * checkpoint every `checkpointEvery` steps. Replaces any earlier tape. */
int vxb_tape_begin(vxb_context* ctx, uint32_t steps, uint32_t checkpointEvery);
/* Steps recorded so far, contacts recorded, checkpoint slots (incl. the final state). */
int vxb_tape_info(vxb_context* ctx, uint32_t* recordedSteps, uint32_t* contacts, uint32_t* checkpoints);
/* Copies the tape out (each pointer nullable): contacts after matching,
 * stepStart[steps + 1], sources (2 per contact: the previous step's contact
 * it inherited impulses / vn0 from, 0xffffffff = none), colours, checkpoints
 * (slots x 4 x n float4: position, orientation, velocity, angular velocity),
 * world flags. */
int vxb_tape_read(vxb_context* ctx, vx_contact* contacts, uint32_t* stepStart, uint32_t* sources, int32_t* colors,
                  float* checkpoints, uint32_t* worldFlags);
/* Backward pass over a fully recorded tape. seed: dL/d(state after the last
 * taped step), n x 13 floats per body (position 3, orientation 4, velocity 3,
 * angular velocity 3), null = zero. Outputs (each nullable): grad = dL/d(state
 * at the tape's first step), n x 13; gradInverseMass = dL/d(invMass) and
 * dL/d(isotropic invInertia), n x 2; gradMass = dL/d(mass) for inertia that
 * scales with mass, n; worldFlags (VXB_ADJ_*), one per world. Worlds with a
 * flag get zero gradients. */
int vxb_adjoint_backward(vxb_context* ctx, const float* seed, float* grad, float* gradInverseMass,
                         float* gradMass, uint32_t* worldFlags);
/* vxb_adjoint_backward that also reports the branch decisions the reverse
 * differentiated (the piece of the piecewise-smooth step the forward took),
 * one byte each, for checking against an independent adjoint. Layout: worlds
 * x steps x blocks of *branchRows bytes (world-local contact index within the
 * step): per substep the live gap's sign (1 = positive); the warm start's
 * activity; per substep and sweep the row bits (1 restitution condition,
 * 2 restitution target, 4 normal impulse unclamped, 8 friction rows,
 * 16 / 32 first / second friction axis bounded, 64 ellipse projection,
 * 128 row without normal mass); per position pass the push's activity.
 * *branchBytes receives the size; a null or smaller buffer returns
 * VXB_ERR_CAPACITY before the reverse runs. */
int vxb_adjoint_backward_branches(vxb_context* ctx, const float* seed, float* grad, float* gradInverseMass,
                                  float* gradMass, uint32_t* worldFlags, uint8_t* branches, size_t capacity,
                                  size_t* branchBytes, uint32_t* branchRows);
/* Releases the tape. */
int vxb_tape_end(vxb_context* ctx);

/* ---- individual stages (parity testing) --------------------------------- */

/* Candidate pairs (i<j) of the sorted-grid broad phase, returned sorted
 * ascending as (i<<32)|j: the pair set of gridPairsKernel/oversizePairsKernel
 * and allPairsContactsKernel (src/backend_cuda.cu:174-299). */
int vxb_stage_pairs(vxb_context* ctx, const vx_body* bodies, uint32_t n, float dt,
                    uint64_t* out, uint32_t cap, uint32_t* count);
/* vxb_stage_pairs for scenes with static meshes, whose root bounds come from
 * the soup (src/backend_cuda.cu:100-129: meshes pair with every body whose
 * swept AABB overlaps those bounds). vxb_stage_pairs rejects mesh bodies. */
int vxb_stage_pairs_soup(vxb_context* ctx, const vx_body* bodies, uint32_t n, const vx_soup* soup,
                         float dt, uint64_t* out, uint32_t cap, uint32_t* count);
/* collidePair (src/narrowphase.h:678-714) for each listed pair; contacts are
 * returned grouped in pair order, counts[p] per pair, *total overall. */
int vxb_stage_collide(vxb_context* ctx, const vx_body* bodies, uint32_t n, const vx_soup* soup,
                      const uint64_t* pairs, uint32_t npairs, float dt, vx_contact* out,
                      uint32_t cap, uint32_t* counts, uint32_t* total);
/* gjkDistance(makeConvex(a), makeConvex(b)) (include/velox/gjk.h:751-777)
 * for each listed pair: out[11*p ..] = distance, normal xyz, pointA xyz,
 * pointB xyz, overlapping (1/0). path 0 = the rewind's query (register GJK,
 * general GJK/EPA on overlap), 1 = the general GJK/EPA only. Convex bodies
 * and planes only (VXB_ERR_UNSUPPORTED for meshes and compounds). */
int vxb_stage_distance(vxb_context* ctx, const vx_body* bodies, uint32_t n, const vx_soup* soup,
                       const uint64_t* pairs, uint32_t npairs, int path, float* out);
/* Greedy first-free-bit colouring (src/backend_cuda.cu:603-630) of contacts
 * already in (a, b, point) order. */
int vxb_stage_color(vxb_context* ctx, const vx_body* bodies, uint32_t n,
                    const vx_contact* contacts, uint32_t m, int32_t* colorOf,
                    uint32_t* numColors);

/* Broad-phase candidate pairs, as vxb_stage_pairs, for callers that must not
 * allocate device memory during the call (frame-locked loops with a fixed
 * memory budget, plugin hosts that own all device memory, code running on a
 * nearly full device). No counterpart in the reference: it exists for such
 * callers only. Needs no context. All device memory it uses is one
 * library-owned array of about 4.3 MB, held on every device that loads the
 * library until exit; after the first call on a device the call allocates
 * nothing (device or host heap). The first call on a device is its set-up: it
 * resolves the array's device address and loads the kernels it launches
 * (with CUDA's lazy module loading, loading may allocate device memory); make
 * that first call before any stream capture. After a device reset do not call
 * it again on that device.
 * Limits: n <= 4096 bodies, <= 32768 body-body and <= 8192 body-plane pairs;
 * beyond them it returns VXB_ERR_CAPACITY (*count still reports the pairs
 * found when the body limit was met; when only `cap` is too small, *count is
 * the number of pairs, so a retry with cap = *count succeeds). Every call
 * shares the array, so calls that overlap on the GPU (other threads or
 * streams) race. Works on the current device and `stream` (null = the
 * default stream); returns after the pairs are in `out`. */
int vxb_stage_pairs_noalloc(const vx_body* bodies, uint32_t n, float dt, uint64_t* out, uint32_t cap,
                            uint32_t* count, void* stream);

/* ---- scene construction (host only) ------------------------------------- */

/* Shape-level specs of a benchmark workload (1..5); `size` overrides its
 * count (lattice side, bodies, pyramids or worlds; 0 = full size). */
int vxb_scene_generate(int config, uint64_t seed, uint32_t size, vx_shape_spec* specs,
                       uint32_t cap, uint32_t* count, vx_vec3* pool, uint32_t poolCap,
                       uint32_t* poolCount);
/* Bodies + hull soup from specs, following World::add* (src/world.cpp:646-985). */
int vxb_bodies_from_specs(const vx_shape_spec* specs, uint32_t n, const vx_vec3* pool,
                          vx_body* bodies, vx_vec3* hullPoints, uint32_t hullCap,
                          uint32_t* hullCount, uint32_t* faceIndices, uint32_t faceCap,
                          uint32_t* faceIndexCount);

#pragma GCC visibility pop

#ifdef __cplusplus
}  /* extern "C" */
#endif

#endif /* VELOX_B200_H */
