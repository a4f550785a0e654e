// Backend context: device buffers and the step orchestration of one
// pipeline instance (the role of class CudaBackend, src/backend_cuda.cu:350-1017,
// re-planned for the device: SoA body state, device-side counts, no host
// round trips inside a step).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>

#include "coop.cuh"
#include "geom.cuh"
#include "radix_sort.cuh"
#include "tuner.h"
#include "velox_b200.h"

namespace vxb {

// Island decomposition of one step's contacts.
struct IslandPlan {
    uint32_t islands = 0;      // including the null island when present
    uint32_t realIslands = 0;  // islands with a dynamic body
    uint32_t segments = 0;     // (island, colour) runs
    uint32_t contacts = 0;     // contacts in the plan
    uint32_t freeFrom = 0, freeTo = 0;  // contact-free bodies (range in the island-sorted body order)
};

// State of one cooperative launch (zeroed before it, except spinLimit).
struct CoopState {
    GridBarrier bar;
    uint32_t changed[3];  // per-round counters, rotated
    uint32_t spill;       // bit 0: fall back to the serial path; bit 1: no progress
    uint32_t rounds;      // rounds the kernel ran (or a count the launch returns)
    uint32_t timeout;     // a barrier wait gave up
    uint32_t queued[3];   // per-round work-queue lengths, rotated like changed[]
    uint32_t spinLimit;   // polls before any wait of the launch gives up (Context::waitLimit)
    uint32_t pad[4];
};

// Grow-only device allocation.
struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
};

// A snapshot of the device world kept in device memory (snapshot.cu).
constexpr uint32_t kSnapshotSlots = 8;
struct DeviceSnapshot {
    DevBuf buf;                    // body arrays, previous contacts and their keys
    alignas(8) char header[256];   // layout, configuration and statistics at save time
    bool valid = false;
};

// Recording of the device world's steps for the adjoint (adjoint.cu).
struct Tape {
    bool active = false;
    uint32_t steps = 0, every = 0, recorded = 0;
    std::vector<uint32_t> stepStart{0u};  // first contact of each recorded step (+ total)
    DevBuf contacts;    // vx_contact per contact, after warm-start matching
    DevBuf src;         // uint2 per contact: impulse source, vn0 source (previous step's index)
    DevBuf color;       // uint32 per contact
    DevBuf worldStart;  // steps x (worlds + 1): first contact of each world within its step
    DevBuf ckpt;        // (J + 1) x 4 x n float4: body state every k steps, then the final state
    DevBuf flags;       // uint32 per world (VXB_ADJ_*)
    DevBuf scratch;     // backward: per-world working memory
    DevBuf host;        // backward: small device arrays (body ranges, seeds, gradients)
    DevBuf branches;    // backward: branch decisions, when requested
};

// Device-side counters and flags (one small allocation, read back once per call).
struct Counters {
    uint32_t pairs;          // convex candidate pairs emitted (may exceed capacity)
    uint32_t planePairs;     // body-plane candidate pairs emitted
    uint32_t contactsTmp;    // contacts appended by the narrow phase
    uint32_t records;        // pairs with at least one contact
    uint32_t contacts;       // contacts after placement (== contactsTmp when no overflow)
    uint32_t islands;        // contact islands
    uint32_t segments;       // (island, colour) segments
    uint32_t maxColors;      // largest colour count of an island
    uint32_t largestIsland;  // contacts in the largest island
    uint32_t caCandidates;   // pairs visited by the serial rewind pass
    uint32_t rewinds;        // conservative-advancement rewinds
    uint32_t caOverflow;     // rewind cascade left the 1-hop candidate set
    uint32_t warmStarted;    // contacts that inherited impulses
    uint32_t overflow;       // bit 0 pairs, bit 1 contacts, bit 2 records
    uint32_t timeout;        // a bounded device wait gave up
    uint32_t cellMinBits[3]; // ordered-int encodings of the minimum AABB centre
    uint32_t cellMaxBits[3]; // ordered-int encodings of the maximum AABB centre
    uint32_t extentBits;     // float bits of the largest non-plane AABB extent
    uint32_t worldBits;      // bits of the world id in cell keys
    uint32_t lastIslandKey;  // island key of the last contact (n = the null island)
    uint32_t maxIslandSize;  // contacts of the largest island (before colouring)
    uint32_t freeFrom, freeTo;  // contact-free bodies: range in the island-sorted body order
    uint32_t planFault;      // a solve kernel found an inconsistent island plan
    uint32_t caGapQueries;   // distance queries of the rewind passes
    uint32_t caCritMicros;   // rewind: evaluation time along the longest dependency chain
    uint32_t caSpecMicros;   // rewind: the longest single speculated pair
    uint32_t tinyIslands;    // islands of at most tinyLimit contacts (packed solve)
    uint32_t tinyPacks;      // warps they were packed into
    uint32_t caFlagged;      // pairs the rewind probe flagged
    uint32_t clusterBodies;  // bodies of the giant islands (clustered solve)
    uint32_t clusterRows;    // their rows
    uint32_t clusterColours; // most colours of a giant island
    uint32_t giantCount;     // islands the block kernels cannot hold
    uint32_t pad[1];
};

// Pipeline stages timed with CUDA events when timing is enabled.
enum Stage : int {
    kStagePrepare = 0, kStageBroadphase, kStageCellSort, kStageNarrowphase, kStagePlacement,
    kStageWarmStart, kStageIslands, kStageSolve, kStageRewind, kStagePositions, kStageCount
};

struct StageTimer {
    std::vector<cudaEvent_t> pool;         // free events
    std::vector<cudaEvent_t> open[kStageCount];
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> done[kStageCount];
    double ms[kStageCount] = {};
    uint64_t calls[kStageCount] = {};
};

// Island sleeping and contact events of the device world (sleep.cu).
struct SleepState {
    vxb_sleep_config config{};
    bool events = false;          // record contact events (vxb_world_enable_events)
    uint32_t sleepable = 0;       // dynamic bodies loaded with enableSleep
    uint32_t asleep = 0;          // bodies asleep after the last step (an upper bound between steps)
    uint32_t pairCount = 0;       // pair keys of the last step (active and resting pairs)
    uint32_t eventCount = 0;      // events of the last step
    DevBuf state;                 // float4 per body: sleepTimer, stable frames, state (0/1/2), enableSleep
    DevBuf pairs;                 // sorted unique pair keys of the last step
    DevBuf pairsNext, eventBuf;   // this step's pair keys (unsorted) and events
    DevBuf keys, vals, flags, ranks, small, list, parent, bodyBits, kept, merge;
};

struct Context {
    int device = 0;
    int smCount = 148;
    int cooperative = 0;  // cudaDevAttrCooperativeLaunch
    uint32_t caRounds = 0;     // rewind dependency depth of the last step (all passes)
    uint32_t caWidenings = 0;  // rewind replays with a widened body set (last step)
    uint32_t planContacts = 0; // contacts of the current island plan
    uint32_t planGiants = 0;   // giant islands of the current plan
    bool giantLinked = false;  // dataflow links of the plan's giant islands are built
    bool clusterBuilt = false; // spatial clusters of the plan's giant islands are built
    bool tinyPacked = false;   // the plan's tiny islands are packed into warps
    uint32_t tinyCount = 0, tinyPackCount = 0;
    uint32_t clusterNB = 0, clusterR = 0, clusterG = 0;  // giant bodies, rows, most colours (clustered solve)
    uint32_t waitLimit = kSpinLimit;  // polls before a device wait gives up (vxb_context_set_wait_limit)
    cudaStream_t ownStream = nullptr;
    cudaStream_t stream = nullptr;
    std::string lastError;
    uint64_t launches = 0;
    uint64_t hostSyncs = 0;  // blocking reads of device counts (the stream drains)
    Tuner tuner;             // launch shapes of the narrow phase and the rewind probe

    // ---- bodies ----
    uint32_t n = 0;
    uint32_t worlds = 1;
    DevBuf bodyBuf;     // all SoA arrays in one allocation
    BodyArrays B{};
    DevBuf aosBuf;      // vx_body staging (upload / download)
    DevBuf worldOfBuf;  // uint32 world id per body
    DevBuf planeStartBuf, planeListBuf;  // per-world plane CSR
    DevBuf prevPoseBuf;                  // float4 prevPos[n], prevRot[n]
    DevBuf snapBuf;                      // call-start snapshot of the mutable state
    std::vector<uint32_t> hostWorldOf;
    bool hasKinematic = false;

    // ---- soup ----
    DevBuf hullPtsBuf, facesBuf;
    size_t hullPointCount = 0, faceIndexCount = 0;
    // triangle meshes and compound children of the soup (static geometry)
    DevBuf vertBuf, indexBuf, meshBuf, nodeBuf, triRefBuf, childBuf;
    DevBuf jointBuf;  // joints of the Backend path, in colour order
    std::vector<vx_mesh> hostMeshes;   // root bounds for the broad phase
    bool complexShapes = false;        // any mesh or compound body loaded
    bool kinematic = false;            // any kinematic body loaded (Backend path)
    // FNV-1a keys of the loaded bodies' shape references and of the soup's
    // array sizes (a snapshot image restores only into the same geometry)
    uint64_t bodyGeometryKey = 0, soupGeometryKey = 0;

    // ---- broad phase ----
    DevBuf aabbBuf;      // float4 lo[n], hi[n]
    DevBuf cellKeyBuf, cellValBuf;
    RadixScratch sortScratch;
    DevBuf sortKeysAlt, sortValsAlt, sortHist;
    DevBuf hashKeyBuf, hashValBuf;
    uint32_t hashCap = 0;
    DevBuf pairBuf;            // convex pairs, then plane pairs
    uint32_t pairCap = 0;
    uint32_t convexPairs = 0;  // last broad phase: convex pairs at [0, convexPairs) of pairBuf
    uint32_t planePairs = 0;   // and plane pairs at [pairCap, pairCap + planePairs)
    std::vector<uint32_t> hostPlaneStart;

    // ---- narrow phase ----
    DevBuf contactTmpBuf;
    uint32_t contactCap = 0;
    DevBuf recKeyBuf, recValBuf, recInfoBuf, recCountBuf;
    uint32_t recCap = 0;
    DevBuf contactBuf[2];  // key-sorted contacts: current / previous step
    int cur = 0;
    uint32_t prevCount = 0;     // contacts held in contactBuf[cur ^ 1]
    uint32_t stepContacts = 0;  // of those, the last step's own (the rest: resting pairs kept for warm starting)
    DevBuf stepPosBuf;          // positions of the last step's own contacts in the cache (when some are kept)
    DevBuf prevKeyBuf;          // (a<<32|b) of the previous contacts
    DevBuf pairKeyBuf;          // (a<<32|b) per record in sorted order (CA pairs)
    DevBuf recOffsetBuf;        // first contact of each sorted record

    // ---- islands / colouring ----
    DevBuf parentBuf, islandOfBodyBuf;
    DevBuf islandKeyBuf, islandValBuf;  // per contact
    DevBuf colorBuf;                    // colour per contact (key-sorted index)
    DevBuf colorKeyBuf;                 // (island << 16 | colour) in island order
    DevBuf maskBuf, nextColorBuf;       // per body
    DevBuf islandStartBuf, islandInfoBuf;  // per island
    DevBuf flagBuf, scanBuf, scanTmp;
    DevBuf segStartBuf, islandSegBuf;
    DevBuf bodyKeyBuf, bodyValBuf, islandBodyStartBuf;
    DevBuf caFlagBuf, caBodyMarkBuf, caCandBuf, caSpecBuf;
    DevBuf localIdxBuf;                 // island-local body index (block solve)
    DevBuf prepBuf, frameBuf;           // per-row pose terms / per-body inertia frames (solve)
    DevBuf fpKeyBuf, fpValBuf, fpSlotBuf, fpColorBuf, fpRunStartBuf, fpIslandBuf;  // parallel colouring
    DevBuf coopBuf;                     // CoopState of cooperative launches
    DevBuf giantBuf;                    // giant island list (solve)
    DevBuf classKeyBuf, classValBuf;    // convex pairs grouped by shape combination (narrow phase)
    DevBuf rowBodyBuf;                  // (a, b) per solve-order row (giant islands)
    DevBuf tinyBuf;                     // tiny-island flags, ranks, list, pack counts/bases/firsts
    DevBuf tinyKeyBuf;                  // tiny islands' colour counts (pack order sort)
    DevBuf clusterInfoBuf, clusterKeyBuf, clusterValBuf, clusterOfBuf, clusterCountBuf, clusterStartBuf,
        clusterRowsBuf;                 // spatial clusters of a giant island
    DevBuf clusterLinkBuf;              // cross-cluster predecessor links + remote-successor flags
    DevBuf caInfoBuf;                   // rewind pass: one record per candidate
    DevBuf tuneSaveBuf;                 // launch-shape trials: device copy of the counters

    DevBuf countersBuf;
    Counters* dCounters = nullptr;
    Counters hostCounters{};

    // ---- configuration ----
    vxb_step_config config{};
    bool configured = false;
    vxb_step_stats stats{};

    // ---- Backend-interface mode ----
    uint32_t backendContacts = 0;   // contacts resident after a find / solve
    bool backendColored = false;
    int backendSweeps = 0;
    vx_solver_options backendOptions{};
    std::vector<vx_contact> hostSorted;
    IslandPlan backendPlan;

    bool timing = false;
    StageTimer timer;

    Tape tape;
    SleepState sleep;
    DeviceSnapshot snapshots[kSnapshotSlots];

    cudaError_t err = cudaSuccess;
};

void stageBegin(Context& c, int stage);
void stageEnd(Context& c, int stage);
int stageResolve(Context& c);

// Records a failure on the context; returns the mapped status.
int fail(Context& c, int status, const std::string& message);
int cudaStatus(Context& c, cudaError_t e, const char* what);

// Zeroes a cooperative launch's state on the context's stream and sets its
// wait limit to the context's.
int resetCoop(Context& c, CoopState* st);

// Grow-only device allocation helper; returns VXB_OK or VXB_ERR_OOM.
int ensure(Context& c, DevBuf& b, size_t bytes);

// Pipeline entry points (pipeline.cu).
// deviceWorld: the device-resident world (vxb_world_load), which does not take
// kinematic bodies; the Backend and stage paths do.
int loadBodies(Context& c, const vx_body* bodies, uint32_t n, const uint32_t* worldOf, bool deviceWorld = false);
int loadSoup(Context& c, const vx_soup* soup);
int readBodies(Context& c, vx_body* out, uint32_t n);
int worldStep(Context& c, int steps);
int stagePairs(Context& c, float dt, uint64_t* out, uint32_t cap, uint32_t* count);
int stageCollide(Context& c, const uint64_t* pairs, uint32_t npairs, float dt, vx_contact* out,
                 uint32_t cap, uint32_t* counts, uint32_t* total);
int stageColor(Context& c, const vx_contact* contacts, uint32_t m, int32_t* colorOf, uint32_t* numColors);
int stageDistance(Context& c, const uint64_t* pairs, uint32_t npairs, int path, float* out);
int backendIntegrate(Context& c, vx_vec3 gravity, float dt);
int backendIntegrateTransforms(Context& c, float dt);
// advanceSubsteps one substep at a time, as the reference CUDA backend runs
// it (joints.cu): contact sweeps, optional joint sweeps, then the integration
// of every body (kinematic ones too) each substep. Bodies must be loaded.
int backendStepwise(Context& c, vx_body* bodies, uint32_t n, vx_contact* contacts, uint32_t m, vx_joint* joints,
                    uint32_t njoints, vx_vec3 gravity, float h, int substeps, const vx_solver_options& o,
                    uint32_t* iterations);
// The reference CUDA backend's joint path of advanceSubsteps (joints.cu).
int backendAdvanceJoints(Context& c, vx_body* bodies, uint32_t n, vx_contact* contacts, uint32_t m,
                         vx_joint* joints, uint32_t njoints, vx_vec3 gravity, float h, int substeps,
                         const vx_solver_options& o, int* advanced, uint32_t* iterations);
int backendFindContacts(Context& c, float dt, uint32_t* count);
int backendCopyContacts(Context& c, vx_contact* out, uint32_t cap);
int backendSolve(Context& c, vx_contact* contacts, uint32_t m, float h, bool warmStart,
                 const vx_solver_options& options, vx_vec3 gravity, int substeps, bool fullSubsteps);
int backendFetchImpulses(Context& c, vx_contact* contacts, uint32_t m);
int readPoses(Context& c, float* out, uint32_t n);
int writeForces(Context& c, const float* in, uint32_t n);
int readContacts(Context& c, vx_contact* out, uint32_t cap, uint32_t* count);
int writeContacts(Context& c, const vx_contact* contacts, uint32_t m);
// Island sleeping and contact events (sleep.cu).
int sleepLoad(Context& c, const vx_body* host, uint32_t n);
int sleepExport(Context& c, vx_body* aosDevice);
bool sleepActive(const Context& c);
int wakePass(Context& c, const vx_contact* cs, uint32_t m);
int sleepAndEvents(Context& c, const vx_contact* cs, uint32_t m, float dt, uint32_t* kept);
int mergeKeptContacts(Context& c, uint32_t m, uint32_t kept);
int readEvents(Context& c, vxb_contact_event* out, uint32_t cap, uint32_t* count);
int readStepContacts(Context& c, vx_contact* out, uint32_t m);
void sleepConfigDefault(vxb_sleep_config* c);
// Pipeline pieces the sleep pass shares (pipeline.cu).
int sortPairs(Context& c, uint64_t* keys, uint32_t* vals, uint32_t n, int bits);
int exclusiveScan(Context& c, const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* grandTotal);
int unionRoots(Context& c, const vx_contact* cs, uint32_t m, uint32_t* parent);

// Snapshots of the device world (snapshot.cu).
int snapshotSave(Context& c, uint32_t slot);
int snapshotRestore(Context& c, uint32_t slot);
int snapshotBytes(Context& c, size_t* bytes);
int snapshotRead(Context& c, void* out, size_t capacity);
int snapshotWrite(Context& c, const void* in, size_t size);

// Input validation (validate.cpp), the reference's per-step checks of public state.
bool validBody(const vx_body& b, const vx_soup* soup, std::string& why);
bool validComplexRefs(const vx_body& b, const vx_soup* soup, std::string& why);
bool validSoup(const vx_soup* soup, std::string& why);
bool validSolverOptions(const vx_solver_options& o, std::string& why);
bool finiteValues(const float* v, size_t count);

// Adjoint (adjoint.cu): tape hooks of the device world's step, and the backward pass.
int tapeBegin(Context& c, uint32_t steps, uint32_t every);
int tapeEnd(Context& c);
int tapeStepBegin(Context& c);
int tapeBeforeMatch(Context& c, const vx_contact* cs, uint32_t m, const vx_contact* prev, const uint64_t* prevKeys,
                    uint32_t mPrev);
int tapeAfterMatch(Context& c, const vx_contact* cs, uint32_t m);
int tapeAfterIslands(Context& c, const uint32_t* color, uint32_t m);
int tapeAfterRewind(Context& c, const uint32_t* rewound);
int tapeStepEnd(Context& c, uint32_t m);
int tapeRead(Context& c, vx_contact* contacts, uint32_t* stepStart, uint32_t* src, int32_t* color, float* ckpt,
             uint32_t* worldFlags);
int adjointBackward(Context& c, const float* seed, float* grad, float* gradInv, float* gradMass,
                    uint32_t* worldFlags, uint8_t* branches = nullptr, size_t branchCapacity = 0,
                    size_t* branchBytes = nullptr, uint32_t* branchRows = nullptr);

}  // namespace vxb
