// The per-step contact pipeline on the device.
//
// Step structure (src/world.cpp:3830-4521 with the CUDA backend's
// advanceSubsteps, src/backend_cuda.cu:691-761):
//   prepare      orientation normalisation, first-substep gravity, pre-solve poses
//   broad phase  swept AABBs, cell keys (world id in the high bits), radix sort,
//                cell hash table, 27-cell pair emission + per-world plane pairs
//   narrow phase collidePair per candidate pair, contacts sorted by (a, b, point)
//   warm start   impulse matching against the previous step's contacts
//   islands      union-find over dynamic-dynamic contacts; contacts grouped by
//                island keep their global order, so island-local greedy
//                colouring equals the reference's global greedy colouring and
//                island-local colour order equals its global colour order
//   solve        one launch runs every island's whole substep loop
//                (integration, warm start, 2*velocityIterations coloured
//                sweeps, transform integration); tiny islands run one thread
//                each, larger ones a block with a barrier between colours
//   rewind       conservative advancement for deep end-of-step overlaps
//   correction   split-impulse position correction, coloured per island
#include <algorithm>
#include <cstddef>
#include <cstring>

#include "context.cuh"

namespace vxb {

static_assert(sizeof(vx_contact) == 128 && offsetof(vx_contact, spinningImpulse) == 116,
              "contact record: 120 bytes of fields, 8 of padding");

// ---------------------------------------------------------------------------
// host helpers
// ---------------------------------------------------------------------------

int fail(Context& c, int status, const std::string& message) {
    c.lastError = message;
    return status;
}

int cudaStatus(Context& c, cudaError_t e, const char* what) {
    if (e == cudaSuccess) return VXB_OK;
    std::string msg = std::string("velox_b200 CUDA failure: ") + cudaGetErrorString(e) + " (" + what + ")";
    if (e == cudaErrorMemoryAllocation) return fail(c, VXB_ERR_OOM, msg);
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return fail(c, VXB_ERR_NO_DEVICE, msg);
    if (e == cudaErrorLaunchFailure || e == cudaErrorLaunchTimeout || e == cudaErrorUnknown ||
        e == cudaErrorIllegalAddress || e == cudaErrorDevicesUnavailable)
        return fail(c, VXB_ERR_DEVICE_LOST, msg);
    return fail(c, VXB_ERR_INVALID, msg);
}

int ensure(Context& c, DevBuf& b, size_t bytes) {
    if (bytes <= b.bytes && b.ptr) return VXB_OK;
    if (b.ptr) cudaFree(b.ptr);
    b.ptr = nullptr;
    b.bytes = 0;
    size_t want = bytes + bytes / 2 + 256;
    cudaError_t e = cudaMalloc(&b.ptr, want);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return cudaStatus(c, e, "cudaMalloc");
    }
    b.bytes = want;
    return VXB_OK;
}

template <class T> T* P(DevBuf& b) { return reinterpret_cast<T*>(b.ptr); }

static cudaEvent_t takeEvent(Context& c) {
    if (c.timer.pool.empty()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        return e;
    }
    cudaEvent_t e = c.timer.pool.back();
    c.timer.pool.pop_back();
    return e;
}

void stageBegin(Context& c, int stage) {
    if (!c.timing) return;
    cudaEvent_t e = takeEvent(c);
    cudaEventRecord(e, c.stream);
    c.timer.open[stage].push_back(e);
}

void stageEnd(Context& c, int stage) {
    if (!c.timing || c.timer.open[stage].empty()) return;
    cudaEvent_t e = takeEvent(c);
    cudaEventRecord(e, c.stream);
    c.timer.done[stage].push_back({c.timer.open[stage].back(), e});
    c.timer.open[stage].pop_back();
}

// Folds completed event pairs into the per-stage totals.
int stageResolve(Context& c) {
    cudaError_t e = cudaStreamSynchronize(c.stream);
    if (e != cudaSuccess) return cudaStatus(c, e, "stage timing");
    for (int s = 0; s < kStageCount; ++s) {
        for (auto& pr : c.timer.done[s]) {
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, pr.first, pr.second);
            c.timer.ms[s] += ms;
            c.timer.calls[s] += 1;
            c.timer.pool.push_back(pr.first);
            c.timer.pool.push_back(pr.second);
        }
        c.timer.done[s].clear();
    }
    return VXB_OK;
}

#define VXB_TRY(expr)                  \
    do {                               \
        int s_ = (expr);               \
        if (s_ != VXB_OK) return s_;   \
    } while (0)

#define VXB_CUDA(c, expr)                                             \
    do {                                                              \
        cudaError_t e_ = (expr);                                      \
        if (e_ != cudaSuccess) return cudaStatus((c), e_, #expr);     \
    } while (0)

static inline uint32_t blocksFor(uint64_t items, int threads, uint32_t cap = 65535u * 16u) {
    uint64_t b = (items + threads - 1) / threads;
    if (b == 0) b = 1;
    return (uint32_t)std::min<uint64_t>(b, cap);
}

static inline int bitsFor(uint64_t maxValue) { return keyBits(maxValue); }

#define LAUNCH(c, kernel, grid, block, ...)                                  \
    do {                                                                     \
        kernel<<<(grid), (block), 0, (c).stream>>>(__VA_ARGS__);            \
        ++(c).launches;                                                      \
    } while (0)


// ---------------------------------------------------------------------------
// device helpers
// ---------------------------------------------------------------------------

VXD uint32_t orderedBits(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
VXD float fromOrdered(uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}
VXD uint64_t mix64(uint64_t k) {
    k ^= k >> 33; k *= 0xff51afd7ed558ccdull; k ^= k >> 33; k *= 0xc4ceb9fe1a85ec53ull; k ^= k >> 33;
    return k;
}
VXD unsigned laneMaskLt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}
// Warp-aggregated slot reservation for the currently active lanes.
VXD uint32_t aggregatedSlot(uint32_t* counter) {
    const unsigned active = __activemask();
    const int leader = __ffs(active) - 1;
    const int lane = threadIdx.x & 31;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(active));
    base = __shfl_sync(active, base, leader);
    return base + __popc(active & laneMaskLt());
}

VXD Mass loadMass(const BodyArrays& B, uint32_t i) {
    const float4 in = B.inertia[i];
    Mass m;
    m.invI = V3{in.x, in.y, in.z};
    m.invMass = in.w;
    m.iq = q4(B.iq[i]);
    m.flags = B.filt[i].x;
    return m;
}

VXD SolverBody loadSolverBody(const BodyArrays& B, uint32_t i) {
    SolverBody s;
    s.p = f3(B.pos[i]);
    s.q = q4(B.rot[i]);
    s.v = f3(B.vel[i]);
    s.w = f3(B.ang[i]);
    s.m = loadMass(B, i);
    s.sphere = shapeOf(s.m.flags) == kSphere;
    return s;
}

VXD void loadRow(const vx_contact& c, RowContact& r) {
    r.normal = V3{c.normal.x, c.normal.y, c.normal.z};
    r.point = V3{c.point.x, c.point.y, c.point.z};
    r.la = V3{c.localAnchorA.x, c.localAnchorA.y, c.localAnchorA.z};
    r.lb = V3{c.localAnchorB.x, c.localAnchorB.y, c.localAnchorB.z};
    r.bias0 = c.bias0; r.vn0 = c.vn0; r.restitution = c.restitution;
    r.friction1 = c.friction1; r.friction2 = c.friction2;
    r.rolling = c.rollingFriction; r.spinning = c.spinningFriction;
    r.nImp = c.normalImpulse; r.t1Imp = c.tangentImpulse1; r.t2Imp = c.tangentImpulse2;
    r.r1Imp = c.rollingImpulse1; r.r2Imp = c.rollingImpulse2; r.sImp = c.spinningImpulse;
}
VXD void storeRow(vx_contact& c, const RowContact& r) {
    c.point = vx_vec3{r.point.x, r.point.y, r.point.z};
    c.normalImpulse = r.nImp; c.tangentImpulse1 = r.t1Imp; c.tangentImpulse2 = r.t2Imp;
    c.rollingImpulse1 = r.r1Imp; c.rollingImpulse2 = r.r2Imp; c.spinningImpulse = r.sImp;
}

// integrateKernel semantics (src/backend_cuda.cu:80-89) for body i.
VXD void integrateVelocity(const BodyArrays& B, uint32_t i, const V3& g, float dt) {
    const Mass m = loadMass(B, i);
    if (!isDynamic(m.flags) || isLocked(m.flags) || isAsleep(m.flags)) return;
    const Q4 q = q4(B.rot[i]);
    V3 v = f3(B.vel[i]);
    V3 w = f3(B.ang[i]);
    const V3 F = f3(B.force[i]);
    const V3 T = f3(B.torque[i]);
    const float4 ex = B.extra[i];
    v += (g * ex.y + F * solverInvMass(m)) * dt;
    w += invInertiaMulAt(m, T, q) * dt;
    v *= 1.0f / (1.0f + ex.z * dt);
    w *= 1.0f / (1.0f + ex.w * dt);
    B.vel[i] = pack(v, 0.0f);
    B.ang[i] = pack(w, 0.0f);
}

// integrateTransformsKernel semantics (src/backend_cuda.cu:91-97).
VXD void integrateTransform(const BodyArrays& B, uint32_t i, float dt) {
    const Mass m = loadMass(B, i);
    if (isStaticBody(m.flags) || isLocked(m.flags) || isAsleep(m.flags)) return;
    V3 p = f3(B.pos[i]);
    Q4 q = q4(B.rot[i]);
    const V3 v = f3(B.vel[i]);
    V3 w = f3(B.ang[i]);
    advanceTransform(m, p, q, v, w, dt);
    B.pos[i] = pack(p, 0.0f);
    B.rot[i] = pack(q);
    B.ang[i] = pack(w, 0.0f);
}

// ---------------------------------------------------------------------------
// body packing
// ---------------------------------------------------------------------------

__global__ void packBodiesKernel(const vx_body* __restrict__ in, uint32_t n, BodyArrays B) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const vx_body& b = in[i];
        B.pos[i] = make_float4(b.position.x, b.position.y, b.position.z, 0.0f);
        B.rot[i] = make_float4(b.orientation.x, b.orientation.y, b.orientation.z, b.orientation.w);
        B.vel[i] = make_float4(b.velocity.x, b.velocity.y, b.velocity.z, 0.0f);
        B.ang[i] = make_float4(b.angularVelocity.x, b.angularVelocity.y, b.angularVelocity.z, 0.0f);
        B.inertia[i] = make_float4(b.invInertia.x, b.invInertia.y, b.invInertia.z, b.invMass);
        B.iq[i] = make_float4(b.inertiaOrientation.x, b.inertiaOrientation.y, b.inertiaOrientation.z,
                              b.inertiaOrientation.w);
        B.dims[i] = make_float4(b.halfExtents.x, b.halfExtents.y, b.halfExtents.z, b.radius);
        B.extra[i] = make_float4(b.capsuleHalfHeight, b.gravityScale, b.linearDamping, b.angularDamping);
        B.mat[i] = make_float4(b.friction, b.restitution, b.rollingFriction, b.spinningFriction);
        B.fscale[i] = make_float4(b.frictionScale.x, b.frictionScale.y, b.frictionScale.z,
                                  b.ccdTuning.speculativeDistance);
        B.ccd[i] = make_float4(b.ccdTuning.collisionMargin, b.ccdTuning.minVelocityForCCD, 0.0f, 0.0f);
        B.plane[i] = make_float4(b.planeNormal.x, b.planeNormal.y, b.planeNormal.z, b.planeOffset);
        // the hull word: a mesh keeps its mesh index there, a compound its child range
        B.hull[i] = b.shape == VX_SHAPE_MESH       ? make_uint4(b.meshIndex, 0u, 0u, 0u)
                    : b.shape == VX_SHAPE_COMPOUND ? make_uint4(b.compoundFirst, b.compoundCount, 0u, 0u)
                                                   : make_uint4(b.hullFirst, b.hullCount, b.hullFaceFirst, b.hullFaceCount);
        const uint32_t flags = (uint32_t)(b.shape & 15u) | ((uint32_t)(b.motionType & 3u) << kMotionShift) |
                               ((uint32_t)(b.ccdTuning.quality & 3u) << kQualityShift) |
                               (b.ccdTuning.enableContinuous ? kContinuousBit : 0u) |
                               (b.sensor ? kSensorBit : 0u) | (b.fixedRotation ? kFixedRotationBit : 0u) |
                               (b.asleep == 1 ? kAsleepBit : 0u) |
                               ((uint32_t)(b.frictionCombine & 7u) << kFrictionCombineShift) |
                               ((uint32_t)(b.restitutionCombine & 7u) << kRestitutionCombineShift) |
                               ((uint32_t)(b.geometryQuality & 3u) << kGeomQualityShift);
        B.filt[i] = make_uint4(flags, b.categoryBits, b.maskBits, (uint32_t)b.groupIndex);
        B.force[i] = make_float4(b.force.x, b.force.y, b.force.z, 0.0f);
        B.torque[i] = make_float4(b.torque.x, b.torque.y, b.torque.z, 0.0f);
    }
}

__global__ void unpackBodiesKernel(vx_body* __restrict__ out, uint32_t n, BodyArrays B) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        vx_body& b = out[i];
        float4 t = B.pos[i]; b.position = vx_vec3{t.x, t.y, t.z};
        t = B.rot[i]; b.orientation = vx_quat{t.x, t.y, t.z, t.w};
        t = B.vel[i]; b.velocity = vx_vec3{t.x, t.y, t.z};
        t = B.ang[i]; b.angularVelocity = vx_vec3{t.x, t.y, t.z};
        t = B.force[i]; b.force = vx_vec3{t.x, t.y, t.z};
        t = B.torque[i]; b.torque = vx_vec3{t.x, t.y, t.z};
    }
}

__global__ void posesKernel(float* __restrict__ out, uint32_t n, BodyArrays B) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 p = B.pos[i], q = B.rot[i];
        float* o = out + 7 * (size_t)i;
        o[0] = p.x; o[1] = p.y; o[2] = p.z; o[3] = q.x; o[4] = q.y; o[5] = q.z; o[6] = q.w;
    }
}

__global__ void forcesKernel(const float* __restrict__ in, uint32_t n, BodyArrays B) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float* f = in + 6 * (size_t)i;
        B.force[i] = make_float4(f[0], f[1], f[2], 0.0f);
        B.torque[i] = make_float4(f[3], f[4], f[5], 0.0f);
    }
}

// ---------------------------------------------------------------------------
// prepare: World::stepImpl orientation normalisation (world.cpp:3930),
// first-substep gravity (world.cpp:4014) and the pre-solve poses (:4186-4188)
// ---------------------------------------------------------------------------

__global__ void prepareKernel(BodyArrays B, uint32_t n, V3 g, float h, float4* prevPos, float4* prevRot,
                              int normalizeOrientation) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (normalizeOrientation) B.rot[i] = pack(qnormalize(q4(B.rot[i])));
        integrateVelocity(B, i, g, h);
        if (prevPos) {
            prevPos[i] = B.pos[i];
            prevRot[i] = B.rot[i];
        }
    }
}

__global__ void integrateKernel(BodyArrays B, uint32_t n, V3 g, float h) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        integrateVelocity(B, i, g, h);
}

__global__ void transformsKernel(BodyArrays B, uint32_t n, float h) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        integrateTransform(B, i, h);
}

// ---------------------------------------------------------------------------
// broad phase
// ---------------------------------------------------------------------------

constexpr int kCellBits = 10;  // per axis; coordinates wrap modulo 1024 (exactness kept by the AABB test)
constexpr uint32_t kCellMask = (1u << kCellBits) - 1u;
constexpr uint64_t kEmptySlot = ~0ull;

// Swept AABBs (bodyAabb, narrowphase.h:369-398); planes unbounded, meshes
// their root bounds (src/backend_cuda.cu:100-129). Neither enters the cell
// size or the cell grid's extent.
__global__ void aabbKernel(BodyArrays B, uint32_t n, float dt, const vx_mesh* meshes, float4* lo, float4* hi,
                           Counters* C) {
    float ext = 0.0f;
    float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t flags = B.filt[i].x;
        if (shapeOf(flags) == kPlane) {
            lo[i] = make_float4(-1e30f, -1e30f, -1e30f, 0.0f);
            hi[i] = make_float4(1e30f, 1e30f, 1e30f, 0.0f);
            continue;
        }
        if (shapeOf(flags) == kMesh) {
            const vx_mesh& m = meshes[B.hull[i].x];
            lo[i] = make_float4(m.aabbMin.x, m.aabbMin.y, m.aabbMin.z, 0.0f);
            hi[i] = make_float4(m.aabbMax.x, m.aabbMax.y, m.aabbMax.z, 0.0f);
            continue;
        }
        const V3 p = f3(B.pos[i]);
        const float4 d = B.dims[i];
        const float reach = aabbReach(flags, V3{d.x, d.y, d.z}, d.w, B.extra[i].x, B.ccd[i].x,
                                      f3(B.vel[i]), f3(B.ang[i]), dt);
        const V3 L = p - V3{reach, reach, reach};
        const V3 H = p + V3{reach, reach, reach};
        lo[i] = pack(L, 0.0f);
        hi[i] = pack(H, 0.0f);
        const float e = fmaxf(H.x - L.x, fmaxf(H.y - L.y, H.z - L.z));
        if (e < 1e6f) ext = fmaxf(ext, e);
        const float c[3] = {(L.x + H.x) * 0.5f, (L.y + H.y) * 0.5f, (L.z + H.z) * 0.5f};
        for (int a = 0; a < 3; ++a) { mn[a] = fminf(mn[a], c[a]); mx[a] = fmaxf(mx[a], c[a]); }
    }
    for (int off = 16; off > 0; off >>= 1) {
        ext = fmaxf(ext, __shfl_xor_sync(0xffffffffu, ext, off));
        for (int a = 0; a < 3; ++a) {
            mn[a] = fminf(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], off));
            mx[a] = fmaxf(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], off));
        }
    }
    if ((threadIdx.x & 31) == 0) {
        if (ext > 0.0f) atomicMax(&C->extentBits, __float_as_uint(ext));
        for (int a = 0; a < 3; ++a)
            if (mn[a] <= mx[a]) {
                atomicMin(&C->cellMinBits[a], orderedBits(mn[a]));
                atomicMax(&C->cellMaxBits[a], orderedBits(mx[a]));
            }
    }
}

VXD float cellSizeOf(const Counters* C) {
    float s = __uint_as_float(C->extentBits);
    return s > 0.0f ? s : 1.0f;
}
VXD int cellCoord(float centre, float inv, float minCentre) {
    float f = floorf(centre * inv) - floorf(minCentre * inv);
    f = fminf(fmaxf(f, -1.0e9f), 1.0e9f);
    return (int)f;
}

__global__ void keyKernel(BodyArrays B, uint32_t n, const uint32_t* worldOf, const float4* lo, const float4* hi,
                          const Counters* C, uint64_t* keys, uint32_t* vals, uint64_t planeKey) {
    const float cs = cellSizeOf(C);
    const float inv = 1.0f / cs;
    const float m0 = fromOrdered(C->cellMinBits[0]), m1 = fromOrdered(C->cellMinBits[1]),
                m2 = fromOrdered(C->cellMinBits[2]);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        vals[i] = i;
        const uint32_t shape = shapeOf(B.filt[i].x);
        if (shape == kPlane || shape == kMesh) { keys[i] = planeKey; continue; }
        const float4 L = lo[i], H = hi[i];
        const int cx = cellCoord((L.x + H.x) * 0.5f, inv, m0);
        const int cy = cellCoord((L.y + H.y) * 0.5f, inv, m1);
        const int cz = cellCoord((L.z + H.z) * 0.5f, inv, m2);
        const uint64_t w = worldOf ? worldOf[i] : 0u;
        keys[i] = (w << (3 * kCellBits)) | ((uint64_t)((uint32_t)cz & kCellMask) << (2 * kCellBits)) |
                  ((uint64_t)((uint32_t)cy & kCellMask) << kCellBits) | (uint64_t)((uint32_t)cx & kCellMask);
    }
}

__global__ void cellTableKernel(const uint64_t* keys, uint32_t n, uint64_t planeKey, uint64_t* hk, uint32_t* hv,
                                uint32_t mask) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        const uint64_t key = keys[s];
        if (key == planeKey) continue;
        if (s > 0 && keys[s - 1] == key) continue;
        uint32_t slot = (uint32_t)mix64(key) & mask;
        for (uint32_t probe = 0; probe <= mask; ++probe) {
            const unsigned long long prev = atomicCAS((unsigned long long*)&hk[slot], (unsigned long long)kEmptySlot,
                                                      (unsigned long long)key);
            if (prev == kEmptySlot) { hv[slot] = s; break; }
            slot = (slot + 1) & mask;
        }
    }
}

VXD uint32_t cellLookup(const uint64_t* hk, const uint32_t* hv, uint32_t mask, uint64_t key) {
    uint32_t slot = (uint32_t)mix64(key) & mask;
    for (uint32_t probe = 0; probe <= mask; ++probe) {
        const uint64_t k = hk[slot];
        if (k == key) return hv[slot];
        if (k == kEmptySlot) return 0xffffffffu;
        slot = (slot + 1) & mask;
    }
    return 0xffffffffu;
}

VXD void emitPair(uint64_t pair, uint64_t* pairs, uint32_t cap, uint32_t* counter, Counters* C) {
    const uint32_t slot = aggregatedSlot(counter);
    if (slot < cap) pairs[slot] = pair;
    else atomicOr(&C->overflow, 1u);
}

// Candidate pairs (src/backend_cuda.cu:174-250): the 27 neighbouring cells of
// each body's cell (same world), pairs i<j discovered from i's side, plus the
// planes and meshes of the body's world (the list `planeList`; a mesh pair
// also needs overlapping AABBs). Plane pairs of simple convex bodies go to
// `planePairs`; mesh pairs and a compound's plane pairs join the general
// pairs, whose narrow phase handles every shape.
__global__ void pairKernel(BodyArrays B, uint32_t n, const uint64_t* keys, const uint32_t* vals, const float4* lo,
                           const float4* hi, const uint64_t* hk, const uint32_t* hv, uint32_t mask, uint64_t planeKey,
                           const uint32_t* worldOf, const uint32_t* planeStart, const uint32_t* planeList,
                           uint64_t* pairs, uint32_t cap, uint64_t* planePairs, uint32_t planeCap, Counters* C) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        const uint64_t key = keys[s];
        if (key == planeKey) continue;
        const uint32_t i = vals[s];
        const uint4 fi = B.filt[i];
        const V3 Li = f3(lo[i]), Hi = f3(hi[i]);
        const int cx = (int)(key & kCellMask), cy = (int)((key >> kCellBits) & kCellMask),
                  cz = (int)((key >> (2 * kCellBits)) & kCellMask);
        const uint64_t wbits = key >> (3 * kCellBits);
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    const uint64_t nk = (wbits << (3 * kCellBits)) |
                                        ((uint64_t)((uint32_t)(cz + dz) & kCellMask) << (2 * kCellBits)) |
                                        ((uint64_t)((uint32_t)(cy + dy) & kCellMask) << kCellBits) |
                                        (uint64_t)((uint32_t)(cx + dx) & kCellMask);
                    const uint32_t start = cellLookup(hk, hv, mask, nk);
                    if (start == 0xffffffffu) continue;
                    for (uint32_t t = start; t < n && keys[t] == nk; ++t) {
                        const uint32_t j = vals[t];
                        if (j <= i) continue;
                        if (!aabbOverlap(Li, Hi, f3(lo[j]), f3(hi[j]))) continue;
                        const uint4 fj = B.filt[j];
                        if (inert(fi.x) && inert(fj.x)) continue;
                        if (!canCollide(fi.y, fi.z, (int32_t)fi.w, fj.y, fj.z, (int32_t)fj.w)) continue;
                        emitPair(((uint64_t)i << 32) | j, pairs, cap, &C->pairs, C);
                    }
                }
        const uint32_t w = worldOf ? worldOf[i] : 0u;
        const bool compound = shapeOf(fi.x) == kCompound;
        for (uint32_t k = planeStart[w]; k < planeStart[w + 1]; ++k) {
            const uint32_t p = planeList[k];
            const uint4 fp = B.filt[p];
            const bool mesh = shapeOf(fp.x) == kMesh;
            if (mesh && !aabbOverlap(Li, Hi, f3(lo[p]), f3(hi[p]))) continue;
            if (inert(fi.x) && inert(fp.x)) continue;
            const uint32_t a = i < p ? i : p, b = i < p ? p : i;
            const uint4 fa = a == i ? fi : fp, fb = a == i ? fp : fi;
            if (!canCollide(fa.y, fa.z, (int32_t)fa.w, fb.y, fb.z, (int32_t)fb.w)) continue;
            if (mesh || compound) emitPair(((uint64_t)a << 32) | b, pairs, cap, &C->pairs, C);
            else emitPair(((uint64_t)a << 32) | b, planePairs, planeCap, &C->planePairs, C);
        }
    }
}

// ---------------------------------------------------------------------------
// narrow phase
// ---------------------------------------------------------------------------

VXD bool pointLess(const vx_contact& x, const vx_contact& y) {
    if (x.point.x != y.point.x) return x.point.x < y.point.x;
    if (x.point.y != y.point.y) return x.point.y < y.point.y;
    return x.point.z < y.point.z;
}

// One thread per candidate pair: collidePair into a local buffer, order the
// pair's contacts by point (the host sort of src/backend_cuda.cu:587-595
// within one (a, b) key), append them and a record keyed for the global sort.
// mode 0: key = (a << bodyBits) | b; mode 1: key = pair index, emission order kept.
// Which pair classes one instantiation handles: plane pairs compile to a
// light kernel (high occupancy), convex pairs to the GJK/EPA kernel.
// Mesh and compound pairs (among the general pairs) take a third
// instantiation, launched only when such bodies are loaded.
enum PairClass : int { kAnyPairs = 0, kPlanePairs = 1, kConvexPairs = 2, kComplexPairs = 3 };

// `order` (optional): the pairs in the order to process them (convex pairs
// grouped by shape combination so that a warp runs one code path).
template <int Class>
__global__ void __launch_bounds__(128) collideKernel(BodyArrays B, Soup soup, const uint64_t* pairs,
                                                     const uint32_t* order, uint32_t npairs, float dt, int mode,
                                                     int bodyBits, vx_contact* tmp, uint32_t contactCap,
                                                     uint64_t* recKeys, uint32_t* recVals, uint2* recInfo,
                                                     uint32_t recCap, Counters* C) {
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t rounded = (npairs + 31u) & ~31u;
    for (uint32_t base = blockIdx.x * blockDim.x; base < rounded; base += stride) {
        const uint32_t slot = base + threadIdx.x;
        const uint32_t p = slot < npairs && order ? order[slot] : slot;
        vx_contact buf[kMaxContactsPerPair];
        int count = 0;
        if (slot < npairs) {
            const uint64_t pr = pairs[p];
            const uint32_t i = (uint32_t)(pr >> 32), j = (uint32_t)pr;
            const BodyView a = loadView(B, i);
            const BodyView b = loadView(B, j);
            const bool complex = isComplexShape(shapeOf(a.flags)) || isComplexShape(shapeOf(b.flags));
            if (Class == kAnyPairs) {
                count = collidePair(a, b, i, j, soup, dt, buf, kMaxContactsPerPair);
            } else if (Class == kPlanePairs) {
                if (shapeOf(b.flags) == kPlane) planeConvex(a, b, i, j, soup, dt, buf, kMaxContactsPerPair, count);
                else planeConvex(b, a, j, i, soup, dt, buf, kMaxContactsPerPair, count);
            } else if (Class == kConvexPairs) {
                if (!complex) convexConvex(a, b, i, j, soup, dt, buf, kMaxContactsPerPair, count);
            } else if (complex) {
                count = collidePair(a, b, i, j, soup, dt, buf, kMaxContactsPerPair);
            }
            if (mode == 0)
                for (int x = 1; x < count; ++x) {
                    vx_contact key = buf[x];
                    int y = x - 1;
                    while (y >= 0 && pointLess(key, buf[y])) { buf[y + 1] = buf[y]; --y; }
                    buf[y + 1] = key;
                }
        }
        // Warp-wide exclusive scan of the counts, one atomic per warp.
        const int lane = threadIdx.x & 31;
        uint32_t incl = (uint32_t)count;
        for (int off = 1; off < 32; off <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, off);
            if (lane >= off) incl += y;
        }
        const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
        const unsigned hasMask = __ballot_sync(0xffffffffu, count > 0);
        uint32_t cbase = 0, rbase = 0;
        if (lane == 0 && total) {
            cbase = atomicAdd(&C->contactsTmp, total);
            rbase = atomicAdd(&C->records, (uint32_t)__popc(hasMask));
        }
        cbase = __shfl_sync(0xffffffffu, cbase, 0);
        rbase = __shfl_sync(0xffffffffu, rbase, 0);
        if (count > 0) {
            const uint32_t off = cbase + incl - (uint32_t)count;
            const uint32_t rec = rbase + __popc(hasMask & laneMaskLt());
            if (off + (uint32_t)count > contactCap || rec >= recCap) {
                atomicOr(&C->overflow, 2u);
            } else {
                for (int x = 0; x < count; ++x) {
                    tmp[off + x] = buf[x];
                    // the record's 8 tail bytes are padding: zero them so contact
                    // images (snapshots, read-back) are deterministic bytes
                    *reinterpret_cast<uint2*>(reinterpret_cast<char*>(tmp + off + x) + 120) = make_uint2(0u, 0u);
                }
                recKeys[rec] = mode == 0 ? (((uint64_t)buf[0].a << bodyBits) | buf[0].b) : (uint64_t)p;
                recVals[rec] = rec;
                recInfo[rec] = make_uint2(off, (uint32_t)count);
            }
        }
    }
}

__global__ void gatherCountsKernel(const uint32_t* recVals, const uint2* recInfo, uint32_t nrec, uint32_t* counts) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nrec; k += gridDim.x * blockDim.x)
        counts[k] = recInfo[recVals[k]].y;
}

// Shape combination of each convex pair (the processing-order sort key).
__global__ void pairClassKernel(const BodyArrays B, const uint64_t* pairs, uint32_t npairs, uint64_t* keys,
                                uint32_t* vals) {
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < npairs; p += gridDim.x * blockDim.x) {
        const uint64_t pr = pairs[p];
        const uint32_t sa = shapeOf(B.filt[(uint32_t)(pr >> 32)].x), sb = shapeOf(B.filt[(uint32_t)pr].x);
        keys[p] = (uint64_t)(sa * 16u + sb);
        vals[p] = p;
    }
}

// Copies each record's contacts to their sorted position.
__global__ void placeKernel(const uint32_t* recVals, const uint2* recInfo, const uint32_t* offsets, uint32_t nrec,
                            const vx_contact* tmp, vx_contact* out, uint64_t* contactKeys, uint64_t* pairKeys,
                            uint32_t* recOffset) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nrec; k += gridDim.x * blockDim.x) {
        const uint2 info = recInfo[recVals[k]];
        const uint32_t dst = offsets[k];
        const float4* src = reinterpret_cast<const float4*>(tmp + info.x);
        float4* d = reinterpret_cast<float4*>(out + dst);
        for (uint32_t x = 0; x < info.y * 8u; ++x) d[x] = src[x];
        const uint64_t key = ((uint64_t)tmp[info.x].a << 32) | tmp[info.x].b;
        if (contactKeys)
            for (uint32_t x = 0; x < info.y; ++x) contactKeys[dst + x] = key;
        if (pairKeys) pairKeys[k] = key;
        if (recOffset) recOffset[k] = dst;
    }
}

// Multi-block exclusive scan: per-block sums, a single-block scan of the sums,
// then per-block scans with the carried offsets.
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr uint32_t kScanTile = kScanThreads * kScanItems;

__device__ uint32_t blockExclusiveScan(uint32_t v, uint32_t* warpSums, uint32_t* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, off);
        if (lane >= off) x += y;
    }
    if (lane == 31) warpSums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        uint32_t w = lane < nw ? warpSums[lane] : 0u;
        for (int off = 1; off < 32; off <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, off);
            if (lane >= off) w += y;
        }
        warpSums[lane] = w;
    }
    __syncthreads();
    const uint32_t r = x - v + (warp > 0 ? warpSums[warp - 1] : 0u);
    if (total) *total = warpSums[(blockDim.x >> 5) - 1];
    __syncthreads();
    return r;
}

__global__ void scanReduceKernel(const uint32_t* in, uint32_t n, uint32_t* blockSums) {
    __shared__ uint32_t ws[32];
    const uint32_t base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    uint32_t s = 0;
    for (int k = 0; k < kScanItems; ++k)
        if (base + k < n) s += in[base + k];
    uint32_t total;
    blockExclusiveScan(s, ws, &total);
    if (threadIdx.x == 0) blockSums[blockIdx.x] = total;
}

__global__ void scanSumsKernel(uint32_t* sums, uint32_t len) {
    __shared__ uint32_t ws[32];
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (uint32_t start = 0; start < len; start += blockDim.x) {
        const uint32_t i = start + threadIdx.x;
        const uint32_t v = i < len ? sums[i] : 0u;
        uint32_t total;
        const uint32_t ex = blockExclusiveScan(v, ws, &total);
        if (i < len) sums[i] = carry + ex;
        __syncthreads();
        if (threadIdx.x == 0) carry += total;
        __syncthreads();
    }
}

__global__ void scanApplyKernel(const uint32_t* in, uint32_t n, const uint32_t* blockSums, uint32_t* out,
                                uint32_t* grandTotal) {
    __shared__ uint32_t ws[32];
    const uint32_t base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t s = 0;
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = base + k < n ? in[base + k] : 0u;
        s += v[k];
    }
    uint32_t total;
    uint32_t ex = blockExclusiveScan(s, ws, &total) + blockSums[blockIdx.x];
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < n) out[base + k] = ex;
        ex += v[k];
    }
    if (grandTotal && blockIdx.x == gridDim.x - 1 && threadIdx.x == blockDim.x - 1) *grandTotal = ex;
}

int exclusiveScan(Context& c, const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* grandTotal) {
    if (n == 0) return VXB_OK;
    const uint32_t blocks = (n + kScanTile - 1) / kScanTile;
    VXB_TRY(ensure(c, c.scanTmp, (size_t)blocks * 4 + 16));
    uint32_t* sums = P<uint32_t>(c.scanTmp);
    LAUNCH(c, scanReduceKernel, blocks, kScanThreads, in, n, sums);
    LAUNCH(c, scanSumsKernel, 1, 1024, sums, blocks);
    LAUNCH(c, scanApplyKernel, blocks, kScanThreads, in, n, sums, out, grandTotal);
    return VXB_OK;
}

// ---------------------------------------------------------------------------
// warm-start matching (src/world.cpp:4133-4184)
// ---------------------------------------------------------------------------

__global__ void matchKernel(vx_contact* cur, uint32_t m, const vx_contact* prev, const uint64_t* prevKeys,
                            uint32_t mPrev, Counters* C) {
    uint32_t warm = 0;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
        vx_contact c = cur[k];
        const uint64_t key = ((uint64_t)c.a << 32) | c.b;
        uint32_t lo = 0, hi = mPrev;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (prevKeys[mid] < key) lo = mid + 1;
            else hi = mid;
        }
        bool copied = false;
        bool matched = false;
        if (c.featureKey != 0) {
            for (uint32_t it = lo; it < mPrev && prevKeys[it] == key; ++it) {
                const vx_contact& p = prev[it];
                if (p.featureKey == c.featureKey) {
                    c.normalImpulse = p.normalImpulse; c.tangentImpulse1 = p.tangentImpulse1;
                    c.tangentImpulse2 = p.tangentImpulse2; c.rollingImpulse1 = p.rollingImpulse1;
                    c.rollingImpulse2 = p.rollingImpulse2; c.spinningImpulse = p.spinningImpulse;
                    if (c.vn0 < -1.0f && p.vn0 < c.vn0) c.vn0 = p.vn0;
                    matched = copied = true;
                    break;
                }
            }
        }
        if (!matched) {
            if (c.vn0 < -1.0f)
                for (uint32_t it = lo; it < mPrev && prevKeys[it] == key; ++it)
                    if (prev[it].vn0 < c.vn0) c.vn0 = prev[it].vn0;
            float best = 2.5e-3f;
            for (uint32_t it = lo; it < mPrev && prevKeys[it] == key; ++it) {
                const vx_contact& p = prev[it];
                const V3 d{p.point.x - c.point.x, p.point.y - c.point.y, p.point.z - c.point.z};
                const float ds = lengthSq(d);
                if (ds < best) {
                    best = ds;
                    c.normalImpulse = p.normalImpulse; c.tangentImpulse1 = p.tangentImpulse1;
                    c.tangentImpulse2 = p.tangentImpulse2; c.rollingImpulse1 = p.rollingImpulse1;
                    c.rollingImpulse2 = p.rollingImpulse2; c.spinningImpulse = p.spinningImpulse;
                    copied = true;
                }
            }
        }
        if (copied) ++warm;
        cur[k] = c;
    }
    for (int off = 16; off > 0; off >>= 1) warm += __shfl_xor_sync(0xffffffffu, warm, off);
    if ((threadIdx.x & 31) == 0 && warm) atomicAdd(&C->warmStarted, warm);
}

// ---------------------------------------------------------------------------
// islands and colouring
// ---------------------------------------------------------------------------

__global__ void iotaKernel(uint32_t* a, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] = i;
}

// Union-find root with path halving. Parent links are read with ld.global.cg
// (L2, not the SM's L1): other SMs relink roots concurrently and a stale L1
// line would otherwise keep a thread spinning on an outdated root.
VXD uint32_t ufFind(uint32_t* parent, uint32_t x) {
    uint32_t p = __ldcg(parent + x);
    while (p != x) {
        const uint32_t gp = __ldcg(parent + p);
        if (gp != p) __stcg(parent + x, gp);  // path halving (benign race: any ancestor is valid)
        x = p;
        p = gp;
    }
    return x;
}

VXD bool solvedContact(uint32_t fa, uint32_t fb) { return !isSensor(fa) && !isSensor(fb); }

// Lock-free linking: a failed CAS means another thread linked that root, so
// the retry loop always makes global progress; the bound only turns a
// malfunction into a reported error instead of a hang.
constexpr uint32_t kUnionRetryLimit = 1u << 24;

__global__ void unionKernel(const vx_contact* cs, uint32_t m, const BodyArrays B, uint32_t* parent, Counters* C) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
        const uint32_t a = cs[k].a, b = cs[k].b;
        const uint32_t fa = B.filt[a].x, fb = B.filt[b].x;
        if (!solvedContact(fa, fb) || !isDynamic(fa) || !isDynamic(fb)) continue;
        uint32_t tries = 0;
        for (;; ++tries) {
            if (tries == kUnionRetryLimit) { atomicOr(&C->timeout, 1u); break; }
            uint32_t ra = ufFind(parent, a), rb = ufFind(parent, b);
            if (ra == rb) break;
            if (ra < rb) { const uint32_t t = ra; ra = rb; rb = t; }
            if (atomicCAS(&parent[ra], ra, rb) == ra) break;
        }
    }
}

// parent[i] = root of i. The walk writes nothing but the final root: a
// path-halving store racing with another thread's final store could leave a
// non-root ancestor behind, splitting one island into two keys.
__global__ void compressKernel(uint32_t* parent, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t x = i, p = __ldcg(parent + x);
        while (p != x) {
            x = p;
            p = __ldcg(parent + x);
        }
        __stcg(parent + i, x);
    }
}

// Island key of each contact: the root of its dynamic endpoint; contacts with
// no dynamic endpoint (or a sensor) go to the "null" island keyed n.
__global__ void islandKeyKernel(const vx_contact* cs, uint32_t m, const BodyArrays B, const uint32_t* root, uint32_t n,
                                uint64_t* keys, uint32_t* vals) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
        const uint32_t a = cs[k].a, b = cs[k].b;
        const uint32_t fa = B.filt[a].x, fb = B.filt[b].x;
        uint32_t key = n;
        if (solvedContact(fa, fb)) {
            if (isDynamic(fa)) key = root[a];
            else if (isDynamic(fb)) key = root[b];
        }
        keys[k] = key;
        vals[k] = k;
    }
}

__global__ void runFlagKernel(const uint64_t* keys, uint32_t m, uint32_t* flags) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x)
        flags[k] = (k == 0 || keys[k] != keys[k - 1]) ? 1u : 0u;
}

// starts[index[k]] = k for run heads; also starts[runs] = m.
__global__ void runStartKernel(const uint32_t* flags, const uint32_t* index, uint32_t m, uint32_t* starts) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
        if (flags[k]) starts[index[k]] = k;
        if (k == m - 1) starts[index[k] + flags[k]] = m;
    }
}

// Greedy first-free-bit colouring (src/backend_cuda.cu:603-630), one thread
// per island, contacts in their global (a, b, point) order. Static,
// kinematic and sensor endpoints do not constrain colours; past 64 colours
// each body continues from its own spill counter.
__global__ void colorKernel(const vx_contact* cs, const uint32_t* order, const uint32_t* islandStart,
                            uint32_t islands, const BodyArrays B, unsigned long long* mask, uint32_t* nextColor,
                            uint32_t* colorOf, uint64_t* colorKeys, Counters* C, uint32_t sizeLimit) {
    for (uint32_t isl = blockIdx.x * blockDim.x + threadIdx.x; isl < islands; isl += gridDim.x * blockDim.x) {
        const uint32_t s0 = islandStart[isl], s1 = islandStart[isl + 1];
        if (s1 - s0 > sizeLimit) continue;  // coloured by the parallel fixed point
        for (uint32_t k = s0; k < s1; ++k) {
            const vx_contact& c = cs[order[k]];
            mask[c.a] = 0ull; mask[c.b] = 0ull;
            nextColor[c.a] = 64u; nextColor[c.b] = 64u;
        }
        uint32_t colors = 0;
        for (uint32_t k = s0; k < s1; ++k) {
            const uint32_t ci = order[k];
            const vx_contact& c = cs[ci];
            const uint32_t fa = B.filt[c.a].x, fb = B.filt[c.b].x;
            const bool sensor = isSensor(fa) || isSensor(fb);
            const bool sa = sensor || !isDynamic(fa);
            const bool sb = sensor || !isDynamic(fb);
            const unsigned long long used = (sa ? 0ull : mask[c.a]) | (sb ? 0ull : mask[c.b]);
            uint32_t color;
            if (~used) {
                color = (uint32_t)(__ffsll((long long)~used) - 1);
            } else {
                const uint32_t na = sa ? 64u : nextColor[c.a];
                const uint32_t nb = sb ? 64u : nextColor[c.b];
                color = na > nb ? na : nb;
                if (!sa) nextColor[c.a] = color + 1;
                if (!sb) nextColor[c.b] = color + 1;
            }
            if (color < 64) {
                if (!sa) mask[c.a] |= 1ull << color;
                if (!sb) mask[c.b] |= 1ull << color;
            }
            colorOf[ci] = color;
            colorKeys[k] = ((uint64_t)isl << 16) | (color < 65535u ? color : 65535u);
            if (color + 1 > colors) colors = color + 1;
        }
        atomicMax(&C->maxColors, colors);
        atomicMax(&C->largestIsland, s1 - s0);
    }
}

// Islands above this many contacts are coloured by the parallel fixed point.
constexpr uint32_t kSerialColorLimit = 4096;

// Run number of each position: inclusive scan of the head flags minus one.
__global__ void runOfKernel(const uint32_t* flags, const uint32_t* index, uint32_t m, uint32_t* runOf) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x)
        runOf[k] = index[k] + flags[k] - 1u;
}

__global__ void lastKeyKernel(const uint64_t* keys, uint32_t m, Counters* C) {
    if (blockIdx.x == 0 && threadIdx.x == 0) C->lastIslandKey = (uint32_t)keys[m - 1];
}

__global__ void islandMaxKernel(const uint32_t* islandStart, Counters* C) {
    const uint32_t islands = C->islands;
    uint32_t mx = 0;
    for (uint32_t isl = blockIdx.x * blockDim.x + threadIdx.x; isl < islands; isl += gridDim.x * blockDim.x)
        mx = max(mx, islandStart[isl + 1] - islandStart[isl]);
    for (int off = 16; off > 0; off >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    if ((threadIdx.x & 31) == 0 && mx) atomicMax(&C->maxIslandSize, mx);
}

// Parallel greedy colouring of large islands. The greedy colour of a contact
// is the first colour below 64 unused by the earlier contacts (island order)
// that share one of its dynamic bodies (past that, one more than their
// highest colour): the unique fixed point of
//   colour[k] = rule({ colour[j] : j < k, j shares a body with k })
// reached by iterating the rule from all-zero colours (a contact is final
// once every earlier neighbour is). Every round runs over all contacts of the
// large islands in parallel; a round without changes is the fixed point.
// Entries (body, 2k + side) sorted by body list each contact's earlier
// neighbours as the entries before its own in the body's run.
__global__ void colorEntryKernel(const vx_contact* cs, const uint32_t* order, uint32_t m, const uint32_t* islandIdx,
                                 const uint32_t* islandStart, const BodyArrays B, uint32_t n, uint64_t* keys,
                                 uint32_t* vals, uint32_t* slot) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
        const uint32_t isl = islandIdx[k];
        const bool big = islandStart[isl + 1] - islandStart[isl] > kSerialColorLimit;
        const vx_contact& c = cs[order[k]];
        const uint32_t fa = B.filt[c.a].x, fb = B.filt[c.b].x;
        const bool sensor = isSensor(fa) || isSensor(fb);
        keys[2 * k] = big && !sensor && isDynamic(fa) ? c.a : n;
        keys[2 * k + 1] = big && !sensor && isDynamic(fb) ? c.b : n;
        vals[2 * k] = 2 * k;
        vals[2 * k + 1] = 2 * k + 1;
        slot[2 * k] = slot[2 * k + 1] = 0xffffffffu;
    }
}

__global__ void colorSlotKernel(const uint64_t* keys, const uint32_t* vals, uint32_t entries, uint32_t n,
                                uint32_t* slot, uint32_t* runStart) {
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < entries; e += gridDim.x * blockDim.x) {
        const uint64_t key = keys[e];
        if (key >= n) continue;
        slot[vals[e]] = e;
        if (e == 0 || keys[e - 1] != key) runStart[key] = e;
    }
}

// Cooperative launch. changed[3] rotate per round: the counter of round r + 1
// is cleared during round r, after every block has read round r - 2's value.
// color[] is indexed by island-order position and zero on entry.
__global__ void colorFixedPointKernel(const uint64_t* keys, const uint32_t* vals, const uint32_t* slot,
                                      const uint32_t* runStart, const uint32_t* islandIdx,
                                      const uint32_t* islandStart, uint32_t m, uint32_t* color, CoopState* st,
                                      uint32_t maxRounds) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    for (uint32_t r = 0; r < maxRounds; ++r) {
        if (tid == 0) st->changed[(r + 1) % 3] = 0u;
        uint32_t local = 0;
        for (uint32_t k = tid; k < m; k += stride) {
            const uint32_t isl = islandIdx[k];
            if (islandStart[isl + 1] - islandStart[isl] <= kSerialColorLimit) continue;
            // Past 64 colours the greedy rule continues from a per-body
            // counter: one past the highest colour (>= 64) of the body's
            // earlier contacts, 64 when there is none.
            unsigned long long used = 0ull;
            uint32_t high = 63u;
            for (int side = 0; side < 2; ++side) {
                const uint32_t e = slot[2 * k + side];
                if (e == 0xffffffffu) continue;
                const uint32_t body = (uint32_t)keys[e];
                for (uint32_t f = runStart[body]; f < e; ++f) {
                    const uint32_t cq = __ldcg(color + (vals[f] >> 1));
                    if (cq < 64u) used |= 1ull << cq;
                    else high = max(high, cq);
                }
            }
            const uint32_t next = ~used != 0ull ? (uint32_t)(__ffsll((long long)~used) - 1) : high + 1u;
            if (next != __ldcg(color + k)) {
                __stcg(color + k, next);
                ++local;
            }
        }
        if (local) atomicAdd(&st->changed[r % 3], local);
        if (!gridSync(&st->bar, &st->timeout, st->spinLimit)) return;
        if (__ldcg(&st->changed[r % 3]) == 0u || __ldcg(&st->spill) != 0u) {
            if (tid == 0) st->rounds = r + 1;
            return;
        }
    }
    if (tid == 0) { st->rounds = maxRounds; atomicOr(&st->spill, 2u); }  // no fixed point within the bound
}

__global__ void colorFinishKernel(const uint32_t* order, uint32_t m, const uint32_t* islandIdx,
                                  const uint32_t* islandStart, const uint32_t* color, uint32_t* colorOf,
                                  uint64_t* colorKeys, Counters* C) {
    uint32_t mx = 0;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
        const uint32_t isl = islandIdx[k];
        const uint32_t size = islandStart[isl + 1] - islandStart[isl];
        if (size <= kSerialColorLimit) continue;
        const uint32_t c = color[k];
        colorOf[order[k]] = c;
        colorKeys[k] = ((uint64_t)isl << 16) | (c < 65535u ? c : 65535u);
        mx = max(mx, c + 1);
        if (k == islandStart[isl]) atomicMax(&C->largestIsland, size);
    }
    for (int off = 16; off > 0; off >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    if ((threadIdx.x & 31) == 0 && mx) atomicMax(&C->maxColors, mx);
}

// islandOfBody for the dynamic bodies of every real island's contacts, one
// thread per island-order position (islandOf[k]: island of position k).
__global__ void islandBodyKernel(const vx_contact* cs, const uint32_t* order, const uint32_t* islandOf, uint32_t m,
                                 uint32_t realIslands, const BodyArrays B, uint32_t* islandOfBody) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
        const uint32_t isl = islandOf[k];
        if (isl >= realIslands) continue;
        const vx_contact& c = cs[order[k]];
        if (isDynamic(B.filt[c.a].x)) islandOfBody[c.a] = isl;
        if (isDynamic(B.filt[c.b].x)) islandOfBody[c.b] = isl;
    }
}

__global__ void bodyKeyKernel(const uint32_t* islandOfBody, uint32_t n, uint32_t freeKey, uint64_t* keys,
                              uint32_t* vals) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t isl = islandOfBody[i];
        keys[i] = isl == 0xffffffffu ? freeKey : isl;
        vals[i] = i;
    }
}

// bodyStart[key] for each run of sorted body keys; bodyStart has islands+2 entries.
__global__ void bodyStartKernel(const uint64_t* keys, uint32_t n, uint32_t* bodyStart, uint32_t entries) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint64_t key = keys[k];
        const uint64_t prevKey = k == 0 ? ~0ull : keys[k - 1];
        if (key != prevKey) {
            // every key in (prevKey, key] starts at k (empty islands get empty ranges)
            const uint64_t from = k == 0 ? 0 : prevKey + 1;
            for (uint64_t x = from; x <= key && x < entries; ++x) bodyStart[x] = k;
        }
        if (k == n - 1)
            for (uint64_t x = key + 1; x < entries; ++x) bodyStart[x] = n;
    }
}

// Islands the block kernels cannot hold (solveClusterKernel's share), counted
// for the host's single read of the plan.
constexpr uint32_t kTinyLimit = 16;   // islands of at most this many contacts: packed tiny solve
constexpr int kBlockBodies = 512;     // islands beyond these sizes: the whole grid (giant islands)
constexpr int kBlockRows = 3072;
__global__ void giantCountKernel(const uint32_t* islandStart, const uint32_t* bodyStart, uint32_t islands,
                                 uint32_t realIslands, Counters* C) {
    uint32_t count = 0;
    for (uint32_t isl = blockIdx.x * blockDim.x + threadIdx.x; isl < islands; isl += gridDim.x * blockDim.x) {
        const uint32_t rows = islandStart[isl + 1] - islandStart[isl];
        const uint32_t nb = isl < realIslands ? bodyStart[isl + 1] - bodyStart[isl] : 0u;
        if (rows > kTinyLimit && (nb > (uint32_t)kBlockBodies || rows > (uint32_t)kBlockRows)) ++count;
    }
    for (int off = 16; off > 0; off >>= 1) count += __shfl_xor_sync(0xffffffffu, count, off);
    if ((threadIdx.x & 31) == 0 && count) atomicAdd(&C->giantCount, count);
}

// Contact-free bodies: the last two bodyStart entries, for the host's single read.
__global__ void freeRangeKernel(const uint32_t* bodyStart, uint32_t entries, Counters* C) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        C->freeFrom = bodyStart[entries - 2];
        C->freeTo = bodyStart[entries - 1];
    }
}

// ---------------------------------------------------------------------------
// island solve (src/backend_cuda.cu:569-761 semantics)
// ---------------------------------------------------------------------------

struct SolveArgs {
    BodyArrays B;
    vx_contact* contacts;        // key-sorted storage
    const uint32_t* order;       // solve order -> contact index
    const uint32_t* islandStart; // islands + 1 (solve-order ranges)
    const uint32_t* segStart;    // segments + 1
    const uint32_t* islandSeg;   // islands + 1 (first segment)
    const uint32_t* bodyOrder;   // bodies sorted by island
    const uint32_t* bodyStart;   // islands + 2
    uint32_t islands;
    uint32_t realIslands;  // islands >= realIslands (the null island) own no bodies
    V3 gravity;
    float h;
    int substeps;
    int sweeps;
    int warmStart;     // warm start on the first substep
    int integrate;     // integrate velocities (s > 0) and transforms each substep
    int coneBlock;
    uint32_t tinyLimit;
    int positionIterations;  // position-correction mode when > 0
    RowPrep* prep;           // per solve-order row, rebuilt every substep (block / global paths)
    float4* frames;          // per body inertia frame, rebuilt every substep (global path)
    int stackStabilization;
    float stackStiffness, stackDamping;
    uint32_t* fault;         // set when the island plan is inconsistent (Counters::planFault)
    const uint2* rowBodies;  // per solve-order row: (a, b) of its contact (giant islands)
};

VXD void positionRow(const SolveArgs& A, uint32_t ci) {
    const vx_contact& cc = A.contacts[ci];
    const uint32_t fa = A.B.filt[cc.a].x, fb = A.B.filt[cc.b].x;
    if (!solvedContact(fa, fb)) return;
    const Mass ma = loadMass(A.B, cc.a), mb = loadMass(A.B, cc.b);
    const float ima = solverInvMass(ma), imb = solverInvMass(mb);
    const float invMassSum = ima + imb;
    if (invMassSum <= 0.0f) return;
    V3 pa = f3(A.B.pos[cc.a]), pb = f3(A.B.pos[cc.b]);
    const Q4 qa = q4(A.B.rot[cc.a]), qb = q4(A.B.rot[cc.b]);
    const V3 n{cc.normal.x, cc.normal.y, cc.normal.z};
    const V3 wa = anchorWorld(shapeOf(fa) == kSphere, pa, qa, V3{cc.localAnchorA.x, cc.localAnchorA.y, cc.localAnchorA.z});
    const V3 wb = anchorWorld(shapeOf(fb) == kSphere, pb, qb, V3{cc.localAnchorB.x, cc.localAnchorB.y, cc.localAnchorB.z});
    const float g = cc.bias0 + dot(n, wa - wb);
    const float slop = 1e-3f;
    if (g >= -slop) return;
    float resolve = 0.6f;
    if (A.stackStabilization) {
        const V3 rv = f3(A.B.vel[cc.a]) - f3(A.B.vel[cc.b]);
        if (lengthSq(rv) < 1e-4f) {
            const float stiffness = A.stackStiffness / 1000.0f;
            const float damping = 1.0f + A.stackDamping * A.h;
            resolve += 0.2f * stiffness / damping;
        }
    }
    const float push = -resolve * (g + slop) / invMassSum;
    if (isDynamic(fa) && !isAsleep(fa)) { pa += n * (push * ima); A.B.pos[cc.a] = pack(pa, 0.0f); }
    if (isDynamic(fb) && !isAsleep(fb)) { pb -= n * (push * imb); A.B.pos[cc.b] = pack(pb, 0.0f); }
}



// Block-cooperative island processing: contacts of one colour in parallel,
// a block barrier between colours. The island's dynamic bodies live in shared
// memory for the whole substep loop (islands of up to kBlockBodies bodies and
// kBlockRows contacts); larger islands run the same schedule on global memory.
constexpr int kBlockThreads = 256;
// Islands of up to kSmallBodies bodies and kSmallRows contacts run on one warp
// each, many per SM (a colour of a small island has a few rows; a 256-thread
// block would leave most of its threads idle and hold a whole SM's share of
// shared memory).
constexpr int kSmallThreads = 32;
constexpr int kSmallBodies = 64;
constexpr int kSmallRows = 256;
constexpr size_t blockSmem(int bodies, int rows) {
    return (size_t)bodies * (7 * sizeof(float4) + sizeof(uint32_t)) + (size_t)rows * sizeof(int2);
}
constexpr size_t kBlockSmem = blockSmem(kBlockBodies, kBlockRows);
constexpr size_t kSmallSmem = blockSmem(kSmallBodies, kSmallRows);

struct SharedBodies {
    float4 *p, *q, *v, *w, *inertia, *iq, *frame;
    uint32_t* flags;
    int2* rowIdx;  // per island row: local index of a / b, -1 = read-only global body
};

template <int Bodies>
VXD SharedBodies carve(float4* base) {
    SharedBodies S;
    S.p = base;
    S.q = S.p + Bodies;
    S.v = S.q + Bodies;
    S.w = S.v + Bodies;
    S.inertia = S.w + Bodies;
    S.iq = S.inertia + Bodies;
    S.frame = S.iq + Bodies;
    S.flags = reinterpret_cast<uint32_t*>(S.frame + Bodies);
    S.rowIdx = reinterpret_cast<int2*>(S.flags + Bodies);
    return S;
}

VXD SolverBody sharedBody(const SharedBodies& S, int li) {
    SolverBody b;
    b.p = f3(S.p[li]);
    b.q = q4(S.q[li]);
    b.v = f3(S.v[li]);
    b.w = f3(S.w[li]);
    const float4 in = S.inertia[li];
    b.m.invI = V3{in.x, in.y, in.z};
    b.m.invMass = in.w;
    b.m.iq = q4(S.iq[li]);
    b.m.flags = S.flags[li];
    b.sphere = shapeOf(b.m.flags) == kSphere;
    b.frame = q4(S.frame[li]);
    return b;
}

// A body outside the island's shared copy (static endpoints): frame computed here.
VXD SolverBody globalBody(const BodyArrays& B, uint32_t id) {
    SolverBody b = loadSolverBody(B, id);
    cacheFrame(b);
    return b;
}

// op: 0 warm start, 1 velocity sweep, 2 position row, 3 prepare (pose terms)
VXD void sharedRow(const SolveArgs& A, const SharedBodies& S, uint32_t k, uint32_t s0, int op) {
    vx_contact& cc = A.contacts[A.order[s0 + k]];
    const int2 li = S.rowIdx[k];
    SolverBody a = li.x >= 0 ? sharedBody(S, li.x) : globalBody(A.B, cc.a);
    SolverBody b = li.y >= 0 ? sharedBody(S, li.y) : globalBody(A.B, cc.b);
    if (!solvedContact(a.m.flags, b.m.flags)) return;
    if (op == 2) {
        const float ima = solverInvMass(a.m), imb = solverInvMass(b.m);
        const float invMassSum = ima + imb;
        if (invMassSum <= 0.0f) return;
        const V3 n{cc.normal.x, cc.normal.y, cc.normal.z};
        const V3 wa = anchorWorld(a.sphere, a.p, a.q, V3{cc.localAnchorA.x, cc.localAnchorA.y, cc.localAnchorA.z});
        const V3 wb = anchorWorld(b.sphere, b.p, b.q, V3{cc.localAnchorB.x, cc.localAnchorB.y, cc.localAnchorB.z});
        const float gap = cc.bias0 + dot(n, wa - wb);
        if (gap >= -1e-3f) return;
        float resolve = 0.6f;
        if (A.stackStabilization && lengthSq(a.v - b.v) < 1e-4f)
            resolve += 0.2f * (A.stackStiffness / 1000.0f) / (1.0f + A.stackDamping * A.h);
        const float push = -resolve * (gap + 1e-3f) / invMassSum;
        if (isDynamic(a.m.flags) && !isAsleep(a.m.flags) && li.x >= 0) S.p[li.x] = pack(a.p + n * (push * ima), 0.0f);
        if (isDynamic(b.m.flags) && !isAsleep(b.m.flags) && li.y >= 0) S.p[li.y] = pack(b.p - n * (push * imb), 0.0f);
        return;
    }
    RowContact r;
    loadRow(cc, r);
    RowPrep& P = A.prep[s0 + k];
    if (op == 3) {  // prepare
        prepRow(a, b, r, A.h, A.coneBlock != 0, P);
        return;
    }
    if (op == 0) warmPrepRow(a, b, r, P);
    else sweepRow(a, b, r, P, A.coneBlock != 0);
    if (li.x >= 0 && isDynamic(a.m.flags)) { S.v[li.x] = pack(a.v, 0.0f); S.w[li.x] = pack(a.w, 0.0f); }
    if (li.y >= 0 && isDynamic(b.m.flags)) { S.v[li.y] = pack(b.v, 0.0f); S.w[li.y] = pack(b.w, 0.0f); }
    storeRow(cc, r);
}

VXD void sharedIntegrateVelocity(const SolveArgs& A, const SharedBodies& S, int li, uint32_t id) {
    SolverBody b = sharedBody(S, li);
    const Mass& m = b.m;
    if (!isDynamic(m.flags) || isLocked(m.flags) || isAsleep(m.flags)) return;
    const float4 ex = A.B.extra[id];
    b.v += (A.gravity * ex.y + f3(A.B.force[id]) * solverInvMass(m)) * A.h;
    b.w += invInertiaMulAt(m, f3(A.B.torque[id]), b.q) * A.h;
    b.v *= 1.0f / (1.0f + ex.z * A.h);
    b.w *= 1.0f / (1.0f + ex.w * A.h);
    S.v[li] = pack(b.v, 0.0f);
    S.w[li] = pack(b.w, 0.0f);
}

VXD void sharedIntegrateTransform(const SolveArgs& A, const SharedBodies& S, int li) {
    SolverBody b = sharedBody(S, li);
    if (isStaticBody(b.m.flags) || isLocked(b.m.flags) || isAsleep(b.m.flags)) return;
    advanceTransform(b.m, b.p, b.q, b.v, b.w, A.h);
    S.p[li] = pack(b.p, 0.0f);
    S.q[li] = pack(b.q);
    S.w[li] = pack(b.w, 0.0f);
}

// Island bodies read from global memory with frames from A.frames.
VXD SolverBody framedBody(const SolveArgs& A, uint32_t id) {
    SolverBody b = loadSolverBody(A.B, id);
    if (isDynamic(b.m.flags)) b.frame = q4(A.frames[id]);
    else cacheFrame(b);
    return b;
}

// op: 0 warm start, 1 velocity sweep, 3 prepare
VXD void globalRow(const SolveArgs& A, uint32_t pos, int op) {
    vx_contact& cc = A.contacts[A.order[pos]];
    SolverBody a = framedBody(A, cc.a), b = framedBody(A, cc.b);
    if (!solvedContact(a.m.flags, b.m.flags)) return;
    RowContact r;
    loadRow(cc, r);
    RowPrep& P = A.prep[pos];
    if (op == 3) { prepRow(a, b, r, A.h, A.coneBlock != 0, P); return; }
    if (op == 0) warmPrepRow(a, b, r, P);
    else sweepRow(a, b, r, P, A.coneBlock != 0);
    if (isDynamic(a.m.flags)) { A.B.vel[cc.a] = pack(a.v, 0.0f); A.B.ang[cc.a] = pack(a.w, 0.0f); }
    if (isDynamic(b.m.flags)) { A.B.vel[cc.b] = pack(b.v, 0.0f); A.B.ang[cc.b] = pack(b.w, 0.0f); }
    storeRow(cc, r);
}

__device__ void solveIslandGlobal(const SolveArgs& A, uint32_t isl) {
    const uint32_t g0 = A.islandSeg[isl], g1 = A.islandSeg[isl + 1];
    if (A.positionIterations > 0) {
        for (int it = 0; it < A.positionIterations; ++it)
            for (uint32_t g = g0; g < g1; ++g) {
                for (uint32_t k = A.segStart[g] + threadIdx.x; k < A.segStart[g + 1]; k += blockDim.x)
                    positionRow(A, A.order[k]);
                __syncthreads();
            }
        return;
    }
    const uint32_t s0 = A.islandStart[isl], s1 = A.islandStart[isl + 1];
    const uint32_t b0 = isl < A.realIslands ? A.bodyStart[isl] : 0u;
    const uint32_t b1 = isl < A.realIslands ? A.bodyStart[isl + 1] : 0u;
    for (int s = 0; s < A.substeps; ++s) {
        for (uint32_t k = b0 + threadIdx.x; k < b1; k += blockDim.x) {
            const uint32_t id = A.bodyOrder[k];
            if (A.integrate && s > 0) integrateVelocity(A.B, id, A.gravity, A.h);
            A.frames[id] = pack(inertiaFrameAt(loadMass(A.B, id), q4(A.B.rot[id])));
        }
        __syncthreads();
        for (uint32_t k = s0 + threadIdx.x; k < s1; k += blockDim.x) globalRow(A, k, 3);
        __syncthreads();
        if (A.warmStart && s == 0)
            for (uint32_t g = g0; g < g1; ++g) {
                for (uint32_t k = A.segStart[g] + threadIdx.x; k < A.segStart[g + 1]; k += blockDim.x)
                    globalRow(A, k, 0);
                __syncthreads();
            }
        for (int it = 0; it < A.sweeps; ++it)
            for (uint32_t g = g0; g < g1; ++g) {
                for (uint32_t k = A.segStart[g] + threadIdx.x; k < A.segStart[g + 1]; k += blockDim.x)
                    globalRow(A, k, 1);
                __syncthreads();
            }
        if (A.integrate) {
            for (uint32_t k = b0 + threadIdx.x; k < b1; k += blockDim.x)
                integrateTransform(A.B, A.bodyOrder[k], A.h);
            __syncthreads();
        }
    }
}

// Small = the island fits the one-warp variant.
VXD bool smallIsland(uint32_t nb, uint32_t rows) { return nb <= (uint32_t)kSmallBodies && rows <= (uint32_t)kSmallRows; }

template <int Threads, int Bodies, int Rows, bool Small>
__global__ void __launch_bounds__(Threads) solveBlockKernel(SolveArgs A, uint32_t* localIdx) {
    extern __shared__ float4 smemRaw[];
    const SharedBodies S = carve<Bodies>(smemRaw);
    for (uint32_t isl = blockIdx.x; isl < A.islands; isl += gridDim.x) {
        const uint32_t s0 = A.islandStart[isl], s1 = A.islandStart[isl + 1];
        if (s1 - s0 <= A.tinyLimit) continue;
        const uint32_t b0 = isl < A.realIslands ? A.bodyStart[isl] : 0u;
        const uint32_t b1 = isl < A.realIslands ? A.bodyStart[isl + 1] : 0u;
        const uint32_t nb = b1 - b0, rows = s1 - s0;
        if (nb > (uint32_t)Bodies || rows > (uint32_t)Rows) continue;  // a giant island
        if (!Small && smallIsland(nb, rows)) continue;                 // the one-warp variant's
        for (uint32_t k = threadIdx.x; k < nb; k += blockDim.x) {
            const uint32_t id = A.bodyOrder[b0 + k];
            S.p[k] = A.B.pos[id]; S.q[k] = A.B.rot[id]; S.v[k] = A.B.vel[id]; S.w[k] = A.B.ang[id];
            S.inertia[k] = A.B.inertia[id]; S.iq[k] = A.B.iq[id]; S.flags[k] = A.B.filt[id].x;
            localIdx[id] = k;
        }
        __syncthreads();
        for (uint32_t k = threadIdx.x; k < rows; k += blockDim.x) {
            const vx_contact& cc = A.contacts[A.order[s0 + k]];
            const bool da = isDynamic(A.B.filt[cc.a].x), db = isDynamic(A.B.filt[cc.b].x);
            int la = da ? (int)localIdx[cc.a] : -1, lb = db ? (int)localIdx[cc.b] : -1;
            // a dynamic body outside this island's list means an inconsistent plan: report it, never index smem
            if (la >= 0 && ((uint32_t)la >= nb || A.bodyOrder[b0 + la] != cc.a)) { atomicOr(A.fault, 1u); la = -1; }
            if (lb >= 0 && ((uint32_t)lb >= nb || A.bodyOrder[b0 + lb] != cc.b)) { atomicOr(A.fault, 1u); lb = -1; }
            S.rowIdx[k] = make_int2(la, lb);
        }
        __syncthreads();
        const uint32_t g0 = A.islandSeg[isl], g1 = A.islandSeg[isl + 1];
        if (A.positionIterations > 0) {
            for (int it = 0; it < A.positionIterations; ++it)
                for (uint32_t g = g0; g < g1; ++g) {
                    for (uint32_t k = A.segStart[g] - s0 + threadIdx.x; k < A.segStart[g + 1] - s0; k += blockDim.x)
                        sharedRow(A, S, k, s0, 2);
                    __syncthreads();
                }
        } else {
            for (int s = 0; s < A.substeps; ++s) {
                if (A.integrate && s > 0)
                    for (uint32_t k = threadIdx.x; k < nb; k += blockDim.x)
                        sharedIntegrateVelocity(A, S, (int)k, A.bodyOrder[b0 + k]);
                for (uint32_t k = threadIdx.x; k < nb; k += blockDim.x) {
                    Mass m;
                    const float4 in = S.inertia[k];
                    m.invI = V3{in.x, in.y, in.z};
                    m.invMass = in.w;
                    m.iq = q4(S.iq[k]);
                    m.flags = S.flags[k];
                    S.frame[k] = pack(inertiaFrameAt(m, q4(S.q[k])));
                }
                __syncthreads();
                for (uint32_t k = threadIdx.x; k < rows; k += blockDim.x) sharedRow(A, S, k, s0, 3);
                __syncthreads();
                if (A.warmStart && s == 0)
                    for (uint32_t g = g0; g < g1; ++g) {
                        for (uint32_t k = A.segStart[g] - s0 + threadIdx.x; k < A.segStart[g + 1] - s0; k += blockDim.x)
                            sharedRow(A, S, k, s0, 0);
                        __syncthreads();
                    }
                for (int it = 0; it < A.sweeps; ++it)
                    for (uint32_t g = g0; g < g1; ++g) {
                        for (uint32_t k = A.segStart[g] - s0 + threadIdx.x; k < A.segStart[g + 1] - s0; k += blockDim.x)
                            sharedRow(A, S, k, s0, 1);
                        __syncthreads();
                    }
                if (A.integrate) {
                    for (uint32_t k = threadIdx.x; k < nb; k += blockDim.x) sharedIntegrateTransform(A, S, (int)k);
                    __syncthreads();
                }
            }
        }
        for (uint32_t k = threadIdx.x; k < nb; k += blockDim.x) {
            const uint32_t id = A.bodyOrder[b0 + k];
            A.B.pos[id] = S.p[k]; A.B.rot[id] = S.q[k]; A.B.vel[id] = S.v[k]; A.B.ang[id] = S.w[k];
        }
        __syncthreads();
    }
}

// ---- tiny islands packed into warps -----------------------------------------
//
// Islands of at most tinyLimit (16) contacts are packed, in island order, into
// warps of at most 32 rows and 64 bodies. Each lane owns one row and keeps its
// contact terms and per-substep pose terms in registers; the pack's bodies live
// in shared memory. A step runs colour slot c of every island in the pack at
// once (rows of different islands share no body; rows of one colour share no
// dynamic body), so each body sees its rows in colour order, as in the serial
// per-island loop. A pack needs (largest colour count) x sweeps x substeps
// warp steps instead of (rows x sweeps x substeps) thread steps, with no
// per-thread arrays in local memory.
constexpr int kPackRows = 32;
constexpr int kPackBodies = 64;
constexpr int kPackChunk = 64;      // tiny islands per packing thread (a serial greedy scan each)
constexpr int kPackWarps = 4;       // warps (packs) per block

// Sort key of a tiny island: its colour count (a pack runs as many colour
// slots per sweep as its most coloured island, so similar islands share packs).
// Over `cap` slots (an upper bound); slots past the device-side count sort last.
__global__ void tinyKeyKernel(SolveArgs A, const uint32_t* list, const uint32_t* countPtr, uint32_t cap,
                              uint64_t* keys, uint32_t* vals) {
    const uint32_t count = *countPtr;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < cap; t += gridDim.x * blockDim.x) {
        if (t < count) {
            const uint32_t isl = list[t];
            keys[t] = A.islandSeg[isl + 1] - A.islandSeg[isl];
            vals[t] = isl;
        } else {
            keys[t] = 0xffu;
            vals[t] = 0xffffffffu;
        }
    }
}

__global__ void tinyFlagKernel(SolveArgs A, uint32_t* flags) {
    for (uint32_t isl = blockIdx.x * blockDim.x + threadIdx.x; isl < A.islands; isl += gridDim.x * blockDim.x) {
        const uint32_t rows = A.islandStart[isl + 1] - A.islandStart[isl];
        flags[isl] = rows > 0 && rows <= A.tinyLimit ? 1u : 0u;
    }
}

VXD uint32_t islandBodies(const SolveArgs& A, uint32_t isl) {
    return isl < A.realIslands ? A.bodyStart[isl + 1] - A.bodyStart[isl] : 0u;
}

// Greedy packing of each chunk of the tiny-island list: pass 0 counts the
// packs of a chunk, pass 1 writes each pack's first list index.
__global__ void tinyPackKernel(SolveArgs A, const uint32_t* list, const uint32_t* countPtr, uint32_t chunksCap,
                               int pass, uint32_t* packCount, const uint32_t* packBase, uint32_t* packFirst) {
    const uint32_t count = *countPtr;
    for (uint32_t ch = blockIdx.x * blockDim.x + threadIdx.x; ch < chunksCap; ch += gridDim.x * blockDim.x) {
        if (ch * kPackChunk >= count) {  // past the list: no packs
            if (pass == 0) packCount[ch] = 0;
            continue;
        }
        const uint32_t t0 = ch * kPackChunk, t1 = min(count, t0 + kPackChunk);
        uint32_t packs = 0, rows = 0, bodies = 0;
        for (uint32_t t = t0; t < t1; ++t) {
            const uint32_t isl = list[t];
            const uint32_t r = A.islandStart[isl + 1] - A.islandStart[isl], b = islandBodies(A, isl);
            if (t == t0 || rows + r > (uint32_t)kPackRows || bodies + b > (uint32_t)kPackBodies) {
                if (pass == 1) packFirst[packBase[ch] + packs] = t;
                ++packs;
                rows = 0;
                bodies = 0;
            }
            rows += r;
            bodies += b;
        }
        if (pass == 0) packCount[ch] = packs;
    }
}

// Per-warp shared memory of the pack kernel: the bodies and their ids.
constexpr size_t kPackBodySmem = blockSmem(kPackBodies, 0);
constexpr size_t kPackWarpSmem = (kPackBodySmem + kPackBodies * sizeof(uint32_t) + 15) / 16 * 16;

VXD void solveTinyPack(const SolveArgs& A, const uint32_t* list, const uint32_t* packFirst, uint32_t packs,
                       uint32_t listCount, uint32_t* localIdx, const SharedBodies& S, uint32_t* ids,
                       uint32_t packIdx, uint32_t lane);

// Packs come from device-side counts (no host read); warps stride over them.
__global__ void __launch_bounds__(32 * kPackWarps) solveTinyPackKernel(SolveArgs A, const uint32_t* list,
                                                                        const uint32_t* packFirst,
                                                                        const Counters* C, uint32_t* localIdx) {
    extern __shared__ float4 smemRaw[];
    const uint32_t warpInBlock = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    float4* base = smemRaw + warpInBlock * (kPackWarpSmem / sizeof(float4));
    const SharedBodies S = carve<kPackBodies>(base);
    uint32_t* ids = reinterpret_cast<uint32_t*>(base + kPackBodySmem / sizeof(float4));
    const uint32_t packs = C->tinyPacks, listCount = C->tinyIslands;
    for (uint32_t packIdx = blockIdx.x * kPackWarps + warpInBlock; packIdx < packs; packIdx += gridDim.x * kPackWarps) {
        solveTinyPack(A, list, packFirst, packs, listCount, localIdx, S, ids, packIdx, lane);
        __syncwarp();
    }
}

VXD void solveTinyPack(const SolveArgs& A, const uint32_t* list, const uint32_t* packFirst, uint32_t packs,
                       uint32_t listCount, uint32_t* localIdx, const SharedBodies& S, uint32_t* ids,
                       uint32_t packIdx, uint32_t lane) {
    const uint32_t first = packFirst[packIdx];
    const uint32_t last = packIdx + 1 < packs ? packFirst[packIdx + 1] : listCount;
    const uint32_t count = last - first;  // islands in this pack (1..32)
    uint32_t isl = 0, r = 0, nb = 0, colours = 0;
    if (lane < count) {
        isl = list[first + lane];
        r = A.islandStart[isl + 1] - A.islandStart[isl];
        nb = islandBodies(A, isl);
        colours = A.islandSeg[isl + 1] - A.islandSeg[isl];
    }
    // inclusive prefix sums of rows and bodies over the pack's islands, largest colour count
    uint32_t rp = r, bp = nb, maxC = colours;
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t x = __shfl_up_sync(0xffffffffu, rp, off), y = __shfl_up_sync(0xffffffffu, bp, off);
        if ((int)lane >= off) { rp += x; bp += y; }
    }
    for (int off = 16; off > 0; off >>= 1) maxC = max(maxC, __shfl_xor_sync(0xffffffffu, maxC, off));
    rp -= r;  // exclusive
    bp -= nb;
    const uint32_t totalBodies = __shfl_sync(0xffffffffu, bp + nb, 31);
    // bodies into shared memory: island j's bodies at slots [bp_j, bp_j + nb_j)
    for (uint32_t j = 0; j < count; ++j) {
        const uint32_t jIsl = __shfl_sync(0xffffffffu, isl, j), jB = __shfl_sync(0xffffffffu, nb, j);
        const uint32_t jBase = __shfl_sync(0xffffffffu, bp, j);
        for (uint32_t k = lane; k < jB; k += 32) {
            const uint32_t id = A.bodyOrder[A.bodyStart[jIsl] + k], t = jBase + k;
            S.p[t] = A.B.pos[id]; S.q[t] = A.B.rot[id]; S.v[t] = A.B.vel[id]; S.w[t] = A.B.ang[id];
            S.inertia[t] = A.B.inertia[id]; S.iq[t] = A.B.iq[id]; S.flags[t] = A.B.filt[id].x;
            ids[t] = id;
            localIdx[id] = t;
        }
    }
    __syncwarp();
    // this lane's row: the island j with rp_j <= lane < rp_j + r_j
    bool has = false;
    uint32_t row = 0, myIsl = 0, myBase = 0, myNb = 0;
    for (uint32_t j = 0; j < count; ++j) {
        const uint32_t jr = __shfl_sync(0xffffffffu, r, j), jrp = __shfl_sync(0xffffffffu, rp, j);
        const uint32_t jIsl = __shfl_sync(0xffffffffu, isl, j), jBase = __shfl_sync(0xffffffffu, bp, j);
        const uint32_t jNb = __shfl_sync(0xffffffffu, nb, j);
        if (lane >= jrp && lane < jrp + jr) {
            has = true;
            myIsl = jIsl;
            row = A.islandStart[jIsl] + (lane - jrp);
            myBase = jBase;
            myNb = jNb;
        }
    }
    vx_contact* cp = nullptr;
    RowContact rc;
    RowPrep P;
    int la = -1, lb = -1;
    uint32_t ida = 0, idb = 0, myC = 0;
    bool live = false;
    if (has) {
        cp = A.contacts + A.order[row];
        loadRow(*cp, rc);
        ida = cp->a;
        idb = cp->b;
        const uint32_t fa = A.B.filt[ida].x, fb = A.B.filt[idb].x;
        live = solvedContact(fa, fb);
        if (isDynamic(fa)) la = (int)localIdx[ida];
        if (isDynamic(fb)) lb = (int)localIdx[idb];
        // a dynamic body outside its island's slots means an inconsistent plan: report it, never index smem
        if (la >= 0 && ((uint32_t)la < myBase || (uint32_t)la >= myBase + myNb || ids[la] != ida)) {
            atomicOr(A.fault, 1u);
            la = -1;
        }
        if (lb >= 0 && ((uint32_t)lb < myBase || (uint32_t)lb >= myBase + myNb || ids[lb] != idb)) {
            atomicOr(A.fault, 1u);
            lb = -1;
        }
        const uint32_t g0 = A.islandSeg[myIsl], g1 = A.islandSeg[myIsl + 1];
        uint32_t g = g0;
        while (g + 1 < g1 && A.segStart[g + 1] <= row) ++g;
        myC = g - g0;
    }
    if (A.positionIterations > 0) {
        for (int it = 0; it < A.positionIterations; ++it)
            for (uint32_t c = 0; c < maxC; ++c) {
                if (live && myC == c) {
                    const SolverBody a = la >= 0 ? sharedBody(S, la) : globalBody(A.B, ida);
                    const SolverBody b = lb >= 0 ? sharedBody(S, lb) : globalBody(A.B, idb);
                    const float ima = solverInvMass(a.m), imb = solverInvMass(b.m);
                    const float invMassSum = ima + imb;
                    if (invMassSum > 0.0f) {
                        const V3 wa = anchorWorld(a.sphere, a.p, a.q, rc.la);
                        const V3 wb = anchorWorld(b.sphere, b.p, b.q, rc.lb);
                        const float gap = rc.bias0 + dot(rc.normal, wa - wb);
                        if (gap < -1e-3f) {
                            float resolve = 0.6f;
                            if (A.stackStabilization && lengthSq(a.v - b.v) < 1e-4f)
                                resolve += 0.2f * (A.stackStiffness / 1000.0f) / (1.0f + A.stackDamping * A.h);
                            const float push = -resolve * (gap + 1e-3f) / invMassSum;
                            if (isDynamic(a.m.flags) && !isAsleep(a.m.flags) && la >= 0)
                                S.p[la] = pack(a.p + rc.normal * (push * ima), 0.0f);
                            if (isDynamic(b.m.flags) && !isAsleep(b.m.flags) && lb >= 0)
                                S.p[lb] = pack(b.p - rc.normal * (push * imb), 0.0f);
                        }
                    }
                }
                __syncwarp();
            }
        for (uint32_t t = lane; t < totalBodies; t += 32)
            if (isDynamic(S.flags[t])) A.B.pos[ids[t]] = S.p[t];
        return;
    }
    for (int s = 0; s < A.substeps; ++s) {
        for (uint32_t t = lane; t < totalBodies; t += 32) {
            if (A.integrate && s > 0) sharedIntegrateVelocity(A, S, (int)t, ids[t]);
            Mass m;
            const float4 in = S.inertia[t];
            m.invI = V3{in.x, in.y, in.z};
            m.invMass = in.w;
            m.iq = q4(S.iq[t]);
            m.flags = S.flags[t];
            S.frame[t] = pack(inertiaFrameAt(m, q4(S.q[t])));
        }
        __syncwarp();
        if (live) {
            const SolverBody a = la >= 0 ? sharedBody(S, la) : globalBody(A.B, ida);
            const SolverBody b = lb >= 0 ? sharedBody(S, lb) : globalBody(A.B, idb);
            prepRow(a, b, rc, A.h, A.coneBlock != 0, P);
        }
        __syncwarp();
        const int units = (A.warmStart && s == 0 ? 1 : 0) + A.sweeps;
        for (int u = 0; u < units; ++u) {
            const bool warm = A.warmStart && s == 0 && u == 0;
            for (uint32_t c = 0; c < maxC; ++c) {
                if (live && myC == c) {
                    SolverBody a = la >= 0 ? sharedBody(S, la) : globalBody(A.B, ida);
                    SolverBody b = lb >= 0 ? sharedBody(S, lb) : globalBody(A.B, idb);
                    if (warm) warmPrepRow(a, b, rc, P);
                    else sweepRow(a, b, rc, P, A.coneBlock != 0);
                    if (la >= 0 && isDynamic(a.m.flags)) { S.v[la] = pack(a.v, 0.0f); S.w[la] = pack(a.w, 0.0f); }
                    if (lb >= 0 && isDynamic(b.m.flags)) { S.v[lb] = pack(b.v, 0.0f); S.w[lb] = pack(b.w, 0.0f); }
                }
                __syncwarp();
            }
        }
        if (A.integrate) {
            for (uint32_t t = lane; t < totalBodies; t += 32) sharedIntegrateTransform(A, S, (int)t);
            __syncwarp();
        }
    }
    for (uint32_t t = lane; t < totalBodies; t += 32) {
        if (!isDynamic(S.flags[t])) continue;
        const uint32_t id = ids[t];
        A.B.pos[id] = S.p[t]; A.B.rot[id] = S.q[t]; A.B.vel[id] = S.v[t]; A.B.ang[id] = S.w[t];
    }
    if (has) storeRow(*cp, rc);
}

// ---- giant islands: the whole grid on one island ----------------------------
//
// Islands too large for one block's shared memory run on every block of a
// cooperative launch, with a grid barrier between colours. Mutable data that
// other blocks wrote since the last barrier (velocities, poses, impulses, row
// terms, frames) is read with ld.global.cg and written with st.global.cg, so
// no SM works from a stale L1 line.

VXD float4 ldcg4(const float4* p) { return __ldcg(p); }

// Acquire load / release store at GPU scope: the dataflow's flag handoff
// without a full fence on either side.
VXD uint32_t ldAcquire(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
VXD void stRelease(uint32_t* p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

VXD SolverBody coherentBody(const SolveArgs& A, uint32_t id) {
    SolverBody b;
    b.p = f3(ldcg4(A.B.pos + id));
    b.q = q4(ldcg4(A.B.rot + id));
    b.v = f3(ldcg4(A.B.vel + id));
    b.w = f3(ldcg4(A.B.ang + id));
    b.m = loadMass(A.B, id);
    b.sphere = shapeOf(b.m.flags) == kSphere;
    if (isDynamic(b.m.flags)) b.frame = q4(ldcg4(A.frames + id));
    else cacheFrame(b);
    return b;
}

// Whole 128-byte contact records through L2 (one thread owns a row per colour).
VXD void loadContactCoherent(const vx_contact* p, vx_contact& c) {
    const float4* src = reinterpret_cast<const float4*>(p);
    float4* dst = reinterpret_cast<float4*>(&c);
#pragma unroll
    for (int i = 0; i < (int)(sizeof(vx_contact) / 16); ++i) dst[i] = __ldcg(src + i);
}

VXD void storeContactCoherent(vx_contact* p, const vx_contact& c) {
    const float4* src = reinterpret_cast<const float4*>(&c);
    float4* dst = reinterpret_cast<float4*>(p);
#pragma unroll
    for (int i = 0; i < (int)(sizeof(vx_contact) / 16); ++i) __stcg(dst + i, src[i]);
}

// A row's prepared terms through L2 as 16-byte words: one sector per word and
// lane, where word-sized loads would fetch each sector four times (the rows of
// a warp lie 176 bytes apart, and L2-only loads do not keep sectors in L1).
static_assert(sizeof(RowPrep) % 16 == 0, "prepared rows must be whole 16-byte words");

VXD void coherentPrep(const RowPrep* p, RowPrep& P) {
    const float4* s = reinterpret_cast<const float4*>(p);
    float* d = reinterpret_cast<float*>(&P);
#pragma unroll
    for (int i = 0; i < (int)(sizeof(RowPrep) / 16); ++i) {
        const float4 v = __ldcg(s + i);
        d[4 * i + 0] = v.x;
        d[4 * i + 1] = v.y;
        d[4 * i + 2] = v.z;
        d[4 * i + 3] = v.w;
    }
}

VXD void storePrepCoherent(RowPrep* p, const RowPrep& P) {
    float4* dst = reinterpret_cast<float4*>(p);
    const float* src = reinterpret_cast<const float*>(&P);
#pragma unroll
    for (int i = 0; i < (int)(sizeof(RowPrep) / 16); ++i)
        __stcg(dst + i, make_float4(src[4 * i + 0], src[4 * i + 1], src[4 * i + 2], src[4 * i + 3]));
}

// Inputs of one giant row that only the row itself writes (its contact
// record and its prepared terms; the body ids are fixed): a row fetches them
// before it waits for its predecessors, so their latency overlaps the wait.
struct GiantRowIn {
    uint2 ab;
    vx_contact* cp;
    vx_contact cc;
    RowPrep P;
};

VXD void giantRowFetch(const SolveArgs& A, uint32_t pos, int op, GiantRowIn& in) {
    in.ab = A.rowBodies[pos];
    in.cp = A.contacts + A.order[pos];
    loadContactCoherent(in.cp, in.cc);
    if (op == 0 || op == 1) coherentPrep(A.prep + pos, in.P);
}

// op: 0 warm start, 1 velocity sweep, 2 position row, 3 prepare
VXD void giantRowRun(const SolveArgs& A, uint32_t pos, int op, GiantRowIn& in) {
    const uint2 ab = in.ab;
    vx_contact* cp = in.cp;
    vx_contact& cc = in.cc;
    SolverBody a = coherentBody(A, ab.x), b = coherentBody(A, ab.y);
    if (!solvedContact(a.m.flags, b.m.flags)) return;
    RowContact r;
    loadRow(cc, r);
    if (op == 2) {
        const float ima = solverInvMass(a.m), imb = solverInvMass(b.m);
        const float invMassSum = ima + imb;
        if (invMassSum <= 0.0f) return;
        const V3 wa = anchorWorld(a.sphere, a.p, a.q, r.la);
        const V3 wb = anchorWorld(b.sphere, b.p, b.q, r.lb);
        const float gap = r.bias0 + dot(r.normal, wa - wb);
        if (gap >= -1e-3f) return;
        float resolve = 0.6f;
        if (A.stackStabilization && lengthSq(a.v - b.v) < 1e-4f)
            resolve += 0.2f * (A.stackStiffness / 1000.0f) / (1.0f + A.stackDamping * A.h);
        const float push = -resolve * (gap + 1e-3f) / invMassSum;
        if (isDynamic(a.m.flags) && !isAsleep(a.m.flags))
            __stcg(A.B.pos + ab.x, pack(a.p + r.normal * (push * ima), 0.0f));
        if (isDynamic(b.m.flags) && !isAsleep(b.m.flags))
            __stcg(A.B.pos + ab.y, pack(b.p - r.normal * (push * imb), 0.0f));
        return;
    }
    RowPrep& P = in.P;
    if (op == 3) {
        prepRow(a, b, r, A.h, A.coneBlock != 0, P);
        storePrepCoherent(A.prep + pos, P);
        return;
    }
    if (op == 0) warmPrepRow(a, b, r, P);
    else sweepRow(a, b, r, P, A.coneBlock != 0);
    if (isDynamic(a.m.flags)) { __stcg(A.B.vel + ab.x, pack(a.v, 0.0f)); __stcg(A.B.ang + ab.x, pack(a.w, 0.0f)); }
    if (isDynamic(b.m.flags)) { __stcg(A.B.vel + ab.y, pack(b.v, 0.0f)); __stcg(A.B.ang + ab.y, pack(b.w, 0.0f)); }
    storeRow(cc, r);
    storeContactCoherent(cp, cc);
}

VXD void giantRow(const SolveArgs& A, uint32_t pos, int op) {
    GiantRowIn in;
    giantRowFetch(A, pos, op, in);
    giantRowRun(A, pos, op, in);
}

// integrateKernel semantics (src/backend_cuda.cu:80-89) on coherent loads.
VXD void giantIntegrateVelocity(const SolveArgs& A, uint32_t i) {
    const Mass m = loadMass(A.B, i);
    if (!isDynamic(m.flags) || isLocked(m.flags) || isAsleep(m.flags)) return;
    const Q4 q = q4(ldcg4(A.B.rot + i));
    V3 v = f3(ldcg4(A.B.vel + i));
    V3 w = f3(ldcg4(A.B.ang + i));
    const V3 F = f3(A.B.force[i]);
    const V3 T = f3(A.B.torque[i]);
    const float4 ex = A.B.extra[i];
    v += (A.gravity * ex.y + F * solverInvMass(m)) * A.h;
    w += invInertiaMulAt(m, T, q) * A.h;
    v *= 1.0f / (1.0f + ex.z * A.h);
    w *= 1.0f / (1.0f + ex.w * A.h);
    __stcg(A.B.vel + i, pack(v, 0.0f));
    __stcg(A.B.ang + i, pack(w, 0.0f));
}

// integrateTransformsKernel semantics (src/backend_cuda.cu:91-97) on coherent loads.
VXD void giantIntegrateTransform(const SolveArgs& A, uint32_t i) {
    const Mass m = loadMass(A.B, i);
    if (isStaticBody(m.flags) || isLocked(m.flags) || isAsleep(m.flags)) return;
    V3 p = f3(ldcg4(A.B.pos + i));
    Q4 q = q4(ldcg4(A.B.rot + i));
    const V3 v = f3(ldcg4(A.B.vel + i));
    V3 w = f3(ldcg4(A.B.ang + i));
    advanceTransform(m, p, q, v, w, A.h);
    __stcg(A.B.pos + i, pack(p, 0.0f));
    __stcg(A.B.rot + i, pack(q));
    __stcg(A.B.ang + i, pack(w, 0.0f));
}

// Giant islands: every row is linked to the previous row on each of its
// dynamic bodies (colour order; the body's last row of the previous sweep for
// its first row). A row may run sweep u once those predecessors have
// published sweep u (u - 1 across the wrap): the order the colour-by-colour
// sweep imposes on every body, without a barrier per colour.
constexpr uint32_t kNoPred = 0xffffffffu;  // no predecessor / empty queue slot
constexpr uint32_t kWrap = 0x80000000u;    // predecessor from the previous sweep

// Dataflow links of the giant islands' rows: entries (dynamic body, 2k + side)
// of every row of a giant island, other endpoints keyed n (no link).
__global__ void giantEntryKernel(SolveArgs A, const uint32_t* islandOf, uint32_t m, uint32_t n, uint64_t* keys,
                                 uint32_t* vals, uint2* rowBodies);
// For each body run of the sorted entries, the position of its last entry.
__global__ void giantLastKernel(const uint64_t* keys, uint32_t entries, uint32_t n, uint32_t* lastOf) {
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < entries; p += gridDim.x * blockDim.x) {
        const uint64_t key = keys[p];
        if (key != (uint64_t)n && (p + 1 == entries || keys[p + 1] != key)) lastOf[key] = p;
    }
}
// pred[2k + side]: the previous row on that body in colour order, or (kWrap |
// the body's last row) for its first row; kNoPred for no dynamic body.
__global__ void giantPredKernel(const uint64_t* keys, const uint32_t* vals, uint32_t entries, uint32_t n,
                                const uint32_t* lastOf, uint32_t* pred) {
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < entries; p += gridDim.x * blockDim.x) {
        const uint64_t key = keys[p];
        uint32_t v = kNoPred;
        if (key != (uint64_t)n)
            v = p > 0 && keys[p - 1] == key ? (vals[p - 1] >> 1) : (kWrap | (vals[lastOf[key]] >> 1));
        pred[vals[p]] = v;
    }
}

// ---- one giant island in spatial clusters -------------------------------
//
// The same dataflow with coarser, local steps: the island's bodies are cut
// into as many spatial clusters (Morton order) as the grid has blocks, each
// row belongs to the cluster of its first dynamic body, and block c runs its
// cluster's rows colour by colour with a block barrier between colours. Rows
// whose predecessor on a body lies in another cluster wait for that row's
// sweep counter; all others are ordered by the block barrier. Most chain steps
// therefore stay inside a block. A block takes its (sweep, colour) steps in
// order, which keeps the earliest unfinished step runnable; waits are bounded.

VXD uint32_t spreadBits10(uint32_t v) {  // 10 bits -> every third bit
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

__global__ void clusterBodyKeyKernel(SolveArgs A, const uint32_t* bodyPos, uint32_t nb, const Counters* C,
                                     uint64_t* keys, uint32_t* vals) {
    const float lo[3] = {fromOrdered(C->cellMinBits[0]), fromOrdered(C->cellMinBits[1]), fromOrdered(C->cellMinBits[2])};
    const float hi[3] = {fromOrdered(C->cellMaxBits[0]), fromOrdered(C->cellMaxBits[1]), fromOrdered(C->cellMaxBits[2])};
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nb; k += gridDim.x * blockDim.x) {
        const uint32_t id = A.bodyOrder[bodyPos[k]];
        const float4 p = A.B.pos[id];
        const float x[3] = {p.x, p.y, p.z};
        uint32_t code = 0;
        for (int a = 0; a < 3; ++a) {
            const float span = fmaxf(hi[a] - lo[a], 1e-6f);
            float t = (x[a] - lo[a]) / span;
            t = t >= 0.0f ? fminf(t, 1.0f) : 0.0f;  // NaN (no bounds) -> 0
            code |= spreadBits10((uint32_t)(t * 1023.0f)) << a;
        }
        keys[k] = code;
        vals[k] = id;
    }
}

// Cluster of each giant-island body: its Morton rank chunked into `clusters`.
__global__ void clusterOfBodyKernel(const uint32_t* sortedIds, uint32_t nb, uint32_t clusters, uint32_t* clusterOf) {
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < nb; r += gridDim.x * blockDim.x)
        clusterOf[sortedIds[r]] = (uint32_t)(((uint64_t)r * clusters) / nb);
}

VXD uint32_t segmentOf(const uint32_t* segStart, uint32_t g0, uint32_t g1, uint32_t k) {
    uint32_t lo = g0, hi = g1;  // last g with segStart[g] <= k
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (segStart[mid] <= k) lo = mid; else hi = mid;
    }
    return lo;
}

VXD uint32_t rowCluster(const SolveArgs& A, uint32_t k, const uint32_t* clusterOf) {
    const uint2 ab = A.rowBodies[k];
    return clusterOf[isDynamic(A.B.filt[ab.x].x) ? ab.x : ab.y];
}

// (cluster, colour slot) cell of a giant row: colour slot = colour within its
// island. Rows of the null island (no dynamic body of their own island) go to
// cluster 0: they are never solved and link to nothing.
VXD uint32_t rowBlock(const SolveArgs& A, uint32_t k, const uint32_t* islandOf, const uint32_t* clusterOf) {
    return islandOf[k] < A.realIslands ? rowCluster(A, k, clusterOf) : 0u;
}

VXD uint32_t rowCell(const SolveArgs& A, uint32_t k, const uint32_t* islandOf, const uint32_t* clusterOf,
                     uint32_t G) {
    const uint32_t isl = islandOf[k];
    const uint32_t g0 = A.islandSeg[isl], g1 = A.islandSeg[isl + 1];
    return rowBlock(A, k, islandOf, clusterOf) * G + (segmentOf(A.segStart, g0, g1, k) - g0);
}

// Links the clustered solve waits on. A predecessor in the row's own cluster
// ran in the same block, in an earlier (sweep, colour) step: a same-sweep
// predecessor has a lower colour of the same island, a wrapped one belongs to
// the previous sweep, and the block barrier after every step orders it. Only
// predecessors in other clusters stay linked (clusterPred), and only rows that
// such a link names publish their sweep counter (remote = 1).
__global__ void clusterLinkKernel(SolveArgs A, const uint32_t* rowList, uint32_t R, const uint32_t* islandOf,
                                  const uint32_t* clusterOf, const uint32_t* pred, uint32_t* clusterPred,
                                  uint32_t* remote) {
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < R; t += gridDim.x * blockDim.x) {
        const uint32_t k = rowList[t];
        const uint32_t own = rowBlock(A, k, islandOf, clusterOf);
        for (int side = 0; side < 2; ++side) {
            const uint32_t p = pred[2 * k + side];
            uint32_t link = kNoPred;
            if (p != kNoPred && rowBlock(A, p & ~kWrap, islandOf, clusterOf) != own) {
                link = p;
                remote[p & ~kWrap] = 1u;
            }
            clusterPred[2 * k + side] = link;
        }
    }
}

__global__ void clusterCountKernel(SolveArgs A, const uint32_t* rowList, uint32_t R, const uint32_t* islandOf,
                                   const uint32_t* clusterOf, uint32_t G, uint32_t* counts) {
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < R; t += gridDim.x * blockDim.x)
        atomicAdd(counts + rowCell(A, rowList[t], islandOf, clusterOf, G), 1u);
}

__global__ void clusterScatterKernel(SolveArgs A, const uint32_t* rowList, uint32_t R, const uint32_t* islandOf,
                                     const uint32_t* clusterOf, uint32_t G, const uint32_t* start, uint32_t* fill,
                                     uint32_t* rows) {
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < R; t += gridDim.x * blockDim.x) {
        const uint32_t k = rowList[t];
        const uint32_t cell = rowCell(A, k, islandOf, clusterOf, G);
        rows[start[cell] + atomicAdd(fill + cell, 1u)] = k;
    }
}

// Shared-memory index of a block's cluster: the start of each of its G colour
// cells relative to the block's first row (G + 1 words, padded to 16 bytes),
// then per row its solve position, contact index and two bodies. A step then
// reads its rows' indices from shared memory instead of three dependent global
// loads (cell start, row, contact index and bodies). A block whose rows do not
// fit reads them from global memory.
constexpr int kClusterThreads = 256;               // threads of a cluster block
constexpr uint32_t kClusterSmemBytes = 64u * 1024u;  // its shared-memory index

VXD uint32_t clusterHeadWords(uint32_t G) { return (G + 1u + 3u) & ~3u; }

VXD bool clusterIndexFits(uint32_t G, uint32_t rowsInBlock) {
    return (uint64_t)clusterHeadWords(G) * 4u + (uint64_t)rowsInBlock * 16u <= (uint64_t)kClusterSmemBytes;
}

// One unit (sweep) step of block c's cluster for colour slot gl; false = abort.
// `pred`: the cross-cluster links (clusterLinkKernel); `remote`: rows that
// publish their sweep counter. `resident`: the block's index is in shared
// memory (cellStart, info); else the rows come from start/rows in global memory.
VXD bool clusterStep(const SolveArgs& A, const uint32_t* start, const uint32_t* rows, bool resident,
                     const uint32_t* cellStart, const uint4* info, uint32_t base, uint32_t gl, int u, int op,
                     const uint32_t* pred, const uint32_t* remote, uint32_t* done, CoopState* st, int* abortFlag) {
    const uint32_t i0 = resident ? cellStart[gl] : start[base + gl];
    const uint32_t i1 = resident ? cellStart[gl + 1] : start[base + gl + 1];
    for (uint32_t idx = i0 + threadIdx.x; idx < i1; idx += blockDim.x) {
        uint32_t k;
        GiantRowIn in;
        if (resident) {
            const uint4 r = info[idx];
            k = r.x;
            in.ab = make_uint2(r.z, r.w);
            in.cp = A.contacts + r.y;
            loadContactCoherent(in.cp, in.cc);
            if (op == 0 || op == 1) coherentPrep(A.prep + k, in.P);
        } else {
            k = rows[idx];
            giantRowFetch(A, k, op, in);
        }
        const uint32_t p0 = pred[2 * k], p1 = pred[2 * k + 1];
        if (p0 != kNoPred || p1 != kNoPred) {
            const uint32_t need0 = (p0 & kWrap) ? (uint32_t)u : (uint32_t)u + 1u;
            const uint32_t need1 = (p1 & kWrap) ? (uint32_t)u : (uint32_t)u + 1u;
            bool ok = true;
            uint32_t nap = 16;
            for (uint32_t spins = 0;; ++spins) {
                const uint32_t d0 = p0 == kNoPred ? 0xffffffffu : ldAcquire(done + (p0 & ~kWrap));
                const uint32_t d1 = p1 == kNoPred ? 0xffffffffu : ldAcquire(done + (p1 & ~kWrap));
                if (d0 >= need0 && d1 >= need1) break;
                if (spins > st->spinLimit || ((spins & 63u) == 63u && __ldcg(&st->timeout))) {
                    atomicOr(&st->timeout, 1u);
                    ok = false;
                    break;
                }
                __nanosleep(nap);
                if (nap < 256u) nap <<= 1;
            }
            if (!ok) { *abortFlag = 1; break; }
        }
        giantRowRun(A, k, op, in);
        if (remote[k]) stRelease(done + k, (uint32_t)u + 1u);
    }
    __syncthreads();
    return *abortFlag == 0;
}

__global__ void __launch_bounds__(kClusterThreads) solveClusterKernel(SolveArgs A, uint32_t G, const uint32_t* start,
                                                          const uint32_t* rows, const uint32_t* rowList, uint32_t R,
                                                          const uint32_t* bodyIds, uint32_t NB, const uint32_t* pred,
                                                          const uint32_t* remote, uint32_t* done, CoopState* st) {
    extern __shared__ uint4 clusterSmem[];  // kClusterSmemBytes: the block's cluster index
    __shared__ int abortFlag;
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    const uint32_t base = blockIdx.x * G;
    const uint32_t s0 = start[base], s1 = start[base + G];
    const bool resident = G > 0 && clusterIndexFits(G, s1 - s0);
    uint32_t* cellStart = reinterpret_cast<uint32_t*>(clusterSmem);
    uint4* info = clusterSmem + clusterHeadWords(G) / 4u;
    if (resident) {
        for (uint32_t t = threadIdx.x; t <= G; t += blockDim.x) cellStart[t] = start[base + t] - s0;
        for (uint32_t i = threadIdx.x; i < s1 - s0; i += blockDim.x) {
            const uint32_t k = rows[s0 + i];
            const uint2 ab = A.rowBodies[k];
            info[i] = make_uint4(k, A.order[k], ab.x, ab.y);
        }
    }
    if (threadIdx.x == 0) abortFlag = 0;
    __syncthreads();
    if (A.positionIterations > 0) {
        for (uint32_t t = tid; t < R; t += stride) __stcg(done + rowList[t], 0u);
        if (!gridSync(&st->bar, &st->timeout, st->spinLimit)) return;
        for (int u = 0; u < A.positionIterations; ++u)
            for (uint32_t gl = 0; gl < G; ++gl)
                if (!clusterStep(A, start, rows, resident, cellStart, info, base, gl, u, 2, pred, remote, done, st,
                                 &abortFlag))
                    return;
        gridSync(&st->bar, &st->timeout, st->spinLimit);
        return;
    }
    for (int s = 0; s < A.substeps; ++s) {
        for (uint32_t t = tid; t < NB; t += stride) {
            const uint32_t id = bodyIds[t];
            if (A.integrate && s > 0) giantIntegrateVelocity(A, id);
            __stcg(A.frames + id, pack(inertiaFrameAt(loadMass(A.B, id), q4(ldcg4(A.B.rot + id)))));
        }
        if (!gridSync(&st->bar, &st->timeout, st->spinLimit)) return;
        for (uint32_t t = tid; t < R; t += stride) {
            const uint32_t k = rowList[t];
            giantRow(A, k, 3);
            __stcg(done + k, 0u);
        }
        if (!gridSync(&st->bar, &st->timeout, st->spinLimit)) return;
        const int warmUnits = A.warmStart && s == 0 ? 1 : 0;
        for (int u = 0; u < warmUnits + A.sweeps; ++u)
            for (uint32_t gl = 0; gl < G; ++gl)
                if (!clusterStep(A, start, rows, resident, cellStart, info, base, gl, u, u < warmUnits ? 0 : 1, pred,
                                 remote, done, st, &abortFlag))
                    return;
        if (!gridSync(&st->bar, &st->timeout, st->spinLimit)) return;
        if (A.integrate) {
            for (uint32_t t = tid; t < NB; t += stride) giantIntegrateTransform(A, bodyIds[t]);
            if (!gridSync(&st->bar, &st->timeout, st->spinLimit)) return;
        }
    }
}

// The block kernel's complement among the islands above tinyLimit.
VXD bool isGiant(const SolveArgs& A, uint32_t isl) {
    const uint32_t rows = A.islandStart[isl + 1] - A.islandStart[isl];
    const uint32_t nb = isl < A.realIslands ? A.bodyStart[isl + 1] - A.bodyStart[isl] : 0u;
    return rows > A.tinyLimit && (nb > (uint32_t)kBlockBodies || rows > (uint32_t)kBlockRows);
}

__global__ void giantEntryKernel(SolveArgs A, const uint32_t* islandOf, uint32_t m, uint32_t n, uint64_t* keys,
                                 uint32_t* vals, uint2* rowBodies) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
        const bool giant = isGiant(A, islandOf[k]);
        const vx_contact& c = A.contacts[A.order[k]];
        rowBodies[k] = make_uint2(c.a, c.b);
        const uint32_t fa = A.B.filt[c.a].x, fb = A.B.filt[c.b].x;
        const bool solved = giant && solvedContact(fa, fb);
        keys[2 * k] = solved && isDynamic(fa) ? c.a : n;
        keys[2 * k + 1] = solved && isDynamic(fb) ? c.b : n;
        vals[2 * k] = 2 * k;
        vals[2 * k + 1] = 2 * k + 1;
    }
}

__global__ void coopTimeoutKernel(const CoopState* st, Counters* C) {
    if (blockIdx.x == 0 && threadIdx.x == 0 && st->timeout) atomicOr(&C->timeout, 1u);
}

__global__ void giantListKernel(SolveArgs A, uint32_t* list, uint32_t* count) {
    for (uint32_t isl = blockIdx.x * blockDim.x + threadIdx.x; isl < A.islands; isl += gridDim.x * blockDim.x)
        if (isGiant(A, isl)) list[atomicAdd(count, 1u)] = isl;
}

// Giant-island membership of the sorted body positions and of the solve
// positions (flags for compaction), and the largest colour count of a giant.
__global__ void giantMemberKernel(SolveArgs A, const uint64_t* bodyKeys, uint32_t n, const uint32_t* islandOf,
                                  uint32_t m, uint32_t* bodyFlags, uint32_t* rowFlags, Counters* C) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride) {
        const uint64_t isl = bodyKeys[k];
        bodyFlags[k] = isl < A.realIslands && isGiant(A, (uint32_t)isl) ? 1u : 0u;
    }
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += stride) {
        const uint32_t isl = islandOf[k];
        const bool g = isGiant(A, isl);
        rowFlags[k] = g ? 1u : 0u;
        if (g && k == A.islandStart[isl]) atomicMax(&C->clusterColours, A.islandSeg[isl + 1] - A.islandSeg[isl]);
    }
}

// Fallback when the device cannot run a cooperative grid: one block per giant island.
__global__ void __launch_bounds__(kBlockThreads) solveGiantBlockKernel(SolveArgs A, const uint32_t* giants) {
    solveIslandGlobal(A, giants[blockIdx.x]);
}

// Bodies without contacts: the substep loop's integration only.
__global__ void freeBodiesKernel(BodyArrays B, const uint32_t* bodyOrder, uint32_t from, uint32_t to, V3 g, float h,
                                 int substeps) {
    for (uint32_t k = from + blockIdx.x * blockDim.x + threadIdx.x; k < to; k += gridDim.x * blockDim.x) {
        const uint32_t i = bodyOrder[k];
        for (int s = 0; s < substeps; ++s) {
            if (s > 0) integrateVelocity(B, i, g, h);
            integrateTransform(B, i, h);
        }
    }
}

// ---------------------------------------------------------------------------
// conservative-advancement rewind (src/world.cpp:4233-4357, gapAt :2916-2958)
// ---------------------------------------------------------------------------

struct GapProbe { float gap; V3 normal; };

VXD BodyView withPose(BodyView b, const V3& p, const Q4& q) {
    b.p = p;
    b.q = q;
    return b;
}

// Distance query of the rewind: gjkDistance's results, the common case in registers.
VXD GjkResult distanceQuery(const Convex& ca, const Convex& cb) { return gjkDistanceQuick(ca, cb); }

// meshSimpleGapProbe (narrowphase.h:719-749): the smallest gap (strictly
// smaller replaces) between `a` and the triangles of mesh `b` whose BVH
// leaves overlap a cube of half width `search` around a's position.
__device__ __noinline__ void meshGap(const BodyView& a, const BodyView& b, const Soup& soup, float search,
                                     GapProbe& best) {
    const vx_mesh& m = soup.meshes[b.hullFirst];
    const V3 lo = a.p - V3{search, search, search}, hi = a.p + V3{search, search, search};
    const Convex ca = makeConvex(a, soup);
    meshVisit(soup, m, lo, hi, [&](uint32_t tri) {
        const GjkResult g = distanceQuery(ca, meshTriangle(soup, m, tri));
        if (g.distance < best.gap) best = GapProbe{g.distance, g.normal};
        return true;
    });
}

// gapAt (world.cpp:2916-2958) for two non-compound bodies, b not a mesh.
VXD GapProbe gapConvex(const BodyView& a, const BodyView& b, const Soup& soup) {
    if (shapeOf(b.flags) == kPlane) {
        const Convex c = makeConvex(a, soup);
        const V3 deep = c.position + supportOffsetBody(c, -b.planeN);
        return GapProbe{dot(b.planeN, deep) - b.planeOff - c.radius, b.planeN};
    }
    const GjkResult r = distanceQuery(makeConvex(a, soup), makeConvex(b, soup));
    return GapProbe{r.distance, r.normal};
}

// gapAt's compound and mesh cases: the minimum over every child pair (A's
// children outer, B's inner) and every searched triangle, the first minimum
// kept, starting from (1e30, +y) as the reference's recursion does.
__device__ __noinline__ GapProbe gapComplex(const BodyView& a, const BodyView& b, const Soup& soup, float search) {
    GapProbe best{1e30f, V3{0.0f, 1.0f, 0.0f}};
    const bool ca = shapeOf(a.flags) == kCompound, cb = shapeOf(b.flags) == kCompound;
    const uint32_t countA = ca ? a.hullCount : 1u, countB = cb ? b.hullCount : 1u;
    for (uint32_t x = 0; x < countA; ++x) {
        const BodyView ga = ca ? compoundChildView(a, soup.children[a.hullFirst + x]) : a;
        for (uint32_t y = 0; y < countB; ++y) {
            const BodyView gb = cb ? compoundChildView(b, soup.children[b.hullFirst + y]) : b;
            if (shapeOf(gb.flags) == kMesh) {
                meshGap(ga, gb, soup, search, best);
            } else {
                const GapProbe g = gapConvex(ga, gb, soup);
                if (g.gap < best.gap) best = g;
            }
        }
    }
    return best;
}

// Signed gap and normal (from b towards a) of the rewind's distance oracle;
// `dt` sizes the mesh search cube as the rewind loop does (world.cpp:4272-4273).
__device__ __noinline__ GapProbe gapAt(const BodyView& a, const BodyView& b, const Soup& soup, float dt) {
    if (isComplexShape(shapeOf(a.flags)) || isComplexShape(shapeOf(b.flags))) {
        const float search = maxPointSpeed(a) * dt + a.radius + length(a.half) + a.hh + 0.1f;
        return gapComplex(a, b, soup, search);
    }
    return gapConvex(a, b, soup);
}

// Bounding spheres more than 1 mm apart give a positive end gap, so the
// rewind's `gap >= -8 mm` test skips the pair (planes, meshes and compounds
// have no bounding sphere here).
VXD bool spheresApart(const BodyView& a, const BodyView& b) {
    const float ea = coreExtent(shapeOf(a.flags), a.half, a.radius, a.hh);
    const float eb = coreExtent(shapeOf(b.flags), b.half, b.radius, b.hh);
    if (ea < 0.0f || eb < 0.0f) return false;
    const float reach = ea + eb + 1e-3f;
    return lengthSq(a.p - b.p) > reach * reach;
}

VXD Mass massOfView(const BodyArrays& B, uint32_t i) { return loadMass(B, i); }

// Conditions of the rewind loop for an oriented pair (a dynamic).
VXD bool caEligible(const BodyView& a, const BodyView& b, const BodyArrays& B, uint32_t ia) {
    if (isSensor(a.flags) || isSensor(b.flags)) return false;
    if (!isDynamic(a.flags)) return false;
    const float minVel = B.ccd[ia].y;
    if (!(a.flags & kContinuousBit) || qualityOf(a.flags) == kQualityLow || isLocked(a.flags) ||
        maxPointSpeed(a) < minVel)
        return false;
    return true;
}

VXD void orientPair(const BodyArrays& B, uint64_t key, uint32_t& i, uint32_t& j) {
    i = (uint32_t)(key >> 32);
    j = (uint32_t)key;
    if (!isDynamic(B.filt[i].x) && isDynamic(B.filt[j].x)) { const uint32_t t = i; i = j; j = t; }
}

// `order` (optional): the pairs grouped by shape combination, so that a warp's
// lanes mostly take the same distance-query path; every outcome is written at
// the pair's own index.
__global__ void caProbeKernel(BodyArrays B, Soup soup, const uint64_t* pairKeys, const uint32_t* order,
                              uint32_t npairs, float dt, uint32_t* flags, uint32_t* bodyMark, float4* endGap) {
    for (uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x; slot < npairs; slot += gridDim.x * blockDim.x) {
        const uint32_t r = order ? order[slot] : slot;
        uint32_t i, j;
        orientPair(B, pairKeys[r], i, j);
        const BodyView a = loadView(B, i), b = loadView(B, j);
        uint32_t flag = 0;
        if (!spheresApart(a, b) && caEligible(a, b, B, i)) {
            const GapProbe end = gapAt(a, b, soup, dt);
            if (end.gap < -8e-3f) {
                flag = 1;
                endGap[r] = make_float4(end.gap, end.normal.x, end.normal.y, end.normal.z);
                bodyMark[i] = 1;  // only dynamic bodies move in a rewind
                if (isDynamic(b.flags)) bodyMark[j] = 1;
            }
        }
        flags[r] = flag;
    }
}

__global__ void caCandidateKernel(const BodyArrays B, const uint64_t* pairKeys, uint32_t npairs, uint32_t* flags,
                                  const uint32_t* bodyMark, uint32_t* candidates, Counters* C) {
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < npairs; r += gridDim.x * blockDim.x) {
        const uint32_t i = (uint32_t)(pairKeys[r] >> 32), j = (uint32_t)pairKeys[r];
        if (flags[r] || bodyMark[i] || bodyMark[j]) candidates[r] = 1;
        else candidates[r] = 0;
    }
}

VXD Q4 orientationAt(const Mass& m, const Q4& start, const V3& L, float elapsed) {
    Q4 q = start;
    V3 w = invInertiaMulAt(m, L, start);
    advanceOrientation(m, q, w, elapsed);
    return q;
}

// Full rewind logic for one oriented pair on the current state. Returns true
// when the pair was rewound.
// `cached`: the probe's end-state gap for this pair when neither body has
// moved since the probe (else null: computed here). `spec` (optional): write
// the rewound states there (a: pos, rot, vel, ang; then b) instead of into B.
__device__ __noinline__ bool caRewind(BodyArrays& B, const Soup& soup, uint32_t i, uint32_t j, float dt,
                                      const float4* prevPos, const float4* prevRot, uint32_t* gapQueries,
                                      const float4* cached, float4* spec = nullptr) {
    BodyView a = loadViewCoherent(B, i), b = loadViewCoherent(B, j);
    if (!caEligible(a, b, B, i)) return false;
    if (spheresApart(a, b)) return false;  // positive end gap, no rewind (the probe's test)
    GapProbe end;
    if (cached) {
        const float4 g = *cached;
        end = GapProbe{g.x, V3{g.y, g.z, g.w}};
    } else {
        end = gapAt(a, b, soup, dt);
    }
    if (end.gap >= -8e-3f) return false;
    const bool bStatic = isStaticBody(b.flags), bDyn = isDynamic(b.flags);
    const V3 pa0 = f3(prevPos[i]), da = a.p - pa0;
    const Q4 qa0 = q4(prevRot[i]);
    const V3 pb0 = bStatic ? b.p : f3(prevPos[j]);
    const V3 db = b.p - pb0;
    const Q4 qb0 = bStatic ? b.q : q4(prevRot[j]);
    const float bound = maxPointSpeed(a) * dt + (bStatic ? 0.0f : maxPointSpeed(b) * dt);
    if (bound < 1e-9f) return false;
    const Mass ma = loadMass(B, i), mb = loadMass(B, j);
    const V3 La = inertiaMulAt(ma, a.w, a.q);
    const V3 Lb = bDyn ? inertiaMulAt(mb, b.w, b.q) : V3{0.0f, 0.0f, 0.0f};
    float t = 0.0f;
    V3 n = end.normal;
    uint32_t queries = 1;
    for (int iter = 0; iter < 24 && t < 1.0f; ++iter) {
        ++queries;
        const Q4 qa = orientationAt(ma, qa0, La, dt * t);
        const Q4 qb = bStatic ? qb0 : orientationAt(mb, qb0, Lb, dt * t);
        const GapProbe g = gapAt(withPose(a, pa0 + da * t, qa), withPose(b, pb0 + db * t, qb), soup, dt);
        n = g.normal;
        if (g.gap < 1e-3f) break;
        t = vmin(1.0f, t + g.gap / bound);
    }
    atomicAdd(gapQueries, queries);
    if (t >= 1.0f) return false;
    a.p = pa0 + da * t;
    a.q = qa0;
    a.w = invInertiaMulAt(ma, La, qa0);
    advanceOrientation(ma, a.q, a.w, dt * t);
    if (bDyn) {
        b.p = pb0 + db * t;
        b.q = qb0;
        b.w = invInertiaMulAt(mb, Lb, qb0);
        advanceOrientation(mb, b.q, b.w, dt * t);
    }
    const float ima = solverInvMass(ma), imb = solverInvMass(mb);
    const float vn = dot(a.v - b.v, n);
    const float invMassSum = ima + imb;
    if (vn < 0.0f && invMassSum > 0.0f) {
        const float restitution = vn < -1.0f
            ? combineMaterial(a.restitution, b.restitution, (a.flags >> kRestitutionCombineShift) & 7u,
                              (b.flags >> kRestitutionCombineShift) & 7u)
            : 0.0f;
        const float impulse = -(1.0f + restitution) * vn / invMassSum;
        a.v += n * (impulse * ima);
        if (bDyn) b.v -= n * (impulse * imb);
    }
    const float remaining = dt * (1.0f - t);
    advanceTransform(ma, a.p, a.q, a.v, a.w, remaining);
    if (bDyn) advanceTransform(mb, b.p, b.q, b.v, b.w, remaining);
    if (spec) {
        spec[0] = pack(a.p, 0.0f); spec[1] = pack(a.q); spec[2] = pack(a.v, 0.0f); spec[3] = pack(a.w, 0.0f);
        spec[4] = pack(b.p, 0.0f); spec[5] = pack(b.q); spec[6] = pack(b.v, 0.0f); spec[7] = pack(b.w, 0.0f);
        return true;
    }
    B.pos[i] = pack(a.p, 0.0f); B.rot[i] = pack(a.q); B.vel[i] = pack(a.v, 0.0f); B.ang[i] = pack(a.w, 0.0f);
    if (bDyn) {
        B.pos[j] = pack(b.p, 0.0f); B.rot[j] = pack(b.q); B.vel[j] = pack(b.v, 0.0f); B.ang[j] = pack(b.w, 0.0f);
    }
    return true;
}

VXD uint64_t globalTimerNs() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Every flagged pair evaluated in parallel on the probe's state (read-only):
// in the ordered pass, a flagged pair whose bodies no earlier rewind has moved
// sees exactly this state, so its outcome can be taken from here.
// `spread` (1..32): threads per pair, so that a few pairs occupy many SMs
// and share warps with few others (each is a long serial loop). The working
// lanes are the first 32 / spread of each warp: local memory interleaves the
// lanes' words, so contiguous lanes share L1 sectors of their stack frames
// (lanes 0-7 use one sector of every line).
__global__ void caSpeculateKernel(BodyArrays B, Soup soup, const uint64_t* pairKeys, const uint32_t* flaggedList,
                                  uint32_t flagged, uint32_t spread, const float4* endGap, float dt,
                                  const float4* prevPos, const float4* prevRot, float4* specState,
                                  uint32_t* specResult, Counters* C) {
    const uint32_t perWarp = 32u / spread, lane = threadIdx.x & 31u;
    if (lane >= perWarp) return;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t k = warp * perWarp + lane; k < flagged; k += warps * perWarp) {
        const uint32_t r = flaggedList[k];
        uint32_t i, j;
        orientPair(B, pairKeys[r], i, j);
        const uint64_t t0 = globalTimerNs();
        specResult[k] = caRewind(B, soup, i, j, dt, prevPos, prevRot, &C->caGapQueries, endGap + r,
                                 specState + 8 * (size_t)k) ? 1u : 0u;
        atomicMax(&C->caSpecMicros, (uint32_t)((globalTimerNs() - t0) / 1000u));
    }
}

// Rewind pass over the candidate pairs as a dataflow. A candidate's
// predecessors are the latest earlier candidates sharing one of its dynamic
// bodies; it becomes ready when both have finished and is then evaluated
// exactly as the reference's single ordered loop would evaluate it: it sees
// the same body states and rewound marks, as long as no rewind moves a body
// outside the marked set (that case is flagged; the caller widens the set and
// replays the pass from a snapshot). Workers (lane 0 of a warp) take ready
// candidates from a queue, so independent chains never wait for one another.
// Cooperative launch (all workers resident); every wait is bounded.
constexpr int kCaWidenLimit = 8;  // replays with a widened marked set before the serial loop
constexpr uint32_t kProbeGroupMin = 8192;  // pairs from which the probe groups them by shape combination
constexpr int kCaWidenHops = 8;   // hops of widening per replay
constexpr int kCaInitialHops = 8; // hops of widening before the first pass
// Workers of the rewind pass: one block of kCaFlowThreads threads per SM, one
// worker lane per warp. A worker's distance queries keep a stack frame of
// about 10 KB (simplex, EPA polytope) in local memory, where one active lane
// takes a 32-byte L1 sector per 4-byte word: several workers on an SM evict
// one another's frames. On a settled 100k-body pile a distance query took
// 18 us with 1 worker per SM, 31 us with 2, 64 us with 4 and 127 us with 8,
// at about the same queries per SM per second. The pass is bound by its
// longest dependency chain, so one fast worker per SM wins (chain 5.0 ms,
// against 8.1 ms with 2 and 12.1 ms with 8; the pass's 24k evaluations still
// fit beside it).
constexpr int kCaFlowThreads = 32;
constexpr int kCaFlowBlocksPerSm = 1;

__global__ void __launch_bounds__(256) caFlowKernel(BodyArrays B, Soup soup, const uint32_t* flagRank,
                                                    const float4* specState, const uint32_t* specResult,
                                                    const uint4* info, uint32_t ncand, const uint32_t* succ,
                                                    uint32_t* pending, uint32_t* queue, uint32_t* depth,
                                                    uint32_t* crit, const uint32_t* bodyMark, uint32_t* rewound,
                                                    float dt, const float4* prevPos, const float4* prevRot,
                                                    Counters* C, CoopState* st) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    uint32_t* tail = &st->queued[0];
    uint32_t* head = &st->queued[1];
    for (uint32_t k = tid; k < ncand; k += stride)  // roots
        if (pending[k] == 0u) {
            const uint32_t t = atomicAdd(tail, 1u);
            if (t < ncand) __stcg(queue + t, k);
            else atomicOr(&st->spill, 4u);  // pushed twice: inconsistent links
        }
    // Every root is queued before any worker starts: a count that a finished
    // candidate has taken to zero must not read as a root.
    if (!gridSync(&st->bar, &st->timeout, st->spinLimit)) return;
    if ((threadIdx.x & 31u) != 0u) return;
    uint32_t rewinds = 0, maxDepth = 0, maxCrit = 0;
    for (;;) {
        const uint32_t h = atomicAdd(head, 1u);
        if (h >= ncand) break;
        // Claimed before it was filled. Idle workers back off (up to ~1 us) and
        // read the shared timeout word only every 16th poll: a thousand warps
        // polling one L2 line at full rate slow the working lanes' own loads.
        uint32_t k, spins = 0, nap = 32;
        while ((k = __ldcg(queue + h)) == kNoPred) {
            if (++spins > st->spinLimit || ((spins & 15u) == 0u && __ldcg(&st->timeout))) {
                atomicOr(&st->timeout, 1u);
                return;
            }
            __nanosleep(nap);
            if (nap < 1024u) nap <<= 1;
        }
        __threadfence();  // acquire the predecessors' writes
        const uint64_t t0 = globalTimerNs();
        // record, successors and chain statistics in one round of loads (the
        // predecessors raised depth and crit before they released this one)
        const uint4 rec = info[k];
        const uint2 next = reinterpret_cast<const uint2*>(succ)[k];
        const uint32_t d = __ldcg(depth + k) + 1u;
        const uint32_t crit0 = __ldcg(crit + k);
        const uint32_t i = rec.y, j = rec.z;
        const bool jDyn = (rec.w & 2u) != 0u;
        const bool touched = __ldcg(rewound + i) || __ldcg(rewound + j);
        if ((rec.w & 1u) || touched) {
            bool rewoundPair;
            if (!touched) {  // flagged, bodies as the probe saw them: the speculative outcome holds
                const uint32_t sk = flagRank[rec.x];
                rewoundPair = specResult[sk] != 0u;
                if (rewoundPair) {
                    const float4* st4 = specState + 8 * (size_t)sk;
                    __stcg(B.pos + i, st4[0]); __stcg(B.rot + i, st4[1]); __stcg(B.vel + i, st4[2]); __stcg(B.ang + i, st4[3]);
                    if (jDyn) {
                        __stcg(B.pos + j, st4[4]); __stcg(B.rot + j, st4[5]); __stcg(B.vel + j, st4[6]);
                        __stcg(B.ang + j, st4[7]);
                    }
                }
            } else {
                rewoundPair = caRewind(B, soup, i, j, dt, prevPos, prevRot, &C->caGapQueries, nullptr);
            }
            if (rewoundPair) {
                ++rewinds;
                __stcg(rewound + i, 1u);
                if (jDyn) __stcg(rewound + j, 1u);
                if (!bodyMark[i] || (jDyn && !bodyMark[j])) atomicOr(&C->caOverflow, 1u);
            }
        }
        const uint64_t elapsed = globalTimerNs() - t0;
        const uint32_t ck = crit0 + (uint32_t)(elapsed < 0x7fffffffull ? elapsed : 0x7fffffffull);
        maxDepth = max(maxDepth, d);
        maxCrit = max(maxCrit, ck);
        __threadfence();  // release this evaluation's writes before the successors can run
        // both successors' counts drop in one round; a count that reaches
        // zero queues its candidate (the same one twice only if it follows
        // this one on both bodies, and then only the second drop reaches zero)
        uint32_t left0 = 0u, left1 = 0u;
        if (next.x != kNoPred) {
            atomicMax(depth + next.x, d);
            atomicMax(crit + next.x, ck);
            left0 = atomicSub(pending + next.x, 1u);
        }
        if (next.y != kNoPred) {
            atomicMax(depth + next.y, d);
            atomicMax(crit + next.y, ck);
            left1 = atomicSub(pending + next.y, 1u);
        }
        const uint32_t ready = (left0 == 1u ? 1u : 0u) + (left1 == 1u ? 1u : 0u);
        if (ready) {
            uint32_t t = atomicAdd(tail, ready);
            if (left0 == 1u) {
                if (t < ncand) __stcg(queue + t, next.x);
                else atomicOr(&st->spill, 4u);
                ++t;
            }
            if (left1 == 1u) {
                if (t < ncand) __stcg(queue + t, next.y);
                else atomicOr(&st->spill, 4u);
            }
        }
    }
    if (rewinds) atomicAdd(&C->rewinds, rewinds);
    atomicMax(&st->rounds, maxDepth);
    atomicMax(&C->caCritMicros, maxCrit / 1000u);
}

// Entries (dynamic body, 2k + side) of the candidates; other endpoints sort last.
// Also the candidate's record for the pass: (pair, oriented bodies i and j,
// bit 0 flagged by the probe | bit 1 j dynamic), one load for the worker.
__global__ void caEntryKernel(const BodyArrays B, const uint64_t* pairKeys, const uint32_t* cand, uint32_t ncand,
                              uint32_t n, const uint32_t* flags, uint64_t* keys, uint32_t* vals, uint4* info) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < ncand; k += gridDim.x * blockDim.x) {
        const uint32_t r = cand[k];
        const uint64_t key = pairKeys[r];
        const uint32_t a = (uint32_t)(key >> 32), b = (uint32_t)key;
        keys[2 * k] = isDynamic(B.filt[a].x) ? a : n;
        keys[2 * k + 1] = isDynamic(B.filt[b].x) ? b : n;
        vals[2 * k] = 2 * k;
        vals[2 * k + 1] = 2 * k + 1;
        uint32_t i, j;
        orientPair(B, key, i, j);
        info[k] = make_uint4(r, i, j, (flags[r] ? 1u : 0u) | (isDynamic(B.filt[j].x) ? 2u : 0u));
    }
}

// Entries sorted stably by body: consecutive entries of one body link a
// candidate to its successor on that body (pending counts its predecessors).
__global__ void caLinkKernel(const uint64_t* keys, const uint32_t* vals, uint32_t entries, uint32_t n,
                             uint32_t* succ, uint32_t* pending) {
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < entries; p += gridDim.x * blockDim.x) {
        const uint64_t key = keys[p];
        const bool body = key != (uint64_t)n;
        const bool next = body && p + 1 < entries && keys[p + 1] == key;
        succ[vals[p]] = next ? (vals[p + 1] >> 1) : kNoPred;
        if (body && p > 0 && keys[p - 1] == key) atomicAdd(pending + (vals[p] >> 1), 1u);
    }
}

// Widen the marked set after a failed pass, one hop per launch: both dynamic
// endpoints of every pair touching a frontier body (the first frontier is
// the set of bodies the pass rewound); bodies marked here form the next one.
// Marking ahead of the cascade means fewer replays.
__global__ void caWidenKernel(const BodyArrays B, const uint64_t* pairKeys, uint32_t npairs, uint32_t* bodyMark,
                              const uint32_t* frontier, uint32_t* next) {
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < npairs; r += gridDim.x * blockDim.x) {
        const uint32_t i = (uint32_t)(pairKeys[r] >> 32), j = (uint32_t)pairKeys[r];
        if (!frontier[i] && !frontier[j]) continue;
        if (isDynamic(B.filt[i].x) && atomicExch(bodyMark + i, 1u) == 0u) next[i] = 1u;
        if (isDynamic(B.filt[j].x) && atomicExch(bodyMark + j, 1u) == 0u) next[j] = 1u;
    }
}

// The reference's loop verbatim in pair order (one thread): the fallback when
// a rewind cascades beyond the candidate neighbourhood.
__global__ void caFullSerialKernel(BodyArrays B, Soup soup, const uint64_t* pairKeys, uint32_t npairs,
                                   const uint32_t* flags, uint32_t* rewound, float dt, const float4* prevPos,
                                   const float4* prevRot, Counters* C) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    uint32_t rewinds = 0;
    for (uint32_t r = 0; r < npairs; ++r) {
        const uint64_t key = pairKeys[r];
        const uint32_t ri = (uint32_t)(key >> 32), rj = (uint32_t)key;
        if (!(flags[r] || rewound[ri] || rewound[rj])) continue;
        uint32_t i, j;
        orientPair(B, key, i, j);
        if (caRewind(B, soup, i, j, dt, prevPos, prevRot, &C->caGapQueries, nullptr)) {
            ++rewinds;
            rewound[i] = 1;
            if (isDynamic(B.filt[j].x)) rewound[j] = 1;
        }
    }
    C->rewinds = rewinds;
}

__global__ void copyStateKernel(const BodyArrays B, uint32_t n, float4* snap, int restore) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4* s = snap + 4 * (size_t)i;
        if (restore) {
            B.pos[i] = s[0]; B.rot[i] = s[1]; B.vel[i] = s[2]; B.ang[i] = s[3];
        } else {
            s[0] = B.pos[i]; s[1] = B.rot[i]; s[2] = B.vel[i]; s[3] = B.ang[i];
        }
    }
}

// prefix ranks of candidate flags -> candidate index list
__global__ void compactKernel(const uint32_t* flags, const uint32_t* ranks, uint32_t n, uint32_t* out) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        if (flags[k]) out[ranks[k]] = k;
}

__global__ void clearForcesKernel(BodyArrays B, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        B.force[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        B.torque[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
}

__global__ void gatherContactsKernel(const vx_contact* in, const uint32_t* order, uint32_t m, vx_contact* out) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x)
        out[k] = in[order[k]];
}

__global__ void contactKeysKernel(const vx_contact* cs, uint32_t m, uint64_t* keys) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x)
        keys[k] = ((uint64_t)cs[k].a << 32) | cs[k].b;
}

// ===========================================================================
// host orchestration
// ===========================================================================

int sortPairs(Context& c, uint64_t* keys, uint32_t* vals, uint32_t n, int bits) {
    if (n <= 1 || bits <= 0) return VXB_OK;
    const uint32_t tiles = (n + kSortTile - 1) / kSortTile;
    VXB_TRY(ensure(c, c.sortKeysAlt, (size_t)n * 8));
    VXB_TRY(ensure(c, c.sortValsAlt, (size_t)n * 4));
    VXB_TRY(ensure(c, c.sortHist, (size_t)tiles * 256 * 4));
    c.sortScratch.keysAlt = P<uint64_t>(c.sortKeysAlt);
    c.sortScratch.valsAlt = P<uint32_t>(c.sortValsAlt);
    c.sortScratch.hist = P<uint32_t>(c.sortHist);
    cudaError_t e = cudaSuccess;
    c.launches += radixSortPairs(keys, vals, n, 0, bits, c.sortScratch, c.stream, &e);
    if (e != cudaSuccess) return cudaStatus(c, e, "radix sort");
    return VXB_OK;
}

// Union-find roots (parent[i] = the root of i) over the dynamic-dynamic
// contacts of `cs` that involve no sensor (the islands of SleepManager::update,
// src/sleep.cpp:63-91, and of the solve).
int unionRoots(Context& c, const vx_contact* cs, uint32_t m, uint32_t* parent) {
    LAUNCH(c, iotaKernel, blocksFor(c.n, 256), 256, parent, c.n);
    if (m) {
        LAUNCH(c, unionKernel, blocksFor(m, 256), 256, cs, m, c.B, parent, c.dCounters);
        LAUNCH(c, compressKernel, blocksFor(c.n, 256), 256, parent, c.n);
    }
    return VXB_OK;
}

int resetCoop(Context& c, CoopState* st) {
    CoopState init;
    std::memset(&init, 0, sizeof(init));
    init.spinLimit = c.waitLimit;
    VXB_CUDA(c, cudaMemcpyAsync(st, &init, sizeof(init), cudaMemcpyHostToDevice, c.stream));
    return VXB_OK;
}

static int readCounters(Context& c) {
    VXB_CUDA(c, cudaMemcpyAsync(&c.hostCounters, c.dCounters, sizeof(Counters), cudaMemcpyDeviceToHost, c.stream));
    ++c.hostSyncs;
    VXB_CUDA(c, cudaStreamSynchronize(c.stream));
    return VXB_OK;
}

// Launch at a tuned site (tuner.h): `launch(shape)` issues the kernel with
// that block size and grid cap. While the size bucket of `items` has no shape,
// every candidate first runs on the same inputs, `restore()` putting back what
// a launch consumes before each trial and before the real launch.
template <class Launch, class Restore>
static int tunedLaunch(Context& c, int site, uint32_t items, Launch launch, Restore restore) {
    if (c.tuner.undecided(site, items)) {
        c.tuner.beginTrials();
        for (int round = 0; round < kTuneSamples; ++round)
            for (int k = 0; k < kTuneCandidates; ++k) {
                VXB_TRY(restore());
                c.tuner.trialStart(c.stream);
                launch(Tuner::candidate(site, k));
                ++c.hostSyncs;
                const cudaError_t e = c.tuner.trialStop(k, c.stream);
                if (e != cudaSuccess) return cudaStatus(c, e, "launch-shape trial");
            }
        c.tuner.decide(site, items);
        VXB_TRY(restore());
    }
    launch(c.tuner.shapeFor(site, items, nullptr));
    return VXB_OK;
}

// Restores the device counters a narrow-phase launch appends to (contacts,
// records, overflow flags): the first call keeps a device copy, later calls
// put it back.
struct CounterRestore {
    Context& c;
    bool saved = false;
    int operator()() {
        if (!saved) {
            VXB_TRY(ensure(c, c.tuneSaveBuf, sizeof(Counters)));
            VXB_CUDA(c, cudaMemcpyAsync(c.tuneSaveBuf.ptr, c.dCounters, sizeof(Counters), cudaMemcpyDeviceToDevice,
                                        c.stream));
            saved = true;
            return VXB_OK;
        }
        VXB_CUDA(c, cudaMemcpyAsync(c.dCounters, c.tuneSaveBuf.ptr, sizeof(Counters), cudaMemcpyDeviceToDevice,
                                    c.stream));
        return VXB_OK;
    }
};

static int resetCounters(Context& c) {
    Counters z;
    std::memset(&z, 0, sizeof(z));
    for (int a = 0; a < 3; ++a) { z.cellMinBits[a] = 0xffffffffu; z.cellMaxBits[a] = 0u; }
    VXB_CUDA(c, cudaMemcpyAsync(c.dCounters, &z, sizeof(Counters), cudaMemcpyHostToDevice, c.stream));
    return VXB_OK;
}

static uint64_t fnv1a(uint64_t h, const void* data, size_t bytes) {
    const unsigned char* p = static_cast<const unsigned char*>(data);
    for (size_t k = 0; k < bytes; ++k) h = (h ^ p[k]) * 0x100000001b3ull;
    return h;
}

int loadSoup(Context& c, const vx_soup* soup) {
    c.hullPointCount = soup ? soup->hullPointCount : 0;
    c.faceIndexCount = soup ? soup->hullFaceIndexCount : 0;
    VXB_TRY(ensure(c, c.hullPtsBuf, c.hullPointCount * 12 + 16));
    VXB_TRY(ensure(c, c.facesBuf, c.faceIndexCount * 4 + 16));
    if (c.hullPointCount)
        VXB_CUDA(c, cudaMemcpyAsync(c.hullPtsBuf.ptr, soup->hullPoints, c.hullPointCount * 12, cudaMemcpyHostToDevice,
                                    c.stream));
    if (c.faceIndexCount)
        VXB_CUDA(c, cudaMemcpyAsync(c.facesBuf.ptr, soup->hullFaceIndices, c.faceIndexCount * 4,
                                    cudaMemcpyHostToDevice, c.stream));
    // triangle meshes, their BVHs and compound children
    struct Part { DevBuf* buf; const void* src; size_t bytes; };
    const Part parts[] = {
        {&c.vertBuf, soup ? soup->vertices : nullptr, soup ? (size_t)soup->vertexCount * 12 : 0},
        {&c.indexBuf, soup ? soup->indices : nullptr, soup ? (size_t)soup->indexCount * 4 : 0},
        {&c.meshBuf, soup ? soup->meshes : nullptr, soup ? (size_t)soup->meshCount * sizeof(vx_mesh) : 0},
        {&c.nodeBuf, soup ? soup->bvhNodes : nullptr, soup ? (size_t)soup->bvhNodeCount * sizeof(vx_bvh_node) : 0},
        {&c.triRefBuf, soup ? soup->bvhTriRefs : nullptr, soup ? (size_t)soup->bvhTriRefCount * 4 : 0},
        {&c.childBuf, soup ? soup->compoundChildren : nullptr,
         soup ? (size_t)soup->compoundChildCount * sizeof(vx_compound_child) : 0}};
    for (const Part& part : parts) {
        VXB_TRY(ensure(c, *part.buf, part.bytes + 16));
        if (part.bytes)
            VXB_CUDA(c, cudaMemcpyAsync(part.buf->ptr, part.src, part.bytes, cudaMemcpyHostToDevice, c.stream));
    }
    if (soup && soup->meshCount) VXB_CUDA(c, cudaStreamSynchronize(c.stream));  // copies read the caller's arrays
    uint64_t key = 0xcbf29ce484222325ull;
    for (const Part& part : parts) key = fnv1a(key, &part.bytes, sizeof(part.bytes));
    const size_t hull[2] = {c.hullPointCount, c.faceIndexCount};
    c.soupGeometryKey = fnv1a(key, hull, sizeof(hull));
    return VXB_OK;
}

static Soup soupOf(Context& c) {
    return Soup{P<float>(c.hullPtsBuf), P<uint32_t>(c.facesBuf),  P<float>(c.vertBuf),
                P<uint32_t>(c.indexBuf), P<vx_mesh>(c.meshBuf),    P<vx_bvh_node>(c.nodeBuf),
                P<uint32_t>(c.triRefBuf), P<vx_compound_child>(c.childBuf)};
}

int loadBodies(Context& c, const vx_body* bodies, uint32_t n, const uint32_t* worldOf, bool deviceWorld) {
    if (n == 0) return fail(c, VXB_ERR_INVALID, "no bodies");
    // The Backend path reloads the same bodies between its calls of one step
    // (integrate between substeps' solves): the coloured contacts stay valid
    // unless the body set changed.
    if (n != c.n) {
        c.backendContacts = 0;
        c.backendColored = false;
    }
    c.complexShapes = false;
    c.kinematic = false;
    uint64_t key = 0xcbf29ce484222325ull;
    for (uint32_t i = 0; i < n; ++i) {
        const vx_body& b = bodies[i];
        const uint32_t refs[6] = {b.shape, b.meshIndex, b.hullFirst, b.hullCount, b.compoundFirst, b.compoundCount};
        key = fnv1a(key, refs, sizeof(refs));
        key = fnv1a(key, &b.hullFaceFirst, 8);  // hullFaceFirst, hullFaceCount
    }
    c.bodyGeometryKey = key;
    for (uint32_t i = 0; i < n; ++i) {
        const uint8_t s = bodies[i].shape;
        if (s == VX_SHAPE_MESH || s == VX_SHAPE_COMPOUND) c.complexShapes = true;
        if (s == VX_SHAPE_MESH && bodies[i].motionType != VX_MOTION_STATIC)
            return fail(c, VXB_ERR_INVALID, "mesh bodies are static");
        if (deviceWorld && bodies[i].motionType == VX_MOTION_KINEMATIC)
            return fail(c, VXB_ERR_UNSUPPORTED, "kinematic bodies are not supported by the device world");
        if (bodies[i].motionType == VX_MOTION_KINEMATIC) c.kinematic = true;
    }
    c.n = n;
    // SoA arrays in one allocation (16 arrays of 16-byte elements).
    const size_t stride = ((size_t)n * 16 + 255) & ~(size_t)255;
    VXB_TRY(ensure(c, c.bodyBuf, stride * 16));
    char* base = P<char>(c.bodyBuf);
    float4** f4[] = {&c.B.pos, &c.B.rot, &c.B.vel, &c.B.ang, &c.B.inertia, &c.B.iq, &c.B.dims, &c.B.extra,
                     &c.B.mat, &c.B.fscale, &c.B.ccd, &c.B.plane, &c.B.force, &c.B.torque};
    int slot = 0;
    for (float4** p : f4) *p = reinterpret_cast<float4*>(base + stride * slot++);
    c.B.hull = reinterpret_cast<uint4*>(base + stride * slot++);
    c.B.filt = reinterpret_cast<uint4*>(base + stride * slot++);
    VXB_TRY(ensure(c, c.aosBuf, (size_t)n * sizeof(vx_body)));
    VXB_CUDA(c, cudaMemcpyAsync(c.aosBuf.ptr, bodies, (size_t)n * sizeof(vx_body), cudaMemcpyHostToDevice, c.stream));
    LAUNCH(c, packBodiesKernel, blocksFor(n, 256), 256, P<vx_body>(c.aosBuf), n, c.B);
    // worlds and per-world lists of planes and meshes (paired with every body of their world)
    c.hostWorldOf.assign(n, 0u);
    uint32_t worlds = 1;
    if (worldOf) {
        for (uint32_t i = 0; i < n; ++i) {
            c.hostWorldOf[i] = worldOf[i];
            if (i > 0 && worldOf[i] < worldOf[i - 1])
                return fail(c, VXB_ERR_INVALID, "bodies of one world must be contiguous and worlds ascending");
            worlds = std::max(worlds, worldOf[i] + 1);
        }
    }
    c.worlds = worlds;
    std::vector<uint32_t> planeStart(worlds + 1, 0), planeList;
    auto boundless = [&](uint32_t i) { return bodies[i].shape == VX_SHAPE_PLANE || bodies[i].shape == VX_SHAPE_MESH; };
    for (uint32_t i = 0; i < n; ++i)
        if (boundless(i)) ++planeStart[c.hostWorldOf[i] + 1];
    for (uint32_t w = 0; w < worlds; ++w) planeStart[w + 1] += planeStart[w];
    planeList.resize(planeStart[worlds]);
    {
        std::vector<uint32_t> fill(planeStart.begin(), planeStart.end() - 1);
        for (uint32_t i = 0; i < n; ++i)
            if (boundless(i)) planeList[fill[c.hostWorldOf[i]]++] = i;
    }
    VXB_TRY(ensure(c, c.worldOfBuf, (size_t)n * 4));
    VXB_TRY(ensure(c, c.planeStartBuf, planeStart.size() * 4));
    VXB_TRY(ensure(c, c.planeListBuf, planeList.size() * 4 + 4));
    c.hostPlaneStart = planeStart;
    VXB_CUDA(c, cudaMemcpyAsync(c.worldOfBuf.ptr, c.hostWorldOf.data(), (size_t)n * 4, cudaMemcpyHostToDevice, c.stream));
    VXB_CUDA(c, cudaMemcpyAsync(c.planeStartBuf.ptr, planeStart.data(), planeStart.size() * 4, cudaMemcpyHostToDevice,
                                c.stream));
    if (!planeList.empty())
        VXB_CUDA(c, cudaMemcpyAsync(c.planeListBuf.ptr, planeList.data(), planeList.size() * 4, cudaMemcpyHostToDevice,
                                    c.stream));
    VXB_CUDA(c, cudaStreamSynchronize(c.stream));  // host vectors above are freed on return
    // Reserve step buffers up front so steady stepping never reallocates
    // (cudaFree synchronises the device).
    if (c.pairCap < 16u * n) c.pairCap = 16u * n + 4096u;
    if (c.contactCap < 8u * n) c.contactCap = 8u * n + 4096u;
    if (c.recCap < 8u * n) c.recCap = 8u * n + 4096u;
    const size_t mcap = c.contactCap;
    VXB_TRY(ensure(c, c.pairBuf, (size_t)c.pairCap * 8));
    VXB_TRY(ensure(c, c.contactTmpBuf, mcap * sizeof(vx_contact)));
    VXB_TRY(ensure(c, c.contactBuf[0], mcap * sizeof(vx_contact) + 128));
    VXB_TRY(ensure(c, c.contactBuf[1], mcap * sizeof(vx_contact) + 128));
    VXB_TRY(ensure(c, c.coopBuf, sizeof(CoopState)));
    for (DevBuf* b : {&c.recValBuf, &c.recCountBuf, &c.recOffsetBuf, &c.islandValBuf, &c.colorBuf, &c.flagBuf,
                      &c.scanBuf, &c.islandStartBuf, &c.segStartBuf, &c.islandSegBuf, &c.fpIslandBuf})
        VXB_TRY(ensure(c, *b, mcap * 4 + 64));
    for (DevBuf* b : {&c.recKeyBuf, &c.recInfoBuf, &c.pairKeyBuf, &c.prevKeyBuf, &c.islandKeyBuf, &c.colorKeyBuf,
                      &c.sortKeysAlt})
        VXB_TRY(ensure(c, *b, mcap * 8 + 64));
    VXB_TRY(ensure(c, c.sortValsAlt, std::max<size_t>(mcap, (size_t)c.pairCap) * 4 + 64));
    c.prevCount = 0;
    c.stepContacts = 0;
    VXB_TRY(sleepLoad(c, bodies, n));
    return VXB_OK;
}

int readBodies(Context& c, vx_body* out, uint32_t n) {
    if (n != c.n) return fail(c, VXB_ERR_INVALID, "body count mismatch");
    LAUNCH(c, unpackBodiesKernel, blocksFor(n, 256), 256, P<vx_body>(c.aosBuf), n, c.B);
    VXB_TRY(sleepExport(c, P<vx_body>(c.aosBuf)));
    VXB_CUDA(c, cudaMemcpyAsync(out, c.aosBuf.ptr, (size_t)n * sizeof(vx_body), cudaMemcpyDeviceToHost, c.stream));
    VXB_CUDA(c, cudaStreamSynchronize(c.stream));
    return VXB_OK;
}

int readPoses(Context& c, float* out, uint32_t n) {
    if (n != c.n) return fail(c, VXB_ERR_INVALID, "body count mismatch");
    VXB_TRY(ensure(c, c.scanBuf, (size_t)n * 28 + 16));
    LAUNCH(c, posesKernel, blocksFor(n, 256), 256, P<float>(c.scanBuf), n, c.B);
    VXB_CUDA(c, cudaMemcpyAsync(out, c.scanBuf.ptr, (size_t)n * 28, cudaMemcpyDeviceToHost, c.stream));
    VXB_CUDA(c, cudaStreamSynchronize(c.stream));
    return VXB_OK;
}

int writeForces(Context& c, const float* in, uint32_t n) {
    if (n != c.n) return fail(c, VXB_ERR_INVALID, "body count mismatch");
    VXB_TRY(ensure(c, c.scanBuf, (size_t)n * 28 + 16));
    VXB_CUDA(c, cudaMemcpyAsync(c.scanBuf.ptr, in, (size_t)n * 24, cudaMemcpyHostToDevice, c.stream));
    LAUNCH(c, forcesKernel, blocksFor(n, 256), 256, P<float>(c.scanBuf), n, c.B);
    return VXB_OK;
}

// ---- broad phase ----------------------------------------------------------

static int broadPhase(Context& c, float dt, uint32_t* pairCount) {
    const uint32_t n = c.n;
    VXB_TRY(ensure(c, c.aabbBuf, (size_t)n * 32));
    float4* lo = P<float4>(c.aabbBuf);
    float4* hi = lo + n;
    stageBegin(c, kStageBroadphase);
    LAUNCH(c, aabbKernel, std::min<uint32_t>(blocksFor(n, 256), (uint32_t)c.smCount * 8), 256, c.B, n, dt,
           (const vx_mesh*)P<vx_mesh>(c.meshBuf), lo, hi, c.dCounters);
    const int worldBits = bitsFor(c.worlds > 1 ? c.worlds - 1 : 0);
    const int keyBitsTotal = 3 * kCellBits + worldBits + 1;
    const uint64_t planeKey = 1ull << (3 * kCellBits + worldBits);
    VXB_TRY(ensure(c, c.cellKeyBuf, (size_t)n * 8));
    VXB_TRY(ensure(c, c.cellValBuf, (size_t)n * 4));
    uint64_t* keys = P<uint64_t>(c.cellKeyBuf);
    uint32_t* vals = P<uint32_t>(c.cellValBuf);
    LAUNCH(c, keyKernel, blocksFor(n, 256), 256, c.B, n, c.worlds > 1 ? P<uint32_t>(c.worldOfBuf) : nullptr, lo, hi,
           c.dCounters, keys, vals, planeKey);
    stageEnd(c, kStageBroadphase);
    stageBegin(c, kStageCellSort);
    VXB_TRY(sortPairs(c, keys, vals, n, keyBitsTotal));
    stageEnd(c, kStageCellSort);
    stageBegin(c, kStageBroadphase);
    uint32_t hashCap = 1024;
    while (hashCap < 2 * n) hashCap <<= 1;
    c.hashCap = hashCap;
    VXB_TRY(ensure(c, c.hashKeyBuf, (size_t)hashCap * 8));
    VXB_TRY(ensure(c, c.hashValBuf, (size_t)hashCap * 4));
    VXB_CUDA(c, cudaMemsetAsync(c.hashKeyBuf.ptr, 0xff, (size_t)hashCap * 8, c.stream));
    LAUNCH(c, cellTableKernel, blocksFor(n, 256), 256, keys, n, planeKey, P<uint64_t>(c.hashKeyBuf),
           P<uint32_t>(c.hashValBuf), hashCap - 1);
    if (c.pairCap == 0) c.pairCap = std::max<uint32_t>(n * 8u, 4096u);
    // plane pairs: at most bodies x planes of a world
    uint32_t planeCap = 16;
    {
        uint32_t maxPlanes = 0;
        for (uint32_t w = 0; w < c.worlds; ++w) maxPlanes = std::max(maxPlanes, c.hostPlaneStart[w + 1] - c.hostPlaneStart[w]);
        planeCap = std::max<uint32_t>(16u, n * std::max<uint32_t>(maxPlanes, 1u));
    }
    for (int attempt = 0; attempt < 3; ++attempt) {
        VXB_TRY(ensure(c, c.pairBuf, ((size_t)c.pairCap + planeCap) * 8));
        VXB_CUDA(c, cudaMemsetAsync(&c.dCounters->pairs, 0, 4, c.stream));
        VXB_CUDA(c, cudaMemsetAsync(&c.dCounters->planePairs, 0, 4, c.stream));
        VXB_CUDA(c, cudaMemsetAsync(&c.dCounters->overflow, 0, 4, c.stream));
        LAUNCH(c, pairKernel, blocksFor(n, 128), 128, c.B, n, keys, vals, lo, hi, P<uint64_t>(c.hashKeyBuf),
               P<uint32_t>(c.hashValBuf), hashCap - 1, planeKey,
               c.worlds > 1 ? P<uint32_t>(c.worldOfBuf) : nullptr, P<uint32_t>(c.planeStartBuf),
               P<uint32_t>(c.planeListBuf), P<uint64_t>(c.pairBuf), c.pairCap, P<uint64_t>(c.pairBuf) + c.pairCap,
               planeCap, c.dCounters);
        stageEnd(c, kStageBroadphase);
        VXB_TRY(readCounters(c));
        if (c.hostCounters.pairs <= c.pairCap && c.hostCounters.planePairs <= planeCap) break;
        c.pairCap = c.hostCounters.pairs + c.hostCounters.pairs / 4 + 1024;
    }
    // Convex pairs live at [0, pairs), plane pairs at [pairCap, pairCap + planePairs).
    c.convexPairs = c.hostCounters.pairs;
    c.planePairs = c.hostCounters.planePairs;
    *pairCount = c.convexPairs + c.planePairs;
    return VXB_OK;
}

// ---- narrow phase ---------------------------------------------------------

// Runs the narrow phase on `npairs` device pairs and leaves the contacts
// sorted in contactBuf[c.cur] (mode 0) or grouped in pair order (mode 1).
// World path: `pairs` holds convexSplit convex-convex pairs and `planePairs`
// holds npairs - convexSplit plane pairs. Stage path (convexSplit = ~0u):
// `pairs` holds npairs unclassified pairs.
static int narrowPhase(Context& c, const uint64_t* pairs, uint32_t npairs, float dt, int mode, uint32_t* contactCount,
                       uint32_t* recordCount, uint32_t convexSplit = ~0u, const uint64_t* planePairs = nullptr) {
    const int bodyBits = std::max(1, bitsFor(c.n - 1));
    if (c.contactCap == 0) c.contactCap = std::max<uint32_t>(npairs * 2u, 4096u);
    if (c.recCap < npairs) c.recCap = npairs + 1024;
    for (int attempt = 0; attempt < 3; ++attempt) {
        VXB_TRY(ensure(c, c.contactTmpBuf, (size_t)c.contactCap * sizeof(vx_contact)));
        VXB_TRY(ensure(c, c.recKeyBuf, (size_t)c.recCap * 8));
        VXB_TRY(ensure(c, c.recValBuf, (size_t)c.recCap * 4));
        VXB_TRY(ensure(c, c.recInfoBuf, (size_t)c.recCap * 8));
        VXB_CUDA(c, cudaMemsetAsync(&c.dCounters->contactsTmp, 0, 8, c.stream));  // contactsTmp + records
        VXB_CUDA(c, cudaMemsetAsync(&c.dCounters->overflow, 0, 4, c.stream));
        stageBegin(c, kStageNarrowphase);
        vx_contact* tmp = P<vx_contact>(c.contactTmpBuf);
        uint64_t* recKeys = P<uint64_t>(c.recKeyBuf);
        uint32_t* recVals = P<uint32_t>(c.recValBuf);
        uint2* recInfo = P<uint2>(c.recInfoBuf);
        if (npairs && convexSplit <= npairs) {
            const uint32_t np = npairs - convexSplit;
            if (convexSplit) {
                // group the convex pairs by shape combination (records are keyed by body pair, so
                // the processing order does not change the result)
                VXB_TRY(ensure(c, c.classKeyBuf, (size_t)convexSplit * 8 + 64));
                VXB_TRY(ensure(c, c.classValBuf, (size_t)convexSplit * 4 + 64));
                if (attempt == 0) {
                    LAUNCH(c, pairClassKernel, blocksFor(convexSplit, 256), 256, c.B, pairs, convexSplit,
                           P<uint64_t>(c.classKeyBuf), P<uint32_t>(c.classValBuf));
                    VXB_TRY(sortPairs(c, P<uint64_t>(c.classKeyBuf), P<uint32_t>(c.classValBuf), convexSplit, 8));
                }
                const uint32_t* order = P<uint32_t>(c.classValBuf);
                VXB_TRY(tunedLaunch(c, kTuneCollideConvex, convexSplit, [&](LaunchShape sh) {
                    LAUNCH(c, collideKernel<kConvexPairs>, sh.grid(convexSplit, c.smCount), sh.threads, c.B, soupOf(c),
                           pairs, order, convexSplit, dt, mode, bodyBits, tmp, c.contactCap, recKeys, recVals, recInfo,
                           c.recCap, c.dCounters);
                }, CounterRestore{c}));
                if (c.complexShapes)
                    VXB_TRY(tunedLaunch(c, kTuneCollideComplex, convexSplit, [&](LaunchShape sh) {
                        LAUNCH(c, collideKernel<kComplexPairs>, sh.grid(convexSplit, c.smCount), sh.threads, c.B,
                               soupOf(c), pairs, order, convexSplit, dt, mode, bodyBits, tmp, c.contactCap, recKeys,
                               recVals, recInfo, c.recCap, c.dCounters);
                    }, CounterRestore{c}));
            }
            if (np)
                VXB_TRY(tunedLaunch(c, kTuneCollidePlane, np, [&](LaunchShape sh) {
                    LAUNCH(c, collideKernel<kPlanePairs>, sh.grid(np, c.smCount), sh.threads, c.B, soupOf(c), planePairs,
                           (const uint32_t*)nullptr, np, dt, mode, bodyBits, tmp, c.contactCap, recKeys, recVals,
                           recInfo, c.recCap, c.dCounters);
                }, CounterRestore{c}));
        } else if (npairs) {
            VXB_TRY(tunedLaunch(c, kTuneCollideAny, npairs, [&](LaunchShape sh) {
                LAUNCH(c, collideKernel<kAnyPairs>, sh.grid(npairs, c.smCount), sh.threads, c.B, soupOf(c), pairs,
                       (const uint32_t*)nullptr, npairs, dt, mode, bodyBits, tmp, c.contactCap, recKeys, recVals,
                       recInfo, c.recCap, c.dCounters);
            }, CounterRestore{c}));
        }
        stageEnd(c, kStageNarrowphase);
        VXB_TRY(readCounters(c));
        if (!(c.hostCounters.overflow & 2u)) break;
        c.contactCap = c.hostCounters.contactsTmp + c.hostCounters.contactsTmp / 4 + 1024;
        c.recCap = std::max(c.recCap, c.hostCounters.records + 1024);
    }
    const uint32_t m = c.hostCounters.contactsTmp, nrec = c.hostCounters.records;
    *contactCount = m;
    *recordCount = nrec;
    const int recBits = mode == 0 ? 2 * bodyBits : bitsFor(npairs);
    stageBegin(c, kStagePlacement);
    VXB_TRY(sortPairs(c, P<uint64_t>(c.recKeyBuf), P<uint32_t>(c.recValBuf), nrec, recBits));
    VXB_TRY(ensure(c, c.recCountBuf, (size_t)nrec * 4 + 16));
    VXB_TRY(ensure(c, c.recOffsetBuf, (size_t)nrec * 4 + 16));
    VXB_TRY(ensure(c, c.pairKeyBuf, (size_t)nrec * 8 + 16));
    VXB_TRY(ensure(c, c.contactBuf[c.cur], (size_t)m * sizeof(vx_contact) + 128));
    VXB_TRY(ensure(c, c.scanBuf, (size_t)nrec * 4 + 16));
    if (nrec) {
        LAUNCH(c, gatherCountsKernel, blocksFor(nrec, 256), 256, P<uint32_t>(c.recValBuf), P<uint2>(c.recInfoBuf), nrec,
               P<uint32_t>(c.recCountBuf));
        VXB_TRY(exclusiveScan(c, P<uint32_t>(c.recCountBuf), P<uint32_t>(c.scanBuf), nrec, nullptr));
        LAUNCH(c, placeKernel, blocksFor(nrec, 128), 128, P<uint32_t>(c.recValBuf), P<uint2>(c.recInfoBuf),
               P<uint32_t>(c.scanBuf), nrec, P<vx_contact>(c.contactTmpBuf), P<vx_contact>(c.contactBuf[c.cur]),
               (uint64_t*)nullptr, P<uint64_t>(c.pairKeyBuf), P<uint32_t>(c.recOffsetBuf));
    }
    stageEnd(c, kStagePlacement);
    return VXB_OK;
}

// ---- islands + colouring --------------------------------------------------

// Groups the m contacts of `cs` into islands, colours them and builds the
// solve order (island, colour, contact order) plus per-island body lists.
// Cooperative launch of `kernel` with as many blocks as fit on the device at
// once (at most maxPerSm per SM when maxPerSm > 0). VXB_ERR_UNSUPPORTED
// (nothing recorded) when the device cannot run it: callers then take their
// serial path.
template <class Kernel, class... Args>
static int launchCooperativeSmem(Context& c, int maxPerSm, size_t smem, Kernel kernel, int threads, Args... args) {
    int perSm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kernel, threads, smem);
    if (e != cudaSuccess) return cudaStatus(c, e, "cooperative occupancy");
    if (perSm <= 0 || !c.cooperative) return VXB_ERR_UNSUPPORTED;
    if (maxPerSm > 0 && perSm > maxPerSm) perSm = maxPerSm;
    void* params[] = {&args...};
    e = cudaLaunchCooperativeKernel((const void*)kernel, dim3(perSm * c.smCount), dim3(threads), params, smem,
                                    c.stream);
    ++c.launches;
    return cudaStatus(c, e, "cudaLaunchCooperativeKernel");
}

template <class Kernel, class... Args>
static int launchCooperativeCapped(Context& c, int maxPerSm, Kernel kernel, int threads, Args... args) {
    return launchCooperativeSmem(c, maxPerSm, 0, kernel, threads, args...);
}

template <class Kernel, class... Args>
static int launchCooperative(Context& c, Kernel kernel, int threads, Args... args) {
    return launchCooperativeSmem(c, 0, 0, kernel, threads, args...);
}

// Colours of the islands above kSerialColorLimit contacts (colorOf, colour
// keys, maxColors). VXB_ERR_UNSUPPORTED / VXB_ERR_TIMEOUT: the caller colours
// every island serially instead.
static int parallelColor(Context& c, const vx_contact* cs, const uint32_t* order, const uint32_t* islandIdx,
                         const uint32_t* islandStart, uint32_t m, uint64_t* colorKeys) {
    const uint32_t n = c.n;
    VXB_TRY(ensure(c, c.fpKeyBuf, (size_t)m * 16 + 64));
    VXB_TRY(ensure(c, c.fpValBuf, (size_t)m * 8 + 64));
    VXB_TRY(ensure(c, c.fpSlotBuf, (size_t)m * 8 + 64));
    VXB_TRY(ensure(c, c.fpColorBuf, (size_t)m * 4 + 64));
    VXB_TRY(ensure(c, c.fpRunStartBuf, (size_t)n * 4 + 64));
    VXB_TRY(ensure(c, c.coopBuf, sizeof(CoopState)));
    uint64_t* keys = P<uint64_t>(c.fpKeyBuf);
    uint32_t* vals = P<uint32_t>(c.fpValBuf);
    uint32_t* slot = P<uint32_t>(c.fpSlotBuf);
    uint32_t* color = P<uint32_t>(c.fpColorBuf);
    uint32_t* runStart = P<uint32_t>(c.fpRunStartBuf);
    CoopState* st = P<CoopState>(c.coopBuf);
    LAUNCH(c, colorEntryKernel, blocksFor(m, 256), 256, cs, order, m, islandIdx, islandStart, c.B, n,
           keys, vals, slot);
    VXB_TRY(sortPairs(c, keys, vals, 2 * m, bitsFor(n)));
    LAUNCH(c, colorSlotKernel, blocksFor(2 * m, 256), 256, keys, vals, 2 * m, n, slot, runStart);
    VXB_CUDA(c, cudaMemsetAsync(color, 0, (size_t)m * 4, c.stream));
    VXB_TRY(resetCoop(c, st));
    const int rc = launchCooperative(c, colorFixedPointKernel, 256, (const uint64_t*)keys, (const uint32_t*)vals,
                                     (const uint32_t*)slot, (const uint32_t*)runStart, islandIdx,
                                     islandStart, m, color, st, 4096u);
    if (rc != VXB_OK) return rc;
    CoopState host;
    VXB_CUDA(c, cudaMemcpyAsync(&host, st, sizeof(host), cudaMemcpyDeviceToHost, c.stream));
    ++c.hostSyncs;
    VXB_CUDA(c, cudaStreamSynchronize(c.stream));
    c.stats.colorRounds = host.rounds;
    if (host.timeout || (host.spill & 2u)) return VXB_ERR_TIMEOUT;
    if (host.spill) return VXB_ERR_UNSUPPORTED;
    LAUNCH(c, colorFinishKernel, blocksFor(m, 256), 256, order, m, islandIdx, islandStart,
           (const uint32_t*)color, P<uint32_t>(c.colorBuf), colorKeys, c.dCounters);
    return VXB_OK;
}

static int buildIslands(Context& c, const vx_contact* cs, uint32_t m, IslandPlan& plan, uint32_t* colorOut) {
    const uint32_t n = c.n;
    plan.contacts = m;
    c.planContacts = m;
    c.giantLinked = false;
    c.clusterBuilt = false;
    c.tinyPacked = false;
    VXB_TRY(ensure(c, c.parentBuf, (size_t)n * 4));
    VXB_TRY(ensure(c, c.islandOfBodyBuf, (size_t)n * 4));
    VXB_TRY(ensure(c, c.maskBuf, (size_t)n * 8));
    VXB_TRY(ensure(c, c.nextColorBuf, (size_t)n * 4));
    VXB_TRY(ensure(c, c.bodyKeyBuf, (size_t)n * 8));
    VXB_TRY(ensure(c, c.bodyValBuf, (size_t)n * 4));
    VXB_TRY(ensure(c, c.islandKeyBuf, (size_t)m * 8 + 16));
    VXB_TRY(ensure(c, c.islandValBuf, (size_t)m * 4 + 16));
    VXB_TRY(ensure(c, c.colorBuf, (size_t)m * 4 + 16));
    VXB_TRY(ensure(c, c.flagBuf, (size_t)m * 4 + 16));
    VXB_TRY(ensure(c, c.scanBuf, (size_t)m * 4 + 16));
    VXB_TRY(ensure(c, c.islandStartBuf, (size_t)m * 4 + 16));
    VXB_TRY(ensure(c, c.segStartBuf, (size_t)m * 4 + 16));
    VXB_TRY(ensure(c, c.islandSegBuf, (size_t)m * 4 + 16));
    uint32_t* parent = P<uint32_t>(c.parentBuf);
    LAUNCH(c, iotaKernel, blocksFor(n, 256), 256, parent, n);
    if (m == 0) {
        plan = IslandPlan{};
        plan.contacts = 0;
        VXB_CUDA(c, cudaMemsetAsync(c.islandOfBodyBuf.ptr, 0xff, (size_t)n * 4, c.stream));
    } else {
        LAUNCH(c, unionKernel, blocksFor(m, 256), 256, cs, m, c.B, parent, c.dCounters);
        LAUNCH(c, compressKernel, blocksFor(n, 256), 256, parent, n);
        uint64_t* ikeys = P<uint64_t>(c.islandKeyBuf);
        uint32_t* ivals = P<uint32_t>(c.islandValBuf);
        LAUNCH(c, islandKeyKernel, blocksFor(m, 256), 256, cs, m, c.B, parent, n, ikeys, ivals);
        VXB_TRY(sortPairs(c, ikeys, ivals, m, bitsFor(n)));
        uint32_t* flags = P<uint32_t>(c.flagBuf);
        uint32_t* index = P<uint32_t>(c.scanBuf);
        uint32_t* islandStart = P<uint32_t>(c.islandStartBuf);
        LAUNCH(c, runFlagKernel, blocksFor(m, 256), 256, ikeys, m, flags);
        VXB_TRY(exclusiveScan(c, flags, index, m, &c.dCounters->islands));
        LAUNCH(c, runStartKernel, blocksFor(m, 256), 256, flags, index, m, islandStart);
        VXB_TRY(ensure(c, c.fpIslandBuf, (size_t)m * 4 + 64));
        uint32_t* islandOf = P<uint32_t>(c.fpIslandBuf);
        LAUNCH(c, runOfKernel, blocksFor(m, 256), 256, flags, index, m, islandOf);
        LAUNCH(c, lastKeyKernel, 1, 32, ikeys, m, c.dCounters);
        LAUNCH(c, islandMaxKernel, std::min<uint32_t>(blocksFor(m, 256), (uint32_t)c.smCount * 4), 256, islandStart,
               c.dCounters);
        VXB_TRY(readCounters(c));
        plan.islands = c.hostCounters.islands;
        // is the last island the null island (key n)?
        plan.realIslands = c.hostCounters.lastIslandKey == n ? plan.islands - 1 : plan.islands;
        // colour each island; colour keys (island << 16 | colour) in island order
        VXB_TRY(ensure(c, c.colorKeyBuf, (size_t)m * 8 + 16));
        uint64_t* ckeys = P<uint64_t>(c.colorKeyBuf);
        bool serialAll = false;
        if (c.hostCounters.maxIslandSize > kSerialColorLimit) {
            const int status = parallelColor(c, cs, ivals, islandOf, islandStart, m, ckeys);
            if (status == VXB_ERR_TIMEOUT || status == VXB_ERR_UNSUPPORTED) serialAll = true;  // exact serial path
            else if (status != VXB_OK) return status;
        }
        LAUNCH(c, colorKernel, blocksFor(plan.islands, 64), 64, cs, ivals, islandStart, plan.islands, c.B,
               P<unsigned long long>(c.maskBuf), P<uint32_t>(c.nextColorBuf), P<uint32_t>(c.colorBuf), ckeys,
               c.dCounters, serialAll ? 0xffffffffu : kSerialColorLimit);
        if (colorOut)
            VXB_CUDA(c, cudaMemcpyAsync(colorOut, c.colorBuf.ptr, (size_t)m * 4, cudaMemcpyDeviceToHost, c.stream));
        // solve order: stable sort by (island, colour)
        VXB_TRY(sortPairs(c, ckeys, ivals, m, 16 + bitsFor(plan.islands)));
        LAUNCH(c, runFlagKernel, blocksFor(m, 256), 256, ckeys, m, flags);
        VXB_TRY(exclusiveScan(c, flags, index, m, &c.dCounters->segments));
        LAUNCH(c, runStartKernel, blocksFor(m, 256), 256, flags, index, m, P<uint32_t>(c.segStartBuf));
        // island bodies
        VXB_CUDA(c, cudaMemsetAsync(c.islandOfBodyBuf.ptr, 0xff, (size_t)n * 4, c.stream));
        LAUNCH(c, islandBodyKernel, blocksFor(m, 256), 256, cs, ivals, (const uint32_t*)islandOf, m, plan.realIslands,
               c.B, P<uint32_t>(c.islandOfBodyBuf));
    }
    const uint32_t freeKey = plan.realIslands;
    LAUNCH(c, bodyKeyKernel, blocksFor(n, 256), 256, P<uint32_t>(c.islandOfBodyBuf), n, freeKey,
           P<uint64_t>(c.bodyKeyBuf), P<uint32_t>(c.bodyValBuf));
    VXB_TRY(sortPairs(c, P<uint64_t>(c.bodyKeyBuf), P<uint32_t>(c.bodyValBuf), n, bitsFor(freeKey)));
    VXB_TRY(ensure(c, c.islandBodyStartBuf, ((size_t)plan.realIslands + 2) * 4 + 16));
    LAUNCH(c, bodyStartKernel, blocksFor(n, 256), 256, P<uint64_t>(c.bodyKeyBuf), n, P<uint32_t>(c.islandBodyStartBuf),
           plan.realIslands + 2);
    LAUNCH(c, freeRangeKernel, 1, 32, P<uint32_t>(c.islandBodyStartBuf), plan.realIslands + 2, c.dCounters);
    VXB_CUDA(c, cudaMemsetAsync(&c.dCounters->giantCount, 0, 4, c.stream));
    if (m)
        LAUNCH(c, giantCountKernel, std::min<uint32_t>(blocksFor(plan.islands, 256), (uint32_t)c.smCount * 4), 256,
               (const uint32_t*)P<uint32_t>(c.islandStartBuf), (const uint32_t*)P<uint32_t>(c.islandBodyStartBuf),
               plan.islands, plan.realIslands, c.dCounters);
    VXB_TRY(readCounters(c));  // one read for the segment count, the free-body range and the giants
    plan.segments = m ? c.hostCounters.segments : 0;
    plan.freeFrom = c.hostCounters.freeFrom;
    plan.freeTo = c.hostCounters.freeTo;
    c.planGiants = m ? c.hostCounters.giantCount : 0u;
    return VXB_OK;
}

__global__ void islandSegKernel(const uint32_t* islandStart, const uint32_t* segIndex, uint32_t islands,
                                uint32_t segments, uint32_t* islandSeg) {
    for (uint32_t isl = blockIdx.x * blockDim.x + threadIdx.x; isl <= islands; isl += gridDim.x * blockDim.x)
        islandSeg[isl] = isl == islands ? segments : segIndex[islandStart[isl]];
}

static SolveArgs solveArgs(Context& c, vx_contact* cs, const IslandPlan& plan) {
    SolveArgs A;
    std::memset(&A, 0, sizeof(A));
    A.B = c.B;
    A.contacts = cs;
    A.order = P<uint32_t>(c.islandValBuf);
    A.islandStart = P<uint32_t>(c.islandStartBuf);
    A.segStart = P<uint32_t>(c.segStartBuf);
    A.islandSeg = P<uint32_t>(c.islandSegBuf);
    A.bodyOrder = P<uint32_t>(c.bodyValBuf);
    A.bodyStart = P<uint32_t>(c.islandBodyStartBuf);
    A.islands = plan.islands;
    A.realIslands = plan.realIslands;
    A.tinyLimit = kTinyLimit;
    A.fault = &c.dCounters->planFault;
    A.prep = P<RowPrep>(c.prepBuf);
    A.frames = P<float4>(c.frameBuf);
    return A;
}

static int prepareSegments(Context& c, const IslandPlan& plan) {
    if (plan.islands == 0) return VXB_OK;
    LAUNCH(c, islandSegKernel, blocksFor(plan.islands + 1, 256), 256, P<uint32_t>(c.islandStartBuf),
           P<uint32_t>(c.scanBuf), plan.islands, plan.segments, P<uint32_t>(c.islandSegBuf));
    return VXB_OK;
}

static int launchSolve(Context& c, const SolveArgs& A) {
    if (A.islands == 0) return VXB_OK;
    // tiny islands: pack them into warps once per island plan
    const uint32_t islands = A.islands, chunksCap = (islands + kPackChunk - 1) / kPackChunk + 1;
    VXB_TRY(ensure(c, c.tinyBuf, ((size_t)islands * 4 + (size_t)chunksCap * 2 + 64) * 4));
    uint32_t* tFlags = P<uint32_t>(c.tinyBuf);
    uint32_t* tRanks = tFlags + islands + 16;
    uint32_t* tList = tRanks + islands + 16;
    uint32_t* tFirst = tList + islands + 16;
    uint32_t* tChunkCount = tFirst + islands + 16;
    uint32_t* tChunkBase = tChunkCount + chunksCap;
    // (counts stay on the device: sizes below are upper bounds, kernels read the counts)
    const uint32_t chunks = (islands + kPackChunk - 1) / kPackChunk;
    if (!c.tinyPacked) {
        LAUNCH(c, tinyFlagKernel, blocksFor(islands, 256), 256, A, tFlags);
        VXB_TRY(exclusiveScan(c, tFlags, tRanks, islands, &c.dCounters->tinyIslands));
        LAUNCH(c, compactKernel, blocksFor(islands, 256), 256, tFlags, tRanks, islands, tList);
        VXB_TRY(ensure(c, c.tinyKeyBuf, (size_t)islands * 8 + 64));
        LAUNCH(c, tinyKeyKernel, blocksFor(islands, 256), 256, A, (const uint32_t*)tList,
               (const uint32_t*)&c.dCounters->tinyIslands, islands, P<uint64_t>(c.tinyKeyBuf), tList);
        VXB_TRY(sortPairs(c, P<uint64_t>(c.tinyKeyBuf), tList, islands, 8));
        LAUNCH(c, tinyPackKernel, blocksFor(chunks, 128), 128, A, (const uint32_t*)tList,
               (const uint32_t*)&c.dCounters->tinyIslands, chunks, 0, tChunkCount, (const uint32_t*)tChunkBase, tFirst);
        VXB_TRY(exclusiveScan(c, tChunkCount, tChunkBase, chunks, &c.dCounters->tinyPacks));
        LAUNCH(c, tinyPackKernel, blocksFor(chunks, 128), 128, A, (const uint32_t*)tList,
               (const uint32_t*)&c.dCounters->tinyIslands, chunks, 1, tChunkCount, (const uint32_t*)tChunkBase, tFirst);
        c.tinyPacked = true;
    }
    VXB_TRY(ensure(c, c.localIdxBuf, (size_t)c.n * 4 + 16));
    {
        static bool packConfigured = false;
        if (!packConfigured) {
            cudaFuncSetAttribute(solveTinyPackKernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(kPackWarpSmem * kPackWarps));
            packConfigured = true;
        }
        const uint32_t grid = std::min<uint32_t>((islands + kPackWarps - 1) / kPackWarps, (uint32_t)c.smCount * 8);
        solveTinyPackKernel<<<grid, 32 * kPackWarps, kPackWarpSmem * kPackWarps, c.stream>>>(
            A, (const uint32_t*)tList, (const uint32_t*)tFirst, (const Counters*)c.dCounters, P<uint32_t>(c.localIdxBuf));
        ++c.launches;
    }
    auto* large = solveBlockKernel<kBlockThreads, kBlockBodies, kBlockRows, false>;
    auto* small = solveBlockKernel<kSmallThreads, kSmallBodies, kSmallRows, true>;
    static int smallPerSm = 0;
    if (!smallPerSm) {
        cudaFuncSetAttribute(large, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBlockSmem);
        cudaFuncSetAttribute(small, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmallSmem);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&smallPerSm, small, kSmallThreads, kSmallSmem) != cudaSuccess ||
            smallPerSm <= 0)
            smallPerSm = 8;
    }
    small<<<std::min<uint32_t>(A.islands, (uint32_t)(c.smCount * smallPerSm)), kSmallThreads, kSmallSmem, c.stream>>>(
        A, P<uint32_t>(c.localIdxBuf));
    ++c.launches;
    large<<<std::min<uint32_t>(A.islands, (uint32_t)c.smCount * 2), kBlockThreads, kBlockSmem, c.stream>>>(
        A, P<uint32_t>(c.localIdxBuf));
    ++c.launches;
    // giant islands: list them, then one cooperative launch over all of them
    VXB_TRY(ensure(c, c.giantBuf, ((size_t)A.islands + 1) * 4 + 64));
    VXB_TRY(ensure(c, c.coopBuf, sizeof(CoopState)));
    CoopState* st = P<CoopState>(c.coopBuf);
    uint32_t* list = P<uint32_t>(c.giantBuf);
    VXB_TRY(resetCoop(c, st));
    const uint32_t giants = c.planGiants;  // counted with the island plan
    if (!giants) return VXB_OK;
    LAUNCH(c, giantListKernel, std::min<uint32_t>(blocksFor(A.islands, 256), (uint32_t)c.smCount * 4), 256, A, list,
           &st->rounds);
    c.stats.giantIslands = std::max(c.stats.giantIslands, giants);
    // dataflow links of the giant islands' rows (once per island plan)
    const uint32_t m = c.planContacts;
    VXB_TRY(ensure(c, c.fpKeyBuf, (size_t)m * 16 + 64));
    VXB_TRY(ensure(c, c.fpValBuf, (size_t)m * 8 + 64));
    VXB_TRY(ensure(c, c.fpSlotBuf, (size_t)m * 8 + 64));
    VXB_TRY(ensure(c, c.fpColorBuf, (size_t)m * 4 + 64));
    VXB_TRY(ensure(c, c.fpRunStartBuf, (size_t)c.n * 4 + 64));
    VXB_TRY(ensure(c, c.rowBodyBuf, (size_t)m * 8 + 64));
    uint32_t* pred = P<uint32_t>(c.fpSlotBuf);
    uint32_t* done = P<uint32_t>(c.fpColorBuf);
    if (!c.giantLinked) {
        uint64_t* keys = P<uint64_t>(c.fpKeyBuf);
        uint32_t* vals = P<uint32_t>(c.fpValBuf);
        LAUNCH(c, giantEntryKernel, blocksFor(m, 256), 256, A, P<uint32_t>(c.fpIslandBuf), m, c.n, keys, vals,
               P<uint2>(c.rowBodyBuf));
        VXB_TRY(sortPairs(c, keys, vals, 2 * m, bitsFor(c.n)));
        LAUNCH(c, giantLastKernel, blocksFor(2 * m, 256), 256, keys, 2 * m, c.n, P<uint32_t>(c.fpRunStartBuf));
        LAUNCH(c, giantPredKernel, blocksFor(2 * m, 256), 256, keys, vals, 2 * m, c.n,
               P<uint32_t>(c.fpRunStartBuf), pred);
        c.giantLinked = true;
    }
    SolveArgs G = A;
    G.rowBodies = P<uint2>(c.rowBodyBuf);
    if (c.cooperative) {
        // the giant islands in spatial clusters, one per block of the cooperative grid
        int perSm = 0;
        VXB_CUDA(c, cudaFuncSetAttribute(solveClusterKernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)kClusterSmemBytes));
        VXB_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, solveClusterKernel, kClusterThreads,
                                                                  kClusterSmemBytes));
        const uint32_t clusters = (uint32_t)(perSm * c.smCount);
        const uint32_t n = c.n;
        VXB_TRY(ensure(c, c.clusterInfoBuf, ((size_t)n * 3 + (size_t)m * 3 + 64) * 4));
        uint32_t* bodyFlags = P<uint32_t>(c.clusterInfoBuf);
        uint32_t* bodyRank = bodyFlags + n + 16;
        uint32_t* bodyPos = bodyRank + n + 16;
        uint32_t* rowFlags = bodyPos + n + 16;
        uint32_t* rowRank = rowFlags + m + 16;
        uint32_t* rowList = rowRank + m + 16;
        if (clusters > 0 && !c.clusterBuilt) {
            VXB_CUDA(c, cudaMemsetAsync(&c.dCounters->clusterColours, 0, 4, c.stream));
            LAUNCH(c, giantMemberKernel, blocksFor(std::max(n, m), 256), 256, G, P<uint64_t>(c.bodyKeyBuf), n,
                   (const uint32_t*)P<uint32_t>(c.fpIslandBuf), m, bodyFlags, rowFlags, c.dCounters);
            VXB_TRY(exclusiveScan(c, bodyFlags, bodyRank, n, &c.dCounters->clusterBodies));
            VXB_TRY(exclusiveScan(c, rowFlags, rowRank, m, &c.dCounters->clusterRows));
            LAUNCH(c, compactKernel, blocksFor(n, 256), 256, bodyFlags, bodyRank, n, bodyPos);
            LAUNCH(c, compactKernel, blocksFor(m, 256), 256, rowFlags, rowRank, m, rowList);
            VXB_TRY(readCounters(c));
            c.clusterNB = c.hostCounters.clusterBodies;
            c.clusterR = c.hostCounters.clusterRows;
            c.clusterG = c.hostCounters.clusterColours;
            const uint32_t nb = c.clusterNB, R = c.clusterR, Gc = c.clusterG, cells = clusters * Gc;
            if (nb > 0 && R > 0 && Gc > 0) {
                VXB_TRY(ensure(c, c.clusterKeyBuf, (size_t)nb * 8 + 64));
                VXB_TRY(ensure(c, c.clusterValBuf, (size_t)nb * 4 + 64));
                VXB_TRY(ensure(c, c.clusterOfBuf, (size_t)n * 4 + 64));
                VXB_TRY(ensure(c, c.clusterCountBuf, (size_t)cells * 8 + 64));
                VXB_TRY(ensure(c, c.clusterStartBuf, ((size_t)cells + 1) * 4 + 64));
                VXB_TRY(ensure(c, c.clusterRowsBuf, (size_t)R * 4 + 64));
                uint32_t* counts = P<uint32_t>(c.clusterCountBuf);
                uint32_t* fill = counts + cells;
                uint32_t* start = P<uint32_t>(c.clusterStartBuf);
                LAUNCH(c, clusterBodyKeyKernel, blocksFor(nb, 256), 256, G, (const uint32_t*)bodyPos, nb,
                       (const Counters*)c.dCounters, P<uint64_t>(c.clusterKeyBuf), P<uint32_t>(c.clusterValBuf));
                VXB_TRY(sortPairs(c, P<uint64_t>(c.clusterKeyBuf), P<uint32_t>(c.clusterValBuf), nb, 30));
                LAUNCH(c, clusterOfBodyKernel, blocksFor(nb, 256), 256, (const uint32_t*)P<uint32_t>(c.clusterValBuf),
                       nb, clusters, P<uint32_t>(c.clusterOfBuf));
                VXB_CUDA(c, cudaMemsetAsync(counts, 0, (size_t)cells * 8, c.stream));
                LAUNCH(c, clusterCountKernel, blocksFor(R, 256), 256, G, (const uint32_t*)rowList, R,
                       (const uint32_t*)P<uint32_t>(c.fpIslandBuf), (const uint32_t*)P<uint32_t>(c.clusterOfBuf), Gc,
                       counts);
                VXB_TRY(exclusiveScan(c, counts, start, cells, start + cells));
                LAUNCH(c, clusterScatterKernel, blocksFor(R, 256), 256, G, (const uint32_t*)rowList, R,
                       (const uint32_t*)P<uint32_t>(c.fpIslandBuf), (const uint32_t*)P<uint32_t>(c.clusterOfBuf), Gc,
                       (const uint32_t*)start, fill, P<uint32_t>(c.clusterRowsBuf));
                VXB_TRY(ensure(c, c.clusterLinkBuf, (size_t)m * 12 + 64));
                uint32_t* remote = P<uint32_t>(c.clusterLinkBuf) + 2 * (size_t)m;
                VXB_CUDA(c, cudaMemsetAsync(remote, 0, (size_t)m * 4, c.stream));
                LAUNCH(c, clusterLinkKernel, blocksFor(R, 256), 256, G, (const uint32_t*)rowList, R,
                       (const uint32_t*)P<uint32_t>(c.fpIslandBuf), (const uint32_t*)P<uint32_t>(c.clusterOfBuf),
                       (const uint32_t*)pred, P<uint32_t>(c.clusterLinkBuf), remote);
                c.clusterBuilt = true;
            }
        }
        if (clusters > 0 && c.clusterBuilt) {
            VXB_TRY(resetCoop(c, st));
            const int rcc = launchCooperativeSmem(c, 0, kClusterSmemBytes, solveClusterKernel, kClusterThreads, G,
                                                  c.clusterG,
                                              (const uint32_t*)P<uint32_t>(c.clusterStartBuf),
                                              (const uint32_t*)P<uint32_t>(c.clusterRowsBuf), (const uint32_t*)rowList,
                                              c.clusterR, (const uint32_t*)P<uint32_t>(c.clusterValBuf), c.clusterNB,
                                              (const uint32_t*)P<uint32_t>(c.clusterLinkBuf),
                                              (const uint32_t*)(P<uint32_t>(c.clusterLinkBuf) + 2 * (size_t)m), done,
                                              st);
            if (rcc != VXB_ERR_UNSUPPORTED) {
                VXB_TRY(rcc);
                // a timed-out wait reaches the host with the step's final counter read
                LAUNCH(c, coopTimeoutKernel, 1, 32, (const CoopState*)st, c.dCounters);
                return VXB_OK;
            }
        }
    }
    // no cooperative grid (or no solvable giant rows): one block per giant island
    LAUNCH(c, solveGiantBlockKernel, giants, kBlockThreads, A, (const uint32_t*)list);
    return VXB_OK;
}

// Substep loop over islands + contact-free bodies (advanceSubsteps).
static int solveBuffers(Context& c, uint32_t m) {
    VXB_TRY(ensure(c, c.prepBuf, (size_t)m * sizeof(RowPrep) + 256));
    VXB_TRY(ensure(c, c.frameBuf, (size_t)c.n * 16 + 256));
    return VXB_OK;
}

static int runSubsteps(Context& c, vx_contact* cs, const IslandPlan& plan, const V3& g, float h, int substeps,
                       const vx_solver_options& o, bool warmStart, bool integrate) {
    VXB_TRY(solveBuffers(c, plan.contacts + 1));
    SolveArgs A = solveArgs(c, cs, plan);
    A.gravity = g;
    A.h = h;
    A.substeps = substeps;
    A.sweeps = 2 * o.velocityIterations;
    A.warmStart = warmStart ? 1 : 0;
    A.integrate = integrate ? 1 : 0;
    A.coneBlock = o.frictionModel == VX_FRICTION_CONE_BLOCK;
    VXB_TRY(launchSolve(c, A));
    if (integrate && plan.freeTo > plan.freeFrom)
        LAUNCH(c, freeBodiesKernel, blocksFor(plan.freeTo - plan.freeFrom, 128), 128, c.B, P<uint32_t>(c.bodyValBuf),
               plan.freeFrom, plan.freeTo, g, h, substeps);
    return VXB_OK;
}

static int positionCorrection(Context& c, vx_contact* cs, const IslandPlan& plan, const vx_solver_options& o, float h) {
    if (o.positionIterations <= 0 || plan.islands == 0) return VXB_OK;
    SolveArgs A = solveArgs(c, cs, plan);
    A.positionIterations = o.positionIterations;
    A.stackStabilization = o.enableStackStabilization;
    A.stackStiffness = o.stackStiffness;
    A.stackDamping = o.stackDamping;
    A.h = h;
    VXB_TRY(launchSolve(c, A));
    return VXB_OK;
}

static int conservativeAdvancement(Context& c, uint32_t npairs, float dt) {
    if (npairs == 0) return VXB_OK;
    const uint32_t n = c.n;
    VXB_TRY(ensure(c, c.caFlagBuf, (size_t)npairs * 28 + 64));
    VXB_TRY(ensure(c, c.caBodyMarkBuf, (size_t)n * 16 + 16));
    VXB_TRY(ensure(c, c.caCandBuf, (size_t)npairs * 28 + 64));
    float4* endGap = P<float4>(c.caFlagBuf);
    uint32_t* flags = reinterpret_cast<uint32_t*>(endGap + npairs);
    uint32_t* candFlags = flags + npairs;
    uint32_t* flagRank = candFlags + npairs;
    uint32_t* bodyMark = P<uint32_t>(c.caBodyMarkBuf);
    uint32_t* rewound = bodyMark + n;
    uint32_t* front[2] = {rewound + n, rewound + 2 * (size_t)n};  // widening frontiers
    uint32_t* queue = P<uint32_t>(c.caCandBuf);  // exclusive-scan ranks first, then the ready queue
    uint32_t* candIndex = queue + npairs;
    uint32_t* succ = candIndex + npairs;          // two per candidate
    uint32_t* pending = succ + 2 * (size_t)npairs;
    uint32_t* depth = pending + npairs;
    uint32_t* crit = depth + npairs;
    VXB_CUDA(c, cudaMemsetAsync(bodyMark, 0, (size_t)n * 8, c.stream));
    const uint64_t* pk = P<uint64_t>(c.pairKeyBuf);
    const float4* prevPos = P<float4>(c.prevPoseBuf);
    const float4* prevRot = prevPos + n;
    // group the pairs by shape combination for the probe (the narrow phase's
    // grouping buffers are free again at this point of the step)
    const uint32_t* probeOrder = nullptr;
    if (npairs >= kProbeGroupMin) {
        VXB_TRY(ensure(c, c.classKeyBuf, (size_t)npairs * 8 + 64));
        VXB_TRY(ensure(c, c.classValBuf, (size_t)npairs * 4 + 64));
        LAUNCH(c, pairClassKernel, blocksFor(npairs, 256), 256, c.B, pk, npairs, P<uint64_t>(c.classKeyBuf),
               P<uint32_t>(c.classValBuf));
        VXB_TRY(sortPairs(c, P<uint64_t>(c.classKeyBuf), P<uint32_t>(c.classValBuf), npairs, 8));
        probeOrder = P<uint32_t>(c.classValBuf);
    }
    // the probe writes each pair's outcome at its own index and only sets marks: trials need no restore
    VXB_TRY(tunedLaunch(c, kTuneProbe, npairs, [&](LaunchShape sh) {
        LAUNCH(c, caProbeKernel, sh.grid(npairs, c.smCount), sh.threads, c.B, soupOf(c), pk, probeOrder, npairs, dt,
               flags, bodyMark, endGap);
    }, [] { return (int)VXB_OK; }));
    // speculative outcomes of the flagged pairs on the probe's state
    VXB_TRY(exclusiveScan(c, flags, flagRank, npairs, &c.dCounters->caFlagged));
    VXB_TRY(readCounters(c));
    const uint32_t flagged = c.hostCounters.caFlagged;
    if (flagged == 0) return VXB_OK;  // nothing flagged: no pair is examined, nothing moves
    VXB_TRY(ensure(c, c.caSpecBuf, (size_t)flagged * (8 * sizeof(float4) + 8) + 64));
    float4* specState = P<float4>(c.caSpecBuf);
    uint32_t* specResult = reinterpret_cast<uint32_t*>(specState + 8 * (size_t)flagged);
    uint32_t* flaggedList = specResult + flagged;
    LAUNCH(c, compactKernel, blocksFor(npairs, 256), 256, flags, flagRank, npairs, flaggedList);
    // Spread the flagged pairs evenly over all SMs, one single-warp block per
    // group of `lanes` pairs: a distance query's latency grows with the number
    // of stack frames live on its SM (local memory shares the SM's L1), so a
    // few flagged pairs run one per SM rather than packed into a few warps.
    uint32_t lanes = 1;
    while (lanes < 32 && (size_t)lanes * c.smCount < flagged) lanes <<= 1;
    const uint32_t spread = 32u / lanes;
    LAUNCH(c, caSpeculateKernel, (flagged + lanes - 1) / lanes, 32, c.B, soupOf(c), pk, (const uint32_t*)flaggedList,
           flagged, spread, (const float4*)endGap, dt, prevPos, prevRot, specState, specResult, c.dCounters);
    // mark ahead of the cascade before the first pass too (fewer replays)
    {
        const uint32_t* frontier = bodyMark;
        for (int hop = 0; hop < kCaInitialHops; ++hop) {
            uint32_t* next = front[hop & 1];
            VXB_CUDA(c, cudaMemsetAsync(next, 0, (size_t)n * 4, c.stream));
            LAUNCH(c, caWidenKernel, blocksFor(npairs, 256), 256, c.B, pk, npairs, bodyMark, frontier, next);
            frontier = next;
        }
    }
    VXB_TRY(ensure(c, c.snapBuf, (size_t)n * 64));
    VXB_TRY(ensure(c, c.coopBuf, sizeof(CoopState)));
    CoopState* st = P<CoopState>(c.coopBuf);
    bool snapped = false, serial = false;
    for (int pass = 0;; ++pass) {
        if (pass == kCaWidenLimit) { serial = true; break; }
        LAUNCH(c, caCandidateKernel, blocksFor(npairs, 256), 256, c.B, pk, npairs, flags, bodyMark, candFlags,
               c.dCounters);
        VXB_TRY(exclusiveScan(c, candFlags, queue, npairs, &c.dCounters->caCandidates));
        VXB_TRY(readCounters(c));
        const uint32_t ncand = c.hostCounters.caCandidates;
        if (ncand == 0) return VXB_OK;
        LAUNCH(c, compactKernel, blocksFor(npairs, 256), 256, candFlags, queue, npairs, candIndex);
        // successors and predecessor counts through shared dynamic bodies
        const size_t valsOffset = ((size_t)ncand * 16 + 255) & ~(size_t)255;  // both arrays 256-byte aligned
        VXB_TRY(ensure(c, c.islandInfoBuf, valsOffset + (size_t)ncand * 8 + 16));
        uint64_t* ekeys = P<uint64_t>(c.islandInfoBuf);
        uint32_t* evals = reinterpret_cast<uint32_t*>(P<char>(c.islandInfoBuf) + valsOffset);
        VXB_TRY(ensure(c, c.caInfoBuf, (size_t)ncand * 16 + 64));
        uint4* info = P<uint4>(c.caInfoBuf);
        LAUNCH(c, caEntryKernel, blocksFor(ncand, 256), 256, c.B, pk, (const uint32_t*)candIndex, ncand, n,
               (const uint32_t*)flags, ekeys, evals, info);
        VXB_TRY(sortPairs(c, ekeys, evals, 2 * ncand, bitsFor(n)));
        VXB_CUDA(c, cudaMemsetAsync(pending, 0, (size_t)ncand * 4, c.stream));
        VXB_CUDA(c, cudaMemsetAsync(depth, 0, (size_t)ncand * 4, c.stream));
        VXB_CUDA(c, cudaMemsetAsync(crit, 0, (size_t)ncand * 4, c.stream));
        LAUNCH(c, caLinkKernel, blocksFor(2 * ncand, 256), 256, ekeys, evals, 2 * ncand, n, succ, pending);
        if (!snapped) {
            LAUNCH(c, copyStateKernel, blocksFor(n, 256), 256, c.B, n, P<float4>(c.snapBuf), 0);
            snapped = true;
        }
        VXB_CUDA(c, cudaMemsetAsync(queue, 0xff, (size_t)ncand * 4, c.stream));
        VXB_TRY(resetCoop(c, st));
        const int rc = launchCooperativeCapped(c, kCaFlowBlocksPerSm, caFlowKernel, kCaFlowThreads, c.B, soupOf(c),
                                               (const uint32_t*)flagRank, (const float4*)specState,
                                               (const uint32_t*)specResult, (const uint4*)info, ncand,
                                               (const uint32_t*)succ, pending, queue, depth, crit,
                                               (const uint32_t*)bodyMark, rewound, dt, prevPos, prevRot, c.dCounters,
                                               st);
        if (rc == VXB_ERR_UNSUPPORTED) { serial = true; break; }
        VXB_TRY(rc);
        CoopState host;
        VXB_CUDA(c, cudaMemcpyAsync(&host, st, sizeof(host), cudaMemcpyDeviceToHost, c.stream));
        VXB_TRY(readCounters(c));
        if (host.timeout) return fail(c, VXB_ERR_TIMEOUT, "a wait timed out in the rewind pass");
        if (host.spill) return fail(c, VXB_ERR_INTERNAL, "inconsistent candidate links in the rewind pass");
        c.caRounds += host.rounds;
        if (!c.hostCounters.caOverflow) return VXB_OK;
        // a rewind reached an unmarked body: widen the marked set and replay from the snapshot
        LAUNCH(c, copyStateKernel, blocksFor(n, 256), 256, c.B, n, P<float4>(c.snapBuf), 1);
        {
            const uint32_t* frontier = rewound;
            for (int hop = 0; hop < kCaWidenHops; ++hop) {
                uint32_t* next = front[hop & 1];
                VXB_CUDA(c, cudaMemsetAsync(next, 0, (size_t)n * 4, c.stream));
                LAUNCH(c, caWidenKernel, blocksFor(npairs, 256), 256, c.B, pk, npairs, bodyMark, frontier, next);
                frontier = next;
            }
        }
        VXB_CUDA(c, cudaMemsetAsync(rewound, 0, (size_t)n * 4, c.stream));
        VXB_CUDA(c, cudaMemsetAsync(&c.dCounters->rewinds, 0, 4, c.stream));
        VXB_CUDA(c, cudaMemsetAsync(&c.dCounters->caOverflow, 0, 4, c.stream));
        ++c.caWidenings;
    }
    if (serial) {
        if (snapped) LAUNCH(c, copyStateKernel, blocksFor(n, 256), 256, c.B, n, P<float4>(c.snapBuf), 1);
        VXB_CUDA(c, cudaMemsetAsync(rewound, 0, (size_t)n * 4, c.stream));
        LAUNCH(c, caFullSerialKernel, 1, 32, c.B, soupOf(c), pk, npairs, flags, rewound, dt, prevPos, prevRot,
               c.dCounters);
    }
    return VXB_OK;
}

// One World::step on the device world.
static int stepOnce(Context& c) {
    const vxb_step_config& cfg = c.config;
    const uint32_t n = c.n;
    const int substeps = cfg.substeps > 0 ? cfg.substeps : 1;
    const float dt = cfg.dt;
    const float h = dt / substeps;
    const V3 g{cfg.gravity.x, cfg.gravity.y, cfg.gravity.z};
    VXB_TRY(resetCounters(c));
    c.stats.colorRounds = 0;
    c.stats.giantIslands = 0;
    c.caRounds = 0;
    c.caWidenings = 0;
    VXB_TRY(ensure(c, c.prevPoseBuf, (size_t)n * 32));
    float4* prevPos = P<float4>(c.prevPoseBuf);
    if (c.tape.active) VXB_TRY(tapeStepBegin(c));
    stageBegin(c, kStagePrepare);
    LAUNCH(c, prepareKernel, blocksFor(n, 256), 256, c.B, n, g, h, prevPos, prevPos + n, 1);
    stageEnd(c, kStagePrepare);
    uint32_t npairs = 0, m = 0, nrec = 0;
    VXB_TRY(broadPhase(c, dt, &npairs));
    c.stats.candidatePairs = npairs;
    VXB_TRY(narrowPhase(c, P<uint64_t>(c.pairBuf), npairs, dt, 0, &m, &nrec, c.convexPairs,
                        P<uint64_t>(c.pairBuf) + c.pairCap));
    vx_contact* cs = P<vx_contact>(c.contactBuf[c.cur]);
    stageBegin(c, kStageWarmStart);
    VXB_TRY(wakePass(c, cs, m));  // src/world.cpp:4106-4128: after detection, before warm starting
    if (c.tape.active)
        VXB_TRY(tapeBeforeMatch(c, cs, m, P<vx_contact>(c.contactBuf[c.cur ^ 1]), P<uint64_t>(c.prevKeyBuf),
                                c.prevCount));
    if (c.prevCount && m)
        LAUNCH(c, matchKernel, blocksFor(m, 128), 128, cs, m, P<vx_contact>(c.contactBuf[c.cur ^ 1]),
               P<uint64_t>(c.prevKeyBuf), c.prevCount, c.dCounters);
    if (c.tape.active) VXB_TRY(tapeAfterMatch(c, cs, m));
    stageEnd(c, kStageWarmStart);
    IslandPlan plan;
    stageBegin(c, kStageIslands);
    VXB_TRY(buildIslands(c, cs, m, plan, nullptr));
    VXB_TRY(prepareSegments(c, plan));
    if (c.tape.active) VXB_TRY(tapeAfterIslands(c, P<uint32_t>(c.colorBuf), m));
    stageEnd(c, kStageIslands);
    stageBegin(c, kStageSolve);
    VXB_TRY(runSubsteps(c, cs, plan, g, h, substeps, cfg.solver, true, true));
    stageEnd(c, kStageSolve);
    stageBegin(c, kStageRewind);
    if (m) VXB_TRY(conservativeAdvancement(c, nrec, dt));
    if (c.tape.active && m && nrec) VXB_TRY(tapeAfterRewind(c, P<uint32_t>(c.caBodyMarkBuf) + n));
    stageEnd(c, kStageRewind);
    stageBegin(c, kStagePositions);
    VXB_TRY(positionCorrection(c, cs, plan, cfg.solver, h));
    stageEnd(c, kStagePositions);
    // events, sleeping and the resting pairs' cached contacts (before the
    // forces are cleared: the calm test reads them)
    uint32_t kept = 0;
    VXB_TRY(sleepAndEvents(c, cs, m, dt, &kept));
    LAUNCH(c, clearForcesKernel, blocksFor(n, 256), 256, c.B, n);
    // previous-contact cache: this step's contacts in (a, b, point) order, and
    // resting pairs' cached contacts merged in by pair
    if (kept) {
        VXB_TRY(mergeKeptContacts(c, m, kept));
        cs = P<vx_contact>(c.contactBuf[c.cur]);
    }
    const uint32_t cacheCount = m + kept;
    VXB_TRY(ensure(c, c.prevKeyBuf, (size_t)cacheCount * 8 + 16));
    if (cacheCount)
        LAUNCH(c, contactKeysKernel, blocksFor(cacheCount, 256), 256, cs, cacheCount, P<uint64_t>(c.prevKeyBuf));
    c.prevCount = cacheCount;
    c.stepContacts = m;
    c.cur ^= 1;
    if (c.tape.active) VXB_TRY(tapeStepEnd(c, m));
    VXB_TRY(readCounters(c));
    c.stats.contacts = m;
    c.stats.islands = plan.realIslands;
    c.stats.colors = c.hostCounters.maxColors;
    c.stats.largestIsland = c.hostCounters.largestIsland;
    c.stats.rewinds = c.hostCounters.rewinds;
    c.stats.rewindRounds = c.caRounds;
    c.stats.rewindReplays = c.caWidenings;
    c.stats.rewindGapQueries = c.hostCounters.caGapQueries;
    c.stats.rewindCriticalMicros = c.hostCounters.caCritMicros;
    c.stats.rewindSpeculateMicros = c.hostCounters.caSpecMicros;
    c.stats.warmStarted = c.hostCounters.warmStarted;
    c.stats.velocityIterations = (uint32_t)(2 * cfg.solver.velocityIterations * substeps);
    if (c.hostCounters.timeout) return fail(c, VXB_ERR_TIMEOUT, "a bounded device wait gave up");
    if (c.hostCounters.planFault) return fail(c, VXB_ERR_INTERNAL, "inconsistent island plan in the solve");
    return VXB_OK;
}

int worldStep(Context& c, int steps) {
    if (!c.configured) return fail(c, VXB_ERR_INVALID, "vxb_world_configure was not called");
    if (c.n == 0) return fail(c, VXB_ERR_INVALID, "no bodies loaded");
    VXB_TRY(ensure(c, c.countersBuf, sizeof(Counters)));
    c.dCounters = P<Counters>(c.countersBuf);
    for (int s = 0; s < steps; ++s) VXB_TRY(stepOnce(c));
    VXB_CUDA(c, cudaStreamSynchronize(c.stream));
    VXB_CUDA(c, cudaGetLastError());
    return VXB_OK;
}

int readContacts(Context& c, vx_contact* out, uint32_t cap, uint32_t* count) {
    const uint32_t m = c.stepContacts;
    if (count) *count = m;
    if (out && m && c.prevCount != m) return readStepContacts(c, out, std::min(m, cap));
    if (out && m) {
        VXB_CUDA(c, cudaMemcpyAsync(out, c.contactBuf[c.cur ^ 1].ptr, (size_t)std::min(m, cap) * sizeof(vx_contact),
                                    cudaMemcpyDeviceToHost, c.stream));
        VXB_CUDA(c, cudaStreamSynchronize(c.stream));
    }
    return VXB_OK;
}

int writeContacts(Context& c, const vx_contact* contacts, uint32_t m) {
    tapeEnd(c);
    VXB_TRY(ensure(c, c.contactBuf[c.cur ^ 1], (size_t)m * sizeof(vx_contact) + 128));
    VXB_TRY(ensure(c, c.prevKeyBuf, (size_t)m * 8 + 16));
    if (m) {
        VXB_CUDA(c, cudaMemcpyAsync(c.contactBuf[c.cur ^ 1].ptr, contacts, (size_t)m * sizeof(vx_contact),
                                    cudaMemcpyHostToDevice, c.stream));
        LAUNCH(c, contactKeysKernel, blocksFor(m, 256), 256, P<vx_contact>(c.contactBuf[c.cur ^ 1]), m,
               P<uint64_t>(c.prevKeyBuf));
    }
    c.prevCount = m;
    c.stepContacts = m;
    VXB_CUDA(c, cudaStreamSynchronize(c.stream));
    return VXB_OK;
}

// ---- stage entry points -----------------------------------------------------

int stagePairs(Context& c, float dt, uint64_t* out, uint32_t cap, uint32_t* count) {
    VXB_TRY(ensure(c, c.countersBuf, sizeof(Counters)));
    c.dCounters = P<Counters>(c.countersBuf);
    VXB_TRY(resetCounters(c));
    uint32_t npairs = 0;
    VXB_TRY(broadPhase(c, dt, &npairs));
    *count = npairs;
    if (out) {
        std::vector<uint64_t> host(npairs);
        if (c.convexPairs)
            VXB_CUDA(c, cudaMemcpyAsync(host.data(), c.pairBuf.ptr, (size_t)c.convexPairs * 8, cudaMemcpyDeviceToHost,
                                        c.stream));
        if (c.planePairs)
            VXB_CUDA(c, cudaMemcpyAsync(host.data() + c.convexPairs, P<uint64_t>(c.pairBuf) + c.pairCap,
                                        (size_t)c.planePairs * 8, cudaMemcpyDeviceToHost, c.stream));
        VXB_CUDA(c, cudaStreamSynchronize(c.stream));
        std::sort(host.begin(), host.end());
        std::memcpy(out, host.data(), (size_t)std::min(npairs, cap) * 8);
    }
    return npairs > cap && out ? fail(c, VXB_ERR_CAPACITY, "pair buffer too small") : VXB_OK;
}

int stageCollide(Context& c, const uint64_t* pairs, uint32_t npairs, float dt, vx_contact* out, uint32_t cap,
                 uint32_t* counts, uint32_t* total) {
    VXB_TRY(ensure(c, c.countersBuf, sizeof(Counters)));
    c.dCounters = P<Counters>(c.countersBuf);
    VXB_TRY(resetCounters(c));
    VXB_TRY(ensure(c, c.pairBuf, (size_t)npairs * 8 + 16));
    if (npairs)
        VXB_CUDA(c, cudaMemcpyAsync(c.pairBuf.ptr, pairs, (size_t)npairs * 8, cudaMemcpyHostToDevice, c.stream));
    uint32_t m = 0, nrec = 0;
    VXB_TRY(narrowPhase(c, P<uint64_t>(c.pairBuf), npairs, dt, 1, &m, &nrec));
    *total = m;
    if (m > cap) return fail(c, VXB_ERR_CAPACITY, "contact buffer too small");
    if (m) VXB_CUDA(c, cudaMemcpyAsync(out, c.contactBuf[c.cur].ptr, (size_t)m * sizeof(vx_contact),
                                       cudaMemcpyDeviceToHost, c.stream));
    if (counts) {
        std::vector<uint64_t> keys(nrec);
        std::vector<uint32_t> cnt(nrec);
        if (nrec) {
            VXB_CUDA(c, cudaMemcpyAsync(keys.data(), c.recKeyBuf.ptr, (size_t)nrec * 8, cudaMemcpyDeviceToHost, c.stream));
            VXB_CUDA(c, cudaMemcpyAsync(cnt.data(), c.recCountBuf.ptr, (size_t)nrec * 4, cudaMemcpyDeviceToHost, c.stream));
        }
        VXB_CUDA(c, cudaStreamSynchronize(c.stream));
        std::fill(counts, counts + npairs, 0u);
        for (uint32_t r = 0; r < nrec; ++r) counts[keys[r]] = cnt[r];
    }
    VXB_CUDA(c, cudaStreamSynchronize(c.stream));
    return VXB_OK;
}

int stageColor(Context& c, const vx_contact* contacts, uint32_t m, int32_t* colorOf, uint32_t* numColors) {
    VXB_TRY(ensure(c, c.countersBuf, sizeof(Counters)));
    c.dCounters = P<Counters>(c.countersBuf);
    VXB_TRY(resetCounters(c));
    VXB_TRY(ensure(c, c.contactBuf[c.cur], (size_t)m * sizeof(vx_contact) + 128));
    if (m) VXB_CUDA(c, cudaMemcpyAsync(c.contactBuf[c.cur].ptr, contacts, (size_t)m * sizeof(vx_contact),
                                       cudaMemcpyHostToDevice, c.stream));
    IslandPlan plan;
    VXB_TRY(buildIslands(c, P<vx_contact>(c.contactBuf[c.cur]), m, plan, reinterpret_cast<uint32_t*>(colorOf)));
    VXB_TRY(readCounters(c));
    *numColors = c.hostCounters.maxColors;
    return VXB_OK;
}

__global__ void distanceKernel(BodyArrays B, Soup soup, const uint64_t* pairs, uint32_t npairs, int path,
                               float* out) {
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < npairs; p += gridDim.x * blockDim.x) {
        const Convex ca = makeConvex(loadView(B, (uint32_t)(pairs[p] >> 32)), soup);
        const Convex cb = makeConvex(loadView(B, (uint32_t)pairs[p]), soup);
        const GjkResult r = path == 0 ? distanceQuery(ca, cb) : gjkDistance(ca, cb);
        float* o = out + 11 * (size_t)p;
        o[0] = r.distance;
        o[1] = r.normal.x; o[2] = r.normal.y; o[3] = r.normal.z;
        o[4] = r.pointA.x; o[5] = r.pointA.y; o[6] = r.pointA.z;
        o[7] = r.pointB.x; o[8] = r.pointB.y; o[9] = r.pointB.z;
        o[10] = r.overlapping ? 1.0f : 0.0f;
    }
}

int stageDistance(Context& c, const uint64_t* pairs, uint32_t npairs, int path, float* out) {
    if (npairs == 0) return VXB_OK;
    VXB_TRY(ensure(c, c.pairBuf, (size_t)npairs * 8 + 16));
    VXB_TRY(ensure(c, c.contactTmpBuf, (size_t)npairs * 44 + 16));
    VXB_CUDA(c, cudaMemcpyAsync(c.pairBuf.ptr, pairs, (size_t)npairs * 8, cudaMemcpyHostToDevice, c.stream));
    LAUNCH(c, distanceKernel, blocksFor(npairs, 64), 64, c.B, soupOf(c), P<uint64_t>(c.pairBuf), npairs, path,
           P<float>(c.contactTmpBuf));
    VXB_CUDA(c, cudaMemcpyAsync(out, c.contactTmpBuf.ptr, (size_t)npairs * 44, cudaMemcpyDeviceToHost, c.stream));
    VXB_CUDA(c, cudaStreamSynchronize(c.stream));
    return VXB_OK;
}

// ---- Backend-interface mode ---------------------------------------------------

int backendIntegrate(Context& c, vx_vec3 gravity, float dt) {
    LAUNCH(c, integrateKernel, blocksFor(c.n, 256), 256, c.B, c.n, V3{gravity.x, gravity.y, gravity.z}, dt);
    return VXB_OK;
}

int backendIntegrateTransforms(Context& c, float dt) {
    LAUNCH(c, transformsKernel, blocksFor(c.n, 256), 256, c.B, c.n, dt);
    return VXB_OK;
}

int backendFindContacts(Context& c, float dt, uint32_t* count) {
    VXB_TRY(ensure(c, c.countersBuf, sizeof(Counters)));
    c.dCounters = P<Counters>(c.countersBuf);
    VXB_TRY(resetCounters(c));
    uint32_t npairs = 0, m = 0, nrec = 0;
    VXB_TRY(broadPhase(c, dt, &npairs));
    VXB_TRY(narrowPhase(c, P<uint64_t>(c.pairBuf), npairs, dt, 0, &m, &nrec, c.convexPairs,
                        P<uint64_t>(c.pairBuf) + c.pairCap));
    c.backendContacts = m;
    c.backendColored = false;
    *count = m;
    return VXB_OK;
}

int backendCopyContacts(Context& c, vx_contact* out, uint32_t cap) {
    const uint32_t m = c.backendContacts;
    if (m > cap) return fail(c, VXB_ERR_CAPACITY, "contact buffer too small");
    if (m) VXB_CUDA(c, cudaMemcpyAsync(out, c.contactBuf[c.cur].ptr, (size_t)m * sizeof(vx_contact),
                                       cudaMemcpyDeviceToHost, c.stream));
    VXB_CUDA(c, cudaStreamSynchronize(c.stream));
    return VXB_OK;
}

static bool hostContactLess(const vx_contact& x, const vx_contact& y) {
    const uint64_t kx = ((uint64_t)x.a << 32) | x.b, ky = ((uint64_t)y.a << 32) | y.b;
    if (kx != ky) return kx < ky;
    if (x.point.x != y.point.x) return x.point.x < y.point.x;
    if (x.point.y != y.point.y) return x.point.y < y.point.y;
    return x.point.z < y.point.z;
}

// solveVelocities / advanceSubsteps. On warm start the contacts are sorted,
// coloured, written back in colour order and kept resident; the solve then
// runs `substeps` substeps (fullSubsteps) or one velocity solve.
int backendSolve(Context& c, vx_contact* contacts, uint32_t m, float h, bool warmStart, const vx_solver_options& o,
                 vx_vec3 gravity, int substeps, bool fullSubsteps) {
    VXB_TRY(ensure(c, c.countersBuf, sizeof(Counters)));
    c.dCounters = P<Counters>(c.countersBuf);
    IslandPlan& plan = c.backendPlan;  // retained between the warm-start call and later calls
    if (warmStart) {
        VXB_TRY(resetCounters(c));
        c.hostSorted.assign(contacts, contacts + m);
        std::stable_sort(c.hostSorted.begin(), c.hostSorted.end(), hostContactLess);
        VXB_TRY(ensure(c, c.contactBuf[c.cur], (size_t)m * sizeof(vx_contact) + 128));
        if (m) VXB_CUDA(c, cudaMemcpyAsync(c.contactBuf[c.cur].ptr, c.hostSorted.data(), (size_t)m * sizeof(vx_contact),
                                           cudaMemcpyHostToDevice, c.stream));
        VXB_TRY(buildIslands(c, P<vx_contact>(c.contactBuf[c.cur]), m, plan, nullptr));
        VXB_TRY(prepareSegments(c, plan));
        // colour order back to the host (pre-solve values, like the reference's sorted_ copy)
        std::vector<uint32_t> order(m);
        if (m) VXB_CUDA(c, cudaMemcpyAsync(order.data(), c.islandValBuf.ptr, (size_t)m * 4, cudaMemcpyDeviceToHost,
                                           c.stream));
        VXB_CUDA(c, cudaStreamSynchronize(c.stream));
        for (uint32_t k = 0; k < m; ++k) contacts[k] = c.hostSorted[order[k]];
        c.backendContacts = m;
        c.backendColored = true;
    }
    if (m == 0 && !fullSubsteps) return VXB_OK;
    const V3 g{gravity.x, gravity.y, gravity.z};
    if (fullSubsteps) {
        VXB_TRY(runSubsteps(c, P<vx_contact>(c.contactBuf[c.cur]), plan, g, h, substeps, o, warmStart, true));
    } else {
        VXB_TRY(runSubsteps(c, P<vx_contact>(c.contactBuf[c.cur]), plan, g, h, 1, o, warmStart, false));
    }
    VXB_CUDA(c, cudaGetLastError());
    VXB_TRY(readCounters(c));
    if (c.hostCounters.timeout) return fail(c, VXB_ERR_TIMEOUT, "a bounded device wait gave up");
    if (c.hostCounters.planFault) return fail(c, VXB_ERR_INTERNAL, "inconsistent island plan in the solve");
    return VXB_OK;
}

int backendFetchImpulses(Context& c, vx_contact* contacts, uint32_t m) {
    if (!c.backendColored || m != c.backendContacts || m == 0) return VXB_OK;
    VXB_TRY(ensure(c, c.contactTmpBuf, (size_t)m * sizeof(vx_contact)));
    LAUNCH(c, gatherContactsKernel, blocksFor(m, 128), 128, P<vx_contact>(c.contactBuf[c.cur]),
           P<uint32_t>(c.islandValBuf), m, P<vx_contact>(c.contactTmpBuf));
    VXB_CUDA(c, cudaMemcpyAsync(contacts, c.contactTmpBuf.ptr, (size_t)m * sizeof(vx_contact), cudaMemcpyDeviceToHost,
                                c.stream));
    VXB_CUDA(c, cudaStreamSynchronize(c.stream));
    return VXB_OK;
}

}  // namespace vxb
