// Island sleeping, the wake pass and contact events of the device world.
//
// The reference runs these on the host after every step:
//   wake pass      src/world.cpp:4106-4128 (after detection, before warm start)
//   contact events src/world.cpp:4398-4488 (after position correction)
//   sleeping       SleepManager::update, src/sleep.cpp:52-237 (union-find
//                  islands, contact stability, calm timers, island minimum,
//                  drowsy / asleep transitions), called by World::updateSleeping
//   cached contacts of resting pairs, src/world.cpp:4496-4521 (after sleeping)
// Here they are kernels over the step's device data. Sleep state per body
// (float4): sleepTimer, consecutive stable frames, state (0 awake, 1 asleep,
// 2 drowsy), enableSleep. The asleep bit of the packed body flags mirrors
// state 1; the rest of the pipeline reads only that bit.
//
// Order-dependent rule: the wake pass walks the contacts in order, and a body
// it wakes can wake a later contact's partner. Only contacts with an asleep
// endpoint can change anything, so a parallel pass lists them and counts those
// that can start a wake; one thread walks the list in order when the count
// is not zero (all worlds at once: they never share bodies).
#include <algorithm>
#include <cstring>
#include <vector>

#include "context.cuh"

namespace vxb {

static_assert(sizeof(vxb_contact_event) == 40, "event record: a, b, point, normal, impulse, type, sensor, pad");

namespace {

#define SL_TRY(expr)                   \
    do {                               \
        int s_ = (expr);               \
        if (s_ != VXB_OK) return s_;   \
    } while (0)

#define SL_CUDA(c, expr)                                              \
    do {                                                              \
        cudaError_t e_ = (expr);                                      \
        if (e_ != cudaSuccess) return cudaStatus((c), e_, #expr);     \
    } while (0)

#define SL_LAUNCH(c, kernel, grid, block, ...)                               \
    do {                                                                     \
        kernel<<<(grid), (block), 0, (c).stream>>>(__VA_ARGS__);            \
        ++(c).launches;                                                      \
    } while (0)

template <class T> T* PT(DevBuf& b) { return reinterpret_cast<T*>(b.ptr); }

inline uint32_t gridFor(uint64_t items, int threads) {
    uint64_t b = (items + threads - 1) / threads;
    return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(b, 65535u * 16u));
}

constexpr float kAwake = 0.0f, kAsleep = 1.0f, kDrowsy = 2.0f;

VXD void setAsleepBit(BodyArrays& B, uint32_t i, bool asleep) {
    uint4 f = B.filt[i];
    f.x = asleep ? (f.x | kAsleepBit) : (f.x & ~kAsleepBit);
    B.filt[i] = f;
}

VXD void markWorld(uint32_t* tapeFlags, const uint32_t* worldOf, uint32_t i) {
    if (tapeFlags) atomicOr(tapeFlags + (worldOf ? worldOf[i] : 0u), (uint32_t)VXB_ADJ_UNSUPPORTED);
}

__global__ void sleepExportKernel(vx_body* out, uint32_t n, const float4* sleep) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 s = sleep[i];
        out[i].sleepTimer = s.x;
        out[i].asleep = s.z == kAsleep ? 1 : s.z == kDrowsy ? 2 : 0;
    }
}

VXD bool moving(const BodyArrays& B, uint32_t i) {
    return lengthSq(f3(B.vel[i])) + lengthSq(f3(B.ang[i])) > 1e-3f;
}

// Contacts with an asleep endpoint (the walk's candidates), and a count of
// those that can start a wake now.
__global__ void wakeScanKernel(const vx_contact* cs, uint32_t m, BodyArrays B, uint32_t* listed, uint32_t* starters) {
    uint32_t count = 0;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
        const uint32_t a = cs[k].a, b = cs[k].b;
        const uint32_t fa = B.filt[a].x, fb = B.filt[b].x;
        uint32_t flag = 0;
        if (!isSensor(fa) && !isSensor(fb) && (isAsleep(fa) || isAsleep(fb))) {
            flag = 1;
            const bool impact = cs[k].vn0 < -0.1f;
            if ((isAsleep(fa) && !isStaticBody(fb) && !isAsleep(fb) && (impact || moving(B, b))) ||
                (isAsleep(fb) && !isStaticBody(fa) && !isAsleep(fa) && (impact || moving(B, a))))
                ++count;
        }
        listed[k] = flag;
    }
    if (count) atomicAdd(starters, count);
}

__global__ void listKernel(const uint32_t* flags, const uint32_t* rank, uint32_t m, uint32_t* list) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x)
        if (flags[k]) list[rank[k]] = k;
}

// The ordered walk (src/world.cpp:4110-4128) over the listed contacts.
__global__ void wakeWalkKernel(const vx_contact* cs, const uint32_t* list, const uint32_t* count,
                               const uint32_t* starters, BodyArrays B, float4* sleep, uint32_t* tapeFlags,
                               const uint32_t* worldOf) {
    if (threadIdx.x != 0 || blockIdx.x != 0 || *starters == 0) return;
    const uint32_t total = *count;
    for (uint32_t t = 0; t < total; ++t) {
        const vx_contact& c = cs[list[t]];
        const bool impact = c.vn0 < -0.1f;
        const uint32_t fa = B.filt[c.a].x, fb = B.filt[c.b].x;
        if (isAsleep(fa) && !isStaticBody(fb) && !isAsleep(fb) && (impact || moving(B, c.b))) {
            setAsleepBit(B, c.a, false);
            float4 s = sleep[c.a];
            s.z = kAwake;
            s.x = 0.0f;
            sleep[c.a] = s;
            markWorld(tapeFlags, worldOf, c.a);
        }
        const uint32_t fa2 = B.filt[c.a].x;
        if (isAsleep(fb) && !isStaticBody(fa2) && !isAsleep(fa2) && (impact || moving(B, c.a))) {
            setAsleepBit(B, c.b, false);
            float4 s = sleep[c.b];
            s.z = kAwake;
            s.x = 0.0f;
            sleep[c.b] = s;
            markWorld(tapeFlags, worldOf, c.b);
        }
    }
}

// Contact stability (src/sleep.cpp:96-122): bit 0 has a contact, bit 1 has an
// unstable one (relative speed at the contact point above the threshold).
__global__ void stabilityKernel(const vx_contact* cs, uint32_t m, BodyArrays B, float threshold, uint32_t* bits) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
        const vx_contact& c = cs[k];
        const uint32_t fa = B.filt[c.a].x, fb = B.filt[c.b].x;
        if (isSensor(fa) || isSensor(fb)) continue;
        const V3 p{c.point.x, c.point.y, c.point.z};
        const V3 va = f3(B.vel[c.a]) + cross(f3(B.ang[c.a]), p - f3(B.pos[c.a]));
        const V3 vb = f3(B.vel[c.b]) + cross(f3(B.ang[c.b]), p - f3(B.pos[c.b]));
        const float rel = length(va - vb);
        const uint32_t v = 1u | (rel > threshold ? 2u : 0u);
        if (isDynamic(fa)) atomicOr(bits + c.a, v);
        if (isDynamic(fb)) atomicOr(bits + c.b, v);
    }
}

// Stability counters (src/sleep.cpp:124-133), calm timers (:135-175) and the
// island minimum timer (:184-200) over union-find roots.
__global__ void sleepTimerKernel(BodyArrays B, uint32_t n, const uint32_t* bits, vxb_sleep_config cfg, float dt,
                                 float4* sleep, const uint32_t* root, uint32_t* islandTimer) {
    const float linTol = cfg.linearVelocityThreshold * cfg.linearVelocityThreshold;
    const float angTol = cfg.angularVelocityThreshold * cfg.angularVelocityThreshold;
    const float accTol = cfg.accelerationThreshold * cfg.accelerationThreshold;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t f = B.filt[i].x;
        if (!isDynamic(f)) continue;
        float4 s = sleep[i];
        if (cfg.enableContactStability) {
            const uint32_t b = bits[i];
            s.y = (b & 1u) && !(b & 2u) ? fminf(s.y + 1.0f, 65535.0f) : 0.0f;
        }
        if (!isAsleep(f) && s.w != 0.0f) {
            const float lin = lengthSq(f3(B.vel[i])), ang = lengthSq(f3(B.ang[i]));
            const float im = B.inertia[i].w;
            const float acc = im > 0.0f ? lengthSq(f3(B.force[i])) * im * im : 0.0f;
            bool calm = lin < linTol && ang < angTol && acc < accTol;
            if (calm && cfg.enableContactStability) calm = s.y >= (float)cfg.contactStabilityFrames;
            if (calm) {
                s.x += dt;
            } else {
                s.x = 0.0f;
                if (s.z == kDrowsy) s.z = kAwake;
            }
        }
        sleep[i] = s;
        if (!isAsleep(f)) {
            const float timer = s.w != 0.0f ? s.x : 0.0f;  // a body that may not sleep holds its island awake
            atomicMin(islandTimer + root[i], __float_as_uint(timer));
        }
    }
}

// Island transitions (src/sleep.cpp:202-237).
__global__ void sleepTransitionKernel(BodyArrays B, uint32_t n, vxb_sleep_config cfg, float4* sleep,
                                      const uint32_t* root, const uint32_t* islandTimer, uint32_t* asleepCount,
                                      uint32_t* tapeFlags, const uint32_t* worldOf) {
    uint32_t slept = 0;
    const float tDrowsy = cfg.enableGradualSleep ? cfg.timeToDrowsy : cfg.timeToSleep;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t f = B.filt[i].x;
        float4 s = sleep[i];
        if (isDynamic(f) && !isAsleep(f) && s.w != 0.0f) {
            const float minTimer = __uint_as_float(islandTimer[root[i]]);
            if (minTimer >= cfg.timeToSleep) {
                s.z = kAsleep;
                s.x = 0.0f;
                B.vel[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                B.ang[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                setAsleepBit(B, i, true);
                markWorld(tapeFlags, worldOf, i);
            } else if (cfg.enableGradualSleep && minTimer >= tDrowsy && s.z != kDrowsy) {
                s.z = kDrowsy;
            }
            sleep[i] = s;
        }
        if (isDynamic(f) && isAsleep(B.filt[i].x)) ++slept;
    }
    if (slept) atomicAdd(asleepCount, slept);
}

// ---- contact events and pair keys ------------------------------------------------

VXD uint64_t canonicalKey(uint32_t a, uint32_t b) {
    const uint32_t lo = a < b ? a : b, hi = a < b ? b : a;
    return ((uint64_t)lo << 32) | hi;
}

VXD uint32_t lowerBound(const uint64_t* keys, uint32_t count, uint64_t key) {
    uint32_t lo = 0, hi = count;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (keys[mid] < key) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

VXD bool inSorted(const uint64_t* keys, uint32_t count, uint64_t key) {
    const uint32_t lo = lowerBound(keys, count, key);
    return lo < count && keys[lo] == key;
}

// Active contacts (src/world.cpp:4418-4432): an impulse, touching live
// anchors, or (sensors) a sweep across the trigger this step. Inactive ones
// get the sentinel key (sorted last).
__global__ void activeKeysKernel(const vx_contact* cs, uint32_t m, BodyArrays B, float dt, uint64_t sentinel,
                                 uint64_t* keys, uint32_t* vals) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
        const vx_contact& c = cs[k];
        const uint32_t fa = B.filt[c.a].x, fb = B.filt[c.b].x;
        const bool sensor = isSensor(fa) || isSensor(fb);
        const V3 n{c.normal.x, c.normal.y, c.normal.z};
        const V3 wa = anchorWorld(shapeOf(fa) == kSphere, f3(B.pos[c.a]), q4(B.rot[c.a]),
                                  V3{c.localAnchorA.x, c.localAnchorA.y, c.localAnchorA.z});
        const V3 wb = anchorWorld(shapeOf(fb) == kSphere, f3(B.pos[c.b]), q4(B.rot[c.b]),
                                  V3{c.localAnchorB.x, c.localAnchorB.y, c.localAnchorB.z});
        const float live = c.bias0 + dot(n, wa - wb);
        const bool swept = sensor && c.vn0 < 0.0f && c.gap <= -c.vn0 * dt + 1e-3f;
        const bool active = !(c.normalImpulse <= 1e-6f && live > 1e-3f && !swept);
        keys[k] = active ? canonicalKey(c.a, c.b) : sentinel;
        vals[k] = k;
    }
}

__global__ void headFlagKernel(const uint64_t* keys, uint32_t m, uint64_t sentinel, uint32_t* flags) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x)
        flags[k] = keys[k] != sentinel && (k == 0 || keys[k - 1] != keys[k]) ? 1u : 0u;
}

// One event per active pair (runs of the sorted keys, indices ascending
// within a run): Begin or Persist by the previous step's pair keys; the
// representative is the first contact with the largest normal impulse
// (src/world.cpp:4433-4457). Writes the pair key at the same rank.
__global__ void activeEventsKernel(const uint64_t* keys, const uint32_t* vals, uint32_t m, uint64_t sentinel,
                                   const uint32_t* rank, const vx_contact* cs, BodyArrays B,
                                   const uint64_t* prevPairs, uint32_t prevPairCount, vxb_contact_event* events,
                                   uint64_t* pairsOut) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
        const uint64_t key = keys[k];
        if (key == sentinel || (k > 0 && keys[k - 1] == key)) continue;
        const uint32_t lo = (uint32_t)(key >> 32), hi = (uint32_t)key;
        vxb_contact_event e;
        memset(&e, 0, sizeof(e));
        e.a = lo;
        e.b = hi;
        e.type = inSorted(prevPairs, prevPairCount, key) ? 1u : 0u;
        e.sensor = (isSensor(B.filt[lo].x) || isSensor(B.filt[hi].x)) ? 1u : 0u;
        bool set = false;
        for (uint32_t t = k; t < m && keys[t] == key; ++t) {
            const vx_contact& c = cs[vals[t]];
            if (!set || c.normalImpulse > e.impulse) {
                set = true;
                e.impulse = c.normalImpulse;
                e.point = c.point;
                // narrow-phase normals point from b towards a; events from lo towards hi
                const float sgn = c.a == lo ? -1.0f : 1.0f;
                e.normal = vx_vec3{c.normal.x * sgn, c.normal.y * sgn, c.normal.z * sgn};
            }
        }
        if (events) events[rank[k]] = e;
        pairsOut[rank[k]] = key;
    }
}

// Pairs of the previous step (src/world.cpp:4458-4482), in their order: a
// pair found among this step's pair keys is skipped; otherwise Persist when
// both bodies are static or asleep (the pair is appended to the pair keys),
// else End. The reference looks pairs up with std::binary_search in a key
// array it appends to as it goes, so after the first appended pair the array
// is no longer sorted and the lookup can miss a pair that is present (which
// then ends although active). This walk keeps that behaviour: one thread, the
// same lower-bound bisection over the same growing array.
VXD bool bisectFind(const uint64_t* keys, uint32_t count, uint64_t key) {
    uint32_t first = 0, len = count;
    while (len > 0) {
        const uint32_t half = len >> 1, middle = first + half;
        if (keys[middle] < key) {
            first = middle + 1;
            len = len - half - 1;
        } else {
            len = half;
        }
    }
    return first != count && !(key < keys[first]);
}

__global__ void endedWalkKernel(const uint64_t* prevPairs, uint32_t prevPairCount, const uint32_t* activeCount,
                                uint32_t n, BodyArrays B, const vx_contact* prevContacts, const uint64_t* prevKeys,
                                uint32_t prevCount, vxb_contact_event* events, uint64_t* pairs, uint32_t* counts) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const uint32_t active = *activeCount;
    uint32_t size = active, emitted = 0;
    for (uint32_t k = 0; k < prevPairCount; ++k) {
        const uint64_t key = prevPairs[k];
        if (bisectFind(pairs, size, key)) continue;
        const uint32_t lo = (uint32_t)(key >> 32), hi = (uint32_t)key;
        if (lo >= n || hi >= n) continue;
        const uint32_t fl = B.filt[lo].x, fh = B.filt[hi].x;
        const bool resting = (isStaticBody(fl) || isAsleep(fl)) && (isStaticBody(fh) || isAsleep(fh));
        if (events) {
            vxb_contact_event e;
            memset(&e, 0, sizeof(e));
            e.a = lo;
            e.b = hi;
            e.sensor = (isSensor(fl) || isSensor(fh)) ? 1u : 0u;
            e.type = resting ? 1u : 2u;
            if (resting) {
                // the pair's first cached contact: raw keys (lo, hi) sort before (hi, lo)
                uint32_t t = lowerBound(prevKeys, prevCount, key);
                if (!(t < prevCount && prevKeys[t] == key))
                    t = lowerBound(prevKeys, prevCount, ((uint64_t)hi << 32) | lo);
                if (t < prevCount && canonicalKey(prevContacts[t].a, prevContacts[t].b) == key) {
                    const vx_contact& c = prevContacts[t];
                    e.point = c.point;
                    const float sgn = c.a == lo ? -1.0f : 1.0f;
                    e.normal = vx_vec3{c.normal.x * sgn, c.normal.y * sgn, c.normal.z * sgn};
                    e.impulse = c.normalImpulse;
                }
            }
            events[active + emitted] = e;
        }
        ++emitted;
        if (resting) pairs[size++] = key;
    }
    counts[0] = emitted;
    counts[1] = size - active;
}

__global__ void iotaU32Kernel(uint32_t* a, uint32_t n) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) a[k] = k;
}

// First of each run of equal keys, ignoring the sentinel tail.
__global__ void uniqueFlagKernel(const uint64_t* keys, uint32_t n, uint64_t sentinel, uint32_t* flags) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        flags[k] = keys[k] != sentinel && (k == 0 || keys[k - 1] != keys[k]) ? 1u : 0u;
}

__global__ void compactKeysKernel(const uint64_t* keys, const uint32_t* flags, const uint32_t* rank, uint32_t n,
                                  uint64_t* out) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        if (flags[k]) out[rank[k]] = keys[k];
}

__global__ void canonicalKeysKernel(const vx_contact* cs, uint32_t m, uint64_t* keys, uint32_t* vals) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
        keys[k] = canonicalKey(cs[k].a, cs[k].b);
        vals[k] = k;
    }
}

// Cached contacts that stay for warm starting (src/world.cpp:4496-4516): the
// pair is a pair key of this step, both bodies are static or asleep (after
// this step's sleeping), and the pair has no contact this step.
__global__ void keptFlagKernel(const vx_contact* prev, uint32_t prevCount, BodyArrays B, const uint64_t* pairs,
                               uint32_t pairCount, const uint64_t* current, uint32_t currentCount, uint32_t* flags,
                               uint32_t* tapeFlags, const uint32_t* worldOf) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < prevCount; k += gridDim.x * blockDim.x) {
        const vx_contact& c = prev[k];
        const uint64_t key = canonicalKey(c.a, c.b);
        const uint32_t fa = B.filt[c.a].x, fb = B.filt[c.b].x;
        const bool keep = inSorted(pairs, pairCount, key) && (isStaticBody(fa) || isAsleep(fa)) &&
                          (isStaticBody(fb) || isAsleep(fb)) && !inSorted(current, currentCount, key);
        flags[k] = keep ? 1u : 0u;
        if (keep) markWorld(tapeFlags, worldOf, isStaticBody(fa) ? c.b : c.a);
    }
}

__global__ void gatherKeptKernel(const vx_contact* prev, const uint32_t* flags, const uint32_t* rank,
                                 uint32_t prevCount, vx_contact* out) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < prevCount; k += gridDim.x * blockDim.x)
        if (flags[k]) out[rank[k]] = prev[k];
}

// Merge of this step's contacts (in pair order) and the kept ones: sort keys
// (raw (a, b), disjoint pair sets) with the record index, then gather.
__global__ void mergeKeysKernel(const vx_contact* cur, uint32_t m, const vx_contact* kept, uint32_t kc,
                                uint64_t* keys, uint32_t* vals) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m + kc; k += gridDim.x * blockDim.x) {
        const vx_contact& c = k < m ? cur[k] : kept[k - m];
        keys[k] = ((uint64_t)c.a << 32) | c.b;
        vals[k] = k;
    }
}

__global__ void mergeGatherKernel(const vx_contact* cur, uint32_t m, const vx_contact* kept, const uint32_t* vals,
                                  uint32_t total, vx_contact* out, uint32_t* stepPos) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < total; k += gridDim.x * blockDim.x) {
        const uint32_t v = vals[k];
        out[k] = v < m ? cur[v] : kept[v - m];
        if (v < m) stepPos[v] = k;
    }
}

__global__ void gatherStepContactsKernel(const vx_contact* cache, const uint32_t* stepPos, uint32_t m,
                                         vx_contact* out) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x)
        out[k] = cache[stepPos[k]];
}

}  // namespace

// ---- host side -------------------------------------------------------------------

void sleepConfigDefault(vxb_sleep_config* c) {
    std::memset(c, 0, sizeof(*c));
    c->linearVelocityThreshold = 0.05f;
    c->angularVelocityThreshold = 0.05f;
    c->accelerationThreshold = 0.01f;
    c->timeToSleep = 0.5f;
    c->timeToDrowsy = 0.25f;
    c->contactStabilityThreshold = 0.02f;
    c->contactStabilityFrames = 10;
    c->enableGradualSleep = 1;
    c->enableContactStability = 1;
}

int sleepLoad(Context& c, const vx_body* host, uint32_t n) {
    SleepState& S = c.sleep;
    S.sleepable = S.asleep = 0;
    std::vector<float4> state(n);
    for (uint32_t i = 0; i < n; ++i) {
        const vx_body& b = host[i];
        const bool dynamic = b.motionType == VX_MOTION_DYNAMIC;
        if (dynamic && b.enableSleep) ++S.sleepable;
        if (dynamic && b.asleep == 1) ++S.asleep;
        const float st = b.asleep == 1 ? kAsleep : b.asleep == 2 ? kDrowsy : kAwake;
        state[i] = make_float4(b.sleepTimer, 0.0f, st, b.enableSleep ? 1.0f : 0.0f);
    }
    SL_TRY(ensure(c, S.state, (size_t)n * 16 + 16));
    SL_CUDA(c, cudaMemcpyAsync(S.state.ptr, state.data(), (size_t)n * 16, cudaMemcpyHostToDevice, c.stream));
    SL_CUDA(c, cudaStreamSynchronize(c.stream));  // `state` is freed on return
    S.pairCount = 0;
    S.eventCount = 0;
    return VXB_OK;
}

int sleepExport(Context& c, vx_body* aosDevice) {
    if (!c.sleep.state.ptr) return VXB_OK;
    SL_LAUNCH(c, sleepExportKernel, gridFor(c.n, 256), 256, aosDevice, c.n, PT<float4>(c.sleep.state));
    return VXB_OK;
}

bool sleepActive(const Context& c) { return c.sleep.sleepable > 0 || c.sleep.asleep > 0; }

static uint32_t* tapeFlagsOf(Context& c) {
    return c.tape.active && c.tape.recorded < c.tape.steps ? PT<uint32_t>(c.tape.flags) : nullptr;
}

int wakePass(Context& c, const vx_contact* cs, uint32_t m) {
    SleepState& S = c.sleep;
    if (S.asleep == 0 || m == 0) return VXB_OK;
    SL_TRY(ensure(c, S.flags, (size_t)m * 4 + 64));
    SL_TRY(ensure(c, S.ranks, (size_t)m * 4 + 64));
    SL_TRY(ensure(c, S.list, (size_t)m * 4 + 64));
    SL_TRY(ensure(c, S.small, 256));
    uint32_t* small = PT<uint32_t>(S.small);  // [8] starters, [9] listed contacts
    SL_CUDA(c, cudaMemsetAsync(small + 8, 0, 8, c.stream));
    SL_LAUNCH(c, wakeScanKernel, gridFor(m, 256), 256, cs, m, c.B, PT<uint32_t>(S.flags), small + 8);
    SL_TRY(exclusiveScan(c, PT<uint32_t>(S.flags), PT<uint32_t>(S.ranks), m, small + 9));
    SL_LAUNCH(c, listKernel, gridFor(m, 256), 256, PT<uint32_t>(S.flags), PT<uint32_t>(S.ranks), m,
              PT<uint32_t>(S.list));
    SL_LAUNCH(c, wakeWalkKernel, 1, 32, cs, PT<uint32_t>(S.list), small + 9, small + 8, c.B, PT<float4>(S.state),
              tapeFlagsOf(c), PT<uint32_t>(c.worldOfBuf));
    return VXB_OK;
}

int sleepAndEvents(Context& c, const vx_contact* cs, uint32_t m, float dt, uint32_t* keptOut) {
    SleepState& S = c.sleep;
    *keptOut = 0;
    const bool sleeping = sleepActive(c);
    if (!sleeping && !S.events) return VXB_OK;
    const uint32_t n = c.n;
    const vx_contact* prevContacts = PT<vx_contact>(c.contactBuf[c.cur ^ 1]);
    const uint64_t* prevKeys = PT<uint64_t>(c.prevKeyBuf);
    const uint32_t prevCount = c.prevCount, prevPairCount = S.pairCount;
    const uint64_t sentinel = (uint64_t)n << 32;  // above every pair key
    const int bits = keyBits(sentinel);
    const size_t cap = (size_t)m + prevPairCount + prevCount + 64;
    SL_TRY(ensure(c, S.small, 256));
    SL_TRY(ensure(c, S.keys, cap * 8));
    SL_TRY(ensure(c, S.vals, cap * 4));
    SL_TRY(ensure(c, S.flags, cap * 4));
    SL_TRY(ensure(c, S.ranks, cap * 4));
    SL_TRY(ensure(c, S.pairsNext, cap * 8));
    if (S.events) SL_TRY(ensure(c, S.eventBuf, cap * sizeof(vxb_contact_event)));
    uint32_t* small = PT<uint32_t>(S.small);  // [0] active pairs, [2] pair keys, [3] asleep, [4] kept,
                                              // [5] other events, [6] resting pairs appended
    uint64_t* keys = PT<uint64_t>(S.keys);
    uint32_t* vals = PT<uint32_t>(S.vals);
    uint32_t* flags = PT<uint32_t>(S.flags);
    uint32_t* ranks = PT<uint32_t>(S.ranks);
    uint64_t* pairsNext = PT<uint64_t>(S.pairsNext);
    const uint64_t* prevPairs = PT<uint64_t>(S.pairs);
    vxb_contact_event* events = S.events ? PT<vxb_contact_event>(S.eventBuf) : nullptr;
    SL_CUDA(c, cudaMemsetAsync(small, 0, 32, c.stream));
    // ---- events (src/world.cpp:4398-4488), with the pre-sleep states
    if (m) {
        SL_LAUNCH(c, activeKeysKernel, gridFor(m, 256), 256, cs, m, c.B, dt, sentinel, keys, vals);
        SL_TRY(sortPairs(c, keys, vals, m, bits));
        SL_LAUNCH(c, headFlagKernel, gridFor(m, 256), 256, keys, m, sentinel, flags);
        SL_TRY(exclusiveScan(c, flags, ranks, m, small + 0));
        SL_LAUNCH(c, activeEventsKernel, gridFor(m, 256), 256, keys, vals, m, sentinel, ranks, cs, c.B, prevPairs,
                  prevPairCount, events, pairsNext);
    }
    if (prevPairCount)
        SL_LAUNCH(c, endedWalkKernel, 1, 32, prevPairs, prevPairCount, small, n, c.B, prevContacts, prevKeys,
                  prevCount, events, pairsNext, small + 5);
    uint32_t host[8];
    SL_CUDA(c, cudaMemcpyAsync(host, small, 32, cudaMemcpyDeviceToHost, c.stream));
    ++c.hostSyncs;
    SL_CUDA(c, cudaStreamSynchronize(c.stream));
    const uint32_t total = host[0] + host[6];  // active pairs and the resting pairs appended
    S.eventCount = S.events ? host[0] + host[5] : 0;
    // ---- this step's pair keys: active pairs and resting ones, sorted and unique
    uint32_t pairCount = 0;
    if (total) {
        SL_LAUNCH(c, iotaU32Kernel, gridFor(total, 256), 256, vals, total);
        SL_TRY(sortPairs(c, pairsNext, vals, total, bits));
        SL_LAUNCH(c, uniqueFlagKernel, gridFor(total, 256), 256, pairsNext, total, sentinel, flags);
        SL_TRY(exclusiveScan(c, flags, ranks, total, small + 2));
        // every kernel reading the previous pair keys is queued before this point
        SL_TRY(ensure(c, S.pairs, (size_t)total * 8 + 64));
        SL_LAUNCH(c, compactKeysKernel, gridFor(total, 256), 256, pairsNext, flags, ranks, total,
                  PT<uint64_t>(S.pairs));
        SL_CUDA(c, cudaMemcpyAsync(host + 2, small + 2, 4, cudaMemcpyDeviceToHost, c.stream));
        ++c.hostSyncs;
        SL_CUDA(c, cudaStreamSynchronize(c.stream));
        pairCount = host[2];
    }
    S.pairCount = pairCount;
    if (!sleeping) return VXB_OK;
    // ---- sleeping (src/sleep.cpp:52-237)
    uint32_t* tapeFlags = tapeFlagsOf(c);
    SL_TRY(ensure(c, S.parent, (size_t)n * 4 + 64));
    SL_TRY(ensure(c, S.bodyBits, (size_t)n * 8 + 64));
    uint32_t* parent = PT<uint32_t>(S.parent);
    uint32_t* bodyBits = PT<uint32_t>(S.bodyBits);
    uint32_t* islandTimer = bodyBits + n + 8;
    SL_TRY(unionRoots(c, cs, m, parent));
    SL_CUDA(c, cudaMemsetAsync(bodyBits, 0, (size_t)n * 4, c.stream));
    SL_CUDA(c, cudaMemsetAsync(islandTimer, 0x7f, (size_t)n * 4, c.stream));  // 3.4e38: above any timer
    if (m && S.config.enableContactStability)
        SL_LAUNCH(c, stabilityKernel, gridFor(m, 256), 256, cs, m, c.B, S.config.contactStabilityThreshold, bodyBits);
    SL_LAUNCH(c, sleepTimerKernel, gridFor(n, 256), 256, c.B, n, bodyBits, S.config, dt, PT<float4>(S.state), parent,
              islandTimer);
    SL_LAUNCH(c, sleepTransitionKernel, gridFor(n, 256), 256, c.B, n, S.config, PT<float4>(S.state), parent,
              islandTimer, small + 3, tapeFlags, PT<uint32_t>(c.worldOfBuf));
    // ---- cached contacts of resting pairs (src/world.cpp:4496-4521), with the post-sleep states
    if (prevCount && pairCount) {
        if (m) {
            SL_LAUNCH(c, canonicalKeysKernel, gridFor(m, 256), 256, cs, m, keys, vals);
            SL_TRY(sortPairs(c, keys, vals, m, bits));
        }
        SL_LAUNCH(c, keptFlagKernel, gridFor(prevCount, 256), 256, prevContacts, prevCount, c.B,
                  PT<uint64_t>(S.pairs), pairCount, keys, m, flags, tapeFlags, PT<uint32_t>(c.worldOfBuf));
        SL_TRY(exclusiveScan(c, flags, ranks, prevCount, small + 4));
        SL_TRY(ensure(c, S.kept, (size_t)prevCount * sizeof(vx_contact) + 128));
        SL_LAUNCH(c, gatherKeptKernel, gridFor(prevCount, 256), 256, prevContacts, flags, ranks, prevCount,
                  PT<vx_contact>(S.kept));
    }
    SL_CUDA(c, cudaMemcpyAsync(host + 3, small + 3, 8, cudaMemcpyDeviceToHost, c.stream));
    ++c.hostSyncs;
    SL_CUDA(c, cudaStreamSynchronize(c.stream));
    S.asleep = host[3];
    *keptOut = prevCount && pairCount ? host[4] : 0;
    return VXB_OK;
}

int mergeKeptContacts(Context& c, uint32_t m, uint32_t kept) {
    SleepState& S = c.sleep;
    const uint32_t total = m + kept;
    SL_TRY(ensure(c, S.keys, (size_t)total * 8 + 64));
    SL_TRY(ensure(c, S.vals, (size_t)total * 4 + 64));
    SL_TRY(ensure(c, S.merge, (size_t)total * sizeof(vx_contact) + 128));
    SL_TRY(ensure(c, c.stepPosBuf, (size_t)m * 4 + 64));
    const vx_contact* cur = PT<vx_contact>(c.contactBuf[c.cur]);
    SL_LAUNCH(c, mergeKeysKernel, gridFor(total, 256), 256, cur, m, PT<vx_contact>(S.kept), kept, PT<uint64_t>(S.keys),
              PT<uint32_t>(S.vals));
    SL_TRY(sortPairs(c, PT<uint64_t>(S.keys), PT<uint32_t>(S.vals), total, keyBits((uint64_t)c.n << 32)));
    SL_LAUNCH(c, mergeGatherKernel, gridFor(total, 256), 256, cur, m, PT<vx_contact>(S.kept), PT<uint32_t>(S.vals),
              total, PT<vx_contact>(S.merge), PT<uint32_t>(c.stepPosBuf));
    std::swap(c.contactBuf[c.cur], S.merge);
    return VXB_OK;
}

int readStepContacts(Context& c, vx_contact* out, uint32_t m) {
    SL_TRY(ensure(c, c.sleep.merge, (size_t)m * sizeof(vx_contact) + 128));
    SL_LAUNCH(c, gatherStepContactsKernel, gridFor(m, 256), 256, PT<vx_contact>(c.contactBuf[c.cur ^ 1]),
              PT<uint32_t>(c.stepPosBuf), m, PT<vx_contact>(c.sleep.merge));
    SL_CUDA(c, cudaMemcpyAsync(out, c.sleep.merge.ptr, (size_t)m * sizeof(vx_contact), cudaMemcpyDeviceToHost,
                               c.stream));
    SL_CUDA(c, cudaStreamSynchronize(c.stream));
    return VXB_OK;
}

int readEvents(Context& c, vxb_contact_event* out, uint32_t cap, uint32_t* count) {
    const uint32_t k = c.sleep.eventCount;
    if (count) *count = k;
    if (out && k) {
        SL_CUDA(c, cudaMemcpyAsync(out, c.sleep.eventBuf.ptr, (size_t)std::min(k, cap) * sizeof(vxb_contact_event),
                                   cudaMemcpyDeviceToHost, c.stream));
        SL_CUDA(c, cudaStreamSynchronize(c.stream));
    }
    return VXB_OK;
}

}  // namespace vxb
