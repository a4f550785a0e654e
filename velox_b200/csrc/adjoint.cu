// Reverse mode of the device world's step: the adjoint of the substep loop.
//
// The reference engine has no adjoint; this differentiates its step as the
// device world runs it (src/world.cpp:4007-4397 with the CUDA backend's
// coloured solve, src/backend_cuda.cu:569-761): orientation normalisation and
// first-substep gravity, per substep the velocity integration
// (backend_cuda.cu:80-89), the warm start (src/narrowphase.h:80-124), the
// colour-major sweeps of solveContact (narrowphase.h:130-366), the transform
// integration (include/velox/body.h:266-321), and the split-impulse position
// correction (world.cpp:4370-4397).
//
// Frozen from the forward pass (recorded while a tape is active): each
// step's contacts after warm-start matching (normal, anchors, bias0,
// coefficients, the inherited impulses, vn0), their colours, the previous
// step's contact each one inherited its impulses and its restitution
// reference from, and the branch of every clamp, friction ellipse and
// position-correction test. Body states are checkpointed every k steps; the
// backward pass recomputes each segment from its checkpoint with the
// pipeline's own row functions (prepRow / warmPrepRow / sweepRow, so the
// recomputed trajectory equals the forward bit for bit), records every row
// update's inputs, and runs the hand-derived reverse of each operation.
// Gradients flow through body poses and velocities, impulses carried between
// steps by warm starting, and approach speeds (vn0) carried by the matching.
//
// Scope of the reverse: two-axis friction, isotropic inverse inertia, zero
// rolling and spinning friction. A world outside it, or one whose recomputed
// trajectory leaves the forward's (a conservative-advancement rewind), is
// reported in its flags and its gradients are not meaningful.
//
// Layout: one warp per world. Rows of one colour share no dynamic body, so a
// colour's rows run on the warp's lanes in parallel, in both directions.
#include <algorithm>
#include <cstring>

#include "context.cuh"

namespace vxb {

namespace {

#define AD_TRY(expr)                   \
    do {                               \
        int s_ = (expr);               \
        if (s_ != VXB_OK) return s_;   \
    } while (0)

#define AD_CUDA(c, expr)                                              \
    do {                                                              \
        cudaError_t e_ = (expr);                                      \
        if (e_ != cudaSuccess) return cudaStatus((c), e_, #expr);     \
    } while (0)

#define AD_LAUNCH(c, kernel, grid, block, ...)                               \
    do {                                                                     \
        kernel<<<(grid), (block), 0, (c).stream>>>(__VA_ARGS__);            \
        ++(c).launches;                                                      \
    } while (0)

template <class T> T* PT(DevBuf& b) { return reinterpret_cast<T*>(b.ptr); }

constexpr uint32_t kNone = 0xffffffffu;
// Row branch bits as the backward reports them (the FP64 restatement's
// numbering): restitution condition, restitution target taken, normal impulse
// unclamped, friction rows present, each friction axis bounded, ellipse
// projection; kBrSkip for a row without normal mass.
constexpr uint32_t kBrRestitution = 1, kBrResMax = 2, kBrClamp = 4, kBrFriction = 8, kBrM1 = 16, kBrM2 = 32,
                   kBrEllipse = 64, kBrSkip = 128;
constexpr uint32_t kNoColour = 0x7fffffffu;

inline uint32_t gridFor(uint64_t items, int threads) {
    uint64_t b = (items + threads - 1) / threads;
    return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(b, 65535u * 16u));
}

// Grow-only allocation that keeps the first `keep` bytes.
int growKeep(Context& c, DevBuf& b, size_t bytes, size_t keep) {
    if (bytes <= b.bytes && b.ptr) return VXB_OK;
    void* fresh = nullptr;
    const size_t want = std::max(bytes, b.bytes * 2) + 256;
    cudaError_t e = cudaMalloc(&fresh, want);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return cudaStatus(c, e, "cudaMalloc (tape)");
    }
    if (b.ptr && keep) AD_CUDA(c, cudaMemcpyAsync(fresh, b.ptr, keep, cudaMemcpyDeviceToDevice, c.stream));
    if (b.ptr) {
        AD_CUDA(c, cudaStreamSynchronize(c.stream));
        cudaFree(b.ptr);
    }
    b.ptr = fresh;
    b.bytes = want;
    return VXB_OK;
}

// ---- recording kernels ------------------------------------------------------

// The previous-step contact each contact inherits its impulses from and the
// one it takes its restitution reference (vn0) from: matchKernel's choices
// (src/world.cpp:4133-4184), made on the unmatched contacts.
__global__ void matchSourceKernel(const vx_contact* cur, uint32_t m, const vx_contact* prev, const uint64_t* prevKeys,
                                  uint32_t mPrev, uint2* src) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
        const vx_contact& c = cur[k];
        const uint64_t key = ((uint64_t)c.a << 32) | c.b;
        uint32_t lo = 0, hi = mPrev;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (prevKeys[mid] < key) lo = mid + 1;
            else hi = mid;
        }
        uint32_t impulseFrom = kNone, vn0From = kNone;
        float vn0 = c.vn0;
        bool matched = false;
        if (c.featureKey != 0) {
            for (uint32_t it = lo; it < mPrev && prevKeys[it] == key; ++it)
                if (prev[it].featureKey == c.featureKey) {
                    impulseFrom = it;
                    if (vn0 < -1.0f && prev[it].vn0 < vn0) vn0From = it;
                    matched = true;
                    break;
                }
        }
        if (!matched) {
            if (vn0 < -1.0f)
                for (uint32_t it = lo; it < mPrev && prevKeys[it] == key; ++it)
                    if (prev[it].vn0 < vn0) { vn0 = prev[it].vn0; vn0From = it; }
            float best = 2.5e-3f;
            for (uint32_t it = lo; it < mPrev && prevKeys[it] == key; ++it) {
                const vx_contact& p = prev[it];
                const V3 d{p.point.x - c.point.x, p.point.y - c.point.y, p.point.z - c.point.z};
                const float ds = lengthSq(d);
                if (ds < best) { best = ds; impulseFrom = it; }
            }
        }
        src[k] = make_uint2(impulseFrom, vn0From);
    }
}

// First contact of each world (contacts are sorted by a; worlds are contiguous
// body ranges), worlds + 1 entries.
__global__ void worldStartKernel(const vx_contact* cs, uint32_t m, const uint32_t* worldOf, uint32_t worlds,
                                 uint32_t* out) {
    for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w <= worlds; w += gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = m;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (worldOf[cs[mid].a] < w) lo = mid + 1;
            else hi = mid;
        }
        out[w] = lo;
    }
}

__global__ void checkpointKernel(BodyArrays B, uint32_t n, float4* out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        out[i] = B.pos[i];
        out[n + i] = B.rot[i];
        out[2 * n + i] = B.vel[i];
        out[3 * n + i] = B.ang[i];
    }
}

__global__ void rewoundWorldsKernel(const uint32_t* rewound, uint32_t n, const uint32_t* worldOf, uint32_t* flags) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (rewound[i]) atomicOr(flags + worldOf[i], (uint32_t)VXB_ADJ_REWOUND);
}

// Largest colour (solved rows) and largest per-world row count of the tape.
__global__ void tapeExtentKernel(const uint32_t* color, uint32_t total, const uint32_t* worldStart, uint32_t steps,
                                 uint32_t worlds, uint32_t* out) {
    uint32_t mc = 0, mr = 0;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < total; k += gridDim.x * blockDim.x)
        if (color[k] < kNoColour) mc = max(mc, color[k]);
    const uint64_t cells = (uint64_t)steps * worlds;
    for (uint64_t k = blockIdx.x * blockDim.x + threadIdx.x; k < cells; k += gridDim.x * blockDim.x) {
        const uint64_t t = k / worlds, w = k % worlds;
        const uint32_t* ws = worldStart + t * (worlds + 1);
        mr = max(mr, ws[w + 1] - ws[w]);
    }
    atomicMax(out, mc);
    atomicMax(out + 1, mr);
}

// Worlds whose bodies or contacts are outside the reverse's scope.
__global__ void scopeKernel(BodyArrays B, uint32_t n, const uint32_t* worldOf, const vx_contact* cs, uint32_t total,
                            uint32_t* flags) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 in = B.inertia[i];
        const uint32_t f = B.filt[i].x;
        if (isDynamic(f) && !isRotationLocked(f) && (in.x != in.y || in.y != in.z))
            atomicOr(flags + worldOf[i], (uint32_t)VXB_ADJ_UNSUPPORTED);
    }
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < total; k += gridDim.x * blockDim.x)
        if (cs[k].rollingFriction > 0.0f || cs[k].spinningFriction > 0.0f)
            atomicOr(flags + worldOf[cs[k].a], (uint32_t)VXB_ADJ_UNSUPPORTED);
}

// ---- reverse-mode helpers (plain arithmetic; isotropic inverse inertia) -------

VXD V3 xc(const V3& a, const V3& b) { return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
VXD void accs(V3& a, const V3& b, float s) { a.x += b.x * s; a.y += b.y * s; a.z += b.z * s; }

// reverse of rotate(q, v) w.r.t. q (rotate = v + 2 qv x (qv x v + w v))
VXD void rotateRevQ(const Q4& q, const V3& v, const V3& ob, Q4& qb) {
    const V3 qv{q.x, q.y, q.z};
    const V3 u = xc(qv, v) + v * q.w;
    const V3 tb = ob * 2.0f;
    V3 qvb = xc(u, tb);
    const V3 ub = xc(tb, qv);
    qvb += xc(v, ub);
    qb.w += dot(ub, v);
    qb.x += qvb.x; qb.y += qvb.y; qb.z += qvb.z;
}

// reverse of q / |q|
VXD Q4 qnormalizeRev(const Q4& q, const Q4& ob) {
    const float len = sqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
    const Q4 n{q.x / len, q.y / len, q.z / len, q.w / len};
    const float d = n.x * ob.x + n.y * ob.y + n.z * ob.z + n.w * ob.w;
    return Q4{(ob.x - n.x * d) / len, (ob.y - n.y * d) / len, (ob.z - n.z * d) / len, (ob.w - n.w * d) / len};
}

// reverse of qintegrate(q, w, h) = normalize(q + (w h/2, 0) (x) q); qb in: after, out: before
VXD void qintegrateRev(const Q4& q, const V3& w, float h, Q4& qb, V3& wb) {
    const float ax = w.x * 0.5f * h, ay = w.y * 0.5f * h, az = w.z * 0.5f * h;
    const Q4 raw{q.x + (ax * q.w + ay * q.z - az * q.y), q.y + (-ax * q.z + ay * q.w + az * q.x),
                 q.z + (ax * q.y - ay * q.x + az * q.w), q.w + (-ax * q.x - ay * q.y - az * q.z)};
    const Q4 rb = qnormalizeRev(raw, qb);
    const float axb = rb.x * q.w - rb.y * q.z + rb.z * q.y - rb.w * q.x;
    const float ayb = rb.x * q.z + rb.y * q.w - rb.z * q.x - rb.w * q.y;
    const float azb = -rb.x * q.y + rb.y * q.x + rb.z * q.w - rb.w * q.z;
    Q4 out = rb;
    out.w += rb.x * ax + rb.y * ay + rb.z * az;
    out.z += rb.x * ay - rb.y * ax - rb.w * az;
    out.y += -rb.x * az + rb.z * ax - rb.w * ay;
    out.x += rb.y * az - rb.z * ay - rb.w * ax;
    qb = out;
    wb.x += axb * 0.5f * h; wb.y += ayb * 0.5f * h; wb.z += azb * 0.5f * h;
}

// Adjoints of one row's pose terms (RowPrep) within a substep.
struct PrepBar {
    V3 ra, rb, raxn, rbxn, raxt1, rbxt1, raxt2, rbxt2;
    float kN, k1, k2, target0;
};

// Per-body adjoint state.
struct BodyBar {
    float4 p, q, v, w;
};

// ---- per-world scratch ----------------------------------------------------------

struct AdjArgs {
    BodyArrays B;
    const float4* ckpt;            // (J + 1) x 4 x n
    uint32_t n, worlds, steps, every, J;
    const uint32_t* bodyStart;     // worlds + 1
    const vx_contact* contacts;    // all recorded steps
    const uint32_t* stepStart;     // steps + 1
    const uint2* src;              // per contact
    const uint32_t* color;         // per contact
    const uint32_t* worldStart;    // steps x (worlds + 1), indices within a step
    V3 gravity;
    float h;
    int substeps, sweeps, posIters;
    int stackStab;
    float stackStiffness, stackDamping;
    uint32_t NB, MR, MC;           // per-world limits of this tape
    const float* seed;             // n x 13
    float* grad;                   // n x 13
    float* gradInv;                // n x 2 (invMass, isotropic invInertia)
    float* gradMass;               // n
    uint32_t* flags;               // worlds
    uint8_t* branches;             // optional: branch decisions, worlds x steps x branchStep
    size_t branchStep;             // (S + 1 + S*W + PI) * MR bytes per world and step
    char* scratch;
    size_t worldBytes;
    // offsets inside a world's slice
    size_t oSt, oSub, oEnd, oCorr, oRin, oPush, oLam, oLamInit, oPrep, oPbar, oOrder, oCstart, oLamb0, oLamb1,
        oCur, oAdj, oGm;
};

struct WorldView {
    float4* st;      // every x 4 x NB (p, q, v, w) step-start states of a segment
    float4* sub;     // S x 4 x NB
    float4* endv;    // S x 2 x NB (v, w)
    float4* corr;    // 4 x NB
    float4* rin;     // S x W x MR x 4 (va|ln, wa|l1, vb|l2, wb)
    float* push;     // PI x MR
    float4* lam;     // MR current impulses (n, t1, t2, -)
    float4* lamInit; // MR
    RowPrep* prep;   // MR
    PrepBar* pbar;   // MR
    uint32_t* order; // MR colour-major world-local row order
    uint32_t* cstart;// MC + 4
    float4* lamb[2]; // MR adjoints (n, t1, t2, vn0), current / previous step
    float4* cur;     // 4 x NB current state
    BodyBar* adj;    // NB
    float2* gm;      // NB (invMass, invI) adjoints
};

VXD WorldView carve(const AdjArgs& A, uint32_t w) {
    char* base = A.scratch + (size_t)w * A.worldBytes;
    WorldView V;
    V.st = reinterpret_cast<float4*>(base + A.oSt);
    V.sub = reinterpret_cast<float4*>(base + A.oSub);
    V.endv = reinterpret_cast<float4*>(base + A.oEnd);
    V.corr = reinterpret_cast<float4*>(base + A.oCorr);
    V.rin = reinterpret_cast<float4*>(base + A.oRin);
    V.push = reinterpret_cast<float*>(base + A.oPush);
    V.lam = reinterpret_cast<float4*>(base + A.oLam);
    V.lamInit = reinterpret_cast<float4*>(base + A.oLamInit);
    V.prep = reinterpret_cast<RowPrep*>(base + A.oPrep);
    V.pbar = reinterpret_cast<PrepBar*>(base + A.oPbar);
    V.order = reinterpret_cast<uint32_t*>(base + A.oOrder);
    V.cstart = reinterpret_cast<uint32_t*>(base + A.oCstart);
    V.lamb[0] = reinterpret_cast<float4*>(base + A.oLamb0);
    V.lamb[1] = reinterpret_cast<float4*>(base + A.oLamb1);
    V.cur = reinterpret_cast<float4*>(base + A.oCur);
    V.adj = reinterpret_cast<BodyBar*>(base + A.oAdj);
    V.gm = reinterpret_cast<float2*>(base + A.oGm);
    return V;
}

// One world inside the kernel.
struct WorldRun {
    const AdjArgs& A;
    WorldView V;
    uint32_t w, b0, nb, lane;
    int colours = 0;

    VXD WorldRun(const AdjArgs& a, uint32_t world) : A(a), w(world) {
        V = carve(A, w);
        b0 = A.bodyStart[w];
        nb = A.bodyStart[w + 1] - b0;
        lane = threadIdx.x & 31u;
    }

    // state array s (4 x NB float4: p, q, v, w)
    VXD float4* P(float4* s) const { return s; }
    VXD float4* Q(float4* s) const { return s + A.NB; }
    VXD float4* Vv(float4* s) const { return s + 2 * A.NB; }
    VXD float4* Wv(float4* s) const { return s + 3 * A.NB; }

    VXD Mass mass(uint32_t li) const {
        const uint32_t i = b0 + li;
        const float4 in = A.B.inertia[i];
        Mass m;
        m.invI = V3{in.x, in.y, in.z};
        m.invMass = in.w;
        m.iq = q4(A.B.iq[i]);
        m.flags = A.B.filt[i].x;
        return m;
    }
    VXD SolverBody body(const float4* s, uint32_t li) const {
        SolverBody b;
        b.p = f3(s[li]);
        b.q = q4(s[A.NB + li]);
        b.v = f3(s[2 * A.NB + li]);
        b.w = f3(s[3 * A.NB + li]);
        b.m = mass(li);
        b.sphere = shapeOf(b.m.flags) == kSphere;
        cacheFrame(b);
        return b;
    }
    VXD void storeVel(float4* s, uint32_t li, const SolverBody& b) const {
        s[2 * A.NB + li] = pack(b.v, 0.0f);
        s[3 * A.NB + li] = pack(b.w, 0.0f);
    }
    VXD void copyState(float4* dst, const float4* from) const {
        for (uint32_t k = lane; k < 4 * A.NB; k += 32) dst[k] = from[k];
        __syncwarp();
    }

    // Branch decisions of step t (null unless requested): per substep the live
    // gap's sign, the warm start's activity, per substep and sweep the row bits,
    // per position pass the push's activity; MR entries each, world-local rows.
    VXD uint8_t* branchesOf(uint32_t t) const {
        return A.branches ? A.branches + ((size_t)w * A.steps + t) * A.branchStep : nullptr;
    }

    VXD uint32_t rowsOf(uint32_t t, uint32_t& c0) const {
        const uint32_t* ws = A.worldStart + (size_t)t * (A.worlds + 1);
        c0 = A.stepStart[t] + ws[w];
        return ws[w + 1] - ws[w];
    }

    // colour-major order of the world's rows of step t (lane 0 counting sort)
    VXD void buildOrder(uint32_t c0, uint32_t m) {
        if (lane == 0) {
            const uint32_t buckets = A.MC + 2;  // colours 0..MC, then the unsolved bucket
            for (uint32_t b = 0; b <= buckets; ++b) V.cstart[b] = 0;
            for (uint32_t j = 0; j < m; ++j) {
                uint32_t col = A.color[c0 + j];
                col = col < kNoColour ? col : A.MC + 1;
                ++V.cstart[col + 1];
            }
            for (uint32_t b = 0; b < buckets; ++b) V.cstart[b + 1] += V.cstart[b];
            for (uint32_t j = 0; j < m; ++j) {  // stable placement; cstart[b] ends at bucket b's end
                uint32_t col = A.color[c0 + j];
                col = col < kNoColour ? col : A.MC + 1;
                V.order[V.cstart[col]++] = j;
            }
            for (uint32_t b = buckets; b > 0; --b) V.cstart[b] = V.cstart[b - 1];
            V.cstart[0] = 0;
        }
        __syncwarp();
        colours = (int)A.MC + 2;
    }

    VXD bool solved(const vx_contact& cc) const {
        return !isSensor(A.B.filt[cc.a].x) && !isSensor(A.B.filt[cc.b].x);
    }

    // ---- forward ----------------------------------------------------------
    VXD void integrateVelocities(float4* s) {
        for (uint32_t li = lane; li < nb; li += 32) {
            const Mass m = mass(li);
            if (!isDynamic(m.flags) || isLocked(m.flags) || isAsleep(m.flags)) continue;
            const float4 ex = A.B.extra[b0 + li];
            V3 v = f3(Vv(s)[li]), wv = f3(Wv(s)[li]);
            const Q4 q = q4(Q(s)[li]);
            v += (A.gravity * ex.y + f3(A.B.force[b0 + li]) * solverInvMass(m)) * A.h;
            wv += invInertiaMulAt(m, f3(A.B.torque[b0 + li]), q) * A.h;
            v *= 1.0f / (1.0f + ex.z * A.h);
            wv *= 1.0f / (1.0f + ex.w * A.h);
            Vv(s)[li] = pack(v, 0.0f);
            Wv(s)[li] = pack(wv, 0.0f);
        }
        __syncwarp();
    }

    VXD void integrateTransforms(float4* s) {
        for (uint32_t li = lane; li < nb; li += 32) {
            const Mass m = mass(li);
            if (isStaticBody(m.flags) || isLocked(m.flags) || isAsleep(m.flags)) continue;
            V3 p = f3(P(s)[li]), wv = f3(Wv(s)[li]);
            Q4 q = q4(Q(s)[li]);
            advanceTransform(m, p, q, f3(Vv(s)[li]), wv, A.h);
            P(s)[li] = pack(p, 0.0f);
            Q(s)[li] = pack(q);
            Wv(s)[li] = pack(wv, 0.0f);
        }
        __syncwarp();
    }

    VXD void loadRowContact(const vx_contact& cc, const float4& lam, RowContact& r) const {
        r.normal = V3{cc.normal.x, cc.normal.y, cc.normal.z};
        r.point = V3{cc.point.x, cc.point.y, cc.point.z};
        r.la = V3{cc.localAnchorA.x, cc.localAnchorA.y, cc.localAnchorA.z};
        r.lb = V3{cc.localAnchorB.x, cc.localAnchorB.y, cc.localAnchorB.z};
        r.bias0 = cc.bias0; r.vn0 = cc.vn0; r.restitution = cc.restitution;
        r.friction1 = cc.friction1; r.friction2 = cc.friction2;
        r.nImp = lam.x; r.t1Imp = lam.y; r.t2Imp = lam.z;
        r.r1Imp = 0.0f; r.r2Imp = 0.0f; r.sImp = 0.0f;
        r.rolling = 0.0f; r.spinning = 0.0f;
    }

    // One step of the frozen-contact model on V.cur; with `tape`, records what
    // the reverse needs.
    VXD void forwardStep(uint32_t t, bool tape) {
        uint32_t c0;
        const uint32_t m = rowsOf(t, c0);
        const vx_contact* cs = A.contacts;
        buildOrder(c0, m);
        float4* s = V.cur;
        for (uint32_t li = lane; li < nb; li += 32) Q(s)[li] = pack(qnormalize(q4(Q(s)[li])));
        __syncwarp();
        integrateVelocities(s);
        for (uint32_t j = lane; j < m; j += 32) {
            const vx_contact& cc = cs[c0 + j];
            V.lam[j] = make_float4(cc.normalImpulse, cc.tangentImpulse1, cc.tangentImpulse2, 0.0f);
            V.lamInit[j] = V.lam[j];
        }
        __syncwarp();
        const int S = A.substeps, W = A.sweeps;
        for (int sub = 0; sub < S; ++sub) {
            if (sub > 0) integrateVelocities(s);
            if (tape) {
                float4* dst = V.sub + (size_t)sub * 4 * A.NB;
                for (uint32_t k = lane; k < 4 * A.NB; k += 32) dst[k] = s[k];
            }
            for (uint32_t j = lane; j < m; j += 32) {
                const vx_contact& cc = cs[c0 + j];
                const SolverBody a = body(s, cc.a - b0), b = body(s, cc.b - b0);
                RowContact r;
                loadRowContact(cc, V.lam[j], r);
                prepRow(a, b, r, A.h, false, V.prep[j]);
            }
            __syncwarp();
            for (int op = (sub == 0 ? 0 : 1); op <= W; ++op) {  // op 0: warm start, 1..W: sweeps
                const int sweep = op - 1;
                for (int col = 0; col < colours; ++col) {
                    const uint32_t r0 = V.cstart[col], r1 = V.cstart[col + 1];
                    for (uint32_t x = r0 + lane; x < r1; x += 32) {
                        const uint32_t j = V.order[x];
                        const vx_contact& cc = cs[c0 + j];
                        if (!solved(cc)) continue;
                        const uint32_t la = cc.a - b0, lb = cc.b - b0;
                        SolverBody a = body(s, la), b = body(s, lb);
                        RowContact r;
                        loadRowContact(cc, V.lam[j], r);
                        if (op == 0) {
                            warmPrepRow(a, b, r, V.prep[j]);
                        } else {
                            if (tape) {
                                float4* rec = V.rin + (((size_t)sub * W + sweep) * A.MR + j) * 4;
                                rec[0] = pack(a.v, r.nImp);
                                rec[1] = pack(a.w, r.t1Imp);
                                rec[2] = pack(b.v, r.t2Imp);
                                rec[3] = pack(b.w, 0.0f);
                            }
                            sweepRow(a, b, r, V.prep[j], false);
                        }
                        if (isDynamic(a.m.flags)) storeVel(s, la, a);
                        if (isDynamic(b.m.flags)) storeVel(s, lb, b);
                        V.lam[j] = make_float4(r.nImp, r.t1Imp, r.t2Imp, 0.0f);
                    }
                    __syncwarp();
                }
            }
            if (tape) {
                float4* dst = V.endv + (size_t)sub * 2 * A.NB;
                for (uint32_t k = lane; k < 2 * A.NB; k += 32) dst[k] = s[2 * A.NB + k];
            }
            __syncwarp();
            integrateTransforms(s);
        }
        if (tape) copyState(V.corr, s);
        for (int it = 0; it < A.posIters; ++it)
            for (int col = 0; col < colours; ++col) {
                const uint32_t r0 = V.cstart[col], r1 = V.cstart[col + 1];
                for (uint32_t x = r0 + lane; x < r1; x += 32) {
                    const uint32_t j = V.order[x];
                    float push = 0.0f;
                    const vx_contact& cc = cs[c0 + j];
                    if (solved(cc)) {
                        const uint32_t la = cc.a - b0, lb = cc.b - b0;
                        const Mass ma = mass(la), mb = mass(lb);
                        const float ima = solverInvMass(ma), imb = solverInvMass(mb);
                        const float sum = ima + imb;
                        if (sum > 0.0f) {
                            V3 pa = f3(P(s)[la]), pb = f3(P(s)[lb]);
                            const Q4 qa = q4(Q(s)[la]), qb = q4(Q(s)[lb]);
                            const V3 n{cc.normal.x, cc.normal.y, cc.normal.z};
                            const V3 wa = anchorWorld(shapeOf(ma.flags) == kSphere, pa, qa,
                                                      V3{cc.localAnchorA.x, cc.localAnchorA.y, cc.localAnchorA.z});
                            const V3 wb = anchorWorld(shapeOf(mb.flags) == kSphere, pb, qb,
                                                      V3{cc.localAnchorB.x, cc.localAnchorB.y, cc.localAnchorB.z});
                            const float g = cc.bias0 + dot(n, wa - wb);
                            if (g < -1e-3f) {
                                float resolve = 0.6f;
                                if (A.stackStab && lengthSq(f3(Vv(s)[la]) - f3(Vv(s)[lb])) < 1e-4f)
                                    resolve += 0.2f * (A.stackStiffness / 1000.0f) / (1.0f + A.stackDamping * A.h);
                                push = -resolve * (g + 1e-3f) / sum;
                                if (isDynamic(ma.flags) && !isAsleep(ma.flags)) {
                                    pa += n * (push * ima);
                                    P(s)[la] = pack(pa, 0.0f);
                                }
                                if (isDynamic(mb.flags) && !isAsleep(mb.flags)) {
                                    pb -= n * (push * imb);
                                    P(s)[lb] = pack(pb, 0.0f);
                                }
                            }
                        }
                    }
                    if (tape) V.push[(size_t)it * A.MR + j] = push;
                }
                __syncwarp();
            }
    }

    // ---- reverse ------------------------------------------------------------
    VXD float isoInvI(const Mass& m) const {
        return isDynamic(m.flags) && !isRotationLocked(m.flags) ? m.invI.x : 0.0f;
    }
    VXD void addGm(uint32_t li, const Mass& m, float gIm, float gIi) {
        float2 g = V.gm[li];
        if (isDynamic(m.flags) && !isLocked(m.flags)) g.x += gIm;
        if (isDynamic(m.flags) && !isRotationLocked(m.flags)) g.y += gIi;
        V.gm[li] = g;
    }

    // Reverse of one sweepRow (two-axis friction) from its recorded inputs.
    VXD void rowReverse(uint32_t j, const vx_contact& cc, const float4* rec, const float4* poseState,
                        uint8_t* bitsOut) {
        const uint32_t la = cc.a - b0, lb = cc.b - b0;
        const RowPrep& P = V.prep[j];
        if (P.kNormal <= 0.0f) {
            if (bitsOut) *bitsOut = kBrSkip;
            return;
        }
        uint32_t bits = 0;
        SolverBody a = body(poseState, la), b = body(poseState, lb);
        a.v = f3(rec[0]); a.w = f3(rec[1]); b.v = f3(rec[2]); b.w = f3(rec[3]);
        const float ln = rec[0].w, l1 = rec[1].w, l2 = rec[2].w;
        const V3 n{cc.normal.x, cc.normal.y, cc.normal.z};
        // replay of sweepRow's arithmetic (identical branch decisions)
        const float ima = solverInvMass(a.m), imb = solverInvMass(b.m);
        const bool dynA = isDynamic(a.m.flags), dynB = isDynamic(b.m.flags);
        const float vn = dot((a.v + cross(a.w, P.ra)) - (b.v + cross(b.w, P.rb)), n);
        float target = P.targetBase;
        bool resMax = false;
        if (cc.vn0 < -1.0f && (P.liveGap <= 0.0f || vn > 0.0f)) {
            bits |= kBrRestitution;
            const float rest = -cc.restitution * cc.vn0;
            if (rest > target) { target = rest; resMax = true; bits |= kBrResMax; }
        }
        const float jn = (target - vn) / P.kNormal;
        const float s = ln + jn;
        const bool clampOn = s > 0.0f;  // vmax(s, 0) == s
        if (clampOn) bits |= kBrClamp;
        const float lnp = vmax(s, 0.0f);
        const float dn = lnp - ln;
        const V3 ni = n * dn;
        SolverBody a1 = a, b1 = b;
        if (dynA) { a1.v += ni * ima; a1.w += invIF(a1, cross(P.ra, ni)); }
        if (dynB) { b1.v -= ni * imb; b1.w -= invIF(b1, cross(P.rb, ni)); }
        const float iA = isoInvI(a.m), iB = isoInvI(b.m);
        const Mass& mA = a.m;
        const Mass& mB = b.m;
        BodyBar& A_ = V.adj[la];
        BodyBar& B_ = V.adj[lb];
        V3 VA = f3(A_.v), WA = f3(A_.w), VB = f3(B_.v), WB = f3(B_.w);
        float4 lb4 = V.lamb[0][j];  // (n, t1, t2, vn0) adjoints of this row's impulses
        float lnpb = lb4.x, l1b = 0.0f, l2b = 0.0f;
        PrepBar& Pb = V.pbar[j];
        float gImA = 0.0f, gIiA = 0.0f, gImB = 0.0f, gIiB = 0.0f;
        if (P.k1 > 0.0f && P.k2 > 0.0f) {
            const V3 rv = (a1.v + cross(a1.w, P.ra)) - (b1.v + cross(b1.w, P.rb));
            const float rv1 = dot(rv, P.t1), rv2 = dot(rv, P.t2);
            const float next1 = l1 - rv1 / P.k1;
            const float next2 = l2 - rv2 / P.k2;
            const float max1 = cc.friction1 * lnp;
            const float max2 = cc.friction2 * lnp;
            const bool m1on = max1 > 0.0f, m2on = max2 > 0.0f;
            bits |= kBrFriction | (m1on ? kBrM1 : 0u) | (m2on ? kBrM2 : 0u);
            const float z1 = m1on ? next1 : 0.0f, z2 = m2on ? next2 : 0.0f;
            const float E = (m1on ? z1 * z1 / (max1 * max1) : 0.0f) + (m2on ? z2 * z2 / (max2 * max2) : 0.0f);
            const bool ell = E > 1.0f;
            if (ell) bits |= kBrEllipse;
            const float sc = ell ? 1.0f / sqrtf(E) : 1.0f;
            const float y1 = z1 * sc, y2 = z2 * sc;
            const float d1 = y1 - l1, d2 = y2 - l2;
            float d1b = 0.0f, d2b = 0.0f;
            const V3 imp = P.t1 * d1 + P.t2 * d2;
            if (dynA) {
                d1b += ima * dot(P.t1, VA) + iA * dot(P.raxt1, WA);
                d2b += ima * dot(P.t2, VA) + iA * dot(P.raxt2, WA);
                gImA += dot(imp, VA);
                gIiA += dot(P.raxt1 * d1 + P.raxt2 * d2, WA);
                accs(Pb.raxt1, WA, iA * d1);
                accs(Pb.raxt2, WA, iA * d2);
            }
            if (dynB) {
                d1b -= imb * dot(P.t1, VB) + iB * dot(P.rbxt1, WB);
                d2b -= imb * dot(P.t2, VB) + iB * dot(P.rbxt2, WB);
                gImB -= dot(imp, VB);
                gIiB -= dot(P.rbxt1 * d1 + P.rbxt2 * d2, WB);
                accs(Pb.rbxt1, WB, -iB * d1);
                accs(Pb.rbxt2, WB, -iB * d2);
            }
            const float y1b = lb4.y + d1b, y2b = lb4.z + d2b;
            l1b -= d1b;
            l2b -= d2b;
            float z1b = y1b * sc, z2b = y2b * sc, Eb = 0.0f;
            if (ell) {
                const float scb = z1 * y1b + z2 * y2b;
                Eb = scb * -0.5f / (E * sqrtf(E));
            }
            float m1b = 0.0f, m2b = 0.0f;
            if (m1on) { z1b += Eb * 2.0f * z1 / (max1 * max1); m1b += Eb * (-2.0f * z1 * z1 / (max1 * max1 * max1)); }
            if (m2on) { z2b += Eb * 2.0f * z2 / (max2 * max2); m2b += Eb * (-2.0f * z2 * z2 / (max2 * max2 * max2)); }
            const float u1b = m1on ? z1b : 0.0f, u2b = m2on ? z2b : 0.0f;
            lnpb += cc.friction1 * m1b + cc.friction2 * m2b;
            l1b += u1b;
            l2b += u2b;
            const float rv1b = -u1b / P.k1, rv2b = -u2b / P.k2;
            Pb.k1 += u1b * rv1 / (P.k1 * P.k1);
            Pb.k2 += u2b * rv2 / (P.k2 * P.k2);
            accs(VA, P.t1, rv1b); accs(VA, P.t2, rv2b);
            accs(WA, P.raxt1, rv1b); accs(WA, P.raxt2, rv2b);
            accs(VB, P.t1, -rv1b); accs(VB, P.t2, -rv2b);
            accs(WB, P.rbxt1, -rv1b); accs(WB, P.rbxt2, -rv2b);
            accs(Pb.raxt1, a1.w, rv1b); accs(Pb.raxt2, a1.w, rv2b);
            accs(Pb.rbxt1, b1.w, -rv1b); accs(Pb.rbxt2, b1.w, -rv2b);
        } else {
            l1b = lb4.y;
            l2b = lb4.z;
        }
        float dnb = 0.0f;
        if (dynA) {
            dnb += ima * dot(n, VA) + iA * dot(P.raxn, WA);
            gImA += dn * dot(n, VA);
            gIiA += dn * dot(P.raxn, WA);
            accs(Pb.raxn, WA, iA * dn);
        }
        if (dynB) {
            dnb -= imb * dot(n, VB) + iB * dot(P.rbxn, WB);
            gImB -= dn * dot(n, VB);
            gIiB -= dn * dot(P.rbxn, WB);
            accs(Pb.rbxn, WB, -iB * dn);
        }
        lnpb += dnb;
        float lnb = -dnb;
        const float sb = clampOn ? lnpb : 0.0f;
        lnb += sb;
        const float jnb = sb;
        const float targetb = jnb / P.kNormal;
        const float vnb = -jnb / P.kNormal;
        Pb.kN += -jnb * jn / P.kNormal;
        if (resMax) lb4.w += -cc.restitution * targetb;  // the row's vn0 adjoint
        else Pb.target0 += targetb;
        accs(VA, n, vnb); accs(WA, P.raxn, vnb);
        accs(VB, n, -vnb); accs(WB, P.rbxn, -vnb);
        accs(Pb.raxn, a.w, vnb); accs(Pb.rbxn, b.w, -vnb);
        if (dynA) { A_.v = pack(VA, 0.0f); A_.w = pack(WA, 0.0f); addGm(la, mA, gImA, gIiA); }
        if (dynB) { B_.v = pack(VB, 0.0f); B_.w = pack(WB, 0.0f); addGm(lb, mB, gImB, gIiB); }
        V.lamb[0][j] = make_float4(lnb, l1b, l2b, lb4.w);
        if (bitsOut) *bitsOut = (uint8_t)bits;
    }

    // Reverse of warmPrepRow (linear impulses; rolling and spinning are zero).
    VXD void warmReverse(uint32_t j, const vx_contact& cc, uint8_t* activeOut) {
        const float4 l = V.lamInit[j];
        const bool active = !(l.x <= 0.0f && l.y == 0.0f && l.z == 0.0f);
        if (activeOut) *activeOut = active ? 1u : 0u;
        if (!active) return;
        const uint32_t la = cc.a - b0, lb = cc.b - b0;
        const RowPrep& P = V.prep[j];
        const Mass mA = mass(la), mB = mass(lb);
        const V3 n{cc.normal.x, cc.normal.y, cc.normal.z};
        const V3 imp = n * l.x + P.t1 * l.y + P.t2 * l.z;
        V3 ib{0.0f, 0.0f, 0.0f};
        PrepBar& Pb = V.pbar[j];
        if (isDynamic(mA.flags)) {
            const V3 VA = f3(V.adj[la].v), WA = f3(V.adj[la].w);
            const float ma = solverInvMass(mA), iA = isoInvI(mA);
            accs(ib, VA, ma);
            accs(ib, xc(WA, P.ra), iA);
            accs(Pb.ra, xc(imp, WA), iA);
            addGm(la, mA, dot(imp, VA), dot(xc(P.ra, imp), WA));
        }
        if (isDynamic(mB.flags)) {
            const V3 VB = f3(V.adj[lb].v), WB = f3(V.adj[lb].w);
            const float mb = solverInvMass(mB), iB = isoInvI(mB);
            accs(ib, VB, -mb);
            accs(ib, xc(WB, P.rb), -iB);
            accs(Pb.rb, xc(imp, WB), -iB);
            addGm(lb, mB, -dot(imp, VB), -dot(xc(P.rb, imp), WB));
        }
        float4 g = V.lamb[0][j];
        g.x += dot(n, ib);
        g.y += dot(P.t1, ib);
        g.z += dot(P.t2, ib);
        V.lamb[0][j] = g;
    }

    // Reverse of prepRow's pose terms into body pose and mass adjoints.
    VXD void prepReverse(uint32_t j, const vx_contact& cc, const float4* poseState) {
        const uint32_t la = cc.a - b0, lb = cc.b - b0;
        const RowPrep& P = V.prep[j];
        PrepBar Pb = V.pbar[j];
        const Mass mA = mass(la), mB = mass(lb);
        const float iA = isoInvI(mA), iB = isoInvI(mB);
        const V3 n{cc.normal.x, cc.normal.y, cc.normal.z};
        const float kb = Pb.kN + Pb.k1 + Pb.k2;
        addGm(la, mA, kb, Pb.kN * dot(P.raxn, P.raxn) + Pb.k1 * dot(P.raxt1, P.raxt1) + Pb.k2 * dot(P.raxt2, P.raxt2));
        addGm(lb, mB, kb, Pb.kN * dot(P.rbxn, P.rbxn) + Pb.k1 * dot(P.rbxt1, P.rbxt1) + Pb.k2 * dot(P.rbxt2, P.rbxt2));
        accs(Pb.raxn, P.raxn, 2.0f * iA * Pb.kN);
        accs(Pb.rbxn, P.rbxn, 2.0f * iB * Pb.kN);
        accs(Pb.raxt1, P.raxt1, 2.0f * iA * Pb.k1);
        accs(Pb.rbxt1, P.rbxt1, 2.0f * iB * Pb.k1);
        accs(Pb.raxt2, P.raxt2, 2.0f * iA * Pb.k2);
        accs(Pb.rbxt2, P.rbxt2, 2.0f * iB * Pb.k2);
        Pb.ra += xc(n, Pb.raxn); Pb.ra += xc(P.t1, Pb.raxt1); Pb.ra += xc(P.t2, Pb.raxt2);
        Pb.rb += xc(n, Pb.rbxn); Pb.rb += xc(P.t1, Pb.rbxt1); Pb.rb += xc(P.t2, Pb.rbxt2);
        const float gapb = P.liveGap > 0.0f ? -Pb.target0 / A.h : 0.0f;
        accs(Pb.ra, n, gapb);
        accs(Pb.rb, n, -gapb);
        if (isDynamic(mA.flags)) {
            BodyBar& X = V.adj[la];
            X.p = pack(f3(X.p) + n * gapb, 0.0f);
            if (shapeOf(mA.flags) != kSphere) {
                Q4 qb = q4(X.q);
                rotateRevQ(q4(poseState[A.NB + la]), V3{cc.localAnchorA.x, cc.localAnchorA.y, cc.localAnchorA.z},
                           Pb.ra, qb);
                X.q = pack(qb);
            }
        }
        if (isDynamic(mB.flags)) {
            BodyBar& X = V.adj[lb];
            X.p = pack(f3(X.p) - n * gapb, 0.0f);
            if (shapeOf(mB.flags) != kSphere) {
                Q4 qb = q4(X.q);
                rotateRevQ(q4(poseState[A.NB + lb]), V3{cc.localAnchorB.x, cc.localAnchorB.y, cc.localAnchorB.z},
                           Pb.rb, qb);
                X.q = pack(qb);
            }
        }
    }

    VXD void reverseStep(uint32_t t, const float4* stepStart) {
        uint32_t c0;
        const uint32_t m = rowsOf(t, c0);
        const vx_contact* cs = A.contacts;
        const int S = A.substeps, W = A.sweeps;
        uint8_t* br = branchesOf(t);
        const size_t MR = A.MR, oWarm = (size_t)S * MR, oRows = oWarm + MR, oPush = oRows + (size_t)S * W * MR;
        // previous step's row adjoints start at zero; sources index the
        // previous step's contacts, whose world range starts at pbase
        uint32_t pc0 = 0, pm = 0, pbase = 0;
        if (t > 0) {
            pm = rowsOf(t - 1, pc0);
            pbase = pc0 - A.stepStart[t - 1];
        }
        for (uint32_t j = lane; j < pm; j += 32) V.lamb[1][j] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        __syncwarp();
        // position correction
        for (int it = A.posIters - 1; it >= 0; --it)
            for (int col = colours - 1; col >= 0; --col) {
                const uint32_t r0 = V.cstart[col], r1 = V.cstart[col + 1];
                for (uint32_t x = r0 + lane; x < r1; x += 32) {
                    const uint32_t j = V.order[x];
                    const float push = V.push[(size_t)it * A.MR + j];
                    if (br) br[oPush + (size_t)it * MR + j] = push != 0.0f ? 1u : 0u;
                    if (push == 0.0f) continue;
                    const vx_contact& cc = cs[c0 + j];
                    const uint32_t la = cc.a - b0, lb = cc.b - b0;
                    const Mass mA = mass(la), mB = mass(lb);
                    const float ma = solverInvMass(mA), mb = solverInvMass(mB), sum = ma + mb;
                    const V3 n{cc.normal.x, cc.normal.y, cc.normal.z};
                    const bool movesA = isDynamic(mA.flags) && !isAsleep(mA.flags);
                    const bool movesB = isDynamic(mB.flags) && !isAsleep(mB.flags);
                    float pushb = 0.0f, gImA = 0.0f, gImB = 0.0f;
                    if (movesA) { const float d = dot(n, f3(V.adj[la].p)); pushb += ma * d; gImA += push * d; }
                    if (movesB) { const float d = dot(n, f3(V.adj[lb].p)); pushb -= mb * d; gImB -= push * d; }
                    float resolve = 0.6f;
                    if (A.stackStab &&
                        lengthSq(f3(V.corr[2 * A.NB + la]) - f3(V.corr[2 * A.NB + lb])) < 1e-4f)
                        resolve += 0.2f * (A.stackStiffness / 1000.0f) / (1.0f + A.stackDamping * A.h);
                    const float gb = -resolve / sum * pushb;
                    const float sumb = -push / sum * pushb;
                    gImA += sumb;
                    gImB += sumb;
                    if (isDynamic(mA.flags)) {
                        BodyBar& X = V.adj[la];
                        X.p = pack(f3(X.p) + n * gb, 0.0f);
                        if (shapeOf(mA.flags) != kSphere) {
                            Q4 qb = q4(X.q);
                            rotateRevQ(q4(V.corr[A.NB + la]),
                                       V3{cc.localAnchorA.x, cc.localAnchorA.y, cc.localAnchorA.z}, n * gb, qb);
                            X.q = pack(qb);
                        }
                        addGm(la, mA, gImA, 0.0f);
                    }
                    if (isDynamic(mB.flags)) {
                        BodyBar& X = V.adj[lb];
                        X.p = pack(f3(X.p) - n * gb, 0.0f);
                        if (shapeOf(mB.flags) != kSphere) {
                            Q4 qb = q4(X.q);
                            rotateRevQ(q4(V.corr[A.NB + lb]),
                                       V3{cc.localAnchorB.x, cc.localAnchorB.y, cc.localAnchorB.z}, n * -gb, qb);
                            X.q = pack(qb);
                        }
                        addGm(lb, mB, gImB, 0.0f);
                    }
                }
                __syncwarp();
            }
        for (int sub = S - 1; sub >= 0; --sub) {
            const float4* ss = V.sub + (size_t)sub * 4 * A.NB;   // state at substep start
            const float4* ev = V.endv + (size_t)sub * 2 * A.NB;  // v, w after the sweeps
            // transform integration
            for (uint32_t li = lane; li < nb; li += 32) {
                const Mass mm = mass(li);
                if (isStaticBody(mm.flags) || isLocked(mm.flags) || isAsleep(mm.flags)) continue;
                BodyBar& X = V.adj[li];
                V3 wb = f3(X.w);
                Q4 qb = q4(X.q);
                if (isRotationLocked(mm.flags)) {
                    wb = V3{0.0f, 0.0f, 0.0f};
                } else {
                    qintegrateRev(q4(ss[A.NB + li]), f3(ev[A.NB + li]), A.h, qb, wb);
                }
                X.v = pack(f3(X.v) + f3(X.p) * A.h, 0.0f);
                X.w = pack(wb, 0.0f);
                X.q = pack(qb);
            }
            __syncwarp();
            // pose terms of this substep, adjoint accumulators zeroed
            for (uint32_t j = lane; j < m; j += 32) {
                const vx_contact& cc = cs[c0 + j];
                const SolverBody a = body(ss, cc.a - b0), b = body(ss, cc.b - b0);
                RowContact r;
                loadRowContact(cc, V.lamInit[j], r);
                prepRow(a, b, r, A.h, false, V.prep[j]);
                if (br) br[(size_t)sub * MR + j] = V.prep[j].liveGap > 0.0f ? 1u : 0u;
                PrepBar z = {};
                V.pbar[j] = z;
            }
            __syncwarp();
            for (int sweep = W - 1; sweep >= 0; --sweep)
                for (int col = colours - 1; col >= 0; --col) {
                    const uint32_t r0 = V.cstart[col], r1 = V.cstart[col + 1];
                    for (uint32_t x = r0 + lane; x < r1; x += 32) {
                        const uint32_t j = V.order[x];
                        const vx_contact& cc = cs[c0 + j];
                        if (!solved(cc)) continue;
                        const float4* rec = V.rin + (((size_t)sub * W + sweep) * A.MR + j) * 4;
                        rowReverse(j, cc, rec, ss, br ? br + oRows + ((size_t)sub * W + sweep) * MR + j : nullptr);
                    }
                    __syncwarp();
                }
            if (sub == 0) {
                for (int col = colours - 1; col >= 0; --col) {
                    const uint32_t r0 = V.cstart[col], r1 = V.cstart[col + 1];
                    for (uint32_t x = r0 + lane; x < r1; x += 32) {
                        const uint32_t j = V.order[x];
                        const vx_contact& cc = cs[c0 + j];
                        if (solved(cc)) warmReverse(j, cc, br ? br + oWarm + j : nullptr);
                    }
                    __syncwarp();
                }
                // restitution references: to the previous step's contact, or to
                // the velocities at detection (the state at substep 0)
                for (int col = 0; col < colours; ++col) {
                    const uint32_t r0 = V.cstart[col], r1 = V.cstart[col + 1];
                    for (uint32_t x = r0 + lane; x < r1; x += 32) {
                        const uint32_t j = V.order[x];
                        const vx_contact& cc = cs[c0 + j];
                        const float g = V.lamb[0][j].w;
                        if (g == 0.0f || !solved(cc)) continue;
                        const uint2 sr = A.src[c0 + j];
                        // carried: handled with the impulses below, or (first taped
                        // step) a constant from before the tape
                        if (sr.y != kNone) continue;
                        const uint32_t la = cc.a - b0, lb = cc.b - b0;
                        const Mass mA = mass(la), mB = mass(lb);
                        const V3 n{cc.normal.x, cc.normal.y, cc.normal.z};
                        const RowPrep& P = V.prep[j];
                        PrepBar& Pb = V.pbar[j];
                        if (isDynamic(mA.flags)) {
                            BodyBar& X = V.adj[la];
                            X.v = pack(f3(X.v) + n * g, 0.0f);
                            X.w = pack(f3(X.w) + P.raxn * g, 0.0f);
                        }
                        if (isDynamic(mB.flags)) {
                            BodyBar& X = V.adj[lb];
                            X.v = pack(f3(X.v) - n * g, 0.0f);
                            X.w = pack(f3(X.w) - P.rbxn * g, 0.0f);
                        }
                        accs(Pb.raxn, f3(ss[3 * A.NB + la]), g);
                        accs(Pb.rbxn, f3(ss[3 * A.NB + lb]), -g);
                    }
                    __syncwarp();
                }
            }
            for (int col = colours - 1; col >= 0; --col) {
                const uint32_t r0 = V.cstart[col], r1 = V.cstart[col + 1];
                for (uint32_t x = r0 + lane; x < r1; x += 32) {
                    const uint32_t j = V.order[x];
                    const vx_contact& cc = cs[c0 + j];
                    if (solved(cc)) prepReverse(j, cc, ss);
                }
                __syncwarp();
            }
            // velocity integration of this substep (substep 0: the prepare's)
            for (uint32_t li = lane; li < nb; li += 32) {
                const Mass mm = mass(li);
                if (!isDynamic(mm.flags) || isLocked(mm.flags) || isAsleep(mm.flags)) continue;
                const float4 ex = A.B.extra[b0 + li];
                BodyBar& X = V.adj[li];
                X.v = pack(f3(X.v) * (1.0f / (1.0f + ex.z * A.h)), 0.0f);
                X.w = pack(f3(X.w) * (1.0f / (1.0f + ex.w * A.h)), 0.0f);
            }
            __syncwarp();
        }
        // orientation normalisation at the step start
        for (uint32_t li = lane; li < nb; li += 32) {
            BodyBar& X = V.adj[li];
            X.q = pack(qnormalizeRev(q4(stepStart[A.NB + li]), q4(X.q)));
        }
        __syncwarp();
        // impulses and restitution references inherited from the previous step
        if (t > 0) {
            for (uint32_t j = lane; j < m; j += 32) {
                const uint2 sr = A.src[c0 + j];
                const float4 g = V.lamb[0][j];
                if (sr.x != kNone && sr.x - pbase < pm) {
                    float* d = reinterpret_cast<float*>(&V.lamb[1][sr.x - pbase]);
                    atomicAdd(d, g.x);
                    atomicAdd(d + 1, g.y);
                    atomicAdd(d + 2, g.z);
                }
                if (sr.y != kNone && sr.y - pbase < pm && g.w != 0.0f)
                    atomicAdd(reinterpret_cast<float*>(&V.lamb[1][sr.y - pbase]) + 3, g.w);
            }
        }
        __syncwarp();
        float4* tmp = V.lamb[0];
        V.lamb[0] = V.lamb[1];
        V.lamb[1] = tmp;
    }

    VXD void loadCheckpoint(uint32_t slot, float4* dst) const {
        const float4* ck = A.ckpt + (size_t)slot * 4 * A.n;
        for (uint32_t li = lane; li < A.NB; li += 32)
            for (int f = 0; f < 4; ++f)
                dst[f * A.NB + li] = li < nb ? ck[(size_t)f * A.n + b0 + li] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        __syncwarp();
    }

    VXD bool matchesCheckpoint(uint32_t slot, const float4* s) const {
        const float4* ck = A.ckpt + (size_t)slot * 4 * A.n;
        bool ok = true;
        for (uint32_t li = lane; li < nb; li += 32)
            for (int f = 0; f < 4; ++f) {
                const float4 x = s[f * A.NB + li], y = ck[(size_t)f * A.n + b0 + li];
                const float tol = 1e-5f * (1.0f + fabsf(y.x) + fabsf(y.y) + fabsf(y.z));
                if (fabsf(x.x - y.x) > tol || fabsf(x.y - y.y) > tol || fabsf(x.z - y.z) > tol ||
                    (f == 1 && fabsf(x.w - y.w) > tol))
                    ok = false;
            }
        return __all_sync(0xffffffffu, ok);
    }
};

__global__ void __launch_bounds__(128) adjointKernel(AdjArgs A) {
    const uint32_t w = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    if (w >= A.worlds) return;
    WorldRun R(A, w);
    if (R.nb > A.NB) {
        if (R.lane == 0) atomicOr(A.flags + w, (uint32_t)VXB_ADJ_UNSUPPORTED);
        return;
    }
    // seeds, zeroed accumulators
    for (uint32_t li = R.lane; li < R.nb; li += 32) {
        const float* s = A.seed + (size_t)(R.b0 + li) * 13;
        BodyBar X;
        X.p = make_float4(s[0], s[1], s[2], 0.0f);
        X.q = make_float4(s[3], s[4], s[5], s[6]);
        X.v = make_float4(s[7], s[8], s[9], 0.0f);
        X.w = make_float4(s[10], s[11], s[12], 0.0f);
        R.V.adj[li] = X;
        R.V.gm[li] = make_float2(0.0f, 0.0f);
    }
    for (uint32_t j = R.lane; j < A.MR; j += 32) {
        R.V.lamb[0][j] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        R.V.lamb[1][j] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
    __syncwarp();
    for (int seg = (int)A.J - 1; seg >= 0; --seg) {
        const uint32_t t0 = (uint32_t)seg * A.every;
        const uint32_t t1 = min(A.steps, t0 + A.every);
        R.loadCheckpoint((uint32_t)seg, R.V.cur);
        for (uint32_t t = t0; t < t1; ++t) {
            R.copyState(R.V.st + (size_t)(t - t0) * 4 * A.NB, R.V.cur);
            R.forwardStep(t, false);
        }
        if (!R.matchesCheckpoint((uint32_t)seg + 1, R.V.cur) && R.lane == 0)
            atomicOr(A.flags + w, (uint32_t)VXB_ADJ_DIVERGED);
        for (int t = (int)t1 - 1; t >= (int)t0; --t) {
            const float4* start = R.V.st + (size_t)(t - t0) * 4 * A.NB;
            R.copyState(R.V.cur, start);
            R.forwardStep((uint32_t)t, true);
            R.reverseStep((uint32_t)t, start);
        }
    }
    // Worlds outside the model (rewound, diverged, unsupported) get zero
    // gradients rather than values of another trajectory.
    __syncwarp();
    const bool flagged = atomicOr(A.flags + w, 0u) != 0u;
    for (uint32_t li = R.lane; li < R.nb; li += 32) {
        BodyBar X = R.V.adj[li];
        float2 gm = R.V.gm[li];
        if (flagged) {
            X.p = X.q = X.v = X.w = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            gm = make_float2(0.0f, 0.0f);
        }
        float* g = A.grad + (size_t)(R.b0 + li) * 13;
        g[0] = X.p.x; g[1] = X.p.y; g[2] = X.p.z;
        g[3] = X.q.x; g[4] = X.q.y; g[5] = X.q.z; g[6] = X.q.w;
        g[7] = X.v.x; g[8] = X.v.y; g[9] = X.v.z;
        g[10] = X.w.x; g[11] = X.w.y; g[12] = X.w.z;
        const Mass m = R.mass(li);
        A.gradInv[2 * (R.b0 + li)] = gm.x;
        A.gradInv[2 * (R.b0 + li) + 1] = gm.y;
        // inverse mass 1/m and isotropic inverse inertia c/m: d/dm = -(1/m^2) gInvMass - (invI/m) gInvI
        const float im = m.invMass;
        A.gradMass[R.b0 + li] = isDynamic(m.flags) ? -im * im * gm.x - m.invI.x * im * gm.y : 0.0f;
    }
}

}  // namespace

// ---- tape recording (called by the device world's step) ------------------------

int tapeStepBegin(Context& c) {
    Tape& T = c.tape;
    if (!T.active || T.recorded >= T.steps || T.recorded % T.every != 0) return VXB_OK;
    const uint32_t slot = T.recorded / T.every;
    AD_LAUNCH(c, checkpointKernel, gridFor(c.n, 256), 256, c.B, c.n, PT<float4>(T.ckpt) + (size_t)slot * 4 * c.n);
    return VXB_OK;
}

int tapeBeforeMatch(Context& c, const vx_contact* cs, uint32_t m, const vx_contact* prev, const uint64_t* prevKeys,
                    uint32_t mPrev) {
    Tape& T = c.tape;
    if (!T.active || T.recorded >= T.steps) return VXB_OK;
    const size_t off = T.stepStart.back();
    AD_TRY(growKeep(c, T.src, (off + m) * sizeof(uint2), off * sizeof(uint2)));
    uint2* src = PT<uint2>(T.src) + off;
    if (m == 0) return VXB_OK;
    if (mPrev)
        AD_LAUNCH(c, matchSourceKernel, gridFor(m, 128), 128, cs, m, prev, prevKeys, mPrev, src);
    else
        AD_CUDA(c, cudaMemsetAsync(src, 0xff, (size_t)m * sizeof(uint2), c.stream));
    return VXB_OK;
}

int tapeAfterMatch(Context& c, const vx_contact* cs, uint32_t m) {
    Tape& T = c.tape;
    if (!T.active || T.recorded >= T.steps) return VXB_OK;
    const size_t off = T.stepStart.back();
    AD_TRY(growKeep(c, T.contacts, (off + m) * sizeof(vx_contact), off * sizeof(vx_contact)));
    if (m)
        AD_CUDA(c, cudaMemcpyAsync(PT<vx_contact>(T.contacts) + off, cs, (size_t)m * sizeof(vx_contact),
                                   cudaMemcpyDeviceToDevice, c.stream));
    AD_LAUNCH(c, worldStartKernel, gridFor(c.worlds + 1, 128), 128, cs, m, PT<uint32_t>(c.worldOfBuf), c.worlds,
              PT<uint32_t>(T.worldStart) + (size_t)T.recorded * (c.worlds + 1));
    return VXB_OK;
}

int tapeAfterIslands(Context& c, const uint32_t* color, uint32_t m) {
    Tape& T = c.tape;
    if (!T.active || T.recorded >= T.steps) return VXB_OK;
    const size_t off = T.stepStart.back();
    AD_TRY(growKeep(c, T.color, (off + m) * sizeof(uint32_t), off * sizeof(uint32_t)));
    if (m)
        AD_CUDA(c, cudaMemcpyAsync(PT<uint32_t>(T.color) + off, color, (size_t)m * sizeof(uint32_t),
                                   cudaMemcpyDeviceToDevice, c.stream));
    return VXB_OK;
}

int tapeAfterRewind(Context& c, const uint32_t* rewound) {
    Tape& T = c.tape;
    if (!T.active || T.recorded >= T.steps || !rewound) return VXB_OK;
    AD_LAUNCH(c, rewoundWorldsKernel, gridFor(c.n, 256), 256, rewound, c.n, PT<uint32_t>(c.worldOfBuf),
              PT<uint32_t>(T.flags));
    return VXB_OK;
}

int tapeStepEnd(Context& c, uint32_t m) {
    Tape& T = c.tape;
    if (!T.active || T.recorded >= T.steps) return VXB_OK;
    T.stepStart.push_back(T.stepStart.back() + m);
    ++T.recorded;
    if (T.recorded == T.steps) {
        const uint32_t slot = (T.steps + T.every - 1) / T.every;
        AD_LAUNCH(c, checkpointKernel, gridFor(c.n, 256), 256, c.B, c.n,
                  PT<float4>(T.ckpt) + (size_t)slot * 4 * c.n);
    }
    return VXB_OK;
}

int tapeBegin(Context& c, uint32_t steps, uint32_t every) {
    if (steps == 0 || every == 0) return fail(c, VXB_ERR_INVALID, "tape: steps and checkpoint interval must be > 0");
    if (c.n == 0) return fail(c, VXB_ERR_INVALID, "tape: no bodies loaded");
    Tape& T = c.tape;
    T.active = true;
    T.steps = steps;
    T.every = every;
    T.recorded = 0;
    T.stepStart.assign(1, 0u);
    const uint32_t J = (steps + every - 1) / every;
    AD_TRY(ensure(c, T.ckpt, (size_t)(J + 1) * 4 * c.n * sizeof(float4)));
    AD_TRY(ensure(c, T.worldStart, (size_t)steps * (c.worlds + 1) * sizeof(uint32_t)));
    AD_TRY(ensure(c, T.flags, (size_t)c.worlds * sizeof(uint32_t)));
    AD_CUDA(c, cudaMemsetAsync(T.flags.ptr, 0, (size_t)c.worlds * sizeof(uint32_t), c.stream));
    return VXB_OK;
}

int tapeEnd(Context& c) {
    Tape& T = c.tape;
    T.active = false;
    T.recorded = 0;
    T.stepStart.assign(1, 0u);
    if (T.contacts.ptr || T.ckpt.ptr || T.scratch.ptr || T.branches.ptr) cudaStreamSynchronize(c.stream);
    for (DevBuf* b : {&T.contacts, &T.src, &T.color, &T.worldStart, &T.ckpt, &T.flags, &T.scratch, &T.host,
                      &T.branches}) {
        if (b->ptr) cudaFree(b->ptr);
        b->ptr = nullptr;
        b->bytes = 0;
    }
    return VXB_OK;
}

int tapeRead(Context& c, vx_contact* contacts, uint32_t* stepStart, uint32_t* src, int32_t* color, float* ckpt,
             uint32_t* worldFlags) {
    Tape& T = c.tape;
    const size_t total = T.stepStart.back();
    if (stepStart) std::memcpy(stepStart, T.stepStart.data(), T.stepStart.size() * sizeof(uint32_t));
    if (contacts && total)
        AD_CUDA(c, cudaMemcpyAsync(contacts, T.contacts.ptr, total * sizeof(vx_contact), cudaMemcpyDeviceToHost,
                                   c.stream));
    if (src && total)
        AD_CUDA(c, cudaMemcpyAsync(src, T.src.ptr, total * sizeof(uint2), cudaMemcpyDeviceToHost, c.stream));
    if (color && total)
        AD_CUDA(c, cudaMemcpyAsync(color, T.color.ptr, total * sizeof(uint32_t), cudaMemcpyDeviceToHost, c.stream));
    if (ckpt) {
        const uint32_t J = (T.steps + T.every - 1) / T.every;
        AD_CUDA(c, cudaMemcpyAsync(ckpt, T.ckpt.ptr, (size_t)(J + 1) * 4 * c.n * sizeof(float4),
                                   cudaMemcpyDeviceToHost, c.stream));
    }
    if (worldFlags)
        AD_CUDA(c, cudaMemcpyAsync(worldFlags, T.flags.ptr, (size_t)c.worlds * sizeof(uint32_t),
                                   cudaMemcpyDeviceToHost, c.stream));
    AD_CUDA(c, cudaStreamSynchronize(c.stream));
    return VXB_OK;
}

int adjointBackward(Context& c, const float* seed, float* grad, float* gradInv, float* gradMass,
                    uint32_t* worldFlags, uint8_t* branches, size_t branchCapacity, size_t* branchBytes,
                    uint32_t* branchRows) {
    Tape& T = c.tape;
    if (!T.active || T.recorded != T.steps)
        return fail(c, VXB_ERR_INVALID, "adjoint: the tape has not recorded all of its steps");
    const vxb_step_config& cfg = c.config;
    if (cfg.solver.frictionModel != VX_FRICTION_TWO_AXIS)
        return fail(c, VXB_ERR_UNSUPPORTED, "adjoint: only the two-axis friction model is differentiated");
    const uint32_t n = c.n, worlds = c.worlds, steps = T.steps;
    const size_t total = T.stepStart.back();
    // per-world body ranges (worlds are contiguous, ascending)
    std::vector<uint32_t> bodyStart(worlds + 1, 0);
    for (uint32_t i = 0; i < n; ++i) ++bodyStart[c.hostWorldOf[i] + 1];
    for (uint32_t w = 0; w < worlds; ++w) bodyStart[w + 1] += bodyStart[w];
    uint32_t NB = 1;
    for (uint32_t w = 0; w < worlds; ++w) NB = std::max(NB, bodyStart[w + 1] - bodyStart[w]);
    AD_TRY(ensure(c, T.host, 64 + (worlds + 1) * 4 + (steps + 1) * 4 + (size_t)n * 13 * 4 * 2 + (size_t)n * 12));
    char* hb = PT<char>(T.host);
    uint32_t* dExtent = reinterpret_cast<uint32_t*>(hb);
    uint32_t* dBodyStart = dExtent + 16;
    uint32_t* dStepStart = dBodyStart + (worlds + 1);
    float* dSeed = reinterpret_cast<float*>(dStepStart + (steps + 1));
    float* dGrad = dSeed + (size_t)n * 13;
    float* dGradInv = dGrad + (size_t)n * 13;
    float* dGradMass = dGradInv + (size_t)n * 2;
    AD_CUDA(c, cudaMemsetAsync(dExtent, 0, 64, c.stream));
    AD_CUDA(c, cudaMemcpyAsync(dBodyStart, bodyStart.data(), (worlds + 1) * 4, cudaMemcpyHostToDevice, c.stream));
    AD_CUDA(c, cudaMemcpyAsync(dStepStart, T.stepStart.data(), (steps + 1) * 4, cudaMemcpyHostToDevice, c.stream));
    if (seed)
        AD_CUDA(c, cudaMemcpyAsync(dSeed, seed, (size_t)n * 13 * 4, cudaMemcpyHostToDevice, c.stream));
    else
        AD_CUDA(c, cudaMemsetAsync(dSeed, 0, (size_t)n * 13 * 4, c.stream));
    AD_LAUNCH(c, tapeExtentKernel, gridFor(std::max<uint64_t>(total, (uint64_t)steps * worlds), 256), 256,
              PT<uint32_t>(T.color), (uint32_t)total, PT<uint32_t>(T.worldStart), steps, worlds, dExtent);
    AD_LAUNCH(c, scopeKernel, gridFor(std::max<uint64_t>(n, total), 256), 256, c.B, n, PT<uint32_t>(c.worldOfBuf),
              PT<vx_contact>(T.contacts), (uint32_t)total, PT<uint32_t>(T.flags));
    uint32_t ext[2];
    AD_CUDA(c, cudaMemcpyAsync(ext, dExtent, 8, cudaMemcpyDeviceToHost, c.stream));
    AD_CUDA(c, cudaStreamSynchronize(c.stream));
    AdjArgs A;
    std::memset(&A, 0, sizeof(A));
    A.B = c.B;
    A.ckpt = PT<float4>(T.ckpt);
    A.n = n;
    A.worlds = worlds;
    A.steps = steps;
    A.every = T.every;
    A.J = (steps + T.every - 1) / T.every;
    A.bodyStart = dBodyStart;
    A.contacts = PT<vx_contact>(T.contacts);
    A.stepStart = dStepStart;
    A.src = PT<uint2>(T.src);
    A.color = PT<uint32_t>(T.color);
    A.worldStart = PT<uint32_t>(T.worldStart);
    const int substeps = cfg.substeps > 0 ? cfg.substeps : 1;
    A.gravity = V3{cfg.gravity.x, cfg.gravity.y, cfg.gravity.z};
    A.h = cfg.dt / substeps;
    A.substeps = substeps;
    A.sweeps = 2 * cfg.solver.velocityIterations;
    A.posIters = cfg.solver.positionIterations;
    A.stackStab = cfg.solver.enableStackStabilization;
    A.stackStiffness = cfg.solver.stackStiffness;
    A.stackDamping = cfg.solver.stackDamping;
    A.NB = NB;
    A.MR = std::max<uint32_t>(ext[1], 1);
    A.MC = ext[0];
    A.seed = dSeed;
    A.grad = dGrad;
    A.gradInv = dGradInv;
    A.gradMass = dGradMass;
    A.flags = PT<uint32_t>(T.flags);
    const bool wantBranches = branchBytes != nullptr || branches != nullptr;
    if (wantBranches) {
        A.branchStep = ((size_t)substeps * (1 + std::max(A.sweeps, 1)) + 1 + (size_t)std::max(A.posIters, 1)) * A.MR;
        const size_t need = A.branchStep * steps * worlds;
        if (branchBytes) *branchBytes = need;
        if (branchRows) *branchRows = A.MR;
        if (!branches || branchCapacity < need)
            return fail(c, VXB_ERR_CAPACITY, "adjoint: branch buffer smaller than the reported size");
        AD_TRY(ensure(c, T.branches, need));
        AD_CUDA(c, cudaMemsetAsync(T.branches.ptr, 0, need, c.stream));
        A.branches = PT<uint8_t>(T.branches);
    }
    // per-world scratch layout
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t NBs = A.NB, MRs = A.MR;
    size_t o = 0;
    A.oSt = o; o += al((size_t)T.every * 4 * NBs * 16);
    A.oSub = o; o += al((size_t)substeps * 4 * NBs * 16);
    A.oEnd = o; o += al((size_t)substeps * 2 * NBs * 16);
    A.oCorr = o; o += al(4 * NBs * 16);
    A.oRin = o; o += al((size_t)substeps * std::max(A.sweeps, 1) * MRs * 64);
    A.oPush = o; o += al((size_t)std::max(A.posIters, 1) * MRs * 4);
    A.oLam = o; o += al(MRs * 16);
    A.oLamInit = o; o += al(MRs * 16);
    A.oPrep = o; o += al(MRs * sizeof(RowPrep));
    A.oPbar = o; o += al(MRs * sizeof(PrepBar));
    A.oOrder = o; o += al(MRs * 4);
    A.oCstart = o; o += al(((size_t)A.MC + 4) * 4);
    A.oLamb0 = o; o += al(MRs * 16);
    A.oLamb1 = o; o += al(MRs * 16);
    A.oCur = o; o += al(4 * NBs * 16);
    A.oAdj = o; o += al(NBs * sizeof(BodyBar));
    A.oGm = o; o += al(NBs * 8);
    A.worldBytes = o;
    AD_TRY(ensure(c, T.scratch, A.worldBytes * worlds));
    A.scratch = PT<char>(T.scratch);
    const int worldsPerBlock = 4;
    AD_LAUNCH(c, adjointKernel, (worlds + worldsPerBlock - 1) / worldsPerBlock, 32 * worldsPerBlock, A);
    AD_CUDA(c, cudaGetLastError());
    if (grad) AD_CUDA(c, cudaMemcpyAsync(grad, dGrad, (size_t)n * 13 * 4, cudaMemcpyDeviceToHost, c.stream));
    if (gradInv) AD_CUDA(c, cudaMemcpyAsync(gradInv, dGradInv, (size_t)n * 2 * 4, cudaMemcpyDeviceToHost, c.stream));
    if (gradMass) AD_CUDA(c, cudaMemcpyAsync(gradMass, dGradMass, (size_t)n * 4, cudaMemcpyDeviceToHost, c.stream));
    if (worldFlags)
        AD_CUDA(c, cudaMemcpyAsync(worldFlags, T.flags.ptr, (size_t)worlds * 4, cudaMemcpyDeviceToHost, c.stream));
    if (A.branches)
        AD_CUDA(c, cudaMemcpyAsync(branches, A.branches, A.branchStep * steps * worlds, cudaMemcpyDeviceToHost,
                                   c.stream));
    AD_CUDA(c, cudaStreamSynchronize(c.stream));
    return VXB_OK;
}

}  // namespace vxb
