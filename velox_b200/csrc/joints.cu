// The substep-wise path of advanceSubsteps on the device (the reference CUDA
// backend's, src/backend_cuda.cu:691-760 and :800-880): with 64 or more
// joints of supported types, every substep runs the contact sweeps, then
// reset + 8 sweeps of the joints colour by colour + the break test, then the
// position integration of every body. Joints are coloured on the host with
// the greedy first-free-bit rule over their dynamic endpoints (64 colours,
// then a per-body spill counter), so no two joints of one colour share a
// dynamic body and one thread per joint solves a colour in parallel.
#include <algorithm>
#include <vector>

#include "context.cuh"
#include "joints.cuh"

namespace vxb {

namespace {

#define JT_TRY(expr)                   \
    do {                               \
        int s_ = (expr);               \
        if (s_ != VXB_OK) return s_;   \
    } while (0)

#define JT_CUDA(c, expr)                                              \
    do {                                                              \
        cudaError_t e_ = (expr);                                      \
        if (e_ != cudaSuccess) return cudaStatus((c), e_, #expr);     \
    } while (0)

#define JT_LAUNCH(c, kernel, grid, block, ...)                               \
    do {                                                                     \
        kernel<<<(grid), (block), 0, (c).stream>>>(__VA_ARGS__);            \
        ++(c).launches;                                                      \
    } while (0)

inline uint32_t gridFor(uint64_t items, int threads) {
    const uint64_t b = (items + threads - 1) / threads;
    return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(b, 65535u * 16u));
}

constexpr uint32_t kDeviceJointThreshold = 64;  // fewer joints: the host path is faster

VXD joint::JBody loadJointBody(const BodyArrays& B, uint32_t i) {
    joint::JBody b;
    b.p = f3(B.pos[i]);
    b.q = q4(B.rot[i]);
    b.v = f3(B.vel[i]);
    b.w = f3(B.ang[i]);
    const float4 in = B.inertia[i];
    b.m.invI = V3{in.x, in.y, in.z};
    b.m.invMass = in.w;
    b.m.iq = q4(B.iq[i]);
    b.m.flags = B.filt[i].x;
    return b;
}

__global__ void jointResetKernel(vx_joint* joints, uint32_t count, int preserveBroken) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
        if (preserveBroken && joints[k].broken) continue;
        joint::reset(joints[k]);
    }
}

// One colour: joints [first, first + count) share no dynamic body.
__global__ void jointColorKernel(BodyArrays B, vx_joint* joints, uint32_t first, uint32_t count, float dt) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
        vx_joint j = joints[first + k];
        if (j.broken) continue;
        joint::JBody a = loadJointBody(B, j.a), b = loadJointBody(B, j.b);
        joint::solve(j, a, b, dt);
        if (joint::movable(a)) { B.vel[j.a] = pack(a.v, 0.0f); B.ang[j.a] = pack(a.w, 0.0f); }
        if (joint::movable(b)) { B.vel[j.b] = pack(b.v, 0.0f); B.ang[j.b] = pack(b.w, 0.0f); }
        joints[first + k] = j;
    }
}

__global__ void jointBreakKernel(vx_joint* joints, uint32_t count, float dt) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x)
        joint::markBroken(joints[k], dt);
}

// Greedy colours of the joints in their order (dynamic endpoints only), the
// colour-major order and each colour's start.
void colourJoints(const vx_body* bodies, uint32_t n, const vx_joint* joints, uint32_t count,
                  std::vector<uint32_t>& order, std::vector<uint32_t>& colourStart) {
    std::vector<uint64_t> mask(n, 0);
    std::vector<int> next(n, 64);
    std::vector<int> colourOf(count);
    int colours = 0;
    for (uint32_t k = 0; k < count; ++k) {
        const vx_joint& j = joints[k];
        const bool staticA = bodies[j.a].motionType != VX_MOTION_DYNAMIC;
        const bool staticB = bodies[j.b].motionType != VX_MOTION_DYNAMIC;
        const uint64_t used = (staticA ? 0 : mask[j.a]) | (staticB ? 0 : mask[j.b]);
        int colour;
        if (~used) {
            colour = 0;
            while (used & (1ull << colour)) ++colour;
        } else {
            const int nextA = staticA ? 64 : next[j.a];
            const int nextB = staticB ? 64 : next[j.b];
            colour = nextA > nextB ? nextA : nextB;
            if (!staticA) next[j.a] = colour + 1;
            if (!staticB) next[j.b] = colour + 1;
        }
        if (colour < 64) {
            if (!staticA) mask[j.a] |= 1ull << colour;
            if (!staticB) mask[j.b] |= 1ull << colour;
        }
        colourOf[k] = colour;
        colours = std::max(colours, colour + 1);
    }
    colourStart.assign((size_t)colours + 1, 0);
    for (int col : colourOf) ++colourStart[(size_t)col + 1];
    for (int col = 0; col < colours; ++col) colourStart[(size_t)col + 1] += colourStart[col];
    std::vector<uint32_t> fill(colourStart.begin(), colourStart.end() - 1);
    order.assign(count, 0);
    for (uint32_t k = 0; k < count; ++k) order[fill[colourOf[k]]++] = k;
}

}  // namespace

int backendAdvanceJoints(Context& c, vx_body* bodies, uint32_t n, vx_contact* contacts, uint32_t m,
                         vx_joint* joints, uint32_t njoints, vx_vec3 gravity, float h, int substeps,
                         const vx_solver_options& o, int* advanced, uint32_t* iterations) {
    *advanced = 0;
    if (iterations) *iterations = 0;
    if (njoints < kDeviceJointThreshold) return VXB_OK;
    for (uint32_t k = 0; k < njoints; ++k)
        if (joints[k].type > VX_JOINT_GEAR) return VXB_OK;
    for (uint32_t k = 0; k < njoints; ++k)
        if (joints[k].a >= n || joints[k].b >= n || joints[k].a == joints[k].b)
            return fail(c, VXB_ERR_INVALID, "joint endpoints must be two distinct bodies");
    // a joint wakes its sleeping endpoint (also when the path below declines)
    for (uint32_t k = 0; k < njoints; ++k) {
        vx_body& a = bodies[joints[k].a];
        vx_body& b = bodies[joints[k].b];
        if (a.asleep == b.asleep) continue;
        a.asleep = b.asleep = 0;
        a.sleepTimer = b.sleepTimer = 0.0f;
    }
    if (o.iterationPolicy != 0) return VXB_OK;  // Adaptive: the host path, like the reference
    JT_TRY(loadBodies(c, bodies, n, nullptr));
    JT_TRY(backendStepwise(c, bodies, n, contacts, m, joints, njoints, gravity, h, substeps, o, iterations));
    *advanced = 1;
    return VXB_OK;
}

int backendStepwise(Context& c, vx_body* bodies, uint32_t n, vx_contact* contacts, uint32_t m, vx_joint* joints,
                    uint32_t njoints, vx_vec3 gravity, float h, int substeps, const vx_solver_options& o,
                    uint32_t* iterations) {
    std::vector<uint32_t> order, colourStart(1, 0);
    std::vector<vx_joint> sorted;
    vx_joint* dj = nullptr;
    if (njoints) {
        colourJoints(bodies, n, joints, njoints, order, colourStart);
        sorted.resize(njoints);
        for (uint32_t s = 0; s < njoints; ++s) sorted[s] = joints[order[s]];
        JT_TRY(ensure(c, c.jointBuf, (size_t)njoints * sizeof(vx_joint)));
        dj = reinterpret_cast<vx_joint*>(c.jointBuf.ptr);
        JT_CUDA(c, cudaMemcpyAsync(dj, sorted.data(), (size_t)njoints * sizeof(vx_joint), cudaMemcpyHostToDevice,
                                    c.stream));
    }
    const uint32_t colours = (uint32_t)colourStart.size() - 1;
    for (int s = 0; s < substeps; ++s) {
        if (s > 0) JT_TRY(backendIntegrate(c, gravity, h));
        // contact sweeps (the first substep warm-starts and colours the contacts)
        if (m) JT_TRY(backendSolve(c, contacts, m, h, s == 0, o, gravity, 1, false));
        if (njoints) {
            JT_LAUNCH(c, jointResetKernel, gridFor(njoints, 128), 128, dj, njoints, s > 0 ? 1 : 0);
            for (int it = 0; it < joint::kIterations; ++it)
                for (uint32_t col = 0; col < colours; ++col) {
                    const uint32_t first = colourStart[col], count = colourStart[col + 1] - first;
                    JT_LAUNCH(c, jointColorKernel, gridFor(count, 128), 128, c.B, dj, first, count, h);
                }
            JT_LAUNCH(c, jointBreakKernel, gridFor(njoints, 128), 128, dj, njoints, h);
        }
        JT_TRY(backendIntegrateTransforms(c, h));
    }
    if (njoints)
        JT_CUDA(c, cudaMemcpyAsync(sorted.data(), dj, (size_t)njoints * sizeof(vx_joint), cudaMemcpyDeviceToHost,
                                    c.stream));
    JT_TRY(readBodies(c, bodies, n));  // synchronises the stream
    for (uint32_t s = 0; s < njoints; ++s) joints[order[s]] = sorted[s];
    if (iterations) *iterations = m ? (uint32_t)(2 * o.velocityIterations * substeps) : 0u;
    return VXB_OK;
}

}  // namespace vxb
