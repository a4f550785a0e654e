// Broad-phase candidate pairs without any allocation.
//
// Who needs this: callers that must not allocate device memory at call time —
// frame-locked game or simulation loops whose device memory budget is fixed
// up front, plugin hosts that own all device memory, or code that runs while
// the device is nearly full. For them a cudaMalloc inside the call could fail
// or stall the frame (it synchronises the device). This entry point takes
// host inputs and outputs and keeps every device byte it touches in one
// file-scope __device__ array of a fixed size, resolved once per device.
//
// Limits (kMaxBodies etc. below): 4,096 bodies, 32,768 body-body pairs and
// 8,192 body-plane pairs per call; larger requests are rejected with
// VXB_ERR_CAPACITY before any device work. The array (about 4.3 MB) is held
// on every device that loads the library until the process exits.
//
// The first call on a device is its set-up: it resolves the array's device
// address and loads every kernel the entry point launches. With CUDA's lazy
// module loading (the default) loading a module allocates device memory, so
// that first call may allocate; calls after it on the same device do not.
// Make the first call before any stream capture. A device reset
// (cudaDeviceReset) discards the loaded module: do not call the entry point
// on that device again in the same process.
#include <atomic>
#include <cstring>
#include <mutex>

#include "broadphase_kernels.cuh"

namespace vxb {
namespace {

constexpr uint32_t kMaxBodies = 4096;
constexpr uint32_t kMaxPairs = 32768;       // body-body candidate pairs
constexpr uint32_t kMaxPlanePairs = 8192;   // body-plane candidate pairs
constexpr uint32_t kMaxAllPairs = kMaxPairs + kMaxPlanePairs;
constexpr uint32_t kHashCap = 2 * kMaxBodies;  // power of two >= 2 * bodies
constexpr uint32_t kMaxDevices = 64;

constexpr size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Byte offsets of the regions inside the scratch array.
constexpr size_t kOffAos = 0;
constexpr size_t kOffSoa = kOffAos + align256((size_t)kMaxBodies * sizeof(vx_body));
constexpr size_t kSoaArray = align256((size_t)kMaxBodies * 16);
constexpr size_t kOffAabb = kOffSoa + 16 * kSoaArray;
constexpr size_t kOffKeys = kOffAabb + align256((size_t)kMaxBodies * 32);
constexpr size_t kOffVals = kOffKeys + align256((size_t)kMaxAllPairs * 8);
constexpr size_t kOffKeysAlt = kOffVals + align256((size_t)kMaxAllPairs * 4);
constexpr size_t kOffValsAlt = kOffKeysAlt + align256((size_t)kMaxAllPairs * 8);
constexpr size_t kOffHist = kOffValsAlt + align256((size_t)kMaxAllPairs * 4);
constexpr size_t kOffHashKeys =
    kOffHist + align256((size_t)256 * ((kMaxAllPairs + kSortTile - 1) / kSortTile) * 4);
constexpr size_t kOffHashVals = kOffHashKeys + align256((size_t)kHashCap * 8);
constexpr size_t kOffPlanes = kOffHashVals + align256((size_t)kHashCap * 4);
constexpr size_t kOffPairs = kOffPlanes + align256((size_t)(kMaxBodies + 2) * 4);
constexpr size_t kOffPlanePairs = kOffPairs + align256((size_t)kMaxPairs * 8);
constexpr size_t kOffOut = kOffPlanePairs + align256((size_t)kMaxPlanePairs * 8);
constexpr size_t kOffCounters = kOffOut + align256((size_t)kMaxAllPairs * 8);
constexpr size_t kScratchBytes = kOffCounters + align256(sizeof(Counters));

// The only device memory this entry point uses. Every call shares it: calls
// that overlap on the GPU (other threads, other streams) race on it.
static __device__ __align__(256) unsigned char g_noallocScratch[kScratchBytes];

// Device address of g_noallocScratch per device, resolved on the first call
// made on that device (with it current). In host code the array's name is
// only a host-side stand-in; kernels must get this address instead. Host
// threads may make first calls concurrently: the set-up runs under a mutex and
// publishes the address atomically.
std::atomic<unsigned char*> g_scratchAddress[kMaxDevices] = {};
std::mutex g_setupMutex;

// Pair (i, j) compressed to 24 bits for the output sort (i, j < 4096).
__global__ void packPairKeysKernel(const uint64_t* convex, uint32_t nc, const uint64_t* plane, uint32_t np,
                                   uint64_t* keys, uint32_t* vals) {
    const uint32_t total = nc + np;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < total; k += gridDim.x * blockDim.x) {
        const uint64_t p = k < nc ? convex[k] : plane[k - nc];
        keys[k] = ((p >> 32) << 12) | (p & 0xfffu);
        vals[k] = k;
    }
}

__global__ void unpackPairKeysKernel(const uint64_t* keys, uint32_t total, uint64_t* out) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < total; k += gridDim.x * blockDim.x)
        out[k] = ((keys[k] >> 12) << 32) | (keys[k] & 0xfffu);
}

int cudaToStatus(cudaError_t e) {
    if (e == cudaSuccess) return VXB_OK;
    cudaGetLastError();
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return VXB_ERR_NO_DEVICE;
    if (e == cudaErrorLaunchFailure || e == cudaErrorIllegalAddress || e == cudaErrorUnknown)
        return VXB_ERR_DEVICE_LOST;
    return VXB_ERR_INVALID;
}

#define NA_CUDA(expr)                                   \
    do {                                                \
        const int s_ = cudaToStatus(expr);              \
        if (s_ != VXB_OK) return s_;                    \
    } while (0)

// Set-up of one device (current): the array's address, and every kernel
// this entry point launches loaded now rather than at its first launch.
int setupDevice(int device, unsigned char** base) {
    std::lock_guard<std::mutex> lock(g_setupMutex);
    unsigned char* known = g_scratchAddress[device].load(std::memory_order_acquire);
    if (known) {
        *base = known;
        return VXB_OK;
    }
    void* address = nullptr;
    NA_CUDA(cudaGetSymbolAddress(&address, g_noallocScratch));
    cudaFuncAttributes a;
    NA_CUDA(cudaFuncGetAttributes(&a, packBodiesKernel));
    NA_CUDA(cudaFuncGetAttributes(&a, aabbKernel));
    NA_CUDA(cudaFuncGetAttributes(&a, keyKernel));
    NA_CUDA(cudaFuncGetAttributes(&a, cellTableKernel));
    NA_CUDA(cudaFuncGetAttributes(&a, pairKernel));
    NA_CUDA(cudaFuncGetAttributes(&a, packPairKeysKernel));
    NA_CUDA(cudaFuncGetAttributes(&a, unpackPairKeysKernel));
    NA_CUDA(radixSortPreload());
    *base = static_cast<unsigned char*>(address);
    g_scratchAddress[device].store(*base, std::memory_order_release);
    return VXB_OK;
}

}  // namespace
}  // namespace vxb

extern "C" int vxb_stage_pairs_noalloc(const vx_body* bodies, uint32_t n, float dt, uint64_t* out, uint32_t cap,
                                       uint32_t* count, void* stream) {
    using namespace vxb;
    if (!bodies || !count || n == 0) return VXB_ERR_INVALID;
    *count = 0;
    if (n > kMaxBodies) return VXB_ERR_CAPACITY;
    uint32_t planeList[kMaxBodies];
    uint32_t planes = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const uint8_t s = bodies[i].shape;
        if (s == VX_SHAPE_MESH || s == VX_SHAPE_COMPOUND || bodies[i].motionType == VX_MOTION_KINEMATIC)
            return VXB_ERR_UNSUPPORTED;  // same body set as vxb_stage_pairs accepts
        if (s == VX_SHAPE_PLANE) planeList[planes++] = i;
    }
    if ((uint64_t)(n - planes) * planes > kMaxPlanePairs) return VXB_ERR_CAPACITY;

    int device = 0;
    NA_CUDA(cudaGetDevice(&device));
    if (device < 0 || device >= (int)kMaxDevices) return VXB_ERR_INVALID;
    unsigned char* base = g_scratchAddress[device].load(std::memory_order_acquire);
    if (!base) {
        const int status = setupDevice(device, &base);
        if (status != VXB_OK) return status;
    }
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);

    vx_body* aos = reinterpret_cast<vx_body*>(base + kOffAos);
    BodyArrays B;
    float4** f4[] = {&B.pos, &B.rot, &B.vel, &B.ang, &B.inertia, &B.iq, &B.dims, &B.extra,
                     &B.mat, &B.fscale, &B.ccd, &B.plane, &B.force, &B.torque};
    int slot = 0;
    for (float4** p : f4) *p = reinterpret_cast<float4*>(base + kOffSoa + kSoaArray * slot++);
    B.hull = reinterpret_cast<uint4*>(base + kOffSoa + kSoaArray * slot++);
    B.filt = reinterpret_cast<uint4*>(base + kOffSoa + kSoaArray * slot++);
    float4* lo = reinterpret_cast<float4*>(base + kOffAabb);
    float4* hi = lo + kMaxBodies;
    uint64_t* keys = reinterpret_cast<uint64_t*>(base + kOffKeys);
    uint32_t* vals = reinterpret_cast<uint32_t*>(base + kOffVals);
    RadixScratch rs;
    rs.keysAlt = reinterpret_cast<uint64_t*>(base + kOffKeysAlt);
    rs.valsAlt = reinterpret_cast<uint32_t*>(base + kOffValsAlt);
    rs.hist = reinterpret_cast<uint32_t*>(base + kOffHist);
    uint64_t* hk = reinterpret_cast<uint64_t*>(base + kOffHashKeys);
    uint32_t* hv = reinterpret_cast<uint32_t*>(base + kOffHashVals);
    uint32_t* planeStart = reinterpret_cast<uint32_t*>(base + kOffPlanes);
    uint32_t* planeDev = planeStart + 2;
    uint64_t* pairs = reinterpret_cast<uint64_t*>(base + kOffPairs);
    uint64_t* planePairs = reinterpret_cast<uint64_t*>(base + kOffPlanePairs);
    uint64_t* outDev = reinterpret_cast<uint64_t*>(base + kOffOut);
    Counters* C = reinterpret_cast<Counters*>(base + kOffCounters);

    // Everything that must start from a known state is reset on every call:
    // the counters, the cell hash table and the plane list.
    Counters zero;
    std::memset(&zero, 0, sizeof(zero));
    for (int a = 0; a < 3; ++a) zero.cellMinBits[a] = 0xffffffffu;
    const uint32_t planeRange[2] = {0u, planes};
    NA_CUDA(cudaMemcpyAsync(C, &zero, sizeof(zero), cudaMemcpyHostToDevice, st));
    NA_CUDA(cudaMemcpyAsync(planeStart, planeRange, sizeof(planeRange), cudaMemcpyHostToDevice, st));
    if (planes) NA_CUDA(cudaMemcpyAsync(planeDev, planeList, planes * 4, cudaMemcpyHostToDevice, st));
    NA_CUDA(cudaMemsetAsync(hk, 0xff, (size_t)kHashCap * 8, st));
    NA_CUDA(cudaMemcpyAsync(aos, bodies, (size_t)n * sizeof(vx_body), cudaMemcpyHostToDevice, st));

    const uint32_t blocks = (n + 255) / 256;
    packBodiesKernel<<<blocks, 256, 0, st>>>(aos, n, B);
    aabbKernel<<<blocks, 256, 0, st>>>(B, n, dt, nullptr, lo, hi, C);  // mesh bodies are rejected above
    const uint64_t planeKey = 1ull << (3 * kCellBitsPerAxis);
    keyKernel<<<blocks, 256, 0, st>>>(B, n, nullptr, lo, hi, C, keys, vals, planeKey);
    cudaError_t e = cudaSuccess;
    radixSortPairs(keys, vals, n, 0, 3 * kCellBitsPerAxis + 1, rs, st, &e);
    NA_CUDA(e);
    cellTableKernel<<<blocks, 256, 0, st>>>(keys, n, planeKey, hk, hv, kHashCap - 1);
    pairKernel<<<(n + 127) / 128, 128, 0, st>>>(B, n, keys, vals, lo, hi, hk, hv, kHashCap - 1, planeKey, nullptr,
                                              planeStart, planeDev, pairs, kMaxPairs, planePairs, kMaxPlanePairs, C);
    Counters got;
    NA_CUDA(cudaMemcpyAsync(&got, C, sizeof(got), cudaMemcpyDeviceToHost, st));
    NA_CUDA(cudaStreamSynchronize(st));
    const uint32_t total = got.pairs + got.planePairs;
    *count = total;
    if (got.pairs > kMaxPairs || got.planePairs > kMaxPlanePairs) return VXB_ERR_CAPACITY;
    if (total == 0) return VXB_OK;
    if (!out || total > cap) return VXB_ERR_CAPACITY;
    // Ascending (i << 32 | j) order, sorted on the device.
    packPairKeysKernel<<<(total + 255) / 256, 256, 0, st>>>(pairs, got.pairs, planePairs, got.planePairs, keys, vals);
    radixSortPairs(keys, vals, total, 0, 24, rs, st, &e);
    NA_CUDA(e);
    unpackPairKeysKernel<<<(total + 255) / 256, 256, 0, st>>>(keys, total, outDev);
    NA_CUDA(cudaMemcpyAsync(out, outDev, (size_t)total * 8, cudaMemcpyDeviceToHost, st));
    NA_CUDA(cudaStreamSynchronize(st));
    return cudaToStatus(cudaGetLastError());
}
