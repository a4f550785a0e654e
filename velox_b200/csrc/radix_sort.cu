#include "radix_sort.cuh"

#include <cstdint>

namespace vxb {

namespace {

constexpr int kWarps = kSortThreads / 32;

__device__ __forceinline__ bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// Stage [base, base + count) of keys into shared memory with 16-byte loads
// when the address is 16-byte aligned (callers may pass sub-buffers).
__device__ void stageKeys(const uint64_t* __restrict__ keys, uint32_t base, uint32_t count,
                          uint64_t* sk) {
    const uint32_t pairs = count / 2;
    if (aligned16(keys + base)) {
        const ulonglong2* src = reinterpret_cast<const ulonglong2*>(keys + base);
        for (uint32_t i = threadIdx.x; i < pairs; i += blockDim.x) {
            ulonglong2 v = src[i];
            sk[2 * i] = v.x;
            sk[2 * i + 1] = v.y;
        }
        if ((count & 1u) && threadIdx.x == 0) sk[count - 1] = keys[base + count - 1];
    } else {
        for (uint32_t i = threadIdx.x; i < count; i += blockDim.x) sk[i] = keys[base + i];
    }
}

__global__ void histogramKernel(const uint64_t* __restrict__ keys, uint32_t n, int shift,
                                uint32_t tiles, uint32_t* __restrict__ hist) {
    __shared__ uint64_t sk[kSortTile];
    __shared__ uint32_t counts[256];
    const uint32_t tile = blockIdx.x;
    const uint32_t base = tile * kSortTile;
    const uint32_t count = min((uint32_t)kSortTile, n - base);
    for (int i = threadIdx.x; i < 256; i += blockDim.x) counts[i] = 0;
    stageKeys(keys, base, count, sk);
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < count; i += blockDim.x)
        atomicAdd(&counts[(sk[i] >> shift) & 255u], 1u);
    __syncthreads();
    for (int d = threadIdx.x; d < 256; d += blockDim.x) hist[d * tiles + tile] = counts[d];
}

// Exclusive scan of `len` counts in place (single block): each thread scans
// a contiguous segment, segment sums are combined with warp shuffles.
__global__ void scanKernel(uint32_t* __restrict__ data, uint32_t len) {
    __shared__ uint32_t warpSums[32];
    const uint32_t per = (len + blockDim.x - 1) / blockDim.x;
    const uint32_t begin = min(len, threadIdx.x * per), end = min(len, begin + per);
    uint32_t sum = 0;
    for (uint32_t i = begin; i < end; ++i) sum += data[i];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = sum;
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, off);
        if (lane >= off) x += y;
    }
    if (lane == 31) warpSums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        uint32_t w = lane < nw ? warpSums[lane] : 0u;
        for (int off = 1; off < 32; off <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, off);
            if (lane >= off) w += y;
        }
        warpSums[lane] = w;
    }
    __syncthreads();
    uint32_t prefix = x - sum + (warp > 0 ? warpSums[warp - 1] : 0u);
    for (uint32_t i = begin; i < end; ++i) {
        const uint32_t v = data[i];
        data[i] = prefix;
        prefix += v;
    }
}

__global__ void scatterKernel(const uint64_t* __restrict__ keysIn, const uint32_t* __restrict__ valsIn,
                              uint64_t* __restrict__ keysOut, uint32_t* __restrict__ valsOut, uint32_t n,
                              int shift, uint32_t tiles, const uint32_t* __restrict__ offsets) {
    __shared__ uint64_t sk[kSortTile];
    __shared__ uint32_t sv[kSortTile];
    __shared__ uint32_t running[256];
    __shared__ uint32_t warpCounts[kWarps][256];
    __shared__ uint32_t chunkTotal[256];
    const uint32_t tile = blockIdx.x;
    const uint32_t base = tile * kSortTile;
    const uint32_t count = min((uint32_t)kSortTile, n - base);
    stageKeys(keysIn, base, count, sk);
    if (aligned16(valsIn + base)) {
        const uint4* src = reinterpret_cast<const uint4*>(valsIn + base);
        for (uint32_t i = threadIdx.x; i < count / 4; i += blockDim.x) {
            uint4 v = src[i];
            sv[4 * i] = v.x; sv[4 * i + 1] = v.y; sv[4 * i + 2] = v.z; sv[4 * i + 3] = v.w;
        }
        for (uint32_t i = (count / 4) * 4 + threadIdx.x; i < count; i += blockDim.x) sv[i] = valsIn[base + i];
    } else {
        for (uint32_t i = threadIdx.x; i < count; i += blockDim.x) sv[i] = valsIn[base + i];
    }
    for (int d = threadIdx.x; d < 256; d += blockDim.x) running[d] = offsets[d * tiles + tile];
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    for (uint32_t chunk = 0; chunk < count; chunk += blockDim.x) {
        const uint32_t i = chunk + threadIdx.x;
        const bool valid = i < count;
        const uint32_t digit = valid ? (uint32_t)((sk[i] >> shift) & 255u) : 256u + lane;
        const unsigned peers = __match_any_sync(0xffffffffu, digit);
        const uint32_t rank = __popc(peers & lt);
        for (int d = threadIdx.x; d < kWarps * 256; d += blockDim.x) (&warpCounts[0][0])[d] = 0;
        __syncthreads();
        if (valid && rank == 0) warpCounts[warp][digit] = __popc(peers);
        __syncthreads();
        // Per digit: exclusive prefix over warps (in place) and chunk total.
        for (int d = threadIdx.x; d < 256; d += blockDim.x) {
            uint32_t sum = 0;
            for (int w = 0; w < kWarps; ++w) {
                const uint32_t c = warpCounts[w][d];
                warpCounts[w][d] = sum;
                sum += c;
            }
            chunkTotal[d] = sum;
        }
        __syncthreads();
        if (valid) {
            const uint32_t pos = running[digit] + warpCounts[warp][digit] + rank;
            keysOut[pos] = sk[i];
            valsOut[pos] = sv[i];
        }
        __syncthreads();
        for (int d = threadIdx.x; d < 256; d += blockDim.x) running[d] += chunkTotal[d];
        __syncthreads();
    }
}

}  // namespace

cudaError_t radixSortPreload() {
    cudaFuncAttributes a;
    cudaError_t e = cudaFuncGetAttributes(&a, histogramKernel);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&a, scanKernel);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&a, scatterKernel);
    return e;
}

int radixSortPairs(uint64_t* keys, uint32_t* vals, uint32_t n, int beginBit, int endBit,
                   RadixScratch& s, cudaStream_t stream, cudaError_t* err) {
    int launches = 0;
    if (n <= 1 || endBit <= beginBit) return 0;
    const uint32_t tiles = (n + kSortTile - 1) / kSortTile;
    uint64_t* kin = keys;
    uint32_t* vin = vals;
    uint64_t* kout = s.keysAlt;
    uint32_t* vout = s.valsAlt;
    for (int shift = beginBit; shift < endBit; shift += 8) {
        histogramKernel<<<tiles, kSortThreads, 0, stream>>>(kin, n, shift, tiles, s.hist);
        scanKernel<<<1, 1024, 0, stream>>>(s.hist, 256u * tiles);
        scatterKernel<<<tiles, kSortThreads, 0, stream>>>(kin, vin, kout, vout, n, shift, tiles, s.hist);
        launches += 3;
        uint64_t* tk = kin; kin = kout; kout = tk;
        uint32_t* tv = vin; vin = vout; vout = tv;
    }
    if (kin != keys) {
        cudaMemcpyAsync(keys, kin, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, stream);
        cudaMemcpyAsync(vals, vin, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, stream);
    }
    if (err) *err = cudaGetLastError();
    return launches;
}

}  // namespace vxb
