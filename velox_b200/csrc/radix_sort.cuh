// Stable LSD radix sort of (uint64 key, uint32 value) pairs on the device.
//
// Replaces the reference's thrust::sort_by_key (src/backend_cuda.cu:514-522).
// Each pass sorts one 8-bit digit in three launches:
//   histogram  per-tile digit counts, tiles staged in shared memory with
//              128-bit loads
//   scan       exclusive scan of the digit-major count matrix (one block)
//   scatter    stable scatter: tiles re-staged with 128-bit loads, ranked with
//              warp __match_any_sync + per-warp digit counts
// Only the digits inside [beginBit, endBit) are sorted, so a key space of
// b bits costs ceil(b/8) passes.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace vxb {

constexpr int kSortThreads = 256;
constexpr int kSortTile = 2048;  // keys per tile (16 KB of keys in shared memory)

struct RadixScratch {
    uint64_t* keysAlt = nullptr;
    uint32_t* valsAlt = nullptr;
    uint32_t* hist = nullptr;  // 256 * tiles
    size_t capacity = 0;       // elements
    size_t histCapacity = 0;   // entries
};

// Sorts keys/vals in place (using scratch as the ping-pong buffer). Returns
// the number of kernel launches issued.
int radixSortPairs(uint64_t* keys, uint32_t* vals, uint32_t n, int beginBit, int endBit,
                   RadixScratch& scratch, cudaStream_t stream, cudaError_t* err);

// Loads the sort's kernels on the current device now (cudaFuncGetAttributes),
// so that a later sort does not load them lazily (which allocates device
// memory) on its first launch.
cudaError_t radixSortPreload();

// Bits needed to represent `maxKey`.
inline int keyBits(uint64_t maxKey) {
    int b = 0;
    while (b < 64 && (maxKey >> b) != 0) ++b;
    return b;
}

}  // namespace vxb
