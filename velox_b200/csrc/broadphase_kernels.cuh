// Declarations of the broad-phase kernels defined in pipeline.cu, for host
// code in other translation units that launches them with its own buffers.
#pragma once
#include "context.cuh"

namespace vxb {

constexpr int kCellBitsPerAxis = 10;  // must equal pipeline.cu's kCellBits

__global__ void packBodiesKernel(const vx_body* __restrict__ in, uint32_t n, BodyArrays B);
// meshes: the soup's mesh records (read for mesh bodies only; may be null
// when no mesh body is loaded)
__global__ void aabbKernel(BodyArrays B, uint32_t n, float dt, const vx_mesh* meshes, float4* lo, float4* hi,
                           Counters* C);
__global__ void keyKernel(BodyArrays B, uint32_t n, const uint32_t* worldOf, const float4* lo, const float4* hi,
                          const Counters* C, uint64_t* keys, uint32_t* vals, uint64_t planeKey);
__global__ void cellTableKernel(const uint64_t* keys, uint32_t n, uint64_t planeKey, uint64_t* hk, uint32_t* hv,
                                uint32_t mask);
__global__ void pairKernel(BodyArrays B, uint32_t n, const uint64_t* keys, const uint32_t* vals, const float4* lo,
                           const float4* hi, const uint64_t* hk, const uint32_t* hv, uint32_t mask, uint64_t planeKey,
                           const uint32_t* worldOf, const uint32_t* planeStart, const uint32_t* planeList,
                           uint64_t* pairs, uint32_t cap, uint64_t* planePairs, uint32_t planeCap, Counters* C);

}  // namespace vxb
