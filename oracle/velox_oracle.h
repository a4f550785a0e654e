/*
 * Test infrastructure: a plain-C restatement of the integer / ordering stages
 * of the reference's per-step contact pipeline, used as an independent
 * checker next to the reference build itself (oracle/_ref). Nothing in the
 * product links it. Each function cites the reference code it restates.
 */
#ifndef VELOX_ORACLE_H
#define VELOX_ORACLE_H

#include "velox_b200_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Swept AABB of one body (src/narrowphase.h:369-398); planes are unbounded. */
void vxo_body_aabb(const vx_body* b, float dt, float lo[3], float hi[3]);

/* Candidate pair set of the reference CUDA backend's broad phase
 * (src/backend_cuda.cu:174-299): every i<j whose AABBs overlap, not both
 * inert (static or fully asleep), passing canCollideWith (body.h:196-202).
 * Written ascending as (i<<32)|j; returns the total (may exceed cap). */
uint32_t vxo_candidate_pairs(const vx_body* bodies, uint32_t n, float dt, uint64_t* out, uint32_t cap);

/* Stable sort by (a, b, point.x, point.y, point.z) — the deterministic contact
 * order of src/backend_cuda.cu:587-595. */
void vxo_sort_contacts(vx_contact* contacts, uint32_t m);

/* Greedy first-free-bit colouring with the >64-colour spill rule
 * (src/backend_cuda.cu:603-630). Returns the colour count. */
uint32_t vxo_color_contacts(const vx_body* bodies, uint32_t n, const vx_contact* contacts, uint32_t m,
                            int32_t* colorOf);

/* Counting sort into colour order (src/backend_cuda.cu:634-640): order[k] is
 * the input index of the k-th contact of the colour-ordered list;
 * colorStart has numColors + 1 entries. */
void vxo_color_order(const int32_t* colorOf, uint32_t m, uint32_t numColors, uint32_t* order,
                     uint32_t* colorStart);

/* Warm-start matching against the previous step's contacts sorted by
 * (a<<32|b) (src/world.cpp:4133-4184): feature-key match copies all six
 * impulses (and the fast-approach vn0), otherwise the vn0 carry and the
 * nearest previous point within 5 cm. Returns the number of contacts that
 * inherited impulses. */
uint32_t vxo_warm_start_match(vx_contact* cur, uint32_t m, const vx_contact* prev, uint32_t mPrev);

#ifdef __cplusplus
}
#endif
#endif
