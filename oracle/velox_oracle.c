/*
 * Test infrastructure: plain-C restatement of the ordering / integer stages of
 * the reference's per-step contact pipeline (see velox_oracle.h). Compiled
 * with -ffp-contract=off so its few float expressions round like the
 * reference's strict build.
 */
#include "velox_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static float vo_max(float a, float b) { return a > b ? a : b; }
static float vo_len(float x, float y, float z) { return sqrtf(x * x + y * y + z * z); }

/* Body::maxPointSpeed, include/velox/body.h:329-344 */
static float vo_max_point_speed(const vx_body* b) {
    float r = b->radius;
    const float hx = b->halfExtents.x, hy = b->halfExtents.y, hz = b->halfExtents.z;
    switch (b->shape) {
    case VX_SHAPE_BOX: r = vo_len(hx, hy, hz); break;
    case VX_SHAPE_ROUNDED_BOX: r = vo_len(hx, hy, hz) + b->radius; break;
    case VX_SHAPE_ELLIPSOID: r = vo_max(hx, vo_max(hy, hz)); break;
    case VX_SHAPE_CAPSULE: r = b->capsuleHalfHeight + b->radius; break;
    case VX_SHAPE_CYLINDER:
        r = sqrtf(b->capsuleHalfHeight * b->capsuleHalfHeight + b->radius * b->radius);
        break;
    case VX_SHAPE_CONE: {
        float top = 1.5f * b->capsuleHalfHeight;
        r = vo_max(top, sqrtf(b->radius * b->radius + 0.25f * b->capsuleHalfHeight * b->capsuleHalfHeight));
        break;
    }
    default: break;
    }
    return vo_len(b->velocity.x, b->velocity.y, b->velocity.z) +
           vo_len(b->angularVelocity.x, b->angularVelocity.y, b->angularVelocity.z) * r;
}

/* bodyAabb, src/narrowphase.h:369-398 */
void vxo_body_aabb(const vx_body* b, float dt, float lo[3], float hi[3]) {
    if (b->shape == VX_SHAPE_PLANE) {
        for (int a = 0; a < 3; ++a) { lo[a] = -1e30f; hi[a] = 1e30f; }
        return;
    }
    const float hx = b->halfExtents.x, hy = b->halfExtents.y, hz = b->halfExtents.z;
    float ext;
    switch (b->shape) {
    case VX_SHAPE_BOX: ext = vo_len(hx, hy, hz); break;
    case VX_SHAPE_ROUNDED_BOX: ext = vo_len(hx, hy, hz) + b->radius; break;
    case VX_SHAPE_ELLIPSOID: ext = vo_max(hx, vo_max(hy, hz)); break;
    case VX_SHAPE_CAPSULE: ext = b->capsuleHalfHeight + b->radius; break;
    case VX_SHAPE_SPHERE: case VX_SHAPE_HULL: case VX_SHAPE_COMPOUND: ext = b->radius; break;
    case VX_SHAPE_CYLINDER:
        ext = sqrtf(b->radius * b->radius + b->capsuleHalfHeight * b->capsuleHalfHeight);
        break;
    case VX_SHAPE_CONE: {
        float top = 1.5f * b->capsuleHalfHeight;
        ext = vo_max(top, sqrtf(b->radius * b->radius + 0.25f * b->capsuleHalfHeight * b->capsuleHalfHeight));
        break;
    }
    default: ext = 0.0f; break;
    }
    const int continuous = b->ccdTuning.enableContinuous && b->ccdTuning.quality != VX_QUALITY_LOW &&
                           b->ccdTuning.quality != VX_QUALITY_LOCKED;
    const float sweep = continuous ? vo_max_point_speed(b) * dt : 0.0f;
    const float reach = ext + sweep + b->ccdTuning.collisionMargin + 1e-2f;
    const float p[3] = {b->position.x, b->position.y, b->position.z};
    for (int a = 0; a < 3; ++a) { lo[a] = p[a] - reach; hi[a] = p[a] + reach; }
}

static int vo_inert(const vx_body* b) { return b->motionType == VX_MOTION_STATIC || b->asleep == 1; }

/* Body::canCollideWith, include/velox/body.h:196-202 */
static int vo_can_collide(const vx_body* a, const vx_body* b) {
    if (a->groupIndex != 0 && a->groupIndex == b->groupIndex) return a->groupIndex > 0;
    return (a->maskBits & b->categoryBits) != 0 && (b->maskBits & a->categoryBits) != 0;
}

static int vo_cmp_u64(const void* x, const void* y) {
    uint64_t a = *(const uint64_t*)x, b = *(const uint64_t*)y;
    return a < b ? -1 : a > b ? 1 : 0;
}

typedef struct { float lo[3], hi[3]; uint32_t index; } vo_box;

static int vo_cmp_box(const void* x, const void* y) {
    const vo_box* a = (const vo_box*)x;
    const vo_box* b = (const vo_box*)y;
    if (a->lo[0] < b->lo[0]) return -1;
    if (a->lo[0] > b->lo[0]) return 1;
    return a->index < b->index ? -1 : a->index > b->index ? 1 : 0;
}

uint32_t vxo_candidate_pairs(const vx_body* bodies, uint32_t n, float dt, uint64_t* out, uint32_t cap) {
    vo_box* boxes = (vo_box*)malloc(sizeof(vo_box) * (n ? n : 1));
    uint32_t* planes = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
    uint32_t nb = 0, np = 0, total = 0, capPairs = 1024;
    uint64_t* pairs = (uint64_t*)malloc(sizeof(uint64_t) * capPairs);
    for (uint32_t i = 0; i < n; ++i) {
        if (bodies[i].shape == VX_SHAPE_PLANE) { planes[np++] = i; continue; }
        vxo_body_aabb(&bodies[i], dt, boxes[nb].lo, boxes[nb].hi);
        boxes[nb].index = i;
        ++nb;
    }
#define VO_EMIT(I, J)                                                               \
    do {                                                                            \
        uint32_t lo_ = (I) < (J) ? (I) : (J), hi_ = (I) < (J) ? (J) : (I);          \
        const vx_body* a_ = &bodies[lo_];                                           \
        const vx_body* b_ = &bodies[hi_];                                           \
        if (!(vo_inert(a_) && vo_inert(b_)) && vo_can_collide(a_, b_)) {            \
            if (total == capPairs) {                                                \
                capPairs *= 2;                                                      \
                pairs = (uint64_t*)realloc(pairs, sizeof(uint64_t) * capPairs);     \
            }                                                                       \
            pairs[total++] = ((uint64_t)lo_ << 32) | hi_;                           \
        }                                                                           \
    } while (0)
    /* planes are unbounded: they pair with every other body */
    for (uint32_t p = 0; p < np; ++p) {
        for (uint32_t k = 0; k < nb; ++k) VO_EMIT(planes[p], boxes[k].index);
        for (uint32_t q = p + 1; q < np; ++q) VO_EMIT(planes[p], planes[q]);
    }
    qsort(boxes, nb, sizeof(vo_box), vo_cmp_box);
    for (uint32_t s = 0; s < nb; ++s)
        for (uint32_t t = s + 1; t < nb; ++t) {
            if (boxes[t].lo[0] > boxes[s].hi[0]) break;
            const vo_box* A = &boxes[s];
            const vo_box* B = &boxes[t];
            if (A->hi[0] >= B->lo[0] && A->lo[0] <= B->hi[0] && A->hi[1] >= B->lo[1] && A->lo[1] <= B->hi[1] &&
                A->hi[2] >= B->lo[2] && A->lo[2] <= B->hi[2])
                VO_EMIT(A->index, B->index);
        }
#undef VO_EMIT
    qsort(pairs, total, sizeof(uint64_t), vo_cmp_u64);
    if (out) memcpy(out, pairs, sizeof(uint64_t) * (total < cap ? total : cap));
    free(pairs);
    free(planes);
    free(boxes);
    return total;
}

static int vo_contact_less(const vx_contact* x, const vx_contact* y) {
    const uint64_t kx = ((uint64_t)x->a << 32) | x->b, ky = ((uint64_t)y->a << 32) | y->b;
    if (kx != ky) return kx < ky;
    if (x->point.x != y->point.x) return x->point.x < y->point.x;
    if (x->point.y != y->point.y) return x->point.y < y->point.y;
    return x->point.z < y->point.z;
}

/* stable merge sort */
void vxo_sort_contacts(vx_contact* c, uint32_t m) {
    if (m < 2) return;
    vx_contact* tmp = (vx_contact*)malloc(sizeof(vx_contact) * m);
    for (uint32_t width = 1; width < m; width *= 2) {
        for (uint32_t lo = 0; lo < m; lo += 2 * width) {
            uint32_t mid = lo + width < m ? lo + width : m;
            uint32_t hi = lo + 2 * width < m ? lo + 2 * width : m;
            uint32_t i = lo, j = mid, k = lo;
            while (i < mid && j < hi) tmp[k++] = vo_contact_less(&c[j], &c[i]) ? c[j++] : c[i++];
            while (i < mid) tmp[k++] = c[i++];
            while (j < hi) tmp[k++] = c[j++];
        }
        memcpy(c, tmp, sizeof(vx_contact) * m);
    }
    free(tmp);
}

uint32_t vxo_color_contacts(const vx_body* bodies, uint32_t n, const vx_contact* contacts, uint32_t m,
                            int32_t* colorOf) {
    uint64_t* mask = (uint64_t*)calloc(n ? n : 1, sizeof(uint64_t));
    int32_t* next = (int32_t*)malloc(sizeof(int32_t) * (n ? n : 1));
    for (uint32_t i = 0; i < n; ++i) next[i] = 64;
    uint32_t colors = 0;
    for (uint32_t k = 0; k < m; ++k) {
        const vx_contact* c = &contacts[k];
        const vx_body* A = &bodies[c->a];
        const vx_body* B = &bodies[c->b];
        const int sensor = A->sensor || B->sensor;
        const int sa = sensor || A->motionType != VX_MOTION_DYNAMIC;
        const int sb = sensor || B->motionType != VX_MOTION_DYNAMIC;
        const uint64_t used = (sa ? 0 : mask[c->a]) | (sb ? 0 : mask[c->b]);
        int32_t color;
        if (~used) {
            color = 0;
            while (used & (1ull << color)) ++color;
        } else {
            int32_t na = sa ? 64 : next[c->a];
            int32_t nb = sb ? 64 : next[c->b];
            color = na > nb ? na : nb;
            if (!sa) next[c->a] = color + 1;
            if (!sb) next[c->b] = color + 1;
        }
        if (color < 64) {
            if (!sa) mask[c->a] |= 1ull << color;
            if (!sb) mask[c->b] |= 1ull << color;
        }
        colorOf[k] = color;
        if ((uint32_t)color + 1 > colors) colors = (uint32_t)color + 1;
    }
    free(next);
    free(mask);
    return colors;
}

void vxo_color_order(const int32_t* colorOf, uint32_t m, uint32_t numColors, uint32_t* order,
                     uint32_t* colorStart) {
    for (uint32_t c = 0; c <= numColors; ++c) colorStart[c] = 0;
    for (uint32_t k = 0; k < m; ++k) ++colorStart[colorOf[k] + 1];
    for (uint32_t c = 0; c < numColors; ++c) colorStart[c + 1] += colorStart[c];
    uint32_t* fill = (uint32_t*)malloc(sizeof(uint32_t) * (numColors + 1));
    memcpy(fill, colorStart, sizeof(uint32_t) * (numColors + 1));
    for (uint32_t k = 0; k < m; ++k) order[fill[colorOf[k]]++] = k;
    free(fill);
}

static void vo_copy_impulses(vx_contact* c, const vx_contact* p) {
    c->normalImpulse = p->normalImpulse;
    c->tangentImpulse1 = p->tangentImpulse1;
    c->tangentImpulse2 = p->tangentImpulse2;
    c->rollingImpulse1 = p->rollingImpulse1;
    c->rollingImpulse2 = p->rollingImpulse2;
    c->spinningImpulse = p->spinningImpulse;
}

uint32_t vxo_warm_start_match(vx_contact* cur, uint32_t m, const vx_contact* prev, uint32_t mPrev) {
    uint32_t warm = 0;
    for (uint32_t k = 0; k < m; ++k) {
        vx_contact* c = &cur[k];
        const uint64_t key = ((uint64_t)c->a << 32) | c->b;
        uint32_t lo = 0, hi = mPrev;
        while (lo < hi) {
            uint32_t mid = (lo + hi) / 2;
            uint64_t pk = ((uint64_t)prev[mid].a << 32) | prev[mid].b;
            if (pk < key) lo = mid + 1; else hi = mid;
        }
        int copied = 0, matched = 0;
        uint32_t it;
        if (c->featureKey != 0)
            for (it = lo; it < mPrev && (((uint64_t)prev[it].a << 32) | prev[it].b) == key; ++it)
                if (prev[it].featureKey == c->featureKey) {
                    vo_copy_impulses(c, &prev[it]);
                    if (c->vn0 < -1.0f && prev[it].vn0 < c->vn0) c->vn0 = prev[it].vn0;
                    matched = copied = 1;
                    break;
                }
        if (!matched) {
            if (c->vn0 < -1.0f)
                for (it = lo; it < mPrev && (((uint64_t)prev[it].a << 32) | prev[it].b) == key; ++it)
                    if (prev[it].vn0 < c->vn0) c->vn0 = prev[it].vn0;
            float best = 2.5e-3f;
            for (it = lo; it < mPrev && (((uint64_t)prev[it].a << 32) | prev[it].b) == key; ++it) {
                const float dx = prev[it].point.x - c->point.x, dy = prev[it].point.y - c->point.y,
                            dz = prev[it].point.z - c->point.z;
                const float d = dx * dx + dy * dy + dz * dz;
                if (d < best) {
                    best = d;
                    vo_copy_impulses(c, &prev[it]);
                    copied = 1;
                }
            }
        }
        warm += (uint32_t)copied;
    }
    return warm;
}
