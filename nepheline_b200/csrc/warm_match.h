/* SPDX-License-Identifier: Apache-2.0
 *
 * Warm-start matching of a contact's points from one step to the next, as the reference's
 * contact update does for a pair of convex shapes (phys_contact_update, contact.c:516-565;
 * warm_by_id and warm_by_place, contact.c:332-380): a new point takes the impulses of last
 * step's point with its feature id; then, if some new point found no id and some old point is
 * still unclaimed, each such new point in order takes the nearest unclaimed old point within
 * 2 x the linear slop on both bodies' anchors. The normal impulse and the tangent impulse (a
 * world vector, so a turn of the tangent basis does not matter) carry over; everything else
 * of a point is the narrow phase's. Plain C with the reference's operations: the device
 * kernel and the CPU restatement include it alike.
 */
#ifndef NPH_WARM_MATCH_H
#define NPH_WARM_MATCH_H

#include "nepheline_b200.h"

#if defined(__CUDACC__)
#define NPH_WM __host__ __device__ static inline
#else
#define NPH_WM static inline
#endif

/* WARM_DISTANCE (contact.c:305): twice NPH_PHYSICS_LINEAR_SLOP (types.h:38). */
#define NPH_WARM_DISTANCE (2.0F * 0.005F)

NPH_WM float nph_wm_distance_sq(const float a[3], const float b[3])
{
    const float x = a[0] - b[0], y = a[1] - b[1], z = a[2] - b[2];
    return x * x + y * y + z * z;
}

/* The points of `fresh` (the narrow phase's, impulses zero) take their impulses from `old`
 * (last step's points of the same contact, with their stored impulses). */
NPH_WM void nph_warm_match(const NphGpuContactPoint *old, uint32_t old_count, NphGpuContactPoint *fresh,
                           uint32_t count)
{
    uint32_t claimed = 0U;
    uint32_t unmatched = 0U;
    for (uint32_t i = 0U; i < count; ++i) {
        NphGpuContactPoint *p = &fresh[i];
        uint32_t o = 0U;
        for (; o < old_count; ++o) {
            if (old[o].id == p->id) {
                break;
            }
        }
        if (o < old_count) {
            p->normal_impulse = old[o].normal_impulse;
            p->tangent_impulse[0] = old[o].tangent_impulse[0];
            p->tangent_impulse[1] = old[o].tangent_impulse[1];
            p->tangent_impulse[2] = old[o].tangent_impulse[2];
            claimed |= 1U << o;
        } else {
            unmatched |= 1U << i;
        }
    }
    if (unmatched == 0U || claimed == (1U << old_count) - 1U) {
        return;
    }
    for (uint32_t i = 0U; i < count; ++i) {
        if ((unmatched & (1U << i)) == 0U) {
            continue;
        }
        NphGpuContactPoint *p = &fresh[i];
        uint32_t best = NPH_GPU_NULL;
        float best_d = NPH_WARM_DISTANCE * NPH_WARM_DISTANCE;
        for (uint32_t o = 0U; o < old_count; ++o) {
            if ((claimed & (1U << o)) != 0U) {
                continue;
            }
            const float da = nph_wm_distance_sq(old[o].anchor_a, p->anchor_a);
            const float db = nph_wm_distance_sq(old[o].anchor_b, p->anchor_b);
            const float d = da > db ? da : db;
            if (d < best_d) {
                best_d = d;
                best = o;
            }
        }
        if (best != NPH_GPU_NULL) {
            p->normal_impulse = old[best].normal_impulse;
            p->tangent_impulse[0] = old[best].tangent_impulse[0];
            p->tangent_impulse[1] = old[best].tangent_impulse[1];
            p->tangent_impulse[2] = old[best].tangent_impulse[2];
            claimed |= 1U << best;
        }
    }
}

/* A contact's record for this step: the pair and its flags (the HIT flag the last solve
 * stored) from last step's record, the manifold (normal, surface, points) from the narrow
 * phase's, the points warm-started from last step's. */
NPH_WM void nph_warm_update(const NphGpuContact *old, const NphGpuContact *fresh, NphGpuContact *out)
{
    NphGpuContact c = *fresh;
    c.body_a = old->body_a;
    c.body_b = old->body_b;
    c.flags = old->flags;
    const uint32_t oc = old->point_count <= NPH_GPU_MAX_POINTS ? old->point_count : 0U;
    const uint32_t nc = c.point_count <= NPH_GPU_MAX_POINTS ? c.point_count : 0U;
    nph_warm_match(old->points, oc, c.points, nc);
    *out = c;
}

#endif /* NPH_WARM_MATCH_H */
