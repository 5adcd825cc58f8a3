// eph_plan.h - host-side planning shared by the context entry points (eph_capi.cu) and the
// fixed-scratch entry point (eph_noalloc.cu): body classes, per-body work estimates, the automatic launch
// shape and the split of bodies over CTAs. Everything works on caller-provided arrays and allocates nothing.
#pragma once
#include <algorithm>
#include <cstddef>

#include "eph_system.cuh"
#include "../../include/eph_planes.h"

namespace eph {

// Body class of the device ordering (eph_system.cuh): full if any term beyond point-mass Newtonian + 1PN
// can be nonzero for the body, as source or as target. `pl` is planes[EPH_NPLANES][n].
inline bool plan_full_class(const double *pl, int n, int i) {
    auto P = [&](int p) { return pl[(size_t)p * n + i]; };
    if (P(EPH_P_K2) != 0 || P(EPH_P_K2R) != 0 || P(EPH_P_DJ2) != 0 || P(EPH_P_LUM) != 0 || P(EPH_P_RR2G_4C) != 0)
        return true;
    if (P(EPH_P_GP_INDEX) >= 0 || P(EPH_P_RING_INDEX) >= 0) return true;
    for (int q = 0; q < 9; ++q)
        if (P(EPH_P_C_STATIC + q) != 0) return true;
    for (int c = 0; c < 3; ++c)
        if (P(EPH_P_W + c) != 0 || P(EPH_P_GL_HI + c) != 0 || P(EPH_P_GL_LO + c) != 0) return true;
    return false;
}

// Work estimate of one body, in units of a point-like body's pass-A pair sweep. A delayed tide costs up to
// four pass-A sweeps (the angular-velocity fixed point re-sweeps it) of a pair term about ten times as
// expensive as the point-mass one, and those sweeps sit on the stage's critical path, so such a body is
// weighted to end up alone in its CTA whenever the grid has room; pass B adds a little per body.
inline double plan_cost(const double *pl, int n, int i, bool full) {
    const bool delayed = pl[(size_t)EPH_P_K2 * n + i] != 0 && pl[(size_t)EPH_P_TIDE_DELAY * n + i] != 0;
    if (delayed) return 46.0;
    return full ? 5.0 : 3.0;
}

// Automatic launch shape for n bodies with at most `maxc` co-resident CTAs: one CTA per SM slot when
// there are enough bodies to spread, each CTA taking up to kOwnMax bodies (the split decides how many).
// A requested grid or bodies-per-CTA (> 0) overrides the choice. Returns false if the request cannot be
// met with co-resident CTAs.
inline bool plan_shape(int n, int maxc, int req_grid, int req_per, int *grid_out, int *per_out) {
    int per = req_per, grid = req_grid;
    if (per <= 0 && grid <= 0) {
        grid = std::min(maxc, n);
        per = (n + grid - 1) / grid;
        grid = (n + per - 1) / per;
        if (n > 64 && grid < maxc) grid = std::min(maxc, n);   // spread work when every SM can take some
        per = kOwnMax;
    } else if (per <= 0) {
        per = (n + grid - 1) / grid;
    } else if (grid <= 0) {
        grid = (n + per - 1) / per;
    }
    per = std::max(1, std::min(per, (int)kOwnMax));
    grid = std::max(grid, (n + per - 1) / per);
    if (grid > maxc) return false;
    *grid_out = grid;
    *per_out = per;
    return true;
}

// Split bodies over CTAs: longest-processing-time-first into `grid` bins of at most `cap` bodies, ties in
// body order; each CTA's list sorted by body index. own[grid][kOwnMax] is -1 padded. Work arrays:
// order[n], load[grid], cnt[grid].
inline void plan_ownership(const double *cost, int n, int grid, int cap, int *order, double *load, int *cnt,
                           int *own) {
    for (int i = 0; i < n; ++i) order[i] = i;
    std::sort(order, order + n, [&](int a, int b) { return cost[a] > cost[b] || (cost[a] == cost[b] && a < b); });
    std::fill(own, own + (size_t)grid * kOwnMax, -1);
    std::fill(load, load + grid, 0.0);
    std::fill(cnt, cnt + grid, 0);
    for (int q = 0; q < n; ++q) {
        const int i = order[q];
        int best = -1;
        for (int g = 0; g < grid; ++g) {
            if (cnt[g] >= cap) continue;
            if (best < 0 || load[g] < load[best]) best = g;
        }
        own[(size_t)best * kOwnMax + cnt[best]++] = i;
        load[best] += cost[i];
    }
    for (int g = 0; g < grid; ++g) std::sort(own + (size_t)g * kOwnMax, own + (size_t)g * kOwnMax + cnt[g]);
}

}  // namespace eph
