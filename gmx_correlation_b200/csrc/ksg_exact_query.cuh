// Exact FP64 KSG statistics of one (pair, query), shared by the brute-force
// kernel and the fast path's hand-over queue.  See ksg_exact.cu for the
// reference semantics.
#pragma once

#include "gc_common.cuh"

namespace gc {

// n_x and n_y of query frame i of pair (a1, a2), x = a1.  X: [3*natoms][T]
// normalised rows; hist: 256 words of this warp's shared memory.  All lanes
// get the same values.
__device__ __forceinline__ void exact_query_nxy(const double* __restrict__ X, int T, int K, int a1, int a2, int i,
                                                int box, int rank_shift, unsigned* hist, int lane, int& nx_out,
                                                int& ny_out)
{
    const double* __restrict__ ra0 = X + (size_t)(a1 * 3 + 0) * T;
    const double* __restrict__ ra1 = X + (size_t)(a1 * 3 + 1) * T;
    const double* __restrict__ ra2 = X + (size_t)(a1 * 3 + 2) * T;
    const double* __restrict__ rb0 = X + (size_t)(a2 * 3 + 0) * T;
    const double* __restrict__ rb1 = X + (size_t)(a2 * 3 + 1) * T;
    const double* __restrict__ rb2 = X + (size_t)(a2 * 3 + 2) * T;
    const ScanGrid g(box);
    const double qa0 = ra0[i], qa1 = ra1[i], qa2 = ra2[i];
    const double qb0 = rb0[i], qb1 = rb1[i], qb2 = rb2[i];
    auto dist = [&](int j, double& dx, double& dy) {
        dx = fmax(fmax(fabs(qa0 - ra0[j]), fabs(qa1 - ra1[j])), fabs(qa2 - ra2[j]));
        dy = fmax(fmax(fabs(qb0 - rb0[j]), fabs(qb1 - rb1[j])), fabs(qb2 - rb2[j]));
    };
    auto vkey = [&](int j, unsigned long long& k) -> bool {
        if (j == i)
            return false;
        double dx, dy;
        dist(j, dx, dy);
        k = dbits(fmax(dx, dy));
        return true;
    };
    int                      below;
    const unsigned long long dkb  = warp_select_u64(vkey, T, K, 56, hist, lane, &below);
    const double             dk   = __longlong_as_double((long long)dkb);
    const int                need = K - below;

    int tied = 0;
    for (int j = lane; j < T; j += 32)
    {
        if (j == i)
            continue;
        double dx, dy;
        dist(j, dx, dy);
        tied += fmax(dx, dy) == dk;
    }
    tied = __reduce_add_sync(kFull, tied);

    const int          ix   = g.qcell(qa0), iy = g.qcell(qb0);
    unsigned long long rcut = ~0ull;
    if (tied > need)
    {
        auto rkey = [&](int j, unsigned long long& k) -> bool {
            if (j == i)
                return false;
            double dx, dy;
            dist(j, dx, dy);
            if (fmax(dx, dy) != dk)
                return false;
            k = g.rank(ix, iy, ra0[j], rb0[j], j, T);
            return true;
        };
        int b2;
        rcut = warp_select_u64(rkey, T, need, rank_shift, hist, lane, &b2);
    }

    double ex = 0.0, ey = 0.0;
    for (int j = lane; j < T; j += 32)
    {
        if (j == i)
            continue;
        double dx, dy;
        dist(j, dx, dy);
        const double v  = fmax(dx, dy);
        bool         in = v < dk;
        if (!in && v == dk)
            in = rcut == ~0ull || g.rank(ix, iy, ra0[j], rb0[j], j, T) <= rcut;
        if (in)
        {
            ex = fmax(ex, dx);
            ey = fmax(ey, dy);
        }
    }
    ex = warp_max(ex);
    ey = warp_max(ey);

    int nx = 0, ny = 0;
    for (int j = lane; j < T; j += 32)
    {
        if (j == i)
            continue;
        double dx, dy;
        dist(j, dx, dy);
        nx += dx <= ex;
        ny += dy <= ey;
    }
    nx_out = __reduce_add_sync(kFull, nx);
    ny_out = __reduce_add_sync(kFull, ny);
}

// The same counts packed as n_x | n_y << 16 (nframes <= 65535).
__device__ __forceinline__ uint32_t exact_query(const double* __restrict__ X, int T, int K, int a1, int a2, int i,
                                                int box, int rank_shift, unsigned* hist, int lane)
{
    int nx, ny;
    exact_query_nxy(X, T, K, a1, a2, i, box, rank_shift, hist, lane, nx, ny);
    return (uint32_t)nx | ((uint32_t)ny << 16);
}

} // namespace gc
