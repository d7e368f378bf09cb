// Exact FP64 transfer-entropy statistics of one (ordered pair, query), one
// warp: the brute-force path (te_exact_kernel) and the hand-over repair of
// the fast path.  Reference: te_matrix, lib/transfer_entropy.cpp:114-193.
#pragma once

#include "gc_common.cuh"

namespace gc {

// Query qi < N_valid = T - lag of the ordered pair (target a1, source a2) on
// the raw coordinates XT [3 * natoms][T] (component-major).  eps is the k-th
// smallest 9-D max-norm distance over j != qi, j < N_valid (byte-wise radix
// selection; only its value matters, so no tie rule); the counts are strict
// (< eps).  Returns (n_xp | n_xfxp << 16, n_ypxp) on every lane.  hist: 256
// words of this warp's shared memory.
__device__ __forceinline__ void te_exact_query_n(const double* __restrict__ XT, int T, int K, int lag, int a1, int a2,
                                                 int qi, unsigned* hist, int lane, int& n_xp, int& n_xfxp, int& n_ypxp)
{
    const double* __restrict__ A0 = XT + (size_t)(a1 * 3 + 0) * T;
    const double* __restrict__ A1 = XT + (size_t)(a1 * 3 + 1) * T;
    const double* __restrict__ A2 = XT + (size_t)(a1 * 3 + 2) * T;
    const double* __restrict__ B0 = XT + (size_t)(a2 * 3 + 0) * T;
    const double* __restrict__ B1 = XT + (size_t)(a2 * 3 + 1) * T;
    const double* __restrict__ B2 = XT + (size_t)(a2 * 3 + 2) * T;
    const int    Nv = T - lag;
    const double f0 = A0[qi + lag], f1 = A1[qi + lag], f2 = A2[qi + lag];
    const double p0 = A0[qi], p1 = A1[qi], p2 = A2[qi];
    const double y0 = B0[qi], y1 = B1[qi], y2 = B2[qi];
    auto sub = [&](int j, double& dfut, double& dpast, double& dy) {
        dfut  = fmax(fmax(fabs(f0 - A0[j + lag]), fabs(f1 - A1[j + lag])), fabs(f2 - A2[j + lag]));
        dpast = fmax(fmax(fabs(p0 - A0[j]), fabs(p1 - A1[j])), fabs(p2 - A2[j]));
        dy    = fmax(fmax(fabs(y0 - B0[j]), fabs(y1 - B1[j])), fabs(y2 - B2[j]));
    };
    auto key = [&](int j, unsigned long long& k) -> bool {
        if (j == qi)
            return false;
        double a, b, c;
        sub(j, a, b, c);
        k = dbits(fmax(fmax(a, b), c));
        return true;
    };
    int          below;
    const double eps = __longlong_as_double((long long)warp_select_u64(key, Nv, K, 56, hist, lane, &below));
    int nxfxp = 0, nypxp = 0, nxp = 0;
    for (int j = lane; j < Nv; j += 32)
    {
        if (j == qi)
            continue;
        double a, b, c;
        sub(j, a, b, c);
        nxfxp += fmax(a, b) < eps;
        nypxp += fmax(b, c) < eps;
        nxp += b < eps;
    }
    n_xfxp = __reduce_add_sync(kFull, nxfxp);
    n_ypxp = __reduce_add_sync(kFull, nypxp);
    n_xp   = __reduce_add_sync(kFull, nxp);
}

// The same counts packed as (n_xp | n_xfxp << 16, n_ypxp) (N_valid <= 65535).
__device__ __forceinline__ uint2 te_exact_query(const double* __restrict__ XT, int T, int K, int lag, int a1, int a2,
                                                int qi, unsigned* hist, int lane)
{
    int xp, xf, yp;
    te_exact_query_n(XT, T, K, lag, a1, a2, qi, hist, lane, xp, xf, yp);
    return make_uint2((unsigned)xp | ((unsigned)xf << 16), (unsigned)yp);
}

} // namespace gc
