// KSG (Kraskov algorithm 2) on B200: normalisation, the exact FP64
// brute-force neighbour statistics, and the ordered MI reduction.
//
// Reference semantics (scdantu/gmx_correlation):
//   kraskov_prepare  lib/kraskov.cpp:2168-2220
//   mir_xnyn         lib/kraskov.cpp:1228-1331 (the estimator per pair)
//   neiK / neiE      lib/kraskov.cpp:257-343 / :113-177 (exact k-NN, counts)
//
// For every (pair, query frame i) the exact kernel finds the k-th smallest
// joint max-norm distance over j != i, breaks exact ties at that distance in
// the reference's grid-scan order, takes eps_x / eps_y as the largest
// marginal distance among the k chosen neighbours, and counts
// n_x = #{j != i : d_x(i,j) <= eps_x} (same for y).  All distance
// arithmetic is IEEE FP64 |a-b| and max, so every count equals the
// reference's.  The counts are stored per query and reduced in frame order
// by ksg_finalize_kernel, which reproduces mir_xnyn's summation exactly.

#include "gc_common.cuh"
#include "gc_internal.h"
#include "ksg_exact_query.cuh"

namespace gc {

// One thread per component c = atom*3 + dim; sequential sums in frame
// order with round-to-nearest intrinsics so no FMA contraction alters a
// bit relative to the reference's plain double arithmetic.
__global__ void ksg_prepare_kernel(const double* __restrict__ xyz, int natoms, int T,
                                   double* __restrict__ X, int* __restrict__ status)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= natoms * 3)
        return;
    const int     atom = c / 3, d = c - 3 * (c / 3);
    const double* src  = xyz + (size_t)atom * T * 3 + d;
    double        me   = 0.0;
    for (int f = 0; f < T; ++f)
        me = __dadd_rn(me, src[(size_t)f * 3]);
    me       = __ddiv_rn(me, (double)T);
    double s = 0.0;
    for (int f = 0; f < T; ++f)
    {
        const double t = __dsub_rn(src[(size_t)f * 3], me);
        s              = __dadd_rn(s, __dmul_rn(t, t));
    }
    s = __ddiv_rn(s, (double)(T - 1));
    s = __dsqrt_rn(s);
    if (!isfinite(s))
    {
        atomicOr(status, kStatNonFinite);
        return;
    }
    if (s == 0.0)
    {
        atomicOr(status, kStatZeroVariance);
        return;
    }
    // min/max seeds of the reference: DBL_MAX/2 with its integer DBL_MAX.
    double  mn = 1000000.0, mx = -1000000.0;
    double* row = X + (size_t)c * T;
    for (int f = 0; f < T; ++f)
    {
        const double z = __ddiv_rn(__dsub_rn(src[(size_t)f * 3], me), s);
        row[f]         = z;
        mn             = z < mn ? z : mn;
        mx             = z > mx ? z : mx;
    }
    for (int f = 0; f < T; ++f)
        row[f] = __dsub_rn(row[f], mn);
}

namespace {
constexpr int kExactWarps  = 8;
constexpr int kExactQBlock = 64;
} // namespace

__global__ void __launch_bounds__(kExactWarps * 32)
    ksg_exact_kernel(const double* __restrict__ X, int T, int K, long pair_begin, long pair_count,
                     const int2* __restrict__ pair_ab, int nqb, int rank_shift, uint32_t* __restrict__ cnt)
{
    __shared__ unsigned hist[kExactWarps][256];
    const int  warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long task = blockIdx.x;
    const long pl   = task / nqb;
    const int  qb   = (int)(task - pl * nqb);
    if (pl >= pair_count)
        return;
    int a1, a2;
    if (pair_ab)
    {
        a1 = pair_ab[pl].x;
        a2 = pair_ab[pl].y;
    }
    else
        pair_from_index(pair_begin + pl, &a1, &a2);
    const int box = ksg_box_count(T, K);
    const int i0  = qb * kExactQBlock;
    const int i1  = min(T, i0 + kExactQBlock);
#pragma unroll 1
    for (int i = i0 + warp; i < i1; i += kExactWarps)
    {
        const uint32_t c = exact_query(X, T, K, a1, a2, i, box, rank_shift, hist[warp], lane);
        if (lane == 0)
            cnt[(size_t)i * pair_count + pl] = c;
    }
}

// MI = psi[N] + (psi[K] - 1/K) - (1/N) * sum_i (psi[n_x,i] + psi[n_y,i]),
// summed over i in frame order (lib/kraskov.cpp:1262, :1303-1318).
__global__ void ksg_finalize_kernel(const uint32_t* __restrict__ cnt, long pair_count, int T, int K,
                                    const double* __restrict__ psi, double* __restrict__ pair_mi)
{
    const long p = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (p >= pair_count)
        return;
    double s = 0.0;
    for (int i = 0; i < T; ++i)
    {
        const uint32_t c = cnt[(size_t)i * pair_count + p];
        s                = __dadd_rn(s, __dadd_rn(psi[c & 0xFFFFu], psi[c >> 16]));
    }
    const double phiK = __dsub_rn(psi[K], __ddiv_rn(1.0, (double)K));
    const double dxy2 = __ddiv_rn(s, (double)T);
    pair_mi[p]        = __dsub_rn(__dadd_rn(psi[T], phiK), dxy2);
}

void launch_ksg_prepare(const double* xyz, int natoms, int T, double* X, int* status, cudaStream_t s)
{
    const int n = natoms * 3;
    ksg_prepare_kernel<<<(n + 127) / 128, 128, 0, s>>>(xyz, natoms, T, X, status);
}

void launch_ksg_exact(const double* X, int T, int K, long pair_begin, long pair_count, uint32_t* cnt,
                      cudaStream_t s, const int2* pair_ab)
{
    const int  nqb   = (T + kExactQBlock - 1) / kExactQBlock;
    const long tasks = pair_count * nqb;
    const int  rank_shift = rank_top_shift(ksg_box_count(T, K), T);
    ksg_exact_kernel<<<(unsigned)tasks, kExactWarps * 32, 0, s>>>(X, T, K, pair_begin, pair_count, pair_ab, nqb,
                                                                  rank_shift, cnt);
}

void launch_ksg_finalize(const uint32_t* cnt, long pair_count, int T, int K, const double* psi,
                         double* pair_mi, cudaStream_t s)
{
    ksg_finalize_kernel<<<(unsigned)((pair_count + 127) / 128), 128, 0, s>>>(cnt, pair_count, T, K, psi,
                                                                            pair_mi);
}

} // namespace gc
