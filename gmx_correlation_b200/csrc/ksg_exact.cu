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

// One CTA per atom, its three components side by side.  The mean and the
// variance are sequential FP64 sums in frame order (one thread per
// component, over chunks of the atom's frames staged in shared memory by
// coalesced loads) with round-to-nearest intrinsics, so no FMA contraction
// or reordering alters a bit relative to the reference's plain double
// arithmetic.  The z-scores, their minimum (an exact operation in any
// order) and the shifted rows are then computed by all threads.
constexpr int kPrepThreads = 192; // a multiple of 3: thread e keeps component e % 3
constexpr int kPrepChunk   = 512; // frames per staged chunk

__global__ void __launch_bounds__(kPrepThreads) ksg_prepare_kernel(const double* __restrict__ xyz, int natoms, int T,
                                                                   double* __restrict__ X, int* __restrict__ status)
{
    __shared__ double buf[kPrepChunk * 3];
    __shared__ double s_me[3], s_sd[3], s_mn[kPrepThreads / 32][3];
    __shared__ int    s_bad;
    const int         atom = blockIdx.x, tid = threadIdx.x;
    const double*     src  = xyz + (size_t)atom * T * 3;
    if (tid == 0)
        s_bad = 0;
    // pass 1: the mean, pass 2: the sum of squared deviations
    for (int pass = 0; pass < 2; ++pass)
    {
        const double me  = pass ? s_me[tid < 3 ? tid : 0] : 0.0;
        double       acc = 0.0;
        for (int f0 = 0; f0 < T; f0 += kPrepChunk)
        {
            const int n = min(kPrepChunk, T - f0);
            __syncthreads(); // the previous chunk is consumed
            for (int e = tid; e < n * 3; e += kPrepThreads)
                buf[e] = src[(size_t)f0 * 3 + e];
            __syncthreads();
            if (tid < 3)
            {
                if (pass == 0)
                {
#pragma unroll 8
                    for (int f = 0; f < n; ++f)
                        acc = __dadd_rn(acc, buf[f * 3 + tid]);
                }
                else
                {
#pragma unroll 8
                    for (int f = 0; f < n; ++f)
                    {
                        const double t = __dsub_rn(buf[f * 3 + tid], me);
                        acc            = __dadd_rn(acc, __dmul_rn(t, t));
                    }
                }
            }
        }
        if (tid < 3)
        {
            if (pass == 0)
                s_me[tid] = __ddiv_rn(acc, (double)T);
            else
            {
                const double sd = __dsqrt_rn(__ddiv_rn(acc, (double)(T - 1)));
                s_sd[tid]       = sd;
                if (!isfinite(sd))
                {
                    atomicOr(status, kStatNonFinite);
                    s_bad = 1;
                }
                else if (sd == 0.0)
                {
                    atomicOr(status, kStatZeroVariance);
                    s_bad = 1;
                }
            }
        }
        __syncthreads();
    }
    if (s_bad)
        return;
    // pass 3: minimum z per component (seeded like the reference's DBL_MAX/2
    // with its integer DBL_MAX); pass 4: the rows z - min
    const int    d  = tid % 3;
    const double me = s_me[d], sd = s_sd[d];
    double       mn = 1000000.0;
    for (int e = tid; e < T * 3; e += kPrepThreads)
    {
        const double z = __ddiv_rn(__dsub_rn(src[e], me), sd);
        mn             = z < mn ? z : mn;
    }
    // lanes of a warp hold components (lane + 32 * warp) % 3; reduce per component
    const int lane = tid & 31, warp = tid >> 5;
    for (int c = 0; c < 3; ++c)
    {
        double v = d == c ? mn : 1000000.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
        {
            const double w = __shfl_xor_sync(0xFFFFFFFFu, v, o);
            v              = w < v ? w : v;
        }
        if (lane == 0)
            s_mn[warp][c] = v;
    }
    __syncthreads();
    double mnd = s_mn[0][d];
    for (int w = 1; w < kPrepThreads / 32; ++w)
        mnd = s_mn[w][d] < mnd ? s_mn[w][d] : mnd;
    double* row = X + (size_t)(atom * 3 + d) * T;
    for (int e = tid; e < T * 3; e += kPrepThreads)
        row[e / 3] = __dsub_rn(__ddiv_rn(__dsub_rn(src[e], me), sd), mnd);
}

namespace {
constexpr int kExactWarps  = 8;
constexpr int kExactQBlock = 64;
} // namespace

__global__ void __launch_bounds__(kExactWarps * 32)
    ksg_exact_kernel(const double* __restrict__ X, int T, int K, long pair_begin, long pair_count,
                     const int2* __restrict__ pair_ab, int nqb, int rank_shift, uint32_t* __restrict__ cnt,
                     uint32_t* __restrict__ cnt_y)
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
        int nx, ny;
        exact_query_nxy(X, T, K, a1, a2, i, box, rank_shift, hist[warp], lane, nx, ny);
        if (lane == 0)
        {
            if (cnt_y) // wide counts: n_x and n_y in separate planes
            {
                cnt[(size_t)pl * T + i]   = (uint32_t)nx;
                cnt_y[(size_t)pl * T + i] = (uint32_t)ny;
            }
            else
                cnt[(size_t)pl * T + i] = (uint32_t)nx | ((uint32_t)ny << 16);
        }
    }
}

// MI = psi[N] + (psi[K] - 1/K) - (1/N) * sum_i (psi[n_x,i] + psi[n_y,i]),
// summed over i in frame order (lib/kraskov.cpp:1262, :1303-1318).
// cnt_y != nullptr: wide counts (n_x in cnt, n_y in cnt_y, 32 bits each).
__global__ void ksg_finalize_kernel(const uint32_t* __restrict__ cnt, const uint32_t* __restrict__ cnt_y,
                                    long pair_count, int T, int K, const double* __restrict__ psi,
                                    double* __restrict__ pair_mi)
{
    const long p = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (p >= pair_count)
        return;
    if (cnt_y)
    {
        double s = 0.0;
        for (int i = 0; i < T; ++i)
            s = __dadd_rn(s, __dadd_rn(psi[cnt[(size_t)p * T + i]], psi[cnt_y[(size_t)p * T + i]]));
        const double phiK = __dsub_rn(psi[K], __ddiv_rn(1.0, (double)K));
        pair_mi[p]        = __dsub_rn(__dadd_rn(psi[T], phiK), __ddiv_rn(s, (double)T));
        return;
    }
    // 16 frames' counts and digamma terms are fetched together; the sum
    // itself stays sequential in frame order
    double s = 0.0;
    int    i = 0;
    for (; i + 16 <= T; i += 16)
    {
        uint32_t c[16];
        double   term[16];
#pragma unroll
        for (int u = 0; u < 16; ++u)
            c[u] = cnt[(size_t)p * T + i + u];
#pragma unroll
        for (int u = 0; u < 16; ++u)
            term[u] = __dadd_rn(psi[c[u] & 0xFFFFu], psi[c[u] >> 16]);
#pragma unroll
        for (int u = 0; u < 16; ++u)
            s = __dadd_rn(s, term[u]);
    }
    for (; i < T; ++i)
    {
        const uint32_t c = cnt[(size_t)p * T + i];
        s                = __dadd_rn(s, __dadd_rn(psi[c & 0xFFFFu], psi[c >> 16]));
    }
    const double phiK = __dsub_rn(psi[K], __ddiv_rn(1.0, (double)K));
    const double dxy2 = __ddiv_rn(s, (double)T);
    pair_mi[p]        = __dsub_rn(__dadd_rn(psi[T], phiK), dxy2);
}

void launch_ksg_prepare(const double* xyz, int natoms, int T, double* X, int* status, cudaStream_t s)
{
    ksg_prepare_kernel<<<natoms, kPrepThreads, 0, s>>>(xyz, natoms, T, X, status);
}

// Rows handed in already normalised (kraskov_corrmatrix_gpu's t_kraskov):
// flags a non-finite value, which is what a constant component becomes
// after the reference's z-scoring (0 / 0).
__global__ void ksg_check_rows_kernel(const double* __restrict__ X, long n, int* __restrict__ status)
{
    bool bad = false;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x)
        bad |= !isfinite(X[e]);
    if (__any_sync(kFull, bad) && (threadIdx.x & 31) == 0)
        atomicOr(status, kStatNonFinite);
}

void launch_ksg_check_rows(const double* X, long n, int* status, cudaStream_t s)
{
    const long blocks = (n + 255) / 256;
    ksg_check_rows_kernel<<<(unsigned)(blocks < 1184 ? (blocks > 0 ? blocks : 1) : 1184), 256, 0, s>>>(X, n, status);
}

void launch_ksg_exact(const double* X, int T, int K, long pair_begin, long pair_count, uint32_t* cnt,
                      cudaStream_t s, const int2* pair_ab, uint32_t* cnt_y)
{
    const int  nqb   = (T + kExactQBlock - 1) / kExactQBlock;
    const long tasks = pair_count * nqb;
    const int  rank_shift = rank_top_shift(ksg_box_count(T, K), T);
    ksg_exact_kernel<<<(unsigned)tasks, kExactWarps * 32, 0, s>>>(X, T, K, pair_begin, pair_count, pair_ab, nqb,
                                                                  rank_shift, cnt, cnt_y);
}

void launch_ksg_finalize(const uint32_t* cnt, long pair_count, int T, int K, const double* psi,
                         double* pair_mi, cudaStream_t s, const uint32_t* cnt_y)
{
    ksg_finalize_kernel<<<(unsigned)((pair_count + 127) / 128), 128, 0, s>>>(cnt, cnt_y, pair_count, T, K, psi,
                                                                            pair_mi);
}

} // namespace gc
