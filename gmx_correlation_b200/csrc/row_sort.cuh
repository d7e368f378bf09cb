// Sorted distance rows on B200: the row sort shared by the KSG and the
// transfer-entropy fast paths (ksg_fast.cu, te_walk.cu).
#pragma once

#include "gc_common.cuh"

namespace gc {

// One CTA per sorted row: a query frame's distances to every other frame,
// sorted ascending with their frames.  Keys are
// (distance bits << 32 | frame).  A bucket pass over the row's own
// distribution (range, coarse CDF, histogram, scan, scatter) leaves about one
// key per bucket, which one thread per bucket insertion-sorts.  R > 0: each
// thread keeps its R distances (entries tid + r * threads) in registers for
// the passes; R = 0: distances are recomputed (from L1-resident coordinate
// rows) in every pass.  THREADS (256 or 512) threads per row; 512
// only for rows longer than 2048 entries, so every thread owns whole
// buckets of the scan.  A row with a crowded bucket (more than 64
// equal-ish distances, e.g. duplicated frames), and rows longer than 8192,
// are sorted by a bitonic network instead.

// Bucket counters and cursors carry one padding word per 32, so the
// contiguous bucket slices a thread scans start in distinct banks.
__device__ __forceinline__ int rows_skew(int b) { return b + (b >> 5); }
__host__ __device__ constexpr int rows_skewed(int nbin) { return nbin + (nbin >> 5); }

// Sorts the row of query frame i over frames 0 .. N (i excluded, N entries
// in all): dist(j) gives the FP32 distance from the query to frame j.  The
// sorted distances and frames go to S / P at base + (m / 4) * gstride + m % 4
// for entry m (the transposed layout of the walk), the last 4-entry group
// padded with NaN and frame 0.  Every thread of the CTA calls it; it uses
// the dynamic shared memory (N2 * 8 + rows_skewed(nbin) * 8 bytes, N2 and
// nbin as in row_sort_smem).  U_row (optional) receives the unsorted
// distances at U_row[j].
// Static shared memory of sort_row: the caller's kernel declares one (so a
// kernel that sorts rows of several kinds holds it once).
template <int THREADS>
struct RowSortShared
{
    unsigned red_min[THREADS / 32], red_max[THREADS / 32];
    unsigned coarse[THREADS / 32][64];
    float    cum[65];
    int      crowded;
};

template <int THREADS, int R, class DistFn>
__device__ __forceinline__ void sort_row(RowSortShared<THREADS>& sh, int N, int i, DistFn&& dist,
                                         float* __restrict__ S, uint16_t* __restrict__ P, size_t base,
                                         size_t gstride, float* __restrict__ U_row = nullptr)
{
    extern __shared__ __align__(16) unsigned char rows_smem[];
    unsigned(&red_min)[THREADS / 32]       = sh.red_min;
    unsigned(&red_max)[THREADS / 32]       = sh.red_max;
    unsigned(&coarse)[THREADS / 32][64]    = sh.coarse;
    float(&cum)[65]                        = sh.cum;
    int&     crowded                       = sh.crowded;

    const int         tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    int               N2  = THREADS; // at least one bucket per thread in the scan
    while (N2 < N)
        N2 <<= 1;
    // bucket pass up to 8192 keys; longer rows use the bitonic network alone
    const int           nbin   = N2 <= 8192 ? (N2 < 4096 ? N2 : 4096) : 0;
    unsigned long long* keys   = reinterpret_cast<unsigned long long*>(rows_smem); // [N2] sorted output
    unsigned*           hist   = reinterpret_cast<unsigned*>(keys + N2);           // [skewed nbin]
    unsigned*           cursor = hist + rows_skewed(nbin);                         // [skewed nbin]
    auto                frame_of = [i](int m) { return m < i ? m : m + 1; };

    // the row's distances (and later their buckets), entry m = tid + k * threads
    float dreg[R > 0 ? R : 1];
    int   breg[R > 0 ? R : 1];
    if constexpr (R > 0)
    {
#pragma unroll
        for (int k = 0; k < R; ++k)
        {
            const int m = tid + k * THREADS;
            dreg[k]     = m < N ? dist(frame_of(m)) : 0.0f;
        }
    }
    auto each = [&](auto&& fn) {
        if constexpr (R > 0)
        {
#pragma unroll
            for (int k = 0; k < R; ++k)
            {
                const int m = tid + k * THREADS;
                if (m < N)
                    fn(k, m, dreg[k]);
            }
        }
        else
        {
            for (int m = tid; m < N; m += THREADS)
                fn(0, m, dist(frame_of(m)));
        }
    };

    // optional unsorted copy of the row, indexed by frame (the query's own
    // frame is left unwritten: no walk reads it)
    if (U_row)
        each([&](int, int m, float d) { U_row[frame_of(m)] = d; });
    unsigned kmin = 0xFFFFFFFFu, kmax = 0u;
    each([&](int, int, float d) {
        const unsigned k = __float_as_uint(d);
        kmin             = min(kmin, k);
        kmax             = max(kmax, k);
    });
    for (int b = tid; b < rows_skewed(nbin); b += THREADS)
        hist[b] = 0u;
    for (int e = lane; e < 64; e += 32)
        coarse[warp][e] = 0u;
    if (tid == 0)
        crowded = nbin == 0; // no bucket pass for very long rows
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
    {
        kmin = min(kmin, __shfl_xor_sync(kFull, kmin, o));
        kmax = max(kmax, __shfl_xor_sync(kFull, kmax, o));
    }
    if (lane == 0)
    {
        red_min[warp] = kmin;
        red_max[warp] = kmax;
    }
    __syncthreads();
    kmin = red_min[0];
    kmax = red_max[0];
    for (int w = 1; w < THREADS / 32; ++w)
    {
        kmin = min(kmin, red_min[w]);
        kmax = max(kmax, red_max[w]);
    }
    // Buckets follow the row's own distribution: a coarse 64-bin histogram
    // (linear in the value) gives a piecewise-linear CDF, and a key's bucket
    // is floor(CDF * nbin), so each bucket holds about one key and the
    // per-bucket insertion sorts stay short and balanced.  Every step is
    // monotone in the value (FP32 products and sums of non-negative terms,
    // the fraction clamped to [0, 1]), so buckets keep key order.
    const float vmin = __uint_as_float(kmin), vmax = __uint_as_float(kmax);
    const float cinv = vmax > vmin ? 64.0f / (vmax - vmin) : 0.0f;
    auto coarse_of = [&](float v, float& frac) -> unsigned {
        const float    t = (v - vmin) * cinv;
        const unsigned c = min((unsigned)t, 63u);
        frac             = fminf(t - (float)c, 1.0f);
        return c;
    };
    if (nbin)
        each([&](int, int, float d) {
            float f;
            atomicAdd(&coarse[warp][coarse_of(d, f)], 1u);
        });
    __syncthreads();
    if (warp == 0)
    {
        // exclusive prefix over the 64 coarse bins (two per lane), as floats
        unsigned c0 = 0u, c1 = 0u;
        for (int w = 0; w < THREADS / 32; ++w)
        {
            c0 += coarse[w][2 * lane];
            c1 += coarse[w][2 * lane + 1];
        }
        unsigned incl = c0 + c1;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1)
        {
            const unsigned y = __shfl_up_sync(kFull, incl, o);
            if (lane >= o)
                incl += y;
        }
        const unsigned excl = incl - c0 - c1;
        cum[2 * lane]       = (float)excl;
        cum[2 * lane + 1]   = (float)(excl + c0);
        if (lane == 31)
            cum[64] = (float)incl;
    }
    __syncthreads();
    const float fscale = (float)nbin / fmaxf((float)N, 1.0f);
    auto bin_of = [&](float v) -> int {
        float          f;
        const unsigned c = coarse_of(v, f);
        const unsigned b = (unsigned)((cum[c] + f * (cum[c + 1] - cum[c])) * fscale);
        return rows_skew(b < (unsigned)nbin ? (int)b : nbin - 1);
    };
    // histogram
    if (nbin)
        each([&](int slot, int, float d) {
            const int b = bin_of(d);
            if constexpr (R > 0)
                breg[slot] = b;
            atomicAdd(&hist[b], 1u);
        });
    __syncthreads();
    // exclusive scan of hist into cursor (each thread a contiguous slice)
    const int per = nbin / THREADS; // 0 without a bucket pass
    unsigned  loc = 0;
    for (int e = 0; e < per; ++e)
        loc += hist[rows_skew(tid * per + e)];
    unsigned incl = loc;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1)
    {
        const unsigned y = __shfl_up_sync(kFull, incl, o);
        if (lane >= o)
            incl += y;
    }
    if (lane == 31)
        red_min[warp] = incl;
    __syncthreads();
    unsigned wbase = 0;
    for (int w = 0; w < warp; ++w)
        wbase += red_min[w];
    unsigned run = wbase + incl - loc;
    for (int e = 0; e < per; ++e)
    {
        const int      b = rows_skew(tid * per + e);
        const unsigned c = hist[b];
        cursor[b]        = run;
        if (c > 64)
            crowded = 1;
        run += c;
    }
    __syncthreads();
    // scatter (or place in frame order for the bitonic network)
    const bool bucketed = !crowded;
    each([&](int slot, int m, float d) {
        const int                j   = frame_of(m);
        const unsigned long long key = ((unsigned long long)__float_as_uint(d) << 32) | (unsigned)j;
        int                      b   = 0;
        if (bucketed)
        {
            if constexpr (R > 0)
                b = breg[slot];
            else
                b = bin_of(d);
        }
        const unsigned pos = bucketed ? atomicAdd(&cursor[b], 1u) : (unsigned)m;
        keys[pos]          = key;
    });
    __syncthreads();
    if (bucketed)
    {
        // cursor[b] now holds the end of bucket b; sort each bucket (thread
        // t takes buckets t, t + threads, ..., so a warp's buckets, and
        // their keys, lie side by side)
        for (int b = tid; b < nbin; b += THREADS)
        {
            const int      bs  = rows_skew(b);
            const unsigned end = cursor[bs], beg = end - hist[bs];
            for (unsigned x = beg + 1; x < end; ++x)
            {
                const unsigned long long v = keys[x];
                unsigned                 y = x;
                while (y > beg && keys[y - 1] > v)
                {
                    keys[y] = keys[y - 1];
                    --y;
                }
                keys[y] = v;
            }
        }
        __syncthreads();
    }
    else
    {
        for (int m = N + tid; m < N2; m += THREADS)
            keys[m] = ~0ull;
        __syncthreads();
        for (int k = 2; k <= N2; k <<= 1)
            for (int j = k >> 1; j > 0; j >>= 1)
            {
                for (int t = tid; t < (N2 >> 1); t += THREADS)
                {
                    const int                idx = ((t / j) * (j << 1)) + (t % j);
                    const int                prt = idx + j;
                    const unsigned long long x = keys[idx], y = keys[prt];
                    if ((x > y) == ((idx & k) == 0))
                    {
                        keys[idx] = y;
                        keys[prt] = x;
                    }
                }
                __syncthreads();
            }
    }
    // transposed layout: groups of 4 consecutive entries per query, the
    // queries of a block side by side (see WalkParams)
    for (int m = tid; m < N; m += THREADS)
    {
        const unsigned long long k   = keys[m];
        const size_t             idx = base + (size_t)(m >> 2) * gstride + (m & 3);
        S[idx]                       = __uint_as_float((unsigned)(k >> 32));
        P[idx]                       = (uint16_t)(k & 0xFFFFu);
    }
    // the last 4-entry group runs out in NaN (never <= any stop value) with
    // frame 0, so the walk reads whole groups without a bounds test
    if (tid < ((N + 3) & ~3) - N)
    {
        const int    m   = N + tid;
        const size_t idx = base + (size_t)(m >> 2) * gstride + (m & 3);
        S[idx]           = __int_as_float(0x7fc00000);
        P[idx]           = 0;
    }
}

// Shared memory of one sorted row of N entries: keys (N2 * 8 bytes) plus the
// bucket counters and cursors; *threads and *regs pick the sort_row
// instantiation (threads per row, distances per thread kept in registers).
#ifndef GC_ROWS_128
#define GC_ROWS_128 0 // a build-time setting: 128 threads x 16 distances for rows up to 2048 entries
#endif

inline size_t row_sort_smem(int N, int* threads, int* regs)
{
    int N2 = 256;
    while (N2 < N)
        N2 <<= 1;
    const int nbin = N2 <= 8192 ? (N2 < 4096 ? N2 : 4096) : 0;
    // distances kept in registers, 8 per thread up to 2048 entries, then
    // 512 threads with 8 or 16 each (measured faster than 256 threads with
    // 16 or 32 at 4999 entries); longer rows recompute them
    *threads = N <= 8 * 256 ? (GC_ROWS_128 ? 128 : 256) : (N <= 16 * 512 ? 512 : 256);
    *regs    = N <= 8 * 256 ? (GC_ROWS_128 ? 16 : 8) : (N <= 8 * 512 ? 8 : (N <= 16 * 512 ? 16 : 0));
    return (size_t)N2 * 8 + (size_t)rows_skewed(nbin) * 8;
}

} // namespace gc
