// KSG fast path on B200: FP32 neighbour search with exact FP64 repair.
//
// Same estimator as ksg_exact.cu (Kraskov alg. 2 as mir_xnyn computes it,
// lib/kraskov.cpp:1228-1331), restructured around one observation: the
// joint distance of a pair is the max of two per-atom marginal distances,
// and each marginal row (atom a, query i) is shared by every pair that
// contains atom a.  So:
//
//   ksg_x32_kernel    FP32 copy of the normalised coordinates, centred per
//                     component, and a per-atom bound eps_a with
//                     |d32 - d64| <= eps_a for every marginal distance.
//   ksg_rows_kernel   per (atom, query): the T-1 marginal distances, sorted
//                     ascending, with their frame indices (S rows, P rows).
//   ksg_walk_kernel   per (pair, query), one warp: walks the sorted row of
//                     the marginal whose k-th distance is larger, gathering
//                     the other marginal, until the joint k-th distance is
//                     provably behind; the k-th value comes from a
//                     shared-memory histogram anchored at the exact lower
//                     bound max(k-th marginal distances) plus a sorted band.
//                     Everything within the proven error band 2*eps of a
//                     decision is re-evaluated in FP64 on the reference's
//                     normalised coordinates, with the reference's grid-scan
//                     order deciding exact ties, so n_x and n_y equal the
//                     reference's counts.  Counts come from warp-parallel
//                     search in the sorted rows, again with FP64 repair of
//                     the band around eps_x / eps_y.
//   ksg_queue_kernel  queries the walk hands over (degenerate histograms,
//                     oversized tie bands) run through the exact FP64 code.
//
// Error bound (x32 = fl32(x64 - c), c the component midrange, |x64-c| <= R):
//   |fl32(x32_i - x32_j) - fl64(x64_i - x64_j)| <= 4 u R (1 + 2^-20),
//   u = 2^-24, and max over components keeps the bound; eps_a = R_a * 2^-21
//   (twice that) is used.

#include "gc_common.cuh"
#include "gc_internal.h"
#include "ksg_exact_query.cuh"
#include "ksg_fast.h"

namespace gc {

__device__ __forceinline__ float dist3f(const float4 a, const float4 b)
{
    return fmaxf(fmaxf(fabsf(a.x - b.x), fabsf(a.y - b.y)), fabsf(a.z - b.z));
}

__device__ __forceinline__ double dist3d(const double* __restrict__ X64, int atom, int T, int i, int j)
{
    const double* r = X64 + (size_t)atom * 3 * T;
    return fmax(fmax(fabs(r[i] - r[j]), fabs(r[T + i] - r[T + j])), fabs(r[2 * T + i] - r[2 * T + j]));
}

// One warp per atom: component midranges (X64 rows are min-shifted, so the
// midrange is max/2), centred FP32 coordinates and the atom's error bound.
__global__ void ksg_x32_kernel(const double* __restrict__ X64, int natoms, int T, float4* __restrict__ X32,
                               float* __restrict__ eps_atom)
{
    const int lane = threadIdx.x & 31;
    const int a    = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (a >= natoms)
        return;
    const double* r = X64 + (size_t)a * 3 * T;
    double        mx[3];
    for (int d = 0; d < 3; ++d)
    {
        double m = 0.0;
        for (int f = lane; f < T; f += 32)
            m = fmax(m, r[(size_t)d * T + f]);
        mx[d] = warp_max(m);
    }
    const double c0 = 0.5 * mx[0], c1 = 0.5 * mx[1], c2 = 0.5 * mx[2];
    for (int f = lane; f < T; f += 32)
        X32[(size_t)a * T + f] = make_float4((float)(r[f] - c0), (float)(r[T + f] - c1),
                                             (float)(r[2 * T + f] - c2), 0.0f);
    if (lane == 0)
    {
        const double R = fmax(fmax(c0, c1), c2) * (1.0 + 0x1p-40);
        eps_atom[a]    = __double2float_ru(R * 0x1p-21) + 1e-30f;
    }
}

// One CTA per (atom, query): the row's T-1 marginal distances (self
// excluded), sorted ascending with their frames.  Keys are
// (distance bits << 32 | frame); a bucket pass over the row's key range
// (histogram, scan, scatter) leaves a few keys per bucket, which one thread
// per bucket insertion-sorts.  A row with a crowded bucket (more than 64
// equal-ish distances, e.g. duplicated frames) is sorted by a bitonic
// network over the same buffer instead.
constexpr int kRowsThreads = 256;

__global__ void __launch_bounds__(kRowsThreads) ksg_rows_kernel(const float4* __restrict__ X32, int T, int i0, int Q,
                                                                int Lpad, int N2, int nbin, float* __restrict__ S,
                                                                uint16_t* __restrict__ P)
{
    extern __shared__ __align__(16) unsigned char rows_smem[];
    unsigned long long* keys   = reinterpret_cast<unsigned long long*>(rows_smem);      // [N2] sorted output
    unsigned long long* in     = keys + N2;                                             // [N2] unsorted (bucket path)
    unsigned*           hist   = reinterpret_cast<unsigned*>(in + (nbin ? N2 : 0));     // [nbin]
    unsigned*           cursor = hist + nbin;                                           // [nbin]
    __shared__ unsigned red_min[kRowsThreads / 32], red_max[kRowsThreads / 32];
    __shared__ int      crowded;

    const int    row = blockIdx.x;
    const int    a   = row / Q;
    const int    iq  = row - a * Q;
    const int    i   = i0 + iq;
    const int    N   = T - 1;
    const int    tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const float4 q   = X32[(size_t)a * T + i];

    unsigned kmin = 0xFFFFFFFFu, kmax = 0u;
    for (int m = tid; m < N; m += kRowsThreads)
    {
        const int      j = m < i ? m : m + 1;
        const unsigned k = __float_as_uint(dist3f(q, X32[(size_t)a * T + j]));
        (nbin ? in : keys)[m] = ((unsigned long long)k << 32) | (unsigned)j;
        kmin             = min(kmin, k);
        kmax             = max(kmax, k);
    }
    for (int b = tid; b < nbin; b += kRowsThreads)
        hist[b] = 0u;
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
    for (int w = 1; w < kRowsThreads / 32; ++w)
    {
        kmin = min(kmin, red_min[w]);
        kmax = max(kmax, red_max[w]);
    }
    // bucket = floor((key - kmin) * nbin / (kmax - kmin + 1)), in FP32: the
    // conversion and the scaling are monotone, so buckets keep key order
    const float scale = (float)nbin / ((float)(kmax - kmin) + 1.0f);
    auto bin_of = [&](unsigned long long key) -> unsigned {
        const unsigned b = (unsigned)((float)((unsigned)(key >> 32) - kmin) * scale);
        return b < (unsigned)nbin ? b : (unsigned)nbin - 1;
    };
    // histogram
    for (int m = tid; m < N && nbin; m += kRowsThreads)
        atomicAdd(&hist[bin_of(in[m])], 1u);
    __syncthreads();
    // exclusive scan of hist into cursor (each thread a contiguous slice)
    const int per = nbin / kRowsThreads; // 0 without a bucket pass
    unsigned  loc = 0;
    for (int e = 0; e < per; ++e)
        loc += hist[tid * per + e];
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
        const unsigned c       = hist[tid * per + e];
        cursor[tid * per + e]  = run;
        if (c > 64)
            crowded = 1;
        run += c;
    }
    __syncthreads();
    // scatter
    if (!crowded)
        for (int m = tid; m < N; m += kRowsThreads)
        {
            const unsigned long long k   = in[m];
            const unsigned           pos = atomicAdd(&cursor[bin_of(k)], 1u);
            keys[pos]                    = k;
        }
    else if (nbin)
        for (int m = tid; m < N; m += kRowsThreads)
            keys[m] = in[m];
    __syncthreads();
    if (!crowded)
    {
        // cursor[b] now holds the end of bucket b; sort each bucket
        for (int e = 0; e < per; ++e)
        {
            const int      b   = tid * per + e;
            const unsigned end = cursor[b], beg = end - hist[b];
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
        for (int m = N + tid; m < N2; m += kRowsThreads)
            keys[m] = ~0ull;
        __syncthreads();
        for (int k = 2; k <= N2; k <<= 1)
            for (int j = k >> 1; j > 0; j >>= 1)
            {
                for (int t = tid; t < (N2 >> 1); t += kRowsThreads)
                {
                    const int idx = ((t / j) * (j << 1)) + (t % j);
                    const int prt = idx + j;
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
    float*    srow = S + (size_t)row * Lpad;
    uint16_t* prow = P + (size_t)row * Lpad;
    for (int m = tid; m < N; m += kRowsThreads)
    {
        const unsigned long long k = keys[m];
        srow[m] = __uint_as_float((unsigned)(k >> 32));
        prow[m] = (uint16_t)(k & 0xFFFFu);
    }
}

namespace {

// Warp-wide count of sorted row values < t (strict) or <= t.
__device__ __noinline__ int warp_rank(const float* __restrict__ row, int n, float t, bool strict, int lane)
{
    int lo = 0, hi = n;
    while (hi - lo > 32)
    {
        const int  step = (hi - lo + 31) >> 5;
        const int  p    = lo + lane * step;
        bool       ok   = false;
        if (p < hi)
        {
            const float v = row[p];
            ok            = strict ? v < t : v <= t;
        }
        const int c = __popc(__ballot_sync(kFull, ok));
        if (c == 0)
            hi = lo;
        else
        {
            const int nlo = lo + (c - 1) * step + 1;
            const int nhi = min(hi, lo + c * step);
            lo            = nlo;
            hi            = nhi;
        }
    }
    const int p  = lo + lane;
    bool      ok = false;
    if (p < hi)
    {
        const float v = row[p];
        ok            = strict ? v < t : v <= t;
    }
    return lo + __popc(__ballot_sync(kFull, ok));
}

__device__ __forceinline__ unsigned lanemask_lt(int lane) { return (1u << lane) - 1u; }

// Warp maximum of non-negative floats / doubles: their IEEE bit patterns
// order like the values, so single-instruction integer reductions do it.
__device__ __forceinline__ float warp_max_nn(float v)
{
    return __uint_as_float(__reduce_max_sync(kFull, __float_as_uint(v)));
}

__device__ __forceinline__ double warp_max_nn(double v)
{
    const unsigned long long b  = (unsigned long long)__double_as_longlong(v);
    const unsigned           hi = __reduce_max_sync(kFull, (unsigned)(b >> 32));
    const unsigned           lo = __reduce_max_sync(kFull, (unsigned)(b >> 32) == hi ? (unsigned)b : 0u);
    return __longlong_as_double((long long)(((unsigned long long)hi << 32) | lo));
}

// Bitonic sort of (key_hi, key_lo, payload) per lane, ascending lexicographic.
__device__ __noinline__ void warp_sort_kv(unsigned long long& kh, unsigned long long& kl, int& pay, int lane)
{
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1)
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1)
        {
            const unsigned long long oh = __shfl_xor_sync(kFull, kh, j);
            const unsigned long long ol = __shfl_xor_sync(kFull, kl, j);
            const int                op = __shfl_xor_sync(kFull, pay, j);
            const bool up   = (lane & k) == 0;
            const bool low  = (lane & j) == 0;
            const bool less = (oh < kh) || (oh == kh && ol < kl); // other < mine
            const bool take = (low == up) ? less : !less && !(oh == kh && ol == kl);
            if (take)
            {
                kh  = oh;
                kl  = ol;
                pay = op;
            }
        }
}

} // namespace

namespace {

// 4 consecutive sorted-row entries of lane `lane` in the 128-element walk
// step starting at g0 (m = g0 + 4*lane + q), padded with NaN / frame 0 (a
// NaN compares false with everything, so padding is never taken).
__device__ __forceinline__ void load_step(const float* __restrict__ Sw, const uint16_t* __restrict__ Pw, int g0,
                                          int Llen, int lane, float4& s4, uint2& j2)
{
    const int m0 = g0 + 4 * lane;
    if (m0 + 3 < Llen)
    {
        s4 = *reinterpret_cast<const float4*>(Sw + m0);
        j2 = *reinterpret_cast<const uint2*>(Pw + m0);
    }
    else
    {
        const float nan = __int_as_float(0x7fc00000);
        float       v[4];
        unsigned    j[4];
#pragma unroll
        for (int q = 0; q < 4; ++q)
        {
            v[q] = m0 + q < Llen ? Sw[m0 + q] : nan;
            j[q] = m0 + q < Llen ? Pw[m0 + q] : 0u;
        }
        s4 = make_float4(v[0], v[1], v[2], v[3]);
        j2 = make_uint2(j[0] | (j[1] << 16), j[2] | (j[3] << 16));
    }
}

__device__ __forceinline__ float f4get(const float4& v, int q)
{
    return q == 0 ? v.x : (q == 1 ? v.y : (q == 2 ? v.z : v.w));
}

__device__ __forceinline__ unsigned u2get16(const uint2& v, int q)
{
    return q < 2 ? ((v.x >> (16 * q)) & 0xFFFFu) : ((v.y >> (16 * (q - 2))) & 0xFFFFu);
}

} // namespace

template <int WARPS>
__global__ void __launch_bounds__(WARPS * 32) ksg_walk_kernel(WalkParams p)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int      warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char* base = smem_raw + (size_t)warp * p.warp_smem;
    unsigned*      hist = reinterpret_cast<unsigned*>(base);
    float*         bsw  = reinterpret_cast<float*>(base + p.nb * 4);
    float*         bdo  = bsw + p.bufcap;
    uint16_t*      bj   = reinterpret_cast<uint16_t*>(bdo + p.bufcap);
    unsigned char* lst  = base + walk_list_offset(p.nb, p.bufcap);
    float*         bv   = reinterpret_cast<float*>(lst);          // [64] band values
    unsigned*      bjj  = reinterpret_cast<unsigned*>(lst + 256); // [64] band frames
    float*         bdx  = reinterpret_cast<float*>(lst + 512);    // [64]
    float*         bdy  = reinterpret_cast<float*>(lst + 768);    // [64]
    unsigned*      aj   = reinterpret_cast<unsigned*>(lst + 1024); // [32] ambiguous: band slot
    unsigned*      cj   = reinterpret_cast<unsigned*>(lst + 1152); // [32] max candidates: frames
    double*        a64  = reinterpret_cast<double*>(lst + 1280);   // [64] ambiguous dx64 | dy64

    const int       T = p.T, K = p.K, Llen = T - 1;
    const ScanGrid  grid(p.box);
    const long long total = (long long)p.Q * p.pair_count;
    const float     inf   = __int_as_float(0x7f800000);

    for (;;)
    {
        long long t0 = 0;
        if (lane == 0)
            t0 = (long long)atomicAdd(p.task_counter, 32ull);
        t0 = __shfl_sync(kFull, t0, 0);
        if (t0 >= total)
            break;
        const long long t1 = min(total, t0 + 32);
        int             iq = (int)(t0 / p.pair_count);
        long            pl = (long)(t0 - (long long)iq * p.pair_count);
        int             a1, a2;
        if (p.pair_ab)
        {
            a1 = p.pair_ab[pl].x;
            a2 = p.pair_ab[pl].y;
        }
        else
            pair_from_index(p.pair_begin + pl, &a1, &a2);
        for (long long t = t0; t < t1; ++t)
        {
            if (t > t0)
            {
                // advance to the next pair (list order, or p = a1*(a1-1)/2 + a2)
                if (++pl == p.pair_count)
                {
                    pl = 0;
                    ++iq;
                }
                if (p.pair_ab)
                {
                    a1 = p.pair_ab[pl].x;
                    a2 = p.pair_ab[pl].y;
                }
                else if (pl == 0)
                    pair_from_index(p.pair_begin, &a1, &a2);
                else if (++a2 == a1)
                {
                    ++a1;
                    a2 = 0;
                }
            }
            const int       i  = p.i0 + iq;
            const float*    Sa = p.S + ((size_t)a1 * p.Q + iq) * p.Lpad;
            const float*    Sb = p.S + ((size_t)a2 * p.Q + iq) * p.Lpad;
            const uint16_t* Pa = p.P + ((size_t)a1 * p.Q + iq) * p.Lpad;
            const uint16_t* Pb = p.P + ((size_t)a2 * p.Q + iq) * p.Lpad;
            const float     Ra = Sa[K - 1], Rb = Sb[K - 1];
            const bool      wx = Ra >= Rb; // walk the x (a1) marginal
            const int       o  = wx ? a2 : a1;
            const float*    Sw = wx ? Sa : Sb;
            const uint16_t* Pw = wx ? Pa : Pb;
            const float*    So = wx ? Sb : Sa;
            const uint16_t* Po = wx ? Pb : Pa;
            const float     L  = wx ? Ra : Rb;
            const unsigned  Lb = __float_as_uint(L);
            const float4    xo = p.X32[(size_t)o * T + i];
            const float4*   X32o = p.X32 + (size_t)o * T;
            const float     ea = p.eps_atom[a1], eb = p.eps_atom[a2];
            const float     ew = wx ? ea : eb, eo = wx ? eb : ea;
            const float     e2 = __fmul_ru(2.0f, fmaxf(ea, eb));
            // probes of the other atom's row for its count (every 64th entry)
            const int   pr0 = (lane + 1) * 64 - 1, pr1 = (lane + 33) * 64 - 1;
            const float probe0 = pr0 < Llen ? So[pr0] : inf;
            const float probe1 = pr1 < Llen ? So[pr1] : inf;
            bool        handoff = false;

            for (int b = 4 * lane; b < p.nb; b += 128)
                *reinterpret_cast<uint4*>(hist + b) = make_uint4(0u, 0u, 0u, 0u);
            __syncwarp();

            // ---- pass 1: walk in 128-entry steps + histogram -------------------
            // Branch-free step: every lane gathers all four coordinates (padding
            // entries read frame 0) and the taken mask only gates the counters.
            int      cnt_lo = 0, R = 0, m_end = 0;
            unsigned thr  = 0;
            float    stop = inf;
            float4   s4;
            uint2    j2;
            load_step(Sw, Pw, 0, Llen, lane, s4, j2);
            for (int g0 = 0; g0 < Llen; g0 += 128)
            {
                if (!(__shfl_sync(kFull, s4.x, 0) <= stop))
                    break;
                float4 ns4 = make_float4(nanf(""), nanf(""), nanf(""), nanf(""));
                uint2  nj2 = make_uint2(0u, 0u);
                if (g0 + 128 < Llen)
                    load_step(Sw, Pw, g0 + 128, Llen, lane, ns4, nj2);
                const float4 x0 = X32o[j2.x & 0xFFFFu], x1 = X32o[j2.x >> 16];
                const float4 x2 = X32o[j2.y & 0xFFFFu], x3 = X32o[j2.y >> 16];
                const float  d0 = dist3f(xo, x0), d1 = dist3f(xo, x1), d2 = dist3f(xo, x2), d3 = dist3f(xo, x3);
                const float  sv[4] = {s4.x, s4.y, s4.z, s4.w};
                const float  dv[4] = {d0, d1, d2, d3};
                int          nlo = 0, ntk = 0;
#pragma unroll
                for (int q = 0; q < 4; ++q)
                {
                    const float    v    = fmaxf(sv[q], dv[q]);
                    const bool     take = sv[q] <= stop;
                    const bool     lo   = take && v < L;
                    const unsigned b    = min((__float_as_uint(v) - Lb) >> p.shift, (unsigned)p.nb - 1);
                    nlo += lo;
                    ntk += take;
                    if (take && !lo)
                        atomicAdd(&hist[b], 1u);
                }
                const int m0 = g0 + 4 * lane;
                if (m0 < p.bufcap)
                {
                    *reinterpret_cast<float4*>(bsw + m0) = s4;
                    *reinterpret_cast<float4*>(bdo + m0) = make_float4(d0, d1, d2, d3);
                    *reinterpret_cast<uint2*>(bj + m0)   = j2;
                }
                cnt_lo += __reduce_add_sync(kFull, nlo);
                const int ntake = __reduce_add_sync(kFull, ntk);
                m_end           = g0 + ntake;
                __syncwarp();
                if (stop == inf && ntake > 0)
                {
                    const int   last = ntake - 1; // taken entries form a prefix of the step
                    const float sl   = __shfl_sync(kFull, f4get(s4, last & 3), last >> 2);
                    if (sl >= L)
                    {
                        const unsigned bn  = min((__float_as_uint(sl) - Lb) >> p.shift, (unsigned)p.nb - 1);
                        int            add = 0;
                        for (unsigned b = thr + lane; b < bn; b += 32)
                            add += hist[b];
                        R += __reduce_add_sync(kFull, add);
                        thr = bn > thr ? bn : thr;
                        if (cnt_lo + R >= K)
                            stop = __fadd_ru(__uint_as_float(Lb + (bn << p.shift)), e2);
                    }
                }
                s4 = ns4;
                j2 = nj2;
            }
            if (p.walk_elems && lane == 0)
                atomicAdd(p.walk_elems, (unsigned long long)m_end);
            // a walk longer than the buffer goes to the exact kernel (rare)
            int reason = 0;
            if (m_end > p.bufcap)
                reason = 1;
            handoff = reason != 0;


            // ---- bucket of the k-th value: one warp scan over nb/32 buckets/lane
            int bstar = -1;
            {
                const int per = p.nb >> 5; // 2..8 buckets per lane
                unsigned  c[8];
                unsigned  own = 0;
#pragma unroll
                for (int e = 0; e < 8; ++e)
                {
                    c[e] = e < per ? hist[lane * per + e] : 0u;
                    own += c[e];
                }
                unsigned incl = own;
#pragma unroll
                for (int sft = 1; sft < 32; sft <<= 1)
                {
                    const unsigned y = __shfl_up_sync(kFull, incl, sft);
                    if (lane >= sft)
                        incl += y;
                }
                const unsigned need  = (unsigned)(K - cnt_lo);
                const unsigned excl  = incl - own;
                const bool     here  = excl < need && need <= incl;
                int            mine  = -1;
                if (here)
                {
                    unsigned acc = excl;
#pragma unroll
                    for (int e = 0; e < 8; ++e)
                        if (mine < 0 && e < per)
                        {
                            acc += c[e];
                            if (acc >= need)
                                mine = lane * per + e;
                        }
                }
                const unsigned who = __ballot_sync(kFull, here);
                bstar              = who ? __shfl_sync(kFull, mine, __ffs(who) - 1) : -1;
            }
            if (!handoff && (bstar < 0 || bstar >= p.nb - 1))
            {
                handoff = true;
                reason  = 2;
            }

            // ---- one pass: certain members, and the band around bucket bstar ----
            // v < inlo: certainly among the k nearest (d32 >= lower bucket edge);
            // inlo <= v <= bandhi: the band, which holds the k-th value and every
            // entry within 2 eps of it; above bandhi: certainly not.
            const double* xa = p.X64 + (size_t)a1 * 3 * T;
            const double* xb = p.X64 + (size_t)a2 * 3 * T;
            float mx = 0.0f, my = 0.0f, inlo = 0.0f, bandhi = 0.0f;
            int   n_in = 0, nband = 0;
            if (!handoff)
            {
                inlo   = __fsub_rd(__uint_as_float(Lb + ((unsigned)bstar << p.shift)), e2);
                bandhi = __fadd_ru(__uint_as_float(Lb + ((unsigned)(bstar + 1) << p.shift)), e2);
                int cin = 0;
                for (int b0 = 0; b0 < m_end; b0 += 128)
                {
                    const int    m0 = b0 + 4 * lane;
                    const int    mc = min(m0, p.bufcap - 4);
                    const float4 a  = *reinterpret_cast<const float4*>(bsw + mc);
                    const float4 d  = *reinterpret_cast<const float4*>(bdo + mc);
                    const float  sv[4] = {a.x, a.y, a.z, a.w};
                    const float  dv[4] = {d.x, d.y, d.z, d.w};
                    bool         bd[4];
                    bool         anyb = false;
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                    {
                        const float v  = fmaxf(sv[q], dv[q]);
                        const bool  ok = m0 + q < m_end;
                        const bool  in = ok && v < inlo;
                        bd[q]          = ok && !in && v <= bandhi;
                        anyb |= bd[q];
                        mx = in ? fmaxf(mx, wx ? sv[q] : dv[q]) : mx;
                        my = in ? fmaxf(my, wx ? dv[q] : sv[q]) : my;
                        cin += in;
                    }
                    if (__any_sync(kFull, anyb))
                    {
                        const uint2 j = *reinterpret_cast<const uint2*>(bj + mc);
#pragma unroll
                        for (int q = 0; q < 4; ++q)
                        {
                            const unsigned bm = __ballot_sync(kFull, bd[q]);
                            const int      sl = nband + __popc(bm & lanemask_lt(lane));
                            if (bd[q] && sl < 64)
                            {
                                bv[sl]  = fmaxf(sv[q], dv[q]);
                                bjj[sl] = u2get16(j, q);
                                bdx[sl] = wx ? sv[q] : dv[q];
                                bdy[sl] = wx ? dv[q] : sv[q];
                            }
                            nband += __popc(bm);
                        }
                    }
                }
                n_in = __reduce_add_sync(kFull, cin);
                if (nband > 64 || K - n_in < 1 || K - n_in > nband)
                {
                    handoff = true;
                    reason  = 3;
                }
                __syncwarp();
            }

            // ---- the k-th value from the band, then exact members and the
            //      ambiguous set (within 2 eps of it) ------------------------------
            int   n_amb = 0;
            float lower = 0.0f;
            if (!handoff)
            {
                const int r = K - n_in; // 1-based rank of the k-th value in the band
                float     d32 = 0.0f;
                if (nband <= 32)
                {
                    const float mine = lane < nband ? bv[lane] : inf;
                    int         rk   = 0;
                    for (int f = 0; f < nband; ++f)
                    {
                        const float u = __shfl_sync(kFull, mine, f);
                        rk += u < mine || (u == mine && f < lane);
                    }
                    const unsigned hit = __ballot_sync(kFull, lane < nband && rk == r - 1);
                    d32                = __shfl_sync(kFull, mine, __ffs(hit) - 1);
                }
                else
                {
                    for (int e = lane; e < nband; e += 32)
                    {
                        const float v  = bv[e];
                        int         rk = 0;
                        for (int f = 0; f < nband; ++f)
                        {
                            const float u = bv[f];
                            rk += u < v || (u == v && f < e);
                        }
                        if (rk == r - 1)
                            d32 = v;
                    }
                    d32 = warp_max_nn(d32);
                }
                lower             = __fsub_rd(d32, e2);
                const float upper = __fadd_ru(d32, e2);
                int         cin = 0;
                for (int e0 = 0; e0 < nband; e0 += 32)
                {
                    const int  e   = e0 + lane;
                    bool       in  = false, amb = false;
                    if (e < nband)
                    {
                        const float v = bv[e];
                        in            = v < lower;
                        amb           = !in && v <= upper;
                        if (in)
                        {
                            mx = fmaxf(mx, bdx[e]);
                            my = fmaxf(my, bdy[e]);
                        }
                    }
                    cin += in;
                    const unsigned am = __ballot_sync(kFull, amb);
                    const int      sl = n_amb + __popc(am & lanemask_lt(lane));
                    if (amb && sl < 32)
                        aj[sl] = (unsigned)e;
                    n_amb += __popc(am);
                }
                n_in += __reduce_add_sync(kFull, cin);
                if (n_amb > 32 || n_amb < 1 || K - n_in < 1 || K - n_in > n_amb)
                {
                    handoff = true;
                    reason  = 4;
                }
                __syncwarp();
            }

            // ---- members whose FP32 marginal is within 2 eps of the members'
            //      maximum: a superset of those that can hold the FP64 maximum ----
            int n_cand = 0;
            if (!handoff)
            {
                mx             = warp_max_nn(mx);
                my             = warp_max_nn(my);
                const float tx = __fsub_rd(mx, __fmul_ru(2.0f, ea));
                const float ty = __fsub_rd(my, __fmul_ru(2.0f, eb));
                for (int b0 = 0; b0 < m_end; b0 += 128)
                {
                    const int    m0 = b0 + 4 * lane;
                    const int    mc = min(m0, p.bufcap - 4);
                    const float4 a  = *reinterpret_cast<const float4*>(bsw + mc);
                    const float4 d  = *reinterpret_cast<const float4*>(bdo + mc);
                    const float  sv[4] = {a.x, a.y, a.z, a.w};
                    const float  dv[4] = {d.x, d.y, d.z, d.w};
                    bool         c[4];
                    bool         anyc = false;
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                    {
                        const float dx = wx ? sv[q] : dv[q], dy = wx ? dv[q] : sv[q];
                        c[q] = m0 + q < m_end && fmaxf(sv[q], dv[q]) < inlo && (dx >= tx || dy >= ty);
                        anyc |= c[q];
                    }
                    if (__any_sync(kFull, anyc))
                    {
                        const uint2 j = *reinterpret_cast<const uint2*>(bj + mc);
#pragma unroll
                        for (int q = 0; q < 4; ++q)
                        {
                            const unsigned cm = __ballot_sync(kFull, c[q]);
                            const int      sl = n_cand + __popc(cm & lanemask_lt(lane));
                            if (c[q] && sl < 32)
                                cj[sl] = u2get16(j, q);
                            n_cand += __popc(cm);
                        }
                    }
                }
                for (int e0 = 0; e0 < nband; e0 += 32)
                {
                    const int  e = e0 + lane;
                    const bool c = e < nband && bv[e] < lower && (bdx[e] >= tx || bdy[e] >= ty);
                    const unsigned cm = __ballot_sync(kFull, c);
                    const int      sl = n_cand + __popc(cm & lanemask_lt(lane));
                    if (c && sl < 32)
                        cj[sl] = bjj[e];
                    n_cand += __popc(cm);
                }
                if (n_cand > 32)
                {
                    handoff = true;
                    reason  = 5;
                }
                __syncwarp();
            }

            uint32_t out_cnt = 0;
            if (!handoff)
            {
                // ---- one FP64 round: ambiguous set + max candidates -------------
                const double qa0 = xa[i], qa1 = xa[T + i], qa2 = xa[2 * T + i];
                const double qb0 = xb[i], qb1 = xb[T + i], qb2 = xb[2 * T + i];
                unsigned long long kh = ~0ull, kl = ~0ull;
                int                slot = lane;
                double             cx = 0.0, cy = 0.0;
                if (lane < n_amb)
                {
                    const int    j  = (int)bjj[aj[lane]];
                    const double x0 = xa[j], y0 = xb[j];
                    const double dx = fmax(fmax(fabs(qa0 - x0), fabs(qa1 - xa[T + j])), fabs(qa2 - xa[2 * T + j]));
                    const double dy = fmax(fmax(fabs(qb0 - y0), fabs(qb1 - xb[T + j])), fabs(qb2 - xb[2 * T + j]));
                    a64[lane]       = dx;
                    a64[32 + lane]  = dy;
                    kh              = dbits(fmax(dx, dy));
                    kl              = n_amb > 1 ? grid.rank(grid.qcell(qa0), grid.qcell(qb0), x0, y0, j, T) : 0ull;
                }
                if (lane < n_cand)
                {
                    const int j = (int)cj[lane];
                    cx = fmax(fmax(fabs(qa0 - xa[j]), fabs(qa1 - xa[T + j])), fabs(qa2 - xa[2 * T + j]));
                    cy = fmax(fmax(fabs(qb0 - xb[j]), fabs(qb1 - xb[T + j])), fabs(qb2 - xb[2 * T + j]));
                }
                __syncwarp();
                if (n_amb > 1)
                    warp_sort_kv(kh, kl, slot, lane);
                if (lane < K - n_in)
                {
                    cx = fmax(cx, a64[slot]);
                    cy = fmax(cy, a64[32 + slot]);
                }
                const double ex64 = warp_max_nn(cx), ey64 = warp_max_nn(cy);

                // ---- counts ----------------------------------------------------
                const double tw = wx ? ex64 : ey64, to = wx ? ey64 : ex64;
                const float  wlo = __double2float_rd(__dsub_rd(tw, (double)ew));
                const float  whi = __double2float_ru(__dadd_ru(tw, (double)ew));
                const float  olo = __double2float_rd(__dsub_rd(to, (double)eo));
                const float  ohi = __double2float_ru(__dadd_ru(to, (double)eo));
                // walked marginal: every entry <= whi lies in the walked prefix
                int w_lo = 0, w_hi = 0;
                {
                    int clo = 0, chi = 0;
                    for (int b0 = 0; b0 < m_end; b0 += 128)
                    {
                        const int m0 = b0 + 4 * lane;
                        if (m0 < m_end)
                        {
                            const float4 a = *reinterpret_cast<const float4*>(bsw + m0);
#pragma unroll
                            for (int q = 0; q < 4; ++q)
                            {
                                const float v = f4get(a, q);
                                clo += m0 + q < m_end && v < wlo;
                                chi += m0 + q < m_end && v <= whi;
                            }
                        }
                    }
                    w_lo = __reduce_add_sync(kFull, clo);
                    w_hi = __reduce_add_sync(kFull, chi);
                }
                // other marginal: chunk from the prefetched probes, then one block
                int       o_lo, o_hi;
                const int clo = __popc(__ballot_sync(kFull, probe0 < olo)) + __popc(__ballot_sync(kFull, probe1 < olo));
                const int chi = __popc(__ballot_sync(kFull, probe0 <= ohi)) + __popc(__ballot_sync(kFull, probe1 <= ohi));
                if (clo == chi && Llen <= 64 * 64)
                {
                    const int   c0 = clo * 64;
                    const int   e0 = c0 + 2 * lane, e1 = e0 + 1;
                    const float v0 = e0 < Llen && e0 < c0 + 64 ? So[e0] : inf;
                    const float v1 = e1 < Llen && e1 < c0 + 64 ? So[e1] : inf;
                    o_lo = c0 + __reduce_add_sync(kFull, (int)(v0 < olo) + (int)(v1 < olo));
                    o_hi = c0 + __reduce_add_sync(kFull, (int)(v0 <= ohi) + (int)(v1 <= ohi));
                }
                else
                {
                    o_lo = warp_rank(So, Llen, olo, true, lane);
                    o_hi = warp_rank(So, Llen, ohi, false, lane);
                }
                // FP64 re-evaluation of both bands in one round
                const int nbw = w_hi - w_lo, nbo = o_hi - o_lo;
                int       addw = 0, addo = 0;
                for (int idx = lane; idx < nbw + nbo; idx += 32)
                {
                    if (idx < nbw)
                    {
                        const int m = w_lo + idx;
                        const int j = (int)bj[m];
                        addw += dist3d(p.X64, wx ? a1 : a2, T, i, j) <= tw;
                    }
                    else
                    {
                        const int j = (int)Po[o_lo + idx - nbw];
                        addo += dist3d(p.X64, o, T, i, j) <= to;
                    }
                }
                const int nw = w_lo + __reduce_add_sync(kFull, addw);
                const int no = o_lo + __reduce_add_sync(kFull, addo);
                const int nx = wx ? nw : no, ny = wx ? no : nw;
                out_cnt      = (uint32_t)nx | ((uint32_t)ny << 16);
            }
            if (lane == 0)
            {
                if (handoff)
                {
                    const unsigned q = atomicAdd(p.queue_len, 1u);
                    if (q < p.queue_cap)
                        p.queue[q] = ((unsigned long long)pl << 16) | (unsigned)i;
                    atomicOr(p.status, q < p.queue_cap ? kStatFallback : kStatQueueOverflow);
                    if (p.reasons)
                        atomicAdd(p.reasons + reason, 1u);
                }
                else
                    p.cnt[(size_t)i * p.pair_count + pl] = out_cnt;
            }
            __syncwarp();
        }
    }
}

// Exact FP64 statistics for the queries the walk handed over.
__global__ void __launch_bounds__(256) ksg_queue_kernel(QueueParams p)
{
    __shared__ unsigned hist[8][256];
    const int      warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned n    = min(*p.queue_len, p.queue_cap);
    for (unsigned e = blockIdx.x * 8 + warp; e < n; e += gridDim.x * 8)
    {
        const unsigned long long q  = p.queue[e];
        const long               pl = (long)(q >> 16);
        const int                i  = (int)(q & 0xFFFFu);
        int                      a1, a2;
        if (p.pair_ab)
        {
            a1 = p.pair_ab[pl].x;
            a2 = p.pair_ab[pl].y;
        }
        else
            pair_from_index(p.pair_begin + pl, &a1, &a2);
        const uint32_t c = exact_query(p.X64, p.T, p.K, a1, a2, i, p.box, p.rank_shift, hist[warp], lane);
        if (lane == 0)
            p.cnt[(size_t)i * p.pair_count + pl] = c;
    }
}

cudaError_t launch_ksg_x32(const double* X64, int natoms, int T, float4* X32, float* eps_atom, cudaStream_t s)
{
    ksg_x32_kernel<<<(natoms * 32 + 255) / 256, 256, 0, s>>>(X64, natoms, T, X32, eps_atom);
    return cudaGetLastError();
}

cudaError_t launch_ksg_rows(const float4* X32, int natoms, int T, int i0, int Q, int Lpad, float* S, uint16_t* P,
                            cudaStream_t s)
{
    int N2 = 256;
    while (N2 < T - 1)
        N2 <<= 1;
    // bucket pass up to 8192 keys (two key arrays + bins); longer rows use
    // the bitonic network alone
    const int    nbin = N2 <= 8192 ? (N2 < 4096 ? N2 : 4096) : 0;
    const size_t smem = (size_t)N2 * 8 * (nbin ? 2 : 1) + (size_t)nbin * 8;
    // static shared memory comes on top of the dynamic part: always raise
    // the limit to what this launch needs
    cudaFuncSetAttribute(ksg_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    ksg_rows_kernel<<<(unsigned)((long)natoms * Q), kRowsThreads, smem, s>>>(X32, T, i0, Q, Lpad, N2, nbin, S, P);
    return cudaGetLastError();
}

cudaError_t launch_ksg_walk(const WalkParams& p, int sms, cudaStream_t s)
{
    const size_t smem = (size_t)p.warp_smem * kWalkWarps;
    cudaFuncSetAttribute(ksg_walk_kernel<kWalkWarps>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ksg_walk_kernel<kWalkWarps>, kWalkWarps * 32, smem);
    if (per_sm < 1)
        per_sm = 1;
    ksg_walk_kernel<kWalkWarps><<<sms * per_sm, kWalkWarps * 32, smem, s>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_ksg_queue(const QueueParams& p, int sms, cudaStream_t s)
{
    ksg_queue_kernel<<<sms * 4, 256, 0, s>>>(p);
    return cudaGetLastError();
}

} // namespace gc
