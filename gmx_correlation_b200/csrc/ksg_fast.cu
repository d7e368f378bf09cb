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

// One CTA per (atom, query): sort the marginal distances of the query's
// row (T-1 values, self excluded) with their frames, as 64-bit keys
// (distance bits << 32 | frame) in shared memory.
__global__ void ksg_rows_kernel(const float4* __restrict__ X32, int T, int i0, int Q, int Lpad, int N2,
                                float* __restrict__ S, uint16_t* __restrict__ P)
{
    extern __shared__ unsigned long long keys[];
    const int row  = blockIdx.x;
    const int a    = row / Q;
    const int iq   = row - a * Q;
    const int i    = i0 + iq;
    const float4 q = X32[(size_t)a * T + i];
    for (int m = threadIdx.x; m < N2; m += blockDim.x)
    {
        unsigned long long k = ~0ull;
        if (m < T - 1)
        {
            const int j = m < i ? m : m + 1;
            const float d = dist3f(q, X32[(size_t)a * T + j]);
            k = ((unsigned long long)__float_as_uint(d) << 32) | (unsigned)j;
        }
        keys[m] = k;
    }
    __syncthreads();
    for (int k = 2; k <= N2; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1)
        {
            for (int t = threadIdx.x; t < (N2 >> 1); t += blockDim.x)
            {
                const int idx = ((t / j) * (j << 1)) + (t % j);
                const int prt = idx + j;
                const unsigned long long x = keys[idx], y = keys[prt];
                const bool up = (idx & k) == 0;
                if ((x > y) == up)
                {
                    keys[idx] = y;
                    keys[prt] = x;
                }
            }
            __syncthreads();
        }
    float*    srow = S + (size_t)row * Lpad;
    uint16_t* prow = P + (size_t)row * Lpad;
    for (int m = threadIdx.x; m < T - 1; m += blockDim.x)
    {
        const unsigned long long k = keys[m];
        srow[m] = __uint_as_float((unsigned)(k >> 32));
        prow[m] = (uint16_t)(k & 0xFFFFu);
    }
}

namespace {

// Warp-wide count of sorted row values < t (strict) or <= t.
__device__ __forceinline__ int warp_rank(const float* __restrict__ row, int n, float t, bool strict, int lane)
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

// n = #{j != i : d64(atom; i, j) <= t64} from the sorted FP32 row, exact.
__device__ int count_le_exact(const float* __restrict__ row, const uint16_t* __restrict__ perm, int n,
                              const double* __restrict__ X64, int atom, int T, int i, double t64, float eps,
                              int lane)
{
    const float lo_t = __double2float_rd(__dsub_rd(t64, (double)eps));
    const float hi_t = __double2float_ru(__dadd_ru(t64, (double)eps));
    const int   lo   = warp_rank(row, n, lo_t, true, lane);
    const int   hi   = warp_rank(row, n, hi_t, false, lane);
    int         add  = 0;
    for (int m = lo + lane; m < hi; m += 32)
        add += dist3d(X64, atom, T, i, perm[m]) <= t64;
    return lo + __reduce_add_sync(kFull, add);
}

__device__ __forceinline__ unsigned lanemask_lt(int lane) { return (1u << lane) - 1u; }

// Bitonic sort of one uint32 per lane, ascending.
__device__ __forceinline__ unsigned warp_sort_u32(unsigned v, int lane)
{
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1)
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1)
        {
            const unsigned o    = __shfl_xor_sync(kFull, v, j);
            const bool     up   = (lane & k) == 0;
            const bool     low  = (lane & j) == 0;
            const unsigned mn   = min(v, o), mxv = max(v, o);
            v                   = (low == up) ? mn : mxv;
        }
    return v;
}

// Bitonic sort of (key_hi, key_lo, payload) per lane, ascending lexicographic.
__device__ __forceinline__ void warp_sort_kv(unsigned long long& kh, unsigned long long& kl, int& pay, int lane)
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

__global__ void __launch_bounds__(kWalkWarps * 32) ksg_walk_kernel(WalkParams p)
{
    extern __shared__ unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char* base = smem_raw + (size_t)warp * p.warp_smem;
    unsigned*  hist = reinterpret_cast<unsigned*>(base);
    float*     bsw  = reinterpret_cast<float*>(base + p.nb * 4);
    float*     bdo  = bsw + p.bufcap;
    uint16_t*  bj   = reinterpret_cast<uint16_t*>(bdo + p.bufcap);
    unsigned*  list = reinterpret_cast<unsigned*>(base + walk_list_offset(p.nb, p.bufcap));
    // list layout: [0,32) u32 band / amb frames, [32,64) f32 amb dx, [64,96) f32 amb dy
    float*     ldx  = reinterpret_cast<float*>(list + 32);
    float*     ldy  = reinterpret_cast<float*>(list + 64);
    double*    l64  = reinterpret_cast<double*>(list + 96); // [0,32) dx64, [32,64) dy64

    const int       T    = p.T, K = p.K, Llen = T - 1;
    const ScanGrid  grid(p.box);
    const long long total = (long long)p.Q * p.pair_count;

    for (;;)
    {
        long long t0 = 0;
        if (lane == 0)
            t0 = (long long)atomicAdd(p.task_counter, 32ull);
        t0 = __shfl_sync(kFull, t0, 0);
        if (t0 >= total)
            break;
        const long long t1 = min(total, t0 + 32);
        for (long long t = t0; t < t1; ++t)
        {
            const int  iq = (int)(t / p.pair_count);
            const long pl = (long)(t - (long long)iq * p.pair_count);
            const int  i  = p.i0 + iq;
            int        a1, a2;
            pair_from_index(p.pair_begin + pl, &a1, &a2);
            const float*    Sa = p.S + ((size_t)a1 * p.Q + iq) * p.Lpad;
            const float*    Sb = p.S + ((size_t)a2 * p.Q + iq) * p.Lpad;
            const uint16_t* Pa = p.P + ((size_t)a1 * p.Q + iq) * p.Lpad;
            const uint16_t* Pb = p.P + ((size_t)a2 * p.Q + iq) * p.Lpad;
            const float     Ra = Sa[K - 1], Rb = Sb[K - 1];
            const bool      wx = Ra >= Rb; // walk the x (a1) marginal
            const int       o  = wx ? a2 : a1;
            const float*    Sw = wx ? Sa : Sb;
            const uint16_t* Pw = wx ? Pa : Pb;
            const float     L  = wx ? Ra : Rb;
            const unsigned  Lb = __float_as_uint(L);
            const float4    xo = p.X32[(size_t)o * T + i];
            const float*    X32o = reinterpret_cast<const float*>(p.X32 + (size_t)o * T);
            const float     ea = p.eps_atom[a1], eb = p.eps_atom[a2];
            const float     e2 = __fmul_ru(2.0f, fmaxf(ea, eb));
            bool            handoff = false;

            for (int b = lane; b < p.nb; b += 32)
                hist[b] = 0u;
            __syncwarp();

            // ---- pass 1: walk + histogram ------------------------------------
            int      cnt_lo = 0, R = 0, m_end = 0;
            unsigned thr    = 0;
            float    stop   = __int_as_float(0x7f800000);
            for (int base0 = 0; base0 < Llen; base0 += 32)
            {
                const int  m     = base0 + lane;
                const bool valid = m < Llen;
                const float sw   = valid ? Sw[m] : __int_as_float(0x7f800000);
                if (__shfl_sync(kFull, sw, 0) > stop)
                    break;
                const bool take = valid && sw <= stop;
                float      Do   = 0.0f;
                int        j    = 0;
                if (take)
                {
                    j  = Pw[m];
                    Do = dist3f(xo, *reinterpret_cast<const float4*>(X32o + 4 * (size_t)j));
                    if (m < p.bufcap)
                    {
                        bsw[m] = sw;
                        bdo[m] = Do;
                        bj[m]  = (uint16_t)j;
                    }
                }
                const float    v     = fmaxf(sw, Do);
                const bool     below = take && v < L;
                cnt_lo += __popc(__ballot_sync(kFull, below));
                if (take && !below)
                    atomicAdd(&hist[min((__float_as_uint(v) - Lb) >> p.shift, (unsigned)p.nb - 1)], 1u);
                const unsigned tm = __ballot_sync(kFull, take);
                m_end = base0 + __popc(tm);
                __syncwarp();
                if (stop == __int_as_float(0x7f800000))
                {
                    const float sl = __shfl_sync(kFull, sw, 31 - __clz(tm));
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
            }

            // element m of the walk (buffered, or re-derived past the buffer)
            auto elem = [&](int m, float& sw, float& Do, int& j) {
                if (m < p.bufcap)
                {
                    sw = bsw[m];
                    Do = bdo[m];
                    j  = bj[m];
                }
                else
                {
                    sw = Sw[m];
                    j  = Pw[m];
                    Do = dist3f(xo, *reinterpret_cast<const float4*>(X32o + 4 * (size_t)j));
                }
            };

            // ---- pass 2: bucket of the k-th value, then the band ---------------
            int acc = cnt_lo, bstar = -1, belowk = 0;
            for (int b0 = 0; b0 < p.nb; b0 += 32)
            {
                const unsigned c    = hist[b0 + lane];
                unsigned       incl = c;
#pragma unroll
                for (int s = 1; s < 32; s <<= 1)
                {
                    const unsigned y = __shfl_up_sync(kFull, incl, s);
                    if (lane >= s)
                        incl += y;
                }
                const unsigned tot = __shfl_sync(kFull, incl, 31);
                if (acc + (int)tot >= K)
                {
                    const bool here = acc + (int)(incl - c) < K && acc + (int)incl >= K;
                    const int  src  = __ffs(__ballot_sync(kFull, here)) - 1;
                    bstar           = b0 + src;
                    belowk          = acc + (int)__shfl_sync(kFull, incl - c, src);
                    break;
                }
                acc += (int)tot;
            }
            const int nband = bstar >= 0 ? (int)hist[bstar] : 0;
            if (bstar < 0 || bstar == p.nb - 1 || nband > 32)
                handoff = true;

            float d32 = 0.0f;
            if (!handoff)
            {
                int nb_seen = 0;
                for (int base0 = 0; base0 < m_end; base0 += 32)
                {
                    const int m = base0 + lane;
                    float     sw = 0.0f, Do = 0.0f;
                    int       j  = 0;
                    bool      in = false;
                    if (m < m_end)
                    {
                        elem(m, sw, Do, j);
                        const float v = fmaxf(sw, Do);
                        in = v >= L && min((__float_as_uint(v) - Lb) >> p.shift, (unsigned)p.nb - 1) == (unsigned)bstar;
                    }
                    const unsigned bm = __ballot_sync(kFull, in);
                    const int      sl = nb_seen + __popc(bm & lanemask_lt(lane));
                    if (in && sl < 32)
                        list[sl] = __float_as_uint(fmaxf(sw, Do));
                    nb_seen += __popc(bm);
                }
                __syncwarp();
                const unsigned mine   = lane < nband ? list[lane] : 0xFFFFFFFFu;
                const unsigned sorted = warp_sort_u32(mine, lane);
                d32                   = __uint_as_float(__shfl_sync(kFull, sorted, K - belowk - 1));
                __syncwarp();
            }

            // ---- pass 3: certain members and the ambiguous band ----------------
            float mx_in = 0.0f, my_in = 0.0f;
            int   n_in = 0, n_amb = 0;
            float lower = 0.0f, upper = 0.0f;
            if (!handoff)
            {
                lower = __fsub_rd(d32, e2);
                upper = __fadd_ru(d32, e2);
                for (int base0 = 0; base0 < m_end; base0 += 32)
                {
                    const int m = base0 + lane;
                    float     sw = 0.0f, Do = 0.0f;
                    int       j  = 0;
                    bool      in = false, amb = false;
                    float     dx = 0.0f, dy = 0.0f;
                    if (m < m_end)
                    {
                        elem(m, sw, Do, j);
                        const float v = fmaxf(sw, Do);
                        dx            = wx ? sw : Do;
                        dy            = wx ? Do : sw;
                        in            = v < lower;
                        amb           = !in && v <= upper;
                        if (in)
                        {
                            mx_in = fmaxf(mx_in, dx);
                            my_in = fmaxf(my_in, dy);
                        }
                    }
                    n_in += __popc(__ballot_sync(kFull, in));
                    const unsigned am = __ballot_sync(kFull, amb);
                    if (amb)
                    {
                        const int slot = n_amb + __popc(am & lanemask_lt(lane));
                        if (slot < 32)
                        {
                            list[slot] = (unsigned)j;
                            ldx[slot]  = dx;
                            ldy[slot]  = dy;
                        }
                    }
                    n_amb += __popc(am);
                }
                if (n_amb > 32 || n_amb < 1)
                    handoff = true;
                __syncwarp();
            }

            uint32_t out_cnt = 0;
            if (!handoff)
            {
                mx_in = warp_max((double)mx_in);
                my_in = warp_max((double)my_in);
                // ---- pass 4: exact order of the ambiguous band ----------------
                const double* xa0 = p.X64 + (size_t)a1 * 3 * T;
                const double* xb0 = p.X64 + (size_t)a2 * 3 * T;
                const int     ix  = grid.qcell(xa0[i]);
                const int     iy  = grid.qcell(xb0[i]);
                unsigned long long kh = ~0ull, kl = ~0ull;
                int                slot = lane;
                if (lane < n_amb)
                {
                    const int    j    = (int)list[lane];
                    const double dx64 = dist3d(p.X64, a1, T, i, j);
                    const double dy64 = dist3d(p.X64, a2, T, i, j);
                    l64[lane]         = dx64;
                    l64[32 + lane]    = dy64;
                    kh                = dbits(fmax(dx64, dy64));
                    kl                = grid.rank(ix, iy, xa0[j], xb0[j], j, T);
                }
                __syncwarp();
                warp_sort_kv(kh, kl, slot, lane);
                const int need   = K - n_in;
                if (need < 1 || need > n_amb)
                    handoff = true; // cannot happen with a valid error bound; stay exact anyway
                const bool chosen = !handoff && lane < need;
                float  cx32 = 0.0f, cy32 = 0.0f;
                double cx64 = 0.0, cy64 = 0.0;
                if (chosen)
                {
                    cx32 = ldx[slot];
                    cy32 = ldy[slot];
                    cx64 = l64[slot];
                    cy64 = l64[32 + slot];
                }
                const float Mx = fmaxf(mx_in, (float)warp_max((double)cx32));
                const float My = fmaxf(my_in, (float)warp_max((double)cy32));
                double ex64 = warp_max(cx64), ey64 = warp_max(cy64);
                // ---- pass 5: certain members that may hold the FP64 maxima -----
                const float tx = __fsub_rd(Mx, __fmul_ru(2.0f, ea));
                const float ty = __fsub_rd(My, __fmul_ru(2.0f, eb));
                for (int base0 = 0; base0 < m_end; base0 += 32)
                {
                    const int m = base0 + lane;
                    if (m < m_end)
                    {
                        float sw, Do;
                        int   j;
                        elem(m, sw, Do, j);
                        const float v = fmaxf(sw, Do);
                        if (v < lower)
                        {
                            const float dx = wx ? sw : Do, dy = wx ? Do : sw;
                            if (dx >= tx)
                                ex64 = fmax(ex64, dist3d(p.X64, a1, T, i, j));
                            if (dy >= ty)
                                ey64 = fmax(ey64, dist3d(p.X64, a2, T, i, j));
                        }
                    }
                }
                ex64 = warp_max(ex64);
                ey64 = warp_max(ey64);
                // ---- counts --------------------------------------------------
                if (!handoff)
                {
                    const int nx = count_le_exact(Sa, Pa, Llen, p.X64, a1, T, i, ex64, ea, lane);
                    const int ny = count_le_exact(Sb, Pb, Llen, p.X64, a2, T, i, ey64, eb, lane);
                    out_cnt      = (uint32_t)nx | ((uint32_t)ny << 16);
                }
            }
            if (lane == 0)
            {
                if (handoff)
                {
                    const unsigned q = atomicAdd(p.queue_len, 1u);
                    if (q < p.queue_cap)
                        p.queue[q] = ((unsigned long long)pl << 16) | (unsigned)i;
                    atomicOr(p.status, q < p.queue_cap ? kStatFallback : kStatQueueOverflow);
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
        pair_from_index(p.pair_begin + pl, &a1, &a2);
        const uint32_t c = exact_query(p.X64, p.T, p.K, a1, a2, i, p.box, p.rank_shift, hist[warp], lane);
        if (lane == 0)
            p.cnt[(size_t)i * p.pair_count + pl] = c;
    }
}

void launch_ksg_x32(const double* X64, int natoms, int T, float4* X32, float* eps_atom, cudaStream_t s)
{
    ksg_x32_kernel<<<(natoms * 32 + 255) / 256, 256, 0, s>>>(X64, natoms, T, X32, eps_atom);
}

void launch_ksg_rows(const float4* X32, int natoms, int T, int i0, int Q, int Lpad, float* S, uint16_t* P,
                     cudaStream_t s)
{
    int N2 = 1;
    while (N2 < T - 1)
        N2 <<= 1;
    const size_t smem = (size_t)N2 * 8;
    if (smem > 48 * 1024)
        cudaFuncSetAttribute(ksg_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    ksg_rows_kernel<<<(unsigned)((long)natoms * Q), 256, smem, s>>>(X32, T, i0, Q, Lpad, N2, S, P);
}

void launch_ksg_walk(const WalkParams& p, int sms, cudaStream_t s)
{
    const size_t smem = (size_t)p.warp_smem * kWalkWarps;
    cudaFuncSetAttribute(ksg_walk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ksg_walk_kernel, kWalkWarps * 32, smem);
    if (per_sm < 1)
        per_sm = 1;
    ksg_walk_kernel<<<sms * per_sm, kWalkWarps * 32, smem, s>>>(p);
}

void launch_ksg_queue(const QueueParams& p, int sms, cudaStream_t s)
{
    ksg_queue_kernel<<<sms * 4, 256, 0, s>>>(p);
}

} // namespace gc
