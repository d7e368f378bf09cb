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
//   ksg_walk_kernel   one pair per CTA task, 32 consecutive queries per warp,
//                     one query per lane.  Each lane walks the sorted row of the
//                     marginal whose k-th distance is larger, gathering the
//                     other marginal, and histograms the joint distances in
//                     its own shared-memory column (anchored at the exact
//                     lower bound max(k-th marginal distances)) until the
//                     joint k-th distance is provably behind.  The bucket of
//                     the k-th value then bounds a band that two short ranges
//                     of the two sorted rows enumerate; the members' marginal
//                     maxima come from backward scans of the same rows.
//                     Everything within the proven error band 2*eps of a
//                     decision is re-evaluated in FP64 on the reference's
//                     normalised coordinates, with the reference's grid-scan
//                     order deciding exact ties, so n_x and n_y equal the
//                     reference's counts.  Counts come from binary search in
//                     the sorted rows, with FP64 repair of the band around
//                     eps_x / eps_y.
//   ksg_fixup_kernel  queries a lane hands over (k-th value outside the
//                     histogram, oversized bands) are marked in the count
//                     array and recomputed here by the exact FP64 code.
//
// Error bound (x32 = fl32(x64 - c), c the component midrange, |x64-c| <= R):
//   |fl32(x32_i - x32_j) - fl64(x64_i - x64_j)| <= 4 u R (1 + 2^-20),
//   u = 2^-24, and max over components keeps the bound; eps_a = R_a * 2^-21
//   (twice that) is used.

#include "gc_common.cuh"
#include "gc_internal.h"
#include "ksg_exact_query.cuh"
#include "ksg_fast.h"
#include "row_sort.cuh"

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

// One warp per atom: component midranges c = (min + max) / 2 (for the
// min-shifted rows kraskov_prepare makes, max / 2), centred FP32 coordinates
// and the atom's error bound from the largest half-range R.
__global__ void ksg_x32_kernel(const double* __restrict__ X64, int natoms, int T, float4* __restrict__ X32,
                               float* __restrict__ eps_atom)
{
    const int lane = threadIdx.x & 31;
    const int a    = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (a >= natoms)
        return;
    const double* r = X64 + (size_t)a * 3 * T;
    double        c[3], R = 0.0;
    for (int d = 0; d < 3; ++d)
    {
        double lo = r[(size_t)d * T], hi = lo;
        for (int f = lane; f < T; f += 32)
        {
            lo = fmin(lo, r[(size_t)d * T + f]);
            hi = fmax(hi, r[(size_t)d * T + f]);
        }
        lo   = -warp_max(-lo);
        hi   = warp_max(hi);
        c[d] = 0.5 * (lo + hi);
        R    = fmax(R, fmax(hi - c[d], c[d] - lo));
    }
    for (int f = lane; f < T; f += 32)
        X32[(size_t)a * T + f] = make_float4((float)(r[f] - c[0]), (float)(r[T + f] - c[1]),
                                             (float)(r[2 * T + f] - c[2]), 0.0f);
    if (lane == 0)
        eps_atom[a] = __double2float_ru(R * (1.0 + 0x1p-40) * 0x1p-21) + 1e-30f;
}

// The descriptor owning task t: the largest d with prefix[d] <= t.
__device__ __forceinline__ int batch_desc(const long long* __restrict__ prefix, int n, long long t)
{
    int lo = 0, hi = n - 1;
    while (lo < hi)
    {
        const int mid = (lo + hi + 1) >> 1;
        if (prefix[mid] <= t)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// One CTA per (atom, query) of the launch's query blocks: the row's T-1
// marginal distances (self excluded), sorted ascending with their frames
// (sort_row).
template <int THREADS, int R>
__global__ void __launch_bounds__(THREADS) ksg_rows_kernel(WalkBatch B)
{
    // row blockIdx.x of the launch -> descriptor, atom, query of its block
    const long long   r   = blockIdx.x;
    const int         dsc = batch_desc(B.rprefix, B.n, r);
    const WalkParams& w   = B.d[dsc];
    const int         T = w.T, Q = w.Q, Qp = w.Qp, Lpad = w.Lpad;
    const int         row = (int)(r - B.rprefix[dsc]);
    const int         a   = row / Q;
    const int         iq  = row - a * Q;
    const int         i   = w.i0 + iq;
    const float4*     xr  = w.X32 + (size_t)a * T;
    const float4      q   = xr[i];
    __shared__ RowSortShared<THREADS> sh;
    sort_row<THREADS, R>(
        sh, T - 1, i, [&](int j) { return dist3f(q, xr[j]); }, w.S, w.P, ((size_t)a * (Lpad >> 2) * Qp + iq) * 4,
        (size_t)Qp * 4, w.U ? w.U + ((size_t)a * Qp + iq) * w.Tpad : nullptr);
}

namespace {

// One lane's view of a transposed sorted row (see WalkParams).
struct LaneRow
{
    const float*    S;
    const uint16_t* P;
    size_t          gstride; // elements between consecutive 4-entry groups

    __device__ __forceinline__ float  s(int m) const { return S[(size_t)(m >> 2) * gstride + (m & 3)]; }
    __device__ __forceinline__ int    j(int m) const { return P[(size_t)(m >> 2) * gstride + (m & 3)]; }
    __device__ __forceinline__ float4 s4(int g) const
    {
        return *reinterpret_cast<const float4*>(S + (size_t)g * gstride);
    }
    __device__ __forceinline__ uint2 j4(int g) const { return *reinterpret_cast<const uint2*>(P + (size_t)g * gstride); }
};

// Entry q (0..3) of a 4-entry group: its distance and its frame.
__device__ __forceinline__ float f4get(const float4& v, int q)
{
    return q == 0 ? v.x : (q == 1 ? v.y : (q == 2 ? v.z : v.w));
}

__device__ __forceinline__ unsigned u2get16(const uint2& v, int q)
{
    return q < 2 ? ((v.x >> (16 * q)) & 0xFFFFu) : ((v.y >> (16 * (q - 2))) & 0xFFFFu);
}

__device__ __forceinline__ LaneRow lane_row(const WalkParams& p, int atom, int iq)
{
    const size_t base = ((size_t)atom * (p.Lpad >> 2) * p.Qp + iq) * 4;
    return LaneRow{p.S + base, p.P + base, (size_t)p.Qp * 4};
}

// Four independent binary searches advanced together, so their loads
// overlap: lo[q] becomes the first position in [lo[q], hi[q]] of row r[q]
// whose value is not < t[q] (strict[q]) / not <= t[q].
__device__ __forceinline__ void row_bounds4(const LaneRow (&r)[4], int (&lo)[4], int (&hi)[4], const float (&t)[4],
                                            const bool (&strict)[4])
{
    for (;;)
    {
        int   mid[4];
        float v[4];
        bool  any = false;
#pragma unroll
        for (int q = 0; q < 4; ++q)
        {
            mid[q] = (lo[q] + hi[q]) >> 1;
            v[q]   = lo[q] < hi[q] ? r[q].s(mid[q]) : 0.0f;
        }
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (lo[q] < hi[q])
            {
                if (strict[q] ? v[q] < t[q] : v[q] <= t[q])
                    lo[q] = mid[q] + 1;
                else
                    hi[q] = mid[q];
                any |= lo[q] < hi[q];
            }
        if (!any)
            break;
    }
}

__device__ __forceinline__ double dist3r(const double* __restrict__ r, int T, double q0, double q1, double q2, int j)
{
    return fmax(fmax(fabs(q0 - r[j]), fabs(q1 - r[T + j])), fabs(q2 - r[2 * T + j]));
}

constexpr int kScanCap = 1024; // row entries a backward scan may visit
constexpr int kAmbCap  = 8;    // ambiguous entries ordered in FP64

// Hand-over causes (WalkParams::reasons index).
enum
{
    kReasonRange    = 2, // k-th value beyond the histogram's two octaves
    kReasonBand     = 3, // band larger than kBandCap or inconsistent with the histogram
    kReasonAmbig    = 4, // ambiguous set inconsistent or larger than kAmbCap
    kReasonScan     = 5, // backward scan for the maxima exceeded kScanCap
    kReasonPrefix   = 6  // count band reaches beyond the walked prefix
};

} // namespace

namespace {

// Per-lane view of one (pair, query): the walked marginal w is the atom with
// the larger k-th marginal distance L (an exact lower bound of the joint
// k-th distance), o the other one.
struct LaneSetup
{
    bool          wx; // the walked marginal is x (atom a1)
    int           w, o;
    LaneRow       rw, ro;
    float         L;
    unsigned      Lb;
    const float4* X32w;
    const float4* X32o;
    float4        xw, xo;
    float         ew, eo, e2;
};

// xa / xb: the coordinate rows of a1 / a2 (global memory or the CTA's
// shared-memory copy).
__device__ __forceinline__ LaneSetup lane_setup(const WalkParams& p, int a1, int a2, int iql, int i, const float4* xa,
                                                const float4* xb)
{
    LaneSetup     u;
    const LaneRow ra = lane_row(p, a1, iql), rb = lane_row(p, a2, iql);
    const float   Ra = ra.s(p.K - 1), Rb = rb.s(p.K - 1);
    u.wx             = Ra >= Rb;
    u.w              = u.wx ? a1 : a2;
    u.o              = u.wx ? a2 : a1;
    u.rw             = u.wx ? ra : rb;
    u.ro             = u.wx ? rb : ra;
    u.L              = u.wx ? Ra : Rb;
    u.Lb             = __float_as_uint(u.L);
    u.X32w           = u.wx ? xa : xb;
    u.X32o           = u.wx ? xb : xa;
    u.xw             = u.X32w[i];
    u.xo             = u.X32o[i];
    const float ea = p.eps_atom[a1], eb = p.eps_atom[a2];
    u.ew             = u.wx ? ea : eb;
    u.eo             = u.wx ? eb : ea;
    u.e2             = __fmul_ru(2.0f, fmaxf(ea, eb));
    return u;
}

// CTA task t of a query block: chunk c of B.chunk query groups of 32
// consecutive queries, which the CTA's warps take one group at a time, for
// the pair pair_order[k] (pairs in atom-tile order, so the rows the running
// tasks read stay in L2).  Every thread of the CTA calls next_task; it ends
// with a barrier.
struct Task
{
    int  c;
    long pl;
    int  a1, a2;
};

__device__ __forceinline__ void task_pair(const WalkParams& p, long k, Task& tk)
{
    tk.pl = p.pair_order ? (long)p.pair_order[k] : k;
    if (p.pair_ab)
    {
        tk.a1 = p.pair_ab[tk.pl].x;
        tk.a2 = p.pair_ab[tk.pl].y;
    }
    else
        pair_from_index(p.pair_begin + tk.pl, &tk.a1, &tk.a2);
}

__device__ __forceinline__ bool next_task(const WalkBatch& B, long long total, long long* s_task, int* s_desc,
                                          int* s_next, Task& tk, int& d)
{
    if (threadIdx.x == 0)
    {
        const long long t = (long long)atomicAdd(B.counter, 1ull);
        *s_task           = t;
        *s_next           = 0;
        if (t < total)
            *s_desc = batch_desc(B.wprefix, B.n, t);
    }
    __syncthreads();
    const long long t = *s_task;
    if (t >= total)
        return false;
    d                   = *s_desc;
    const WalkParams& p = B.d[d];
    const long long   lt = t - B.wprefix[d];
    tk.c                 = (int)(lt / p.pair_count);
    task_pair(p, (long)(lt - (long long)tk.c * p.pair_count), tk);
    return true;
}

// Walk result of one (pair, query): bucket of the k-th value, the number of
// entries below that bucket, the walked length, and a hand-over cause.
__device__ __forceinline__ unsigned long long pack_walk(int bstar, int prefix, int m_end, int reason)
{
    return (unsigned long long)(bstar & 0xFF) | ((unsigned long long)(prefix & 0xFFFF) << 8) |
           ((unsigned long long)(m_end & 0xFFFF) << 24) | ((unsigned long long)(reason & 0xFF) << 40);
}

} // namespace

// One query group of a walk task (pass 1 below): lane iq = g * 32 + lane
// walks the sorted row of its query and histograms v = max(s, d), d the other
// marginal's FP32 distance to the entry's frame, dist_other(frame).  Writes
// the lane's walk result; clears and uses this warp's histogram at base.
template <bool LO, class DistFn>
__device__ __forceinline__ void walk_query_group(const WalkParams& p, long pl, int iq, bool live, const LaneSetup& u,
                                                 DistFn&& dist_other, unsigned char* base, int lane)
{
    const int          K = p.K, Llen = p.T - 1, shift = p.shift;
    uint8_t*           hist = base + lane * 4;
    auto               H    = [hist](unsigned b) -> uint8_t& { return hist[(b >> 2) * 128 + (b & 3)]; };
    constexpr unsigned kTop = kWalkBuckets - 1; // open-ended index above the range, never read
    const float        inf  = __int_as_float(0x7f800000);
    {
        uint4* h4 = reinterpret_cast<uint4*>(base);
        for (int e = lane; e < kWalkBuckets * 32 / 16; e += 32)
            h4[e] = make_uint4(0u, 0u, 0u, 0u);
    }
    __syncwarp();

    // Histogram index of v: LO: 0 for v < L, then buckets of 2^shift
    // float ulps from L; otherwise buckets from L (v < L counted in
    // cnt_lo).  Index b starts at value bits Lh + (b << shift) (b >= 1
    // when LO); the last index takes everything above the range.
    const unsigned Lh   = LO ? u.Lb - (1u << shift) : u.Lb;
    auto           hidx = [Lh, shift](float v) -> unsigned {
        if (LO)
            return (unsigned)min(max((int)(__float_as_uint(v) - Lh) >> shift, 0), (int)kTop);
        return min((__float_as_uint(v) - Lh) >> shift, kTop);
    };
    // Every 16 entries the indices below the current value are final
    // (later entries have v >= s), so their running sum R decides the stop
    // value.  The rows end in NaN up to a 4-entry boundary, which the
    // take test (s <= stop) never passes, so taken entries form a prefix
    // of each group and a group short of 4 ends the walk.
    const float4* Sg = reinterpret_cast<const float4*>(u.rw.S); // 4-entry groups of this lane's row
    const uint2*  Pg = reinterpret_cast<const uint2*>(u.rw.P);
    const size_t  gs = (size_t)p.Qp;                            // group stride
    int           m_end = 0, cnt_lo = 0, R = 0, thr = 0, grp = 0;
    unsigned      wrap = 0u; // bit 8 set once a counter below the top passed 255
    float         stop = inf;
    bool          walking = live;
    float4        s4      = make_float4(inf, inf, inf, inf);
    uint2         j4      = make_uint2(0u, 0u);
    if (live)
    {
        s4 = Sg[0];
        j4 = Pg[0];
    }
    const int last = (Llen - 1) >> 2; // the last (possibly partial) group
    while (walking)
    {
        if (grp > last) // the whole row walked
        {
            m_end = Llen;
            break;
        }
        // prefetch the next group (the last group again at the end)
        const int      nxt   = grp < last ? grp + 1 : grp;
        const float4   ns4   = Sg[(size_t)nxt * gs];
        const uint2    nj4   = Pg[(size_t)nxt * gs];
        const float    sv[4] = {s4.x, s4.y, s4.z, s4.w};
        const unsigned jv[4] = {j4.x & 0xFFFFu, j4.x >> 16, j4.y & 0xFFFFu, j4.y >> 16};
        bool           tkn[4];
        // Branch-free: every slot gathers and adds 0 or 1 to its counter.
#pragma unroll
        for (int q = 0; q < 4; ++q)
        {
            tkn[q]          = sv[q] <= stop;
            const float v   = fmaxf(sv[q], dist_other(jv[q]));
            bool        inc = tkn[q];
            if (!LO)
            {
                const bool below = v < u.L;
                cnt_lo += inc && below;
                inc = inc && !below;
            }
            uint8_t&       c  = H(hidx(v));
            const unsigned h1 = (unsigned)c + (inc ? 1u : 0u);
            c                 = (uint8_t)h1;
            wrap |= h1;
        }
        ++grp;
        if (!tkn[3])
        {
            walking = false;
            m_end   = (grp - 1) * 4 + (int)tkn[0] + (int)tkn[1] + (int)tkn[2];
        }
        else if ((grp & 3) == 0)
        {
            H(kTop) = 0; // at most 16 increments between clears: never wraps
            if (stop == inf)
            {
                const float sl = sv[3];
                const int   bn = (LO || sl >= u.L) ? (int)hidx(sl) : 0;
                for (int b = thr; b < bn; ++b)
                    R += H(b);
                thr = max(thr, bn);
                if (cnt_lo + R >= K)
                    stop = __fadd_ru(__uint_as_float(Lh + ((unsigned)bn << shift)), u.e2);
            }
        }
        s4 = ns4;
        j4 = nj4;
    }

    // histogram index of the k-th value
    if (live)
    {
        int bstar, prefix;
        if (stop != inf)
        {
            // cum = #{v below index b + 1} >= K; step down while still >= K
            int cum = cnt_lo + R, b = thr - 1;
            while (b > 0 && cum - (int)H(b) >= K)
            {
                cum -= H(b);
                --b;
            }
            bstar  = b;
            prefix = cum - H(b);
        }
        else
        {
            int cum = cnt_lo, b = 0;
            while (b < (int)kTop && cum + (int)H(b) < K)
            {
                cum += H(b);
                ++b;
            }
            bstar  = b;
            prefix = cum;
        }
        // index 0 under LO holds fewer than k entries, so the k-th value
        // lies above it unless the input is not finite
        const int reason = (wrap > 255u || (LO && bstar == 0)) ? kReasonBand
                           : (bstar >= (int)kTop ? kReasonRange : 0);
        // the result names buckets from L (index - 1 under LO)
        p.wres[(size_t)pl * p.Q + iq] = pack_walk(LO ? bstar - 1 : bstar, prefix, m_end, reason);
    }
    if (p.walk_elems)
    {
        const unsigned we = __reduce_add_sync(kFull, live ? (unsigned)m_end : 0u);
        if (lane == 0 && we)
            atomicAdd(p.walk_elems, (unsigned long long)we);
    }}

// Pass 1: walk the sorted row, histogram v = max(s, d) per lane.  STAGED:
// the pair's coordinate rows are copied into shared memory per task.  LO
// (every k of the launch below 256): entries below the lower bound L count
// in histogram index 0 (at most k - 1 of them: they all have s < L, the k-th
// walked-row value), so the per-entry update needs no separate test.  GU:
// the other marginal's distance d is read from its unsorted row in HBM
// (WalkParams::U) instead of being recomputed from coordinates.
template <bool STAGED, bool LO, bool GU>
__global__ void __launch_bounds__(1024, 1) ksg_walk_kernel(WalkBatch B)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ long long s_task;
    __shared__ int       s_desc, s_next;
    const int            warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float4*              sx   = reinterpret_cast<float4*>(smem_raw);
    // this warp's histogram: index b of a lane is byte b % 4 of word
    // (b / 4) * 32 + lane, so the 32 lanes of a warp always hit 32 different banks
    unsigned char*       base = smem_raw + (STAGED ? (size_t)2 * B.maxT * 16 : 0) + (size_t)warp * kWalkBuckets * 32;

    const long long total = B.wprefix[B.n];
    Task            tk;
    int             dsc;
    while (next_task(B, total, &s_task, &s_desc, &s_next, tk, dsc))
    {
        const WalkParams& p       = B.d[dsc];
        const int         T       = p.T;
        const int         ngroups = (p.Q + 31) >> 5;
        const float4* xa = p.X32 + (size_t)tk.a1 * T;
        const float4* xb = p.X32 + (size_t)tk.a2 * T;
        if (STAGED)
        {
            for (int e = threadIdx.x; e < T; e += blockDim.x)
            {
                sx[e]     = xa[e];
                sx[T + e] = xb[e];
            }
            __syncthreads();
            xa = sx;
            xb = sx + T;
        }
        // the task's query groups go to whichever warp asks next, so warps
        // that finish early take more groups of the same pair
        for (;;)
        {
        int gi = 0;
        if (lane == 0)
            gi = atomicAdd(&s_next, 1);
        gi = __shfl_sync(kFull, gi, 0);
        const int g = tk.c * B.chunk + gi;
        if (gi >= B.chunk || g >= ngroups)
            break;
        const int       iq   = g * 32 + lane;
        const bool      live = g < ngroups && iq < p.Q;
        const int       iql  = live ? iq : 0;
        const LaneSetup u    = lane_setup(p, tk.a1, tk.a2, iql, p.i0 + iql, xa, xb);
        // the other atom's coordinate row (shared memory when staged), or
        // its unsorted distance row of this query
        const float4* X32o = STAGED ? (u.wx ? sx + T : sx) : u.X32o;
        const float*  Uo   = GU ? p.U + ((size_t)u.o * p.Qp + iql) * p.Tpad : nullptr;
        if (GU)
            walk_query_group<LO>(p, tk.pl, iq, live, u, [&](unsigned j) { return Uo[j]; }, base, lane);
        else
            walk_query_group<LO>(p, tk.pl, iq, live, u, [&](unsigned j) { return dist3f(u.xo, X32o[j]); }, base,
                                 lane);
        __syncwarp(); // the next group clears this warp's histogram
        }
        __syncthreads(); // every warp is done with the staged rows
    }
}

// Pass 1, double-buffered: the CTA holds two walk tasks' coordinate rows in
// shared memory, x and y as float2 and z apart (12 bytes a frame, so two
// pairs and 32 warps' histograms fit), and warps move from a task to the
// next without a CTA barrier: a warp that finds no query group left in task
// i goes on to task i + 1 (the other buffer), and the last warp to leave
// task i refills its buffer with task i + 2.  Tasks are fetched from the
// global counter in local-index order (the refill of task i + 2 follows
// every warp's leaving task i, hence the refill of task i + 1), so once a
// slot finds no task none of the later ones can.  The distances are computed
// with the same FP32 operations as dist3f, so the results equal the
// single-buffered walk's.
struct WalkSlot
{
    long long    t;      // global walk task, or -1: no more tasks
    int          desc;   // descriptor of the task
    int          next;   // query groups handed out
    int          left;   // warps done with the task
    volatile int gen;    // CTA-local index of the task this slot holds
    Task         tk;
};

// Fills slot s with the next global walk task as CTA-local task `gen`: one
// warp (lane 0 takes the task, all lanes copy the pair's rows).
__device__ __forceinline__ void walk_slot_fill(const WalkBatch& B, WalkSlot& S, float2* xy, float* z, int gen,
                                               int lane)
{
    long long t = 0;
    int       d = 0;
    if (lane == 0)
    {
        t = (long long)atomicAdd(B.counter, 1ull);
        if (t < B.wprefix[B.n])
            d = batch_desc(B.wprefix, B.n, t);
        else
            t = -1;
    }
    t = __shfl_sync(kFull, t, 0);
    d = __shfl_sync(kFull, d, 0);
    Task tk{};
    if (t >= 0)
    {
        const WalkParams& p  = B.d[d];
        const long long   lt = t - B.wprefix[d];
        tk.c                 = (int)(lt / p.pair_count);
        task_pair(p, (long)(lt - (long long)tk.c * p.pair_count), tk);
        const int     T  = p.T;
        const float4* xa = p.X32 + (size_t)tk.a1 * T;
        const float4* xb = p.X32 + (size_t)tk.a2 * T;
        for (int e = lane; e < T; e += 32)
        {
            const float4 va = xa[e], vb = xb[e];
            xy[e]     = make_float2(va.x, va.y);
            z[e]      = va.z;
            xy[T + e] = make_float2(vb.x, vb.y);
            z[T + e]  = vb.z;
        }
    }
    __syncwarp();
    if (lane == 0)
    {
        S.t    = t;
        S.desc = d;
        S.tk   = tk;
        S.next = 0;
        S.left = 0;
        __threadfence_block(); // the rows and fields before the generation
        S.gen = gen;
    }
    __syncwarp();
}

template <bool LO>
__global__ void __launch_bounds__(1024, 1) ksg_walk_db_kernel(WalkBatch B)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ WalkSlot slot[2];
    const int           warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    const int           maxT = B.maxT;
    // buffer b: xy [2 * maxT] float2 then z [2 * maxT] float (atom a1's rows, then a2's)
    auto xyb = [&](int b) { return reinterpret_cast<float2*>(smem_raw + (size_t)b * 24 * maxT); };
    auto zb  = [&](int b) { return reinterpret_cast<float*>(smem_raw + (size_t)b * 24 * maxT + (size_t)16 * maxT); };
    unsigned char* base = smem_raw + (size_t)48 * maxT + (size_t)warp * kWalkBuckets * 32;
    // A CTA's tasks must be fetched in the order of their local index: a warp
    // stops at the first slot without a task, so no later slot may hold one.
    // One warp therefore fills both slots, slot 0 first.
    if (warp == 0)
    {
        walk_slot_fill(B, slot[0], xyb(0), zb(0), 0, lane);
        walk_slot_fill(B, slot[1], xyb(1), zb(1), 1, lane);
    }
    __syncthreads();
    for (int i = 0;; ++i)
    {
        const int b  = i & 1;
        WalkSlot& S  = slot[b];
        // the slot holds task i once the warp that refilled it has published it;
        // the wait is bounded (the refilling warp is resident and never waits)
        int spins = 0;
        while (S.gen != i)
        {
            if (++spins > (1 << 24))
            {
                if (lane == 0)
                    atomicOr(B.d[0].status, kStatTimeout);
                return;
            }
            __nanosleep(64);
        }
        __threadfence_block();
        if (S.t < 0)
            break;
        const WalkParams& p       = B.d[S.desc];
        const Task        tk      = S.tk;
        const int         T       = p.T;
        const int         ngroups = (p.Q + 31) >> 5;
        const float2*     xy      = xyb(b);
        const float*      z       = zb(b);
        const float4*     ga      = p.X32 + (size_t)tk.a1 * T;
        const float4*     gb      = p.X32 + (size_t)tk.a2 * T;
        for (;;)
        {
            int gi = 0;
            if (lane == 0)
                gi = atomicAdd(&S.next, 1);
            gi          = __shfl_sync(kFull, gi, 0);
            const int g = tk.c * B.chunk + gi;
            if (gi >= B.chunk || g >= ngroups)
                break;
            const int       iq   = g * 32 + lane;
            const bool      live = iq < p.Q;
            const int       iql  = live ? iq : 0;
            const LaneSetup u    = lane_setup(p, tk.a1, tk.a2, iql, p.i0 + iql, ga, gb);
            const float2*   oxy  = u.wx ? xy + T : xy;
            const float*    oz   = u.wx ? z + T : z;
            walk_query_group<LO>(
                p, tk.pl, iq, live, u,
                [&](unsigned j) {
                    const float2 v = oxy[j];
                    return fmaxf(fmaxf(fabsf(u.xo.x - v.x), fabsf(u.xo.y - v.y)), fabsf(u.xo.z - oz[j]));
                },
                base, lane);
            __syncwarp(); // the next group clears this warp's histogram
        }
        int last = 0;
        if (lane == 0)
            last = atomicAdd(&S.left, 1) == nwarps - 1;
        last = __shfl_sync(kFull, last, 0);
        if (last) // every warp has left task i: its buffer takes task i + 2
            walk_slot_fill(B, S, xyb(b), zb(b), i + 2, lane);
    }
}

// Pass 2: from the walk's k-th bucket to n_x, n_y (or a hand-over).
__global__ void __launch_bounds__(kFinishWarps * 32, 1) ksg_finish_kernel(WalkBatch B)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int      warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char* base = smem_raw + (size_t)warp * kBandSlotBytes * kBandCap * 32;
    // per-lane columns: band entry e of lane l at [e * 32 + l]: joint value v,
    // walked-marginal value s, other-marginal value d and the row position as
    // an offset from the start of its range (the walked-row range holds the
    // first entries, the other-row range the rest)
    float*    bv = reinterpret_cast<float*>(base) + lane;
    float*    bs = bv + kBandCap * 32;
    float*    bd = bs + kBandCap * 32;
    uint16_t* bo = reinterpret_cast<uint16_t*>(bd + kBandCap * 32 - lane) + lane;

    const long long total = B.fprefix[B.n];
    for (;;)
    {
        // warp task: query group g outer, pairs (in tile order) inner, so
        // the warps running at once share the sorted rows of a query group
        long long t   = 0;
        int       dsc = 0;
        if (lane == 0)
        {
            t = (long long)atomicAdd(B.counter + 1, 1ull);
            if (t < total)
                dsc = batch_desc(B.fprefix, B.n, t);
        }
        t   = __shfl_sync(kFull, t, 0);
        dsc = __shfl_sync(kFull, dsc, 0);
        if (t >= total)
            break;
        const WalkParams& p  = B.d[dsc];
        const int         T  = p.T, K = p.K, Llen = T - 1, shift = p.shift;
        const ScanGrid    grid(p.box);
        const long long   lt = t - B.fprefix[dsc];
        Task              tk;
        const int         g = (int)(lt / p.pair_count);
        task_pair(p, (long)(lt - (long long)g * p.pair_count), tk);
        const float4* xa   = p.X32 + (size_t)tk.a1 * T;
        const float4* xb   = p.X32 + (size_t)tk.a2 * T;
        const int     iq   = g * 32 + lane;
        const bool    live = iq < p.Q;
        if (live)
        {
            const int                a1 = tk.a1, a2 = tk.a2;
            const int                i  = p.i0 + iq;
            const unsigned long long wr = p.wres[(size_t)tk.pl * p.Q + iq];
            const int                bstar = (int)(wr & 0xFF), prefix = (int)((wr >> 8) & 0xFFFF);
            const int                m_end = (int)((wr >> 24) & 0xFFFF);
            int                      reason = (int)((wr >> 40) & 0xFF);
            if (m_end > Llen) // not a walk result: never read past the row
                reason = kReasonBand;
            uint32_t                 out    = kHandOver;
            const LaneSetup          u      = lane_setup(p, a1, a2, iq, i, xa, xb);
            const bool     wx = u.wx;
            const LaneRow& rw = u.rw;
            const LaneRow& ro = u.ro;
            const unsigned Lb = u.Lb;
            const float4*  X32w = u.X32w;
            const float4*  X32o = u.X32o;
            const float4   xw = u.xw, xo = u.xo;
            const float    ew = u.ew, eo = u.eo, e2 = u.e2;
            if (reason == 0)
            {
                // ---- band: every entry with inlo <= v <= bandhi, from two row ranges
                const float elo    = __uint_as_float(Lb + ((unsigned)bstar << shift));
                const float ehi    = __uint_as_float(Lb + ((unsigned)(bstar + 1) << shift));
                const float inlo   = __fsub_rd(elo, e2);
                const float bandhi = __fadd_ru(ehi, e2);
                if (m_end < Llen && rw.s(m_end) <= bandhi)
                    reason = kReasonPrefix;
                const LaneRow rr[4] = {rw, rw, ro, ro};
                int           lo[4] = {0, 0, 0, 0}, hi[4] = {m_end, m_end, Llen, Llen};
                const float   tt[4] = {inlo, bandhi, inlo, bandhi};
                const bool    st[4] = {true, false, true, false};
                row_bounds4(rr, lo, hi, tt, st);
                const int mw0 = lo[0], mw1 = lo[1], mo0 = lo[2], mo1 = lo[3];
                int       nband = 0, nlo = 0;
                auto add = [&](float v, float sv, float dv, int off) {
                    if (nband < kBandCap)
                    {
                        bv[nband * 32] = v;
                        bs[nband * 32] = sv;
                        bd[nband * 32] = dv;
                        bo[nband * 32] = (uint16_t)off;
                    }
                    ++nband;
                    nlo += v < elo;
                };
                // Both ranges by aligned 4-entry groups of the row (one 16-byte
                // and one 8-byte load per group), kFinishRound groups per round
                // (the loads of a round, then its gathers).  One group per round
                // keeps the kernel at 96 registers, so a CTA holds 20 warps.
                for (int g0 = mw0 >> 2; g0 * 4 < mw1; g0 += kFinishRound) // s in the band, d <= bandhi
                {
                    float4 s4[kFinishRound];
                    uint2  j4[kFinishRound];
#pragma unroll
                    for (int h = 0; h < kFinishRound; ++h)
                        if ((g0 + h) * 4 < mw1)
                        {
                            s4[h] = rw.s4(g0 + h);
                            j4[h] = rw.j4(g0 + h);
                        }
#pragma unroll
                    for (int h = 0; h < kFinishRound; ++h)
#pragma unroll
                        for (int q = 0; q < 4; ++q)
                        {
                            const int   mm = (g0 + h) * 4 + q;
                            const bool  in = mm >= mw0 && mm < mw1;
                            const int   j  = (int)u2get16(j4[h], q);
                            const float sv = f4get(s4[h], q);
                            const float dv = dist3f(xo, X32o[in ? j : 0]);
                            if (in && dv <= bandhi)
                                add(fmaxf(sv, dv), sv, dv, mm - mw0);
                        }
                }
                const int nW = nband; // band entries from the walked row come first
                for (int g0 = mo0 >> 2; g0 * 4 < mo1; g0 += kFinishRound) // d in the band, s < inlo
                {
                    float4 d4[kFinishRound];
                    uint2  j4[kFinishRound];
#pragma unroll
                    for (int h = 0; h < kFinishRound; ++h)
                        if ((g0 + h) * 4 < mo1)
                        {
                            d4[h] = ro.s4(g0 + h);
                            j4[h] = ro.j4(g0 + h);
                        }
#pragma unroll
                    for (int h = 0; h < kFinishRound; ++h)
#pragma unroll
                        for (int q = 0; q < 4; ++q)
                        {
                            const int   mm = (g0 + h) * 4 + q;
                            const bool  in = mm >= mo0 && mm < mo1;
                            const int   j  = (int)u2get16(j4[h], q);
                            const float dv = f4get(d4[h], q);
                            const float sv = dist3f(xw, X32w[in ? j : 0]);
                            if (in && sv < inlo)
                                add(dv, sv, dv, mm - mo0);
                        }
                }
                // frame of band entry e (for the FP64 paths)
                auto band_frame = [&](int e) -> int {
                    return e < nW ? rw.j(mw0 + bo[e * 32]) : ro.j(mo0 + bo[e * 32]);
                };
                int       n_in = prefix - nlo; // #{v < inlo}
                const int r    = K - n_in;     // 1-based rank of the k-th value in the band
                if (!reason && (nband > kBandCap || r < 1 || r > nband))
                    reason = kReasonBand;

                // ---- the k-th FP32 value; certain members and the ambiguous set ---
                unsigned amb  = 0u;
                float    lower = 0.0f;
                int      need  = 0;
                if (!reason)
                {
                    float d32 = 0.0f;
                    for (int e = 0; e < nband; ++e)
                    {
                        const float v  = bv[e * 32];
                        int         rk = 0;
                        for (int f = 0; f < nband; ++f)
                        {
                            const float u = bv[f * 32];
                            rk += u < v || (u == v && f < e);
                        }
                        if (rk == r - 1)
                        {
                            d32 = v;
                            break;
                        }
                    }
                    lower             = __fsub_rd(d32, e2);
                    const float upper = __fadd_ru(d32, e2);
                    for (int e = 0; e < nband; ++e)
                    {
                        const float v = bv[e * 32];
                        if (v < lower)
                            ++n_in;
                        else if (v <= upper)
                            amb |= 1u << e;
                    }
                    need = K - n_in;
                    if (need < 1 || need > __popc(amb))
                        reason = kReasonAmbig;
                }

                // ---- marginal maxima over the members, then the counts -----------
                // Fast path: when no other member lies within 2 eps below the
                // FP32 maximum member of a marginal, that member holds the FP64
                // maximum; when no other row entry lies within 2 eps of it
                // either, its row position gives the count.  Otherwise every
                // member within 2 eps gets an FP64 look and an FP64-repaired
                // binary search counts.
                const double* xa64 = p.X64 + (size_t)a1 * 3 * T;
                const double* xb64 = p.X64 + (size_t)a2 * 3 * T;
                const double* xw64 = wx ? xa64 : xb64;
                const double* xo64 = wx ? xb64 : xa64;
                unsigned      amem = 0u; // ambiguous band entries that are members
                if (!reason)
                {
                    const int n_amb = __popc(amb);
                    if (n_amb == need)
                        amem = amb;
                    else if (n_amb > kAmbCap)
                        reason = kReasonAmbig;
                    else
                    {
                        // order the ambiguous entries by (FP64 joint distance, scan rank)
                        unsigned long long kh[kAmbCap], kl[kAmbCap];
                        int                slot[kAmbCap];
                        const double       qw0 = xw64[i], qw1 = xw64[T + i], qw2 = xw64[2 * T + i];
                        const double       qo0 = xo64[i], qo1 = xo64[T + i], qo2 = xo64[2 * T + i];
                        const int          ix = grid.qcell(xa64[i]), iy = grid.qcell(xb64[i]);
                        int                c  = 0;
                        for (unsigned am = amb; am; am &= am - 1, ++c)
                        {
                            const int    e  = __ffs(am) - 1;
                            const int    j  = band_frame(e);
                            const double dw = dist3r(xw64, T, qw0, qw1, qw2, j);
                            const double dq = dist3r(xo64, T, qo0, qo1, qo2, j);
                            slot[c]         = e;
                            kh[c]           = dbits(fmax(dw, dq));
                            kl[c]           = grid.rank(ix, iy, xa64[j], xb64[j], j, T);
                        }
                        for (int x = 0; x < n_amb; ++x)
                        {
                            int rk = 0;
                            for (int y = 0; y < n_amb; ++y)
                                rk += kh[y] < kh[x] || (kh[y] == kh[x] && kl[y] < kl[x]);
                            if (rk < need)
                                amem |= 1u << slot[x];
                        }
                    }
                }
                int ncount[2] = {0, 0}; // counts of the walked and the other marginal
                int steps     = 0;
                for (int side = 0; side < 2 && !reason; ++side)
                {
                    const LaneRow& row  = side == 0 ? rw : ro;
                    const float4*  Xc   = side == 0 ? X32o : X32w; // membership: the other marginal < inlo
                    const float4   xc   = side == 0 ? xo : xw;
                    const double*  x64  = side == 0 ? xw64 : xo64;
                    const float    eps  = side == 0 ? ew : eo;
                    const float*   bval = side == 0 ? bs : bd;
                    // band members
                    float top = -1.0f, sec = -1.0f;
                    int   ptop = -1;
                    for (int e = 0; e < nband; ++e)
                    {
                        if (!(bv[e * 32] < lower || ((amem >> e) & 1u)))
                            continue;
                        const float val  = bval[e * 32];
                        // row position of the entry in this side's row (-1: other row)
                        const int   prow = (side == 0) == (e < nW) ? (side == 0 ? mw0 : mo0) + bo[e * 32] : -1;
                        if (val > top)
                        {
                            sec  = top;
                            top  = val;
                            ptop = prow;
                        }
                        else if (val > sec)
                            sec = val;
                    }
                    // members with v < inlo: the first one below the band start
                    // in this row holds their maximum (a 4-entry group per round).
                    // Row values below the band start are < inlo, so when a band
                    // member already tops inlo by 2 eps they can neither be the
                    // maximum nor lie within 2 eps of it: no scan.
                    const bool settled = top >= 0.0f && __fsub_rd(top, __fmul_ru(2.0f, eps)) >= inlo;
                    int        mm = (side == 0 ? mw0 : mo0) - 1, first = -1;
                    float      fval = -1.0f, fsec = -1.0f;
                    while (!settled && mm >= 0 && first < 0)
                    {
                        const int    g  = mm >> 2;
                        const float4 s4 = row.s4(g);
                        const uint2  j4 = row.j4(g);
                        bool         ok[4];
#pragma unroll
                        for (int q = 0; q < 4; ++q)
                        {
                            const bool in = g * 4 + q <= mm;
                            ok[q] = in && dist3f(xc, Xc[in ? u2get16(j4, q) : 0u]) < inlo;
                        }
#pragma unroll
                        for (int q = 3; q >= 0; --q)
                            if (ok[q])
                            {
                                if (first < 0)
                                {
                                    first = g * 4 + q;
                                    fval  = f4get(s4, q);
                                }
                                else
                                    fsec = fmaxf(fsec, f4get(s4, q));
                            }
                        steps += mm - g * 4 + 1;
                        mm = g * 4 - 1; // the next unexamined position
                        if (first < 0 && steps > kScanCap)
                            reason = kReasonScan;
                    }
                    if (reason)
                        break;
                    if (first >= 0)
                    {
                        if (fval > top)
                        {
                            sec  = fmaxf(sec, top);
                            top  = fval;
                            ptop = first;
                        }
                        else
                            sec = fmaxf(sec, fval);
                        sec = fmaxf(sec, fsec);
                    }
                    const float tie = __fsub_rd(top, __fmul_ru(2.0f, eps));
                    const float chi = __fadd_ru(top, __fmul_ru(2.0f, eps));
                    // members below the examined entries that are still within 2 eps
                    for (; first >= 0 && mm >= 0; --mm)
                    {
                        const float sv = row.s(mm);
                        if (sv < tie)
                            break;
                        if (++steps > kScanCap)
                        {
                            reason = kReasonScan;
                            break;
                        }
                        if (dist3f(xc, Xc[row.j(mm)]) < inlo)
                            sec = fmaxf(sec, sv);
                    }
                    if (reason)
                        break;
                    bool fast = ptop >= 0 && sec < tie;
                    if (fast && ptop > 0 && row.s(ptop - 1) >= tie)
                        fast = false;
                    if (fast && ptop + 1 < Llen && row.s(ptop + 1) <= chi)
                        fast = false;
                    if (fast)
                    {
                        ncount[side] = ptop + 1;
                        continue;
                    }
                    // FP64 maximum over every member within 2 eps of top
                    const double q0 = x64[i], q1 = x64[T + i], q2 = x64[2 * T + i];
                    double       best = -1.0;
                    for (int e = 0; e < nband; ++e)
                        if ((bv[e * 32] < lower || ((amem >> e) & 1u)) && bval[e * 32] >= tie)
                            best = fmax(best, dist3r(x64, T, q0, q1, q2, band_frame(e)));
                    for (int pos = first; pos >= 0; --pos)
                    {
                        const float sv = row.s(pos);
                        if (sv < tie)
                            break;
                        if (++steps > kScanCap)
                        {
                            reason = kReasonScan;
                            break;
                        }
                        const int j = row.j(pos);
                        if (dist3f(xc, Xc[j]) < inlo)
                            best = fmax(best, dist3r(x64, T, q0, q1, q2, j));
                    }
                    if (reason)
                        break;
                    // count: every entry below the FP64 band, plus the band in FP64
                    const float   tlo   = __double2float_rd(__dsub_rd(best, (double)eps));
                    const float   thi   = __double2float_ru(__dadd_ru(best, (double)eps));
                    const LaneRow rr[4] = {row, row, row, row};
                    int           lo[4] = {0, 0, 0, 0}, hi[4] = {Llen, Llen, 0, 0};
                    const float   tt[4] = {tlo, thi, 0.0f, 0.0f};
                    const bool    st[4] = {true, false, true, true};
                    row_bounds4(rr, lo, hi, tt, st);
                    int n = lo[0];
                    for (int pos = lo[0]; pos < lo[1]; ++pos)
                        n += dist3r(x64, T, q0, q1, q2, row.j(pos)) <= best;
                    ncount[side] = n;
                }
                if (!reason)
                {
                    const int nx = wx ? ncount[0] : ncount[1], ny = wx ? ncount[1] : ncount[0];
                    out          = (uint32_t)nx | ((uint32_t)ny << 16);
                }
            }
            if (reason)
            {
                out = kHandOver;
                atomicOr(p.status, kStatFallback);
                if (p.reasons)
                    atomicAdd(p.reasons + reason, 1u);
                if (p.hq)
                {
                    const unsigned q = atomicAdd(p.hq_len, 1u);
                    if (q < p.hq_cap)
                        p.hq[q] = (unsigned long long)tk.pl * p.T + i;
                }
            }
            p.cnt[(size_t)tk.pl * p.T + i] = out;
        }
        __syncwarp(); // band columns of every lane are free for the next task
    }
}

// Exact FP64 statistics of one handed-over (query, pair): cnt index idx.
__device__ __forceinline__ void fixup_one(const WalkParams& p, long long idx, unsigned* hist, int lane)
{
    const long pl = (long)(idx / p.T);
    const int  i  = (int)(idx - (long long)pl * p.T);
    int        a1, a2;
    if (p.pair_ab)
    {
        a1 = p.pair_ab[pl].x;
        a2 = p.pair_ab[pl].y;
    }
    else
        pair_from_index(p.pair_begin + pl, &a1, &a2);
    const uint32_t c = exact_query(p.X64, p.T, p.K, a1, a2, i, p.box, p.rank_shift, hist, lane);
    if (lane == 0)
        p.cnt[idx] = c;
    __syncwarp();
}

// The queued hand-overs of every descriptor, one warp each, spread over the grid.
__global__ void __launch_bounds__(256) ksg_fixup_queue_kernel(WalkBatch B)
{
    __shared__ unsigned hist[8][256];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int d = 0; d < B.n; ++d)
    {
        const WalkParams& p = B.d[d];
        if (!p.hq)
            continue;
        const unsigned n = min(*p.hq_len, p.hq_cap);
        for (unsigned e = blockIdx.x * 8 + warp; e < n; e += gridDim.x * 8)
            fixup_one(p, (long long)p.hq[e], hist[warp], lane);
    }
}

// Any kHandOver mark left (a queue overflowed): scan the counts.
__global__ void __launch_bounds__(256) ksg_fixup_kernel(WalkBatch B)
{
    __shared__ unsigned hist[8][256];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int d = 0; d < B.n; ++d)
    {
        const WalkParams& p = B.d[d];
        if (p.hq && *p.hq_len <= p.hq_cap) // every hand-over was queued (and is done)
            continue;
        const long long   n = (long long)p.T * p.pair_count;
        for (long long c0 = ((long long)blockIdx.x * 8 + warp) * 32; c0 < n; c0 += (long long)gridDim.x * 8 * 32)
        {
            const long long e  = c0 + lane;
            unsigned        hm = __ballot_sync(kFull, e < n && p.cnt[e] == kHandOver);
            while (hm)
            {
                const int src = __ffs(hm) - 1;
                hm &= hm - 1;
                fixup_one(p, c0 + src, hist[warp], lane);
            }
        }
    }
}

cudaError_t launch_ksg_x32(const double* X64, int natoms, int T, float4* X32, float* eps_atom, cudaStream_t s)
{
    ksg_x32_kernel<<<(natoms * 32 + 255) / 256, 256, 0, s>>>(X64, natoms, T, X32, eps_atom);
    return cudaGetLastError();
}

cudaError_t launch_ksg_rows(const WalkBatch& b, long long rows, cudaStream_t s)
{
    if (rows <= 0)
        return cudaSuccess;
    int          threads = 256, regs = 0;
    const size_t smem    = row_sort_smem(b.maxT - 1, &threads, &regs);
    void (*kernel)(WalkBatch) = ksg_rows_kernel<256, 0>;
    if (threads == 256 && regs == 8)
        kernel = ksg_rows_kernel<256, 8>;
    else if (threads == 512 && regs == 8)
        kernel = ksg_rows_kernel<512, 8>;
    else if (threads == 512 && regs == 16)
        kernel = ksg_rows_kernel<512, 16>;
#if GC_ROWS_128
    else if (threads == 128 && regs == 16)
        kernel = ksg_rows_kernel<128, 16>;
#endif
    // static shared memory comes on top of the dynamic part: always raise
    // the limit to what this launch needs
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess)
        return e;
    kernel<<<(unsigned)rows, threads, smem, s>>>(b);
    return cudaGetLastError();
}

// Shared memory budget of one CTA (the 227 KB opt-in maximum on sm_100, less
// room for the static variables).
constexpr size_t kSmemBudget = 226 * 1024;

int walk_max_staged_warps(int maxT)
{
    const size_t rows = (size_t)2 * maxT * 16;
    if (rows >= kSmemBudget)
        return 0;
    int w = (int)((kSmemBudget - rows) / ((size_t)kWalkBuckets * 32));
    w     = w > kWalkWarps ? kWalkWarps : w;
    return w >= 8 ? w : 0;
}

int walk_max_db_warps(int maxT)
{
    const size_t rows = (size_t)48 * maxT;
    if (rows >= kSmemBudget)
        return 0;
    const int w = (int)((kSmemBudget - rows) / ((size_t)kWalkBuckets * 32));
    return w > kWalkWarps ? kWalkWarps : w;
}

void walk_shape(int maxT, int* warps, bool* staged)
{
    const int w = walk_max_staged_warps(maxT);
    *staged     = w > 0;
    *warps      = w > 0 ? w : kWalkWarps;
}

cudaError_t launch_ksg_walk(const WalkBatch& b, int warps, bool staged, int sms, cudaStream_t s, bool gather_u,
                            bool double_buffer)
{
    const bool lo = b.maxK < 256;
    if (double_buffer && !gather_u)
    {
        void (*kernel)(WalkBatch) = lo ? ksg_walk_db_kernel<true> : ksg_walk_db_kernel<false>;
        const size_t smem = (size_t)48 * b.maxT + (size_t)warps * kWalkBuckets * 32;
        cudaError_t  e    = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess)
            return e;
        kernel<<<sms, warps * 32, smem, s>>>(b);
        return cudaGetLastError();
    }
    staged        = staged && !gather_u;
    void (*kernel)(WalkBatch) =
        gather_u ? (lo ? ksg_walk_kernel<false, true, true> : ksg_walk_kernel<false, false, true>)
                 : (staged ? (lo ? ksg_walk_kernel<true, true, false> : ksg_walk_kernel<true, false, false>)
                           : (lo ? ksg_walk_kernel<false, true, false> : ksg_walk_kernel<false, false, false>));
    const size_t smem = (staged ? (size_t)2 * b.maxT * 16 : 0) + (size_t)warps * kWalkBuckets * 32;
    cudaError_t  e    = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess)
        return e;
    int per_sm = 0;
    e          = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, warps * 32, smem);
    if (e != cudaSuccess)
        return e;
    per_sm = per_sm < 1 ? 1 : per_sm;
    kernel<<<sms * per_sm, warps * 32, smem, s>>>(b);
    return cudaGetLastError();
}

cudaError_t launch_ksg_finish(const WalkBatch& b, int sms, cudaStream_t s)
{
    const size_t smem = (size_t)kFinishWarps * kBandSlotBytes * kBandCap * 32;
    cudaError_t  e    = cudaFuncSetAttribute(ksg_finish_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess)
        return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ksg_finish_kernel, kFinishWarps * 32, smem);
    if (e != cudaSuccess)
        return e;
    per_sm = per_sm < 1 ? 1 : per_sm;
    ksg_finish_kernel<<<sms * per_sm, kFinishWarps * 32, smem, s>>>(b);
    return cudaGetLastError();
}

cudaError_t launch_ksg_fixup(const WalkBatch& b, int sms, cudaStream_t s)
{
    ksg_fixup_queue_kernel<<<sms * 4, 256, 0, s>>>(b);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return e;
    ksg_fixup_kernel<<<sms * 4, 256, 0, s>>>(b);
    return cudaGetLastError();
}

} // namespace gc
