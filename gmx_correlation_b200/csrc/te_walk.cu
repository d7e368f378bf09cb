// Transfer entropy on B200: sorted-row walk with exact FP64 repair.
//
// Reference: te_matrix, lib/transfer_entropy.cpp:63-221 (the FP64 brute
// force te_exact_kernel restates it query by query).  Restructured around
// the split of te_walk.h: the 9-D distance of an ordered pair is
// max(G, Y), G the target's 6-D (future, past) embedding distance and Y the
// source's 3-D distance, and both are rows of one atom shared by every pair
// it takes part in.
//
//   te_rows_kernel    per (atom, query): the G row and the M row (3-D
//                     distances over frames j < N_valid), sorted, with frames.
//   te_walk_kernel    one ordered pair per CTA task, one query per lane: walk
//                     the row (target G or source M) whose k-th value is
//                     larger, gathering the other distance from the pair's
//                     coordinates staged in shared memory, and histogram the
//                     joint values from the lower bound until the k-th is
//                     provably passed (the KSG walk's scheme, ksg_fast.cu).
//   te_finish_kernel  band around the k-th bucket from two row ranges, the
//                     FP32 k-th value, the FP64 eps from the few values
//                     within the error bound of it; then n_xfxp and n_xp by
//                     binary search in the target's G and M rows and n_ypxp
//                     by enumerating the shorter of the target's and the
//                     source's M-row prefixes, every decision within the
//                     error bound of eps re-evaluated in FP64.
//   te_fixup_*        queries handed over (too many values near a bound, a
//                     histogram overflow) get the exact FP64 query.
//   te_reduce_kernel  the reference's te_sum in query order.
//
// Error bound: x32 = fl32(x64 - c) (te_x32_kernel) gives |d32 - d64| <=
// eps_a for every 3-D distance of atom a, so a G value is within eps_a1, a
// Y value within eps_a2 and a 9-D value within e = max of the two.  Only the
// value of eps enters the counts (strict <), so there is no tie rule.

#include "gc_common.cuh"
#include "gc_internal.h"
#include "ksg_fast.h"
#include "row_sort.cuh"
#include "te_exact_query.cuh"
#include "te_walk.h"

namespace gc {

namespace {

__device__ __forceinline__ float te3(const float4 a, const float4 b)
{
    return fmaxf(fmaxf(fabsf(a.x - b.x), fabsf(a.y - b.y)), fabsf(a.z - b.z));
}

// The descriptor owning task t: the largest d with prefix[d] <= t.
__device__ __forceinline__ int te_desc_of(const long long* __restrict__ prefix, int n, long long t)
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

// One lane's view of a transposed sorted row.
struct TeRow
{
    const float*    S;
    const uint16_t* P;
    size_t          gstride; // elements between consecutive 4-entry groups

    __device__ __forceinline__ float s(int m) const { return S[(size_t)(m >> 2) * gstride + (m & 3)]; }
    __device__ __forceinline__ int   j(int m) const { return P[(size_t)(m >> 2) * gstride + (m & 3)]; }
    __device__ __forceinline__ float4 s4(int g) const
    {
        return *reinterpret_cast<const float4*>(S + (size_t)g * gstride);
    }
    __device__ __forceinline__ uint2 j4(int g) const { return *reinterpret_cast<const uint2*>(P + (size_t)g * gstride); }
};

__device__ __forceinline__ TeRow te_row(const float* S, const uint16_t* P, const TeParams& p, int atom, int iq)
{
    const size_t base = ((size_t)atom * (p.Lpad >> 2) * p.Qp + iq) * 4;
    return TeRow{S + base, P + base, (size_t)p.Qp * 4};
}

__device__ __forceinline__ float f4at(const float4& v, int q)
{
    return q == 0 ? v.x : (q == 1 ? v.y : (q == 2 ? v.z : v.w));
}

__device__ __forceinline__ unsigned u2at16(const uint2& v, int q)
{
    return q < 2 ? ((v.x >> (16 * q)) & 0xFFFFu) : ((v.y >> (16 * (q - 2))) & 0xFFFFu);
}

// Ordered pair of walk / finish task k of descriptor p.
__device__ __forceinline__ void te_pair(const TeParams& p, long k, long& q, int& a1, int& a2)
{
    q            = p.pair_order ? (long)p.pair_order[k] : k;
    a1           = (int)(q / (p.natoms - 1));
    const int rr = (int)(q - (long)a1 * (p.natoms - 1));
    a2           = rr < a1 ? rr : rr + 1;
}

// Independent binary searches advanced together: lo[q] becomes the first
// position in [lo[q], hi[q]) of row r[q] whose value is not < t[q]
// (strict[q]) / not <= t[q].
template <int NS>
__device__ __forceinline__ void te_bounds(const TeRow (&r)[NS], int (&lo)[NS], int (&hi)[NS], const float (&t)[NS],
                                          const bool (&strict)[NS])
{
    for (;;)
    {
        int   mid[NS];
        float v[NS];
        bool  any = false;
#pragma unroll
        for (int q = 0; q < NS; ++q)
        {
            mid[q] = (lo[q] + hi[q]) >> 1;
            v[q]   = lo[q] < hi[q] ? r[q].s(mid[q]) : 0.0f;
        }
#pragma unroll
        for (int q = 0; q < NS; ++q)
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

// Hand-over causes (TeParams::reasons index).
enum
{
    kTeReasonRange  = 2, // k-th value beyond the histogram's range
    kTeReasonBand   = 3, // band larger than kTeBandCap or inconsistent with the histogram
    kTeReasonAmbig  = 4, // more than kTeAmbCap values within the error bound of the k-th
    kTeReasonPrefix = 6  // band reaches beyond the walked prefix
};
constexpr int kTeAmbCap = 8;

__device__ __forceinline__ unsigned long long te_pack_walk(int bstar, int prefix, int m_end, int reason)
{
    return (unsigned long long)(bstar & 0xFF) | ((unsigned long long)(prefix & 0xFFFF) << 8) |
           ((unsigned long long)(m_end & 0xFFFF) << 24) | ((unsigned long long)(reason & 0xFF) << 40);
}

} // namespace

// ---------------------------------------------------------------------------
// Sorted rows: blocks [0, natoms * Q) of a descriptor are G rows, the next
// natoms * Q the M rows, each over the frames j < N_valid, j != qi.
// ---------------------------------------------------------------------------
template <int THREADS, int R>
__global__ void __launch_bounds__(THREADS) te_rows_kernel(TeBatch B)
{
    const long long r   = blockIdx.x;
    const int       dsc = te_desc_of(B.rprefix, B.n, r);
    const TeParams& p   = B.d[dsc];
    const int       row = (int)(r - B.rprefix[dsc]);
    const int       per = p.natoms * p.Q;
    const bool      g   = row < per;
    const int       rem = g ? row : row - per;
    const int       a   = rem / p.Q;
    const int       iq  = rem - a * p.Q;
    const int       qi  = p.i0 + iq;
    const int       lag = p.lag;
    const float4*   xr  = p.X32 + (size_t)a * p.T;
    const float4    qp  = xr[qi];
    const size_t    base = ((size_t)a * (p.Lpad >> 2) * p.Qp + iq) * 4, gs = (size_t)p.Qp * 4;
    __shared__ RowSortShared<THREADS> sh;
    if (g)
    {
        const float4 qf = xr[qi + lag];
        sort_row<THREADS, R>(
            sh, p.Nv - 1, qi, [&](int j) { return fmaxf(te3(qf, xr[j + lag]), te3(qp, xr[j])); }, p.SG, p.PG, base,
            gs);
    }
    else
        sort_row<THREADS, R>(sh, p.Nv - 1, qi, [&](int j) { return te3(qp, xr[j]); }, p.SM, p.PM, base, gs);
}

// ---------------------------------------------------------------------------
// Walk
// ---------------------------------------------------------------------------
namespace {

struct TeTask
{
    int  c;  // chunk of query groups
    long pl; // ordered pair (local index)
    int  a1, a2;
};

__device__ __forceinline__ bool te_next_task(const TeBatch& B, long long total, long long* s_task, int* s_desc,
                                             int* s_next, TeTask& tk, int& d)
{
    if (threadIdx.x == 0)
    {
        const long long t = (long long)atomicAdd(B.counter, 1ull);
        *s_task           = t;
        *s_next           = 0;
        if (t < total)
            *s_desc = te_desc_of(B.wprefix, B.n, t);
    }
    __syncthreads();
    const long long t = *s_task;
    if (t >= total)
        return false;
    d                 = *s_desc;
    const TeParams& p = B.d[d];
    const long long lt = t - B.wprefix[d];
    tk.c               = (int)(lt / p.pair_count);
    te_pair(p, (long)(lt - (long long)tk.c * p.pair_count), tk.pl, tk.a1, tk.a2);
    return true;
}

} // namespace

// Pass 1 (see ksg_walk_kernel for the histogram scheme): per lane, walk the
// row whose k-th value L is larger (the target's G row, gathering the
// source's Y, or the source's M row, gathering the target's G from two
// staged frames) and histogram the joint value max(s, other).  STAGED: the
// pair's two coordinate rows in shared memory.  LO (every k < 256): values
// below L counted in histogram index 0.
// An atom's FP32 coordinate row as float4 (global or shared memory) ...
struct TeRows4
{
    const float4* x;
    __device__ __forceinline__ float4 at(int j) const { return x[j]; }
    __device__ __forceinline__ float  d3(const float4& q, int j) const { return te3(q, x[j]); }
};

// ... or as x,y float2 and z float in shared memory (12 bytes a frame).
struct TeRows12
{
    const float2* xy;
    const float*  z;
    __device__ __forceinline__ float4 at(int j) const
    {
        const float2 v = xy[j];
        return make_float4(v.x, v.y, z[j], 0.0f);
    }
    __device__ __forceinline__ float d3(const float4& q, int j) const
    {
        const float2 v = xy[j];
        return fmaxf(fmaxf(fabsf(q.x - v.x), fabsf(q.y - v.y)), fabsf(q.z - z[j]));
    }
};

// Walk of query group g of a staged pair task (x1, x2: the pair's FP32
// rows; base: this warp's histogram): the body of both walk kernels.
template <bool LO, class V>
__device__ __forceinline__ void te_walk_group(const TeParams& p, const TeTask& tk, int g, const V& x1, const V& x2,
                                              unsigned char* base, int lane)
{
    uint8_t*           hist = base + lane * 4;
    auto               H    = [hist](unsigned b) -> uint8_t& { return hist[(b >> 2) * 128 + (b & 3)]; };
    constexpr unsigned kTop = kWalkBuckets - 1;
    const float        inf  = __int_as_float(0x7f800000);
    const int          K = p.K, lag = p.lag, Llen = p.Nv - 1, shift = p.shift;
    const float        ebig = fmaxf(p.eps_atom[tk.a1], p.eps_atom[tk.a2]);
    const float        e2   = __fmul_ru(2.0f, ebig);
    const int   iq   = g * 32 + lane;
    const bool  live = iq < p.Q;
    const int   iql  = live ? iq : 0;
    const int   qi   = p.i0 + iql;
    const TeRow G1   = te_row(p.SG, p.PG, p, tk.a1, iql);
    const TeRow M2   = te_row(p.SM, p.PM, p, tk.a2, iql);
    const float gk = G1.s(K - 1), yk = M2.s(K - 1);
    const bool  wg = gk >= yk; // walk the target's G row (gather the source's Y)
    const TeRow rw = wg ? G1 : M2;
    const float L  = wg ? gk : yk;
    const unsigned Lb = __float_as_uint(L);
    // other distance of frame j: Y = |y(qi) - y(j)| or G = max over the
    // target's past (qi, j) and future (qi + lag, j + lag)
    const V&      oa = wg ? x2 : x1;
    const float4  oq = oa.at(qi);
    const float4  fq = x1.at(qi + lag);
    {
        uint4* h4 = reinterpret_cast<uint4*>(base);
        for (int e = lane; e < kWalkBuckets * 32 / 16; e += 32)
            h4[e] = make_uint4(0u, 0u, 0u, 0u);
    }
    __syncwarp();
    const unsigned Lh   = LO ? Lb - (1u << shift) : Lb;
    auto           hidx = [Lh, shift](float v) -> unsigned {
        if (LO)
            return (unsigned)min(max((int)(__float_as_uint(v) - Lh) >> shift, 0), (int)kTop);
        return min((__float_as_uint(v) - Lh) >> shift, kTop);
    };
    const float4* Sg = reinterpret_cast<const float4*>(rw.S);
    const uint2*  Pg = reinterpret_cast<const uint2*>(rw.P);
    const size_t  gs = (size_t)p.Qp;
    int           m_end = 0, cnt_lo = 0, Rs = 0, thr = 0, grp = 0;
    unsigned      wrap = 0u;
    float         stop = inf;
    bool          walking = live;
    float4        s4      = make_float4(inf, inf, inf, inf);
    uint2         j4      = make_uint2(0u, 0u);
    if (live)
    {
        s4 = Sg[0];
        j4 = Pg[0];
    }
    const int last = (Llen - 1) >> 2;
    while (walking)
    {
        if (grp > last)
        {
            m_end = Llen;
            break;
        }
        const int      nxt   = grp < last ? grp + 1 : grp;
        const float4   ns4   = Sg[(size_t)nxt * gs];
        const uint2    nj4   = Pg[(size_t)nxt * gs];
        const float    sv[4] = {s4.x, s4.y, s4.z, s4.w};
        const unsigned jv[4] = {j4.x & 0xFFFFu, j4.x >> 16, j4.y & 0xFFFFu, j4.y >> 16};
        bool           tkn[4];
#pragma unroll
        for (int q = 0; q < 4; ++q)
        {
            tkn[q] = sv[q] <= stop;
            float o = oa.d3(oq, (int)jv[q]);
            if (!wg)
                o = fmaxf(o, x1.d3(fq, (int)jv[q] + lag));
            const float v   = fmaxf(sv[q], o);
            bool        inc = tkn[q];
            if (!LO)
            {
                const bool below = v < L;
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
            H(kTop) = 0;
            if (stop == inf)
            {
                const float sl = sv[3];
                const int   bn = (LO || sl >= L) ? (int)hidx(sl) : 0;
                for (int b = thr; b < bn; ++b)
                    Rs += H(b);
                thr = max(thr, bn);
                if (cnt_lo + Rs >= K)
                    stop = __fadd_ru(__uint_as_float(Lh + ((unsigned)bn << shift)), e2);
            }
        }
        s4 = ns4;
        j4 = nj4;
    }
    if (live)
    {
        int bstar, prefix;
        if (stop != inf)
        {
            int cum = cnt_lo + Rs, b = thr - 1;
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
        const int reason = (wrap > 255u || (LO && bstar == 0)) ? kTeReasonBand
                           : (bstar >= (int)kTop ? kTeReasonRange : 0);
        p.wres[(size_t)tk.pl * p.Q + iq] = te_pack_walk(LO ? bstar - 1 : bstar, prefix, m_end, reason);
    }
    if (p.walk_elems)
    {
        const unsigned we = __reduce_add_sync(kFull, live ? (unsigned)m_end : 0u);
        if (lane == 0 && we)
            atomicAdd(p.walk_elems, (unsigned long long)we);
    }
    __syncwarp();
}

template <bool STAGED, bool LO>
__global__ void __launch_bounds__(1024, 1) te_walk_kernel(TeBatch B)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ long long s_task;
    __shared__ int       s_desc, s_next;
    const int            warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float4*              sx   = reinterpret_cast<float4*>(smem_raw);
    unsigned char*       base = smem_raw + (STAGED ? (size_t)2 * B.maxT * 16 : 0) + (size_t)warp * kWalkBuckets * 32;

    const long long total = B.wprefix[B.n];
    TeTask          tk;
    int             dsc;
    while (te_next_task(B, total, &s_task, &s_desc, &s_next, tk, dsc))
    {
        const TeParams& p       = B.d[dsc];
        const int       T       = p.T;
        const int       ngroups = (p.Q + 31) >> 5;
        const float4*   x1      = p.X32 + (size_t)tk.a1 * T;
        const float4*   x2      = p.X32 + (size_t)tk.a2 * T;
        if (STAGED)
        {
            for (int e = threadIdx.x; e < T; e += blockDim.x)
            {
                sx[e]     = x1[e];
                sx[T + e] = x2[e];
            }
            __syncthreads();
            x1 = sx;
            x2 = sx + T;
        }
        for (;;)
        {
            int gi = 0;
            if (lane == 0)
                gi = atomicAdd(&s_next, 1);
            gi          = __shfl_sync(kFull, gi, 0);
            const int g = tk.c * B.chunk + gi;
            if (gi >= B.chunk || g >= ngroups)
                break;
            te_walk_group<LO>(p, tk, g, TeRows4{x1}, TeRows4{x2}, base, lane);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Finish
// ---------------------------------------------------------------------------
namespace {

// FP64 distances of one query on the raw coordinates (the reference's
// arithmetic: |q - x| per component, max over components).
struct TeQuery64
{
    const double* a; // target rows [3][T]
    const double* b; // source rows [3][T]
    int           T, lag, qi;
    double        f0, f1, f2, p0, p1, p2, y0, y1, y2;

    __device__ __forceinline__ TeQuery64(const double* XT, int T_, int lag_, int a1, int a2, int qi_)
        : a(XT + (size_t)a1 * 3 * T_), b(XT + (size_t)a2 * 3 * T_), T(T_), lag(lag_), qi(qi_)
    {
        f0 = a[qi + lag];
        f1 = a[T + qi + lag];
        f2 = a[2 * T + qi + lag];
        p0 = a[qi];
        p1 = a[T + qi];
        p2 = a[2 * T + qi];
        y0 = b[qi];
        y1 = b[T + qi];
        y2 = b[2 * T + qi];
    }
    __device__ __forceinline__ double past(int j) const
    {
        return fmax(fmax(fabs(p0 - a[j]), fabs(p1 - a[T + j])), fabs(p2 - a[2 * T + j]));
    }
    __device__ __forceinline__ double fut(int j) const
    {
        const int jj = j + lag;
        return fmax(fmax(fabs(f0 - a[jj]), fabs(f1 - a[T + jj])), fabs(f2 - a[2 * T + jj]));
    }
    __device__ __forceinline__ double src(int j) const
    {
        return fmax(fmax(fabs(y0 - b[j]), fabs(y1 - b[T + j])), fabs(y2 - b[2 * T + j]));
    }
};

} // namespace

__global__ void __launch_bounds__(kTeFinishWarps * 32, 1) te_finish_kernel(TeBatch B)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int      warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char* base = smem_raw + (size_t)warp * 6 * kTeBandCap * 32;
    // per-lane columns: band entry e of lane l at [e * 32 + l]: joint FP32
    // value and frame
    float*    bv = reinterpret_cast<float*>(base) + lane;
    uint16_t* bj = reinterpret_cast<uint16_t*>(base + 4 * kTeBandCap * 32) + lane;

    const long long total = B.fprefix[B.n];
    for (;;)
    {
        long long t   = 0;
        int       dsc = 0;
        if (lane == 0)
        {
            t = (long long)atomicAdd(B.counter + 1, 1ull);
            if (t < total)
                dsc = te_desc_of(B.fprefix, B.n, t);
        }
        t   = __shfl_sync(kFull, t, 0);
        dsc = __shfl_sync(kFull, dsc, 0);
        if (t >= total)
            break;
        const TeParams& p  = B.d[dsc];
        const int       T = p.T, K = p.K, lag = p.lag, Nv = p.Nv, Llen = Nv - 1, shift = p.shift;
        const long long lt = t - B.fprefix[dsc];
        const int       g  = (int)(lt / p.pair_count);
        long            pl;
        int             a1, a2;
        te_pair(p, (long)(lt - (long long)g * p.pair_count), pl, a1, a2);
        const int  iq   = g * 32 + lane;
        const bool live = iq < p.Q;
        if (live)
        {
            const int                qi = p.i0 + iq;
            const unsigned long long wr = p.wres[(size_t)pl * p.Q + iq];
            const int                bstar = (int)(wr & 0xFF), prefix = (int)((wr >> 8) & 0xFFFF);
            const int                m_end = (int)((wr >> 24) & 0xFFFF);
            int                      reason = (int)((wr >> 40) & 0xFF);
            if (m_end > Llen) // not a walk result: never read past the row
                reason = kTeReasonBand;
            uint2                    out    = make_uint2(kTeHandOver, kTeHandOver);
            const TeRow   G1 = te_row(p.SG, p.PG, p, a1, iq);
            const TeRow   M1 = te_row(p.SM, p.PM, p, a1, iq);
            const TeRow   M2 = te_row(p.SM, p.PM, p, a2, iq);
            const float   gk = G1.s(K - 1), yk = M2.s(K - 1);
            const bool    wg = gk >= yk;
            const TeRow&  rw = wg ? G1 : M2;
            const TeRow&  ro = wg ? M2 : G1;
            const unsigned Lb = __float_as_uint(wg ? gk : yk);
            const float4* x1 = p.X32 + (size_t)a1 * T;
            const float4* x2 = p.X32 + (size_t)a2 * T;
            const float4  qp = x1[qi], qf = x1[qi + lag], qy = x2[qi];
            auto gval = [&](int j) { return fmaxf(te3(qf, x1[j + lag]), te3(qp, x1[j])); };
            auto yval = [&](int j) { return te3(qy, x2[j]); };
            const float e1 = p.eps_atom[a1], e2a = p.eps_atom[a2];
            const float e2 = __fmul_ru(2.0f, fmaxf(e1, e2a));
            if (reason == 0)
            {
                // ---- band: every joint value in [inlo, bandhi], from two row ranges
                const float elo    = __uint_as_float(Lb + ((unsigned)bstar << shift));
                const float ehi    = __uint_as_float(Lb + ((unsigned)(bstar + 1) << shift));
                const float inlo   = __fsub_rd(elo, e2);
                const float bandhi = __fadd_ru(ehi, e2);
                if (m_end < Llen && rw.s(m_end) <= bandhi)
                    reason = kTeReasonPrefix;
                const TeRow rr[4] = {rw, rw, ro, ro};
                int         lo[4] = {0, 0, 0, 0}, hi[4] = {m_end, m_end, Llen, Llen};
                const float tt[4] = {inlo, bandhi, inlo, bandhi};
                const bool  st[4] = {true, false, true, false};
                te_bounds<4>(rr, lo, hi, tt, st);
                const int mw0 = lo[0], mw1 = lo[1], mo0 = lo[2], mo1 = lo[3];
                int       nband = 0, nlo = 0;
                auto add = [&](float v, int j) {
                    if (nband < kTeBandCap)
                    {
                        bv[nband * 32] = v;
                        bj[nband * 32] = (uint16_t)j;
                    }
                    ++nband;
                    nlo += v < elo;
                };
                for (int g0 = mw0 >> 2; g0 * 4 < mw1; ++g0) // walked value in the band, other <= bandhi
                {
                    const float4 s4 = rw.s4(g0);
                    const uint2  j4 = rw.j4(g0);
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                    {
                        const int mm = g0 * 4 + q;
                        if (mm >= mw0 && mm < mw1)
                        {
                            const int   j  = (int)u2at16(j4, q);
                            const float sv = f4at(s4, q);
                            const float ov = wg ? yval(j) : gval(j);
                            if (ov <= bandhi)
                                add(fmaxf(sv, ov), j);
                        }
                    }
                }
                for (int g0 = mo0 >> 2; g0 * 4 < mo1; ++g0) // other value in the band, walked < inlo
                {
                    const float4 d4 = ro.s4(g0);
                    const uint2  j4 = ro.j4(g0);
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                    {
                        const int mm = g0 * 4 + q;
                        if (mm >= mo0 && mm < mo1)
                        {
                            const int   j  = (int)u2at16(j4, q);
                            const float dv = f4at(d4, q);
                            const float wv = wg ? gval(j) : yval(j);
                            if (wv < inlo)
                                add(dv, j);
                        }
                    }
                }
                int       n_in = prefix - nlo; // #{v < inlo}
                const int r    = K - n_in;     // rank of the k-th value in the band
                if (!reason && (nband > kTeBandCap || r < 1 || r > nband))
                    reason = kTeReasonBand;

                // ---- the FP32 k-th value, then eps in FP64 from the values near it
                double eps = 0.0;
                const TeQuery64 q64(p.XT, T, lag, a1, a2, qi);
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
                    const float lower = __fsub_rd(d32, e2), upper = __fadd_ru(d32, e2);
                    unsigned    amb   = 0u;
                    for (int e = 0; e < nband; ++e)
                    {
                        const float v = bv[e * 32];
                        if (v < lower)
                            ++n_in;
                        else if (v <= upper)
                            amb |= 1u << e;
                    }
                    const int need = K - n_in, n_amb = __popc(amb);
                    if (need < 1 || need > n_amb || n_amb > kTeAmbCap)
                        reason = kTeReasonAmbig;
                    else
                    {
                        double val[kTeAmbCap];
                        int    c = 0;
                        for (unsigned am = amb; am; am &= am - 1, ++c)
                        {
                            const int j = bj[(__ffs(am) - 1) * 32];
                            val[c]      = fmax(fmax(q64.fut(j), q64.past(j)), q64.src(j));
                        }
                        for (int x = 0; x < n_amb; ++x)
                        {
                            int rk = 0;
                            for (int y = 0; y < n_amb; ++y)
                                rk += val[y] < val[x] || (val[y] == val[x] && y < x);
                            if (rk == need - 1)
                                eps = val[x];
                        }
                    }
                }

                // ---- counts, strict < eps ------------------------------------------
                if (!reason)
                {
                    const float tlo1 = __double2float_rd(__dsub_rd(eps, (double)e1));
                    const float thi1 = __double2float_ru(__dadd_ru(eps, (double)e1));
                    const float tlo2 = __double2float_rd(__dsub_rd(eps, (double)e2a));
                    const float thi2 = __double2float_ru(__dadd_ru(eps, (double)e2a));
                    const TeRow cr[5] = {G1, G1, M1, M1, M2};
                    int         clo[5] = {0, 0, 0, 0, 0}, chi[5] = {Llen, Llen, Llen, Llen, Llen};
                    const float ct[5] = {tlo1, thi1, tlo1, thi1, thi2};
                    const bool  cs[5] = {true, false, true, false, false};
                    te_bounds<5>(cr, clo, chi, ct, cs);
                    // n_xfxp: G row of the target; n_xp: its M row
                    int n_xfxp = clo[0];
                    for (int pos = clo[0]; pos < clo[1]; ++pos)
                    {
                        const int j = G1.j(pos);
                        n_xfxp += fmax(q64.fut(j), q64.past(j)) < eps;
                    }
                    int n_xp = clo[2];
                    for (int pos = clo[2]; pos < clo[3]; ++pos)
                        n_xp += q64.past(M1.j(pos)) < eps;
                    // n_ypxp is counted by te_count_kernel over the shorter of
                    // the two M-row prefixes that can hold a value below eps:
                    // it gets eps (in wres) and the prefix (in cnt.y).
                    const int  end1 = clo[3], end2 = clo[4];
                    const bool on1  = end1 <= end2;
                    const int  ne   = on1 ? end1 : end2;
                    p.wres[(size_t)pl * p.Q + iq] = (unsigned long long)__double_as_longlong(eps);
                    out = make_uint2((unsigned)n_xp | ((unsigned)n_xfxp << 16),
                                     (unsigned)ne | (on1 ? kTeCountOn1 : 0u));
                }
            }
            if (reason)
            {
                out = make_uint2(kTeHandOver, kTeHandOver);
                atomicOr(p.status, kStatFallback);
                if (p.reasons)
                    atomicAdd(p.reasons + reason, 1u);
                if (p.hq)
                {
                    const unsigned hqi = atomicAdd(p.hq_len, 1u);
                    if (hqi < p.hq_cap)
                        p.hq[hqi] = (unsigned long long)pl * Nv + qi;
                }
            }
            p.cnt[(size_t)pl * Nv + qi] = out;
        }
        __syncwarp();
    }
}

// n_ypxp of query iq of a staged pair task (x1, x2: the pair's FP32 rows,
// in shared or global memory): the body of both count kernels.
__device__ __forceinline__ void te_count_query(const TeParams& p, const TeTask& tk, int iq, const float4* x1,
                                               const float4* x2, float e1, float e2a)
{
    const int T = p.T, Nv = p.Nv;
    const int    qi = p.i0 + iq;
    uint2* const cp = p.cnt + (size_t)tk.pl * Nv + qi;
    const uint2  c  = *cp;
    if (c.x != kTeHandOver)
    {
        const double eps = __longlong_as_double((long long)p.wres[(size_t)tk.pl * p.Q + iq]);
        const int    ne  = (int)(c.y & 0xFFFFu);
        const bool   on1 = (c.y & kTeCountOn1) != 0u;
        const double es = on1 ? (double)e1 : (double)e2a, eo = on1 ? (double)e2a : (double)e1;
        const float  tlo_s = __double2float_rd(__dsub_rd(eps, es));
        const float  tlo_o = __double2float_rd(__dsub_rd(eps, eo));
        const float  thi_o = __double2float_ru(__dadd_ru(eps, eo));
        const TeRow  er = te_row(p.SM, p.PM, p, on1 ? tk.a1 : tk.a2, iq);
        const float4* ox = on1 ? x2 : x1;
        const float4  oq = ox[qi];
        const float4* Sg = reinterpret_cast<const float4*>(er.S);
        const uint2*  Pg = reinterpret_cast<const uint2*>(er.P);
        const size_t  gs = (size_t)p.Qp;
        const int     ng = (ne + 3) >> 2;
        int           n  = 0;
        float4        s4 = make_float4(0.f, 0.f, 0.f, 0.f);
        uint2         j4 = make_uint2(0u, 0u);
        if (ng > 0)
        {
            s4 = Sg[0];
            j4 = Pg[0];
        }
        for (int g0 = 0; g0 < ng; ++g0)
        {
            // the next group is loaded while this one is counted
            const int    nx  = g0 + 1 < ng ? g0 + 1 : g0;
            const float4 ns4 = Sg[(size_t)nx * gs];
            const uint2  nj4 = Pg[(size_t)nx * gs];
            const float  sv[4] = {s4.x, s4.y, s4.z, s4.w};
            const unsigned jv[4] = {j4.x & 0xFFFFu, j4.x >> 16, j4.y & 0xFFFFu, j4.y >> 16};
            unsigned     amb = 0u;
#pragma unroll
            for (int q = 0; q < 4; ++q)
            {
                const bool  in = g0 * 4 + q < ne;
                const float ov = te3(oq, ox[jv[q]]);
                if (in && sv[q] < tlo_s && ov < tlo_o)
                    ++n;
                else if (in && ov <= thi_o)
                    amb |= 1u << q;
            }
            for (; amb; amb &= amb - 1) // rare: FP64 on the raw coordinates
            {
                const int     j  = (int)u2at16(j4, __ffs(amb) - 1);
                const double* ra = p.XT + (size_t)tk.a1 * 3 * T;
                const double* rb = p.XT + (size_t)tk.a2 * 3 * T;
                double        d  = 0.0;
#pragma unroll 1
                for (int c3 = 0; c3 < 3; ++c3)
                    d = fmax(d, fmax(fabs(ra[c3 * T + qi] - ra[c3 * T + j]),
                                     fabs(rb[c3 * T + qi] - rb[c3 * T + j])));
                n += d < eps;
            }
            s4 = ns4;
            j4 = nj4;
        }
        cp->y = (unsigned)n;
    }
}

// ---------------------------------------------------------------------------
// n_ypxp = #{j : max(D1(qi, j), Y(qi, j)) < eps}: one ordered pair per CTA
// task with its two coordinate rows staged in shared memory (the walk's
// task scheme), one query per lane.  Each lane enumerates the prefix the
// finish kernel chose (the target's or the source's M row, every entry whose
// FP32 value may lie below eps), gathers the other marginal from shared
// memory, and re-evaluates in FP64 every entry within the error bound of
// eps.
// ---------------------------------------------------------------------------
template <bool STAGED>
__global__ void __launch_bounds__(1024, 1) te_count_kernel(TeBatch B)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ long long s_task;
    __shared__ int       s_desc, s_next;
    const int            lane = threadIdx.x & 31;
    float4*              sx   = reinterpret_cast<float4*>(smem_raw);
    const long long      total = B.wprefix[B.n];
    TeTask               tk;
    int                  dsc;
    while (te_next_task(B, total, &s_task, &s_desc, &s_next, tk, dsc))
    {
        const TeParams& p       = B.d[dsc];
        const int       T = p.T, Nv = p.Nv;
        const int       ngroups = (p.Q + 31) >> 5;
        const float4*   x1      = p.X32 + (size_t)tk.a1 * T;
        const float4*   x2      = p.X32 + (size_t)tk.a2 * T;
        if (STAGED)
        {
            for (int e = threadIdx.x; e < T; e += blockDim.x)
            {
                sx[e]     = x1[e];
                sx[T + e] = x2[e];
            }
            __syncthreads();
            x1 = sx;
            x2 = sx + T;
        }
        const float e1 = p.eps_atom[tk.a1], e2a = p.eps_atom[tk.a2];
        for (;;)
        {
            int gi = 0;
            if (lane == 0)
                gi = atomicAdd(&s_next, 1);
            gi          = __shfl_sync(kFull, gi, 0);
            const int g = tk.c * B.chunk + gi;
            if (gi >= B.chunk || g >= ngroups)
                break;
            const int iq = g * 32 + lane;
            if (iq < p.Q)
                te_count_query(p, tk, iq, x1, x2, e1, e2a);
        }
        __syncthreads(); // every warp is done with the staged rows
    }
}

// A staged pair task of the double-buffered count kernel.
struct TeSlot
{
    long long    t;    // global task, or -1: no more tasks
    int          desc; // descriptor of the task
    int          next; // query groups handed out
    int          left; // warps done with the task
    volatile int gen;  // CTA-local index of the task this slot holds
    TeTask       tk;
};

// Fills slot S with the next global task as CTA-local task `gen`: one warp
// (lane 0 takes the task, all lanes copy the pair's two FP32 rows through
// put(T, frame e, a1's value, a2's value)).
template <class Put>
__device__ __forceinline__ void te_slot_fill_with(const TeBatch& B, long long total, TeSlot& S, int gen, int lane,
                                                  Put put)
{
    long long t = 0;
    int       d = 0;
    if (lane == 0)
    {
        t = (long long)atomicAdd(B.counter, 1ull);
        if (t < total)
            d = te_desc_of(B.wprefix, B.n, t);
        else
            t = -1;
    }
    t = __shfl_sync(kFull, t, 0);
    d = __shfl_sync(kFull, d, 0);
    TeTask tk{};
    if (t >= 0)
    {
        const TeParams& p  = B.d[d];
        const long long lt = t - B.wprefix[d];
        tk.c               = (int)(lt / p.pair_count);
        te_pair(p, (long)(lt - (long long)tk.c * p.pair_count), tk.pl, tk.a1, tk.a2);
        const int     T  = p.T;
        const float4* x1 = p.X32 + (size_t)tk.a1 * T;
        const float4* x2 = p.X32 + (size_t)tk.a2 * T;
        for (int e = lane; e < T; e += 32)
            put(T, e, x1[e], x2[e]);
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

__device__ __forceinline__ void te_slot_fill(const TeBatch& B, long long total, TeSlot& S, float4* rows, int gen,
                                             int lane)
{
    te_slot_fill_with(B, total, S, gen, lane, [rows](int T, int e, const float4& a, const float4& b) {
        rows[e]     = a;
        rows[T + e] = b;
    });
}

__device__ __forceinline__ void te_slot_fill12(const TeBatch& B, long long total, TeSlot& S, float2* xy, float* z,
                                               int gen, int lane)
{
    te_slot_fill_with(B, total, S, gen, lane, [xy, z](int T, int e, const float4& a, const float4& b) {
        xy[e]     = make_float2(a.x, a.y);
        z[e]      = a.z;
        xy[T + e] = make_float2(b.x, b.y);
        z[T + e]  = b.z;
    });
}

// The count kernel with two staged pair tasks per CTA (2 x 2 x maxT float4):
// a warp done with its query groups of task i moves on to task i + 1 without
// waiting for the CTA; the last warp to leave task i refills its buffer with
// task i + 2.  Tasks reach a CTA in its local index order (one warp fills
// both buffers first), so a warp stops at the first slot without a task.
__global__ void __launch_bounds__(1024, 1) te_count_db_kernel(TeBatch B)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ TeSlot slot[2];
    const int         warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    const long long   total = B.wprefix[B.n];
    auto              rows  = [&](int b) { return reinterpret_cast<float4*>(smem_raw) + (size_t)b * 2 * B.maxT; };
    if (warp == 0)
    {
        te_slot_fill(B, total, slot[0], rows(0), 0, lane);
        te_slot_fill(B, total, slot[1], rows(1), 1, lane);
    }
    __syncthreads();
    for (int i = 0;; ++i)
    {
        const int b = i & 1;
        TeSlot&   S = slot[b];
        // bounded wait for the refilling warp (resident, never waiting itself)
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
        const TeParams& p       = B.d[S.desc];
        const TeTask    tk      = S.tk;
        const int       ngroups = (p.Q + 31) >> 5;
        const float4*   x1      = rows(b);
        const float4*   x2      = x1 + p.T;
        const float     e1 = p.eps_atom[tk.a1], e2a = p.eps_atom[tk.a2];
        for (;;)
        {
            int gi = 0;
            if (lane == 0)
                gi = atomicAdd(&S.next, 1);
            gi          = __shfl_sync(kFull, gi, 0);
            const int g = tk.c * B.chunk + gi;
            if (gi >= B.chunk || g >= ngroups)
                break;
            const int iq = g * 32 + lane;
            if (iq < p.Q)
                te_count_query(p, tk, iq, x1, x2, e1, e2a);
        }
        int last = 0;
        if (lane == 0)
            last = atomicAdd(&S.left, 1) == nwarps - 1;
        last = __shfl_sync(kFull, last, 0);
        if (last) // every warp has left task i: its buffer takes task i + 2
            te_slot_fill(B, total, S, rows(b), i + 2, lane);
    }
}

// The walk with two staged pair tasks per CTA (the count kernel's scheme):
// per buffer the pair's rows as x,y float2 [2 maxT] and z float [2 maxT]
// (24 maxT bytes), then each warp's histogram.
template <bool LO>
__global__ void __launch_bounds__(1024, 1) te_walk_db_kernel(TeBatch B)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ TeSlot slot[2];
    const int         warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    const long long   total = B.wprefix[B.n];
    const int         maxT  = B.maxT;
    auto              xyb   = [&](int b) { return reinterpret_cast<float2*>(smem_raw + (size_t)b * 24 * maxT); };
    auto zb = [&](int b) { return reinterpret_cast<float*>(smem_raw + (size_t)b * 24 * maxT + (size_t)16 * maxT); };
    unsigned char* base = smem_raw + (size_t)48 * maxT + (size_t)warp * kWalkBuckets * 32;
    if (warp == 0)
    {
        te_slot_fill12(B, total, slot[0], xyb(0), zb(0), 0, lane);
        te_slot_fill12(B, total, slot[1], xyb(1), zb(1), 1, lane);
    }
    __syncthreads();
    for (int i = 0;; ++i)
    {
        const int b = i & 1;
        TeSlot&   S = slot[b];
        int       spins = 0;
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
        const TeParams& p       = B.d[S.desc];
        const TeTask    tk      = S.tk;
        const int       ngroups = (p.Q + 31) >> 5;
        const TeRows12  r1{xyb(b), zb(b)}, r2{xyb(b) + p.T, zb(b) + p.T};
        for (;;)
        {
            int gi = 0;
            if (lane == 0)
                gi = atomicAdd(&S.next, 1);
            gi          = __shfl_sync(kFull, gi, 0);
            const int g = tk.c * B.chunk + gi;
            if (gi >= B.chunk || g >= ngroups)
                break;
            te_walk_group<LO>(p, tk, g, r1, r2, base, lane);
        }
        int last = 0;
        if (lane == 0)
            last = atomicAdd(&S.left, 1) == nwarps - 1;
        last = __shfl_sync(kFull, last, 0);
        if (last)
            te_slot_fill12(B, total, S, xyb(b), zb(b), i + 2, lane);
    }
}

// ---------------------------------------------------------------------------
// Hand-overs, reduction
// ---------------------------------------------------------------------------
__device__ __forceinline__ void te_fixup_one(const TeParams& p, long long idx, unsigned* hist, int lane)
{
    const long pl = (long)(idx / p.Nv);
    const int  qi = (int)(idx - (long long)pl * p.Nv);
    const int  a1 = (int)(pl / (p.natoms - 1));
    const int  rr = (int)(pl - (long)a1 * (p.natoms - 1));
    const int  a2 = rr < a1 ? rr : rr + 1;
    const uint2 c = te_exact_query(p.XT, p.T, p.K, p.lag, a1, a2, qi, hist, lane);
    if (lane == 0)
        p.cnt[idx] = c;
    __syncwarp();
}

__global__ void __launch_bounds__(256) te_fixup_queue_kernel(TeBatch B)
{
    __shared__ unsigned hist[8][256];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int d = 0; d < B.n; ++d)
    {
        const TeParams& p = B.d[d];
        if (!p.hq)
            continue;
        const unsigned n = min(*p.hq_len, p.hq_cap);
        for (unsigned e = blockIdx.x * 8 + warp; e < n; e += gridDim.x * 8)
            te_fixup_one(p, (long long)p.hq[e], hist[warp], lane);
    }
}

__global__ void __launch_bounds__(256) te_fixup_scan_kernel(TeBatch B)
{
    __shared__ unsigned hist[8][256];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int d = 0; d < B.n; ++d)
    {
        const TeParams& p = B.d[d];
        if (p.hq && *p.hq_len <= p.hq_cap)
            continue;
        const long long n = (long long)p.Nv * p.pair_count;
        for (long long c0 = ((long long)blockIdx.x * 8 + warp) * 32; c0 < n; c0 += (long long)gridDim.x * 8 * 32)
        {
            const long long e  = c0 + lane;
            unsigned        hm = __ballot_sync(kFull, e < n && p.cnt[e].x == kTeHandOver);
            while (hm)
            {
                const int src = __ffs(hm) - 1;
                hm &= hm - 1;
                te_fixup_one(p, c0 + src, hist[warp], lane);
            }
        }
    }
}

// te_sum += psi_k + psi[n_xp + 1] - psi[n_xfxp + 1] - psi[n_ypxp + 1] with
// the counts clamped to N_valid, in query order; te_sum / N_valid
// (lib/transfer_entropy.cpp:188-204).  cnt is pair-major [q][Nv].
__global__ void te_reduce_kernel(const uint2* __restrict__ cnt, int natoms, int Nv, int K,
                                 const double* __restrict__ psi, double* __restrict__ te_mat)
{
    const long npairs = (long)natoms * (natoms - 1);
    const long q      = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (q >= npairs)
        return;
    const uint2* c   = cnt + (size_t)q * Nv;
    const double pk  = psi[K];
    double       sum = 0.0;
    auto term = [&](uint2 v) {
        const int xp = min((int)(v.x & 0xFFFFu), Nv);
        const int xf = min((int)(v.x >> 16), Nv);
        const int yp = min((int)v.y, Nv);
        return __dsub_rn(__dsub_rn(__dadd_rn(pk, psi[xp + 1]), psi[xf + 1]), psi[yp + 1]);
    };
    int i = 0;
    for (; i + 8 <= Nv; i += 8)
    {
        uint2  v[8];
        double t[8];
#pragma unroll
        for (int u = 0; u < 8; ++u)
            v[u] = c[i + u];
#pragma unroll
        for (int u = 0; u < 8; ++u)
            t[u] = term(v[u]);
#pragma unroll
        for (int u = 0; u < 8; ++u)
            sum = __dadd_rn(sum, t[u]);
    }
    for (; i < Nv; ++i)
        sum = __dadd_rn(sum, term(c[i]));
    const int a1 = (int)(q / (natoms - 1));
    const int rr = (int)(q - (long)a1 * (natoms - 1));
    const int a2 = rr < a1 ? rr : rr + 1;
    te_mat[(size_t)a1 * natoms + a2] = __ddiv_rn(sum, (double)Nv);
}

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
cudaError_t launch_te_rows(const TeBatch& b, long long rows, cudaStream_t s)
{
    if (rows <= 0)
        return cudaSuccess;
    int          threads = 256, regs = 0;
    const size_t smem    = row_sort_smem(b.maxNv - 1, &threads, &regs);
    void (*kernel)(TeBatch) = te_rows_kernel<256, 0>;
    if (threads == 256 && regs == 8)
        kernel = te_rows_kernel<256, 8>;
    else if (threads == 512 && regs == 8)
        kernel = te_rows_kernel<512, 8>;
    else if (threads == 512 && regs == 16)
        kernel = te_rows_kernel<512, 16>;
#if GC_ROWS_128
    else if (threads == 128 && regs == 16)
        kernel = te_rows_kernel<128, 16>;
#endif
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess)
        return e;
    kernel<<<(unsigned)rows, threads, smem, s>>>(b);
    return cudaGetLastError();
}

cudaError_t launch_te_walk(const TeBatch& b, int warps, bool staged, int sms, cudaStream_t s)
{
    const bool lo = b.maxK < 256;
    // two staged pair tasks per CTA (12-byte rows) where they fit beside the
    // warps' histograms, else one (16-byte rows)
    const size_t hist = (size_t)warps * kWalkBuckets * 32;
    const bool   dbuf = staged && (size_t)48 * b.maxT + hist <= (size_t)226 * 1024;
    void (*kernel)(TeBatch) = dbuf     ? (lo ? te_walk_db_kernel<true> : te_walk_db_kernel<false>)
                              : staged ? (lo ? te_walk_kernel<true, true> : te_walk_kernel<true, false>)
                                       : (lo ? te_walk_kernel<false, true> : te_walk_kernel<false, false>);
    const size_t smem = (dbuf ? (size_t)48 * b.maxT : (staged ? (size_t)2 * b.maxT * 16 : 0)) + hist;
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

cudaError_t launch_te_finish(const TeBatch& b, int sms, cudaStream_t s)
{
    const size_t smem = (size_t)kTeFinishWarps * 6 * kTeBandCap * 32;
    cudaError_t  e    = cudaFuncSetAttribute(te_finish_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess)
        return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, te_finish_kernel, kTeFinishWarps * 32, smem);
    if (e != cudaSuccess)
        return e;
    per_sm = per_sm < 1 ? 1 : per_sm;
    te_finish_kernel<<<sms * per_sm, kTeFinishWarps * 32, smem, s>>>(b);
    return cudaGetLastError();
}

cudaError_t launch_te_count(const TeBatch& b, int warps, bool staged, int sms, cudaStream_t s)
{
    // two staged pair tasks per CTA where they fit (rows of up to 3584
    // frames), else one
    const size_t db      = (size_t)4 * b.maxT * 16;
    const bool   dbuf    = staged && db <= (size_t)224 * 1024;
    void (*kernel)(TeBatch) = dbuf ? te_count_db_kernel : (staged ? te_count_kernel<true> : te_count_kernel<false>);
    const size_t smem = dbuf ? db : (staged ? (size_t)2 * b.maxT * 16 : 0);
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

cudaError_t launch_te_fixup(const TeBatch& b, int sms, cudaStream_t s)
{
    te_fixup_queue_kernel<<<sms * 4, 256, 0, s>>>(b);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return e;
    te_fixup_scan_kernel<<<sms * 4, 256, 0, s>>>(b);
    return cudaGetLastError();
}

cudaError_t launch_te_reduce(const uint2* cnt, int natoms, int Nv, int K, const double* psi, double* te_mat,
                             cudaStream_t s)
{
    const long npairs = (long)natoms * (natoms - 1);
    te_reduce_kernel<<<(unsigned)((npairs + 127) / 128), 128, 0, s>>>(cnt, natoms, Nv, K, psi, te_mat);
    return cudaGetLastError();
}

} // namespace gc
