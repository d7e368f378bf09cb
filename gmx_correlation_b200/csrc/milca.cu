// The MILCA estimator family (lib/kraskov.cpp:347-2155) on the GPU: one warp
// per query frame, exact FP64 arithmetic throughout.
//
// Every variant of the family does, per query frame i (neiK, :257-343, then
// the per-variant loops):
//   1. the K nearest frames j != i in the joint max-norm over all
//      components, exact distance ties broken in neiK's grid-scan order
//      (square shells of the 2-D grid on components grid1/grid2, frames in
//      ascending order inside a cell);
//   2. per variable g, eps_g = the largest distance in that variable's
//      components over those K neighbours (over the first k, for the
//      k = 1 .. K variants); Eps = max_g eps_g and the variable owning it;
//   3. counts per variable: n2_g at eps_g and n1_g at Eps, either the exact
//      max-norm count #{j != i : d_g(i,j) <= t} (neiE / neiEK) or, for the
//      one-component variables of mi2 / red / ..., the reference's 1-D box
//      count neiE1 (:92-112), which checks the distance only in the two end
//      boxes of [x - t, x + t] and counts every frame of the boxes between.
// The ordered digamma sums are reduced by milca_sum_kernel.  The selection
// reuses the radix selection of the KSG exact path (gc_common.cuh), so the
// neighbour sets, maxima and counts are the reference's exactly.

#include "gc_common.cuh"
#include "gc_internal.h"
#include "milca.h"

namespace gc {

namespace {

constexpr int kMilcaWarps = 4; // warps per CTA

// Dynamic shared memory of one warp: the radix histogram, then (k = 1 .. K
// variants) the sort buffer; 16-byte multiples so every warp's 64-bit keys
// stay aligned.
__host__ __device__ inline size_t milca_smem_per_warp(int krange, int Kp)
{
    return (256 * sizeof(unsigned) + (krange ? (size_t)Kp * 20 : 0) + 15) & ~(size_t)15;
}

__device__ __forceinline__ double comp(const MilcaParams& p, int c, int t) { return p.X[(size_t)c * p.N + t]; }

// Max-norm distance of frames i and j over components [c0, c0 + n).
__device__ __forceinline__ double range_dist(const MilcaParams& p, int c0, int n, int i, int j)
{
    double d = fabs(comp(p, c0, i) - comp(p, c0, j));
    for (int c = 1; c < n; ++c)
        d = fmax(d, fabs(comp(p, c0 + c, i) - comp(p, c0 + c, j)));
    return d;
}

// The 1-D box count's two end boxes and its "box between" test for the
// threshold t around the value xc (neiE1: mp = lrint((xc + t) * scal) capped
// at bs, mm = lrint((xc - t) * scal) floored at 0; box(x) = (int)(x * scal)).
struct Box1
{
    int    mp, mm;
    double t, xc;
    __device__ void set(double xc_, double t_, double scal, int bs)
    {
        t                 = t_;
        xc                = xc_;
        const long long a = (long long)rint(__dmul_rn(__dadd_rn(xc, t), scal));
        const long long b = (long long)rint(__dmul_rn(__dsub_rn(xc, t), scal));
        mp                = (int)(a > bs ? bs : a);
        mm                = (int)(b < 0 ? 0 : b);
    }
    // is frame value x (in box bx) counted
    __device__ __forceinline__ bool in(double x, int bx) const
    {
        if (bx == mp)
            return fabs(x - xc) <= t;
        if (mm >= mp)
            return false;
        if (bx == mm)
            return fabs(xc - x) <= t;
        return bx > mm && bx < mp;
    }
};

__device__ __forceinline__ int box1_of(double x, double scal) { return (int)__dmul_rn(x, scal); }

// Per variable, eps and the Eps owner from the per-group maxima (the
// variant's tie rule).
__device__ __forceinline__ void owner(const MilcaParams& p, const double* e, double& Eps, int& md)
{
    if (p.tie_xy)
    {
        md  = e[0] > e[1] ? 0 : 1;
        Eps = e[md];
        return;
    }
    Eps = 0.0;
    md  = -1;
    for (int g = 0; g < p.G; ++g)
        if (e[g] > Eps)
        {
            Eps = e[g];
            md  = g;
        }
}

} // namespace

// One warp per query frame.  Dynamic shared memory per warp: the radix
// histogram (256 words) and, for the k = 1 .. K variants, the sort buffer of
// the K nearest (Kp = K rounded up to a power of two: two 64-bit keys and a
// frame index each).
__global__ void __launch_bounds__(kMilcaWarps * 32) milca_query_kernel(MilcaParams p, int Kp)
{
    extern __shared__ unsigned char smem[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int i    = blockIdx.x * kMilcaWarps + w;
    if (i >= p.N)
        return;
    unsigned char* base = smem + milca_smem_per_warp(p.krange, Kp) * w;
    unsigned*      hist  = reinterpret_cast<unsigned*>(base);
    const ScanGrid sg(p.box);
    const int      ix = sg.qcell(comp(p, p.grid1, i)), iy = sg.qcell(comp(p, p.grid2, i));
    auto           joint = [&](int j) { return range_dist(p, 0, p.D, i, j); };
    auto           rank  = [&](int j) { return sg.rank(ix, iy, comp(p, p.grid1, j), comp(p, p.grid2, j), j, p.N); };

    // 1. the K-th smallest joint distance and, on an exact tie there, the
    //    cut in scan order
    auto vkey = [&](int j, unsigned long long& k) -> bool {
        if (j == i)
            return false;
        k = dbits(joint(j));
        return true;
    };
    int                      below;
    const unsigned long long dkb  = warp_select_u64(vkey, p.N, p.K, 56, hist, lane, &below);
    const double             dk   = __longlong_as_double((long long)dkb);
    const int                need = p.K - below;
    int                      tied = 0;
    for (int j = lane; j < p.N; j += 32)
        tied += j != i && joint(j) == dk;
    tied                    = __reduce_add_sync(kFull, tied);
    unsigned long long rcut = ~0ull;
    if (tied > need)
    {
        auto rkey = [&](int j, unsigned long long& k) -> bool {
            if (j == i || joint(j) != dk)
                return false;
            k = rank(j);
            return true;
        };
        int b2;
        rcut = warp_select_u64(rkey, p.N, need, p.rank_shift, hist, lane, &b2);
    }
    auto chosen = [&](int j, double d) { return d < dk || (d == dk && (rcut == ~0ull || rank(j) <= rcut)); };

    const int Kr = p.krange ? p.K : 1;
    double*   epsq = p.eps + (size_t)i * Kr * (p.G + 1);

    if (!p.krange)
    {
        // 2. per-variable maxima over the K chosen neighbours
        double e[kMilcaMaxGroups];
        for (int g = 0; g < p.G; ++g)
            e[g] = 0.0;
        for (int j = lane; j < p.N; j += 32)
        {
            if (j == i || !chosen(j, joint(j)))
                continue;
            for (int g = 0; g < p.G; ++g)
                e[g] = fmax(e[g], range_dist(p, p.gfirst[g], p.gdim[g], i, j));
        }
        for (int g = 0; g < p.G; ++g)
            e[g] = warp_max(e[g]);
        double Eps;
        int    md;
        owner(p, e, Eps, md);
        // 3. counts at eps_g and at Eps (self included, then removed, as the
        //    reference's neighbour counts do)
        int  n1[kMilcaMaxGroups], n2[kMilcaMaxGroups];
        Box1 b1[kMilcaMaxGroups], b2[kMilcaMaxGroups];
        for (int g = 0; g < p.G; ++g)
        {
            n1[g] = n2[g] = 0;
            if (p.gbox1d[g])
            {
                const double xc = comp(p, p.gfirst[g], i);
                b2[g].set(xc, e[g], p.gscal[g], p.bs1);
                b1[g].set(xc, Eps, p.gscal[g], p.bs1);
            }
        }
        for (int j = lane; j < p.N; j += 32)
            for (int g = 0; g < p.G; ++g)
            {
                if (p.gbox1d[g])
                {
                    const double x  = comp(p, p.gfirst[g], j);
                    const int    bx = box1_of(x, p.gscal[g]);
                    n2[g] += b2[g].in(x, bx);
                    n1[g] += b1[g].in(x, bx);
                }
                else
                {
                    const double d = range_dist(p, p.gfirst[g], p.gdim[g], i, j);
                    n2[g] += d <= e[g];
                    n1[g] += d <= Eps;
                }
            }
        for (int g = 0; g < p.G; ++g)
        {
            n1[g] = __reduce_add_sync(kFull, n1[g]) - 1;
            n2[g] = __reduce_add_sync(kFull, n2[g]) - 1;
        }
        if (lane == 0)
        {
            int* c = p.cnt + (size_t)i * p.G * 2;
            for (int g = 0; g < p.G; ++g)
            {
                c[2 * g]     = g == md ? n2[g] : n1[g];
                c[2 * g + 1] = n2[g];
                epsq[g] = e[g];
            }
            epsq[p.G] = Eps;
            p.maxd[i] = md;
        }
        return;
    }

    // k = 1 .. K: the K chosen neighbours, sorted by (distance, scan rank)
    unsigned long long* kd = reinterpret_cast<unsigned long long*>(base + 256 * sizeof(unsigned));
    unsigned long long* kr = kd + Kp;
    int*                kj = reinterpret_cast<int*>(kr + Kp);
    int                 slot = 0;
    for (int j0 = 0; j0 < p.N; j0 += 32)
    {
        const int    j  = j0 + lane;
        const double d  = j < p.N && j != i ? joint(j) : 0.0;
        const bool   on = j < p.N && j != i && chosen(j, d);
        const unsigned m = __ballot_sync(kFull, on);
        const int s = slot + __popc(m & ((1u << lane) - 1u));
        if (on && s < Kp)
        {
            kd[s]       = dbits(d);
            kr[s]       = rank(j);
            kj[s]       = j;
        }
        slot += __popc(m);
    }
    for (int s = p.K + lane; s < Kp; s += 32)
    {
        kd[s] = ~0ull;
        kr[s] = ~0ull;
        kj[s] = -1;
    }
    __syncwarp();
    // bitonic sort of Kp entries by (kd, kr)
    for (int size = 2; size <= Kp; size <<= 1)
        for (int stride = size >> 1; stride > 0; stride >>= 1)
        {
            for (int t = lane; t < Kp / 2; t += 32)
            {
                const int  a   = 2 * t - (t & (stride - 1));
                const int  b   = a + stride;
                const bool up  = (a & size) == 0;
                const bool gt  = kd[a] > kd[b] || (kd[a] == kd[b] && kr[a] > kr[b]);
                if (gt == up)
                {
                    const unsigned long long td = kd[a], tr = kr[a];
                    const int                tj = kj[a];
                    kd[a] = kd[b];
                    kr[a] = kr[b];
                    kj[a] = kj[b];
                    kd[b] = td;
                    kr[b] = tr;
                    kj[b] = tj;
                }
            }
            __syncwarp();
        }
    // prefix maxima per variable (lane g), then Eps and its owner per k
    if (lane < p.G)
    {
        double m = 0.0;
        for (int k = 0; k < p.K; ++k)
        {
            m                                 = fmax(m, range_dist(p, p.gfirst[lane], p.gdim[lane], i, kj[k]));
            epsq[(size_t)k * (p.G + 1) + lane] = m;
        }
    }
    __syncwarp();
    for (int k = lane; k < p.K; k += 32)
    {
        double* ek = epsq + (size_t)k * (p.G + 1);
        double  Eps;
        int     md;
        owner(p, ek, Eps, md);
        ek[p.G]                 = Eps;
        p.maxd[(size_t)i * Kr + k] = md;
        // counts of this k, one lane per k over all frames
        int* c = p.cnt + ((size_t)i * Kr + k) * p.G * 2;
        for (int g = 0; g < p.G; ++g)
        {
            int a1 = 0, a2 = 0;
            if (p.gbox1d[g])
            {
                const double xc = comp(p, p.gfirst[g], i);
                Box1         b1, b2;
                b2.set(xc, ek[g], p.gscal[g], p.bs1);
                b1.set(xc, Eps, p.gscal[g], p.bs1);
                for (int j = 0; j < p.N; ++j)
                {
                    const double x  = comp(p, p.gfirst[g], j);
                    const int    bx = box1_of(x, p.gscal[g]);
                    a2 += b2.in(x, bx);
                    a1 += b1.in(x, bx);
                }
            }
            else
                for (int j = 0; j < p.N; ++j)
                {
                    const double d = range_dist(p, p.gfirst[g], p.gdim[g], i, j);
                    a2 += d <= ek[g];
                    a1 += d <= Eps;
                }
            a1 -= 1;
            a2 -= 1;
            c[2 * g]     = g == md ? a2 : a1;
            c[2 * g + 1] = a2;
        }
    }
}

// Ordered digamma sums, one thread per k: the reference's loop over query
// frames (in its order), its association (dxy += psi_a + psi_b for two
// variables, term by term for the redundancy forms), then
// (G-1) psi[N] + psi[k] - dxy1 / N and the same with phi[k] for dxy2.
__global__ void milca_sum_kernel(MilcaSum s, const int* __restrict__ cnt, const int* __restrict__ maxd)
{
    const int Kr = s.krange ? s.K : 1;
    const int k  = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= Kr)
        return;
    const int kk  = s.krange ? k + 1 : s.K;
    double    dx1 = 0.0, dx2 = 0.0;
    for (int q = 0; q < s.N; ++q)
    {
        const int  i  = s.order[q];
        const int* c  = cnt + ((size_t)i * Kr + k) * s.G * 2;
        const int  md = maxd[(size_t)i * Kr + k];
        // a 1-D box count can be -1 (the query's own box outside [x - t,
        // x + t]'s end boxes): the reference then reads psi[-1], the word
        // before its table; it is taken as 0 here, the value of psi[0]
        auto ps = [&](int n) { return n < 0 ? 0.0 : s.psi[n]; };
        if (s.pair_sum)
        {
            const double a1 = ps(c[0] + (md != 0)), b1 = ps(c[2] + (md != 1));
            dx1             = __dadd_rn(dx1, __dadd_rn(a1, b1));
            dx2             = __dadd_rn(dx2, __dadd_rn(ps(c[1]), ps(c[3])));
        }
        else
            for (int g = 0; g < s.G; ++g)
            {
                dx1 = __dadd_rn(dx1, ps(c[2 * g] + (md != g)));
                dx2 = __dadd_rn(dx2, ps(c[2 * g + 1]));
            }
    }
    dx1               = __ddiv_rn(dx1, (double)s.N);
    dx2               = __ddiv_rn(dx2, (double)s.N);
    const double base = __dmul_rn((double)(s.G - 1), s.psi[s.N]);
    const double phik = s.phi ? s.phi[kk] : __dsub_rn(s.psi[kk], __ddiv_rn((double)(s.G - 1), (double)kk));
    if (s.mic)
        s.mic[k] = __dsub_rn(__dadd_rn(base, s.psi[kk]), dx1);
    if (s.mir)
        s.mir[k] = __dsub_rn(__dadd_rn(base, phik), dx2);
}

cudaError_t launch_milca(const MilcaParams& p, const MilcaSum& s, cudaStream_t st)
{
    int Kp = 1;
    while (p.krange && Kp < p.K)
        Kp <<= 1;
    const size_t smem = milca_smem_per_warp(p.krange, Kp) * kMilcaWarps;
    if (smem > 48 * 1024)
    {
        const cudaError_t e = cudaFuncSetAttribute(milca_query_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)smem);
        if (e != cudaSuccess)
            return e;
    }
    milca_query_kernel<<<(p.N + kMilcaWarps - 1) / kMilcaWarps, kMilcaWarps * 32, smem, st>>>(p, Kp);
    const int Kr = p.krange ? p.K : 1;
    milca_sum_kernel<<<(Kr + 127) / 128, 128, 0, st>>>(s, p.cnt, p.maxd);
    return cudaGetLastError();
}

} // namespace gc
