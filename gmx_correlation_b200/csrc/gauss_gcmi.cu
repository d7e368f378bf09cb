// Gaussian (-linear) and Gaussian-copula (GCMI) mutual information on B200.
//
// Reference:
//   gauss_corrmatrix / covarianceMatrix / matrixDet / entropy
//       lib/correlation_core.cpp:280-311, :140-166, :49-98, :100-111
//   gcmi_corrmatrix / copula_transform / gcmi_erfinv / lu_det / gcmi_pair
//       lib/gcmi.cpp:246-317, :95-146, :26-79, :152-184, :190-231
//
// Both estimators need, per atom pair, the 6x6 co-moment matrix of the two
// atoms' 3-D series.  Its 3x3 blocks depend only on the two atoms, so one
// kernel sums every block (lo <= hi) once, sequentially over frames with
// round-to-nearest intrinsics (the reference's plain double loop, so the
// sums are bit-identical), and a second kernel assembles each pair's
// matrices and log-determinants.

#include "gc_common.cuh"
#include "gc_internal.h"

namespace gc {

__global__ void frame_major_kernel(const double* __restrict__ xyz, int natoms, int T, double* __restrict__ XF,
                                   int* __restrict__ status)
{
    const long n  = (long)natoms * T * 3;
    const int  nc = natoms * 3;
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < n; idx += (long)gridDim.x * blockDim.x)
    {
        const long   a = idx / ((long)T * 3);
        const long   r = idx - a * (long)T * 3;
        const int    f = (int)(r / 3), d = (int)(r - (r / 3) * 3);
        const double v = xyz[idx];
        if (!isfinite(v))
            atomicOr(status, kStatNonFinite);
        XF[(size_t)f * nc + a * 3 + d] = v;
    }
}

// gcmi_erfinv (lib/gcmi.cpp:26-79): Acklam's rational approximation of the
// inverse normal CDF (published coefficients), mapped to erfinv, then one
// Newton step with erf/exp.
__device__ double acklam_erfinv(double x)
{
    const double a0 = -3.969683028665376e+01, a1 = 2.209460984245205e+02, a2 = -2.759285104469687e+02,
                 a3 = 1.383577518672690e+02, a4 = -3.066479806614716e+01, a5 = 2.506628277459239e+00;
    const double b0 = -5.447609879822406e+01, b1 = 1.615858368580409e+02, b2 = -1.556989798598866e+02,
                 b3 = 6.680131188771972e+01, b4 = -1.328068155288572e+01;
    const double c0 = -7.784894002430293e-03, c1 = -3.223964580411365e-01, c2 = -2.400758277161838e+00,
                 c3 = -2.549732539343734e+00, c4 = 4.374664141464968e+00, c5 = 2.938163982698783e+00;
    const double d0 = 7.784695709041462e-03, d1 = 3.224671290700398e-01, d2 = 2.445134137142996e+00,
                 d3 = 3.754408661907416e+00;
    if (x >= 1.0)
        return 1e30;
    if (x <= -1.0)
        return -1e30;
    if (x == 0.0)
        return 0.0;
    const double p = __dmul_rn(__dadd_rn(x, 1.0), 0.5);
    double       r, q;
#define M_(u, v) __dmul_rn(u, v)
#define A_(u, v) __dadd_rn(u, v)
    if (p < 0.02425)
    {
        q = sqrt(M_(-2.0, log(p)));
        r = __ddiv_rn(A_(M_(A_(M_(A_(M_(A_(M_(A_(M_(c0, q), c1), q), c2), q), c3), q), c4), q), c5),
                      A_(M_(A_(M_(A_(M_(A_(M_(d0, q), d1), q), d2), q), d3), q), 1.0));
    }
    else if (p <= 0.97575)
    {
        q              = __dsub_rn(p, 0.5);
        const double s = M_(q, q);
        r = __ddiv_rn(M_(A_(M_(A_(M_(A_(M_(A_(M_(A_(M_(a0, s), a1), s), a2), s), a3), s), a4), s), a5), q),
                      A_(M_(A_(M_(A_(M_(A_(M_(A_(M_(b0, s), b1), s), b2), s), b3), s), b4), s), 1.0));
    }
    else
    {
        q = sqrt(M_(-2.0, log(__dsub_rn(1.0, p))));
        r = -__ddiv_rn(A_(M_(A_(M_(A_(M_(A_(M_(A_(M_(c0, q), c1), q), c2), q), c3), q), c4), q), c5),
                       A_(M_(A_(M_(A_(M_(A_(M_(d0, q), d1), q), d2), q), d3), q), 1.0));
    }
    r = __ddiv_rn(r, sqrt(2.0));
    r = __dsub_rn(r, M_(M_(M_(__dsub_rn(erf(r), x), sqrt(3.14159265358979323846)), 0.5), exp(M_(r, r))));
#undef M_
#undef A_
    return r;
}

// zt[t] = sqrt(2) * erfinv(2 p - 1), p = (t + 0.5) / T (lib/gcmi.cpp:133-136).
__global__ void probit_table_kernel(int T, double* __restrict__ zt)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T)
        return;
    const double p = __ddiv_rn(__dadd_rn((double)t, 0.5), (double)T);
    zt[t]          = __dmul_rn(sqrt(2.0), acklam_erfinv(__dsub_rn(__dmul_rn(2.0, p), 1.0)));
}

// Longest series the shared-memory sort below takes (next_pow2(T) * 12 bytes).
constexpr int kCopulaSortMax = 16384;

// One CTA per component: bitonic sort of (value, frame) in shared memory,
// then midrank averaging of the probit scores over runs of equal values
// (lib/gcmi.cpp:113-143).  Requires next_pow2(T) * 12 bytes of shared memory.
__global__ void copula_kernel(const double* __restrict__ XF, int natoms, int T, int P,
                              const double* __restrict__ zt, double* __restrict__ Z)
{
    extern __shared__ unsigned char smem_raw[];
    double* val = reinterpret_cast<double*>(smem_raw);
    int*    idx = reinterpret_cast<int*>(val + P);
    const int nc = natoms * 3, comp = blockIdx.x;
    for (int t = threadIdx.x; t < P; t += blockDim.x)
    {
        val[t] = t < T ? XF[(size_t)t * nc + comp] : __longlong_as_double(0x7ff0000000000000LL);
        idx[t] = t < T ? t : -1;
    }
    __syncthreads();
    for (int k = 2; k <= P; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1)
        {
            for (int t = threadIdx.x; t < P; t += blockDim.x)
            {
                const int u = t ^ j;
                if (u > t)
                {
                    const bool   up = (t & k) == 0;
                    const double vt = val[t], vu = val[u];
                    if ((vt > vu) == up)
                    {
                        val[t] = vu;
                        val[u] = vt;
                        const int it = idx[t];
                        idx[t]       = idx[u];
                        idx[u]       = it;
                    }
                }
            }
            __syncthreads();
        }
    for (int r = threadIdx.x; r < T; r += blockDim.x)
    {
        if (r > 0 && val[r] == val[r - 1])
            continue; // not the start of a run
        int s = r + 1;
        while (s < T && val[s] == val[r])
            ++s;
        double avg = 0.0;
        for (int t = r; t < s; ++t)
            avg = __dadd_rn(avg, zt[t]);
        avg = __ddiv_rn(avg, (double)(s - r));
        for (int t = r; t < s; ++t)
            Z[(size_t)idx[t] * nc + comp] = avg;
    }
}

// The same copula scores for series too long to sort in shared memory: a
// frame's run of equal values starts at rank r = #{g : x_g < x_f} and holds
// m = #{g : x_g == x_f} frames, so its score is the average of zt[r .. r+m)
// summed in rank order, as in the sorted form.  Grid (frame blocks,
// components); the component's values pass through shared memory in tiles.
constexpr int kCopulaTile = 4096;

__global__ void __launch_bounds__(256) copula_count_kernel(const double* __restrict__ XF, int natoms, int T,
                                                           const double* __restrict__ zt, double* __restrict__ Z)
{
    __shared__ double tile[kCopulaTile];
    const int    nc   = natoms * 3, comp = blockIdx.y;
    const int    f    = blockIdx.x * blockDim.x + threadIdx.x;
    const double v    = f < T ? XF[(size_t)f * nc + comp] : 0.0;
    int          lt = 0, eq = 0;
    for (int t0 = 0; t0 < T; t0 += kCopulaTile)
    {
        const int n = min(kCopulaTile, T - t0);
        __syncthreads(); // the previous tile is consumed
        for (int e = threadIdx.x; e < n; e += blockDim.x)
            tile[e] = XF[(size_t)(t0 + e) * nc + comp];
        __syncthreads();
        for (int e = 0; e < n; ++e)
        {
            const double u = tile[e];
            lt += u < v;
            eq += u == v;
        }
    }
    if (f >= T)
        return;
    double avg = 0.0;
    for (int t = lt; t < lt + eq; ++t)
        avg = __dadd_rn(avg, zt[t]);
    Z[(size_t)f * nc + comp] = __ddiv_rn(avg, (double)eq);
}

// Block b = hi*(hi+1)/2 + lo (lo <= hi): 9 co-moments summed over frames in order.
__global__ void blocks_kernel(const double* __restrict__ V, int natoms, int T, double* __restrict__ blk)
{
    const long nb = (long)natoms * (natoms + 1) / 2;
    const long b  = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (b >= nb)
        return;
    long hi = (long)((sqrt(8.0 * (double)b + 1.0) - 1.0) * 0.5);
    while (hi * (hi + 1) / 2 > b)
        --hi;
    while ((hi + 1) * (hi + 2) / 2 <= b)
        ++hi;
    const long lo = b - hi * (hi + 1) / 2;
    const int  nc = natoms * 3;
    double     acc[9];
#pragma unroll
    for (int e = 0; e < 9; ++e)
        acc[e] = 0.0;
    const double* pl = V + lo * 3;
    const double* ph = V + hi * 3;
    for (int f = 0; f < T; ++f)
    {
        const double l0 = pl[(size_t)f * nc], l1 = pl[(size_t)f * nc + 1], l2 = pl[(size_t)f * nc + 2];
        const double h0 = ph[(size_t)f * nc], h1 = ph[(size_t)f * nc + 1], h2 = ph[(size_t)f * nc + 2];
        acc[0] = __dadd_rn(acc[0], __dmul_rn(l0, h0));
        acc[1] = __dadd_rn(acc[1], __dmul_rn(l0, h1));
        acc[2] = __dadd_rn(acc[2], __dmul_rn(l0, h2));
        acc[3] = __dadd_rn(acc[3], __dmul_rn(l1, h0));
        acc[4] = __dadd_rn(acc[4], __dmul_rn(l1, h1));
        acc[5] = __dadd_rn(acc[5], __dmul_rn(l1, h2));
        acc[6] = __dadd_rn(acc[6], __dmul_rn(l2, h0));
        acc[7] = __dadd_rn(acc[7], __dmul_rn(l2, h1));
        acc[8] = __dadd_rn(acc[8], __dmul_rn(l2, h2));
    }
#pragma unroll
    for (int e = 0; e < 9; ++e)
        blk[b * 9 + e] = acc[e];
}

// Determinant by LU with partial pivoting (lib/correlation_core.cpp:49-98,
// lib/gcmi.cpp:152-184; the two differ only in a store that never feeds
// the determinant).
__device__ double lu_det(double* m, int n)
{
    double sign = 1.0;
    for (int col = 0; col < n; ++col)
    {
        int    pivot = col;
        double best  = fabs(m[col * n + col]);
        for (int row = col + 1; row < n; ++row)
        {
            const double v = fabs(m[row * n + col]);
            if (v > best)
            {
                best  = v;
                pivot = row;
            }
        }
        if (best == 0.0)
            return 0.0;
        if (pivot != col)
        {
            for (int j = 0; j < n; ++j)
            {
                const double t   = m[col * n + j];
                m[col * n + j]   = m[pivot * n + j];
                m[pivot * n + j] = t;
            }
            sign = -sign;
        }
        const double diag = m[col * n + col];
        for (int row = col + 1; row < n; ++row)
        {
            const double factor = __ddiv_rn(m[row * n + col], diag);
            for (int j = col + 1; j < n; ++j)
                m[row * n + j] = __dsub_rn(m[row * n + j], __dmul_rn(factor, m[col * n + j]));
        }
    }
    double det = sign;
    for (int i = 0; i < n; ++i)
        det = __dmul_rn(det, m[i * n + i]);
    return det;
}

__device__ __forceinline__ long block_index(long lo, long hi) { return hi * (hi + 1) / 2 + lo; }

// entropy (lib/correlation_core.cpp:100-111).
__device__ double gauss_entropy(double* m, int n, double log2pi)
{
    const double det = lu_det(m, n);
    if (det <= 0.0)
        return 0.0;
    return __dmul_rn(0.5, __dadd_rn(__dmul_rn((double)n, __dadd_rn(1.0, log2pi)), log(det)));
}

__global__ void pair_logdet_kernel(const double* __restrict__ blk, int natoms, int T, int mode, double log2pi,
                                   double* __restrict__ mat)
{
    const long np = (long)natoms * (natoms - 1) / 2;
    const long p  = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (p < natoms)
        mat[(size_t)p * natoms + p] = 2000.0;
    if (p >= np)
        return;
    int hi, lo;
    pair_from_index(p, &hi, &lo); // hi > lo
    const double* bll = blk + block_index(lo, lo) * 9;
    const double* bhh = blk + block_index(hi, hi) * 9;
    const double* blh = blk + block_index(lo, hi) * 9; // sum V_lo,r * V_hi,c
    double        mi;
    if (mode == 0)
    {
        // gauss_corrmatrix iterates a1 < a2: first = a1 = lo, second = hi.
        double first[9], second[9], comb[36];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c)
            {
                first[r * 3 + c]          = __ddiv_rn(bll[r * 3 + c], (double)T);
                second[r * 3 + c]         = __ddiv_rn(bhh[r * 3 + c], (double)T);
                const double cr           = __ddiv_rn(blh[r * 3 + c], (double)T);
                comb[r * 6 + c]           = first[r * 3 + c];
                comb[(r + 3) * 6 + c + 3] = second[r * 3 + c];
                comb[r * 6 + c + 3]       = cr;
                comb[(c + 3) * 6 + r]     = cr;
            }
        const double e1 = gauss_entropy(first, 3, log2pi);
        const double e2 = gauss_entropy(second, 3, log2pi);
        mi              = __dsub_rn(__dadd_rn(e1, e2), gauss_entropy(comb, 6, log2pi));
    }
    else
    {
        // gcmi_pair(z, N, a1, a2) with a1 = hi > a2 = lo: v = [hi, lo].
        const double invN = __ddiv_rn(1.0, (double)T);
        double       c6[36], c1[9], c2[9];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c)
            {
                c6[r * 6 + c]           = __dmul_rn(bhh[r * 3 + c], invN);
                c6[(r + 3) * 6 + c + 3] = __dmul_rn(bll[r * 3 + c], invN);
                c6[r * 6 + c + 3]       = __dmul_rn(blh[c * 3 + r], invN); // sum z_hi,r z_lo,c
                c6[(r + 3) * 6 + c]     = __dmul_rn(blh[r * 3 + c], invN); // sum z_lo,r z_hi,c
            }
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c)
            {
                c1[r * 3 + c] = c6[r * 6 + c];
                c2[r * 3 + c] = c6[(r + 3) * 6 + c + 3];
            }
        const double d1 = lu_det(c1, 3), d2 = lu_det(c2, 3), dJ = lu_det(c6, 6);
        if (d1 <= 0.0 || d2 <= 0.0 || dJ <= 0.0)
            mi = 0.0;
        else
            mi = __dmul_rn(0.5, __dsub_rn(__dadd_rn(log(d1), log(d2)), log(dJ)));
    }
    mat[(size_t)hi * natoms + lo] = mi;
    mat[(size_t)lo * natoms + hi] = mi;
}

void launch_frame_major(const double* xyz, int natoms, int T, double* XF, int* status, cudaStream_t s)
{
    frame_major_kernel<<<1184, 256, 0, s>>>(xyz, natoms, T, XF, status);
}

void launch_copula(const double* XF, int natoms, int T, double* zt, double* Z, cudaStream_t s)
{
    probit_table_kernel<<<(T + 127) / 128, 128, 0, s>>>(T, zt);
    if (T > kCopulaSortMax)
    {
        copula_count_kernel<<<dim3((unsigned)((T + 255) / 256), (unsigned)(natoms * 3)), 256, 0, s>>>(XF, natoms, T,
                                                                                                     zt, Z);
        return;
    }
    int P = 1;
    while (P < T)
        P <<= 1;
    const size_t smem = (size_t)P * (sizeof(double) + sizeof(int));
    if (smem > 48 * 1024)
        cudaFuncSetAttribute(copula_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    copula_kernel<<<natoms * 3, 512, smem, s>>>(XF, natoms, T, P, zt, Z);
}

void launch_blocks(const double* V, int natoms, int T, double* blk, cudaStream_t s)
{
    const long nb = (long)natoms * (natoms + 1) / 2;
    blocks_kernel<<<(unsigned)((nb + 127) / 128), 128, 0, s>>>(V, natoms, T, blk);
}

void launch_pair_logdet(const double* blk, int natoms, int T, int mode, double log2pi, double* mat,
                        cudaStream_t s)
{
    long np = (long)natoms * (natoms - 1) / 2;
    if (np < natoms)
        np = natoms;
    pair_logdet_kernel<<<(unsigned)((np + 127) / 128), 128, 0, s>>>(blk, natoms, T, mode, log2pi, mat);
}

} // namespace gc
