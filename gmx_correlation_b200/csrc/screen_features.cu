// Per-pair features of the learned KSG screen (no counterpart in the
// reference; the screen predicts KSG r(MI) so that exact KSG runs only on
// the pairs the prediction cannot settle).
//
// Feature row of one atom pair (a1, a2), width kScreenBase + H:
//   [0]       Gaussian MI 0.5 (log|C_11| + log|C_22| - log|C|) of the pair's
//             6x6 covariance C (the -linear estimator, divide by T)
//   [1..6]    eigenvalues of the 6x6 joint correlation matrix, descending
//   [7..12]   excess kurtosis of the six components: each atom's three
//             sorted descending, the atom with the larger maximum first
//   [13..21]  |3x3 cross-correlation| corr(x_a1,d, x_a2,e), sorted descending
//   [22]      k / T (the KSG bias depends on the neighbour fraction)
//   [23..]    8x8 joint histogram of the two atoms' first-principal-axis
//             projections in rank space (8 equal-count bins per atom),
//             oriented so that its rank correlation is >= 0 and symmetrised
//             (h + h^T) / 2, as fractions of T.  With a PCA basis
//             (mean[64], comp[H][64]) the row holds the H projections; with
//             none it holds the 64 raw cells (used to fit the basis).
// Every statistic is over all T frames of the mean-centred coordinates.

#include "gc_common.cuh"
#include "gc_internal.h"

namespace gc {

namespace {

// Cyclic Jacobi diagonalisation of a symmetric n x n matrix (n <= 6) in
// place; eigenvalues descending into ev, and (when vec != nullptr) the
// matching unit eigenvectors as columns of vec [n][n].
__device__ void jacobi_sym(double* a, int n, double* ev, double* vec)
{
    double v[36];
    for (int i = 0; i < n * n; ++i)
        v[i] = (i % (n + 1) == 0) ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 40; ++sweep)
    {
        double off = 0.0, dia = 0.0;
        for (int p = 0; p < n; ++p)
        {
            dia += a[p * n + p] * a[p * n + p];
            for (int q = p + 1; q < n; ++q)
                off += a[p * n + q] * a[p * n + q];
        }
        if (off <= 1e-30 * dia)
            break;
        for (int p = 0; p < n; ++p)
            for (int q = p + 1; q < n; ++q)
            {
                const double apq = a[p * n + q];
                if (apq == 0.0)
                    continue;
                const double theta = (a[q * n + q] - a[p * n + p]) / (2.0 * apq);
                const double t     = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < n; ++k)
                {
                    const double akp = a[k * n + p], akq = a[k * n + q];
                    a[k * n + p] = c * akp - s * akq;
                    a[k * n + q] = s * akp + c * akq;
                }
                for (int k = 0; k < n; ++k)
                {
                    const double apk = a[p * n + k], aqk = a[q * n + k];
                    a[p * n + k] = c * apk - s * aqk;
                    a[q * n + k] = s * apk + c * aqk;
                }
                for (int k = 0; k < n; ++k)
                {
                    const double vkp = v[k * n + p], vkq = v[k * n + q];
                    v[k * n + p] = c * vkp - s * vkq;
                    v[k * n + q] = s * vkp + c * vkq;
                }
            }
    }
    int order[6];
    for (int i = 0; i < n; ++i)
        order[i] = i;
    for (int i = 1; i < n; ++i)
    {
        const int o = order[i];
        int       j = i - 1;
        while (j >= 0 && a[order[j] * n + order[j]] < a[o * n + o])
        {
            order[j + 1] = order[j];
            --j;
        }
        order[j + 1] = o;
    }
    for (int i = 0; i < n; ++i)
    {
        ev[i] = a[order[i] * n + order[i]];
        if (vec)
            for (int k = 0; k < n; ++k)
                vec[k * n + i] = v[k * n + order[i]];
    }
}

// Determinant by LU with partial pivoting (destroys m).
__device__ double det_lu(double* m, int n)
{
    double det = 1.0;
    for (int c = 0; c < n; ++c)
    {
        int    piv  = c;
        double best = fabs(m[c * n + c]);
        for (int r = c + 1; r < n; ++r)
            if (fabs(m[r * n + c]) > best)
            {
                best = fabs(m[r * n + c]);
                piv  = r;
            }
        if (best == 0.0)
            return 0.0;
        if (piv != c)
        {
            for (int j = 0; j < n; ++j)
            {
                const double t = m[c * n + j];
                m[c * n + j]   = m[piv * n + j];
                m[piv * n + j] = t;
            }
            det = -det;
        }
        for (int r = c + 1; r < n; ++r)
        {
            const double f = m[r * n + c] / m[c * n + c];
            for (int j = c + 1; j < n; ++j)
                m[r * n + j] -= f * m[c * n + j];
        }
        det *= m[c * n + c];
    }
    return det;
}

__device__ void sort_desc(double* v, int n)
{
    for (int i = 1; i < n; ++i)
    {
        const double x = v[i];
        int          j = i - 1;
        while (j >= 0 && v[j] < x)
        {
            v[j + 1] = v[j];
            --j;
        }
        v[j + 1] = x;
    }
}

__device__ double block_sum(double v, double* red)
{
    const int tid = threadIdx.x;
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(kFull, v, o);
    __syncthreads();
    if ((tid & 31) == 0)
        red[tid >> 5] = v;
    __syncthreads();
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
        s += red[w];
    return s;
}

} // namespace

// One CTA (256 threads) per atom: means, covariance, kurtoses, the first
// principal axis, and the rank bin (0..7) of every frame's projection on it.
// stats[a * kScreenStat + ...]: [0..2] means, [3..5] standard deviations,
// [6..8] excess kurtoses (component order), [9..14] covariance (xx, xy, xz,
// yy, yz, zz), all divided by T.
__global__ void __launch_bounds__(256) screen_atom_kernel(const double* __restrict__ xyz, int T, int P,
                                                          double* __restrict__ stats,
                                                          unsigned char* __restrict__ bins)
{
    extern __shared__ __align__(16) unsigned char sm[];
    unsigned long long* keys = reinterpret_cast<unsigned long long*>(sm); // [P]
    __shared__ double   red[8];
    __shared__ double   mom[12];
    __shared__ double   axis[3];
    const int           a = blockIdx.x, tid = threadIdx.x;
    const double*       x = xyz + (size_t)a * T * 3;

    for (int d = 0; d < 3; ++d)
    {
        double s = 0.0;
        for (int f = tid; f < T; f += 256)
            s += x[(size_t)f * 3 + d];
        s = block_sum(s, red);
        if (tid == 0)
            mom[d] = s / T;
    }
    __syncthreads();
    const double m0 = mom[0], m1 = mom[1], m2 = mom[2];
    double       acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int f = tid; f < T; f += 256)
    {
        const double u = x[(size_t)f * 3] - m0, v = x[(size_t)f * 3 + 1] - m1, w = x[(size_t)f * 3 + 2] - m2;
        acc[0] += u * u;
        acc[1] += u * v;
        acc[2] += u * w;
        acc[3] += v * v;
        acc[4] += v * w;
        acc[5] += w * w;
        acc[6] += (u * u) * (u * u);
        acc[7] += (v * v) * (v * v);
        acc[8] += (w * w) * (w * w);
    }
    for (int e = 0; e < 9; ++e)
    {
        const double s = block_sum(acc[e], red);
        if (tid == 0)
            mom[3 + e] = s / T;
    }
    __syncthreads();
    if (tid == 0)
    {
        double*      st     = stats + (size_t)a * kScreenStat;
        const double c[6]   = {mom[3], mom[4], mom[5], mom[6], mom[7], mom[8]};
        const double var[3] = {c[0], c[3], c[5]};
        for (int d = 0; d < 3; ++d)
        {
            st[d]     = mom[d];
            st[3 + d] = sqrt(var[d]);
            st[6 + d] = var[d] > 0.0 ? mom[9 + d] / (var[d] * var[d]) - 3.0 : 0.0;
        }
        for (int e = 0; e < 6; ++e)
            st[9 + e] = c[e];
        double m[9] = {c[0], c[1], c[2], c[1], c[3], c[4], c[2], c[4], c[5]};
        double ev[3], vec[9];
        jacobi_sym(m, 3, ev, vec);
        // sign: the largest-magnitude component positive
        int big = 0;
        for (int d = 1; d < 3; ++d)
            if (fabs(vec[d * 3]) > fabs(vec[big * 3]))
                big = d;
        const double sg = vec[big * 3] < 0.0 ? -1.0 : 1.0;
        for (int d = 0; d < 3; ++d)
            axis[d] = sg * vec[d * 3];
    }
    __syncthreads();
    // order-preserving keys of the float projection, frame in the low word
    for (int f = tid; f < P; f += 256)
    {
        unsigned long long k = ~0ull;
        if (f < T)
        {
            const double pr = (x[(size_t)f * 3] - m0) * axis[0] + (x[(size_t)f * 3 + 1] - m1) * axis[1] +
                              (x[(size_t)f * 3 + 2] - m2) * axis[2];
            unsigned u = __float_as_uint((float)pr);
            u          = (u & 0x80000000u) ? ~u : (u | 0x80000000u);
            k          = ((unsigned long long)u << 32) | (unsigned)f;
        }
        keys[f] = k;
    }
    __syncthreads();
    for (int k = 2; k <= P; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1)
        {
            for (int t = tid; t < (P >> 1); t += 256)
            {
                const int                idx = ((t / j) * (j << 1)) + (t % j);
                const int                prt = idx + j;
                const unsigned long long u = keys[idx], w = keys[prt];
                const bool               up = (idx & k) == 0;
                if ((u > w) == up)
                {
                    keys[idx] = w;
                    keys[prt] = u;
                }
            }
            __syncthreads();
        }
    for (int r = tid; r < T; r += 256)
        bins[(size_t)a * T + (unsigned)(keys[r] & 0xFFFFFFFFu)] = (unsigned char)((8 * r) / T);
}

// One warp per pair (a1 > a2).  Pair pl of the launch is the pair_ab entry
// when a list is given, else p = pair_begin + pl in the order
// p = a1 (a1 - 1) / 2 + a2.
__global__ void __launch_bounds__(256) screen_pair_kernel(const double* __restrict__ xyz, int T, int K,
                                                          const double* __restrict__ stats,
                                                          const unsigned char* __restrict__ bins, long pair_begin,
                                                          long pair_count, const int2* __restrict__ pair_ab,
                                                          const float* __restrict__ pca, int ncomp,
                                                          float* __restrict__ out, int width)
{
    __shared__ unsigned hist[8][64];
    const int           warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long          pl   = (long)blockIdx.x * 8 + warp;
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
    const double*        s1 = stats + (size_t)a1 * kScreenStat;
    const double*        s2 = stats + (size_t)a2 * kScreenStat;
    const double*        x1 = xyz + (size_t)a1 * T * 3;
    const double*        x2 = xyz + (size_t)a2 * T * 3;
    const unsigned char* b1 = bins + (size_t)a1 * T;
    const unsigned char* b2 = bins + (size_t)a2 * T;
    unsigned*            h  = hist[warp];
    h[lane]                 = 0u;
    h[lane + 32]            = 0u;
    __syncwarp();
    const double mu1[3] = {s1[0], s1[1], s1[2]}, mu2[3] = {s2[0], s2[1], s2[2]};
    double       cr[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int f = lane; f < T; f += 32)
    {
        double u[3], v[3];
#pragma unroll
        for (int d = 0; d < 3; ++d)
        {
            u[d] = x1[(size_t)f * 3 + d] - mu1[d];
            v[d] = x2[(size_t)f * 3 + d] - mu2[d];
        }
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c)
                cr[r * 3 + c] += u[r] * v[c];
        atomicAdd(&h[b1[f] * 8 + b2[f]], 1u);
    }
#pragma unroll
    for (int e = 0; e < 9; ++e)
        for (int o = 16; o > 0; o >>= 1)
            cr[e] += __shfl_xor_sync(kFull, cr[e], o);
    __syncwarp();
    // orientation: rank correlation of the binned projections >= 0
    double sc = 0.0;
    for (int c = lane; c < 64; c += 32)
        sc += (double)h[c] * ((c >> 3) - 3.5) * ((c & 7) - 3.5);
    for (int o = 16; o > 0; o >>= 1)
        sc += __shfl_xor_sync(kFull, sc, o);
    const bool flip = sc < 0.0;
    const float inv = 1.0f / (float)T;
    auto cell = [&](int c) -> float {
        const int i = c >> 3, j = c & 7;
        const unsigned hij = flip ? h[i * 8 + (7 - j)] : h[i * 8 + j];
        const unsigned hji = flip ? h[j * 8 + (7 - i)] : h[j * 8 + i];
        return 0.5f * (float)(hij + hji) * inv;
    };
    float* row = out + (size_t)pl * width;
    if (pca)
    {
        for (int q = lane; q < ncomp; q += 32)
        {
            float acc = 0.0f;
            for (int c = 0; c < 64; ++c)
                acc += (cell(c) - pca[c]) * pca[64 + q * 64 + c];
            row[kScreenBase + q] = acc;
        }
    }
    else
        for (int c = lane; c < 64; c += 32)
            row[kScreenBase + c] = cell(c);
    if (lane != 0)
        return;

    double C[36];
    const double* c1 = s1 + 9;
    const double* c2 = s2 + 9;
    const double  A1[9] = {c1[0], c1[1], c1[2], c1[1], c1[3], c1[4], c1[2], c1[4], c1[5]};
    const double  A2[9] = {c2[0], c2[1], c2[2], c2[1], c2[3], c2[4], c2[2], c2[4], c2[5]};
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
        {
            C[r * 6 + c]           = A1[r * 3 + c];
            C[(r + 3) * 6 + c + 3] = A2[r * 3 + c];
            C[r * 6 + c + 3]       = cr[r * 3 + c] / T;
            C[(c + 3) * 6 + r]     = cr[r * 3 + c] / T;
        }
    double m1[9], m2[9], m6[36];
    for (int e = 0; e < 9; ++e)
    {
        m1[e] = A1[e];
        m2[e] = A2[e];
    }
    for (int e = 0; e < 36; ++e)
        m6[e] = C[e];
    const double d1 = det_lu(m1, 3), d2 = det_lu(m2, 3), d6 = det_lu(m6, 6);
    row[0] = (d1 > 0.0 && d2 > 0.0 && d6 > 0.0) ? (float)(0.5 * (log(d1) + log(d2) - log(d6))) : 0.0f;

    const double sd[6] = {s1[3], s1[4], s1[5], s2[3], s2[4], s2[5]};
    double       R[36];
    for (int r = 0; r < 6; ++r)
        for (int c = 0; c < 6; ++c)
            R[r * 6 + c] = (sd[r] > 0.0 && sd[c] > 0.0) ? C[r * 6 + c] / (sd[r] * sd[c]) : (r == c ? 1.0 : 0.0);
    double cc[9];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            cc[r * 3 + c] = fabs(R[r * 6 + c + 3]);
    double ev[6];
    jacobi_sym(R, 6, ev, nullptr);
    for (int e = 0; e < 6; ++e)
        row[1 + e] = (float)ev[e];

    double k1[3] = {s1[6], s1[7], s1[8]}, k2[3] = {s2[6], s2[7], s2[8]};
    sort_desc(k1, 3);
    sort_desc(k2, 3);
    const bool swap = k2[0] > k1[0];
    for (int d = 0; d < 3; ++d)
    {
        row[7 + d]  = (float)(swap ? k2[d] : k1[d]);
        row[10 + d] = (float)(swap ? k1[d] : k2[d]);
    }
    sort_desc(cc, 9);
    for (int e = 0; e < 9; ++e)
        row[13 + e] = (float)cc[e];
    row[22] = (float)K / (float)T;
}

cudaError_t launch_screen_features(const double* xyz, int natoms, int T, int K, long pair_begin, long pair_count,
                                   const int2* pair_ab, const float* pca, int ncomp, double* stats,
                                   unsigned char* bins, float* out, int width, cudaStream_t s)
{
    int P = 256;
    while (P < T)
        P <<= 1;
    const size_t smem = (size_t)P * 8;
    cudaError_t  e    = cudaFuncSetAttribute(screen_atom_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess)
        return e;
    screen_atom_kernel<<<natoms, 256, smem, s>>>(xyz, T, P, stats, bins);
    if (pair_count > 0)
        screen_pair_kernel<<<(unsigned)((pair_count + 7) / 8), 256, 0, s>>>(xyz, T, K, stats, bins, pair_begin,
                                                                           pair_count, pair_ab, pca, ncomp, out, width);
    return cudaGetLastError();
}

} // namespace gc
