// Transfer entropy (Frenzel-Pompe conditional MI) on B200.
//
// Reference: te_matrix, lib/transfer_entropy.cpp:63-221.  For an ordered
// pair (a1, a2) and query qi < N_valid = T - lag the 9-D vector is
// [x_a1(qi+lag), x_a1(qi), x_a2(qi)] on the raw mean-centred coordinates;
// eps is the k-th smallest max-norm distance over j != qi, j < N_valid, and
// the three subspace counts use a strict `<` eps.  Only the value of eps
// enters (never the neighbour identities), so no tie rule is needed.  The
// per-query counts are stored and reduced in query order by
// te_finalize_kernel, reproducing the reference's te_sum exactly.

#include "gc_common.cuh"
#include "gc_internal.h"
#include "te_exact_query.cuh"

namespace gc {

__global__ void transpose_components_kernel(const double* __restrict__ xyz, int natoms, int T,
                                            double* __restrict__ XT, int* __restrict__ status)
{
    const long n   = (long)natoms * T * 3;
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < n; idx += (long)gridDim.x * blockDim.x)
    {
        const long   a = idx / ((long)T * 3);
        const long   r = idx - a * (long)T * 3;
        const int    f = (int)(r / 3), d = (int)(r - (r / 3) * 3);
        const double v = xyz[idx];
        if (!isfinite(v))
            atomicOr(status, kStatNonFinite);
        XT[(size_t)(a * 3 + d) * T + f] = v;
    }
}

namespace {
constexpr int kTeWarps  = 8;
constexpr int kTeQBlock = 64;
} // namespace

__global__ void __launch_bounds__(kTeWarps * 32)
    te_exact_kernel(const double* __restrict__ XT, int natoms, int T, int K, int lag, int nqb,
                    uint2* __restrict__ cnt, bool wide)
{
    __shared__ unsigned hist[kTeWarps][256];
    const int  warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long npairs = (long)natoms * (natoms - 1);
    const long q      = blockIdx.x / nqb;
    const int  qb     = (int)(blockIdx.x - q * nqb);
    if (q >= npairs)
        return;
    const int a1 = (int)(q / (natoms - 1));
    const int rr = (int)(q - (long)a1 * (natoms - 1));
    const int a2 = rr < a1 ? rr : rr + 1;
    const int Nv = T - lag;
    const int i0 = qb * kTeQBlock, i1 = min(Nv, i0 + kTeQBlock);
#pragma unroll 1
    for (int qi = i0 + warp; qi < i1; qi += kTeWarps)
    {
        int xp, xf, yp;
        te_exact_query_n(XT, T, K, lag, a1, a2, qi, hist[warp], lane, xp, xf, yp);
        if (lane == 0)
        {
            if (wide)
            {
                cnt[(size_t)qi * npairs + q]        = make_uint2((unsigned)xp, (unsigned)xf);
                cnt[(size_t)(Nv + qi) * npairs + q] = make_uint2((unsigned)yp, 0u);
            }
            else
                cnt[(size_t)qi * npairs + q] = make_uint2((unsigned)xp | ((unsigned)xf << 16), (unsigned)yp);
        }
    }
}

// FP32 copy of the raw coordinates for the fast TE kernel: x32 =
// fl32(x64 - c), c the component midrange, and a per-atom bound eps_a =
// 2^-21 R_a (R_a the largest half-range of its components), so every FP32
// marginal max-norm distance is within eps_a of the FP64 one:
// |fl32(x32_i - x32_j) - fl64(x64_i - x64_j)| <= 4 u R (1 + 2^-20), u = 2^-24.
__global__ void te_x32_kernel(const double* __restrict__ XT, int natoms, int T, float4* __restrict__ X32,
                              float* __restrict__ eps_atom)
{
    const int lane = threadIdx.x & 31;
    const int a    = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (a >= natoms)
        return;
    const double* r = XT + (size_t)a * 3 * T;
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

namespace {
__device__ __forceinline__ float te_d3(const float4 a, const float4 b)
{
    return fmaxf(fmaxf(fabsf(a.x - b.x), fabsf(a.y - b.y)), fabsf(a.z - b.z));
}
} // namespace

// The same statistics as te_exact_kernel from FP32 distances with an exact
// FP64 repair.  eps: the k-th smallest FP32 9-D distance d32 is selected;
// the FP64 k-th distance lies within e = max(eps_a1, eps_a2) of it, so the
// frames with FP32 distance below d32 - 2e are certainly nearer, those above
// d32 + 2e certainly farther, and the FP64 eps is the right order statistic
// of the (few) frames in between, evaluated in FP64.  Counts: an FP32
// subspace distance below eps - e (above eps + e) is certainly (not) below
// eps; the rest are compared in FP64.  More than 32 frames in the band
// (exact ties) fall back to the FP64 selection.  The counts equal the exact
// kernel's.
__global__ void __launch_bounds__(kTeWarps * 32)
    te_fast_kernel(const double* __restrict__ XT, const float4* __restrict__ X32, const float* __restrict__ eps_atom,
                   int natoms, int T, int K, int lag, int nqb, uint2* __restrict__ cnt)
{
    __shared__ unsigned hist[kTeWarps][256];
    __shared__ int      amb[kTeWarps][32];
    const int  warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long npairs = (long)natoms * (natoms - 1);
    const long q      = blockIdx.x / nqb;
    const int  qb     = (int)(blockIdx.x - q * nqb);
    if (q >= npairs)
        return;
    const int a1 = (int)(q / (natoms - 1));
    const int rr = (int)(q - (long)a1 * (natoms - 1));
    const int a2 = rr < a1 ? rr : rr + 1;
    const double* __restrict__ A0 = XT + (size_t)(a1 * 3 + 0) * T;
    const double* __restrict__ A1 = XT + (size_t)(a1 * 3 + 1) * T;
    const double* __restrict__ A2 = XT + (size_t)(a1 * 3 + 2) * T;
    const double* __restrict__ B0 = XT + (size_t)(a2 * 3 + 0) * T;
    const double* __restrict__ B1 = XT + (size_t)(a2 * 3 + 1) * T;
    const double* __restrict__ B2 = XT + (size_t)(a2 * 3 + 2) * T;
    const float4* __restrict__ A = X32 + (size_t)a1 * T;
    const float4* __restrict__ Bq = X32 + (size_t)a2 * T;
    const float e1 = eps_atom[a1], e = fmaxf(e1, eps_atom[a2]);
    const int   Nv = T - lag;
    const int   i0 = qb * kTeQBlock, i1 = min(Nv, i0 + kTeQBlock);
    unsigned*   h  = hist[warp];
    const unsigned lt = (1u << lane) - 1u;

#pragma unroll 1
    for (int qi = i0 + warp; qi < i1; qi += kTeWarps)
    {
        const double f0 = A0[qi + lag], f1 = A1[qi + lag], f2 = A2[qi + lag];
        const double p0 = A0[qi], p1 = A1[qi], p2 = A2[qi];
        const double y0 = B0[qi], y1 = B1[qi], y2 = B2[qi];
        auto sub = [&](int j, double& dfut, double& dpast, double& dy) {
            dfut  = fmax(fmax(fabs(f0 - A0[j + lag]), fabs(f1 - A1[j + lag])), fabs(f2 - A2[j + lag]));
            dpast = fmax(fmax(fabs(p0 - A0[j]), fabs(p1 - A1[j])), fabs(p2 - A2[j]));
            dy    = fmax(fmax(fabs(y0 - B0[j]), fabs(y1 - B1[j])), fabs(y2 - B2[j]));
        };
        const float4 fq = A[qi + lag], pq = A[qi], yq = Bq[qi];
        auto d32 = [&](int j) { return fmaxf(fmaxf(te_d3(fq, A[j + lag]), te_d3(pq, A[j])), te_d3(yq, Bq[j])); };
        auto key32 = [&](int j, unsigned long long& kv) -> bool {
            if (j == qi)
                return false;
            kv = __float_as_uint(d32(j));
            return true;
        };
        int         below;
        const float dk = __uint_as_float((unsigned)warp_select_u64(key32, Nv, K, 24, h, lane, &below));
        const float two_e = __fmul_ru(2.0f, e);
        const float lo = __fsub_rd(dk, two_e), hi = __fadd_ru(dk, two_e);
        // frames certainly nearer, and the band in between
        int nbelow = 0, namb = 0;
        for (int j0 = 0; j0 < Nv; j0 += 32)
        {
            const int j     = j0 + lane;
            bool      inamb = false;
            if (j < Nv && j != qi)
            {
                const float D = d32(j);
                nbelow += D < lo;
                inamb = D >= lo && D <= hi;
            }
            const unsigned m = __ballot_sync(kFull, inamb);
            const int      pos = namb + __popc(m & lt);
            if (inamb && pos < 32)
                amb[warp][pos] = j;
            namb += __popc(m);
        }
        nbelow = __reduce_add_sync(kFull, nbelow);
        __syncwarp();
        double eps   = 0.0;
        bool   exact = namb > 32;
        if (!exact)
        {
            double v = __longlong_as_double(0x7FF0000000000000ll);
            if (lane < namb)
            {
                double a, b, c;
                sub(amb[warp][lane], a, b, c);
                v = fmax(fmax(a, b), c);
            }
            int rank = 0;
            for (int m = 0; m < 32; ++m)
            {
                const double w = __shfl_sync(kFull, v, m);
                rank += w < v || (w == v && m < lane);
            }
            const int      need = K - nbelow;
            const unsigned sel  = __ballot_sync(kFull, lane < namb && rank == need - 1);
            if (need < 1 || need > namb || !sel)
                exact = true;
            else
                eps = __shfl_sync(kFull, v, __ffs(sel) - 1);
        }
        if (exact)
        {
            auto key = [&](int j, unsigned long long& kv) -> bool {
                if (j == qi)
                    return false;
                double a, b, c;
                sub(j, a, b, c);
                kv = dbits(fmax(fmax(a, b), c));
                return true;
            };
            int b2;
            eps = __longlong_as_double((long long)warp_select_u64(key, Nv, K, 56, h, lane, &b2));
        }
        // strict counts, FP32 first
        const float p_lo = __double2float_rd(__dsub_rd(eps, (double)e1));
        const float p_hi = __double2float_ru(__dadd_ru(eps, (double)e1));
        const float y_lo = __double2float_rd(__dsub_rd(eps, (double)e));
        const float y_hi = __double2float_ru(__dadd_ru(eps, (double)e));
        int nxfxp = 0, nypxp = 0, nxp = 0;
        for (int j = lane; j < Nv; j += 32)
        {
            if (j == qi)
                continue;
            const float F = te_d3(fq, A[j + lag]), P = te_d3(pq, A[j]), Y = te_d3(yq, Bq[j]);
            const float FP = fmaxf(F, P), YP = fmaxf(Y, P);
            const bool  uxp = P >= p_lo && P <= p_hi, ufp = FP >= p_lo && FP <= p_hi, uyp = YP >= y_lo && YP <= y_hi;
            if (uxp || ufp || uyp)
            {
                double a, b, c;
                sub(j, a, b, c);
                nxp += b < eps;
                nxfxp += fmax(a, b) < eps;
                nypxp += fmax(b, c) < eps;
            }
            else
            {
                nxp += P < p_lo;
                nxfxp += FP < p_lo;
                nypxp += YP < y_lo;
            }
        }
        nxfxp = __reduce_add_sync(kFull, nxfxp);
        nypxp = __reduce_add_sync(kFull, nypxp);
        nxp   = __reduce_add_sync(kFull, nxp);
        if (lane == 0)
            cnt[(size_t)qi * npairs + q] = make_uint2((unsigned)nxp | ((unsigned)nxfxp << 16), (unsigned)nypxp);
        __syncwarp(); // amb[warp] is rewritten for the next query
    }
}

// te_sum += psi_k + psi[n_xp+1] - psi[n_xfxp+1] - psi[n_ypxp+1] over qi in
// order, then te_sum / N_valid (lib/transfer_entropy.cpp:195-204).
__global__ void te_finalize_kernel(const uint2* __restrict__ cnt, int natoms, int T, int K, int lag,
                                   const double* __restrict__ psi, double* __restrict__ te_mat, bool wide)
{
    const long npairs = (long)natoms * (natoms - 1);
    const long q      = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (q >= npairs)
        return;
    const int Nv  = T - lag;
    double    sum = 0.0;
    for (int qi = 0; qi < Nv; ++qi)
    {
        const uint2 c   = cnt[(size_t)qi * npairs + q];
        if (wide)
        {
            const int    xp = min((int)c.x, Nv), xf = min((int)c.y, Nv);
            const int    yp = min((int)cnt[(size_t)(Nv + qi) * npairs + q].x, Nv);
            const double t  = __dsub_rn(__dsub_rn(__dadd_rn(psi[K], psi[xp + 1]), psi[xf + 1]), psi[yp + 1]);
            sum             = __dadd_rn(sum, t);
            continue;
        }
        const int   xp  = min((int)(c.x & 0xFFFFu), Nv);
        const int   xf  = min((int)(c.x >> 16), Nv);
        const int   yp  = min((int)c.y, Nv);
        const double t  = __dsub_rn(__dsub_rn(__dadd_rn(psi[K], psi[xp + 1]), psi[xf + 1]), psi[yp + 1]);
        sum             = __dadd_rn(sum, t);
    }
    const int a1 = (int)(q / (natoms - 1));
    const int rr = (int)(q - (long)a1 * (natoms - 1));
    const int a2 = rr < a1 ? rr : rr + 1;
    te_mat[(size_t)a1 * natoms + a2] = __ddiv_rn(sum, (double)Nv);
}

void launch_transpose_components(const double* xyz, int natoms, int T, double* XT, int* status, cudaStream_t s)
{
    transpose_components_kernel<<<1184, 256, 0, s>>>(xyz, natoms, T, XT, status);
}

void launch_te_exact(const double* XT, int natoms, int T, int K, int lag, uint2* cnt, cudaStream_t s, bool wide)
{
    const int  Nv     = T - lag;
    const int  nqb    = (Nv + kTeQBlock - 1) / kTeQBlock;
    const long npairs = (long)natoms * (natoms - 1);
    te_exact_kernel<<<(unsigned)(npairs * nqb), kTeWarps * 32, 0, s>>>(XT, natoms, T, K, lag, nqb, cnt, wide);
}

void launch_te_x32(const double* XT, int natoms, int T, float4* X32, float* eps_atom, cudaStream_t s)
{
    te_x32_kernel<<<(natoms * 32 + 255) / 256, 256, 0, s>>>(XT, natoms, T, X32, eps_atom);
}

void launch_te_fast(const double* XT, const float4* X32, const float* eps_atom, int natoms, int T, int K, int lag,
                    uint2* cnt, cudaStream_t s)
{
    const int  Nv     = T - lag;
    const int  nqb    = (Nv + kTeQBlock - 1) / kTeQBlock;
    const long npairs = (long)natoms * (natoms - 1);
    te_fast_kernel<<<(unsigned)(npairs * nqb), kTeWarps * 32, 0, s>>>(XT, X32, eps_atom, natoms, T, K, lag, nqb, cnt);
}

void launch_te_finalize(const uint2* cnt, int natoms, int T, int K, int lag, const double* psi, double* te_mat,
                        cudaStream_t s, bool wide)
{
    const long npairs = (long)natoms * (natoms - 1);
    te_finalize_kernel<<<(unsigned)((npairs + 127) / 128), 128, 0, s>>>(cnt, natoms, T, K, lag, psi, te_mat, wide);
}

} // namespace gc
