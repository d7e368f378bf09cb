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
                    uint2* __restrict__ cnt)
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
    const double* __restrict__ A0 = XT + (size_t)(a1 * 3 + 0) * T;
    const double* __restrict__ A1 = XT + (size_t)(a1 * 3 + 1) * T;
    const double* __restrict__ A2 = XT + (size_t)(a1 * 3 + 2) * T;
    const double* __restrict__ B0 = XT + (size_t)(a2 * 3 + 0) * T;
    const double* __restrict__ B1 = XT + (size_t)(a2 * 3 + 1) * T;
    const double* __restrict__ B2 = XT + (size_t)(a2 * 3 + 2) * T;
    const int Nv = T - lag;
    const int i0 = qb * kTeQBlock, i1 = min(Nv, i0 + kTeQBlock);
    unsigned* h  = hist[warp];

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
        auto key = [&](int j, unsigned long long& k) -> bool {
            if (j == qi)
                return false;
            double a, b, c;
            sub(j, a, b, c);
            k = dbits(fmax(fmax(a, b), c));
            return true;
        };
        int          below;
        const double eps = __longlong_as_double((long long)warp_select_u64(key, Nv, K, 56, h, lane, &below));
        int nxfxp = 0, nypxp = 0, nxp = 0;
        for (int j = lane; j < Nv; j += 32)
        {
            if (j == qi)
                continue;
            double a, b, c;
            sub(j, a, b, c);
            nxfxp += fmax(a, b) < eps;
            nypxp += fmax(b, c) < eps;
            nxp += b < eps;
        }
        nxfxp = __reduce_add_sync(kFull, nxfxp);
        nypxp = __reduce_add_sync(kFull, nypxp);
        nxp   = __reduce_add_sync(kFull, nxp);
        if (lane == 0)
            cnt[(size_t)qi * npairs + q] = make_uint2((unsigned)nxp | ((unsigned)nxfxp << 16), (unsigned)nypxp);
    }
}

// te_sum += psi_k + psi[n_xp+1] - psi[n_xfxp+1] - psi[n_ypxp+1] over qi in
// order, then te_sum / N_valid (lib/transfer_entropy.cpp:195-204).
__global__ void te_finalize_kernel(const uint2* __restrict__ cnt, int natoms, int T, int K, int lag,
                                   const double* __restrict__ psi, double* __restrict__ te_mat)
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

void launch_te_exact(const double* XT, int natoms, int T, int K, int lag, uint2* cnt, cudaStream_t s)
{
    const int  Nv     = T - lag;
    const int  nqb    = (Nv + kTeQBlock - 1) / kTeQBlock;
    const long npairs = (long)natoms * (natoms - 1);
    te_exact_kernel<<<(unsigned)(npairs * nqb), kTeWarps * 32, 0, s>>>(XT, natoms, T, K, lag, nqb, cnt);
}

void launch_te_finalize(const uint2* cnt, int natoms, int T, int K, int lag, const double* psi, double* te_mat,
                        cudaStream_t s)
{
    const long npairs = (long)natoms * (natoms - 1);
    te_finalize_kernel<<<(unsigned)((npairs + 127) / 128), 128, 0, s>>>(cnt, natoms, T, K, lag, psi, te_mat);
}

} // namespace gc
