// Training and inference kernels of the learned KSG screen's networks (no
// counterpart in the reference).
//
// Every matrix product of the forward and backward passes goes through one
// batched tensor-core GEMM: operands are rounded to BF16 as they are staged
// into shared memory, products accumulate in FP32 (mma.sync m16n8k16), and
// the epilogue fuses the bias and GELU of the forward layers.  Ensemble
// members are the grid's z dimension.  The remaining steps of a training
// step (row gather with standardisation, loss gradient, GELU derivative,
// bias gradients, Adam) are small elementwise kernels, so one step is a
// fixed sequence of launches that the host captures once into a CUDA graph.

#include "gc_common.cuh"
#include "gc_internal.h"

#include <cuda_bf16.h>

namespace gc {

namespace {

constexpr int kBM = 64, kBN = 64, kBK = 32, kPad = 8;
constexpr int kGemmThreads = 128;

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }

__device__ __forceinline__ float gelu_grad(float z)
{
    return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * expf(-0.5f * z * z) * 0.39894228040143268f;
}

__device__ __forceinline__ void mma_bf16(float* c, const uint32_t* a, const uint32_t* b)
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};\n"
                 : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Stages a kBM x kBK tile of op(r, k) = P[r*sr + k*sk] (zero outside
// rows x K) into S[r][k] as BF16.  Threads run along whichever of r and k
// has unit stride, so the global reads coalesce.
__device__ __forceinline__ void stage_tile(__nv_bfloat16 (*S)[kBK + kPad], const float* __restrict__ P, long sr,
                                           long sk, int r0, int rows, int k0, int K)
{
    const bool k_fast = (sk == 1) || (sr != 1);
#pragma unroll 4
    for (int i = 0; i < (kBM * kBK) / kGemmThreads; ++i)
    {
        const int e = threadIdx.x + i * kGemmThreads;
        const int r = k_fast ? (e / kBK) : (e % kBM);
        const int c = k_fast ? (e % kBK) : (e / kBM);
        const int gr = r0 + r, gk = k0 + c;
        float     v  = 0.0f;
        if (gr < rows && gk < K)
            v = P[(long)gr * sr + (long)gk * sk];
        S[r][c] = __float2bfloat16_rn(v);
    }
}

__global__ void __launch_bounds__(kGemmThreads) mlp_gemm_kernel(MlpGemm g)
{
    __shared__ __align__(16) __nv_bfloat16 As[kBM][kBK + kPad];
    __shared__ __align__(16) __nv_bfloat16 Bs[kBN][kBK + kPad];
    const int   z = blockIdx.z, m0 = blockIdx.y * kBM, n0 = blockIdx.x * kBN;
    const int   warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int   wm = warp >> 1, wn = warp & 1, gq = lane >> 2, tq = lane & 3;
    const float* A = g.A + (long)z * g.sAz;
    const float* B = g.B + (long)z * g.sBz;

    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int q = 0; q < 4; ++q)
                acc[i][j][q] = 0.0f;

    for (int k0 = 0; k0 < g.K; k0 += kBK)
    {
        stage_tile(As, A, g.sAm, g.sAk, m0, g.M, k0, g.K);
        stage_tile(Bs, B, g.sBn, g.sBk, n0, g.N, k0, g.K);
        __syncthreads();
#pragma unroll
        for (int ks = 0; ks < kBK; ks += 16)
        {
            uint32_t af[2][4], bf[4][2];
#pragma unroll
            for (int mt = 0; mt < 2; ++mt)
            {
                const int r = wm * 32 + mt * 16 + gq;
                af[mt][0]   = *reinterpret_cast<const uint32_t*>(&As[r][ks + 2 * tq]);
                af[mt][1]   = *reinterpret_cast<const uint32_t*>(&As[r + 8][ks + 2 * tq]);
                af[mt][2]   = *reinterpret_cast<const uint32_t*>(&As[r][ks + 2 * tq + 8]);
                af[mt][3]   = *reinterpret_cast<const uint32_t*>(&As[r + 8][ks + 2 * tq + 8]);
            }
#pragma unroll
            for (int nt = 0; nt < 4; ++nt)
            {
                const int n = wn * 32 + nt * 8 + gq;
                bf[nt][0]   = *reinterpret_cast<const uint32_t*>(&Bs[n][ks + 2 * tq]);
                bf[nt][1]   = *reinterpret_cast<const uint32_t*>(&Bs[n][ks + 2 * tq + 8]);
            }
#pragma unroll
            for (int mt = 0; mt < 2; ++mt)
#pragma unroll
                for (int nt = 0; nt < 4; ++nt)
                    mma_bf16(acc[mt][nt], af[mt], bf[nt]);
        }
        __syncthreads();
    }

    float*       C    = g.C + (long)z * g.sCz;
    float*       H    = g.H ? g.H + (long)z * g.sCz : nullptr;
    const float* bias = g.bias ? g.bias + (long)z * g.sbz : nullptr;
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
#pragma unroll
            for (int q = 0; q < 4; ++q)
            {
                const int m = m0 + wm * 32 + mt * 16 + gq + (q >> 1) * 8;
                const int n = n0 + wn * 32 + nt * 8 + 2 * tq + (q & 1);
                if (m >= g.M || n >= g.N)
                    continue;
                float      v   = acc[mt][nt][q];
                const long off = (long)m * g.ldc + n;
                if (g.epi == kEpiStore)
                {
                    C[off] = g.accumulate ? C[off] + v : v;
                    continue;
                }
                v += bias[n];
                C[off] = v;
                if (g.epi == kEpiBiasGelu)
                    H[off] = gelu(v);
            }
}

__global__ void mlp_gather_kernel(const float* __restrict__ F, const long* __restrict__ idx, const int* step, int M,
                                  const float* __restrict__ mean, const float* __restrict__ sd, float* __restrict__ X)
{
    const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long)M * kScreenIn)
        return;
    const int  m = (int)(e / kScreenIn), c = (int)(e % kScreenIn);
    const long base = step ? (long)(*step) * M : 0;
    const long row  = idx ? idx[base + m] : base + m;
    X[e]            = (F[row * kScreenIn + c] - mean[c]) / sd[c];
}

__global__ void mlp_loss_kernel(const float* __restrict__ Y, const float* __restrict__ target,
                                const long* __restrict__ idx, const int* step, int M, int Z, float* __restrict__ dY,
                                float* __restrict__ loss)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x, z = blockIdx.y;
    float     l = 0.0f;
    if (m < M)
    {
        const long base = step ? (long)(*step) * M : 0;
        const long row  = idx ? idx[base + m] : base + m;
        const float d   = Y[(long)z * M + m] - target[row];
        dY[(long)z * M + m] = 2.0f * d / (float)M;
        l                   = d * d / (float)M;
    }
    for (int o = 16; o > 0; o >>= 1)
        l += __shfl_xor_sync(kFull, l, o);
    if ((threadIdx.x & 31) == 0)
        atomicAdd(loss + z, l);
}

__global__ void mlp_gelu_back_kernel(const float* __restrict__ Zpre, float* __restrict__ dH, long n)
{
    const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < n)
        dH[e] *= gelu_grad(Zpre[e]);
}

__global__ void mlp_colsum_kernel(const float* __restrict__ dZ, int M, int N, int Z, float* __restrict__ db, long sbz)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x, z = blockIdx.y;
    if (c >= N)
        return;
    const float* p = dZ + (long)z * M * N + c;
    float        s = 0.0f;
    for (int m = 0; m < M; ++m)
        s += p[(long)m * N];
    db[(long)z * sbz + c] = s;
}

__global__ void mlp_adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                                float* __restrict__ v, long n, const float* __restrict__ hyper, const int* tstep)
{
    const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n)
        return;
    const float lr = hyper[0], b1 = hyper[1], b2 = hyper[2], eps = hyper[3];
    const float t   = (float)(*tstep + 1);
    const float bc1 = 1.0f - powf(b1, t), bc2 = 1.0f - powf(b2, t);
    const float gr  = g[e];
    const float mm  = b1 * m[e] + (1.0f - b1) * gr;
    const float vv  = b2 * v[e] + (1.0f - b2) * gr * gr;
    m[e]            = mm;
    v[e]            = vv;
    p[e] -= lr * (mm / bc1) / (sqrtf(vv / bc2) + eps);
}

__global__ void mlp_tick_kernel(int* a, int* b)
{
    if (a)
        ++*a;
    if (b)
        ++*b;
}

__global__ void mlp_ensemble_kernel(const float* __restrict__ Y, long n, int Z, float* __restrict__ mean,
                                    float* __restrict__ sd)
{
    const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n)
        return;
    float s = 0.0f;
    for (int z = 0; z < Z; ++z)
        s += Y[(long)z * n + e];
    const float mu = s / (float)Z;
    float       q  = 0.0f;
    for (int z = 0; z < Z; ++z)
    {
        const float d = Y[(long)z * n + e] - mu;
        q += d * d;
    }
    mean[e] = mu;
    sd[e]   = sqrtf(q / (float)Z);
}

unsigned blocks_for(long n, int t) { return (unsigned)((n + t - 1) / t); }

} // namespace

cudaError_t launch_mlp_gemm(const MlpGemm& g, cudaStream_t s)
{
    if (g.M <= 0 || g.N <= 0 || g.Z <= 0)
        return cudaSuccess;
    const dim3 grid((unsigned)((g.N + kBN - 1) / kBN), (unsigned)((g.M + kBM - 1) / kBM), (unsigned)g.Z);
    mlp_gemm_kernel<<<grid, kGemmThreads, 0, s>>>(g);
    return cudaGetLastError();
}

cudaError_t launch_mlp_gather(const float* F, const long* idx, const int* step, int M, const float* mean,
                              const float* sd, float* X, cudaStream_t s)
{
    const long n = (long)M * kScreenIn;
    mlp_gather_kernel<<<blocks_for(n, 256), 256, 0, s>>>(F, idx, step, M, mean, sd, X);
    return cudaGetLastError();
}

cudaError_t launch_mlp_loss(const float* Y, const float* target, const long* idx, const int* step, int M, int Z,
                            float* dY, float* loss, cudaStream_t s)
{
    mlp_loss_kernel<<<dim3(blocks_for(M, 256), (unsigned)Z), 256, 0, s>>>(Y, target, idx, step, M, Z, dY, loss);
    return cudaGetLastError();
}

cudaError_t launch_mlp_gelu_back(const float* Zpre, float* dH, long n, cudaStream_t s)
{
    mlp_gelu_back_kernel<<<blocks_for(n, 256), 256, 0, s>>>(Zpre, dH, n);
    return cudaGetLastError();
}

cudaError_t launch_mlp_colsum(const float* dZ, int M, int N, int Z, float* db, long sbz, cudaStream_t s)
{
    mlp_colsum_kernel<<<dim3(blocks_for(N, 128), (unsigned)Z), 128, 0, s>>>(dZ, M, N, Z, db, sbz);
    return cudaGetLastError();
}

cudaError_t launch_mlp_adam(float* p, const float* g, float* m, float* v, long n, const float* hyper,
                            const int* tstep, cudaStream_t s)
{
    mlp_adam_kernel<<<blocks_for(n, 256), 256, 0, s>>>(p, g, m, v, n, hyper, tstep);
    return cudaGetLastError();
}

cudaError_t launch_mlp_tick(int* a, int* b, cudaStream_t s)
{
    mlp_tick_kernel<<<1, 1, 0, s>>>(a, b);
    return cudaGetLastError();
}

cudaError_t launch_mlp_ensemble(const float* Y, long n, int Z, float* mean, float* sd, cudaStream_t s)
{
    mlp_ensemble_kernel<<<blocks_for(n, 256), 256, 0, s>>>(Y, n, Z, mean, sd);
    return cudaGetLastError();
}

} // namespace gc
