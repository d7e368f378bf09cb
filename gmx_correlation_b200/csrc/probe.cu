// Measurement support: the FP32 non-tensor rates that bound the KSG
// neighbour kernels, measured on the device in use.
//
//   mix: one FADD and one FMNMX per step (|q - c| then max), the instruction
//        pair of a max-norm distance; reported as lane-ops/s (each FADD or
//        FMNMX lane result counts one op, the unit of the 12-op
//        distance-eval).
//   fma: FFMA chains, reported as flop/s (2 per FFMA).
// Eight independent chains per thread hide latency; grid = 4 x SMs x 8 warps.

#include "gmx_corr_b200.h"
#include <cuda_runtime.h>

namespace {

__global__ void probe_mix_kernel(float* out, int iters, float c0, float c1)
{
    float v[8], q[8];
#pragma unroll
    for (int u = 0; u < 8; ++u)
    {
        v[u] = 0.0f;
        q[u] = (float)(threadIdx.x + u) * 1e-3f;
    }
    for (int it = 0; it < iters; ++it)
    {
#pragma unroll
        for (int u = 0; u < 8; ++u)
        {
            v[u] = fmaxf(v[u], fabsf(q[u] - c0));
            q[u] = fmaxf(q[u], fabsf(v[u] - c1));
        }
    }
    float s = 0.0f;
#pragma unroll
    for (int u = 0; u < 8; ++u)
        s += v[u] + q[u];
    if (s == 1234.5f)
        out[0] = s;
}

__global__ void probe_fma_kernel(float* out, int iters, float a, float b)
{
    float v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u)
        v[u] = (float)(threadIdx.x + u);
    for (int it = 0; it < iters; ++it)
    {
#pragma unroll
        for (int u = 0; u < 8; ++u)
            v[u] = fmaf(v[u], a, b);
    }
    float s = 0.0f;
#pragma unroll
    for (int u = 0; u < 8; ++u)
        s += v[u];
    if (s == 1234.5f)
        out[0] = s;
}

} // namespace

extern "C" gc_status gc_probe_fp32(int device, double* mix_ops_per_s, double* fma_flops_per_s)
{
    int prev = 0;
    if (cudaGetDevice(&prev) != cudaSuccess)
        return GC_ERR_NO_DEVICE;
    if (device >= 0 && cudaSetDevice(device) != cudaSuccess)
        return GC_ERR_CUDA;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    float* d = nullptr;
    if (cudaMalloc(&d, sizeof(float)) != cudaSuccess)
        return GC_ERR_OUT_OF_MEMORY;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int  blocks = sms * 4, threads = 256, iters = 1 << 14;
    double     best_mix = 0.0, best_fma = 0.0;
    for (int rep = 0; rep < 4; ++rep)
    {
        float ms = 0.0f;
        cudaEventRecord(e0);
        probe_mix_kernel<<<blocks, threads>>>(d, iters, 0.5f, 0.25f);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&ms, e0, e1);
        // 2 chains-steps x 2 ops x 8 lanes-chains per iteration per thread
        const double ops = (double)blocks * threads * iters * 8 * 4;
        if (rep > 0 && ms > 0)
            best_mix = ops / (ms * 1e-3) > best_mix ? ops / (ms * 1e-3) : best_mix;
        cudaEventRecord(e0);
        probe_fma_kernel<<<blocks, threads>>>(d, iters * 2, 1.0000001f, 1e-7f);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&ms, e0, e1);
        const double flops = (double)blocks * threads * iters * 2 * 8 * 2;
        if (rep > 0 && ms > 0)
            best_fma = flops / (ms * 1e-3) > best_fma ? flops / (ms * 1e-3) : best_fma;
    }
    const cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d);
    cudaSetDevice(prev);
    if (err != cudaSuccess)
        return GC_ERR_CUDA;
    if (mix_ops_per_s)
        *mix_ops_per_s = best_mix;
    if (fma_flops_per_s)
        *fma_flops_per_s = best_fma;
    return GC_OK;
}
