// KSG pair MI without any device allocation, for callers that cannot call
// cudaMalloc: for example a plugin inside a host application that owns all
// device memory through its own pool and forbids allocations from library
// code, or a caller on a latency-critical path where an allocation (and the
// implicit device synchronisation cudaFree brings) is not acceptable.
//
// The exact FP64 KSG pipeline (the same kernels as gc_ksg_matrix's exact
// path: normalisation, neighbour statistics, frame-ordered MI reduction)
// runs with every piece of scratch memory taken from one fixed array,
// g_noalloc_scratch, that lives for the life of the process on every device
// that loads this library.  The caller passes device pointers for the
// coordinates and the pair MI output.
//
// Limits: natoms <= 64, nframes <= 1024 (larger calls are rejected with
// GC_ERR_INVALID); the array is ~9.8 MB.
//
// Host code must not use the array's name as a device address: the name is
// a host-side stand-in.  Its device address is looked up with
// cudaGetSymbolAddress once per device (with that device current) on the
// first call made on that device; that first call should therefore come
// before any stream capture.  Under CUDA's lazy module loading that first
// call is also what reserves the array on the device (it loads this file's
// module), so it can fail for lack of memory where later calls cannot; an
// application that hands all device memory to its own pool makes one
// warm-up call first.  A cudaDeviceReset leaves the looked-up address stale.
//
// Every call shares the one array, which keeps the previous call's
// contents; the status word is cleared on each call and every other region
// is fully rewritten before it is read.  Calls whose work overlaps on the
// GPU (other threads, other streams) race on the array.

#include "gmx_corr_b200.h"
#include "gc_geom.h"
#include "gc_internal.h"

#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>

namespace {

constexpr int kNoAllocMaxAtoms  = 64;
constexpr int kNoAllocMaxFrames = 1024;
constexpr long kMaxPairs        = (long)kNoAllocMaxAtoms * (kNoAllocMaxAtoms - 1) / 2;

// Byte layout of the scratch array (each region 256-byte aligned).
constexpr size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }
constexpr size_t kOffX      = 0;                                                       // double [3*64][1024]
constexpr size_t kOffCnt    = kOffX + align256(sizeof(double) * 3 * kNoAllocMaxAtoms * kNoAllocMaxFrames);
constexpr size_t kOffPsi    = kOffCnt + align256(sizeof(uint32_t) * kMaxPairs * kNoAllocMaxFrames);
constexpr size_t kOffStatus = kOffPsi + align256(sizeof(double) * (kNoAllocMaxFrames + 1));
constexpr size_t kScratchBytes = kOffStatus + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex    g_setup_mutex;
void*         g_scratch_addr[kMaxDevices] = {};

// psi[0] = 0, psi[1] = -0.57721566490153, psi[n+1] = psi[n] + 1/n, in the
// reference's sequential order (lib/kraskov.cpp:2217-2219).
__global__ void noalloc_psi_kernel(double* psi, int N)
{
    if (blockIdx.x != 0 || threadIdx.x != 0)
        return;
    psi[0] = 0.0;
    psi[1] = -0.57721566490153;
    for (int n = 1; n < N; ++n)
        psi[n + 1] = __dadd_rn(psi[n], __ddiv_rn(1.0, (double)n));
}

// Records `msg` as the calling thread's gc_last_error() text and returns st.
gc_status noalloc_fail(gc_status st, const std::string& msg)
{
    gc::set_last_error(msg.c_str());
    return st;
}

} // namespace

extern "C" gc_status gc_ksg_pair_mi_noalloc(const double* d_xyz, int natoms, int nframes, int k, double* d_pair_mi,
                                            void* stream)
{
    if (!d_xyz || !d_pair_mi)
    {
        return noalloc_fail(GC_ERR_INVALID, "gc_ksg_pair_mi_noalloc: null device pointer");
    }
    if (natoms < 2 || k < 1 || nframes <= k)
    {
        return noalloc_fail(GC_ERR_INVALID, "gc_ksg_pair_mi_noalloc: need natoms >= 2, k >= 1 and nframes > k");
    }
    if (natoms > kNoAllocMaxAtoms || nframes > kNoAllocMaxFrames)
    {
        return noalloc_fail(GC_ERR_INVALID,
                            "gc_ksg_pair_mi_noalloc: limited to " + std::to_string(kNoAllocMaxAtoms) + " atoms and " +
                                std::to_string(kNoAllocMaxFrames) + " frames (got " + std::to_string(natoms) + " x " +
                                std::to_string(nframes) + "); use gc_ksg_matrix or a gc_ksg_plan for larger trajectories");
    }
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    {
        cudaGetLastError();
        return noalloc_fail(GC_ERR_NO_DEVICE, "gc_ksg_pair_mi_noalloc: no usable current CUDA device");
    }
    void* base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_scratch_addr[dev])
        {
            void*             addr = nullptr;
            const cudaError_t e    = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
            if (e != cudaSuccess || !addr)
            {
                cudaGetLastError();
                return noalloc_fail(GC_ERR_CUDA, std::string("gc_ksg_pair_mi_noalloc: cudaGetSymbolAddress failed: ") +
                                                     cudaGetErrorString(e));
            }
            g_scratch_addr[dev] = addr;
        }
        base = g_scratch_addr[dev];
    }
    unsigned char* b      = static_cast<unsigned char*>(base);
    double*        X      = reinterpret_cast<double*>(b + kOffX);
    uint32_t*      cnt    = reinterpret_cast<uint32_t*>(b + kOffCnt);
    double*        psi    = reinterpret_cast<double*>(b + kOffPsi);
    int*           status = reinterpret_cast<int*>(b + kOffStatus);
    cudaStream_t   s      = static_cast<cudaStream_t>(stream);
    const long     npairs = (long)natoms * (natoms - 1) / 2;

    cudaError_t e = cudaMemsetAsync(status, 0, sizeof(int), s);
    if (e == cudaSuccess)
    {
        noalloc_psi_kernel<<<1, 1, 0, s>>>(psi, nframes);
        gc::launch_ksg_prepare(d_xyz, natoms, nframes, X, status, s);
        gc::launch_ksg_exact(X, nframes, k, 0, npairs, cnt, s);
        gc::launch_ksg_finalize(cnt, npairs, nframes, k, psi, d_pair_mi, s);
        e = cudaGetLastError();
    }
    int st = 0;
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&st, status, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
    {
        cudaGetLastError();
        return noalloc_fail(GC_ERR_CUDA, std::string("gc_ksg_pair_mi_noalloc: ") + cudaGetErrorString(e));
    }
    if (st & gc::kStatNonFinite)
        return noalloc_fail(GC_ERR_NONFINITE, "gc_ksg_pair_mi_noalloc: non-finite coordinate");
    if (st & gc::kStatZeroVariance)
        return noalloc_fail(GC_ERR_ZERO_VARIANCE, "gc_ksg_pair_mi_noalloc: a coordinate component has zero variance");
    return GC_OK;
}
