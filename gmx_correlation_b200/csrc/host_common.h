// Host-side helpers shared by the C-ABI translation units: error text,
// CUDA-call checks, device and stream scopes, owned device buffers, trajectory
// upload and the reference's digamma table.  Not part of the public ABI.
#pragma once

#include "gmx_corr_b200.h"
#include "gc_internal.h"

#include <cuda_runtime.h>

#include <string>
#include <vector>

namespace gc {
namespace host {

inline gc_status fail(gc_status st, const std::string& msg)
{
    gc::set_last_error(msg.c_str());
    return st;
}

#define GC_TRY_CUDA(call)                                                                            \
    do                                                                                               \
    {                                                                                                \
        cudaError_t e_ = (call);                                                                     \
        if (e_ != cudaSuccess)                                                                       \
        {                                                                                            \
            cudaGetLastError(); /* a non-sticky error must not resurface in the next call */         \
            return fail(e_ == cudaErrorMemoryAllocation ? GC_ERR_OUT_OF_MEMORY : GC_ERR_CUDA,         \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                          \
        }                                                                                            \
    } while (0)

#define GC_TRY(expr)                                                                                 \
    do                                                                                               \
    {                                                                                                \
        gc_status s_ = (expr);                                                                       \
        if (s_ != GC_OK)                                                                             \
            return s_;                                                                               \
    } while (0)

// Switches to the requested device for the lifetime of the guard.
struct DeviceScope
{
    int       prev = -1;
    gc_status st   = GC_OK;
    explicit DeviceScope(int dev)
    {
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0)
        {
            cudaGetLastError();
            st = fail(GC_ERR_NO_DEVICE, "no CUDA device available (this build has no CPU path)");
            return;
        }
        cudaGetDevice(&prev);
        if (dev >= 0)
        {
            if (dev >= n)
            {
                st = fail(GC_ERR_INVALID, "device ordinal out of range");
                return;
            }
            if (cudaSetDevice(dev) != cudaSuccess)
                st = fail(GC_ERR_CUDA, "cudaSetDevice failed");
        }
    }
    ~DeviceScope()
    {
        if (prev >= 0)
            cudaSetDevice(prev);
    }
};

template <class T>
struct DevBuf
{
    T*     p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { reset(); }
    void reset()
    {
        if (p)
            cudaFree(p);
        p = nullptr;
        n = 0;
    }
    gc_status alloc(size_t count)
    {
        reset();
        if (count == 0)
            count = 1;
        cudaError_t e = cudaMalloc(&p, count * sizeof(T));
        if (e != cudaSuccess)
        {
            cudaGetLastError();
            p = nullptr;
            return fail(e == cudaErrorMemoryAllocation ? GC_ERR_OUT_OF_MEMORY : GC_ERR_CUDA,
                        std::string("cudaMalloc: ") + cudaGetErrorString(e));
        }
        n = count;
        return GC_OK;
    }
};

// Per-device pool of large device blocks (exact-size reuse): plans of the
// same shape created one after another reuse the blocks instead of calling
// cudaMalloc / cudaFree.  pool_release frees every pooled block.
// The smallest pooled block of at least `bytes` and at most 1.25 x `bytes`
// (its size in *got), or nullptr.
void*  pool_take(size_t bytes, size_t* got);
void   pool_give(void* p, size_t bytes);   // keeps the block (or frees it when the pool is full)
// Size of a fresh block for `bytes`: above 2 MiB rounded up to an eighth of
// its power of two, so blocks of similar requests can be reused; below, to
// 256 bytes.
size_t pool_round(size_t bytes);
void  pool_release();

// DevBuf whose blocks come from and return to the pool.
template <class T>
struct PoolBuf
{
    T*     p   = nullptr;
    size_t n   = 0;
    size_t cap = 0; // bytes of the block
    PoolBuf() = default;
    PoolBuf(const PoolBuf&) = delete;
    PoolBuf& operator=(const PoolBuf&) = delete;
    ~PoolBuf() { reset(); }
    void reset()
    {
        if (p)
            pool_give(p, cap);
        p   = nullptr;
        n   = 0;
        cap = 0;
    }
    gc_status alloc(size_t count)
    {
        reset();
        if (count == 0)
            count = 1;
        size_t got = 0;
        void*  q   = pool_take(count * sizeof(T), &got);
        if (!q)
        {
            got           = pool_round(count * sizeof(T));
            cudaError_t e = cudaMalloc(&q, got);
            if (e == cudaErrorMemoryAllocation)
            {
                cudaGetLastError();
                pool_release(); // free what the pool holds and try once more
                e = cudaMalloc(&q, got);
            }
            if (e != cudaSuccess)
            {
                cudaGetLastError();
                return fail(e == cudaErrorMemoryAllocation ? GC_ERR_OUT_OF_MEMORY : GC_ERR_CUDA,
                            std::string("cudaMalloc: ") + cudaGetErrorString(e));
            }
        }
        p   = static_cast<T*>(q);
        n   = count;
        cap = got;
        return GC_OK;
    }
};

inline gc_opts defaults()
{
    gc_opts o;
    gc_opts_init(&o);
    return o;
}

// digamma table of kraskov_prepare (lib/kraskov.cpp:2217-2219) and
// digamma_table (lib/transfer_entropy.cpp:41-48): psi[0] = 0,
// psi[1] = -0.57721566490153, psi[n+1] = psi[n] + 1/n.
inline std::vector<double> digamma_table(int N)
{
    std::vector<double> psi((size_t)N + 1, 0.0);
    if (N >= 1)
        psi[1] = -0.57721566490153;
    for (int n = 1; n < N; ++n)
        psi[n + 1] = psi[n] + 1 / (1.0 * n);
    return psi;
}

inline gc_status check_view(const gc_traj_view* v)
{
    if (!v)
        return fail(GC_ERR_INVALID, "null trajectory view");
    if ((v->xyz == nullptr) == (v->rows == nullptr))
        return fail(GC_ERR_INVALID, "trajectory view needs exactly one of xyz / rows");
    if (v->natoms < 0 || v->nframes < 0)
        return fail(GC_ERR_INVALID, "negative trajectory size");
    if (v->rows)
        for (int a = 0; a < v->natoms; ++a)
            if (!v->rows[a])
                return fail(GC_ERR_INVALID, "null atom row in trajectory view");
    return GC_OK;
}

// Uploads the view's coordinates into a contiguous device block.
inline gc_status upload_traj(const gc_traj_view* v, double* d_xyz, cudaStream_t s)
{
    const size_t row = (size_t)v->nframes * 3;
    if (v->xyz)
    {
        GC_TRY_CUDA(cudaMemcpyAsync(d_xyz, v->xyz, sizeof(double) * row * v->natoms, cudaMemcpyHostToDevice, s));
    }
    else
    {
        for (int a = 0; a < v->natoms; ++a)
            GC_TRY_CUDA(cudaMemcpyAsync(d_xyz + row * a, v->rows[a], sizeof(double) * row, cudaMemcpyHostToDevice, s));
    }
    return GC_OK;
}

inline gc_status status_to_error(int st)
{
    if (st & gc::kStatNonFinite)
        return fail(GC_ERR_NONFINITE, "non-finite coordinate in the trajectory");
    if (st & gc::kStatZeroVariance)
        return fail(GC_ERR_ZERO_VARIANCE,
                    "a coordinate component has zero variance over the frames (the reference divides by it)");
    if (st & gc::kStatTimeout)
        return fail(GC_ERR_TIMEOUT, "a bounded device wait ran out");
    if (st & gc::kStatInternal)
        return fail(GC_ERR_INTERNAL, "device-side consistency check failed");
    return GC_OK;
}

struct StreamScope
{
    cudaStream_t s     = nullptr;
    bool         owned = false;
    gc_status    init(void* user)
    {
        if (user)
        {
            s = (cudaStream_t)user;
            return GC_OK;
        }
        GC_TRY_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        owned = true;
        return GC_OK;
    }
    ~StreamScope()
    {
        if (owned && s)
            cudaStreamDestroy(s);
    }
};

} // namespace host
} // namespace gc
