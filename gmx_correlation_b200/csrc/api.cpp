// C ABI of gmx_correlation_b200 (declared in include/gmx_corr_b200.h).
//
// Host side of the all-pairs path: argument checks with the reference's
// messages, device selection, workspace plans, host<->device staging and
// matrix assembly.  Every estimator computes on the GPU; there is no CPU
// fallback (a missing device is an error).

#include "gmx_corr_b200.h"
#include "gc_internal.h"
#include "gc_geom.h"
#include "ksg_fast.h"
#include "host_common.h"
#include "ksg_host.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

namespace {

thread_local std::string g_last_error;

} // namespace

using namespace gc::host;

void gc::set_last_error(const char* msg) { g_last_error = msg ? msg : ""; }

namespace {

constexpr size_t kPoolCap = (size_t)48 << 30; // bytes a device's pool may hold

struct DevicePool
{
    std::multimap<size_t, void*> blocks;
    size_t                       bytes = 0;
};
// Never destroyed: blocks may still be returned while statics are torn down.
std::mutex& g_pool_mutex = *new std::mutex;
DevicePool* g_pool       = new DevicePool[64];

int current_device()
{
    int d = -1;
    if (cudaGetDevice(&d) != cudaSuccess)
    {
        cudaGetLastError();
        return -1;
    }
    return d < 64 ? d : -1;
}

} // namespace

size_t gc::host::pool_round(size_t bytes)
{
    if (bytes <= ((size_t)2 << 20))
        return (bytes + 255) & ~(size_t)255;
    size_t step = (size_t)2 << 20;
    while (step * 16 <= bytes)
        step <<= 1; // an eighth to a sixteenth of the size
    return (bytes + step - 1) / step * step;
}

void* gc::host::pool_take(size_t bytes, size_t* got)
{
    const int d = current_device();
    if (d < 0)
        return nullptr;
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    auto                        it = g_pool[d].blocks.lower_bound(bytes);
    if (it == g_pool[d].blocks.end() || it->first > bytes + bytes / 4)
        return nullptr;
    void* p = it->second;
    *got    = it->first;
    g_pool[d].bytes -= it->first;
    g_pool[d].blocks.erase(it);
    return p;
}

void gc::host::pool_give(void* p, size_t bytes)
{
    cudaPointerAttributes attr{};
    int                   d = -1;
    if (cudaPointerGetAttributes(&attr, p) == cudaSuccess)
        d = attr.device;
    else
        cudaGetLastError();
    // A full pool gives up its largest blocks for the newest one, so it holds
    // the sizes in current use (a workload after a much larger one would
    // otherwise allocate and free every block of every call).
    std::vector<void*> evicted;
    bool               kept = false;
    {
        std::lock_guard<std::mutex> lock(g_pool_mutex);
        if (d >= 0 && d < 64 && bytes <= kPoolCap)
        {
            DevicePool& pool = g_pool[d];
            while (pool.bytes + bytes > kPoolCap && !pool.blocks.empty())
            {
                auto big = std::prev(pool.blocks.end());
                pool.bytes -= big->first;
                evicted.push_back(big->second);
                pool.blocks.erase(big);
            }
            pool.blocks.emplace(bytes, p);
            pool.bytes += bytes;
            kept = true;
        }
    }
    for (void* q : evicted)
        cudaFree(q);
    if (!kept)
        cudaFree(p);
}

void gc::host::pool_release()
{
    std::multimap<size_t, void*> all[64];
    {
        std::lock_guard<std::mutex> lock(g_pool_mutex);
        for (int d = 0; d < 64; ++d)
        {
            all[d].swap(g_pool[d].blocks);
            g_pool[d].bytes = 0;
        }
    }
    int prev = -1;
    cudaGetDevice(&prev);
    for (int d = 0; d < 64; ++d)
        if (!all[d].empty())
        {
            cudaSetDevice(d);
            for (auto& kv : all[d])
                cudaFree(kv.second);
        }
    if (prev >= 0)
        cudaSetDevice(prev);
}

// ---------------------------------------------------------------------------
// KSG plan
// ---------------------------------------------------------------------------

struct gc_ksg_plan
{
    int          device = 0, sms = 148;
    int          natoms = 0, T = 0, K = 0, path = GC_PATH_AUTO;
    long         pair_begin = 0, pair_count = 0;
    cudaStream_t stream = nullptr;
    PoolBuf<double>   X, psi;
    PoolBuf<uint32_t> cnt;
    DevBuf<int>      status;
    DevBuf<int2>     pair_ab; // explicit pair list as (a1, a2), empty for a range
    int              launches = 0;
    cudaEvent_t      ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t      ev_done = nullptr; // recorded after the last kernel of a run, on the run's stream
    bool             wide    = false;   // counts above 16 bits: n_x and n_y in two planes of cnt
    // fast path workspace
    bool                  fast = false;
    gc::host::KsgTraj     ft;
    gc::host::KsgLaunch   fl;
    PoolBuf<double>       io_xyz, io_mi; // gc_ksg_matrix staging of inputs and outputs
    long                         reason_counts[8] = {};
    double                       walk_mean = 0.0;
    long                         handoffs = 0;
    const double*                last_xyz = nullptr;
    double*                      last_mi  = nullptr;
    cudaStream_t                 last_stream = nullptr;
};

namespace {

gc_status validate_ksg(int natoms, int T, int k, const gc_opts& o, long* pb, long* pc)
{
    if (natoms < 2)
        return fail(GC_ERR_INVALID, "kraskov_corrmatrix: need at least 2 atoms");
    if (T <= k)
        return fail(GC_ERR_INVALID, "kraskov_corrmatrix: nframes must exceed k (number of nearest neighbours)");
    if (k < 1)
        return fail(GC_ERR_INVALID, "kraskov_corrmatrix: k must be at least 1");
    if (T > gc::kMaxFrames)
        return fail(GC_ERR_INVALID, "kraskov_corrmatrix: this build supports at most 16777216 frames");
    if (o.variant != GC_VARIANT_DEFAULT && o.variant != GC_VARIANT_HBM_GATHER)
        return fail(GC_ERR_INVALID, "unknown gc_opts.variant");
    const long np = (long)natoms * (natoms - 1) / 2;
    if (o.pair_list)
    {
        if (o.pair_list_len < 0)
            return fail(GC_ERR_INVALID, "negative pair list length");
        for (long q = 0; q < o.pair_list_len; ++q)
            if (o.pair_list[q] < 0 || o.pair_list[q] >= np)
                return fail(GC_ERR_INVALID, "pair list entry out of range");
        *pb = 0;
        *pc = o.pair_list_len;
        return GC_OK;
    }
    long b = o.pair_begin, e = o.pair_end <= 0 ? np : o.pair_end;
    if (b < 0 || b > e || e > np)
        return fail(GC_ERR_INVALID, "pair shard out of range");
    *pb = b;
    *pc = e - b;
    return GC_OK;
}

} // namespace

extern "C" {

void gc_opts_init(gc_opts* o)
{
    if (!o)
        return;
    std::memset(o, 0, sizeof(*o));
    o->device = -1;
    o->path   = GC_PATH_AUTO;
}

const char* gc_last_error(void) { return g_last_error.c_str(); }

int gc_device_count(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess)
    {
        cudaGetLastError();
        return 0;
    }
    return n;
}

int gc_gpu_available(void)
{
    const int n = gc_device_count();
    for (int d = 0; d < n; ++d)
    {
        cudaDeviceProp p{};
        if (cudaGetDeviceProperties(&p, d) == cudaSuccess && p.major == 10)
            return 1;
    }
    return 0;
}

gc_status gc_ksg_plan_create(int natoms, int nframes, int k, const gc_opts* opts, gc_ksg_plan** out)
{
    if (!out)
        return fail(GC_ERR_INVALID, "null plan output");
    *out          = nullptr;
    const gc_opts o = opts ? *opts : defaults();
    long pb = 0, pc = 0;
    GC_TRY(validate_ksg(natoms, nframes, k, o, &pb, &pc));
    DeviceScope dev(o.device);
    GC_TRY(dev.st);
    std::unique_ptr<gc_ksg_plan> p(new gc_ksg_plan);
    cudaGetDevice(&p->device);
    p->natoms     = natoms;
    p->T          = nframes;
    p->K          = k;
    p->path       = o.path;
    p->pair_begin = pb;
    p->pair_count = pc;
    GC_TRY_CUDA(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
    GC_TRY_CUDA(cudaEventCreate(&p->ev0));
    GC_TRY_CUDA(cudaEventCreate(&p->ev1));
    GC_TRY_CUDA(cudaEventCreateWithFlags(&p->ev_done, cudaEventDisableTiming));
    GC_TRY(p->X.alloc((size_t)3 * natoms * nframes));
    GC_TRY(p->psi.alloc((size_t)nframes + 1));
    // more than 65535 frames: counts need 32 bits each (the exact kernels'
    // wide layout; the fast path stops at 16385 frames anyway)
    p->wide = nframes > 65535;
    GC_TRY(p->cnt.alloc((size_t)nframes * (size_t)(pc > 0 ? pc : 1) * (p->wide ? 2 : 1)));
    GC_TRY(p->status.alloc(1));
    GC_TRY_CUDA(cudaDeviceGetAttribute(&p->sms, cudaDevAttrMultiProcessorCount, p->device));
    // The fast path sorts each marginal row in shared memory (<= 16384
    // frames); longer trajectories use the exact kernels throughout.
    p->fast = o.path != GC_PATH_EXACT_FP64 && nframes - 1 <= 16384 && pc > 0;
    const std::vector<double> psi = digamma_table(nframes);
    GC_TRY_CUDA(cudaMemcpy(p->psi.p, psi.data(), sizeof(double) * psi.size(), cudaMemcpyHostToDevice));
    if (o.pair_list && pc > 0)
    {
        std::vector<int2> ab((size_t)pc);
        for (long q = 0; q < pc; ++q)
        {
            int a1, a2;
            gc::pair_from_index((long)o.pair_list[q], &a1, &a2);
            ab[(size_t)q] = make_int2(a1, a2);
        }
        GC_TRY(p->pair_ab.alloc((size_t)pc));
        GC_TRY_CUDA(cudaMemcpy(p->pair_ab.p, ab.data(), sizeof(int2) * ab.size(), cudaMemcpyHostToDevice));
    }
    if (p->fast)
    {
        gc::host::WalkConfig cfg = gc::host::walk_config(nframes, k);
        const bool           hbm = o.variant == GC_VARIANT_HBM_GATHER;
        if (hbm)
        {
            // the other marginal comes from unsorted distance rows in HBM: no
            // staged coordinates, so the walk CTA takes the most warps
            cfg.gather_u   = true;
            cfg.staged     = false;
            cfg.walk_warps = gc::kWalkWarps;
        }
        GC_TRY(p->ft.create(natoms, nframes, k, pb, pc, o.pair_list, p->pair_ab.p,
                            gc::host::ksg_block_queries(natoms, nframes, 16.0 * (1 << 30), 32 * cfg.walk_warps,
                                                        hbm ? 4.0 * ((nframes + 3) & ~3) / (((nframes - 1) + 31) & ~31)
                                                            : 0.0),
                            cfg.pair_tile, hbm));
        std::vector<std::vector<gc::WalkParams>> waves;
        for (int b = 0; b < p->ft.blocks(); ++b)
            waves.push_back({p->ft.desc(p->X.p, p->cnt.p, p->status.p, b)});
        GC_TRY(p->fl.build(waves, {p->ft.desc(p->X.p, p->cnt.p, p->status.p, 0)}, cfg));
    }
    *out = p.release();
    return GC_OK;
}

} // extern "C"

namespace {

// One run of a plan: the normalisation of d_xyz into the plan's rows (or,
// with d_xyz == nullptr, a finiteness check of rows the caller already
// placed there), then the neighbour statistics and the MI reduction.
gc_status plan_run(gc_ksg_plan* p, const double* d_xyz, double* d_pair_mi, cudaStream_t s)
{
    p->launches = 0;
    GC_TRY_CUDA(cudaMemsetAsync(p->status.p, 0, sizeof(int), s));
    if (d_xyz)
        gc::launch_ksg_prepare(d_xyz, p->natoms, p->T, p->X.p, p->status.p, s);
    else
        gc::launch_ksg_check_rows(p->X.p, (long)3 * p->natoms * p->T, p->status.p, s);
    ++p->launches;
    p->last_xyz    = d_xyz;
    p->last_mi     = d_pair_mi;
    p->last_stream = s;
    if (p->pair_count > 0)
    {
        GC_TRY_CUDA(cudaEventRecord(p->ev0, s));
        if (p->fast)
        {
            GC_TRY_CUDA(gc::launch_ksg_x32(p->X.p, p->natoms, p->T, p->ft.X32.p, p->ft.eps.p, s));
            GC_TRY(p->ft.clear(s));
            GC_TRY(p->fl.enqueue(p->sms, s));
            p->launches += 1 + p->fl.launches;
        }
        else
        {
            gc::launch_ksg_exact(p->X.p, p->T, p->K, p->pair_begin, p->pair_count, p->cnt.p, s, p->pair_ab.p,
                                 p->wide ? p->cnt.p + (size_t)p->T * p->pair_count : nullptr);
            p->launches += 1;
        }
        GC_TRY_CUDA(cudaEventRecord(p->ev1, s));
        gc::launch_ksg_finalize(p->cnt.p, p->pair_count, p->T, p->K, p->psi.p, d_pair_mi, s,
                                p->wide ? p->cnt.p + (size_t)p->T * p->pair_count : nullptr);
        p->launches += 1;
    }
    GC_TRY_CUDA(cudaGetLastError());
    GC_TRY_CUDA(cudaEventRecord(p->ev_done, s));
    return GC_OK;
}

} // namespace

extern "C" {

gc_status gc_ksg_plan_run(gc_ksg_plan* p, const double* d_xyz, double* d_pair_mi, void* stream)
{
    if (!p || !d_xyz || !d_pair_mi)
        return fail(GC_ERR_INVALID, "null plan or device buffer");
    DeviceScope dev(p->device);
    GC_TRY(dev.st);
    return plan_run(p, d_xyz, d_pair_mi, stream ? (cudaStream_t)stream : p->stream);
}

gc_status gc_ksg_plan_sync(gc_ksg_plan* p)
{
    if (!p)
        return fail(GC_ERR_INVALID, "null plan");
    DeviceScope dev(p->device);
    GC_TRY(dev.st);
    // The run may have been ordered on a caller's stream: wait for its last
    // kernel only, not for the caller's other work on the device.
    GC_TRY_CUDA(cudaEventSynchronize(p->ev_done));
    int st = 0;
    GC_TRY_CUDA(cudaMemcpy(&st, p->status.p, sizeof(int), cudaMemcpyDeviceToHost));
    p->handoffs = 0;
    if (p->fast)
    {
        unsigned long long we = 0;
        GC_TRY_CUDA(cudaMemcpy(&we, p->ft.walk_elems.p, sizeof(we), cudaMemcpyDeviceToHost));
        p->walk_mean = (double)we / ((double)p->pair_count * p->T);
        unsigned rc[8] = {};
        GC_TRY_CUDA(cudaMemcpy(rc, p->ft.reasons.p, sizeof(rc), cudaMemcpyDeviceToHost));
        for (int r = 0; r < 8; ++r)
        {
            p->reason_counts[r] = (long)rc[r];
            p->handoffs += (long)rc[r];
        }
    }
    st &= ~gc::kStatFallback;
    return status_to_error(st);
}

long gc_ksg_plan_pairs(const gc_ksg_plan* p) { return p ? p->pair_count : 0; }

int gc_ksg_plan_launches(const gc_ksg_plan* p) { return p ? p->launches : 0; }

long gc_ksg_plan_handoffs(const gc_ksg_plan* p) { return p ? p->handoffs : 0; }

double gc_ksg_plan_walk_mean(const gc_ksg_plan* p) { return p ? p->walk_mean : 0.0; }

long gc_ksg_plan_handoff_reason(const gc_ksg_plan* p, int reason)
{
    return (p && reason >= 0 && reason < 8) ? p->reason_counts[reason] : 0;
}

int gc_ksg_plan_is_fast(const gc_ksg_plan* p) { return p && p->fast ? 1 : 0; }

float gc_ksg_plan_kernel_ms(const gc_ksg_plan* p)
{
    if (!p || !p->ev0 || !p->ev1 || p->pair_count <= 0)
        return 0.0f;
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, p->ev0, p->ev1) != cudaSuccess)
    {
        cudaGetLastError();
        return 0.0f;
    }
    return ms;
}

void gc_ksg_plan_destroy(gc_ksg_plan* p)
{
    if (!p)
        return;
    {
        DeviceScope dev(p->device);
        // The plan's pooled blocks go back to the device pool below, where the
        // next plan may take them at once: the last run's kernels (on whatever
        // stream it was ordered) must be done writing them first.
        if (p->ev_done)
        {
            cudaEventSynchronize(p->ev_done);
            cudaEventDestroy(p->ev_done);
        }
        if (p->stream)
            cudaStreamDestroy(p->stream);
        if (p->ev0)
            cudaEventDestroy(p->ev0);
        if (p->ev1)
            cudaEventDestroy(p->ev1);
        delete p; // the remaining buffers are freed with this device current
    }
}

} // extern "C"

namespace {

// One cached plan per device for gc_ksg_matrix: a repeated call with the same
// shape (atoms, frames, k, path, pair range) reuses the plan's device
// workspace instead of allocating and freeing it again.  Explicit pair lists
// are not cached.  gc_release_cache() frees the cached plans.
struct PlanKey
{
    int  natoms = 0, nframes = 0, k = 0, path = 0, variant = 0;
    long pair_begin = 0, pair_count = 0;
    bool operator==(const PlanKey& o) const
    {
        return natoms == o.natoms && nframes == o.nframes && k == o.k && path == o.path && variant == o.variant &&
               pair_begin == o.pair_begin && pair_count == o.pair_count;
    }
};

constexpr int kCacheDevices = 64;
std::mutex    g_cache_mutex;
gc_ksg_plan*  g_cache_plan[kCacheDevices] = {};
PlanKey       g_cache_key[kCacheDevices];

// Takes the cached plan for (device, key) if there is one, else nullptr.
gc_ksg_plan* cache_take(int dev, const PlanKey& key)
{
    if (dev < 0 || dev >= kCacheDevices)
        return nullptr;
    std::lock_guard<std::mutex> lock(g_cache_mutex);
    if (g_cache_plan[dev] && g_cache_key[dev] == key)
    {
        gc_ksg_plan* p    = g_cache_plan[dev];
        g_cache_plan[dev] = nullptr;
        return p;
    }
    return nullptr;
}

// Returns a plan to the cache; an older cached plan of that device is freed.
void cache_put(int dev, const PlanKey& key, gc_ksg_plan* p)
{
    gc_ksg_plan* old = nullptr;
    if (dev >= 0 && dev < kCacheDevices)
    {
        std::lock_guard<std::mutex> lock(g_cache_mutex);
        old               = g_cache_plan[dev];
        g_cache_plan[dev] = p;
        g_cache_key[dev]  = key;
    }
    else
        old = p;
    if (old)
        gc_ksg_plan_destroy(old);
}

} // namespace

extern "C" {

void gc_release_cache(void)
{
    gc_ksg_plan* plans[kCacheDevices];
    {
        std::lock_guard<std::mutex> lock(g_cache_mutex);
        for (int d = 0; d < kCacheDevices; ++d)
        {
            plans[d]        = g_cache_plan[d];
            g_cache_plan[d] = nullptr;
        }
    }
    for (gc_ksg_plan* p : plans)
        if (p)
            gc_ksg_plan_destroy(p);
    gc::host::pool_release();
}

} // extern "C"

namespace {

// gc_ksg_matrix and gc_ksg_matrix_prepared: either trajectory coordinates
// (traj) or already-normalised component rows X [3n][T] with their digamma
// table psi [T+1].
gc_status ksg_matrix_impl(const gc_traj_view* traj, const double* X, const double* psi_in, int n, int T, int k,
                          const gc_opts* opts, double* mi)
{
    if (!mi)
        return fail(GC_ERR_INVALID, "null output matrix");
    const gc_opts o = opts ? *opts : defaults();
    long          pb = 0, pc = 0;
    GC_TRY(validate_ksg(n, T, k, o, &pb, &pc));
    DeviceScope dev(o.device);
    GC_TRY(dev.st);
    int cur = -1;
    cudaGetDevice(&cur);
    PlanKey key;
    key.natoms     = n;
    key.nframes    = T;
    key.k          = k;
    key.path       = o.path;
    key.variant    = o.variant;
    key.pair_begin = pb;
    key.pair_count = pc;
    // A plan that holds a caller's digamma table is not kept for later calls.
    const bool   cacheable = o.pair_list == nullptr && traj != nullptr;
    gc_ksg_plan* raw       = cacheable ? cache_take(cur, key) : nullptr;
    if (!raw)
        GC_TRY(gc_ksg_plan_create(n, T, k, &o, &raw));
    std::unique_ptr<gc_ksg_plan, void (*)(gc_ksg_plan*)> plan(raw, gc_ksg_plan_destroy);
    if (!plan->io_mi.p)
        GC_TRY(plan->io_mi.alloc((size_t)(pc > 0 ? pc : 1)));
    cudaStream_t s = plan->stream;
    if (traj)
    {
        if (!plan->io_xyz.p)
            GC_TRY(plan->io_xyz.alloc((size_t)n * T * 3));
        GC_TRY(upload_traj(traj, plan->io_xyz.p, s));
        GC_TRY(plan_run(plan.get(), plan->io_xyz.p, plan->io_mi.p, s));
    }
    else
    {
        GC_TRY_CUDA(cudaMemcpyAsync(plan->X.p, X, sizeof(double) * 3 * (size_t)n * T, cudaMemcpyHostToDevice, s));
        GC_TRY_CUDA(cudaMemcpyAsync(plan->psi.p, psi_in, sizeof(double) * ((size_t)T + 1), cudaMemcpyHostToDevice, s));
        GC_TRY(plan_run(plan.get(), nullptr, plan->io_mi.p, s));
    }
    GC_TRY(gc_ksg_plan_sync(plan.get()));
    std::vector<double> pm((size_t)pc);
    if (pc > 0)
        GC_TRY_CUDA(cudaMemcpy(pm.data(), plan->io_mi.p, sizeof(double) * pc, cudaMemcpyDeviceToHost));
    if (o.detail_nx || o.detail_ny)
    {
        const bool            wide = plan->wide;
        const size_t          m    = (size_t)T * pc;
        std::vector<uint32_t> c(m * (wide ? 2 : 1));
        if (pc > 0)
            GC_TRY_CUDA(cudaMemcpy(c.data(), plan->cnt.p, sizeof(uint32_t) * c.size(), cudaMemcpyDeviceToHost));
        for (size_t e = 0; e < m; ++e)
        {
            const uint32_t v = c[e];
            if (o.detail_nx)
                o.detail_nx[e] = (int32_t)(wide ? v : (v & 0xFFFFu));
            if (o.detail_ny)
                o.detail_ny[e] = (int32_t)(wide ? c[m + e] : (v >> 16));
        }
    }
    // kraskov_corrmatrix: zero fill, diagonal 2000, symmetric entries.
    std::memset(mi, 0, sizeof(double) * (size_t)n * n);
    for (int a = 0; a < n; ++a)
        mi[(size_t)a * n + a] = 2000.0;
    for (long pl = 0; pl < pc; ++pl)
    {
        int a1, a2;
        gc::pair_from_index(o.pair_list ? (long)o.pair_list[pl] : pb + pl, &a1, &a2);
        mi[(size_t)a1 * n + a2] = pm[(size_t)pl];
        mi[(size_t)a2 * n + a1] = pm[(size_t)pl];
    }
    if (cacheable)
        cache_put(cur, key, plan.release());
    return GC_OK;
}

} // namespace

extern "C" {

gc_status gc_ksg_matrix(const gc_traj_view* traj, int k, const gc_opts* opts, double* mi)
{
    GC_TRY(check_view(traj));
    return ksg_matrix_impl(traj, nullptr, nullptr, traj->natoms, traj->nframes, k, opts, mi);
}

gc_status gc_ksg_matrix_prepared(const double* X, const double* psi, int natoms, int nframes, int k,
                                 const gc_opts* opts, double* mi)
{
    if (!X || !psi)
        return fail(GC_ERR_INVALID, "null normalised rows or digamma table");
    return ksg_matrix_impl(nullptr, X, psi, natoms, nframes, k, opts, mi);
}

static gc_status gauss_like(const gc_traj_view* traj, const gc_opts* opts, double* mi, int mode)
{
    GC_TRY(check_view(traj));
    if (!mi)
        return fail(GC_ERR_INVALID, "null output matrix");
    const gc_opts o = opts ? *opts : defaults();
    const int     n = traj->natoms, T = traj->nframes;
    if (mode == 1)
    {
        if (n < 2)
            return fail(GC_ERR_INVALID, "gcmi_corrmatrix: need at least 2 atoms");
        if (T < 6)
            return fail(GC_ERR_INVALID, "gcmi_corrmatrix: need at least 6 frames for a non-singular 6x6 covariance");
        if (T > gc::kMaxFrames)
            return fail(GC_ERR_INVALID, "gcmi_corrmatrix: this build supports at most 16777216 frames");
    }
    else if (n < 1 || T < 1)
        return fail(GC_ERR_INVALID, "gauss_corrmatrix: empty trajectory");
    DeviceScope dev(o.device);
    GC_TRY(dev.st);
    StreamScope ss;
    GC_TRY(ss.init(o.stream));
    const long     nb = (long)n * (n + 1) / 2;
    DevBuf<double> d_xyz, d_XF, d_Z, d_zt, d_blk, d_mat;
    DevBuf<int>    d_st;
    GC_TRY(d_xyz.alloc((size_t)n * T * 3));
    GC_TRY(d_XF.alloc((size_t)n * T * 3));
    GC_TRY(d_blk.alloc((size_t)nb * 9));
    GC_TRY(d_mat.alloc((size_t)n * n));
    GC_TRY(d_st.alloc(1));
    if (mode == 1)
    {
        GC_TRY(d_Z.alloc((size_t)n * T * 3));
        GC_TRY(d_zt.alloc((size_t)T));
    }
    GC_TRY(upload_traj(traj, d_xyz.p, ss.s));
    GC_TRY_CUDA(cudaMemsetAsync(d_st.p, 0, sizeof(int), ss.s));
    GC_TRY_CUDA(cudaMemsetAsync(d_mat.p, 0, sizeof(double) * (size_t)n * n, ss.s));
    gc::launch_frame_major(d_xyz.p, n, T, d_XF.p, d_st.p, ss.s);
    const double* V = d_XF.p;
    if (mode == 1)
    {
        gc::launch_copula(d_XF.p, n, T, d_zt.p, d_Z.p, ss.s);
        V = d_Z.p;
    }
    gc::launch_blocks(V, n, T, d_blk.p, ss.s);
    const double log2pi = std::log(2.0 * 3.14159265358979323846);
    gc::launch_pair_logdet(d_blk.p, n, T, mode, log2pi, d_mat.p, ss.s);
    GC_TRY_CUDA(cudaGetLastError());
    GC_TRY_CUDA(cudaStreamSynchronize(ss.s));
    int st = 0;
    GC_TRY_CUDA(cudaMemcpy(&st, d_st.p, sizeof(int), cudaMemcpyDeviceToHost));
    GC_TRY(status_to_error(st & gc::kStatNonFinite));
    GC_TRY_CUDA(cudaMemcpy(mi, d_mat.p, sizeof(double) * (size_t)n * n, cudaMemcpyDeviceToHost));
    return GC_OK;
}

gc_status gc_gauss_matrix(const gc_traj_view* traj, const gc_opts* opts, double* mi)
{
    return gauss_like(traj, opts, mi, 0);
}

gc_status gc_gcmi_matrix(const gc_traj_view* traj, const gc_opts* opts, double* mi)
{
    return gauss_like(traj, opts, mi, 1);
}


gc_status gc_ksg_prepare(const gc_traj_view* traj, const gc_opts* opts, double* X, double* psi, double* scal)
{
    GC_TRY(check_view(traj));
    if (!X || !psi)
        return fail(GC_ERR_INVALID, "null output array");
    const gc_opts o = opts ? *opts : defaults();
    const int     n = traj->natoms, T = traj->nframes;
    if (n < 1 || T < 2)
        return fail(GC_ERR_INVALID, "kraskov_prepare: need at least one atom and two frames");
    DeviceScope dev(o.device);
    GC_TRY(dev.st);
    StreamScope ss;
    GC_TRY(ss.init(o.stream));
    DevBuf<double> d_xyz, d_X;
    DevBuf<int>    d_st;
    GC_TRY(d_xyz.alloc((size_t)n * T * 3));
    GC_TRY(d_X.alloc((size_t)n * T * 3));
    GC_TRY(d_st.alloc(1));
    GC_TRY(upload_traj(traj, d_xyz.p, ss.s));
    GC_TRY_CUDA(cudaMemsetAsync(d_st.p, 0, sizeof(int), ss.s));
    gc::launch_ksg_prepare(d_xyz.p, n, T, d_X.p, d_st.p, ss.s);
    GC_TRY_CUDA(cudaGetLastError());
    GC_TRY_CUDA(cudaStreamSynchronize(ss.s));
    int st = 0;
    GC_TRY_CUDA(cudaMemcpy(&st, d_st.p, sizeof(int), cudaMemcpyDeviceToHost));
    GC_TRY(status_to_error(st));
    GC_TRY_CUDA(cudaMemcpy(X, d_X.p, sizeof(double) * (size_t)n * T * 3, cudaMemcpyDeviceToHost));
    const std::vector<double> tab = digamma_table(T);
    std::memcpy(psi, tab.data(), sizeof(double) * tab.size());
    if (scal)
        for (int c = 0; c < 3 * n; ++c)
        {
            // X is min-shifted, so max - min is the row maximum.
            double mx = 0.0;
            for (int f = 0; f < T; ++f)
                mx = X[(size_t)c * T + f] > mx ? X[(size_t)c * T + f] : mx;
            scal[c] = (T - 5) / mx;
        }
    return GC_OK;
}

gc_status gc_ksg_pair(const double* rows6, int nframes, int k, const double* psi, const gc_opts* opts, double* mi)
{
    if (!rows6 || !psi || !mi)
        return fail(GC_ERR_INVALID, "null argument");
    const gc_opts o = opts ? *opts : defaults();
    const int     T = nframes;
    long          pb, pc;
    gc_opts       one = o;
    one.pair_begin = 0;
    one.pair_end   = 0;
    one.pair_list  = nullptr;
    GC_TRY(validate_ksg(2, T, k, one, &pb, &pc));
    DeviceScope dev(o.device);
    GC_TRY(dev.st);
    StreamScope ss;
    GC_TRY(ss.init(o.stream));
    // Two-atom system whose single pair (1, 0) has a1 = atom 1: the
    // x-marginal (first three rows, the grid's first axis) goes to atom 1.
    DevBuf<double>   d_X, d_psi, d_mi;
    DevBuf<uint32_t> d_cnt;
    GC_TRY(d_X.alloc((size_t)6 * T));
    GC_TRY(d_psi.alloc((size_t)T + 1));
    GC_TRY(d_mi.alloc(1));
    const bool wide = T > 65535;
    GC_TRY(d_cnt.alloc((size_t)T * (wide ? 2 : 1)));
    GC_TRY_CUDA(cudaMemcpyAsync(d_X.p + (size_t)3 * T, rows6, sizeof(double) * 3 * T, cudaMemcpyHostToDevice, ss.s));
    GC_TRY_CUDA(cudaMemcpyAsync(d_X.p, rows6 + (size_t)3 * T, sizeof(double) * 3 * T, cudaMemcpyHostToDevice, ss.s));
    GC_TRY_CUDA(cudaMemcpyAsync(d_psi.p, psi, sizeof(double) * (T + 1), cudaMemcpyHostToDevice, ss.s));
    gc::launch_ksg_exact(d_X.p, T, k, 0, 1, d_cnt.p, ss.s, nullptr, wide ? d_cnt.p + T : nullptr);
    gc::launch_ksg_finalize(d_cnt.p, 1, T, k, d_psi.p, d_mi.p, ss.s, wide ? d_cnt.p + T : nullptr);
    GC_TRY_CUDA(cudaGetLastError());
    GC_TRY_CUDA(cudaMemcpyAsync(mi, d_mi.p, sizeof(double), cudaMemcpyDeviceToHost, ss.s));
    GC_TRY_CUDA(cudaStreamSynchronize(ss.s));
    return GC_OK;
}

} // extern "C"
