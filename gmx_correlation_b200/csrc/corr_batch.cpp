// Transfer-entropy and GCMI matrices of many trajectories in one batched run
// (no counterpart in the reference, which computes te_matrix and
// gcmi_corrmatrix once per trajectory: lib/transfer_entropy.cpp:63-221,
// lib/gcmi.cpp:246-317).
//
// TE: every trajectory gets the single-trajectory plan's workspace
// (TeTraj); trajectories are grouped by row length, and within a group each
// wave is one launch of the row sort, the walk, the finish and the count
// whose tasks are drawn from every trajectory still active, with query-block
// sizes from the smallest number of waves whose sorted rows fit the group's
// share of the row budget.  GCMI: the copula, co-moment and log-determinant
// kernels of every trajectory.  Either sequence (everything after the input
// upload) is captured once into a CUDA graph and replayed on later calls
// with the same shapes.

#include "gc_internal.h"
#include "host_common.h"
#include "ksg_fast.h"
#include "ksg_host.h"
#include "te_host.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>

using namespace gc::host;

namespace {

// Sorted rows: one trajectory's query block is sized as the single-trajectory
// plan sizes it (so every pair task holds whole rounds of the walk CTA's
// warps); the blocks of one wave share an arena of at most kTeArenaBudget
// bytes, or the largest block where that is larger.
constexpr double kTeBlockBudget = 16.0 * (1ull << 30);
constexpr double kTeArenaBudget = 32.0 * (1ull << 30);
constexpr int    kMaxDev        = 64;

gc_status capture_graph(cudaStream_t s, cudaGraphExec_t* exec, gc_status (*fn)(void*, cudaStream_t), void* ctx)
{
    if (*exec)
    {
        cudaGraphExecDestroy(*exec);
        *exec = nullptr;
    }
    cudaGraph_t graph = nullptr;
    GC_TRY_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    const gc_status   st = fn(ctx, s);
    const cudaError_t ce = cudaStreamEndCapture(s, &graph);
    if (st != GC_OK)
    {
        if (graph)
            cudaGraphDestroy(graph);
        return st;
    }
    GC_TRY_CUDA(ce);
    const cudaError_t ie = cudaGraphInstantiate(exec, graph, 0);
    cudaGraphDestroy(graph);
    GC_TRY_CUDA(ie);
    return GC_OK;
}

// ---------------------------------------------------------------------------
// Transfer entropy
// ---------------------------------------------------------------------------

struct TeItem
{
    int                     natoms = 0, T = 0, K = 0;
    bool                    active = false; // N_valid > k and two atoms or more
    PoolBuf<double>         xyz, te;
    std::unique_ptr<TeTraj> tt;
    std::vector<double>     host;
};

struct TeBatchPlan
{
    int                                    device = 0, sms = 148, lag = 0;
    std::vector<int>                       key;
    std::vector<std::unique_ptr<TeItem>>   items;
    DevBuf<int>                            status;
    PoolBuf<unsigned char>                 arena;
    std::vector<std::unique_ptr<TeLaunch>> groups;
    cudaStream_t                           stream = nullptr;
    cudaGraphExec_t                        exec   = nullptr;
    ~TeBatchPlan()
    {
        if (stream)
            cudaStreamSynchronize(stream);
        if (exec)
            cudaGraphExecDestroy(exec);
        if (stream)
            cudaStreamDestroy(stream);
    }
};

int te_row_class(int Nv)
{
    const int N = Nv - 1;
    return N <= 2048 ? 0 : (N <= 4096 ? 1 : (N <= 8192 ? 2 : 3));
}

gc_status te_enqueue_all(void* ctx, cudaStream_t s)
{
    TeBatchPlan& bp = *static_cast<TeBatchPlan*>(ctx);
    GC_TRY_CUDA(cudaMemsetAsync(bp.status.p, 0, sizeof(int) * bp.items.size(), s));
    for (size_t i = 0; i < bp.items.size(); ++i)
    {
        TeItem& it = *bp.items[i];
        GC_TRY_CUDA(cudaMemsetAsync(it.te.p, 0, sizeof(double) * (size_t)it.natoms * it.natoms, s));
        if (it.active)
            GC_TRY(it.tt->prepare(it.xyz.p, bp.status.p + i, s));
    }
    for (auto& g : bp.groups)
        GC_TRY(g->enqueue(bp.sms, s));
    for (auto& ip : bp.items)
        if (ip->active)
            GC_TRY_CUDA(gc::launch_te_reduce(ip->tt->cnt.p, ip->natoms, ip->tt->Nv, ip->K, ip->tt->psi.p, ip->te.p, s));
    GC_TRY_CUDA(cudaGetLastError());
    return GC_OK;
}

gc_status te_create_plan(const gc_traj_view* trajs, const int* ks, int ntraj, int lag, int device,
                         std::unique_ptr<TeBatchPlan>& out)
{
    auto bp    = std::make_unique<TeBatchPlan>();
    bp->device = device;
    bp->lag    = lag;
    GC_TRY_CUDA(cudaDeviceGetAttribute(&bp->sms, cudaDevAttrMultiProcessorCount, device));
    GC_TRY_CUDA(cudaStreamCreateWithFlags(&bp->stream, cudaStreamNonBlocking));
    GC_TRY(bp->status.alloc((size_t)ntraj));
    for (int i = 0; i < ntraj; ++i)
        bp->items.push_back(std::make_unique<TeItem>());
    int                              gid[4] = {-1, -1, -1, -1};
    std::vector<std::vector<size_t>> members;
    for (int i = 0; i < ntraj; ++i)
    {
        TeItem& it = *bp->items[(size_t)i];
        it.natoms  = trajs[i].natoms;
        it.T       = trajs[i].nframes;
        it.K       = ks[i];
        it.active  = it.natoms >= 2 && it.T - lag > it.K;
        GC_TRY(it.xyz.alloc((size_t)it.natoms * it.T * 3));
        GC_TRY(it.te.alloc((size_t)it.natoms * it.natoms));
        bp->key.insert(bp->key.end(), {it.natoms, it.T, it.K});
        if (!it.active)
            continue;
        const int c = te_row_class(it.T - lag);
        if (gid[c] < 0)
        {
            gid[c] = (int)members.size();
            members.emplace_back();
        }
        members[(size_t)gid[c]].push_back((size_t)i);
    }
    // Per row class: the walk shape of its longest trajectory, each member's
    // block size, then the (trajectory, block) pairs packed into waves by
    // first fit in decreasing row bytes, at most one block of a trajectory
    // per wave (its walk results and hand-over queue hold one block).
    struct Slot
    {
        size_t item;
        int    block;
        size_t bytes;
    };
    std::vector<std::vector<std::vector<Slot>>> plan(members.size());
    size_t                                      arena = 0;
    for (size_t g = 0; g < members.size(); ++g)
    {
        int maxT = 0;
        for (size_t i : members[g])
            maxT = std::max(maxT, bp->items[i]->T);
        int  warps  = 0;
        bool staged = false;
        gc::walk_shape(maxT, &warps, &staged);
        std::vector<Slot> slots;
        size_t            largest = 0;
        for (size_t i : members[g])
        {
            TeItem&   it = *bp->items[i];
            const int Nv = it.T - lag;
            const int Q  = ksg_block_queries(2 * it.natoms, Nv, kTeBlockBudget, 32 * warps);
            it.tt        = std::make_unique<TeTraj>();
            GC_TRY(it.tt->create(it.natoms, it.T, it.K, lag, Q, false));
            const size_t b = it.tt->block_row_bytes();
            largest        = std::max(largest, b);
            for (int w = 0; w < it.tt->blocks(); ++w)
                slots.push_back({i, w, b});
        }
        std::stable_sort(slots.begin(), slots.end(), [](const Slot& a, const Slot& b) { return a.bytes > b.bytes; });
        const size_t        cap = std::max(largest, (size_t)kTeArenaBudget);
        std::vector<size_t> used;
        auto&               waves = plan[g];
        for (const Slot& sl : slots)
        {
            size_t w = 0;
            for (; w < waves.size(); ++w)
            {
                bool clash = false;
                for (const Slot& o : waves[w])
                    clash = clash || o.item == sl.item;
                if (!clash && used[w] + sl.bytes <= cap)
                    break;
            }
            if (w == waves.size())
            {
                waves.emplace_back();
                used.push_back(0);
            }
            waves[w].push_back(sl);
            used[w] += sl.bytes;
            arena = std::max(arena, used[w]);
        }
    }
    GC_TRY(bp->arena.alloc(arena));
    for (size_t g = 0; g < members.size(); ++g)
    {
        std::vector<std::vector<gc::TeParams>> waves;
        for (const auto& wv : plan[g])
        {
            waves.emplace_back();
            size_t off = 0;
            for (const Slot& sl : wv)
            {
                const TeTraj&  tt   = *bp->items[sl.item]->tt;
                const size_t   e    = (size_t)tt.natoms * tt.Qp * tt.Lpad;
                auto           a    = [](size_t b) { return (b + 255) & ~(size_t)255; };
                unsigned char* base = bp->arena.p + off;
                float*         SG   = reinterpret_cast<float*>(base);
                float*         SM   = reinterpret_cast<float*>(base + a(e * sizeof(float)));
                uint16_t*      PG   = reinterpret_cast<uint16_t*>(base + 2 * a(e * sizeof(float)));
                uint16_t*      PM   = reinterpret_cast<uint16_t*>(base + 2 * a(e * sizeof(float)) + a(e * sizeof(uint16_t)));
                waves.back().push_back(tt.desc_rows(bp->status.p + sl.item, sl.block, SG, PG, SM, PM));
                off += sl.bytes;
            }
        }
        std::vector<gc::TeParams> fix;
        for (size_t i : members[g])
            fix.push_back(bp->items[i]->tt->desc_rows(bp->status.p + i, 0, nullptr, nullptr, nullptr, nullptr));
        auto tl = std::make_unique<TeLaunch>();
        GC_TRY(tl->build(waves, fix));
        bp->groups.push_back(std::move(tl));
    }
    out = std::move(bp);
    return GC_OK;
}

std::mutex   g_te_mutex;
TeBatchPlan* g_te[kMaxDev] = {}; // the last batch per device (its blocks return to the pool when replaced)

// ---------------------------------------------------------------------------
// GCMI
// ---------------------------------------------------------------------------

struct GcmiItem
{
    int                 natoms = 0, T = 0;
    PoolBuf<double>     xyz, XF, Z, zt, blk, mat;
    std::vector<double> host;
};

struct GcmiBatchPlan
{
    int                   device = 0;
    std::vector<int>      key;
    std::vector<std::unique_ptr<GcmiItem>> items;
    DevBuf<int>           status;
    cudaStream_t          stream = nullptr;
    cudaGraphExec_t       exec   = nullptr;
    ~GcmiBatchPlan()
    {
        if (stream)
            cudaStreamSynchronize(stream);
        if (exec)
            cudaGraphExecDestroy(exec);
        if (stream)
            cudaStreamDestroy(stream);
    }
};

gc_status gcmi_enqueue_all(void* ctx, cudaStream_t s)
{
    GcmiBatchPlan& bp     = *static_cast<GcmiBatchPlan*>(ctx);
    const double   log2pi = std::log(2.0 * 3.14159265358979323846);
    GC_TRY_CUDA(cudaMemsetAsync(bp.status.p, 0, sizeof(int) * bp.items.size(), s));
    for (size_t i = 0; i < bp.items.size(); ++i)
    {
        GcmiItem& it = *bp.items[i];
        GC_TRY_CUDA(cudaMemsetAsync(it.mat.p, 0, sizeof(double) * (size_t)it.natoms * it.natoms, s));
        gc::launch_frame_major(it.xyz.p, it.natoms, it.T, it.XF.p, bp.status.p + i, s);
        gc::launch_copula(it.XF.p, it.natoms, it.T, it.zt.p, it.Z.p, s);
        gc::launch_blocks(it.Z.p, it.natoms, it.T, it.blk.p, s);
        gc::launch_pair_logdet(it.blk.p, it.natoms, it.T, 1, log2pi, it.mat.p, s);
    }
    GC_TRY_CUDA(cudaGetLastError());
    return GC_OK;
}

std::mutex     g_gcmi_mutex;
GcmiBatchPlan* g_gcmi[kMaxDev] = {};

gc_status batch_device(const gc_opts* opts, int* cur)
{
    (void)opts;
    *cur = 0;
    cudaGetDevice(cur);
    if (*cur < 0 || *cur >= kMaxDev)
        return fail(GC_ERR_INVALID, "batch: device ordinal beyond the batch cache");
    return GC_OK;
}

} // namespace

extern "C" {

gc_status gc_te_batch(const gc_traj_view* trajs, const int* ks, int ntraj, int lag, const gc_opts* opts,
                      double* const* te)
{
    if (!trajs || !ks || !te || ntraj < 1)
        return fail(GC_ERR_INVALID, "gc_te_batch: need trajectories, k values and output matrices");
    if (lag < 0)
        return fail(GC_ERR_INVALID, "te_matrix: lag must be non-negative");
    const gc_opts o = opts ? *opts : defaults();
    for (int i = 0; i < ntraj; ++i)
    {
        GC_TRY(check_view(&trajs[i]));
        if (!te[i])
            return fail(GC_ERR_INVALID, "gc_te_batch: null output matrix");
        if (ks[i] < 1)
            return fail(GC_ERR_INVALID, "te_matrix: k must be at least 1");
        if (trajs[i].nframes - lag - 1 > 16384)
            return fail(GC_ERR_INVALID, "gc_te_batch: nframes - lag <= 16385 (use gc_te_matrix for longer trajectories)");
        if (trajs[i].natoms >= 2 && trajs[i].nframes - lag <= ks[i])
            std::fprintf(stderr, "Warning: TE: N_valid=%d <= k=%d; skipping.\n", trajs[i].nframes - lag, ks[i]);
    }
    DeviceScope dev(o.device);
    GC_TRY(dev.st);
    int cur = 0;
    GC_TRY(batch_device(&o, &cur));
    std::vector<int> key;
    for (int i = 0; i < ntraj; ++i)
        key.insert(key.end(), {trajs[i].natoms, trajs[i].nframes, ks[i]});

    std::lock_guard<std::mutex> lock(g_te_mutex);
    if (!g_te[cur] || g_te[cur]->lag != lag || g_te[cur]->key != key)
    {
        // the previous batch gives its blocks back to the pool, where the new
        // one (another lag of the same trajectories) finds them again
        delete g_te[cur];
        g_te[cur] = nullptr;
        std::unique_ptr<TeBatchPlan> made;
        GC_TRY(te_create_plan(trajs, ks, ntraj, lag, cur, made));
        g_te[cur] = made.release();
    }
    TeBatchPlan* bp = g_te[cur];
    cudaStream_t s  = bp->stream;
    for (int i = 0; i < ntraj; ++i)
        GC_TRY(upload_traj(&trajs[i], bp->items[(size_t)i]->xyz.p, s));
    if (!bp->exec)
        GC_TRY(capture_graph(s, &bp->exec, te_enqueue_all, bp));
    GC_TRY_CUDA(cudaGraphLaunch(bp->exec, s));
    std::vector<int> st((size_t)ntraj);
    GC_TRY_CUDA(cudaMemcpyAsync(st.data(), bp->status.p, sizeof(int) * ntraj, cudaMemcpyDeviceToHost, s));
    for (int i = 0; i < ntraj; ++i)
    {
        TeItem& it = *bp->items[(size_t)i];
        GC_TRY_CUDA(cudaMemcpyAsync(te[i], it.te.p, sizeof(double) * (size_t)it.natoms * it.natoms,
                                    cudaMemcpyDeviceToHost, s));
    }
    GC_TRY_CUDA(cudaStreamSynchronize(s));
    for (int i = 0; i < ntraj; ++i)
        GC_TRY(status_to_error(st[(size_t)i] & gc::kStatNonFinite));
    return GC_OK;
}

void gc_te_batch_release(void)
{
    std::lock_guard<std::mutex> lock(g_te_mutex);
    for (TeBatchPlan*& b : g_te)
        if (b)
        {
            DeviceScope dev(b->device);
            delete b;
            b = nullptr;
        }
}

gc_status gc_gcmi_batch(const gc_traj_view* trajs, int ntraj, const gc_opts* opts, double* const* mi)
{
    if (!trajs || !mi || ntraj < 1)
        return fail(GC_ERR_INVALID, "gc_gcmi_batch: need trajectories and output matrices");
    const gc_opts o = opts ? *opts : defaults();
    for (int i = 0; i < ntraj; ++i)
    {
        GC_TRY(check_view(&trajs[i]));
        if (!mi[i])
            return fail(GC_ERR_INVALID, "gc_gcmi_batch: null output matrix");
        if (trajs[i].natoms < 2)
            return fail(GC_ERR_INVALID, "gcmi_corrmatrix: need at least 2 atoms");
        if (trajs[i].nframes < 6)
            return fail(GC_ERR_INVALID, "gcmi_corrmatrix: need at least 6 frames for a non-singular 6x6 covariance");
        if (trajs[i].nframes > gc::kMaxFrames)
            return fail(GC_ERR_INVALID, "gcmi_corrmatrix: this build supports at most 16777216 frames");
    }
    DeviceScope dev(o.device);
    GC_TRY(dev.st);
    int cur = 0;
    GC_TRY(batch_device(&o, &cur));
    std::vector<int> key;
    for (int i = 0; i < ntraj; ++i)
        key.insert(key.end(), {trajs[i].natoms, trajs[i].nframes});

    std::lock_guard<std::mutex> lock(g_gcmi_mutex);
    if (!g_gcmi[cur] || g_gcmi[cur]->key != key)
    {
        delete g_gcmi[cur];
        g_gcmi[cur] = nullptr;
        auto bp     = std::make_unique<GcmiBatchPlan>();
        bp->device  = cur;
        bp->key     = key;
        GC_TRY_CUDA(cudaStreamCreateWithFlags(&bp->stream, cudaStreamNonBlocking));
        GC_TRY(bp->status.alloc((size_t)ntraj));
        for (int i = 0; i < ntraj; ++i)
        {
            bp->items.push_back(std::make_unique<GcmiItem>());
            GcmiItem& it = *bp->items.back();
            it.natoms    = trajs[i].natoms;
            it.T         = trajs[i].nframes;
            const size_t c = (size_t)it.natoms * it.T * 3;
            GC_TRY(it.xyz.alloc(c));
            GC_TRY(it.XF.alloc(c));
            GC_TRY(it.Z.alloc(c));
            GC_TRY(it.zt.alloc((size_t)it.T));
            GC_TRY(it.blk.alloc((size_t)it.natoms * (it.natoms + 1) / 2 * 9));
            GC_TRY(it.mat.alloc((size_t)it.natoms * it.natoms));
        }
        g_gcmi[cur] = bp.release();
    }
    GcmiBatchPlan* bp = g_gcmi[cur];
    cudaStream_t   s  = bp->stream;
    for (int i = 0; i < ntraj; ++i)
        GC_TRY(upload_traj(&trajs[i], bp->items[(size_t)i]->xyz.p, s));
    if (!bp->exec)
        GC_TRY(capture_graph(s, &bp->exec, gcmi_enqueue_all, bp));
    GC_TRY_CUDA(cudaGraphLaunch(bp->exec, s));
    std::vector<int> st((size_t)ntraj);
    GC_TRY_CUDA(cudaMemcpyAsync(st.data(), bp->status.p, sizeof(int) * ntraj, cudaMemcpyDeviceToHost, s));
    for (int i = 0; i < ntraj; ++i)
    {
        GcmiItem& it = *bp->items[(size_t)i];
        GC_TRY_CUDA(cudaMemcpyAsync(mi[i], it.mat.p, sizeof(double) * (size_t)it.natoms * it.natoms,
                                    cudaMemcpyDeviceToHost, s));
    }
    GC_TRY_CUDA(cudaStreamSynchronize(s));
    for (int i = 0; i < ntraj; ++i)
        GC_TRY(status_to_error(st[(size_t)i] & gc::kStatNonFinite));
    return GC_OK;
}

void gc_gcmi_batch_release(void)
{
    std::lock_guard<std::mutex> lock(g_gcmi_mutex);
    for (GcmiBatchPlan*& b : g_gcmi)
        if (b)
        {
            DeviceScope dev(b->device);
            delete b;
            b = nullptr;
        }
}

} // extern "C"
