// KSG matrices of many trajectories in one batched run (no counterpart in
// the reference, which runs kraskov_corrmatrix once per trajectory,
// lib/correlation_core.cpp:324-459).
//
// Every trajectory gets the single-trajectory plan's workspace; the query
// blocks of all trajectories then run together: each wave is one launch of
// the row sort, the walk and the finish whose tasks are drawn from every
// trajectory still active (a global task counter over a prefix table of
// per-trajectory descriptors), so trajectories of uneven atom and frame
// counts and different k share the GPU.  Trajectories are grouped by row
// length (up to 2048, 4096, 8192 or more sorted entries per row), and each
// group runs its own waves with the row-sort and walk shapes of its longest
// rows, so short trajectories do not take the shapes long ones need.  The
// whole sequence (normalisation, FP32 rows, every group's waves, exact
// fix-up, MI reduction) is captured once into a CUDA graph and replayed; each
// group's walk launch shape (atom-tile size of the pair order, query groups
// per warp task) is chosen by timing the candidates on its first wave the
// first time a shape class is seen.

#include "gc_geom.h"
#include "gc_internal.h"
#include "host_common.h"
#include "ksg_host.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

using namespace gc::host;

namespace {

// Sorted rows: one trajectory's query block is sized as the single-trajectory
// plan sizes it, and the blocks of one wave share an arena of at most
// kArenaBudget bytes (or the largest block, where that is larger).
constexpr double kBlockBudget = 16.0 * (1ull << 30);
constexpr double kArenaBudget = 32.0 * (1ull << 30);

// One trajectory's query block in a wave, at an offset of the row arena.
struct WaveSlot
{
    size_t item;
    int    block;
    size_t bytes, offset;
};

struct BatchTraj
{
    int                 natoms = 0, T = 0, K = 0;
    long                pairs  = 0;
    DevBuf<double>      xyz, X, psi, mi;
    DevBuf<uint32_t>    cnt;
    KsgTraj             ft;
    std::vector<double> host_mi;
};

// Trajectories of one row-length class and their launch tables.
struct BatchGroup
{
    std::vector<size_t> members; // indices into BatchPlan::t
    int                 maxT = 0, maxK = 0;
    std::vector<std::vector<WaveSlot>> waves;
    KsgLaunch           fl;
    WalkConfig          cfg;
};

// Row-length class of a trajectory: its rows' sorted-entry count up to 2048,
// 4096, 8192 or beyond (the row sort's and the walk's shapes change there).
int row_class(int T)
{
    const int N = T - 1;
    return N <= 2048 ? 0 : (N <= 4096 ? 1 : (N <= 8192 ? 2 : 3));
}

struct BatchPlan
{
    int                                     device = 0, sms = 148;
    std::vector<std::unique_ptr<BatchTraj>> t;
    DevBuf<int>                             status;
    PoolBuf<unsigned char>                  arena; // sorted rows of one wave
    std::vector<std::unique_ptr<BatchGroup>> groups;
    bool                                    tuned  = false;
    cudaStream_t                            stream = nullptr;
    cudaGraphExec_t                         exec   = nullptr;
    std::vector<int>                        key; // natoms, T, k per trajectory
    ~BatchPlan()
    {
        if (exec)
            cudaGraphExecDestroy(exec);
        if (stream)
            cudaStreamDestroy(stream);
    }
};

// Kept batches, one per device.  Deliberately never destroyed at process
// exit (the driver frees device memory then), so no destructor runs after
// the CUDA context is gone.
std::mutex  g_batch_mutex;
BatchPlan*  g_batch[64] = {};

// Packs the (trajectory, block) pairs of a group into waves: first fit in
// decreasing row bytes, at most one block of a trajectory per wave (its walk
// results and hand-over queue hold one block).  Returns the largest wave's
// bytes.
size_t pack_waves(BatchPlan& bp, BatchGroup& g)
{
    std::vector<WaveSlot> slots;
    size_t                largest = 0;
    for (size_t i : g.members)
    {
        const KsgTraj& ft = bp.t[i]->ft;
        const size_t   b  = ft.block_row_bytes();
        largest           = std::max(largest, b);
        for (int w = 0; w < ft.blocks(); ++w)
            slots.push_back({i, w, b, 0});
    }
    std::stable_sort(slots.begin(), slots.end(), [](const WaveSlot& a, const WaveSlot& b) { return a.bytes > b.bytes; });
    const size_t        cap = std::max(largest, (size_t)kArenaBudget);
    std::vector<size_t> used;
    size_t              most = 0;
    g.waves.clear();
    for (WaveSlot sl : slots)
    {
        size_t w = 0;
        for (; w < g.waves.size(); ++w)
        {
            bool clash = false;
            for (const WaveSlot& o : g.waves[w])
                clash = clash || o.item == sl.item;
            if (!clash && used[w] + sl.bytes <= cap)
                break;
        }
        if (w == g.waves.size())
        {
            g.waves.emplace_back();
            used.push_back(0);
        }
        sl.offset = used[w];
        g.waves[w].push_back(sl);
        used[w] += sl.bytes;
        most = std::max(most, used[w]);
    }
    return most;
}

gc_status build_launch(BatchPlan& bp, BatchGroup& g, const WalkConfig& cfg)
{
    for (size_t i : g.members)
        GC_TRY(bp.t[i]->ft.set_pair_tile(cfg.pair_tile));
    std::vector<std::vector<gc::WalkParams>> waves;
    for (const auto& wv : g.waves)
    {
        waves.emplace_back();
        for (const WaveSlot& sl : wv)
        {
            BatchTraj&     b    = *bp.t[sl.item];
            const size_t   e    = (size_t)b.ft.natoms * b.ft.Qp * b.ft.Lpad;
            unsigned char* base = bp.arena.p + sl.offset;
            float*         S    = reinterpret_cast<float*>(base);
            uint16_t*      P    = reinterpret_cast<uint16_t*>(base + ((e * sizeof(float) + 255) & ~(size_t)255));
            waves.back().push_back(b.ft.desc_rows(b.X.p, b.cnt.p, bp.status.p + sl.item, sl.block, S, P));
        }
    }
    std::vector<gc::WalkParams> traj;
    for (size_t i : g.members)
    {
        BatchTraj& b = *bp.t[i];
        traj.push_back(b.ft.desc_rows(b.X.p, b.cnt.p, bp.status.p + i, 0, nullptr, nullptr));
    }
    g.cfg = cfg;
    return g.fl.build(waves, traj, cfg);
}

// Everything after the input upload, in stream order (graph-capturable).
gc_status enqueue_all(BatchPlan& bp, cudaStream_t s)
{
    GC_TRY_CUDA(cudaMemsetAsync(bp.status.p, 0, sizeof(int) * bp.t.size(), s));
    for (size_t i = 0; i < bp.t.size(); ++i)
    {
        BatchTraj& b = *bp.t[i];
        gc::launch_ksg_prepare(b.xyz.p, b.natoms, b.T, b.X.p, bp.status.p + i, s);
        GC_TRY_CUDA(gc::launch_ksg_x32(b.X.p, b.natoms, b.T, b.ft.X32.p, b.ft.eps.p, s));
        GC_TRY(b.ft.clear(s));
    }
    for (auto& g : bp.groups)
        GC_TRY(g->fl.enqueue(bp.sms, s));
    for (auto& b : bp.t)
        gc::launch_ksg_finalize(b->cnt.p, b->pairs, b->T, b->K, b->psi.p, b->mi.p, s);
    GC_TRY_CUDA(cudaGetLastError());
    return GC_OK;
}

// Times each candidate walk configuration on every group's first wave and
// keeps the fastest per group (inputs must be uploaded; the status words are
// ignored here).
gc_status autotune(BatchPlan& bp)
{
    cudaStream_t s = bp.stream;
    for (size_t i = 0; i < bp.t.size(); ++i)
    {
        BatchTraj& b = *bp.t[i];
        gc::launch_ksg_prepare(b.xyz.p, b.natoms, b.T, b.X.p, bp.status.p + i, s);
        GC_TRY_CUDA(gc::launch_ksg_x32(b.X.p, b.natoms, b.T, b.ft.X32.p, b.ft.eps.p, s));
    }
    cudaEvent_t e0, e1;
    GC_TRY_CUDA(cudaEventCreate(&e0));
    GC_TRY_CUDA(cudaEventCreate(&e1));
    gc_status st = GC_OK;
    for (auto& gp : bp.groups)
    {
        BatchGroup& g    = *gp;
        float      best = 1e30f;
        WalkConfig best_cfg;
        for (const WalkConfig& c : walk_candidates(g.maxT))
        {
            if ((st = build_launch(bp, g, c)) != GC_OK)
                break;
            float ms = 0.0f;
            for (int rep = 0; rep < 2 && st == GC_OK; ++rep) // the first run warms up
            {
                for (size_t i : g.members)
                    if ((st = bp.t[i]->ft.clear(s)) != GC_OK)
                        break;
                cudaEventRecord(e0, s);
                if (st == GC_OK)
                    st = g.fl.enqueue(bp.sms, s, 0, 0, false);
                cudaEventRecord(e1, s);
                if (cudaEventSynchronize(e1) != cudaSuccess)
                    st = fail(GC_ERR_CUDA, "autotune run failed");
                cudaEventElapsedTime(&ms, e0, e1);
            }
            if (st != GC_OK)
                break;
            if (ms < best)
            {
                best     = ms;
                best_cfg = c;
            }
        }
        if (st != GC_OK)
            break;
        remember_walk_config(g.maxT, g.maxK, best_cfg);
        if ((st = build_launch(bp, g, best_cfg)) != GC_OK)
            break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    GC_TRY(st);
    bp.tuned = true;
    return GC_OK;
}

gc_status create_plan(const gc_traj_view* trajs, const int* ks, int ntraj, int device, std::unique_ptr<BatchPlan>& out)
{
    auto bp    = std::make_unique<BatchPlan>();
    bp->device = device;
    GC_TRY_CUDA(cudaDeviceGetAttribute(&bp->sms, cudaDevAttrMultiProcessorCount, device));
    GC_TRY_CUDA(cudaStreamCreateWithFlags(&bp->stream, cudaStreamNonBlocking));
    GC_TRY(bp->status.alloc((size_t)ntraj));
    for (int i = 0; i < ntraj; ++i)
    {
        auto b    = std::make_unique<BatchTraj>();
        b->natoms = trajs[i].natoms;
        b->T      = trajs[i].nframes;
        b->K      = ks[i];
        b->pairs  = (long)b->natoms * (b->natoms - 1) / 2;
        GC_TRY(b->xyz.alloc((size_t)b->natoms * b->T * 3));
        GC_TRY(b->X.alloc((size_t)b->natoms * b->T * 3));
        GC_TRY(b->psi.alloc((size_t)b->T + 1));
        GC_TRY(b->mi.alloc((size_t)b->pairs));
        GC_TRY(b->cnt.alloc((size_t)b->T * b->pairs));
        const std::vector<double> psi = digamma_table(b->T);
        GC_TRY_CUDA(cudaMemcpy(b->psi.p, psi.data(), sizeof(double) * psi.size(), cudaMemcpyHostToDevice));
        bp->key.insert(bp->key.end(), {b->natoms, b->T, b->K});
        bp->t.push_back(std::move(b));
    }
    // groups by row length, each with the walk shape of its longest
    // trajectory and single-plan query blocks packed into waves
    int gid[4] = {-1, -1, -1, -1};
    for (size_t i = 0; i < bp->t.size(); ++i)
    {
        const BatchTraj& b = *bp->t[i];
        const int        c = row_class(b.T);
        if (gid[c] < 0)
        {
            gid[c] = (int)bp->groups.size();
            bp->groups.push_back(std::make_unique<BatchGroup>());
        }
        BatchGroup& g = *bp->groups[(size_t)gid[c]];
        g.members.push_back(i);
        g.maxT = std::max(g.maxT, b.T);
        g.maxK = std::max(g.maxK, b.K);
    }
    size_t arena = 0;
    std::vector<WalkConfig> cfgs;
    for (auto& gp : bp->groups)
    {
        BatchGroup&      g   = *gp;
        const WalkConfig cfg = walk_config(g.maxT, g.maxK);
        for (size_t i : g.members)
        {
            BatchTraj& b = *bp->t[i];
            const int  Q = ksg_block_queries(b.natoms, b.T, kBlockBudget, 32 * cfg.walk_warps);
            GC_TRY(b.ft.create(b.natoms, b.T, b.K, 0, b.pairs, nullptr, nullptr, Q, cfg.pair_tile, false, false));
        }
        arena = std::max(arena, pack_waves(*bp, g));
        cfgs.push_back(cfg);
    }
    GC_TRY(bp->arena.alloc(arena));
    for (size_t gi = 0; gi < bp->groups.size(); ++gi)
        GC_TRY(build_launch(*bp, *bp->groups[gi], cfgs[gi]));
    out = std::move(bp);
    return GC_OK;
}

gc_status capture(BatchPlan& bp)
{
    if (bp.exec)
    {
        cudaGraphExecDestroy(bp.exec);
        bp.exec = nullptr;
    }
    cudaGraph_t graph = nullptr;
    GC_TRY_CUDA(cudaStreamBeginCapture(bp.stream, cudaStreamCaptureModeThreadLocal));
    const gc_status   st = enqueue_all(bp, bp.stream);
    const cudaError_t ce = cudaStreamEndCapture(bp.stream, &graph);
    if (st != GC_OK)
    {
        if (graph)
            cudaGraphDestroy(graph);
        return st;
    }
    GC_TRY_CUDA(ce);
    const cudaError_t ie = cudaGraphInstantiate(&bp.exec, graph, 0);
    cudaGraphDestroy(graph);
    GC_TRY_CUDA(ie);
    return GC_OK;
}

} // namespace

extern "C" {

gc_status gc_ksg_batch(const gc_traj_view* trajs, const int* ks, int ntraj, const gc_opts* opts, double* const* mi)
{
    if (!trajs || !ks || !mi || ntraj < 1)
        return fail(GC_ERR_INVALID, "gc_ksg_batch: need trajectories, k values and output matrices");
    const gc_opts o = opts ? *opts : defaults();
    for (int i = 0; i < ntraj; ++i)
    {
        GC_TRY(check_view(&trajs[i]));
        if (!mi[i])
            return fail(GC_ERR_INVALID, "gc_ksg_batch: null output matrix");
        const int n = trajs[i].natoms, T = trajs[i].nframes, k = ks[i];
        if (n < 2 || k < 1 || T <= k)
            return fail(GC_ERR_INVALID, "gc_ksg_batch: every trajectory needs >= 2 atoms and nframes > k >= 1");
        if (T - 1 > 16384)
            return fail(GC_ERR_INVALID, "gc_ksg_batch: nframes <= 16385 (use gc_ksg_matrix for longer trajectories)");
    }
    DeviceScope dev(o.device);
    GC_TRY(dev.st);
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur < 0 || cur >= 64)
        return fail(GC_ERR_INVALID, "gc_ksg_batch: device ordinal beyond the batch cache");
    std::vector<int> key;
    for (int i = 0; i < ntraj; ++i)
        key.insert(key.end(), {trajs[i].natoms, trajs[i].nframes, ks[i]});

    std::lock_guard<std::mutex> lock(g_batch_mutex); // one batch per process at a time
    if (!g_batch[cur] || g_batch[cur]->key != key)
    {
        delete g_batch[cur];
        g_batch[cur] = nullptr;
        std::unique_ptr<BatchPlan> made;
        GC_TRY(create_plan(trajs, ks, ntraj, cur, made));
        g_batch[cur] = made.release();
    }
    BatchPlan* bp = g_batch[cur];
    cudaStream_t s = bp->stream;
    for (int i = 0; i < ntraj; ++i)
        GC_TRY(upload_traj(&trajs[i], bp->t[(size_t)i]->xyz.p, s));
    if (!bp->tuned)
    {
        GC_TRY(autotune(*bp));
        GC_TRY(capture(*bp));
    }
    else if (!bp->exec)
        GC_TRY(capture(*bp));
    GC_TRY_CUDA(cudaGraphLaunch(bp->exec, s));
    std::vector<int> st((size_t)ntraj);
    GC_TRY_CUDA(cudaMemcpyAsync(st.data(), bp->status.p, sizeof(int) * ntraj, cudaMemcpyDeviceToHost, s));
    for (auto& b : bp->t)
    {
        b->host_mi.resize((size_t)b->pairs);
        GC_TRY_CUDA(cudaMemcpyAsync(b->host_mi.data(), b->mi.p, sizeof(double) * b->pairs, cudaMemcpyDeviceToHost, s));
    }
    GC_TRY_CUDA(cudaStreamSynchronize(s));
    for (int i = 0; i < ntraj; ++i)
        GC_TRY(status_to_error(st[(size_t)i] & ~gc::kStatFallback));
    for (int i = 0; i < ntraj; ++i)
    {
        const BatchTraj& b = *bp->t[(size_t)i];
        double*          m = mi[i];
        const int        n = b.natoms;
        std::memset(m, 0, sizeof(double) * (size_t)n * n);
        for (int a = 0; a < n; ++a)
            m[(size_t)a * n + a] = 2000.0;
        for (long p = 0; p < b.pairs; ++p)
        {
            int a1, a2;
            gc::pair_from_index(p, &a1, &a2);
            m[(size_t)a1 * n + a2] = b.host_mi[(size_t)p];
            m[(size_t)a2 * n + a1] = b.host_mi[(size_t)p];
        }
    }
    return GC_OK;
}

void gc_ksg_batch_release(void)
{
    std::lock_guard<std::mutex> lock(g_batch_mutex);
    for (BatchPlan*& b : g_batch)
        if (b)
        {
            DeviceScope dev(b->device);
            delete b;
            b = nullptr;
        }
}

} // extern "C"
