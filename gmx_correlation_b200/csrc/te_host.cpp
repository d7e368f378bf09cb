// Host side of transfer entropy: the device-resident TE plan (sorted-row
// walk, or the brute-force kernels for the exact path and for rows too long
// to sort in shared memory) and gc_te_matrix on top of it.
//
// Reference: te_matrix, lib/transfer_entropy.cpp:63-221 (argument checks,
// the zero fill, the N_valid <= k early return, mat[a1 * n + a2] =
// TE(a2 -> a1) with a zero diagonal).

#include "gmx_corr_b200.h"
#include "gc_internal.h"
#include "host_common.h"
#include "ksg_fast.h"
#include "ksg_host.h"
#include "te_walk.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>

using namespace gc::host;

struct gc_te_plan
{
    int          device = 0, sms = 148;
    int          natoms = 0, T = 0, K = 0, lag = 0, Nv = 0, path = GC_PATH_AUTO;
    long         npairs = 0; // ordered pairs
    bool         walk   = false;
    cudaStream_t stream = nullptr;
    cudaEvent_t  ev0 = nullptr, ev1 = nullptr, ev_done = nullptr;
    PoolBuf<double> XT, psi;
    PoolBuf<float4> X32;
    PoolBuf<float>  eps;
    PoolBuf<uint2>  cnt;
    DevBuf<int>     status;
    int             launches = 0;
    // walk path
    int                         Q = 0, Qp = 0, Lpad = 0, warps = 0;
    bool                        staged = false;
    PoolBuf<float>              SG, SM;
    PoolBuf<uint16_t>           PG, PM;
    PoolBuf<unsigned long long> wres, hq, walk_elems;
    PoolBuf<unsigned>           hq_len, reasons;
    PoolBuf<int>                pair_order;
    DevBuf<gc::TeParams>        descs;
    DevBuf<long long>           prefix;
    DevBuf<unsigned long long>  counters;
    std::vector<gc::TeBatch>    waves;
    std::vector<long long>      wave_rows;
    gc::TeBatch                 fix{};
    long                        handoffs = 0;
    double                      walk_mean = 0.0;
};

namespace {

gc_status te_validate(int natoms, int T, int k, int lag)
{
    if (k < 1)
        return fail(GC_ERR_INVALID, "te_matrix: k must be at least 1");
    if (lag < 0)
        return fail(GC_ERR_INVALID, "te_matrix: lag must be non-negative");
    if (natoms < 0 || T < 0)
        return fail(GC_ERR_INVALID, "te_matrix: negative trajectory size");
    if (T > 65535)
        return fail(GC_ERR_INVALID, "te_matrix: this build supports at most 65535 frames");
    return GC_OK;
}

// Walk tasks visit the ordered pairs by 16 x 16 atom tiles, so the rows of
// the atoms the running tasks read stay in L2.
std::vector<int> te_tile_order(int n)
{
    const long             np = (long)n * (n - 1);
    std::vector<long long> key((size_t)np);
    for (long q = 0; q < np; ++q)
    {
        const int a1 = (int)(q / (n - 1));
        const int rr = (int)(q - (long)a1 * (n - 1));
        const int a2 = rr < a1 ? rr : rr + 1;
        key[(size_t)q] = (((long long)(a1 >> 4) * 65536 + (a2 >> 4)) << 32) | (long long)q;
    }
    std::sort(key.begin(), key.end());
    std::vector<int> order((size_t)np);
    for (long q = 0; q < np; ++q)
        order[(size_t)q] = (int)(key[(size_t)q] & 0xFFFFFFFFll);
    return order;
}

gc_status te_build_walk(gc_te_plan* p)
{
    const int n = p->natoms, Nv = p->Nv;
    gc::walk_shape(p->T, &p->warps, &p->staged);
    const int chunk = p->warps * 4;
    // Sorted rows of one query block: G and M rows of every atom, within 16 GiB.
    p->Q    = ksg_block_queries(2 * n, Nv, 16.0 * (1 << 30), 32 * p->warps);
    p->Qp   = (p->Q + 31) & ~31;
    p->Lpad = ((Nv - 1) + 31) & ~31;
    const size_t rows = (size_t)n * p->Qp * p->Lpad;
    GC_TRY(p->SG.alloc(rows));
    GC_TRY(p->SM.alloc(rows));
    GC_TRY(p->PG.alloc(rows));
    GC_TRY(p->PM.alloc(rows));
    GC_TRY(p->wres.alloc((size_t)p->Q * p->npairs));
    const double hq_want = 0.01 * (double)p->npairs * Nv + 4096.0;
    const unsigned hq_cap = (unsigned)(hq_want < 16777216.0 ? hq_want : 16777216.0);
    GC_TRY(p->hq.alloc(hq_cap));
    GC_TRY(p->hq_len.alloc(1));
    GC_TRY(p->walk_elems.alloc(1));
    GC_TRY(p->reasons.alloc(8));
    const std::vector<int> order = te_tile_order(n);
    GC_TRY(p->pair_order.alloc(order.size()));
    GC_TRY_CUDA(cudaMemcpy(p->pair_order.p, order.data(), sizeof(int) * order.size(), cudaMemcpyHostToDevice));

    const int                  nblocks = (Nv + p->Q - 1) / p->Q;
    std::vector<gc::TeParams>  all;
    std::vector<long long>     pre;
    for (int b = 0; b <= nblocks; ++b)
    {
        gc::TeParams d{};
        d.X32        = p->X32.p;
        d.XT         = p->XT.p;
        d.eps_atom   = p->eps.p;
        d.SG         = p->SG.p;
        d.PG         = p->PG.p;
        d.SM         = p->SM.p;
        d.PM         = p->PM.p;
        d.natoms     = n;
        d.T          = p->T;
        d.lag        = p->lag;
        d.Nv         = Nv;
        d.K          = p->K;
        d.Lpad       = p->Lpad;
        d.Qp         = p->Qp;
        d.i0         = b < nblocks ? b * p->Q : 0;
        d.Q          = b < nblocks ? std::min(p->Q, Nv - b * p->Q) : p->Q;
        d.pair_count = p->npairs;
        d.pair_order = p->pair_order.p;
        d.shift      = gc::walk_histogram_shift(p->K);
        d.cnt        = p->cnt.p;
        d.wres       = p->wres.p;
        d.hq         = p->hq.p;
        d.hq_len     = p->hq_len.p;
        d.hq_cap     = hq_cap;
        d.status     = p->status.p;
        d.walk_elems = p->walk_elems.p;
        d.reasons    = p->reasons.p;
        all.push_back(d); // the last one is the fix-up's descriptor
        if (b < nblocks)
        {
            const long long grp = (d.Q + 31) / 32;
            pre.insert(pre.end(), {0, 2LL * n * d.Q, 0, (grp + chunk - 1) / chunk * p->npairs, 0, grp * p->npairs});
        }
    }
    GC_TRY(p->descs.alloc(all.size()));
    GC_TRY(p->prefix.alloc(pre.size()));
    GC_TRY(p->counters.alloc(2 * (size_t)nblocks));
    GC_TRY_CUDA(cudaMemcpy(p->descs.p, all.data(), sizeof(gc::TeParams) * all.size(), cudaMemcpyHostToDevice));
    GC_TRY_CUDA(cudaMemcpy(p->prefix.p, pre.data(), sizeof(long long) * pre.size(), cudaMemcpyHostToDevice));
    p->waves.clear();
    p->wave_rows.clear();
    for (int b = 0; b < nblocks; ++b)
    {
        gc::TeBatch w{};
        w.d       = p->descs.p + b;
        w.rprefix = p->prefix.p + 6 * b;
        w.wprefix = w.rprefix + 2;
        w.fprefix = w.rprefix + 4;
        w.n       = 1;
        w.maxT    = p->T;
        w.maxNv   = Nv;
        w.maxK    = p->K;
        w.chunk   = chunk;
        w.counter = p->counters.p + 2 * b;
        p->waves.push_back(w);
        p->wave_rows.push_back(2LL * n * all[(size_t)b].Q);
    }
    p->fix       = gc::TeBatch{};
    p->fix.d     = p->descs.p + nblocks;
    p->fix.n     = 1;
    p->fix.maxT  = p->T;
    p->fix.maxNv = Nv;
    p->fix.maxK  = p->K;
    return GC_OK;
}

} // namespace

extern "C" {

gc_status gc_te_plan_create(int natoms, int nframes, int k, int lag, const gc_opts* opts, gc_te_plan** out)
{
    if (!out)
        return fail(GC_ERR_INVALID, "null plan output");
    *out            = nullptr;
    const gc_opts o = opts ? *opts : defaults();
    GC_TRY(te_validate(natoms, nframes, k, lag));
    if (natoms < 2 || nframes - lag <= k)
        return fail(GC_ERR_INVALID, "te plan: needs at least 2 atoms and nframes - lag > k");
    DeviceScope dev(o.device);
    GC_TRY(dev.st);
    std::unique_ptr<gc_te_plan> p(new gc_te_plan);
    cudaGetDevice(&p->device);
    p->natoms = natoms;
    p->T      = nframes;
    p->K      = k;
    p->lag    = lag;
    p->Nv     = nframes - lag;
    p->path   = o.path;
    p->npairs = (long)natoms * (natoms - 1);
    p->walk   = o.path != GC_PATH_EXACT_FP64 && p->Nv - 1 <= 16384;
    GC_TRY_CUDA(cudaDeviceGetAttribute(&p->sms, cudaDevAttrMultiProcessorCount, p->device));
    GC_TRY_CUDA(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
    GC_TRY_CUDA(cudaEventCreate(&p->ev0));
    GC_TRY_CUDA(cudaEventCreate(&p->ev1));
    GC_TRY_CUDA(cudaEventCreateWithFlags(&p->ev_done, cudaEventDisableTiming));
    GC_TRY(p->XT.alloc((size_t)natoms * nframes * 3));
    // psi[0 .. N_valid + 1]: a count clamped to N_valid indexes psi[N_valid + 1]
    GC_TRY(p->psi.alloc((size_t)p->Nv + 2));
    GC_TRY(p->X32.alloc((size_t)natoms * nframes));
    GC_TRY(p->eps.alloc((size_t)natoms));
    GC_TRY(p->cnt.alloc((size_t)p->Nv * p->npairs));
    GC_TRY(p->status.alloc(1));
    const std::vector<double> psi = digamma_table(p->Nv + 1);
    GC_TRY_CUDA(cudaMemcpy(p->psi.p, psi.data(), sizeof(double) * psi.size(), cudaMemcpyHostToDevice));
    if (p->walk)
        GC_TRY(te_build_walk(p.get()));
    *out = p.release();
    return GC_OK;
}

gc_status gc_te_plan_run(gc_te_plan* p, const double* d_xyz, double* d_te, void* stream)
{
    if (!p || !d_xyz || !d_te)
        return fail(GC_ERR_INVALID, "null plan or device buffer");
    DeviceScope dev(p->device);
    GC_TRY(dev.st);
    cudaStream_t s = stream ? (cudaStream_t)stream : p->stream;
    const int    n = p->natoms;
    p->launches    = 0;
    GC_TRY_CUDA(cudaMemsetAsync(p->status.p, 0, sizeof(int), s));
    GC_TRY_CUDA(cudaMemsetAsync(d_te, 0, sizeof(double) * (size_t)n * n, s));
    gc::launch_transpose_components(d_xyz, n, p->T, p->XT.p, p->status.p, s);
    gc::launch_te_x32(p->XT.p, n, p->T, p->X32.p, p->eps.p, s);
    p->launches += 2;
    GC_TRY_CUDA(cudaEventRecord(p->ev0, s));
    if (p->walk)
    {
        GC_TRY_CUDA(cudaMemsetAsync(p->counters.p, 0, sizeof(unsigned long long) * 2 * p->waves.size(), s));
        GC_TRY_CUDA(cudaMemsetAsync(p->hq_len.p, 0, sizeof(unsigned), s));
        GC_TRY_CUDA(cudaMemsetAsync(p->reasons.p, 0, 8 * sizeof(unsigned), s));
        GC_TRY_CUDA(cudaMemsetAsync(p->walk_elems.p, 0, sizeof(unsigned long long), s));
        for (size_t w = 0; w < p->waves.size(); ++w)
        {
            GC_TRY_CUDA(gc::launch_te_rows(p->waves[w], p->wave_rows[w], s));
            GC_TRY_CUDA(gc::launch_te_walk(p->waves[w], p->warps, p->staged, p->sms, s));
            GC_TRY_CUDA(gc::launch_te_finish(p->waves[w], p->sms, s));
            GC_TRY_CUDA(cudaMemsetAsync(p->waves[w].counter, 0, sizeof(unsigned long long), s));
            GC_TRY_CUDA(gc::launch_te_count(p->waves[w], p->warps, p->staged, p->sms, s));
            p->launches += 4;
        }
        GC_TRY_CUDA(gc::launch_te_fixup(p->fix, p->sms, s));
        GC_TRY_CUDA(cudaEventRecord(p->ev1, s));
        GC_TRY_CUDA(gc::launch_te_reduce(p->cnt.p, n, p->Nv, p->K, p->psi.p, d_te, s));
        p->launches += 3;
    }
    else
    {
        if (p->path == GC_PATH_EXACT_FP64)
            gc::launch_te_exact(p->XT.p, n, p->T, p->K, p->lag, p->cnt.p, s);
        else
            gc::launch_te_fast(p->XT.p, p->X32.p, p->eps.p, n, p->T, p->K, p->lag, p->cnt.p, s);
        GC_TRY_CUDA(cudaEventRecord(p->ev1, s));
        gc::launch_te_finalize(p->cnt.p, n, p->T, p->K, p->lag, p->psi.p, d_te, s);
        p->launches += 2;
    }
    GC_TRY_CUDA(cudaGetLastError());
    GC_TRY_CUDA(cudaEventRecord(p->ev_done, s));
    return GC_OK;
}

gc_status gc_te_plan_sync(gc_te_plan* p)
{
    if (!p)
        return fail(GC_ERR_INVALID, "null plan");
    DeviceScope dev(p->device);
    GC_TRY(dev.st);
    GC_TRY_CUDA(cudaEventSynchronize(p->ev_done));
    int st = 0;
    GC_TRY_CUDA(cudaMemcpy(&st, p->status.p, sizeof(int), cudaMemcpyDeviceToHost));
    p->handoffs  = 0;
    p->walk_mean = 0.0;
    if (p->walk)
    {
        unsigned rc[8] = {};
        GC_TRY_CUDA(cudaMemcpy(rc, p->reasons.p, sizeof(rc), cudaMemcpyDeviceToHost));
        for (unsigned r : rc)
            p->handoffs += (long)r;
        unsigned long long we = 0;
        GC_TRY_CUDA(cudaMemcpy(&we, p->walk_elems.p, sizeof(we), cudaMemcpyDeviceToHost));
        p->walk_mean = (double)we / ((double)p->npairs * p->Nv);
    }
    return status_to_error(st & gc::kStatNonFinite);
}

long gc_te_plan_pairs(const gc_te_plan* p) { return p ? p->npairs : 0; }

int gc_te_plan_launches(const gc_te_plan* p) { return p ? p->launches : 0; }

int gc_te_plan_is_walk(const gc_te_plan* p) { return p && p->walk ? 1 : 0; }

long gc_te_plan_handoffs(const gc_te_plan* p) { return p ? p->handoffs : 0; }

double gc_te_plan_walk_mean(const gc_te_plan* p) { return p ? p->walk_mean : 0.0; }

float gc_te_plan_kernel_ms(const gc_te_plan* p)
{
    if (!p)
        return 0.0f;
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, p->ev0, p->ev1) != cudaSuccess)
    {
        cudaGetLastError();
        return 0.0f;
    }
    return ms;
}

gc_status gc_te_plan_counts(gc_te_plan* p, int a1, int a2, int32_t* n_xp, int32_t* n_xfxp, int32_t* n_ypxp)
{
    if (!p || a1 < 0 || a2 < 0 || a1 >= p->natoms || a2 >= p->natoms || a1 == a2)
        return fail(GC_ERR_INVALID, "te plan counts: bad plan or atom pair");
    DeviceScope dev(p->device);
    GC_TRY(dev.st);
    GC_TRY_CUDA(cudaEventSynchronize(p->ev_done));
    const long q = (long)a1 * (p->natoms - 1) + (a2 < a1 ? a2 : a2 - 1);
    std::vector<uint2> c((size_t)p->Nv);
    if (p->walk) // pair-major [q][Nv]
        GC_TRY_CUDA(cudaMemcpy(c.data(), p->cnt.p + (size_t)q * p->Nv, sizeof(uint2) * c.size(),
                               cudaMemcpyDeviceToHost));
    else // query-major [qi][npairs]
        GC_TRY_CUDA(cudaMemcpy2D(c.data(), sizeof(uint2), p->cnt.p + q, sizeof(uint2) * p->npairs, sizeof(uint2),
                                 (size_t)p->Nv, cudaMemcpyDeviceToHost));
    for (int i = 0; i < p->Nv; ++i)
    {
        if (n_xp)
            n_xp[i] = (int32_t)(c[(size_t)i].x & 0xFFFFu);
        if (n_xfxp)
            n_xfxp[i] = (int32_t)(c[(size_t)i].x >> 16);
        if (n_ypxp)
            n_ypxp[i] = (int32_t)c[(size_t)i].y;
    }
    return GC_OK;
}

void gc_te_plan_destroy(gc_te_plan* p)
{
    if (!p)
        return;
    DeviceScope dev(p->device);
    // pooled blocks go back to the pool: the last run must be done with them
    if (p->ev_done)
    {
        cudaEventSynchronize(p->ev_done);
        cudaEventDestroy(p->ev_done);
    }
    if (p->ev0)
        cudaEventDestroy(p->ev0);
    if (p->ev1)
        cudaEventDestroy(p->ev1);
    if (p->stream)
        cudaStreamDestroy(p->stream);
    delete p;
}

gc_status gc_te_matrix(const gc_traj_view* traj, int k, int lag, const gc_opts* opts, double* te)
{
    GC_TRY(check_view(traj));
    if (!te)
        return fail(GC_ERR_INVALID, "null output matrix");
    const gc_opts o = opts ? *opts : defaults();
    const int     n = traj->natoms, T = traj->nframes;
    GC_TRY(te_validate(n, T, k, lag));
    std::memset(te, 0, sizeof(double) * (size_t)n * n);
    const int Nv = T - lag;
    if (Nv <= k)
    {
        std::fprintf(stderr, "Warning: TE: N_valid=%d <= k=%d; skipping.\n", Nv, k);
        return GC_OK;
    }
    if (n < 2)
        return GC_OK;
    DeviceScope dev(o.device);
    GC_TRY(dev.st);
    // declared before the plan, so the plan (which waits for its last run)
    // is destroyed first and these blocks return to the pool idle
    PoolBuf<double> d_xyz, d_te;
    gc_te_plan*     raw = nullptr;
    GC_TRY(gc_te_plan_create(n, T, k, lag, &o, &raw));
    std::unique_ptr<gc_te_plan, void (*)(gc_te_plan*)> plan(raw, gc_te_plan_destroy);
    GC_TRY(d_xyz.alloc((size_t)n * T * 3));
    GC_TRY(d_te.alloc((size_t)n * n));
    cudaStream_t s = o.stream ? (cudaStream_t)o.stream : plan->stream;
    GC_TRY(upload_traj(traj, d_xyz.p, s));
    GC_TRY(gc_te_plan_run(plan.get(), d_xyz.p, d_te.p, s));
    GC_TRY(gc_te_plan_sync(plan.get()));
    GC_TRY_CUDA(cudaMemcpy(te, d_te.p, sizeof(double) * (size_t)n * n, cudaMemcpyDeviceToHost));
    return GC_OK;
}

} // extern "C"
