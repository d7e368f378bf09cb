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
#include "te_host.h"
#include "te_walk.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>

using namespace gc::host;

namespace {

gc_status te_validate(int natoms, int T, int k, int lag)
{
    if (k < 1)
        return fail(GC_ERR_INVALID, "te_matrix: k must be at least 1");
    if (lag < 0)
        return fail(GC_ERR_INVALID, "te_matrix: lag must be non-negative");
    if (natoms < 0 || T < 0)
        return fail(GC_ERR_INVALID, "te_matrix: negative trajectory size");
    if (T > gc::kMaxFrames)
        return fail(GC_ERR_INVALID, "te_matrix: this build supports at most 16777216 frames");
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

} // namespace

namespace gc {
namespace host {

double te_row_bytes_per_query(int natoms, int Nv)
{
    // G and M rows of every atom: (distance + frame) per entry
    return 2.0 * natoms * (double)(((Nv - 1) + 31) & ~31) * 6.0;
}

gc_status TeTraj::create(int n, int nframes, int k, int lg, int q, bool own_rows)
{
    natoms = n;
    T      = nframes;
    K      = k;
    lag    = lg;
    Nv     = T - lag;
    npairs = (long)n * (n - 1);
    GC_TRY(XT.alloc((size_t)n * T * 3));
    // psi[0 .. N_valid + 1]: a count clamped to N_valid indexes psi[N_valid + 1]
    GC_TRY(psi.alloc((size_t)Nv + 2));
    GC_TRY(X32.alloc((size_t)n * T));
    GC_TRY(eps.alloc((size_t)n));
    GC_TRY(cnt.alloc((size_t)Nv * npairs));
    const std::vector<double> tab = digamma_table(Nv + 1);
    GC_TRY_CUDA(cudaMemcpy(psi.p, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice));
    Q = q;
    if (Q <= 0)
        return GC_OK;
    Qp   = (Q + 31) & ~31;
    Lpad = ((Nv - 1) + 31) & ~31;
    const size_t rows = (size_t)n * Qp * Lpad;
    if (own_rows)
    {
        GC_TRY(SG.alloc(rows));
        GC_TRY(SM.alloc(rows));
        GC_TRY(PG.alloc(rows));
        GC_TRY(PM.alloc(rows));
    }
    GC_TRY(wres.alloc((size_t)Q * npairs));
    const double hq_want = 0.01 * (double)npairs * Nv + 4096.0;
    hq_cap               = (unsigned)(hq_want < 16777216.0 ? hq_want : 16777216.0);
    GC_TRY(hq.alloc(hq_cap));
    GC_TRY(hq_len.alloc(1));
    GC_TRY(walk_elems.alloc(1));
    GC_TRY(reasons.alloc(8));
    const std::vector<int> order = te_tile_order(n);
    GC_TRY(pair_order.alloc(order.size()));
    GC_TRY_CUDA(cudaMemcpy(pair_order.p, order.data(), sizeof(int) * order.size(), cudaMemcpyHostToDevice));
    return GC_OK;
}

TeParams TeTraj::desc(int* status, int b) const
{
    TeParams d{};
    d.X32        = X32.p;
    d.XT         = XT.p;
    d.eps_atom   = eps.p;
    d.SG         = SG.p;
    d.PG         = PG.p;
    d.SM         = SM.p;
    d.PM         = PM.p;
    d.natoms     = natoms;
    d.T          = T;
    d.lag        = lag;
    d.Nv         = Nv;
    d.K          = K;
    d.Lpad       = Lpad;
    d.Qp         = Qp;
    d.i0         = b * Q;
    d.Q          = std::min(Q, Nv - b * Q);
    d.pair_count = npairs;
    d.pair_order = pair_order.p;
    d.shift      = gc::walk_histogram_shift(K);
    d.cnt        = cnt.p;
    d.wres       = wres.p;
    d.hq         = hq.p;
    d.hq_len     = hq_len.p;
    d.hq_cap     = hq_cap;
    d.status     = status;
    d.walk_elems = walk_elems.p;
    d.reasons    = reasons.p;
    return d;
}

TeParams TeTraj::desc_rows(int* status, int b, float* SG_, uint16_t* PG_, float* SM_, uint16_t* PM_) const
{
    TeParams d = desc(status, b);
    d.SG       = SG_;
    d.PG       = PG_;
    d.SM       = SM_;
    d.PM       = PM_;
    return d;
}

size_t TeTraj::block_row_bytes() const
{
    const size_t e = (size_t)natoms * Qp * Lpad;
    auto         a = [](size_t b) { return (b + 255) & ~(size_t)255; };
    return 2 * a(e * sizeof(float)) + 2 * a(e * sizeof(uint16_t));
}

gc_status TeTraj::prepare(const double* d_xyz, int* status, cudaStream_t s) const
{
    gc::launch_transpose_components(d_xyz, natoms, T, XT.p, status, s);
    gc::launch_te_x32(XT.p, natoms, T, X32.p, eps.p, s);
    if (Q > 0)
    {
        GC_TRY_CUDA(cudaMemsetAsync(hq_len.p, 0, sizeof(unsigned), s));
        GC_TRY_CUDA(cudaMemsetAsync(reasons.p, 0, 8 * sizeof(unsigned), s));
        GC_TRY_CUDA(cudaMemsetAsync(walk_elems.p, 0, sizeof(unsigned long long), s));
    }
    GC_TRY_CUDA(cudaGetLastError());
    return GC_OK;
}

gc_status TeLaunch::build(const std::vector<std::vector<TeParams>>& wave_descs, const std::vector<TeParams>& traj_descs)
{
    int maxT = 0, maxNv = 0, maxK = 0;
    for (const auto& wv : wave_descs)
        for (const TeParams& d : wv)
        {
            maxT  = std::max(maxT, d.T);
            maxNv = std::max(maxNv, d.Nv);
            maxK  = std::max(maxK, d.K);
        }
    gc::walk_shape(maxT, &warps, &staged);
    const long long        chunk = (long long)warps * 4;
    std::vector<TeParams>  all;
    std::vector<long long> pre;
    std::vector<size_t>    dofs, pofs;
    for (const auto& wv : wave_descs)
    {
        dofs.push_back(all.size());
        pofs.push_back(pre.size());
        std::vector<long long> rp{0}, wp{0}, fp{0};
        for (const TeParams& d : wv)
        {
            all.push_back(d);
            const long long grp = (d.Q + 31) / 32;
            rp.push_back(rp.back() + 2LL * d.natoms * d.Q);
            wp.push_back(wp.back() + (grp + chunk - 1) / chunk * d.pair_count);
            fp.push_back(fp.back() + grp * d.pair_count);
        }
        pre.insert(pre.end(), rp.begin(), rp.end());
        pre.insert(pre.end(), wp.begin(), wp.end());
        pre.insert(pre.end(), fp.begin(), fp.end());
    }
    const size_t tofs = all.size();
    all.insert(all.end(), traj_descs.begin(), traj_descs.end());
    GC_TRY(descs.alloc(all.size()));
    GC_TRY(prefix.alloc(pre.size()));
    GC_TRY(counters.alloc(2 * wave_descs.size() + 1));
    GC_TRY_CUDA(cudaMemcpy(descs.p, all.data(), sizeof(TeParams) * all.size(), cudaMemcpyHostToDevice));
    GC_TRY_CUDA(cudaMemcpy(prefix.p, pre.data(), sizeof(long long) * pre.size(), cudaMemcpyHostToDevice));
    waves.clear();
    wave_rows.clear();
    for (size_t v = 0; v < wave_descs.size(); ++v)
    {
        const int n = (int)wave_descs[v].size();
        TeBatch   b{};
        b.d       = descs.p + dofs[v];
        b.rprefix = prefix.p + pofs[v];
        b.wprefix = b.rprefix + (n + 1);
        b.fprefix = b.wprefix + (n + 1);
        b.n       = n;
        b.maxT    = maxT;
        b.maxNv   = maxNv;
        b.maxK    = maxK;
        b.chunk   = (int)chunk;
        b.counter = counters.p + 2 * v;
        waves.push_back(b);
        wave_rows.push_back(pre[pofs[v] + n]);
    }
    fix       = TeBatch{};
    fix.d     = descs.p + tofs;
    fix.n     = (int)traj_descs.size();
    fix.maxT  = maxT;
    fix.maxNv = maxNv;
    fix.maxK  = maxK;
    return GC_OK;
}

gc_status TeLaunch::enqueue(int sms, cudaStream_t s)
{
    launches = 0;
    if (!waves.empty())
        GC_TRY_CUDA(cudaMemsetAsync(counters.p, 0, sizeof(unsigned long long) * 2 * waves.size(), s));
    for (const TeBatch& w : waves)
    {
        GC_TRY_CUDA(gc::launch_te_rows(w, wave_rows[(size_t)(&w - waves.data())], s));
        GC_TRY_CUDA(gc::launch_te_walk(w, warps, staged, sms, s));
        GC_TRY_CUDA(gc::launch_te_finish(w, sms, s));
        // the walk's task counter serves the count kernel
        GC_TRY_CUDA(cudaMemsetAsync(w.counter, 0, sizeof(unsigned long long), s));
        GC_TRY_CUDA(gc::launch_te_count(w, warps, staged, sms, s));
        launches += 4;
    }
    if (fix.n > 0)
    {
        GC_TRY_CUDA(gc::launch_te_fixup(fix, sms, s));
        launches += 2;
    }
    return GC_OK;
}

} // namespace host
} // namespace gc

struct gc_te_plan
{
    int                 device = 0, sms = 148;
    int                 natoms = 0, T = 0, K = 0, lag = 0, Nv = 0, path = GC_PATH_AUTO;
    long                npairs = 0; // ordered pairs
    bool                walk   = false;
    bool                wide   = false; // counts above 16 bits (exact kernel, two planes)
    cudaStream_t        stream = nullptr;
    cudaEvent_t         ev0 = nullptr, ev1 = nullptr, ev_done = nullptr;
    gc::host::TeTraj    tt;
    gc::host::TeLaunch  tl;
    DevBuf<int>         status;
    int                 launches = 0;
    long                handoffs = 0;
    double              walk_mean = 0.0;
};

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
    // more than 65535 valid frames: 32-bit counts, which only the exact
    // kernel writes (the walk stops at 16385 frames anyway)
    p->wide = p->Nv > 65535;
    if (p->wide)
        p->path = GC_PATH_EXACT_FP64;
    GC_TRY_CUDA(cudaDeviceGetAttribute(&p->sms, cudaDevAttrMultiProcessorCount, p->device));
    GC_TRY_CUDA(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
    GC_TRY_CUDA(cudaEventCreate(&p->ev0));
    GC_TRY_CUDA(cudaEventCreate(&p->ev1));
    GC_TRY_CUDA(cudaEventCreateWithFlags(&p->ev_done, cudaEventDisableTiming));
    GC_TRY(p->status.alloc(1));
    int Q = 0;
    if (p->walk)
    {
        int  warps  = 0;
        bool staged = false;
        gc::walk_shape(nframes, &warps, &staged);
        // sorted G and M rows of one query block within 16 GiB
        Q = ksg_block_queries(2 * natoms, p->Nv, 16.0 * (1 << 30), 32 * warps);
    }
    GC_TRY(p->tt.create(natoms, nframes, k, lag, Q));
    if (p->wide) // (n_xp, n_xfxp) then (n_ypxp, 0): two planes
        GC_TRY(p->tt.cnt.alloc((size_t)2 * p->Nv * p->npairs));
    if (p->walk)
    {
        std::vector<std::vector<gc::TeParams>> waves;
        for (int b = 0; b < p->tt.blocks(); ++b)
            waves.push_back({p->tt.desc(p->status.p, b)});
        GC_TRY(p->tl.build(waves, {p->tt.desc(p->status.p, 0)}));
    }
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
    GC_TRY_CUDA(cudaMemsetAsync(p->status.p, 0, sizeof(int), s));
    GC_TRY_CUDA(cudaMemsetAsync(d_te, 0, sizeof(double) * (size_t)n * n, s));
    GC_TRY(p->tt.prepare(d_xyz, p->status.p, s));
    p->launches = 2;
    GC_TRY_CUDA(cudaEventRecord(p->ev0, s));
    if (p->walk)
    {
        GC_TRY(p->tl.enqueue(p->sms, s));
        GC_TRY_CUDA(cudaEventRecord(p->ev1, s));
        GC_TRY_CUDA(gc::launch_te_reduce(p->tt.cnt.p, n, p->Nv, p->K, p->tt.psi.p, d_te, s));
        p->launches += p->tl.launches + 1;
    }
    else
    {
        if (p->path == GC_PATH_EXACT_FP64)
            gc::launch_te_exact(p->tt.XT.p, n, p->T, p->K, p->lag, p->tt.cnt.p, s, p->wide);
        else
            gc::launch_te_fast(p->tt.XT.p, p->tt.X32.p, p->tt.eps.p, n, p->T, p->K, p->lag, p->tt.cnt.p, s);
        GC_TRY_CUDA(cudaEventRecord(p->ev1, s));
        gc::launch_te_finalize(p->tt.cnt.p, n, p->T, p->K, p->lag, p->tt.psi.p, d_te, s, p->wide);
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
        GC_TRY_CUDA(cudaMemcpy(rc, p->tt.reasons.p, sizeof(rc), cudaMemcpyDeviceToHost));
        for (unsigned r : rc)
            p->handoffs += (long)r;
        unsigned long long we = 0;
        GC_TRY_CUDA(cudaMemcpy(&we, p->tt.walk_elems.p, sizeof(we), cudaMemcpyDeviceToHost));
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
        GC_TRY_CUDA(cudaMemcpy(c.data(), p->tt.cnt.p + (size_t)q * p->Nv, sizeof(uint2) * c.size(),
                               cudaMemcpyDeviceToHost));
    else // query-major [qi][npairs]
        GC_TRY_CUDA(cudaMemcpy2D(c.data(), sizeof(uint2), p->tt.cnt.p + q, sizeof(uint2) * p->npairs,
                                 sizeof(uint2), (size_t)p->Nv, cudaMemcpyDeviceToHost));
    std::vector<uint2> c2;
    if (p->wide) // the n_ypxp plane
    {
        c2.resize((size_t)p->Nv);
        GC_TRY_CUDA(cudaMemcpy2D(c2.data(), sizeof(uint2), p->tt.cnt.p + (size_t)p->Nv * p->npairs + q,
                                 sizeof(uint2) * p->npairs, sizeof(uint2), (size_t)p->Nv, cudaMemcpyDeviceToHost));
    }
    for (int i = 0; i < p->Nv; ++i)
    {
        const uint2 v = c[(size_t)i];
        if (n_xp)
            n_xp[i] = (int32_t)(p->wide ? v.x : (v.x & 0xFFFFu));
        if (n_xfxp)
            n_xfxp[i] = (int32_t)(p->wide ? v.y : (v.x >> 16));
        if (n_ypxp)
            n_ypxp[i] = (int32_t)(p->wide ? c2[(size_t)i].x : v.y);
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
