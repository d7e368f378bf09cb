// Host side of the KSG fast path: per-trajectory workspaces, the device
// descriptor tables of a launch sequence, and the walk configurations the
// autotuner found.

#include "ksg_host.h"
#include "gc_geom.h"
#include "gc_internal.h"

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>

namespace gc {
namespace host {

int ksg_block_queries(int natoms, int T, double budget, int quantum, double extra_bytes_per_entry)
{
    const int    Lpad = ((T - 1) + 31) & ~31;
    const double row  = (double)natoms * Lpad * (6.0 + extra_bytes_per_entry);
    long         q    = (long)(budget / row) / 32 * 32;
    q                 = q < 32 ? 32 : q;
    if (q >= T)
        return T;
    // whole rounds of the walk CTA's warps: a block of q queries gives each
    // pair q / 32 query groups, which the CTA's warps take one at a time
    if (quantum > 32 && q >= quantum)
        q = q / quantum * quantum;
    return (int)q;
}

gc_status KsgTraj::create(int n, int nframes, int k, long pb, long pc, const int64_t* lst, const int2* d_ab, int q,
                          int tile, bool unsorted_rows, bool own_rows)
{
    natoms     = n;
    T          = nframes;
    K          = k;
    pair_begin = pb;
    pair_count = pc;
    d_pair_ab  = d_ab;
    Q          = q;
    Qp         = (Q + 31) & ~31;
    Lpad       = ((T - 1) + 31) & ~31;
    shift      = walk_histogram_shift(k);
    list.clear();
    if (lst)
        list.assign(lst, lst + pc);
    GC_TRY(X32.alloc((size_t)natoms * T));
    GC_TRY(eps.alloc((size_t)natoms));
    if (own_rows)
    {
        GC_TRY(S.alloc((size_t)natoms * Qp * Lpad));
        GC_TRY(P.alloc((size_t)natoms * Qp * Lpad));
    }
    else
    {
        S.reset();
        P.reset();
    }
    Tpad = (T + 3) & ~3;
    if (unsorted_rows)
        GC_TRY(U.alloc((size_t)natoms * Qp * Tpad));
    else
        U.reset();
    GC_TRY(wres.alloc((size_t)Q * (pc > 0 ? pc : 1)));
    // hand-over queue: ample for the rare hand-overs; overflow is caught by
    // the fix-up's scan of the counts
    const double hq_want = 0.01 * (double)pc * T + 4096.0;
    hq_cap               = (unsigned)(hq_want < 16777216.0 ? hq_want : 16777216.0);
    GC_TRY(hq.alloc(hq_cap));
    GC_TRY(hq_len.alloc(1));
    GC_TRY(walk_elems.alloc(1));
    GC_TRY(reasons.alloc(8));
    pair_tile = 0;
    return set_pair_tile(tile);
}

gc_status KsgTraj::set_pair_tile(int tile)
{
    if (tile == pair_tile || pair_count <= 0)
    {
        pair_tile = tile;
        return GC_OK;
    }
    // Walk tasks visit the pairs tile by tile (tile x tile atoms), so the
    // sorted rows of the atoms the running tasks read stay in L2.
    int sh = 0;
    while ((1 << sh) < tile)
        ++sh;
    std::vector<long long> key((size_t)pair_count);
    for (long q = 0; q < pair_count; ++q)
    {
        int a1, a2;
        gc::pair_from_index(list.empty() ? pair_begin + q : list[(size_t)q], &a1, &a2);
        key[(size_t)q] = (((long long)(a1 >> sh) * 65536 + (a2 >> sh)) << 32) | (long long)q;
    }
    std::sort(key.begin(), key.end());
    std::vector<int> order((size_t)pair_count);
    for (long q = 0; q < pair_count; ++q)
        order[(size_t)q] = (int)(key[(size_t)q] & 0xFFFFFFFFll);
    if (!pair_order.p)
        GC_TRY(pair_order.alloc((size_t)pair_count));
    GC_TRY_CUDA(cudaMemcpy(pair_order.p, order.data(), sizeof(int) * order.size(), cudaMemcpyHostToDevice));
    pair_tile = tile;
    return GC_OK;
}

WalkParams KsgTraj::desc(const double* X, uint32_t* cnt, int* status, int b) const
{
    WalkParams w{};
    w.X32        = X32.p;
    w.X64        = X;
    w.eps_atom   = eps.p;
    w.S          = S.p;
    w.P          = P.p;
    w.natoms     = natoms;
    w.Lpad       = Lpad;
    w.Qp         = Qp;
    w.i0         = b * Q;
    w.Q          = std::min(Q, T - b * Q);
    w.T          = T;
    w.K          = K;
    w.box        = ksg_box_count(T, K);
    w.rank_shift = rank_top_shift(w.box, T);
    w.pair_begin = pair_begin;
    w.pair_count = pair_count;
    w.pair_ab    = d_pair_ab;
    w.pair_order = pair_order.p;
    w.shift      = shift;
    w.cnt        = cnt;
    w.wres       = wres.p;
    w.hq         = hq.p;
    w.hq_len     = hq_len.p;
    w.hq_cap     = hq_cap;
    w.status     = status;
    w.walk_elems = walk_elems.p;
    w.reasons    = reasons.p;
    w.U          = U.p;
    w.Tpad       = Tpad;
    return w;
}

WalkParams KsgTraj::desc_rows(const double* X, uint32_t* cnt, int* status, int b, float* S_, uint16_t* P_) const
{
    WalkParams w = desc(X, cnt, status, b);
    w.S          = S_;
    w.P          = P_;
    return w;
}

size_t KsgTraj::block_row_bytes() const
{
    const size_t e = (size_t)natoms * Qp * Lpad;
    auto         a = [](size_t b) { return (b + 255) & ~(size_t)255; };
    return a(e * sizeof(float)) + a(e * sizeof(uint16_t));
}

gc_status KsgTraj::clear(cudaStream_t s)
{
    GC_TRY_CUDA(cudaMemsetAsync(reasons.p, 0, 8 * sizeof(unsigned), s));
    GC_TRY_CUDA(cudaMemsetAsync(walk_elems.p, 0, sizeof(unsigned long long), s));
    GC_TRY_CUDA(cudaMemsetAsync(hq_len.p, 0, sizeof(unsigned), s));
    return GC_OK;
}

gc_status KsgLaunch::build(const std::vector<std::vector<WalkParams>>& wave_descs,
                           const std::vector<WalkParams>& traj_descs, const WalkConfig& c)
{
    cfg = c;
    // descriptor table: every wave's descriptors, then the per-trajectory ones
    std::vector<WalkParams> all;
    std::vector<long long>  pre;
    std::vector<size_t>     dofs, pofs;
    int                     maxT = 0, maxK = 0;
    for (const auto& wv : wave_descs)
    {
        dofs.push_back(all.size());
        pofs.push_back(pre.size());
        long long r = 0, w = 0, f = 0;
        std::vector<long long> rp{0}, wp{0}, fp{0};
        for (const WalkParams& d : wv)
        {
            all.push_back(d);
            maxT                 = std::max(maxT, d.T);
            maxK                 = std::max(maxK, d.K);
            const long long grp  = (d.Q + 31) / 32;
            r += (long long)d.natoms * d.Q;
            const long long chunk = (long long)cfg.walk_warps * cfg.chunk_mult;
            w += (grp + chunk - 1) / chunk * d.pair_count;
            f += grp * d.pair_count;
            rp.push_back(r);
            wp.push_back(w);
            fp.push_back(f);
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
    GC_TRY_CUDA(cudaMemcpy(descs.p, all.data(), sizeof(WalkParams) * all.size(), cudaMemcpyHostToDevice));
    GC_TRY_CUDA(cudaMemcpy(prefix.p, pre.data(), sizeof(long long) * pre.size(), cudaMemcpyHostToDevice));
    waves.clear();
    wave_rows.clear();
    for (size_t v = 0; v < wave_descs.size(); ++v)
    {
        const int  n = (int)wave_descs[v].size();
        WalkBatch  b{};
        b.d        = descs.p + dofs[v];
        b.rprefix  = prefix.p + pofs[v];
        b.wprefix  = b.rprefix + (n + 1);
        b.fprefix  = b.wprefix + (n + 1);
        b.n        = n;
        b.maxT     = maxT;
        b.maxK     = maxK;
        b.chunk    = cfg.walk_warps * cfg.chunk_mult;
        b.counter  = counters.p + 2 * v;
        waves.push_back(b);
        wave_rows.push_back(pre[pofs[v] + n]);
    }
    fix      = WalkBatch{};
    fix.d    = descs.p + tofs;
    fix.n    = (int)traj_descs.size();
    fix.maxT = maxT;
    fix.maxK = maxK;
    return GC_OK;
}

gc_status KsgLaunch::enqueue(int sms, cudaStream_t s, int first_wave, int last_wave, bool fixup)
{
    if (last_wave < 0)
        last_wave = (int)waves.size() - 1;
    launches = 0;
    if (!waves.empty())
        GC_TRY_CUDA(cudaMemsetAsync(counters.p, 0, sizeof(unsigned long long) * 2 * waves.size(), s));
    for (int v = first_wave; v <= last_wave; ++v)
    {
        GC_TRY_CUDA(launch_ksg_rows(waves[(size_t)v], wave_rows[(size_t)v], s));
        GC_TRY_CUDA(launch_ksg_walk(waves[(size_t)v], cfg.walk_warps, cfg.staged, sms, s, cfg.gather_u,
                                    cfg.double_buf));
        GC_TRY_CUDA(launch_ksg_finish(waves[(size_t)v], sms, s));
        launches += 3;
    }
    if (fixup && fix.n > 0)
    {
        GC_TRY_CUDA(launch_ksg_fixup(fix, sms, s));
        launches += 2;
    }
    return GC_OK;
}

namespace {
std::mutex                              g_cfg_mutex;
std::map<std::pair<int, int>, WalkConfig> g_cfg; // (frames / 256, k) -> tuned configuration
} // namespace

WalkConfig walk_config(int maxT, int k)
{
    {
        std::lock_guard<std::mutex> lock(g_cfg_mutex);
        const auto                  it = g_cfg.find({maxT / 256, k});
        if (it != g_cfg.end())
        {
            // tuned on trajectories of up to 255 fewer frames: the staged rows
            // of maxT frames may leave room for fewer warps
            WalkConfig c = it->second;
            if (c.double_buf && walk_max_db_warps(maxT) < c.walk_warps)
            {
                c.double_buf = false;
                walk_shape(maxT, &c.walk_warps, &c.staged);
            }
            else if (c.staged && !c.double_buf)
            {
                const int w = walk_max_staged_warps(maxT);
                if (w > 0)
                    c.walk_warps = std::min(c.walk_warps, w);
                else
                {
                    c.staged     = false;
                    c.walk_warps = kWalkWarps;
                }
            }
            return c;
        }
    }
    WalkConfig c;
    walk_shape(maxT, &c.walk_warps, &c.staged);
    c.pair_tile = 16;
    // the double-buffered walk where its two staged tasks leave room for 32
    // warps (rows up to about 2,090 frames): 82.9 against 89.2 ms on the
    // 247 x 2000 matrix, the per-task barrier's idle warps gone
    if (walk_max_db_warps(maxT) >= kWalkWarps)
    {
        c.double_buf = true;
        c.walk_warps = kWalkWarps;
    }
    return c;
}

void remember_walk_config(int maxT, int k, const WalkConfig& cfg)
{
    std::lock_guard<std::mutex> lock(g_cfg_mutex);
    g_cfg[{maxT / 256, k}] = cfg;
}

std::vector<WalkConfig> walk_candidates(int maxT)
{
    // Measured on 247 x 2000 and 128 x 5000 matrices: fewer warps than the
    // staged rows allow (24, 16, or two CTAs of 11-12 per SM) and chunks of
    // one group per warp were always slower, so the search spans the atom
    // tile and chunks of two or four groups per warp.
    std::vector<WalkConfig> out;
    const int               wmax = walk_max_staged_warps(maxT);
    std::vector<int>        warps;
    if (wmax > 0)
        warps.push_back(wmax);
    for (int tile : {16, 32})
        for (int mult : {2, 4})
        {
            if (warps.empty())
            {
                WalkConfig c;
                c.walk_warps = kWalkWarps;
                c.staged     = false;
                c.pair_tile  = tile;
                c.chunk_mult = mult;
                out.push_back(c);
            }
            for (int w : warps)
            {
                WalkConfig c;
                c.walk_warps = w;
                c.staged     = true;
                c.pair_tile  = tile;
                c.chunk_mult = mult;
                out.push_back(c);
            }
            if (walk_max_db_warps(maxT) >= kWalkWarps)
            {
                WalkConfig c;
                c.walk_warps = kWalkWarps;
                c.staged     = true;
                c.double_buf = true;
                c.pair_tile  = tile;
                c.chunk_mult = mult;
                out.push_back(c);
            }
        }
    return out;
}

} // namespace host
} // namespace gc
