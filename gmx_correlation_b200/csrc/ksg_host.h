// Host side of the KSG fast path, shared by the single-trajectory plan
// (api.cpp) and the batched entry point (ksg_batch.cpp).  Not public ABI.
#pragma once

#include "gmx_corr_b200.h"
#include "host_common.h"
#include "ksg_fast.h"

#include <vector>

namespace gc {
namespace host {

// Launch configuration of the walk: warps per CTA, staging of the pair's
// coordinate rows, and the side of the atom tiles that order the pairs.
struct WalkConfig
{
    int  walk_warps = 0;
    bool staged     = false;
    int  pair_tile  = 16;
    int  chunk_mult = 4; // query groups per walk task = chunk_mult * walk_warps
    bool gather_u   = false; // other marginal from precomputed HBM rows (GC_VARIANT_HBM_GATHER)
    bool double_buf = false; // the double-buffered walk kernel
};

// Fast-path workspace of one trajectory (all pairs, a shard, or a list): the
// FP32 coordinates, the sorted rows of one query block, the walk results,
// the hand-over queue and the counters.  The prepared FP64 rows (X), the
// per-query counts (cnt) and the status word belong to the caller.
struct KsgTraj
{
    int      natoms = 0, T = 0, K = 0;
    long     pair_begin = 0, pair_count = 0;
    int      Q = 0, Qp = 0, Lpad = 0, shift = 0, pair_tile = 0;
    unsigned hq_cap = 0;
    const int2* d_pair_ab = nullptr; // explicit list as (a1, a2) (owned by the caller), or null
    std::vector<long> list;          // host copy of the list's pair indices (for the tile order)
    PoolBuf<float4>             X32;
    PoolBuf<float>              eps, S;
    PoolBuf<uint16_t>           P;
    PoolBuf<unsigned long long> wres, hq, walk_elems;
    PoolBuf<unsigned>           hq_len, reasons;
    PoolBuf<int>                pair_order;
    PoolBuf<float>              U; // unsorted distance rows (GC_VARIANT_HBM_GATHER only)
    int                         Tpad = 0;

    // Sizes the workspace for query blocks of Q frames (a multiple of 32, or T).
    // own_rows false: the sorted rows live elsewhere (a batch's shared arena)
    // and are passed to desc_rows.
    gc_status create(int natoms, int T, int K, long pair_begin, long pair_count, const int64_t* list,
                     const int2* d_pair_ab, int Q, int pair_tile, bool unsorted_rows = false, bool own_rows = true);
    // Reorders the pairs by atom tiles of the given side (device upload).
    gc_status set_pair_tile(int tile);
    int       blocks() const { return (T + Q - 1) / Q; }
    // Descriptor of query block b (first query b * Q).
    WalkParams desc(const double* X, uint32_t* cnt, int* status, int b) const;
    // The same with the block's sorted rows at the given addresses.
    WalkParams desc_rows(const double* X, uint32_t* cnt, int* status, int b, float* S_, uint16_t* P_) const;
    // Bytes of one block's sorted rows (256-byte aligned parts: distances, then frames).
    size_t block_row_bytes() const;
    // Clears the counters and the hand-over queue (stream-ordered).
    gc_status clear(cudaStream_t s);
};

// Query-block size for one trajectory whose sorted rows of a block must fit
// in budget bytes; when the trajectory needs several blocks, a multiple of
// quantum queries if the budget allows one.
int ksg_block_queries(int natoms, int T, double budget, int quantum = 32, double extra_bytes_per_entry = 0.0);

// Device tables of a sequence of waves: each wave one launch of the row
// sort, the walk and the finish over the descriptors of that wave; then one
// fix-up over one descriptor per trajectory.
struct KsgLaunch
{
    DevBuf<WalkParams>         descs;
    DevBuf<long long>          prefix;
    DevBuf<unsigned long long> counters;
    std::vector<WalkBatch>     waves;
    std::vector<long long>     wave_rows;
    WalkBatch                  fix{};
    WalkConfig                 cfg;
    int                        launches = 0;

    gc_status build(const std::vector<std::vector<WalkParams>>& wave_descs, const std::vector<WalkParams>& traj_descs,
                    const WalkConfig& cfg);
    // Enqueues every wave and the fix-up (no allocation, graph-capturable).
    gc_status enqueue(int sms, cudaStream_t s, int first_wave = 0, int last_wave = -1, bool fixup = true);
};

// The walk configuration to use for trajectories of up to maxT frames and k:
// the autotuned one when known, else the widest staged shape.
WalkConfig walk_config(int maxT, int k);
// Records a tuned configuration.
void remember_walk_config(int maxT, int k, const WalkConfig& cfg);
// Candidate configurations for the autotuner.
std::vector<WalkConfig> walk_candidates(int maxT);

} // namespace host
} // namespace gc
