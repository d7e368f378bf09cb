// Host side of the transfer-entropy walk, shared by the single-trajectory
// plan (te_host.cpp) and the batched entry point (corr_batch.cpp).  Not
// public ABI.
#pragma once

#include "gmx_corr_b200.h"
#include "host_common.h"
#include "te_walk.h"

#include <vector>

namespace gc {
namespace host {

// Device workspace of one trajectory at one lag: raw coordinates (FP64
// component-major and centred FP32), the digamma table, the per-query
// counts, and for the walk the G and M rows of one query block of Q
// queries, the walk results, the hand-over queue and counters.
struct TeTraj
{
    int      natoms = 0, T = 0, K = 0, lag = 0, Nv = 0;
    long     npairs = 0; // ordered pairs
    int      Q = 0, Qp = 0, Lpad = 0;
    unsigned hq_cap = 0;
    PoolBuf<double>             XT, psi;
    PoolBuf<float4>             X32;
    PoolBuf<float>              eps, SG, SM;
    PoolBuf<uint2>              cnt;
    PoolBuf<uint16_t>           PG, PM;
    PoolBuf<unsigned long long> wres, hq, walk_elems;
    PoolBuf<unsigned>           hq_len, reasons;
    PoolBuf<int>                pair_order;

    // Q > 0: the walk's workspace for query blocks of Q queries; Q == 0: the
    // brute-force kernels' (coordinates, counts and digamma table only).
    // own_rows false: the G and M rows live elsewhere (a batch's shared
    // arena) and are passed to desc_rows.
    gc_status create(int natoms, int T, int K, int lag, int Q, bool own_rows = true);
    int       blocks() const { return Q > 0 ? (Nv + Q - 1) / Q : 0; }
    // Descriptor of query block b; the per-trajectory (fix-up) descriptor is block 0's.
    TeParams desc(int* status, int b) const;
    // The same with the block's rows at the given addresses.
    TeParams desc_rows(int* status, int b, float* SG_, uint16_t* PG_, float* SM_, uint16_t* PM_) const;
    // Bytes of one block's G and M rows (256-byte aligned parts).
    size_t block_row_bytes() const;
    // Transpose and FP32 copy of device coordinates d_xyz, then the counters
    // cleared (stream-ordered; no allocation, graph-capturable).
    gc_status prepare(const double* d_xyz, int* status, cudaStream_t s) const;
};

// Sorted rows of a TE query block: bytes per query of a trajectory.
double te_row_bytes_per_query(int natoms, int Nv);

// Device tables of a sequence of waves (one launch of the row sort, the
// walk, the finish and the count per wave over that wave's descriptors) and
// of the fix-up over one descriptor per trajectory.
struct TeLaunch
{
    DevBuf<TeParams>           descs;
    DevBuf<long long>          prefix;
    DevBuf<unsigned long long> counters;
    std::vector<TeBatch>       waves;
    std::vector<long long>     wave_rows;
    TeBatch                    fix{};
    int                        warps = 0;
    bool                       staged = false;
    int                        launches = 0;

    gc_status build(const std::vector<std::vector<TeParams>>& wave_descs, const std::vector<TeParams>& traj_descs);
    // Enqueues every wave and the fix-up (no allocation, graph-capturable).
    gc_status enqueue(int sms, cudaStream_t s);
};

} // namespace host
} // namespace gc
