// Parameters of the KSG fast-path kernels (host and device).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace gc {

constexpr int kWalkWarps   = 32;       // most warps per walk CTA
#ifndef GC_FINISH_WARPS
#define GC_FINISH_WARPS 20 // a build-time setting for timing other finish CTA shapes
#endif
constexpr int kFinishWarps = GC_FINISH_WARPS; // warps per finish CTA
#ifndef GC_FINISH_ROUND
#define GC_FINISH_ROUND 1 // a build-time setting: 4-entry row groups loaded per band round
#endif
constexpr int kFinishRound = GC_FINISH_ROUND;
constexpr int kWalkBuckets = 128;      // per-lane histogram buckets
#ifndef GC_BAND_CAP
#define GC_BAND_CAP 20 // a build-time setting for timing other capacities
#endif
constexpr int kBandCap     = GC_BAND_CAP; // band entries kept per lane
constexpr int kBandSlotBytes = 14;     // v, s, d (f32), row position in its range (u16)
constexpr uint32_t kHandOver = 0xFFFFFFFFu; // cnt value of a query handed to the exact kernel

// Sorted marginal rows of one query block, transposed so that the 32
// queries of a warp read consecutive addresses: entry m of the row of
// (atom a, query i0 + iq) is element ((a * Lq + m / 4) * Qp + iq) * 4 + m % 4
// of S (distances) and of P (frames), Lq = Lpad / 4.
struct WalkParams
{
    const float4*   X32;      // [natoms][T] centred FP32 coordinates
    const double*   X64;      // [3*natoms][T] normalised rows (reference arithmetic)
    const float*    eps_atom; // [natoms] |d32 - d64| bound
    float*          S;
    uint16_t*       P;
    int             natoms, Lpad, Qp, i0, Q, T, K, box, rank_shift;
    long            pair_begin, pair_count;
    const int2*     pair_ab;    // optional [pair_count] (a1, a2) of an explicit pair list
    const int*      pair_order; // optional task order: task k computes local pair pair_order[k]
    int             shift;      // histogram bucket = 2^shift float ulps above the lower bound
    uint32_t*       cnt;        // [pair_count][T] n_x | n_y << 16, or kHandOver
    unsigned long long* wres;   // [pair_count][Q] walk results of the block (a warp's 32 queries side by side)
    unsigned long long* hq;     // hand-over queue: cnt indices pl * T + i
    unsigned*           hq_len;
    unsigned            hq_cap;
    int*                status;
    unsigned long long* walk_elems; // optional: total walked row entries
    unsigned*           reasons;    // optional [8]: hand-overs by cause
    // optional unsorted distance rows of the block: the distance from query
    // i0 + iq of atom a to frame j at U[((size_t)a * Qp + iq) * Tpad + j]
    // (GC_VARIANT_HBM_GATHER: the walk reads the other marginal here)
    float* U;
    int    Tpad;
};

// One launch over the query blocks of several trajectories (or of one): the
// launch's tasks are numbered across the descriptors, descriptor d owning
// tasks [prefix[d], prefix[d + 1]).  Every array lives in device memory.
struct WalkBatch
{
    const WalkParams*   d;       // [n]
    const long long*    rprefix; // [n + 1] row-sort tasks: natoms * Q per descriptor
    const long long*    wprefix; // [n + 1] walk tasks: ceil(groups / chunk) * pairs
    const long long*    fprefix; // [n + 1] finish tasks: query groups * pairs
    int                 n;
    int                 maxT;    // largest frame count (shared-memory layout)
    int                 maxK;    // largest k
    int                 chunk;   // query groups per walk task (shared by the CTA's warps)
    unsigned long long* counter; // [2] walk and finish task counters, zero at launch
};

// Bucket width of the walk histogram for k: about 1.3/k of the value
// (around eight entries per bucket near the k-th value), at least 2^17
// ulps so that the 128 buckets span two octaves above the lower bound.
inline int walk_histogram_shift(int K)
{
    const double target = 24.0 + __builtin_log2(0.67 / (double)K);
    int          s      = (int)(target + 0.5);
    return s < 17 ? 17 : (s > 21 ? 21 : s);
}

// Walk launch shape for trajectories of up to maxT frames: warps per CTA and
// whether the pair's coordinate rows are staged in shared memory.
void walk_shape(int maxT, int* warps, bool* staged);
// Largest walk warps per CTA that the staged layout allows (0: not staged).
int walk_max_staged_warps(int maxT);

// Each launcher returns the launch status (cudaGetLastError right after it).
cudaError_t launch_ksg_x32(const double* X64, int natoms, int T, float4* X32, float* eps_atom, cudaStream_t s);
cudaError_t launch_ksg_rows(const WalkBatch& b, long long rows, cudaStream_t s);
// gather_u: the other marginal's distances come from the descriptors' U rows;
// double_buffer: the double-buffered walk (two staged tasks per CTA).
cudaError_t launch_ksg_walk(const WalkBatch& b, int warps, bool staged, int sms, cudaStream_t s,
                            bool gather_u = false, bool double_buffer = false);
// Warps per CTA the double-buffered walk leaves room for (0: its rows do not fit).
int walk_max_db_warps(int maxT);
cudaError_t launch_ksg_finish(const WalkBatch& b, int sms, cudaStream_t s);
// Exact FP64 statistics for every queued hand-over of the batch's
// descriptors, then for any hand-over mark a queue could not hold (a scan of
// cnt).  One descriptor per trajectory.
cudaError_t launch_ksg_fixup(const WalkBatch& b, int sms, cudaStream_t s);

} // namespace gc
