// Parameters of the KSG fast-path kernels (host and device).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace gc {

constexpr int kWalkWarps   = 32;       // most warps per walk CTA
constexpr int kFinishWarps = 16;       // warps per finish CTA
constexpr int kWalkBuckets = 128;      // per-lane histogram buckets
constexpr int kBandCap     = 20;       // band entries kept per lane
constexpr int kBandSlotBytes = 18;     // v, s, d (f32), row position (i32), frame (u16)
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
    const float*    S;
    const uint16_t* P;
    int             Lpad, Qp, i0, Q, T, K, box;
    long            pair_begin, pair_count;
    const int2*     pair_ab; // optional [pair_count] (a1, a2) of an explicit pair list
    const int*      pair_order; // optional task order: task k computes local pair pair_order[k]
    int             staged;     // set by the launchers: coordinate rows staged in shared memory
    int             shift;   // histogram bucket = 2^shift float ulps above the lower bound
    uint32_t*       cnt;     // [T][pair_count] n_x | n_y << 16, or kHandOver
    unsigned long long* wres;         // [Q][pair_count] walk results of the block
    unsigned long long* hq;           // hand-over queue: cnt indices i * pair_count + pl
    unsigned*           hq_len;
    unsigned            hq_cap;
    unsigned long long* task_counter; // [2]: walk, finish
    int*                status;
    unsigned long long* walk_elems; // optional: total walked row entries
    unsigned*           reasons;    // optional [8]: hand-overs by cause
};

struct FixupParams
{
    const double* X64;
    int           T, K, box, rank_shift;
    long          pair_begin, pair_count;
    const int2*   pair_ab;
    uint32_t*     cnt;
    const unsigned long long* hq; // hand-over queue (may be null): entries are cnt indices
    const unsigned*           hq_len;
    unsigned                  hq_cap;
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

// Each launcher returns the launch status (cudaGetLastError right after it).
cudaError_t launch_ksg_x32(const double* X64, int natoms, int T, float4* X32, float* eps_atom, cudaStream_t s);
cudaError_t launch_ksg_rows(const float4* X32, int natoms, int T, int i0, int Q, int Qp, int Lpad, float* S,
                            uint16_t* P, cudaStream_t s);
cudaError_t launch_ksg_walk(const WalkParams& p, int sms, cudaStream_t s);
cudaError_t launch_ksg_finish(const WalkParams& p, int sms, cudaStream_t s);
// Exact FP64 statistics for every queued hand-over, then for any hand-over
// mark the queue could not hold (a scan of cnt).
cudaError_t launch_ksg_fixup(const FixupParams& p, int sms, cudaStream_t s);

} // namespace gc
