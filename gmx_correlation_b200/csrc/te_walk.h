// Parameters of the transfer-entropy fast path (host and device).
//
// For an ordered pair (target a1, source a2) and query qi < N_valid the 9-D
// max-norm distance of te_matrix (lib/transfer_entropy.cpp:114-204) is
//   J(qi, j) = max(G(qi, j), Y(qi, j)),
//   G(qi, j) = max(D1(qi + lag, j + lag), D1(qi, j))   (target future, past)
//   Y(qi, j) = D2(qi, j)                                (source)
// with Da the 3-D max-norm distance of atom a.  G depends on the target
// alone and Y on the source alone, so each (atom, query) has two sorted
// rows shared by every pair it takes part in: its G row (the 6-D embedding
// distances) and its M row (the 3-D distances Da(qi, j), j < N_valid).  The
// counts are n_xfxp = #{G < eps}, n_xp = #{D1 < eps} (binary searches in
// the target's G and M rows) and n_ypxp = #{max(D1, Y) < eps}.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace gc {

constexpr int kTeBandCap = 24; // band entries kept per lane in the finish kernel
#ifndef GC_TE_FINISH_WARPS
#define GC_TE_FINISH_WARPS 24 // a build-time setting for timing other finish CTA shapes
#endif
constexpr int kTeFinishWarps = GC_TE_FINISH_WARPS; // warps per TE finish CTA

// One query block of one trajectory.  Entry m of the G row of (atom a,
// query i0 + iq) is element ((a * Lq + m / 4) * Qp + iq) * 4 + m % 4 of
// SG / PG (distance / frame), Lq = Lpad / 4; the M rows likewise in SM / PM.
struct TeParams
{
    const float4*   X32;      // [natoms][T] centred FP32 raw coordinates
    const double*   XT;       // [3 * natoms][T] raw FP64 coordinates, component-major
    const float*    eps_atom; // [natoms] |d32 - d64| bound of the atom's 3-D distances
    float*          SG;
    uint16_t*       PG;
    float*          SM;
    uint16_t*       PM;
    int             natoms, T, lag, Nv, K, Lpad, Qp, i0, Q;
    long            pair_count; // ordered pairs q = a1 * (natoms - 1) + (a2 < a1 ? a2 : a2 - 1)
    const int*      pair_order; // walk / finish task k computes ordered pair pair_order[k]
    int             shift;      // walk histogram bucket = 2^shift float ulps above the lower bound
    uint2*          cnt;        // [pair_count][Nv]: (n_xp | n_xfxp << 16, n_ypxp), or kTeHandOver in .x
    unsigned long long* wres;   // [pair_count][Q] walk results of the block
    unsigned long long* hq;     // hand-over queue: cnt indices q * Nv + qi
    unsigned*           hq_len;
    unsigned            hq_cap;
    int*                status;
    unsigned long long* walk_elems; // optional: total walked row entries
    unsigned*           reasons;    // optional [8]: hand-overs by cause
};

constexpr uint32_t kTeHandOver = 0xFFFFFFFFu;
// Between te_finish_kernel and te_count_kernel cnt.y holds the prefix length
// to enumerate for n_ypxp, with this bit set when it is the target's M row.
constexpr uint32_t kTeCountOn1 = 1u << 16;

// One launch over the query blocks of several trajectories (or of one), as
// WalkBatch for the KSG kernels.  Every array lives in device memory.
struct TeBatch
{
    const TeParams*     d;       // [n]
    const long long*    rprefix; // [n + 1] row-sort tasks: 2 * natoms * Q per descriptor
    const long long*    wprefix; // [n + 1] walk tasks: ceil(groups / chunk) * pairs
    const long long*    fprefix; // [n + 1] finish tasks: query groups * pairs
    int                 n;
    int                 maxT;  // largest frame count (shared-memory layout)
    int                 maxNv; // largest row length + 1
    int                 maxK;  // largest k
    int                 chunk; // query groups per walk task
    unsigned long long* counter; // [2] walk and finish task counters, zero at launch
};

cudaError_t launch_te_rows(const TeBatch& b, long long rows, cudaStream_t s);
cudaError_t launch_te_walk(const TeBatch& b, int warps, bool staged, int sms, cudaStream_t s);
cudaError_t launch_te_finish(const TeBatch& b, int sms, cudaStream_t s);
// n_ypxp of every (pair, query) the finish settled (its walk launch shape).
cudaError_t launch_te_count(const TeBatch& b, int warps, bool staged, int sms, cudaStream_t s);
// Exact FP64 statistics of every queued hand-over of the trajectories'
// descriptors, then of any mark a full queue could not hold.
cudaError_t launch_te_fixup(const TeBatch& b, int sms, cudaStream_t s);
// te[a1 * natoms + a2] = mean over qi of psi[k] + psi[n_xp + 1] - psi[n_xfxp + 1]
// - psi[n_ypxp + 1], summed in query order (lib/transfer_entropy.cpp:195-204).
cudaError_t launch_te_reduce(const uint2* cnt, int natoms, int Nv, int K, const double* psi, double* te_mat,
                             cudaStream_t s);

} // namespace gc
