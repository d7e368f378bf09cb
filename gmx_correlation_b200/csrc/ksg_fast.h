// Parameters of the KSG fast-path kernels (host and device).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace gc {

constexpr int kWalkWarps = 24;

struct WalkParams
{
    const float4*   X32;       // [natoms][T] centred FP32 coordinates
    const double*   X64;       // [3*natoms][T] normalised rows (reference arithmetic)
    const float*    eps_atom;  // [natoms] |d32 - d64| bound
    const float*    S;         // [natoms][Q][Lpad] sorted marginal distances
    const uint16_t* P;         // [natoms][Q][Lpad] their frames
    int             Lpad, i0, Q, T, K, box;
    long            pair_begin, pair_count;
    const int2*     pair_ab;   // optional [pair_count] (a1, a2) of an explicit pair list
    int             shift, nb, bufcap, warp_smem;
    uint32_t*       cnt;        // [T][pair_count] n_x | n_y << 16
    unsigned long long* task_counter;
    unsigned long long* queue;  // hand-over entries pl << 16 | frame
    unsigned*       queue_len;
    unsigned        queue_cap;
    int*            status;
    unsigned long long* walk_elems; // optional: total walked row entries
    unsigned*           reasons;    // optional [8]: hand-overs by cause (1 walk > buffer,
                                    // 2 k-th bucket open-ended, 3 band, 4 ambiguous set, 5 max candidates)
};

struct QueueParams
{
    const double*       X64;
    int                 T, K, box, rank_shift;
    long                pair_begin, pair_count;
    const int2*         pair_ab;
    uint32_t*           cnt;
    const unsigned long long* queue;
    const unsigned*     queue_len;
    unsigned            queue_cap;
};

// Histogram shift / bucket count for k: buckets of 2^shift float ulps
// (about 1.3/k relative width, so about 10 entries around the k-th value)
// spanning at least four octaves above the lower bound.
inline void walk_histogram_shape(int K, int* shift, int* nb)
{
    double target = 24.0 + __builtin_log2(0.67 / (double)K);
    int    s      = (int)(target + 0.5);
    s             = s < 10 ? 10 : (s > 21 ? 21 : s);
    int n         = 1 << (27 - s);
    n             = n < 64 ? 64 : (n > 256 ? 256 : n);
    *shift        = s;
    *nb           = n;
}

// Per-warp shared-memory layout: hist[nb] u32 | bsw[bufcap] f32 |
// bdo[bufcap] f32 | bj[bufcap] u16 | (16-byte aligned) band values[64] f32,
// band frames[64] u32, band dx[64] f32, band dy[64] f32, ambiguous band
// slots[32] u32, candidate frames[32] u32, ambiguous dx64|dy64 [64] f64.
// bufcap is a multiple of 128.
__host__ __device__ inline int walk_list_offset(int nb, int bufcap) { return ((nb * 4 + bufcap * 10) + 15) & ~15; }
__host__ __device__ inline int walk_warp_smem(int nb, int bufcap) { return walk_list_offset(nb, bufcap) + 1280 + 512; }

// Each launcher returns the launch status (cudaGetLastError right after it).
cudaError_t launch_ksg_x32(const double* X64, int natoms, int T, float4* X32, float* eps_atom, cudaStream_t s);
cudaError_t launch_ksg_rows(const float4* X32, int natoms, int T, int i0, int Q, int Lpad, float* S, uint16_t* P,
                            cudaStream_t s);
cudaError_t launch_ksg_walk(const WalkParams& p, int sms, cudaStream_t s);
cudaError_t launch_ksg_queue(const QueueParams& p, int sms, cudaStream_t s);

} // namespace gc
