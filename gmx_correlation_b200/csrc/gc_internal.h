// Internal launcher interface between the host library (api.cpp) and the
// CUDA translation units.  Not part of the public ABI.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace gc {

// Device status bits raised by kernels (checked by the host after a run).
enum : int
{
    kStatNonFinite    = 1,
    kStatZeroVariance = 2,
    kStatFallback     = 4, // fast path handed queries to the exact repair kernel
    kStatTimeout      = 8,
    kStatInternal     = 16,
    kStatQueueOverflow = 32 // more hand-overs than the queue holds: rerun exact
};

// Sets the calling thread's gc_last_error() text.
void set_last_error(const char* msg);

// ---- KSG -------------------------------------------------------------------
// xyz [natoms][T][3] (mean-centred) -> X [3*natoms][T] normalised, min-shifted
// (kraskov_prepare arithmetic), status bits on error.
void launch_ksg_prepare(const double* xyz, int natoms, int T, double* X, int* status, cudaStream_t s);

// Exact FP64 brute-force KSG statistics for pairs [pair_begin, pair_begin+pair_count):
// writes cnt[i * pair_count + pl] = n_x | n_y << 16 for every query frame i.
// pair_ab (optional): device (a1, a2) per local pair index of an explicit list.
void launch_ksg_exact(const double* X, int T, int K, long pair_begin, long pair_count, uint32_t* cnt,
                      cudaStream_t s, const int2* pair_ab = nullptr);

// MI per pair from the per-query counts, summed in frame order as mir_xnyn does.
void launch_ksg_finalize(const uint32_t* cnt, long pair_count, int T, int K, const double* psi,
                         double* pair_mi, cudaStream_t s);

// ---- Transfer entropy ------------------------------------------------------
// xyz [natoms][T][3] -> XT [3*natoms][T] (component-major copy, raw values),
// status bits on non-finite input.
void launch_transpose_components(const double* xyz, int natoms, int T, double* XT, int* status,
                                 cudaStream_t s);
// Exact FP64 TE statistics for every ordered pair; cnt[qi * npairs + q] =
// {n_xp | n_xfxp << 16, n_ypxp}.
void launch_te_exact(const double* XT, int natoms, int T, int K, int lag, uint2* cnt, cudaStream_t s);
// TE per ordered pair q = a1*(natoms-1) + (a2 < a1 ? a2 : a2-1), into te[a1*n+a2].
void launch_te_finalize(const uint2* cnt, int natoms, int T, int K, int lag, const double* psi,
                        double* te_mat, cudaStream_t s);

// ---- Gaussian and copula MI ------------------------------------------------
// xyz [natoms][T][3] -> XF [T][3*natoms] (frame-major), status on non-finite.
void launch_frame_major(const double* xyz, int natoms, int T, double* XF, int* status, cudaStream_t s);
// Copula transform (lib/gcmi.cpp:95-146) of XF into Z [T][3*natoms] (frame-major).
// zt: [T] probit table sqrt(2)*erfinv(2(t+0.5)/T - 1).
void launch_copula(const double* XF, int natoms, int T, double* zt, double* Z, cudaStream_t s);
// 3x3 co-moment blocks of every atom pair lo <= hi, summed over frames in
// order: blk[(hi*(hi+1)/2 + lo)*9 + r*3 + c] = sum_f V[f][lo*3+r] * V[f][hi*3+c].
void launch_blocks(const double* V, int natoms, int T, double* blk, cudaStream_t s);
// Per pair MI from the blocks.  mode 0: Gaussian (cov = sum / T, entropy
// form); mode 1: GCMI (cov = sum * (1.0/T), log-det form).  Writes the full
// symmetric matrix with diagonal 2000.
void launch_pair_logdet(const double* blk, int natoms, int T, int mode, double log2pi, double* mat,
                        cudaStream_t s);

} // namespace gc
