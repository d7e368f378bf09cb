// Internal launcher interface between the host library (api.cpp) and the
// CUDA translation units.  Not part of the public ABI.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace gc {

// Largest frame count the C ABI accepts (32-bit count and index arithmetic).
constexpr int kMaxFrames = 1 << 24;

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
// Sets kStatNonFinite when any of the n doubles of already-normalised rows is not finite.
void launch_ksg_check_rows(const double* X, long n, int* status, cudaStream_t s);

// Exact FP64 brute-force KSG statistics for pairs [pair_begin, pair_begin+pair_count):
// writes cnt[pl * T + i] = n_x | n_y << 16 for every query frame i, or with
// cnt_y (wide counts, any frame count) cnt[pl * T + i] = n_x and
// cnt_y[pl * T + i] = n_y.
// pair_ab (optional): device (a1, a2) per local pair index of an explicit list.
void launch_ksg_exact(const double* X, int T, int K, long pair_begin, long pair_count, uint32_t* cnt,
                      cudaStream_t s, const int2* pair_ab = nullptr, uint32_t* cnt_y = nullptr);

// MI per pair from the per-query counts, summed in frame order as mir_xnyn does.
void launch_ksg_finalize(const uint32_t* cnt, long pair_count, int T, int K, const double* psi,
                         double* pair_mi, cudaStream_t s, const uint32_t* cnt_y = nullptr);

// ---- Transfer entropy ------------------------------------------------------
// xyz [natoms][T][3] -> XT [3*natoms][T] (component-major copy, raw values),
// status bits on non-finite input.
void launch_transpose_components(const double* xyz, int natoms, int T, double* XT, int* status,
                                 cudaStream_t s);
// Exact FP64 TE statistics for every ordered pair; cnt[qi * npairs + q] =
// {n_xp | n_xfxp << 16, n_ypxp}, or with wide (any frame count) {n_xp,
// n_xfxp} there and {n_ypxp, 0} at cnt[(Nv + qi) * npairs + q].
void launch_te_exact(const double* XT, int natoms, int T, int K, int lag, uint2* cnt, cudaStream_t s,
                     bool wide = false);
// FP32 copy of the raw coordinates and per-atom error bounds for launch_te_fast.
void launch_te_x32(const double* XT, int natoms, int T, float4* X32, float* eps_atom, cudaStream_t s);
// TE statistics from FP32 distances with exact FP64 repair (same counts as launch_te_exact).
void launch_te_fast(const double* XT, const float4* X32, const float* eps_atom, int natoms, int T, int K, int lag,
                    uint2* cnt, cudaStream_t s);
// TE per ordered pair q = a1*(natoms-1) + (a2 < a1 ? a2 : a2-1), into te[a1*n+a2].
void launch_te_finalize(const uint2* cnt, int natoms, int T, int K, int lag, const double* psi,
                        double* te_mat, cudaStream_t s, bool wide = false);

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

// ---- Learned screen --------------------------------------------------------
constexpr int kScreenStat = 16; // doubles of per-atom statistics
constexpr int kScreenBase = 23; // scalar features before the histogram part
constexpr int kScreenHist = 64; // raw 8x8 histogram cells
constexpr int kScreenComp = 17; // histogram principal components kept
constexpr int kScreenIn   = kScreenBase + kScreenComp; // 40 network inputs

// Feature rows of pairs [pair_begin, pair_begin + pair_count) (or of the
// pair_ab list): out[pl][width], width = kScreenIn with a basis pca
// (mean[64] then comp[ncomp][64]), else kScreenBase + kScreenHist raw.
// stats: [natoms][kScreenStat] doubles, bins: [natoms][T] bytes (scratch).
cudaError_t launch_screen_features(const double* xyz, int natoms, int T, int K, long pair_begin, long pair_count,
                                   const int2* pair_ab, const float* pca, int ncomp, double* stats,
                                   unsigned char* bins, float* out, int width, cudaStream_t s);

// Network: kScreenIn -> kMlpHidden x 3 (GELU) -> 1, per ensemble member.
constexpr int  kMlpHidden = 128;
constexpr long kMlpOffW1  = 0;
constexpr long kMlpOffB1  = kMlpOffW1 + (long)kMlpHidden * kScreenIn;
constexpr long kMlpOffW2  = kMlpOffB1 + kMlpHidden;
constexpr long kMlpOffB2  = kMlpOffW2 + (long)kMlpHidden * kMlpHidden;
constexpr long kMlpOffW3  = kMlpOffB2 + kMlpHidden;
constexpr long kMlpOffB3  = kMlpOffW3 + (long)kMlpHidden * kMlpHidden;
constexpr long kMlpOffW4  = kMlpOffB3 + kMlpHidden;
constexpr long kMlpOffB4  = kMlpOffW4 + kMlpHidden;
constexpr long kMlpParams = kMlpOffB4 + 1;
constexpr long kMlpStride = (kMlpParams + 63) / 64 * 64; // floats per member

// C[z] (+)= A[z] . B[z]^T with A(m,k) = A[z*sAz + m*sAm + k*sAk] and
// B(n,k) = B[z*sBz + n*sBn + k*sBk]; operands rounded to BF16, FP32
// accumulation on the tensor cores.  Epilogue: kEpiStore writes (or adds,
// when accumulate) the product to C[z*sCz + m*ldc + n]; kEpiBias adds
// bias[z*sbz + n]; kEpiBiasGelu adds the bias, keeps the pre-activation in
// C and writes GELU of it to H (same layout as C).
enum
{
    kEpiStore    = 0,
    kEpiBias     = 1,
    kEpiBiasGelu = 2
};
struct MlpGemm
{
    const float* A;
    long         sAz, sAm, sAk;
    const float* B;
    long         sBz, sBn, sBk;
    float*       C;
    long         sCz, ldc;
    const float* bias;
    long         sbz;
    float*       H;
    int          M, N, K, Z;
    int          epi, accumulate;
};
cudaError_t launch_mlp_gemm(const MlpGemm& g, cudaStream_t s);
// X[m][c] = (F[row][c] - mean[c]) / sd[c] with row = idx[base + m] (idx may
// be null: row = base + m); base = *step * M when step is non-null, else 0.
cudaError_t launch_mlp_gather(const float* F, const long* idx, const int* step, int M, const float* mean,
                              const float* sd, float* X, cudaStream_t s);
// Targets gathered the same way; dY[z][m] = 2 (Y[z][m] - t) / M, and
// loss[z] += (Y - t)^2 / M.
cudaError_t launch_mlp_loss(const float* Y, const float* target, const long* idx, const int* step, int M, int Z,
                            float* dY, float* loss, cudaStream_t s);
// dZ = dH * GELU'(Zpre), elementwise over n elements.
cudaError_t launch_mlp_gelu_back(const float* Zpre, float* dH, long n, cudaStream_t s);
// db[z*sbz + c] = sum over m of dZ[z][m][c] (dZ: [Z][M][N]).
cudaError_t launch_mlp_colsum(const float* dZ, int M, int N, int Z, float* db, long sbz, cudaStream_t s);
// Adam over n parameters; hyper = {lr, beta1, beta2, eps}; t = *tstep + 1.
cudaError_t launch_mlp_adam(float* p, const float* g, float* m, float* v, long n, const float* hyper,
                            const int* tstep, cudaStream_t s);
// ++*counter for each pointer that is non-null (one thread).
cudaError_t launch_mlp_tick(int* a, int* b, cudaStream_t s);
// Ensemble mean and standard deviation (population) over Z members of Y[z][n].
cudaError_t launch_mlp_ensemble(const float* Y, long n, int Z, float* mean, float* sd, cudaStream_t s);

} // namespace gc
