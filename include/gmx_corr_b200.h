/*
 * gmx_corr_b200.h -- C ABI of the B200 (sm_100a) all-pairs generalized
 * correlation library.
 *
 * Plain pointers and sizes only.  Every entry point returns a gc_status
 * (0 = success); gc_last_error() gives the message of the calling thread's
 * last failure.  There is no CPU fallback: without a usable CUDA device the
 * compute entry points fail with GC_ERR_NO_DEVICE.
 *
 * Coordinates are the reference's t_traj block (lib/correlation_core.h:31-37):
 * mean-centred doubles x[atom][frame][dim], dim = 3, passed either as one
 * contiguous block or as the per-atom row pointers t_traj::x holds.
 *
 * Matrix outputs are natoms*natoms doubles, row-major mat[a1*natoms + a2],
 * with the reference's conventions: zero fill, diagonal 2000 for the
 * symmetric estimators, both triangles written; transfer entropy is
 * mat[a1*natoms + a2] = TE(a2 -> a1) with a zero diagonal.
 */
#ifndef GMX_CORR_B200_H
#define GMX_CORR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int gc_status;

enum
{
    GC_OK                = 0,
    GC_ERR_INVALID       = 1, /* bad argument (the reference throws std::runtime_error) */
    GC_ERR_NO_DEVICE     = 2, /* no CUDA device usable by this library */
    GC_ERR_CUDA          = 3, /* a CUDA call failed */
    GC_ERR_ZERO_VARIANCE = 4, /* a coordinate component is constant over all frames */
    GC_ERR_NONFINITE     = 5, /* NaN or infinite coordinate */
    GC_ERR_OUT_OF_MEMORY = 6,
    GC_ERR_IO            = 7, /* file could not be written */
    GC_ERR_INTERNAL      = 8,
    GC_ERR_TIMEOUT       = 9  /* a bounded device-side wait ran out */
};

/* Which kernels compute the KSG / TE neighbour statistics. */
enum
{
    GC_PATH_AUTO       = 0, /* the fast FP32 path with exact FP64 repair */
    GC_PATH_EXACT_FP64 = 1, /* brute-force FP64 kernels for every query */
    GC_PATH_FAST       = 2  /* same as AUTO */
};

/* Zero-copy view of a t_traj: set exactly one of xyz / rows. */
typedef struct gc_traj_view
{
    int                  natoms;
    int                  nframes;
    const double*        xyz;  /* contiguous [natoms][nframes][3], or NULL */
    const double* const* rows; /* rows[atom] -> nframes*3 doubles (t_traj::x), or NULL */
} gc_traj_view;

typedef struct gc_opts
{
    int   device;     /* CUDA ordinal; -1 = the calling thread's current device */
    int   path;       /* GC_PATH_* */
    long  pair_begin; /* shard of the unordered pair list p = a1*(a1-1)/2 + a2 (a2 < a1) */
    long  pair_end;   /* one past the last pair; <= 0 means all pairs */
    void* stream;     /* cudaStream_t to order the work on, or NULL for the library's own */
    /* Optional per-query detail of the KSG estimator, host arrays laid out
     * [pair - pair_begin][frame]: the counts n_x, n_y that index psi
     * (x = atom a1, y = atom a2 of pair p, a1 > a2). */
    int32_t* detail_nx;
    int32_t* detail_ny;
    /* Optional explicit pair list (host array of pair indices
     * p = a1*(a1-1)/2 + a2): when non-NULL the KSG entry points compute
     * exactly these pairs, in this order, instead of [pair_begin, pair_end);
     * detail arrays and plan outputs then follow the list order. */
    const int64_t* pair_list;
    long           pair_list_len;
    /* GC_VARIANT_*: how the KSG fast path's walk obtains the distance of the
     * marginal it does not walk (results are identical either way). */
    int variant;
} gc_opts;

enum
{
    GC_VARIANT_DEFAULT    = 0, /* recomputed from the pair's coordinates staged in shared memory */
    GC_VARIANT_HBM_GATHER = 1  /* read from per-(atom, query) distance rows precomputed in HBM */
};

/* Fills *o with the defaults (device -1, GC_PATH_AUTO, all pairs). */
void gc_opts_init(gc_opts* o);

/* Message of the calling thread's last failure ("" if none). */
const char* gc_last_error(void);

/* Number of CUDA devices this library can use (0 when none). */
int gc_device_count(void);

/* 1 if a compute capability 10.x device (B200 class) is present, else 0.
 * Replaces gpu_available() / kraskov_gpu_probe()
 * (lib/correlation_core.cpp:313-322, lib/kraskov_gpu.cu:210-219). */
int gc_gpu_available(void);

/* KSG (Kraskov algorithm 2) mutual-information matrix, k nearest
 * neighbours.  Replaces kraskov_corrmatrix (lib/correlation_core.h:79,
 * lib/correlation_core.cpp:324-459) and kraskov_corrmatrix_gpu
 * (lib/kraskov_gpu.h:32).  With a pair shard only the shard's entries and
 * the diagonal are written; the rest stays zero.  mi: natoms*natoms. */
gc_status gc_ksg_matrix(const gc_traj_view* traj, int k, const gc_opts* opts, double* mi);

/* The same KSG matrix from rows that kraskov_prepare already normalised:
 * X [3*natoms][nframes] host doubles, component-major (comp = atom*3 + dim,
 * the order of t_kraskov::x) and psi [nframes+1] the digamma table the
 * neighbour counts index.  Replaces kraskov_corrmatrix_gpu
 * (lib/kraskov_gpu.h:32, lib/kraskov_gpu.cu:225-308), which takes the
 * prepared t_kraskov; unlike it there is no k <= 128 limit and exact ties
 * follow mir_xnyn's scan order.  A non-finite row value (what a constant
 * component becomes after z-scoring) gives GC_ERR_NONFINITE.  opts and mi
 * as for gc_ksg_matrix. */
gc_status gc_ksg_matrix_prepared(const double* X, const double* psi, int natoms, int nframes, int k,
                                 const gc_opts* opts, double* mi);

/* gc_ksg_matrix keeps the device workspace of its last call on each device
 * (a few GB at 247 atoms x 2000 frames) and reuses it when the next call has
 * the same shape (atoms, frames, k, path, pair range); explicit pair lists are
 * not kept.  gc_release_cache frees every kept workspace. */
void gc_release_cache(void);

/* KSG MI matrices of ntraj trajectories in one batched run: trajectory i
 * (its own atom and frame counts, nframes <= 16385) with k = ks[i] into
 * mi[i] (natoms_i * natoms_i, the conventions of gc_ksg_matrix).  The query
 * blocks of all trajectories share each launch of the row sort, walk and
 * finish kernels (tasks drawn from every trajectory through one counter),
 * the whole sequence runs as one captured CUDA graph, and the walk's launch
 * shape is autotuned on the first call for a shape class.  The device
 * workspace and graph of the last batch are kept for a repeated call with
 * the same shapes; gc_ksg_batch_release frees them.  No counterpart in the
 * reference, which handles one trajectory per run.  opts: device only. */
gc_status gc_ksg_batch(const gc_traj_view* trajs, const int* ks, int ntraj, const gc_opts* opts, double* const* mi);
void      gc_ksg_batch_release(void);

/* Gaussian (linearized) MI matrix.  Replaces gauss_corrmatrix
 * (lib/correlation_core.h:76, lib/correlation_core.cpp:280-311). */
gc_status gc_gauss_matrix(const gc_traj_view* traj, const gc_opts* opts, double* mi);

/* Transfer-entropy matrices of ntraj trajectories at one lag in one batched
 * run: trajectory i (its own atom and frame counts, nframes - lag <= 16385)
 * with k = ks[i] into te[i] (natoms_i * natoms_i, the conventions of
 * gc_te_matrix; all zeros when nframes - lag <= k, as in the reference).
 * The query blocks of all trajectories share each launch of the row sort,
 * walk, finish and count kernels, and the sequence runs as a captured CUDA
 * graph; the workspace and graph of the last batch (shapes and lag) are
 * kept for a repeated call (gc_te_batch_release frees them; the per-query
 * counts take 8 bytes per ordered pair and frame, about 22 GB for 16
 * trajectories of up to 400 atoms x 4000 frames, beside one arena of
 * sorted rows shared by all waves: 32 GiB, or one trajectory's largest query
 * block of at most 16 GiB where that is larger).  No counterpart in the reference, which computes te_matrix
 * per trajectory.  opts: device only. */
gc_status gc_te_batch(const gc_traj_view* trajs, const int* ks, int ntraj, int lag, const gc_opts* opts,
                      double* const* te);
void      gc_te_batch_release(void);

/* Gaussian-copula MI matrices of ntraj trajectories
 * in one captured CUDA graph, with the conventions of gc_gcmi_matrix.  The
 * last batch's workspace and graph are kept for a repeated call with the
 * same shapes; gc_gcmi_batch_release frees them.  No counterpart in the
 * reference (gcmi_corrmatrix is per trajectory).  opts: device only. */
gc_status gc_gcmi_batch(const gc_traj_view* trajs, int ntraj, const gc_opts* opts, double* const* mi);
void      gc_gcmi_batch_release(void);

/* Gaussian-copula MI matrix.  Replaces gcmi_corrmatrix (lib/gcmi.h:8-9,
 * lib/gcmi.cpp:246-317). */
gc_status gc_gcmi_matrix(const gc_traj_view* traj, const gc_opts* opts, double* mi);

/* Transfer-entropy matrix, mat[a1*n+a2] = TE(a2 -> a1, lag).  Replaces
 * te_matrix (lib/transfer_entropy.h:8-9, lib/transfer_entropy.cpp:63-221).
 * When nframes - lag <= k the matrix is all zeros, as in the reference. */
gc_status gc_te_matrix(const gc_traj_view* traj, int k, int lag, const gc_opts* opts, double* te);

/* ---- Device-resident transfer-entropy plan ------------------------------
 * Owns every device workspace of one (natoms, nframes, k, lag) shape;
 * gc_te_matrix runs one.  gc_te_plan_run reads device coordinates d_xyz
 * ([natoms][nframes][3] doubles) and writes the whole TE matrix to device
 * memory d_te (natoms*natoms, the conventions of gc_te_matrix), ordered on
 * `stream` (NULL = the plan's stream); nothing is synchronised.  The
 * default path sorts each atom's target-embedding and marginal distance
 * rows and walks them with FP32 distances and an exact FP64 repair (rows of
 * up to 16385 frames); GC_PATH_EXACT_FP64 and longer trajectories use the
 * brute-force kernels.  Requires natoms >= 2 and nframes - lag > k.
 * No counterpart type in the reference (te_matrix computes and returns). */
typedef struct gc_te_plan gc_te_plan;

gc_status gc_te_plan_create(int natoms, int nframes, int k, int lag, const gc_opts* opts, gc_te_plan** plan);
gc_status gc_te_plan_run(gc_te_plan* plan, const double* d_xyz, double* d_te, void* stream);
/* Waits for the last run; reports a non-finite coordinate. */
gc_status gc_te_plan_sync(gc_te_plan* plan);
/* Ordered pairs natoms * (natoms - 1). */
long   gc_te_plan_pairs(const gc_te_plan* plan);
int    gc_te_plan_launches(const gc_te_plan* plan);
/* 1 when the plan runs the sorted-row walk. */
int    gc_te_plan_is_walk(const gc_te_plan* plan);
/* Queries of the last run handed to the exact FP64 kernel, and the mean
 * number of sorted-row entries walked per (ordered pair, query) (valid
 * after gc_te_plan_sync; 0 off the walk path). */
long   gc_te_plan_handoffs(const gc_te_plan* plan);
double gc_te_plan_walk_mean(const gc_te_plan* plan);
/* Device time in milliseconds of the neighbour-statistics kernels of the
 * last run (CUDA events on the run's stream). */
float  gc_te_plan_kernel_ms(const gc_te_plan* plan);
/* Per-query counts of the last run for TE(a2 -> a1), host arrays of
 * nframes - lag entries (any may be NULL): the strict counts n_xp, n_xfxp
 * and n_ypxp of lib/transfer_entropy.cpp:167-186. */
gc_status gc_te_plan_counts(gc_te_plan* plan, int a1, int a2, int32_t* n_xp, int32_t* n_xfxp, int32_t* n_ypxp);
void   gc_te_plan_destroy(gc_te_plan* plan);

/* r = sqrt(1 - exp(-2/dim * MI)) for MI > 0, else 0; the 2000 diagonal
 * maps to 1.  Replaces pearsify (lib/correlation_core.cpp:461-469). */
void gc_pearsify(double* mat, int n, int dim);

/* correl.dat writer, byte-compatible with write_matrix
 * (lib/correlation_core.cpp:202-225). */
gc_status gc_write_matrix(const double* mat, int n, const char* path);

/* Grey-scale XPM writer, byte-compatible with write_xpm_matrix
 * (lib/correlation_core.cpp:227-278). */
gc_status gc_write_xpm(const double* mat, int n, const char* path, const char* title, const char* legend);

/* kraskov_prepare on the GPU (lib/kraskov.cpp:2168-2220): X [3*natoms][nframes]
 * gets each component z-scored with the (N-1) standard deviation and shifted
 * to a zero minimum, bit-identical to the reference; psi [nframes+1] the
 * digamma table; scal [3*natoms] (optional) (nframes-5)/(max-min).
 * Replaces kraskov_prepare (lib/correlation_core.h:65). */
gc_status gc_ksg_prepare(const gc_traj_view* traj, const gc_opts* opts, double* X, double* psi, double* scal);

/* MI of one atom pair from already-normalised component rows, as
 * kraskov_wrap does (lib/kraskov.cpp:2222-2282): rows6 [6][nframes] holds
 * the three rows of atom a1 followed by the three rows of atom a2; psi is
 * the [nframes+1] digamma table.  Replaces kraskov_wrap
 * (lib/correlation_core.h:67). */
gc_status gc_ksg_pair(const double* rows6, int nframes, int k, const double* psi, const gc_opts* opts, double* mi);

/* ---- Device-resident KSG plan (inputs already in HBM) ----------------
 * A plan owns every device workspace for one (natoms, nframes, k, shard)
 * shape, so repeated runs allocate nothing.  gc_ksg_plan_run reads
 * coordinates from device memory d_xyz ([natoms][nframes][3] doubles) and
 * writes the shard's pair MI values (pair order p = a1*(a1-1)/2 + a2) to
 * device memory d_pair_mi, ordered on `stream` (cudaStream_t, NULL = the
 * plan's stream).  Nothing is synchronised; call gc_ksg_plan_sync or
 * synchronise the stream before reading results. */
typedef struct gc_ksg_plan gc_ksg_plan;

gc_status gc_ksg_plan_create(int natoms, int nframes, int k, const gc_opts* opts, gc_ksg_plan** plan);
gc_status gc_ksg_plan_run(gc_ksg_plan* plan, const double* d_xyz, double* d_pair_mi, void* stream);
gc_status gc_ksg_plan_sync(gc_ksg_plan* plan);
/* Number of pairs in the plan's shard. */
long gc_ksg_plan_pairs(const gc_ksg_plan* plan);
/* Kernel launches issued by the last gc_ksg_plan_run. */
int gc_ksg_plan_launches(const gc_ksg_plan* plan);
/* 1 if the plan runs the FP32 fast path (0: exact FP64 kernels only). */
int gc_ksg_plan_is_fast(const gc_ksg_plan* plan);
/* Queries of the last run that the fast path handed to the exact FP64
 * kernel (valid after gc_ksg_plan_sync). */
long gc_ksg_plan_handoffs(const gc_ksg_plan* plan);
/* Mean number of sorted-row entries the fast path walked per (pair, query) in the
 * last run (valid after gc_ksg_plan_sync; 0 for the exact path). */
double gc_ksg_plan_walk_mean(const gc_ksg_plan* plan);
/* Hand-overs of the last run by cause: 2 k-th value beyond the walk
 * histogram's range, 3 band around the k-th value larger than the per-query
 * store or inconsistent, 4 ambiguous set inconsistent or too large, 5 scan
 * for the marginal maxima too long, 6 count band outside the walked prefix
 * (valid after gc_ksg_plan_sync). */
long gc_ksg_plan_handoff_reason(const gc_ksg_plan* plan, int reason);
/* Device time in milliseconds of the neighbour-statistics kernel(s) of the
 * last run, measured with CUDA events on the run's stream (valid after the
 * run has completed). */
float gc_ksg_plan_kernel_ms(const gc_ksg_plan* plan);
void gc_ksg_plan_destroy(gc_ksg_plan* plan);

/* Measured FP32 non-tensor rates of `device` (-1 = current): *mix_ops_per_s
 * for the FADD + FMNMX pair of a max-norm distance (one op per lane
 * result), *fma_flops_per_s for FFMA (2 flop each).  The KSG roofline
 * denominator. */
gc_status gc_probe_fp32(int device, double* mix_ops_per_s, double* fma_flops_per_s);

/* ---- Learned KSG screen ----------------------------------------------------
 * No counterpart in the reference.  An ensemble of small BF16 networks
 * (GC_SCREEN_IN -> 128 -> 128 -> 128 -> 1, GELU, FP32 accumulation, trained
 * and evaluated by this library's own kernels) predicts the KSG r(MI) of an
 * atom pair from cheap per-pair features.  gc_ksg_screened then runs exact
 * KSG only on the pairs whose prediction is uncertain (ensemble spread) or
 * close to the reported threshold, plus a seeded random audit sample whose
 * exact values measure the prediction error.
 *
 * Feature row (floats): [0] Gaussian MI of the pair's 6x6 covariance;
 * [1..6] eigenvalues of the 6x6 joint correlation, descending; [7..12] the
 * six excess kurtoses (each atom's sorted descending, larger maximum first);
 * [13..21] |3x3 cross-correlation| sorted descending; [22] k / nframes;
 * [23..] the 8x8 joint histogram of the atoms' first-principal-axis
 * projections in rank space (oriented to a non-negative rank correlation,
 * symmetrised), either projected on GC_SCREEN_COMP principal components or
 * as the GC_SCREEN_HIST raw cells. */
#define GC_SCREEN_BASE 23
#define GC_SCREEN_HIST 64
#define GC_SCREEN_COMP 17
#define GC_SCREEN_IN (GC_SCREEN_BASE + GC_SCREEN_COMP) /* 40 */
#define GC_SCREEN_RAW (GC_SCREEN_BASE + GC_SCREEN_HIST) /* 87 */
#define GC_SCREEN_HIDDEN 128

typedef struct gc_screen_model gc_screen_model;

/* Features of the pairs opts selects (all pairs, a shard or a list), host
 * out[pair][GC_SCREEN_IN] projected on the basis pca_mean[64],
 * pca_comp[GC_SCREEN_COMP][64]; with pca_mean == NULL the raw rows
 * out[pair][GC_SCREEN_RAW] (used to fit the basis).  nframes <= 16384. */
gc_status gc_screen_features(const gc_traj_view* traj, int k, const gc_opts* opts, const float* pca_mean,
                             const float* pca_comp, float* out);

/* An ensemble of `members` networks on `device` (-1 = current), weights
 * drawn uniform(+-1/sqrt(fan_in)) from `seed`, biases likewise. */
gc_status gc_screen_model_create(int members, uint64_t seed, int device, gc_screen_model** model);
void      gc_screen_model_destroy(gc_screen_model* model);
int       gc_screen_model_members(const gc_screen_model* model);
/* Floats per member of the parameter block: W1[128][40] b1[128]
 * W2[128][128] b2[128] W3[128][128] b3[128] W4[1][128] b4[1], then padding. */
long      gc_screen_param_stride(void);
/* Host copy of all members' parameters, members * stride floats. */
gc_status gc_screen_model_get_params(const gc_screen_model* model, float* params);
gc_status gc_screen_model_set_params(gc_screen_model* model, const float* params);
/* Standardisation (f - feat_mean) / feat_sd applied to every feature row
 * before the first layer, and the histogram basis gc_ksg_screened uses
 * (pca_mean[64], pca_comp[GC_SCREEN_COMP][64]). */
gc_status gc_screen_model_set_input(gc_screen_model* model, const float* feat_mean, const float* feat_sd,
                                    const float* pca_mean, const float* pca_comp);
/* Adam (beta 0.9 / 0.999, eps 1e-8) on the mean squared error of every
 * member against target[n], over `epochs` passes of shuffled minibatches of
 * `batch` rows (<= 8192); the learning rate falls from lr to lr / 20 on a
 * cosine.  feats: host [n][GC_SCREEN_IN].  loss_per_epoch (may be NULL):
 * mean training loss of each epoch, averaged over members. */
gc_status gc_screen_train(gc_screen_model* model, const float* feats, const float* target, long n, int epochs,
                          int batch, float lr, uint64_t seed, float* loss_per_epoch);
/* One forward and backward pass over all n rows (n <= 8192) with no
 * update: grad[members * stride] (mean squared error gradient), loss[members]. */
gc_status gc_screen_grad(gc_screen_model* model, const float* feats, const float* target, long n, float* grad,
                         float* loss);
/* Prediction of every member: out[member][n]. */
gc_status gc_screen_predict(gc_screen_model* model, const float* feats, long n, float* out);

typedef struct gc_screen_opts
{
    double   audit_frac; /* random audit sample, fraction of the pairs (0.05) */
    double   sigma_max;  /* flag a pair when the ensemble's spread exceeds this */
    double   margin;     /* flag a pair when |r_hat - threshold| < margin */
    uint64_t seed;       /* audit sample seed */
} gc_screen_opts;

typedef struct gc_screen_report
{
    long   pairs;          /* pairs in the matrix */
    long   flagged;        /* pairs the screen sent to exact KSG */
    long   audited;        /* pairs in the random audit sample */
    long   exact;          /* pairs computed by exact KSG (flagged or audited) */
    long   audit_accepted; /* audited pairs the screen did not flag */
    double threshold;      /* reported threshold: mean + 0.5 sd of the positive predicted r */
    double audit_max_dr;   /* max |r_hat - r_ksg| over audit_accepted pairs */
    double audit_rms_dr;   /* rms of the same */
    double final_max_dr;   /* max |r_out - r_ksg| over the audit sample */
    /* device time of each stage; when at least half of the pairs are exact,
       ms_ksg is the host time of one whole-matrix gc_ksg_matrix call */
    float  ms_features, ms_mlp, ms_ksg;
} gc_screen_report;

void gc_screen_opts_init(gc_screen_opts* o);
/* r(MI) matrix [natoms * natoms] (pearsified, diagonal 1): exact KSG r on
 * the flagged and audited pairs, the ensemble mean elsewhere.  opts selects
 * the device, path and stream as for gc_ksg_matrix (pair selection ignored). */
gc_status gc_ksg_screened(const gc_traj_view* traj, int k, gc_screen_model* model, const gc_screen_opts* sopts,
                          const gc_opts* opts, double* r, gc_screen_report* report);

/* ---- KSG without device allocation ---------------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory (a plugin whose host application owns all device memory through its
 * own pool, or a latency-critical caller that cannot take cudaMalloc /
 * cudaFree): computes the pair MI of every atom pair with the exact FP64 KSG
 * kernels, taking all scratch from one fixed array of about 9.8 MB that the
 * library holds on every device that loads it until the process exits.
 * Limits: natoms <= 64, nframes <= 1024; larger calls fail with
 * GC_ERR_INVALID.  d_xyz: device [natoms][nframes][3] mean-centred
 * coordinates; d_pair_mi: device [natoms*(natoms-1)/2], pair order
 * p = a1*(a1-1)/2 + a2 (a2 < a1); stream: cudaStream_t (NULL = the legacy
 * default stream).  Runs on the calling thread's current device and returns
 * after the work has finished (it synchronises the stream to check the
 * input-status word).  The first call on a device looks up the array's
 * device address, so it should come before any stream capture.  With CUDA's
 * lazy module loading (the default) that first call is also what reserves
 * the array on the device (CUDA_MODULE_LOADING=EAGER reserves it when the
 * library loads), so a host application that gives all device memory to its
 * own pool should make one warm-up call before doing so; later calls reserve
 * nothing.  After a cudaDeviceReset the looked-up address is stale: do not
 * call this entry point on that device again in the same process.  All calls
 * share the one array: calls whose work overlaps on the GPU race. */
gc_status gc_ksg_pair_mi_noalloc(const double* d_xyz, int natoms, int nframes, int k, double* d_pair_mi, void* stream);

/* ---- Trajectory ingest ----------------------------------------------------
 * Replaces the GROMACS front end's frame collection (src/gmx_correlation.cpp:
 * 158-182 analyzeFrame: a static atom selection, every skip-th analysed
 * frame; :184-223 finishAnalysis: per-atom mean over the kept frames, summed
 * in frame order, subtracted).  Host-only: no device is needed.  Formats are
 * told apart by content: GROMACS XTC (compressed, magic 1995), TRR (magic
 * 1993, float or double; positions only, velocities and forces skipped) and
 * the reference's -dump text file (src/gmx_correlation.cpp:225-244; frame
 * times are the frame indices).  Positions are in the file's units (nm).
 * XTC positions come out as GROMACS' mixed-precision reader gives them
 * (integer times float(1/precision)); double TRR positions are rounded to
 * float unless GC_TRAJ_KEEP_DOUBLE is set.  No periodic-boundary treatment or
 * fitting is applied (the reference asks for a trajectory pre-fitted with
 * gmx trjconv). */
/* ---- The MILCA estimator family (lib/kraskov.cpp:347-2155) ----------------
 * One entry point per reference function, same arguments (x: one host row of
 * N doubles per component, psi: digamma table psi[0..N], scal: per-row scale
 * of the 1-D box counts, whose boxes (int)(x*scal) must lie in 0..N-5).  Each
 * runs the exact FP64 neighbour search on the GPU and returns the
 * reference's values bit for bit; like the reference, every function but
 * redr_embed leaves the rows of x sorted by the cells of its search grid.
 * mi_cr: 2K values, (mic, mir) for k = 1..K.  Errors: GC_ERR_INVALID (bad
 * sizes, K >= N, a scale outside the box range), GC_ERR_NONFINITE, device
 * errors.  Where a 1-D box count comes out at -1 (the query's own box lies
 * outside the end boxes of [x - eps, x + eps]) the reference reads psi[-1],
 * the word before its table; that term is taken as 0 here (= psi[0]).
 * lib/kraskov.cpp: mi2 :347, mi2c :443, mi2r :529, red :615, redc :712,
 * redr :799, redr_embed :883, mi_xnyn :1004, mic_xnyn :1121, mir_xnyn :1228,
 * redK :1333, mi2K :1456, mi_xnynK :1579, mi_xnynKembed :1713, mi2h :1811,
 * mi_d :1950, mi2r_ :2071. */
gc_status gc_milca_mi2(double** x, int N, int K, const double* psi, const double* scal, double* mic, double* mir);
gc_status gc_milca_mi2c(double** x, int N, int K, const double* psi, const double* scal, double* mic);
gc_status gc_milca_mi2r(double** x, int N, int K, const double* psi, const double* scal, double* mir);
gc_status gc_milca_mi2r_(double** x, int N, int K, const double* psi, const double* scal, double* mir);
gc_status gc_milca_mi2K(double** x, int N, int K, const double* psi, const double* scal, double* mi_cr);
/* also prints the reference's entropy lines to stdout */
gc_status gc_milca_mi2h(double** x, int N, int K, const double* psi, const double* scal, double* mic, double* mir,
                        double* hc, double* hr);
gc_status gc_milca_red(double** x, int dim, int N, int K, const double* psi, const double* scal, double* mic,
                       double* mir);
gc_status gc_milca_redc(double** x, int dim, int N, int K, const double* psi, const double* scal, double* mic);
gc_status gc_milca_redr(double** x, int dim, int N, int K, const double* psi, const double* scal, double* mir);
gc_status gc_milca_redK(double** x, int dim, int N, int K, const double* psi, const double* scal, double* mi_cr);
gc_status gc_milca_redr_embed(double** x, int dim, int edim, int tau, int N, int K, const double* psi, double* mir);
gc_status gc_milca_mi_xnyn(double** x, int dimx, int dimy, int N, int K, const double* psi, const double* scal,
                           double* mic, double* mir);
gc_status gc_milca_mic_xnyn(double** x, int dimx, int dimy, int N, int K, const double* psi, const double* scal,
                            double* mic);
gc_status gc_milca_mir_xnyn(double** x, int dimx, int dimy, int N, int K, const double* psi, const double* scal,
                            double* mir);
gc_status gc_milca_mi_xnynK(double** x, int dimx, int dimy, int N, int K, const double* psi, const double* scal,
                            double* mi_cr);
/* the reference's caller-built marginal grids are not needed (exact counts) */
gc_status gc_milca_mi_xnynKembed(double** x, int dim, int N, int K, const double* psi, double* mi_cr);
gc_status gc_milca_mi_d(double** x, int dim, int N, int K, float* mi_cr, const double* psi, const double* phi,
                        double minx, double maxx, double miny, double maxy);

#define GC_TRAJ_XTC  1
#define GC_TRAJ_TRR  2
#define GC_TRAJ_DUMP 3

#define GC_TRAJ_CENTER      1 /* subtract each atom's mean position (the reference's centring) */
#define GC_TRAJ_KEEP_DOUBLE 2 /* read: double TRR positions unrounded; write: a double-precision TRR */
#define GC_TRAJ_BEGIN       4 /* ignore frames with time < t_begin (GROMACS -b) */
#define GC_TRAJ_END         8 /* ignore frames with time > t_end (GROMACS -e) */

typedef struct gc_traj_select
{
    const int* atoms;  /* 0-based atom indices in output order (the selection); NULL: all atoms */
    int        natoms; /* entries of atoms (0 with atoms NULL) */
    int        skip;   /* keep every skip-th frame inside the time window, counted from the first (>= 1) */
    double     t_begin, t_end; /* ps, with GC_TRAJ_BEGIN / GC_TRAJ_END */
    int        flags;  /* GC_TRAJ_* flags */
} gc_traj_select;

/* Format, atom count and frame count of a trajectory (reads the whole file). */
gc_status gc_traj_info(const char* path, int* format, int* natoms, int* nframes);
/* Positions of the selected atoms in the kept frames as a malloc'd host array
 * x[atom][frame][dim] (release with gc_traj_free), the layout of t_traj and
 * of gc_traj_view.  sel NULL: all atoms, all frames, no centring.  Fails with
 * GC_ERR_INVALID (message in gc_last_error) on a malformed or truncated
 * frame, an atom count that changes between frames, a selected index outside
 * the file, or no frame kept; GC_ERR_IO when the file cannot be opened. */
gc_status gc_traj_read(const char* path, const gc_traj_select* sel, double** xyz, int* natoms, int* nframes);
void      gc_traj_free(double* xyz);
/* Writes nframes frames of positions xyz[frame][atom][dim] (nm) as XTC
 * (precision: 1000 = 0.001 nm when <= 0) or TRR (float; double with
 * GC_TRAJ_KEEP_DOUBLE in flags).  box: 9 floats per frame or NULL (zero box);
 * times: ps per frame or NULL (the frame index); steps are frame indices. */
gc_status gc_traj_write(const char* path, int format, const float* xyz, int natoms, int nframes, const float* box,
                        const double* times, float precision, int flags);

#ifdef __cplusplus
}
#endif

#endif /* GMX_CORR_B200_H */
