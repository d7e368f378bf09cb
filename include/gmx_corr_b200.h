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
} gc_opts;

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

/* Gaussian (linearized) MI matrix.  Replaces gauss_corrmatrix
 * (lib/correlation_core.h:76, lib/correlation_core.cpp:280-311). */
gc_status gc_gauss_matrix(const gc_traj_view* traj, const gc_opts* opts, double* mi);

/* Gaussian-copula MI matrix.  Replaces gcmi_corrmatrix (lib/gcmi.h:8-9,
 * lib/gcmi.cpp:246-317). */
gc_status gc_gcmi_matrix(const gc_traj_view* traj, const gc_opts* opts, double* mi);

/* Transfer-entropy matrix, mat[a1*n+a2] = TE(a2 -> a1, lag).  Replaces
 * te_matrix (lib/transfer_entropy.h:8-9, lib/transfer_entropy.cpp:63-221).
 * When nframes - lag <= k the matrix is all zeros, as in the reference. */
gc_status gc_te_matrix(const gc_traj_view* traj, int k, int lag, const gc_opts* opts, double* te);

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
/* Mean number of sorted-row entries the fast path walked per query in the
 * last run (valid after gc_ksg_plan_sync; 0 for the exact path). */
double gc_ksg_plan_walk_mean(const gc_ksg_plan* plan);
/* Hand-overs of the last run by cause: 1 walk longer than the per-warp
 * buffer, 2 k-th value outside the histogram range, 3 band around the k-th
 * value too wide, 4 ambiguous set too large, 5 too many candidates for the
 * FP64 maxima (valid after gc_ksg_plan_sync). */
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
 * device address, so it should come before any stream capture.  All calls
 * share the one array: calls whose work overlaps on the GPU race. */
gc_status gc_ksg_pair_mi_noalloc(const double* d_xyz, int natoms, int nframes, int k, double* d_pair_mi, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GMX_CORR_B200_H */
