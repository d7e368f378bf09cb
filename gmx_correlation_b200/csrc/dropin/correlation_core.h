// Drop-in C++ interface of the all-pairs path.
//
// Same types, names, signatures and default arguments as the reference's
// lib/correlation_core.h:22-88 (scdantu/gmx_correlation), so the reference's
// front end (src/gmx_correlation.cpp) links against this library unchanged.
// The declarations must match the reference for that reason; the
// implementations (dropin.cpp) forward to the C ABI in gmx_corr_b200.h and
// compute on the GPU.
#ifndef GMX_CORRELATION_CORE_H
#define GMX_CORRELATION_CORE_H

#include <cstddef>
#include <cstdlib>
#include <type_traits>

#ifndef DIM
#define DIM 3
#endif

typedef double gcorr_rvec[DIM];

// Mean-centred trajectory: x[atom][frame][dim], xav[atom][dim].
struct t_traj
{
    int          nframes = 0;
    int          natoms  = 0;
    gcorr_rvec** x       = nullptr;
    gcorr_rvec*  xav     = nullptr;
};

// Normalised KSG workspace: x[comp][frame] (comp = atom*3 + dim), the
// digamma table psi[N+1] and scal[3*natoms].
struct t_kraskov
{
    double** x    = nullptr;
    double*  psi  = nullptr;
    double*  scal = nullptr;
    int      N    = 0;
    int      dim  = 0;
};

// calloc / free helpers with the reference's names.
#define snew(ptr, n) \
    ((ptr) = static_cast<std::remove_reference_t<decltype(ptr)>>(std::calloc((n), sizeof(*(ptr)))))
#define sfree(ptr)       \
    do                   \
    {                    \
        std::free(ptr);  \
        (ptr) = nullptr; \
    } while (0)

void   kraskov_prepare(t_traj* gmx_traj, t_kraskov* kr);
void   kraskov_done(t_kraskov* kr);
double kraskov_wrap(t_kraskov* kr, int a1, int a2, int param_k);
void   write_matrix(const double* mat, int natoms, const char* outfile);
void   write_xpm_matrix(const double* mat, int natoms, const char* outfile, const char* title, const char* legend);
void   gauss_corrmatrix(const t_traj* traj, double* mat);
void   kraskov_corrmatrix(const t_traj* traj, double* mat, int k, bool use_gpu = false, int nthreads = 0);
bool   gpu_available();
void   pearsify(double* mat, int n, int dim);
void   done_traj(t_traj* traj);

#endif
