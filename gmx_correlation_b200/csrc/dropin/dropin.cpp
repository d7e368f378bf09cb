// C++ drop-in implementation of the reference's estimator interface
// (lib/correlation_core.h, lib/gcmi.h, lib/transfer_entropy.h) over the C ABI.
//
// Behaviour kept from the reference: input violations throw
// std::runtime_error with the reference's messages; the matrix conventions
// (zero fill, diagonal 2000 / 0, symmetric writes) are those of
// kraskov_corrmatrix, gauss_corrmatrix, gcmi_corrmatrix and te_matrix.
// Changed on purpose: every estimator runs on the GPU whatever use_gpu says
// (the reference's CPU path is the oracle, not a fallback), nthreads is
// accepted and ignored, and CUDA / device failures throw instead of
// exit(1) (lib/kraskov_gpu.cu:202-208).

#include "correlation_core.h"
#include "gcmi.h"
#include "kraskov_gpu.h"
#include "transfer_entropy.h"
#include "gmx_corr_b200.h"

#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

gc_traj_view view_of(const t_traj* traj)
{
    gc_traj_view v;
    v.natoms  = traj->natoms;
    v.nframes = traj->nframes;
    v.xyz     = nullptr;
    v.rows    = reinterpret_cast<const double* const*>(traj->x);
    return v;
}

void check(gc_status st)
{
    if (st != GC_OK)
        throw std::runtime_error(gc_last_error());
}

} // namespace

void kraskov_corrmatrix(const t_traj* traj, double* mat, int k, bool /*use_gpu*/, int /*nthreads*/)
{
    if (traj->natoms < 2)
        throw std::runtime_error("kraskov_corrmatrix: need at least 2 atoms");
    if (traj->nframes <= k)
        throw std::runtime_error("kraskov_corrmatrix: nframes must exceed k (number of nearest neighbours)");
    const gc_traj_view v = view_of(traj);
    check(gc_ksg_matrix(&v, k, nullptr, mat));
}

void gauss_corrmatrix(const t_traj* traj, double* mat)
{
    const gc_traj_view v = view_of(traj);
    check(gc_gauss_matrix(&v, nullptr, mat));
}

void gcmi_corrmatrix(const t_traj* traj, double* mat, bool /*use_gpu*/, int /*nthreads*/)
{
    if (traj->natoms < 2)
        throw std::runtime_error("gcmi_corrmatrix: need at least 2 atoms");
    if (traj->nframes < 6)
        throw std::runtime_error("gcmi_corrmatrix: need at least 6 frames for a non-singular 6x6 covariance");
    const gc_traj_view v = view_of(traj);
    check(gc_gcmi_matrix(&v, nullptr, mat));
}

void te_matrix(const t_traj* traj, double* mat, int k, int lag, bool /*use_gpu*/, int /*nthreads*/)
{
    const gc_traj_view v = view_of(traj);
    check(gc_te_matrix(&v, k, lag, nullptr, mat));
}

bool gpu_available() { return gc_gpu_available() != 0; }
bool kraskov_gpu_probe() { return gc_gpu_available() != 0; }

void kraskov_corrmatrix_gpu(const t_kraskov* kr, int natoms, double* mat, int k)
{
    const int           N = kr->N;
    std::vector<double> X((size_t)natoms * DIM * N);
    for (int c = 0; c < natoms * DIM; ++c)
        std::memcpy(X.data() + (size_t)c * N, kr->x[c], sizeof(double) * N);
    check(gc_ksg_matrix_prepared(X.data(), kr->psi, natoms, N, k, nullptr, mat));
}
bool gcmi_gpu_available() { return gc_gpu_available() != 0; }
bool te_gpu_available() { return gc_gpu_available() != 0; }

void pearsify(double* mat, int n, int dim) { gc_pearsify(mat, n, dim); }

void write_matrix(const double* mat, int natoms, const char* outfile)
{
    if (gc_write_matrix(mat, natoms, outfile) != GC_OK)
        throw std::runtime_error(std::string("Could not open output file: ") + outfile);
}

void write_xpm_matrix(const double* mat, int natoms, const char* outfile, const char* title, const char* legend)
{
    if (gc_write_xpm(mat, natoms, outfile, title, legend) != GC_OK)
        throw std::runtime_error(std::string("Could not open output file: ") + outfile);
}

void done_traj(t_traj* traj)
{
    if (traj->x != nullptr)
    {
        for (int i = 0; i < traj->natoms; ++i)
            sfree(traj->x[i]);
        sfree(traj->x);
    }
    sfree(traj->xav);
}

void kraskov_prepare(t_traj* gmx_traj, t_kraskov* kr)
{
    const int n = gmx_traj->natoms, N = gmx_traj->nframes;
    kr->N   = N;
    kr->dim = n * DIM;
    std::vector<double> X((size_t)n * DIM * N);
    snew(kr->psi, N + 1);
    snew(kr->scal, kr->dim);
    const gc_traj_view v = view_of(gmx_traj);
    check(gc_ksg_prepare(&v, nullptr, X.data(), kr->psi, kr->scal));
    snew(kr->x, kr->dim);
    for (int c = 0; c < kr->dim; ++c)
    {
        snew(kr->x[c], N);
        std::memcpy(kr->x[c], X.data() + (size_t)c * N, sizeof(double) * N);
    }
}

void kraskov_done(t_kraskov* kr)
{
    for (int d = 0; d < kr->dim; ++d)
        sfree(kr->x[d]);
    sfree(kr->psi);
    sfree(kr->scal);
    sfree(kr->x);
}

double kraskov_wrap(t_kraskov* kr, int a1, int a2, int param_k)
{
    const int           N = kr->N;
    std::vector<double> rows((size_t)6 * N);
    for (int d = 0; d < DIM; ++d)
    {
        std::memcpy(rows.data() + (size_t)d * N, kr->x[a1 * DIM + d], sizeof(double) * N);
        std::memcpy(rows.data() + (size_t)(d + 3) * N, kr->x[a2 * DIM + d], sizeof(double) * N);
    }
    double mi = 0.0;
    check(gc_ksg_pair(rows.data(), N, param_k, kr->psi, nullptr, &mi));
    return mi;
}
