// Test infrastructure only (never part of the product path).
//
// C-ABI shim over the UNMODIFIED reference sources of scdantu/gmx_correlation
// (lib/correlation_core.cpp, lib/kraskov.cpp, lib/gcmi.cpp,
// lib/transfer_entropy.cpp), compiled together by oracle/Makefile into
// oracle/_ref/libgcref.so.  Tests use it to pin the C restatement in
// oracle/gc_oracle.c, and bench.py's reference arm times the reference's own
// OpenMP CPU path through it.
//
// Nothing here re-implements an estimator: every number comes out of the
// reference's functions.  gcref_ksg_pair_detail() replays the per-query
// driver loop of mir_xnyn (lib/kraskov.cpp:1294-1318) through the reference's
// own make_box2ind / neiK / neiE so the per-query neighbour counts, marginal
// radii and the k-th neighbour can be compared one by one.

#include "correlation_core.h"
#include "gcmi.h"
#include "transfer_entropy.h"
#ifdef GMX_CORRELATION_USE_CUDA
#include "kraskov_gpu.h"
#endif

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

// External-linkage helpers of lib/kraskov.cpp (:56, :113, :257).
void make_box2ind(double** x, int dim, int N, int comp1, int comp2, int bs, int inveps,
                  int* ind, int** box, int* lis);
int  neiE(double** x, int i, int comp1, int comp2, int dim, int bs, double epsgrid, double eps,
          int** box, int* lis);
void neiK(double** x, int dim, int comp1, int comp2, int i, int bs, double epsgrid, int K,
          int** box, int* lis, int* nn);

// The unused MILCA estimators of lib/kraskov.cpp (:347-2155), by their own
// definitions' signatures; gcref_milca() calls them for the parity tests.
void mi2(double** x, int N, int K, double* psi, double* scal, double* mic, double* mir);
void mi2c(double** x, int N, int K, double* psi, double* scal, double* mic);
void mi2r(double** x, int N, int K, double* psi, double* scal, double* mir);
void mi2r_(double** x, int N, int K, double* psi, double* scal, double* mir);
void mi2K(double** x, int N, int K, double* psi, double* scal, double* mi_cr);
void mi2h(double** x, int N, int K, double* psi, double* scal, double* mic, double* mir, double* hc, double* hr);
void red(double** x, int dim, int N, int K, double* psi, double* scal, double* mic, double* mir);
void redc(double** x, int dim, int N, int K, double* psi, double* scal, double* mic);
void redr(double** x, int dim, int N, int K, double* psi, double* scal, double* mir);
void redK(double** x, int dim, int N, int K, double* psi, double* scal, double* mi_cr);
void redr_embed(double** x, int dim, int edim, int tau, int N, int K, double* psi, double* mir);
void mi_xnyn(double** x, int dimx, int dimy, int N, int K, double* psi, double* scal, double* mic, double* mir);
void mic_xnyn(double** x, int dimx, int dimy, int N, int K, double* psi, double* scal, double* mic);
void mir_xnyn(double** x, int dimx, int dimy, int N, int K, double* psi, double* scal, double* mir);
void mi_xnynK(double** x, int dimx, int dimy, int N, int K, double* psi, double* scal, double* mi_cr);
void mi_xnynKembed(double** x, int dim, int N, int K, double** xx, double** yy, int** boxx, int* lisx, int* indx,
                   int** boxy, int* lisy, int* indy, double* psi, double* mi_cr);
void mi_d(double** x, int dim, int N, int K, float* mi_cr, double* psi, double* phi, double minx, double maxx,
          double miny, double maxy);

namespace {

thread_local std::string g_err;

// Builds a t_traj (lib/correlation_core.h:31-37) from a contiguous
// [natoms][nframes][3] block of mean-centred coordinates.
t_traj make_traj(const double* xyz, int natoms, int nframes)
{
    t_traj t;
    t.natoms  = natoms;
    t.nframes = nframes;
    snew(t.x, natoms);
    snew(t.xav, natoms);
    for (int a = 0; a < natoms; ++a)
    {
        snew(t.x[a], nframes);
        std::memcpy(t.x[a], xyz + (size_t)a * nframes * 3, sizeof(double) * 3 * (size_t)nframes);
    }
    return t;
}

template <class F>
int guarded(F&& f)
{
    try
    {
        f();
        return 0;
    }
    catch (const std::exception& e)
    {
        g_err = e.what();
        return 1;
    }
}

int** alloc_box(int bs)
{
    int** b = (int**)std::calloc(bs, sizeof(int*));
    for (int i = 0; i < bs; ++i)
        b[i] = (int*)std::calloc(bs, sizeof(int));
    return b;
}

void free_box(int** b, int bs)
{
    for (int i = 0; i < bs; ++i)
        std::free(b[i]);
    std::free(b);
}

} // namespace

extern "C" {

const char* gcref_last_error(void) { return g_err.c_str(); }

int gcref_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

int gcref_ksg_matrix(const double* xyz, int natoms, int nframes, int k, int nthreads, double* mat)
{
    t_traj t = make_traj(xyz, natoms, nframes);
    int rc = guarded([&] { kraskov_corrmatrix(&t, mat, k, false, nthreads); });
    done_traj(&t);
    return rc;
}

int gcref_gauss_matrix(const double* xyz, int natoms, int nframes, double* mat)
{
    t_traj t = make_traj(xyz, natoms, nframes);
    int rc = guarded([&] { gauss_corrmatrix(&t, mat); });
    done_traj(&t);
    return rc;
}

int gcref_gcmi_matrix(const double* xyz, int natoms, int nframes, int nthreads, double* mat)
{
    t_traj t = make_traj(xyz, natoms, nframes);
    int rc = guarded([&] { gcmi_corrmatrix(&t, mat, false, nthreads); });
    done_traj(&t);
    return rc;
}

int gcref_te_matrix(const double* xyz, int natoms, int nframes, int k, int lag, int nthreads, double* mat)
{
    t_traj t = make_traj(xyz, natoms, nframes);
    int rc = guarded([&] { te_matrix(&t, mat, k, lag, false, nthreads); });
    done_traj(&t);
    return rc;
}

void gcref_pearsify(double* mat, int n, int dim) { pearsify(mat, n, dim); }

int gcref_write_matrix(const double* mat, int n, const char* path)
{
    return guarded([&] { write_matrix(mat, n, path); });
}

int gcref_write_xpm(const double* mat, int n, const char* path, const char* title, const char* legend)
{
    return guarded([&] { write_xpm_matrix(mat, n, path, title, legend); });
}

// kraskov_prepare (lib/kraskov.cpp:2168-2220): normalised component rows
// X[comp][frame] (comp = atom*3 + dim) and the digamma table psi[0..N].
int gcref_prepare(const double* xyz, int natoms, int nframes, double* X, double* psi)
{
    t_traj t = make_traj(xyz, natoms, nframes);
    t_kraskov kr;
    kraskov_prepare(&t, &kr);
    for (int c = 0; c < kr.dim; ++c)
        std::memcpy(X + (size_t)c * nframes, kr.x[c], sizeof(double) * nframes);
    std::memcpy(psi, kr.psi, sizeof(double) * (nframes + 1));
    kraskov_done(&kr);
    done_traj(&t);
    return 0;
}

// Sampled pairs through kraskov_prepare + kraskov_wrap under the same
// `omp parallel for schedule(dynamic,1)` shape as kraskov_corrmatrix
// (lib/correlation_core.cpp:403-439).  Used for bounded CPU-baseline timing.
int gcref_ksg_pairs(const double* xyz, int natoms, int nframes, int k, const int* a1, const int* a2,
                    int npairs, int nthreads, double* mi_out)
{
    t_traj t = make_traj(xyz, natoms, nframes);
    t_kraskov kr;
    kraskov_prepare(&t, &kr);
#ifdef _OPENMP
    if (nthreads > 0)
        omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1)
#endif
    for (int p = 0; p < npairs; ++p)
        mi_out[p] = kraskov_wrap(&kr, a1[p], a2[p], k);
    kraskov_done(&kr);
    done_traj(&t);
    return 0;
}

// Per-query detail of KSG algorithm 2 for one pair (a1, a2): replays
// mir_xnyn's driver loop (lib/kraskov.cpp:1260-1318, with the box sizing of
// :1260-1263) through the reference's make_box2ind / neiK / neiE.
// Outputs, indexed by original frame i: nx[i], ny[i] (the counts that index
// psi), epsx[i], epsy[i], kth[i] (original frame index of the k-th joint
// neighbour) and dk[i] (its joint distance).  Returns the pair MI through
// *mi, computed exactly as mir_xnyn does.
int gcref_ksg_pair_detail(const double* xyz, int natoms, int nframes, int k, int a1, int a2,
                          int* nx, int* ny, double* epsx_out, double* epsy_out, int* kth,
                          double* dk, double* mi)
{
    t_traj t = make_traj(xyz, natoms, nframes);
    t_kraskov kr;
    kraskov_prepare(&t, &kr);
    const int N = kr.N, K = k;

    double* x[6];
    double* xx[3];
    double* yy[3];
    for (int d = 0; d < 3; ++d)
    {
        x[d]     = (double*)std::malloc(sizeof(double) * N);
        x[d + 3] = (double*)std::malloc(sizeof(double) * N);
        std::memcpy(x[d], kr.x[a1 * 3 + d], sizeof(double) * N);
        std::memcpy(x[d + 3], kr.x[a2 * 3 + d], sizeof(double) * N);
        xx[d] = (double*)std::malloc(sizeof(double) * N);
        yy[d] = (double*)std::malloc(sizeof(double) * N);
        std::memcpy(xx[d], x[d], sizeof(double) * N);
        std::memcpy(yy[d], x[d + 3], sizeof(double) * N);
    }
    int BOX = 1;
    while (0.5 * BOX * BOX * K < N)
        BOX *= 2;
    const double epsilon = 4.0 / BOX;
    const int    inveps  = BOX / 4;

    int** box  = alloc_box(BOX);
    int** boxx = alloc_box(BOX);
    int** boxy = alloc_box(BOX);
    std::vector<int> lis(N), lisx(N), lisy(N), ind(N), indx(N), indy(N), inv(N), nn(K + 1);

    make_box2ind(x, 6, N, 0, 3, BOX, inveps, ind.data(), box, lis.data());
    make_box2ind(xx, 3, N, 0, 2, BOX, inveps, indx.data(), boxx, lisx.data());
    make_box2ind(yy, 3, N, 0, 2, BOX, inveps, indy.data(), boxy, lisy.data());
    for (int i = 0; i < N; ++i)
        inv[ind[i]] = i;

    double dxy2 = 0.0;
    for (int i = 0; i < N; ++i)
    {
        double xc[6];
        for (int d = 0; d < 6; ++d)
            xc[d] = x[d][ind[i]];
        neiK(x, 6, 0, 3, ind[i], BOX, epsilon, K, box, lis.data(), nn.data());
        double ex = 0, ey = 0, dd = 0;
        for (int d = 0; d < 3; ++d)
            for (int kk = 1; kk <= K; ++kk)
            {
                const double v = std::fabs(xc[d] - x[d][nn[kk]]);
                if (v > ex)
                    ex = v;
            }
        for (int d = 3; d < 6; ++d)
            for (int kk = 1; kk <= K; ++kk)
            {
                const double v = std::fabs(xc[d] - x[d][nn[kk]]);
                if (v > ey)
                    ey = v;
            }
        for (int d = 0; d < 6; ++d)
        {
            const double v = std::fabs(xc[d] - x[d][nn[K]]);
            if (v > dd)
                dd = v;
        }
        const int n2x = neiE(xx, indx[i], 0, 2, 3, BOX, epsilon, ex, boxx, lisx.data());
        const int n2y = neiE(yy, indy[i], 0, 2, 3, BOX, epsilon, ey, boxy, lisy.data());
        nx[i]       = n2x;
        ny[i]       = n2y;
        epsx_out[i] = ex;
        epsy_out[i] = ey;
        kth[i]      = inv[nn[K]];
        dk[i]       = dd;
        dxy2 += kr.psi[n2x] + kr.psi[n2y];
    }
    const double phiK = kr.psi[K] - 1 / (1.0 * K);
    dxy2 /= N;
    *mi = kr.psi[N] + phiK - dxy2;

    free_box(box, BOX);
    free_box(boxx, BOX);
    free_box(boxy, BOX);
    for (int d = 0; d < 6; ++d)
        std::free(x[d]);
    for (int d = 0; d < 3; ++d)
    {
        std::free(xx[d]);
        std::free(yy[d]);
    }
    kraskov_done(&kr);
    done_traj(&t);
    return 0;
}

#ifdef GMX_CORRELATION_USE_CUDA
// The reference's legacy CUDA KSG (lib/kraskov_gpu.cu, kraskov_mi_kernel),
// reached the way kraskov_corrmatrix(use_gpu = true) reaches it
// (lib/correlation_core.cpp:331-347) but without its silent CPU fallback:
// k > 128 or no CUDA device is an error here.  Only in libgcrefgpu.so.
int gcref_ksg_matrix_legacy_gpu(const double* xyz, int natoms, int nframes, int k, double* mat)
{
    if (k > 128 || !kraskov_gpu_probe())
    {
        g_err = "legacy GPU KSG unavailable: k > 128 or no CUDA device";
        return 1;
    }
    t_traj t  = make_traj(xyz, natoms, nframes);
    int    rc = guarded([&] {
        std::fill(mat, mat + (size_t)natoms * natoms, 0.0);
        t_kraskov kr;
        kraskov_prepare(&t, &kr);
        kraskov_corrmatrix_gpu(&kr, natoms, mat, k);
        kraskov_done(&kr);
    });
    done_traj(&t);
    return rc;
}
#endif

// One MILCA estimator of the reference on rows[D][N] (sorted in place by the
// reference, as it does to its caller's rows).  dim / dimx / dimy / edim /
// tau as the function takes them; out: mic, mir (hc, hr for mi2h) or 2K
// values; outf: mi_d's 2K floats.  mi_xnynKembed gets the marginal copies
// and grids the reference expects its caller to build (make_box2ind on each
// block, BOX from N and K).
int gcref_milca(const char* name, double* rows, int D, int N, int K, int dim, int dimx, int dimy, int edim, int tau,
                double* psi, double* scal, double* phi, double minx, double maxx, double miny, double maxy,
                double* out, float* outf)
{
    std::vector<double*> x((size_t)D);
    for (int d = 0; d < D; ++d)
        x[(size_t)d] = rows + (size_t)d * N;
    const std::string n(name);
    return guarded([&] {
        double** X = x.data();
        if (n == "mi2")
            mi2(X, N, K, psi, scal, out, out + 1);
        else if (n == "mi2c")
            mi2c(X, N, K, psi, scal, out);
        else if (n == "mi2r")
            mi2r(X, N, K, psi, scal, out + 1);
        else if (n == "mi2r_")
            mi2r_(X, N, K, psi, scal, out + 1);
        else if (n == "mi2K")
            mi2K(X, N, K, psi, scal, out);
        else if (n == "mi2h")
            mi2h(X, N, K, psi, scal, out, out + 1, out + 2, out + 3);
        else if (n == "red")
            red(X, dim, N, K, psi, scal, out, out + 1);
        else if (n == "redc")
            redc(X, dim, N, K, psi, scal, out);
        else if (n == "redr")
            redr(X, dim, N, K, psi, scal, out + 1);
        else if (n == "redK")
            redK(X, dim, N, K, psi, scal, out);
        else if (n == "redr_embed")
            redr_embed(X, dim, edim, tau, N, K, psi, out + 1);
        else if (n == "mi_xnyn")
            mi_xnyn(X, dimx, dimy, N, K, psi, scal, out, out + 1);
        else if (n == "mic_xnyn")
            mic_xnyn(X, dimx, dimy, N, K, psi, scal, out);
        else if (n == "mir_xnyn")
            mir_xnyn(X, dimx, dimy, N, K, psi, scal, out + 1);
        else if (n == "mi_xnynK")
            mi_xnynK(X, dimx, dimy, N, K, psi, scal, out);
        else if (n == "mi_d")
            mi_d(X, dim, N, K, outf, psi, phi, minx, maxx, miny, maxy);
        else if (n == "mi_xnynKembed")
        {
            int BOX = 1;
            while (0.5 * BOX * BOX * K < N)
                BOX *= 2;
            std::vector<std::vector<double>> cx((size_t)dim), cy((size_t)dim);
            std::vector<double*>             xx((size_t)dim), yy((size_t)dim);
            for (int d = 0; d < dim; ++d)
            {
                cx[(size_t)d].assign(X[d], X[d] + N);
                cy[(size_t)d].assign(X[dim + d], X[dim + d] + N);
                xx[(size_t)d] = cx[(size_t)d].data();
                yy[(size_t)d] = cy[(size_t)d].data();
            }
            int**            bx = alloc_box(BOX);
            int**            by = alloc_box(BOX);
            std::vector<int> lx((size_t)N), ly((size_t)N), ixv((size_t)N), iyv((size_t)N);
            make_box2ind(xx.data(), dim, N, 0, dim - 1, BOX, BOX / 4, ixv.data(), bx, lx.data());
            make_box2ind(yy.data(), dim, N, 0, dim - 1, BOX, BOX / 4, iyv.data(), by, ly.data());
            mi_xnynKembed(X, dim, N, K, xx.data(), yy.data(), bx, lx.data(), ixv.data(), by, ly.data(), iyv.data(), psi,
                          out);
            free_box(bx, BOX);
            free_box(by, BOX);
        }
        else
            throw std::runtime_error("unknown MILCA function " + n);
    });
}

} // extern "C"
