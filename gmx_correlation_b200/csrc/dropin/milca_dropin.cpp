// The reference's MILCA functions (lib/kraskov.cpp:347-2155) with their own
// signatures, over the gc_milca_* C entry points.

#include "gmx_corr_b200.h"
#include "kraskov_milca.h"

#include <stdexcept>
#include <string>

namespace {

void check(gc_status st)
{
    if (st != GC_OK)
        throw std::runtime_error(gc_last_error());
}

} // namespace

void mi2(double** x, int N, int K, double* psi, double* scal, double* mic, double* mir)
{
    check(gc_milca_mi2(x, N, K, psi, scal, mic, mir));
}
void mi2c(double** x, int N, int K, double* psi, double* scal, double* mic)
{
    check(gc_milca_mi2c(x, N, K, psi, scal, mic));
}
void mi2r(double** x, int N, int K, double* psi, double* scal, double* mir)
{
    check(gc_milca_mi2r(x, N, K, psi, scal, mir));
}
void mi2r_(double** x, int N, int K, double* psi, double* scal, double* mir)
{
    check(gc_milca_mi2r_(x, N, K, psi, scal, mir));
}
void mi2K(double** x, int N, int K, double* psi, double* scal, double* mi_cr)
{
    check(gc_milca_mi2K(x, N, K, psi, scal, mi_cr));
}
void mi2h(double** x, int N, int K, double* psi, double* scal, double* mic, double* mir, double* hc, double* hr)
{
    check(gc_milca_mi2h(x, N, K, psi, scal, mic, mir, hc, hr));
}
void red(double** x, int dim, int N, int K, double* psi, double* scal, double* mic, double* mir)
{
    check(gc_milca_red(x, dim, N, K, psi, scal, mic, mir));
}
void redc(double** x, int dim, int N, int K, double* psi, double* scal, double* mic)
{
    check(gc_milca_redc(x, dim, N, K, psi, scal, mic));
}
void redr(double** x, int dim, int N, int K, double* psi, double* scal, double* mir)
{
    check(gc_milca_redr(x, dim, N, K, psi, scal, mir));
}
void redK(double** x, int dim, int N, int K, double* psi, double* scal, double* mi_cr)
{
    check(gc_milca_redK(x, dim, N, K, psi, scal, mi_cr));
}
void redr_embed(double** x, int dim, int edim, int tau, int N, int K, double* psi, double* mir)
{
    check(gc_milca_redr_embed(x, dim, edim, tau, N, K, psi, mir));
}
void mi_xnyn(double** x, int dimx, int dimy, int N, int K, double* psi, double* scal, double* mic, double* mir)
{
    check(gc_milca_mi_xnyn(x, dimx, dimy, N, K, psi, scal, mic, mir));
}
void mic_xnyn(double** x, int dimx, int dimy, int N, int K, double* psi, double* scal, double* mic)
{
    check(gc_milca_mic_xnyn(x, dimx, dimy, N, K, psi, scal, mic));
}
void mir_xnyn(double** x, int dimx, int dimy, int N, int K, double* psi, double* scal, double* mir)
{
    check(gc_milca_mir_xnyn(x, dimx, dimy, N, K, psi, scal, mir));
}
void mi_xnynK(double** x, int dimx, int dimy, int N, int K, double* psi, double* scal, double* mi_cr)
{
    check(gc_milca_mi_xnynK(x, dimx, dimy, N, K, psi, scal, mi_cr));
}
void mi_xnynKembed(double** x, int dim, int N, int K, double** /*xx*/, double** /*yy*/, int** /*boxx*/,
                   int* /*lisx*/, int* /*indx*/, int** /*boxy*/, int* /*lisy*/, int* /*indy*/, double* psi,
                   double* mi_cr)
{
    check(gc_milca_mi_xnynKembed(x, dim, N, K, psi, mi_cr));
}
void mi_d(double** x, int dim, int N, int K, float* mi_cr, double* psi, double* phi, double minx, double maxx,
          double miny, double maxy)
{
    check(gc_milca_mi_d(x, dim, N, K, mi_cr, psi, phi, minx, maxx, miny, maxy));
}
