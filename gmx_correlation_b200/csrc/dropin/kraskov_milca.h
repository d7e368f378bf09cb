// Drop-in declarations of the MILCA estimator family that the reference
// defines in lib/kraskov.cpp (:347-2155) without a header: the same names,
// C++ linkage and argument lists, so code written against those definitions
// links against libgmxcorr_b200.so unchanged.  Each runs on the GPU through
// the gc_milca_* C entry points (include/gmx_corr_b200.h) and throws
// std::runtime_error where the C entry point reports an error.
//
// As in the reference, x holds one row of N doubles per variable component
// (the normalised rows kraskov_prepare produces, or any non-negative data
// for the 1-D box counts), psi the digamma table psi[0 .. N], scal the
// per-row scale of the 1-D box counts (boxes (int)(x * scal) in 0 .. N-5).
// Every function except redr_embed leaves x sorted by the cells of its
// search grid, as the reference's make_box2 / make_box2ind do.
#pragma once

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
// The caller's marginal copies and grids (xx, yy, boxx, lisx, indx, boxy,
// lisy, indy) are not read: the counts are the exact marginal counts, which
// is what the reference computes from grids that make_box2ind built on the
// same rows with the same BOX.
void mi_xnynKembed(double** x, int dim, int N, int K, double** xx, double** yy, int** boxx, int* lisx, int* indx,
                   int** boxy, int* lisy, int* indy, double* psi, double* mi_cr);
void mi_d(double** x, int dim, int N, int K, float* mi_cr, double* psi, double* phi, double minx, double maxx,
          double miny, double maxy);
