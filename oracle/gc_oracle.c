/*
 * gc_oracle.c -- TEST INFRASTRUCTURE ONLY: the CPU oracle.
 *
 * A plain-C restatement of the reference algorithms on the all-pairs
 * generalized-correlation path of scdantu/gmx_correlation.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it, and
 * only as the checker: the product (gmx_correlation_b200) never links or
 * calls it.
 *
 * Each function names the reference file:line it restates.  The oracle is
 * pinned against the reference itself: tests/test_oracle_vs_ref.py compares
 * it with oracle/_ref/libgcref.so (the unmodified reference sources compiled
 * here) and tests/test_oracle_golden.py with the committed fixtures under
 * tests/golden/ that the same library generated.
 *
 * KSG is restated as an exact brute force instead of the reference's box
 * grids.  Exact k-NN over the max-norm is unique up to ties; on an exact tie
 * at the k-th distance the reference keeps the neighbour its grid scan meets
 * first (lib/kraskov.cpp:282-285 inserts only on a strict `<`), so the
 * restatement orders tied candidates by that scan position
 * (gco_scan_pos) and then by ascending frame index (the in-cell order that
 * make_box2ind produces, lib/kraskov.cpp:56-91).
 */

#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define GCO_DIM 3

/* ------------------------------------------------------------------ */
/* Front end: mean-centring (src/gmx_correlation.cpp:195-223)          */
/* ------------------------------------------------------------------ */

/* raw and x are [natoms][nframes][3]; xav is [natoms][3]. */
void gco_center(const double* raw, int natoms, int nframes, double* x, double* xav)
{
    for (int a = 0; a < natoms; ++a)
    {
        double s[3] = {0.0, 0.0, 0.0};
        const double* r = raw + (size_t)a * nframes * 3;
        for (int f = 0; f < nframes; ++f)
            for (int d = 0; d < 3; ++d)
                s[d] += r[(size_t)f * 3 + d];
        for (int d = 0; d < 3; ++d)
            s[d] /= nframes;
        for (int f = 0; f < nframes; ++f)
            for (int d = 0; d < 3; ++d)
                x[(size_t)a * nframes * 3 + (size_t)f * 3 + d] = r[(size_t)f * 3 + d] - s[d];
        if (xav)
            for (int d = 0; d < 3; ++d)
                xav[a * 3 + d] = s[d];
    }
}

/* ------------------------------------------------------------------ */
/* kraskov_prepare (lib/kraskov.cpp:2168-2220)                          */
/* ------------------------------------------------------------------ */

/* x: [natoms][N][3] mean-centred; X: [3*natoms][N] normalised and
 * min-shifted; psi: [N+1].  The min/max seeds are the reference's
 * DBL_MAX/2 and -DBL_MAX/2 with its integer DBL_MAX (lib/kraskov.cpp:8-9). */
void gco_prepare(const double* x, int natoms, int N, double* X, double* psi)
{
    const int dim = natoms * GCO_DIM;
    for (int c = 0; c < dim; ++c)
    {
        const int atom = c / 3, d = c % 3;
        double* row = X + (size_t)c * N;
        for (int f = 0; f < N; ++f)
            row[f] = x[(size_t)atom * N * 3 + (size_t)f * 3 + d];
        double me = 0.0, s = 0.0;
        for (int f = 0; f < N; ++f)
            me += row[f];
        me /= N;
        for (int f = 0; f < N; ++f)
            s += (row[f] - me) * (row[f] - me);
        s /= (N - 1);
        s = sqrt(s);
        double mn = 2000000 / 2, mx = -2000000 / 2;
        for (int f = 0; f < N; ++f)
        {
            row[f] = (row[f] - me) / s;
            if (row[f] < mn)
                mn = row[f];
            if (row[f] > mx)
                mx = row[f];
        }
        for (int f = 0; f < N; ++f)
            row[f] = row[f] - mn;
    }
    psi[0] = 0.0;
    psi[1] = -(double).57721566490153;
    for (int n = 1; n < N; ++n)
        psi[n + 1] = psi[n] + 1 / (1.0 * n);
}

/* ------------------------------------------------------------------ */
/* Neighbour scan order of neiK (lib/kraskov.cpp:257-343)               */
/* ------------------------------------------------------------------ */

/* Box count of mir_xnyn (lib/kraskov.cpp:1260-1263). */
int gco_box_count(int N, int K)
{
    int box = 1;
    while (0.5 * box * box * K < N)
        box *= 2;
    return box;
}

/* Position, in neiK's traversal, of the cell whose offset from the query
 * cell is (dxm, dym) modulo bs: square shells jj = 0 .. bs/2-1 (rows
 * iy-jj / iy+jj for ascending ix, then columns ix-jj / ix+jj), then the
 * half layer jj = bs/2 (lib/kraskov.cpp:273-341). */
int64_t gco_scan_pos(int dxm, int dym, int bs)
{
    const int h  = bs / 2;
    const int rx = dxm >= h ? dxm - bs : dxm;
    const int ry = dym >= h ? dym - bs : dym;
    const int ax = rx < 0 ? -rx : rx, ay = ry < 0 ? -ry : ry;
    const int jj = ax > ay ? ax : ay;
    if (jj < h)
    {
        if (jj == 0)
            return 0;
        const int64_t base = (int64_t)(2 * jj - 1) * (2 * jj - 1);
        if (ay == jj)
            return base + (int64_t)(rx + jj) * 2 + (ry == jj ? 1 : 0);
        return base + 2 * (2 * jj + 1) + (rx == jj ? (2 * jj - 1) : 0) + (ry + jj - 1);
    }
    const int64_t base = (int64_t)(2 * h - 1) * (2 * h - 1);
    if (ry == -h)
        return base + (rx + h);
    return base + 2 * h + (ry + h - 1);
}

/* Tie-break rank of candidate j for query i of pair (a1, a2): scan
 * position of j's joint-grid cell, then frame index.  The joint grid is
 * built on component 0 of a1 and component 0 of a2
 * (make_box2ind(x, 6, N, 0, dimx, ...), lib/kraskov.cpp:1294); cells use
 * (int)(x*inveps) (:69-71) and the query cell (int)(x/epsgrid) (:271). */
static int64_t scan_rank(const double* c1, const double* c2, int N, int i, int j, int bs)
{
    const int    ib      = bs - 1;
    const int    inveps  = bs / 4;
    const double epsgrid = 4.0 / bs;
    const int    ix      = ((int)(c1[i] / epsgrid)) & ib;
    const int    iy      = ((int)(c2[i] / epsgrid)) & ib;
    const int    cx      = ((int)(c1[j] * inveps)) & ib;
    const int    cy      = ((int)(c2[j] * inveps)) & ib;
    return gco_scan_pos((cx - ix) & ib, (cy - iy) & ib, bs) * (int64_t)N + j;
}

/* k-th smallest (0-based kk) of a[0..n-1]; a is permuted. */
static double select_kth(double* a, int n, int kk)
{
    int lo = 0, hi = n - 1;
    while (lo < hi)
    {
        const int mid = lo + (hi - lo) / 2;
        /* median of three as pivot */
        double p0 = a[lo], p1 = a[mid], p2 = a[hi], piv;
        if ((p0 <= p1 && p1 <= p2) || (p2 <= p1 && p1 <= p0))
            piv = p1;
        else if ((p1 <= p0 && p0 <= p2) || (p2 <= p0 && p0 <= p1))
            piv = p0;
        else
            piv = p2;
        int i = lo, j = hi;
        while (i <= j)
        {
            while (a[i] < piv)
                ++i;
            while (a[j] > piv)
                --j;
            if (i <= j)
            {
                const double t = a[i];
                a[i] = a[j];
                a[j] = t;
                ++i;
                --j;
            }
        }
        if (kk <= j)
            hi = j;
        else if (kk >= i)
            lo = i;
        else
            return a[kk];
    }
    return a[kk];
}

static int cmp_i64(const void* x, const void* y)
{
    const int64_t a = *(const int64_t*)x, b = *(const int64_t*)y;
    return (a > b) - (a < b);
}

/* ------------------------------------------------------------------ */
/* KSG algorithm 2 for one pair: mir_xnyn (lib/kraskov.cpp:1228-1331)   */
/* as called by kraskov_wrap (lib/kraskov.cpp:2222-2282)                 */
/* ------------------------------------------------------------------ */

/* X: [3n][N] from gco_prepare; the x-marginal is atom a1, the y-marginal
 * atom a2 (kraskov_wrap copies a1's rows first).  Per-query outputs may be
 * NULL.  Returns MI = psi[N] + psi[K] - 1/K - (1/N) sum_i (psi[nx]+psi[ny])
 * with the sum taken in frame order, as mir_xnyn does (:1303-1318). */
double gco_ksg_pair_detail(const double* X, int N, int K, int a1, int a2, const double* psi,
                           int* nx_out, int* ny_out, double* epsx_out, double* epsy_out,
                           int* kth_out, double* dk_out)
{
    const double* xa[3] = {X + (size_t)(a1 * 3 + 0) * N, X + (size_t)(a1 * 3 + 1) * N,
                           X + (size_t)(a1 * 3 + 2) * N};
    const double* xb[3] = {X + (size_t)(a2 * 3 + 0) * N, X + (size_t)(a2 * 3 + 1) * N,
                           X + (size_t)(a2 * 3 + 2) * N};
    const int bs = gco_box_count(N, K);
    double*  dxv  = (double*)malloc(sizeof(double) * N);
    double*  dyv  = (double*)malloc(sizeof(double) * N);
    double*  v    = (double*)malloc(sizeof(double) * N);
    double*  tmp  = (double*)malloc(sizeof(double) * N);
    int64_t* tied = (int64_t*)malloc(sizeof(int64_t) * N);
    double   dxy2 = 0.0;
    for (int i = 0; i < N; ++i)
    {
        int m = 0;
        for (int j = 0; j < N; ++j)
        {
            double dx = 0.0, dy = 0.0;
            for (int d = 0; d < 3; ++d)
            {
                const double tx = fabs(xa[d][i] - xa[d][j]);
                const double ty = fabs(xb[d][i] - xb[d][j]);
                if (tx > dx)
                    dx = tx;
                if (ty > dy)
                    dy = ty;
            }
            dxv[j] = dx;
            dyv[j] = dy;
            v[j]   = dx > dy ? dx : dy;
            if (j != i)
                tmp[m++] = v[j];
        }
        const double dk = select_kth(tmp, m, K - 1);
        int c_less = 0, nt = 0;
        for (int j = 0; j < N; ++j)
        {
            if (j == i)
                continue;
            if (v[j] < dk)
                ++c_less;
            else if (v[j] == dk)
                tied[nt++] = scan_rank(xa[0], xb[0], N, i, j, bs);
        }
        const int need = K - c_less;
        qsort(tied, nt, sizeof(int64_t), cmp_i64);
        const int64_t rcut = tied[need - 1];
        double ex = 0.0, ey = 0.0;
        for (int j = 0; j < N; ++j)
        {
            if (j == i)
                continue;
            int in = v[j] < dk;
            if (!in && v[j] == dk)
                in = scan_rank(xa[0], xb[0], N, i, j, bs) <= rcut;
            if (in)
            {
                if (dxv[j] > ex)
                    ex = dxv[j];
                if (dyv[j] > ey)
                    ey = dyv[j];
            }
        }
        int nx = 0, ny = 0;
        for (int j = 0; j < N; ++j)
        {
            if (j == i)
                continue;
            if (dxv[j] <= ex)
                ++nx;
            if (dyv[j] <= ey)
                ++ny;
        }
        if (nx_out)
            nx_out[i] = nx;
        if (ny_out)
            ny_out[i] = ny;
        if (epsx_out)
            epsx_out[i] = ex;
        if (epsy_out)
            epsy_out[i] = ey;
        if (kth_out)
            kth_out[i] = (int)(rcut % N);
        if (dk_out)
            dk_out[i] = dk;
        dxy2 += psi[nx] + psi[ny];
    }
    free(dxv);
    free(dyv);
    free(v);
    free(tmp);
    free(tied);
    const double phiK = psi[K] - 1 / (1.0 * K);
    dxy2 /= N;
    return psi[N] + phiK - dxy2;
}

/* kraskov_corrmatrix (lib/correlation_core.cpp:324-459), CPU path:
 * zero fill, diagonal 2000, pairs a1 in [1,n), a2 < a1, symmetric write.
 * Returns nonzero on the reference's input errors (:327-330). */
int gco_ksg_matrix(const double* x, int natoms, int N, int K, int nthreads, double* mat)
{
    if (natoms < 2 || N <= K)
        return 1;
    double* X   = (double*)malloc(sizeof(double) * (size_t)3 * natoms * N);
    double* psi = (double*)malloc(sizeof(double) * (N + 1));
    gco_prepare(x, natoms, N, X, psi);
    memset(mat, 0, sizeof(double) * (size_t)natoms * natoms);
    for (int a = 0; a < natoms; ++a)
        mat[(size_t)a * natoms + a] = 2000.0;
#ifdef _OPENMP
    if (nthreads > 0)
        omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1)
#endif
    for (int a1 = 1; a1 < natoms; ++a1)
        for (int a2 = 0; a2 < a1; ++a2)
        {
            const double mi = gco_ksg_pair_detail(X, N, K, a1, a2, psi, NULL, NULL, NULL, NULL, NULL, NULL);
            mat[(size_t)a1 * natoms + a2] = mi;
            mat[(size_t)a2 * natoms + a1] = mi;
        }
    free(X);
    free(psi);
    return 0;
}

/* ------------------------------------------------------------------ */
/* Gaussian MI (lib/correlation_core.cpp:49-111, 140-166, 280-311)      */
/* ------------------------------------------------------------------ */

/* matrixDet: LU with partial pivoting on a copy (:49-98). */
static double gco_det(const double* m_in, int n)
{
    double m[36];
    memcpy(m, m_in, sizeof(double) * n * n);
    double sign = 1.0;
    for (int col = 0; col < n; ++col)
    {
        int    pivot = col;
        double best  = fabs(m[col * n + col]);
        for (int row = col + 1; row < n; ++row)
        {
            const double v = fabs(m[row * n + col]);
            if (v > best)
            {
                best  = v;
                pivot = row;
            }
        }
        if (best == 0.0)
            return 0.0;
        if (pivot != col)
        {
            for (int j = 0; j < n; ++j)
            {
                const double t   = m[col * n + j];
                m[col * n + j]   = m[pivot * n + j];
                m[pivot * n + j] = t;
            }
            sign = -sign;
        }
        const double diag = m[col * n + col];
        for (int row = col + 1; row < n; ++row)
        {
            const double factor = m[row * n + col] / diag;
            m[row * n + col]    = factor;
            for (int j = col + 1; j < n; ++j)
                m[row * n + j] -= factor * m[col * n + j];
        }
    }
    double det = sign;
    for (int i = 0; i < n; ++i)
        det *= m[i * n + i];
    return det;
}

/* entropy (:100-111). */
static double gco_entropy(const double* m, int n)
{
    const double det = gco_det(m, n);
    if (det <= 0.0)
        return 0.0;
    return 0.5 * (n * (1.0 + log(2.0 * 3.14159265358979323846)) + log(det));
}

/* covarianceMatrix (:140-166) into cov [3n][3n]. */
void gco_covariance(const double* x, int natoms, int N, double* cov)
{
    const int ncov = natoms * 3;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1)
#endif
    for (int i = 0; i < ncov; ++i)
    {
        const int a1 = i / 3, d1 = i % 3;
        for (int j = 0; j < ncov; ++j)
        {
            const int a2 = j / 3, d2 = j % 3;
            double    sum = 0.0;
            for (int f = 0; f < N; ++f)
                sum += x[(size_t)a1 * N * 3 + (size_t)f * 3 + d1] * x[(size_t)a2 * N * 3 + (size_t)f * 3 + d2];
            cov[(size_t)i * ncov + j] = sum / N;
        }
    }
}

/* gauss_corrmatrix (:280-311).  mat is not zero-filled first, as in the
 * reference; every entry is written. */
void gco_gauss_matrix(const double* x, int natoms, int N, double* mat)
{
    const int ncov = natoms * 3;
    double*   cov  = (double*)malloc(sizeof(double) * (size_t)ncov * ncov);
    gco_covariance(x, natoms, N, cov);
    for (int a1 = 0; a1 < natoms; ++a1)
    {
        mat[(size_t)a1 * natoms + a1] = 2000.0;
        for (int a2 = a1 + 1; a2 < natoms; ++a2)
        {
            double first[9], second[9], comb[36];
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c)
                {
                    first[r * 3 + c]        = cov[(size_t)(a1 * 3 + r) * ncov + a1 * 3 + c];
                    second[r * 3 + c]       = cov[(size_t)(a2 * 3 + r) * ncov + a2 * 3 + c];
                    const double cr         = cov[(size_t)(a1 * 3 + r) * ncov + a2 * 3 + c];
                    comb[r * 6 + c]         = first[r * 3 + c];
                    comb[(r + 3) * 6 + c + 3] = second[r * 3 + c];
                    comb[r * 6 + c + 3]     = cr;
                    comb[(c + 3) * 6 + r]   = cr;
                }
            const double e1 = gco_entropy(first, 3);
            const double e2 = gco_entropy(second, 3);
            const double mi = e1 + e2 - gco_entropy(comb, 6);
            mat[(size_t)a2 * natoms + a1] = mat[(size_t)a1 * natoms + a2] = mi;
        }
    }
    free(cov);
}

/* ------------------------------------------------------------------ */
/* GCMI (lib/gcmi.cpp)                                                  */
/* ------------------------------------------------------------------ */

/* gcmi_erfinv (lib/gcmi.cpp:26-79): Acklam's rational approximation of
 * the inverse normal CDF, mapped to erfinv, plus one Newton step. */
double gco_erfinv(double x)
{
    static const double a[] = {-3.969683028665376e+01, 2.209460984245205e+02, -2.759285104469687e+02,
                               1.383577518672690e+02,  -3.066479806614716e+01, 2.506628277459239e+00};
    static const double b[] = {-5.447609879822406e+01, 1.615858368580409e+02, -1.556989798598866e+02,
                               6.680131188771972e+01,  -1.328068155288572e+01};
    static const double c[] = {-7.784894002430293e-03, -3.223964580411365e-01, -2.400758277161838e+00,
                               -2.549732539343734e+00, 4.374664141464968e+00,  2.938163982698783e+00};
    static const double d[] = {7.784695709041462e-03, 3.224671290700398e-01, 2.445134137142996e+00,
                               3.754408661907416e+00};
    if (x >= 1.0)
        return 1e30;
    if (x <= -1.0)
        return -1e30;
    if (x == 0.0)
        return 0.0;
    const double p = (x + 1.0) * 0.5;
    double       r, q;
    if (p < 0.02425)
    {
        q = sqrt(-2.0 * log(p));
        r = (((((c[0] * q + c[1]) * q + c[2]) * q + c[3]) * q + c[4]) * q + c[5]) /
            ((((d[0] * q + d[1]) * q + d[2]) * q + d[3]) * q + 1.0);
    }
    else if (p <= 0.97575)
    {
        q              = p - 0.5;
        const double s = q * q;
        r = (((((a[0] * s + a[1]) * s + a[2]) * s + a[3]) * s + a[4]) * s + a[5]) * q /
            (((((b[0] * s + b[1]) * s + b[2]) * s + b[3]) * s + b[4]) * s + 1.0);
    }
    else
    {
        q = sqrt(-2.0 * log(1.0 - p));
        r = -(((((c[0] * q + c[1]) * q + c[2]) * q + c[3]) * q + c[4]) * q + c[5]) /
            ((((d[0] * q + d[1]) * q + d[2]) * q + d[3]) * q + 1.0);
    }
    r /= sqrt(2.0);
    r -= (erf(r) - x) * sqrt(3.14159265358979323846) * 0.5 * exp(r * r);
    return r;
}

static const double* g_sort_vals;
static int cmp_by_val(const void* x, const void* y)
{
    const double a = g_sort_vals[*(const int*)x], b = g_sort_vals[*(const int*)y];
    return (a > b) - (a < b);
}

/* copula_transform (lib/gcmi.cpp:95-146): z[comp][frame], midrank ties.
 * Not thread-safe (qsort comparator state). */
void gco_copula(const double* x, int natoms, int N, double* z)
{
    int*    idx = (int*)malloc(sizeof(int) * N);
    double* col = (double*)malloc(sizeof(double) * N);
    for (int atom = 0; atom < natoms; ++atom)
        for (int dim = 0; dim < 3; ++dim)
        {
            const int comp = atom * 3 + dim;
            for (int f = 0; f < N; ++f)
            {
                col[f] = x[(size_t)atom * N * 3 + (size_t)f * 3 + dim];
                idx[f] = f;
            }
            g_sort_vals = col;
            qsort(idx, N, sizeof(int), cmp_by_val);
            int r = 0;
            while (r < N)
            {
                int s = r + 1;
                while (s < N && col[idx[s]] == col[idx[r]])
                    ++s;
                double avg = 0.0;
                for (int t = r; t < s; ++t)
                {
                    const double p = (t + 0.5) / N;
                    avg += sqrt(2.0) * gco_erfinv(2.0 * p - 1.0);
                }
                avg /= (s - r);
                for (int t = r; t < s; ++t)
                    z[(size_t)comp * N + idx[t]] = avg;
                r = s;
            }
        }
    free(idx);
    free(col);
}

/* lu_det (lib/gcmi.cpp:152-184). */
static double gco_lu_det(const double* m_in, int n)
{
    double m[36];
    memcpy(m, m_in, sizeof(double) * n * n);
    double sign = 1.0;
    for (int col = 0; col < n; ++col)
    {
        int    pivot = col;
        double best  = fabs(m[col * n + col]);
        for (int row = col + 1; row < n; ++row)
        {
            const double v = fabs(m[row * n + col]);
            if (v > best)
            {
                best  = v;
                pivot = row;
            }
        }
        if (best == 0.0)
            return 0.0;
        if (pivot != col)
        {
            for (int j = 0; j < n; ++j)
            {
                const double t   = m[col * n + j];
                m[col * n + j]   = m[pivot * n + j];
                m[pivot * n + j] = t;
            }
            sign = -sign;
        }
        const double diag = m[col * n + col];
        for (int row = col + 1; row < n; ++row)
        {
            const double factor = m[row * n + col] / diag;
            for (int j = col + 1; j < n; ++j)
                m[row * n + j] -= factor * m[col * n + j];
        }
    }
    double det = sign;
    for (int i = 0; i < n; ++i)
        det *= m[i * n + i];
    return det;
}

/* gcmi_pair (lib/gcmi.cpp:190-231). */
double gco_gcmi_pair(const double* z, int N, int a1, int a2)
{
    double       cov6[36] = {0};
    const double invN     = 1.0 / N;
    for (int f = 0; f < N; ++f)
    {
        double v[6];
        for (int d = 0; d < 3; ++d)
        {
            v[d]     = z[(size_t)(a1 * 3 + d) * N + f];
            v[d + 3] = z[(size_t)(a2 * 3 + d) * N + f];
        }
        for (int r = 0; r < 6; ++r)
            for (int c = 0; c < 6; ++c)
                cov6[r * 6 + c] += v[r] * v[c];
    }
    for (int i = 0; i < 36; ++i)
        cov6[i] *= invN;
    double c1[9], c2[9];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
        {
            c1[r * 3 + c] = cov6[r * 6 + c];
            c2[r * 3 + c] = cov6[(r + 3) * 6 + c + 3];
        }
    const double d1 = gco_lu_det(c1, 3), d2 = gco_lu_det(c2, 3), dJ = gco_lu_det(cov6, 6);
    if (d1 <= 0.0 || d2 <= 0.0 || dJ <= 0.0)
        return 0.0;
    return 0.5 * (log(d1) + log(d2) - log(dJ));
}

/* gcmi_corrmatrix (lib/gcmi.cpp:246-317). */
int gco_gcmi_matrix(const double* x, int natoms, int N, double* mat)
{
    if (natoms < 2 || N < 6)
        return 1;
    memset(mat, 0, sizeof(double) * (size_t)natoms * natoms);
    double* z = (double*)malloc(sizeof(double) * (size_t)3 * natoms * N);
    gco_copula(x, natoms, N, z);
    for (int a = 0; a < natoms; ++a)
        mat[(size_t)a * natoms + a] = 2000.0;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1)
#endif
    for (int a1 = 1; a1 < natoms; ++a1)
        for (int a2 = 0; a2 < a1; ++a2)
        {
            const double mi = gco_gcmi_pair(z, N, a1, a2);
            mat[(size_t)a1 * natoms + a2] = mi;
            mat[(size_t)a2 * natoms + a1] = mi;
        }
    free(z);
    return 0;
}

/* ------------------------------------------------------------------ */
/* Transfer entropy (lib/transfer_entropy.cpp:41-221)                   */
/* ------------------------------------------------------------------ */

/* TE(a2 -> a1, lag) for one ordered pair, on raw mean-centred
 * coordinates x [natoms][N][3] (lib/transfer_entropy.cpp:121-204).  psi
 * is the table of digamma_table(N - lag) (:41-48).  Optional per-query
 * outputs (length N - lag): counts n_xp, n_xfxp, n_ypxp and eps_k. */
double gco_te_pair(const double* x, int N, int K, int lag, int a1, int a2, const double* psi,
                   int* nxp_out, int* nxfxp_out, int* nypxp_out, double* eps_out)
{
    const int     Nv = N - lag;
    const double* A  = x + (size_t)a1 * N * 3;
    const double* B  = x + (size_t)a2 * N * 3;
    double*       tmp = (double*)malloc(sizeof(double) * Nv);
    double        te  = 0.0;
    for (int qi = 0; qi < Nv; ++qi)
    {
        double q[9];
        for (int d = 0; d < 3; ++d)
        {
            q[d]     = A[(size_t)(qi + lag) * 3 + d];
            q[d + 3] = A[(size_t)qi * 3 + d];
            q[d + 6] = B[(size_t)qi * 3 + d];
        }
        int m = 0;
        for (int j = 0; j < Nv; ++j)
        {
            if (j == qi)
                continue;
            double dist = 0.0;
            for (int d = 0; d < 3; ++d)
            {
                dist = fmax(dist, fabs(q[d] - A[(size_t)(j + lag) * 3 + d]));
                dist = fmax(dist, fabs(q[d + 3] - A[(size_t)j * 3 + d]));
                dist = fmax(dist, fabs(q[d + 6] - B[(size_t)j * 3 + d]));
            }
            tmp[m++] = dist;
        }
        const double eps = select_kth(tmp, m, K - 1);
        int nxfxp = 0, nypxp = 0, nxp = 0;
        for (int j = 0; j < Nv; ++j)
        {
            if (j == qi)
                continue;
            double dfp = 0.0, dyp = 0.0, dp = 0.0;
            for (int d = 0; d < 3; ++d)
            {
                dfp = fmax(dfp, fabs(q[d] - A[(size_t)(j + lag) * 3 + d]));
                dfp = fmax(dfp, fabs(q[d + 3] - A[(size_t)j * 3 + d]));
            }
            for (int d = 0; d < 3; ++d)
            {
                dyp = fmax(dyp, fabs(q[d + 3] - A[(size_t)j * 3 + d]));
                dyp = fmax(dyp, fabs(q[d + 6] - B[(size_t)j * 3 + d]));
            }
            for (int d = 0; d < 3; ++d)
                dp = fmax(dp, fabs(q[d + 3] - A[(size_t)j * 3 + d]));
            if (dfp < eps)
                ++nxfxp;
            if (dyp < eps)
                ++nypxp;
            if (dp < eps)
                ++nxp;
        }
        const int ixf = nxfxp < Nv ? nxfxp : Nv;
        const int iyp = nypxp < Nv ? nypxp : Nv;
        const int ixp = nxp < Nv ? nxp : Nv;
        if (nxp_out)
            nxp_out[qi] = nxp;
        if (nxfxp_out)
            nxfxp_out[qi] = nxfxp;
        if (nypxp_out)
            nypxp_out[qi] = nypxp;
        if (eps_out)
            eps_out[qi] = eps;
        te += psi[K] + psi[ixp + 1] - psi[ixf + 1] - psi[iyp + 1];
    }
    free(tmp);
    return te / Nv;
}

/* digamma_table (lib/transfer_entropy.cpp:41-48). */
void gco_te_psi(int n, double* psi)
{
    for (int i = 0; i <= n; ++i)
        psi[i] = 0.0;
    psi[1] = -0.57721566490153;
    for (int i = 1; i < n; ++i)
        psi[i + 1] = psi[i] + 1.0 / i;
}

/* te_matrix (lib/transfer_entropy.cpp:63-221): mat[a1*n+a2] = TE(a2->a1),
 * zero diagonal; all zeros when N - lag <= k. */
void gco_te_matrix(const double* x, int natoms, int N, int K, int lag, int nthreads, double* mat)
{
    const int Nv = N - lag;
    memset(mat, 0, sizeof(double) * (size_t)natoms * natoms);
    if (Nv <= K)
        return;
    double* psi = (double*)malloc(sizeof(double) * (Nv + 1));
    gco_te_psi(Nv, psi);
#ifdef _OPENMP
    if (nthreads > 0)
        omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1) collapse(2)
#endif
    for (int a1 = 0; a1 < natoms; ++a1)
        for (int a2 = 0; a2 < natoms; ++a2)
        {
            if (a1 == a2)
                continue;
            mat[(size_t)a1 * natoms + a2] = gco_te_pair(x, N, K, lag, a1, a2, psi, NULL, NULL, NULL, NULL);
        }
    free(psi);
}

/* ------------------------------------------------------------------ */
/* pearsify and writers (lib/correlation_core.cpp:202-278, 461-469)     */
/* ------------------------------------------------------------------ */

void gco_pearsify(double* mat, int n, int dim)
{
    for (int i = 0; i < n * n; ++i)
        mat[i] = mat[i] > 0.0 ? sqrt(1.0 - exp(-2.0 / dim * mat[i])) : 0.0;
}

int gco_write_matrix(const double* mat, int n, const char* path)
{
    FILE* out = fopen(path, "w");
    if (!out)
        return 1;
    fprintf(out, "%d x %d [\n", n, n);
    int ncol = 0;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
        {
            fprintf(out, "%10.6g ", mat[(size_t)j * n + i]);
            if (++ncol > 20)
            {
                ncol = 0;
                fprintf(out, "\n");
            }
        }
    fprintf(out, "]\n");
    fclose(out);
    return 0;
}
