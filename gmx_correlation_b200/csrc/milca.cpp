// Host side of the MILCA estimator family (lib/kraskov.cpp:347-2155): one
// C-ABI entry point per reference function, each a description of the
// variant for the shared engine in milca.cu.
//
// What the variants share and where they differ (all from lib/kraskov.cpp):
//  * variables: mi2 / mi2c / mi2r / mi2K / mi2h / mi2r_ take two 1-D rows;
//    red / redc / redr / redK / mi_d take dim 1-D rows; the *_xnyn forms take
//    an x block of dimx rows and a y block of dimy rows; redr_embed delay-
//    embeds each of dim rows into edim components (x[d][t + tau * e]);
//    mi_xnynKembed takes two blocks of dim rows.
//  * counts: 1-D variables of the make_box2 forms (and the 1-D blocks of the
//    *_xnyn forms) use the 1-D box count neiE1 with the caller's scal;
//    every other variable is counted exactly (neiE / neiEK).
//  * search grid: neiK's 2-D grid on components (0, dim-1) for red*, (0, 1)
//    for mi2* and mi_d, (0, dimx) for *_xnyn, (0, dim) for mi_xnynKembed,
//    (0, edim) of the embedded rows for redr_embed; BOX is the smallest power
//    of two with 0.5 BOX^2 K >= N (0.5 BOX^2 >= N for mi2r_; N before
//    embedding for redr_embed).
//  * order of the sums: the make_box2 forms loop over the frames in the
//    grid's cell order (make_box2 sorts the caller's rows in place); the
//    make_box2ind forms loop in frame order (make_box2ind also sorts the
//    caller's rows in place).  Both in-place sorts are repeated here on the
//    caller's rows after the estimate, so a caller sees the same arrays.
//  * the owner of Eps: first strict maximum over the variables (-1 when every
//    eps is 0) for the make_box2 forms; x when eps_x > eps_y, else y, for the
//    *_xnyn forms.
//  * association: *_xnyn add the two variables' terms first
//    (dxy += psi_x + psi_y); the others add term by term.

#include "gc_geom.h"
#include "gc_internal.h"
#include "gmx_corr_b200.h"
#include "host_common.h"
#include "milca.h"

#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

using namespace gc::host;

namespace gc {
cudaError_t launch_milca(const MilcaParams& p, const MilcaSum& s, cudaStream_t st);
}

namespace {

struct Group
{
    int    first, dim;
    bool   box1d;
    double scal;
};

struct Call
{
    const char*                name;
    std::vector<const double*> rows; // component rows of N frames (after any embedding)
    int                        N = 0, K = 0;
    int                        Nbox = 0, Kbox = 0; // BOX = f(Nbox, Kbox)
    std::vector<Group>         groups;
    int                        grid1 = 0, grid2 = 1;
    bool                       krange = false, tie_xy = false, pair_sum = false, box_order = false;
    const double*              psi = nullptr; // host, N + 1 entries
    const double*              phi = nullptr; // host, K + 1 entries, or null
    // results (k = K, or k = 1 .. K)
    std::vector<double> mic, mir;
    // per query (in summation order), for mi2h: eps per variable and Eps, counts, owner
    bool                want_detail = false;
    std::vector<double> eps;
    std::vector<int>    cnt, maxd, order;
};

gc_status bad(const Call& c, const std::string& m) { return fail(GC_ERR_INVALID, std::string(c.name) + ": " + m); }

// The permutation make_box2 / make_box2ind apply to the rows: cells of the
// 2-D grid (components grid1, grid2; cell = (int)(x * inveps) & (BOX-1)) in
// row-major order, frames of a cell in descending frame order (the cell
// lists are built by head insertion).  order[p] = frame at new position p.
std::vector<int> box_order(const double* c1, const double* c2, int N, int box)
{
    const int        inveps = box / 4, ib = box - 1;
    std::vector<int> head((size_t)box * box, -1), next((size_t)N, -1), order;
    order.reserve((size_t)N);
    for (int i = 0; i < N; ++i)
    {
        const int ix = ((int)(c1[i] * inveps)) & ib, iy = ((int)(c2[i] * inveps)) & ib;
        next[(size_t)i]                    = head[(size_t)ix * box + iy];
        head[(size_t)ix * box + iy]        = i;
    }
    for (int cell = 0; cell < box * box; ++cell)
        for (int e = head[(size_t)cell]; e >= 0; e = next[(size_t)e])
            order.push_back(e);
    return order;
}

gc_status run(Call& c)
{
    const int G = (int)c.groups.size(), D = (int)c.rows.size();
    if (G < 1 || G > gc::kMilcaMaxGroups)
        return bad(c, "between 1 and 8 variables");
    if (c.K < 1 || c.K >= c.N)
        return bad(c, "need 1 <= K < N (K neighbours besides the query frame)");
    if (c.krange && c.K > gc::kMilcaMaxRangeK)
        return bad(c, "the k = 1 .. K forms take K <= 1024");
    if (!c.psi)
        return bad(c, "null psi table");
    for (const double* r : c.rows)
        if (!r)
            return bad(c, "null coordinate row");
    for (int d = 0; d < D; ++d)
        for (int t = 0; t < c.N; ++t)
            if (!std::isfinite(c.rows[(size_t)d][t]))
                return fail(GC_ERR_NONFINITE, std::string(c.name) + ": non-finite coordinate");
    const int bs1 = c.N - 5;
    for (const Group& g : c.groups)
        if (g.box1d)
        {
            if (bs1 < 1)
                return bad(c, "the 1-D box counts need N > 5");
            const double* r = c.rows[(size_t)g.first];
            for (int t = 0; t < c.N; ++t)
            {
                const double v = r[t] * g.scal;
                if (!(v > -1.0 && v < (double)bs1 + 1.0))
                    return bad(c, "scal puts a value outside the 1-D boxes 0 .. N-5 (values must lie in [0, (N-5)/scal])");
            }
        }
    const int box = gc::ksg_box_count(c.Nbox, c.Kbox);

    DeviceScope dev(-1);
    GC_TRY(dev.st);
    // the call's own stream; pooled buffers, returned only after the stream
    // has drained (the guard is destroyed before them, on every path)
    StreamScope ss;
    GC_TRY(ss.init(nullptr));
    const cudaStream_t st = ss.s;
    const int          Kr = c.krange ? c.K : 1;
    const size_t       nq = (size_t)c.N * Kr;
    PoolBuf<double>    X, psi, phi, eps, mic, mir;
    PoolBuf<int>       cnt, maxd, order, status;
    struct Drain
    {
        cudaStream_t s;
        ~Drain() { cudaStreamSynchronize(s); }
    } drain{st};
    GC_TRY(X.alloc((size_t)D * c.N));
    for (int d = 0; d < D; ++d)
        GC_TRY_CUDA(cudaMemcpyAsync(X.p + (size_t)d * c.N, c.rows[(size_t)d], sizeof(double) * c.N,
                                    cudaMemcpyHostToDevice, st));
    GC_TRY(psi.alloc((size_t)c.N + 1));
    GC_TRY_CUDA(cudaMemcpyAsync(psi.p, c.psi, sizeof(double) * (c.N + 1), cudaMemcpyHostToDevice, st));
    if (c.phi)
    {
        GC_TRY(phi.alloc((size_t)c.K + 1));
        GC_TRY_CUDA(cudaMemcpyAsync(phi.p, c.phi, sizeof(double) * (c.K + 1), cudaMemcpyHostToDevice, st));
    }
    GC_TRY(eps.alloc(nq * (G + 1)));
    GC_TRY(cnt.alloc(nq * G * 2));
    GC_TRY(maxd.alloc(nq));
    GC_TRY(status.alloc(1));
    GC_TRY(mic.alloc((size_t)Kr));
    GC_TRY(mir.alloc((size_t)Kr));
    c.order.resize((size_t)c.N);
    if (c.box_order)
        c.order = box_order(c.rows[(size_t)c.grid1], c.rows[(size_t)c.grid2], c.N, box);
    else
        for (int i = 0; i < c.N; ++i)
            c.order[(size_t)i] = i;
    GC_TRY(order.alloc((size_t)c.N));
    GC_TRY_CUDA(cudaMemcpyAsync(order.p, c.order.data(), sizeof(int) * c.N, cudaMemcpyHostToDevice, st));
    GC_TRY_CUDA(cudaMemsetAsync(status.p, 0, sizeof(int), st));

    gc::MilcaParams p{};
    p.X = X.p;
    p.D = D;
    p.N = c.N;
    p.G = G;
    p.K = c.K;
    for (int g = 0; g < G; ++g)
    {
        p.gfirst[g] = c.groups[(size_t)g].first;
        p.gdim[g]   = c.groups[(size_t)g].dim;
        p.gbox1d[g] = c.groups[(size_t)g].box1d;
        p.gscal[g]  = c.groups[(size_t)g].scal;
    }
    p.bs1        = bs1;
    p.grid1      = c.grid1;
    p.grid2      = c.grid2;
    p.box        = box;
    p.rank_shift = gc::rank_top_shift(box, c.N);
    p.krange     = c.krange;
    p.tie_xy     = c.tie_xy;
    p.cnt        = cnt.p;
    p.maxd       = maxd.p;
    p.eps        = eps.p;
    p.status     = status.p;
    gc::MilcaSum s{};
    s.order    = order.p;
    s.psi      = psi.p;
    s.phi      = c.phi ? phi.p : nullptr;
    s.N        = c.N;
    s.G        = G;
    s.K        = c.K;
    s.krange   = c.krange;
    s.pair_sum = c.pair_sum;
    s.mic      = mic.p;
    s.mir      = mir.p;
    GC_TRY_CUDA(gc::launch_milca(p, s, st));
    int stw = 0;
    GC_TRY_CUDA(cudaMemcpyAsync(&stw, status.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    GC_TRY_CUDA(cudaStreamSynchronize(st));
    GC_TRY(status_to_error(stw));
    c.mic.resize((size_t)Kr);
    c.mir.resize((size_t)Kr);
    GC_TRY_CUDA(cudaMemcpyAsync(c.mic.data(), mic.p, sizeof(double) * Kr, cudaMemcpyDeviceToHost, st));
    GC_TRY_CUDA(cudaMemcpyAsync(c.mir.data(), mir.p, sizeof(double) * Kr, cudaMemcpyDeviceToHost, st));
    if (c.want_detail)
    {
        c.eps.resize(nq * (G + 1));
        c.cnt.resize(nq * G * 2);
        c.maxd.resize(nq);
        GC_TRY_CUDA(cudaMemcpyAsync(c.eps.data(), eps.p, sizeof(double) * c.eps.size(), cudaMemcpyDeviceToHost, st));
        GC_TRY_CUDA(cudaMemcpyAsync(c.cnt.data(), cnt.p, sizeof(int) * c.cnt.size(), cudaMemcpyDeviceToHost, st));
        GC_TRY_CUDA(cudaMemcpyAsync(c.maxd.data(), maxd.p, sizeof(int) * c.maxd.size(), cudaMemcpyDeviceToHost, st));
    }
    GC_TRY_CUDA(cudaStreamSynchronize(st));
    return GC_OK;
}

// The in-place row sort of make_box2 / make_box2ind on the caller's rows.
void permute_rows(double** x, int D, const std::vector<int>& order)
{
    std::vector<double> tmp(order.size());
    for (int d = 0; d < D; ++d)
    {
        for (size_t p = 0; p < order.size(); ++p)
            tmp[p] = x[d][order[p]];
        std::copy(tmp.begin(), tmp.end(), x[d]);
    }
}

gc_status check_rows(const char* name, double** x, int D)
{
    if (!x)
        return fail(GC_ERR_INVALID, std::string(name) + ": null coordinate rows");
    for (int d = 0; d < D; ++d)
        if (!x[d])
            return fail(GC_ERR_INVALID, std::string(name) + ": null coordinate row");
    return GC_OK;
}

// dim 1-D variables counted by the 1-D box rule, make_box2 forms.
gc_status run_1d(const char* name, double** x, int dim, int N, int K, int Kbox, int grid2, const double* psi,
                 const double* scal, const double* phi, bool krange, Call& c)
{
    GC_TRY(check_rows(name, x, dim));
    if (dim < 1)
        return fail(GC_ERR_INVALID, std::string(name) + ": dim >= 1");
    if (!scal)
        return fail(GC_ERR_INVALID, std::string(name) + ": null scal");
    c.name = name;
    for (int d = 0; d < dim; ++d)
    {
        c.rows.push_back(x[d]);
        c.groups.push_back({d, 1, true, scal[d]});
    }
    c.N         = N;
    c.K         = K;
    c.Nbox      = N;
    c.Kbox      = Kbox;
    c.grid1     = 0;
    c.grid2     = grid2;
    c.krange    = krange;
    c.box_order = true;
    c.psi       = psi;
    c.phi       = phi;
    GC_TRY(run(c));
    permute_rows(x, dim, c.order);
    return GC_OK;
}

// Two blocks (x: dimx rows, y: dimy rows), make_box2ind forms.
gc_status run_xy(const char* name, double** x, int dimx, int dimy, int N, int K, const double* psi,
                 const double* scal, bool krange, bool box1d, Call& c)
{
    if (dimx < 1 || dimy < 1)
        return fail(GC_ERR_INVALID, std::string(name) + ": dimx, dimy >= 1");
    GC_TRY(check_rows(name, x, dimx + dimy));
    if (box1d && (dimx == 1 || dimy == 1) && !scal)
        return fail(GC_ERR_INVALID, std::string(name) + ": null scal");
    c.name = name;
    for (int d = 0; d < dimx + dimy; ++d)
        c.rows.push_back(x[d]);
    c.groups.push_back({0, dimx, box1d && dimx == 1, box1d && dimx == 1 ? scal[0] : 0.0});
    c.groups.push_back({dimx, dimy, box1d && dimy == 1, box1d && dimy == 1 ? scal[dimx] : 0.0});
    c.N        = N;
    c.K        = K;
    c.Nbox     = N;
    c.Kbox     = K;
    c.grid1    = 0;
    c.grid2    = dimx;
    c.krange   = krange;
    c.tie_xy   = true;
    c.pair_sum = true;
    c.psi      = psi;
    GC_TRY(run(c));
    // make_box2ind sorted the joint rows in place by the same cells
    const int ND = dimx + dimy;
    permute_rows(x, ND, box_order(x[0], x[dimx], N, gc::ksg_box_count(N, K)));
    return GC_OK;
}

void put_range(const Call& c, double* mi_cr)
{
    for (int k = 0; k < c.K; ++k)
    {
        mi_cr[2 * k]     = c.mic[(size_t)k];
        mi_cr[2 * k + 1] = c.mir[(size_t)k];
    }
}

} // namespace

extern "C" {

gc_status gc_milca_mi2(double** x, int N, int K, const double* psi, const double* scal, double* mic, double* mir)
{
    Call c;
    GC_TRY(run_1d("mi2", x, 2, N, K, K, 1, psi, scal, nullptr, false, c));
    if (mic)
        *mic = c.mic[0];
    if (mir)
        *mir = c.mir[0];
    return GC_OK;
}

gc_status gc_milca_mi2c(double** x, int N, int K, const double* psi, const double* scal, double* mic)
{
    return gc_milca_mi2(x, N, K, psi, scal, mic, nullptr);
}

gc_status gc_milca_mi2r(double** x, int N, int K, const double* psi, const double* scal, double* mir)
{
    return gc_milca_mi2(x, N, K, psi, scal, nullptr, mir);
}

gc_status gc_milca_mi2r_(double** x, int N, int K, const double* psi, const double* scal, double* mir)
{
    Call c;
    GC_TRY(run_1d("mi2r_", x, 2, N, K, 1, 1, psi, scal, nullptr, false, c));
    if (mir)
        *mir = c.mir[0];
    return GC_OK;
}

gc_status gc_milca_red(double** x, int dim, int N, int K, const double* psi, const double* scal, double* mic,
                       double* mir)
{
    Call c;
    GC_TRY(run_1d("red", x, dim, N, K, K, dim - 1, psi, scal, nullptr, false, c));
    if (mic)
        *mic = c.mic[0];
    if (mir)
        *mir = c.mir[0];
    return GC_OK;
}

gc_status gc_milca_redc(double** x, int dim, int N, int K, const double* psi, const double* scal, double* mic)
{
    return gc_milca_red(x, dim, N, K, psi, scal, mic, nullptr);
}

gc_status gc_milca_redr(double** x, int dim, int N, int K, const double* psi, const double* scal, double* mir)
{
    return gc_milca_red(x, dim, N, K, psi, scal, nullptr, mir);
}

gc_status gc_milca_redK(double** x, int dim, int N, int K, const double* psi, const double* scal, double* mi_cr)
{
    if (!mi_cr)
        return fail(GC_ERR_INVALID, "redK: null mi_cr");
    Call c;
    GC_TRY(run_1d("redK", x, dim, N, K, K, dim - 1, psi, scal, nullptr, true, c));
    put_range(c, mi_cr);
    return GC_OK;
}

gc_status gc_milca_mi2K(double** x, int N, int K, const double* psi, const double* scal, double* mi_cr)
{
    if (!mi_cr)
        return fail(GC_ERR_INVALID, "mi2K: null mi_cr");
    Call c;
    GC_TRY(run_1d("mi2K", x, 2, N, K, K, 1, psi, scal, nullptr, true, c));
    put_range(c, mi_cr);
    return GC_OK;
}

gc_status gc_milca_mi_d(double** x, int dim, int N, int K, float* mi_cr, const double* psi, const double* phi,
                        double minx, double maxx, double miny, double maxy)
{
    if (!mi_cr || !phi)
        return fail(GC_ERR_INVALID, "mi_d: null mi_cr or phi");
    if (dim < 2)
        return fail(GC_ERR_INVALID, "mi_d: dim >= 2");
    // scal[d & 1] = BOX1 / (max - min) of x (even rows) and y (odd rows)
    const double sc[2] = {(double)(N - 5) / (maxx - minx), (double)(N - 5) / (maxy - miny)};
    std::vector<double> scal((size_t)dim);
    for (int d = 0; d < dim; ++d)
        scal[(size_t)d] = sc[d & 1];
    Call c;
    GC_TRY(run_1d("mi_d", x, dim, N, K, K, 1, psi, scal.data(), phi, true, c));
    for (int k = 0; k < K; ++k)
    {
        mi_cr[2 * k]     = (float)c.mic[(size_t)k];
        mi_cr[2 * k + 1] = (float)c.mir[(size_t)k];
    }
    return GC_OK;
}

gc_status gc_milca_mi2h(double** x, int N, int K, const double* psi, const double* scal, double* mic, double* mir,
                        double* hc, double* hr)
{
    Call c;
    c.want_detail = true;
    GC_TRY(run_1d("mi2h", x, 2, N, K, K, 1, psi, scal, nullptr, false, c));
    // the entropy terms of mi2h (lib/kraskov.cpp:1811-1949), summed on the
    // host in the reference's order from the device's per-frame eps and counts
    const int           dim = 2;
    std::vector<double> phi((size_t)N + 1, 0.0);
    for (int i = 1; i <= N; ++i)
        phi[(size_t)i] = psi[i] - (dim - 1) / (1.0 * i);
    double h1[2] = {0.0, 0.0}, h2[2] = {0.0, 0.0}, hj1 = 0.0, hj2 = 0.0;
    for (int q = 0; q < N; ++q)
    {
        const int     i  = c.order[(size_t)q];
        const double* e  = &c.eps[(size_t)i * (dim + 1)];
        const int*    n  = &c.cnt[(size_t)i * dim * 2];
        const int     md = c.maxd[(size_t)i];
        const double  Eps = e[dim];
        // a count of -1 reads the word before the table in the reference;
        // taken as 0, as on the device
        auto ps = [&](int v) { return v < 0 ? 0.0 : psi[v]; };
        auto ph = [&](int v) { return v < 0 ? 0.0 : phi[(size_t)v]; };
        for (int d = 0; d < dim; ++d)
        {
            if (d == md)
                h1[d] += std::log(Eps) - ps(n[2 * d]);
            else
                h1[d] += std::log(Eps) - ps(n[2 * d] + 1);
            h2[d] += std::log(e[d]) - ph(n[2 * d + 1]);
            hj1 += std::log(Eps);
            hj2 += std::log(e[d]);
        }
    }
    hj1 /= N;
    double vhc = psi[N] - psi[K] + hj1;
    hj2 /= N;
    double vhr = psi[N] - phi[(size_t)K] + hj2;
    double t_d1 = +1e30, t_d2 = +1e30;
    std::fprintf(stdout, "hj_c\t%1.3f\t\t\t\thj_r\t%1.3f\n", vhc, vhr);
    for (int d = 0; d < dim; ++d)
    {
        h1[d] /= N;
        h1[d] += psi[N];
        h2[d] /= N;
        h2[d] += psi[N];
        if (h1[d] < t_d1)
            t_d1 = h1[d];
        if (h2[d] < t_d2)
            t_d2 = h2[d];
        if ((vhc - h1[d]) < t_d1)
            t_d1 = vhc - h1[d];
        if ((vhr - h2[d]) < t_d2)
            t_d2 = vhr - h2[d];
        std::fprintf(stdout, "h[%d]_c\t%1.3f\thcond[%d]_c\t%1.3f\th[%d]_r\t%1.3f\thcond[%d]_r\t%1.3f\n", d, h1[d], d,
                     vhc - h1[d], d, h2[d], d, vhr - h2[d]);
    }
    vhc -= 2 * t_d1;
    vhr -= 2 * t_d2;
    if (mic)
        *mic = c.mic[0];
    if (mir)
        *mir = c.mir[0];
    if (hc)
        *hc = vhc;
    if (hr)
        *hr = vhr;
    return GC_OK;
}

gc_status gc_milca_mi_xnyn(double** x, int dimx, int dimy, int N, int K, const double* psi, const double* scal,
                           double* mic, double* mir)
{
    Call c;
    GC_TRY(run_xy("mi_xnyn", x, dimx, dimy, N, K, psi, scal, false, true, c));
    if (mic)
        *mic = c.mic[0];
    if (mir)
        *mir = c.mir[0];
    return GC_OK;
}

gc_status gc_milca_mic_xnyn(double** x, int dimx, int dimy, int N, int K, const double* psi, const double* scal,
                            double* mic)
{
    return gc_milca_mi_xnyn(x, dimx, dimy, N, K, psi, scal, mic, nullptr);
}

gc_status gc_milca_mir_xnyn(double** x, int dimx, int dimy, int N, int K, const double* psi, const double* scal,
                            double* mir)
{
    return gc_milca_mi_xnyn(x, dimx, dimy, N, K, psi, scal, nullptr, mir);
}

gc_status gc_milca_mi_xnynK(double** x, int dimx, int dimy, int N, int K, const double* psi, const double* scal,
                            double* mi_cr)
{
    if (!mi_cr)
        return fail(GC_ERR_INVALID, "mi_xnynK: null mi_cr");
    Call c;
    GC_TRY(run_xy("mi_xnynK", x, dimx, dimy, N, K, psi, scal, true, true, c));
    put_range(c, mi_cr);
    return GC_OK;
}

gc_status gc_milca_mi_xnynKembed(double** x, int dim, int N, int K, const double* psi, double* mi_cr)
{
    if (!mi_cr)
        return fail(GC_ERR_INVALID, "mi_xnynKembed: null mi_cr");
    Call c;
    GC_TRY(run_xy("mi_xnynKembed", x, dim, dim, N, K, psi, nullptr, true, false, c));
    put_range(c, mi_cr);
    return GC_OK;
}

gc_status gc_milca_redr_embed(double** x, int dim, int edim, int tau, int N, int K, const double* psi, double* mir)
{
    GC_TRY(check_rows("redr_embed", x, dim));
    if (dim < 2 || edim < 1 || tau < 0)
        return fail(GC_ERR_INVALID, "redr_embed: dim >= 2, edim >= 1, tau >= 0");
    const int N_ = N - (edim - 1) * tau;
    if (N_ < 2)
        return fail(GC_ERR_INVALID, "redr_embed: N - (edim-1)*tau frames must remain");
    // component d*edim + e of frame t is x[d][t + tau*e] (the reference
    // copies these rows and leaves the caller's rows in place)
    Call c;
    c.name = "redr_embed";
    for (int d = 0; d < dim * edim; ++d)
        c.rows.push_back(x[d / edim] + (size_t)tau * (d % edim));
    for (int d = 0; d < dim; ++d)
        c.groups.push_back({d * edim, edim, false, 0.0});
    c.N     = N_;
    c.K     = K;
    c.Nbox  = N;
    c.Kbox  = K;
    c.grid1 = 0;
    c.grid2 = edim;
    c.psi   = psi;
    GC_TRY(run(c));
    if (mir)
        *mir = c.mir[0];
    return GC_OK;
}

} // extern "C"
