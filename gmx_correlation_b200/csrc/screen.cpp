// C ABI of the learned KSG screen (no counterpart in the reference): feature
// extraction, the networks' training and inference, and screened KSG.
//
// The reference computes KSG on every pair (lib/correlation_core.cpp:324-459).
// The screen predicts r(MI) for every pair from cheap features with an
// ensemble of small BF16 networks, then runs the exact KSG path on the pairs
// whose prediction is uncertain or close to the reported threshold (the
// mean + 0.5 sd of positive off-diagonal values, bin/analyze_matrix.py:173-190),
// and on a seeded random audit sample whose exact values measure the error
// of the predictions the screen kept.

#include "gmx_corr_b200.h"
#include "gc_geom.h"
#include "gc_internal.h"
#include "host_common.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>
#include <string>
#include <vector>

using namespace gc::host;

static_assert(GC_SCREEN_IN == gc::kScreenIn, "feature width");
static_assert(GC_SCREEN_BASE == gc::kScreenBase && GC_SCREEN_HIST == gc::kScreenHist, "feature layout");
static_assert(GC_SCREEN_HIDDEN == gc::kMlpHidden, "hidden width");

namespace {

constexpr int kMaxBatch   = 8192;
constexpr int kMaxMembers = 16;

// Activations and gradients of one batch of M rows for every member.
struct Workspace
{
    int           M = 0;
    DevBuf<float> X, Z1, H1, Z2, H2, Z3, H3, Y, dY, dA, dB;
};

} // namespace

struct gc_screen_model
{
    int           device  = 0;
    int           members = 0;
    DevBuf<float> params, grad, adam_m, adam_v;
    DevBuf<float> feat_mean, feat_sd, pca; // pca: mean[64] then comp[kScreenComp][64]
    bool          has_input = false;
    DevBuf<float> hyper, loss;
    DevBuf<int>   counters; // [0] Adam step, [1] batch index within the epoch
    Workspace     ws;
    cudaStream_t  stream = nullptr;
    ~gc_screen_model()
    {
        if (stream)
            cudaStreamDestroy(stream);
    }
};

namespace {

gc_status ensure_ws(gc_screen_model* m, int M)
{
    Workspace& w = m->ws;
    if (w.M >= M)
        return GC_OK;
    const size_t E = (size_t)m->members, H = gc::kMlpHidden;
    GC_TRY(w.X.alloc((size_t)M * gc::kScreenIn));
    for (DevBuf<float>* b : {&w.Z1, &w.H1, &w.Z2, &w.H2, &w.Z3, &w.H3, &w.dA, &w.dB})
        GC_TRY(b->alloc(E * M * H));
    GC_TRY(w.Y.alloc(E * M));
    GC_TRY(w.dY.alloc(E * M));
    w.M = M;
    return GC_OK;
}

gc::MlpGemm gemm_base(int M, int N, int K, int Z)
{
    gc::MlpGemm g;
    std::memset(&g, 0, sizeof(g));
    g.M = M;
    g.N = N;
    g.K = K;
    g.Z = Z;
    return g;
}

// Forward pass of M standardised rows in ws.X through every member; the
// outputs go to Y[z * sYz + m].
gc_status forward(gc_screen_model* m, int M, float* Y, long sYz, cudaStream_t s)
{
    Workspace&   w = m->ws;
    const long   P = gc::kMlpStride, Hd = gc::kMlpHidden, act = (long)M * Hd;
    const float* W = m->params.p;
    const int    E = m->members;
    const float* in[3]  = {w.X.p, w.H1.p, w.H2.p};
    float*       zp[3]  = {w.Z1.p, w.Z2.p, w.Z3.p};
    float*       hp[3]  = {w.H1.p, w.H2.p, w.H3.p};
    const long   ow[3]  = {gc::kMlpOffW1, gc::kMlpOffW2, gc::kMlpOffW3};
    const long   ob[3]  = {gc::kMlpOffB1, gc::kMlpOffB2, gc::kMlpOffB3};
    const int    kin[3] = {gc::kScreenIn, gc::kMlpHidden, gc::kMlpHidden};
    for (int l = 0; l < 3; ++l)
    {
        gc::MlpGemm g = gemm_base(M, (int)Hd, kin[l], E);
        g.A           = in[l];
        g.sAz         = l == 0 ? 0 : act;
        g.sAm         = kin[l];
        g.sAk         = 1;
        g.B           = W + ow[l];
        g.sBz         = P;
        g.sBn         = kin[l];
        g.sBk         = 1;
        g.C           = zp[l];
        g.sCz         = act;
        g.ldc         = Hd;
        g.bias        = W + ob[l];
        g.sbz         = P;
        g.H           = hp[l];
        g.epi         = gc::kEpiBiasGelu;
        GC_TRY_CUDA(gc::launch_mlp_gemm(g, s));
    }
    gc::MlpGemm g = gemm_base(M, 1, (int)Hd, E);
    g.A           = w.H3.p;
    g.sAz         = act;
    g.sAm         = Hd;
    g.sAk         = 1;
    g.B           = W + gc::kMlpOffW4;
    g.sBz         = P;
    g.sBn         = Hd;
    g.sBk         = 1;
    g.C           = Y;
    g.sCz         = sYz;
    g.ldc         = 1;
    g.bias        = W + gc::kMlpOffB4;
    g.sbz         = P;
    g.epi         = gc::kEpiBias;
    GC_TRY_CUDA(gc::launch_mlp_gemm(g, s));
    return GC_OK;
}

// Backward pass of the mean squared error: ws.dY must hold dLoss/dY; writes
// the gradient of every parameter to m->grad.
gc_status backward(gc_screen_model* m, int M, cudaStream_t s)
{
    Workspace& w = m->ws;
    const long P = gc::kMlpStride, Hd = gc::kMlpHidden, act = (long)M * Hd;
    const int  E = m->members;
    float*     G = m->grad.p;
    const float* W = m->params.p;

    // layer 4: dW4 = dY^T H3, db4 = sum dY, dH3 = dY W4
    {
        gc::MlpGemm g = gemm_base(1, (int)Hd, M, E);
        g.A = w.dY.p, g.sAz = M, g.sAm = 1, g.sAk = 1;
        g.B = w.H3.p, g.sBz = act, g.sBn = 1, g.sBk = Hd;
        g.C = G + gc::kMlpOffW4, g.sCz = P, g.ldc = Hd;
        g.epi = gc::kEpiStore;
        GC_TRY_CUDA(gc::launch_mlp_gemm(g, s));
        GC_TRY_CUDA(gc::launch_mlp_colsum(w.dY.p, M, 1, E, G + gc::kMlpOffB4, P, s));
        gc::MlpGemm h = gemm_base(M, (int)Hd, 1, E);
        h.A = w.dY.p, h.sAz = M, h.sAm = 1, h.sAk = 1;
        h.B = W + gc::kMlpOffW4, h.sBz = P, h.sBn = 1, h.sBk = Hd;
        h.C = w.dA.p, h.sCz = act, h.ldc = Hd;
        h.epi = gc::kEpiStore;
        GC_TRY_CUDA(gc::launch_mlp_gemm(h, s));
        GC_TRY_CUDA(gc::launch_mlp_gelu_back(w.Z3.p, w.dA.p, (long)E * act, s));
    }
    // hidden layers 3, 2, 1: dZ in cur; X is the layer's input
    float*       cur[3]   = {w.dA.p, w.dB.p, w.dA.p}; // dZ3, dZ2, dZ1
    float*       nxt[3]   = {w.dB.p, w.dA.p, nullptr};
    const float* xin[3]   = {w.H2.p, w.H1.p, w.X.p};
    const float* zprev[3] = {w.Z2.p, w.Z1.p, nullptr};
    const long   ow[3]    = {gc::kMlpOffW3, gc::kMlpOffW2, gc::kMlpOffW1};
    const long   ob[3]    = {gc::kMlpOffB3, gc::kMlpOffB2, gc::kMlpOffB1};
    for (int l = 0; l < 3; ++l)
    {
        const int  kin = l == 2 ? gc::kScreenIn : gc::kMlpHidden;
        const long sx  = l == 2 ? 0 : act;
        gc::MlpGemm g  = gemm_base((int)Hd, kin, M, E);
        g.A = cur[l], g.sAz = act, g.sAm = 1, g.sAk = Hd;
        g.B = xin[l], g.sBz = sx, g.sBn = 1, g.sBk = kin;
        g.C = G + ow[l], g.sCz = P, g.ldc = kin;
        g.epi = gc::kEpiStore;
        GC_TRY_CUDA(gc::launch_mlp_gemm(g, s));
        GC_TRY_CUDA(gc::launch_mlp_colsum(cur[l], M, (int)Hd, E, G + ob[l], P, s));
        if (!nxt[l])
            break;
        gc::MlpGemm h = gemm_base(M, (int)Hd, (int)Hd, E);
        h.A = cur[l], h.sAz = act, h.sAm = Hd, h.sAk = 1;
        h.B = W + ow[l], h.sBz = P, h.sBn = 1, h.sBk = Hd;
        h.C = nxt[l], h.sCz = act, h.ldc = Hd;
        h.epi = gc::kEpiStore;
        GC_TRY_CUDA(gc::launch_mlp_gemm(h, s));
        GC_TRY_CUDA(gc::launch_mlp_gelu_back(zprev[l], nxt[l], (long)E * act, s));
    }
    return GC_OK;
}

// One training step on batch `step` of the permutation idx: gather,
// forward, loss, backward, Adam, step counters.
gc_status train_step(gc_screen_model* m, const float* F, const float* t, const long* idx, int M, cudaStream_t s)
{
    Workspace& w = m->ws;
    int*       c = m->counters.p;
    GC_TRY_CUDA(gc::launch_mlp_gather(F, idx, c + 1, M, m->feat_mean.p, m->feat_sd.p, w.X.p, s));
    GC_TRY(forward(m, M, w.Y.p, M, s));
    GC_TRY_CUDA(gc::launch_mlp_loss(w.Y.p, t, idx, c + 1, M, m->members, w.dY.p, m->loss.p, s));
    GC_TRY(backward(m, M, s));
    GC_TRY_CUDA(gc::launch_mlp_adam(m->params.p, m->grad.p, m->adam_m.p, m->adam_v.p,
                                    (long)m->members * gc::kMlpStride, m->hyper.p, c, s));
    GC_TRY_CUDA(gc::launch_mlp_tick(c, c + 1, s));
    return GC_OK;
}

gc_status check_model(const gc_screen_model* m, bool need_input)
{
    if (!m)
        return fail(GC_ERR_INVALID, "null screen model");
    if (need_input && !m->has_input)
        return fail(GC_ERR_INVALID, "screen model has no input standardisation (gc_screen_model_set_input)");
    return GC_OK;
}

// Host (a1, a2) table of an explicit pair list, validated against npairs.
gc_status list_to_ab(const int64_t* list, long n, long npairs, std::vector<int2>& ab)
{
    ab.resize((size_t)n);
    for (long i = 0; i < n; ++i)
    {
        if (list[i] < 0 || list[i] >= npairs)
            return fail(GC_ERR_INVALID, "pair list entry out of range");
        int a1, a2;
        gc::pair_from_index(list[i], &a1, &a2);
        ab[(size_t)i] = make_int2(a1, a2);
    }
    return GC_OK;
}

// Features of `count` pairs (pair_begin.. or the device list d_ab) of the
// device coordinates d_xyz into the device rows d_out.
gc_status features_device(const double* d_xyz, int natoms, int T, int k, long pair_begin, long count,
                          const int2* d_ab, const float* d_pca, float* d_out, cudaStream_t s)
{
    // pooled scratch (no cudaMalloc / cudaFree per call); the stream is
    // synchronised before the blocks return to the pool
    PoolBuf<double>        stats;
    PoolBuf<unsigned char> bins;
    GC_TRY(stats.alloc((size_t)natoms * gc::kScreenStat));
    GC_TRY(bins.alloc((size_t)natoms * T));
    const int         width = d_pca ? gc::kScreenIn : gc::kScreenBase + gc::kScreenHist;
    const cudaError_t e     = gc::launch_screen_features(d_xyz, natoms, T, k, pair_begin, count, d_ab, d_pca,
                                                         gc::kScreenComp, stats.p, bins.p, d_out, width, s);
    const cudaError_t w     = cudaStreamSynchronize(s);
    GC_TRY_CUDA(e);
    GC_TRY_CUDA(w);
    return GC_OK;
}

gc_status check_screen_traj(const gc_traj_view* traj, int k)
{
    GC_TRY(check_view(traj));
    if (traj->natoms < 2)
        return fail(GC_ERR_INVALID, "the screen needs at least two atoms");
    if (k < 1 || traj->nframes <= k)
        return fail(GC_ERR_INVALID, "need k >= 1 and nframes > k");
    if (traj->nframes > 16384)
        return fail(GC_ERR_INVALID, "the screen's features support nframes <= 16384");
    return GC_OK;
}

// Predictions of every member for n device rows F (raw features) into
// Y[z * n + i], in batches of the workspace size.
gc_status predict_device(gc_screen_model* m, const float* d_F, long n, float* d_Y, cudaStream_t s)
{
    const int M = (int)std::min<long>(kMaxBatch, std::max<long>(n, 1));
    GC_TRY(ensure_ws(m, M));
    for (long off = 0; off < n; off += M)
    {
        const int Mc = (int)std::min<long>(M, n - off);
        GC_TRY_CUDA(gc::launch_mlp_gather(d_F + off * gc::kScreenIn, nullptr, nullptr, Mc, m->feat_mean.p,
                                          m->feat_sd.p, m->ws.X.p, s));
        GC_TRY(forward(m, Mc, d_Y + off, n, s));
    }
    return GC_OK;
}

// r(MI) of one value through gc_pearsify, so screened and plain matrices agree bit for bit.
double pearsify_r(double mi)
{
    gc_pearsify(&mi, 1, 3);
    return mi;
}

} // namespace

extern "C" {

long gc_screen_param_stride(void) { return gc::kMlpStride; }

int gc_screen_model_members(const gc_screen_model* m) { return m ? m->members : 0; }

gc_status gc_screen_model_create(int members, uint64_t seed, int device, gc_screen_model** out)
{
    if (!out)
        return fail(GC_ERR_INVALID, "null output pointer");
    *out = nullptr;
    if (members < 1 || members > kMaxMembers)
        return fail(GC_ERR_INVALID, "members must be in [1, 16]");
    DeviceScope dev(device);
    GC_TRY(dev.st);
    auto* m    = new gc_screen_model();
    m->members = members;
    cudaGetDevice(&m->device);
    const size_t n = (size_t)members * gc::kMlpStride;
    gc_status    st = GC_OK;
    if ((st = m->params.alloc(n)) || (st = m->grad.alloc(n)) || (st = m->adam_m.alloc(n)) ||
        (st = m->adam_v.alloc(n)) || (st = m->feat_mean.alloc(gc::kScreenIn)) ||
        (st = m->feat_sd.alloc(gc::kScreenIn)) || (st = m->pca.alloc(64 + 64 * gc::kScreenComp)) ||
        (st = m->hyper.alloc(4)) || (st = m->loss.alloc(kMaxMembers)) || (st = m->counters.alloc(2)))
    {
        delete m;
        return st;
    }
    if (cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess)
    {
        cudaGetLastError();
        delete m;
        return fail(GC_ERR_CUDA, "cudaStreamCreate failed");
    }
    // uniform(+-1/sqrt(fan_in)) weights and biases, per member from the seed
    std::vector<float> h(n, 0.0f);
    std::mt19937_64    rng(seed);
    struct Seg
    {
        long off, count;
        int  fan_in;
    };
    const Seg segs[] = {{gc::kMlpOffW1, (long)gc::kMlpHidden * gc::kScreenIn, gc::kScreenIn},
                        {gc::kMlpOffB1, gc::kMlpHidden, gc::kScreenIn},
                        {gc::kMlpOffW2, (long)gc::kMlpHidden * gc::kMlpHidden, gc::kMlpHidden},
                        {gc::kMlpOffB2, gc::kMlpHidden, gc::kMlpHidden},
                        {gc::kMlpOffW3, (long)gc::kMlpHidden * gc::kMlpHidden, gc::kMlpHidden},
                        {gc::kMlpOffB3, gc::kMlpHidden, gc::kMlpHidden},
                        {gc::kMlpOffW4, gc::kMlpHidden, gc::kMlpHidden},
                        {gc::kMlpOffB4, 1, gc::kMlpHidden}};
    for (int z = 0; z < members; ++z)
        for (const Seg& sg : segs)
        {
            std::uniform_real_distribution<float> u(-1.0f / std::sqrt((float)sg.fan_in),
                                                    1.0f / std::sqrt((float)sg.fan_in));
            for (long i = 0; i < sg.count; ++i)
                h[(size_t)z * gc::kMlpStride + sg.off + i] = u(rng);
        }
    cudaError_t e = cudaMemcpy(m->params.p, h.data(), n * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemset(m->grad.p, 0, n * sizeof(float));
    if (e == cudaSuccess)
        e = cudaMemset(m->adam_m.p, 0, n * sizeof(float));
    if (e == cudaSuccess)
        e = cudaMemset(m->adam_v.p, 0, n * sizeof(float));
    if (e == cudaSuccess)
        e = cudaMemset(m->counters.p, 0, 2 * sizeof(int));
    if (e != cudaSuccess)
    {
        cudaGetLastError();
        delete m;
        return fail(GC_ERR_CUDA, std::string("screen model set-up: ") + cudaGetErrorString(e));
    }
    *out = m;
    return GC_OK;
}

void gc_screen_model_destroy(gc_screen_model* m)
{
    if (!m)
        return;
    DeviceScope dev(m->device);
    delete m;
}

gc_status gc_screen_model_get_params(const gc_screen_model* m, float* params)
{
    GC_TRY(check_model(m, false));
    if (!params)
        return fail(GC_ERR_INVALID, "null parameter buffer");
    DeviceScope dev(m->device);
    GC_TRY(dev.st);
    GC_TRY_CUDA(cudaMemcpy(params, m->params.p, sizeof(float) * m->members * gc::kMlpStride, cudaMemcpyDeviceToHost));
    return GC_OK;
}

gc_status gc_screen_model_set_params(gc_screen_model* m, const float* params)
{
    GC_TRY(check_model(m, false));
    if (!params)
        return fail(GC_ERR_INVALID, "null parameter buffer");
    DeviceScope dev(m->device);
    GC_TRY(dev.st);
    const size_t n = (size_t)m->members * gc::kMlpStride;
    GC_TRY_CUDA(cudaMemcpy(m->params.p, params, sizeof(float) * n, cudaMemcpyHostToDevice));
    GC_TRY_CUDA(cudaMemset(m->adam_m.p, 0, sizeof(float) * n));
    GC_TRY_CUDA(cudaMemset(m->adam_v.p, 0, sizeof(float) * n));
    GC_TRY_CUDA(cudaMemset(m->counters.p, 0, 2 * sizeof(int)));
    return GC_OK;
}

gc_status gc_screen_model_set_input(gc_screen_model* m, const float* feat_mean, const float* feat_sd,
                                    const float* pca_mean, const float* pca_comp)
{
    GC_TRY(check_model(m, false));
    if (!feat_mean || !feat_sd || !pca_mean || !pca_comp)
        return fail(GC_ERR_INVALID, "null standardisation or basis array");
    for (int c = 0; c < gc::kScreenIn; ++c)
        if (!(feat_sd[c] > 0.0f) || !std::isfinite(feat_sd[c]) || !std::isfinite(feat_mean[c]))
            return fail(GC_ERR_INVALID, "feature standard deviations must be finite and positive");
    DeviceScope dev(m->device);
    GC_TRY(dev.st);
    GC_TRY_CUDA(cudaMemcpy(m->feat_mean.p, feat_mean, sizeof(float) * gc::kScreenIn, cudaMemcpyHostToDevice));
    GC_TRY_CUDA(cudaMemcpy(m->feat_sd.p, feat_sd, sizeof(float) * gc::kScreenIn, cudaMemcpyHostToDevice));
    GC_TRY_CUDA(cudaMemcpy(m->pca.p, pca_mean, sizeof(float) * 64, cudaMemcpyHostToDevice));
    GC_TRY_CUDA(cudaMemcpy(m->pca.p + 64, pca_comp, sizeof(float) * 64 * gc::kScreenComp, cudaMemcpyHostToDevice));
    m->has_input = true;
    return GC_OK;
}

gc_status gc_screen_features(const gc_traj_view* traj, int k, const gc_opts* opts, const float* pca_mean,
                             const float* pca_comp, float* out)
{
    GC_TRY(check_screen_traj(traj, k));
    if (!out)
        return fail(GC_ERR_INVALID, "null output");
    if ((pca_mean == nullptr) != (pca_comp == nullptr))
        return fail(GC_ERR_INVALID, "give both pca_mean and pca_comp, or neither");
    const gc_opts o      = opts ? *opts : defaults();
    const long    npairs = (long)traj->natoms * (traj->natoms - 1) / 2;
    long          begin = 0, count = npairs;
    std::vector<int2> ab;
    if (o.pair_list)
    {
        if (o.pair_list_len < 0)
            return fail(GC_ERR_INVALID, "negative pair list length");
        GC_TRY(list_to_ab(o.pair_list, o.pair_list_len, npairs, ab));
        count = o.pair_list_len;
    }
    else if (o.pair_end > 0 || o.pair_begin > 0)
    {
        const long end = o.pair_end > 0 ? o.pair_end : npairs;
        if (o.pair_begin < 0 || o.pair_begin > end || end > npairs)
            return fail(GC_ERR_INVALID, "pair range outside [0, natoms*(natoms-1)/2]");
        begin = o.pair_begin;
        count = end - begin;
    }
    DeviceScope dev(o.device);
    GC_TRY(dev.st);
    StreamScope ss;
    GC_TRY(ss.init(o.stream));
    const int      width = pca_mean ? gc::kScreenIn : gc::kScreenBase + gc::kScreenHist;
    DevBuf<double> d_xyz;
    DevBuf<float>  d_out, d_pca;
    DevBuf<int2>   d_ab;
    GC_TRY(d_xyz.alloc((size_t)traj->natoms * traj->nframes * 3));
    GC_TRY(d_out.alloc((size_t)std::max<long>(count, 1) * width));
    GC_TRY(upload_traj(traj, d_xyz.p, ss.s));
    if (pca_mean)
    {
        GC_TRY(d_pca.alloc(64 + 64 * gc::kScreenComp));
        GC_TRY_CUDA(cudaMemcpyAsync(d_pca.p, pca_mean, 64 * sizeof(float), cudaMemcpyHostToDevice, ss.s));
        GC_TRY_CUDA(cudaMemcpyAsync(d_pca.p + 64, pca_comp, 64 * gc::kScreenComp * sizeof(float),
                                    cudaMemcpyHostToDevice, ss.s));
    }
    if (!ab.empty())
    {
        GC_TRY(d_ab.alloc(ab.size()));
        GC_TRY_CUDA(cudaMemcpyAsync(d_ab.p, ab.data(), ab.size() * sizeof(int2), cudaMemcpyHostToDevice, ss.s));
    }
    GC_TRY(features_device(d_xyz.p, traj->natoms, traj->nframes, k, begin, count, ab.empty() ? nullptr : d_ab.p,
                           pca_mean ? d_pca.p : nullptr, d_out.p, ss.s));
    if (count > 0)
        GC_TRY_CUDA(cudaMemcpy(out, d_out.p, sizeof(float) * count * width, cudaMemcpyDeviceToHost));
    return GC_OK;
}

gc_status gc_screen_train(gc_screen_model* m, const float* feats, const float* target, long n, int epochs, int batch,
                          float lr, uint64_t seed, float* loss_per_epoch)
{
    GC_TRY(check_model(m, true));
    if (!feats || !target)
        return fail(GC_ERR_INVALID, "null training data");
    if (batch < 1 || batch > kMaxBatch)
        return fail(GC_ERR_INVALID, "batch must be in [1, 8192]");
    if (n < batch || epochs < 1 || !(lr > 0.0f))
        return fail(GC_ERR_INVALID, "need n >= batch, epochs >= 1 and lr > 0");
    DeviceScope dev(m->device);
    GC_TRY(dev.st);
    cudaStream_t  s = m->stream;
    DevBuf<float> d_F, d_t;
    DevBuf<long>  d_idx;
    GC_TRY(d_F.alloc((size_t)n * gc::kScreenIn));
    GC_TRY(d_t.alloc((size_t)n));
    GC_TRY(d_idx.alloc((size_t)n));
    GC_TRY_CUDA(cudaMemcpyAsync(d_F.p, feats, sizeof(float) * n * gc::kScreenIn, cudaMemcpyHostToDevice, s));
    GC_TRY_CUDA(cudaMemcpyAsync(d_t.p, target, sizeof(float) * n, cudaMemcpyHostToDevice, s));
    GC_TRY(ensure_ws(m, batch));

    // One training step captured into a graph; the batch index and the Adam
    // step live in device counters, so the same graph serves every step.
    cudaGraph_t     graph = nullptr;
    cudaGraphExec_t exec  = nullptr;
    GC_TRY_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    const gc_status cst = train_step(m, d_F.p, d_t.p, d_idx.p, batch, s);
    const cudaError_t ce = cudaStreamEndCapture(s, &graph);
    if (cst != GC_OK)
    {
        if (graph)
            cudaGraphDestroy(graph);
        return cst;
    }
    GC_TRY_CUDA(ce);
    cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    GC_TRY_CUDA(ie);
    struct ExecGuard
    {
        cudaGraphExec_t e;
        ~ExecGuard() { cudaGraphExecDestroy(e); }
    } guard{exec};

    const long         steps = n / batch;
    std::vector<long>  perm((size_t)n);
    std::mt19937_64    rng(seed);
    std::vector<float> loss((size_t)m->members);
    for (int ep = 0; ep < epochs; ++ep)
    {
        std::iota(perm.begin(), perm.end(), 0L);
        std::shuffle(perm.begin(), perm.end(), rng);
        const double c        = 0.5 * (1.0 + std::cos(3.14159265358979323846 * ep / std::max(1, epochs - 1)));
        const float  hyper[4] = {(float)(lr * (0.05 + 0.95 * c)), 0.9f, 0.999f, 1e-8f};
        GC_TRY_CUDA(cudaMemcpyAsync(d_idx.p, perm.data(), sizeof(long) * n, cudaMemcpyHostToDevice, s));
        GC_TRY_CUDA(cudaMemcpyAsync(m->hyper.p, hyper, sizeof(hyper), cudaMemcpyHostToDevice, s));
        GC_TRY_CUDA(cudaMemsetAsync(m->counters.p + 1, 0, sizeof(int), s));
        GC_TRY_CUDA(cudaMemsetAsync(m->loss.p, 0, sizeof(float) * m->members, s));
        for (long st = 0; st < steps; ++st)
            GC_TRY_CUDA(cudaGraphLaunch(exec, s));
        GC_TRY_CUDA(cudaMemcpyAsync(loss.data(), m->loss.p, sizeof(float) * m->members, cudaMemcpyDeviceToHost, s));
        GC_TRY_CUDA(cudaStreamSynchronize(s));
        if (loss_per_epoch)
        {
            double acc = 0.0;
            for (float l : loss)
                acc += l;
            loss_per_epoch[ep] = (float)(acc / (m->members * (double)steps));
        }
    }
    return GC_OK;
}

gc_status gc_screen_grad(gc_screen_model* m, const float* feats, const float* target, long n, float* grad, float* loss)
{
    GC_TRY(check_model(m, true));
    if (!feats || !target || !grad)
        return fail(GC_ERR_INVALID, "null argument");
    if (n < 1 || n > kMaxBatch)
        return fail(GC_ERR_INVALID, "gc_screen_grad takes 1..8192 rows");
    DeviceScope dev(m->device);
    GC_TRY(dev.st);
    cudaStream_t  s = m->stream;
    DevBuf<float> d_F, d_t;
    GC_TRY(d_F.alloc((size_t)n * gc::kScreenIn));
    GC_TRY(d_t.alloc((size_t)n));
    GC_TRY_CUDA(cudaMemcpyAsync(d_F.p, feats, sizeof(float) * n * gc::kScreenIn, cudaMemcpyHostToDevice, s));
    GC_TRY_CUDA(cudaMemcpyAsync(d_t.p, target, sizeof(float) * n, cudaMemcpyHostToDevice, s));
    GC_TRY(ensure_ws(m, (int)n));
    const int M = (int)n;
    GC_TRY_CUDA(cudaMemsetAsync(m->loss.p, 0, sizeof(float) * m->members, s));
    GC_TRY_CUDA(gc::launch_mlp_gather(d_F.p, nullptr, nullptr, M, m->feat_mean.p, m->feat_sd.p, m->ws.X.p, s));
    GC_TRY(forward(m, M, m->ws.Y.p, M, s));
    GC_TRY_CUDA(gc::launch_mlp_loss(m->ws.Y.p, d_t.p, nullptr, nullptr, M, m->members, m->ws.dY.p, m->loss.p, s));
    GC_TRY(backward(m, M, s));
    GC_TRY_CUDA(cudaMemcpyAsync(grad, m->grad.p, sizeof(float) * m->members * gc::kMlpStride, cudaMemcpyDeviceToHost, s));
    if (loss)
        GC_TRY_CUDA(cudaMemcpyAsync(loss, m->loss.p, sizeof(float) * m->members, cudaMemcpyDeviceToHost, s));
    GC_TRY_CUDA(cudaStreamSynchronize(s));
    return GC_OK;
}

gc_status gc_screen_predict(gc_screen_model* m, const float* feats, long n, float* out)
{
    GC_TRY(check_model(m, true));
    if (!feats || !out || n < 0)
        return fail(GC_ERR_INVALID, "null argument or negative row count");
    if (n == 0)
        return GC_OK;
    DeviceScope dev(m->device);
    GC_TRY(dev.st);
    cudaStream_t  s = m->stream;
    DevBuf<float> d_F, d_Y;
    GC_TRY(d_F.alloc((size_t)n * gc::kScreenIn));
    GC_TRY(d_Y.alloc((size_t)n * m->members));
    GC_TRY_CUDA(cudaMemcpyAsync(d_F.p, feats, sizeof(float) * n * gc::kScreenIn, cudaMemcpyHostToDevice, s));
    GC_TRY(predict_device(m, d_F.p, n, d_Y.p, s));
    GC_TRY_CUDA(cudaMemcpyAsync(out, d_Y.p, sizeof(float) * n * m->members, cudaMemcpyDeviceToHost, s));
    GC_TRY_CUDA(cudaStreamSynchronize(s));
    return GC_OK;
}

void gc_screen_opts_init(gc_screen_opts* o)
{
    if (!o)
        return;
    o->audit_frac = 0.05;
    o->sigma_max  = 0.0;
    o->margin     = 0.0;
    o->seed       = 12345;
}

gc_status gc_ksg_screened(const gc_traj_view* traj, int k, gc_screen_model* m, const gc_screen_opts* sopts,
                          const gc_opts* opts, double* r, gc_screen_report* report)
{
    GC_TRY(check_model(m, true));
    GC_TRY(check_screen_traj(traj, k));
    if (!r)
        return fail(GC_ERR_INVALID, "null output matrix");
    gc_screen_opts so;
    gc_screen_opts_init(&so);
    if (sopts)
        so = *sopts;
    if (!(so.audit_frac >= 0.0 && so.audit_frac <= 1.0))
        return fail(GC_ERR_INVALID, "audit_frac must be in [0, 1]");
    gc_opts o = opts ? *opts : defaults();
    o.pair_list     = nullptr;
    o.pair_list_len = 0;
    o.pair_begin    = 0;
    o.pair_end      = 0;
    o.detail_nx = o.detail_ny = nullptr;
    if (o.device < 0)
        o.device = m->device;
    if (o.device != m->device)
        return fail(GC_ERR_INVALID, "the screen model lives on another device");
    DeviceScope dev(o.device);
    GC_TRY(dev.st);
    StreamScope ss;
    GC_TRY(ss.init(o.stream));
    cudaStream_t s = ss.s;
    o.stream       = s;

    const int  n = traj->natoms, T = traj->nframes;
    const long P = (long)n * (n - 1) / 2;
    cudaEvent_t ev[4];
    for (auto& e : ev)
        GC_TRY_CUDA(cudaEventCreate(&e));
    struct EvGuard
    {
        cudaEvent_t* e;
        ~EvGuard()
        {
            for (int i = 0; i < 4; ++i)
                cudaEventDestroy(e[i]);
        }
    } evg{ev};

    DevBuf<double> d_xyz;
    DevBuf<float>  d_F, d_Y, d_mean, d_sd;
    GC_TRY(d_xyz.alloc((size_t)n * T * 3));
    GC_TRY(d_F.alloc((size_t)P * gc::kScreenIn));
    GC_TRY(d_Y.alloc((size_t)P * m->members));
    GC_TRY(d_mean.alloc((size_t)P));
    GC_TRY(d_sd.alloc((size_t)P));
    GC_TRY(upload_traj(traj, d_xyz.p, s));
    GC_TRY_CUDA(cudaEventRecord(ev[0], s));
    GC_TRY(features_device(d_xyz.p, n, T, k, 0, P, nullptr, m->pca.p, d_F.p, s));
    GC_TRY_CUDA(cudaEventRecord(ev[1], s));
    GC_TRY(predict_device(m, d_F.p, P, d_Y.p, s));
    GC_TRY_CUDA(gc::launch_mlp_ensemble(d_Y.p, P, m->members, d_mean.p, d_sd.p, s));
    GC_TRY_CUDA(cudaEventRecord(ev[2], s));
    std::vector<float> mean((size_t)P), sd((size_t)P);
    GC_TRY_CUDA(cudaMemcpyAsync(mean.data(), d_mean.p, sizeof(float) * P, cudaMemcpyDeviceToHost, s));
    GC_TRY_CUDA(cudaMemcpyAsync(sd.data(), d_sd.p, sizeof(float) * P, cudaMemcpyDeviceToHost, s));
    GC_TRY_CUDA(cudaStreamSynchronize(s));

    // reported threshold of the predicted matrix (analyze_matrix auto_threshold)
    double sum = 0.0, sum2 = 0.0;
    long   npos = 0;
    for (long p = 0; p < P; ++p)
        if (mean[(size_t)p] > 0.0f)
        {
            sum += mean[(size_t)p];
            ++npos;
        }
    const double mu = npos ? sum / npos : 0.0;
    for (long p = 0; p < P; ++p)
        if (mean[(size_t)p] > 0.0f)
            sum2 += (mean[(size_t)p] - mu) * (mean[(size_t)p] - mu);
    const double thr = npos ? mu + 0.5 * std::sqrt(sum2 / npos) : 0.0;

    std::vector<char> flag((size_t)P, 0), audit((size_t)P, 0);
    long              nflag = 0;
    for (long p = 0; p < P; ++p)
        if (sd[(size_t)p] > so.sigma_max || std::fabs(mean[(size_t)p] - thr) < so.margin)
        {
            flag[(size_t)p] = 1;
            ++nflag;
        }
    const long         naudit = (long)std::llround(so.audit_frac * P);
    std::vector<long>  order((size_t)P);
    std::iota(order.begin(), order.end(), 0L);
    std::mt19937_64 rng(so.seed);
    for (long i = 0; i < naudit; ++i)
    {
        std::uniform_int_distribution<long> u(i, P - 1);
        std::swap(order[(size_t)i], order[(size_t)u(rng)]);
        audit[(size_t)order[(size_t)i]] = 1;
    }
    std::vector<int64_t> list;
    for (long p = 0; p < P; ++p)
        if (flag[(size_t)p] || audit[(size_t)p])
            list.push_back(p);

    std::vector<double> mi_exact(list.size(), 0.0);
    float               ms_ksg = 0.0f;
    if (2 * (long)list.size() >= P)
    {
        // Most pairs exact: the whole matrix through gc_ksg_matrix (its plan
        // stays cached between calls) costs less than a plan over the list.
        const auto          t0 = std::chrono::steady_clock::now();
        std::vector<double> full((size_t)n * n);
        GC_TRY(gc_ksg_matrix(traj, k, &o, full.data()));
        for (size_t i = 0; i < list.size(); ++i)
        {
            int a1, a2;
            gc::pair_from_index(list[i], &a1, &a2);
            mi_exact[i] = full[(size_t)a1 * n + a2];
        }
        ms_ksg = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    else if (!list.empty())
    {
        gc_opts lo       = o;
        lo.pair_list     = list.data();
        lo.pair_list_len = (long)list.size();
        gc_ksg_plan* plan = nullptr;
        GC_TRY(gc_ksg_plan_create(n, T, k, &lo, &plan));
        struct PlanGuard
        {
            gc_ksg_plan* p;
            ~PlanGuard() { gc_ksg_plan_destroy(p); }
        } pg{plan};
        DevBuf<double> d_mi;
        GC_TRY(d_mi.alloc(list.size()));
        GC_TRY_CUDA(cudaEventRecord(ev[3], s));
        GC_TRY(gc_ksg_plan_run(plan, d_xyz.p, d_mi.p, s));
        GC_TRY(gc_ksg_plan_sync(plan));
        cudaEvent_t done;
        GC_TRY_CUDA(cudaEventCreate(&done));
        cudaEventRecord(done, s);
        GC_TRY_CUDA(cudaMemcpyAsync(mi_exact.data(), d_mi.p, sizeof(double) * list.size(), cudaMemcpyDeviceToHost, s));
        GC_TRY_CUDA(cudaStreamSynchronize(s));
        cudaEventElapsedTime(&ms_ksg, ev[3], done);
        cudaEventDestroy(done);
    }

    // assemble: pearsified r, diagonal 1
    for (int a = 0; a < n; ++a)
        r[(size_t)a * n + a] = 1.0;
    for (long p = 0; p < P; ++p)
    {
        int a1, a2;
        gc::pair_from_index(p, &a1, &a2);
        const double v           = std::max(0.0, (double)mean[(size_t)p]);
        r[(size_t)a1 * n + a2]   = v;
        r[(size_t)a2 * n + a1]   = v;
    }
    double maxdr = 0.0, sq = 0.0, fmax = 0.0;
    long   acc_n = 0;
    for (size_t i = 0; i < list.size(); ++i)
    {
        const long p = list[i];
        int        a1, a2;
        gc::pair_from_index(p, &a1, &a2);
        const double rx = pearsify_r(mi_exact[i]);
        if (audit[(size_t)p])
        {
            const double pred = std::max(0.0, (double)mean[(size_t)p]);
            if (!flag[(size_t)p])
            {
                const double d = std::fabs(pred - rx);
                maxdr          = std::max(maxdr, d);
                sq += d * d;
                ++acc_n;
            }
        }
        r[(size_t)a1 * n + a2] = rx;
        r[(size_t)a2 * n + a1] = rx;
        if (audit[(size_t)p])
            fmax = std::max(fmax, std::fabs(r[(size_t)a1 * n + a2] - rx));
    }
    if (report)
    {
        std::memset(report, 0, sizeof(*report));
        report->pairs          = P;
        report->flagged        = nflag;
        report->audited        = naudit;
        report->exact          = (long)list.size();
        report->audit_accepted = acc_n;
        report->threshold      = thr;
        report->audit_max_dr   = maxdr;
        report->audit_rms_dr   = acc_n ? std::sqrt(sq / acc_n) : 0.0;
        report->final_max_dr   = fmax;
        cudaEventElapsedTime(&report->ms_features, ev[0], ev[1]);
        cudaEventElapsedTime(&report->ms_mlp, ev[1], ev[2]);
        report->ms_ksg = ms_ksg;
    }
    return GC_OK;
}

} // extern "C"
