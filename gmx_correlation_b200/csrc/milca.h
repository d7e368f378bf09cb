// The MILCA estimator family of the reference's lib/kraskov.cpp (:347-2155:
// mi2, mi2c, mi2r, red, redc, redr, redr_embed, mi_xnyn, mic_xnyn, mir_xnyn,
// redK, mi2K, mi_xnynK, mi_xnynKembed, mi2h, mi_d, mi2r_) on one exact FP64
// engine.  Shared by the kernels (milca.cu) and the host (milca.cpp).
#pragma once

#include <cstdint>

namespace gc {

constexpr int kMilcaMaxGroups = 8;
constexpr int kMilcaMaxRangeK = 1024; // k = 1 .. K variants: the K nearest are sorted in shared memory

// One estimator call.  Coordinates are component-major, X[c * N + t], in the
// caller's frame order.  Variables ("groups") are contiguous component
// ranges; the joint space is the max-norm over all components.
struct MilcaParams
{
    const double* X;
    int           D, N, G, K;
    int           gfirst[kMilcaMaxGroups], gdim[kMilcaMaxGroups];
    // 1: the group (one component) is counted by the reference's 1-D box
    // rule (neiE1, lib/kraskov.cpp:92-112) with gscal; 0: exact max-norm count
    // (neiE / neiEK, :113-255)
    int    gbox1d[kMilcaMaxGroups];
    double gscal[kMilcaMaxGroups];
    int    bs1;          // the 1-D boxes' last index (N - 5)
    int    grid1, grid2; // components of neiK's 2-D search grid
    int    box;          // that grid's BOX
    int    rank_shift;   // top byte of the tie-break rank keys
    int    krange;       // 0: k = K only; 1: every k = 1 .. K
    int    tie_xy;       // 1: the first group owns Eps only when eps_0 > eps_1 (two groups), else the first strict argmax
    int*    cnt;         // [N][Kr][G][2]: count at Eps (n1), count at the group's own eps (n2)
    int*    maxd;        // [N][Kr]: the group owning Eps (-1: none)
    double* eps;         // [N][Kr][G + 1]: per-group eps, then Eps
    int*    status;
};

// Summation of one variant (the reference's association order).
struct MilcaSum
{
    const int*    order;   // queries in the order the reference sums them
    const double* psi;     // digamma table, psi[0 .. N]
    const double* phi;     // phi[k] table or null (then psi[k] - (G-1)/k)
    int           N, G, K, krange;
    int           pair_sum; // 1: dxy += (term_0 + term_1); 0: dxy += term, group by group
    double*       mic;      // [Kr] or null
    double*       mir;      // [Kr] or null
};

} // namespace gc
