// Drop-in transfer-entropy interface: the signatures of the reference's
// lib/transfer_entropy.h:8-10.  mat[a1*n+a2] = TE(a2 -> a1, lag).
#pragma once
#include "correlation_core.h"

void te_matrix(const t_traj* traj, double* mat, int k, int lag, bool use_gpu = false, int nthreads = 0);
bool te_gpu_available();
