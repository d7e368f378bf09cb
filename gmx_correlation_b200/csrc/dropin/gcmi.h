// Drop-in GCMI interface: the signatures of the reference's lib/gcmi.h:8-10.
#pragma once
#include "correlation_core.h"

void gcmi_corrmatrix(const t_traj* traj, double* mat, bool use_gpu = false, int nthreads = 0);
bool gcmi_gpu_available();
