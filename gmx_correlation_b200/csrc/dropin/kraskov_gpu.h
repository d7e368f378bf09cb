// Drop-in declarations of the reference's legacy device-facing KSG entry
// points (lib/kraskov_gpu.h:20,32).  The reference declares them only in
// builds configured with its CUDA switch (GMX_CORRELATION_USE_CUDA); this
// library always exports them, so a front end built with or without that
// switch links.  Implemented in dropin.cpp over gc_gpu_available and
// gc_ksg_matrix_prepared.
#pragma once

#include "correlation_core.h"

// True when a B200-class (compute capability 10.x) device is present.
bool kraskov_gpu_probe();

// KSG MI matrix mat [natoms*natoms] from the prepared workspace kr
// (kraskov_prepare): diagonal 2000, both triangles written.  No k limit.
void kraskov_corrmatrix_gpu(const t_kraskov* kr, int natoms, double* mat, int k);
