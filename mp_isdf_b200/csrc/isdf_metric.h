// Grid Coulomb metric of interpolation vectors (python/isdf.py:48-97).
#pragma once

#include "isdf_internal.h"

namespace isdf {

constexpr int kMaxMetricAnchors = 64;

// left: kl x n, right: kr x n (row-major, leading dimensions >= n, not
// weight-scaled), xyz: n x 3, w: n (device); metric_host: kl x kr, symmetrised
// when requested (left = right, kl = kr).
void grid_metric(const double* left, int64_t ldl, int kl, const double* right, int64_t ldr, int kr,
                 const double* xyz, const double* w, int64_t n, bool symmetrize, double* metric_host,
                 cudaStream_t s);

// ISDF J and K of a density matrix on the device (X: k x nao anchor AO values,
// Z: k x k metric, D: nao x nao; J, K: nao x nao, symmetrised; either may be null).
void isdf_jk_device(int64_t nao, int64_t k, const double* X, const double* Z, const double* D, double* J,
                    double* K, cudaStream_t s);

}  // namespace isdf
