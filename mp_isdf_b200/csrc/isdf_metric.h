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

}  // namespace isdf
