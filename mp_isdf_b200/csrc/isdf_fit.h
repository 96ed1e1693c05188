// Internal declarations of the fit / pair-error stages.
#pragma once

#include "isdf_select.h"

#include <functional>

namespace isdf {

struct AnchorFactor {
    int64_t k = 0;
    DeviceBuffer<double> phi_a, phi_aT;   // k x nao, nao x k
    DeviceBuffer<double> M;               // (Phi_a Phi_a^T)^2, k x k
    DeviceBuffer<double> T;               // pseudo-inverse of M (SVD cutoff 1e-12 on C)
    DeviceBuffer<double> wa;              // anchor weights
    DeviceBuffer<double> anchor_pts;      // anchor coordinates, k x 3
    std::vector<double> sv;               // singular values of C^T, descending
    int retained = 0;
    double condition = 0;
    bool gram_fallback = false;           // singular values from M (well-separated from the cutoff, or C^T too large)
};

struct FitOutput {
    int64_t n = 0;
    double err2 = 0, exact2 = 0, max_abs_coeff = 0;
    std::vector<double> theta_w;          // sum_g Theta[a, g] w_g
    double mixed_bound = 0;               // bound on the refined mixed fit's relative pair-error excess over FP64
    int path = 0;                         // 0 FP64, 1 mixed, 3 mixed + FP64 refinement, 2 bound too loose -> FP64
};

// Largest relative pair-error excess over the FP64 fit that the refined mixed
// fit accepts (the 1e-8 target); beyond it the fit is redone with FP64 AO values.
constexpr double kMixedFitTolerance = 1e-8;

AnchorFactor factor_anchors(const Context& c, const double* anchor_pts, const double* anchor_w,
                            int64_t k, cudaStream_t s);

// Grid pass over the kept points: writes Theta[a*ldt + g] (unless have_theta,
// in which case Theta is read) and accumulates the pair-space error terms.
FitOutput fit_grid(const Context& c, const double* pts, const double* w, const KeptPoints& kp,
                   const AnchorFactor& f, double* theta, int64_t ldt, bool have_theta,
                   cudaStream_t s);

// Mixed precision: G from the fused FP32-AO / split-BF16 tensor-core projection,
// then h, X0 = T h and Theta0 in FP64 (path 1) with an a-posteriori bound on
// its relative pair-error excess over the FP64 fit; when that bound exceeds
// the tolerance, one FP64 iterative-refinement step over the stored AO tiles
// follows (path 3), whose (hi, lo, remainder) BF16 terms add up to the FP32
// values exactly: G in FP64 against FP64 anchor values, X1 = X0 + T (h - M X0),
// and mixed_bound then bounds the refined Theta's excess.  The pair-space error is not
// evaluated here (see fit_grid with have_theta).  With `ao_tiles` (the AO
// value tiles a mixed sketch of the same kept points left in HBM) and their
// per-point sums of squares `ao_psq`, G comes from a GEMM over the tiles
// instead of a new projection (which otherwise stores the tiles itself); then,
// with `on_chunk`, the points are fitted in a few chunks and on_chunk(g0, m) is
// called after the launches that write Theta's columns [g0, g0 + m) on s (a
// caller can start copying those columns out while the next chunk runs).
bool fit_mixed_supported(int64_t k);
using FitChunkHook = std::function<void(int64_t g0, int64_t m)>;
FitOutput fit_grid_mixed(const Context& c, const double* pts, const double* w, const KeptPoints& kp,
                         const AnchorFactor& f, double* theta, int64_t ldt, cudaStream_t s,
                         const uint8_t* ao_tiles = nullptr, const uint8_t* ao_tiles_r = nullptr,
                         const float* ao_psq = nullptr, const FitChunkHook* on_chunk = nullptr,
                         const uint8_t* ao_chunk_zero = nullptr);

void gather_points(const double* pts, const double* w, const int64_t* idx, int64_t n,
                   int64_t npts_total, double* out_pts, double* out_w, cudaStream_t s);

// Pair-space error reduction from precomputed Gram terms (device pointers):
// out2 = {sum |w| (q^2 - 2 x.h + x^T M x), sum |w| q^2}.
void pair_error_terms(int64_t n, int64_t k, const double* q, const double* H, const double* X,
                      const double* M, const double* w, double* out2, cudaStream_t s);

}  // namespace isdf
