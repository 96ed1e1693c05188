// AO-only robust blockwise random pivoting and its ID (cpp/src/anchor_select_rbrp.cpp).
#pragma once

#include "isdf_internal.h"
#include "isdf_reduce.cuh"

#include <string>
#include <vector>

namespace isdf {

struct RbrpParams {
    int64_t batch_size = 128;   // validated only: the pair rows are never batched in memory here
    int64_t block_size = 16;
    double tolerance = 1e-10;
    int64_t max_rank = 0;
    uint64_t seed = 7;
    double tau_block = std::numeric_limits<double>::quiet_NaN();   // NaN: 1 / block_size
    double rank_rtol = 1e-12;
    int64_t refresh_every = 8;
    double svd_rtol = 1e-12;
    bool compute_id = false;
};

struct RbrpResult {
    std::vector<int64_t> indices;        // into the supplied AO rows
    std::vector<double> interp_vecs;     // rank x n (compute_id)
    std::vector<double> transform;       // rank x nao*nao (compute_id)
    std::vector<double> history;         // per block: rank, candidates, retained, residual
    double relative_residual = 0, condition = 0;
    int64_t retained_rank = 0;
    std::string status;
};

// ao: n x nao row-major, w: n (device memory).
RbrpResult rbrp_ao(const double* ao, const double* w, int64_t n, int nao, const RbrpParams& prm, cudaStream_t s);

}  // namespace isdf
