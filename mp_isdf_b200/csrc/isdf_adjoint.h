// Nuclear gradient of the ISDF density functional (see adjoint.cu).
#pragma once

#include "isdf_fit.h"

namespace isdf {

struct AdjointResult {
    double energy = 0;
    std::vector<double> grad;   // natm x 3, row-major
};

// E = sum_g w_g rho_ISDF(g)^2 and dE/dR over the kept points, for the anchors
// factored in `f` and the AO density matrix `dm_host` (nao x nao, row-major).
// want_grad = false computes E alone (AO values only, no gradient sweep).
AdjointResult energy_gradient(const Context& c, const double* pts, const double* w,
                              const KeptPoints& kp, const AnchorFactor& f, const double* dm_host,
                              bool want_grad, cudaStream_t s);

// The same in two steps, for grid shards: the sums over one set of kept
// points, [E, v (k), per-atom grid terms (natm x 3), B = alpha^T Phi_g
// (k x nao), per-AO grid terms (3 x nao)] (adjoint_partial_size doubles;
// what the fused grid pass folds per atom leaves B and the per-AO terms
// zero), and the energy and gradient from the sums over all shards.
size_t adjoint_partial_size(const Context& c, int64_t k);
std::vector<double> energy_gradient_partial(const Context& c, const double* pts, const double* w,
                                            const KeptPoints& kp, const AnchorFactor& f, const double* dm_host,
                                            bool want_grad, cudaStream_t s);
AdjointResult energy_gradient_finish(const Context& c, const AnchorFactor& f, const double* dm_host,
                                     const double* sums_host, bool want_grad, cudaStream_t s);

// Moves the atoms (and their shells) to new coordinates (natm x 3, bohr).
void set_atom_coords(Context& c, const double* coords_host);

}  // namespace isdf
