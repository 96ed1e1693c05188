/*
 * C-ABI of the B200 ISDF hot-path library (libisdf_b200.so).
 *
 * Every entry point returns an int status (0 = ok, see isdf_status); no C++
 * exception crosses the boundary.  isdf_last_error() returns the message of
 * the calling thread's last failure.  Arrays are plain pointers with explicit
 * sizes; "dev" pointers are CUDA device pointers, "host" pointers are host
 * memory.  `stream` is a cudaStream_t passed as void* (NULL = legacy default
 * stream).  A context belongs to the device that was current when it was
 * created; calls on distinct streams with distinct outputs may run
 * concurrently.
 *
 * Each declaration names the interface of mikovtun/mp_isdf it replaces
 * (file:line within that project).
 */
#ifndef ISDF_B200_H
#define ISDF_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct isdf_ctx isdf_ctx;

enum isdf_status {
    ISDF_OK = 0,
    ISDF_ERR_INVALID = 1,         /* std::invalid_argument -> ValueError */
    ISDF_ERR_OVERFLOW = 2,        /* std::overflow_error */
    ISDF_ERR_RUNTIME = 3,         /* std::runtime_error */
    ISDF_ERR_CUDA = 4,            /* CUDA runtime failure */
    ISDF_ERR_NOT_IMPLEMENTED = 5, /* NotImplementedError */
    ISDF_ERR_LOGIC = 6            /* std::logic_error */
};

/* AxisType codes (cpp/include/enums.hpp:8-14). */
enum isdf_axis { ISDF_AXIS_AO = 0, ISDF_AXIS_DX = 1, ISDF_AXIS_DY = 2, ISDF_AXIS_DZ = 3, ISDF_AXIS_OCC = 4 };

/* LocalAnchorSelectionAlgorithm codes (cpp/include/enums.hpp:23-30). */
enum isdf_algorithm {
    ISDF_QRCP_DENSE = 0,             /* QRColumnPivoting */
    ISDF_QRCP_ONLINE = 1,            /* OnlineQRColumnPivoting */
    ISDF_RAND_SKETCH_QUADRATURE = 2, /* RandomizedQuadratureKhatriRao */
    ISDF_CVT = 3,                    /* CentroidalVoronoi (not on this path) */
    ISDF_RAND_SKETCH_DENSITY = 4,    /* RandomizedAODensityKhatriRao (FP64 form) */
    ISDF_RAND_SKETCH_DENSITY_NORM = 5 /* RandomizedAODensityNormalizedKhatriRao (FP64 form) */
};

enum isdf_precision { ISDF_FP64 = 0, ISDF_MIXED = 1 };

/* Human-readable name of a status code. */
const char* isdf_status_string(int status);
/* Message of the calling thread's last failure ("" if none). */
const char* isdf_last_error(void);
/* 1 when a CUDA device is usable, else 0 (never fails). */
int isdf_cuda_available(void);

/* ---- context --------------------------------------------------------------
 * Replaces LibcintContext(atm, bas, env) (cpp/src/ao_eval.cpp:78-158,
 * cpp/src/ao_eval_pybind.cpp:33-46): copies the libcint ATM[natm,6],
 * BAS[nbas,8] int32 tables and ENV[nenv] and uploads the shell table to the
 * current device. */
int isdf_ctx_create(const int32_t* atm_host, int32_t natm, const int32_t* bas_host, int32_t nbas,
                    const double* env_host, int64_t nenv, isdf_ctx** out);
int isdf_ctx_destroy(isdf_ctx* ctx);
/* LibcintContext.nao (cpp/src/ao_eval_pybind.cpp:91) and atom count. */
int isdf_ctx_info(const isdf_ctx* ctx, int64_t* nao, int32_t* natm, int32_t* nshell);
/* Atom owning each AO (nao int32), for nuclear derivatives. */
int isdf_ctx_ao_atoms(const isdf_ctx* ctx, int32_t* out_host);

/* ---- AO evaluation --------------------------------------------------------
 * Replaces LibcintContext::eval_ao / eval_ao_gradient (cpp/src/ao_eval.cpp:164-310).
 * xyz_dev[ng,3] bohr.  values_dev (ng x nao, row-major) and/or
 * grad_dev (3 x ng x nao, component-major) may be NULL when not wanted.
 * dtype: 0 = float64, 1 = float32 outputs. */
int isdf_eval_ao(isdf_ctx* ctx, const double* xyz_dev, int64_t ng, int32_t dtype,
                 void* values_dev, void* grad_dev, void* stream);
/* Host-buffer form of the same call (copies in, evaluates, copies out). */
int isdf_eval_ao_host(isdf_ctx* ctx, const double* xyz_host, int64_t ng, double* values_host,
                      double* grad_host);

/* ---- axis features ----------------------------------------------------------
 * Replaces AnchorSelection::evaluate_axis (cpp/include/anchor_select_impl.hpp:11-81,
 * cpp/src/anchor_select_pybind.cpp:211-222): concatenated unscaled axis
 * blocks, out (ng x naxes*nao) row-major. */
int isdf_evaluate_axis(isdf_ctx* ctx, const double* xyz_dev, int64_t ng, const int32_t* axes_host,
                       int32_t naxes, double* out_dev, void* stream);
int isdf_evaluate_axis_host(isdf_ctx* ctx, const double* xyz_host, int64_t ng,
                            const int32_t* axes_host, int32_t naxes, double* out_host);
/* The same with OccupiedOrbital entries allowed (anchor_select.cpp:18-52,
 * anchor_select_impl.hpp:69-72): their block is psi_j = sum_mu phi_mu C[mu][j],
 * j < nocc, with mo_coeff_host row-major nao x nao and 1 <= nocc <= nao; the
 * output has ng x (sum of the entries' widths) features (nao per AO/gradient
 * entry, nocc per occupied entry).  out_dev / out_host as above. */
int isdf_evaluate_axis_mo(isdf_ctx* ctx, const double* xyz_dev, int64_t ng, const int32_t* axes_host,
                          int32_t naxes, const double* mo_coeff_host, int64_t nocc, double* out_dev,
                          void* stream);
int isdf_evaluate_axis_mo_host(isdf_ctx* ctx, const double* xyz_host, int64_t ng, const int32_t* axes_host,
                               int32_t naxes, const double* mo_coeff_host, int64_t nocc, double* out_host);

/* ---- anchor selection ------------------------------------------------------
 * Replaces AnchorSelection::select (cpp/src/anchor_select.cpp:79-173,
 * cpp/src/anchor_select_pybind.cpp:162-210) for QRColumnPivoting,
 * OnlineQRColumnPivoting and RandomizedQuadratureKhatriRao.  Pivots are
 * original grid indices in pivot order. */
typedef struct isdf_select_args {
    int32_t algorithm;           /* enum isdf_algorithm */
    int32_t naxes;
    const int32_t* axes;         /* host, naxes AxisType codes */
    const double* axis_weights;  /* host, naxes factors, or NULL */
    double tolerance;            /* default 1e-10 */
    int64_t max_rank;            /* 0 = tolerance only */
    int64_t batch_size;          /* default 128 (validated; results are batch invariant) */
    int64_t sketch_size;         /* default 128 */
    int64_t oversampling;        /* default 16 */
    uint64_t seed;               /* default 7 */
    int32_t precision;           /* enum isdf_precision (rand_sketch only) */
    int32_t debug;               /* print a summary line on stderr */
    /* density sketches (ISDF_RAND_SKETCH_DENSITY[_NORM], FP64 form, axes = {AO}):
     * ngrid finite nonnegative importances m_g (device memory for isdf_select /
     * isdf_select_fit, host memory for the _host variants); points with m_g = 0
     * or squared AO norm <= ao_screening_threshold are not candidates
     * (cpp/src/anchor_select_randomized_id.cpp:104-115, 231-260). */
    const double* point_importance;
    double ao_screening_threshold;   /* default 1e-24 */
    /* OccupiedOrbital axis: row-major nao x nao MO coefficients in host memory
     * and the occupied count (cpp/src/anchor_select.cpp:43-49).  The FP64 forms
     * evaluate it; a mixed rand_sketch with an occupied entry runs in FP64. */
    const double* mo_coeff;
    int64_t nocc;
} isdf_select_args;

typedef struct isdf_select_info {
    int64_t n_kept;              /* nonzero-weight points */
    int64_t sketch_rows;         /* rand_sketch: ell */
    int64_t numerical_rank;      /* rand_sketch */
    int64_t verifications;       /* exact recomputations (pair QR: winners; mixed sketch: candidates) */
    int64_t reselections;
    double relative_residual;    /* sketch tail / pair-QR last |R_jj| / |R_00| */
    int64_t precision_used;      /* form that ran: 0 FP64, 1 mixed.  A mixed request runs the
                                  * FP64 form (and reports 0 here) for the pair-QR algorithms,
                                  * the density sketches, an OccupiedOrbital axis, more AOs than
                                  * the FP64 re-verification holds, or projections wider than
                                  * the tensor-core kernel's accumulators */
} isdf_select_info;

void isdf_select_args_default(isdf_select_args* args);
/* pivots_host must hold at least `capacity` entries; *npivots receives the count. */
int isdf_select(isdf_ctx* ctx, const isdf_select_args* args, const double* xyz_dev,
                const double* w_dev, int64_t ng, int64_t* pivots_host, int64_t capacity,
                int64_t* npivots, isdf_select_info* info, void* stream);
int isdf_select_host(isdf_ctx* ctx, const isdf_select_args* args, const double* xyz_host,
                     const double* w_host, int64_t ng, int64_t* pivots_host, int64_t capacity,
                     int64_t* npivots, isdf_select_info* info);

/* ---- interpolation-vector fit + pair-space error ---------------------------
 * Replaces _physical_pair_refit and the pair-space error functions
 * (python/isdf.py:238-263, 154-191).  anchors_host: k original grid indices.
 * theta_dev receives Theta (k x n_kept, row-major, leading dimension n_kept);
 * it must hold k*ng doubles.  want_error != 0 also evaluates the pair-space
 * error with FP64 AO values. */
typedef struct isdf_fit_info {
    int64_t n_kept;
    int64_t retained_rank;
    double condition;
    double max_abs_physical_coefficient;
    double pair_l2;              /* sqrt(sum |w| |p - rec|^2) */
    double pair_relative;
    double theta_w[64];          /* sum_g Theta[a,g] w_g (first 64 anchors) */
    int64_t fit_path;            /* 0 FP64; 1 mixed (tensor-core Gram); 3 mixed followed by one
                                  * FP64 iterative-refinement step of Theta over the stored AO
                                  * tiles (taken when the bound of path 1 exceeds 1e-8);
                                  * 2 mixed requested, refined bound above 1e-8 -> FP64 AO values */
    double mixed_bound;          /* a-posteriori bound on the accepted mixed Theta's relative
                                  * pair-error excess over the FP64 fit */
} isdf_fit_info;

int isdf_fit(isdf_ctx* ctx, const double* xyz_dev, const double* w_dev, int64_t ng,
             const int64_t* anchors_host, int64_t k, int32_t precision, int32_t want_error,
             double* theta_dev, isdf_fit_info* info, void* stream);
int isdf_fit_host(isdf_ctx* ctx, const double* xyz_host, const double* w_host, int64_t ng,
                  const int64_t* anchors_host, int64_t k, int32_t precision, int32_t want_error,
                  double* theta_host, isdf_fit_info* info);
/* Anchor selection followed by the fit on the same points in one call: the
 * path of build_isdf from selector.select to _physical_pair_refit
 * (python/isdf.py:591-652).  Same results as isdf_select then isdf_fit with
 * args->precision; in the mixed rand_sketch form the split-BF16 AO value
 * tiles of the sketch pass stay in HBM and the fit contracts them instead of
 * evaluating the AOs again (the reference likewise evaluates Phi once and
 * hands it to the fit).  A mixed request whose selection kept no AO tiles
 * (pair-QR algorithms, no plain AO value axis) fits in FP64 below 2^28 AO
 * values (ng * nao), where that is the cheaper fit (fit_info->fit_path 0).
 * theta_dev needs capacity k * ng (k <= capacity). */
int isdf_select_fit(isdf_ctx* ctx, const isdf_select_args* args, const double* xyz_dev,
                    const double* w_dev, int64_t ng, int64_t* pivots_host, int64_t capacity,
                    int64_t* npivots, isdf_select_info* select_info, int32_t want_error,
                    double* theta_dev, isdf_fit_info* fit_info, void* stream);
/* Host-buffer twin; theta_host needs capacity npivots * ng. */
int isdf_select_fit_host(isdf_ctx* ctx, const isdf_select_args* args, const double* xyz_host,
                         const double* w_host, int64_t ng, int64_t* pivots_host, int64_t capacity,
                         int64_t* npivots, isdf_select_info* select_info, int32_t want_error,
                         double* theta_host, isdf_fit_info* fit_info);
/* ---- grid-sharded rand_sketch (one rank per GPU) ---------------------------------
 * The distributed form of AnchorSelection::select + the fit for
 * RandomizedQuadratureKhatriRao (cpp/src/anchor_select_randomized_id.cpp:92-374;
 * the reference's DistributedAnchorSelection is a stub that throws,
 * cpp/src/anchor_select.cpp:175-181, cpp/src/anchor_select_pybind.cpp:224-240).  Every rank holds a contiguous
 * shard of the grid, in grid order; the caller supplies the collectives:
 *  1. isdf_sketch_shard_project: compaction and projection of this shard;
 *     returns its per-component sums of squares (sum them over ranks);
 *  2. isdf_sketch_shard_combine: this shard's sketch columns yt[ell][n_kept]
 *     with the global axis scales, their error bounds (mixed form), kept grid
 *     indices, coordinates and weights (gather all of them over ranks);
 *  3. isdf_sketch_select_gathered (every rank, same gathered inputs):
 *     pivoted QR of the gathered sketch + rank logic; pivots are positions in
 *     the gathered kept-point order;
 *  4. isdf_fit_at on each shard with the anchors' coordinates and weights;
 *     sums_host = {err2, exact2} of the shard (sum over ranks).
 * The result equals the single-GPU selection on the concatenated grid. */
typedef struct isdf_sketch_shard isdf_sketch_shard;
int isdf_sketch_shard_project(isdf_ctx* ctx, const isdf_select_args* args, const double* xyz_dev,
                              const double* w_dev, int64_t ng, int64_t ng_total, isdf_sketch_shard** out,
                              int64_t* n_kept, int64_t* ell, double* sumsq_host, void* stream);
/* yt_dev: ell x n_kept (leading dimension n_kept); delta_dev: n_kept (mixed
 * form; zeros in the FP64 form; may be null there); kept_dev: n_kept grid
 * indices within the shard; kept_xyz_dev/kept_w_dev: n_kept x 3 / n_kept;
 * scales_host: one per axis entry.  The shard's grid must still be valid. */
int isdf_sketch_shard_combine(isdf_sketch_shard* shard, const double* sumsq_global_host, double* yt_dev,
                              double* delta_dev, int64_t* kept_dev, double* kept_xyz_dev,
                              double* kept_w_dev, double* scales_host, void* stream);
void isdf_sketch_shard_free(isdf_sketch_shard* shard);
/* Distributed pivoted QR of the sketch: each rank keeps its own columns
 * (yt_dev: ell x n_local from isdf_sketch_shard_combine) and the ranks
 * exchange only per-step keys and the winning column (instead of gathering
 * the whole sketch).  pos_offset: the number of kept points on lower ranks
 * (global positions of this rank's columns start there); n_total: all
 * ranks' kept points.  Per step j = 0 .. ell-1, on every rank:
 *  a. isdf_qr_shard_update(j): applies reflector j-1; returns this rank's
 *     share of row j-1's energy and either its best key (value = squared
 *     trailing norm, global position, local column; value -1: none) or, in
 *     the mixed form (verified = 1), its best lower bound;
 *  b. mixed form only: the global maximum of the bounds, then
 *     isdf_qr_shard_verify(j, bound) returns the key (candidates recomputed
 *     exactly in FP64);
 *  c. the global best key (largest value, ties to the smaller position); its
 *     owner reads the column (isdf_qr_shard_column, ell rows) for all ranks;
 *  d. isdf_qr_shard_pivot(j, rows, ...) with pivot_col / moved_col the local
 *     pivot column and the local column at position j (-1 on other ranks);
 *     returns R_jj.
 * A final isdf_qr_shard_update(ell) returns the last row's energy shares.
 * isdf_sketch_rank applies the tail / numerical-rank / exact-rank rules
 * (cpp/src/anchor_select_randomized_id.cpp:320-374) to the per-step |R_jj|
 * and row energies (summed over ranks, plus R_jj^2).  Same pivots as
 * isdf_sketch_select_gathered. */
typedef struct isdf_qr_shard isdf_qr_shard;
int isdf_qr_shard_create(isdf_ctx* ctx, const isdf_select_args* args, double* yt_dev, int64_t n_local,
                         int64_t n_total, int64_t pos_offset, const double* kept_xyz_dev, const double* kept_w_dev,
                         double* delta_dev, const double* scales_host, isdf_qr_shard** out, int64_t* ell,
                         int32_t* verified, void* stream);
int isdf_qr_shard_update(isdf_qr_shard* h, int64_t j, double* key_value, int64_t* key_pos, int64_t* key_col,
                         double* energy_part, double* lower_bound);
int isdf_qr_shard_verify(isdf_qr_shard* h, int64_t j, double lower_bound, double* key_value, int64_t* key_pos,
                         int64_t* key_col);
int isdf_qr_shard_column(isdf_qr_shard* h, int64_t col, double* rows_host);
int isdf_qr_shard_pivot(isdf_qr_shard* h, int64_t j, const double* rows_host, int64_t pivot_col, int64_t pivot_pos,
                        int64_t moved_col, double* r_jj);
int isdf_qr_shard_reverified(isdf_qr_shard* h, int64_t* count);
void isdf_qr_shard_free(isdf_qr_shard* h);
/* The pair-space QR of qrcp_dense / qrcp_online (cpp/src/anchor_select_qrcp.cpp:95-225,
 * cpp/src/anchor_select_online_qr.cpp:176-375) over grid shards, one rank per
 * GPU: a rank holds the features and residual estimates of its kept points,
 * the explicit pair basis is replicated.  create: compaction and features of
 * the shard (n_kept, d, the 5 per-component sums of squares for the
 * multi-axis scales); init: global sums -> scales, estimates, positions from
 * pos_offset (the global kept position of the shard's first kept point),
 * out2 = (sum of K_gg, non-finite flag) to be summed over ranks.  Per pivot:
 * argmax gives the shard's best (estimate, position, global kept index; -1
 * when none); the owner exports the winner's row (d features, sqrt|w|, grid
 * index, x, y, z, w: d + 6 doubles), every rank verifies it (exact CGS2 in a
 * fixed reduction order: the same exact2 everywhere) and accepts it; scan
 * recomputes the shard's uncertain columns exactly before a stop.  Driven by
 * mp_isdf_b200.sharded.select_pair_qr_sharded; same anchors as isdf_select. */
typedef struct isdf_pairqr_shard isdf_pairqr_shard;
int isdf_pairqr_shard_create(isdf_ctx* ctx, const isdf_select_args* args, const double* xyz_dev,
                             const double* w_dev, int64_t ng, int64_t grid_offset, isdf_pairqr_shard** out,
                             int64_t* n_kept, int64_t* features, double* sumsq_host, void* stream);
int isdf_pairqr_shard_init(isdf_pairqr_shard* h, const double* sumsq_global, int64_t pos_offset, double* out2);
int isdf_pairqr_shard_argmax(isdf_pairqr_shard* h, double* key3);
int isdf_pairqr_shard_row(isdf_pairqr_shard* h, int64_t col, double* row_host);
int isdf_pairqr_shard_verify(isdf_pairqr_shard* h, const double* row_host, int64_t j, int64_t col,
                             double* exact2);
int isdf_pairqr_shard_accept(isdf_pairqr_shard* h, const double* row_host, int64_t j, int64_t col, double exact2,
                             int64_t winner_pos, int32_t dense);
int isdf_pairqr_shard_scan(isdf_pairqr_shard* h, int64_t j, double thr2, int64_t* count);
void isdf_pairqr_shard_free(isdf_pairqr_shard* h);
int isdf_sketch_rank(isdf_ctx* ctx, const isdf_select_args* args, int64_t n_total, const double* diag_host,
                     const double* energy_host, int64_t steps, int64_t* rank, int64_t* numerical_rank,
                     double* relative_tail);
int isdf_sketch_select_gathered(isdf_ctx* ctx, const isdf_select_args* args, double* yt_dev, int64_t n,
                                const double* kept_xyz_dev, const double* kept_w_dev, double* delta_dev,
                                const double* scales_host, int64_t* pivots_host, int64_t capacity,
                                int64_t* npivots, isdf_select_info* info, void* stream);
/* isdf_fit with anchors given by host coordinates (k x 3) and weights. */
int isdf_fit_at(isdf_ctx* ctx, const double* xyz_dev, const double* w_dev, int64_t ng,
                const double* anchor_xyz_host, const double* anchor_w_host, int64_t k, int32_t precision,
                int32_t want_error, double* theta_dev, isdf_fit_info* info, double* sums_host, void* stream);

/* Pair-space error of a given Theta (k x n_kept, leading dimension n_kept),
 * recomputed with FP64 AO values. */
int isdf_pair_error(isdf_ctx* ctx, const double* xyz_dev, const double* w_dev, int64_t ng,
                    const int64_t* anchors_host, int64_t k, const double* theta_dev,
                    double* l2, double* relative, void* stream);
/* Pair-space error reduction from Gram terms (device arrays): q[n] = |p_g|,
 * H[n,k] = C p_g, X[n,k] = Theta_g * w_anchor, M[k,k] = C C^T, w[n].
 * out_host = {l2, relative}.  Same reduction as isdf_fit's error
 * (python/isdf.py:154-173). */
int isdf_pair_error_terms(int64_t n, int64_t k, const double* q_dev, const double* H_dev,
                          const double* X_dev, const double* M_dev, const double* w_dev,
                          double* out_host, void* stream);

/* Same reduction as isdf_pair_error_terms, for callers that cannot allocate
 * device memory on the call path (a fixed device-memory budget, their own
 * pool or arena, no cudaFree synchronisation allowed).  No counterpart in the
 * reference.  It allocates nothing: its scratch is a fixed 16 KB device array
 * inside the library that every GPU loading the library keeps until exit.
 * Limits: k <= 64 anchors (larger k returns ISDF_ERR_INVALID); any n.  All
 * calls share that array, so calls whose GPU work overlaps race; serialise
 * them.  The first call on a device looks up the array's address once for
 * that device; make it before any stream capture.  The address is kept until
 * exit, so the entry point must not be used on a device after
 * cudaDeviceReset.  Each call waits for its stream before returning (the two
 * sums are copied to out_host).  Null q/w (n > 0) or H/X/M (n > 0, k > 0)
 * return ISDF_ERR_INVALID before any launch. */
int isdf_pair_error_terms_noalloc(int64_t n, int64_t k, const double* q_dev, const double* H_dev,
                                  const double* X_dev, const double* M_dev, const double* w_dev,
                                  double* out_host, void* stream);

/* ---- nuclear-gradient adjoint (no counterpart in the reference, which has no
 * nuclear derivatives: python/isdf.py:7-8) ------------------------------------
 * E = sum_g w_g rho_ISDF(g)^2, rho_ISDF(g) = sum_k Theta_kg w_k rho_a(k),
 * rho_a(k) = phi(a_k)^T D phi(a_k), with grid, anchors (original grid
 * indices) and weights held fixed; grad_host receives dE/dR (natm x 3, bohr).
 * dm_host: AO density matrix (nao x nao, row-major).  AO values/gradients are
 * recomputed per grid chunk (FP64).  grad_host = NULL computes the energy
 * alone (AO values only; no gradient sweep). */
int isdf_energy_gradient(isdf_ctx* ctx, const double* xyz_dev, const double* w_dev, int64_t ng,
                         const int64_t* anchors_host, int64_t k, const double* dm_host,
                         double* energy, double* grad_host, void* stream);
/* The adjoint over grid shards (one rank per GPU, the grid split into
 * contiguous shards): isdf_energy_gradient_shard returns a rank's partial sums
 * over its own points for anchors given by coordinates (k x 3, bohr) and
 * weights (isdf_adjoint_partial_size doubles: [E, v (k), per-atom grid terms
 * (natm x 3), alpha^T Phi_g (k x nao), per-AO grid terms (3 x nao)]); after the
 * element-wise sum of the partials over ranks (one all-reduce),
 * isdf_energy_gradient_finish gives E and dE/dR, the same on every rank and
 * equal to isdf_energy_gradient over the whole grid.  want_grad = 0 / grad_host
 * = NULL: the energy alone. */
int isdf_adjoint_partial_size(isdf_ctx* ctx, int64_t k, int64_t* size);
int isdf_energy_gradient_shard(isdf_ctx* ctx, const double* xyz_dev, const double* w_dev, int64_t ng,
                               const double* anchor_xyz_host, const double* anchor_w_host, int64_t k,
                               const double* dm_host, int32_t want_grad, double* partial_host, void* stream);
int isdf_energy_gradient_finish(isdf_ctx* ctx, const double* anchor_xyz_host, const double* anchor_w_host,
                                int64_t k, const double* dm_host, const double* sums_host, double* energy,
                                double* grad_host, void* stream);
/* Moves the atoms of a context (natm x 3, bohr; the basis functions follow). */
int isdf_ctx_set_coords(isdf_ctx* ctx, const double* coords_host);

/* ---- axis-feature projection -------------------------------------------------
 * The contraction at the core of the Khatri-Rao sketch
 * (cpp/src/anchor_select_randomized_id.cpp:299-309, the f_g . u_s and
 * f_g . v_s sums) and of the fit Gram (python/isdf.py:251-256), exposed on
 * its own: out[g][a][j] = sum_mu comp_a(g, mu) * W[a*nao + mu][j] for the
 * unscaled axis blocks, W_host row-major [naxes*nao][nout].  precision
 * ISDF_FP64: FP64 AO values and FP64 products; ISDF_MIXED: FP32 AO values
 * evaluated in shared memory and split-BF16 tensor-core products (requires
 * naxes <= 4, nout <= 64).  out_dev: ng x naxes x nout float64. */
int isdf_project_axes(isdf_ctx* ctx, const double* xyz_dev, int64_t ng, const int32_t* axes_host,
                      int32_t naxes, const double* W_host, int32_t nout, int32_t precision,
                      double* out_dev, void* stream);

/* Spherical-cell grid Coulomb metric between two sets of interpolation
 * vectors (grid_cross_metric, python/isdf.py:80-97; with left = right and
 * symmetrize = 1 it is grid_coulomb_metric, :48-68):
 *   V[a][b] = sum_{g,h} left[a][g] w_g K_gh w_h right[b][h],
 *   K_gh = 1/|r_g - r_h| (g != h; 0 for coincident points),
 *   K_gg = (32/15) pi^2 (3/(4 pi))^(5/3) |w_g|^(-1/3).
 * left: kl x n, right: kr x n (row-major, leading dimensions ldl, ldr >= n,
 * not weight-scaled), xyz: n x 3, w: n; kr <= 64.  metric_host: kl x kr,
 * (V + V^T)/2 when symmetrize (requires kl = kr).  FP64 throughout.  When
 * symmetrize is set and left and right are the same pointer (and leading
 * dimension), the symmetry of K is used: half the pairs are summed.  The
 * device variant takes device pointers and a stream; the _host variant host
 * buffers (ctx may be NULL there: the current device). */
int isdf_grid_metric(isdf_ctx* ctx, const double* left_dev, int64_t ldl, int64_t kl, const double* right_dev,
                     int64_t ldr, int64_t kr, const double* xyz_dev, const double* w_dev, int64_t n,
                     int32_t symmetrize, double* metric_host, void* stream);
int isdf_grid_metric_host(isdf_ctx* ctx, const double* left_host, int64_t kl, const double* right_host,
                          int64_t kr, const double* xyz_host, const double* w_host, int64_t n,
                          int32_t symmetrize, double* metric_host);

/* ---- ISDF Coulomb and exchange matrices --------------------------------------
 * Replaces evaluate_isdf_jk (python/isdf.py:130-151):
 *   (mu nu|lam sig) ~ sum_pq X[p,mu] X[p,nu] Z[p,q] X[q,lam] X[q,sig],
 *   J = X^T diag(Z diag(X D X^T)) X,  K = X^T (Z o (X D X^T)) X,
 * both symmetrised, (A + A^T)/2.  x: k x nao anchor AO values, z: k x k
 * metric (already carrying both anchors' quadrature weights), dm: nao x nao
 * (symmetric; validated by the caller), j / k_out: nao x nao, either may be
 * NULL.  FP64 tensor-core GEMMs.  The device variant takes device pointers
 * and a stream; the _host variant host buffers. */
int isdf_jk(isdf_ctx* ctx, const double* x_dev, int64_t k, const double* z_dev, const double* dm_dev,
            double* j_dev, double* k_out_dev, void* stream);
int isdf_jk_host(isdf_ctx* ctx, const double* x_host, int64_t k, const double* z_host, const double* dm_host,
                 double* j_host, double* k_out_host);

/* ---- RBRP (robust blockwise random pivoting) ---------------------------------
 * Replaces rbrp_ao_cpu / rbrp_ao_device (cpp/src/anchor_select_rbrp.cpp:195-320,
 * cpp/src/anchor_select_rbrp_device.cpp, cpp/src/anchor_select_pybind.cpp:68-140):
 * AO-only pivoting over the weighted AO pair rows of the grid points, with the
 * optional interpolative decomposition (interp_vecs rank x n, transform
 * rank x nao*nao).  The AO rows live on the GPU; sampling uses the reference's
 * std::discrete_distribution over std::mt19937_64(seed). */
typedef struct isdf_rbrp_args {
    int64_t batch_size;      /* default 128 (validated; results do not depend on it) */
    int64_t block_size;      /* default 16 */
    double tolerance;        /* default 1e-10 */
    int64_t max_rank;        /* 0 = min(n, pairs) */
    uint64_t seed;           /* default 7 */
    double tau_block;        /* NaN (default) = 1 / block_size */
    double rank_rtol;        /* default 1e-12 */
    int64_t refresh_every;   /* default 8 */
    double svd_rtol;         /* default 1e-12 */
    int32_t compute_id;      /* default 0 */
} isdf_rbrp_args;
void isdf_rbrp_args_default(isdf_rbrp_args* args);
typedef struct isdf_rbrp_result isdf_rbrp_result;
/* ao_host: n x nao row-major AO values, w_host: n nonzero weights (ctx may be NULL). */
int isdf_rbrp_ao(isdf_ctx* ctx, const double* ao_host, const double* w_host, int64_t n, int64_t nao,
                 const isdf_rbrp_args* args, isdf_rbrp_result** out);
/* xyz_host: n x 3 points (AOs evaluated on the device), w_host: n nonzero weights. */
int isdf_rbrp_points(isdf_ctx* ctx, const double* xyz_host, const double* w_host, int64_t n,
                     const isdf_rbrp_args* args, isdf_rbrp_result** out);
/* status: NUL-terminated, at most status_capacity bytes. */
int isdf_rbrp_result_info(const isdf_rbrp_result* r, int64_t* rank, int64_t* nblocks, int64_t* n, int64_t* nao,
                          double* relative_residual, double* condition, int64_t* retained_rank, char* status,
                          int64_t status_capacity);
/* indices: rank; history: nblocks x 4; interp_vecs: rank x n; transform: rank x nao*nao
 * (the last two only with compute_id; any pointer may be NULL). */
int isdf_rbrp_result_copy(const isdf_rbrp_result* r, int64_t* indices, double* history, double* interp_vecs,
                          double* transform);
void isdf_rbrp_result_free(isdf_rbrp_result* r);

/* Gaussian sketch factors of rand_sketch: U, V (d x ell, row-major u[a*ell+s])
 * from std::mt19937_64(seed) and std::mt19937_64(seed ^ 0x9e3779b97f4a7c15)
 * through std::normal_distribution<double>
 * (cpp/src/anchor_select_randomized_id.cpp:269-279).  Host only, no device
 * work; u_host and v_host hold d*ell doubles each. */
int isdf_sketch_factors(int64_t d, int64_t ell, uint64_t seed, double* u_host, double* v_host);

/* ---- profiling ---------------------------------------------------------------
 * No counterpart in the reference beyond its per-stage wall times
 * (python/isdf.py:384-396): CUDA-event timing per kernel family, off by
 * default.  isdf_profile_read synchronises the recorded events, returns up to
 * `max` families sorted by total time (names: 48 bytes each) and clears the
 * record. */
/* Number of kernels this library has launched in the process so far (all
 * devices); differences around a call count its launches. */
int64_t isdf_launch_count(void);
int isdf_profile_enable(int32_t on);
int isdf_profile_read(int32_t max, char* names, double* total_ms, int64_t* launches, int32_t* count);

#ifdef __cplusplus
}
#endif

#endif /* ISDF_B200_H */
