// Internal declarations of the anchor-selection stages.
#pragma once

#include "isdf_internal.h"

#include <memory>

namespace isdf {

struct KeptPoints {
    // original indices of the nonzero-weight points: ascending, or, when
    // `rank` is set, ascending between windows of kSpatialWindow positions
    // and in spatial (Morton) order inside each window
    DeviceBuffer<int64_t> index;
    DeviceBuffer<int64_t> rank;   // empty, or the ascending position of each position
    int64_t n = 0;
    bool spatial() const { return rank.get() != nullptr; }
};

// Positions per window of the spatial order (whole 128-point tiles).  A
// window holds the same points in both orders, so position ranges made of
// whole windows can be mapped back to ascending order on their own.
constexpr int64_t kSpatialWindow = 131072;

// Flags non-finite weights (always) and non-finite coordinates of kept points,
// and compacts the nonzero-weight points in their original order.  With an
// importance vector (density sketches) every entry must be finite and
// nonnegative, and points of zero importance are dropped too.  With `spatial`
// the points inside each window of kSpatialWindow positions are then ordered
// by the Morton code of their 1-bohr cell, so that consecutive points (the
// 32-point warps and 128-point tiles of the evaluators) lie close together
// and screen more pieces; `rank` maps positions back to ascending order.
KeptPoints compact_points(const double* pts, const double* w, int64_t n, cudaStream_t s,
                          const double* importance = nullptr, bool spatial = false);

// dst[a*ld + rank[p]] = src[a*ld + p] for the k rows and positions
// [p0, p0 + m), a range of whole windows (dst and src distinct).
void unpermute_columns(const double* src, double* dst, int64_t ld, int64_t k, const int64_t* rank, int64_t p0,
                       int64_t m, cudaStream_t s);

struct SelectOptions {
    int algorithm = 0;               // LocalAnchorSelectionAlgorithm code
    std::vector<int32_t> axes;       // AxisType codes
    std::vector<double> axis_weights;
    double tolerance = 1e-10;
    int64_t max_rank = 0;
    int64_t batch_size = 128;
    int64_t sketch_size = 128;
    int64_t oversampling = 16;
    uint64_t seed = 7;
    int precision = 0;               // 0 FP64, 1 mixed
    bool debug = false;
    const double* importance = nullptr;  // density sketches: per grid point (device)
    double ao_threshold = 1e-24;         // density sketches: squared AO norm screen
    const double* mo_host = nullptr;     // OccupiedOrbital: row-major nao x nao (host)
    int64_t nocc = 0;
};

// Device copy of the MO coefficients of the options (empty without them) and
// the axis spec built with it.
struct AxisSetup {
    DeviceBuffer<double> mo;
    AxisSpec ax;
};
AxisSetup make_axis_setup(const Context& c, const SelectOptions& o, cudaStream_t s);

struct SketchDiagnostics {
    int64_t ell = 0, numerical_rank = 0, cap = 0, rank = 0;
    double relative_tail = 0;
    int64_t reverified = 0;          // mixed path: candidates recomputed in FP64
    int64_t precision_used = 0;      // form that ran: 0 FP64, 1 mixed
    std::vector<double> diag, tails;
};

struct PairQrDiagnostics {
    int64_t rank = 0, verifications = 0, reselections = 0, exact_scans = 0;
    double first = 0, last = 0, floor = 0;
    std::vector<double> rdiag;       // |R_jj| of the selected pivots
    std::vector<double> gap;         // relative gap to the runner-up at each step
};

struct SketchQR {
    std::vector<int64_t> jpvt;       // 0-based pivot columns, per step
    std::vector<double> diag;        // |R_jj|
    std::vector<double> energy;      // sum of squares of row j of R
    int64_t reverified = 0;          // columns recomputed exactly (verified mode)
};

// Everything needed to recompute a sketch column exactly in FP64 (device
// pointers): used by the verified QR of a mixed-precision sketch.
struct ExactSketchSource {
    const Context* ctx = nullptr;
    int naxes = 0;
    int comp[16] = {};
    const double* scales = nullptr;  // naxes
    const double* WT = nullptr;      // (2 ell) x d, row-major
    const double* pts = nullptr;
    const int64_t* index = nullptr;  // kept-point gather
    const double* w = nullptr;
    int64_t ell = 0;
    double* delta = nullptr;         // per-column absolute error bounds (0 = exact)
};

// mo (device, row-major nao x nao) and nocc are needed for the OccupiedOrbital axis.
AxisSpec make_axis_spec(const Context& c, const int32_t* axes, int naxes, const double* mo = nullptr,
                        int64_t nocc = 0);
void validate_axis_weights(const double* axis_weights, int naxes);
std::vector<double> axis_scales_from_sumsq(const AxisSpec& ax, const double* sumsq4,
                                           const double* axis_weights, bool any_eligible);
// Page-locked host memory for vectors that are copied to the device, from a
// process-wide cache of blocks (a block goes back to the cache when its vector
// is freed, so repeated calls pin nothing new); pageable memory if pinning
// fails.  Copies from it are true asynchronous DMA transfers.
void* pinned_host_alloc(size_t bytes);
void pinned_host_free(void* p, size_t bytes) noexcept;
template <class T>
struct PinnedAllocator {
    using value_type = T;
    PinnedAllocator() = default;
    template <class U> PinnedAllocator(const PinnedAllocator<U>&) {}
    T* allocate(size_t n) { return static_cast<T*>(pinned_host_alloc(n * sizeof(T))); }
    void deallocate(T* p, size_t n) noexcept { pinned_host_free(p, n * sizeof(T)); }
    template <class U> bool operator==(const PinnedAllocator<U>&) const { return true; }
    template <class U> bool operator!=(const PinnedAllocator<U>&) const { return false; }
};
// Host copies of the sketch factors (uploaded once per selection).
using HostFactors = std::vector<double, PinnedAllocator<double>>;

// Gaussian sketch factors U, V (d x ell, u[a*ell+s]): std::normal_distribution
// over std::mt19937_64(seed) and std::mt19937_64(seed ^ 0x9e3779b97f4a7c15).
void sketch_factors(int64_t d, int64_t ell, uint64_t seed, double* u, double* v);
void sketch_factors(int64_t d, int64_t ell, uint64_t seed, HostFactors& u, HostFactors& v);

// Full column-pivoted Householder QR of the ell x n sketch stored row-wise
// (Yt[s*ldy + g]); modifies Yt.  With `exact`, columns whose error interval
// reaches the best candidate are recomputed in FP64 before each pivot choice.
SketchQR qrcp_sketch(double* Yt, int64_t ldy, int64_t m, int64_t n, cudaStream_t s,
                     const ExactSketchSource* exact = nullptr);

// One rank's share of the column-pivoted QR of a sketch whose columns are
// split over ranks (the distributed form of qrcp_sketch, same kernels and
// arithmetic).  Per step j the caller runs update(j) on every rank (exact
// mode: returns the rank's best (squared trailing norm, global position,
// local column) key; verified mode: the rank's best lower bound, then, after
// the global maximum of the bounds, verify(j, bound) returns the key), picks
// the global best key (ties to the smaller position), fetches the winner's
// rows from its owner (column) and calls pivot(j, ...) on every rank with the
// same rows.  energy_part is the rank's share of row j-1's energy.  Columns
// carry global positions offset + local index (dgeqp3's swap order).
struct QrShardKey {
    double v;        // squared trailing norm (-1 when the rank has no candidate)
    int64_t pos;     // global position
    int64_t col;     // local column
};
class QrShard {
public:
    QrShard(double* Yt, int64_t ldy, int64_t m, int64_t n, int64_t pos_offset, const ExactSketchSource* exact,
            cudaStream_t s);
    ~QrShard();
    QrShard(const QrShard&) = delete;
    QrShard& operator=(const QrShard&) = delete;
    QrShardKey update(int64_t j, double* energy_part, double* lower_bound);
    QrShardKey verify(int64_t j, double lower_bound);
    void column(int64_t col, double* rows_host);
    // pivot_col / moved_col: this rank's pivot column and the column it holds
    // at position j (-1 when another rank holds them); returns R_jj (signed)
    double pivot(int64_t j, const double* rows_host, int64_t pivot_col, int64_t pivot_pos, int64_t moved_col);
    int64_t reverified() const;

private:
    struct Impl;
    std::unique_ptr<Impl> d_;
};

struct MixedSketch {
    DeviceBuffer<double> scales, WT, delta;
    ExactSketchSource source;
};

// Largest basis the FP64 re-verification of sketch columns holds in shared
// memory (four components of one point, FP64).
constexpr int kMaxVerifiedNao = 6144;

// AO data of a mixed-precision rand_sketch selection kept for the fit that
// follows it on the same points: the split-BF16 AO value tiles of the fused
// projection and the per-point sums of squares, over the kept points.
// The tiles and the projections live in the context's workspace: the caller
// holds ctx.ws_mu from the selection to the end of the fit.
struct RetainedAo {
    KeptPoints kp;
    const uint8_t* tiles = nullptr;  // [tile][K-chunk] (hi, lo) A tiles of the AO values
    const uint8_t* tiles_r = nullptr;  // [tile][K-chunk] remainder tiles (hi + lo + r = FP32 value)
    const uint8_t* chunk_zero = nullptr;  // [tile][K-chunk] 1 where the chunk's tiles are zeros (screened)
    DeviceBuffer<float> psq;       // [n][4] per-point sums of squares (component 0 = values)
    bool valid = false;
};

// Fills Yt with the mixed-precision sketch of the kept points and returns the
// FP64 recomputation source (scales, W^T, error bounds) for the verified QR.
// With `keep`, the AO value tiles and sums of squares stay in `keep` when an
// axis entry is the plain AO value and the tiles fit in free device memory.
MixedSketch sketch_mixed(const Context& c, const double* pts, const KeptPoints& kp, const double* w,
                         const AxisSpec& ax, const double* axis_weights, int64_t ell,
                         const HostFactors& u, const HostFactors& v, double* Yt,
                         int64_t ldy, cudaStream_t s, RetainedAo* keep = nullptr);

std::vector<int64_t> select_rand_sketch(const Context& c, const double* pts, const double* w,
                                        int64_t ng, const SelectOptions& o, cudaStream_t s,
                                        SketchDiagnostics* diag = nullptr, RetainedAo* keep = nullptr);

// Validated sketch parameters for n kept points (cpp/src/anchor_select_randomized_id.cpp:116-191).
struct SketchSetup {
    AxisSpec ax{};
    int64_t d = 0, ell = 0, physical_rank = 0;
    bool mixed = false;              // mixed-precision form applies
    DeviceBuffer<double> mo;         // device MO coefficients (occupied-orbital axis)
};
// n = 0: option checks only; n > 0 also copies the MO coefficients to the device (on s).
SketchSetup sketch_setup(const Context& c, const SelectOptions& o, int64_t n, cudaStream_t s = nullptr);

// Tails, numerical rank, cap and the selected rank of a sketch QR
// (cpp/src/anchor_select_randomized_id.cpp:320-374).
struct SketchRank {
    int64_t rank = 0, numerical_rank = 0, cap = 0;
    double relative_tail = 0;
    std::vector<double> tails;
};
SketchRank sketch_rank(const SketchQR& qr, int64_t ell, int64_t n, const SelectOptions& o,
                       int64_t physical_rank);

// Grid-sharded rand_sketch.  Each rank projects its shard (sketch_shard_project,
// returning per-component sums of squares), the ranks sum those, each rank
// forms its shard's sketch columns with the global axis scales
// (sketch_shard_combine), and every rank runs the pivoted QR of the gathered
// sketch (select_sketch_gathered), which returns positions in the gathered
// kept-point order.
struct SketchShard {
    SelectOptions o;
    SketchSetup su;
    KeptPoints kp;
    HostFactors u, v;
    DeviceBuffer<float> Pf, psq;     // mixed: projections, per-point sums of squares
    DeviceBuffer<double> Pd;         // FP64: projections
    double sumsq[4] = {0, 0, 0, 0};
    const double* pts = nullptr;     // the shard's grid (caller's device arrays)
    const double* w = nullptr;
    int64_t ng = 0;
};
void sketch_shard_project(const Context& c, const double* pts, const double* w, int64_t ng,
                          const SelectOptions& o, int64_t n_total, SketchShard& st, cudaStream_t s);
void sketch_shard_combine(const Context& c, SketchShard& st, const double* sumsq_global, double* Yt,
                          double* delta, int64_t* kept_out, double* kept_xyz, double* kept_w,
                          std::vector<double>& scales, cudaStream_t s);
std::vector<int64_t> select_sketch_gathered(const Context& c, const SelectOptions& o, double* Yt, int64_t n,
                                            const double* kept_xyz, const double* kept_w, double* delta,
                                            const std::vector<double>& scales, SketchDiagnostics* diag,
                                            cudaStream_t s);

// One rank's share of the distributed sketch QR over its own kept points
// (Yt: ell x n_local, leading dimension n_local): the QR state and, in the
// mixed form (delta non-null), the FP64 recomputation source of its columns.
struct SketchQrShard {
    SketchSetup su;
    int64_t n_total = 0;
    DeviceBuffer<double> WT, scales;
    DeviceBuffer<int64_t> index;
    ExactSketchSource src;
    std::unique_ptr<QrShard> qr;
};
std::unique_ptr<SketchQrShard> make_sketch_qr_shard(const Context& c, const SelectOptions& o, double* Yt,
                                                    int64_t n_local, int64_t n_total, const double* kept_xyz,
                                                    const double* kept_w, double* delta,
                                                    const std::vector<double>& scales, int64_t pos_offset,
                                                    cudaStream_t s);

// qrcp_dense / qrcp_online: greedy max-residual pivoting of the weighted
// pair columns sqrt|w_g| f_g (x) f_g, computed without materialising them.
// One rank's share of the pair-space QR (qrcp_dense / qrcp_online) over a grid
// shard: its kept points' features, residual estimates and L rows, with the
// explicit pair basis Q replicated.  Every rank makes the same calls in the
// same order; verify() and accept() give bit-identical results on every rank
// (fixed-order reductions), so the ranks' bases stay equal.
class PairQrShard {
public:
    // pos_offset: the global kept position of this shard's first kept point;
    // grid_offset: the global grid index of its first grid point
    PairQrShard(const Context& c, const SelectOptions& o, const double* pts, const double* w, int64_t ng,
                int64_t grid_offset, cudaStream_t s);
    ~PairQrShard();
    int64_t n_kept() const;
    int64_t features() const;   // d
    void local_sumsq(double out[5]) const;
    // the global multi-axis sums and position offset -> local (sum K_gg, non-finite flag)
    void init(const double* sumsq_global, int64_t pos_offset, double out[2]);
    // best unselected local column: (estimate, global position, global kept index; -1 when none)
    void argmax(double key[3]);
    // row of global kept column gcol (local), kRowExtra + d doubles: its d
    // features, sqrt|w|, global grid index, x, y, z, w
    static constexpr int kRowExtra = 6;
    void row(int64_t gcol, double* out) const;
    // exact squared residual of the row's pair vector against the j basis vectors
    // (also the owner's estimate of it)
    double verify(const double* row_host, int j, int64_t gcol);
    // take the verified column as pivot j (the coefficients of its last verify)
    void accept(const double* row_host, int j, int64_t gcol, double exact2, int64_t winner_pos, bool dense);
    // exact recomputation of every local column whose estimate could exceed thr2
    int64_t scan(int j, double thr2);

private:
    struct Impl;
    Impl* p_;
};

std::vector<int64_t> select_pair_qr(const Context& c, const double* pts, const double* w,
                                    int64_t ng, const SelectOptions& o, cudaStream_t s,
                                    PairQrDiagnostics* diag = nullptr);

}  // namespace isdf
