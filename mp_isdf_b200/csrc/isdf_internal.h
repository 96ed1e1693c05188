// Internal declarations of the B200 ISDF library (not part of the C-ABI).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

namespace isdf {

constexpr int kMaxL = 6;          // highest angular momentum the AO kernels handle
constexpr int kMaxCtrGroup = 4;   // contractions evaluated per exponential sweep
constexpr double kExpCut = 100.0; // alpha*r^2 beyond which a primitive is skipped (<4e-44)

// Piece screening of the tiled evaluators.  A piece (contraction group of one
// shell) is written as zeros for a warp of points where amin r^2 >= X_sh at all
// of them; X_sh <= kExpCut is chosen per shell (screening_argument) so that no
// value or d/dx, d/dy, d/dz component dropped that way exceeds kScreenFp64 in
// absolute value (FP64 tables: far below the reference's AO tolerance of
// 1e-12) or kScreenFp32 (the FP32 tables of the fused projection, whose error
// bounds carry it as an absolute term).  The one-point-per-block kernels and
// the FP64 re-verification do not screen.
constexpr double kScreenFp64 = 1e-15;
constexpr double kScreenFp32 = 1e-11;

// ---- errors -----------------------------------------------------------------
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};
enum : int {
    kOk = 0,
    kInvalid = 1,        // -> ValueError (std::invalid_argument in the reference)
    kOverflow = 2,       // -> OverflowError / RuntimeError family (std::overflow_error)
    kRuntime = 3,        // -> RuntimeError
    kCuda = 4,           // CUDA runtime failure
    kNotImplemented = 5, // -> NotImplementedError
    kLogic = 6,          // -> RuntimeError (std::logic_error)
};
[[noreturn]] inline void fail(int code, const std::string& msg) { throw Error(code, msg); }
// Message returned by isdf_last_error() on the calling thread.
void set_last_error(const std::string& msg);
inline void require(bool ok, const std::string& msg) { if (!ok) fail(kInvalid, msg); }

#define ISDF_CUDA(expr)                                                                  \
    do {                                                                                 \
        cudaError_t err__ = (expr);                                                      \
        if (err__ != cudaSuccess)                                                        \
            ::isdf::fail(::isdf::kCuda, std::string(#expr) + ": " + cudaGetErrorString(err__)); \
    } while (0)
// Counts this library's kernel launches (isdf_launch_count) and checks them.
void count_launches(int64_t k);
#define ISDF_LAUNCH_CHECK()                  \
    do {                                     \
        ISDF_CUDA(cudaGetLastError());       \
        ::isdf::count_launches(1);           \
    } while (0)

// ---- profiling -----------------------------------------------------------------
// Scoped CUDA-event pair around the launches of one kernel family (no-op
// unless enabled through isdf_profile_enable).
bool profiling_enabled();
class ProfileScope {
public:
    ProfileScope(const char* name, cudaStream_t s);
    ~ProfileScope();
    ProfileScope(const ProfileScope&) = delete;
    ProfileScope& operator=(const ProfileScope&) = delete;

private:
    const char* name_;
    cudaStream_t s_;
    cudaEvent_t a_ = nullptr, b_ = nullptr;
};
#define ISDF_PROFILE_CAT2(a, b) a##b
#define ISDF_PROFILE_CAT(a, b) ISDF_PROFILE_CAT2(a, b)
#define ISDF_PROFILE(name, stream) ::isdf::ProfileScope ISDF_PROFILE_CAT(prof_, __LINE__)(name, stream)

// ---- device buffers ----------------------------------------------------------
// Stream-ordered allocation from the device's default memory pool.
template <class T>
class DeviceBuffer {
public:
    DeviceBuffer() = default;
    DeviceBuffer(size_t n, cudaStream_t s) { reset(n, s); }
    ~DeviceBuffer() { release(); }
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    DeviceBuffer(DeviceBuffer&& o) noexcept : p_(o.p_), n_(o.n_), s_(o.s_) { o.p_ = nullptr; o.n_ = 0; }
    DeviceBuffer& operator=(DeviceBuffer&& o) noexcept {
        if (this != &o) { release(); p_ = o.p_; n_ = o.n_; s_ = o.s_; o.p_ = nullptr; o.n_ = 0; }
        return *this;
    }
    void reset(size_t n, cudaStream_t s) {
        release();
        s_ = s;
        n_ = n;
        if (n) ISDF_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&p_), n * sizeof(T), s));
    }
    void release() {
        if (p_) cudaFreeAsync(p_, s_);
        p_ = nullptr;
        n_ = 0;
    }
    T* get() const { return p_; }
    size_t size() const { return n_; }
    void zero(cudaStream_t s) { if (n_) ISDF_CUDA(cudaMemsetAsync(p_, 0, n_ * sizeof(T), s)); }

private:
    T* p_ = nullptr;
    size_t n_ = 0;
    cudaStream_t s_ = nullptr;
};

// ---- shell table ---------------------------------------------------------------
struct ShellDesc {
    int l, nprim, nctr, ao_off;
    int prim_off;   // exponents at prim_off .. prim_off+nprim
    int coef_off;   // coefficients [nctr][nprim] at coef_off
    int atom;
    float amin;     // smallest exponent: the shell is exactly zero where amin r^2 > kExpCut
    // screening exponents amin * kExpCut / X_sh for the FP32 and FP64 bounds:
    // the piece is dropped for a warp where scr r^2 > kExpCut at every point
    float scr32, scr64;
    double x, y, z;
};

// Angular momentum group: a run of shells with equal l (kernels specialise on l).
struct Context {
    int device = 0;
    int nsm = 148;       // streaming multiprocessors of the device
    int natm = 0;
    int nao = 0;
    int nshell = 0;
    int lmax = 0;
    std::vector<int32_t> atm, bas;
    std::vector<double> env;
    std::vector<ShellDesc> shells;        // host copy
    std::vector<int32_t> ao_atom;         // atom of each AO
    std::vector<double> atom_xyz;         // natm x 3
    ShellDesc* d_shells = nullptr;
    double* d_exp = nullptr;
    double* d_coef = nullptr;
    float* d_expf = nullptr;
    float* d_coeff = nullptr;
    int32_t* d_ao_atom = nullptr;
    // shell centres as FP32 hi + lo pairs (x = hi + lo to ~2^-48 relative) and
    // the smallest exponent: (x_hi, y_hi, z_hi, amin), (x_lo, y_lo, z_lo, 0)
    float4* d_shell_hi = nullptr;
    float4* d_shell_lo = nullptr;
    // K-chunk layout of the tensor-core projection (built with the context):
    // chunks of 32 AO slots holding whole contraction groups ("pieces").
    int nchunks = 0;
    int4* d_pieces = nullptr;             // (shell, first contraction, contractions, first slot)
    int piece_lanes = 0;                  // producer lanes per point the layout is balanced for
    int* d_piece_begin = nullptr;         // lane j of chunk c: [begin[c*lanes + j], begin[c*lanes + j + 1])
    int* d_fill = nullptr;                // used slots per chunk
    int* d_chunk_ao0 = nullptr;           // first AO of each chunk (a chunk is a contiguous AO range)
    int2* d_ao_slot = nullptr;            // (chunk, slot) of each AO
    int* d_piece_chunk = nullptr;         // chunk of each piece (d_pieces order)
    int npieces = 0;
    // AO-window layout of the tiled evaluators: window w covers the AOs
    // [32w, 32w + 32), so each stored row segment is a whole, aligned run of
    // the output row; its entries are the pieces that overlap it (a piece
    // across a window boundary appears in both), each as (piece, offset of the
    // piece's first AO from 32w), balanced over the producer lanes:
    // lane j of window w owns [win_begin[w*lanes + j], win_begin[w*lanes + j + 1]).
    int nwin = 0;
    int2* d_win_entry = nullptr;
    int* d_win_begin = nullptr;
    // Packed piece records of the fused kernel, in the order of d_pieces: per
    // piece three float4 -- (x_hi, y_hi, z_hi, FP32 screening exponent), (x_lo, y_lo, z_lo,
    // prim_off as bits), (l, nprim, contractions, first slot as int bits) --
    // and per piece, group of three contractions and primitive one float4
    // (alpha, c_j, c_j+1, c_j+2) at prim_off (FP32, zero-padded contractions).
    float4* d_piece_rec = nullptr;
    float4* d_piece_prim = nullptr;
    // FP64 twins for the tiled evaluators: centre and FP64 screening exponent
    // as two double2 (x, y), (z, scr64) per piece, and two double2 (alpha, c_j),
    // (c_j+1, c_j+2) per entry of the primitive table (same entry index).
    double2* d_piece_c64 = nullptr;
    double2* d_piece_prim64 = nullptr;
    std::vector<int4> h_pieces;           // host copy of the pieces
    std::vector<float> h_expf, h_coeff;   // host FP32 exponents / coefficients (shell order)
    std::vector<double> h_exp64, h_coef64;   // the same in FP64
    // Grow-only device workspace of the fused selection + fit (the stored AO
    // tiles and the sketch projections), kept across calls so that repeated
    // calls allocate nothing large; a call holds ws_mu while it uses it.
    mutable std::mutex ws_mu;
    mutable uint8_t* ws = nullptr;
    mutable size_t ws_bytes = 0;
    // At least `bytes` of workspace (the caller holds ws_mu; growing waits for
    // the device and invalidates earlier pointers).
    uint8_t* workspace(size_t bytes) const;
    ~Context();
};

// Copies the shells' centres (FP32 hi + lo) and smallest exponents to the device
// (and refreshes the packed piece records, which hold them too).
void upload_shell_centres(Context& c);
// (Re)writes the packed piece records and primitive table (d_piece_rec/prim).
void upload_piece_records(Context& c);
// Fills the context's K-chunk layout (defined with the projection kernel).
void build_chunk_layout(Context& c);
// Fills the AO-window layout from the pieces of the K-chunk layout.
void build_window_layout(Context& c);
constexpr int kWin = 32;   // AOs per window of the tiled evaluators
// Producer lanes per point of the projection kernel for a basis' largest l.
inline int piece_lanes_for_lmax(int lmax) { return lmax <= 2 ? 6 : 2; }

Context* create_context(const int32_t* atm, int natm, const int32_t* bas, int nbas,
                        const double* env, int64_t nenv);

// Real-spherical transform of one angular momentum: nsph x ncart, row-major.

// ---- AO evaluation ---------------------------------------------------------------
// Component codes used by the kernels: 0 value, 1 d/dx, 2 d/dy, 3 d/dz.
enum AoOut : int { kAoValues = 1, kAoGrad = 2 };

// Values [p*ld + ao] and/or gradients [(c*n + p)*ld + ao] (component-major as
// in the reference).  `out_grad` may alias a separate buffer.
template <class T>
void eval_ao(const Context& c, const double* pts, int64_t n, T* out_val, T* out_grad,
             int64_t ld, cudaStream_t s);

// Concatenated axis features F[g*d + off_a + j] = scale_a * comp_a(g, j) over
// the given points (gathered through `index` when non-null), with per-component
// sums of squares accumulated into sumsq[4] (FP64) over points whose weight
// (through `weights`, may be null) is nonzero.
struct AxisSpec {
    int naxes = 0;
    int comp[16];      // component of each axis entry (0..3)
    double scale[16];  // scale of each axis entry
    int need_mask = 0; // bit c set if component c is needed
    // feature layout: entry a occupies features [offset[a], offset[a] + width[a])
    int offset[16];
    int width[16];
    int64_t d = 0;               // total features
    // occupied-orbital entries: psi_j = sum_mu phi_mu C[mu][j], j < nocc, with
    // C row-major nao x nao in device memory (mo)
    bool occ[16];
    int nocc = 0;
    const double* mo = nullptr;
    bool has_occ = false;
};
template <class T>
void eval_axis_features(const Context& c, const double* pts, const int64_t* index, int64_t n,
                        const AxisSpec& ax, T* out, int64_t ld, double* sumsq,
                        const double* weights, cudaStream_t s);

// ---- small dense kernels ---------------------------------------------------------
void iota_i64(int64_t* out, int64_t n, cudaStream_t s);
void widen_f32(const float* x, int64_t n, double* y, cudaStream_t s);
// out[g] = F[g,:] . x (warp per row); |F[g,:]|^2 when x is null.
void row_dot(const double* F, int64_t n, int64_t d, const double* x, double* out, cudaStream_t s);
// a[i*d + k] = scale * f[i] * f[k]   (explicit weighted pair vector)
void pair_vector(const double* f, int64_t d, double scale, double* a, cudaStream_t s);
// out[r] += Q[r,:] . x  for r < rows (Q row-major rows x m); out must be pre-zeroed
void rows_dot(const double* Q, int rows, int64_t m, const double* x, double* out, cudaStream_t s);
// y = x - Q^T t ; *norm2 += |y|^2 when norm2 is non-null (x and y may alias)
void rows_axpy(const double* Q, int rows, int64_t m, const double* t, const double* x, double* y,
               double* norm2, cudaStream_t s);
void scale_copy(const double* x, double scale, int64_t m, double* y, cudaStream_t s);
// C[z][m][n] (+)= A[z][m][k] B[z][k][n], FP64, row-major with explicit strides.
void gemm_f64(int64_t M, int64_t N, int64_t K, const double* A, int64_t lda, int64_t strideA,
              const double* B, int64_t ldb, int64_t strideB, double* C, int64_t ldc,
              int64_t strideC, int batch, bool accumulate, cudaStream_t s);

}  // namespace isdf
