// Grid-point compaction, multi-axis Frobenius scales, the quadrature
// Khatri-Rao pair sketch and the column-pivoted QR of the sketch.
//
// Reference behaviour restated (mikovtun/mp_isdf):
//   eligibility (weights finite, zero weights skipped, kept coordinates finite)
//       cpp/src/anchor_select_randomized_id.cpp:131-146
//   multi-axis global Frobenius scales      cpp/src/anchor_select.cpp:437-480
//   sketch rows, caps and validation        cpp/src/anchor_select_randomized_id.cpp:116-191
//   U/V streams (mt19937_64, normal_distribution, u[a*ell+s])
//                                           cpp/src/anchor_select_randomized_id.cpp:269-279
//   Y[s,g] = sqrt|w_g|/sqrt(ell) (f_g.u_s)(f_g.v_s)   :297-309
//   dgeqp3 of Y, row energies -> tails, numerical rank, exact-rank / tolerance
//   rank selection                          cpp/src/anchor_select_randomized_id.cpp:320-374
#include "isdf_fit.h"
#include "isdf_project.h"
#include "isdf_select.h"
#include "isdf_reduce.cuh"

#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <future>
#include <limits>
#include <mutex>
#include <new>
#include <random>
#include <condition_variable>
#include <functional>
#include <thread>
#include <unistd.h>
#include <immintrin.h>

namespace isdf {

// ------------------------------------------------------------------------------
// eligibility + compaction
// ------------------------------------------------------------------------------
namespace {

__global__ void flag_points_kernel(const double* __restrict__ pts, const double* __restrict__ w,
                                   const double* __restrict__ importance, int64_t n,
                                   char* __restrict__ keep, int* __restrict__ bad) {
    const int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g >= n) return;
    bool important = true;
    if (importance) {
        const double m = importance[g];
        if (!isfinite(m) || m < 0.0) atomicOr(bad, 4);
        important = m != 0.0;
    }
    const double wg = w[g];
    if (!isfinite(wg)) { atomicOr(bad, 1); keep[g] = 0; return; }
    const bool k = wg != 0.0 && important;
    keep[g] = k;
    if (k && !(isfinite(pts[3 * g]) && isfinite(pts[3 * g + 1]) && isfinite(pts[3 * g + 2])))
        atomicOr(bad, 2);
}

// 16 bits of v spread to every third bit
__device__ __forceinline__ uint64_t spread3(uint64_t v) {
    v &= 0xffffull;
    v = (v | v << 16) & 0x0000ff0000ffull;
    v = (v | v << 8) & 0x00f00f00f00full;
    v = (v | v << 4) & 0x0c30c30c30c3ull;
    v = (v | v << 2) & 0x249249249249ull;
    return v;
}

// key of position i: window (i / kSpatialWindow) above the Morton code of the
// point's 1-bohr cell (16 bits per axis, cells offset by 2^15); the value is i
__global__ void spatial_key_kernel(const double* __restrict__ pts, const int64_t* __restrict__ index, int64_t n,
                                   uint64_t* __restrict__ key, int64_t* __restrict__ val) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t g = index[i];
    uint64_t m = 0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double c = floor(pts[3 * g + d]) + 32768.0;
        const uint64_t q = c < 0.0 ? 0ull : c > 65535.0 ? 65535ull : static_cast<uint64_t>(c);
        m |= spread3(q) << d;
    }
    key[i] = (static_cast<uint64_t>(i / kSpatialWindow) << 48) | m;
    val[i] = i;
}

__global__ void gather_index_kernel(const int64_t* __restrict__ asc, const int64_t* __restrict__ perm, int64_t n,
                                    int64_t* __restrict__ out) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) out[i] = asc[perm[i]];
}

__global__ void unpermute_columns_kernel(const double* __restrict__ src, double* __restrict__ dst, int64_t ld,
                                         int64_t k, const int64_t* __restrict__ rank, int64_t p0, int64_t m) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const int64_t p = p0 + i, r = rank[p];
    for (int64_t a = 0; a < k; ++a) dst[a * ld + r] = src[a * ld + p];
}

}  // namespace

void unpermute_columns(const double* src, double* dst, int64_t ld, int64_t k, const int64_t* rank, int64_t p0,
                       int64_t m, cudaStream_t s) {
    if (m <= 0 || k <= 0) return;
    unpermute_columns_kernel<<<static_cast<unsigned>((m + 255) / 256), 256, 0, s>>>(src, dst, ld, k, rank, p0, m);
    ISDF_LAUNCH_CHECK();
}

KeptPoints compact_points(const double* pts, const double* w, int64_t n, cudaStream_t s,
                          const double* importance, bool spatial) {
    KeptPoints kp;
    kp.index.reset(std::max<int64_t>(n, 1), s);
    if (n == 0) return kp;
    DeviceBuffer<char> keep(n, s);
    DeviceBuffer<int> bad(1, s);
    DeviceBuffer<int64_t> count(1, s);
    bad.zero(s);
    flag_points_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(pts, w, importance, n,
                                                                              keep.get(), bad.get());
    ISDF_LAUNCH_CHECK();
    size_t tmp_bytes = 0;
    thrust::counting_iterator<int64_t> it(0);
    ISDF_CUDA(cub::DeviceSelect::Flagged(nullptr, tmp_bytes, it, keep.get(), kp.index.get(),
                                         count.get(), n, s));
    DeviceBuffer<char> tmp(tmp_bytes, s);
    ISDF_CUDA(cub::DeviceSelect::Flagged(tmp.get(), tmp_bytes, it, keep.get(), kp.index.get(),
                                         count.get(), n, s));
    count_launches(2);   // the selection's initialisation and sweep kernels
    int hbad = 0;
    int64_t hcount = 0;
    ISDF_CUDA(cudaMemcpyAsync(&hbad, bad.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaMemcpyAsync(&hcount, count.get(), sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaStreamSynchronize(s));
    if (hbad & 4) fail(kInvalid, "point_importance must be finite and nonnegative");
    if (hbad & 1) fail(kInvalid, "grid weights must be finite");
    if (hbad & 2) fail(kInvalid, "grid coordinates must be finite");
    kp.n = hcount;
    if (spatial && hcount > 128 && hcount < (int64_t(1) << 31)) {
        // Morton order inside each window: (key, position) pairs sorted by key
        const int64_t m = hcount;
        DeviceBuffer<uint64_t> key(m, s), key2(m, s);
        DeviceBuffer<int64_t> val(m, s), perm(m, s), index(m, s);
        const unsigned nb = static_cast<unsigned>((m + 255) / 256);
        spatial_key_kernel<<<nb, 256, 0, s>>>(pts, kp.index.get(), m, key.get(), val.get());
        ISDF_LAUNCH_CHECK();
        size_t sort_bytes = 0;
        ISDF_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, key.get(), key2.get(), val.get(), perm.get(),
                                                  static_cast<int>(m), 0, 64, s));
        DeviceBuffer<char> sort_tmp(sort_bytes, s);
        ISDF_CUDA(cub::DeviceRadixSort::SortPairs(sort_tmp.get(), sort_bytes, key.get(), key2.get(), val.get(),
                                                  perm.get(), static_cast<int>(m), 0, 64, s));
        count_launches(8);   // the sort's passes (upper bound)
        gather_index_kernel<<<nb, 256, 0, s>>>(kp.index.get(), perm.get(), m, index.get());
        ISDF_LAUNCH_CHECK();
        kp.index = std::move(index);
        kp.rank = std::move(perm);
    }
    return kp;
}

// ------------------------------------------------------------------------------
// axis bookkeeping
// ------------------------------------------------------------------------------
AxisSpec make_axis_spec(const Context& c, const int32_t* axes, int naxes, const double* mo, int64_t nocc) {
    require(naxes > 0, "axis list must not be empty");
    if (naxes > 16) fail(kNotImplemented, "more than 16 axis entries are not supported");
    AxisSpec ax{};
    ax.naxes = naxes;
    int64_t d = 0;
    for (int a = 0; a < naxes; ++a) {
        const int t = axes[a];
        require(t >= 0 && t <= 4, "unknown AxisType");
        ax.occ[a] = t == 4;
        if (t == 4) {
            // cpp/src/anchor_select.cpp:43-49
            if (!mo || nocc < 1 || nocc > c.nao)
                fail(kInvalid, "OccupiedOrbital requires row-major (nao,nao) RHF mo_coeff and 1 <= nocc <= nao");
            ax.has_occ = true;
            ax.nocc = static_cast<int>(nocc);
            ax.mo = mo;
        }
        ax.comp[a] = t == 4 ? 0 : t;
        ax.scale[a] = 1.0;
        ax.need_mask |= 1 << ax.comp[a];
        ax.width[a] = t == 4 ? static_cast<int>(nocc) : c.nao;
        ax.offset[a] = static_cast<int>(d);
        d += ax.width[a];
    }
    require(c.nao > 0 && d > 0, "no orbital features available");
    require(d < (int64_t(1) << 30), "axis feature count is too large");
    ax.d = d;
    return ax;
}

AxisSetup make_axis_setup(const Context& c, const SelectOptions& o, cudaStream_t s) {
    AxisSetup st;
    if (o.mo_host && c.nao > 0) {
        st.mo.reset(static_cast<size_t>(c.nao) * c.nao, s);
        ISDF_CUDA(cudaMemcpyAsync(st.mo.get(), o.mo_host, static_cast<size_t>(c.nao) * c.nao * sizeof(double),
                                  cudaMemcpyHostToDevice, s));
    }
    st.ax = make_axis_spec(c, o.axes.data(), static_cast<int>(o.axes.size()), st.mo.get(), o.nocc);
    return st;
}

std::vector<double> axis_scales_from_sumsq(const AxisSpec& ax, const double* sumsq4,
                                           const double* axis_weights, bool any_eligible) {
    std::vector<double> scales;
    if (!any_eligible) return scales;
    for (int a = 0; a < ax.naxes; ++a) {
        // slot 4 holds the occupied-orbital features' sum of squares
        const double norm = std::sqrt(sumsq4[ax.occ[a] ? 4 : ax.comp[a]]);
        if (!(norm > 0) || !std::isfinite(norm))
            fail(kInvalid, "axis Frobenius norm must be finite and positive");
        const double scale = (axis_weights ? axis_weights[a] : 1.0) / norm;
        if (!(scale > 0) || !std::isfinite(scale))
            fail(kInvalid, "normalized axis scale must be finite and positive");
        scales.push_back(scale);
    }
    return scales;
}

void validate_axis_weights(const double* axis_weights, int naxes) {
    if (!axis_weights) return;
    for (int a = 0; a < naxes; ++a)
        if (!std::isfinite(axis_weights[a]) || axis_weights[a] <= 0)
            fail(kInvalid, "axis weights must be finite and positive");
}

// ------------------------------------------------------------------------------
// pinned host blocks
// ------------------------------------------------------------------------------
namespace {
struct PinnedBlock { void* p; size_t bytes; bool pinned; };
std::mutex g_pinned_mu;
std::vector<PinnedBlock> g_pinned_free;   // blocks returned by freed vectors
std::vector<PinnedBlock> g_pinned_live;
}  // namespace

void* pinned_host_alloc(size_t bytes) {
    if (bytes == 0) bytes = 1;
    {
        std::lock_guard<std::mutex> lock(g_pinned_mu);
        // the smallest cached block that is large enough
        size_t best = g_pinned_free.size();
        for (size_t i = 0; i < g_pinned_free.size(); ++i)
            if (g_pinned_free[i].bytes >= bytes &&
                (best == g_pinned_free.size() || g_pinned_free[i].bytes < g_pinned_free[best].bytes))
                best = i;
        if (best < g_pinned_free.size()) {
            const PinnedBlock b = g_pinned_free[best];
            g_pinned_free.erase(g_pinned_free.begin() + static_cast<std::ptrdiff_t>(best));
            g_pinned_live.push_back(b);
            return b.p;
        }
    }
    PinnedBlock b{nullptr, bytes, true};
    if (cudaHostAlloc(&b.p, bytes, cudaHostAllocPortable) != cudaSuccess) {
        cudaGetLastError();   // not sticky: fall back to pageable memory
        b.p = std::malloc(bytes);
        b.pinned = false;
        if (!b.p) throw std::bad_alloc();
    }
    std::lock_guard<std::mutex> lock(g_pinned_mu);
    g_pinned_live.push_back(b);
    return b.p;
}

void pinned_host_free(void* p, size_t) noexcept {
    if (!p) return;
    std::lock_guard<std::mutex> lock(g_pinned_mu);
    for (size_t i = 0; i < g_pinned_live.size(); ++i)
        if (g_pinned_live[i].p == p) {
            const PinnedBlock b = g_pinned_live[i];
            g_pinned_live.erase(g_pinned_live.begin() + static_cast<std::ptrdiff_t>(i));
            if (b.pinned && g_pinned_free.size() < 8) {
                g_pinned_free.push_back(b);   // kept for the next selection
            } else if (b.pinned) {
                cudaFreeHost(b.p);
            } else {
                std::free(b.p);
            }
            return;
        }
}

// ------------------------------------------------------------------------------
// sketch
// ------------------------------------------------------------------------------
namespace {

// std::normal_distribution<double>(0, 1) over std::mt19937_64, drawn as
// libstdc++ does it (Marsaglia's polar method): an attempt takes two engine
// outputs, each made a uniform in [0, 1) by generate_canonical<double, 53>
// (one 64-bit output rounded once to double and scaled by 2^-64; 1.0 becomes
// the largest double below 1), x = 2u - 1, y = 2u' - 1, and is rejected
// unless 0 < x^2 + y^2 <= 1; an accepted attempt yields y f, then x f, with
// f = sqrt(-2 ln(r2) / r2).  Only the engine is sequential: one thread per
// stream draws the outputs and counts the accepted attempts per block of
// attempts, and worker threads transform each block into its known place as
// soon as it is published.
inline double canonical53(uint64_t r) {
    // the exact value hi 2^32 + lo rounded once: the correctly rounded conversion
    const double x = (static_cast<double>(static_cast<uint32_t>(r >> 32)) * 0x1p32 +
                      static_cast<double>(static_cast<uint32_t>(r))) * 0x1p-64;
    return x >= 1.0 ? 0x1.fffffffffffffp-1 : x;   // the largest double below 1
}

constexpr double kStdDev = 1.0, kMean = 0.0;
constexpr int64_t kPolarBlock = 2048;   // attempts per block of the transform

// std::mt19937_64 as the C++ standard defines it ([rand.eng.mers], [rand.predef]:
// w 64, n 312, m 156, r 31, a 0xb5026f5aa96619e9, u 29 d 0x5555555555555555,
// s 17 b 0x71d67fffeda60000, t 37 c 0xfff7eee000000000, l 43,
// f 6364136223846793005), producing its outputs 312 at a time: the state
// transition runs over the whole array in branch-free loops and the tempering
// in a separate loop, both of which the compiler vectorises.  The output
// sequence is the standard engine's for the same seed.
class Mt64Blocks {
public:
    static constexpr int kN = 312, kM = 156;
    explicit Mt64Blocks(uint64_t seed) {
        x_[0] = seed;
        for (int i = 1; i < kN; ++i) x_[i] = 6364136223846793005ULL * (x_[i - 1] ^ (x_[i - 1] >> 62)) + i;
    }
    uint64_t operator()() {
        if (idx_ == kN) { transition(); temper(buf_); idx_ = 0; }
        return buf_[idx_++];
    }
    // the next `count` outputs, in order
    void fill(uint64_t* out, int64_t count) {
        while (count > 0) {
            if (idx_ == kN) {
                transition();
                if (count >= kN) {   // a whole block straight into the output
                    temper(out);
                    out += kN;
                    count -= kN;
                    continue;
                }
                temper(buf_);
                idx_ = 0;
            }
            const int64_t take = std::min<int64_t>(count, kN - idx_);
            std::memcpy(out, buf_ + idx_, static_cast<size_t>(take) * sizeof(uint64_t));
            out += take;
            count -= take;
            idx_ += static_cast<int>(take);
        }
    }

private:
    static uint64_t twist(uint64_t cur, uint64_t next, uint64_t far) {
        constexpr uint64_t kUpper = ~((uint64_t(1) << 31) - 1), kLower = (uint64_t(1) << 31) - 1;
        const uint64_t y = (cur & kUpper) | (next & kLower);
        return far ^ (y >> 1) ^ ((uint64_t(0) - (y & 1)) & 0xb5026f5aa96619e9ULL);
    }
    __attribute__((optimize("O3"), target_clones("avx2", "default"))) void transition() {
        for (int i = 0; i < kN - kM; ++i) x_[i] = twist(x_[i], x_[i + 1], x_[i + kM]);
        for (int i = kN - kM; i < kN - 1; ++i) x_[i] = twist(x_[i], x_[i + 1], x_[i + kM - kN]);
        x_[kN - 1] = twist(x_[kN - 1], x_[0], x_[kM - 1]);
    }
    __attribute__((optimize("O3"), target_clones("avx2", "default"))) void temper(uint64_t* out) const {
        for (int i = 0; i < kN; ++i) {
            uint64_t z = x_[i];
            z ^= (z >> 29) & 0x5555555555555555ULL;
            z ^= (z << 17) & 0x71d67fffeda60000ULL;
            z ^= (z << 37) & 0xfff7eee000000000ULL;
            out[i] = z ^ (z >> 43);
        }
    }
    uint64_t x_[kN];
    uint64_t buf_[kN];
    int idx_ = kN;
};

// Worker threads for the sketch-factor draw, created once per process (a
// call used to start a dozen threads, 20-50 us each): start(n, job) has n pool
// threads call job(0..n-1) while the caller works on; wait() returns when all
// have finished.  One run at a time (start takes a lock that wait releases); a
// process forked after the pool started gets a fresh pool.
class DrawPool {
public:
    static DrawPool& get(int size) {
        static std::mutex mu;
        static DrawPool* pool = nullptr;
        std::lock_guard<std::mutex> lk(mu);
        if (!pool || pool->pid_ != getpid() || pool->size() < size) pool = new DrawPool(size);   // old one leaks
        return *pool;
    }
    int size() const { return static_cast<int>(threads_.size()); }
    void start(int n, const std::function<void(int)>& job) {
        run_mu_.lock();
        {
            std::lock_guard<std::mutex> lk(m_);
            job_ = &job;
            njobs_ = n;
            pending_ = n;
            ++gen_;
        }
        cv_.notify_all();
    }
    void wait() {
        {
            std::unique_lock<std::mutex> lk(m_);
            done_.wait(lk, [this] { return pending_ == 0; });
            job_ = nullptr;
        }
        run_mu_.unlock();
    }

private:
    explicit DrawPool(int size) : pid_(getpid()) {
        for (int i = 0; i < size; ++i) {
            threads_.emplace_back([this, i] { loop(i); });
            threads_.back().detach();
        }
    }
    void loop(int id) {
        uint64_t seen = 0;
        std::unique_lock<std::mutex> lk(m_);
        for (;;) {
            cv_.wait(lk, [&] { return gen_ != seen; });
            seen = gen_;
            if (id >= njobs_) continue;
            const std::function<void(int)>* job = job_;
            lk.unlock();
            (*job)(id);
            lk.lock();
            if (--pending_ == 0) done_.notify_all();
        }
    }
    pid_t pid_;
    std::vector<std::thread> threads_;
    std::mutex m_, run_mu_;
    std::condition_variable cv_, done_;
    const std::function<void(int)>* job_ = nullptr;
    int njobs_ = 0, pending_ = 0;
    uint64_t gen_ = 0;
};

// Accepted attempts among the 2 * attempts engine outputs at raw.
int64_t polar_accepted(const uint64_t* raw, int64_t attempts) {
    int64_t n_ok = 0;
    for (int64_t a = 0; a < attempts; ++a) {
        const double x = 2.0 * canonical53(raw[2 * a]) - 1.0;
        const double y = 2.0 * canonical53(raw[2 * a + 1]) - 1.0;
        const double r2 = x * x + y * y;
        n_ok += (r2 <= 1.0) & (r2 != 0.0);
    }
    return n_ok;
}

// The same count, four attempts per step.  Each operation is the scalar
// one's: the 64-bit output becomes a double through its two exactly converted
// 32-bit halves (each placed in the mantissa of 2^84 or 2^52 and that power
// subtracted) added with one rounding, then 2u - 1 and x^2 + y^2 by separate
// multiplies and adds (the target has no FMA), so the count is identical.
// 2 canonical53(r) - 1 for four outputs.
__attribute__((target("avx2"))) inline __m256d centred_avx2(__m256i r) {
    const __m256d hi = _mm256_sub_pd(
        _mm256_castsi256_pd(_mm256_or_si256(_mm256_srli_epi64(r, 32), _mm256_set1_epi64x(0x4530000000000000LL))),
        _mm256_set1_pd(0x1p84));
    const __m256d lo = _mm256_sub_pd(
        _mm256_castsi256_pd(_mm256_or_si256(_mm256_and_si256(r, _mm256_set1_epi64x(0xffffffffLL)),
                                            _mm256_set1_epi64x(0x4330000000000000LL))),
        _mm256_set1_pd(0x1p52));
    // the largest double below 1 where the rounded value is 1
    const __m256d u = _mm256_min_pd(_mm256_mul_pd(_mm256_add_pd(hi, lo), _mm256_set1_pd(0x1p-64)),
                                    _mm256_set1_pd(0x1.fffffffffffffp-1));
    return _mm256_sub_pd(_mm256_mul_pd(_mm256_set1_pd(2.0), u), _mm256_set1_pd(1.0));
}

__attribute__((target("avx2"))) int64_t polar_accepted_avx2(const uint64_t* raw, int64_t attempts) {
    const __m256d one = _mm256_set1_pd(1.0), zero = _mm256_setzero_pd();
    int64_t n_ok = 0, a = 0;
    for (; a + 4 <= attempts; a += 4) {
        // (x0 y0 x1 y1), (x2 y2 x3 y3) -> x_i^2 + y_i^2 for i = 0, 2, 1, 3
        const __m256d t0 = centred_avx2(_mm256_loadu_si256(reinterpret_cast<const __m256i*>(raw + 2 * a)));
        const __m256d t1 = centred_avx2(_mm256_loadu_si256(reinterpret_cast<const __m256i*>(raw + 2 * a + 4)));
        const __m256d r2 = _mm256_hadd_pd(_mm256_mul_pd(t0, t0), _mm256_mul_pd(t1, t1));
        const __m256d ok = _mm256_and_pd(_mm256_cmp_pd(r2, one, _CMP_LE_OQ), _mm256_cmp_pd(r2, zero, _CMP_NEQ_UQ));
        n_ok += __builtin_popcount(static_cast<unsigned>(_mm256_movemask_pd(ok)));
    }
    return n_ok + polar_accepted(raw + 2 * a, attempts - a);
}

struct PolarDraws {
    std::vector<uint64_t> raw;        // two engine outputs per attempt
    std::vector<int64_t> block_out;   // deviates produced before each block
    int64_t nblocks = 0;              // blocks drawn (read after the join)
    std::atomic<int64_t> published{0};
    std::atomic<bool> done{false};
};

// The sequential part: engine outputs until `pairs` attempts are accepted,
// published block by block with the deviates produced so far (at most
// max_blocks; the caller finishes a stream that needs more).  Returns the
// engine for that tail: it stands right after the last block's outputs,
// which are then all consumed.
Mt64Blocks polar_draw(uint64_t seed, int64_t pairs, int64_t max_blocks, PolarDraws& pd) {
    Mt64Blocks gen(seed);
    static const bool avx2 = __builtin_cpu_supports("avx2");
    int64_t acc = 0, b = 0;
    pd.block_out[0] = 0;
    while (acc < pairs && b < max_blocks) {
        const uint64_t* raw = pd.raw.data() + 2 * b * kPolarBlock;
        gen.fill(pd.raw.data() + 2 * b * kPolarBlock, 2 * kPolarBlock);
        acc += avx2 ? polar_accepted_avx2(raw, kPolarBlock) : polar_accepted(raw, kPolarBlock);
        pd.block_out[b + 1] = 2 * acc;
        pd.published.store(++b, std::memory_order_release);
    }
    pd.nblocks = b;
    pd.done.store(true, std::memory_order_release);
    return gen;
}

// Deviates of a published block b, written at their place in out[0, count).
void polar_block(const PolarDraws& pd, int64_t b, double* out, int64_t count) {
    int64_t o = pd.block_out[b];
    const int64_t o1 = std::min(count, pd.block_out[b + 1]);
    for (int64_t a = b * kPolarBlock; o < o1; ++a) {
        const double x = 2.0 * canonical53(pd.raw[2 * a]) - 1.0;
        const double y = 2.0 * canonical53(pd.raw[2 * a + 1]) - 1.0;
        const double r2 = x * x + y * y;
        if (r2 > 1.0 || r2 == 0.0) continue;
        const double f = std::sqrt(-2 * std::log(r2) / r2);
        out[o++] = y * f * kStdDev + kMean;
        if (o < o1) out[o++] = x * f * kStdDev + kMean;
    }
}

}  // namespace

void sketch_factors(int64_t d, int64_t ell, uint64_t seed, double* u, double* v) {
    // Two independent streams; fill order i = a*ell + s.
    const int64_t count = d * ell;
    if (count <= 0) return;
    const uint64_t seeds[2] = {seed, seed ^ 0x9e3779b97f4a7c15ULL};
    double* outs[2] = {u, v};
    const int64_t pairs = (count + 1) / 2;
    // attempts are accepted with probability pi/4: far more blocks than any
    // stream needs in practice; a stream that needs more is finished below
    const int64_t max_blocks = (pairs * 3 / 2) / kPolarBlock + 4;
    // the calling thread's buffers, kept so later calls touch no fresh pages
    thread_local std::vector<uint64_t> raw_keep[2];
    thread_local std::vector<int64_t> out_keep[2];
    PolarDraws pd[2];
    for (int k = 0; k < 2; ++k) {
        raw_keep[k].resize(static_cast<size_t>(2 * max_blocks * kPolarBlock));
        out_keep[k].resize(static_cast<size_t>(max_blocks + 1));
        pd[k].raw.swap(raw_keep[k]);
        pd[k].block_out.swap(out_keep[k]);
    }
    // two threads draw (one per stream) while the others transform each
    // published block; a worker takes every nw-th block of each stream
    const int nw = static_cast<int>(std::clamp(std::thread::hardware_concurrency(), 3u, 12u)) - 2;
    Mt64Blocks tail_gen[2] = {Mt64Blocks(seeds[0]), Mt64Blocks(seeds[1])};
    auto work = [&pd, &outs, count, nw](int w) {
        for (int k = 0; k < 2; ++k)
            for (int64_t b = w;; b += nw) {
                // wait until block b is drawn or the stream ended before it
                while (pd[k].published.load(std::memory_order_acquire) <= b &&
                       !pd[k].done.load(std::memory_order_acquire))
                    std::this_thread::yield();
                if (b >= pd[k].published.load(std::memory_order_acquire)) break;
                polar_block(pd[k], b, outs[k], count);
            }
    };
    {
        // pool job 0 draws stream 1, jobs 1..nw transform; this thread draws stream 0
        DrawPool& pool = DrawPool::get(nw + 1);
        std::exception_ptr err;
        std::mutex err_mu;
        const std::function<void(int)> job = [&](int i) {
            try {
                if (i == 0) tail_gen[1] = polar_draw(seeds[1], pairs, max_blocks, pd[1]);
                else work(i - 1);
            } catch (...) {
                std::lock_guard<std::mutex> lk(err_mu);
                if (!err) err = std::current_exception();
            }
        };
        pool.start(nw + 1, job);
        try {
            tail_gen[0] = polar_draw(seeds[0], pairs, max_blocks, pd[0]);
        } catch (...) {
            pd[0].done.store(true, std::memory_order_release);   // release the transform workers
            pool.wait();
            throw;
        }
        pool.wait();
        if (err) std::rethrow_exception(err);
    }
    for (int k = 0; k < 2; ++k) {
        // practically never: continue the engine where the blocks end
        int64_t o = pd[k].block_out[pd[k].nblocks];
        while (o < count) {
            const double x = 2.0 * canonical53(tail_gen[k]()) - 1.0;
            const double y = 2.0 * canonical53(tail_gen[k]()) - 1.0;
            const double r2 = x * x + y * y;
            if (r2 > 1.0 || r2 == 0.0) continue;
            const double f = std::sqrt(-2 * std::log(r2) / r2);
            outs[k][o++] = y * f * kStdDev + kMean;
            if (o < count) outs[k][o++] = x * f * kStdDev + kMean;
        }
        pd[k].raw.swap(raw_keep[k]);
        pd[k].block_out.swap(out_keep[k]);
    }
    // the first deviates must be the standard library's own (another library
    // may draw differently): otherwise draw everything through it
    bool same = true;
    for (int k = 0; k < 2 && same; ++k) {
        std::mt19937_64 gen(seeds[k]);
        std::normal_distribution<double> normal(kMean, kStdDev);
        for (int64_t i = 0; i < std::min<int64_t>(count, 64) && same; ++i) same = normal(gen) == outs[k][i];
    }
    if (!same) {
        auto fill = [count](uint64_t sd, double* o) {
            std::mt19937_64 gen(sd);
            std::normal_distribution<double> normal(kMean, kStdDev);
            for (int64_t i = 0; i < count; ++i) o[i] = normal(gen);
        };
        std::thread tv(fill, seeds[1], v);
        fill(seeds[0], u);
        tv.join();
    }
}

void sketch_factors(int64_t d, int64_t ell, uint64_t seed, HostFactors& u, HostFactors& v) {
    u.resize(static_cast<size_t>(d * ell));
    v.resize(static_cast<size_t>(d * ell));
    sketch_factors(d, ell, seed, u.data(), v.data());
}

namespace {

// Yt[s*ldy + g] = sqrt|w|/sqrt(ell) * (sum_a sc_a P[g][a][s]) * (sum_a sc_a P[g][a][ell+s])
__global__ void combine_sketch_kernel(const double* __restrict__ P, int naxes, int64_t ell,
                                      const double* __restrict__ scales,
                                      const double* __restrict__ w,
                                      const int64_t* __restrict__ index, int64_t n,
                                      double* __restrict__ Yt, int64_t ldy, int* __restrict__ bad) {
    const int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g >= n) return;
    const double sw = sqrt(fabs(w[index[g]])) / sqrt(static_cast<double>(ell));
    const double* pg = P + g * naxes * 2 * ell;
    bool ok = true;
    for (int64_t s = 0; s < ell; ++s) {
        double left = 0, right = 0;
        for (int a = 0; a < naxes; ++a) {
            const double sc = scales ? scales[a] : 1.0;
            left += sc * pg[a * 2 * ell + s];
            right += sc * pg[a * 2 * ell + ell + s];
        }
        const double y = sw * left * right;
        ok = ok && isfinite(y);
        Yt[s * ldy + g] = y;
    }
    if (!ok) atomicOr(bad, 1);
}

// The same combine for blocks of kCombinePts points: their projections (one
// contiguous block of P) are staged in shared memory, so the loads are
// coalesced and consecutive threads write consecutive columns of a sketch row.
constexpr int kCombinePts = 16;

__global__ void __launch_bounds__(256)
combine_sketch_tiled_kernel(const double* __restrict__ P, int naxes, int64_t ell,
                            const double* __restrict__ scales, const double* __restrict__ w,
                            const int64_t* __restrict__ index, int64_t n, double* __restrict__ Yt,
                            int64_t ldy, int* __restrict__ bad) {
    extern __shared__ double sP[];
    const int64_t width = naxes * 2 * ell;
    const int64_t g0 = static_cast<int64_t>(blockIdx.x) * kCombinePts;
    const int64_t np = min(static_cast<int64_t>(kCombinePts), n - g0);
    for (int64_t i = threadIdx.x; i < np * width; i += blockDim.x) sP[i] = P[g0 * width + i];
    __syncthreads();
    bool ok = true;
    const double inv_sqrt_ell = 1.0 / sqrt(static_cast<double>(ell));
    for (int64_t i = threadIdx.x; i < kCombinePts * ell; i += blockDim.x) {
        const int64_t sidx = i / kCombinePts, pp = i % kCombinePts;
        if (pp >= np) continue;
        const int64_t g = g0 + pp;
        const double* pg = sP + pp * width;
        double left = 0, right = 0;
        for (int a = 0; a < naxes; ++a) {
            const double sc = scales ? scales[a] : 1.0;
            left += sc * pg[a * 2 * ell + sidx];
            right += sc * pg[a * 2 * ell + ell + sidx];
        }
        const double y = sqrt(fabs(w[index[g]])) * inv_sqrt_ell * left * right;
        ok = ok && isfinite(y);
        Yt[sidx * ldy + g] = y;
    }
    if (!ok) atomicOr(bad, 1);
}

// Two-buffer pipeline between the stream s and a side stream: work item i
// runs its producer on side(i), which first waits until s has consumed item
// i - 2 (same buffer); hand_back(i) makes s wait for that producer, and
// consumed(i) marks the point on s after which buffer i % 2 is free again.
// Without `on` everything stays on s.  join() makes s wait for the side
// stream, so stream-ordered frees on s come after its last use.
class StreamPair {
public:
    StreamPair(cudaStream_t s, bool on) : s_(s), on_(on) {
        if (!on_) return;
        ISDF_CUDA(cudaStreamCreateWithFlags(&side_, cudaStreamNonBlocking));
        for (auto& e : ev_) ISDF_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        ISDF_CUDA(cudaEventRecord(ev_[4], s_));          // everything enqueued on s so far
        ISDF_CUDA(cudaStreamWaitEvent(side_, ev_[4], 0));
    }
    cudaStream_t side(int64_t i) {
        if (!on_) return s_;
        if (i >= 2) ISDF_CUDA(cudaStreamWaitEvent(side_, ev_[2 + (i & 1)], 0));
        return side_;
    }
    void hand_back(int64_t i) {
        if (!on_) return;
        ISDF_CUDA(cudaEventRecord(ev_[i & 1], side_));
        ISDF_CUDA(cudaStreamWaitEvent(s_, ev_[i & 1], 0));
    }
    void consumed(int64_t i) {
        if (on_) ISDF_CUDA(cudaEventRecord(ev_[2 + (i & 1)], s_));
    }
    void join() {
        if (!on_ || joined_) return;
        ISDF_CUDA(cudaEventRecord(ev_[4], side_));
        ISDF_CUDA(cudaStreamWaitEvent(s_, ev_[4], 0));
        joined_ = true;
    }
    ~StreamPair() {
        if (!on_) return;
        if (!joined_) {   // an error path: let the side stream drain first
            cudaEventRecord(ev_[4], side_);
            cudaStreamWaitEvent(s_, ev_[4], 0);
        }
        cudaStreamSynchronize(side_);
        for (auto e : ev_) cudaEventDestroy(e);
        cudaStreamDestroy(side_);
    }
    StreamPair(const StreamPair&) = delete;
    StreamPair& operator=(const StreamPair&) = delete;

private:
    cudaStream_t s_, side_ = nullptr;
    bool on_, joined_ = false;
    cudaEvent_t ev_[5] = {};
};

}  // namespace

void sketch_fp64(const Context& c, const double* pts, const KeptPoints& kp, const double* w,
                 const AxisSpec& ax, const double* axis_weights, int64_t ell,
                 const HostFactors& u, const HostFactors& v, double* Yt,
                 int64_t ldy, int64_t chunk, cudaStream_t s) {
    const int naxes = ax.naxes;
    const int64_t d = ax.d;
    const int64_t n = kp.n;
    // W[j][0..ell) = U row j, W[j][ell..2ell) = V row j
    std::vector<double> hw(static_cast<size_t>(d * 2 * ell));
    for (int64_t j = 0; j < d; ++j)
        for (int64_t t = 0; t < ell; ++t) {
            hw[j * 2 * ell + t] = u[j * ell + t];
            hw[j * 2 * ell + ell + t] = v[j * ell + t];
        }
    DeviceBuffer<double> W(hw.size(), s);
    ISDF_CUDA(cudaMemcpyAsync(W.get(), hw.data(), hw.size() * sizeof(double),
                              cudaMemcpyHostToDevice, s));
    DeviceBuffer<double> P(static_cast<size_t>(n * naxes * 2 * ell), s);
    DeviceBuffer<double> sumsq(5, s);
    sumsq.zero(s);
    chunk = std::max<int64_t>(1, std::min(chunk, n));
    bool uniform = true;   // every entry nao wide: one batched GEMM
    for (int a = 0; a < naxes; ++a) uniform = uniform && ax.width[a] == c.nao && ax.offset[a] == a * c.nao;
    // The feature evaluation of chunk i + 1 runs on a second stream while the
    // DMMA GEMM of chunk i runs on s, from two feature buffers: both kernels
    // leave most of an SM idle (the evaluator is latency-bound at 24 warps per
    // SM, the GEMM has 4 warps per block), and one block of each fits an SM.
    const int nbuf = n > chunk ? 2 : 1;
    DeviceBuffer<double> F[2];
    for (int i = 0; i < nbuf; ++i) F[i].reset(static_cast<size_t>(chunk * d), s);
    StreamPair sp(s, nbuf == 2);
    int64_t i = 0;
    for (int64_t g0 = 0; g0 < n; g0 += chunk, ++i) {
        const int64_t b = std::min(chunk, n - g0);
        double* Fi = F[i % nbuf].get();
        cudaStream_t se = sp.side(i);   // waits for the GEMM that last read this buffer
        eval_axis_features<double>(c, pts, kp.index.get() + g0, b, ax, Fi, d,
                                   naxes > 1 ? sumsq.get() : nullptr, nullptr, se);
        sp.hand_back(i);                // s waits for these features
        // per-axis partial projections P[g][a][0..2ell)
        if (uniform) {
            gemm_f64(b, 2 * ell, c.nao, Fi, d, c.nao, W.get(), 2 * ell, c.nao * 2 * ell,
                     P.get() + g0 * naxes * 2 * ell, naxes * 2 * ell, 2 * ell, naxes, false, s);
        } else {
            for (int a = 0; a < naxes; ++a)
                gemm_f64(b, 2 * ell, ax.width[a], Fi + ax.offset[a], d, 0,
                         W.get() + static_cast<int64_t>(ax.offset[a]) * 2 * ell, 2 * ell, 0,
                         P.get() + g0 * naxes * 2 * ell + a * 2 * ell, naxes * 2 * ell, 0, 1, false, s);
        }
        sp.consumed(i);                 // the buffer may be refilled after this GEMM
    }
    sp.join();
    DeviceBuffer<double> dscales;
    if (naxes > 1) {
        double h[5];
        ISDF_CUDA(cudaMemcpyAsync(h, sumsq.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
        ISDF_CUDA(cudaStreamSynchronize(s));
        auto sc = axis_scales_from_sumsq(ax, h, axis_weights, n > 0);
        dscales.reset(sc.size(), s);
        ISDF_CUDA(cudaMemcpyAsync(dscales.get(), sc.data(), sc.size() * sizeof(double),
                                  cudaMemcpyHostToDevice, s));
    }
    DeviceBuffer<int> bad(1, s);
    bad.zero(s);
    ISDF_PROFILE("sketch_combine", s);
    const size_t csmem = static_cast<size_t>(kCombinePts) * naxes * 2 * ell * sizeof(double);
    if (csmem <= 48 * 1024) {
        combine_sketch_tiled_kernel<<<static_cast<unsigned>((n + kCombinePts - 1) / kCombinePts), 256, csmem, s>>>(
            P.get(), naxes, ell, naxes > 1 ? dscales.get() : nullptr, w, kp.index.get(), n, Yt, ldy, bad.get());
    } else {
        combine_sketch_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(
            P.get(), naxes, ell, naxes > 1 ? dscales.get() : nullptr, w, kp.index.get(), n, Yt, ldy,
            bad.get());
    }
    ISDF_LAUNCH_CHECK();
    int hbad = 0;
    ISDF_CUDA(cudaMemcpyAsync(&hbad, bad.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaStreamSynchronize(s));
    if (hbad) fail(kOverflow, "non-finite randomized ID sketch");
}

namespace {

// Squared norm of each feature row (one warp per row).
__global__ void row_sumsq_kernel(const double* __restrict__ F, int64_t rows, int64_t d,
                                 double* __restrict__ out) {
    const int64_t r = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) / 32;
    const int lane = threadIdx.x % 32;
    if (r >= rows) return;
    double acc = 0;
    for (int64_t a = lane; a < d; a += 32) {
        const double x = F[r * d + a];
        acc += x * x;
    }
    acc = warp_allsum(acc);
    if (lane == 0) out[r] = acc;
}

__global__ void flag_screen_kernel(const double* __restrict__ q, int64_t n, double threshold,
                                   char* __restrict__ keep, int* __restrict__ bad) {
    const int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g >= n) return;
    const double v = q[g];
    if (!isfinite(v)) atomicOr(bad, 1);
    keep[g] = v > threshold;
}

// Y[s][i] = sqrt(m_g)/sqrt(ell) (f.u_s)(f.v_s) for the screened points g =
// pos[i] (f = phi_g, or phi_g / |phi_g| in the normalized form); also the
// surviving grid indices.
__global__ void combine_density_kernel(const double* __restrict__ P, const double* __restrict__ q,
                                       const int64_t* __restrict__ pos, int64_t n2, int64_t ell,
                                       const double* __restrict__ importance,
                                       const int64_t* __restrict__ index, bool normalized,
                                       double* __restrict__ Yt, int64_t* __restrict__ index2,
                                       int* __restrict__ bad) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n2) return;
    const int64_t g = pos[i];
    const int64_t gi = index[g];
    index2[i] = gi;
    const double sw = sqrt(importance[gi]);
    const double inv = normalized ? 1.0 / sqrt(q[g]) : 1.0;
    const double scaling = 1.0 / sqrt(static_cast<double>(ell));
    const double* pg = P + g * 2 * ell;
    bool ok = true;
    for (int64_t s = 0; s < ell; ++s) {
        const double y = scaling * sw * (inv * pg[s]) * (inv * pg[ell + s]);
        ok = ok && isfinite(y);
        Yt[s * n2 + i] = y;
    }
    if (!ok) atomicOr(bad, 1);
}

}  // namespace

// AO-density Khatri-Rao sketch in FP64 (anchor_select_randomized_id.cpp:231-309):
// features are the AO values of the kept points; points whose squared AO norm
// is <= threshold leave the candidate set (kp is compacted to the survivors,
// in order), and column g of the sketch is sqrt(m_g)/sqrt(ell) (f.u_s)(f.v_s)
// with f = phi_g, or phi_g/|phi_g| in the normalized form.  Returns Yt
// (ell x kp.n, leading dimension kp.n).
DeviceBuffer<double> sketch_density_fp64(const Context& c, const double* pts, KeptPoints& kp,
                                         const double* importance, int64_t ell,
                                         const HostFactors& u, const HostFactors& v,
                                         bool normalized, double threshold, int64_t chunk,
                                         cudaStream_t s) {
    const int nao = c.nao;
    const int64_t d = nao;
    const int64_t n = kp.n;
    const int32_t ao_axis = 0;
    const AxisSpec ax = make_axis_spec(c, &ao_axis, 1);
    std::vector<double> hw(static_cast<size_t>(d * 2 * ell));
    for (int64_t j = 0; j < d; ++j)
        for (int64_t t = 0; t < ell; ++t) {
            hw[j * 2 * ell + t] = u[j * ell + t];
            hw[j * 2 * ell + ell + t] = v[j * ell + t];
        }
    DeviceBuffer<double> W(hw.size(), s);
    ISDF_CUDA(cudaMemcpyAsync(W.get(), hw.data(), hw.size() * sizeof(double), cudaMemcpyHostToDevice, s));
    DeviceBuffer<double> P(static_cast<size_t>(std::max<int64_t>(n, 1) * 2 * ell), s), q(std::max<int64_t>(n, 1), s);
    chunk = std::max<int64_t>(1, std::min(chunk, n));
    DeviceBuffer<double> F(static_cast<size_t>(chunk * d), s);
    for (int64_t g0 = 0; g0 < n; g0 += chunk) {
        const int64_t b = std::min(chunk, n - g0);
        eval_axis_features<double>(c, pts, kp.index.get() + g0, b, ax, F.get(), d, nullptr, nullptr, s);
        gemm_f64(b, 2 * ell, nao, F.get(), d, 0, W.get(), 2 * ell, 0, P.get() + g0 * 2 * ell, 2 * ell, 0, 1,
                 false, s);
        row_sumsq_kernel<<<static_cast<unsigned>((b * 32 + 255) / 256), 256, 0, s>>>(F.get(), b, d,
                                                                                     q.get() + g0);
        ISDF_LAUNCH_CHECK();
    }
    // screening: the surviving positions, in order
    DeviceBuffer<char> keep(std::max<int64_t>(n, 1), s);
    DeviceBuffer<int> bad(1, s);
    DeviceBuffer<int64_t> pos(std::max<int64_t>(n, 1), s), count(1, s);
    bad.zero(s);
    flag_screen_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(q.get(), n, threshold, keep.get(),
                                                                            bad.get());
    ISDF_LAUNCH_CHECK();
    size_t tmp_bytes = 0;
    thrust::counting_iterator<int64_t> it(0);
    ISDF_CUDA(cub::DeviceSelect::Flagged(nullptr, tmp_bytes, it, keep.get(), pos.get(), count.get(), n, s));
    DeviceBuffer<char> tmp(tmp_bytes, s);
    ISDF_CUDA(cub::DeviceSelect::Flagged(tmp.get(), tmp_bytes, it, keep.get(), pos.get(), count.get(), n, s));
    count_launches(2);
    int hbad = 0;
    int64_t n2 = 0;
    ISDF_CUDA(cudaMemcpyAsync(&hbad, bad.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaMemcpyAsync(&n2, count.get(), sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaStreamSynchronize(s));
    if (hbad) fail(kOverflow, "non-finite AO squared norm");
    DeviceBuffer<double> Yt(static_cast<size_t>(std::max<int64_t>(n2, 1) * ell), s);
    KeptPoints kp2;
    kp2.index.reset(std::max<int64_t>(n2, 1), s);
    kp2.n = n2;
    if (n2 > 0) {
        bad.zero(s);
        ISDF_PROFILE("sketch_combine", s);
        combine_density_kernel<<<static_cast<unsigned>((n2 + 255) / 256), 256, 0, s>>>(
            P.get(), q.get(), pos.get(), n2, ell, importance, kp.index.get(), normalized, Yt.get(),
            kp2.index.get(), bad.get());
        ISDF_LAUNCH_CHECK();
        ISDF_CUDA(cudaMemcpyAsync(&hbad, bad.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
        ISDF_CUDA(cudaStreamSynchronize(s));
        if (hbad) fail(kOverflow, "non-finite randomized ID sketch");
    }
    kp = std::move(kp2);
    return Yt;
}

// ------------------------------------------------------------------------------
// mixed-precision sketch: fused FP32 AO evaluation + split-BF16 tensor-core
// projection, FP64 combination with per-column error bounds
// ------------------------------------------------------------------------------
namespace {

// Relative accuracy of a split-BF16 (hi*hi + hi*lo + lo*hi) dot product of
// FP32 features with FP64 weights, with a 10x margin over its ~2^-16
// representation error: |d(f.u)| <= kSplitBf16Bound * |f| * |u_scale|.
constexpr double kSplitBf16Bound = 1.5e-4;

// Per-axis absolute column sums A[a][t] = sum_mu |f[(a*nao + mu)*ell + t]| of
// a sketch factor (rows j = a*nao + mu, ell columns).
std::vector<double> factor_abs_sums(const HostFactors& f, int naxes, int64_t nao, int64_t ell) {
    std::vector<double> out(static_cast<size_t>(naxes) * ell, 0.0);
    for (int a = 0; a < naxes; ++a)
        for (int64_t mu = 0; mu < nao; ++mu) {
            const double* row = f.data() + (a * nao + mu) * ell;
            double* o = out.data() + a * ell;
            for (int64_t t = 0; t < ell; ++t) o[t] += std::fabs(row[t]);
        }
    return out;
}

// Bound on how far any projection f_g . u_s or f_g . v_s (axis entries scaled
// by sc) moves when every feature entry is off by at most eps: the screening
// of the fused kernel's FP32 evaluation (kScreenFp32 per value or gradient).
double projection_abs_error(const std::vector<double>& au, const std::vector<double>& av,
                            const std::vector<double>& sc, int64_t ell, double eps) {
    double worst = 0.0;
    for (int64_t t = 0; t < ell; ++t) {
        double su = 0.0, sv = 0.0;
        for (size_t a = 0; a < sc.size(); ++a) {
            su += sc[a] * au[a * ell + t];
            sv += sc[a] * av[a * ell + t];
        }
        worst = std::max(worst, std::max(su, sv));
    }
    return eps * worst;
}

// Yt[s][g] = sw/sqrt(ell) L_s R_s from the FP32 per-axis partials, and the
// absolute error bound of the column's norm: with e = k|f_g| + tabs bounding
// the error of each partial (split-BF16 products, and tabs for the screened
// pieces),
//   delta_g = sw/sqrt(ell) * e * sqrt(sum_s (|L_s| + |R_s| + e)^2)
__global__ void combine_mixed_kernel(const float* __restrict__ P, const float* __restrict__ psq,
                                     int naxes, const int* __restrict__ comp, int64_t ell,
                                     const double* __restrict__ scales, const double* __restrict__ w,
                                     const int64_t* __restrict__ index, int64_t n,
                                     double* __restrict__ Yt, int64_t ldy, double* __restrict__ delta,
                                     int* __restrict__ bad, double tabs) {
    const int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g >= n) return;
    const double sw = sqrt(fabs(w[index[g]])) / sqrt(static_cast<double>(ell));
    const float* pg = P + g;   // column-major, leading dimension n
    double f2 = 0;
    for (int a = 0; a < naxes; ++a) {
        const double sc = scales ? scales[a] : 1.0;
        f2 += sc * sc * static_cast<double>(psq[g * 4 + comp[a]]);
    }
    const double fn = sqrt(f2);
    const double e_abs = kSplitBf16Bound * fn + tabs;
    double bound2 = 0;
    bool ok = true;
    for (int64_t s = 0; s < ell; ++s) {
        double left = 0, right = 0;
        for (int a = 0; a < naxes; ++a) {
            const double sc = scales ? scales[a] : 1.0;
            left += sc * static_cast<double>(pg[(a * 2 * ell + s) * n]);
            right += sc * static_cast<double>(pg[(a * 2 * ell + ell + s) * n]);
        }
        const double y = sw * left * right;
        ok = ok && isfinite(y);
        Yt[s * ldy + g] = y;
        const double e = fabs(left) + fabs(right) + e_abs;
        bound2 += e * e;
    }
    delta[g] = sw * e_abs * sqrt(bound2);
    if (!ok) atomicOr(bad, 1);
}

// WT[t*d + j] = u[j*ell + t] (t < ell), v[j*ell + t - ell] (t >= ell): the
// projection weights row-major for the FP64 re-verification.
__global__ void factors_transpose_kernel(const double* __restrict__ u, const double* __restrict__ v,
                                         int64_t d, int64_t ell, double* __restrict__ WT) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= d * 2 * ell) return;
    const int64_t t = i / d, j = i % d;
    WT[i] = t < ell ? u[j * ell + t] : v[j * ell + t - ell];
}

}  // namespace

MixedSketch sketch_mixed(const Context& c, const double* pts, const KeptPoints& kp, const double* w,
                         const AxisSpec& ax, const double* axis_weights, int64_t ell,
                         const HostFactors& u, const HostFactors& v, double* Yt,
                         int64_t ldy, cudaStream_t s, RetainedAo* keep) {
    MixedSketch ms;
    const int nao = c.nao;
    const int naxes = ax.naxes;
    const int64_t d = static_cast<int64_t>(naxes) * nao;
    const int64_t n = kp.n;
    const int nout = static_cast<int>(2 * ell);
    std::vector<int> comps(ax.comp, ax.comp + naxes);
    ProjectPlan plan;
    DeviceBuffer<double> du(static_cast<size_t>(d * ell), s), dv(static_cast<size_t>(d * ell), s);
    ms.WT.reset(static_cast<size_t>(d * nout), s);
    {
        ISDF_PROFILE("phase:sketch_plan", s);
        ISDF_CUDA(cudaMemcpyAsync(du.get(), u.data(), u.size() * sizeof(double), cudaMemcpyHostToDevice, s));
        ISDF_CUDA(cudaMemcpyAsync(dv.get(), v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice, s));
        // feature j = a*nao + mu feeds column s of u (left) and ell + s of v (right)
        const WSource srcs[2] = {{du.get(), static_cast<int64_t>(nao) * ell, ell, 1, static_cast<int>(ell), 0},
                                 {dv.get(), static_cast<int64_t>(nao) * ell, ell, 1, static_cast<int>(ell),
                                  static_cast<int>(ell)}};
        plan = make_project_plan(c, comps, nout, srcs, 2, s);
        factors_transpose_kernel<<<static_cast<unsigned>((d * nout + 255) / 256), 256, 0, s>>>(
            du.get(), dv.get(), d, ell, ms.WT.get());
        ISDF_LAUNCH_CHECK();
    }
    DeviceBuffer<float> P_own, psq(static_cast<size_t>(n * 4), s);
    float* P = nullptr;
    DeviceBuffer<double> sumsq(4, s);
    DeviceBuffer<int> err(1, s), dcomp(naxes, s);
    psq.zero(s);
    sumsq.zero(s);
    err.zero(s);
    // the AO value tiles of the first plain-AO axis entry can stay in HBM for the fit
    int store_axis = -1;
    for (int a = 0; a < naxes && store_axis < 0; ++a)
        if (comps[a] == 0) store_axis = a;
    const size_t p_bytes = (static_cast<size_t>(n) * naxes * nout * sizeof(float) + 255) / 256 * 256;
    uint8_t* tiles = nullptr;
    uint8_t* tiles_r = nullptr;
    uint8_t* chunk_zero = nullptr;
    if (keep) {
        // tiles (when they fit in free memory), their screening flags and the
        // projections in the workspace
        size_t tile_bytes = store_axis >= 0 ? stored_tile_bytes(c, n) + stored_remainder_bytes(c, n) +
                                                  stored_flag_bytes(c, n)
                                            : 0;
        if (tile_bytes + p_bytes > c.ws_bytes && tile_bytes > 0) {
            size_t free_b = 0, total_b = 0;
            ISDF_CUDA(cudaMemGetInfo(&free_b, &total_b));
            if (tile_bytes + p_bytes - c.ws_bytes > free_b / 2) {
                tile_bytes = 0;
                store_axis = -1;
            }
        }
        uint8_t* base = c.workspace(tile_bytes + p_bytes);
        if (store_axis >= 0) {
            tiles = base;
            tiles_r = base + stored_tile_bytes(c, n);
            chunk_zero = tiles_r + stored_remainder_bytes(c, n);
        }
        P = reinterpret_cast<float*>(base + tile_bytes);
    } else {
        P_own.reset(static_cast<size_t>(n) * naxes * nout, s);
        P = P_own.get();
    }
    // column-major projections P[a*nout + j][g] (coalesced for the combine pass)
    project_tc(c, plan, pts, kp.index.get(), n, w, P, 1, n, sumsq.get(), psq.get(),
               err.get(), s, tiles, std::max(store_axis, 0), tiles_r, chunk_zero);
    // host work under the kernel: the factors' absolute column sums for the
    // screening term of the error bounds
    const std::vector<double> au = factor_abs_sums(u, naxes, nao, ell), av = factor_abs_sums(v, naxes, nao, ell);
    double h[4] = {0, 0, 0, 0};
    int herr = 0;
    ISDF_CUDA(cudaMemcpyAsync(h, sumsq.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaMemcpyAsync(&herr, err.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaStreamSynchronize(s));
    if (herr) fail(kRuntime, "tensor-core sketch pipeline timed out (error flags " + std::to_string(herr) + ")");
    std::vector<double> sc(naxes, 1.0);
    if (naxes > 1) sc = axis_scales_from_sumsq(ax, h, axis_weights, n > 0);
    ms.scales.reset(naxes, s);
    ms.delta.reset(n, s);
    ISDF_CUDA(cudaMemcpyAsync(ms.scales.get(), sc.data(), naxes * sizeof(double), cudaMemcpyHostToDevice, s));
    ISDF_CUDA(cudaMemcpyAsync(dcomp.get(), comps.data(), naxes * sizeof(int), cudaMemcpyHostToDevice, s));
    DeviceBuffer<int> bad(1, s);
    bad.zero(s);
    {
        ISDF_PROFILE("sketch_combine", s);
        combine_mixed_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(
            P, psq.get(), naxes, dcomp.get(), ell, naxes > 1 ? ms.scales.get() : nullptr, w,
            kp.index.get(), n, Yt, ldy, ms.delta.get(), bad.get(),
            projection_abs_error(au, av, sc, ell, kScreenFp32));
        ISDF_LAUNCH_CHECK();
    }
    int hbad = 0;
    ISDF_CUDA(cudaMemcpyAsync(&hbad, bad.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaStreamSynchronize(s));   // host staging vectors go out of scope
    if (hbad) fail(kOverflow, "non-finite randomized ID sketch");
    ms.source.ctx = &c;
    ms.source.naxes = naxes;
    for (int a = 0; a < naxes; ++a) ms.source.comp[a] = comps[a];
    ms.source.scales = ms.scales.get();
    ms.source.WT = ms.WT.get();
    ms.source.pts = pts;
    ms.source.index = kp.index.get();
    ms.source.w = w;
    ms.source.ell = ell;
    ms.source.delta = ms.delta.get();
    if (keep && store_axis >= 0) {
        keep->tiles = tiles;
        keep->tiles_r = tiles_r;
        keep->chunk_zero = chunk_zero;
        keep->psq = std::move(psq);
        keep->valid = true;
    }
    return ms;
}

// ------------------------------------------------------------------------------
// rand_sketch (quadrature) driver
// ------------------------------------------------------------------------------
SketchSetup sketch_setup(const Context& c, const SelectOptions& o, int64_t n, cudaStream_t s) {
    if (!std::isfinite(o.tolerance) || o.tolerance < 0 || o.batch_size <= 0 ||
        o.oversampling <= 0 || (!o.max_rank && o.sketch_size <= o.oversampling))
        fail(kInvalid, "invalid randomized ID grid, tolerance, batch, sketch or rank/oversampling");
    SketchSetup su;
    // the host MO pointer only validates here; the device copy is made below
    su.ax = make_axis_spec(c, o.axes.data(), static_cast<int>(o.axes.size()), o.mo_host, o.nocc);
    su.ax.mo = nullptr;
    su.d = su.ax.d;
    if (o.max_rank > std::numeric_limits<int64_t>::max() - o.oversampling)
        fail(kOverflow, "randomized ID rank + oversampling overflows size_t");
    const int64_t requested = o.max_rank ? o.max_rank + o.oversampling : o.sketch_size;
    su.physical_rank = su.d * (su.d + 1) / 2;
    if (n == 0) return su;
    const int64_t physical_limit = su.physical_rank + o.oversampling;
    const int64_t backend_limit = std::numeric_limits<int64_t>::max() / n;
    su.ell = requested <= backend_limit ? requested : std::min({requested, physical_limit, backend_limit});
    if (su.ell <= o.oversampling ||
        (o.max_rank && std::min(o.max_rank, su.physical_rank) > su.ell - o.oversampling))
        fail(kInvalid, "randomized ID sketch/rank exceeds the ILP64 QRCP backend limit for this "
                       "grid; reduce the sketch/rank or use a tiled QRCP backend");
    if (o.max_rank > std::min(n, su.physical_rank))
        fail(kInvalid, "requested anchor_rank exceeds eligible candidates or physical pair rank");
    // the mixed form needs the tensor-core shape and room for one point's AO
    // components in shared memory for the FP64 re-verification of candidates
    su.mixed = o.precision == 1 && project_tc_supported(su.ax.naxes, static_cast<int>(2 * su.ell)) &&
               su.ell <= 64 && c.nao <= kMaxVerifiedNao && !su.ax.has_occ;
    if (su.ax.has_occ) {
        // occupied-orbital features are FP64 only: the FP64 form runs
        su.mo.reset(static_cast<size_t>(c.nao) * c.nao, s);
        ISDF_CUDA(cudaMemcpyAsync(su.mo.get(), o.mo_host, static_cast<size_t>(c.nao) * c.nao * sizeof(double),
                                  cudaMemcpyHostToDevice, s));
        su.ax.mo = su.mo.get();
    }
    return su;
}

SketchRank sketch_rank(const SketchQR& qr, int64_t ell, int64_t n, const SelectOptions& o,
                       int64_t physical_rank) {
    SketchRank r;
    const int64_t steps = std::min(ell, n);
    r.tails.assign(steps + 1, 0.0);
    double diag_max = 0;
    for (int64_t i = steps; i-- > 0;) {
        r.tails[i] = std::hypot(r.tails[i + 1], std::sqrt(qr.energy[i]));
        diag_max = std::max(diag_max, qr.diag[i]);
    }
    if (!std::isfinite(r.tails[0]) || !std::isfinite(diag_max))
        fail(kOverflow, "non-finite randomized ID QR residual");
    const double norm = r.tails[0];
    const double floor = std::numeric_limits<double>::epsilon() *
                         static_cast<double>(std::max(ell, n)) * diag_max;
    r.numerical_rank = steps;
    for (int64_t i = 0; i < steps; ++i)
        if (qr.diag[i] <= floor) { r.numerical_rank = i; break; }
    r.cap = std::min({o.max_rank ? o.max_rank : ell - o.oversampling, ell - o.oversampling, steps,
                      physical_rank, r.numerical_rank});
    if (o.max_rank && r.numerical_rank < o.max_rank)
        fail(kInvalid, "requested anchor_rank exceeds the numerical rank of the randomized sketch");
    r.rank = o.max_rank ? o.max_rank : r.cap;
    if (!o.max_rank)
        for (int64_t i = 0; i <= r.cap; ++i)
            if (r.tails[i] <= o.tolerance * norm) { r.rank = i; break; }
    r.relative_tail = norm ? r.tails[r.rank] / norm : 0.0;
    for (int64_t i = 0; i < r.rank; ++i)
        if (qr.jpvt[i] < 0 || qr.jpvt[i] >= n) fail(kRuntime, "randomized ID QRCP returned invalid pivot");
    return r;
}

namespace {

void fill_diag(SketchDiagnostics* d, int64_t ell, const SketchRank& r, const SketchQR& qr) {
    if (!d) return;
    d->ell = ell;
    d->numerical_rank = r.numerical_rank;
    d->cap = r.cap;
    d->rank = r.rank;
    d->relative_tail = r.relative_tail;
    d->diag = qr.diag;
    d->reverified = qr.reverified;
    d->tails = r.tails;
}

}  // namespace

std::vector<int64_t> select_rand_sketch(const Context& c, const double* pts, const double* w,
                                        int64_t ng, const SelectOptions& o, cudaStream_t s,
                                        SketchDiagnostics* diag_out, RetainedAo* keep) {
    sketch_setup(c, o, 0);   // option checks before any device work
    const bool density = o.algorithm == 4 || o.algorithm == 5;
    if (density) {
        if (!o.importance) fail(kInvalid, "point_importance must have shape (ngrid,)");
        if (!std::isfinite(o.ao_threshold) || o.ao_threshold < 0)
            fail(kInvalid, "AO screening threshold must be finite and nonnegative");
        if (o.axes.size() != 1 || o.axes[0] != 0)
            fail(kInvalid, "density Khatri-Rao sketches with non-AO axis features are NYI");
        if (o.precision != 0)
            fail(kNotImplemented, "density Khatri-Rao sketches are implemented in the FP64 form only");
    }
    ISDF_PROFILE("phase:select", s);
    // The Gaussian factors depend on (d, ell, seed) only, and ell on the kept
    // count only through the ILP64 limit: when the requested ell is within the
    // limit for the whole grid it is the final one, so the factors are drawn on
    // a host thread while the device compacts the points.
    HostFactors u, v;
    const int64_t d_pre = static_cast<int64_t>(o.axes.size()) * c.nao;
    const int64_t ell_req = o.max_rank ? o.max_rank + o.oversampling : o.sketch_size;
    int64_t ell_pre = -1;
    std::future<void> pre;
    if (ng > 0 && ell_req > o.oversampling && ell_req <= std::numeric_limits<int64_t>::max() / ng &&
        d_pre > 0 && d_pre <= (int64_t(1) << 40) / ell_req) {
        ell_pre = ell_req;
        pre = std::async(std::launch::async, [&u, &v, d_pre, ell_pre, &o] {
            sketch_factors(d_pre, ell_pre, o.seed, u, v);
        });
    }
    KeptPoints kp;
    {
        ISDF_PROFILE("phase:compact", s);
        // the sketch evaluates the kept points in spatial order (the pivots
        // are mapped back through the index; a kept mixed fit restores Theta's
        // ascending column order)
        kp = compact_points(pts, w, ng, s, density ? o.importance : nullptr, !density);
    }
    int64_t n = kp.n;
    if (n == 0) {
        if (density && o.max_rank) fail(kInvalid, "requested anchor_rank exceeds eligible candidates");
        return {};
    }
    const SketchSetup su = sketch_setup(c, o, n, s);
    const AxisSpec& ax = su.ax;
    const int64_t ell = su.ell;
    {
        ISDF_PROFILE("phase:sketch_factors", s);
        if (pre.valid()) pre.get();
        if (ell_pre != ell || d_pre != su.d) sketch_factors(su.d, ell, o.seed, u, v);
    }
    const double* aw = o.axis_weights.empty() ? nullptr : o.axis_weights.data();
    SketchQR qr;
    if (density) {
        const int64_t candidates = n;
        const int64_t chunk = std::max<int64_t>(1024, std::min<int64_t>(n, (int64_t(1) << 28) / su.d));
        DeviceBuffer<double> Yd = sketch_density_fp64(c, pts, kp, o.importance, ell, u, v, o.algorithm == 5,
                                                      o.ao_threshold, chunk, s);
        n = kp.n;
        if (o.max_rank > std::min(n, su.physical_rank))
            fail(kInvalid, "requested anchor_rank exceeds eligible candidates or physical pair rank");
        if (o.debug)
            std::fprintf(stderr,
                         "[density sketch screening] candidates=%lld eligible=%lld screened_ao=%lld "
                         "ao_norm2_threshold=%g\n",
                         static_cast<long long>(candidates), static_cast<long long>(n),
                         static_cast<long long>(candidates - n), o.ao_threshold);
        if (n == 0) return {};
        ISDF_PROFILE("phase:qrcp", s);
        qr = qrcp_sketch(Yd.get(), n, ell, n, s);
        const SketchRank r = sketch_rank(qr, ell, n, o, su.physical_rank);
        std::vector<int64_t> selected(r.rank);
        for (int64_t i = 0; i < r.rank; ++i)
            ISDF_CUDA(cudaMemcpyAsync(&selected[i], kp.index.get() + qr.jpvt[i], sizeof(int64_t),
                                      cudaMemcpyDeviceToHost, s));
        ISDF_CUDA(cudaStreamSynchronize(s));
        fill_diag(diag_out, ell, r, qr);
        return selected;
    }
    // an even row stride keeps every row 16-byte aligned for the QR update's
    // paired copies (the padding column is never read)
    const int64_t ldy = n + (n & 1);
    DeviceBuffer<double> Yt(static_cast<size_t>(ell * ldy), s);
    if (su.mixed) {
        MixedSketch ms = sketch_mixed(c, pts, kp, w, ax, aw, ell, u, v, Yt.get(), ldy, s, keep);
        ISDF_PROFILE("phase:qrcp", s);
        qr = qrcp_sketch(Yt.get(), ldy, ell, n, s, &ms.source);
    } else {
        const int64_t chunk = std::max<int64_t>(1024, std::min<int64_t>(n, (int64_t(1) << 28) / su.d));
        sketch_fp64(c, pts, kp, w, ax, aw, ell, u, v, Yt.get(), ldy, chunk, s);
        qr = qrcp_sketch(Yt.get(), ldy, ell, n, s);
    }
    const SketchRank r = sketch_rank(qr, ell, n, o, su.physical_rank);
    // original grid ids of the pivots (a gather of `rank` entries of the kept index)
    std::vector<int64_t> selected(r.rank);
    for (int64_t i = 0; i < r.rank; ++i)
        ISDF_CUDA(cudaMemcpyAsync(&selected[i], kp.index.get() + qr.jpvt[i], sizeof(int64_t),
                                  cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaStreamSynchronize(s));
    fill_diag(diag_out, ell, r, qr);
    if (diag_out) diag_out->precision_used = su.mixed ? 1 : 0;
    if (keep && keep->valid) keep->kp = std::move(kp);
    return selected;
}

// ------------------------------------------------------------------------------
// grid-sharded rand_sketch: per-shard projection, global scales, per-shard
// sketch columns, then the pivoted QR of the gathered sketch on every rank
// ------------------------------------------------------------------------------
void sketch_shard_project(const Context& c, const double* pts, const double* w, int64_t ng,
                          const SelectOptions& o, int64_t n_total, SketchShard& st, cudaStream_t s) {
    st.o = o;
    st.pts = pts;
    st.w = w;
    st.ng = ng;
    st.kp = compact_points(pts, w, ng, s);
    st.su = sketch_setup(c, o, std::max<int64_t>(n_total, 1), s);
    if (st.su.ax.has_occ) fail(kInvalid, "grid-sharded selection supports the ao, dx, dy, dz axes");
    const int64_t n = st.kp.n, ell = st.su.ell, d = st.su.d;
    const int naxes = st.su.ax.naxes, nout = static_cast<int>(2 * ell);
    sketch_factors(d, ell, o.seed, st.u, st.v);
    for (double& x : st.sumsq) x = 0.0;
    if (n == 0) return;
    DeviceBuffer<double> sumsq(4, s);
    sumsq.zero(s);
    if (st.su.mixed) {
        std::vector<int> comps(st.su.ax.comp, st.su.ax.comp + naxes);
        DeviceBuffer<double> du(st.u.size(), s), dv(st.v.size(), s);
        ISDF_CUDA(cudaMemcpyAsync(du.get(), st.u.data(), st.u.size() * sizeof(double), cudaMemcpyHostToDevice, s));
        ISDF_CUDA(cudaMemcpyAsync(dv.get(), st.v.data(), st.v.size() * sizeof(double), cudaMemcpyHostToDevice, s));
        const WSource srcs[2] = {{du.get(), static_cast<int64_t>(c.nao) * ell, ell, 1, static_cast<int>(ell), 0},
                                 {dv.get(), static_cast<int64_t>(c.nao) * ell, ell, 1, static_cast<int>(ell),
                                  static_cast<int>(ell)}};
        ProjectPlan plan = make_project_plan(c, comps, nout, srcs, 2, s);
        st.Pf.reset(static_cast<size_t>(n) * naxes * nout, s);
        st.psq.reset(static_cast<size_t>(n) * 4, s);
        st.psq.zero(s);
        DeviceBuffer<int> err(1, s);
        err.zero(s);
        project_tc(c, plan, pts, st.kp.index.get(), n, w, st.Pf.get(), 1, n, sumsq.get(), st.psq.get(),
                   err.get(), s);
        int herr = 0;
        ISDF_CUDA(cudaMemcpyAsync(&herr, err.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
        ISDF_CUDA(cudaStreamSynchronize(s));
        if (herr) fail(kRuntime, "tensor-core sketch pipeline timed out (error flags " + std::to_string(herr) + ")");
    } else {
        std::vector<double> hw(static_cast<size_t>(d * nout));
        for (int64_t j = 0; j < d; ++j)
            for (int64_t t = 0; t < ell; ++t) {
                hw[j * nout + t] = st.u[j * ell + t];
                hw[j * nout + ell + t] = st.v[j * ell + t];
            }
        DeviceBuffer<double> W(hw.size(), s);
        ISDF_CUDA(cudaMemcpyAsync(W.get(), hw.data(), hw.size() * sizeof(double), cudaMemcpyHostToDevice, s));
        st.Pd.reset(static_cast<size_t>(n) * naxes * nout, s);
        const int64_t chunk = std::max<int64_t>(1, std::min<int64_t>(n, std::max<int64_t>(1024, (int64_t(1) << 28) / d)));
        DeviceBuffer<double> F(static_cast<size_t>(chunk * d), s);
        for (int64_t g0 = 0; g0 < n; g0 += chunk) {
            const int64_t b = std::min(chunk, n - g0);
            eval_axis_features<double>(c, pts, st.kp.index.get() + g0, b, st.su.ax, F.get(), d, sumsq.get(),
                                       nullptr, s);
            gemm_f64(b, nout, c.nao, F.get(), d, c.nao, W.get(), nout, static_cast<int64_t>(c.nao) * nout,
                     st.Pd.get() + g0 * naxes * nout, naxes * nout, nout, naxes, false, s);
        }
        ISDF_CUDA(cudaStreamSynchronize(s));   // host weight image goes out of scope
    }
    ISDF_CUDA(cudaMemcpyAsync(st.sumsq, sumsq.get(), sizeof(st.sumsq), cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaStreamSynchronize(s));
}

void sketch_shard_combine(const Context& c, SketchShard& st, const double* sumsq_global, double* Yt,
                          double* delta, int64_t* kept_out, double* kept_xyz, double* kept_w,
                          std::vector<double>& scales, cudaStream_t s) {
    const int64_t n = st.kp.n, ell = st.su.ell;
    const int naxes = st.su.ax.naxes;
    const double* aw = st.o.axis_weights.empty() ? nullptr : st.o.axis_weights.data();
    scales.assign(naxes, 1.0);
    // every shard derives the same scales from the same global sums
    if (naxes > 1) scales = axis_scales_from_sumsq(st.su.ax, sumsq_global, aw, true);
    if (n == 0) return;
    DeviceBuffer<double> dsc(naxes, s);
    ISDF_CUDA(cudaMemcpyAsync(dsc.get(), scales.data(), naxes * sizeof(double), cudaMemcpyHostToDevice, s));
    DeviceBuffer<int> bad(1, s);
    bad.zero(s);
    if (st.su.mixed) {
        require(delta != nullptr, "the mixed sketch needs its per-column error bounds");
        DeviceBuffer<int> dcomp(naxes, s);
        ISDF_CUDA(cudaMemcpyAsync(dcomp.get(), st.su.ax.comp, naxes * sizeof(int), cudaMemcpyHostToDevice, s));
        ISDF_PROFILE("sketch_combine", s);
        combine_mixed_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(
            st.Pf.get(), st.psq.get(), naxes, dcomp.get(), ell, naxes > 1 ? dsc.get() : nullptr, st.w,
            st.kp.index.get(), n, Yt, n, delta, bad.get(),
            projection_abs_error(factor_abs_sums(st.u, naxes, c.nao, ell), factor_abs_sums(st.v, naxes, c.nao, ell),
                                 scales, ell, kScreenFp32));
        ISDF_LAUNCH_CHECK();
        ISDF_CUDA(cudaStreamSynchronize(s));
    } else {
        ISDF_PROFILE("sketch_combine", s);
        combine_sketch_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(
            st.Pd.get(), naxes, ell, naxes > 1 ? dsc.get() : nullptr, st.w, st.kp.index.get(), n, Yt, n,
            bad.get());
        ISDF_LAUNCH_CHECK();
        if (delta) ISDF_CUDA(cudaMemsetAsync(delta, 0, n * sizeof(double), s));
    }
    if (kept_out)
        ISDF_CUDA(cudaMemcpyAsync(kept_out, st.kp.index.get(), n * sizeof(int64_t), cudaMemcpyDeviceToDevice, s));
    if (kept_xyz && kept_w) gather_points(st.pts, st.w, st.kp.index.get(), n, st.ng, kept_xyz, kept_w, s);
    int hbad = 0;
    ISDF_CUDA(cudaMemcpyAsync(&hbad, bad.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaStreamSynchronize(s));
    if (hbad) fail(kOverflow, "non-finite randomized ID sketch");
}

std::unique_ptr<SketchQrShard> make_sketch_qr_shard(const Context& c, const SelectOptions& o, double* Yt,
                                                    int64_t n_local, int64_t n_total, const double* kept_xyz,
                                                    const double* kept_w, double* delta,
                                                    const std::vector<double>& scales, int64_t pos_offset,
                                                    cudaStream_t s) {
    require(n_local >= 0 && n_total >= n_local && pos_offset >= 0 && pos_offset + n_local <= n_total,
            "invalid distributed sketch QR shard sizes");
    auto sh = std::make_unique<SketchQrShard>();
    sh->n_total = n_total;
    sh->su = sketch_setup(c, o, std::max<int64_t>(n_total, 1), s);
    const SketchSetup& su = sh->su;
    if (su.ax.has_occ) fail(kInvalid, "grid-sharded selection supports the ao, dx, dy, dz axes");
    require(static_cast<int>(scales.size()) == su.ax.naxes, "one scale per axis entry is required");
    const ExactSketchSource* ex = nullptr;
    if (delta && su.mixed && n_local > 0) {
        HostFactors u, v;
        sketch_factors(su.d, su.ell, o.seed, u, v);
        const int64_t d = su.d, nout = 2 * su.ell;
        std::vector<double> hwt(static_cast<size_t>(d * nout));
        for (int64_t jj = 0; jj < d; ++jj)
            for (int64_t t = 0; t < su.ell; ++t) {
                hwt[t * d + jj] = u[jj * su.ell + t];
                hwt[(su.ell + t) * d + jj] = v[jj * su.ell + t];
            }
        sh->WT.reset(hwt.size(), s);
        sh->scales.reset(scales.size(), s);
        sh->index.reset(n_local, s);
        ISDF_CUDA(cudaMemcpyAsync(sh->WT.get(), hwt.data(), hwt.size() * sizeof(double), cudaMemcpyHostToDevice, s));
        ISDF_CUDA(cudaMemcpyAsync(sh->scales.get(), scales.data(), scales.size() * sizeof(double),
                                  cudaMemcpyHostToDevice, s));
        iota_i64(sh->index.get(), n_local, s);
        ExactSketchSource& src = sh->src;
        src.ctx = &c;
        src.naxes = su.ax.naxes;
        for (int a = 0; a < su.ax.naxes; ++a) src.comp[a] = su.ax.comp[a];
        src.scales = sh->scales.get();
        src.WT = sh->WT.get();
        src.pts = kept_xyz;
        src.index = sh->index.get();
        src.w = kept_w;
        src.ell = su.ell;
        src.delta = delta;
        ex = &src;
        ISDF_CUDA(cudaStreamSynchronize(s));   // the host staging vector goes out of scope
    }
    sh->qr = std::make_unique<QrShard>(Yt, n_local, su.ell, n_local, pos_offset, ex, s);
    return sh;
}

std::vector<int64_t> select_sketch_gathered(const Context& c, const SelectOptions& o, double* Yt, int64_t n,
                                            const double* kept_xyz, const double* kept_w, double* delta,
                                            const std::vector<double>& scales, SketchDiagnostics* diag_out,
                                            cudaStream_t s) {
    if (n == 0) return {};
    const SketchSetup su = sketch_setup(c, o, n, s);
    if (su.ax.has_occ) fail(kInvalid, "grid-sharded selection supports the ao, dx, dy, dz axes");
    require(static_cast<int>(scales.size()) == su.ax.naxes, "one scale per axis entry is required");
    SketchQR qr;
    if (delta && su.mixed) {
        // FP64 re-verification source over the gathered kept points
        HostFactors u, v;
        sketch_factors(su.d, su.ell, o.seed, u, v);
        const int64_t d = su.d, nout = 2 * su.ell;
        std::vector<double> hwt(static_cast<size_t>(d * nout));
        for (int64_t j = 0; j < d; ++j)
            for (int64_t t = 0; t < su.ell; ++t) {
                hwt[t * d + j] = u[j * su.ell + t];
                hwt[(su.ell + t) * d + j] = v[j * su.ell + t];
            }
        DeviceBuffer<double> WT(hwt.size(), s), dsc(scales.size(), s);
        DeviceBuffer<int64_t> idx(n, s);
        ISDF_CUDA(cudaMemcpyAsync(WT.get(), hwt.data(), hwt.size() * sizeof(double), cudaMemcpyHostToDevice, s));
        ISDF_CUDA(cudaMemcpyAsync(dsc.get(), scales.data(), scales.size() * sizeof(double), cudaMemcpyHostToDevice, s));
        iota_i64(idx.get(), n, s);
        ExactSketchSource src;
        src.ctx = &c;
        src.naxes = su.ax.naxes;
        for (int a = 0; a < su.ax.naxes; ++a) src.comp[a] = su.ax.comp[a];
        src.scales = dsc.get();
        src.WT = WT.get();
        src.pts = kept_xyz;
        src.index = idx.get();
        src.w = kept_w;
        src.ell = su.ell;
        src.delta = delta;
        qr = qrcp_sketch(Yt, n, su.ell, n, s, &src);
    } else {
        qr = qrcp_sketch(Yt, n, su.ell, n, s);
    }
    const SketchRank r = sketch_rank(qr, su.ell, n, o, su.physical_rank);
    fill_diag(diag_out, su.ell, r, qr);
    if (diag_out) diag_out->precision_used = (delta && su.mixed) ? 1 : 0;
    return std::vector<int64_t>(qr.jpvt.begin(), qr.jpvt.begin() + r.rank);
}

}  // namespace isdf
