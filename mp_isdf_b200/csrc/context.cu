// Context construction (libcint ATM/BAS/ENV tables -> device shell table) and
// the fused per-contracted-shell AO evaluator.
//
// Reference behaviour restated (mikovtun/mp_isdf):
//   table validation and shell metadata  cpp/src/ao_eval.cpp:54-65, 94-121
//   cartesian order x^l, x^(l-1)y, ...    cpp/src/ao_eval.cpp:30-44
//   s/p spherical scaling                 cpp/src/ao_eval.cpp:132-138
//   value / gradient formulas             cpp/src/ao_eval.cpp:207-249
//   value layout [p*nao+ao], gradient layout [(axis*Ng+p)*nao+ao]
//                                         cpp/include/ao_eval.hpp:83-99
#include "ao_device.cuh"
#include "isdf_internal.h"

#include <algorithm>
#include <cmath>
#include <limits>
#include <memory>
#include <type_traits>

namespace isdf {

Context::~Context() {
    cudaFree(d_shells);
    cudaFree(d_exp);
    cudaFree(d_coef);
    cudaFree(d_expf);
    cudaFree(d_coeff);
    cudaFree(d_ao_atom);
    cudaFree(d_pieces);
    cudaFree(d_shell_hi);
    cudaFree(d_shell_lo);
    cudaFree(d_piece_begin);
    cudaFree(d_fill);
    cudaFree(d_chunk_ao0);
    cudaFree(d_ao_slot);
    cudaFree(d_piece_chunk);
    cudaFree(d_piece_rec);
    cudaFree(d_piece_prim);
    cudaFree(d_piece_c64);
    cudaFree(d_piece_prim64);
    cudaFree(ws);
}

void upload_shell_centres(Context& c) {
    if (c.shells.empty()) return;
    std::vector<float4> hi, lo;
    for (const auto& sh : c.shells) {
        const float xh = static_cast<float>(sh.x), yh = static_cast<float>(sh.y), zh = static_cast<float>(sh.z);
        hi.push_back(make_float4(xh, yh, zh, sh.amin));
        lo.push_back(make_float4(static_cast<float>(sh.x - xh), static_cast<float>(sh.y - yh),
                                 static_cast<float>(sh.z - zh), 0.f));
    }
    ISDF_CUDA(cudaMemcpy(c.d_shell_hi, hi.data(), hi.size() * sizeof(float4), cudaMemcpyHostToDevice));
    ISDF_CUDA(cudaMemcpy(c.d_shell_lo, lo.data(), lo.size() * sizeof(float4), cudaMemcpyHostToDevice));
    if (c.d_piece_rec) upload_piece_records(c);   // the piece records carry the centres too
}

uint8_t* Context::workspace(size_t bytes) const {
    if (bytes > ws_bytes) {
        if (ws) ISDF_CUDA(cudaFree(ws));   // waits for the device
        ws = nullptr;
        ws_bytes = 0;
        ISDF_CUDA(cudaMalloc(reinterpret_cast<void**>(&ws), bytes));
        ws_bytes = bytes;
    }
    return ws;
}

// Bound on |P_lm(x)| / |x|^l over the components m of the spherical
// polynomials: the sum of the absolute cartesian coefficients, since every
// monomial x^a y^b z^c of degree l is at most |x|^l in absolute value.
static double c2s_abs_bound(int l) {
    double best = 0.0;
    const int ncart = (l + 1) * (l + 2) / 2;
    for (int sidx = 0; sidx < 2 * l + 1; ++sidx) {
        double sum = 0.0;
        for (int cidx = 0; cidx < ncart; ++cidx) sum += std::fabs(c2s_coef(l, sidx, cidx));
        best = std::max(best, sum);
    }
    return best;
}

// Largest value or d/dx, d/dy, d/dz component of any contraction of the
// shell at a point with amin r^2 >= X.  A primitive term is
// c exp(-a r^2) P(x) with |P| <= S r^l and |dP/dx| <= l S r^(l-1), so one
// component is at most |c| S exp(-a r^2) max(r^l, l r^(l-1) + 2 a r^(l+1)).
// Each of these falls with r where a r^2 >= (l+1)/2, which holds at every
// r >= r0 = sqrt(X / amin) for X >= (l+1)/2 (a >= amin): the maximum is at r0.
static double screened_term_bound(int l, int nprim, int nctr, const double* exps, const double* coefs,
                                  double amin, double X, double S) {
    const double r0 = std::sqrt(X / amin);
    double total = 0.0;
    for (int p = 0; p < nprim; ++p) {
        double c = 0.0;
        for (int j = 0; j < nctr; ++j) c = std::max(c, std::fabs(coefs[j * nprim + p]));
        const double a = exps[p];
        const double rl = std::pow(r0, l);
        const double grad = (l > 0 ? l * std::pow(r0, l - 1) : 0.0) + 2.0 * a * r0 * rl;
        total += c * S * std::exp(-a * r0 * r0) * std::max(rl, grad);
    }
    return total;
}

// Smallest screening argument X in [(l+1)/2 + 1, kExpCut] whose dropped terms
// stay within eps / 2 (the half leaves room for the FP32 rounding of the
// screening test); kExpCut (exact zeros only) when none does.
double screening_argument(int l, int nprim, int nctr, const double* exps, const double* coefs, double eps) {
    double amin = exps[0];
    for (int p = 1; p < nprim; ++p) amin = std::min(amin, exps[p]);
    if (!(amin > 0.0)) return kExpCut;
    const double S = c2s_abs_bound(l);
    double lo = 0.5 * (l + 1) + 1.0, hi = kExpCut;
    if (screened_term_bound(l, nprim, nctr, exps, coefs, amin, hi, S) > 0.5 * eps) return kExpCut;
    if (screened_term_bound(l, nprim, nctr, exps, coefs, amin, lo, S) <= 0.5 * eps) return lo;
    for (int it = 0; it < 64; ++it) {
        const double mid = 0.5 * (lo + hi);
        if (screened_term_bound(l, nprim, nctr, exps, coefs, amin, mid, S) <= 0.5 * eps) hi = mid;
        else lo = mid;
    }
    return hi;
}

Context* create_context(const int32_t* atm, int natm, const int32_t* bas, int nbas,
                        const double* env, int64_t nenv) {
    require(natm >= 0 && nbas >= 0 && nenv >= 20, "invalid libcint ATM/BAS/ENV table sizes");
    auto c = std::make_unique<Context>();
    ISDF_CUDA(cudaGetDevice(&c->device));
    {
        // Scratch buffers come from this process's default stream-ordered pool;
        // keep freed blocks cached across calls instead of returning them to
        // the driver at every synchronisation (the pool's default).
        cudaMemPool_t pool;
        ISDF_CUDA(cudaDeviceGetDefaultMemPool(&pool, c->device));
        uint64_t keep = std::numeric_limits<uint64_t>::max();
        ISDF_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    }
    c->natm = natm;
    c->atm.assign(atm, atm + static_cast<size_t>(natm) * 6);
    c->bas.assign(bas, bas + static_cast<size_t>(nbas) * 8);
    c->env.assign(env, env + nenv);
    auto range_ok = [&](int64_t off, int64_t len) {
        return off >= 0 && len >= 0 && off <= nenv && len <= nenv - off;
    };
    std::vector<double> exps, coefs;
    int64_t nao = 0;
    for (int a = 0; a < natm; ++a) {
        const int pc = atm[6 * a + 1];
        require(range_ok(pc, 3), "libcint table contains an invalid ENV offset");
        c->atom_xyz.insert(c->atom_xyz.end(), env + pc, env + pc + 3);
    }
    for (int i = 0; i < nbas; ++i) {
        const int32_t* b = bas + 8 * i;
        const int atom = b[0], l = b[1], np = b[2], nc = b[3];
        require(atom >= 0 && atom < natm && l >= 0 && np > 0 && nc > 0 && np <= 64 && nc <= 64,
                "invalid libcint basis shell");
        if (l > kMaxL) fail(kNotImplemented, "angular momentum above l=6 is not supported");
        require(range_ok(b[5], np) && range_ok(b[6], static_cast<int64_t>(np) * nc),
                "libcint table contains an invalid ENV offset");
        ShellDesc s{};
        s.l = l; s.nprim = np; s.nctr = nc;
        if (nao + static_cast<int64_t>(2 * l + 1) * nc > std::numeric_limits<int>::max())
            fail(kOverflow, "AO or transformation index exceeds int range");
        s.ao_off = static_cast<int>(nao);
        s.prim_off = static_cast<int>(exps.size());
        s.coef_off = static_cast<int>(coefs.size());
        s.atom = atom;
        s.amin = static_cast<float>(*std::min_element(env + b[5], env + b[5] + np));
        {
            const double amin = *std::min_element(env + b[5], env + b[5] + np);
            const double x32 = screening_argument(l, np, nc, env + b[5], env + b[6], kScreenFp32);
            const double x64 = screening_argument(l, np, nc, env + b[5], env + b[6], kScreenFp64);
            s.scr32 = static_cast<float>(amin * (kExpCut / x32));
            s.scr64 = static_cast<float>(amin * (kExpCut / x64));
        }
        const double* xyz = &c->atom_xyz[3 * atom];
        s.x = xyz[0]; s.y = xyz[1]; s.z = xyz[2];
        exps.insert(exps.end(), env + b[5], env + b[5] + np);
        coefs.insert(coefs.end(), env + b[6], env + b[6] + static_cast<int64_t>(np) * nc);
        c->shells.push_back(s);
        for (int k = 0; k < (2 * l + 1) * nc; ++k) c->ao_atom.push_back(atom);
        nao += static_cast<int64_t>(2 * l + 1) * nc;
        c->lmax = std::max(c->lmax, l);
    }
    c->nao = static_cast<int>(nao);
    c->nshell = static_cast<int>(c->shells.size());
    auto up = [](auto*& dst, const auto& src) {
        using V = std::remove_pointer_t<std::remove_reference_t<decltype(dst)>>;
        if (src.empty()) return;
        ISDF_CUDA(cudaMalloc(reinterpret_cast<void**>(&dst), src.size() * sizeof(V)));
        ISDF_CUDA(cudaMemcpy(dst, src.data(), src.size() * sizeof(V), cudaMemcpyHostToDevice));
    };
    std::vector<float> expf_(exps.begin(), exps.end()), coeff_(coefs.begin(), coefs.end());
    c->h_expf = expf_;
    c->h_coeff = coeff_;
    c->h_exp64 = exps;
    c->h_coef64 = coefs;
    up(c->d_shells, c->shells);
    up(c->d_exp, exps);
    up(c->d_coef, coefs);
    up(c->d_expf, expf_);
    up(c->d_coeff, coeff_);
    up(c->d_ao_atom, c->ao_atom);
    if (!c->shells.empty()) {
        ISDF_CUDA(cudaMalloc(reinterpret_cast<void**>(&c->d_shell_hi), c->shells.size() * sizeof(float4)));
        ISDF_CUDA(cudaMalloc(reinterpret_cast<void**>(&c->d_shell_lo), c->shells.size() * sizeof(float4)));
        upload_shell_centres(*c);
    }
    build_chunk_layout(*c);
    return c.release();
}

// ------------------------------------------------------------------------------
// AO kernels
// ------------------------------------------------------------------------------
namespace {

template <class T>
struct RawSink {
    T* val; T* grad; int64_t p, n, ld; bool want_val;
    template <int C> __device__ __forceinline__ void put(int ao, T v) {
        if (C == 0) { if (want_val) val[p * ld + ao] = v; }
        else grad[((C - 1) * n + p) * ld + ao] = v;
    }
};

template <class T>
struct AxisSink {
    T* out; int64_t p, ld; const AxisSpec* ax; const int* off; double sq[4]; bool count;
    template <int C> __device__ __forceinline__ void put(int ao, T v) {
        if (!((ax->need_mask >> C) & 1)) return;
        if (count) sq[C] += static_cast<double>(v) * static_cast<double>(v);
        for (int a = 0; a < ax->naxes; ++a)
            if (ax->comp[a] == C && !ax->occ[a])
                out[p * ld + off[a] + ao] = static_cast<T>(ax->scale[a] * static_cast<double>(v));
    }
};

constexpr int kPtsPerBlock = 32;
constexpr int kShellLanes = 4;

template <class T, bool GRAD>
__global__ void __launch_bounds__(kPtsPerBlock * kShellLanes)
ao_raw_kernel(const ShellDesc* __restrict__ shells, int nshell, const T* __restrict__ exps,
              const T* __restrict__ coefs, const double* __restrict__ pts,
              int64_t n, T* val, T* grad, int64_t ld, bool want_val) {
    const int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const double px = pts[3 * p], py = pts[3 * p + 1], pz = pts[3 * p + 2];
    RawSink<T> sink{val, grad, p, n, ld, want_val};
    for (int sh = threadIdx.y; sh < nshell; sh += blockDim.y) {
        const ShellDesc b = shells[sh];
        eval_shell_any<T, GRAD>(b, px - b.x, py - b.y, pz - b.z, exps, coefs, sink);
    }
}

// Tiled evaluation for the (Ng, nao) / (3, Ng, nao) layouts: a block takes 64
// points (two warps per piece lane, lane = point) and walks the K-chunks of
// the context's chunk layout (contiguous AO ranges of at most 32 slots holding
// whole contraction groups); the two warps of lane j evaluate the pieces that
// the layout balanced onto lane j, for points 0-31 and 32-63, so each piece's
// metadata is read twice close together.  The chunk's values go to a padded
// shared tile [comp][slot][point]; then every (component, point) row of the
// chunk is written as one contiguous run of `fill` values from a row pointer
// formed once per block, so a warp store covers up to 256 bytes instead of 32
// scattered words.  The values are those of ao_raw_kernel up to the
// contraction of products into FMAs (same offsets, same per-contraction
// arithmetic), except that a piece whose every primitive is beyond the cutoff
// at all 32 points of a warp is written as +0 without evaluation (the
// evaluation gives zeros there as well, possibly signed).
constexpr int kTilePts = 64;
constexpr int kTileStride = kTilePts + 1;   // padded point stride: conflict-free row reads

template <class T>
struct TileSink {
    T* st; int p, base;
    template <int C> __device__ __forceinline__ void put(int ao, T v) {
        st[(C * 32 + ao + base) * kTileStride + p] = v;
    }
};

struct TileArgs {
    const float4* piece_rec; const double2* piece_c64; const void* prims;   // packed piece records
    const int* lane_begin; const int* fill; const int* chunk_ao0; int nchunks;
    const double* pts; int64_t n, ld; void* val; void* grad; bool want_val;
};

// The packed primitive table of T (float4 entries, or two double2 per entry).
template <class T>
__device__ __forceinline__ const typename PackedPrim<T>::rec* packed_prims(const void* p, int prim_off) {
    return static_cast<const typename PackedPrim<T>::rec*>(p) + (sizeof(T) == 8 ? 2 : 1) * prim_off;
}

// Shared tiles per block: two for the value-only tiles (chunk c evaluated into
// one while other warps still store chunk c - 1 from the other, one barrier
// per chunk; FP64 values 12.5 -> 12.2 ms at C5), else one (two barriers per
// chunk: doubling the 33 KB FP32 gradient tile left less L1 and was slower).
template <class T, bool GRAD>
constexpr int tile_bufs() {
    return 2 * (GRAD ? 4 : 1) * 32 * kTileStride * sizeof(T) <= 40 * 1024 ? 2 : 1;
}
template <class T, bool GRAD>
constexpr size_t tile_elems() { return static_cast<size_t>(GRAD ? 4 : 1) * 32 * kTileStride; }

template <class T, bool GRAD>
constexpr size_t tile_smem_bytes() {
    return tile_bufs<T, GRAD>() * tile_elems<T, GRAD>() * sizeof(T) + (GRAD ? 4 : 1) * kTilePts * sizeof(T*);
}

template <class T, bool GRAD, int LMAX, int PPT>
__global__ void __launch_bounds__(kTilePts / 32 * PPT * 32) ao_tile_kernel(TileArgs a) {
    constexpr int kNComp = GRAD ? 4 : 1;
    constexpr int kWarps = kTilePts / 32 * PPT;
    extern __shared__ __align__(16) uint8_t tile_raw[];
    T** rowp = reinterpret_cast<T**>(tile_raw);                       // [kNComp][kTilePts]
    T* const st0 = reinterpret_cast<T*>(tile_raw + kNComp * kTilePts * sizeof(T*));
    const int lane = threadIdx.x % 32, warp = threadIdx.x / 32;
    const int lanegrp = warp % PPT, p = (warp / PPT) * 32 + lane;
    const int64_t b0 = static_cast<int64_t>(blockIdx.x) * kTilePts;
    const int64_t g = b0 + p;
    const bool valid = g < a.n;
    const double px = valid ? a.pts[3 * g] : 0.0, py = valid ? a.pts[3 * g + 1] : 0.0,
                 pz = valid ? a.pts[3 * g + 2] : 0.0;
    // output row of (component, point), or null where nothing is written
    for (int i = threadIdx.x; i < kNComp * kTilePts; i += blockDim.x) {
        const int cc = i / kTilePts;
        const int64_t gp = b0 + i % kTilePts;
        T* r = nullptr;
        if (gp < a.n) {
            if (cc == 0) r = a.want_val ? static_cast<T*>(a.val) + gp * a.ld : nullptr;
            else r = static_cast<T*>(a.grad) + ((cc - 1) * a.n + gp) * a.ld;
        }
        rowp[i] = r;
    }
    // a piece is written as zeros where its FP64 screening exponent puts all
    // 32 points of the warp beyond kExpCut (nothing dropped above kScreenFp64);
    // the margin covers the exponent's rounding to FP32
    const double cut = kExpCut * 1.0001;
    for (int c = 0; c < a.nchunks; ++c) {
        T* const st = st0 + (tile_bufs<T, GRAD>() == 2 ? (c & 1) * tile_elems<T, GRAD>() : 0);
        const int pb = a.lane_begin[c * PPT + lanegrp], pe = a.lane_begin[c * PPT + lanegrp + 1];
        for (int pi = pb; pi < pe; ++pi) {
            // packed record: (l, primitives, contractions, first slot), centre and
            // smallest exponent, primitive-table offset
            const int4 meta = __ldg(reinterpret_cast<const int4*>(a.piece_rec) + 3 * pi + 2);
            const int poff = __float_as_int(__ldg(a.piece_rec + 3 * pi + 1).w);
            const double2 cxy = __ldg(a.piece_c64 + 2 * pi), cza = __ldg(a.piece_c64 + 2 * pi + 1);
            const int l = meta.x, nprim = meta.y, nc = meta.z, slot0 = meta.w;
            const int ns = 2 * l + 1;
            const double dx = px - cxy.x, dy = py - cxy.y, dz = pz - cza.x;
            const double r2 = dx * dx + dy * dy + dz * dz;
            if (__all_sync(0xffffffffu, !valid || cza.y * r2 > cut)) {
                for (int k = slot0; k < slot0 + nc * ns; ++k)
#pragma unroll
                    for (int cc = 0; cc < kNComp; ++cc) st[(cc * 32 + k) * kTileStride + p] = T(0);
                continue;
            }
            TileSink<T> sink{st, p, slot0};
            eval_piece<T, GRAD, LMAX>(l, static_cast<T>(dx), static_cast<T>(dy), static_cast<T>(dz),
                                      static_cast<T>(r2), packed_prims<T>(a.prims, poff), nprim, nc, sink);
        }
        __syncthreads();
        const int fill = a.fill[c], ao0 = a.chunk_ao0[c];
        for (int r = warp; r < kNComp * kTilePts; r += kWarps) {
            T* row = rowp[r];
            if (row != nullptr && lane < fill)
                row[ao0 + lane] = st[((r / kTilePts) * 32 + lane) * kTileStride + r % kTilePts];
        }
        if constexpr (tile_bufs<T, GRAD>() == 1) __syncthreads();   // the tile is refilled next
    }
}

template <class T, bool GRAD, int LMAX, int PPT>
void launch_tile(const TileArgs& a, cudaStream_t s) {
    const int64_t nb = (a.n + kTilePts - 1) / kTilePts;
    require(nb < (1ll << 31), "too many grid points for one launch");
    constexpr size_t smem = tile_smem_bytes<T, GRAD>();
    auto kern = ao_tile_kernel<T, GRAD, LMAX, PPT>;
    if constexpr (smem > 48 * 1024)
        ISDF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    kern<<<static_cast<unsigned>(nb), kTilePts / 32 * PPT * 32, smem, s>>>(a);
    ISDF_LAUNCH_CHECK();
}

template <class T, bool GRAD>
void launch_tile_l(const Context& c, const TileArgs& a, cudaStream_t s) {
    // lane counts as in piece_lanes_for_lmax()
    if (c.lmax <= 2) launch_tile<T, GRAD, 2, 6>(a, s);
    else if (c.lmax <= 4) launch_tile<T, GRAD, 4, 2>(a, s);
    else launch_tile<T, GRAD, kMaxL, 2>(a, s);
}

// Tiled axis features F[p*ld + offset[a] + ao] = scale[a] * comp_a(p, ao): the
// layout of ao_tile_kernel (64 points per block, piece lanes of the chunk
// layout, a padded shared tile [comp][slot][point] per K-chunk), with the
// points gathered through `index`, one contiguous row store per (axis entry,
// point) and chunk, and the per-component sums of squares of the points with
// nonzero weight accumulated by the evaluating threads (FP64).
template <class T>
struct TileSqSink {
    T* st; int p, base; bool count; double sq[4];
    template <int C> __device__ __forceinline__ void put(int ao, T v) {
        st[(C * 32 + ao + base) * kTileStride + p] = v;
        if (count) sq[C] += static_cast<double>(v) * static_cast<double>(v);
    }
};

struct AxisTileArgs {
    const float4* piece_rec; const double2* piece_c64; const void* prims;   // packed piece records
    const int* lane_begin; const int* fill; const int* chunk_ao0; int nchunks;
    const double* pts; const int64_t* index; int64_t n; const double* weights;
    void* out; int64_t ld; double* sumsq;
    int nent; int comp[16]; int off[16]; double scale[16];   // the non-occupied axis entries
};

template <class T, bool GRAD>
constexpr size_t axis_tile_smem_bytes() {
    return tile_bufs<T, GRAD>() * tile_elems<T, GRAD>() * sizeof(T) + kTilePts * sizeof(T*);
}

template <class T, bool GRAD, int LMAX, int PPT>
__global__ void __launch_bounds__(kTilePts / 32 * PPT * 32) axis_tile_kernel(AxisTileArgs a) {
    constexpr int kNComp = GRAD ? 4 : 1;
    constexpr int kWarps = kTilePts / 32 * PPT;
    extern __shared__ __align__(16) uint8_t tile_raw[];
    T** rowp = reinterpret_cast<T**>(tile_raw);                       // [kTilePts]
    T* const st0 = reinterpret_cast<T*>(tile_raw + kTilePts * sizeof(T*));
    __shared__ double red[kWarps][4];
    const int lane = threadIdx.x % 32, warp = threadIdx.x / 32;
    const int lanegrp = warp % PPT, p = (warp / PPT) * 32 + lane;
    const int64_t b0 = static_cast<int64_t>(blockIdx.x) * kTilePts;
    const int64_t g = b0 + p;
    const bool valid = g < a.n;
    const int64_t gi = valid ? (a.index ? a.index[g] : g) : 0;
    const double px = valid ? a.pts[3 * gi] : 0.0, py = valid ? a.pts[3 * gi + 1] : 0.0,
                 pz = valid ? a.pts[3 * gi + 2] : 0.0;
    const bool count = valid && a.sumsq != nullptr && (a.weights == nullptr || a.weights[gi] != 0.0);
    for (int i = threadIdx.x; i < kTilePts; i += blockDim.x) {
        const int64_t gp = b0 + i;
        rowp[i] = gp < a.n ? static_cast<T*>(a.out) + gp * a.ld : nullptr;
    }
    double sq[4] = {0.0, 0.0, 0.0, 0.0};
    const double cut = kExpCut * 1.0001;
    for (int c = 0; c < a.nchunks; ++c) {
        T* const st = st0 + (tile_bufs<T, GRAD>() == 2 ? (c & 1) * tile_elems<T, GRAD>() : 0);
        const int pb = a.lane_begin[c * PPT + lanegrp], pe = a.lane_begin[c * PPT + lanegrp + 1];
        for (int pi = pb; pi < pe; ++pi) {
            const int4 meta = __ldg(reinterpret_cast<const int4*>(a.piece_rec) + 3 * pi + 2);
            const int poff = __float_as_int(__ldg(a.piece_rec + 3 * pi + 1).w);
            const double2 cxy = __ldg(a.piece_c64 + 2 * pi), cza = __ldg(a.piece_c64 + 2 * pi + 1);
            const int l = meta.x, nprim = meta.y, nc = meta.z, slot0 = meta.w;
            const int ns = 2 * l + 1;
            const double dx = px - cxy.x, dy = py - cxy.y, dz = pz - cza.x;
            const double r2 = dx * dx + dy * dy + dz * dz;
            if (__all_sync(0xffffffffu, !valid || cza.y * r2 > cut)) {
                for (int k = slot0; k < slot0 + nc * ns; ++k)
#pragma unroll
                    for (int cc = 0; cc < kNComp; ++cc) st[(cc * 32 + k) * kTileStride + p] = T(0);
                continue;
            }
            TileSqSink<T> sink{st, p, slot0, count, {0.0, 0.0, 0.0, 0.0}};
            eval_piece<T, GRAD, LMAX>(l, static_cast<T>(dx), static_cast<T>(dy), static_cast<T>(dz),
                                      static_cast<T>(r2), packed_prims<T>(a.prims, poff), nprim, nc, sink);
#pragma unroll
            for (int cc = 0; cc < 4; ++cc) sq[cc] += sink.sq[cc];
        }
        __syncthreads();
        const int fill = a.fill[c], ao0 = a.chunk_ao0[c];
        for (int r = warp; r < a.nent * kTilePts; r += kWarps) {
            const int e = r / kTilePts, pp = r % kTilePts;
            T* row = rowp[pp];
            if (row != nullptr && lane < fill)
                row[a.off[e] + ao0 + lane] =
                    static_cast<T>(a.scale[e] * static_cast<double>(st[(a.comp[e] * 32 + lane) * kTileStride + pp]));
        }
        if constexpr (tile_bufs<T, GRAD>() == 1) __syncthreads();   // the tile is refilled next
    }
    if (a.sumsq) {
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) {
            double v = sq[cc];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if (lane == 0) red[warp][cc] = v;
        }
        __syncthreads();
        if (threadIdx.x < 4) {
            double v = 0.0;
            for (int w2 = 0; w2 < kWarps; ++w2) v += red[w2][threadIdx.x];
            if (v != 0.0) atomicAdd(&a.sumsq[threadIdx.x], v);
        }
    }
}

template <class T, bool GRAD, int LMAX, int PPT>
void launch_axis_tile(const AxisTileArgs& a, cudaStream_t s) {
    const int64_t nb = (a.n + kTilePts - 1) / kTilePts;
    require(nb < (1ll << 31), "too many grid points for one launch");
    constexpr size_t smem = axis_tile_smem_bytes<T, GRAD>();
    auto kern = axis_tile_kernel<T, GRAD, LMAX, PPT>;
    if constexpr (smem > 48 * 1024)
        ISDF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    kern<<<static_cast<unsigned>(nb), kTilePts / 32 * PPT * 32, smem, s>>>(a);
    ISDF_LAUNCH_CHECK();
}

template <class T, bool GRAD>
void launch_axis_tile_l(const Context& c, const AxisTileArgs& a, cudaStream_t s) {
    if (c.lmax <= 2) launch_axis_tile<T, GRAD, 2, 6>(a, s);
    else if (c.lmax <= 4) launch_axis_tile<T, GRAD, 4, 2>(a, s);
    else launch_axis_tile<T, GRAD, kMaxL, 2>(a, s);
}

template <class T, bool GRAD>
__global__ void __launch_bounds__(kPtsPerBlock * kShellLanes)
ao_axis_kernel(const ShellDesc* __restrict__ shells, int nshell, const T* __restrict__ exps,
               const T* __restrict__ coefs, const double* __restrict__ pts,
               const int64_t* __restrict__ index, int64_t n, AxisSpec ax, T* out, int64_t ld,
               double* sumsq, const double* __restrict__ weights, int nao) {
    __shared__ double red[kPtsPerBlock * kShellLanes][4];
    __shared__ int off[16];
    const int tid = threadIdx.y * kPtsPerBlock + threadIdx.x;
    if (tid < ax.naxes) off[tid] = ax.offset[tid];
    __syncthreads();
    const int64_t p = static_cast<int64_t>(blockIdx.x) * kPtsPerBlock + threadIdx.x;
    AxisSink<T> sink{out, p, ld, &ax, off, {0, 0, 0, 0}, false};
    if (p < n) {
        const int64_t gi = index ? index[p] : p;
        const double px = pts[3 * gi], py = pts[3 * gi + 1], pz = pts[3 * gi + 2];
        sink.count = sumsq != nullptr && (weights == nullptr || weights[gi] != 0.0);
        for (int sh = threadIdx.y; sh < nshell; sh += kShellLanes) {
            const ShellDesc b = shells[sh];
            eval_shell_any<T, GRAD>(b, px - b.x, py - b.y, pz - b.z, exps, coefs, sink);
        }
    }
    if (sumsq) {
#pragma unroll
        for (int c = 0; c < 4; ++c) red[tid][c] = sink.sq[c];
        __syncthreads();
        for (int stride = kPtsPerBlock * kShellLanes / 2; stride > 0; stride >>= 1) {
            if (tid < stride)
                for (int c = 0; c < 4; ++c) red[tid][c] += red[tid + stride][c];
            __syncthreads();
        }
        if (tid < 4 && ((ax.need_mask >> tid) & 1)) atomicAdd(&sumsq[tid], red[0][tid]);
    }
}

// Occupied-orbital block: out[p][j] *= scale, and the squared unscaled values
// of the counted points added into sumsq[4].
__global__ void occ_block_kernel(double* out, int64_t ld, int64_t n, int nocc, double scale,
                                 const int64_t* __restrict__ index, const double* __restrict__ weights,
                                 double* sumsq) {
    __shared__ double red[256];
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    double sq = 0;
    if (i < n * nocc) {
        const int64_t p = i / nocc, j = i % nocc;
        const double v = out[p * ld + j];
        const int64_t gi = index ? index[p] : p;
        if (sumsq && (weights == nullptr || weights[gi] != 0.0)) sq = v * v;
        out[p * ld + j] = scale * v;
    }
    if (!sumsq) return;
    red[threadIdx.x] = sq;
    __syncthreads();
    for (int st = blockDim.x / 2; st > 0; st >>= 1) {
        if (threadIdx.x < st) red[threadIdx.x] += red[threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x == 0 && red[0] != 0.0) atomicAdd(&sumsq[4], red[0]);
}

template <class T> const T* exps_of(const Context& c);
template <> const double* exps_of<double>(const Context& c) { return c.d_exp; }
template <> const float* exps_of<float>(const Context& c) { return c.d_expf; }
template <class T> const void* prims_of(const Context& c);
template <> const void* prims_of<double>(const Context& c) { return c.d_piece_prim64; }
template <> const void* prims_of<float>(const Context& c) { return c.d_piece_prim; }
template <class T> const T* coefs_of(const Context& c);
template <> const double* coefs_of<double>(const Context& c) { return c.d_coef; }
template <> const float* coefs_of<float>(const Context& c) { return c.d_coeff; }

}  // namespace

template <class T>
void eval_ao(const Context& c, const double* pts, int64_t n, T* out_val, T* out_grad,
             int64_t ld, cudaStream_t s) {
    require(out_val != nullptr || out_grad != nullptr, "AO evaluation needs a values or a gradient output");
    if (n == 0 || c.nao == 0) return;
    ISDF_PROFILE(sizeof(T) == 8 ? "ao_eval_f64" : "ao_eval_f32", s);
    // few points (anchors, candidate columns): one point per block, its shells
    // spread over the block; otherwise 32 points x 4 shell lanes
    const bool few = n <= 2048;
    if (!few) {
        TileArgs a{c.d_piece_rec, c.d_piece_c64, prims_of<T>(c), c.d_piece_begin, c.d_fill,
                   c.d_chunk_ao0, c.nchunks, pts, n, ld, out_val, out_grad, out_val != nullptr};
        if (out_grad) launch_tile_l<T, true>(c, a, s);
        else launch_tile_l<T, false>(c, a, s);
        return;
    }
    const dim3 block = few ? dim3(1, kPtsPerBlock * kShellLanes) : dim3(kPtsPerBlock, kShellLanes);
    const int64_t nb = (n + block.x - 1) / block.x;
    require(nb < (1ll << 31), "too many grid points for one launch");
    if (out_grad)
        ao_raw_kernel<T, true><<<static_cast<unsigned>(nb), block, 0, s>>>(
            c.d_shells, c.nshell, exps_of<T>(c), coefs_of<T>(c), pts, n, out_val,
            out_grad, ld, out_val != nullptr);
    else
        ao_raw_kernel<T, false><<<static_cast<unsigned>(nb), block, 0, s>>>(
            c.d_shells, c.nshell, exps_of<T>(c), coefs_of<T>(c), pts, n, out_val,
            nullptr, ld, true);
    ISDF_LAUNCH_CHECK();
}

template <class T>
void eval_axis_features(const Context& c, const double* pts, const int64_t* index, int64_t n,
                        const AxisSpec& ax, T* out, int64_t ld, double* sumsq,
                        const double* weights, cudaStream_t s) {
    if (n == 0 || c.nao == 0) return;
    require(ax.naxes > 0 && ax.naxes <= 16, "between 1 and 16 axes are supported");
    ISDF_PROFILE(sizeof(T) == 8 ? "ao_axis_f64" : "ao_axis_f32", s);
    dim3 block(kPtsPerBlock, kShellLanes);
    const int64_t nb = (n + kPtsPerBlock - 1) / kPtsPerBlock;
    require(nb < (1ll << 31), "too many grid points for one launch");
    const bool grad = (ax.need_mask & 0xE) != 0;
    if (n > 2048) {
        // tiled: contiguous row stores per (axis entry, point) and K-chunk
        AxisTileArgs ta{c.d_piece_rec, c.d_piece_c64, prims_of<T>(c), c.d_piece_begin, c.d_fill,
                        c.d_chunk_ao0, c.nchunks, pts, index, n, weights, out, ld, sumsq, 0, {}, {}, {}};
        for (int e = 0; e < ax.naxes; ++e) {
            if (ax.occ[e]) continue;
            ta.comp[ta.nent] = ax.comp[e];
            ta.off[ta.nent] = ax.offset[e];
            ta.scale[ta.nent] = ax.scale[e];
            ++ta.nent;
        }
        if (grad) launch_axis_tile_l<T, true>(c, ta, s);
        else launch_axis_tile_l<T, false>(c, ta, s);
    } else if (grad) {
        ao_axis_kernel<T, true><<<static_cast<unsigned>(nb), block, 0, s>>>(
            c.d_shells, c.nshell, exps_of<T>(c), coefs_of<T>(c), pts, index, n, ax,
            out, ld, sumsq, weights, c.nao);
        ISDF_LAUNCH_CHECK();
    } else {
        ao_axis_kernel<T, false><<<static_cast<unsigned>(nb), block, 0, s>>>(
            c.d_shells, c.nshell, exps_of<T>(c), coefs_of<T>(c), pts, index, n, ax,
            out, ld, sumsq, weights, c.nao);
        ISDF_LAUNCH_CHECK();
    }
    if (!ax.has_occ) return;
    // occupied-orbital entries: psi = Phi C_occ (anchor_select_impl.hpp:69-72),
    // from the AO values of the same points, then scaled (sumsq slot 4)
    if constexpr (sizeof(T) != 8) {
        fail(kNotImplemented, "the OccupiedOrbital axis is evaluated in FP64 only");
    } else {
        AxisSpec vs{};
        vs.naxes = 1;
        vs.comp[0] = 0;
        vs.scale[0] = 1.0;
        vs.need_mask = 1;
        vs.offset[0] = 0;
        vs.width[0] = c.nao;
        vs.occ[0] = false;
        vs.d = c.nao;
        DeviceBuffer<double> phi(static_cast<size_t>(n) * c.nao, s);
        ao_axis_kernel<double, false><<<static_cast<unsigned>(nb), block, 0, s>>>(
            c.d_shells, c.nshell, c.d_exp, c.d_coef, pts, index, n, vs, phi.get(), c.nao, nullptr, nullptr,
            c.nao);
        ISDF_LAUNCH_CHECK();
        bool counted = false;   // repeated occupied entries add their sum of squares once
        for (int a = 0; a < ax.naxes; ++a) {
            if (!ax.occ[a]) continue;
            gemm_f64(n, ax.nocc, c.nao, phi.get(), c.nao, 0, ax.mo, c.nao, 0, out + ax.offset[a], ld, 0, 1,
                     false, s);
            occ_block_kernel<<<static_cast<unsigned>((n * ax.nocc + 255) / 256), 256, 0, s>>>(
                out + ax.offset[a], ld, n, ax.nocc, ax.scale[a], index, weights, counted ? nullptr : sumsq);
            ISDF_LAUNCH_CHECK();
            counted = true;
        }
    }
}

template void eval_ao<double>(const Context&, const double*, int64_t, double*, double*, int64_t, cudaStream_t);
template void eval_ao<float>(const Context&, const double*, int64_t, float*, float*, int64_t, cudaStream_t);
template void eval_axis_features<double>(const Context&, const double*, const int64_t*, int64_t,
                                         const AxisSpec&, double*, int64_t, double*, const double*, cudaStream_t);
template void eval_axis_features<float>(const Context&, const double*, const int64_t*, int64_t,
                                        const AxisSpec&, float*, int64_t, double*, const double*, cudaStream_t);

}  // namespace isdf
