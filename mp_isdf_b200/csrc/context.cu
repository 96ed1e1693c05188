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
    cudaFree(d_win_entry);
    cudaFree(d_win_begin);
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
    ISDF_CUDA(cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, c->device));
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
    build_window_layout(*c);
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
// points (two warps per piece lane, lane = point) and walks the AO windows
// [32w, 32w + 32) of the context's window layout; the two warps of lane j
// evaluate the window's pieces that the layout balanced onto lane j, for
// points 0-31 and 32-63, into a padded shared tile [comp][slot][point].  Then
// every (component, point) row segment of the window leaves as one aligned run
// of up to 32 values -- a whole 128-byte line of FP32 (two of FP64) when the
// row length is a multiple of 32 values -- and the store pass leaves zeros
// behind in the tile, so a screened piece costs no shared-memory writes.  A
// piece across a window boundary is evaluated in each window and writes the
// slots inside it.  The values are those of ao_raw_kernel up to the contraction
// of products into FMAs (same offsets, same per-contraction arithmetic), with
// +0 where a piece is screened for a whole warp.  Written without any
// evaluation, the C5 layout's rows took 26.7 ms as 28-32 value runs from the
// arbitrary starts of contraction-group chunks (FP32, 4 components: 1.8 TB/s)
// and 9.5 ms as aligned 32-value windows (5.1 TB/s).
//
// Screening, in two steps: the bounding box of the tile's points against each
// piece's FP64 screening radius (a candidate bit per piece in shared memory:
// the record of a piece that is not a candidate is never read), then each
// warp's 32 points against the candidate's radius.  The FP64 screening
// exponent drops nothing above kScreenFp64 (1e-15) for either table.
constexpr int kTilePts = 64;
constexpr int kTileStride = kTilePts + 1;   // padded point stride: conflict-free row reads
constexpr double kScreenCut = kExpCut * 1.0001;   // margin for the exponent's rounding to FP32

template <class T>
struct WinSink {
    T* st; int p, base;
    template <int C> __device__ __forceinline__ void put(int ao, T v) {
        const int s = ao + base;
        if (static_cast<unsigned>(s) < static_cast<unsigned>(kWin)) st[(C * kWin + s) * kTileStride + p] = v;
    }
};

// the same, with the sums of squares of the slots it writes (each AO once)
template <class T>
struct WinSqSink {
    T* st; int p, base; bool count; double sq[4];
    template <int C> __device__ __forceinline__ void put(int ao, T v) {
        const int s = ao + base;
        if (static_cast<unsigned>(s) < static_cast<unsigned>(kWin)) {
            st[(C * kWin + s) * kTileStride + p] = v;
            if (count) sq[C] += static_cast<double>(v) * static_cast<double>(v);
        }
    }
};

// The packed primitive table of T (float4 entries, or two double2 per entry).
template <class T>
__device__ __forceinline__ const typename PackedPrim<T>::rec* packed_prims(const void* p, int prim_off) {
    return static_cast<const typename PackedPrim<T>::rec*>(p) + (sizeof(T) == 8 ? 2 : 1) * prim_off;
}

// Candidate pieces of a tile: bit pi of cand is set where piece pi's FP64
// screening radius reaches the bounding box of the tile's valid points (its
// half-widths widened by 1e-9 bohr, far above the rounding of the box
// arithmetic, so that a piece left out is screened at every point by the
// per-warp test as well).  The warps that hold each point once (box_warp)
// reduce the box; called by every thread, ends with a block barrier.
__device__ void tile_candidates(const double2* __restrict__ c64, int npieces, double px, double py, double pz,
                                bool valid, bool box_warp, int half, double (*box)[6], uint32_t* cand) {
    const int lane = threadIdx.x % 32;
    if (box_warp) {
        const double pc[3] = {px, py, pz};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            double lo = valid ? pc[d] : INFINITY, hi = valid ? pc[d] : -INFINITY;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
                hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
            }
            if (lane == 0) { box[half][d] = lo; box[half][3 + d] = hi; }
        }
    }
    for (int i = threadIdx.x; i < (npieces + 31) / 32; i += blockDim.x) cand[i] = 0u;
    __syncthreads();
    double mid[3], hw[3];
    bool any = true;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        double lo = box[0][d], hi = box[0][3 + d];
#pragma unroll
        for (int h = 1; h < kTilePts / 32; ++h) { lo = fmin(lo, box[h][d]); hi = fmax(hi, box[h][3 + d]); }
        any = any && lo <= hi;
        mid[d] = 0.5 * (lo + hi);
        hw[d] = 0.5 * (hi - lo) + 1e-9;
    }
    if (any)
        for (int pi = threadIdx.x; pi < npieces; pi += blockDim.x) {
            const double2 cxy = __ldg(c64 + 2 * pi), cza = __ldg(c64 + 2 * pi + 1);
            const double ex = fmax(fabs(cxy.x - mid[0]) - hw[0], 0.0);
            const double ey = fmax(fabs(cxy.y - mid[1]) - hw[1], 0.0);
            const double ez = fmax(fabs(cza.x - mid[2]) - hw[2], 0.0);
            if (!(cza.y * (ex * ex + ey * ey + ez * ez) > kScreenCut)) atomicOr(&cand[pi >> 5], 1u << (pi & 31));
        }
    __syncthreads();
}

struct TileArgs {
    const float4* piece_rec; const double2* piece_c64; const void* prims;   // packed piece records
    const int2* win_entry; const int* win_begin; int nwin, nao, npieces, lanes;   // window layout
    const double* pts; int64_t n, ld; void* val; void* grad; bool want_val;
};

// Shared tiles per block: two for the value-only tiles (window w is evaluated
// into one while other warps still store window w - 1 from the other, one
// barrier per window), else one (two barriers per window).
template <class T, bool GRAD>
constexpr int tile_bufs() {
    return 2 * (GRAD ? 4 : 1) * kWin * kTileStride * sizeof(T) <= 40 * 1024 ? 2 : 1;
}
template <class T, bool GRAD>
constexpr size_t tile_elems() { return static_cast<size_t>(GRAD ? 4 : 1) * kWin * kTileStride; }

// dynamic shared memory: row pointers, tiles, candidate bits
template <class T, bool GRAD>
size_t tile_smem_bytes(int nrowp, int npieces) {
    return nrowp * sizeof(T*) + tile_bufs<T, GRAD>() * tile_elems<T, GRAD>() * sizeof(T) +
           4 * static_cast<size_t>((npieces + 31) / 32);
}

// One piece of a window for the warp's 32 points: nothing where the piece is
// not a candidate of the tile or where every point of the warp lies beyond its
// screening radius, else its values into the tile through the sink.
__device__ __forceinline__ bool piece_live(const float4* __restrict__ rec, const double2* __restrict__ c64,
                                           const uint32_t* cand, int pi, double px, double py, double pz,
                                           bool valid, int4& meta, int& poff, double& dx, double& dy,
                                           double& dz, double& r2) {
    if (!((cand[pi >> 5] >> (pi & 31)) & 1u)) return false;
    meta = __ldg(reinterpret_cast<const int4*>(rec) + 3 * pi + 2);
    poff = __float_as_int(__ldg(rec + 3 * pi + 1).w);
    const double2 cxy = __ldg(c64 + 2 * pi), cza = __ldg(c64 + 2 * pi + 1);
    dx = px - cxy.x; dy = py - cxy.y; dz = pz - cza.x;
    r2 = dx * dx + dy * dy + dz * dz;
    return !__all_sync(0xffffffffu, !valid || cza.y * r2 > kScreenCut);
}

template <class T, bool GRAD, int LMAX, int PPT>
__global__ void __launch_bounds__(kTilePts / 32 * PPT * 32) ao_tile_kernel(TileArgs a) {
    constexpr int kNComp = GRAD ? 4 : 1;
    constexpr int kWarps = kTilePts / 32 * PPT;
    constexpr int kBufs = tile_bufs<T, GRAD>();
    extern __shared__ __align__(16) uint8_t tile_raw[];
    __shared__ double box[kTilePts / 32][6];
    T** rowp = reinterpret_cast<T**>(tile_raw);                       // [kNComp][kTilePts]
    T* const st0 = reinterpret_cast<T*>(tile_raw + kNComp * kTilePts * sizeof(T*));
    uint32_t* const cand = reinterpret_cast<uint32_t*>(st0 + kBufs * tile_elems<T, GRAD>());
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
    // the tiles start as zeros; the store pass zeroes every entry it reads
    for (size_t i = threadIdx.x; i < kBufs * tile_elems<T, GRAD>() * sizeof(T) / 16; i += blockDim.x)
        reinterpret_cast<uint4*>(st0)[i] = make_uint4(0u, 0u, 0u, 0u);
    tile_candidates(a.piece_c64, a.npieces, px, py, pz, valid, lanegrp == 0, warp / PPT, box, cand);
    for (int w = 0; w < a.nwin; ++w) {
        T* const st = st0 + (kBufs == 2 ? (w & 1) * tile_elems<T, GRAD>() : 0);
        const int eb = __ldg(a.win_begin + w * PPT + lanegrp), ee = __ldg(a.win_begin + w * PPT + lanegrp + 1);
        for (int e = eb; e < ee; ++e) {
            const int2 en = __ldg(a.win_entry + e);
            int4 meta; int poff; double dx, dy, dz, r2;
            if (!piece_live(a.piece_rec, a.piece_c64, cand, en.x, px, py, pz, valid, meta, poff, dx, dy, dz, r2))
                continue;
            WinSink<T> sink{st, p, en.y};
            eval_piece<T, GRAD, LMAX>(meta.x, static_cast<T>(dx), static_cast<T>(dy), static_cast<T>(dz),
                                      static_cast<T>(r2), packed_prims<T>(a.prims, poff), meta.y, meta.z, sink);
        }
        __syncthreads();
        // a warp takes whole point columns: it stores each component's row
        // segment and zeroes the column behind it
        const int ao0 = w * kWin, fill = min(kWin, a.nao - ao0);
        for (int pp = warp; pp < kTilePts; pp += kWarps) {
#pragma unroll
            for (int cc = 0; cc < kNComp; ++cc) {
                T* const row = rowp[cc * kTilePts + pp];
                T& slot = st[(cc * kWin + lane) * kTileStride + pp];
                const T v = slot;
                slot = T(0);
                if (row != nullptr && lane < fill) row[ao0 + lane] = v;
            }
        }
        if constexpr (kBufs == 1) __syncthreads();   // the tile is refilled next
    }
}

template <class T, bool GRAD, int LMAX, int PPT>
void launch_tile(const TileArgs& a, cudaStream_t s) {
    const int64_t nb = (a.n + kTilePts - 1) / kTilePts;
    require(nb < (1ll << 31), "too many grid points for one launch");
    constexpr int kNComp = GRAD ? 4 : 1;
    const size_t smem = tile_smem_bytes<T, GRAD>(kNComp * kTilePts, a.npieces);
    require(smem <= 227 * 1024, "basis too large for the tiled AO evaluator's shared memory");
    auto kern = ao_tile_kernel<T, GRAD, LMAX, PPT>;
    if (smem > 48 * 1024)
        ISDF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    kern<<<static_cast<unsigned>(nb), kTilePts / 32 * PPT * 32, smem, s>>>(a);
    ISDF_LAUNCH_CHECK();
}

// Values only, one warp per 32 points and no block barriers: the warp keeps a
// private padded tile [slot][point] of one AO window, takes as candidates the
// pieces whose FP64 screening radius reaches the bounding box of its points
// (lane = piece, a ballot per 32 pieces), and per window loads the window's
// entries with one coalesced load (lane = entry), keeps the candidates in a
// ballot mask and evaluates them one by one (lane = point, each warp-uniform
// piece screened as in ao_tile_kernel); then it stores its 32 aligned row
// segments (lane = slot) and zeroes the tile behind them.  Same values as
// ao_tile_kernel.  At C5 (FP64, 1.99 M points) the block form spent most of its
// stalls at the per-window barrier and on the per-entry record chains.
constexpr int kValWarps = 4;                      // independent warps per block
constexpr int kWarpTileStride = 33;               // padded point stride of the warp tile

template <class T>
struct WarpSink {
    T* st; int p, base;
    template <int C> __device__ __forceinline__ void put(int ao, T v) {
        static_assert(C == 0, "value tiles only");
        const int s = ao + base;
        if (static_cast<unsigned>(s) < static_cast<unsigned>(kWin)) st[s * kWarpTileStride + p] = v;
    }
};

template <class T>
size_t value_warp_bytes(int npieces) {
    const size_t b = kWin * kWarpTileStride * sizeof(T) + 4 * static_cast<size_t>((npieces + 31) / 32);
    return (b + 15) / 16 * 16;
}

template <class T, int LMAX>
__global__ void __launch_bounds__(kValWarps * 32, 6) ao_value_warp_kernel(TileArgs a, int warp_bytes) {
    extern __shared__ __align__(16) uint8_t warp_raw[];
    const int lane = threadIdx.x % 32, warp = threadIdx.x / 32;
    T* const st = reinterpret_cast<T*>(warp_raw + static_cast<size_t>(warp) * warp_bytes);
    uint32_t* const cand = reinterpret_cast<uint32_t*>(warp_raw + static_cast<size_t>(warp) * warp_bytes +
                                                       kWin * kWarpTileStride * sizeof(T));
    const int64_t g0 = (static_cast<int64_t>(blockIdx.x) * kValWarps + warp) * 32;
    if (g0 >= a.n) return;   // whole warps only; nothing below synchronises the block
    const int64_t g = g0 + lane;
    const bool valid = g < a.n;
    const double px = valid ? a.pts[3 * g] : 0.0, py = valid ? a.pts[3 * g + 1] : 0.0,
                 pz = valid ? a.pts[3 * g + 2] : 0.0;
    for (int i = lane; i < kWin * kWarpTileStride * static_cast<int>(sizeof(T)) / 16; i += 32)
        reinterpret_cast<uint4*>(st)[i] = make_uint4(0u, 0u, 0u, 0u);
    // candidates: the bounding box of the warp's valid points (every lane
    // holds it after the butterfly), widened by 1e-9 bohr
    double mid[3], hw[3];
    {
        const double pc[3] = {px, py, pz};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            double lo = valid ? pc[d] : INFINITY, hi = valid ? pc[d] : -INFINITY;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
                hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
            }
            mid[d] = 0.5 * (lo + hi);
            hw[d] = 0.5 * (hi - lo) + 1e-9;
        }
    }
    for (int k = 0; k < (a.npieces + 31) / 32; ++k) {
        const int pi = k * 32 + lane;
        bool c = false;
        if (pi < a.npieces) {
            const double2 cxy = __ldg(a.piece_c64 + 2 * pi), cza = __ldg(a.piece_c64 + 2 * pi + 1);
            const double ex = fmax(fabs(cxy.x - mid[0]) - hw[0], 0.0);
            const double ey = fmax(fabs(cxy.y - mid[1]) - hw[1], 0.0);
            const double ez = fmax(fabs(cza.x - mid[2]) - hw[2], 0.0);
            c = !(cza.y * (ex * ex + ey * ey + ez * ez) > kScreenCut);
        }
        const uint32_t m = __ballot_sync(0xffffffffu, c);
        if (lane == 0) cand[k] = m;
    }
    __syncwarp();
    const int np = a.n - g0 < 32 ? static_cast<int>(a.n - g0) : 32;
    for (int w = 0; w < a.nwin; ++w) {
        const int eb = __ldg(a.win_begin + w * a.lanes), ee = __ldg(a.win_begin + (w + 1) * a.lanes);
        for (int base = eb; base < ee; base += 32) {
            const int e = base + lane;
            const int2 en = e < ee ? __ldg(a.win_entry + e) : make_int2(0, 0);
            const bool c = e < ee && ((cand[en.x >> 5] >> (en.x & 31)) & 1u);
            // candidates one by one, the next one's record loaded while the
            // current one is evaluated
            uint32_t m = __ballot_sync(0xffffffffu, c);
            int4 meta_n{}; int poff_n = 0, off_n = 0; double2 cxy_n{}, cza_n{};
            auto fetch = [&](uint32_t mm) {
                const int k = __ffs(mm) - 1;
                const int pi = __shfl_sync(0xffffffffu, en.x, k);
                off_n = __shfl_sync(0xffffffffu, en.y, k);
                meta_n = __ldg(reinterpret_cast<const int4*>(a.piece_rec) + 3 * pi + 2);
                poff_n = __float_as_int(__ldg(a.piece_rec + 3 * pi + 1).w);
                cxy_n = __ldg(a.piece_c64 + 2 * pi);
                cza_n = __ldg(a.piece_c64 + 2 * pi + 1);
            };
            if (m != 0u) fetch(m);
            while (m != 0u) {
                const int4 meta = meta_n;
                const int poff = poff_n, off = off_n;
                const double2 cxy = cxy_n, cza = cza_n;
                m &= m - 1u;
                if (m != 0u) fetch(m);
                const double dx = px - cxy.x, dy = py - cxy.y, dz = pz - cza.x;
                const double r2 = dx * dx + dy * dy + dz * dz;
                if (__all_sync(0xffffffffu, !valid || cza.y * r2 > kScreenCut)) continue;
                WarpSink<T> sink{st, lane, off};
                eval_piece<T, false, LMAX>(meta.x, static_cast<T>(dx), static_cast<T>(dy), static_cast<T>(dz),
                                           static_cast<T>(r2), packed_prims<T>(a.prims, poff), meta.y, meta.z, sink);
            }
        }
        __syncwarp();
        const int ao0 = w * kWin, fill = min(kWin, a.nao - ao0);
        T* const out = static_cast<T*>(a.val) + g0 * a.ld + ao0 + lane;
#pragma unroll 4
        for (int pp = 0; pp < 32; ++pp) {
            T& slot = st[lane * kWarpTileStride + pp];
            const T v = slot;
            slot = T(0);
            if (pp < np && lane < fill) out[pp * a.ld] = v;
        }
        __syncwarp();
    }
}

template <class T, int LMAX>
void launch_value_warp(const TileArgs& a, cudaStream_t s) {
    const int64_t nb = (a.n + kValWarps * 32 - 1) / (kValWarps * 32);
    require(nb < (1ll << 31), "too many grid points for one launch");
    const size_t wb = value_warp_bytes<T>(a.npieces);
    const size_t smem = kValWarps * wb;
    require(smem <= 227 * 1024, "basis too large for the tiled AO evaluator's shared memory");
    auto kern = ao_value_warp_kernel<T, LMAX>;
    if (smem > 48 * 1024)
        ISDF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    kern<<<static_cast<unsigned>(nb), kValWarps * 32, smem, s>>>(a, static_cast<int>(wb));
    ISDF_LAUNCH_CHECK();
}

template <class T, bool GRAD>
void launch_tile_l(const Context& c, const TileArgs& a, cudaStream_t s) {
    // the warp form has one warp per 32 points, a sixth of the block form's
    // warps: it takes launches of at least two waves of its resident blocks
    // (the FP64 fit's 43 690-point chunks at C5 ran 16 ms longer per step on it)
    const bool warp_form = a.n >= static_cast<int64_t>(c.nsm) * 2 * 6 * kValWarps * 32;
    if constexpr (!GRAD) {
        if (!warp_form) {
            if (c.lmax <= 2) launch_tile<T, false, 2, 6>(a, s);
            else if (c.lmax <= 4) launch_tile<T, false, 4, 2>(a, s);
            else launch_tile<T, false, kMaxL, 2>(a, s);
            return;
        }
        if (c.lmax <= 2) launch_value_warp<T, 2>(a, s);
        else if (c.lmax <= 4) launch_value_warp<T, 4>(a, s);
        else launch_value_warp<T, kMaxL>(a, s);
    } else {
        // lane counts as in piece_lanes_for_lmax()
        if (c.lmax <= 2) launch_tile<T, GRAD, 2, 6>(a, s);
        else if (c.lmax <= 4) launch_tile<T, GRAD, 4, 2>(a, s);
        else launch_tile<T, GRAD, kMaxL, 2>(a, s);
    }
}

// Tiled axis features F[p*ld + offset[a] + ao] = scale[a] * comp_a(p, ao): the
// layout of ao_tile_kernel (64 points per block, piece lanes of the window
// layout, a padded shared tile [comp][slot][point] per AO window), with the
// points gathered through `index`, one aligned row segment per (axis entry,
// point) and window, and the per-component sums of squares of the points with
// nonzero weight accumulated by the evaluating threads (FP64).
struct AxisTileArgs {
    const float4* piece_rec; const double2* piece_c64; const void* prims;   // packed piece records
    const int2* win_entry; const int* win_begin; int nwin, nao, npieces;     // window layout
    const double* pts; const int64_t* index; int64_t n; const double* weights;
    void* out; int64_t ld; double* sumsq;
    int nent; int comp[16]; int off[16]; double scale[16];   // the non-occupied axis entries
};

template <class T, bool GRAD, int LMAX, int PPT>
__global__ void __launch_bounds__(kTilePts / 32 * PPT * 32) axis_tile_kernel(AxisTileArgs a) {
    constexpr int kNComp = GRAD ? 4 : 1;
    constexpr int kWarps = kTilePts / 32 * PPT;
    constexpr int kBufs = tile_bufs<T, GRAD>();
    extern __shared__ __align__(16) uint8_t tile_raw[];
    __shared__ double box[kTilePts / 32][6];
    __shared__ double red[kWarps][4];
    T** rowp = reinterpret_cast<T**>(tile_raw);                       // [kTilePts]
    T* const st0 = reinterpret_cast<T*>(tile_raw + kTilePts * sizeof(T*));
    uint32_t* const cand = reinterpret_cast<uint32_t*>(st0 + kBufs * tile_elems<T, GRAD>());
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
    for (size_t i = threadIdx.x; i < kBufs * tile_elems<T, GRAD>() * sizeof(T) / 16; i += blockDim.x)
        reinterpret_cast<uint4*>(st0)[i] = make_uint4(0u, 0u, 0u, 0u);
    tile_candidates(a.piece_c64, a.npieces, px, py, pz, valid, lanegrp == 0, warp / PPT, box, cand);
    double sq[4] = {0.0, 0.0, 0.0, 0.0};
    for (int w = 0; w < a.nwin; ++w) {
        T* const st = st0 + (kBufs == 2 ? (w & 1) * tile_elems<T, GRAD>() : 0);
        const int eb = __ldg(a.win_begin + w * PPT + lanegrp), ee = __ldg(a.win_begin + w * PPT + lanegrp + 1);
        for (int e = eb; e < ee; ++e) {
            const int2 en = __ldg(a.win_entry + e);
            int4 meta; int poff; double dx, dy, dz, r2;
            if (!piece_live(a.piece_rec, a.piece_c64, cand, en.x, px, py, pz, valid, meta, poff, dx, dy, dz, r2))
                continue;
            WinSqSink<T> sink{st, p, en.y, count, {0.0, 0.0, 0.0, 0.0}};
            eval_piece<T, GRAD, LMAX>(meta.x, static_cast<T>(dx), static_cast<T>(dy), static_cast<T>(dz),
                                      static_cast<T>(r2), packed_prims<T>(a.prims, poff), meta.y, meta.z, sink);
#pragma unroll
            for (int cc = 0; cc < 4; ++cc) sq[cc] += sink.sq[cc];
        }
        __syncthreads();
        // a warp takes whole point columns: every axis entry's row segment,
        // then the column's components zeroed
        const int ao0 = w * kWin, fill = min(kWin, a.nao - ao0);
        for (int pp = warp; pp < kTilePts; pp += kWarps) {
            T* const row = rowp[pp];
            if (row != nullptr && lane < fill)
                for (int e = 0; e < a.nent; ++e)
                    row[a.off[e] + ao0 + lane] =
                        static_cast<T>(a.scale[e] * static_cast<double>(st[(a.comp[e] * kWin + lane) * kTileStride + pp]));
#pragma unroll
            for (int cc = 0; cc < kNComp; ++cc) st[(cc * kWin + lane) * kTileStride + pp] = T(0);
        }
        if constexpr (kBufs == 1) __syncthreads();   // the tile is refilled next
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
    const size_t smem = tile_smem_bytes<T, GRAD>(kTilePts, a.npieces);
    require(smem <= 227 * 1024, "basis too large for the tiled AO evaluator's shared memory");
    auto kern = axis_tile_kernel<T, GRAD, LMAX, PPT>;
    if (smem > 48 * 1024)
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

void build_window_layout(Context& c) {
    const int lanes = c.piece_lanes;
    const int nwin = (c.nao + kWin - 1) / kWin;
    std::vector<std::vector<int2>> per_win(nwin);
    for (int i = 0; i < c.npieces; ++i) {
        const int4 pc = c.h_pieces[i];
        const ShellDesc& sh = c.shells[pc.x];
        const int ns = 2 * sh.l + 1;
        const int a0 = sh.ao_off + pc.y * ns, a1 = a0 + pc.z * ns;
        for (int w = a0 / kWin; w * kWin < a1; ++w) per_win[w].push_back(make_int2(i, a0 - w * kWin));
    }
    // balance each window's pieces over the lanes (longest first onto the
    // least-loaded lane) with the chunk layout's estimate of their cost
    auto cost = [&](const int2& e) {
        const int4 pc = c.h_pieces[e.x];
        const ShellDesc& sh = c.shells[pc.x];
        return 6 + sh.nprim * (2 + pc.z) + pc.z * (2 * sh.l + 1) * 3;
    };
    std::vector<int2> entries;
    std::vector<int> begin;
    for (const auto& win : per_win) {
        std::vector<int> order(win.size());
        for (size_t i = 0; i < order.size(); ++i) order[i] = static_cast<int>(i);
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cost(win[x]) > cost(win[y]); });
        std::vector<std::vector<int2>> per_lane(lanes);
        std::vector<int> load(lanes, 0);
        for (int i : order) {
            const int l = static_cast<int>(std::min_element(load.begin(), load.end()) - load.begin());
            per_lane[l].push_back(win[i]);
            load[l] += cost(win[i]);
        }
        for (int l = 0; l < lanes; ++l) {
            begin.push_back(static_cast<int>(entries.size()));
            entries.insert(entries.end(), per_lane[l].begin(), per_lane[l].end());
        }
    }
    begin.push_back(static_cast<int>(entries.size()));
    if (entries.empty()) entries.push_back(make_int2(0, 0));
    c.nwin = nwin;
    ISDF_CUDA(cudaMalloc(reinterpret_cast<void**>(&c.d_win_entry), entries.size() * sizeof(int2)));
    ISDF_CUDA(cudaMemcpy(c.d_win_entry, entries.data(), entries.size() * sizeof(int2), cudaMemcpyHostToDevice));
    ISDF_CUDA(cudaMalloc(reinterpret_cast<void**>(&c.d_win_begin), begin.size() * sizeof(int)));
    ISDF_CUDA(cudaMemcpy(c.d_win_begin, begin.data(), begin.size() * sizeof(int), cudaMemcpyHostToDevice));
}

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
        TileArgs a{c.d_piece_rec, c.d_piece_c64, prims_of<T>(c), c.d_win_entry, c.d_win_begin, c.nwin, c.nao,
                   c.npieces, c.piece_lanes, pts, n, ld, out_val, out_grad, out_val != nullptr};
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
        // tiled: one aligned row segment per (axis entry, point) and AO window
        AxisTileArgs ta{c.d_piece_rec, c.d_piece_c64, prims_of<T>(c), c.d_win_entry, c.d_win_begin, c.nwin, c.nao,
                        c.npieces, pts, index, n, weights, out, ld, sumsq, 0, {}, {}, {}};
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
