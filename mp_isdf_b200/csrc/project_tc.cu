// Fused AO evaluation + tensor-core projection (sm_100a, tcgen05).
//
// For a tile of 128 grid points (one UMMA M=128 tile) the CTA evaluates the
// needed AO components (value and/or d/dx, d/dy, d/dz) in FP32, one K-chunk of
// 32 AO slots at a time, splits them into BF16 hi + lo parts and multiplies them on
// the tensor cores with a pre-split BF16 hi + lo weight matrix:
//     P[g][a][n] = sum_mu comp_a(g, mu) W_a[mu][n]
//                ~ A_hi B_hi + A_hi B_lo + A_lo B_hi   (FP32 accumulate in TMEM)
// One accumulator of NT columns per axis entry a.  Nothing of the AO matrix
// is written to HBM.  Used for
//   * the Khatri-Rao sketch projections f_g . [u_s v_s] (all selected axes);
//   * the fit Gram G[g][k] = phi_g . phi_a(k) (AO values only).
// K-chunks hold whole contraction groups ("pieces") padded to 32 slots, so a
// producer thread evaluates each (point, piece) once, writes its values at
// fixed slots and needs no range checks.  A piece is written as zeros for a
// warp of points that all lie beyond its shell's FP32 screening radius (no
// dropped value or gradient above kScreenFp32).
// The per-component sums of squares of the FP32 values are accumulated (FP32
// per piece, FP64 across pieces) for the multi-axis Frobenius scales and the
// error bounds.
//
// Warp roles: 4*PPT producer warps evaluate AOs (thread = point x piece lane),
// convert to the UMMA operand layout and, warps 0-3, run the TMEM epilogue;
// one warp issues the MMAs; one warp streams W chunks by bulk copy.  The FP32
// staging buffer lets chunk c+1 be evaluated while the MMAs of chunk c run.
#include "ao_device.cuh"
#include "isdf_project.h"
#include "isdf_reduce.cuh"
#include "tc_sm100.cuh"

#include <cuda_bf16.h>

#include <algorithm>
#include <cstring>
#include <type_traits>
#include <vector>

namespace isdf {

namespace {

inline float __int_as_float_host(int v) {
    float f;
    std::memcpy(&f, &v, sizeof(f));
    return f;
}

constexpr int kRows = 128;            // points per tile (UMMA M)
constexpr int kChunk = 32;            // AO slots per K-chunk
constexpr uint32_t kTileA = kRows * kChunk * 2;       // bytes of one BF16 A tile (8 KB)
constexpr uint32_t kLboA = (kRows / 8) * 128;          // K-adjacent core matrices
constexpr uint32_t kSboA = 128;                        // M-adjacent core matrices
constexpr int kLiveWords = 8;          // chunk-liveness bits per tile (up to 256 chunks)
constexpr int kCandWords = 32;         // piece-candidate bits per tile (up to 1024 pieces)
static_assert(128 + 4 * kCandWords <= 256, "candidate bits exceed the barrier area");
constexpr float kBoxMargin = 1e-3f;    // bohr: covers FP32 rounding of points and centres

// Writes the component values of one piece into the FP32 staging buffer
// stage[comp][slot][point]; slot = ao + base.
struct StageSink {
    float* stage;
    int p, base;
    float sq[4];
    template <int C>
    __device__ __forceinline__ void put(int ao, float v) {
        stage[(C * kChunk + ao + base) * kRows + p] = v;
        sq[C] += v * v;
    }
};

__device__ __forceinline__ uint32_t bf162_bits(__nv_bfloat162 v) {
    uint32_t u;
    memcpy(&u, &v, sizeof(u));
    return u;
}

// hi = bf16(x), lo = bf16(x - hi) (round to nearest) for 8 values, packed for
// two 16-byte stores; pairs are converted with one packed instruction each.
__device__ __forceinline__ void split8(const float* x, uint4& hi, uint4& lo) {
    uint32_t h[4], l[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        h[i] = bf162_bits(__floats2bfloat162_rn(x[2 * i], x[2 * i + 1]));
        const float h0 = __uint_as_float(h[i] << 16), h1 = __uint_as_float(h[i] & 0xffff0000u);
        l[i] = bf162_bits(__floats2bfloat162_rn(x[2 * i] - h0, x[2 * i + 1] - h1));
    }
    hi = make_uint4(h[0], h[1], h[2], h[3]);
    lo = make_uint4(l[0], l[1], l[2], l[3]);
}

// The remainder r = bf16(x - hi - lo) of that split: x - hi and (x - hi) - lo
// are exact in FP32 and the remainder has at most 8 significant bits, so
// hi + lo + r == x exactly.
__device__ __forceinline__ uint4 remainder8(const float* x, const uint4& hi, const uint4& lo) {
    const uint32_t h[4] = {hi.x, hi.y, hi.z, hi.w}, l[4] = {lo.x, lo.y, lo.z, lo.w};
    uint32_t r[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float h0 = __uint_as_float(h[i] << 16), h1 = __uint_as_float(h[i] & 0xffff0000u);
        const float l0 = __uint_as_float(l[i] << 16), l1 = __uint_as_float(l[i] & 0xffff0000u);
        r[i] = bf162_bits(__floats2bfloat162_rn((x[2 * i] - h0) - l0, (x[2 * i + 1] - h1) - l1));
    }
    return make_uint4(r[0], r[1], r[2], r[3]);
}

__device__ __forceinline__ void named_bar_sync(int id, int count) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

template <int PPT>
struct Roles {
    static constexpr int kProducers = kRows * PPT;
    static constexpr int kThreads = kProducers + 64;
};

// Shared-memory plan of one instantiation: A tiles, 1 or 2 W stages (2 when
// they fit), two FP32 staging buffers and the barriers.
template <int NAX, int NT, bool GRAD>
struct Smem {
    static constexpr uint32_t kTileB = NT * kChunk * 2;
    static constexpr uint32_t kABytes = NAX * 2 * kTileA;
    static constexpr uint32_t kBStage = NAX * 2 * kTileB;
    static constexpr int kNComp = GRAD ? 4 : 1;
    static constexpr uint32_t kStage = kNComp * kChunk * kRows * 4;
    static constexpr uint32_t kBarBytes = 256;
    static constexpr uint32_t kLimit = 232448;   // opt-in shared memory per block
    static constexpr int kBStages =
        (kABytes + 2 * kBStage + 2 * kStage + kBarBytes + 1024 <= kLimit) ? 2 : 1;
    static constexpr size_t kBytes = kABytes + kBStages * kBStage + 2 * kStage + kBarBytes + 1024;
    static_assert(kABytes + kBStage + 2 * kStage + kBarBytes + 1024 <= kLimit, "shared memory plan too large");
};

template <int NAX, int NT, bool GRAD, int LMAX, int PPT>
__global__ void __launch_bounds__(Roles<PPT>::kThreads, 1)
project_tc_kernel(ProjectArgs args) {
    using SM = Smem<NAX, NT, GRAD>;
    constexpr int kProducers = Roles<PPT>::kProducers;
    constexpr int kThreads = Roles<PPT>::kThreads;
    constexpr uint32_t kTileB = SM::kTileB;
    constexpr uint32_t kBStage = SM::kBStage;
    constexpr int kBStages = SM::kBStages;
    constexpr int kNComp = SM::kNComp;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    // layout: [A: NAX x (hi, lo) tiles][B: kBStages x NAX x (hi, lo)][2 x FP32 staging][barriers]
    uint8_t* sA = smem_raw;
    uint8_t* sB = sA + SM::kABytes;
    float* sStage0 = reinterpret_cast<float*>(sB + kBStages * kBStage);
    uint64_t* bars = reinterpret_cast<uint64_t*>(reinterpret_cast<uint8_t*>(sStage0) + 2 * SM::kStage);
    uint64_t* a_full = bars + 0;
    uint64_t* a_empty = bars + 1;
    uint64_t* b_full = bars + 2;     // [kBStages]
    uint64_t* b_empty = bars + 4;    // [kBStages]
    uint64_t* acc_full = bars + 6;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 7);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(bars + 8);
    volatile int* prod_abort = reinterpret_cast<volatile int*>(bars + 9);   // [2]
    // pieces of the current tile that are not screened (bytes 128-255 of the
    // barrier area: static shared memory stays within its 1 KB, so the
    // 1 KB-aligned dynamic plan still fits)
    uint32_t* cand_s = reinterpret_cast<uint32_t*>(bars + 16);   // [kCandWords]
    __shared__ double red[kThreads / 32][4];
    __shared__ uint32_t live_s[kLiveWords];   // chunks of the current tile that are not screened
    __shared__ float tile_box[4][6];          // per point warp: coordinate minima, maxima

    const int tid = threadIdx.x;
    const int warp = tid / 32, lane = tid % 32;
    constexpr int kMmaWarp = kProducers / 32;
    constexpr uint32_t kTmemCols = (NAX * NT <= 32) ? 32 : (NAX * NT <= 64) ? 64
                                   : (NAX * NT <= 128) ? 128 : (NAX * NT <= 256) ? 256 : 512;
    static_assert(NAX * NT <= 512, "accumulators exceed TMEM");

    if (tid == 0) {
        tc::mbar_init(a_full, kProducers);
        // released by the MMAs' commit and, when tiles are stored, by the store's read
        tc::mbar_init(a_empty, args.a_store ? 2 : 1);
        for (int i = 0; i < kBStages; ++i) {
            tc::mbar_init(&b_full[i], 1);
            tc::mbar_init(&b_empty[i], 1);
        }
        tc::mbar_init(acc_full, 1);
        *abort_flag = 0;
        prod_abort[0] = 0;
        prod_abort[1] = 0;
        tc::mbar_init_fence();
    }
    if (warp == 0) tc::tmem_alloc(tmem_slot, kTmemCols);
    // with zero-behind conversion the staging buffers start as zeros and stay
    // zero wherever nothing is evaluated
    if (args.zero_behind && warp < kMmaWarp)
        for (uint32_t u = tid; u < 2 * SM::kStage / 16; u += kProducers)
            reinterpret_cast<uint4*>(sStage0)[u] = make_uint4(0u, 0u, 0u, 0u);
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;

    const int64_t n = args.n;
    const int64_t ntiles = (n + kRows - 1) / kRows;
    const int nchunks = args.nchunks;
    double sq[4] = {0, 0, 0, 0};

    auto fail_wait = [&](int where) {
        atomicOr(args.error, 1 << where);
        *abort_flag = 1;
    };

    if (warp < kMmaWarp) {
        // ------------------------------ producers ------------------------------
        // Chunk q is evaluated into staging buffer q & 1; one barrier per chunk
        // separates evaluation from conversion, and the next chunk's evaluation
        // (other buffer) needs no barrier against this chunk's conversion.
        const int p = tid & (kRows - 1);
        const int lanegrp = tid / kRows;     // piece lane of this thread
        uint32_t q = 0;   // chunk sequence number of this CTA
        uint32_t t = 0;   // tile sequence number of this CTA
        bool stop = false;
        bool a_zero = false;   // the A tiles hold zeros from a screened chunk
        const bool use_live = args.piece_chunk != nullptr && nchunks <= 32 * kLiveWords;
        const bool zb = args.zero_behind != 0;
        // per-piece candidate bits of the tile: a piece outside them is skipped
        // without reading its record (only with zero-behind conversion, which
        // needs no zero fill for it)
        const bool use_cand = use_live && zb && args.npieces <= 32 * kCandWords;
        for (int64_t tile = blockIdx.x; tile < ntiles && !stop; tile += gridDim.x, ++t) {
            const int64_t g = tile * kRows + p;
            const bool valid = g < n;
            // point as FP32 hi + lo: offsets from a shell centre are formed in FP32
            // to about one rounding of the offset itself
            float pxh = 0.f, pyh = 0.f, pzh = 0.f, pxl = 0.f, pyl = 0.f, pzl = 0.f;
            bool count = false;
            if (valid) {
                const int64_t gi = args.index ? args.index[g] : g;
                const double px = args.pts[3 * gi], py = args.pts[3 * gi + 1], pz = args.pts[3 * gi + 2];
                pxh = static_cast<float>(px); pyh = static_cast<float>(py); pzh = static_cast<float>(pz);
                pxl = static_cast<float>(px - pxh); pyl = static_cast<float>(py - pyh); pzl = static_cast<float>(pz - pzh);
                count = args.sumsq && (args.weights == nullptr || args.weights[gi] != 0.0);
            }
            // Chunks screened for the whole tile: a chunk every piece of which
            // lies beyond its FP32 screening radius from the tile's bounding box
            // is zero at every point of the tile (each warp's own test would drop
            // every piece); it is neither evaluated nor converted, and its A
            // tiles are written as zeros.
            if (use_live) {
                if (tid < kLiveWords) live_s[tid] = 0u;
                if (tid < kCandWords) cand_s[tid] = 0u;
                if (tid < kRows) {   // warps 0-3 hold each of the tile's points once
                    const float pc[3] = {pxh + pxl, pyh + pyl, pzh + pzl};
                    float lo3[3], hi3[3];
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        lo3[d] = valid ? pc[d] : INFINITY;
                        hi3[d] = valid ? pc[d] : -INFINITY;
#pragma unroll
                        for (int o = 16; o > 0; o >>= 1) {
                            lo3[d] = fminf(lo3[d], __shfl_xor_sync(0xffffffffu, lo3[d], o));
                            hi3[d] = fmaxf(hi3[d], __shfl_xor_sync(0xffffffffu, hi3[d], o));
                        }
                    }
                    if (lane == 0)
#pragma unroll
                        for (int d = 0; d < 3; ++d) { tile_box[warp][d] = lo3[d]; tile_box[warp][3 + d] = hi3[d]; }
                }
                named_bar_sync(1, kProducers);
                float mid[3], half[3];
                bool any = true;
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    float lo = tile_box[0][d], hi = tile_box[0][3 + d];
#pragma unroll
                    for (int w = 1; w < 4; ++w) { lo = fminf(lo, tile_box[w][d]); hi = fmaxf(hi, tile_box[w][3 + d]); }
                    any = any && lo <= hi;
                    mid[d] = 0.5f * (lo + hi);
                    half[d] = 0.5f * (hi - lo) + kBoxMargin;
                }
                if (any)
                    for (int pi = tid; pi < args.npieces; pi += kProducers) {
                        const float4 ch = __ldg(args.piece_rec + 3 * pi), cl = __ldg(args.piece_rec + 3 * pi + 1);
                        const float ex = fmaxf(fabsf((ch.x + cl.x) - mid[0]) - half[0], 0.f);
                        const float ey = fmaxf(fabsf((ch.y + cl.y) - mid[1]) - half[1], 0.f);
                        const float ez = fmaxf(fabsf((ch.z + cl.z) - mid[2]) - half[2], 0.f);
                        if (!(ch.w * (ex * ex + ey * ey + ez * ez) > static_cast<float>(kExpCut))) {
                            const int pc = __ldg(args.piece_chunk + pi);
                            atomicOr(&live_s[pc >> 5], 1u << (pc & 31));
                            if (pi < 32 * kCandWords) atomicOr(&cand_s[pi >> 5], 1u << (pi & 31));
                        }
                    }
                named_bar_sync(1, kProducers);
            }
            float psq[4] = {0.f, 0.f, 0.f, 0.f};
            // the chunk's piece range and fill are read one chunk ahead
            int pb_n = args.lane_begin[lanegrp], pe_n = args.lane_begin[lanegrp + 1], fill_n = args.chunk_fill[0];
            for (int c = 0; c < nchunks; ++c, ++q) {
                float* sStage = sStage0 + (q & 1) * (SM::kStage / 4);
                const int pb = pb_n, pe = pe_n, fill = fill_n;
                if (c + 1 < nchunks) {
                    pb_n = __ldg(args.lane_begin + (c + 1) * PPT + lanegrp);
                    pe_n = __ldg(args.lane_begin + (c + 1) * PPT + lanegrp + 1);
                    fill_n = __ldg(args.chunk_fill + c + 1);
                }
                const bool live = !use_live || ((live_s[c >> 5] >> (c & 31)) & 1u);
                if (args.chunk_zero && tid == 0)
                    args.chunk_zero[static_cast<size_t>(tile) * nchunks + c] = live ? 0 : 1;
                // 1. evaluate this chunk's pieces into the FP32 staging buffer
                if (live && !zb)
                    for (int k = (valid ? fill : 0) + lanegrp; k < kChunk; k += PPT)
#pragma unroll
                        for (int cc = 0; cc < kNComp; ++cc) sStage[(cc * kChunk + k) * kRows + p] = 0.f;
                float csq[4] = {0.f, 0.f, 0.f, 0.f};
                if (valid && live) {
                    for (int pi = pb; pi < pe; ++pi) {
                        if (use_cand && !((cand_s[pi >> 5] >> (pi & 31)) & 1u)) continue;   // warp-uniform
                        // one packed record per piece: centre (hi, lo), smallest exponent,
                        // primitive offset, l, primitive and contraction counts, first slot
                        const float4 ch = __ldg(args.piece_rec + 3 * pi), cl = __ldg(args.piece_rec + 3 * pi + 1);
                        const int4 meta = __ldg(reinterpret_cast<const int4*>(args.piece_rec) + 3 * pi + 2);
                        const int l = meta.x, nprim = meta.y, nc = meta.z, slot0 = meta.w;
                        const int ns = 2 * l + 1;
                        const float dx = (pxh - ch.x) + (pxl - cl.x);
                        const float dy = (pyh - ch.y) + (pyl - cl.y);
                        const float dz = (pzh - ch.z) + (pzl - cl.z);
                        const float r2 = dx * dx + dy * dy + dz * dz;
                        // ch.w is the shell's FP32 screening exponent: where it puts
                        // every point of the warp beyond kExpCut, no value or gradient
                        // of the piece exceeds kScreenFp32 there (the mixed form's error
                        // bounds carry that as an absolute term); taken only for the
                        // whole warp, so the evaluation does not split
                        if (__all_sync(__activemask(), ch.w * r2 > static_cast<float>(kExpCut))) {
                            if (!zb)
                                for (int k = slot0; k < slot0 + nc * ns; ++k)
#pragma unroll
                                for (int cc = 0; cc < kNComp; ++cc) sStage[(cc * kChunk + k) * kRows + p] = 0.f;
                            continue;
                        }
                        StageSink sink{sStage, p, slot0, {0.f, 0.f, 0.f, 0.f}};
                        eval_piece<float, GRAD, LMAX>(l, dx, dy, dz, r2, args.piece_prim + __float_as_int(cl.w), nprim,
                                                      nc, sink);
#pragma unroll
                        for (int cc = 0; cc < 4; ++cc) csq[cc] += sink.sq[cc];
                    }
                }
#pragma unroll
                for (int cc = 0; cc < 4; ++cc) {
                    if (count) sq[cc] += csq[cc];
                    psq[cc] += csq[cc];
                }
                // uniform abort decision: one producer samples the flag before the
                // barrier (alternating slots, so a late reader sees its chunk's value)
                if (tid == 0) prod_abort[q & 1] = *abort_flag;
                named_bar_sync(1, kProducers);
                if (prod_abort[q & 1]) { stop = true; break; }
                // 2. wait until the previous chunk's MMAs (and tile store) released A
                if (q > 0 && !tc::mbar_wait(a_empty, (q - 1) & 1)) fail_wait(0);
                // 3. convert staging -> BF16 hi/lo A tiles (UMMA interleaved K-major);
                // a screened chunk leaves zeros (A and, when kept, its remainder tile)
                if (!live) {
                    if (!a_zero)
                        for (uint32_t u = tid; u < NAX * 2 * kTileA / 16; u += kProducers)
                            *reinterpret_cast<uint4*>(sA + 16 * u) = make_uint4(0u, 0u, 0u, 0u);
                    a_zero = true;
                    if (args.a_store_r)
                        for (uint32_t u = tid; u < kTileA / 16; u += kProducers)
                            *reinterpret_cast<uint4*>(args.a_store_r + (static_cast<size_t>(tile) * nchunks + c) * kTileA +
                                                      16 * u) = make_uint4(0u, 0u, 0u, 0u);
                } else {
                    a_zero = false;
                }
                for (int u = tid; live && u < kRows * NAX * (kChunk / 8); u += kProducers) {
                    const int row = u % kRows;
                    const int rest = u / kRows;
                    const int kg = rest % (kChunk / 8);
                    const int a = rest / (kChunk / 8);
                    const int slot = GRAD ? args.axis_comp[a] : 0;
                    float x[8];
#pragma unroll
                    for (int i = 0; i < 8; ++i) x[i] = sStage[(slot * kChunk + kg * 8 + i) * kRows + row];
                    if (zb)
#pragma unroll
                        for (int i = 0; i < 8; ++i) sStage[(slot * kChunk + kg * 8 + i) * kRows + row] = 0.f;
                    uint4 hi, lo;
                    split8(x, hi, lo);
                    const uint32_t off = tc::interleaved_offset(row, kg * 8, kLboA, kSboA);
                    *reinterpret_cast<uint4*>(sA + (a * 2 + 0) * kTileA + off) = hi;
                    *reinterpret_cast<uint4*>(sA + (a * 2 + 1) * kTileA + off) = lo;
                    if (args.a_store_r && a == args.store_axis)   // warp-uniform: a is fixed per 128 u
                        *reinterpret_cast<uint4*>(args.a_store_r + (static_cast<size_t>(tile) * nchunks + c) * kTileA +
                                                  off) = remainder8(x, hi, lo);
                }
                tc::fence_proxy_async_smem();
                tc::mbar_arrive(a_full);
            }
            if (stop) break;
            // per-point sums of squares of each component (the piece lanes add up)
            if (args.point_sq && valid)
                for (int cc = 0; cc < 4; ++cc)
                    if ((args.comp_mask >> cc) & 1) atomicAdd(&args.point_sq[g * 4 + cc], psq[cc]);
            // 4. epilogue over every producer warp: a warp reads TMEM lane quarter
            // warp % 4 and takes every PPT-th group of 16 accumulator columns
            // (groups past nout are never read).  The next tile's first MMA waits
            // for every producer's arrival, so it cannot overwrite the
            // accumulators before they are read here.
            constexpr int kGroups = NT / 16;
            if ((warp >> 2) < NAX * kGroups) {
                if (!tc::mbar_wait(acc_full, t & 1)) fail_wait(1);
                tc::tc_fence_after();
                const int quarter = warp & 3;
                const int row = quarter * 32 + lane;
                const int64_t gg = tile * kRows + row;
                for (int gi = warp >> 2; gi < NAX * kGroups; gi += PPT) {
                    const int a = gi / kGroups, c0 = (gi % kGroups) * 16;
                    if (c0 >= args.nout) continue;
                    uint32_t r[16];
                    tc::tmem_ld16(tmem_base + (static_cast<uint32_t>(quarter * 32) << 16) +
                                      static_cast<uint32_t>(a * NT + c0), r);
                    tc::tmem_ld_wait();
                    if (gg < n) {
                        const int64_t cs = args.col_stride;
                        float* out = args.out + gg * args.ld_out + (a * args.nout + c0) * cs;
#pragma unroll
                        for (int i = 0; i < 16; ++i)
                            if (c0 + i < args.nout) out[i * cs] = __uint_as_float(r[i]);
                    }
                }
                tc::tc_fence_before();
            }
        }
    } else if (warp == kMmaWarp) {
        // ------------------------------ MMA issuer ------------------------------
        if (lane == 0) {
            constexpr uint32_t idesc = tc::idesc_bf16_f32(kRows, NT);
            constexpr uint32_t kLboB = (NT / 8) * 128;
            // The operand descriptors are affine in the tile offsets: a base
            // descriptor plus (byte offset >> 4) in its start-address field
            // (bits 0-13; shared addresses stay below 2^18, so nothing carries
            // out of the field).
            const uint64_t dA0 = tc::smem_desc_kmajor_noswizzle(tc::smem_addr(sA), kLboA, kSboA);
            const uint64_t dB00 = tc::smem_desc_kmajor_noswizzle(tc::smem_addr(sB), kLboB, 128);
            const uint64_t dB01 = tc::smem_desc_kmajor_noswizzle(tc::smem_addr(sB + (kBStages - 1) * kBStage), kLboB, 128);
            uint32_t q = 0;
            bool ok = true;
            for (int64_t tile = blockIdx.x; tile < ntiles && ok && !*abort_flag; tile += gridDim.x) {
                for (int c = 0; c < nchunks; ++c, ++q) {
                    const int s = q % kBStages;
                    if (!tc::mbar_wait(&b_full[s], (q / kBStages) & 1)) { fail_wait(2); ok = false; break; }
                    if (!tc::mbar_wait(a_full, q & 1)) { fail_wait(3); ok = false; break; }
                    tc::tc_fence_after();
                    const uint64_t dB0 = s == 0 ? dB00 : dB01;
                    const uint32_t acc0 = c == 0 ? 0u : 1u;
#pragma unroll
                    for (int a = 0; a < NAX; ++a) {
                        const uint32_t d = tmem_base + static_cast<uint32_t>(a * NT);
#pragma unroll
                        for (int kk = 0; kk < kChunk / 16; ++kk) {
                            const uint64_t dah = dA0 + (((a * 2 + 0) * kTileA + kk * 2 * kLboA) >> 4);
                            const uint64_t dal = dA0 + (((a * 2 + 1) * kTileA + kk * 2 * kLboA) >> 4);
                            const uint64_t dbh = dB0 + (((a * 2 + 0) * kTileB + kk * 2 * kLboB) >> 4);
                            const uint64_t dbl = dB0 + (((a * 2 + 1) * kTileB + kk * 2 * kLboB) >> 4);
                            tc::mma_bf16(d, dah, dbh, idesc, kk == 0 ? acc0 : 1u);
                            tc::mma_bf16(d, dah, dbl, idesc, 1u);
                            tc::mma_bf16(d, dal, dbh, idesc, 1u);
                        }
                    }
                    tc::mma_commit(a_empty);
                    tc::mma_commit(&b_empty[s]);
                    if (args.a_store) {
                        // keep the (hi, lo) tiles of one axis entry in HBM for a later
                        // GEMM; A is released once the copy has read it
                        tc::bulk_s2g(args.a_store + (static_cast<size_t>(tile) * nchunks + c) * 2 * kTileA,
                                     sA + args.store_axis * 2 * kTileA, 2 * kTileA);
                        tc::bulk_commit();
                        tc::bulk_wait_read_all();
                        tc::mbar_arrive(a_empty);
                    }
                }
                if (ok) tc::mma_commit(acc_full);
            }
            if (args.a_store) tc::bulk_wait_all();
        }
        __syncwarp();
    } else {
        // ------------------------------ W streamer ------------------------------
        if (lane == 0) {
            uint32_t q = 0;
            for (int64_t tile = blockIdx.x; tile < ntiles && !*abort_flag; tile += gridDim.x) {
                for (int c = 0; c < nchunks; ++c, ++q) {
                    const int s = q % kBStages;
                    if (q >= static_cast<uint32_t>(kBStages) &&
                        !tc::mbar_wait(&b_empty[s], ((q / kBStages) - 1) & 1)) { fail_wait(4); break; }
                    tc::mbar_arrive_expect_tx(&b_full[s], kBStage);
                    tc::bulk_g2s(sB + s * kBStage, args.wimg + static_cast<size_t>(c) * kBStage, kBStage,
                                 &b_full[s]);
                }
            }
        }
        __syncwarp();
    }

    // sums of squares (FP64) over the producers
    if (args.sumsq) {
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            double v = warp_sum(sq[c]);
            if (lane == 0) red[warp][c] = v;
        }
    }
    tc::tc_fence_before();
    __syncthreads();
    if (args.sumsq && tid < 4 && ((args.comp_mask >> tid) & 1)) {
        double v = 0;
        for (int w = 0; w < kMmaWarp; ++w) v += red[w][tid];
        atomicAdd(&args.sumsq[tid], v);
    }
    tc::tc_fence_after();
    if (warp == 0) tc::tmem_dealloc(tmem_base, kTmemCols);
}

template <int NAX, int NT, bool GRAD, int LMAX, int PPT>
void launch(const ProjectArgs& a, int nsm, cudaStream_t s) {
    const size_t smem = Smem<NAX, NT, GRAD>::kBytes;
    auto kern = project_tc_kernel<NAX, NT, GRAD, LMAX, PPT>;
    ISDF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(smem)));
    const int64_t ntiles = (a.n + kRows - 1) / kRows;
    const int grid = static_cast<int>(std::min<int64_t>(ntiles, nsm));
    kern<<<grid, Roles<PPT>::kThreads, smem, s>>>(a);
    ISDF_LAUNCH_CHECK();
}

// Specialisation on the basis' largest angular momentum: small l leaves room
// for six piece lanes (24 producer warps) within the register file.
template <int NAX, int NT, bool GRAD>
void launch_l(const ProjectArgs& a, int lmax, int nsm, cudaStream_t s) {
    // lane counts as in piece_lanes_for_lmax()
    if (lmax <= 2) launch<NAX, NT, GRAD, 2, 6>(a, nsm, s);
    else if (lmax <= 4) launch<NAX, NT, GRAD, 4, 2>(a, nsm, s);
    else launch<NAX, NT, GRAD, kMaxL, 2>(a, nsm, s);
}

}  // namespace

// K-chunk layout of a basis: pieces are runs of whole contractions of one
// shell; a chunk takes pieces in shell order until the next contraction no
// longer fits in its 32 slots.
void build_chunk_layout(Context& c) {
    const int nao = c.nao;
    const int lanes = piece_lanes_for_lmax(c.lmax);
    std::vector<std::vector<int4>> chunks;     // pieces of each chunk, in shell order
    std::vector<int> fill;
    std::vector<int2> ao_slot(std::max(nao, 1), make_int2(0, 0));
    std::vector<int4> cur;
    int used = 0;
    auto close_chunk = [&]() {
        chunks.push_back(cur);
        fill.push_back(used);
        cur.clear();
        used = 0;
    };
    for (int i = 0; i < c.nshell; ++i) {
        const auto& sh = c.shells[i];
        const int ns = 2 * sh.l + 1;
        for (int j = 0; j < sh.nctr;) {
            const int room = (kChunk - used) / ns;
            if (room == 0) { close_chunk(); continue; }
            const int take = std::min(room, sh.nctr - j);
            cur.push_back(make_int4(i, j, take, used));
            for (int u = 0; u < take * ns; ++u)
                ao_slot[sh.ao_off + j * ns + u] = make_int2(static_cast<int>(chunks.size()), used + u);
            used += take * ns;
            j += take;
        }
    }
    if (used > 0 || chunks.empty()) close_chunk();
    // balance each chunk's pieces over the producer lanes (longest first onto
    // the least-loaded lane) with an estimate of their evaluation cost
    auto cost = [&](const int4& p) {
        const auto& sh = c.shells[p.x];
        return 6 + sh.nprim * (2 + p.z) + p.z * (2 * sh.l + 1) * 3;
    };
    std::vector<int4> pieces;
    std::vector<int> lane_begin;
    for (auto& ch : chunks) {
        std::vector<int> order(ch.size());
        for (size_t i = 0; i < order.size(); ++i) order[i] = static_cast<int>(i);
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost(ch[a]) > cost(ch[b]); });
        std::vector<std::vector<int4>> per_lane(lanes);
        std::vector<int> load(lanes, 0);
        for (int i : order) {
            const int l = static_cast<int>(std::min_element(load.begin(), load.end()) - load.begin());
            per_lane[l].push_back(ch[i]);
            load[l] += cost(ch[i]);
        }
        for (int l = 0; l < lanes; ++l) {
            lane_begin.push_back(static_cast<int>(pieces.size()));
            pieces.insert(pieces.end(), per_lane[l].begin(), per_lane[l].end());
        }
    }
    lane_begin.push_back(static_cast<int>(pieces.size()));
    std::vector<int> piece_chunk(std::max<size_t>(pieces.size(), 1), 0);
    for (size_t ch = 0; ch < chunks.size(); ++ch)
        for (int i = lane_begin[ch * lanes]; i < lane_begin[(ch + 1) * lanes]; ++i) piece_chunk[i] = static_cast<int>(ch);
    c.npieces = static_cast<int>(pieces.size());
    if (pieces.empty()) pieces.push_back(make_int4(0, 0, 0, 0));
    c.nchunks = static_cast<int>(fill.size());
    c.piece_lanes = lanes;
    auto up = [](auto*& dst, const auto& src) {
        using V = std::remove_pointer_t<std::remove_reference_t<decltype(dst)>>;
        ISDF_CUDA(cudaMalloc(reinterpret_cast<void**>(&dst), src.size() * sizeof(V)));
        ISDF_CUDA(cudaMemcpy(dst, src.data(), src.size() * sizeof(V), cudaMemcpyHostToDevice));
    };
    up(c.d_pieces, pieces);
    c.h_pieces = pieces;
    upload_piece_records(c);
    up(c.d_piece_begin, lane_begin);
    up(c.d_fill, fill);
    std::vector<int> ao0(fill.size(), 0);
    for (size_t i = 1; i < fill.size(); ++i) ao0[i] = ao0[i - 1] + fill[i - 1];
    up(c.d_chunk_ao0, ao0);
    up(c.d_ao_slot, ao_slot);
    up(c.d_piece_chunk, piece_chunk);
}

void upload_piece_records(Context& c) {
    std::vector<float4> rec, prim;
    std::vector<double2> c64, prim64;
    rec.reserve(c.h_pieces.size() * 3);
    for (const int4& pc : c.h_pieces) {
        const ShellDesc& sh = c.shells[pc.x];
        c64.push_back(make_double2(sh.x, sh.y));
        // the screening exponents (FP64 table: kScreenFp64, FP32: kScreenFp32)
        c64.push_back(make_double2(sh.z, static_cast<double>(sh.scr64)));
        const float xh = static_cast<float>(sh.x), yh = static_cast<float>(sh.y), zh = static_cast<float>(sh.z);
        const int off = static_cast<int>(prim.size());
        rec.push_back(make_float4(xh, yh, zh, sh.scr32));
        rec.push_back(make_float4(static_cast<float>(sh.x - xh), static_cast<float>(sh.y - yh),
                                  static_cast<float>(sh.z - zh), __int_as_float_host(off)));
        int4 meta = make_int4(sh.l, sh.nprim, pc.z, pc.w);
        float4 mf;
        std::memcpy(&mf, &meta, sizeof(mf));
        rec.push_back(mf);
        for (int g0 = 0; g0 < pc.z; g0 += 3)
            for (int p = 0; p < sh.nprim; ++p) {
                double cc[3] = {0.0, 0.0, 0.0};
                for (int j = 0; j < 3 && g0 + j < pc.z; ++j)
                    cc[j] = c.h_coef64[sh.coef_off + (pc.y + g0 + j) * sh.nprim + p];
                const double a = c.h_exp64[sh.prim_off + p];
                prim.push_back(make_float4(static_cast<float>(a), static_cast<float>(cc[0]),
                                           static_cast<float>(cc[1]), static_cast<float>(cc[2])));
                prim64.push_back(make_double2(a, cc[0]));
                prim64.push_back(make_double2(cc[1], cc[2]));
            }
    }
    if (rec.empty()) rec.push_back(make_float4(0.f, 0.f, 0.f, 0.f));
    if (prim.empty()) prim.push_back(make_float4(0.f, 0.f, 0.f, 0.f));
    if (c64.empty()) c64.push_back(make_double2(0.0, 0.0));
    if (prim64.empty()) prim64.push_back(make_double2(0.0, 0.0));
    auto put = [](auto*& dst, const auto& src) {
        using V = std::remove_pointer_t<std::remove_reference_t<decltype(dst)>>;
        if (!dst) ISDF_CUDA(cudaMalloc(reinterpret_cast<void**>(&dst), src.size() * sizeof(V)));
        ISDF_CUDA(cudaMemcpy(dst, src.data(), src.size() * sizeof(V), cudaMemcpyHostToDevice));
    };
    put(c.d_piece_rec, rec);
    put(c.d_piece_prim, prim);
    put(c.d_piece_c64, c64);
    put(c.d_piece_prim64, prim64);
}

namespace {

// One thread per (axis, AO, source column): FP64 weight -> BF16 hi + lo at the
// AO's (chunk, slot) in the interleaved K-major B tiles of its axis.
__global__ void w_image_kernel(WSource src, int nax, int nao, const int2* __restrict__ ao_slot,
                               int nt, uint16_t* __restrict__ img) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t total = static_cast<int64_t>(nax) * nao * src.ncols;
    if (i >= total) return;
    const int j = static_cast<int>(i % src.ncols);
    const int mu = static_cast<int>((i / src.ncols) % nao);
    const int a = static_cast<int>(i / (static_cast<int64_t>(src.ncols) * nao));
    const double wv = src.p[a * src.s_axis + mu * src.s_ao + j * src.s_col];
    const __nv_bfloat16 hb = __float2bfloat16_rn(static_cast<float>(wv));
    const __nv_bfloat16 lb = __float2bfloat16_rn(static_cast<float>(wv - static_cast<double>(__bfloat162float(hb))));
    const uint32_t tileB = static_cast<uint32_t>(nt) * kChunk * 2;
    const size_t stage = static_cast<size_t>(nax) * 2 * tileB;
    const int2 cs = ao_slot[mu];
    const uint32_t off = tc::interleaved_offset(src.col0 + j, cs.y, (nt / 8) * 128, 128);
    const size_t base = (cs.x * stage + (a * 2) * tileB + off) / 2;
    img[base] = __bfloat16_as_ushort(hb);
    img[base + tileB / 2] = __bfloat16_as_ushort(lb);
}

}  // namespace

// The split BF16 weight image, built on the device: per chunk, per axis,
// (hi, lo) tiles of NT rows x 32 K in the interleaved K-major layout.
ProjectPlan make_project_plan(const Context& c, const std::vector<int>& axis_comp, int nout,
                              const WSource* src, int nsrc, cudaStream_t s) {
    ProjectPlan pl;
    const int nax = static_cast<int>(axis_comp.size());
    pl.nax = nax;
    pl.nout = nout;
    pl.nt = nout <= 16 ? 16 : nout <= 32 ? 32 : nout <= 64 ? 64 : 128;
    pl.grad = false;
    pl.comp_mask = 0;
    pl.lmax = c.lmax;
    pl.nchunks = c.nchunks;
    for (int a = 0; a < nax; ++a) {
        pl.axis_comp[a] = axis_comp[a];
        pl.comp_mask |= 1 << axis_comp[a];
        if (axis_comp[a] > 0) pl.grad = true;
    }
    const size_t stage = static_cast<size_t>(nax) * 2 * pl.nt * kChunk * 2;
    pl.wimg.reset(stage / 2 * pl.nchunks, s);
    ISDF_CUDA(cudaMemsetAsync(pl.wimg.get(), 0, stage * pl.nchunks, s));
    for (int i = 0; i < nsrc; ++i) {
        require(src[i].col0 >= 0 && src[i].ncols >= 0 && src[i].col0 + src[i].ncols <= nout,
                "projection weight columns out of range");
        const int64_t total = static_cast<int64_t>(nax) * c.nao * src[i].ncols;
        if (total == 0) continue;
        w_image_kernel<<<static_cast<unsigned>((total + 255) / 256), 256, 0, s>>>(
            src[i], nax, c.nao, c.d_ao_slot, pl.nt, pl.wimg.get());
        ISDF_LAUNCH_CHECK();
    }
    return pl;
}

// Accumulator widths NT of 16, 32, 64 (up to 4 axis entries) or 128 (up to 3:
// four 128-column accumulators with gradients exceed the shared-memory plan).
bool project_tc_supported(int nax, int nout) {
    if (nax < 1 || nax > 4 || nout < 1 || nout > 128) return false;
    const int nt = nout <= 16 ? 16 : nout <= 32 ? 32 : nout <= 64 ? 64 : 128;
    return nt < 128 ? nax * nt <= 256 : nax <= 3;
}

void project_tc(const Context& c, const ProjectPlan& pl, const double* pts, const int64_t* index,
                int64_t n, const double* weights, float* out, int64_t ld_out, int64_t col_stride,
                double* sumsq,
                float* point_sq, int* error, cudaStream_t s, uint8_t* a_store, int store_axis,
                uint8_t* a_store_r, uint8_t* chunk_zero) {
    if (n == 0) return;
    ProjectArgs a{};
    a.shells = c.d_shells;
    a.shell_hi = c.d_shell_hi;
    a.shell_lo = c.d_shell_lo;
    a.piece_rec = c.d_piece_rec;
    a.piece_prim = c.d_piece_prim;
    a.expf_ = c.d_expf;
    a.coeff_ = c.d_coeff;
    a.point_sq = point_sq;
    a.nao = c.nao;
    a.pts = pts;
    a.index = index;
    a.weights = weights;
    a.n = n;
    a.nchunks = pl.nchunks;
    a.pieces = c.d_pieces;
    a.lane_begin = c.d_piece_begin;
    a.piece_chunk = c.d_piece_chunk;
    a.npieces = c.npieces;
    require(c.piece_lanes == piece_lanes_for_lmax(pl.lmax), "chunk layout built for other producer lanes");
    a.chunk_fill = c.d_fill;
    a.wimg = reinterpret_cast<const uint8_t*>(pl.wimg.get());
    a.comp_mask = pl.comp_mask;
    for (int i = 0; i < pl.nax; ++i) a.axis_comp[i] = pl.axis_comp[i];
    a.zero_behind = 1;
    for (int i = 0; i < pl.nax; ++i)
        for (int j = 0; j < i; ++j)
            if (pl.axis_comp[i] == pl.axis_comp[j]) a.zero_behind = 0;
    a.out = out;
    a.ld_out = ld_out;
    a.col_stride = col_stride;
    a.a_store = a_store;
    a.a_store_r = a_store_r;
    a.chunk_zero = chunk_zero;
    a.store_axis = store_axis;
    require(a_store == nullptr || (store_axis >= 0 && store_axis < pl.nax), "invalid stored axis entry");
    a.nout = pl.nout;
    a.sumsq = sumsq;
    a.error = error;
    int dev = 0, nsm = 148;
    ISDF_CUDA(cudaGetDevice(&dev));
    ISDF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    ISDF_PROFILE(pl.grad ? "project_tc_grad" : "project_tc_val", s);
#define ISDF_TC_CASE(NAX, NT, G) \
    if (pl.nax == NAX && pl.nt == NT && pl.grad == G) { launch_l<NAX, NT, G>(a, pl.lmax, nsm, s); return; }
    ISDF_TC_CASE(1, 16, false) ISDF_TC_CASE(1, 32, false) ISDF_TC_CASE(1, 64, false)
    ISDF_TC_CASE(1, 16, true) ISDF_TC_CASE(1, 32, true) ISDF_TC_CASE(1, 64, true)
    ISDF_TC_CASE(2, 64, true) ISDF_TC_CASE(3, 64, true) ISDF_TC_CASE(4, 64, true)
    ISDF_TC_CASE(2, 32, true) ISDF_TC_CASE(3, 32, true) ISDF_TC_CASE(4, 32, true)
    ISDF_TC_CASE(2, 16, true) ISDF_TC_CASE(3, 16, true) ISDF_TC_CASE(4, 16, true)
    ISDF_TC_CASE(2, 64, false) ISDF_TC_CASE(2, 32, false) ISDF_TC_CASE(2, 16, false)
    ISDF_TC_CASE(1, 128, false) ISDF_TC_CASE(1, 128, true) ISDF_TC_CASE(2, 128, false)
    ISDF_TC_CASE(2, 128, true) ISDF_TC_CASE(3, 128, true)
#undef ISDF_TC_CASE
    fail(kNotImplemented, "tensor-core projection shape not instantiated");
}

}  // namespace isdf
