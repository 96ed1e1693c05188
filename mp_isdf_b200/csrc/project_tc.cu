// Fused AO evaluation + tensor-core projection (sm_100a, tcgen05).
//
// For a tile of 128 grid points (one UMMA M=128 tile) the CTA evaluates the
// needed AO components (value and/or d/dx, d/dy, d/dz) in FP32, one K-chunk of
// 32 AOs at a time, splits them into BF16 hi + lo parts and multiplies them on
// the tensor cores with a pre-split BF16 hi + lo weight matrix:
//     P[g][a][n] = sum_mu comp_a(g, mu) W_a[mu][n]
//                ~ A_hi B_hi + A_hi B_lo + A_lo B_hi   (FP32 accumulate in TMEM)
// One accumulator of NT columns per axis entry a.  Nothing of the AO matrix
// is written to HBM.  Used for
//   * the Khatri-Rao sketch projections f_g . [u_s v_s] (all selected axes);
//   * the fit Gram G[g][k] = phi_g . phi_a(k) (AO values only).
// The per-component sums of squares of the FP32 values are accumulated in FP64
// for the multi-axis Frobenius scales.
//
// Warp roles (320 threads): warps 0-7 evaluate AOs (thread = point, two shell
// lanes), convert to the UMMA operand layout and, warps 0-3, run the TMEM
// epilogue; warp 8 issues the MMAs; warp 9 streams W chunks by bulk copy.
#include "ao_device.cuh"
#include "isdf_project.h"
#include "isdf_reduce.cuh"
#include "tc_sm100.cuh"

#include <cuda_bf16.h>

#include <algorithm>
#include <cstring>

namespace isdf {

namespace {

constexpr int kRows = 128;            // points per tile (UMMA M)
constexpr int kChunk = 32;            // AOs per K-chunk
constexpr int kProducers = 256;       // 8 warps
constexpr int kThreads = kProducers + 64;
constexpr uint32_t kTileA = kRows * kChunk * 2;       // bytes of one BF16 A tile (8 KB)
constexpr uint32_t kLboA = (kRows / 8) * 128;          // K-adjacent core matrices
constexpr uint32_t kSboA = 128;                        // M-adjacent core matrices

// Writes component values of AO column k (0..31 within the chunk) of point p
// into the FP32 staging buffer stage[comp][k][p].
struct StageSink {
    float* stage;        // [ncomp][kChunk][kRows]
    int p, ao_lo, ao_hi, ao0;  // AOs in [ao_lo, ao_hi) belong to this chunk; ao0 = chunk start
    int comp_slot[4];    // slot of each component in the staging buffer, -1 if unused
    bool count;
    double sq[4];
    __device__ __forceinline__ bool wants(int first, int last) const {
        return last > ao_lo && first < ao_hi;
    }
    template <int C>
    __device__ __forceinline__ void put(int ao, float v) {
        const int slot = comp_slot[C];
        if (slot < 0 || ao < ao_lo || ao >= ao_hi) return;
        stage[(slot * kChunk + (ao - ao0)) * kRows + p] = v;
        if (count) sq[C] += static_cast<double>(v) * static_cast<double>(v);
    }
};

__device__ __forceinline__ uint32_t pack_bf16(float lo_elem, float hi_elem) {
    const uint32_t a = __bfloat16_as_ushort(__float2bfloat16_rn(lo_elem));
    const uint32_t b = __bfloat16_as_ushort(__float2bfloat16_rn(hi_elem));
    return a | (b << 16);
}

// hi = bf16(x), lo = bf16(x - hi) for 8 values, packed for two 16-byte stores.
__device__ __forceinline__ void split8(const float* x, uint4& hi, uint4& lo) {
    float h[8], l[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const __nv_bfloat16 hb = __float2bfloat16_rn(x[i]);
        h[i] = __bfloat162float(hb);
        l[i] = x[i] - h[i];
    }
    hi = make_uint4(pack_bf16(h[0], h[1]), pack_bf16(h[2], h[3]), pack_bf16(h[4], h[5]),
                    pack_bf16(h[6], h[7]));
    lo = make_uint4(pack_bf16(l[0], l[1]), pack_bf16(l[2], l[3]), pack_bf16(l[4], l[5]),
                    pack_bf16(l[6], l[7]));
}

__device__ __forceinline__ void named_bar_sync(int id, int count) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

template <int NAX, int NT, bool GRAD>
__global__ void __launch_bounds__(kThreads, 1)
project_tc_kernel(ProjectArgs args) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    // layout: [A: NAX x (hi, lo) tiles][B: 2 stages x NAX x (hi, lo)][stage FP32][barriers]
    constexpr uint32_t kTileB = NT * kChunk * 2;
    constexpr uint32_t kABytes = NAX * 2 * kTileA;
    constexpr uint32_t kBStage = NAX * 2 * kTileB;
    constexpr int kNComp = GRAD ? 4 : 1;
    uint8_t* sA = smem_raw;
    uint8_t* sB = sA + kABytes;
    float* sStage = reinterpret_cast<float*>(sB + 2 * kBStage);
    uint64_t* bars = reinterpret_cast<uint64_t*>(sStage + kNComp * kChunk * kRows);
    uint64_t* a_full = bars + 0;
    uint64_t* a_empty = bars + 1;
    uint64_t* b_full = bars + 2;     // [2]
    uint64_t* b_empty = bars + 4;    // [2]
    uint64_t* acc_full = bars + 6;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 7);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(bars + 8);
    volatile int* prod_abort = reinterpret_cast<volatile int*>(bars + 9);
    __shared__ double red[kThreads / 32][4];

    const int tid = threadIdx.x;
    const int warp = tid / 32, lane = tid % 32;
    constexpr uint32_t kTmemCols = (NAX * NT <= 32) ? 32 : (NAX * NT <= 64) ? 64
                                   : (NAX * NT <= 128) ? 128 : (NAX * NT <= 256) ? 256 : 512;
    static_assert(NAX * NT <= 512, "accumulators exceed TMEM");

    if (tid == 0) {
        tc::mbar_init(a_full, kProducers);
        tc::mbar_init(a_empty, 1);
        tc::mbar_init(&b_full[0], 1);
        tc::mbar_init(&b_full[1], 1);
        tc::mbar_init(&b_empty[0], 1);
        tc::mbar_init(&b_empty[1], 1);
        tc::mbar_init(acc_full, 1);
        *abort_flag = 0;
        *prod_abort = 0;
        tc::mbar_init_fence();
    }
    if (warp == 0) tc::tmem_alloc(tmem_slot, kTmemCols);
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

    if (warp < 8) {
        // ------------------------------ producers ------------------------------
        const int p = tid & (kRows - 1);
        const int half = tid >> 7;
        int comp_slot[4] = {-1, -1, -1, -1};
        {
            int s = 0;
            for (int c = 0; c < 4; ++c)
                if ((args.comp_mask >> c) & 1) comp_slot[c] = s++;
        }
        uint32_t q = 0;   // chunk sequence number of this CTA
        uint32_t t = 0;   // tile sequence number of this CTA
        for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++t) {
            const int64_t g = tile * kRows + p;
            const bool valid = g < n;
            double px = 0, py = 0, pz = 0;
            bool count = false;
            if (valid) {
                const int64_t gi = args.index ? args.index[g] : g;
                px = args.pts[3 * gi]; py = args.pts[3 * gi + 1]; pz = args.pts[3 * gi + 2];
                count = args.sumsq && (args.weights == nullptr || args.weights[gi] != 0.0);
            }
            float psq[4] = {0.f, 0.f, 0.f, 0.f};
            for (int c = 0; c < nchunks; ++c, ++q) {
                // 1. evaluate this chunk's AOs into the FP32 staging buffer
                StageSink sink{sStage, p, c * kChunk, min((c + 1) * kChunk, args.nao), c * kChunk,
                               {comp_slot[0], comp_slot[1], comp_slot[2], comp_slot[3]},
                               count || args.point_sq != nullptr, {0, 0, 0, 0}};
                if (half == 0) {
                    for (int s = 0; s < kNComp; ++s)
                        for (int k = 0; k < kChunk; ++k) sStage[(s * kChunk + k) * kRows + p] = 0.f;
                }
                named_bar_sync(1, kProducers);
                if (valid) {
                    for (int sh = args.chunk_shell_begin[c] + half; sh < args.chunk_shell_end[c]; sh += 2) {
                        const ShellDesc b = args.shells[sh];
                        const double dx = px - b.x, dy = py - b.y, dz = pz - b.z;
                        eval_shell_any<float, GRAD>(b, dx, dy, dz, args.expf_, args.coeff_,
                                                    args.c2sf, sink);
                    }
                }
#pragma unroll
                for (int cc = 0; cc < 4; ++cc) {
                    if (count) sq[cc] += sink.sq[cc];
                    psq[cc] += static_cast<float>(sink.sq[cc]);
                }
                named_bar_sync(1, kProducers);
                // 2. wait until the MMAs of the previous chunk released the A tiles
                if (q > 0 && !tc::mbar_wait(a_empty, (q - 1) & 1)) fail_wait(0);
                // 3. convert staging -> BF16 hi/lo A tiles (UMMA interleaved K-major)
                for (int u = tid; u < kRows * NAX * (kChunk / 8); u += kProducers) {
                    const int row = u % kRows;
                    const int rest = u / kRows;
                    const int kg = rest % (kChunk / 8);
                    const int a = rest / (kChunk / 8);
                    const int slot = comp_slot[args.axis_comp[a]];
                    float x[8];
#pragma unroll
                    for (int i = 0; i < 8; ++i) x[i] = sStage[(slot * kChunk + kg * 8 + i) * kRows + row];
                    uint4 hi, lo;
                    split8(x, hi, lo);
                    const uint32_t off = tc::interleaved_offset(row, kg * 8, kLboA, kSboA);
                    *reinterpret_cast<uint4*>(sA + (a * 2 + 0) * kTileA + off) = hi;
                    *reinterpret_cast<uint4*>(sA + (a * 2 + 1) * kTileA + off) = lo;
                }
                tc::fence_proxy_async_smem();
                tc::mbar_arrive(a_full);
                // uniform abort decision: one producer samples the flag before the barrier
                if (tid == 0) *prod_abort = *abort_flag;
                named_bar_sync(1, kProducers);
                if (*prod_abort) break;
            }
            // per-point sums of squares of each component (two shell lanes add up)
            if (args.point_sq && valid)
                for (int cc = 0; cc < 4; ++cc)
                    if ((args.comp_mask >> cc) & 1) atomicAdd(&args.point_sq[g * 4 + cc], psq[cc]);
            // 4. epilogue (warps 0-3: TMEM lane quarter = warp)
            if (warp < 4) {
                if (!tc::mbar_wait(acc_full, t & 1)) fail_wait(1);
                tc::tc_fence_after();
                const int row = warp * 32 + lane;
                const int64_t gg = tile * kRows + row;
                for (int a = 0; a < NAX; ++a) {
                    for (int c0 = 0; c0 < NT; c0 += 16) {
                        uint32_t r[16];
                        tc::tmem_ld16(tmem_base + (static_cast<uint32_t>(warp * 32) << 16) +
                                          static_cast<uint32_t>(a * NT + c0), r);
                        tc::tmem_ld_wait();
                        if (gg < n) {
                            float* out = args.out + gg * args.ld_out + a * args.nout;
#pragma unroll
                            for (int i = 0; i < 16; ++i)
                                if (c0 + i < args.nout) out[c0 + i] = __uint_as_float(r[i]);
                        }
                    }
                }
                tc::tc_fence_before();
            }
            if (tid == 0) *prod_abort = *abort_flag;
            named_bar_sync(1, kProducers);
            if (*prod_abort) break;
        }
    } else if (warp == 8) {
        // ------------------------------ MMA issuer ------------------------------
        if (lane == 0) {
            constexpr uint32_t idesc = tc::idesc_bf16_f32(kRows, NT);
            constexpr uint32_t kLboB = (NT / 8) * 128;
            uint32_t q = 0;
            for (int64_t tile = blockIdx.x; tile < ntiles && !*abort_flag; tile += gridDim.x) {
                for (int c = 0; c < nchunks; ++c, ++q) {
                    const int s = q & 1;
                    if (!tc::mbar_wait(&b_full[s], (q >> 1) & 1)) { fail_wait(2); break; }
                    if (!tc::mbar_wait(a_full, q & 1)) { fail_wait(3); break; }
                    tc::tc_fence_after();
                    for (int a = 0; a < NAX; ++a) {
                        const uint32_t d = tmem_base + static_cast<uint32_t>(a * NT);
                        const uint32_t a_hi = tc::smem_addr(sA + (a * 2 + 0) * kTileA);
                        const uint32_t a_lo = tc::smem_addr(sA + (a * 2 + 1) * kTileA);
                        const uint32_t b_hi = tc::smem_addr(sB + s * kBStage + (a * 2 + 0) * kTileB);
                        const uint32_t b_lo = tc::smem_addr(sB + s * kBStage + (a * 2 + 1) * kTileB);
                        for (int kk = 0; kk < kChunk / 16; ++kk) {
                            const uint64_t dah = tc::smem_desc_kmajor_noswizzle(a_hi + kk * 2 * kLboA, kLboA, kSboA);
                            const uint64_t dal = tc::smem_desc_kmajor_noswizzle(a_lo + kk * 2 * kLboA, kLboA, kSboA);
                            const uint64_t dbh = tc::smem_desc_kmajor_noswizzle(b_hi + kk * 2 * kLboB, kLboB, 128);
                            const uint64_t dbl = tc::smem_desc_kmajor_noswizzle(b_lo + kk * 2 * kLboB, kLboB, 128);
                            const uint32_t first = (c == 0 && kk == 0) ? 0u : 1u;
                            tc::mma_bf16(d, dah, dbh, idesc, first);
                            tc::mma_bf16(d, dah, dbl, idesc, 1u);
                            tc::mma_bf16(d, dal, dbh, idesc, 1u);
                        }
                    }
                    tc::mma_commit(a_empty);
                    tc::mma_commit(&b_empty[s]);
                }
                tc::mma_commit(acc_full);
            }
        }
        __syncwarp();
    } else {
        // ------------------------------ W streamer ------------------------------
        if (lane == 0) {
            uint32_t q = 0;
            for (int64_t tile = blockIdx.x; tile < ntiles && !*abort_flag; tile += gridDim.x) {
                for (int c = 0; c < nchunks; ++c, ++q) {
                    const int s = q & 1;
                    if (q >= 2 && !tc::mbar_wait(&b_empty[s], ((q >> 1) - 1) & 1)) { fail_wait(4); break; }
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
        for (int w = 0; w < 8; ++w) v += red[w][tid];
        atomicAdd(&args.sumsq[tid], v);
    }
    tc::tc_fence_after();
    if (warp == 0) tc::tmem_dealloc(tmem_base, kTmemCols);
}

template <int NAX, int NT, bool GRAD>
size_t smem_bytes() {
    constexpr uint32_t kTileB = NT * kChunk * 2;
    constexpr int kNComp = GRAD ? 4 : 1;
    return NAX * 2 * kTileA + 2 * NAX * 2 * kTileB + kNComp * kChunk * kRows * 4 + 256 + 1024;
}

template <int NAX, int NT, bool GRAD>
void launch(const ProjectArgs& a, int nsm, cudaStream_t s) {
    const size_t smem = smem_bytes<NAX, NT, GRAD>();
    auto kern = project_tc_kernel<NAX, NT, GRAD>;
    ISDF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(smem)));
    const int64_t ntiles = (a.n + kRows - 1) / kRows;
    const int grid = static_cast<int>(std::min<int64_t>(ntiles, nsm));
    kern<<<grid, kThreads, smem, s>>>(a);
    ISDF_LAUNCH_CHECK();
}

}  // namespace

// Host-side preparation of the chunk plan and of the BF16 hi/lo weight image.
ProjectPlan make_project_plan(const Context& c, const std::vector<int>& axis_comp,
                              const std::vector<double>& W, int nout, cudaStream_t s) {
    ProjectPlan pl;
    const int nao = c.nao;
    const int nax = static_cast<int>(axis_comp.size());
    pl.nax = nax;
    pl.nout = nout;
    pl.nt = nout <= 16 ? 16 : nout <= 32 ? 32 : nout <= 64 ? 64 : 128;
    pl.grad = false;
    pl.comp_mask = 0;
    for (int a = 0; a < nax; ++a) {
        pl.axis_comp[a] = axis_comp[a];
        pl.comp_mask |= 1 << axis_comp[a];
        if (axis_comp[a] > 0) pl.grad = true;
    }
    pl.nchunks = (nao + kChunk - 1) / kChunk;
    // shells overlapping each chunk
    std::vector<int> sb(pl.nchunks), se(pl.nchunks);
    for (int ch = 0; ch < pl.nchunks; ++ch) {
        const int lo = ch * kChunk, hi = std::min(nao, lo + kChunk);
        int b = -1, e = -1;
        for (int i = 0; i < c.nshell; ++i) {
            const auto& sh = c.shells[i];
            const int s0 = sh.ao_off, s1 = sh.ao_off + (2 * sh.l + 1) * sh.nctr;
            if (s1 > lo && s0 < hi) { if (b < 0) b = i; e = i + 1; }
        }
        sb[ch] = b < 0 ? 0 : b;
        se[ch] = e < 0 ? 0 : e;
    }
    // W image: per chunk, per axis, (hi, lo) tiles of NT rows x 32 K in the
    // interleaved K-major layout.  W is row-major [nax*nao][nout].
    const uint32_t tileB = pl.nt * kChunk * 2;
    const size_t stage = static_cast<size_t>(nax) * 2 * tileB;
    std::vector<uint16_t> img(stage / 2 * pl.nchunks, 0);
    const uint32_t lbo = (pl.nt / 8) * 128;
    for (int ch = 0; ch < pl.nchunks; ++ch)
        for (int a = 0; a < nax; ++a)
            for (int nrow = 0; nrow < nout; ++nrow)
                for (int k = 0; k < kChunk; ++k) {
                    const int mu = ch * kChunk + k;
                    if (mu >= nao) continue;
                    const double wv = W[(static_cast<size_t>(a) * nao + mu) * nout + nrow];
                    const float f = static_cast<float>(wv);
                    const __nv_bfloat16 hb = __float2bfloat16_rn(f);
                    const float hf = __bfloat162float(hb);
                    const __nv_bfloat16 lb = __float2bfloat16_rn(static_cast<float>(wv - hf));
                    const uint32_t off = tc::interleaved_offset(nrow, k, lbo, 128);
                    const size_t base = (ch * stage + (a * 2) * tileB + off) / 2;
                    img[base] = __bfloat16_as_ushort(hb);
                    img[base + tileB / 2] = __bfloat16_as_ushort(lb);
                }
    pl.wimg.reset(img.size(), s);
    ISDF_CUDA(cudaMemcpyAsync(pl.wimg.get(), img.data(), img.size() * 2, cudaMemcpyHostToDevice, s));
    pl.chunk_begin.reset(pl.nchunks, s);
    pl.chunk_end.reset(pl.nchunks, s);
    ISDF_CUDA(cudaMemcpyAsync(pl.chunk_begin.get(), sb.data(), sb.size() * 4, cudaMemcpyHostToDevice, s));
    ISDF_CUDA(cudaMemcpyAsync(pl.chunk_end.get(), se.data(), se.size() * 4, cudaMemcpyHostToDevice, s));
    ISDF_CUDA(cudaStreamSynchronize(s));   // host image is a temporary
    return pl;
}

bool project_tc_supported(int nax, int nout) {
    if (nax < 1 || nax > 4 || nout < 1 || nout > 64) return false;
    const int nt = nout <= 16 ? 16 : nout <= 32 ? 32 : 64;
    return nax * nt <= 256;
}

void project_tc(const Context& c, const ProjectPlan& pl, const double* pts, const int64_t* index,
                int64_t n, const double* weights, float* out, int64_t ld_out, double* sumsq,
                float* point_sq, int* error, cudaStream_t s) {
    if (n == 0) return;
    ProjectArgs a{};
    a.shells = c.d_shells;
    a.expf_ = c.d_expf;
    a.coeff_ = c.d_coeff;
    a.c2sf = c.d_c2sf;
    a.point_sq = point_sq;
    a.nao = c.nao;
    a.pts = pts;
    a.index = index;
    a.weights = weights;
    a.n = n;
    a.nchunks = pl.nchunks;
    a.chunk_shell_begin = pl.chunk_begin.get();
    a.chunk_shell_end = pl.chunk_end.get();
    a.wimg = reinterpret_cast<const uint8_t*>(pl.wimg.get());
    a.comp_mask = pl.comp_mask;
    for (int i = 0; i < pl.nax; ++i) a.axis_comp[i] = pl.axis_comp[i];
    a.out = out;
    a.ld_out = ld_out;
    a.nout = pl.nout;
    a.sumsq = sumsq;
    a.error = error;
    int dev = 0, nsm = 148;
    ISDF_CUDA(cudaGetDevice(&dev));
    ISDF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    ISDF_PROFILE(pl.grad ? "project_tc_grad" : "project_tc_val", s);
#define ISDF_TC_CASE(NAX, NT, G) \
    if (pl.nax == NAX && pl.nt == NT && pl.grad == G) { launch<NAX, NT, G>(a, nsm, s); return; }
    ISDF_TC_CASE(1, 16, false) ISDF_TC_CASE(1, 32, false) ISDF_TC_CASE(1, 64, false)
    ISDF_TC_CASE(1, 16, true) ISDF_TC_CASE(1, 32, true) ISDF_TC_CASE(1, 64, true)
    ISDF_TC_CASE(2, 64, true) ISDF_TC_CASE(3, 64, true) ISDF_TC_CASE(4, 64, true)
    ISDF_TC_CASE(2, 32, true) ISDF_TC_CASE(3, 32, true) ISDF_TC_CASE(4, 32, true)
    ISDF_TC_CASE(2, 16, true) ISDF_TC_CASE(3, 16, true) ISDF_TC_CASE(4, 16, true)
    ISDF_TC_CASE(2, 64, false) ISDF_TC_CASE(2, 32, false) ISDF_TC_CASE(2, 16, false)
#undef ISDF_TC_CASE
    fail(kNotImplemented, "tensor-core projection shape not instantiated");
}

}  // namespace isdf
