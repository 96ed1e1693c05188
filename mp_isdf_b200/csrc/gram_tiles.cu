// Tensor-core GEMM over stored split-BF16 AO tiles (sm_100a, tcgen05).
//
// The fused AO + projection kernel can leave the (hi, lo) BF16 A tiles of the
// AO values in HBM ([tile of 128 points][K-chunk] x 16 KB, UMMA interleaved
// K-major).  This kernel contracts them with a one-axis split weight image
// (ProjectPlan) without evaluating any AO again:
//     G[g][j] = sum_mu phi_mu(g) W[mu][j]  ~  A_hi B_hi + A_hi B_lo + A_lo B_hi
// with the same split products and per-chunk FP32 accumulation as the fused
// kernel.  It streams the tiles once (HBM-bound).
//
// Warp roles (192 threads): warp 0 streams A and B chunks into a 4-stage ring
// by bulk copy; warp 1 issues the MMAs into one of two TMEM accumulators;
// warps 2-5 drain the other accumulator (TMEM lane quarter = warp % 4) into G.
#include "isdf_project.h"
#include "tc_sm100.cuh"

#include <algorithm>

namespace isdf {
namespace {

constexpr int kRows = 128;
constexpr int kChunk = 32;
constexpr uint32_t kTileA = kRows * kChunk * 2;   // one BF16 A tile (8 KB)
constexpr uint32_t kLboA = (kRows / 8) * 128;
constexpr uint32_t kSboA = 128;
constexpr int kStages = 4;
constexpr int kThreads = 192;

struct GramArgs {
    const uint8_t* a_tiles;
    const uint8_t* wimg;
    int64_t n;
    int nchunks;
    float* out;
    int64_t ld_out;
    int nout;
    int* error;
    const uint8_t* chunk_zero;   // null, or [tile][chunk] nonzero where the tiles are zeros
};

// A chunk whose stored tiles are zeros is skipped by the loader and the MMA
// thread alike, except the last chunk of a tile none of whose chunks was
// taken (its zero tiles initialise the accumulator).
__device__ __forceinline__ bool skip_chunk(const GramArgs& a, int64_t tile, int c, bool taken) {
    return a.chunk_zero && a.chunk_zero[tile * a.nchunks + c] && (taken || c + 1 < a.nchunks);
}

template <int NT>
__global__ void __launch_bounds__(kThreads, 1) gram_tiles_kernel(GramArgs args) {
    constexpr uint32_t kTileB = NT * kChunk * 2;
    constexpr uint32_t kStageBytes = 2 * kTileA + 2 * kTileB;
    constexpr uint32_t kTmemCols = (2 * NT <= 32) ? 32 : (2 * NT <= 64) ? 64 : 128;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw + kStages * kStageBytes);
    uint64_t* full = bars;                    // [kStages]
    uint64_t* empty = bars + kStages;         // [kStages]
    uint64_t* acc_full = bars + 2 * kStages;  // [2]
    uint64_t* acc_empty = bars + 2 * kStages + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kStages + 4);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(bars + 2 * kStages + 5);

    const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
    if (tid == 0) {
        for (int i = 0; i < kStages; ++i) {
            tc::mbar_init(&full[i], 1);
            tc::mbar_init(&empty[i], 1);
        }
        for (int i = 0; i < 2; ++i) {
            tc::mbar_init(&acc_full[i], 1);
            tc::mbar_init(&acc_empty[i], 128);
        }
        *abort_flag = 0;
        tc::mbar_init_fence();
    }
    if (warp == 0) tc::tmem_alloc(tmem_slot, kTmemCols);
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;
    const int64_t ntiles = (args.n + kRows - 1) / kRows;
    const int nchunks = args.nchunks;
    auto fail_wait = [&](int where) {
        atomicOr(args.error, 1 << where);
        *abort_flag = 1;
    };

    if (warp == 0) {
        // ------------------------------ loader ------------------------------
        if (lane == 0) {
            uint32_t q = 0;
            for (int64_t tile = blockIdx.x; tile < ntiles && !*abort_flag; tile += gridDim.x) {
                bool taken = false;
                for (int c = 0; c < nchunks; ++c) {
                    if (skip_chunk(args, tile, c, taken)) continue;
                    taken = true;
                    const uint32_t s = q % kStages;
                    ++q;
                    if (q > kStages && !tc::mbar_wait(&empty[s], ((q - 1) / kStages - 1) & 1)) {
                        fail_wait(8);
                        break;
                    }
                    uint8_t* st = smem_raw + s * kStageBytes;
                    tc::mbar_arrive_expect_tx(&full[s], kStageBytes);
                    tc::bulk_g2s(st, args.a_tiles + (static_cast<size_t>(tile) * nchunks + c) * 2 * kTileA,
                                 2 * kTileA, &full[s]);
                    tc::bulk_g2s(st + 2 * kTileA, args.wimg + static_cast<size_t>(c) * 2 * kTileB, 2 * kTileB,
                                 &full[s]);
                }
            }
        }
        __syncwarp();
    } else if (warp == 1) {
        // ------------------------------ MMA issuer ------------------------------
        if (lane == 0) {
            constexpr uint32_t idesc = tc::idesc_bf16_f32(kRows, NT);
            constexpr uint32_t kLboB = (NT / 8) * 128;
            constexpr int pa[3] = {0, 0, 1};
            constexpr int pb[3] = {0, 1, 0};
            uint32_t q = 0, t = 0;
            for (int64_t tile = blockIdx.x; tile < ntiles && !*abort_flag; tile += gridDim.x, ++t) {
                const uint32_t ab = t & 1;
                if (t >= 2 && !tc::mbar_wait(&acc_empty[ab], ((t >> 1) - 1) & 1)) {
                    fail_wait(9);
                    break;
                }
                tc::tc_fence_after();
                const uint32_t d = tmem_base + ab * NT;
                bool ok = true;
                bool taken = false;
                for (int c = 0; c < nchunks; ++c) {
                    if (skip_chunk(args, tile, c, taken)) continue;
                    const bool first = !taken;
                    taken = true;
                    const uint32_t s = q % kStages;
                    const uint32_t ph = (q / kStages) & 1;
                    ++q;
                    if (!tc::mbar_wait(&full[s], ph)) {
                        fail_wait(10);
                        ok = false;
                        break;
                    }
                    tc::tc_fence_after();
                    const uint8_t* st = smem_raw + s * kStageBytes;
                    for (int kk = 0; kk < kChunk / 16; ++kk) {
#pragma unroll
                        for (int pr = 0; pr < 3; ++pr) {
                            const uint32_t aa = tc::smem_addr(st + pa[pr] * kTileA) + kk * 2 * kLboA;
                            const uint32_t bb = tc::smem_addr(st + 2 * kTileA + pb[pr] * kTileB) + kk * 2 * kLboB;
                            tc::mma_bf16(d, tc::smem_desc_kmajor_noswizzle(aa, kLboA, kSboA),
                                         tc::smem_desc_kmajor_noswizzle(bb, kLboB, 128), idesc,
                                         (first && kk == 0 && pr == 0) ? 0u : 1u);
                        }
                    }
                    tc::mma_commit(&empty[s]);
                }
                if (!ok) break;
                tc::mma_commit(&acc_full[ab]);
            }
        }
        __syncwarp();
    } else {
        // ------------------------------ epilogue ------------------------------
        const int quarter = warp % 4;
        const int row = quarter * 32 + lane;
        uint32_t t = 0;
        for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++t) {
            const uint32_t ab = t & 1;
            if (!tc::mbar_wait(&acc_full[ab], (t >> 1) & 1)) {
                fail_wait(11);
                break;
            }
            tc::tc_fence_after();
            const int64_t g = tile * kRows + row;
#pragma unroll
            for (int c0 = 0; c0 < NT; c0 += 16) {
                uint32_t r[16];
                tc::tmem_ld16(tmem_base + (static_cast<uint32_t>(quarter * 32) << 16) + ab * NT + c0, r);
                tc::tmem_ld_wait();
                if (g < args.n) {
                    float* o = args.out + g * args.ld_out + c0;
#pragma unroll
                    for (int i = 0; i < 16; ++i)
                        if (c0 + i < args.nout) o[i] = __uint_as_float(r[i]);
                }
            }
            tc::tc_fence_before();
            tc::mbar_arrive(&acc_empty[ab]);
            if (*abort_flag) break;
        }
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    if (warp == 0) tc::tmem_dealloc(tmem_base, kTmemCols);
}

template <int NT>
void launch_gram(const GramArgs& a, int nsm, cudaStream_t s) {
    constexpr size_t smem = kStages * (2 * kTileA + 2 * NT * kChunk * 2) + 128 + 1024;
    ISDF_CUDA(cudaFuncSetAttribute(gram_tiles_kernel<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(smem)));
    const int64_t ntiles = (a.n + kRows - 1) / kRows;
    const int grid = static_cast<int>(std::min<int64_t>(ntiles, nsm));
    gram_tiles_kernel<NT><<<grid, kThreads, smem, s>>>(a);
    ISDF_LAUNCH_CHECK();
}

}  // namespace

void gram_from_tiles(const Context& c, const ProjectPlan& pl, const uint8_t* a_tiles, int64_t n, float* out,
                     int64_t ld_out, int* error, cudaStream_t s, const uint8_t* chunk_zero) {
    if (n == 0) return;
    require(pl.nax == 1 && !pl.grad, "stored-tile GEMM takes a one-axis value plan");
    require(pl.nchunks == c.nchunks, "weight image and stored tiles disagree on the K-chunks");
    GramArgs a{a_tiles, reinterpret_cast<const uint8_t*>(pl.wimg.get()), n, pl.nchunks, out, ld_out,
               pl.nout, error, chunk_zero};
    int dev = 0, nsm = 148;
    ISDF_CUDA(cudaGetDevice(&dev));
    ISDF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    ISDF_PROFILE("gram_tiles", s);
    if (pl.nt == 16) launch_gram<16>(a, nsm, s);
    else if (pl.nt == 32) launch_gram<32>(a, nsm, s);
    else if (pl.nt == 64) launch_gram<64>(a, nsm, s);
    else fail(kNotImplemented, "stored-tile GEMM width not instantiated");
}

}  // namespace isdf
