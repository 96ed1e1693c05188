// Fused AO-evaluation + tensor-core projection (see project_tc.cu).
#pragma once

#include "isdf_internal.h"

namespace isdf {

struct ProjectArgs {
    const ShellDesc* shells;
    const float4* shell_hi;    // (x_hi, y_hi, z_hi, amin) per shell
    const float4* shell_lo;    // (x_lo, y_lo, z_lo, 0) per shell
    const float4* piece_rec;   // packed piece records (Context::d_piece_rec)
    const float4* piece_prim;  // packed primitives (Context::d_piece_prim)
    const float* expf_;
    const float* coeff_;
    float* point_sq;           // [n][4] per-point sums of squares per component, or null
    int nao;
    const double* pts;
    const int64_t* index;      // kept-point gather (may be null)
    const double* weights;     // for the sums of squares (may be null)
    int64_t n;
    int nchunks;
    const int4* pieces;        // (shell, first contraction, contractions, first slot in chunk)
    const int* lane_begin;     // pieces of lane j in chunk c: [lane_begin[c*PPT+j], lane_begin[c*PPT+j+1])
    const int* chunk_fill;     // slots of chunk c in use; the rest are zero
    const int* piece_chunk;    // chunk of each piece
    int npieces;
    const uint8_t* wimg;       // per chunk: nax x (hi, lo) BF16 tiles
    int comp_mask;
    int axis_comp[4];
    float* out;                // out[g*ld_out + (a*nout + j)*col_stride]
    int64_t ld_out, col_stride;
    int nout;
    double* sumsq;             // [4] or null
    int* error;                // bit flags of bounded waits that gave up
    uint8_t* a_store;          // null, or [tile][chunk] (hi, lo) A tiles of axis entry store_axis
    uint8_t* a_store_r;        // null, or [tile][chunk] BF16 remainder tiles x - hi - lo of that entry
    uint8_t* chunk_zero;       // null, or [tile][chunk]: 1 where the chunk was screened for the tile
    int store_axis;
    // 1 where the axis entries read distinct components: the conversion then
    // writes zeros back behind every staged value it reads, so a piece that is
    // not evaluated needs no zero fill (else screened pieces are zero-filled)
    int zero_behind;
};

struct ProjectPlan {
    int nax = 0, nout = 0, nt = 0, nchunks = 0, comp_mask = 0, lmax = 0;
    int axis_comp[4] = {0, 0, 0, 0};
    bool grad = false;
    DeviceBuffer<uint16_t> wimg;
};

// Device FP64 weights feeding output columns [col0, col0 + ncols) of the
// projection: W_a[mu][col0 + j] = p[a*s_axis + mu*s_ao + j*s_col].
struct WSource {
    const double* p;
    int64_t s_axis, s_ao, s_col;
    int ncols, col0;
};

// Builds the BF16 hi + lo weight image on the device from the sources.
ProjectPlan make_project_plan(const Context& c, const std::vector<int>& axis_comp, int nout,
                              const WSource* src, int nsrc, cudaStream_t s);
bool project_tc_supported(int nax, int nout);
void project_tc(const Context& c, const ProjectPlan& plan, const double* pts, const int64_t* index,
                int64_t n, const double* weights, float* out, int64_t ld_out, int64_t col_stride,
                double* sumsq,
                float* point_sq, int* error, cudaStream_t s, uint8_t* a_store = nullptr,
                int store_axis = 0, uint8_t* a_store_r = nullptr, uint8_t* chunk_zero = nullptr);

// G[g*ld_out + j] from A tiles stored by project_tc (a_store) over n points and
// a one-axis value plan: the same split-BF16 products as project_tc.
// chunk_zero (optional): one byte per stored (tile, K-chunk), nonzero where the
// fused projection screened the chunk for the whole tile (its tiles are zeros
// and the GEMM skips them).
void gram_from_tiles(const Context& c, const ProjectPlan& pl, const uint8_t* a_tiles, int64_t n,
                     float* out, int64_t ld_out, int* error, cudaStream_t s,
                     const uint8_t* chunk_zero = nullptr);

// Bytes of the stored A tiles of one axis entry over n points.
inline size_t stored_tile_bytes(const Context& c, int64_t n) {
    return static_cast<size_t>((n + 127) / 128) * c.nchunks * 2 * 128 * 32 * 2;
}

// Bytes of the stored remainder tiles over n points: the third BF16 term
// r = x - hi - lo of each FP32 value x, so that hi + lo + r == x exactly (one
// 8 KB tile per 128 points and K-chunk, same layout as the A tiles).
inline size_t stored_remainder_bytes(const Context& c, int64_t n) { return stored_tile_bytes(c, n) / 2; }
// Bytes of the per-(tile, K-chunk) screening flags over n points (256-byte multiple).
inline size_t stored_flag_bytes(const Context& c, int64_t n) {
    return ((static_cast<size_t>((n + 127) / 128) * c.nchunks + 255) / 256) * 256;
}

}  // namespace isdf
