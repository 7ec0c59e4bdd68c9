// Argument block of the H^2 product kernel (one kernel for every stage).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace nca {

enum { STAGE_UP = 0, STAGE_COUPLE = 1, STAGE_DOWN = 2, STAGE_LEAVES = 3, STAGE_GATHER = 4 };

// out_o = sum over segments op(M_seg) v_seg for every output node o of a launch.
//   STAGE_UP:     o a node of the input side; one segment XT_o (rank x nrows) times the gathered
//                 input slice (leaf) or the children's xhat; writes xhat_o.
//   STAGE_COUPLE: o a node of the output side; segments over its far list (CSR ptr/other),
//                 blocks M + moff[e] (rank_out x rank_in), vectors xhat of the partner; writes yhat_o.
//   STAGE_DOWN:   o a node of the output side; one segment X_o (nrows x rank) times yhat_o, added
//                 to the children's yhat.
//   STAGE_LEAVES: o a leaf of the output side; segments X_o yhat_o (if ranked) and the near
//                 blocks M + moff[e] times the partner's input slice; scattered into y.
//   STAGE_GATHER: generic block-sparse gather (directional products): output o has g_rows[o]
//                 rows at row g_out[o] of dst (or, with y set, scattered through perm from
//                 position g_out[o]); its segments e in [g_segptr[o], g_segptr[o+1]) are blocks
//                 at g_moff[e] (>= 0: in M, < 0: at -1 - g_moff[e] in M2) with g_w[e] columns,
//                 times the vector rows g_voff[e].. of src.
template <typename S>
struct RowArgs {
    int stage;
    const int32_t *begin, *end, *firstchild, *nchildren, *rank, *nrows, *perm;
    const int64_t *cptr;
    const S *M;
    const int64_t *moff;
    const S *X;
    const int64_t *xoff;
    const int32_t *ptr, *other;
    const int32_t *rank_in, *rank_out;
    const int64_t *cptr_in, *cptr_out;
    const int32_t *o_begin, *o_end;
    const double2 *src;
    double2 *coef;
    double2 *dst;
    // STAGE_GATHER over a complex-FP32 vector arena (the kernels' VT = float2): src32 / dst32 in
    // place of src / dst; accumulation stays FP64
    const float2 *src32;
    float2 *dst32;
    double2 *y;
    int64_t ldy;
    double2 alpha, beta;
    int usebeta;
    int b, bc, q0;
    int vs;           // row stride of the vector buffers (>= b)
    int conj;
    int maxrows;      // largest output block of the launch (picks the register tile)
    int32_t *error;   // 1: misaligned copy skipped, 2: a bounded wait gave up
    // tangent products: UP / DOWN write into coef_out (nullptr: coef) while reading coef;
    // UP and COUPLE add to the existing output with accumulate; UP skips leaves with skip_leaves
    double2 *coef_out;
    int accumulate, skip_leaves;
    const int32_t *g_rows, *g_segptr, *g_w;
    const int64_t *g_out, *g_moff, *g_voff;
    const S *M2;
};

size_t rows_smem_bytes();
int rows_capacity(int bc);  // largest output block one CTA computes for bc right-hand sides

__global__ void k_gather(const double2 *x, int64_t ldx, const int32_t *perm, int64_t n, int b, int vs,
                         double2 *xt);
// k_gather into a complex-FP32 vector buffer (x rounded to FP32)
__global__ void k_gather_to_f32(const double2 *x, int64_t ldx, const int32_t *perm, int64_t n, int b, int vs,
                                float2 *xt);
int vector_stride(int b);  // row stride of the internal vector buffers for b right-hand sides

// smem_bytes: dynamic shared memory of each CTA (0: rows_smem_bytes()); a larger request only
// lowers how many CTAs of the launch share an SM. priority: 0 for the stream's, else the launch's
// own scheduling priority (a CUDA stream priority value).
template <typename S>
void launch_rows(const RowArgs<S> &a, const int32_t *nodes, int count, cudaStream_t s, size_t smem_bytes = 0,
                 int priority = 0);

// STAGE_GATHER for outputs of at most 64 rows: one warp per output, operands read straight from
// global memory, complex FP64 FMA (directional products, whose outputs are many small blocks).
template <typename S, typename VT = double2>
void launch_gather_small(const RowArgs<S> &a, const int32_t *nodes, int count, cudaStream_t s);
// One output of a launch group, in launch order, as the all-column FP32 gather reads it.
struct WideOut {
    int32_t R, W, e0, e1;  // rows, block columns over all its segments, its segments [e0, e1)
    int64_t out;           // position of the record's first row (the output's g_out + r0)
    int32_t ld, r0;        // the output's blocks' leading dimension (its rows) and the record's
                           // first row in them: an output of many rows is taken as row slices
};
// STAGE_GATHER over complex-FP32 stores and arena for outputs of at most 32 rows, all a.b
// right-hand sides in one launch (a.q0, a.bc, a.g_rows, a.g_out, a.g_segptr unused; the outputs
// come as WideOut records): a warp streams a sequence of outputs, two columns per lane, FP32
// accumulation.
// STAGE_GATHER over complex-FP32 stores and arena on the tcgen05 tensor cores (3xTF32), for outputs
// of at most 64 rows, all a.b right-hand sides (passes of 128) in one launch; the outputs come as
// WideOut records (ld = R, r0 = 0). A CTA per output at a time, two per SM (tc_gather.cu).
bool gather_tc_fits(int maxrows);
size_t gather_tc_smem_bytes();
void launch_gather_tc(const RowArgs<float2> &a, const WideOut *outs, int count, cudaStream_t s);
bool gather_wide_fits(int maxrows);
// the register tile (rows) of the kernel instance that takes an output of R <= 32 rows: R rounded
// up to even up to 24, then 28 or 32; a launch's outputs all have tile nr
int wide_rows_class(int R);
void launch_gather_wide(const RowArgs<float2> &a, const WideOut *outs, int count, int nr, cudaStream_t s);
// STAGE_GATHER through the streaming kernel with vectors of type VT (launch_rows: VT = double2)
template <typename S, typename VT>
void launch_gather_rows(const RowArgs<S> &a, const int32_t *nodes, int count, cudaStream_t s);

// STAGE_GATHER for many outputs of at most 32 rows with 2..16 right-hand sides per pass: one
// warp streams a sequence of outputs, double-buffering their block columns and vector rows in
// shared memory with asynchronous copies, and multiplies on the FP64 tensor cores.
bool gather_tiny_fits(int maxrows, int bc);
template <typename S, typename VT = double2>
void launch_gather_tiny(const RowArgs<S> &a, const int32_t *nodes, int count, cudaStream_t s);

// dst[doff[e] + i + j * rows[e]] = src[soff[e] + i + j * sld[e]]: sub-matrix copies into
// contiguous column-major blocks.
template <typename S>
void launch_copy_blocks(const S *src, const int64_t *soff, const int32_t *sld, const int32_t *rows,
                        const int32_t *cols, const int64_t *doff, int64_t nblocks, S *dst, cudaStream_t s);

// out block e = (in block e)^T for R_e x C_e column-major blocks.
template <typename S>
void launch_transpose_blocks(const S *in, const int64_t *inoff, const int32_t *rows, const int32_t *cols,
                             const int64_t *outoff, int64_t nblocks, S *out, cudaStream_t s);

}  // namespace nca
