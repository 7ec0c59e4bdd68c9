// Argument blocks of the H^2 product kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace nca {

// Upward / downward sweep over one side's interpolation operators.
template <typename S>
struct SweepArgs {
    const int32_t *begin, *firstchild, *nchildren, *rank, *nrows;
    const int64_t *xoff, *cptr;
    const S *X;
    const double2 *xt;  // tree-ordered input (upward sweep at the leaves)
    double2 *coef;      // xhat (upward) or yhat (downward)
    int b;
    bool conj;
};

// Coupling stage: forward gathers over the test node's far list, reverse over the trial
// node's transposed list (pairs[] maps it to the coupling block).
template <typename S>
struct CoupleArgs {
    const int32_t *ptr, *other, *pairs;
    const int32_t *rank_out, *rank_in;
    const int64_t *cptr_out, *cptr_in, *coff;
    const S *C;
    const double2 *xhat;
    double2 *yhat;
    int b;
    bool reverse, conj;
};

// Leaf stage: op(X_t) yhat_t plus the near field, scattered to the caller's layout.
template <typename S>
struct LeafArgs {
    const int32_t *perm, *begin, *end, *rank, *nrows;
    const int64_t *xoff, *cptr;
    const S *X;
    const double2 *yhat;
    const int32_t *nptr, *nnodes, *coloff;  // near lists of the output leaves
    const int32_t *o_begin, *o_end;         // the other side's nodes (input points)
    const int64_t *noff;                    // near row-block offsets (test nodes)
    const S *N;
    const double2 *xt;  // tree-ordered input
    double2 *y;
    int64_t ldy;
    double2 alpha, beta;
    int b;
    bool reverse, conj;
};

size_t apply_smem_bytes(int mcap, int bc, int tile_bytes);

__global__ void k_gather(const double2 *x, int64_t ldx, const int32_t *perm, int64_t n, int b,
                         double2 *xt);

// Host launchers (one per stage); each raises the kernel's dynamic shared-memory limit once.
template <typename S>
void launch_up(const SweepArgs<S> &a, const int32_t *nodes, int count, int mcap, int tile, cudaStream_t s);
template <typename S>
void launch_down(const SweepArgs<S> &a, const int32_t *nodes, int count, int mcap, int tile, cudaStream_t s);
template <typename S>
void launch_couple(const CoupleArgs<S> &a, const int32_t *nodes, int count, int mcap, int tile, cudaStream_t s);
template <typename S>
void launch_leaves(const LeafArgs<S> &a, const int32_t *nodes, int count, int mcap, int tile, cudaStream_t s);

}  // namespace nca
