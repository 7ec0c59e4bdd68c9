// Argument blocks and launch declarations of the build and apply kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "entry.cuh"

namespace nca {

// One side of the batched build (side 0: test rows against trial far pivots; side 1: trial
// rows, entries evaluated transposed, as assemble_level(...; transposed=true)).
struct LevelArgs {
    KernelParams K;
    int side;
    const double *own_pts;  // xyz of this side's points
    const double *far_pts;  // xyz of the other side's points
    const int32_t *perm, *begin, *end, *firstchild, *nchildren;
    const int32_t *fpptr, *fpidx;  // phase-1 far pivots (CSR over nodes)
    int32_t *rank, *nrows, *piv;   // outputs: rank, block rows, pivots (maxrank per node)
    int32_t *cpiv;                 // optional output: column pivots (far-side point ids)
    double2 *X;                    // interpolation operators, node slot at xoff[node]
    const int64_t *xoff;
    int maxrank;
    double tol;
    int sampled;
    int32_t *status;  // [flag, node, npivots, rank] of the first singular cross matrix
};

size_t level_smem_bytes(int mcap, int ncap);
__global__ void k_level_compress(LevelArgs a, const int32_t *nodes, int mcap, int ncap);

// Frozen-skeleton values of the interpolation operators: with the row pivots tau (piv) and
// column pivots sigma (cpiv) of a finished build, mode 0 recomputes X = K[rows, sigma]
// K[tau, sigma]^{-1} for the kernel K (a new wavenumber; bit-identical to the build at the same
// one), mode 1 computes dX/dk = (dK[rows, sigma] - X dK[tau, sigma]) K[tau, sigma]^{-1} from X.
struct ValueArgs {
    KernelParams K, dK;
    int side, mode;
    const double *own_pts, *far_pts;
    const int32_t *perm, *begin, *end, *firstchild, *nchildren, *rank, *piv, *cpiv;
    // directional items (null: one item per node): the item's cluster, whether its rows are the
    // cluster's points, and otherwise its children's items (whose pivots form the rows)
    const int32_t *item_node, *item_basis, *item_chptr, *item_chidx;
    int maxrank;
    const double2 *Xin;  // mode 1: X at the wavenumber of K
    double2 *Xout;
    const int64_t *xoff;
    int32_t *status;  // [flag, node, npivots, rank]: 1 singular cross matrix, 2 capacity
};
size_t values_smem_bytes(int mcap, int rcap, int mode);
__global__ void k_level_values(ValueArgs a, const int32_t *nodes, int mcap, int rcap);

struct CouplingArgs {
    KernelParams K;
    const double *test_pts, *trial_pts;
    const int32_t *pair_t, *pair_s;
    const int32_t *rank_t, *rank_s, *piv_t, *piv_s;
    int maxrank;
    const int64_t *coff;
    int64_t npairs;
    double2 *C;
    float2 *C32;
};
__global__ void k_couplings(CouplingArgs a);

struct NearArgs {
    KernelParams K;
    const double *test_pts, *trial_pts;
    const int32_t *pair_t, *pair_s;
    const int32_t *t_perm, *t_begin, *t_end, *s_perm, *s_begin, *s_end;
    const int64_t *poff;  // block offset of each near pair
    int64_t npairs;
    double2 *N;
};
__global__ void k_near(NearArgs a);

__global__ void k_blocks_aca(const double2 *buf, int64_t ld, const int64_t *rowoff,
                             const int32_t *ncols, int maxrank, double tol, int sampled, int mcap,
                             int ncap, int32_t *ranks, int32_t *rowpiv, int32_t *colpiv);
__global__ void k_blocks_factors(const double2 *buf, int64_t ld, const int64_t *rowoff,
                                 const int32_t *ranks, const int32_t *rowpiv,
                                 const int32_t *colpiv, int maxrank, const int64_t *zoff,
                                 double2 *Z, int32_t *status);
__global__ void k_entries(KernelParams K, const double *tp, const double *sp, const int64_t *ii,
                          const int64_t *jj, int64_t n, double2 *out);
__global__ void k_to_f32(const double2 *in, float2 *out, int64_t n);

// Phase-1 far pivots (tree mimicry) of many items, one warp each (mimicry.cu). Item i belongs to
// own-side cluster item_node[i] (null: cluster i), whose centroid and point count are given; its
// far field is ffnodes[ffptr[i] .. ffptr[i + 1]) (far-tree node ids, in the reference's farfield
// order). Writes count[i] pivots (far point ids) to piv[i * maxrank ..].
struct MimicryArgs {
    const int32_t *begin, *end, *firstchild, *nchildren, *perm;  // far tree
    const double *center;                                         // far node centres, 3 each
    const double *pts;                                            // far points by id, 3 each
    int nitems;
    const int64_t *ffptr;
    const int32_t *ffnodes;
    int ff_by_position;  // 1: ffptr is indexed by the item's position in the launch (IACA levels)
    const int32_t *item_node;
    const double *centroid;   // own clusters, 3 each
    const int32_t *own_size;  // own clusters' point counts
    int maxrank;
    int32_t *count, *piv;
    int32_t *error;   // 1: an item ran out of candidates before its pivot count
    int32_t *cursor;  // next item to take (zero at launch): warps take items one at a time
};
// IACA per item (tree-mimicry columns, maximum-value rows, extrapolated Frobenius stop) fused with
// the tree mimicry and the interpolation operator, one warp per item (mimicry.cu). The far tree,
// the items' far fields (ffptr/ffnodes), item_node and the own clusters' centroids come in `mim`
// (its count, piv, error and cursor are unused). Rows of an item: its cluster's points when it is a
// basis item, else its children's pivots (item_chptr/item_chidx; node mode: the tree's children).
struct IacaArgs {
    MimicryArgs mim;
    KernelParams K;
    int side;
    const double *own_pts;
    const int32_t *perm, *begin, *end, *firstchild, *nchildren;  // own tree
    const int32_t *item_basis, *item_chptr, *item_chidx;          // item mode (mim.item_node set)
    const int32_t *items;  // the launch's items
    int nitems;
    int32_t *rank, *nrows, *piv, *cpiv;  // piv, cpiv: maxrank per item (cpiv optional)
    double2 *X;            // item slots of rows x min(maxrank, rows, far points) entries at xoff
    const int64_t *xoff;   // indexed by item, or by position in `items` with xoff_by_position
    int xoff_by_position;
    int32_t *rank_pos;     // optional: rank_pos[i] = rank, rank_pos[nitems + i] = rows of items[i]
    int maxrank;
    double tol;
    int32_t *status;       // [flag, item, a, b], see k_iaca
};
size_t iaca_smem_bytes(int maxrank);
int iaca_max_rows();
// mcap: the largest row count of the launch's items (at most iaca_max_rows())
void launch_iaca(const IacaArgs &a, int mcap, cudaStream_t s);
size_t mimicry_smem_bytes(int maxrank);
void launch_mimicry(const MimicryArgs &a, cudaStream_t s);
// packs count[i] pivots of every item from its maxrank-wide slot into the CSR list fpidx
void launch_compact_pivots(const int32_t *piv, int maxrank, const int32_t *count, const int32_t *fpptr,
                           int nitems, int32_t *fpidx, cudaStream_t s);

}  // namespace nca
