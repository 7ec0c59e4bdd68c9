// Internal declarations shared by the host planner (host_plan.cpp) and the CUDA sources.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "nca_b200.h"

namespace nca {

// Thread-local error state behind nca_last_error / nca_last_singular.
void set_error(const std::string &msg);
void set_singular(int side, int node, int npivots, int rank);

// k-means cluster tree, node ids in breadth-first order (root 0, siblings consecutive,
// every level a contiguous id range).
struct Tree {
    int64_t npoints = 0;
    int nnodes = 0, nlevels = 0;
    std::vector<int32_t> perm, iperm;
    std::vector<int32_t> begin, end, parent, firstchild, nchildren, level;
    std::vector<double> center, radius;
    std::vector<int32_t> levelptr;
    bool isleaf(int n) const { return nchildren[n] == 0; }
    int size(int n) const { return end[n] - begin[n]; }
};

Tree build_kmeans_tree(const double *pts, int64_t n, int minvalues);
// the same tree, bit for bit, built on the current CUDA device (tree_kernels.cu); `stream` is a
// cudaStream_t
Tree build_kmeans_tree_device(const double *pts, int64_t n, int minvalues, void *stream);

// Near/far interaction lists over test nodes, plus the trial-side transposes.
struct Partition {
    std::vector<int32_t> nearptr, nearnodes, farptr, farnodes;
    std::vector<int32_t> tnearptr, tnearnodes, tfarptr, tfarnodes;
};

Partition build_partition(const Tree &test, const Tree &trial, double eta);

// Phase 1 of the batched compressor for one cluster (tree mimicry on the far tree).
// centroid of the reference points (sequential sums in index order, then one division each)
void cluster_centroid(const double *ownpts, const int32_t *refidcs, int nref, double *c);
// select_farpivots with the centroid of the nref reference points given
int select_farpivots_at(const Tree &far, const double *farpts, const double *centroid, int nref,
                        const int32_t *farnodes, int nfar, int maxrank, int32_t *out);
int select_farpivots(const Tree &far, const double *ownpts, const double *farpts,
                     const int32_t *refidcs, int nref, const int32_t *farnodes, int nfar,
                     int maxrank, int32_t *out);

// Phase 1 for every node of one side, in parallel over nodes: CSR of far pivots.
void all_farpivots(const Tree &own, const Tree &far, const double *ownpts, const double *farpts,
                   const std::vector<int32_t> &ptr, const std::vector<int32_t> &nodes,
                   int maxrank, std::vector<int32_t> &fpptr, std::vector<int32_t> &fpidx);

// Worker count of the host planner.
int host_threads();

// ---- directional (wideband) planning, directional.cpp ----
struct Wideband {
    double k, etalf, etahf, gamma;
};
Partition build_partition_wideband(const Tree &test, const Tree &trial, const Wideband &w);
bool is_lowfrequency(const Tree &T, int node, const Wideband &w);

// Directional far data of one side and its basis items (one per (cluster, direction)).
struct DirSide {
    std::vector<int32_t> farptr, farnodes;  // far nodes of each node, grouped by direction
    std::vector<int32_t> dirptr;            // node -> its first item (nnodes + 1)
    std::vector<int32_t> dirs;              // item -> direction (0: low frequency; else 1-based candidate id)
    std::vector<double> dirvec;             // item -> unit direction (zero for low frequency)
    std::vector<int32_t> dirfarptr;         // item -> its own far nodes in farnodes (nitems + 1)
    std::vector<int32_t> chdirptr, chdirmap;  // node -> for each parent direction its own (1-based)
    std::vector<int32_t> invptr, invidx;      // item -> the parent directions (1-based, ascending) mapped onto it
    std::vector<int32_t> item_node, item_basis;
    std::vector<int32_t> item_chptr, item_chidx;  // nested items: the children's items in child order
};
DirSide directional_plan(const Tree &T, const Tree &F, const std::vector<int32_t> &farptr,
                         const std::vector<int32_t> &farnodes, const Wideband &w);
void item_farfield(const Tree &T, const DirSide &D, int item, std::vector<int32_t> &ff);
void all_item_farpivots(const Tree &own, const Tree &far, const DirSide &D, const double *ownpts,
                        const double *farpts, int maxrank, std::vector<int32_t> &fpptr, std::vector<int32_t> &fpidx);

}  // namespace nca

struct nca_tree {
    nca::Tree t;
};
struct nca_dirplan {
    const nca::Tree *tree;  // borrowed: the plan's own tree
    nca::DirSide d;
};
struct nca_partition {
    nca::Partition p;
    bool wideband = false;  // built with the wideband admissibility: the core becomes directional
    nca::Wideband w{};
};
