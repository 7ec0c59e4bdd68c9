/*
 * nca_b200.h -- C ABI of the B200 batched NCA build and H^2 product.
 *
 * Every entry point returns an nca_status; on failure nca_last_error() holds a message
 * (thread-local). No C++ exception or device trap crosses this boundary. Indices are
 * 0-based; complex numbers are interleaved (re, im) doubles (or floats where stated);
 * matrices are column-major, as in Julia.
 *
 * Each declaration names the reference interface of NestedCrossApproximation.jl (paths
 * inside that project) that it replaces on the batched bottom-up build / H^2 product path.
 */
#ifndef NCA_B200_H
#define NCA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    NCA_OK = 0,
    NCA_ERR_SINGULAR = 1, /* SingularCrossMatrixError (src/utils/utils.jl:38-54) */
    NCA_ERR_DIM = 2,      /* DimensionMismatch */
    NCA_ERR_ARG = 3,      /* ArgumentError */
    NCA_ERR_CUDA = 4,     /* CUDA runtime failure */
    NCA_ERR_TIMEOUT = 5,  /* a bounded device wait gave up */
    NCA_ERR_OOM = 6,      /* device allocation failed */
    NCA_ERR_BUSY = 7      /* ConcurrentWorkspaceError (src/nca/petrovgalerkinnca.jl:210-218) */
} nca_status;

/* Kernel families of the entry generator (AdaptiveCrossApproximation.AbstractKernelMatrix
 * for point kernels: README.md:100-108, test/testutils.jl:14-21). */
typedef enum {
    NCA_KERNEL_HELMHOLTZ = 0, /* cis(sign * k r) / (4 pi r); 0 where r == 0 or r < rmin */
    NCA_KERNEL_LAPLACE = 1,   /* 1 / (4 pi r) */
    NCA_KERNEL_MATRIX = 2     /* entry (i, j) of a given matrix (AdaptiveCrossApproximation.PointMatrix) */
} nca_kernel_kind;

typedef struct {
    int32_t kind;          /* nca_kernel_kind */
    int32_t sign;          /* +1: exp(+ikr), -1: exp(-ikr) */
    double k;              /* wavenumber */
    double rmin;           /* distances below rmin give 0 */
    const double *matrix;  /* NCA_KERNEL_MATRIX: host matrix, ldmatrix x ntrial complex */
    int64_t ldmatrix;
} nca_kernel_desc;

/* Apply modes of LinearMaps: A, transpose(A), adjoint(A) (src/nca/petrovgalerkinnca.jl:431-589). */
typedef enum { NCA_MODE_N = 0, NCA_MODE_T = 1, NCA_MODE_C = 2 } nca_mode;

/* Stores the product reads: complex FP64, or complex FP32 copies (FP64 arithmetic either way). */
typedef enum { NCA_PREC_F64 = 0, NCA_PREC_F32 = 1 } nca_precision;

typedef struct nca_tree nca_tree;
typedef struct nca_partition nca_partition;
typedef struct nca_core nca_core;
typedef struct nca_workspace nca_workspace;
typedef struct nca_dirplan nca_dirplan;

int32_t nca_version(void);
/* Copies the last error message of this thread into buf (always NUL-terminated). */
int32_t nca_last_error(char *buf, size_t len);
/* Details of the last NCA_ERR_SINGULAR on this thread: side (0 test, 1 trial), node,
 * number of pivots and numerical rank (SingularCrossMatrixError(kind, npivots, rank)). */
int32_t nca_last_singular(int32_t *side, int32_t *node, int32_t *npivots, int32_t *rank);

/* ---- cluster trees (H2Trees.KMeansTree(points; builder=KMeansTreeBuilder(numberofclusters=2,
 *      minvalues)), used by test/testutils.jl:27-39; the tree is an input of the reference's
 *      PetrovGalerkinNCA, src/nca/petrovgalerkinnca.jl:138-142) ---- */
int32_t nca_tree_kmeans(const double *points, int64_t npoints, int32_t minvalues,
                        int32_t nclusters, nca_tree **out);
void nca_tree_destroy(nca_tree *tree);
int32_t nca_tree_sizes(const nca_tree *tree, int32_t *nnodes, int32_t *nlevels, int64_t *npoints);
int32_t nca_tree_export(const nca_tree *tree, int32_t *perm, int32_t *begin, int32_t *end,
                        int32_t *parent, int32_t *firstchild, int32_t *nchildren, int32_t *level,
                        double *center, double *radius);

/* ---- admissibility: interactions(tree, isnear(eta)) -> near/far CSR over test nodes
 *      (AdaptiveCrossApproximation.interactions; consumed by src/nca/abstractnca.jl:148 and
 *      src/admissibility/farinteractions.jl:66-92) ---- */
int32_t nca_interactions(const nca_tree *test, const nca_tree *trial, double eta,
                         nca_partition **out);
/* isnearwideband(k; eta_lf, eta_hf, gamma) (src/admissibility/nearinteractions.jl:62-95, bounding
 * balls): low frequency when k min(d) <= gamma, then near iff max(d) > eta_lf sep; high
 * frequency near iff 4 k max(r)^2 > eta_hf sep. A core built on this partition is directional. */
int32_t nca_interactions_wideband(const nca_tree *test, const nca_tree *trial, double k, double etalf,
                                  double etahf, double gamma, nca_partition **out);
void nca_partition_destroy(nca_partition *part);
int32_t nca_partition_sizes(const nca_partition *part, int64_t *nnear, int64_t *nfar);
int32_t nca_partition_export(const nca_partition *part, int32_t *nearptr, int32_t *nearnodes,
                             int32_t *farptr, int32_t *farnodes, int32_t *trialfarptr,
                             int32_t *trialfarnodes);

/* ---- directional far data of one side (directionalfardata(fardata, tree, fartree, isnear),
 *      src/admissibility/directionalsubdivision/boundingballdirections.jl:44-152 and
 *      abstractdirections.jl:57-116) and its basis items, one per (cluster, direction): the
 *      plan the directional core is built on, exposed for inspection. side 0: test tree
 *      (far nodes in the trial tree), 1: trial tree. ---- */
int32_t nca_directional_plan(const nca_tree *tree, const nca_tree *fartree, const nca_partition *part,
                             int32_t side, nca_dirplan **out);
void nca_dirplan_destroy(nca_dirplan *plan);
int32_t nca_dirplan_sizes(const nca_dirplan *plan, int32_t *nitems, int64_t *nfar, int64_t *nchildren);
/* farnodes[nfar] (grouped by direction), dirptr[nnodes+1], dirs[nitems] (0: low frequency, else the
 * 1-based candidate direction), dirvec[3 nitems], dirfarptr[nitems+1], item_basis[nitems],
 * item_chptr[nitems+1], item_chidx[nchildren] (the children's items of nested items). */
int32_t nca_dirplan_export(const nca_dirplan *plan, int32_t *farnodes, int32_t *dirptr, int32_t *dirs, double *dirvec,
                           int32_t *dirfarptr, int32_t *item_basis, int32_t *item_chptr, int32_t *item_chidx);
/* dirfarfield(tree, data, node, dir) of one item (abstractdirections.jl:192-231): its own far
 * nodes, then those of the ancestors' directions that map onto it. Writes min(n, cap) entries. */
int32_t nca_dirplan_farfield(const nca_dirplan *plan, int32_t item, int32_t *out, int32_t cap, int32_t *n);

/* ---- phase 1 for one cluster: _selectfarpivots with tree-mimicry pivoting
 *      (src/compressors/batchedbottomup.jl:54-72) ---- */
int32_t nca_select_farpivots(const nca_tree *fartree, const double *ownpoints,
                             const double *farpoints, const int32_t *refidcs, int32_t nref,
                             const int32_t *farnodes, int32_t nfar, int32_t maxrank,
                             int32_t *pivots, int32_t *npivots);

/* ---- the whole build on one GPU: PetrovGalerkinNCACore(...) with the compressor below on both
 *      sides (src/nca/petrovgalerkinnca.jl:138-198 -> src/nca/abstractnca.jl:134-216 ->
 *      src/compressors/batchedbottomup.jl:246-447 or src/compressors/bottomup.jl:48-424 ->
 *      src/couplingmatrices.jl:11-111) ---- */
/* The compressor of both sides:
 *   NCA_COMPRESSOR_BATCHED_ACA   BatchedBottomUp(pivotselector=TreeMimicryPivoting, compressor=
 *                                ACA(FullPivoting(), FullPivoting(), FNormEstimator(tol)))
 *                                (src/compressors/batchedbottomup.jl:30-51); not for wideband
 *                                partitions, which it refuses with NCA_ERR_ARG as
 *                                src/compressors/abstractcompressor.jl:39-47 does;
 *   NCA_COMPRESSOR_BOTTOMUP_IACA BottomUp(factorization=IACA(MaximumValue(), TreeMimicryPivoting,
 *                                FNormExtrapolator(tol))) on the test side and the mirrored IACA on
 *                                the trial side (src/compressors/bottomup.jl:48-424), per cluster or,
 *                                on a wideband partition, per (cluster, direction). */
typedef enum { NCA_COMPRESSOR_BATCHED_ACA = 0, NCA_COMPRESSOR_BOTTOMUP_IACA = 1 } nca_compressor;

typedef struct {
    double tol_test, tol_trial; /* tolerances of the two compressors */
    int32_t maxrank;            /* maximum rank per cluster (default 50) */
    int32_t sampled;            /* 1: sampled FNorm stop (batchedbottomup.jl:120-125); ACA only */
    int32_t device;             /* CUDA device ordinal */
    int32_t store_f32;          /* 1: also keep complex FP32 copies of all stores */
    int32_t compressor;         /* nca_compressor */
} nca_build_opts;

/* The host planning runs on the process's cores (its CPU affinity mask, capped by a cgroup CPU
 * quota); a directional build also runs its two sides, and then its eight gather plans, on host
 * threads and streams of their own. The call returns once the core is complete. */
int32_t nca_core_build(const double *testpoints, int64_t ntest, const double *trialpoints,
                       int64_t ntrial, const nca_tree *testtree, const nca_tree *trialtree,
                       const nca_partition *part, const nca_kernel_desc *kernel,
                       const nca_build_opts *opts, nca_core **out);
void nca_core_destroy(nca_core *core);

/* Sizes: number of nodes per side and the totals of the device stores. */
typedef struct {
    int64_t ntest, ntrial;
    int32_t nnodes_test, nnodes_trial;
    int64_t ncoeff_test, ncoeff_trial;  /* coefficient vector lengths (plan_from_pivots) */
    int64_t near_entries, coupling_entries, basis_entries_test, basis_entries_trial,
        transfer_entries_test, transfer_entries_trial;
    int64_t nfarpairs, nnearpairs;
    double build_seconds;             /* span of the build's device work (events) */
    double build_seconds_host;        /* host time outside that span */
} nca_core_info;
/* ---- differentiation on frozen skeletons (no counterpart in the reference, which has no
 *      gradients): the tree, partition, ranks and row/column pivots of a build stay fixed. ---- */
/* ---- serialised cores (the reference saves a built matrix's stores and plans with JLD2 for reuse
 *      across runs, scripts/create_test_matrix.jl:50-68) ----
 * nca_core_save writes the core's inputs and skeleton to a file: points, trees, partition, kernel,
 * options and per side (cluster, or directional item) the ranks, block rows, pivots and
 * interpolation operators, plus the directional plan. nca_core_load reads it and rebuilds the
 * couplings, the near field and the product plans on the given device: the loaded core's products
 * equal the saved core's bit for bit. Batches are not saved (save their members); a file that is
 * not a saved core, or is truncated, gives NCA_ERR_ARG. */
int32_t nca_core_save(const nca_core *core, const char *path);
int32_t nca_core_load(const char *path, int32_t device, nca_core **out);

/* Refills every store at wavenumber k with the frozen skeleton: X = K[rows, sigma] K[tau, sigma]^{-1},
 * couplings, near field (and FP32 copies); bit-identical to the build at the build's own k. A
 * singular frozen cross matrix returns NCA_ERR_SINGULAR and leaves the core unchanged. Drops
 * the d/dk stores. */
int32_t nca_core_set_wavenumber(nca_core *core, double k);
/* Prepares the d/dk stores at the core's wavenumber: dX = (dK[rows, sigma] - X dK[tau, sigma])
 * K[tau, sigma]^{-1} per node, dS and dN from the derivative entries (as much memory as the
 * complex FP64 stores). */
int32_t nca_core_prepare_dk(nca_core *core);
/* Batched uneven problems (no counterpart in the reference, which applies one H^2 at a time):
 * one block-diagonal core over ncores built cores of one device, so a product covers all of them
 * in one launch per stage level. x and y are the members' vectors stacked in member order. The
 * batch copies the members' stores (the members may be destroyed afterwards); with
 * NCA_BATCH_MOVE_STORES each member's device stores are released as soon as they are copied, so
 * the peak stays near one copy, and the members may afterwards only be destroyed (every other
 * call on them returns NCA_ERR_ARG). Exports of a batch list the members' nodes, points and
 * pairs renumbered in member order. */
#define NCA_BATCH_MOVE_STORES 1
int32_t nca_core_batch(nca_core *const *cores, int32_t ncores, int32_t flags, nca_core **out);
int32_t nca_core_get_info(const nca_core *core, nca_core_info *info);

/* Pivots per node of one side (the third return value of testbases/trialbases,
 * batchedbottomup.jl:344,446): ranks[nnodes], ptr[nnodes+1], idx[ptr[nnodes]]. */
int32_t nca_core_export_pivots(const nca_core *core, int32_t side, int32_t *ranks, int32_t *nrows,
                               int32_t *ptr, int32_t *idx);
/* Directional cores: the basis items of one side (the plan's items, in its order) with their
 * ranks, block rows and row pivots (tpivots/spivots of the directional compressor,
 * src/compressors/bottomup.jl:214-424). Call with ranks = NULL for the item count. */
int32_t nca_core_dir_items(const nca_core *core, int32_t side, int32_t *nitems, int32_t *ranks, int32_t *nrows,
                           int32_t *ptr, int32_t *idx);
/* Far pivots of phase 1 per node of one side: ptr[nnodes+1], idx. */
int32_t nca_core_farpivots_total(const nca_core *core, int32_t side, int64_t *total);
int32_t nca_core_export_farpivots(const nca_core *core, int32_t side, int32_t *ptr, int32_t *idx);
/* Interpolation operator X_t = A[rows, sigma] A[tau, sigma]^{-1} of every node (nrows x rank,
 * column-major): the leaf basis (test: X, trial: X^T) or the stacked transfer matrices
 * (nestedbasis.jl:43-57, transfermatrices.jl:183-211). off[nnodes+1] counts complex entries. */
int32_t nca_core_export_x(const nca_core *core, int32_t side, int64_t *off, double *X);
/* Coupling matrices in test-node CSR order (couplingmatrices.jl:11-53). */
int32_t nca_core_export_couplings(const nca_core *core, int64_t *off, double *C);
/* Near-field block rows per test node (abstractnca.jl:134-178). */
int32_t nca_core_export_near(const nca_core *core, int64_t *off, int32_t *ncols, double *N);

/* ---- the H^2 product: H2Workspace + _unsafe_mul!/_mul! (petrovgalerkinnca.jl:253-271,
 *      :415-589). A workspace owns the coefficient buffers and two CUDA streams (the product
 *      stream and, for non-directional cores, a higher-priority stream for the far-field
 *      sweeps, joined back before the leaf bases). ---- */
int32_t nca_workspace_create(nca_core *core, int32_t max_nrhs, nca_workspace **out);
void nca_workspace_destroy(nca_workspace *ws);
/* y = alpha * op(H) x + beta * y for nrhs columns. memspace 0: x and y are host pointers
 * (copies are part of the call); 1: device pointers. x, y are complex FP64 (interleaved). */
int32_t nca_apply(nca_workspace *ws, int32_t mode, int32_t precision, const void *x, int64_t ldx,
                  void *y, int64_t ldy, int64_t nrhs, double alpha_re, double alpha_im,
                  double beta_re, double beta_im, int32_t memspace);
/* Allocation-free product (no counterpart in the reference, whose products always run on an
 * H2Workspace's own buffers): y = alpha * op(H) x + beta * y with x, y DEVICE arrays (16-byte
 * aligned) on the caller's stream (NULL: the legacy default stream), every intermediate buffer
 * in one fixed device array of NCA_STATIC_SCRATCH_BYTES per device that the library's module
 * holds. The call makes no cudaMalloc/cudaFree or other allocation, for callers whose own pool
 * owns device memory. It needs (nin + input coefficients + output coefficients) *
 * (nrhs + 3) * 16 bytes + 1 KiB at most; larger products return NCA_ERR_ARG naming the size.
 * Non-directional cores only: a directional (wideband) core returns NCA_ERR_ARG (use
 * nca_apply). The first call on a device does the one-time setup (module load, symbol lookup),
 * which reserves the array on that device unless CUDA_MODULE_LOADING=EAGER reserved it when the
 * library was loaded: make that call before the caller's pool reserves HBM. The scratch is shared
 * by every core on the device, so overlapping calls would race on it: a call made while another is
 * in progress on the same device returns NCA_ERR_BUSY. The call waits for the stream and returns
 * the kernels' status, so it cannot be captured in a CUDA graph: on a capturing stream it returns
 * NCA_ERR_ARG. */
#define NCA_STATIC_SCRATCH_BYTES (32ull << 20)
int32_t nca_apply_static(nca_core *core, int32_t mode, int32_t precision, const void *x, int64_t ldx,
                         void *y, int64_t ldy, int64_t nrhs, double alpha_re, double alpha_im,
                         double beta_re, double beta_im, void *stream);
/* Tangent product y = alpha (dH/dk) x + beta y (forward mode, complex FP64, after
 * nca_core_prepare_dk): the sweeps of nca_apply carried as dual numbers. With the adjoint product
 * it gives the gradients of a loss through y = H(k) x: x_bar = H^H y_bar (nca_apply mode C) and
 * k_bar = Re(y_bar^H (dH/dk) x). No counterpart in the reference. */
int32_t nca_apply_dk(nca_workspace *ws, const void *x, int64_t ldx, void *y, int64_t ldy, int64_t nrhs,
                     double alpha_re, double alpha_im, double beta_re, double beta_im, int32_t memspace);
/* Device time of the last nca_apply of this workspace (CUDA events), in seconds. */
int32_t nca_workspace_last_time(const nca_workspace *ws, double *seconds);
/* Kernel launches of the last nca_apply of this workspace. */
int32_t nca_workspace_last_launches(const nca_workspace *ws, int32_t *launches);
/* Which parts the workspace applies: the far field (nested bases, transfers, couplings) and/or
 * the near field. farmatrix / nearmatrix of the reference (petrovgalerkinnca.jl:344-371). */
int32_t nca_workspace_set_parts(nca_workspace *ws, int32_t far, int32_t near);
/* Stage timers (CUDA events around each stage). With profiling on, nca_workspace_stage_times
 * returns the device seconds and launches of the last nca_apply per stage: 0 gather of x,
 * 1 upward sweep, 2 coupling, 3 downward sweep, 4 near field, 5 leaves. A workspace runs the
 * three sweeps on a second stream of its own beside the near field (stage 4) and then adds the
 * leaf bases (stage 5); with only one part present, stage 5 is the whole leaf launch and
 * stage 4 is empty. Stages 1-3 and 4 overlap in time. */
int32_t nca_workspace_set_profiling(nca_workspace *ws, int32_t on);
/* CUDA-graph replay (no counterpart in the reference, whose products run on the CPU; off by
 * default): an nca_apply on device arrays (memspace 1) whose arguments
 * (mode, precision, pointers, leading dimensions, nrhs, alpha, beta, parts, profiling) equal one
 * of the workspace's last few calls is captured once into a CUDA graph, and later identical calls
 * launch that graph instead of enqueueing every stage. Results are bitwise those of the enqueued
 * product. It pays off for launch-bound products (small problems); for large ones it is slower,
 * because the graph loses the overlap of the far-field sweeps with the near field (measured on the
 * 65,536-point sphere: 1.53 ms per step with graphs, 1.46 ms without). */
int32_t nca_workspace_set_graphs(nca_workspace *ws, int32_t on);
/* Schedule autotuner (no counterpart in the reference): times the product (mode, precision, nrhs
 * columns, on zero device arrays of
 * the workspace's own) under each schedule — near field beside the far-field sweeps or after
 * them, with or without CUDA-graph replay — and keeps the fastest for the workspace. choice
 * (nullable) receives bit 0 = overlap, bit 1 = graphs. Results do not depend on the schedule
 * beyond the rounding of the final sum (overlap) and are bitwise equal with and without graphs. */
int32_t nca_workspace_autotune(nca_workspace *ws, int32_t mode, int32_t precision, int64_t nrhs, int32_t *choice);
int32_t nca_workspace_stage_times(const nca_workspace *ws, double *seconds, int32_t *launches,
                                  int32_t nstages);

/* ---- level seams on caller-given blocks (batchedbottomup.jl:101-244, the CUDA extension's
 *      ext/NestedCrossApproximationCUDAExt/compresslevel.jl:31-137): fully pivoted ACA and
 *      the interpolation solve of every block of a packed level buffer
 *      (rows rowoffsets[i]..rowoffsets[i+1]-1, columns 0..ncols[i]-1 of a (sum m) x ldcols
 *      column-major complex FP64 host buffer). ---- */
int32_t nca_blocks_aca(const double *buffer, int64_t ldbuffer, int32_t ldcols,
                       const int64_t *rowoffsets, const int32_t *ncols, int32_t nblocks,
                       int32_t maxrank, double tol, int32_t sampled, int32_t device,
                       int32_t *ranks, int32_t *rowpivots, int32_t *colpivots);
/* Z_i = X_i^T with X_i = L_i P_i^{-1}, L_i = A_i[:, colpivots], P_i = L_i[rowpivots, :]
 * (compresslevel.jl:88-137). Z is rank_i x m_i per block at zoff[i] (complex entries).
 * Singular cross matrices give NCA_ERR_SINGULAR and nca_last_singular(node = block). */
int32_t nca_blocks_factors(const double *buffer, int64_t ldbuffer, int32_t ldcols,
                           const int64_t *rowoffsets, int32_t nblocks, const int32_t *ranks,
                           const int32_t *rowpivots, const int32_t *colpivots, int32_t maxrank,
                           int32_t device, const int64_t *zoff, double *Z);

/* ---- kernel entries: A(i, j) for index pairs (AbstractKernelMatrix entry evaluation) ---- */
int32_t nca_entries(const nca_kernel_desc *kernel, const double *testpoints, int64_t ntest,
                    const double *trialpoints, int64_t ntrial, const int64_t *ii,
                    const int64_t *jj, int64_t n, int32_t device, double *out);

/* d/dk of the point-kernel entries (Helmholtz: (-sin(kr) + i sign cos(kr)) / (4 pi); Laplace: 0);
 * no counterpart in the reference. Matrix kernels return NCA_ERR_ARG. */
int32_t nca_entries_dk(const nca_kernel_desc *kernel, const double *testpoints, int64_t ntest,
                       const double *trialpoints, int64_t ntrial, const int64_t *ii,
                       const int64_t *jj, int64_t n, int32_t device, double *out);

#ifdef __cplusplus
}
#endif
#endif
