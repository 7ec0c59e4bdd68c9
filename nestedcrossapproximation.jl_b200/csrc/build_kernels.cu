// Device kernels of the batched bottom-up build (phases 2 and 3 of
// src/compressors/batchedbottomup.jl, fused):
//
//   k_level_compress  one CTA per active cluster of a level: gathers the block rows (the
//                     cluster's points for a leaf, the children's pivots otherwise,
//                     batchedbottomup.jl:285-303), evaluates K[rows, farpivots] into shared
//                     memory (assemble_level, :101-116; trial side transposed, :98-99),
//                     runs the fully pivoted ACA with the sampled Frobenius stop
//                     (_compressblock, :120-125), factorises the cross matrix with partial
//                     pivoting and the singular check of _crossfactorization
//                     (src/utils/utils.jl:57-80), and writes X = A[:, sigma] A[tau, sigma]^{-1}
//                     (nestedbasis.jl:43-57, transfermatrices.jl:183-211) plus the pivots.
//   k_couplings       S_ts = K[tau_t, sigma_s] for every admissible pair (couplingmatrices.jl:11-53).
//   k_near            dense near-field blocks (src/nca/abstractnca.jl:134-178).
//
// The ACA reproduces the host restatement bit for bit: explicit _rn intrinsics (the file is
// also compiled with --fmad=false), argmax ties to the lowest column-major index, and the
// residual norm summed in one fixed order (256 strided partial sums, halving trees inside
// each warp, then over the 8 warp totals).
#include <cuda_runtime.h>

#include <cstdint>

#include "build_kernels.cuh"
#include "entry.cuh"

namespace nca {

namespace {

constexpr int NT = 256;  // the fixed reduction order is defined for 256 partial sums
constexpr int NWARP = NT / 32;

struct Scan {
    double sum;
    double vmax;
    int emax;
};

// Block reduction of per-thread (partial sum, local argmax) in the fixed order.
__device__ Scan block_scan(double acc, double bv, int be, double *wsum, double *wmax, int *widx) {
    const unsigned full = 0xffffffffu;
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int off = 16; off >= 1; off >>= 1) {
        double o = __shfl_down_sync(full, acc, off);
        double ov = __shfl_down_sync(full, bv, off);
        int oe = __shfl_down_sync(full, be, off);
        acc = __dadd_rn(acc, o);
        if (ov > bv || (ov == bv && oe >= 0 && (be < 0 || oe < be))) {
            bv = ov;
            be = oe;
        }
    }
    if (lane == 0) {
        wsum[warp] = acc;
        wmax[warp] = bv;
        widx[warp] = be;
    }
    __syncthreads();
    Scan s;
    {
        double w[NWARP];
        for (int k = 0; k < NWARP; ++k) w[k] = wsum[k];
        for (int off = NWARP / 2; off >= 1; off >>= 1)
            for (int k = 0; k < off; ++k) w[k] = __dadd_rn(w[k], w[k + off]);
        s.sum = w[0];
        double v = -1.0;
        int e = -1;
        for (int k = 0; k < NWARP; ++k) {
            double ov = wmax[k];
            int oe = widx[k];
            if (ov > v || (ov == v && oe >= 0 && (e < 0 || oe < e))) {
                v = ov;
                e = oe;
            }
        }
        s.vmax = v;
        s.emax = e;
    }
    __syncthreads();
    return s;
}

__device__ __forceinline__ double2 block_entry(const LevelArgs &a, const double *rowxyz,
                                               const int32_t *rowid, const double *colxyz,
                                               const int32_t *colid, int i, int j) {
    const double *p = rowxyz + 3 * i;
    const double *q = colxyz + 3 * j;
    if (a.side == 0)
        return kernel_entry(a.K, p[0], p[1], p[2], q[0], q[1], q[2], rowid[i], colid[j]);
    return kernel_entry(a.K, q[0], q[1], q[2], p[0], p[1], p[2], colid[j], rowid[i]);
}

}  // namespace

size_t level_smem_bytes(int mcap, int ncap) {
    size_t b = 0;
    b += sizeof(double2) * size_t(mcap) * ncap;  // R (the cross matrix P lives in the node's X slot)
    b += sizeof(double2) * (mcap + ncap);        // u, v
    b += sizeof(double) * 3 * (mcap + ncap);     // coordinates
    b += sizeof(int32_t) * (mcap + 3 * ncap);    // row ids, col ids, rp, cp, ipiv
    b += sizeof(int32_t) * ncap;
    return (b + 15) & ~size_t(15);
}

// Fully pivoted ACA of the m x n block in R (column-major, overwritten by the residual).
// Writes the local row/column pivots, returns the rank. All threads of the CTA call it.
__device__ int aca_smem(double2 *R, int m, int n, int maxrank, double tol, int sampled,
                        double2 *u, double2 *v, int32_t *rp, int32_t *cp, double *wsum,
                        double *wmax, int *widx) {
    const int tid = threadIdx.x;
    const int len = m * n;
    double acc = 0.0, bv = -1.0;
    int be = -1;
    for (int e = tid; e < len; e += NT) {
        double s2 = cabs2_rn(R[e]);
        acc = __dadd_rn(acc, s2);
        if (s2 > bv) {
            bv = s2;
            be = e;
        }
    }
    Scan sc = block_scan(acc, bv, be, wsum, wmax, widx);
    const double normA2 = sc.sum;
    const double rhs = __dmul_rn(__dmul_rn(tol, tol), normA2);
    double normR2 = normA2;
    int limit = maxrank < m ? maxrank : m;
    if (n < limit) limit = n;
    int r = 0;
    while (r < limit) {
        if (!(sc.vmax > 0.0)) break;
        double lhs = sampled ? __ddiv_rn(__dmul_rn(normR2, double(n)), double(n - r)) : normR2;
        if (lhs <= rhs) break;
        const int ip = sc.emax % m, jp = sc.emax / m;
        if (tid == 0) {
            rp[r] = ip;
            cp[r] = jp;
        }
        double2 p = R[ip + jp * m];
        double d = cabs2_rn(p);
        double2 w = make_double2(__ddiv_rn(p.x, d), -__ddiv_rn(p.y, d));
        for (int i = tid; i < m; i += NT) u[i] = R[i + jp * m];
        for (int j = tid; j < n; j += NT) v[j] = cmul_rn(R[ip + j * m], w);
        __syncthreads();
        acc = 0.0;
        bv = -1.0;
        be = -1;
        for (int e = tid; e < len; e += NT) {
            int i = e % m, j = e / m;
            double2 val;
            if (i == ip || j == jp) {
                val = make_double2(0.0, 0.0);
            } else {
                double2 t = cmul_rn(u[i], v[j]);
                double2 x = R[e];
                val = make_double2(__dsub_rn(x.x, t.x), __dsub_rn(x.y, t.y));
            }
            R[e] = val;
            double s2 = cabs2_rn(val);
            acc = __dadd_rn(acc, s2);
            if (s2 > bv) {
                bv = s2;
                be = e;
            }
        }
        sc = block_scan(acc, bv, be, wsum, wmax, widx);
        normR2 = sc.sum;
        ++r;
    }
    __syncthreads();
    return r;
}

// LU with partial pivoting of the r x r cross matrix P (the CTA's shared or global memory, in
// place, ordered by the block barriers) and the singular check of _crossfactorization:
// |U_ii|^2 <= (10 eps)^2 max|U_jj|^2 for some i, or an exactly zero pivot. Returns 1 if singular
// (*rank_out: numerical rank). All threads call it.
__device__ int cross_factor_smem(double2 *P, int r, int32_t *ipiv, int *s_flag, int *rank_out) {
    const int tid = threadIdx.x;
    if (tid == 0) *s_flag = 0;
    __syncthreads();
    for (int k = 0; k < r; ++k) {
        if (tid < 32) {
            double best = -1.0;
            int arg = -1;
            for (int i = k + tid; i < r; i += 32) {
                double av = cabs2_rn(P[i + k * r]);
                if (av > best) {
                    best = av;
                    arg = i;
                }
            }
            for (int off = 16; off >= 1; off >>= 1) {
                double ob = __shfl_down_sync(0xffffffffu, best, off);
                int oa = __shfl_down_sync(0xffffffffu, arg, off);
                if (ob > best || (ob == best && oa >= 0 && (arg < 0 || oa < arg))) {
                    best = ob;
                    arg = oa;
                }
            }
            if (tid == 0) ipiv[k] = arg;
        }
        __syncthreads();
        const int pr = ipiv[k];
        if (pr != k) {
            for (int j = tid; j < r; j += NT) {
                double2 t = P[k + j * r];
                P[k + j * r] = P[pr + j * r];
                P[pr + j * r] = t;
            }
        }
        __syncthreads();
        double2 pv = P[k + k * r];
        double dd = cabs2_rn(pv);
        if (dd == 0.0) {
            if (tid == 0) *s_flag = 1;
            __syncthreads();
            continue;
        }
        double2 wi = make_double2(__ddiv_rn(pv.x, dd), -__ddiv_rn(pv.y, dd));
        for (int i = k + 1 + tid; i < r; i += NT) P[i + k * r] = cmul_rn(P[i + k * r], wi);
        __syncthreads();
        const int tr = r - k - 1;
        for (int e = tid; e < tr * tr; e += NT) {
            int i = k + 1 + e % tr, j = k + 1 + e / tr;
            double2 t = cmul_rn(P[i + k * r], P[k + j * r]);
            P[i + j * r].x -= t.x;
            P[i + j * r].y -= t.y;
        }
        __syncthreads();
    }
    double d2max = 0.0, d2min = 1.0 / 0.0;
    for (int i = 0; i < r; ++i) {
        double d2 = cabs2_rn(P[i + i * r]);
        d2max = d2 > d2max ? d2 : d2max;
        d2min = d2 < d2min ? d2 : d2min;
    }
    const double eps = 0x1p-52;
    const double tol2 = (10.0 * eps) * (10.0 * eps) * d2max;
    int singular = *s_flag || !(d2min > tol2);
    if (singular) {
        int rank = 0;
        for (int i = 0; i < r; ++i) rank += cabs2_rn(P[i + i * r]) > tol2;
        *rank_out = rank;
    }
    __syncthreads();
    return singular;
}

// One row x of X P = L (length r, elements x[j * stride]) with P = Pi^T L U factored:
// x <- ((x U^{-1}) L^{-1}) Pi.
__device__ void solve_row(double2 *x, int stride, int r, const double2 *P, const int32_t *ipiv) {
    for (int j = 0; j < r; ++j) {
        double2 acc2 = x[j * stride];
        for (int l = 0; l < j; ++l) {
            double2 t = cmul_rn(x[l * stride], P[l + j * r]);
            acc2.x -= t.x;
            acc2.y -= t.y;
        }
        double2 uu = P[j + j * r];
        double du = cabs2_rn(uu);
        x[j * stride] = cmul_rn(acc2, make_double2(uu.x / du, -(uu.y / du)));
    }
    for (int j = r - 1; j >= 0; --j) {
        double2 acc2 = x[j * stride];
        for (int l = j + 1; l < r; ++l) {
            double2 t = cmul_rn(x[l * stride], P[l + j * r]);
            acc2.x -= t.x;
            acc2.y -= t.y;
        }
        x[j * stride] = acc2;
    }
    for (int k = r - 1; k >= 0; --k) {
        int pk = ipiv[k];
        if (pk != k) {
            double2 t = x[k * stride];
            x[k * stride] = x[pk * stride];
            x[pk * stride] = t;
        }
    }
}

__global__ void __launch_bounds__(NT) k_level_compress(LevelArgs a, const int32_t *nodes, int mcap,
                                                       int ncap) {
    extern __shared__ __align__(16) unsigned char smem[];
    double2 *R = reinterpret_cast<double2 *>(smem);
    double2 *u = R + size_t(mcap) * ncap;
    double2 *v = u + mcap;
    double *rowxyz = reinterpret_cast<double *>(v + ncap);
    double *colxyz = rowxyz + 3 * mcap;
    int32_t *rowid = reinterpret_cast<int32_t *>(colxyz + 3 * ncap);
    int32_t *colid = rowid + mcap;
    int32_t *rp = colid + ncap;
    int32_t *cp = rp + ncap;
    int32_t *ipiv = cp + ncap;
    __shared__ double wsum[NWARP], wmax[NWARP];
    __shared__ int widx[NWARP];
    __shared__ int s_m, s_flag;

    const int tid = threadIdx.x;
    const int node = nodes[blockIdx.x];
    const int n = a.fpptr[node + 1] - a.fpptr[node];
    const int32_t *fp = a.fpidx + a.fpptr[node];
    const bool leaf = a.nchildren[node] == 0;
    const int nch = a.nchildren[node];
    auto child = [&](int c) { return a.firstchild[node] + c; };

    // rows of the block: the cluster's points, or the children's pivots in child order
    if (tid == 0) {
        int m = 0;
        if (leaf) {
            m = a.end[node] - a.begin[node];
        } else {
            for (int c = 0; c < nch; ++c) m += a.rank[child(c)];
        }
        s_m = m;
    }
    __syncthreads();
    const int m = s_m;
    if (m > mcap || n > ncap) {
        if (tid == 0 && atomicCAS(a.status, 0, 2) == 0) {
            a.status[1] = node;
            a.status[2] = m;
            a.status[3] = n;
        }
        return;
    }
    if (leaf) {
        for (int i = tid; i < m; i += NT) rowid[i] = a.perm[a.begin[node] + i];
    } else {
        int off = 0;
        for (int c = 0; c < nch; ++c) {
            const int ch = child(c);
            const int kc = a.rank[ch];
            for (int k = tid; k < kc; k += NT) rowid[off + k] = a.piv[int64_t(ch) * a.maxrank + k];
            off += kc;
        }
    }
    for (int j = tid; j < n; j += NT) colid[j] = fp[j];
    __syncthreads();
    for (int e = tid; e < 3 * m; e += NT) rowxyz[e] = a.own_pts[3 * int64_t(rowid[e / 3]) + e % 3];
    for (int e = tid; e < 3 * n; e += NT) colxyz[e] = a.far_pts[3 * int64_t(colid[e / 3]) + e % 3];
    __syncthreads();

    // phase 2: the block against the far pivots
    for (int e = tid; e < m * n; e += NT)
        R[e] = block_entry(a, rowxyz, rowid, colxyz, colid, e % m, e / m);
    __syncthreads();

    // phase 3a: pivots
    const int r = aca_smem(R, m, n, a.maxrank, a.tol, a.sampled, u, v, rp, cp, wsum, wmax, widx);
    for (int k = tid; k < r; k += NT) a.piv[int64_t(node) * a.maxrank + k] = rowid[rp[k]];
    if (a.cpiv)
        for (int k = tid; k < r; k += NT) a.cpiv[int64_t(node) * a.maxrank + k] = colid[cp[k]];
    if (tid == 0) {
        a.rank[node] = r;
        a.nrows[node] = m;
    }
    if (r == 0) return;

    // phase 3b: L = A[:, cp] regenerated into R, P = L[rp, :], X = L P^{-1}. The r x r cross
    // matrix is factorised in the node's own X slot (m x rank bound >= r x r entries, in L2),
    // which keeps shared memory to the block and lets more CTAs share an SM; X overwrites it
    // once every row is solved.
    double2 *P = a.X + a.xoff[node];
    for (int e = tid; e < m * r; e += NT)
        R[e] = block_entry(a, rowxyz, rowid, colxyz, colid, e % m, cp[e / m]);
    __syncthreads();
    for (int e = tid; e < r * r; e += NT) P[e] = R[rp[e % r] + (e / r) * m];
    __syncthreads();
    int rank = 0;
    if (cross_factor_smem(P, r, ipiv, &s_flag, &rank)) {
        if (tid == 0 && atomicCAS(a.status, 0, 1) == 0) {
            a.status[1] = node;
            a.status[2] = r;
            a.status[3] = rank;
        }
        return;
    }
    for (int i = tid; i < m; i += NT) solve_row(R + i, m, r, P, ipiv);
    __syncthreads();
    double2 *X = a.X + a.xoff[node];
    for (int e = tid; e < m * r; e += NT) X[e] = R[e];
}

size_t values_smem_bytes(int mcap, int rcap, int mode) {
    size_t b = sizeof(double2) * (size_t(mcap) * rcap + size_t(rcap) * rcap * (mode ? 2 : 1));
    b += sizeof(double) * 3 * (size_t(mcap) + 2 * rcap);
    b += sizeof(int32_t) * (size_t(mcap) + 3 * rcap);
    return (b + 15) & ~size_t(15);
}

namespace {
// K(row point i, column point j) with the side's orientation (test rows / trial columns on side 0)
__device__ __forceinline__ double2 oriented_entry(const KernelParams &K, int side, const double *rowxyz,
                                                  const int32_t *rowid, const double *colxyz,
                                                  const int32_t *colid, int i, int j) {
    const double *p = rowxyz + 3 * i;
    const double *q = colxyz + 3 * j;
    if (side == 0) return kernel_entry(K, p[0], p[1], p[2], q[0], q[1], q[2], rowid[i], colid[j]);
    return kernel_entry(K, q[0], q[1], q[2], p[0], p[1], p[2], colid[j], rowid[i]);
}
}  // namespace

__global__ void __launch_bounds__(NT) k_level_values(ValueArgs a, const int32_t *nodes, int mcap, int rcap) {
    extern __shared__ __align__(16) unsigned char smem[];
    double2 *L = reinterpret_cast<double2 *>(smem);
    double2 *P = L + size_t(mcap) * rcap;
    double2 *dP = P + size_t(rcap) * rcap;
    double *rowxyz = reinterpret_cast<double *>(dP + (a.mode ? size_t(rcap) * rcap : 0));
    double *colxyz = rowxyz + 3 * mcap;
    double *tauxyz = colxyz + 3 * rcap;
    int32_t *rowid = reinterpret_cast<int32_t *>(tauxyz + 3 * rcap);
    int32_t *colid = rowid + mcap;
    int32_t *tauid = colid + rcap;
    int32_t *ipiv = tauid + rcap;
    __shared__ int s_m, s_flag;
    const int tid = threadIdx.x;
    const int node = nodes[blockIdx.x];  // the node, or the directional item
    const int r = a.rank[node];
    if (r <= 0) return;
    const bool items = a.item_node != nullptr;
    const int cl = items ? a.item_node[node] : node;
    const bool leaf = items ? a.item_basis[node] != 0 : a.nchildren[node] == 0;
    const int nch = leaf ? 0 : items ? a.item_chptr[node + 1] - a.item_chptr[node] : a.nchildren[node];
    auto child = [&](int c) { return items ? a.item_chidx[a.item_chptr[node] + c] : a.firstchild[node] + c; };
    if (tid == 0) {
        int m = 0;
        if (leaf) {
            m = a.end[cl] - a.begin[cl];
        } else {
            for (int c = 0; c < nch; ++c) m += a.rank[child(c)];
        }
        s_m = m;
    }
    __syncthreads();
    const int m = s_m;
    if (m > mcap || r > rcap) {
        if (tid == 0 && atomicCAS(a.status, 0, 2) == 0) {
            a.status[1] = node;
            a.status[2] = m;
            a.status[3] = r;
        }
        return;
    }
    if (leaf) {
        for (int i = tid; i < m; i += NT) rowid[i] = a.perm[a.begin[cl] + i];
    } else {
        int off = 0;
        for (int c = 0; c < nch; ++c) {
            const int ch = child(c);
            const int kc = a.rank[ch];
            for (int k = tid; k < kc; k += NT) rowid[off + k] = a.piv[int64_t(ch) * a.maxrank + k];
            off += kc;
        }
    }
    for (int j = tid; j < r; j += NT) {
        colid[j] = a.cpiv[int64_t(node) * a.maxrank + j];
        tauid[j] = a.piv[int64_t(node) * a.maxrank + j];
    }
    __syncthreads();
    for (int e = tid; e < 3 * m; e += NT) rowxyz[e] = a.own_pts[3 * int64_t(rowid[e / 3]) + e % 3];
    for (int e = tid; e < 3 * r; e += NT) {
        colxyz[e] = a.far_pts[3 * int64_t(colid[e / 3]) + e % 3];
        tauxyz[e] = a.own_pts[3 * int64_t(tauid[e / 3]) + e % 3];
    }
    __syncthreads();
    const KernelParams &KL = a.mode ? a.dK : a.K;
    for (int e = tid; e < m * r; e += NT) L[e] = oriented_entry(KL, a.side, rowxyz, rowid, colxyz, colid, e % m, e / m);
    for (int e = tid; e < r * r; e += NT) {
        P[e] = oriented_entry(a.K, a.side, tauxyz, tauid, colxyz, colid, e % r, e / r);
        if (a.mode) dP[e] = oriented_entry(a.dK, a.side, tauxyz, tauid, colxyz, colid, e % r, e / r);
    }
    __syncthreads();
    if (a.mode) {
        // M = dL - X dP, row by row into L
        const double2 *X = a.Xin + a.xoff[node];
        for (int e = tid; e < m * r; e += NT) {
            const int i = e % m, j = e / m;
            double2 acc = L[e];
            for (int l = 0; l < r; ++l) {
                const double2 t = cmul_rn(X[i + int64_t(l) * m], dP[l + j * r]);
                acc.x -= t.x;
                acc.y -= t.y;
            }
            L[e] = acc;
        }
        __syncthreads();
    }
    int rank = 0;
    if (cross_factor_smem(P, r, ipiv, &s_flag, &rank)) {
        if (tid == 0 && atomicCAS(a.status, 0, 1) == 0) {
            a.status[1] = node;
            a.status[2] = r;
            a.status[3] = rank;
        }
        return;
    }
    for (int i = tid; i < m; i += NT) solve_row(L + i, m, r, P, ipiv);
    __syncthreads();
    double2 *X = a.Xout + a.xoff[node];
    for (int e = tid; e < m * r; e += NT) X[e] = L[e];
}

// Level seam on caller-given blocks: block i holds rows rowoff[i]..rowoff[i+1]-1 and
// columns 0..ncols[i]-1 of a column-major buffer with leading dimension ld.
__global__ void __launch_bounds__(NT) k_blocks_aca(const double2 *buf, int64_t ld,
                                                   const int64_t *rowoff, const int32_t *ncols,
                                                   int maxrank, double tol, int sampled, int mcap,
                                                   int ncap, int32_t *ranks, int32_t *rowpiv,
                                                   int32_t *colpiv) {
    extern __shared__ __align__(16) unsigned char smem[];
    double2 *R = reinterpret_cast<double2 *>(smem);
    double2 *u = R + size_t(mcap) * ncap;
    double2 *v = u + mcap;
    int32_t *rp = reinterpret_cast<int32_t *>(v + ncap);
    int32_t *cp = rp + ncap;
    __shared__ double wsum[NWARP], wmax[NWARP];
    __shared__ int widx[NWARP];
    const int blk = blockIdx.x;
    const int m = int(rowoff[blk + 1] - rowoff[blk]), n = ncols[blk];
    for (int e = threadIdx.x; e < m * n; e += NT) R[e] = buf[rowoff[blk] + e % m + (e / m) * ld];
    __syncthreads();
    const int r = (m > 0 && n > 0) ? aca_smem(R, m, n, maxrank, tol, sampled, u, v, rp, cp, wsum, wmax, widx) : 0;
    for (int k = threadIdx.x; k < maxrank; k += NT) {
        rowpiv[int64_t(blk) * maxrank + k] = k < r ? rp[k] : -1;
        colpiv[int64_t(blk) * maxrank + k] = k < r ? cp[k] : -1;
    }
    if (threadIdx.x == 0) ranks[blk] = r;
}

// Z_i = (L_i P_i^{-1})^T per block (the transposed interpolation operator). Only the r x r
// cross matrix lives in shared memory; each thread solves one row of X in place in Z, where
// that row is a contiguous column (any block height fits).
__global__ void __launch_bounds__(NT) k_blocks_factors(const double2 *buf, int64_t ld,
                                                       const int64_t *rowoff, const int32_t *ranks,
                                                       const int32_t *rowpiv, const int32_t *colpiv,
                                                       int maxrank, const int64_t *zoff, double2 *Z,
                                                       int32_t *status) {
    extern __shared__ __align__(16) unsigned char smem[];
    double2 *P = reinterpret_cast<double2 *>(smem);
    int32_t *ipiv = reinterpret_cast<int32_t *>(P + size_t(maxrank) * maxrank);
    __shared__ int s_flag;
    const int blk = blockIdx.x;
    const int m = int(rowoff[blk + 1] - rowoff[blk]), r = ranks[blk];
    if (r == 0) return;
    const int32_t *rp = rowpiv + int64_t(blk) * maxrank;
    const int32_t *cp = colpiv + int64_t(blk) * maxrank;
    const double2 *A = buf + rowoff[blk];
    for (int e = threadIdx.x; e < r * r; e += NT) P[e] = A[rp[e % r] + int64_t(cp[e / r]) * ld];
    __syncthreads();
    double2 *z = Z + zoff[blk];
    for (int e = threadIdx.x; e < m * r; e += NT) {
        int i = e % m, k = e / m;
        z[k + int64_t(i) * r] = A[i + int64_t(cp[k]) * ld];
    }
    int rank = 0;
    // LU of P; the rows are solved below with leading dimension 1 and stride r per row
    if (cross_factor_smem(P, r, ipiv, &s_flag, &rank)) {
        if (threadIdx.x == 0 && atomicCAS(status, 0, 1) == 0) {
            status[1] = blk;
            status[2] = r;
            status[3] = rank;
        }
        return;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < m; i += NT) solve_row(z + int64_t(i) * r, 1, r, P, ipiv);
}

// ---------------------------------------------------------------------------------------
// Coupling and near-field entries
// ---------------------------------------------------------------------------------------

__global__ void __launch_bounds__(256) k_couplings(CouplingArgs a) {
    __shared__ double tx[3 * 256], sx[3 * 256];
    __shared__ int32_t tid_[256], sid_[256];
    for (int64_t pair = blockIdx.x; pair < a.npairs; pair += gridDim.x) {
        int t = a.pair_t[pair], s = a.pair_s[pair];
        int kt = a.rank_t[t], ks = a.rank_s[s];
        __syncthreads();
        for (int i = threadIdx.x; i < kt; i += blockDim.x) {
            int32_t id = a.piv_t[int64_t(t) * a.maxrank + i];
            tid_[i] = id;
            for (int d = 0; d < 3; ++d) tx[3 * i + d] = a.test_pts[3 * int64_t(id) + d];
        }
        for (int j = threadIdx.x; j < ks; j += blockDim.x) {
            int32_t id = a.piv_s[int64_t(s) * a.maxrank + j];
            sid_[j] = id;
            for (int d = 0; d < 3; ++d) sx[3 * j + d] = a.trial_pts[3 * int64_t(id) + d];
        }
        __syncthreads();
        double2 *S = a.C + a.coff[pair];
        float2 *S32 = a.C32 ? a.C32 + a.coff[pair] : nullptr;
        for (int e = threadIdx.x; e < kt * ks; e += blockDim.x) {
            int i = e % kt, j = e / kt;
            double2 v = kernel_entry(a.K, tx[3 * i], tx[3 * i + 1], tx[3 * i + 2], sx[3 * j],
                                     sx[3 * j + 1], sx[3 * j + 2], tid_[i], sid_[j]);
            S[e] = v;
            if (S32) S32[e] = make_float2(float(v.x), float(v.y));
        }
    }
}

__global__ void __launch_bounds__(256) k_near(NearArgs a) {
    for (int64_t pair = blockIdx.x; pair < a.npairs; pair += gridDim.x) {
        int t = a.pair_t[pair], s = a.pair_s[pair];
        int tb = a.t_begin[t], mt = a.t_end[t] - tb;
        int sb = a.s_begin[s], ms = a.s_end[s] - sb;
        double2 *N = a.N + a.poff[pair];
        for (int e = threadIdx.x; e < mt * ms; e += blockDim.x) {
            int i = e % mt, j = e / mt;
            int64_t gi = a.t_perm[tb + i], gj = a.s_perm[sb + j];
            const double *x = a.test_pts + 3 * gi;
            const double *y = a.trial_pts + 3 * gj;
            double2 v = kernel_entry(a.K, x[0], x[1], x[2], y[0], y[1], y[2], gi, gj);
            N[e] = v;
        }
    }
}

__global__ void k_entries(KernelParams K, const double *tp, const double *sp, const int64_t *ii,
                          const int64_t *jj, int64_t n, double2 *out) {
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n;
         e += int64_t(gridDim.x) * blockDim.x) {
        const double *x = tp + 3 * ii[e];
        const double *y = sp + 3 * jj[e];
        out[e] = kernel_entry(K, x[0], x[1], x[2], y[0], y[1], y[2], ii[e], jj[e]);
    }
}

__global__ void k_to_f32(const double2 *in, float2 *out, int64_t n) {
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n;
         e += int64_t(gridDim.x) * blockDim.x) {
        double2 v = in[e];
        out[e] = make_float2(float(v.x), float(v.y));
    }
}

}  // namespace nca
