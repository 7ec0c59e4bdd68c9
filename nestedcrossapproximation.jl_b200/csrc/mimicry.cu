// Phase 1 of the batched build on the device: tree-mimicry far pivots of many clusters (or
// directional items) at once, one warp per item.
//
// The selection is the host planner's (host_plan.cpp, class Mimicry), which restates
// _selectfarpivots (src/compressors/batchedbottomup.jl:54-72) with the tree-mimicry rule this
// project fixes:
//   n = min(maxrank, |t|) capped by the far points available (the far nodes in list order);
//   pick p: among the item's far nodes (roots) with untaken points, the one whose centre
//   maximises score(y) = dmin2(y) / max(|y - c|^2, 1e-300) (c: the cluster centroid; dmin2(y):
//   1 before the first pick, else the smallest squared distance from y to the pivots chosen so
//   far); descend by the same score through the children with untaken points to a leaf; take
//   the leaf's untaken point of the largest score. Ties go to the first candidate (root list
//   order, child order, point position).
// The host keeps running minima between picks; here the far nodes' minima (and their counts of
// taken points) are kept running per lane for items with at most 128 far nodes, and every other
// minimum is taken afresh over the chosen pivots. A minimum does not depend on the order it is
// taken in and every squared distance uses the host's operation order (fma(dx, dx, fma(dy, dy,
// dz * dz)); compiled with --fmad=false), so the pivots agree with the host's bit for bit.
#include <cuda_runtime.h>

#include <cstdint>

#include "build_kernels.cuh"

namespace nca {

namespace {

constexpr int kWarps = 8;  // warps per CTA, each on one item at a time
constexpr int kRootSlots = 4;  // roots a lane keeps running minima for (items with <= 128 far nodes)

__device__ __forceinline__ double dist2(double ax, double ay, double az, double bx, double by, double bz) {
    const double dx = ax - bx, dy = ay - by, dz = az - bz;
    return fma(dx, dx, fma(dy, dy, __dmul_rn(dz, dz)));
}

struct Chosen {
    double *x, *y, *z;
    int32_t *pos;
};

// score of y for the centroid c and the squared distance dmin2 to the chosen pivots
__device__ __forceinline__ double score(double yx, double yy, double yz, const double *c, double dmin2) {
    double d2 = dist2(yx, yy, yz, c[0], c[1], c[2]);
    if (d2 < 1e-300) d2 = 1e-300;
    return __ddiv_rn(dmin2, d2);
}

// dmin2 of y over the nch chosen pivots, every lane taking a share, the same value on all lanes
__device__ double warp_dmin(const Chosen &ch, int nch, double yx, double yy, double yz, int lane) {
    if (nch == 0) return 1.0;
    double m = INFINITY;
    for (int q = lane; q < nch; q += 32) {
        const double d = dist2(yx, yy, yz, ch.x[q], ch.y[q], ch.z[q]);
        m = d < m ? d : m;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const double o = __shfl_xor_sync(0xffffffffu, m, off);
        m = o < m ? o : m;
    }
    return m;
}

// chosen positions inside [lo, hi), the same value on all lanes
__device__ int warp_taken(const Chosen &ch, int nch, int lo, int hi, int lane) {
    int n = 0;
    for (int q0 = 0; q0 < nch; q0 += 32) {
        const int q = q0 + lane;
        const bool in = q < nch && ch.pos[q] >= lo && ch.pos[q] < hi;
        n += __popc(__ballot_sync(0xffffffffu, in));
    }
    return n;
}

// warp argmax: largest score, ties to the smallest index
__device__ __forceinline__ void warp_argmax(double &sc, int &idx) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const double os = __shfl_xor_sync(0xffffffffu, sc, off);
        const int oi = __shfl_xor_sync(0xffffffffu, idx, off);
        if (os > sc || (os == sc && oi < idx)) {
            sc = os;
            idx = oi;
        }
    }
}

// One warp's tree-mimicry state for one item: its far nodes (roots), the cluster centroid, the
// pivots chosen so far (shared memory) and, for items with at most 32 * kRootSlots far nodes,
// lane-held running minima and taken counts of the roots.
struct MimWarp {
    const int32_t *roots;
    int nroots;
    double c[3];
    bool running;
    double rdm[kRootSlots];
    int rtk[kRootSlots];
    Chosen ch;
    int nch;
};

__device__ __forceinline__ void mim_start(const MimicryArgs &a, MimWarp &w, int item, int own) {
    const int64_t f0 = a.ffptr[item], f1 = a.ffptr[item + 1];
    w.nroots = int(f1 - f0);
    w.roots = a.ffnodes + f0;
    w.c[0] = a.centroid[3 * size_t(own)];
    w.c[1] = a.centroid[3 * size_t(own) + 1];
    w.c[2] = a.centroid[3 * size_t(own) + 2];
    w.running = w.nroots <= 32 * kRootSlots;
#pragma unroll
    for (int r = 0; r < kRootSlots; ++r) {
        w.rdm[r] = INFINITY;
        w.rtk[r] = 0;
    }
    w.nch = 0;
}

// The next pivot: returns its position in the far tree's permutation (the same on all lanes) and
// stores its point id in *id, or returns -1 when no far point is left (cannot happen for disjoint
// far nodes with points to spare). Lane 0 appends the pivot to the chosen list.
__device__ __forceinline__ int mim_pick(const MimicryArgs &a, MimWarp &w, int lane, int32_t *id) {
    const Chosen &ch = w.ch;
    const int nch = w.nch;
    const int32_t *roots = w.roots;
    const int nroots = w.nroots;
    const double *c = w.c;
    // root: the far node of the best centre score among those with untaken points
    double best = -1.0;
    int bi = 0x7fffffff;
    if (w.running) {
#pragma unroll
        for (int r = 0; r < kRootSlots; ++r) {
            const int i = lane + 32 * r;
            if (i < nroots) {
                const int f = roots[i];
                if (a.end[f] - a.begin[f] - w.rtk[r] > 0) {
                    const double sc = score(a.center[3 * size_t(f)], a.center[3 * size_t(f) + 1],
                                            a.center[3 * size_t(f) + 2], c, nch == 0 ? 1.0 : w.rdm[r]);
                    if (sc > best) {
                        best = sc;
                        bi = i;
                    }
                }
            }
        }
    } else {
        for (int i = lane; i < nroots; i += 32) {
            const int f = roots[i];
            const int lo = a.begin[f], hi = a.end[f];
            int taken = 0;
            double dm = nch == 0 ? 1.0 : INFINITY;
            const double yx = a.center[3 * size_t(f)], yy = a.center[3 * size_t(f) + 1],
                         yz = a.center[3 * size_t(f) + 2];
            for (int q = 0; q < nch; ++q) {
                taken += ch.pos[q] >= lo && ch.pos[q] < hi;
                const double d = dist2(yx, yy, yz, ch.x[q], ch.y[q], ch.z[q]);
                dm = d < dm ? d : dm;
            }
            if (hi - lo - taken <= 0) continue;
            const double sc = score(yx, yy, yz, c, dm);
            if (sc > best) {
                best = sc;
                bi = i;
            }
        }
    }
    warp_argmax(best, bi);
    if (bi == 0x7fffffff) return -1;
    int node = roots[bi];
    // descent through the children with untaken points, best centre score first
    while (a.nchildren[node] > 0) {
        int pick = -1;
        double pbest = -1.0;
        for (int k = 0; k < a.nchildren[node]; ++k) {
            const int cnode = a.firstchild[node] + k;
            const int lo = a.begin[cnode], hi = a.end[cnode];
            if (hi - lo - warp_taken(ch, nch, lo, hi, lane) <= 0) continue;
            const double yx = a.center[3 * size_t(cnode)], yy = a.center[3 * size_t(cnode) + 1],
                         yz = a.center[3 * size_t(cnode) + 2];
            const double sc = score(yx, yy, yz, c, warp_dmin(ch, nch, yx, yy, yz, lane));
            if (sc > pbest) {
                pbest = sc;
                pick = cnode;
            }
        }
        node = pick;
        if (node < 0) return -1;
    }
    // leaf: the untaken point of the best score; the taken positions of each 32-point window come
    // from one OR-reduction per 32 chosen pivots
    double pb = -1.0;
    int bp = 0x7fffffff;
    const int lend = a.end[node];
    for (int base = a.begin[node]; base < lend; base += 32) {
        unsigned tmask = 0;
        for (int q0 = 0; q0 < nch; q0 += 32) {
            const int q = q0 + lane;
            const int off = q < nch ? ch.pos[q] - base : -1;
            tmask |= __reduce_or_sync(0xffffffffu, off >= 0 && off < 32 ? 1u << off : 0u);
        }
        const int pos = base + lane;
        if (pos >= lend || ((tmask >> lane) & 1u)) continue;
        const int pid = a.perm[pos];
        const double yx = a.pts[3 * size_t(pid)], yy = a.pts[3 * size_t(pid) + 1], yz = a.pts[3 * size_t(pid) + 2];
        double dm = nch == 0 ? 1.0 : INFINITY;
        for (int q = 0; q < nch; ++q) {
            const double d = dist2(yx, yy, yz, ch.x[q], ch.y[q], ch.z[q]);
            dm = d < dm ? d : dm;
        }
        const double sc = score(yx, yy, yz, c, dm);
        if (sc > pb) {
            pb = sc;
            bp = pos;
        }
    }
    warp_argmax(pb, bp);
    if (bp == 0x7fffffff) return -1;
    const int pid = a.perm[bp];
    if (lane == 0) {
        ch.x[nch] = a.pts[3 * size_t(pid)];
        ch.y[nch] = a.pts[3 * size_t(pid) + 1];
        ch.z[nch] = a.pts[3 * size_t(pid) + 2];
        ch.pos[nch] = bp;
    }
    __syncwarp();
    if (w.running) {
        const double px = ch.x[nch], py = ch.y[nch], pz = ch.z[nch];
#pragma unroll
        for (int r = 0; r < kRootSlots; ++r) {
            const int i = lane + 32 * r;
            if (i < nroots) {
                const int f = roots[i];
                w.rtk[r] += bp >= a.begin[f] && bp < a.end[f];
                const double d = dist2(a.center[3 * size_t(f)], a.center[3 * size_t(f) + 1],
                                       a.center[3 * size_t(f) + 2], px, py, pz);
                w.rdm[r] = d < w.rdm[r] ? d : w.rdm[r];
            }
        }
    }
    w.nch = nch + 1;
    *id = pid;
    return bp;
}

__global__ void __launch_bounds__(kWarps * 32, 4) k_mimicry(MimicryArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m = a.maxrank;
    double *base = reinterpret_cast<double *>(smem) + size_t(warp) * 3 * m;
    MimWarp w;
    w.ch = Chosen{base, base + m, base + 2 * m,
                  reinterpret_cast<int32_t *>(reinterpret_cast<double *>(smem) + size_t(kWarps) * 3 * m) + warp * m};
    for (;;) {
        // items differ widely in cost: each warp takes the next untaken one
        int item = 0;
        if (lane == 0) item = atomicAdd(a.cursor, 1);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= a.nitems) break;
        const int own = a.item_node ? a.item_node[item] : item;
        mim_start(a, w, item, own);
        const int nref = a.own_size[own];
        const int limit = nref < m ? nref : m;
        int n = 0;
        for (int i = 0; i < w.nroots && limit - n > 0; ++i) {
            const int f = w.roots[i];
            const int sz = a.end[f] - a.begin[f];
            n += limit - n < sz ? limit - n : sz;
        }
        int32_t *out = a.piv + size_t(item) * m;
        for (int p = 0; p < n; ++p) {
            int32_t id = 0;
            if (mim_pick(a, w, lane, &id) < 0) {
                if (lane == 0) atomicCAS(a.error, 0, 1);
                break;
            }
            if (lane == 0) out[p] = id;
        }
        if (lane == 0) a.count[item] = w.nch;
        __syncwarp();
    }
}

constexpr int kIacaWarps = 8;  // warps per CTA of the IACA kernel, each on one item at a time
constexpr unsigned kFull = 0xffffffffu;

// sum over the warp in the xor butterfly order (offsets 16, 8, 4, 2, 1): every lane gets the value
// of the oracle's restatement
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v = __dadd_rn(v, __shfl_xor_sync(kFull, v, off));
    return v;
}

// value of slot q (a warp-uniform index) of a lane's register array
template <int RPL, typename T>
__device__ __forceinline__ T slot(const T (&v)[RPL], int q) {
    T out = v[0];
#pragma unroll
    for (int k = 1; k < RPL; ++k)
        if (q == k) out = v[k];
    return out;
}

// K(own point, far point) in the side's orientation (side 0: own points are test points). Kept
// out of line: the k_iaca loop calls it once per held row, and one copy of the entry code keeps
// the kernel's instruction footprint small (an inlined copy per row and orientation made
// instruction fetch the kernel's top stall).
__device__ __noinline__ double2 oriented_entry(KernelParams K, bool own_is_test, double rx, double ry, double rz,
                                              int32_t rid, double qx, double qy, double qz, int32_t qid) {
    if (own_is_test) return kernel_entry(K, rx, ry, rz, qx, qy, qz, rid, qid);
    return kernel_entry(K, qx, qy, qz, rx, ry, rz, qid, rid);
}

// IACA of every item of one level, one warp per item: tree
// mimicry picks the geometric columns one at a time, the column is evaluated on the item's rows
// (lane l holds rows l + 32 q), eliminated against the accepted crosses, tested by the
// extrapolated Frobenius stop (||r||^2 k <= tol^2 ||sampled block||_F^2; the build stops, rejecting
// the column, when two consecutive columns pass or r is exactly zero) and, if kept, pivoted at its
// largest entry (lowest row on ties); the cross matrix is
// unit lower triangular in the eliminated columns, so X = U L^{-1} is solved in place in the
// item's X slot. Status: [1, item, npivots, rank] singular cross matrix, [2, item, rows, limit]
// more rows than the warp holds, [3, item, 0, 0] tree mimicry out of far points.
// The CTA's warps take their items in rounds (one round per CTA as launched: CTAs retire as their
// items end, so the kernels of other streams find room on the SMs between them) and run the pivot
// steps in lockstep (one CTA-wide barrier per step), so that the warps of an SM execute the same
// part of the item loop at a time:
// instruction fetch bounded the free-running form (8 lockstep warps per CTA took 11 % less time
// than 4 free-running ones; refilling a warp as soon as its item ends was slower still, as the
// refill holds up the step barrier). Warps whose item is done, or that hold none, wait at the
// barriers; the item's closing work (singular check, X = U L^{-1}) runs between the rounds' steps.
template <int RPL>
__global__ void __launch_bounds__(kIacaWarps * 32) k_iaca(IacaArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int mr = a.maxrank;
    double *dbase = reinterpret_cast<double *>(smem) + size_t(warp) * 4 * mr;
    int32_t *ibase = reinterpret_cast<int32_t *>(reinterpret_cast<double *>(smem) + size_t(kIacaWarps) * 4 * mr) +
                     size_t(warp) * 2 * mr;
    MimWarp w;
    w.ch = Chosen{dbase, dbase + mr, dbase + 2 * mr, ibase};
    double *pivabs = dbase + 3 * mr;  // |pivot|^2 of every accepted cross
    int32_t *rp = ibase + mr;         // local pivot row of every accepted cross
    const MimicryArgs &F = a.mim;
    const bool items = F.item_node != nullptr;
    for (int64_t round = 0;; ++round) {
        const int64_t at = (round * gridDim.x + blockIdx.x) * kIacaWarps + warp;
        const int idx = int(at < a.nitems ? at : a.nitems);
        const bool valid = at < a.nitems;
        if (__syncthreads_and(!valid)) break;  // every warp of the CTA is out of items
        const int item = valid ? a.items[idx] : 0;
        const int cl = items ? F.item_node[item] : item;
        const bool basis = items ? a.item_basis[item] != 0 : a.nchildren[cl] == 0;
        const int nchd = basis ? 0 : items ? a.item_chptr[item + 1] - a.item_chptr[item] : a.nchildren[cl];
        auto child = [&](int c) { return items ? a.item_chidx[a.item_chptr[item] + c] : a.firstchild[cl] + c; };
        int m = 0;
        if (!valid) {
            m = 0;
        } else if (basis) {
            m = a.end[cl] - a.begin[cl];
        } else {
            for (int c = 0; c < nchd; ++c) m += a.rank[child(c)];
        }
        const int limit = mr < m ? mr : m;
        bool ok = valid;  // the warp holds an item it works on
        if (valid && m > 32 * RPL) {
            if (lane == 0 && atomicCAS(a.status, 0, 2) == 0) {
                a.status[1] = item;
                a.status[2] = m;
                a.status[3] = 32 * RPL;
            }
            ok = false;
        }
        if (!ok) m = 0;  // no rows: the steps below do nothing for this warp
        // the lane's rows: the cluster's points or the children's pivots, in order
        int32_t rid[RPL];
        double rx[RPL], ry[RPL], rz[RPL];
#pragma unroll
        for (int q = 0; q < RPL; ++q) {
            const int i = lane + 32 * q;
            rid[q] = -1;
            if (i < m) {
                if (basis) {
                    rid[q] = a.perm[a.begin[cl] + i];
                } else {
                    int off = 0;
                    for (int c = 0; c < nchd; ++c) {
                        const int ch = child(c), kc = a.rank[ch];
                        if (i < off + kc) {
                            rid[q] = a.piv[int64_t(ch) * mr + (i - off)];
                            break;
                        }
                        off += kc;
                    }
                }
                rx[q] = a.own_pts[3 * int64_t(rid[q])];
                ry[q] = a.own_pts[3 * int64_t(rid[q]) + 1];
                rz[q] = a.own_pts[3 * int64_t(rid[q]) + 2];
            } else {
                rx[q] = ry[q] = rz[q] = 0.0;
            }
        }
        // rank limit: min(maxrank, rows, far points)
        int n = 0;
        double2 *U = a.X;
        if (ok) {
            mim_start(F, w, F.ff_by_position ? idx : item, cl);
            for (int i = 0; i < w.nroots && limit - n > 0; ++i) {
                const int f = w.roots[i];
                const int sz = F.end[f] - F.begin[f];
                n += limit - n < sz ? limit - n : sz;
            }
            U = a.X + a.xoff[a.xoff_by_position ? idx : item];
        }
        const double tol2 = __dmul_rn(a.tol, a.tol);
        double S = 0.0;
        int k = 0;
        bool lost = false, passed = false, active = ok;
        for (;;) {
            const bool go = active && k < n;
            if (!__syncthreads_or(go)) break;  // the CTA's items of this round are done
            if (!go) continue;
            int32_t jid = 0;
            if (mim_pick(F, w, lane, &jid) < 0) {
                lost = true;
                active = false;
                continue;
            }
            const double qx = w.ch.x[k], qy = w.ch.y[k], qz = w.ch.z[k];
            double2 r[RPL];
            double cs = 0.0;
#pragma unroll
            for (int q = 0; q < RPL; ++q) {
                r[q] = make_double2(0.0, 0.0);
                if (rid[q] >= 0) {
                    r[q] = oriented_entry(a.K, a.side == 0, rx[q], ry[q], rz[q], rid[q], qx, qy, qz, jid);
                    cs = __dadd_rn(cs, cabs2_rn(r[q]));
                }
            }
            S = __dadd_rn(S, warp_sum(cs));
            // elimination against the accepted crosses, in order
            for (int l = 0; l < k; ++l) {
                const int il = rp[l];
                const double2 v = slot<RPL>(r, il >> 5);
                const double2 p = make_double2(__shfl_sync(kFull, v.x, il & 31), __shfl_sync(kFull, v.y, il & 31));
                const double2 *ul = U + int64_t(l) * m;
#pragma unroll
                for (int q = 0; q < RPL; ++q)
                    if (rid[q] >= 0) {
                        const double2 t = cmul_rn(ul[lane + 32 * q], p);
                        r[q] = make_double2(__dsub_rn(r[q].x, t.x), __dsub_rn(r[q].y, t.y));
                    }
            }
            double e2 = 0.0, best = -1.0;
            int bi = 0x7fffffff;
#pragma unroll
            for (int q = 0; q < RPL; ++q)
                if (rid[q] >= 0) {
                    const double s2 = cabs2_rn(r[q]);
                    e2 = __dadd_rn(e2, s2);
                    if (s2 > best) {
                        best = s2;
                        bi = lane + 32 * q;
                    }
                }
            e2 = warp_sum(e2);
            // extrapolated Frobenius stop, confirmed on two consecutive columns
            const bool pass = !(__dmul_rn(e2, double(k + 1)) > __dmul_rn(tol2, S));
            if (pass && (passed || e2 == 0.0)) {
                active = false;
                continue;
            }
            passed = pass;
            warp_argmax(best, bi);
            if (bi >= m) {  // no finite residual entry (non-finite kernel values): stop here
                active = false;
                continue;
            }
            const double2 v = slot<RPL>(r, bi >> 5);
            const double px = __shfl_sync(kFull, v.x, bi & 31), py = __shfl_sync(kFull, v.y, bi & 31);
            const int32_t pid = __shfl_sync(kFull, slot<RPL>(rid, bi >> 5), bi & 31);
            const double d = cabs2_rn(make_double2(px, py));
            const double2 wv = make_double2(__ddiv_rn(px, d), -__ddiv_rn(py, d));
            double2 *uk = U + int64_t(k) * m;
#pragma unroll
            for (int q = 0; q < RPL; ++q)
                if (rid[q] >= 0) {
                    const int i = lane + 32 * q;
                    uk[i] = i == bi ? make_double2(1.0, 0.0) : cmul_rn(r[q], wv);
                }
            if (lane == 0) {
                rp[k] = bi;
                pivabs[k] = d;
                a.piv[int64_t(item) * mr + k] = pid;
                if (a.cpiv) a.cpiv[int64_t(item) * mr + k] = jid;
            }
            __syncwarp();
            ++k;
        }
        if (lost) {
            if (lane == 0 && atomicCAS(a.status, 0, 3) == 0) a.status[1] = item;
            continue;
        }
        const int rank = k;
        if (rank > 0) {
            // singular check of _crossfactorization on the pivots
            double d2max = 0.0, d2min = INFINITY;
            for (int l = 0; l < rank; ++l) {
                const double d = pivabs[l];
                d2max = d > d2max ? d : d2max;
                d2min = d < d2min ? d : d2min;
            }
            const double eps = 0x1p-52;
            const double thr = (10.0 * eps) * (10.0 * eps) * d2max;
            if (!(d2min > thr)) {
                if (lane == 0 && atomicCAS(a.status, 0, 1) == 0) {
                    int nr = 0;
                    for (int l = 0; l < rank; ++l) nr += pivabs[l] > thr;
                    a.status[1] = item;
                    a.status[2] = limit;
                    a.status[3] = nr;
                }
                continue;
            }
        }
        // X L = U with L[l][kk] = U[i_l, kk]: columns from the last, each row summed over l ascending
        for (int kk = rank - 1; kk >= 0; --kk) {
            double2 val[RPL];
#pragma unroll
            for (int q = 0; q < RPL; ++q) {
                val[q] = make_double2(0.0, 0.0);
                if (rid[q] >= 0) {
                    const int i = lane + 32 * q;
                    double2 acc = U[i + int64_t(kk) * m];
                    for (int l = kk + 1; l < rank; ++l) {
                        const double2 t = cmul_rn(U[i + int64_t(l) * m], U[rp[l] + int64_t(kk) * m]);
                        acc = make_double2(__dsub_rn(acc.x, t.x), __dsub_rn(acc.y, t.y));
                    }
                    val[q] = acc;
                }
            }
            __syncwarp();
#pragma unroll
            for (int q = 0; q < RPL; ++q)
                if (rid[q] >= 0) U[lane + 32 * q + int64_t(kk) * m] = val[q];
            __syncwarp();
        }
        if (lane == 0 && ok) {
            a.rank[item] = rank;
            a.nrows[item] = m;
            if (a.rank_pos) {
                a.rank_pos[idx] = rank;
                a.rank_pos[a.nitems + idx] = m;
            }
        }
        __syncwarp();
    }
}

// fpidx[fpptr[i] + r] = piv[i * maxrank + r] for r < count[i]: the padded pivot slots of every
// item packed into one CSR list
__global__ void k_compact_pivots(const int32_t *piv, int maxrank, const int32_t *count, const int32_t *fpptr,
                                 int64_t nslots, int32_t *fpidx) {
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < nslots; e += int64_t(gridDim.x) * blockDim.x) {
        const int64_t i = e / maxrank;
        const int r = int(e - i * maxrank);
        if (r < count[i]) fpidx[fpptr[i] + r] = piv[e];
    }
}

}  // namespace

void launch_compact_pivots(const int32_t *piv, int maxrank, const int32_t *count, const int32_t *fpptr,
                           int nitems, int32_t *fpidx, cudaStream_t s) {
    const int64_t nslots = int64_t(nitems) * maxrank;
    if (nslots <= 0) return;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t need = (nslots + 255) / 256;
    k_compact_pivots<<<int(need < int64_t(sms) * 16 ? need : int64_t(sms) * 16), 256, 0, s>>>(piv, maxrank, count, fpptr,
                                                                                              nslots, fpidx);
}

size_t iaca_smem_bytes(int maxrank) {
    return size_t(kIacaWarps) * maxrank * (4 * sizeof(double) + 2 * sizeof(int32_t));
}

int iaca_max_rows() { return 256; }

void launch_iaca(const IacaArgs &a, int mcap, cudaStream_t s) {
    if (a.nitems <= 0) return;
    const size_t sm = iaca_smem_bytes(a.maxrank);
    const int grid = (a.nitems + kIacaWarps - 1) / kIacaWarps;  // one round of items per CTA
    auto go = [&](auto kern) {
        if (sm > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm));
        kern<<<grid, kIacaWarps * 32, sm, s>>>(a);
    };
    if (mcap <= 32) {
        go(k_iaca<1>);
    } else if (mcap <= 64) {
        go(k_iaca<2>);
    } else if (mcap <= 128) {
        go(k_iaca<4>);
    } else {
        go(k_iaca<8>);
    }
}

size_t mimicry_smem_bytes(int maxrank) { return size_t(kWarps) * maxrank * (3 * sizeof(double) + sizeof(int32_t)); }

void launch_mimicry(const MimicryArgs &a, cudaStream_t s) {
    if (a.nitems <= 0) return;
    const size_t sm = mimicry_smem_bytes(a.maxrank);
    cudaFuncSetAttribute(k_mimicry, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm));
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int need = (a.nitems + kWarps - 1) / kWarps;
    const int grid = need < sms * 8 ? need : sms * 8;
    k_mimicry<<<grid, kWarps * 32, sm, s>>>(a);
}

}  // namespace nca
