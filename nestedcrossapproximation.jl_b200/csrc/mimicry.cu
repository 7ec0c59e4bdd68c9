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

__global__ void __launch_bounds__(kWarps * 32, 4) k_mimicry(MimicryArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m = a.maxrank;
    double *base = reinterpret_cast<double *>(smem) + size_t(warp) * 3 * m;
    Chosen ch{base, base + m, base + 2 * m,
              reinterpret_cast<int32_t *>(reinterpret_cast<double *>(smem) + size_t(kWarps) * 3 * m) + warp * m};
    for (;;) {
        // items differ widely in cost: each warp takes the next untaken one
        int item = 0;
        if (lane == 0) item = atomicAdd(a.cursor, 1);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= a.nitems) break;
        const int64_t f0 = a.ffptr[item], f1 = a.ffptr[item + 1];
        const int nroots = int(f1 - f0);
        const int32_t *roots = a.ffnodes + f0;
        const int own = a.item_node ? a.item_node[item] : item;
        const int nref = a.own_size[own];
        const int limit = nref < m ? nref : m;
        int n = 0;
        for (int i = 0; i < nroots && limit - n > 0; ++i) {
            const int f = roots[i];
            const int sz = a.end[f] - a.begin[f];
            n += limit - n < sz ? limit - n : sz;
        }
        const double c[3] = {a.centroid[3 * size_t(own)], a.centroid[3 * size_t(own) + 1],
                             a.centroid[3 * size_t(own) + 2]};
        int32_t *out = a.piv + size_t(item) * m;
        int nch = 0;
        // Items with at most 32 * kRootSlots far nodes: lane l keeps, for its roots l + 32 r, the
        // running minimum of the squared distances to the chosen pivots and the count of chosen
        // positions inside the root (updated once per pick; a minimum is exact in any order).
        const bool running = nroots <= 32 * kRootSlots;
        double rdm[kRootSlots];
        int rtk[kRootSlots];
#pragma unroll
        for (int r = 0; r < kRootSlots; ++r) {
            rdm[r] = INFINITY;
            rtk[r] = 0;
        }
        for (int p = 0; p < n; ++p) {
            // root: the far node of the best centre score among those with untaken points
            double best = -1.0;
            int bi = 0x7fffffff;
            if (running) {
#pragma unroll
                for (int r = 0; r < kRootSlots; ++r) {
                    const int i = lane + 32 * r;
                    if (i < nroots) {
                        const int f = roots[i];
                        if (a.end[f] - a.begin[f] - rtk[r] > 0) {
                            const double sc = score(a.center[3 * size_t(f)], a.center[3 * size_t(f) + 1],
                                                    a.center[3 * size_t(f) + 2], c, nch == 0 ? 1.0 : rdm[r]);
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
            if (bi == 0x7fffffff) {  // no far point left (cannot happen for disjoint far nodes)
                if (lane == 0) atomicCAS(a.error, 0, 1);
                break;
            }
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
                if (node < 0) break;
            }
            if (node < 0) {  // no child with untaken points (cannot happen: the node had some)
                if (lane == 0) atomicCAS(a.error, 0, 1);
                break;
            }
            // leaf: the untaken point of the best score; the taken positions of each 32-point
            // window come from one OR-reduction per 32 chosen pivots
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
                const int id = a.perm[pos];
                const double yx = a.pts[3 * size_t(id)], yy = a.pts[3 * size_t(id) + 1], yz = a.pts[3 * size_t(id) + 2];
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
            if (bp == 0x7fffffff) {  // every point of the leaf taken (cannot happen, as above)
                if (lane == 0) atomicCAS(a.error, 0, 1);
                break;
            }
            if (lane == 0) {
                const int id = a.perm[bp];
                ch.x[nch] = a.pts[3 * size_t(id)];
                ch.y[nch] = a.pts[3 * size_t(id) + 1];
                ch.z[nch] = a.pts[3 * size_t(id) + 2];
                ch.pos[nch] = bp;
                out[p] = id;
            }
            __syncwarp();
            if (running) {
                const double px = ch.x[nch], py = ch.y[nch], pz = ch.z[nch];
#pragma unroll
                for (int r = 0; r < kRootSlots; ++r) {
                    const int i = lane + 32 * r;
                    if (i < nroots) {
                        const int f = roots[i];
                        rtk[r] += bp >= a.begin[f] && bp < a.end[f];
                        const double d = dist2(a.center[3 * size_t(f)], a.center[3 * size_t(f) + 1],
                                               a.center[3 * size_t(f) + 2], px, py, pz);
                        rdm[r] = d < rdm[r] ? d : rdm[r];
                    }
                }
            }
            ++nch;
        }
        if (lane == 0) a.count[item] = nch;
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
