// The k-means cluster tree on the device, bit for bit the host planner's (host_plan.cpp) and the
// oracle's tree: the same rules (2-means splits seeded by the point farthest from the centroid and
// the point farthest from that one, at most 50 Lloyd iterations with ties to the first cluster,
// stable partition, breadth-first numbering) and the same arithmetic order — every sum over a
// cluster is taken in ordered chunks of 256 points (each chunk from zero in point order, the chunk
// sums added in chunk order), distances as fma(dx, dx, fma(dy, dy, dz * dz)), farthest points the
// first of equal distances. One CTA of 1024 threads splits one cluster: thread t sums chunks t,
// t + 1024, ...; a few threads add the chunk sums in order. One launch per tree level.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

#include "nca_internal.h"

namespace nca {

namespace {

constexpr int kTreeChunk = 256;
constexpr int kSplitThreads = 1024;
constexpr int kLloyd = 50;

__device__ __forceinline__ double tdist2(const double *p, const double *c) {
    const double dx = __dsub_rn(p[0], c[0]), dy = __dsub_rn(p[1], c[1]), dz = __dsub_rn(p[2], c[2]);
    return __fma_rn(dx, dx, __fma_rn(dy, dy, __dmul_rn(dz, dz)));
}

struct SplitArgs {
    const double *pts;
    int32_t *perm, *tmp;
    int8_t *side;
    const int32_t *nb, *ne;  // the level's clusters to split: [nb, ne) of perm
    const int64_t *cbase;    // first chunk slot of each cluster in the scratch below
    double *part;            // 6 per chunk: the chunk's sums (group 0, group 1), or the centroid sum
    int32_t *num;            // 2 per chunk: the chunk's group sizes; also zero counts
    int32_t *farg;           // per chunk: farthest point (first of equals)
    double *fd;              // per chunk: its squared distance
    int8_t *chg;             // per chunk: an assignment changed
    int32_t *first;          // out: size of the first group of each cluster
    int count;
};

__global__ void __launch_bounds__(kSplitThreads) k_kmeans_split(SplitArgs a) {
    const int node = blockIdx.x;
    if (node >= a.count) return;
    const int tid = threadIdx.x;
    const int b = a.nb[node], e = a.ne[node], cnt = e - b;
    const int nch = (cnt + kTreeChunk - 1) / kTreeChunk;
    double *P = a.part + 6 * a.cbase[node];
    int32_t *Nn = a.num + 2 * a.cbase[node];
    int32_t *FA = a.farg + a.cbase[node];
    double *FD = a.fd + a.cbase[node];
    int8_t *CH = a.chg + a.cbase[node];
    const int32_t *ids = a.perm + b;
    int8_t *side = a.side + b;
    __shared__ double g[3], from[3], c[2][3], spread;
    __shared__ int ia, stop, nfirst;
    // the centroid
    for (int q = tid; q < nch; q += blockDim.x) {
        const int i0 = q * kTreeChunk, i1 = min(cnt, i0 + kTreeChunk);
        double t0 = 0.0, t1 = 0.0, t2 = 0.0;
        for (int i = i0; i < i1; ++i) {
            const double *p = a.pts + 3 * int64_t(ids[i]);
            t0 = __dadd_rn(t0, p[0]);
            t1 = __dadd_rn(t1, p[1]);
            t2 = __dadd_rn(t2, p[2]);
        }
        P[6 * q] = t0;
        P[6 * q + 1] = t1;
        P[6 * q + 2] = t2;
    }
    for (int i = tid; i < cnt; i += blockDim.x) side[i] = -1;
    __syncthreads();
    if (tid < 3) {
        double s = 0.0;
        for (int q = 0; q < nch; ++q) s = __dadd_rn(s, P[6 * q + tid]);
        g[tid] = __ddiv_rn(s, double(cnt));
        from[tid] = g[tid];
    }
    __syncthreads();
    // the farthest point from `from` (twice: from the centroid, then from that point)
    for (int round = 0; round < 2; ++round) {
        for (int q = tid; q < nch; q += blockDim.x) {
            const int i0 = q * kTreeChunk, i1 = min(cnt, i0 + kTreeChunk);
            int arg = i0;
            double best = -1.0;
            for (int i = i0; i < i1; ++i) {
                const double d = tdist2(a.pts + 3 * int64_t(ids[i]), from);
                if (d > best) {
                    best = d;
                    arg = i;
                }
            }
            FA[q] = arg;
            FD[q] = best;
        }
        __syncthreads();
        if (tid == 0) {
            int arg = 0;
            double best = -1.0;
            for (int q = 0; q < nch; ++q)
                if (FD[q] > best) {
                    best = FD[q];
                    arg = FA[q];
                }
            if (round == 0) {
                ia = arg;
                for (int d = 0; d < 3; ++d) from[d] = a.pts[3 * int64_t(ids[arg]) + d];
            } else {
                spread = best;
                stop = !(best > 0.0);
                if (best > 0.0)
                    for (int d = 0; d < 3; ++d) {
                        c[0][d] = a.pts[3 * int64_t(ids[ia]) + d];
                        c[1][d] = a.pts[3 * int64_t(ids[arg]) + d];
                    }
            }
        }
        __syncthreads();
    }
    // Lloyd iterations: assignment and the groups' chunk sums, then the ordered combination
    for (int it = 0; it < kLloyd; ++it) {
        if (stop) break;
        for (int q = tid; q < nch; q += blockDim.x) {
            const int i0 = q * kTreeChunk, i1 = min(cnt, i0 + kTreeChunk);
            bool changed = false;
            double t[2][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
            int m0 = 0, m1 = 0;
            for (int i = i0; i < i1; ++i) {
                const double *p = a.pts + 3 * int64_t(ids[i]);
                const int8_t sd = tdist2(p, c[1]) < tdist2(p, c[0]) ? 1 : 0;
                if (sd != side[i]) {
                    side[i] = sd;
                    changed = true;
                }
                if (sd) {
                    t[1][0] = __dadd_rn(t[1][0], p[0]);
                    t[1][1] = __dadd_rn(t[1][1], p[1]);
                    t[1][2] = __dadd_rn(t[1][2], p[2]);
                    ++m1;
                } else {
                    t[0][0] = __dadd_rn(t[0][0], p[0]);
                    t[0][1] = __dadd_rn(t[0][1], p[1]);
                    t[0][2] = __dadd_rn(t[0][2], p[2]);
                    ++m0;
                }
            }
            CH[q] = changed;
            for (int k = 0; k < 2; ++k)
                for (int d = 0; d < 3; ++d) P[6 * q + 3 * k + d] = t[k][d];
            Nn[2 * q] = m0;
            Nn[2 * q + 1] = m1;
        }
        __syncthreads();
        // threads 0..5 add the six sums in chunk order; 6, 7 the counts; 8 the changes
        __shared__ double sum6[6];
        __shared__ int n2[2], anychg;
        if (tid < 6) {
            double s = 0.0;
            for (int q = 0; q < nch; ++q) s = __dadd_rn(s, P[6 * q + tid]);
            sum6[tid] = s;
        } else if (tid < 8) {
            int s = 0;
            for (int q = 0; q < nch; ++q) s += Nn[2 * q + (tid - 6)];
            n2[tid - 6] = s;
        } else if (tid == 8) {
            int s = 0;
            for (int q = 0; q < nch; ++q) s |= CH[q];
            anychg = s;
        }
        __syncthreads();
        if (tid == 0) {
            if (!anychg || n2[0] == 0 || n2[1] == 0) {
                stop = 1;
            } else {
                for (int k = 0; k < 2; ++k)
                    for (int d = 0; d < 3; ++d) c[k][d] = __ddiv_rn(sum6[3 * k + d], double(n2[k]));
            }
        }
        __syncthreads();
    }
    // the first group's size; both groups nonempty or the halves by position
    for (int q = tid; q < nch; q += blockDim.x) {
        const int i0 = q * kTreeChunk, i1 = min(cnt, i0 + kTreeChunk);
        int z = 0;
        for (int i = i0; i < i1; ++i) z += side[i] == 0;
        Nn[2 * q] = z;
    }
    __syncthreads();
    if (tid == 0) {
        int f = 0;
        if (spread > 0.0)
            for (int q = 0; q < nch; ++q) f += Nn[2 * q];
        nfirst = f;
    }
    __syncthreads();
    const bool halves = nfirst == 0 || nfirst == cnt;
    const int f = halves ? (cnt + 1) / 2 : nfirst;
    if (halves) {
        for (int i = tid; i < cnt; i += blockDim.x) side[i] = i < f ? 0 : 1;
        __syncthreads();
        for (int q = tid; q < nch; q += blockDim.x) {
            const int i0 = q * kTreeChunk, i1 = min(cnt, i0 + kTreeChunk);
            int z = 0;
            for (int i = i0; i < i1; ++i) z += side[i] == 0;
            Nn[2 * q] = z;
        }
        __syncthreads();
    }
    // stable partition: the chunks' zero counts as exclusive prefix sums, then each chunk places its
    // points
    if (tid == 0) {
        int s = 0;
        for (int q = 0; q < nch; ++q) {
            const int z = Nn[2 * q];
            Nn[2 * q + 1] = s;
            s += z;
        }
    }
    __syncthreads();
    for (int q = tid; q < nch; q += blockDim.x) {
        const int i0 = q * kTreeChunk, i1 = min(cnt, i0 + kTreeChunk);
        int p0 = Nn[2 * q + 1], p1 = f + (i0 - Nn[2 * q + 1]);
        for (int i = i0; i < i1; ++i) {
            if (side[i] == 0)
                a.tmp[b + p0++] = ids[i];
            else
                a.tmp[b + p1++] = ids[i];
        }
    }
    __syncthreads();
    for (int i = tid; i < cnt; i += blockDim.x) a.perm[b + i] = a.tmp[b + i];
    if (tid == 0) a.first[node] = f;
}

// centre (chunked ordered sums, one division) and radius (largest distance) of every node
__global__ void __launch_bounds__(256) k_node_balls(const double *pts, const int32_t *perm, const int32_t *nb,
                                                    const int32_t *ne, int nnodes, double *center, double *radius) {
    const int node = blockIdx.x;
    if (node >= nnodes) return;
    const int b = nb[node], e = ne[node], cnt = e - b;
    const int nch = (cnt + kTreeChunk - 1) / kTreeChunk;
    extern __shared__ double red[];  // 3 per chunk slot of this block's pass, then maxima
    __shared__ double cc[3];
    const int tid = threadIdx.x;
    // chunk sums, kept per chunk in shared memory in rounds of blockDim chunks
    double acc[3] = {0.0, 0.0, 0.0};  // thread 0's running ordered total
    for (int q0 = 0; q0 < nch; q0 += blockDim.x) {
        const int q = q0 + tid;
        double t0 = 0.0, t1 = 0.0, t2 = 0.0;
        if (q < nch) {
            const int i0 = q * kTreeChunk, i1 = min(cnt, i0 + kTreeChunk);
            for (int i = b + i0; i < b + i1; ++i) {
                const double *p = pts + 3 * int64_t(perm[i]);
                t0 = __dadd_rn(t0, p[0]);
                t1 = __dadd_rn(t1, p[1]);
                t2 = __dadd_rn(t2, p[2]);
            }
        }
        red[3 * tid] = t0;
        red[3 * tid + 1] = t1;
        red[3 * tid + 2] = t2;
        __syncthreads();
        if (tid < 3) {
            const int top = min(int(blockDim.x), nch - q0);
            for (int k = 0; k < top; ++k) acc[tid] = __dadd_rn(acc[tid], red[3 * k + tid]);
        }
        __syncthreads();
    }
    if (tid < 3) cc[tid] = cnt > 0 ? __ddiv_rn(acc[tid], double(cnt)) : 0.0;
    __syncthreads();
    double m = 0.0;
    for (int i = b + tid; i < e; i += blockDim.x) m = fmax(m, tdist2(pts + 3 * int64_t(perm[i]), cc));
    red[tid] = m;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (tid < s) red[tid] = fmax(red[tid], red[tid + s]);
        __syncthreads();
    }
    if (tid == 0) {
        for (int d = 0; d < 3; ++d) center[3 * int64_t(node) + d] = cc[d];
        radius[node] = sqrt(red[0]);
    }
}

__global__ void k_iota(int32_t *v, int64_t n) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        v[i] = int32_t(i);
}

void ck(cudaError_t e) {
    if (e != cudaSuccess) throw std::runtime_error(std::string("CUDA error in the device tree: ") + cudaGetErrorString(e));
}

template <typename T>
struct TBuf {
    T *p = nullptr;
    explicit TBuf(size_t n) { ck(cudaMalloc(&p, sizeof(T) * std::max<size_t>(n, 1))); }
    ~TBuf() {
        if (p) cudaFree(p);
    }
    TBuf(const TBuf &) = delete;
    TBuf &operator=(const TBuf &) = delete;
};

}  // namespace

Tree build_kmeans_tree_device(const double *pts, int64_t n, int minvalues, void *stream) {
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    Tree T;
    T.npoints = n;
    T.begin.push_back(0);
    T.end.push_back(int32_t(n));
    T.parent.push_back(-1);
    T.level.push_back(0);
    TBuf<double> dpts{size_t(3 * n)};
    TBuf<int32_t> dperm{size_t(n)}, dtmp{size_t(n)};
    TBuf<int8_t> dside{size_t(n)};
    ck(cudaMemcpyAsync(dpts.p, pts, sizeof(double) * 3 * size_t(n), cudaMemcpyHostToDevice, s));
    if (n > 0) k_iota<<<int(std::min<int64_t>((n + 255) / 256, 4096)), 256, 0, s>>>(dperm.p, n);
    ck(cudaGetLastError());
    // chunk scratch: at most n / 256 + (clusters of a level) slots per level
    const int64_t slots = n / kTreeChunk + int64_t(n / std::max(minvalues, 1)) + 2;
    TBuf<double> dpart{size_t(6 * slots)}, dfd{size_t(slots)};
    TBuf<int32_t> dnum{size_t(2 * slots)}, dfarg{size_t(slots)};
    TBuf<int8_t> dchg{size_t(slots)};
    const int64_t maxnodes = 2 * (n / std::max(minvalues, 1)) + 2;
    TBuf<int32_t> dnb{size_t(maxnodes)}, dne{size_t(maxnodes)}, dfirst{size_t(maxnodes)};
    TBuf<int64_t> dcbase{size_t(maxnodes)};
    std::vector<int32_t> cb, ce, idx, first;
    std::vector<int64_t> cbase;
    for (size_t lev0 = 0, lev1 = T.begin.size(); lev0 < lev1; lev0 = lev1, lev1 = T.begin.size()) {
        cb.clear();
        ce.clear();
        idx.clear();
        cbase.clear();
        int64_t nslot = 0;
        for (size_t node = lev0; node < lev1; ++node) {
            const int cnt = T.end[node] - T.begin[node];
            if (cnt > minvalues && cnt >= 2) {
                cb.push_back(T.begin[node]);
                ce.push_back(T.end[node]);
                idx.push_back(int32_t(node));
                cbase.push_back(nslot);
                nslot += (cnt + kTreeChunk - 1) / kTreeChunk;
            }
        }
        first.assign(idx.size(), -1);
        if (!idx.empty()) {
            if (nslot > slots || int64_t(idx.size()) > maxnodes) throw std::runtime_error("device tree scratch too small");
            ck(cudaMemcpyAsync(dnb.p, cb.data(), sizeof(int32_t) * cb.size(), cudaMemcpyHostToDevice, s));
            ck(cudaMemcpyAsync(dne.p, ce.data(), sizeof(int32_t) * ce.size(), cudaMemcpyHostToDevice, s));
            ck(cudaMemcpyAsync(dcbase.p, cbase.data(), sizeof(int64_t) * cbase.size(), cudaMemcpyHostToDevice, s));
            SplitArgs a{dpts.p, dperm.p, dtmp.p, dside.p, dnb.p, dne.p, dcbase.p, dpart.p, dnum.p, dfarg.p, dfd.p,
                        dchg.p, dfirst.p, int(idx.size())};
            k_kmeans_split<<<int(idx.size()), kSplitThreads, 0, s>>>(a);
            ck(cudaGetLastError());
            ck(cudaMemcpyAsync(first.data(), dfirst.p, sizeof(int32_t) * first.size(), cudaMemcpyDeviceToHost, s));
            ck(cudaStreamSynchronize(s));
        }
        size_t k = 0;
        for (size_t node = lev0; node < lev1; ++node) {
            const int b = T.begin[node], e = T.end[node];
            if (k < idx.size() && idx[k] == int32_t(node)) {
                const int f = first[k++];
                T.firstchild.push_back(int32_t(T.begin.size()));
                T.nchildren.push_back(2);
                const int bounds[3] = {b, b + f, e};
                for (int c = 0; c < 2; ++c) {
                    T.begin.push_back(bounds[c]);
                    T.end.push_back(bounds[c + 1]);
                    T.parent.push_back(int32_t(node));
                    T.level.push_back(T.level[node] + 1);
                }
            } else {
                T.firstchild.push_back(-1);
                T.nchildren.push_back(0);
            }
        }
    }
    T.nnodes = int(T.begin.size());
    T.center.resize(3 * size_t(T.nnodes));
    T.radius.resize(T.nnodes);
    {
        TBuf<int32_t> ab{size_t(T.nnodes)}, ae{size_t(T.nnodes)};
        TBuf<double> cen{3 * size_t(T.nnodes)}, rad{size_t(T.nnodes)};
        ck(cudaMemcpyAsync(ab.p, T.begin.data(), sizeof(int32_t) * T.nnodes, cudaMemcpyHostToDevice, s));
        ck(cudaMemcpyAsync(ae.p, T.end.data(), sizeof(int32_t) * T.nnodes, cudaMemcpyHostToDevice, s));
        k_node_balls<<<T.nnodes, 256, sizeof(double) * 3 * 256, s>>>(dpts.p, dperm.p, ab.p, ae.p, T.nnodes, cen.p, rad.p);
        ck(cudaGetLastError());
        T.perm.resize(size_t(n));
        ck(cudaMemcpyAsync(T.perm.data(), dperm.p, sizeof(int32_t) * size_t(n), cudaMemcpyDeviceToHost, s));
        ck(cudaMemcpyAsync(T.center.data(), cen.p, sizeof(double) * 3 * T.nnodes, cudaMemcpyDeviceToHost, s));
        ck(cudaMemcpyAsync(T.radius.data(), rad.p, sizeof(double) * T.nnodes, cudaMemcpyDeviceToHost, s));
        ck(cudaStreamSynchronize(s));
    }
    T.nlevels = T.level.back() + 1;
    T.levelptr.assign(T.nlevels + 1, T.nnodes);
    for (int node = T.nnodes - 1; node >= 0; --node) T.levelptr[T.level[node]] = node;
    T.iperm.resize(size_t(n));
    for (int64_t i = 0; i < n; ++i) T.iperm[T.perm[i]] = int32_t(i);
    return T;
}

}  // namespace nca
