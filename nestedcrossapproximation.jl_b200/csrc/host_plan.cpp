// Host planner of the batched build: cluster tree, admissible partition, phase-1 far pivots.
//
// These steps run on the host in the reference too (they decide index sets, not entries):
//   - the k-means tree (H2Trees.KMeansTree with numberofclusters = 2; an input of
//     PetrovGalerkinNCA, src/nca/petrovgalerkinnca.jl:138-142),
//   - interactions(tree, isnear(eta)) with the ball admissibility
//     2 max(r_t, r_s) > eta max(|c_t - c_s| - r_t - r_s, 0)  ->  near
//     (the low-frequency branch of src/admissibility/nearinteractions.jl:84-95),
//   - FarData and its test->trial transpose (src/admissibility/farinteractions.jl:16-92),
//   - farfield: own far nodes, then each ancestor's (farinteractions.jl:38-60),
//   - _selectfarpivots with tree mimicry (src/compressors/batchedbottomup.jl:54-72).
//
// Rules fixed by this project where the reference's dependencies are not available
// (AdaptiveCrossApproximation.jl, H2Trees.jl): 2-means splits seeded by the point farthest
// from the centroid and the point farthest from that one, Lloyd iterations with ties to the
// first cluster, sums over a cluster taken in ordered chunks of 256 points, stable partition;
// tree mimicry picks, for each pivot, the far node whose centre maximises dmin^2/|y - c_t|^2
// (dmin: distance to the pivots chosen so far), descends
// by the same score to a leaf and takes the best untaken point there; ties go to the first
// candidate. Compiled with -ffp-contract=off: every fused multiply-add is an explicit
// std::fma, so results are reproducible bit for bit.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <thread>

#include <immintrin.h>
#include <sched.h>

#include "nca_internal.h"

namespace nca {

namespace {

inline double dist2(const double *a, const double *b) {
    double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
    return std::fma(dx, dx, std::fma(dy, dy, dz * dz));
}

constexpr int kLloydIterations = 50;
// Sums over a cluster's points are taken in chunks of kChunk consecutive points: each chunk summed
// in order from zero, the chunk sums added in chunk order (one chunk: the plain ordered sum).
// Clusters of at least kTeamPoints points are split by a team of host threads over the chunks;
// the fixed chunking makes the result independent of the team size.
constexpr int kChunk = 256;
constexpr int kTeamPoints = 16384;

// reusable barrier of a fixed team of threads: arrivals counted atomically, the last one opens
// the next generation; waiters spin briefly (a Lloyd step of a team is tens of microseconds, and a
// sleeping wait through a condition variable cost about as much as the step), then yield
struct TeamBarrier {
    std::atomic<int> waiting{0};
    std::atomic<unsigned> gen{0};
    const int n;
    explicit TeamBarrier(int count) : n(count) {}
    void wait() {
        const unsigned g = gen.load(std::memory_order_acquire);
        if (waiting.fetch_add(1, std::memory_order_acq_rel) + 1 == n) {
            waiting.store(0, std::memory_order_relaxed);
            gen.store(g + 1, std::memory_order_release);
            return;
        }
        for (int spin = 0; gen.load(std::memory_order_acquire) == g; ++spin) {
            if (spin < 4096)
                _mm_pause();
            else
                std::this_thread::yield();
        }
    }
};

struct Splitter {
    const double *pts;
    std::vector<int32_t> side, scratch;
    std::vector<double> px, py, pz;  // the cluster's points, gathered once per split (same values)

    // Reorders ids[0:cnt) into two stable groups; returns the size of the first one. nteam > 1
    // spreads the chunks of one cluster over that many threads.
    int split(int32_t *ids, int cnt, int nteam = 1) {
        side.assign(cnt, -1);
        scratch.resize(cnt);
        px.resize(cnt);
        py.resize(cnt);
        pz.resize(cnt);
        const int nch = (cnt + kChunk - 1) / kChunk;
        nteam = std::max(1, std::min(nteam, nch));
        // per chunk: partial sums of both groups, their counts, the farthest point, changes
        std::vector<double> part(size_t(nch) * 6);
        std::vector<int> num(size_t(nch) * 2), far_arg(nch);
        std::vector<double> far_d(nch);
        std::vector<char> chg(nch);
        double g[3] = {0.0, 0.0, 0.0}, from[3] = {0.0, 0.0, 0.0}, c[2][3];
        int a = 0, bidx = 0, first = 0;
        double spread = 0.0;
        bool stop = false;
        TeamBarrier bar(nteam);
        auto chunk_range = [&](int q, int &i0, int &i1) {
            i0 = q * kChunk;
            i1 = std::min(cnt, i0 + kChunk);
        };
        // the farthest point from `from` in every chunk of this thread (first on ties)
        auto farthest_local = [&](int tid) {
            for (int q = tid; q < nch; q += nteam) {
                int i0, i1;
                chunk_range(q, i0, i1);
                int arg = i0;
                double best = -1.0;
                for (int i = i0; i < i1; ++i) {
                    const double p[3] = {px[i], py[i], pz[i]};
                    const double d = dist2(p, from);
                    if (d > best) {
                        best = d;
                        arg = i;
                    }
                }
                far_arg[q] = arg;
                far_d[q] = best;
            }
        };
        auto farthest_combine = [&](double &best) {
            int arg = 0;
            best = -1.0;
            for (int q = 0; q < nch; ++q)
                if (far_d[q] > best) {
                    best = far_d[q];
                    arg = far_arg[q];
                }
            return arg;
        };
        auto body = [&](int tid) {
            // centroid of the cluster
            for (int q = tid; q < nch; q += nteam) {
                int i0, i1;
                chunk_range(q, i0, i1);
                double t[3] = {0.0, 0.0, 0.0};
                for (int i = i0; i < i1; ++i) {
                    const double *p = pts + 3 * int64_t(ids[i]);
                    px[i] = p[0];
                    py[i] = p[1];
                    pz[i] = p[2];
                    t[0] += p[0];
                    t[1] += p[1];
                    t[2] += p[2];
                }
                for (int d = 0; d < 3; ++d) part[6 * size_t(q) + d] = t[d];
            }
            bar.wait();
            if (tid == 0) {
                for (int q = 0; q < nch; ++q)
                    for (int d = 0; d < 3; ++d) g[d] += part[6 * size_t(q) + d];
                for (double &v : g) v /= cnt;
                std::memcpy(from, g, sizeof(from));
            }
            bar.wait();
            farthest_local(tid);
            bar.wait();
            if (tid == 0) {
                double best;
                a = farthest_combine(best);
                std::memcpy(from, pts + 3 * int64_t(ids[a]), sizeof(from));
            }
            bar.wait();
            farthest_local(tid);
            bar.wait();
            if (tid == 0) {
                bidx = farthest_combine(spread);
                if (spread > 0.0) {
                    std::memcpy(c[0], pts + 3 * int64_t(ids[a]), sizeof(c[0]));
                    std::memcpy(c[1], pts + 3 * int64_t(ids[bidx]), sizeof(c[1]));
                }
                stop = !(spread > 0.0);
            }
            bar.wait();
            for (int it = 0; it < kLloydIterations && !stop; ++it) {
                // assignment, and the groups' sums under the new assignment, chunk by chunk
                for (int q = tid; q < nch; q += nteam) {
                    int i0, i1;
                    chunk_range(q, i0, i1);
                    bool changed = false;
                    double t[2][3] = {{0, 0, 0}, {0, 0, 0}};
                    int m[2] = {0, 0};
                    for (int i = i0; i < i1; ++i) {
                        const double p[3] = {px[i], py[i], pz[i]};
                        const int32_t sd = dist2(p, c[1]) < dist2(p, c[0]) ? 1 : 0;
                        if (sd != side[i]) {
                            side[i] = sd;
                            changed = true;
                        }
                        for (int d = 0; d < 3; ++d) t[sd][d] += p[d];
                        ++m[sd];
                    }
                    chg[q] = changed;
                    for (int k = 0; k < 2; ++k) {
                        for (int d = 0; d < 3; ++d) part[6 * size_t(q) + 3 * k + d] = t[k][d];
                        num[2 * size_t(q) + k] = m[k];
                    }
                }
                bar.wait();
                if (tid == 0) {
                    bool changed = false;
                    for (int q = 0; q < nch; ++q) changed = changed || chg[q];
                    if (!changed) {
                        stop = true;
                    } else {
                        double sum[2][3] = {{0, 0, 0}, {0, 0, 0}};
                        int n2[2] = {0, 0};
                        for (int q = 0; q < nch; ++q)
                            for (int k = 0; k < 2; ++k) {
                                for (int d = 0; d < 3; ++d) sum[k][d] += part[6 * size_t(q) + 3 * k + d];
                                n2[k] += num[2 * size_t(q) + k];
                            }
                        if (n2[0] == 0 || n2[1] == 0) {
                            stop = true;
                        } else {
                            for (int k = 0; k < 2; ++k)
                                for (int d = 0; d < 3; ++d) c[k][d] = sum[k][d] / n2[k];
                        }
                    }
                }
                bar.wait();
            }
        };
        if (nteam == 1) {
            body(0);
        } else {
            std::vector<std::thread> team;
            for (int t = 1; t < nteam; ++t) team.emplace_back(body, t);
            body(0);
            for (auto &th : team) th.join();
        }
        if (spread > 0.0) first = int(std::count(side.begin(), side.end(), 0));
        if (first == 0 || first == cnt) {
            first = (cnt + 1) / 2;
            for (int i = 0; i < cnt; ++i) side[i] = i < first ? 0 : 1;
        }
        int k = 0;
        for (int grp = 0; grp < 2; ++grp)
            for (int i = 0; i < cnt; ++i)
                if (side[i] == grp) scratch[k++] = ids[i];
        std::copy(scratch.begin(), scratch.end(), ids);
        return first;
    }
};

}  // namespace

Tree build_kmeans_tree(const double *pts, int64_t n, int minvalues) {
    Tree T;
    T.npoints = n;
    T.perm.resize(n);
    for (int64_t i = 0; i < n; ++i) T.perm[i] = int32_t(i);
    T.begin.push_back(0);
    T.end.push_back(int32_t(n));
    T.parent.push_back(-1);
    T.level.push_back(0);
    // Breadth-first, one level at a time: the nodes of a level split their own ranges of perm
    // independently on the host threads, then their children are numbered in node order.
    const int nth = n >= 32768 ? host_threads() : 1;  // small trees: no thread start-up
    auto parallel_for = [&](int n0, int n1, auto &&fn) {
        std::atomic<int> cursor{n0};
        auto work = [&]() {
            for (;;) {
                const int i = cursor.fetch_add(1);
                if (i >= n1) break;
                fn(i);
            }
        };
        const int use = std::max(1, std::min(nth, n1 - n0));
        std::vector<std::thread> pool;
        for (int t = 1; t < use; ++t) pool.emplace_back(work);
        work();
        for (auto &th : pool) th.join();
    };
    std::vector<int32_t> first;
    for (size_t lev0 = 0, lev1 = T.begin.size(); lev0 < lev1; lev0 = lev1, lev1 = T.begin.size()) {
        first.assign(lev1 - lev0, -1);
        parallel_for(int(lev0), int(lev1), [&](int node) {
            thread_local Splitter sp{nullptr, {}, {}};
            sp.pts = pts;
            const int b = T.begin[node], cnt = T.end[node] - b;
            // a level of few nodes (the top of the tree) gives each large cluster a team of threads
            const int team = cnt >= kTeamPoints ? std::max(1, nth / std::max(1, int(lev1 - lev0))) : 1;
            if (cnt > minvalues && cnt >= 2) first[node - lev0] = sp.split(T.perm.data() + b, cnt, team);
        });
        for (size_t node = lev0; node < lev1; ++node) {
            const int b = T.begin[node], e = T.end[node];
            if (first[node - lev0] >= 0) {
                T.firstchild.push_back(int32_t(T.begin.size()));
                T.nchildren.push_back(2);
                const int bounds[3] = {b, b + first[node - lev0], e};
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
    parallel_for(0, T.nnodes, [&](int node) {
        double s[3] = {0, 0, 0};
        for (int c0 = T.begin[node]; c0 < T.end[node]; c0 += kChunk) {
            const int c1 = std::min(T.end[node], c0 + kChunk);
            double part[3] = {0, 0, 0};
            for (int i = c0; i < c1; ++i)
                for (int d = 0; d < 3; ++d) part[d] += pts[3 * int64_t(T.perm[i]) + d];
            for (int d = 0; d < 3; ++d) s[d] += part[d];
        }
        int cnt = T.size(node);
        double *c = &T.center[3 * size_t(node)];
        for (int d = 0; d < 3; ++d) c[d] = cnt > 0 ? s[d] / cnt : 0.0;
        double m = 0.0;
        for (int i = T.begin[node]; i < T.end[node]; ++i)
            m = std::max(m, dist2(pts + 3 * int64_t(T.perm[i]), c));
        T.radius[node] = std::sqrt(m);
    });
    T.nlevels = T.level.back() + 1;
    T.levelptr.assign(T.nlevels + 1, T.nnodes);
    for (int node = T.nnodes - 1; node >= 0; --node) T.levelptr[T.level[node]] = node;
    T.iperm.resize(n);
    for (int64_t i = 0; i < n; ++i) T.iperm[T.perm[i]] = int32_t(i);
    return T;
}

namespace {

bool isnear(const Tree &A, const Tree &B, int a, int b, double eta) {
    double ra = A.radius[a], rb = B.radius[b];
    double gap = std::sqrt(dist2(&A.center[3 * size_t(a)], &B.center[3 * size_t(b)])) - (ra + rb);
    double sep = gap > 0.0 ? gap : 0.0;
    return 2.0 * std::max(ra, rb) > eta * sep;
}

struct PairSink {
    std::vector<int32_t> nt, ns, ft, fs;
};

void traverse(const Tree &T, const Tree &S, int t, int s, double eta, PairSink &out) {
    if (!isnear(T, S, t, s, eta)) {
        out.ft.push_back(t);
        out.fs.push_back(s);
        return;
    }
    bool lt = T.isleaf(t), ls = S.isleaf(s);
    if (lt && ls) {
        out.nt.push_back(t);
        out.ns.push_back(s);
    } else if (lt) {
        for (int c = 0; c < S.nchildren[s]; ++c) traverse(T, S, t, S.firstchild[s] + c, eta, out);
    } else if (ls) {
        for (int c = 0; c < T.nchildren[t]; ++c) traverse(T, S, T.firstchild[t] + c, s, eta, out);
    } else {
        for (int c = 0; c < T.nchildren[t]; ++c)
            for (int d = 0; d < S.nchildren[s]; ++d)
                traverse(T, S, T.firstchild[t] + c, S.firstchild[s] + d, eta, out);
    }
}

void to_csr(const std::vector<int32_t> &key, const std::vector<int32_t> &val, int nrows,
            std::vector<int32_t> &ptr, std::vector<int32_t> &idx) {
    ptr.assign(nrows + 1, 0);
    for (int32_t k : key) ++ptr[k + 1];
    for (int r = 0; r < nrows; ++r) ptr[r + 1] += ptr[r];
    idx.resize(key.size());
    std::vector<int32_t> cursor(ptr.begin(), ptr.end() - 1);
    for (size_t i = 0; i < key.size(); ++i) idx[cursor[key[i]]++] = val[i];
    for (int r = 0; r < nrows; ++r) std::sort(idx.begin() + ptr[r], idx.begin() + ptr[r + 1]);
}

}  // namespace

Partition build_partition(const Tree &test, const Tree &trial, double eta) {
    PairSink sink;
    if (test.nnodes > 0 && trial.nnodes > 0) traverse(test, trial, 0, 0, eta, sink);
    Partition P;
    to_csr(sink.nt, sink.ns, test.nnodes, P.nearptr, P.nearnodes);
    to_csr(sink.ft, sink.fs, test.nnodes, P.farptr, P.farnodes);
    to_csr(sink.ns, sink.nt, trial.nnodes, P.tnearptr, P.tnearnodes);
    to_csr(sink.fs, sink.ft, trial.nnodes, P.tfarptr, P.tfarnodes);
    return P;
}

namespace {

// Per-thread caches of the tree-mimicry selection, valid for one selection (generation stamp):
// the running minimum squared distance of a point / node centre to the chosen pivots and how
// many pivots it already accounts for, the pivots taken inside each node, the taken positions.
// Minima and counts are exact, so the cached selection equals the direct one bit for bit.
struct MimicryCache {
    uint32_t gen = 0;
    std::vector<uint32_t> pst, nst, tst, kst;
    std::vector<double> pd, nd;
    std::vector<int32_t> pc, nc, taken;
    void prepare(const Tree &F) {
        if (pst.size() < size_t(F.npoints)) {
            pst.assign(F.npoints, 0);
            kst.assign(F.npoints, 0);
            pd.assign(F.npoints, 0.0);
            pc.assign(F.npoints, 0);
        }
        if (nst.size() < size_t(F.nnodes)) {
            nst.assign(F.nnodes, 0);
            tst.assign(F.nnodes, 0);
            nd.assign(F.nnodes, 0.0);
            nc.assign(F.nnodes, 0);
            taken.assign(F.nnodes, 0);
        }
        if (++gen == 0) {  // wrapped: clear every stamp
            std::fill(pst.begin(), pst.end(), 0);
            std::fill(kst.begin(), kst.end(), 0);
            std::fill(nst.begin(), nst.end(), 0);
            std::fill(tst.begin(), tst.end(), 0);
            gen = 1;
        }
    }
};
thread_local MimicryCache t_cache;

// Greedy tree-mimicry selection state for one cluster.
class Mimicry {
  public:
    Mimicry(const Tree &far, const double *farpts, const double *centroid, const int32_t *roots,
            int nroots, int capacity)
        : F_(far), pts_(farpts), roots_(roots), nroots_(nroots), C_(t_cache) {
        std::memcpy(c_, centroid, sizeof(c_));
        chosen_xyz_.reserve(3 * size_t(capacity));
        root_dmin_.assign(nroots, 1.0);
        root_taken_.assign(nroots, 0);
        C_.prepare(far);
    }

    int32_t next() {
        int node = -1;
        double best = -1.0;
        for (int i = 0; i < nroots_; ++i) {
            int f = roots_[i];
            if (F_.size(f) - root_taken_[i] <= 0) continue;
            double sc = score(&F_.center[3 * size_t(f)], root_dmin_[i]);
            if (sc > best) {
                best = sc;
                node = f;
            }
        }
        while (!F_.isleaf(node)) {
            int pick = -1;
            double pbest = -1.0;
            for (int c = 0; c < F_.nchildren[node]; ++c) {
                int ch = F_.firstchild[node] + c;
                if (F_.size(ch) - taken_inside(ch) <= 0) continue;
                const double *cc = &F_.center[3 * size_t(ch)];
                double sc = score(cc, dmin_cached(C_.nst, C_.nd, C_.nc, ch, cc));
                if (sc > pbest) {
                    pbest = sc;
                    pick = ch;
                }
            }
            node = pick;
        }
        int bestpos = -1;
        best = -1.0;
        for (int pos = F_.begin[node]; pos < F_.end[node]; ++pos) {
            if (C_.kst[pos] == C_.gen) continue;  // already chosen
            const double *y = pts_ + 3 * int64_t(F_.perm[pos]);
            double sc = score(y, dmin_cached(C_.pst, C_.pd, C_.pc, pos, y));
            if (sc > best) {
                best = sc;
                bestpos = pos;
            }
        }
        int32_t id = F_.perm[bestpos];
        const double *y = pts_ + 3 * int64_t(id);
        bool firstpick = nchosen_ == 0;
        C_.kst[bestpos] = C_.gen;
        chosen_xyz_.insert(chosen_xyz_.end(), y, y + 3);
        ++nchosen_;
        for (int a = node; a >= 0; a = F_.parent[a]) {
            if (C_.tst[a] != C_.gen) {
                C_.tst[a] = C_.gen;
                C_.taken[a] = 0;
            }
            ++C_.taken[a];
        }
        for (int i = 0; i < nroots_; ++i) {
            int f = roots_[i];
            double d = dist2(&F_.center[3 * size_t(f)], y);
            if (firstpick || d < root_dmin_[i]) root_dmin_[i] = d;
            if (bestpos >= F_.begin[f] && bestpos < F_.end[f]) ++root_taken_[i];
        }
        return id;
    }

  private:
    double score(const double *y, double dmin2) const {
        double d2 = dist2(y, c_);
        if (d2 < 1e-300) d2 = 1e-300;
        return dmin2 / d2;
    }
    // min over the chosen pivots of the squared distance to y (1 before the first pick),
    // caught up from the pivots this entry has not seen yet
    double dmin_cached(std::vector<uint32_t> &st, std::vector<double> &dv, std::vector<int32_t> &cnt, int idx,
                       const double *y) {
        if (nchosen_ == 0) return 1.0;
        if (st[idx] != C_.gen) {
            st[idx] = C_.gen;
            dv[idx] = INFINITY;
            cnt[idx] = 0;
        }
        double m = dv[idx];
        for (int q = cnt[idx]; q < nchosen_; ++q) m = std::min(m, dist2(y, &chosen_xyz_[3 * size_t(q)]));
        dv[idx] = m;
        cnt[idx] = nchosen_;
        return m;
    }
    int taken_inside(int node) const { return C_.tst[node] == C_.gen ? C_.taken[node] : 0; }

    const Tree &F_;
    const double *pts_;
    const int32_t *roots_;
    int nroots_;
    MimicryCache &C_;
    double c_[3];
    std::vector<double> chosen_xyz_;
    int nchosen_ = 0;
    std::vector<double> root_dmin_;
    std::vector<int> root_taken_;
};

}  // namespace

void cluster_centroid(const double *ownpts, const int32_t *refidcs, int nref, double *c) {
    double s[3] = {0, 0, 0};
    for (int i = 0; i < nref; ++i)
        for (int d = 0; d < 3; ++d) s[d] += ownpts[3 * int64_t(refidcs[i]) + d];
    for (int d = 0; d < 3; ++d) c[d] = s[d] / nref;
}

int select_farpivots_at(const Tree &far, const double *farpts, const double *centroid, int nref,
                        const int32_t *farnodes, int nfar, int maxrank, int32_t *out) {
    int limit = std::min(maxrank, nref);
    int n = 0;
    for (int i = 0; i < nfar && limit - n > 0; ++i) {
        n += std::min(limit - n, far.size(farnodes[i]));
    }
    if (n <= 0) return 0;
    Mimicry M(far, farpts, centroid, farnodes, nfar, n);
    for (int p = 0; p < n; ++p) out[p] = M.next();
    return n;
}

int select_farpivots(const Tree &far, const double *ownpts, const double *farpts,
                     const int32_t *refidcs, int nref, const int32_t *farnodes, int nfar,
                     int maxrank, int32_t *out) {
    double c[3];
    cluster_centroid(ownpts, refidcs, nref, c);
    return select_farpivots_at(far, farpts, c, nref, farnodes, nfar, maxrank, out);
}

// The cores this process may run on: its CPU affinity mask, capped by a cgroup CPU quota
// (cpu.max) when there is one, at most 64. The machine's processor count alone overstates it in a
// container that is given a share of a larger host.
int host_threads() {
    static const int n = [] {
        int c = 0;
        cpu_set_t set;
        CPU_ZERO(&set);
        if (sched_getaffinity(0, sizeof(set), &set) == 0) c = CPU_COUNT(&set);
        if (c <= 0) c = int(std::thread::hardware_concurrency());
        if (FILE *f = std::fopen("/sys/fs/cgroup/cpu.max", "r")) {
            char quota[32] = {0};
            long long period = 0;
            if (std::fscanf(f, "%31s %lld", quota, &period) == 2 && std::strcmp(quota, "max") != 0 && period > 0) {
                const long long q = std::atoll(quota);
                if (q > 0) c = std::min<long long>(c, std::max<long long>(1, (q + period - 1) / period));
            }
            std::fclose(f);
        }
        return std::max(1, std::min(c, 64));
    }();
    return n;
}

void all_farpivots(const Tree &own, const Tree &far, const double *ownpts, const double *farpts,
                   const std::vector<int32_t> &ptr, const std::vector<int32_t> &nodes,
                   int maxrank, std::vector<int32_t> &fpptr, std::vector<int32_t> &fpidx) {
    int nn = own.nnodes;
    std::vector<int32_t> count(nn, 0);
    std::vector<int32_t> buf(size_t(nn) * std::max(maxrank, 1));
    std::atomic<int> cursor{0};
    auto work = [&]() {
        std::vector<int32_t> ff;
        for (;;) {
            int t = cursor.fetch_add(1);
            if (t >= nn) break;
            ff.clear();
            for (int a = t; a >= 0; a = own.parent[a])
                ff.insert(ff.end(), nodes.begin() + ptr[a], nodes.begin() + ptr[a + 1]);
            if (ff.empty()) continue;
            count[t] = select_farpivots(far, ownpts, farpts, own.perm.data() + own.begin[t],
                                        own.size(t), ff.data(), int(ff.size()), maxrank,
                                        buf.data() + size_t(t) * maxrank);
        }
    };
    int nth = std::max(1, std::min(host_threads(), nn));
    std::vector<std::thread> pool;
    for (int i = 1; i < nth; ++i) pool.emplace_back(work);
    work();
    for (auto &th : pool) th.join();
    fpptr.assign(nn + 1, 0);
    for (int t = 0; t < nn; ++t) fpptr[t + 1] = fpptr[t] + count[t];
    fpidx.resize(fpptr[nn]);
    for (int t = 0; t < nn; ++t)
        std::copy(buf.begin() + size_t(t) * maxrank, buf.begin() + size_t(t) * maxrank + count[t],
                  fpidx.begin() + fpptr[t]);
}

}  // namespace nca
