// Host planning of directional (wideband) H^2 matrices:
//
//   build_partition_wideband  near/far pairs with the wideband admissibility
//                             (src/admissibility/nearinteractions.jl:84-95 for bounding balls):
//                             low frequency (k min(d) <= gamma): near iff max(d) > eta_lf sep,
//                             high frequency: near iff 4 k max(r)^2 > eta_hf sep.
//   directional_plan          per cluster the direction set, the far nodes grouped by their
//                             nearest direction and the parent-to-child direction map
//                             (src/admissibility/directionalsubdivision/boundingballdirections.jl:44-152,
//                             abstractdirections.jl:73-116), then the basis items: one per
//                             (cluster, direction), a basis item if the cluster is a leaf or a
//                             high-frequency cluster with low-frequency children
//                             (abstractdirections.jl:238-243), otherwise nested in the children's
//                             items of the mapped directions (src/compressors/bottomup.jl:214-320).
//   item_farfield             the far field of an item: its own far nodes followed by those of
//                             the ancestors' directions that map onto it (dirfarfield,
//                             abstractdirections.jl:192-231).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <functional>
#include <stdexcept>
#include <thread>

#include <immintrin.h>

#include "nca_internal.h"

namespace nca {

namespace {

inline double d2(const double *a, const double *b) {
    const double x = a[0] - b[0], y = a[1] - b[1], z = a[2] - b[2];
    return x * x + y * y + z * z;
}

bool isnear_wideband(const Tree &A, const Tree &B, int a, int b, const Wideband &w) {
    const double ra = A.radius[a], rb = B.radius[b];
    const double gap = std::sqrt(d2(&A.center[3 * size_t(a)], &B.center[3 * size_t(b)])) - (ra + rb);
    const double sep = gap > 0.0 ? gap : 0.0;
    if (w.k * std::min(2.0 * ra, 2.0 * rb) <= w.gamma) return 2.0 * std::max(ra, rb) > w.etalf * sep;
    return 4.0 * w.k * std::max(ra * ra, rb * rb) > w.etahf * sep;
}

struct Pairs {
    std::vector<int32_t> nt, ns, ft, fs;
};

void traverse_wideband(const Tree &T, const Tree &S, int t, int s, const Wideband &w, Pairs &out) {
    if (!isnear_wideband(T, S, t, s, w)) {
        out.ft.push_back(t);
        out.fs.push_back(s);
        return;
    }
    const bool lt = T.isleaf(t), ls = S.isleaf(s);
    if (lt && ls) {
        out.nt.push_back(t);
        out.ns.push_back(s);
    } else if (lt) {
        for (int c = 0; c < S.nchildren[s]; ++c) traverse_wideband(T, S, t, S.firstchild[s] + c, w, out);
    } else if (ls) {
        for (int c = 0; c < T.nchildren[t]; ++c) traverse_wideband(T, S, T.firstchild[t] + c, s, w, out);
    } else {
        for (int c = 0; c < T.nchildren[t]; ++c)
            for (int d = 0; d < S.nchildren[s]; ++d)
                traverse_wideband(T, S, T.firstchild[t] + c, S.firstchild[s] + d, w, out);
    }
}

void csr(const std::vector<int32_t> &key, const std::vector<int32_t> &val, int nrows, std::vector<int32_t> &ptr,
         std::vector<int32_t> &idx) {
    ptr.assign(nrows + 1, 0);
    for (int32_t k : key) ++ptr[k + 1];
    for (int r = 0; r < nrows; ++r) ptr[r + 1] += ptr[r];
    idx.resize(key.size());
    std::vector<int32_t> cursor(ptr.begin(), ptr.end() - 1);
    for (size_t i = 0; i < key.size(); ++i) idx[cursor[key[i]]++] = val[i];
    for (int r = 0; r < nrows; ++r) std::sort(idx.begin() + ptr[r], idx.begin() + ptr[r + 1]);
}

// Generalised radius of a node: the smaller of the parent's and the mean radius of the
// siblings, so that siblings share one low/high-frequency class
// (nearinteractions.jl:142-153).
double genradius(const Tree &T, int node) {
    const int p = T.parent[node];
    if (p < 0) return T.radius[node];
    double sum = 0.0;
    for (int c = 0; c < T.nchildren[p]; ++c) sum += T.radius[T.firstchild[p] + c];
    return std::min(genradius(T, p), sum / T.nchildren[p]);
}

// Candidate directions of a cluster of diameter diam: n = max(6, ceil(6 * 4^log2(
// acos(1/sqrt 3) / asin(min(1, gamma / (k diam)))))) spherical Fibonacci points
// (boundingballdirections.jl:12-29).
int64_t candidate_count(double diam, double k, double gamma) {
    const double kd = std::max(k * diam, 0x1p-52);
    const double ratio = std::acos(1.0 / std::sqrt(3.0)) / std::asin(std::min(1.0, gamma / kd));
    const int64_t n = int64_t(std::ceil(6.0 * std::pow(4.0, std::log(ratio) / std::log(2.0))));
    return std::max<int64_t>(6, n);
}

// the n spherical Fibonacci points (a function of n alone)
void fibonacci_points(int64_t n, std::vector<double> &out) {
    out.resize(3 * size_t(n));
    const double ga = M_PI * (3.0 - std::sqrt(5.0));
    for (int64_t i = 0; i < n; ++i) {
        const double z = 1.0 - 2.0 * (double(i) + 0.5) / double(n);
        const double r = std::sqrt(std::max(0.0, 1.0 - z * z));
        out[3 * i] = r * std::cos(double(i) * ga);
        out[3 * i + 1] = r * std::sin(double(i) * ga);
        out[3 * i + 2] = z;
    }
}

void candidate_directions(double diam, double k, double gamma, std::vector<double> &out) {
    fibonacci_points(candidate_count(diam, k, gamma), out);
}

// 0-based index of the direction with the largest dot product (first on ties), one candidate
// at a time: the reference form of the search (the checks compare the planner's search with it).
int nearest_direction(const std::vector<double> &dirs, const double *v) {
    const size_t n = dirs.size() / 3;
    int best = 0;
    double bd = dirs[0] * v[0] + dirs[1] * v[1] + dirs[2] * v[2];
    for (size_t i = 1; i < n; ++i) {
        const double d = dirs[3 * i] * v[0] + dirs[3 * i + 1] * v[1] + dirs[3 * i + 2] * v[2];
        if (d > bd) {
            bd = d;
            best = int(i);
        }
    }
    return best;
}

// The candidates of one cluster as coordinate arrays (x[i], y[i], z[i]), i < n.
struct Candidates {
    std::vector<double> xyz;
    const double *x = nullptr, *y = nullptr, *z = nullptr;
    int64_t n = 0;
    double band = 0.0, cb = 0.0, sb = 0.0;  // the search band's half angle, its cosine and sine
    void set(const std::vector<double> &dirs) {
        n = int64_t(dirs.size() / 3);
        band = 4.0 * std::sqrt(4.0 * M_PI / double(n));
        cb = std::cos(band);
        sb = std::sin(band);
        xyz.resize(3 * size_t(n));
        for (int64_t i = 0; i < n; ++i) {
            xyz[i] = dirs[3 * i];
            xyz[n + i] = dirs[3 * i + 1];
            xyz[2 * n + i] = dirs[3 * i + 2];
        }
        x = xyz.data();
        y = x + n;
        z = y + n;
    }
};

// Index of the largest x_i v0 + y_i v1 + z_i v2 over i0 <= i <= i1, the first on ties. Every dot is
// formed as (x v0 + y v1) + z v2 with each product and sum rounded (no fused multiply-add), four
// candidates at a time: each lane keeps its largest dot and the first index reaching it, the lanes
// are merged by value then index, and the tail follows in order.
// Eight candidates at a time where the host has AVX-512 (same rule: lanes merged by value, then
// index, the tail in order).
__attribute__((target("avx512f"))) int64_t argmax_dot8(const Candidates &c, int64_t i0, int64_t i1,
                                                       const double *v) {
    int64_t i = i0, best = i0;
    double bd = -INFINITY;
    if (i1 - i0 + 1 >= 16) {
        const __m512d v0 = _mm512_set1_pd(v[0]), v1 = _mm512_set1_pd(v[1]), v2 = _mm512_set1_pd(v[2]);
        const __m512d eight = _mm512_set1_pd(8.0);
        __m512d bv = _mm512_set1_pd(-INFINITY), bi = _mm512_setzero_pd();
        __m512d idx = _mm512_add_pd(_mm512_set1_pd(double(i)), _mm512_setr_pd(0, 1, 2, 3, 4, 5, 6, 7));
        for (; i + 7 <= i1; i += 8) {
            const __m512d d = _mm512_add_pd(
                _mm512_add_pd(_mm512_mul_pd(_mm512_loadu_pd(c.x + i), v0), _mm512_mul_pd(_mm512_loadu_pd(c.y + i), v1)),
                _mm512_mul_pd(_mm512_loadu_pd(c.z + i), v2));
            const __mmask8 gt = _mm512_cmp_pd_mask(d, bv, _CMP_GT_OQ);
            bv = _mm512_mask_blend_pd(gt, bv, d);
            bi = _mm512_mask_blend_pd(gt, bi, idx);
            idx = _mm512_add_pd(idx, eight);
        }
        alignas(64) double lv[8], li[8];
        _mm512_store_pd(lv, bv);
        _mm512_store_pd(li, bi);
        for (int l = 0; l < 8; ++l)
            if (lv[l] > bd || (lv[l] == bd && int64_t(li[l]) < best)) {
                bd = lv[l];
                best = int64_t(li[l]);
            }
    }
    for (; i <= i1; ++i) {
        const double d = c.x[i] * v[0] + c.y[i] * v[1] + c.z[i] * v[2];
        if (d > bd) {
            bd = d;
            best = i;
        }
    }
    return best;
}

int64_t argmax_dot4(const Candidates &c, int64_t i0, int64_t i1, const double *v) {
    int64_t i = i0, best = i0;
    double bd = -INFINITY;
    if (i1 - i0 + 1 >= 8) {
        const __m256d v0 = _mm256_set1_pd(v[0]), v1 = _mm256_set1_pd(v[1]), v2 = _mm256_set1_pd(v[2]);
        const __m256d four = _mm256_set1_pd(4.0);
        __m256d bv = _mm256_set1_pd(-INFINITY), bi = _mm256_setzero_pd();
        __m256d idx = _mm256_setr_pd(double(i), double(i + 1), double(i + 2), double(i + 3));
        for (; i + 3 <= i1; i += 4) {
            const __m256d d = _mm256_add_pd(
                _mm256_add_pd(_mm256_mul_pd(_mm256_loadu_pd(c.x + i), v0), _mm256_mul_pd(_mm256_loadu_pd(c.y + i), v1)),
                _mm256_mul_pd(_mm256_loadu_pd(c.z + i), v2));
            const __m256d gt = _mm256_cmp_pd(d, bv, _CMP_GT_OQ);
            bv = _mm256_blendv_pd(bv, d, gt);
            bi = _mm256_blendv_pd(bi, idx, gt);
            idx = _mm256_add_pd(idx, four);
        }
        alignas(32) double lv[4], li[4];
        _mm256_store_pd(lv, bv);
        _mm256_store_pd(li, bi);
        for (int l = 0; l < 4; ++l)
            if (lv[l] > bd || (lv[l] == bd && int64_t(li[l]) < best)) {
                bd = lv[l];
                best = int64_t(li[l]);
            }
    }
    for (; i <= i1; ++i) {
        const double d = c.x[i] * v[0] + c.y[i] * v[1] + c.z[i] * v[2];
        if (d > bd) {
            bd = d;
            best = i;
        }
    }
    return best;
}

int64_t argmax_dot(const Candidates &c, int64_t i0, int64_t i1, const double *v) {
    static const bool wide = __builtin_cpu_supports("avx512f");
    return wide ? argmax_dot8(c, i0, i1, v) : argmax_dot4(c, i0, i1, v);
}

// Index of the candidate nearest to direction v: the largest dot product, the first on ties
// (nearest_direction). Over the spherical Fibonacci candidates of candidate_directions (z_i =
// 1 - 2 (i + 1/2) / n, descending) only the indices whose z lies within an angle of
// 4 sqrt(4 pi / n) of v's polar angle are searched. That band holds every candidate within twice
// the lattice's covering radius of v, so the largest dot product lies inside it, ahead of every
// candidate outside by about 75 / n of |v|, far above the rounding of a three-term dot product.
// Inside the band the dots are formed and compared as in the full search, so the result is the
// full search's.
// The band's z limits cos(max(0, theta - band)) and cos(min(pi, theta + band)) are formed from
// cos theta = v_z / |v| by the angle-sum formulas; their rounding (~1e-16) is far inside the one
// index of slack added on each side (2 / n in z).
int nearest_candidate(const Candidates &c, const double *v) {
    const int64_t n = c.n;
    const double r = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    if (!(r > 0.0) || !std::isfinite(r) || c.band >= 0.5 * M_PI) return int(argmax_dot(c, 0, n - 1, v));
    const double ct = std::max(-1.0, std::min(1.0, v[2] / r));
    const double st = std::sqrt(std::max(0.0, 1.0 - ct * ct));
    const double zhi = ct >= c.cb ? 1.0 : ct * c.cb + st * c.sb;
    const double zlo = ct <= -c.cb ? -1.0 : ct * c.cb - st * c.sb;
    // z_i <= zhi  <=>  i >= (1 - zhi) n / 2 - 1/2;  z_i >= zlo  <=>  i <= (1 - zlo) n / 2 - 1/2
    const int64_t i0 = std::max<int64_t>(0, int64_t(std::floor((1.0 - zhi) * double(n) / 2.0 - 0.5)) - 1);
    const int64_t i1 = std::min<int64_t>(n - 1, int64_t(std::ceil((1.0 - zlo) * double(n) / 2.0 - 0.5)) + 1);
    return int(argmax_dot(c, i0, i1, v));
}

}  // namespace

// The lists of a node come out of csr sorted, so the pairs may be found in any order: the top of
// the traversal is expanded breadth first (near leaf pairs and far pairs found there kept) until
// it offers enough independent (test, trial) subtrees, which the host threads then traverse into
// their own lists; the four CSR lists are made side by side.
Partition build_partition_wideband(const Tree &test, const Tree &trial, const Wideband &w) {
    Pairs sink;
    std::vector<std::pair<int, int>> frontier, next;
    if (test.nnodes > 0 && trial.nnodes > 0) frontier.emplace_back(0, 0);
    const int nth = host_threads();
    while (!frontier.empty() && frontier.size() < size_t(16) * nth) {
        next.clear();
        for (const auto &ts : frontier) {
            const int t = ts.first, s = ts.second;
            if (!isnear_wideband(test, trial, t, s, w)) {
                sink.ft.push_back(t);
                sink.fs.push_back(s);
                continue;
            }
            const bool lt = test.isleaf(t), ls = trial.isleaf(s);
            if (lt && ls) {
                sink.nt.push_back(t);
                sink.ns.push_back(s);
            } else if (lt) {
                for (int c = 0; c < trial.nchildren[s]; ++c) next.emplace_back(t, trial.firstchild[s] + c);
            } else if (ls) {
                for (int c = 0; c < test.nchildren[t]; ++c) next.emplace_back(test.firstchild[t] + c, s);
            } else {
                for (int c = 0; c < test.nchildren[t]; ++c)
                    for (int d = 0; d < trial.nchildren[s]; ++d)
                        next.emplace_back(test.firstchild[t] + c, trial.firstchild[s] + d);
            }
        }
        frontier.swap(next);
    }
    const int use = std::max(1, std::min(nth, int(frontier.size())));
    std::vector<Pairs> part(use);
    std::atomic<size_t> cursor{0};
    auto work = [&](int i) {
        for (;;) {
            const size_t f = cursor.fetch_add(1);
            if (f >= frontier.size()) break;
            traverse_wideband(test, trial, frontier[f].first, frontier[f].second, w, part[i]);
        }
    };
    {
        std::vector<std::thread> pool;
        for (int i = 1; i < use; ++i) pool.emplace_back(work, i);
        work(0);
        for (auto &th : pool) th.join();
    }
    for (const Pairs &q : part) {
        sink.nt.insert(sink.nt.end(), q.nt.begin(), q.nt.end());
        sink.ns.insert(sink.ns.end(), q.ns.begin(), q.ns.end());
        sink.ft.insert(sink.ft.end(), q.ft.begin(), q.ft.end());
        sink.fs.insert(sink.fs.end(), q.fs.begin(), q.fs.end());
    }
    Partition P;
    std::thread a([&] { csr(sink.nt, sink.ns, test.nnodes, P.nearptr, P.nearnodes); });
    std::thread b([&] { csr(sink.ft, sink.fs, test.nnodes, P.farptr, P.farnodes); });
    std::thread c([&] { csr(sink.ns, sink.nt, trial.nnodes, P.tnearptr, P.tnearnodes); });
    csr(sink.fs, sink.ft, trial.nnodes, P.tfarptr, P.tfarnodes);
    a.join();
    b.join();
    c.join();
    return P;
}

bool is_lowfrequency(const Tree &T, int node, const Wideband &w) { return w.k * (2.0 * genradius(T, node)) <= w.gamma; }

DirSide directional_plan(const Tree &T, const Tree &F, const std::vector<int32_t> &farptr,
                         const std::vector<int32_t> &farnodes_in, const Wideband &w) {
    const int nn = T.nnodes;
    DirSide D;
    D.farptr = farptr;
    D.farnodes = farnodes_in;
    std::vector<std::vector<int32_t>> dirs(nn), dircount(nn), pmap(nn);
    std::vector<std::vector<double>> dirvec(nn);
    std::vector<char> hasvec(nn, 0);
    std::vector<int32_t> pcount(nn, 0);
    std::vector<char> lf(nn);
    for (int node = 0; node < nn; ++node) lf[node] = is_lowfrequency(T, node, w);
    // the nodes of one level depend on their parents only: a level's nodes run on the host
    // threads, each writing its own entries (and its own range of the far-node list)
    auto plan_node = [&](int level, int node, std::vector<double> &total, Candidates &cand,
                         std::vector<int32_t> &slot) {
            const int p = T.parent[node];
            const bool hasfars = farptr[node + 1] > farptr[node];
            const bool hasparentvecs = p >= 0 && hasvec[p];
            const bool hasparentdirs = p >= 0 && !dirs[p].empty();
            if (lf[node]) {
                const bool inherit = hasparentdirs && level > 0 && lf[p];
                if (hasfars || inherit) dirs[node] = {0};
                if (inherit) pmap[node] = {1};
                return;
            }
            if (!hasfars && !hasparentvecs) return;
            // the candidates depend on their count alone: a thread keeps its last set, which the
            // next nodes of the level (of about the same size) mostly share
            const int64_t ncand = candidate_count(2.0 * T.radius[node], w.k, w.gamma);
            if (int64_t(total.size()) != 3 * ncand) {
                fibonacci_points(ncand, total);
                cand.set(total);
            }
            const int b = farptr[node], nfar = farptr[node + 1] - b;
            std::vector<int32_t> nd(nfar);
            const double *c = &T.center[3 * size_t(node)];
            for (int i = 0; i < nfar; ++i) {
                const double *cf = &F.center[3 * size_t(D.farnodes[b + i])];
                const double v[3] = {c[0] - cf[0], c[1] - cf[1], c[2] - cf[2]};
                nd[i] = nearest_candidate(cand, v) + 1;
            }
            // far nodes grouped by direction (stable)
            std::vector<int32_t> order(nfar);
            for (int i = 0; i < nfar; ++i) order[i] = i;
            std::stable_sort(order.begin(), order.end(), [&](int a, int q) { return nd[a] < nd[q]; });
            std::vector<int32_t> permuted(nfar), sorted(nfar);
            for (int i = 0; i < nfar; ++i) {
                permuted[i] = D.farnodes[b + order[i]];
                sorted[i] = nd[order[i]];
            }
            std::copy(permuted.begin(), permuted.end(), D.farnodes.begin() + b);
            std::vector<int32_t> uniq(sorted);
            uniq.erase(std::unique(uniq.begin(), uniq.end()), uniq.end());
            const size_t noriginal = uniq.size();
            // the child's direction of every parent direction, seen from the child's centre
            std::vector<int32_t> map;
            if (p >= 0) {
                map.assign(dirs[p].size(), 0);
                const double *cp = &T.center[3 * size_t(p)];
                const double rp2 = 2.0 * T.radius[p];
                const double mult = w.k * rp2 / w.etahf + rp2;
                for (size_t di = 0; di < dirs[p].size(); ++di) {
                    const double *pv = &dirvec[p][3 * di];
                    const double v[3] = {c[0] - cp[0] + mult * pv[0], c[1] - cp[1] + mult * pv[1],
                                         c[2] - cp[2] + mult * pv[2]};
                    map[di] = nearest_candidate(cand, v) + 1;
                }
                // candidate -> 1-based position in uniq (0: not yet listed), instead of a search
                // of uniq per parent direction
                slot.assign(total.size() / 3 + 1, 0);
                for (size_t u = 0; u < uniq.size(); ++u) slot[uniq[u]] = int32_t(u) + 1;
                for (size_t di = 0; di < map.size(); ++di) {
                    int32_t &at = slot[map[di]];
                    if (at == 0) {
                        uniq.push_back(map[di]);
                        at = int32_t(uniq.size());
                    }
                    map[di] = at;
                }
            }
            std::vector<int32_t> count(uniq.size(), 0);
            for (size_t u = 0, i = 0; u < noriginal; ++u)
                while (i < size_t(nfar) && sorted[i] == uniq[u]) {
                    ++count[u];
                    ++i;
                }
            dirvec[node].resize(3 * uniq.size());
            for (size_t u = 0; u < uniq.size(); ++u)
                for (int d = 0; d < 3; ++d) dirvec[node][3 * u + d] = total[3 * size_t(uniq[u] - 1) + d];
            hasvec[node] = 1;
            pcount[node] = int32_t(std::count_if(map.begin(), map.end(), [](int32_t x) { return x != 0; }));
            pmap[node] = map;
            dirs[node] = uniq;
            dircount[node] = count;
    };
    const int nth = host_threads();
    for (int level = 0; level < T.nlevels; ++level) {
        const int n0 = T.levelptr[level], n1 = T.levelptr[level + 1];
        std::atomic<int> cursor{n0};
        auto work = [&]() {
            std::vector<double> total;
            Candidates cand;
            std::vector<int32_t> slot;
            for (;;) {
                const int node = cursor.fetch_add(1);
                if (node >= n1) break;
                plan_node(level, node, total, cand, slot);
            }
        };
        const int use = std::max(1, std::min(nth, n1 - n0));
        std::vector<std::thread> pool;
        for (int i = 1; i < use; ++i) pool.emplace_back(work);
        work();
        for (auto &th : pool) th.join();
    }
    for (int node = 0; node < nn; ++node)
        if (!dirs[node].empty() && dircount[node].empty()) {
            dircount[node] = {std::max(0, farptr[node + 1] - farptr[node])};
            pcount[node] = int32_t(pmap[node].size());
        }
    // CSR: items (node, direction), far ranges per item, parent-to-child maps per node
    D.dirptr.assign(nn + 1, 0);
    D.chdirptr.assign(nn + 1, 0);
    for (int node = 0; node < nn; ++node) {
        D.dirptr[node + 1] = D.dirptr[node] + int32_t(dirs[node].size());
        D.chdirptr[node + 1] = D.chdirptr[node] + pcount[node];
    }
    const int ni = D.dirptr[nn];
    // The rest fills disjoint ranges per node or per item, on the host threads: fn(b, e) over
    // consecutive ranges of [0, n)
    auto in_ranges = [nth](int n, auto fn) {
        const int use = std::max(1, std::min(nth, n / 4096));
        std::vector<std::thread> pool;
        for (int k = 1; k < use; ++k)
            pool.emplace_back([&, k] { fn(int(int64_t(n) * k / use), int(int64_t(n) * (k + 1) / use)); });
        fn(0, int(int64_t(n) / use));
        for (auto &th : pool) th.join();
    };
    D.dirs.resize(ni);
    D.dirvec.assign(3 * size_t(ni), 0.0);
    D.dirfarptr.resize(ni + 1);
    D.chdirmap.resize(D.chdirptr[nn]);
    D.item_node.resize(ni);
    in_ranges(nn, [&](int n0, int n1) {
        for (int node = n0; node < n1; ++node) {
            int32_t off = farptr[node];
            for (size_t u = 0; u < dirs[node].size(); ++u) {
                const int item = D.dirptr[node] + int(u);
                D.dirs[item] = dirs[node][u];
                D.item_node[item] = node;
                if (hasvec[node])
                    for (int d = 0; d < 3; ++d) D.dirvec[3 * size_t(item) + d] = dirvec[node][3 * u + d];
                D.dirfarptr[item] = off;
                off += dircount[node][u];
            }
            std::copy(pmap[node].begin(), pmap[node].end(), D.chdirmap.begin() + D.chdirptr[node]);
        }
    });
    D.dirfarptr[ni] = farptr[nn];
    // the inverse of the parent-to-child maps: for every item the parent directions mapped onto it
    // (a node's map points at the node's own items only)
    D.invptr.assign(ni + 1, 0);
    in_ranges(nn, [&](int n0, int n1) {
        for (int node = n0; node < n1; ++node) {
            const int nown = D.dirptr[node + 1] - D.dirptr[node];
            for (int i = D.chdirptr[node]; i < D.chdirptr[node + 1]; ++i)
                if (D.chdirmap[i] >= 1 && D.chdirmap[i] <= nown) ++D.invptr[D.dirptr[node] + D.chdirmap[i]];
        }
    });
    for (int item = 0; item < ni; ++item) D.invptr[item + 1] += D.invptr[item];
    D.invidx.resize(D.invptr[ni]);
    {
        std::vector<int32_t> fill(D.invptr.begin(), D.invptr.end() - 1);
        in_ranges(nn, [&](int n0, int n1) {
            for (int node = n0; node < n1; ++node) {
                const int nown = D.dirptr[node + 1] - D.dirptr[node];
                for (int i = D.chdirptr[node]; i < D.chdirptr[node + 1]; ++i)
                    if (D.chdirmap[i] >= 1 && D.chdirmap[i] <= nown)
                        D.invidx[fill[D.dirptr[node] + D.chdirmap[i] - 1]++] = i - D.chdirptr[node] + 1;
            }
        });
    }
    // basis items and the children's items of nested ones: the basis flags and child counts per
    // item, their prefix, then the children's items
    D.item_basis.resize(ni);
    D.item_chptr.assign(ni + 1, 0);
    in_ranges(ni, [&](int i0, int i1) {
        for (int item = i0; item < i1; ++item) {
            const int node = D.item_node[item];
            bool basis;
            if (T.isleaf(node)) {
                basis = true;
            } else if (D.dirs[item] == 0) {
                basis = false;
            } else {
                const int fc = T.firstchild[node];
                basis = D.dirptr[fc + 1] == D.dirptr[fc] ||
                        (D.dirptr[fc + 1] - D.dirptr[fc] == 1 && D.dirs[D.dirptr[fc]] == 0);
            }
            D.item_basis[item] = basis;
            D.item_chptr[item + 1] = basis ? 0 : T.nchildren[node];
        }
    });
    for (int item = 0; item < ni; ++item) D.item_chptr[item + 1] += D.item_chptr[item];
    D.item_chidx.assign(size_t(D.item_chptr[ni]), 0);
    std::atomic<bool> missing{false};
    in_ranges(ni, [&](int i0, int i1) {
        for (int item = i0; item < i1; ++item) {
            if (D.item_basis[item]) continue;
            const int node = D.item_node[item];
            const int local = item - D.dirptr[node];  // 0-based local direction of the parent
            int32_t at = D.item_chptr[item];
            for (int c = 0; c < T.nchildren[node]; ++c) {
                const int ch = T.firstchild[node] + c;
                const int cnt = D.chdirptr[ch + 1] - D.chdirptr[ch];
                const int m = local < cnt ? D.chdirmap[D.chdirptr[ch] + local] : 0;  // 1-based local direction
                if (m <= 0) {
                    missing = true;
                    return;
                }
                D.item_chidx[at++] = D.dirptr[ch] + m - 1;
            }
        }
    });
    if (missing) throw std::runtime_error("directional plan: a child has no direction for its parent's");
    return D;
}

void item_farfield(const Tree &T, const DirSide &D, int item, std::vector<int32_t> &ff) {
    ff.clear();
    const int node = D.item_node[item];
    auto append = [&](int it) {
        ff.insert(ff.end(), D.farnodes.begin() + D.dirfarptr[it], D.farnodes.begin() + D.dirfarptr[it + 1]);
    };
    if (D.dirs[item] == 0) {
        for (int cur = node; cur >= 0; cur = T.parent[cur]) {
            int found = -1;
            for (int it = D.dirptr[cur]; it < D.dirptr[cur + 1]; ++it)
                if (D.dirs[it] == 0) {
                    found = it;
                    break;
                }
            if (found < 0) break;
            append(found);
        }
        return;
    }
    append(item);
    // idcs: the 1-based local directions of cur on the chain; next: the parent directions that map
    // onto any of them, ascending (each parent direction maps onto one child direction, so the
    // inverse lists are disjoint and their sorted union is the reference's scan in order)
    thread_local std::vector<int32_t> idcs, next;  // reused by every call on this thread
    idcs.assign(1, item - D.dirptr[node] + 1);
    for (int cur = node; T.parent[cur] >= 0; cur = T.parent[cur]) {
        const int p = T.parent[cur];
        next.clear();
        for (int32_t c : idcs) {
            const int it = D.dirptr[cur] + c - 1;
            next.insert(next.end(), D.invidx.begin() + D.invptr[it], D.invidx.begin() + D.invptr[it + 1]);
        }
        std::sort(next.begin(), next.end());
        for (int32_t pi : next) append(D.dirptr[p] + pi - 1);
        if (next.empty()) break;  // no ancestor direction maps onto the chain any more
        idcs.swap(next);
    }
}

void all_item_farpivots(const Tree &own, const Tree &far, const DirSide &D, const double *ownpts,
                        const double *farpts, int maxrank, std::vector<int32_t> &fpptr, std::vector<int32_t> &fpidx) {
    const int ni = int(D.item_node.size());
    std::vector<int32_t> count(ni, 0);
    std::vector<int32_t> buf(size_t(ni) * std::max(maxrank, 1));
    // every direction of a cluster shares its centroid: computed once per cluster
    std::vector<double> centroid(3 * size_t(own.nnodes));
    std::atomic<int> cursor{0};
    auto cwork = [&]() {
        for (;;) {
            const int t = cursor.fetch_add(1);
            if (t >= own.nnodes) break;
            if (own.size(t) > 0)
                cluster_centroid(ownpts, own.perm.data() + own.begin[t], own.size(t), &centroid[3 * size_t(t)]);
        }
    };
    auto work = [&]() {
        std::vector<int32_t> ff;
        for (;;) {
            const int item = cursor.fetch_add(1);
            if (item >= ni) break;
            item_farfield(own, D, item, ff);
            if (ff.empty()) continue;
            const int t = D.item_node[item];
            count[item] = select_farpivots_at(far, farpts, &centroid[3 * size_t(t)], own.size(t), ff.data(),
                                              int(ff.size()), maxrank, buf.data() + size_t(item) * maxrank);
        }
    };
    const int nth = std::max(1, std::min(host_threads(), ni));
    auto run = [&](const std::function<void()> &job) {
        cursor = 0;
        std::vector<std::thread> pool;
        for (int i = 1; i < nth; ++i) pool.emplace_back(job);
        job();
        for (auto &th : pool) th.join();
    };
    run(cwork);
    run(work);
    fpptr.assign(ni + 1, 0);
    for (int i = 0; i < ni; ++i) fpptr[i + 1] = fpptr[i] + count[i];
    fpidx.resize(fpptr[ni]);
    for (int i = 0; i < ni; ++i)
        std::copy(buf.begin() + size_t(i) * maxrank, buf.begin() + size_t(i) * maxrank + count[i],
                  fpidx.begin() + fpptr[i]);
}

}  // namespace nca
