// Randomised check of the banded, vectorised nearest-direction search against the full
// one-at-a-time search (and of the four- and eight-wide scans over all candidates against it): the
// candidate sets of candidate_directions for cluster diameters 0.01-3 and wavenumbers 1-120
// (6 to ~680,000 spherical Fibonacci points), queried with Gaussian directions of magnitudes
// 1e-30 to 1e30, many of them near the poles or on the equator. Both searches must return the
// same index for every query. Built and run by tests/test_nearest_candidate.py.
#include <cstdio>
#include <cstdlib>
#include <random>

#include "directional.cpp"  // the helpers live in that file's anonymous namespace

int main(int argc, char **argv) {
    const int per_set = argc > 1 ? std::atoi(argv[1]) : 400;
    std::mt19937_64 g(7);
    std::normal_distribution<double> nd;
    std::uniform_real_distribution<double> ud(-30, 30);
    long bad = 0, total = 0;
    std::vector<double> dirs;
    nca::Candidates cand;
    const bool wide = __builtin_cpu_supports("avx512f");
    for (double diam = 0.01; diam < 3.0; diam *= 1.07) {
        for (double k : {1.0, 10.0, 50.0, 120.0}) {
            nca::candidate_directions(diam, k, 1.0, dirs);
            cand.set(dirs);
            for (int t = 0; t < per_set; ++t) {
                double v[3] = {nd(g), nd(g), nd(g)};
                if (t % 5 == 0) {  // near the poles
                    v[0] *= 1e-6;
                    v[1] *= 1e-6;
                }
                if (t % 7 == 0) v[2] = 0.0;  // on the equator
                const double scale = std::pow(10.0, ud(g));
                for (double &x : v) x *= scale;
                ++total;
                const int full = nca::nearest_direction(dirs, v);
                if (nca::nearest_candidate(cand, v) != full) ++bad;
                if (t % 3 == 0) {  // the four- and (where the host has it) eight-wide scans over all
                    if (int(nca::argmax_dot4(cand, 0, cand.n - 1, v)) != full) ++bad;
                    if (wide && int(nca::argmax_dot8(cand, 0, cand.n - 1, v)) != full) ++bad;
                }
            }
        }
    }
    std::printf("queries %ld mismatches %ld\n", total, bad);
    return bad != 0;
}
