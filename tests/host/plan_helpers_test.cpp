// Host-planner helpers against their direct definitions (built and run by
// tests/test_host_helpers.py with g++; no GPU):
//   * stable_order_by_key equals std::stable_sort with a key comparison,
//     including unsorted inputs, keys outside the counting range and keys
//     far larger than the list;
//   * Plan::far_pairs_of_level equals a per-pair search of the target box's
//     level and point range, for equal and distinct point sets.
#include "plan.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

using namespace ifgf;

static int check_stable_order()
{
    std::mt19937 rng(3);
    int bad = 0;
    for (int trial = 0; trial < 60; trial++)
    {
        const int n = trial < 40 ? (int)(rng() % 3000) : 50000 + (int)(rng() % 50000);
        const int nk = 1 + (int)(rng() % (trial % 3 == 0 ? 4 : 5000));
        std::vector<int> key(n + 7);
        for (auto& k : key)
            k = (int)(rng() % nk);
        if (trial == 5)
            key[0] = -3; // a negative key: the comparison-sort path
        if (trial == 6)
            key[1] = 1 << 27; // a key beyond the counting range
        if (trial == 7 || trial == 8)
            key[2] = (1 << 25) + trial; // one large key over a short list: the comparison sort
        std::vector<int> idx;
        for (int i = 0; i < n + 7; i++)
            if (rng() % 3)
                idx.push_back(i);
        if (trial % 4 == 1)
            std::shuffle(idx.begin(), idx.end(), rng);
        std::vector<int> a = idx, b = idx;
        std::stable_sort(a.begin(), a.end(), [&](int x, int y) { return key[x] < key[y]; });
        stable_order_by_key(b, key);
        if (a != b)
        {
            std::printf("stable_order_by_key differs (trial %d)\n", trial);
            bad++;
        }
    }
    return bad;
}

static std::vector<double> surface(int64_t n, double az, double scale, std::mt19937_64& rng)
{
    std::normal_distribution<double> nd;
    std::vector<double> p(3 * n);
    for (int64_t i = 0; i < n; i++)
    {
        double v[3] = {nd(rng), nd(rng), nd(rng)};
        const double s = scale / std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2] / (az * az));
        for (int d = 0; d < 3; d++)
            p[3 * i + d] = v[d] * s;
    }
    return p;
}

static int check_far_pairs(bool distinct)
{
    std::mt19937_64 rng(7);
    const int64_t n = 40000;
    std::vector<double> ps = surface(n, 0.5, 1.0, rng), pt = surface(n / 3, 1.0, 1.3, rng);
    Plan P;
    P.src.build(ps.data(), n, 60);
    if (distinct)
        P.tgt.build(pt.data(), n / 3, 30);
    else
        P.tgt = P.src;
    P.build_lists(nullptr);
    std::vector<int> tf, tl;
    P.target_box_ranges(tf, tl);
    const Tree& T = P.tgt;
    int bad = 0;
    int64_t total = 0;
    for (int l = 0; l < P.src.num_levels(); l++)
    {
        std::vector<int> fs, f0, f1;
        for (int64_t g = P.src.level_off[l]; g < P.src.level_off[l + 1]; g++)
            for (const int32_t* tp = P.far.begin(g); tp != P.far.end(g); tp++)
            {
                const int lev = (int)(std::upper_bound(T.level_off.begin(), T.level_off.end(),
                                                       (int64_t)*tp) -
                                      T.level_off.begin()) - 1;
                const int64_t b = *tp - T.level_off[lev];
                fs.push_back((int)g);
                f0.push_back((int)T.levels[lev].first[b]);
                f1.push_back((int)T.levels[lev].last[b]);
            }
        std::vector<int> a, b, c;
        P.far_pairs_of_level(l, tf, tl, a, b, c);
        if (a != fs || b != f0 || c != f1)
        {
            std::printf("far_pairs_of_level differs at level %d (distinct %d)\n", l, (int)distinct);
            bad++;
        }
        total += (int64_t)fs.size();
    }
    if (total == 0)
    {
        std::printf("no far pairs (distinct %d): the case tests nothing\n", (int)distinct);
        bad++;
    }
    return bad;
}

int main()
{
    const int bad = check_stable_order() + check_far_pairs(false) + check_far_pairs(true);
    std::printf(bad ? "FAILED\n" : "OK\n");
    return bad ? 1 : 0;
}
