// Host-planner helpers against their direct definitions (built and run by
// tests/test_host_helpers.py with g++; no GPU):
//   * stable_order_by_key equals std::stable_sort with a key comparison,
//     including unsorted inputs, keys outside the counting range and keys
//     far larger than the list;
//   * Plan::target_parents equals the per-level parent indices, and the
//     target-leaf lists of Plan::build_target_lists equal their definition
//     (per target leaf: the far sources of the leaf and of each ancestor,
//     leaf first, each group with sources ascending; then its near source
//     leaves ascending), for equal and distinct point sets; the array form
//     of target_list_work gives the host form's sums and checksum.
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

static int check_target_lists(bool distinct)
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
    P.build_target_lists(-1);
    const Tree& T = P.tgt;
    int bad = 0;
    const std::vector<int> par = P.target_parents();
    for (int l = 0; l < T.num_levels(); l++)
        for (size_t b = 0; b < T.levels[l].size(); b++)
        {
            const int want = l == 0 ? -1 : (int)(T.level_off[l - 1] + T.levels[l].parent[b]);
            if (par[T.level_off[l] + (int64_t)b] != want)
                bad++;
        }
    if (bad)
        std::printf("target_parents differs at %d boxes (distinct %d)\n", bad, (int)distinct);
    // per target box, its far and near sources ascending (the transposes)
    const int64_t ntb = T.num_boxes_total();
    std::vector<std::vector<int>> fin((size_t)ntb), nin((size_t)ntb);
    for (int64_t s = 0; s < P.src.num_boxes_total(); s++)
    {
        for (const int32_t* t = P.far.begin(s); t != P.far.end(s); t++)
            fin[*t].push_back((int)s);
        for (const int32_t* t = P.near.begin(s); t != P.near.end(s); t++)
            nin[*t].push_back((int)s);
    }
    std::vector<long long> fo{0}, no{0};
    std::vector<int> fs, ns;
    for (size_t i = 0; i < P.tleaf_gid.size(); i++)
    {
        for (int a = (int)P.tleaf_gid[i]; a >= 0; a = par[a])
            fs.insert(fs.end(), fin[a].begin(), fin[a].end());
        ns.insert(ns.end(), nin[P.tleaf_gid[i]].begin(), nin[P.tleaf_gid[i]].end());
        fo.push_back((long long)fs.size());
        no.push_back((long long)ns.size());
    }
    const bool same = fo.size() == P.tleaf_far_off.size() &&
                      std::equal(fo.begin(), fo.end(), P.tleaf_far_off.begin()) &&
                      std::equal(no.begin(), no.end(), P.tleaf_near_off.begin()) &&
                      fs.size() == P.tleaf_far_src.size() &&
                      std::equal(fs.begin(), fs.end(), P.tleaf_far_src.begin()) &&
                      ns.size() == P.tleaf_near_src.size() &&
                      std::equal(ns.begin(), ns.end(), P.tleaf_near_src.begin());
    if (!same)
    {
        std::printf("target-leaf lists differ from their definition (distinct %d)\n",
                    (int)distinct);
        bad++;
    }
    int64_t w0[4], w1[4];
    uint64_t h0 = 0, h1 = 1;
    P.target_list_work(w0, &h0);
    P.target_list_work(fo, fs, no, ns, w1, &h1);
    if (!std::equal(w0, w0 + 4, w1) || h0 != h1)
    {
        std::printf("target_list_work forms differ (distinct %d)\n", (int)distinct);
        bad++;
    }
    if (fs.empty() || ns.empty())
    {
        std::printf("empty lists (distinct %d): the case tests nothing\n", (int)distinct);
        bad++;
    }
    return bad;
}

int main()
{
    const int bad = check_stable_order() + check_target_lists(false) + check_target_lists(true);
    std::printf(bad ? "FAILED\n" : "OK\n");
    return bad ? 1 : 0;
}
