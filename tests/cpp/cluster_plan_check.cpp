// Invariants of the cluster-synchronous solve plan (fm_setup.cpp
// cluster_plan), checked on the host for a mesh given as argv:
//   cluster_plan_check N [seed]
// builds the N^3 unit cube (seed != 0: node ids randomly relabelled, which
// gives irregular levels and long-lived values) and, for both directions:
//   * every node appears at exactly one position, with a record that
//     matches its neighbour list;
//   * every neighbour a node reads on the solve's side sits at an earlier
//     level, and its slot is the one recorded for that neighbour entry;
//   * a slot is handed out again only from the second window after the
//     window of its last read, and each retirement is listed once in the
//     reset list of that window and the slot's CTA;
//   * slots stay inside their CTA's pool and belong to the writer's CTA;
// and the ILU(0) update map (ilu_edge_maps) against a direct search.
// Prints "ok" and exits 0, or names the first violation and exits 1.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <random>
#include <vector>

#include "fm_setup.hpp"

using namespace fm;

static int fail(const char* what, long a, long b) {
    std::printf("violation: %s (%ld, %ld)\n", what, a, b);
    return 1;
}

int main(int argc, char** argv) {
    const int N = argc > 1 ? std::atoi(argv[1]) : 8;
    const unsigned seed = argc > 2 ? (unsigned)std::atoi(argv[2]) : 0;
    const uint32_t nn = (N + 1) * (N + 1) * (N + 1), ne = 6 * N * N * N;
    std::vector<double> xyz(3 * (size_t)nn);
    std::vector<uint32_t> conn(4 * (size_t)ne);
    unit_cube(N, xyz.data(), conn.data());
    if (seed) {
        std::vector<uint32_t> perm(nn);
        for (uint32_t i = 0; i < nn; ++i) perm[i] = i;
        std::mt19937 rng(seed);
        std::shuffle(perm.begin(), perm.end(), rng);
        for (auto& v : conn) v = perm[v];
    }
    const NodeGraph g = build_node_graph(nn, ne, conn.data());
    for (int lower = 1; lower >= 0; --lower) {
        std::vector<uint32_t> ptr, order;
        node_levels(g, lower != 0, ptr, order);
        for (int lanes = 0; lanes < 2; ++lanes)
        for (uint32_t cs : {8u, 16u})
        for (uint32_t win : {1u, 8u}) {
            const uint32_t wpc = lanes ? 6 : 32, W = cs * wpc;
            ClusterPlan P;
            std::vector<uint32_t> nslot;
            if (!cluster_plan(g, lower != 0, ptr, order, cs, wpc, win, 1u << 16, P, nslot,
                              lanes != 0))
                return fail("plan refused", cs, lower);
            std::vector<long> level(nn, -1), slot(nn, -1), last(nn, -1);
            for (uint32_t l = 0; l < P.n_levels; ++l)
                for (uint32_t p = P.lvl_ptr[l]; p < P.lvl_ptr[l + 1]; ++p) {
                    const uint32_t* r = &P.rec[4 * (size_t)p];
                    const uint32_t n = r[0];
                    if (n >= nn || level[n] >= 0) return fail("position", p, n);
                    level[n] = l;
                    const uint32_t deg = r[2] & 0xff, sk = (r[2] >> 8) & 0xff, cnt = r[2] >> 16;
                    if (r[1] != g.ptr[n] || deg != g.ptr[n + 1] - g.ptr[n] || sk != g.self[n] ||
                        cnt != (lower ? sk : deg - sk - 1))
                        return fail("record", p, n);
                    const uint32_t i = p - P.lvl_ptr[l];
                    const uint32_t warp = lanes ? (P.lvl_gptr[l] + i / 32) % W : i % W;
                    const uint32_t cta = warp / wpc;
                    if (r[3] >= P.slots_per_cta) return fail("slot range", p, r[3]);
                    slot[n] = (long)((cta << 16) | r[3]);
                }
            for (uint32_t n = 0; n < nn; ++n)
                if (level[n] < 0) return fail("missing node", n, 0);
            // readers: dependency levels and recorded slots
            for (uint32_t n = 0; n < nn; ++n)
                for (uint32_t k = g.ptr[n]; k < g.ptr[n + 1]; ++k) {
                    const uint32_t m = g.nbr[k];
                    if (lower ? m < n : m > n) {
                        if (level[m] >= level[n]) return fail("level order", n, m);
                        if ((long)nslot[k] != slot[m]) return fail("neighbour slot", n, m);
                        last[m] = std::max(last[m], level[n]);
                    }
                }
            // per slot, lifetimes [level, last read] of successive writers
            std::map<long, std::vector<std::pair<long, long>>> life;
            for (uint32_t n = 0; n < nn; ++n)
                life[slot[n]].push_back({level[n], std::max(last[n], level[n])});
            std::map<std::pair<long, long>, int> retired;  // (slot, window) -> count
            for (auto& kv : life) {
                auto& v = kv.second;
                std::sort(v.begin(), v.end());
                for (size_t i = 0; i < v.size(); ++i) {
                    retired[{kv.first, v[i].second / win}]++;
                    if (i > 0 && v[i].first / win < v[i - 1].second / win + 2)
                        return fail("slot reuse", kv.first, (long)i);
                }
            }
            const long n_win = ((long)P.n_levels + win - 1) / win;
            if ((long)P.reset_ptr.size() != n_win * cs + 1) return fail("reset ptr", n_win, cs);
            long listed = 0;
            for (long t = 0; t < n_win; ++t)
                for (uint32_t c = 0; c < cs; ++c)
                    for (uint32_t i = P.reset_ptr[t * cs + c]; i < P.reset_ptr[t * cs + c + 1]; ++i) {
                        auto it = retired.find({(long)((c << 16) | P.reset[i]), t});
                        if (it == retired.end() || it->second <= 0) return fail("reset entry", t, c);
                        it->second--;
                        ++listed;
                    }
            if (listed != (long)nn) return fail("reset count", listed, nn);
            if (lanes) {
                // lane groups: ceil(width / 32) per level, numbered consecutively
                uint32_t gsum = 0;
                for (uint32_t l = 0; l < P.n_levels; ++l) {
                    if (P.lvl_gptr[l] != gsum) return fail("group ptr", l, gsum);
                    gsum += (P.lvl_ptr[l + 1] - P.lvl_ptr[l] + 31) / 32;
                }
                if (P.lvl_gptr[P.n_levels] != gsum || P.n_groups != gsum)
                    return fail("group count", gsum, P.n_groups);
                continue;
            }
            // cards: a bijection onto [0, nn) that keeps each level's cards in
            // the level's range and each warp's cards of a level consecutive
            std::vector<uint32_t> card;
            cluster_card_index(P.lvl_ptr, W, card);
            std::vector<char> seen(nn, 0);
            for (uint32_t l = 0; l < P.n_levels; ++l)
                for (uint32_t p = P.lvl_ptr[l]; p < P.lvl_ptr[l + 1]; ++p) {
                    const uint32_t c = card[p];
                    if (c < P.lvl_ptr[l] || c >= P.lvl_ptr[l + 1] || seen[c]) return fail("card", p, c);
                    seen[c] = 1;
                    const uint32_t i = p - P.lvl_ptr[l];
                    if (i >= W && card[p - W] + 1 != c) return fail("card order", p, c);
                }
        }
    }
    // ILU(0) update map: for node i and lower neighbour m, entry t names the
    // position in i's list of m's neighbour self(m) + t, or 0xff
    {
        std::vector<uint32_t> eptr;
        std::vector<uint8_t> emap;
        ilu_edge_maps(g, eptr, emap);
        if (eptr.size() != nn + 1 || emap.size() != eptr[nn]) return fail("edge map size", 0, 0);
        for (uint32_t i = 0; i < nn; ++i) {
            uint32_t o = eptr[i];
            for (uint32_t k = g.ptr[i]; k < g.ptr[i] + g.self[i]; ++k) {
                const uint32_t m = g.nbr[k];
                for (uint32_t q = g.ptr[m] + g.self[m]; q < g.ptr[m + 1]; ++q, ++o) {
                    uint32_t want = 0xff;
                    for (uint32_t r = g.ptr[i]; r < g.ptr[i + 1]; ++r)
                        if (g.nbr[r] == g.nbr[q]) want = r - g.ptr[i];
                    if (emap[o] != want) return fail("edge map entry", i, o);
                }
            }
            if (o != eptr[i + 1]) return fail("edge map extent", i, o);
        }
    }
    std::printf("ok\n");
    return 0;
}
