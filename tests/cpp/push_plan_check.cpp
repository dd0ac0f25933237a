// Invariants of the slab-partitioned push solve plan (fm_setup.cpp
// push_plan), checked on the host for a mesh given as argv:
//   push_plan_check N seed clusters cluster [block [max_slots]]
// builds the N^3 unit cube (seed > 0: node ids randomly relabelled; seed
// < 0: relabelled inside blocks of 8 consecutive ids) and checks, for both
// directions:
//   * a refused plan only where some node has more than 16 neighbours on
//     one side;
//   * the position ranges of the CTAs tile the orders; each CTA's range lists
//     exactly the nodes push_cta assigns it plus holes, with non-decreasing
//     dependency level (so every warp meets a node only after all nodes it
//     waits on are reachable); the range has even length and positions 2i,
//     2i + 1 (resolved together by one warp) are never two nodes of
//     different levels; no CTA holds more than max_level_share nodes of one
//     level;
//   * every neighbour entry on the solve's side reads from a slot exactly
//     when the neighbour is in the reader's slab; that slot lies inside the
//     reader CTA's slot count, holds only that neighbour, and the
//     neighbour's push list names it (reader rank, slot);
//   * every push list entry is read by some entry, lists are terminated
//     by ~0u and hold no duplicates; entries off the solve's side are ~0u
//     for the side's own walk;
//   * the kernels' schedule cannot deadlock: with W warps per CTA, warp w
//     resolves positions (2w + qH, 2w + 1 + qH), H = 2W, q = 0, 1, ... of
//     its CTA in order, a pair only once every dependency of both nodes is
//     resolved; simulated to a fixpoint for several W, every node resolves.
// Prints "ok" and exits 0, or names the first violation and exits 1.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <set>
#include <vector>

#include "fm_setup.hpp"

using namespace fm;

static int fail(const char* what, long a, long b) {
    std::printf("violation: %s (%ld, %ld)\n", what, a, b);
    return 1;
}

int main(int argc, char** argv) {
    const int N = argc > 1 ? std::atoi(argv[1]) : 8;
    const int seed = argc > 2 ? std::atoi(argv[2]) : 0;
    const uint32_t ncl = argc > 3 ? (uint32_t)std::atoi(argv[3]) : 16;
    const uint32_t cs = argc > 4 ? (uint32_t)std::atoi(argv[4]) : 8;
    const uint32_t block = argc > 5 ? (uint32_t)std::atoi(argv[5]) : 0;
    const uint32_t max_slots = argc > 6 ? (uint32_t)std::atoi(argv[6]) : (1u << 20);
    const uint32_t nn = (N + 1) * (N + 1) * (N + 1), ne = 6 * N * N * N;
    std::vector<double> xyz(3 * (size_t)nn);
    std::vector<uint32_t> conn(4 * (size_t)ne);
    unit_cube(N, xyz.data(), conn.data());
    if (seed) {
        std::vector<uint32_t> perm(nn);
        for (uint32_t i = 0; i < nn; ++i) perm[i] = i;
        std::mt19937 rng((unsigned)std::abs(seed));
        if (seed > 0)
            std::shuffle(perm.begin(), perm.end(), rng);
        else
            for (uint32_t b = 0; b < nn; b += 8)
                std::shuffle(perm.begin() + b, perm.begin() + std::min(nn, b + 8), rng);
        for (auto& v : conn) v = perm[v];
    }
    const NodeGraph g = build_node_graph(nn, ne, conn.data());
    std::vector<uint32_t> fp, fo, bp, bo;
    node_levels(g, true, fp, fo);
    node_levels(g, false, bp, bo);
    PushPlan P;
    if (!push_plan(g, fp, fo, bp, bo, ncl, cs, block, max_slots, P)) {
        uint32_t side = 0;
        for (uint32_t n = 0; n < nn; ++n) {
            uint32_t lo = 0, hi = 0;
            for (uint32_t k = g.ptr[n]; k < g.ptr[n + 1]; ++k) {
                lo += g.nbr[k] < n;
                hi += g.nbr[k] > n;
            }
            side = std::max(side, std::max(lo, hi));
        }
        if (side > 16) {
            std::printf("ok\n");  // refused as documented
            return 0;
        }
        return fail("plan refused", ncl, cs);
    }
    const uint32_t nc = ncl * cs;
    if (P.n_ctas != nc || P.cluster != cs || P.pos_f.size() != nc + 1 ||
        P.pos_b.size() != nc + 1 || !P.block || (block && P.block != block))
        return fail("plan shape", P.n_ctas, P.block);
    std::vector<uint32_t> cta(nn);
    for (uint32_t n = 0; n < nn; ++n) {
        cta[n] = push_cta(n, nn, ncl, cs, P.block);
        if (cta[n] >= nc) return fail("CTA out of range", n, cta[n]);
        const uint32_t sl = cta[n] / cs;
        if (n < push_slab_begin(sl, nn, ncl) || n >= push_slab_begin(sl + 1, nn, ncl))
            return fail("node outside its slab", n, sl);
    }
    for (int lower = 1; lower >= 0; --lower) {
        const std::vector<uint32_t>& lp = lower ? fp : bp;
        const std::vector<uint32_t>& lo = lower ? fo : bo;
        std::vector<uint32_t> level(nn);
        for (uint32_t l = 0; l + 1 < lp.size(); ++l)
            for (uint32_t t = lp[l]; t < lp[l + 1]; ++t) level[lo[t]] = l;
        const std::vector<uint32_t>& ord = lower ? P.order_f : P.order_b;
        const std::vector<uint32_t>& pos = lower ? P.pos_f : P.pos_b;
        if (pos[0] != 0 || pos[nc] != ord.size()) return fail("position range ends", 0, lower);
        const std::vector<uint32_t>& push = lower ? P.push_f : P.push_b;
        const std::vector<uint32_t>& nslot = lower ? P.nslot_f : P.nslot_b;
        const uint32_t max_slot = lower ? P.max_slot_f : P.max_slot_b;
        if (ord.size() < nn || push.size() != (size_t)nn * kPushMax || nslot.size() != nc)
            return fail("array sizes", lower, 0);
        if (max_slot > max_slots) return fail("slots above the limit", max_slot, max_slots);
        std::vector<uint32_t> seen(nn, 0);
        for (uint32_t c = 0; c < nc; ++c) {
            if (nslot[c] > max_slot) return fail("slot count above max", c, nslot[c]);
            if (pos[c] > pos[c + 1] || ((pos[c + 1] - pos[c]) & 1))
                return fail("position range decreasing or odd", c, 0);
            uint32_t run = 0;
            long prev = -1;  // last node of the range so far
            for (uint32_t t = pos[c]; t < pos[c + 1]; ++t) {
                const uint32_t n = ord[t];
                if (((t - pos[c]) & 1) && n != ~0u && ord[t - 1] != ~0u &&
                    level[n] != level[ord[t - 1]])
                    return fail("a warp's pair spans two levels", c, t);
                if (n == ~0u) continue;
                if (n >= nn || cta[n] != c) return fail("node in foreign CTA", c, t);
                if (seen[n]++) return fail("node listed twice", c, n);
                if (prev >= 0 && level[n] < level[prev]) return fail("CTA order not by level", c, t);
                run = prev >= 0 && level[n] == level[prev] ? run + 1 : 1;
                if (run > P.max_level_share) return fail("level share above max", c, t);
                prev = n;
            }
        }
        // (reader CTA, slot) -> producer; push entries actually read
        std::vector<std::vector<long>> owner(nc);
        for (uint32_t c = 0; c < nc; ++c) owner[c].assign(nslot[c], -1);
        std::set<std::pair<uint32_t, uint32_t>> used;  // (producer, entry)
        for (uint32_t n = 0; n < nn; ++n) {
            if (seen[n] != 1) return fail("node missing from the orders", n, lower);
            const uint32_t c = cta[n], slab = c / cs;
            for (uint32_t k = g.ptr[n]; k < g.ptr[n + 1]; ++k) {
                const uint32_t m = g.nbr[k];
                if (m == n) {
                    if (P.src[k] != ~0u) return fail("self entry has a slot", n, k);
                    continue;
                }
                if ((m < n) != (lower != 0)) continue;
                if (level[m] >= level[n]) return fail("dependency not at an earlier level", n, m);
                const bool same = cta[m] / cs == slab;
                const uint32_t sl = P.src[k];
                if (!same) {
                    if (sl != ~0u) return fail("cross-slab entry has a slot", n, m);
                    continue;
                }
                if (sl == ~0u || sl >= nslot[c]) return fail("slot missing or out of range", n, m);
                if (owner[c][sl] != -1 && owner[c][sl] != (long)m)
                    return fail("slot shared by two producers", c, sl);
                owner[c][sl] = m;
                const uint32_t want = (c % cs) << 20 | sl;
                bool found = false;
                for (uint32_t j = 0; j < kPushMax; ++j)
                    if (push[(size_t)m * kPushMax + j] == want) {
                        found = true;
                        used.insert({m, j});
                    }
                if (!found) return fail("producer does not push to its reader", m, n);
            }
        }
        // schedule simulation: every warp advances while its next pair is ready
        for (uint32_t W : {1u, 3u, 16u, 24u}) {
            const uint32_t H = 2 * W;
            std::vector<uint8_t> done(nn, 0);
            std::vector<uint32_t> q((size_t)nc * W, 0);
            auto ready = [&](uint32_t t) {
                const uint32_t n = ord[t];
                if (n == ~0u) return true;
                for (uint32_t k = g.ptr[n]; k < g.ptr[n + 1]; ++k) {
                    const uint32_t m = g.nbr[k];
                    if (m != n && (m < n) == (lower != 0) && !done[m]) return false;
                }
                return true;
            };
            uint32_t resolved = 0;
            for (bool moved = true; moved;) {
                moved = false;
                for (uint32_t c = 0; c < nc; ++c)
                    for (uint32_t w = 0; w < W; ++w) {
                        uint32_t& qq = q[(size_t)c * W + w];
                        for (;;) {
                            const uint32_t t = pos[c] + 2 * w + qq * H;
                            if (t >= pos[c + 1]) break;
                            if (!ready(t) || !ready(t + 1)) break;
                            for (uint32_t u : {t, t + 1})
                                if (ord[u] != ~0u) {
                                    done[ord[u]] = 1;
                                    ++resolved;
                                }
                            ++qq;
                            moved = true;
                        }
                    }
            }
            if (resolved != nn) return fail("schedule deadlocks", W, resolved);
        }
        for (uint32_t m = 0; m < nn; ++m) {
            bool ended = false;
            std::set<uint32_t> ents;
            for (uint32_t j = 0; j < kPushMax; ++j) {
                const uint32_t pe = push[(size_t)m * kPushMax + j];
                if (pe == ~0u) {
                    ended = true;
                    continue;
                }
                if (ended) return fail("push entry after the terminator", m, j);
                if ((pe >> 20) >= cs) return fail("push rank out of range", m, pe >> 20);
                if (!ents.insert(pe).second) return fail("duplicate push entry", m, j);
                if (!used.count({m, j})) return fail("push entry nobody reads", m, j);
            }
        }
    }
    std::printf("ok\n");
    return 0;
}
