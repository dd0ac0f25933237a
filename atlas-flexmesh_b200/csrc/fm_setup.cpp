// fm_setup.cpp — host-side integer setup (see fm_setup.hpp).
#include "fm_setup.hpp"

#include <algorithm>
#include <cstring>

namespace fm {

namespace {
// 6-tet split of a hex and its corner offsets; the tables fix the node and
// element numbering and must equal the reference's
// (FEM/adaptive_fem_engine.hpp:2240-2247).
constexpr int kCorner[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                               {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
constexpr int kTet[6][4] = {{0, 1, 3, 4}, {1, 2, 3, 6}, {1, 3, 4, 6},
                            {3, 4, 6, 7}, {1, 4, 5, 6}, {0, 3, 4, 7}};
}  // namespace

void unit_cube(int N, double* xyz, uint32_t* conn) {
    const int s = N + 1;
    const double h = 1.0 / N;
    size_t id = 0;
    for (int k = 0; k <= N; ++k)
        for (int j = 0; j <= N; ++j)
            for (int i = 0; i <= N; ++i, ++id) {
                xyz[3 * id] = i * h;
                xyz[3 * id + 1] = j * h;
                xyz[3 * id + 2] = k * h;
            }
    size_t e = 0;
    for (int k = 0; k < N; ++k)
        for (int j = 0; j < N; ++j)
            for (int i = 0; i < N; ++i) {
                uint32_t c[8];
                for (int q = 0; q < 8; ++q)
                    c[q] = (uint32_t)((k + kCorner[q][2]) * s * s + (j + kCorner[q][1]) * s +
                                      (i + kCorner[q][0]));
                for (int t = 0; t < 6; ++t, ++e)
                    for (int v = 0; v < 4; ++v) conn[4 * e + v] = c[kTet[t][v]];
            }
}

NodeGraph build_node_graph(uint32_t n_nodes, uint32_t n_elems, const uint32_t* conn) {
    NodeGraph g;
    g.n_nodes = n_nodes;
    // incident-element buckets first, then per node a small sort of the
    // union of the incident elements' vertices
    Incidence inc = build_incidence(n_nodes, n_elems, conn);
    g.ptr.assign(n_nodes + 1, 0);
    g.self.assign(n_nodes, 0);
    std::vector<uint32_t> tmp;
    g.nbr.reserve((size_t)n_nodes * 16);
    for (uint32_t n = 0; n < n_nodes; ++n) {
        tmp.clear();
        for (uint32_t k = inc.ptr[n]; k < inc.ptr[n + 1]; ++k) {
            const uint32_t* c = conn + 4 * (size_t)inc.elem[k];
            tmp.insert(tmp.end(), c, c + 4);
        }
        std::sort(tmp.begin(), tmp.end());
        tmp.erase(std::unique(tmp.begin(), tmp.end()), tmp.end());
        g.ptr[n] = (uint32_t)g.nbr.size();
        for (size_t q = 0; q < tmp.size(); ++q)
            if (tmp[q] == n) g.self[n] = (uint32_t)q;
        g.nbr.insert(g.nbr.end(), tmp.begin(), tmp.end());
        g.max_deg = std::max<uint32_t>(g.max_deg, (uint32_t)tmp.size());
    }
    g.ptr[n_nodes] = (uint32_t)g.nbr.size();
    return g;
}

Incidence build_incidence(uint32_t n_nodes, uint32_t n_elems, const uint32_t* conn) {
    Incidence inc;
    inc.ptr.assign(n_nodes + 1, 0);
    for (size_t q = 0; q < 4 * (size_t)n_elems; ++q) inc.ptr[conn[q] + 1]++;
    for (uint32_t n = 0; n < n_nodes; ++n) {
        inc.max_inc = std::max(inc.max_inc, inc.ptr[n + 1]);
        inc.ptr[n + 1] += inc.ptr[n];
    }
    inc.elem.resize(inc.ptr[n_nodes]);
    std::vector<uint32_t> fill(inc.ptr.begin(), inc.ptr.end() - 1);
    for (uint32_t e = 0; e < n_elems; ++e)
        for (int v = 0; v < 4; ++v) inc.elem[fill[conn[4 * (size_t)e + v]]++] = e;
    return inc;
}

void csr_row_ptr(const NodeGraph& g, uint32_t* row_ptr) {
    row_ptr[0] = 0;
    for (uint32_t n = 0; n < g.n_nodes; ++n) {
        uint32_t deg = g.ptr[n + 1] - g.ptr[n];
        for (int d = 0; d < 3; ++d) row_ptr[3 * n + d + 1] = row_ptr[3 * n + d] + 3 * deg;
    }
}

void csr_solve_cols(const NodeGraph& g, uint32_t* col_idx) {
    size_t w = 0;
    for (uint32_t n = 0; n < g.n_nodes; ++n)
        for (int d = 0; d < 3; ++d)
            for (uint32_t k = g.ptr[n]; k < g.ptr[n + 1]; ++k)
                for (uint32_t q = 0; q < 3; ++q) col_idx[w++] = 3 * g.nbr[k] + q;
}

void csr_reference_cols(const NodeGraph& g, uint32_t* col_idx) {
    // the reference writes, for each neighbour, 3 (d_self) x 3 (d_neigh)
    // entries consecutively, walking the node's three rows as one run
    size_t w = 0;
    for (uint32_t n = 0; n < g.n_nodes; ++n)
        for (uint32_t k = g.ptr[n]; k < g.ptr[n + 1]; ++k)
            for (int ds = 0; ds < 3; ++ds)
                for (uint32_t q = 0; q < 3; ++q) col_idx[w++] = 3 * g.nbr[k] + q;
}

void slot_map(const uint32_t* row_ptr, const uint32_t* col_idx, uint32_t n_elems,
              const uint32_t* conn, int32_t* slot) {
    for (uint32_t e = 0; e < n_elems; ++e) {
        const uint32_t* c = conn + 4 * (size_t)e;
        int32_t* s = slot + 144 * (size_t)e;
        for (int i = 0; i < 4; ++i)
            for (int di = 0; di < 3; ++di) {
                const uint32_t gi = 3 * c[i] + di;
                for (int j = 0; j < 4; ++j)
                    for (int dj = 0; dj < 3; ++dj) {
                        const uint32_t gj = 3 * c[j] + dj;
                        int32_t found = -1;
                        for (uint32_t k = row_ptr[gi]; k < row_ptr[gi + 1]; ++k)
                            if (col_idx[k] == gj) found = (int32_t)k;
                        s[(i * 3 + di) * 12 + j * 3 + dj] = found;
                    }
            }
    }
}

static uint32_t levels_from_depth(const std::vector<uint32_t>& depth, uint32_t maxd,
                                  std::vector<uint32_t>& ptr, std::vector<uint32_t>& rows) {
    const uint32_t n = (uint32_t)depth.size();
    const uint32_t nl = n ? maxd + 1 : 0;
    ptr.assign(nl + 1, 0);
    for (uint32_t i = 0; i < n; ++i) ptr[depth[i] + 1]++;
    for (uint32_t l = 0; l < nl; ++l) ptr[l + 1] += ptr[l];
    rows.resize(n);
    std::vector<uint32_t> fill(ptr.begin(), ptr.end() - (nl ? 1 : 0));
    for (uint32_t i = 0; i < n; ++i) rows[fill[depth[i]]++] = i;
    return nl;
}

uint32_t csr_levels(uint32_t n, const uint32_t* row_ptr, const uint32_t* col_idx, bool lower,
                    std::vector<uint32_t>& ptr, std::vector<uint32_t>& rows) {
    std::vector<uint32_t> depth(n, 0);
    uint32_t maxd = 0;
    for (uint32_t t = 0; t < n; ++t) {
        const uint32_t i = lower ? t : n - 1 - t;
        uint32_t d = 0;
        for (uint32_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k) {
            const uint32_t c = col_idx[k];
            if (lower ? c < i : c > i) d = std::max(d, depth[c] + 1);
        }
        depth[i] = d;
        maxd = std::max(maxd, d);
    }
    return levels_from_depth(depth, maxd, ptr, rows);
}

bool push_plan(const NodeGraph& g, const std::vector<uint32_t>& fwd_ptr,
               const std::vector<uint32_t>& fwd_order, const std::vector<uint32_t>& bwd_ptr,
               const std::vector<uint32_t>& bwd_order, uint32_t n_clusters, uint32_t cluster,
               uint32_t block, uint32_t max_slots, PushPlan& plan) {
    const uint32_t nn = g.n_nodes;
    plan = PushPlan();
    if (!nn || !n_clusters || !cluster || cluster > kPushMax || fwd_order.size() != nn ||
        bwd_order.size() != nn || fwd_ptr.size() < 2 || bwd_ptr.size() < 2)
        return false;
    const uint32_t nc = n_clusters * cluster;
    max_slots = std::min(max_slots, 1u << 20);
    // Every node read inside its own slab takes at least one slot in some
    // CTA of the slab, so a slab with more such nodes than cluster *
    // max_slots cannot fit with any block size: refuse before the search.
    for (int lower = 1; lower >= 0; --lower) {
        for (uint32_t s = 0; s < n_clusters; ++s) {
            const uint32_t b = push_slab_begin(s, nn, n_clusters);
            const uint32_t e = push_slab_begin(s + 1, nn, n_clusters);
            uint64_t read = 0;
            for (uint32_t m = b; m < e; ++m)
                for (uint32_t k = g.ptr[m]; k < g.ptr[m + 1]; ++k) {
                    const uint32_t n = g.nbr[k];  // a reader of m on this side?
                    if (n >= b && n < e && (lower ? n > m : n < m)) {
                        ++read;
                        break;
                    }
                }
            if (read > (uint64_t)cluster * max_slots) return false;
        }
    }
    const uint32_t nlf = (uint32_t)fwd_ptr.size() - 1, nlb = (uint32_t)bwd_ptr.size() - 1;
    std::vector<uint32_t> lf(nn), lb(nn);
    for (uint32_t l = 0; l < nlf; ++l)
        for (uint32_t t = fwd_ptr[l]; t < fwd_ptr[l + 1]; ++t) lf[fwd_order[t]] = l;
    for (uint32_t l = 0; l < nlb; ++l)
        for (uint32_t t = bwd_ptr[l]; t < bwd_ptr[l + 1]; ++t) lb[bwd_order[t]] = l;
    // busiest CTA's share of one level, either direction
    std::vector<uint32_t> cf((size_t)nc * nlf), cb((size_t)nc * nlb);
    auto share = [&](uint32_t R) {
        std::fill(cf.begin(), cf.end(), 0u);
        std::fill(cb.begin(), cb.end(), 0u);
        uint32_t mx = 0;
        for (uint32_t n = 0; n < nn; ++n) {
            const uint32_t c = push_cta(n, nn, n_clusters, cluster, R);
            mx = std::max(mx, ++cf[(size_t)c * nlf + lf[n]]);
            mx = std::max(mx, ++cb[(size_t)c * nlb + lb[n]]);
        }
        return mx;
    };
    std::vector<std::pair<uint32_t, uint32_t>> cand;  // (share, block)
    if (block) {
        cand.push_back({share(block), block});
    } else {
        for (uint32_t R = 16; R <= 512; R += R < 128 ? 1 : 8) cand.push_back({share(R), R});
        std::sort(cand.begin(), cand.end());
    }
    std::vector<uint32_t> cta(nn);
    auto slots = [&](bool lower, std::vector<uint32_t>& push, std::vector<uint32_t>& nslot,
                     uint32_t& max_slot) {
        push.assign((size_t)nn * kPushMax, ~0u);
        nslot.assign(nc, 0);
        std::vector<uint8_t> npush(nn, 0);
        for (uint32_t s = 0; s < n_clusters; ++s) {
            const uint32_t b = push_slab_begin(s, nn, n_clusters);
            const uint32_t e = push_slab_begin(s + 1, nn, n_clusters);
            // slot of producer m in the slab's CTA of rank r: slot[(m - b) * cluster + r]
            std::vector<uint32_t> slot((size_t)(e - b) * cluster, ~0u);
            for (uint32_t n = b; n < e; ++n) {
                const uint32_t c = cta[n], r = c - s * cluster;
                uint32_t cnt = 0;
                for (uint32_t k = g.ptr[n]; k < g.ptr[n + 1]; ++k) {
                    const uint32_t m = g.nbr[k];
                    if (m == n || (m < n) != lower) continue;
                    ++cnt;
                    if (m < b || m >= e) continue;  // another slab: through global memory
                    uint32_t& sl = slot[(size_t)(m - b) * cluster + r];
                    if (sl == ~0u) {
                        sl = nslot[c]++;
                        if (sl >= max_slots) return false;
                        push[(size_t)m * kPushMax + npush[m]++] = r << 20 | sl;
                    }
                    plan.src[k] = sl;
                }
                if (cnt > 16) return false;
            }
        }
        max_slot = *std::max_element(nslot.begin(), nslot.end());
        return true;
    };
    for (const auto& cs : cand) {
        const uint32_t R = cs.second;
        for (uint32_t n = 0; n < nn; ++n) cta[n] = push_cta(n, nn, n_clusters, cluster, R);
        plan.src.assign(g.nbr.size(), ~0u);
        if (!slots(true, plan.push_f, plan.nslot_f, plan.max_slot_f) ||
            !slots(false, plan.push_b, plan.nslot_b, plan.max_slot_b))
            continue;
        plan.n_ctas = nc;
        plan.cluster = cluster;
        plan.block = R;
        plan.max_level_share = cs.first;
        // each CTA's nodes keep the relative order of the global level order;
        // a level that would start at an odd position of its CTA gets a hole first
        auto split = [&](const std::vector<uint32_t>& order, const std::vector<uint32_t>& lev,
                         std::vector<uint32_t>& pos, std::vector<uint32_t>& out) {
            std::vector<std::vector<uint32_t>> per(nc);
            for (uint32_t n : order) {
                std::vector<uint32_t>& v = per[cta[n]];
                if ((v.size() & 1) && lev[v.back()] != lev[n]) v.push_back(~0u);
                v.push_back(n);
            }
            pos.assign(nc + 1, 0);
            out.clear();
            for (uint32_t c = 0; c < nc; ++c) {
                if (per[c].size() & 1) per[c].push_back(~0u);
                out.insert(out.end(), per[c].begin(), per[c].end());
                pos[c + 1] = (uint32_t)out.size();
            }
        };
        split(fwd_order, lf, plan.pos_f, plan.order_f);
        split(bwd_order, lb, plan.pos_b, plan.order_b);
        return true;
    }
    plan = PushPlan();
    return false;
}

void ilu_edge_maps(const NodeGraph& g, std::vector<uint32_t>& ptr, std::vector<uint8_t>& map) {
    const uint32_t n = g.n_nodes;
    ptr.assign(n + 1, 0);
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t c = 0;
        for (uint32_t k = g.ptr[i]; k < g.ptr[i] + g.self[i]; ++k) {
            const uint32_t m = g.nbr[k];
            c += (g.ptr[m + 1] - g.ptr[m]) - g.self[m];
        }
        ptr[i + 1] = ptr[i] + c;
    }
    map.assign(ptr[n], 0xff);
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t* ni = g.nbr.data() + g.ptr[i];
        const uint32_t di = g.ptr[i + 1] - g.ptr[i];
        uint32_t o = ptr[i];
        for (uint32_t k = 0; k < g.self[i]; ++k) {
            const uint32_t m = ni[k];
            for (uint32_t q = g.ptr[m] + g.self[m]; q < g.ptr[m + 1]; ++q, ++o) {
                const uint32_t* hit = std::lower_bound(ni, ni + di, g.nbr[q]);
                if (hit != ni + di && *hit == g.nbr[q]) map[o] = (uint8_t)(hit - ni);
            }
        }
    }
}

uint32_t node_levels(const NodeGraph& g, bool lower, std::vector<uint32_t>& ptr,
                     std::vector<uint32_t>& order) {
    const uint32_t n = g.n_nodes;
    std::vector<uint32_t> depth(n, 0);
    uint32_t maxd = 0;
    for (uint32_t t = 0; t < n; ++t) {
        const uint32_t i = lower ? t : n - 1 - t;
        uint32_t d = 0;
        for (uint32_t k = g.ptr[i]; k < g.ptr[i + 1]; ++k) {
            const uint32_t c = g.nbr[k];
            if (lower ? c < i : c > i) d = std::max(d, depth[c] + 1);
        }
        depth[i] = d;
        maxd = std::max(maxd, d);
    }
    return levels_from_depth(depth, maxd, ptr, order);
}

}  // namespace fm
