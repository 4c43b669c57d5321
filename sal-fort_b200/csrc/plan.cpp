// Flattening of a tree and its interaction lists into the device work plan.
//
// The device never walks the tree.  Every solve is four data-parallel passes
// over flat arrays built here once per grid:
//   upward   : per (source slot, chunk) unit, proxy weights W from the slot
//              panel's points (fast_sum_module.f90:99-111,
//              mom6_fast_sum_module.f90:33-74);
//   proxy    : per target slot, proxy potentials at the target panel's
//              Chebyshev nodes from CP sources (points) and CC sources
//              (proxies) (fast_sum_module.f90:172-183, :254-271);
//   leaf     : per leaf, PP sources (points) and PC sources (proxies) of the
//              leaf and all its ancestors, plus one DOWN item per ancestor
//              target slot that interpolates the proxy potentials
//              (fast_sum_module.f90:58-72, :113-129, :185-199).
// All sources live in one pool of (x, y, z, w) records: the n points in
// leaf-contiguous order, then (d+1)^2 proxies per source slot, so every item
// is a contiguous pool range the kernels stage with one bulk copy.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <string>
#include <unordered_map>
#include <vector>

#include "sal_internal.hpp"

namespace sal {

static constexpr int kUpChunk = 4096;          // points per upward unit
static constexpr double kProxyUnitPairs = 81.0 * 8192.0;  // pair budget of one proxy work unit (FP64 pass)

static void panel_proxies(const Panel &q, int d, double *xyz, double *nodes, double *box) {
    int n = d + 1;
    double cx[kMaxDegree + 1], ce[kMaxDegree + 1];
    cheb_nodes(q.min_xi, q.max_xi, d, cx);
    cheb_nodes(q.min_eta, q.max_eta, d, ce);
    // proxy p = i + j*n sits at (xi_i, eta_j): the loop order of
    // fast_sum_module.f90:119-127 and mom6_fast_sum_module.f90:96-105
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            double *o = xyz + 3 * (i + j * n);
            xyz_from_xieta(cx[i], ce[j], q.face, &o[0], &o[1], &o[2]);
        }
    if (nodes) {
        for (int i = 0; i < n; ++i) { nodes[i] = cx[i]; nodes[n + i] = ce[i]; }
    }
    if (box) { box[0] = q.min_xi; box[1] = q.max_xi; box[2] = q.min_eta; box[3] = q.max_eta; }
}

// interp_vals_bli's one-dimensional basis (bli_module.f90:67-105): the
// exact-node test, then the second barycentric form normalised by its
// denominator; weights 1/2, -1, 1, ..., (-1)^d / 2 (bli_module.f90:13-24).
void bli_basis_host(double x, const double *nodes, int n, double *f) {
    bool found = false;
    for (int i = 0; i < n; ++i) {
        f[i] = 0.0;
        if (std::fabs(x - nodes[i]) < 1e-16) { found = true; f[i] = 1.0; }
    }
    if (found) return;
    double denom = 0.0;
    for (int i = 0; i < n; ++i) {
        double c = (i & 1) ? -1.0 : 1.0;
        if (n == 1) c = 1.0;
        else if (i == 0 || i == n - 1) c *= 0.5;
        f[i] = c / (x - nodes[i]);
        denom += f[i];
    }
    for (int i = 0; i < n; ++i) f[i] /= denom;
}

static void push_range(std::vector<Item> &v, int64_t off, int64_t cnt, int kind, int32_t mask) {
    for (int64_t b = 0; b < cnt; b += kMaxStage) {
        int64_t c = std::min<int64_t>(kMaxStage, cnt - b);
        v.push_back(Item{(int32_t)(off + b), (int32_t)c, mask, kind});
    }
}

bool plan_build(const Tree &t, int d, int mode, const int32_t *list, int64_t nlist, const int32_t *pc, int64_t npc,
                const int32_t *pp, int64_t npp, Plan *pl, std::string *err) {
    if (d < 1 || d > kMaxDegree) { *err = "interp_degree must be in 1.." + std::to_string(kMaxDegree); return false; }
    const int n = t.n, np = (int)t.p.size(), nd = d + 1, P = nd * nd;
    pl->n = n; pl->d = d; pl->P = P; pl->mode = mode; pl->npanels = np;
    pl->perm = t.order;
    // ---------------------------------------------------------------- leaves
    std::vector<int32_t> leaves;                 // panel indices of leaves with points, by range start
    for (int k = 0; k < np; ++k)
        if (t.p[k].is_leaf && t.p[k].count() > 0) leaves.push_back(k);
    std::sort(leaves.begin(), leaves.end(), [&](int a, int b) { return t.p[a].begin < t.p[b].begin; });
    pl->nleaves = (int)leaves.size();
    std::vector<int64_t> leaf_begin(leaves.size());
    for (size_t i = 0; i < leaves.size(); ++i) leaf_begin[i] = t.p[leaves[i]].begin;
    for (auto k : leaves)
        if (t.p[k].count() > 256) { *err = "leaves with more than 256 points are not supported (cluster_thresh <= 257)"; return false; }
    // leaves under panel k: contiguous in range order
    auto leaf_range = [&](int k, int32_t *lb, int32_t *le) {
        const Panel &q = t.p[k];
        *lb = (int32_t)(std::lower_bound(leaf_begin.begin(), leaf_begin.end(), q.begin) - leaf_begin.begin());
        *le = (int32_t)(std::lower_bound(leaf_begin.begin(), leaf_begin.end(), q.end) - leaf_begin.begin());
    };
    std::vector<int32_t> leaf_of_pos(n, -1);
    for (size_t i = 0; i < leaves.size(); ++i)
        for (int64_t p = t.p[leaves[i]].begin; p < t.p[leaves[i]].end; ++p) leaf_of_pos[p] = (int32_t)i;
    // ---------------------------------------------------------------- slots
    std::vector<int32_t> src_slot(np, -1), tgt_slot(np, -1);
    const bool dtt = (mode == 0);
    if (dtt) {
        for (int64_t i = 0; i < nlist; ++i) {
            int32_t it = list[3 * i], is = list[3 * i + 1], ty = list[3 * i + 2];
            if (it < 1 || it > np || is < 1 || is > np || ty < 0 || ty > 3) {
                *err = "interaction " + std::to_string(i + 1) + " is out of range";
                return false;
            }
            if (ty == 1 || ty == 3) src_slot[is - 1] = 0;
            if (ty == 2 || ty == 3) tgt_slot[it - 1] = 0;
        }
    } else {
        for (int k = 0; k < np; ++k) src_slot[k] = 0;  // slot == panel index: the reference's flat weight layout
    }
    for (int k = 0; k < np; ++k)
        if (src_slot[k] == 0) { src_slot[k] = (int32_t)pl->src_slot_panel.size(); pl->src_slot_panel.push_back(k); }
    for (int k = 0; k < np; ++k)
        if (tgt_slot[k] == 0) { tgt_slot[k] = (int32_t)pl->tgt_slot_panel.size(); pl->tgt_slot_panel.push_back(k); }
    const int32_t nsrc = (int32_t)pl->src_slot_panel.size(), ntgt = (int32_t)pl->tgt_slot_panel.size();
    if ((int64_t)n + (int64_t)nsrc * P > INT32_MAX / 2) { *err = "grid too large for 32-bit pool offsets"; return false; }
    pl->src_proxy_xyz.resize((size_t)nsrc * P * 3);
    pl->src_nodes.resize((size_t)nsrc * 2 * nd);
    pl->src_box.resize((size_t)nsrc * 4);
    for (int32_t s = 0; s < nsrc; ++s)
        panel_proxies(t.p[pl->src_slot_panel[s]], d, &pl->src_proxy_xyz[(size_t)s * P * 3], &pl->src_nodes[(size_t)s * 2 * nd],
                      &pl->src_box[(size_t)s * 4]);
    pl->tgt_proxy_xyz.resize((size_t)ntgt * P * 3);
    pl->tgt_nodes.resize((size_t)ntgt * 2 * nd);
    pl->tgt_box.resize((size_t)ntgt * 4);
    for (int32_t s = 0; s < ntgt; ++s)
        panel_proxies(t.p[pl->tgt_slot_panel[s]], d, &pl->tgt_proxy_xyz[(size_t)s * P * 3], &pl->tgt_nodes[(size_t)s * 2 * nd],
                      &pl->tgt_box[(size_t)s * 4]);
    // ---------------------------------------------------------------- upward units
    pl->up_unit_beg.assign(nsrc + 1, 0);
    for (int32_t s = 0; s < nsrc; ++s) {
        const Panel &q = t.p[pl->src_slot_panel[s]];
        pl->up_unit_beg[s] = (int32_t)pl->up_units.size();
        for (int64_t b = q.begin; b < q.end; b += kUpChunk)
            pl->up_units.push_back(UpUnit{s, (int32_t)b, (int32_t)std::min<int64_t>(q.end, b + kUpChunk), pl->src_slot_panel[s]});
        pl->macs_up += (double)q.count() * P;
    }
    pl->up_unit_beg[nsrc] = (int32_t)pl->up_units.size();
    // ---------------------------------------------------------------- per-leaf and per-target-slot items
    const int64_t pool_proxy0 = n;
    auto proxy_off = [&](int k) { return pool_proxy0 + (int64_t)src_slot[k] * P; };
    std::vector<std::vector<Item>> litems(leaves.size()), titems(ntgt);
    std::vector<double> lcost(leaves.size(), 0.0), tcost(ntgt, 0.0);
    pl->masks.clear();
    if (dtt) {
        for (int64_t i = 0; i < nlist; ++i) {
            int k_t = list[3 * i] - 1, k_s = list[3 * i + 1] - 1, ty = list[3 * i + 2];
            const Panel &T = t.p[k_t], &S = t.p[k_s];
            if (T.count() == 0 || S.count() == 0) continue;
            if (ty == 0 || ty == 1) {
                int32_t lb, le;
                leaf_range(k_t, &lb, &le);
                for (int32_t l = lb; l < le; ++l) {
                    if (ty == 0) push_range(litems[l], S.begin, S.count(), 0, -1);
                    else push_range(litems[l], proxy_off(k_s), P, 1, -1);
                    lcost[l] += (double)(ty == 0 ? S.count() : P) * t.p[leaves[l]].count();
                }
                pl->pairs[ty] += (double)T.count() * (ty == 0 ? S.count() : P);
            } else {
                int32_t ts = tgt_slot[k_t];
                if (ty == 2) push_range(titems[ts], S.begin, S.count(), 0, -1);
                else push_range(titems[ts], proxy_off(k_s), P, 1, -1);
                tcost[ts] += (double)P * (ty == 2 ? S.count() : P);
                pl->pairs[ty] += (double)P * (ty == 2 ? S.count() : P);
            }
        }
        // DOWN items: every leaf under a target slot interpolates its potentials
        for (int32_t s = 0; s < ntgt; ++s) {
            int32_t lb, le;
            leaf_range(pl->tgt_slot_panel[s], &lb, &le);
            for (int32_t l = lb; l < le; ++l) {
                litems[l].push_back(Item{s, 0, -1, 2});
                lcost[l] += (double)P * t.p[leaves[l]].count() * 0.5;
            }
            pl->macs_down += (double)t.p[pl->tgt_slot_panel[s]].count() * P;
        }
    } else {
        // STT: per-point pairs become per-leaf items with per-target bitmasks.
        struct PairRec { int32_t key, local; };
        for (int64_t i = 0; i < npc + npp; ++i) {
            const int32_t *e = i < npc ? pc + 2 * i : pp + 2 * (i - npc);
            if (e[0] < 1 || e[0] > n || e[1] < 1 || e[1] > np) { *err = "STT list entry out of range"; return false; }
        }
        std::vector<int32_t> pos_of(n);
        for (int32_t p = 0; p < n; ++p) pos_of[t.order[p]] = p;
        // bucket pairs by leaf: key = panel*2 + kind
        std::vector<int64_t> off(leaves.size() + 1, 0);
        auto leaf_of_point = [&](int32_t ip) { return leaf_of_pos[pos_of[ip]]; };
        for (int64_t i = 0; i < npc; ++i) off[leaf_of_point(pc[2 * i] - 1) + 1]++;
        for (int64_t i = 0; i < npp; ++i) off[leaf_of_point(pp[2 * i] - 1) + 1]++;
        for (size_t l = 0; l < leaves.size(); ++l) off[l + 1] += off[l];
        std::vector<PairRec> recs(off.back());
        {
            std::vector<int64_t> w(off.begin(), off.end() - 1);
            auto put = [&](const int32_t *L, int64_t m, int kind) {
                for (int64_t i = 0; i < m; ++i) {
                    int32_t ip = L[2 * i] - 1, is = L[2 * i + 1] - 1;
                    int32_t pos = pos_of[ip], l = leaf_of_pos[pos];
                    recs[w[l]++] = PairRec{is * 2 + kind, (int32_t)(pos - t.p[leaves[l]].begin)};
                }
            };
            put(pc, npc, 1);
            put(pp, npp, 0);
        }
        std::vector<std::vector<uint32_t>> lmask(leaves.size());
#pragma omp parallel for schedule(dynamic, 16)
        for (int64_t l = 0; l < (int64_t)leaves.size(); ++l) {
            const int64_t nt = t.p[leaves[l]].count();
            const int words = (int)((nt + 31) / 32);
            std::unordered_map<int32_t, int32_t> idx;
            std::vector<int32_t> keys;
            std::vector<uint32_t> &mk = lmask[l];
            for (int64_t r = off[l]; r < off[l + 1]; ++r) {
                auto it = idx.find(recs[r].key);
                int32_t slot;
                if (it == idx.end()) {
                    slot = (int32_t)keys.size();
                    idx.emplace(recs[r].key, slot);
                    keys.push_back(recs[r].key);
                    mk.resize(mk.size() + words, 0u);
                } else {
                    slot = it->second;
                }
                mk[(size_t)slot * words + recs[r].local / 32] |= 1u << (recs[r].local % 32);
            }
            // emit items in (kind, panel) order for locality; mask offsets are
            // leaf-local here and rebased below
            std::vector<int32_t> ordk(keys.size());
            std::iota(ordk.begin(), ordk.end(), 0);
            std::sort(ordk.begin(), ordk.end(), [&](int a, int b) { return keys[a] < keys[b]; });
            double c = 0;
            for (int32_t a : ordk) {
                int32_t k_s = keys[a] / 2, kind = keys[a] % 2;
                if (kind == 0) push_range(litems[l], t.p[k_s].begin, t.p[k_s].count(), 0, a * words);
                else push_range(litems[l], proxy_off(k_s), P, 1, a * words);
                c += (double)(kind == 0 ? t.p[k_s].count() : P) * nt;
            }
            lcost[l] = c;
        }
        for (size_t l = 0; l < leaves.size(); ++l) {
            int32_t base = (int32_t)pl->masks.size();
            for (auto &it : litems[l]) it.mask += base;
            pl->masks.insert(pl->masks.end(), lmask[l].begin(), lmask[l].end());
        }
        for (int64_t i = 0; i < npc; ++i) pl->pairs[1] += P;
        for (int64_t i = 0; i < npp; ++i) pl->pairs[0] += (double)t.p[pp[2 * i + 1] - 1].count();
    }
    // ---------------------------------------------------------------- groups, sorted by cost
    {
        std::vector<int32_t> ord(leaves.size());
        std::iota(ord.begin(), ord.end(), 0);
        std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return lcost[a] > lcost[b]; });
        pl->leaf_groups.clear();
        pl->leaf_items.clear();
        pl->max_nt = 0;
        for (int32_t l : ord) {
            const Panel &L = t.p[leaves[l]];
            Group g{};
            g.tgt = (int32_t)L.begin; g.nt = (int32_t)L.count();
            g.ib = (int32_t)pl->leaf_items.size();
            pl->leaf_items.insert(pl->leaf_items.end(), litems[l].begin(), litems[l].end());
            g.ie = (int32_t)pl->leaf_items.size();
            g.out = l;
            pl->max_nt = std::max(pl->max_nt, g.nt);
            pl->leaf_groups.push_back(g);
        }
    }
    {
        // proxy groups: each target slot's items split into units of bounded work
        pl->proxy_groups.clear();
        pl->proxy_items.clear();
        pl->proxy_unit_beg.assign(ntgt + 1, 0);
        std::vector<Group> units;
        std::vector<double> ucost;
        pl->proxy_slot_items.assign(ntgt + 1, 0);
        for (int32_t s = 0; s < ntgt; ++s) {
            pl->proxy_unit_beg[s] = (int32_t)units.size();
            pl->proxy_slot_items[s] = (int32_t)pl->proxy_items.size();
            const auto &v = titems[s];
            size_t i = 0;
            while (i < v.size()) {
                Group g{};
                g.tgt = s; g.nt = P;
                g.ib = (int32_t)pl->proxy_items.size();
                double c = 0;
                while (i < v.size() && (c == 0 || c + (double)v[i].cnt * P <= kProxyUnitPairs)) {
                    pl->proxy_items.push_back(v[i]);
                    c += (double)v[i].cnt * P;
                    ++i;
                }
                g.ie = (int32_t)pl->proxy_items.size();
                g.out = (int32_t)units.size();
                units.push_back(g);
                ucost.push_back(c);
            }
        }
        pl->proxy_unit_beg[ntgt] = (int32_t)units.size();
        pl->proxy_slot_items[ntgt] = (int32_t)pl->proxy_items.size();
        std::vector<int32_t> ord(units.size());
        std::iota(ord.begin(), ord.end(), 0);
        std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return ucost[a] > ucost[b]; });
        for (int32_t u : ord) pl->proxy_groups.push_back(units[u]);
    }
    pl->leaf_panel = leaves;
    pl->mix_built = false;
    if (dtt && !plan_build_tc(t, pl, TcOptions{}, err)) return false;
    // ---------------------------------------------------------------- point data in pool order
    pl->pxi.resize(n); pl->peta.resize(n);
    for (int32_t p = 0; p < n; ++p) { pl->pxi[p] = t.xi[t.order[p]]; pl->peta[p] = t.eta[t.order[p]]; }
    return true;
}

// ---------------------------------------------------------------- 32-field groups
// The batched form's work re-cut for the mma.sync kernels (32-field blocks):
// items of at most kMixStage sources, groups of at most kMixRows targets, and
// a local coordinate origin per group (the panel centre) so the FP32 kernel
// tiles see small coordinate differences.  Built only for grids that use
// 32-field blocks (plan_build leaves it out: it is a third of the plan's time).
void plan_build_mix(const Tree &t, Plan *pl) {
    const int P = pl->P;
    const bool dtt = pl->mode == 0;
    const std::vector<int32_t> &leaves = pl->leaf_panel;
    {
        auto rechunk = [&](const std::vector<Item> &src, int32_t ib, int32_t ie, std::vector<Item> &dst) {
            for (int32_t i = ib; i < ie; ++i) {
                const Item &it = src[i];
                if (it.kind == 2) {
                    for (int r = 0; r < 3 * P; r += kMixStage)
                        dst.push_back(Item{it.off, std::min(kMixStage, 3 * P - r), r, 2});
                } else {
                    for (int b = 0; b < it.cnt; b += kMixStage)
                        dst.push_back(Item{it.off + b, std::min(kMixStage, it.cnt - b), it.mask, it.kind});
                }
            }
        };
        pl->mix_leaf_groups.clear();
        pl->mix_leaf_items.clear();
        if (dtt) {
            for (const Group &g : pl->leaf_groups) {
                int32_t ib = (int32_t)pl->mix_leaf_items.size();
                rechunk(pl->leaf_items, g.ib, g.ie, pl->mix_leaf_items);
                int32_t ie = (int32_t)pl->mix_leaf_items.size();
                const int k = leaves[g.out];
                for (int32_t r = 0; r < g.nt; r += kMixRows) {
                    MixGroup m{};
                    m.tgt = g.tgt + r; m.nt = std::min(kMixRows, g.nt - r); m.ib = ib; m.ie = ie; m.out = g.out;
                    m.cx = t.cx[k]; m.cy = t.cy[k]; m.cz = t.cz[k];
                    pl->mix_leaf_groups.push_back(m);
                }
            }
            pl->mix_proxy_groups.clear();
            pl->mix_proxy_items.clear();
            for (const Group &g : pl->proxy_groups) {
                int32_t ib = (int32_t)pl->mix_proxy_items.size();
                rechunk(pl->proxy_items, g.ib, g.ie, pl->mix_proxy_items);
                int32_t ie = (int32_t)pl->mix_proxy_items.size();
                const int k = pl->tgt_slot_panel[g.tgt];
                for (int32_t r = 0; r < P; r += kMixRows) {
                    MixGroup m{};
                    m.tgt = g.tgt; m.nt = std::min(kMixRows, P - r); m.ib = ib; m.ie = ie; m.out = g.out; m.row0 = r;
                    m.cx = t.cx[k]; m.cy = t.cy[k]; m.cz = t.cz[k];
                    pl->mix_proxy_groups.push_back(m);
                }
            }
            pl->mix_up_groups.clear();
            for (size_t u = 0; u < pl->up_units.size(); ++u)
                for (int32_t r = 0; r < P; r += kMixRows) {
                    MixGroup m{};
                    m.tgt = pl->up_units[u].slot; m.nt = std::min(kMixRows, P - r); m.ib = pl->up_units[u].beg;
                    m.ie = pl->up_units[u].end; m.out = (int32_t)u; m.row0 = r;
                    pl->mix_up_groups.push_back(m);
                }
        }
    }
    pl->mix_built = true;
}

// ---------------------------------------------------------------- tcgen05 passes
// The split weight store holds every source row of the leaf pass once, as
// TF32 hi/lo tiles per k-step of 8 rows: each leaf's points, then each source
// slot's P proxies, then the potential rows (3P per target slot in the direct
// passes, per leaf under a target slot in the tree passes), every range padded
// with zero rows to a multiple of 8 so that each item starts on a k-step
// boundary and its padding columns meet zero weights.
//
// Tree passes (opt.tree_passes).  Upward: the weights of every leaf below a
// source slot come from its own points (one tcgen05 work unit per leaf), and
// every refined panel below a source slot sums its children's weights moved
// onto its own Chebyshev nodes (child-to-parent BLI transfer, exact for the
// degree-d polynomials both grids reproduce), level by level from the
// deepest.  Downward: every panel below a target slot adds its parent's
// potentials interpolated at its own nodes (parent-to-child transfer), level
// by level from the top, so a leaf needs one DOWN item (its own potentials)
// instead of one per target slot above it.  The FP64 forms keep the
// reference's direct passes.
// Kernel-tile store of the FP16 leaf pass: a group's stored items follow one
// another (an item is one stage: kTcChunk sources at most), every `every`-th
// item of the group (items every-1, 2 every-1, ...; all with every = 1).  A
// stage of c sources holds ceil(ceil(c / 8) / 2) MMA steps of 16 sources,
// each four chunks (hi, lo x east, north) of the group's rows rounded up to
// 16, 32 bytes per row.
void plan_tile_offsets(Plan *pl, int every) {
    pl->tc_tile_off.assign(pl->tc_leaf_groups.size() + 1, 0);
    for (size_t gi = 0; gi < pl->tc_leaf_groups.size(); ++gi) {
        const MixGroup &m = pl->tc_leaf_groups[gi];
        const int64_t cb = (int64_t)((m.nt + 15) & ~15) * 32;
        int64_t b = 0;
        for (int32_t i = m.ib; i < m.ie; ++i)
            if ((i - m.ib) % every == every - 1) b += (int64_t)(((pl->tc_items[i].cnt + 7) / 8 + 1) / 2) * 4 * cb;
        pl->tc_tile_off[gi + 1] = pl->tc_tile_off[gi] + b;
    }
}

bool plan_build_tc(const Tree &t, Plan *pl, const TcOptions &opt, std::string *err) {
    const int n = t.n, np = (int)t.p.size(), d = pl->d, nd = d + 1, P = pl->P;
    const int32_t nsrc = (int32_t)pl->src_slot_panel.size(), ntgt = (int32_t)pl->tgt_slot_panel.size();
    if (opt.chain_ksteps < 1 || opt.up_chunk < 1 || opt.proxy_unit_kpairs < 1 || opt.cta_groups < 1) {
        *err = "tcgen05 options must be positive";
        return false;
    }
    pl->tc_opt = opt;
    if (d > kMaxTreeDegree) pl->tc_opt.tree_passes = 0;   // the transfer tiles fit shared memory up to kMaxTreeDegree
    std::vector<int32_t> leaves;
    for (int k = 0; k < np; ++k)
        if (t.p[k].is_leaf && t.p[k].count() > 0) leaves.push_back(k);
    std::sort(leaves.begin(), leaves.end(), [&](int a, int b) { return t.p[a].begin < t.p[b].begin; });
    std::vector<int64_t> leaf_begin(leaves.size());
    for (size_t i = 0; i < leaves.size(); ++i) leaf_begin[i] = t.p[leaves[i]].begin;
    auto leaf_range = [&](int k, int32_t *lb, int32_t *le) {
        const Panel &q = t.p[k];
        *lb = (int32_t)(std::lower_bound(leaf_begin.begin(), leaf_begin.end(), q.begin) - leaf_begin.begin());
        *le = (int32_t)(std::lower_bound(leaf_begin.begin(), leaf_begin.end(), q.end) - leaf_begin.begin());
    };
    std::vector<int32_t> leaf_of_pos(n, -1);
    for (size_t i = 0; i < leaves.size(); ++i)
        for (int64_t q = t.p[leaves[i]].begin; q < t.p[leaves[i]].end; ++q) leaf_of_pos[q] = (int32_t)i;
    std::vector<int32_t> src_slot(np, -1), tgt_slot(np, -1);
    for (int32_t s = 0; s < nsrc; ++s) src_slot[pl->src_slot_panel[s]] = s;
    for (int32_t s = 0; s < ntgt; ++s) tgt_slot[pl->tgt_slot_panel[s]] = s;
    const bool tree = pl->tc_opt.tree_passes != 0;

    // ---- slots of the tree passes: panels with points below a source
    // (target) slot, BFS order is parents before children
    std::vector<int32_t> wslot(np, -1), dslot(np, -1);
    int32_t nw = nsrc, ndn = ntgt;
    std::vector<int32_t> wpanel(pl->src_slot_panel), dpanel(pl->tgt_slot_panel);
    for (int32_t s = 0; s < nsrc; ++s) wslot[pl->src_slot_panel[s]] = s;
    for (int32_t s = 0; s < ntgt; ++s) dslot[pl->tgt_slot_panel[s]] = s;
    if (tree) {
        for (int k = 0; k < np; ++k) {
            const Panel &q = t.p[k];
            if (q.count() == 0 || q.parent < 1) continue;
            const int par = q.parent - 1;
            if (wslot[k] < 0 && wslot[par] >= 0) { wslot[k] = nw++; wpanel.push_back(k); }
            if (dslot[k] < 0 && dslot[par] >= 0) { dslot[k] = ndn++; dpanel.push_back(k); }
        }
    }
    pl->n_wslots = nw;
    pl->n_dslots = ndn;
    auto nodes_of = [&](const std::vector<int32_t> &panels, std::vector<double> &out) {
        out.assign(panels.size() * 2 * (size_t)nd, 0.0);
        for (size_t i = 0; i < panels.size(); ++i) {
            const Panel &q = t.p[panels[i]];
            cheb_nodes(q.min_xi, q.max_xi, d, &out[i * 2 * nd]);
            cheb_nodes(q.min_eta, q.max_eta, d, &out[i * 2 * nd + nd]);
        }
    };
    nodes_of(wpanel, pl->tc_up_nodes);
    nodes_of(dpanel, pl->tc_down_nodes);
    pl->m2m_tasks.clear();
    pl->m2m_level_beg.clear();
    pl->l2l_tasks.clear();
    pl->l2l_level_beg.clear();
    if (tree) {
        const int maxl = t.max_level();
        std::vector<std::vector<int32_t>> up(maxl + 1), down(maxl + 1);
        for (int k = 0; k < np; ++k) {
            const Panel &q = t.p[k];
            if (wslot[k] >= 0 && !q.is_leaf && q.count() > 0) up[q.level].push_back(k);
            if (dslot[k] >= 0 && q.parent >= 1 && dslot[q.parent - 1] >= 0) down[q.level].push_back(k);
        }
        // which half of its parent's xi (bit 0) and eta (bit 1) interval a
        // child covers: 0 the lower half, 1 the upper
        auto halves = [&](int ch) {
            const Panel &c = t.p[ch], &q = t.p[c.parent - 1];
            return (c.min_xi < q.mid_xi ? 0 : 1) | (c.min_eta < q.mid_eta ? 0 : 2);
        };
        for (int l = maxl; l >= 0; --l) {
            if (up[l].empty()) continue;
            pl->m2m_level_beg.push_back((int32_t)(pl->m2m_tasks.size() / 6));
            for (int k : up[l]) {
                pl->m2m_tasks.push_back(wslot[k]);
                int32_t code = 0;
                for (int c = 0; c < 4; ++c) {
                    const int ch = t.p[k].child[c];
                    const bool live = ch >= 1 && t.p[ch - 1].count() > 0;
                    pl->m2m_tasks.push_back(live ? wslot[ch - 1] : -1);
                    if (live) code |= halves(ch - 1) << (2 * c);
                }
                pl->m2m_tasks.push_back(code);
            }
        }
        pl->m2m_level_beg.push_back((int32_t)(pl->m2m_tasks.size() / 6));
        for (int l = 0; l <= maxl; ++l) {
            if (down[l].empty()) continue;
            pl->l2l_level_beg.push_back((int32_t)(pl->l2l_tasks.size() / 4));
            for (int k : down[l]) {
                pl->l2l_tasks.push_back(dslot[k]);
                pl->l2l_tasks.push_back(dslot[t.p[k].parent - 1]);
                pl->l2l_tasks.push_back(tgt_slot[k] >= 0 ? 1 : 0);
                pl->l2l_tasks.push_back(halves(k));
            }
        }
        pl->l2l_level_beg.push_back((int32_t)(pl->l2l_tasks.size() / 4));
        // The transfer matrices.  Barycentric Lagrange bases are invariant
        // under affine maps of the interval, so one pair serves every panel:
        // H[h][j][i] = the parent's basis j (nodes on [-1, 1]) at node i of
        // its lower (h = 0, [-1, 0]) or upper (h = 1, [0, 1]) half.
        pl->tc_transfer.assign(2 * (size_t)nd * nd, 0.0);
        double pn[kMaxDegree + 1], cn[kMaxDegree + 1];
        cheb_nodes(-1.0, 1.0, d, pn);
        for (int h = 0; h < 2; ++h) {
            cheb_nodes(h ? 0.0 : -1.0, h ? 1.0 : 0.0, d, cn);
            for (int i = 0; i < nd; ++i) {
                double f[kMaxDegree + 1];
                bli_basis_host(cn[i], pn, nd, f);
                for (int j = 0; j < nd; ++j) pl->tc_transfer[((size_t)h * nd + j) * nd + i] = f[j];
            }
        }
    }

    // ---- the split weight store's row map
    pl->tc_items.clear();
    pl->tc_proxy_items.clear();
    pl->tc_proxy_groups.clear();
    pl->tc_up_groups.clear();
    pl->tc_up_items.clear();
    pl->tc_up_unit_beg.clear();
    pl->tc_bas.clear();
    pl->bsrc.clear();
    pl->sloc_ranges.clear();
    pl->sloc_centres.clear();
    pl->tc_leaf_groups.clear();
    auto add_range = [&](int64_t b, int64_t e, int k) {
        pl->sloc_ranges.push_back((int32_t)b);
        pl->sloc_ranges.push_back((int32_t)e);
        pl->sloc_centres.push_back(t.cx[k]);
        pl->sloc_centres.push_back(t.cy[k]);
        pl->sloc_centres.push_back(t.cz[k]);
    };
    for (int k : leaves) add_range(t.p[k].begin, t.p[k].end, k);
    for (int32_t s = 0; s < nsrc; ++s) add_range(n + (int64_t)s * P, n + (int64_t)(s + 1) * P, pl->src_slot_panel[s]);
    auto up8 = [](int64_t x) { return (x + 7) & ~int64_t(7); };
    std::vector<int64_t> leaf_b(leaves.size());
    int64_t nb = 0;
    for (size_t i = 0; i < leaves.size(); ++i) { leaf_b[i] = nb; nb += up8(t.p[leaves[i]].count()); }
    const int64_t src_b0 = nb, P8 = up8(P), P38 = up8(3 * P);
    pl->tc_pt_ksteps = src_b0 / 8;
    nb += (int64_t)nsrc * P8;
    const int64_t phi_b0 = nb;
    pl->tc_src_ksteps = phi_b0 / 8;
    // potential blocks: per target slot (direct) or per leaf below a target
    // slot (tree); phi_blocks[b] = the dslot whose rows block b holds
    std::vector<int32_t> phi_blocks, leaf_phi_block(leaves.size(), -1);
    if (tree) {
        for (size_t i = 0; i < leaves.size(); ++i)
            if (dslot[leaves[i]] >= 0) { leaf_phi_block[i] = (int32_t)phi_blocks.size(); phi_blocks.push_back(dslot[leaves[i]]); }
    } else {
        for (int32_t s = 0; s < ntgt; ++s) phi_blocks.push_back(s);
    }
    nb += (int64_t)phi_blocks.size() * P38;
    if (nb / 8 > INT32_MAX / 2) { *err = "grid too large for the split weight store"; return false; }
    pl->bsrc.assign((size_t)nb, -1);
    for (size_t i = 0; i < leaves.size(); ++i) {
        const Panel &q = t.p[leaves[i]];
        for (int64_t r = q.begin; r < q.end; ++r) pl->bsrc[leaf_b[i] + (r - q.begin)] = (int32_t)r;
    }
    for (int32_t s = 0; s < nsrc; ++s)
        for (int r = 0; r < P; ++r) pl->bsrc[src_b0 + s * P8 + r] = (int32_t)(n + (int64_t)s * P + r);
    for (size_t b = 0; b < phi_blocks.size(); ++b)
        for (int r = 0; r < 3 * P; ++r)
            pl->bsrc[phi_b0 + (int64_t)b * P38 + r] = (int32_t)(-2 - ((int64_t)phi_blocks[b] * 3 * P + r));

    // One work list (items [ib, ie) of `src`) as tcgen05 items relative to the
    // centre of target panel kt, with the accumulator-chain flags.  DOWN items
    // of the direct passes read their target slot's potential block.
    auto convert = [&](const std::vector<Item> &src, int32_t ib0, int32_t ie0, int kt, std::vector<TcItem> &dst,
                       int32_t extra_down_leaf) -> bool {
        const int32_t ib = (int32_t)dst.size();
        auto push = [&](int kind, int64_t off, int64_t total, int64_t base, int ks) {
            TcItem r{};
            r.kind = kind;
            if (ks >= 0) {
                r.dx = (float)(t.cx[ks] - t.cx[kt]);
                r.dy = (float)(t.cy[ks] - t.cy[kt]);
                r.dz = (float)(t.cz[ks] - t.cz[kt]);
            }
            for (int64_t b = 0; b < total; b += kTcChunk) {
                r.cnt = (int32_t)std::min<int64_t>(kTcChunk, total - b);
                r.kb = (int32_t)((base + b) / 8);
                r.off = (int32_t)(kind == 2 ? off : off + b);
                r.row0 = kind == 2 ? (int32_t)b : 0;
                dst.push_back(r);
            }
        };
        for (int32_t i = ib0; i < ie0; ++i) {
            const Item &it = src[i];
            if (it.kind == 0) {
                // a point source panel's range, re-joined across the
                // staging splits and cut at leaf boundaries
                int64_t b = it.off, e = (int64_t)it.off + it.cnt;
                while (i + 1 < ie0 && src[i + 1].kind == 0 && src[i + 1].off == e) e += src[++i].cnt;
                while (b < e) {
                    const int32_t l = leaf_of_pos[b];
                    const Panel &q = t.p[leaves[l]];
                    const int64_t le = std::min<int64_t>(e, q.end);
                    if ((b - q.begin) % 8 != 0) return false;   // a point range starting inside a leaf
                    push(0, b, le - b, leaf_b[l] + (b - q.begin), leaves[l]);
                    b = le;
                }
            } else if (it.kind == 1) {
                const int64_t s = ((int64_t)it.off - n) / P;
                push(1, it.off, it.cnt, src_b0 + s * P8, pl->src_slot_panel[s]);
            } else if (!tree) {
                push(2, it.off, 3 * P, phi_b0 + (int64_t)it.off * P38, -1);
            }
        }
        if (extra_down_leaf >= 0 && leaf_phi_block[extra_down_leaf] >= 0)
            push(2, dslot[leaves[extra_down_leaf]], 3 * P, phi_b0 + (int64_t)leaf_phi_block[extra_down_leaf] * P38, -1);
        const int32_t ie = (int32_t)dst.size();
        // accumulator chains: end one after the item that brings it to
        // chain_ksteps k-steps, and always after the list's last item.  The
        // FP16 leaf pass scales kernel tiles and interpolation rows apart, so
        // there DOWN items form chains of their own.
        for (int32_t i = ib, chain = 0; i < ie; ++i) {
            TcItem &r = dst[i];
            chain += (r.cnt + 7) / 8;
            const bool kind_changes = opt.f16 && i + 1 < ie && ((r.kind & 3) == 2) != ((dst[i + 1].kind & 3) == 2);
            if (chain >= opt.chain_ksteps || i == ie - 1 || kind_changes) { r.kind |= kTcFlush; chain = 0; }
        }
        return true;
    };

    // Many work lists at once, on every host thread: job j's items land in
    // dst[range[j].first, range[j].second), the jobs in order.
    struct Job {
        int32_t ib, ie, kt, extra;
    };
    auto convert_all = [&](const std::vector<Item> &src, const std::vector<Job> &jobs, std::vector<TcItem> &dst,
                           std::vector<std::pair<int32_t, int32_t>> &range) -> bool {
        const int64_t nj = (int64_t)jobs.size();
        std::vector<std::vector<TcItem>> part(nj);
        int bad = 0;
#pragma omp parallel for schedule(dynamic, 32) reduction(| : bad)
        for (int64_t j = 0; j < nj; ++j)
            if (!convert(src, jobs[j].ib, jobs[j].ie, jobs[j].kt, part[j], jobs[j].extra)) bad |= 1;
        if (bad) { *err = "internal: point range starts inside a leaf"; return false; }
        std::vector<int64_t> off(nj + 1, (int64_t)dst.size());
        for (int64_t j = 0; j < nj; ++j) off[j + 1] = off[j] + (int64_t)part[j].size();
        if (off[nj] > INT32_MAX) { *err = "tcgen05 work list too long"; return false; }
        dst.resize((size_t)off[nj]);
        range.resize(nj);
#pragma omp parallel for schedule(dynamic, 32)
        for (int64_t j = 0; j < nj; ++j) {
            std::copy(part[j].begin(), part[j].end(), dst.begin() + off[j]);
            range[j] = {(int32_t)off[j], (int32_t)off[j + 1]};
        }
        return true;
    };

    // ---- leaf pass: groups of at most kTcRows targets in pool order
    std::vector<int32_t> gord(pl->leaf_groups.size());
    std::iota(gord.begin(), gord.end(), 0);
    std::sort(gord.begin(), gord.end(), [&](int a, int b) { return pl->leaf_groups[a].tgt < pl->leaf_groups[b].tgt; });
    pl->tc_macs_down = 0;
    std::vector<Job> jobs;
    std::vector<std::pair<int32_t, int32_t>> range;
    jobs.reserve(gord.size());
    for (int32_t gi : gord) {
        const Group &g = pl->leaf_groups[gi];
        jobs.push_back(Job{g.ib, g.ie, leaves[g.out], tree ? g.out : -1});
    }
    if (!convert_all(pl->leaf_items, jobs, pl->tc_items, range)) return false;
    for (size_t x = 0; x < gord.size(); ++x) {
        const Group &g = pl->leaf_groups[gord[x]];
        const int kt = leaves[g.out];
        const int32_t ib = range[x].first, ie = range[x].second;
        if (tree && leaf_phi_block[g.out] >= 0) pl->tc_macs_down += (double)g.nt * P;
        for (int32_t r = 0; r < g.nt; r += kTcRows) {
            MixGroup m{};
            m.tgt = g.tgt + r; m.nt = std::min(kTcRows, g.nt - r); m.ib = ib; m.ie = ie; m.out = g.out;
            m.cx = t.cx[kt]; m.cy = t.cy[kt]; m.cz = t.cz[kt];
            pl->tc_leaf_groups.push_back(m);
        }
    }
    if (!tree) pl->tc_macs_down = pl->macs_down;
    plan_tile_offsets(pl, opt.tile_store > 1 ? opt.tile_store : 1);

    // ---- proxy pass: each target slot's items cut into units of at most
    // proxy_unit_kpairs * 1024 pairs; rows of at most kTcProxyRows proxies
    // (three Cartesian components each fill the MMA's N = 256)
    {
        const double budget = 1024.0 * opt.proxy_unit_kpairs;
        pl->tc_proxy_unit_beg.assign(ntgt + 1, 0);
        struct U { int32_t slot, ib, ie; double cost; };
        std::vector<U> units;
        for (int32_t s = 0; s < ntgt; ++s) {
            pl->tc_proxy_unit_beg[s] = (int32_t)units.size();
            int32_t i = pl->proxy_slot_items[s];
            const int32_t e = pl->proxy_slot_items[s + 1];
            while (i < e) {
                U u{s, i, i, 0.0};
                while (u.ie < e && (u.cost == 0 || u.cost + (double)pl->proxy_items[u.ie].cnt * P <= budget)) {
                    u.cost += (double)pl->proxy_items[u.ie].cnt * P;
                    ++u.ie;
                }
                i = u.ie;
                units.push_back(u);
            }
        }
        pl->tc_proxy_unit_beg[ntgt] = (int32_t)units.size();
        pl->tc_nproxy_units = (int32_t)units.size();
        std::vector<int32_t> ord(units.size());
        std::iota(ord.begin(), ord.end(), 0);
        std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return units[a].cost > units[b].cost; });
        jobs.clear();
        for (int32_t uo : ord) jobs.push_back(Job{units[uo].ib, units[uo].ie, pl->tgt_slot_panel[units[uo].slot], -1});
        if (!convert_all(pl->proxy_items, jobs, pl->tc_proxy_items, range)) return false;
        for (size_t x = 0; x < ord.size(); ++x) {
            const int32_t uo = ord[x];
            const U &u = units[uo];
            const int kt = pl->tgt_slot_panel[u.slot];
            const int32_t ib = range[x].first, ie = range[x].second;
            for (int32_t r = 0; r < P; r += kTcProxyRows) {
                MixGroup m{};
                m.tgt = u.slot; m.nt = std::min(kTcProxyRows, P - r); m.ib = ib; m.ie = ie; m.out = uo; m.row0 = r;
                m.cx = t.cx[kt]; m.cy = t.cy[kt]; m.cz = t.cz[kt];
                pl->tc_proxy_groups.push_back(m);
            }
        }
    }

    // ---- upward pass.  Direct: per source slot, units of whole leaves of
    // its panel (at least up_chunk points, or the panel's rest).  Tree: one
    // unit per leaf below a source slot, written straight to the leaf's
    // wslot rows.  Rows of at most kTcRows proxies; every item gets its own
    // k-steps in the basis store (per-point BLI factors over the nodes of
    // the unit's panel: tc_bas holds nodes slot, first pool row, rows).
    pl->tc_up_unit_beg.assign(nsrc + 1, 0);
    int32_t nunits = 0;
    int64_t nbk = 0;
    pl->tc_macs_up = 0;
    auto add_unit = [&](int ks, int64_t b, int64_t e, int32_t out, int32_t nodes_slot) -> bool {
        const std::vector<Item> range{Item{(int32_t)b, (int32_t)(e - b), -1, 0}};
        const int32_t ib = (int32_t)pl->tc_up_items.size();
        if (!convert(range, 0, 1, ks, pl->tc_up_items, -1)) { *err = "internal: point range starts inside a leaf"; return false; }
        const int32_t ie = (int32_t)pl->tc_up_items.size();
        for (int32_t i = ib; i < ie; ++i) {
            TcItem &r = pl->tc_up_items[i];
            r.row0 = (int32_t)nbk;
            for (int32_t k = 0; k < r.cnt; k += 8) {
                pl->tc_bas.push_back(nodes_slot);
                pl->tc_bas.push_back(r.off + k);
                pl->tc_bas.push_back(std::min(8, r.cnt - k));
                ++nbk;
            }
        }
        for (int32_t r = 0; r < P; r += kTcRows) {
            MixGroup m{};
            m.tgt = nodes_slot; m.nt = std::min(kTcRows, P - r); m.ib = ib; m.ie = ie; m.out = out; m.row0 = r;
            pl->tc_up_groups.push_back(m);
        }
        pl->tc_macs_up += (double)(e - b) * P;
        return true;
    };
    if (tree) {
        for (size_t i = 0; i < leaves.size(); ++i) {
            const int k = leaves[i];
            if (wslot[k] < 0) continue;
            if (!add_unit(k, t.p[k].begin, t.p[k].end, wslot[k], wslot[k])) return false;
            ++nunits;
        }
    } else {
        for (int32_t s = 0; s < nsrc; ++s) {
            const int ks = pl->src_slot_panel[s];
            pl->tc_up_unit_beg[s] = nunits;
            int32_t lb, le;
            leaf_range(ks, &lb, &le);
            for (int32_t l = lb; l < le;) {
                const int64_t b = t.p[leaves[l]].begin;
                int64_t e = b;
                int32_t l2 = l;
                while (l2 < le && e - b < opt.up_chunk) e = t.p[leaves[l2++]].end;
                if (!add_unit(ks, b, e, nunits, s)) return false;
                ++nunits;
                l = l2;
            }
        }
        pl->tc_up_unit_beg[nsrc] = nunits;
    }
    if (nbk > INT32_MAX / 2) { *err = "grid too large for the basis store"; return false; }
    return true;
}

}  // namespace sal
