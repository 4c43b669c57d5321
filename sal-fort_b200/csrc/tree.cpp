// Host-side cubed-sphere quadtree and interaction lists.
//
// Tree and MAC decisions must equal the reference's exactly, so the geometry
// below restates cube_sphere_module.f90 with glibc libm (the library gfortran
// calls) and no FMA contraction (this file is built with -ffp-contract=off).
// The data layout is this library's own: points are partitioned in place into
// one permutation array, so every panel is a contiguous range of it.
#include <cmath>
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "sal_internal.hpp"
#ifdef _OPENMP
#include <omp.h>
#endif

namespace sal {

static constexpr int kTreeMaxLevel = 40;  // the reference refines identical points forever

// face_from_xyz, cube_sphere_module.f90:7-35.
int face_from_xyz(double x, double y, double z) {
    double ax = std::fabs(x), ay = std::fabs(y), az = std::fabs(z);
    if (ax >= ay && ax >= az) return x >= 0 ? 1 : 3;
    if (ay >= ax && ay >= az) return y >= 0 ? 2 : 4;
    return z >= 0 ? 5 : 6;
}

// xieta_from_xyz, cube_sphere_module.f90:38-61.
void face_xieta(double x, double y, double z, int face, double *xi, double *eta) {
    switch (face) {
        case 1: *xi = std::atan(y / x); *eta = std::atan(z / x); break;
        case 2: *xi = std::atan(-x / y); *eta = std::atan(z / y); break;
        case 3: *xi = std::atan(y / x); *eta = std::atan(-z / x); break;
        case 4: *xi = std::atan(-x / y); *eta = std::atan(-z / y); break;
        case 5: *xi = std::atan(y / z); *eta = std::atan(-x / z); break;
        default: *xi = std::atan(-y / z); *eta = std::atan(-x / z); break;
    }
}

// xyz_from_xieta, cube_sphere_module.f90:64-95.
void xyz_from_xieta(double xi, double eta, int face, double *x, double *y, double *z) {
    double ax = std::tan(xi), ay = std::tan(eta);
    double r = std::sqrt(1 + ax * ax + ay * ay);
    switch (face) {
        case 1: *x = 1.0 / r; *y = ax * *x; *z = ay * *x; break;
        case 2: *y = 1.0 / r; *x = -ax * *y; *z = ay * *y; break;
        case 3: *x = -1.0 / r; *y = ax * *x; *z = -ay * *x; break;
        case 4: *y = -1.0 / r; *x = -ax * *y; *z = -ay * *y; break;
        case 5: *z = 1.0 / r; *x = -ay * *z; *y = ax * *z; break;
        default: *z = -1.0 / r; *x = -ay * *z; *y = -ax * *z; break;
    }
}

// bli_interp_points_shift, bli_module.f90:28-48.
void cheb_nodes(double min_x, double max_x, int degree, double *out) {
    double pi = 4.0 * std::atan(1.0);
    double range = 0.5 * (max_x - min_x), shift = 0.5 * (max_x + min_x);
    if (degree == 0) { out[0] = shift; return; }
    for (int i = 0; i <= degree; ++i) out[i] = std::cos(pi / degree * (double)i) * range + shift;
}

static double clamp_acos(double v) {
    v = v > -1.0 ? v : -1.0;
    v = v < 1.0 ? v : 1.0;
    return std::acos(v);
}

int32_t Tree::max_level() const {
    int32_t m = 0;
    for (auto &q : p) m = std::max(m, q.level);
    return m;
}

std::vector<int32_t> Tree::points_inside(int32_t k) const {
    const Panel &q = p[k - 1];
    std::vector<int32_t> v(order.begin() + q.begin, order.begin() + q.end);
    std::sort(v.begin(), v.end());
    for (auto &x : v) x += 1;
    return v;
}

// Per-point face and (xi, eta) on that face: the values tree_traverse
// recomputes at every refinement (tree_module.f90:179), computed once.
void tree_set_points(Tree *t, const double *xs, const double *ys, const double *zs) {
    int32_t n = t->n;
    t->xi.resize(n); t->eta.resize(n); t->face.resize(n);
#pragma omp parallel for schedule(static)
    for (int32_t i = 0; i < n; ++i) {
        int f = face_from_xyz(xs[i], ys[i], zs[i]);
        t->face[i] = (int8_t)f;
        face_xieta(xs[i], ys[i], zs[i], f, &t->xi[i], &t->eta[i]);
    }
}

// Panel radius (tree_module.f90:224-244) and MAC centre.
void tree_finish_panels(Tree *t) {
    size_t np = t->p.size();
    t->cx.resize(np); t->cy.resize(np); t->cz.resize(np);
#pragma omp parallel for schedule(static)
    for (size_t k = 0; k < np; ++k) {
        Panel &q = t->p[k];
        double x1, x2, x3, y1, y2, y3;
        xyz_from_xieta(q.mid_xi, q.mid_eta, q.face, &x1, &x2, &x3);
        t->cx[k] = x1; t->cy[k] = x2; t->cz[k] = x3;
        const double cxi[4] = {q.min_xi, q.min_xi, q.max_xi, q.max_xi};
        const double ceta[4] = {q.min_eta, q.max_eta, q.max_eta, q.min_eta};
        double r = 0;
        for (int c = 0; c < 4; ++c) {
            xyz_from_xieta(cxi[c], ceta[c], q.face, &y1, &y2, &y3);
            double dd = clamp_acos(x1 * y1 + x2 * y2 + x3 * y3);
            r = c == 0 ? dd : (dd > r ? dd : r);
        }
        q.radius = r;
    }
}

// tree_traverse, tree_module.f90:59-246: six face roots, then BFS refinement of
// every leaf holding >= thresh points into SW, SE, NE, NW children by
// xi < mid_xi, eta < mid_eta.  Each refinement is a stable 4-way partition of
// the parent's range, which keeps every leaf's range in the reference's
// points_inside order.
Tree *tree_build(const double *xs, const double *ys, const double *zs, int32_t n, int32_t thresh) {
    Tree *t = new Tree();
    t->n = n;
    tree_set_points(t, xs, ys, zs);
    double pi = 4.0 * std::atan(1.0);
    int64_t cnt[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int32_t i = 0; i < n; ++i) cnt[t->face[i]]++;
    t->order.resize(n);
    int64_t start[7];
    start[1] = 0;
    for (int f = 2; f <= 6; ++f) start[f] = start[f - 1] + cnt[f - 1];
    {
        int64_t pos[7];
        std::memcpy(pos, start, sizeof(pos));
        for (int32_t i = 0; i < n; ++i) t->order[pos[t->face[i]]++] = i;
    }
    t->p.reserve(6 + 4 * (size_t)(n / std::max(1, thresh) + 8) * 2);
    for (int f = 1; f <= 6; ++f) {
        Panel q;
        q.id = f; q.face = f;
        q.min_xi = -pi / 4.0; q.mid_xi = 0.0; q.max_xi = pi / 4.0;
        q.min_eta = -pi / 4.0; q.mid_eta = 0.0; q.max_eta = pi / 4.0;
        q.begin = start[f]; q.end = start[f] + cnt[f];
        t->p.push_back(q);
    }
    std::vector<int32_t> tmp;
    for (size_t i = 0; i < t->p.size(); ++i) {
        if (!(t->p[i].count() >= thresh && t->p[i].is_leaf && t->p[i].level < kTreeMaxLevel)) continue;
        Panel par = t->p[i];
        int32_t pc = (int32_t)t->p.size();
        t->p[i].is_leaf = 0;
        for (int j = 0; j < 4; ++j) t->p[i].child[j] = pc + j + 1;
        double mnx = par.min_xi, mdx = par.mid_xi, mxx = par.max_xi;
        double mne = par.min_eta, mde = par.mid_eta, mxe = par.max_eta;
        int64_t qc[4] = {0, 0, 0, 0};
        int64_t m = par.count();
        tmp.resize(m);
        std::vector<int8_t> which(m);
        for (int64_t j = 0; j < m; ++j) {
            int32_t idx = t->order[par.begin + j];
            double xi = t->xi[idx], eta = t->eta[idx];
            int w = (xi < mdx) ? ((eta < mde) ? 0 : 3) : ((eta < mde) ? 1 : 2);
            which[j] = (int8_t)w;
            qc[w]++;
        }
        int64_t qs[4] = {0, qc[0], qc[0] + qc[1], qc[0] + qc[1] + qc[2]};
        int64_t qp[4] = {qs[0], qs[1], qs[2], qs[3]};
        for (int64_t j = 0; j < m; ++j) tmp[qp[which[j]]++] = t->order[par.begin + j];
        std::copy(tmp.begin(), tmp.end(), t->order.begin() + par.begin);
        const double bx[4][2] = {{mnx, mdx}, {mdx, mxx}, {mdx, mxx}, {mnx, mdx}};
        const double be[4][2] = {{mne, mde}, {mne, mde}, {mde, mxe}, {mde, mxe}};
        for (int j = 0; j < 4; ++j) {
            Panel c;
            c.parent = (int32_t)i + 1; c.level = par.level + 1; c.face = par.face; c.id = pc + j + 1;
            c.min_xi = bx[j][0]; c.max_xi = bx[j][1]; c.mid_xi = 0.5 * (bx[j][0] + bx[j][1]);
            c.min_eta = be[j][0]; c.max_eta = be[j][1]; c.mid_eta = 0.5 * (be[j][0] + be[j][1]);
            c.begin = par.begin + qs[j]; c.end = c.begin + qc[j];
            t->p.push_back(c);
        }
    }
    tree_finish_panels(t);
    return t;
}

// A tree flattened by the caller (its own tree_traverse).  Leaves' points_inside
// are laid out in DFS order (children 1..4), which gives every panel a
// contiguous range; counts are checked against the caller's arrays.
Tree *tree_import(int32_t np, const int32_t *I, const double *D, const int64_t *off, const int32_t *idx, int32_t n,
                  const double *xs, const double *ys, const double *zs, std::string *err) {
    Tree *t = new Tree();
    t->n = n;
    t->p.resize(np);
    for (int32_t k = 0; k < np; ++k) {
        Panel &q = t->p[k];
        const int32_t *a = I + 9 * (size_t)k;
        const double *b = D + 7 * (size_t)k;
        q.level = a[0]; q.is_leaf = a[1]; q.id = a[2]; q.parent = a[3];
        for (int j = 0; j < 4; ++j) q.child[j] = a[4 + j];
        q.face = a[8];
        q.min_xi = b[0]; q.mid_xi = b[1]; q.max_xi = b[2];
        q.min_eta = b[3]; q.mid_eta = b[4]; q.max_eta = b[5]; q.radius = b[6];
        if (q.face < 1 || q.face > 6) { *err = "panel " + std::to_string(k + 1) + " has face outside 1..6"; delete t; return nullptr; }
        for (int j = 0; j < 4 && !q.is_leaf; ++j)
            if (q.child[j] < 1 || q.child[j] > np) { *err = "panel " + std::to_string(k + 1) + " has an invalid child"; delete t; return nullptr; }
    }
    t->order.clear();
    t->order.reserve(n);
    std::vector<uint8_t> seen(n, 0);
    // iterative DFS over the six roots
    std::vector<std::pair<int32_t, int>> st;
    for (int32_t r = 6; r >= 1; --r) st.push_back({r, 0});
    std::vector<int32_t> path;
    while (!st.empty()) {
        auto [k, phase] = st.back();
        st.pop_back();
        Panel &q = t->p[k - 1];
        if (phase == 0) {
            q.begin = (int64_t)t->order.size();
            if (q.is_leaf) {
                for (int64_t j = off[k - 1]; j < off[k]; ++j) {
                    int32_t v = idx[j];
                    if (v < 1 || v > n || seen[v - 1]) { *err = "points_inside of leaf " + std::to_string(k) + " is not a partition"; delete t; return nullptr; }
                    seen[v - 1] = 1;
                    t->order.push_back(v - 1);
                }
                q.end = (int64_t)t->order.size();
            } else {
                st.push_back({k, 1});
                for (int j = 3; j >= 0; --j) st.push_back({q.child[j], 0});
            }
        } else {
            q.end = (int64_t)t->order.size();
        }
    }
    for (int32_t k = 0; k < np; ++k)
        if (t->p[k].count() != off[k + 1] - off[k]) {
            *err = "panel " + std::to_string(k + 1) + " count differs from its children's";
            delete t;
            return nullptr;
        }
    if ((int32_t)t->order.size() != n) { *err = "leaves do not cover every point"; delete t; return nullptr; }
    tree_set_points(t, xs, ys, zs);
    // the caller's radii are kept; only the MAC centres are derived here
    std::vector<double> radius(np);
    for (int32_t k = 0; k < np; ++k) radius[k] = t->p[k].radius;
    tree_finish_panels(t);
    for (int32_t k = 0; k < np; ++k) t->p[k].radius = radius[k];
    return t;
}

// One queued pair of dual_tree_traversal (tree_module.f90:300-392):
// 0 an empty panel, 1..4 a list entry of type code - 1, 5 refine the
// source, 6 refine the target.
int dtt_decide(const Tree &t, int32_t it, int32_t is, double theta, int32_t thresh) {
    const Panel &T = t.p[it - 1], &S = t.p[is - 1];
    int64_t ct = T.count(), cs = S.count();
    if (!(ct > 0 && cs > 0)) return 0;
    double dist = clamp_acos(t.cx[it - 1] * t.cx[is - 1] + t.cy[it - 1] * t.cy[is - 1] + t.cz[it - 1] * t.cz[is - 1]);
    double sep = (T.radius + S.radius) / dist;
    if (dist > 0 && sep < theta) return 1 + (ct > thresh ? 2 : 0) + (cs > thresh ? 1 : 0);
    if ((ct < thresh && cs < thresh) || (T.is_leaf && S.is_leaf)) return 1;
    bool refine_source = T.is_leaf ? true : (S.is_leaf ? false : !(ct >= cs));
    return refine_source ? 5 : 6;
}

// dual_tree_traversal, tree_module.f90:277-398: BFS over panel pairs seeded
// with the 6x6 root pairs; the queue grows as needed.
std::vector<int32_t> dual_tree_traversal(const Tree &t, double theta, int32_t thresh) {
    std::vector<int32_t> tq, sq, L;
    for (int i = 1; i <= 6; ++i)
        for (int j = 1; j <= 6; ++j) { tq.push_back(i); sq.push_back(j); }
    for (size_t cur = 0; cur < tq.size(); ++cur) {
        int32_t it = tq[cur], is = sq[cur];
        const int c = dtt_decide(t, it, is, theta, thresh);
        if (c >= 1 && c <= 4) {
            L.insert(L.end(), {it, is, c - 1});
        } else if (c >= 5) {
            for (int k = 0; k < 4; ++k) {
                if (c == 5) { tq.push_back(it); sq.push_back(t.p[is - 1].child[k]); }
                else { tq.push_back(t.p[it - 1].child[k]); sq.push_back(is); }
            }
        }
    }
    return L;
}

// single_tree_traversal, tree_module.f90:401-487, parallel over targets; the
// per-target lists are concatenated in target order, as the reference emits them.
void single_tree_traversal(const Tree &t, double theta, int32_t thresh, const double *xs, const double *ys,
                           const double *zs, int32_t own, std::vector<int32_t> *pc, std::vector<int32_t> *pp) {
    (void)thresh;
    int nth = 1;
#ifdef _OPENMP
    nth = omp_get_max_threads();
#endif
    int32_t chunk = std::max<int32_t>(1, (own + 8 * nth - 1) / (8 * nth));
    int32_t nchunks = (own + chunk - 1) / chunk;
    std::vector<std::vector<int32_t>> cpc(nchunks), cpp(nchunks);
#pragma omp parallel for schedule(dynamic, 1)
    for (int32_t c = 0; c < nchunks; ++c) {
        std::vector<int32_t> q;
        q.reserve(t.p.size());
        for (int32_t i = c * chunk; i < std::min(own, (c + 1) * chunk); ++i) {
            q.clear();
            for (int j = 1; j <= 6; ++j) q.push_back(j);
            double x = xs[i], y = ys[i], z = zs[i];
            for (size_t cur = 0; cur < q.size(); ++cur) {
                int32_t is = q[cur];
                const Panel &S = t.p[is - 1];
                if (!(S.count() > 0)) continue;
                double dist = clamp_acos(x * t.cx[is - 1] + y * t.cy[is - 1] + z * t.cz[is - 1]);
                double sep = S.radius / dist;
                if (dist > 0 && sep < theta) { cpc[c].push_back(i + 1); cpc[c].push_back(is); }
                else if (S.is_leaf) { cpp[c].push_back(i + 1); cpp[c].push_back(is); }
                else for (int k = 0; k < 4; ++k) q.push_back(S.child[k]);
            }
        }
    }
    pc->clear(); pp->clear();
    for (int32_t c = 0; c < nchunks; ++c) {
        pc->insert(pc->end(), cpc[c].begin(), cpc[c].end());
        pp->insert(pp->end(), cpp[c].begin(), cpp[c].end());
    }
}

// contains_point, tree_module.f90:39-56.
static bool contains_point(const Panel &q, double x, double y, double z) {
    int f = face_from_xyz(x, y, z);
    if (f != q.face) return false;
    double xi, eta;
    face_xieta(x, y, z, f, &xi, &eta);
    return xi >= q.min_xi && xi < q.max_xi && eta >= q.min_eta && eta < q.max_eta;
}

// assign_points_to_panels, tree_module.f90:249-273.  Returns 0 or -(point id)
// for a point that lies in no panel (where the reference walks off the array).
int assign_points_to_panels(const Tree &t, const double *xs, const double *ys, const double *zs, int32_t own,
                            int32_t *pp, int32_t nlev) {
    int bad = 0;
    int32_t np = (int32_t)t.p.size();
#pragma omp parallel for schedule(static)
    for (int32_t i = 0; i < own; ++i) {
        int32_t level = 1, j = 1;
        for (;;) {
            if (j == -1) break;
            if (j > np || level > nlev) {
#pragma omp critical
                bad = bad ? bad : -(i + 1);
                break;
            }
            if (contains_point(t.p[j - 1], xs[i], ys[i], zs[i])) {
                pp[(size_t)(level - 1) + (size_t)nlev * i] = j;
                ++level;
                j = t.p[j - 1].child[0];
            } else {
                ++j;
            }
        }
    }
    return bad;
}

}  // namespace sal
