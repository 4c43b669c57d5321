// Host-only part of the C ABI: errors and the tree_module.f90 mirrors.
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/salgpu.h"
#include "sal_internal.hpp"

namespace sal {
static thread_local std::string g_last_error;
int set_error(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}
}  // namespace sal

using namespace sal;

struct sal_tree : Tree {};

extern "C" const char *sal_last_error(void) { return g_last_error.c_str(); }

extern "C" void sal_free(void *p) { std::free(p); }

static int32_t *copy_out(const std::vector<int32_t> &v) {
    int32_t *p = (int32_t *)std::malloc(std::max<size_t>(1, v.size()) * sizeof(int32_t));
    if (p && !v.empty()) std::memcpy(p, v.data(), v.size() * sizeof(int32_t));
    return p;
}

extern "C" int sal_tree_traverse(const double *xs, const double *ys, const double *zs, int32_t n, int32_t thresh,
                                 sal_tree **out) {
    if (!xs || !ys || !zs || !out) return set_error(SAL_EINVAL, "null argument");
    if (n < 0) return set_error(SAL_EINVAL, "negative point_count");
    if (thresh < 2) return set_error(SAL_EINVAL, "cluster_thresh must be >= 2");
    Tree *t = tree_build(xs, ys, zs, n, thresh);
    sal_tree *s = new sal_tree();
    static_cast<Tree &>(*s) = std::move(*t);
    delete t;
    *out = s;
    return SAL_OK;
}

extern "C" int sal_tree_import(int32_t np, const int32_t *ints9, const double *dbl7, const int64_t *pt_off,
                               const int32_t *pt_idx, int32_t n, const double *xs, const double *ys, const double *zs,
                               sal_tree **out) {
    if (!ints9 || !dbl7 || !pt_off || !pt_idx || !xs || !ys || !zs || !out) return set_error(SAL_EINVAL, "null argument");
    if (np < 6) return set_error(SAL_EINVAL, "a cubed-sphere tree has at least 6 panels");
    std::string err;
    Tree *t = tree_import(np, ints9, dbl7, pt_off, pt_idx, n, xs, ys, zs, &err);
    if (!t) return set_error(SAL_EINVAL, err);
    sal_tree *s = new sal_tree();
    static_cast<Tree &>(*s) = std::move(*t);
    delete t;
    *out = s;
    return SAL_OK;
}

extern "C" int sal_tree_info(const sal_tree *t, int32_t *np, int64_t *total, int32_t *max_level) {
    if (!t) return set_error(SAL_EINVAL, "null tree");
    if (np) *np = (int32_t)t->p.size();
    if (total) {
        int64_t s = 0;
        for (auto &q : t->p) s += q.count();
        *total = s;
    }
    if (max_level) *max_level = t->max_level();
    return SAL_OK;
}

extern "C" int sal_tree_export(const sal_tree *t, int32_t *I, double *D, int64_t *off, int32_t *idx) {
    if (!t || !I || !D || !off) return set_error(SAL_EINVAL, "null argument");
    int64_t o = 0;
    for (size_t k = 0; k < t->p.size(); ++k) {
        const Panel &q = t->p[k];
        int32_t *a = I + 9 * k;
        a[0] = q.level; a[1] = q.is_leaf; a[2] = q.id; a[3] = q.parent;
        for (int j = 0; j < 4; ++j) a[4 + j] = q.child[j];
        a[8] = q.face;
        double *b = D + 7 * k;
        b[0] = q.min_xi; b[1] = q.mid_xi; b[2] = q.max_xi; b[3] = q.min_eta; b[4] = q.mid_eta; b[5] = q.max_eta;
        b[6] = q.radius;
        off[k] = o;
        if (idx) {
            std::vector<int32_t> v = t->points_inside((int32_t)k + 1);
            std::memcpy(idx + o, v.data(), v.size() * sizeof(int32_t));
        }
        o += q.count();
    }
    off[t->p.size()] = o;
    return SAL_OK;
}

extern "C" int sal_tree_destroy(sal_tree *t) {
    delete t;
    return SAL_OK;
}

extern "C" int sal_dual_tree_traversal(const sal_tree *t, double theta, int32_t thresh, int32_t **list,
                                       int64_t *count) {
    if (!t || !list || !count) return set_error(SAL_EINVAL, "null argument");
    std::vector<int32_t> L = dual_tree_traversal(*t, theta, thresh);
    *list = copy_out(L);
    if (!*list) return set_error(SAL_ENOMEM, "out of host memory");
    *count = (int64_t)(L.size() / 3);
    return SAL_OK;
}

extern "C" int sal_tree_traverse_device(const double *xs, const double *ys, const double *zs, int32_t n,
                                        int32_t thresh, int32_t device, sal_tree **out) {
    if (!xs || !ys || !zs || !out) return set_error(SAL_EINVAL, "null argument");
    if (n < 0) return set_error(SAL_EINVAL, "negative point_count");
    if (thresh < 2) return set_error(SAL_EINVAL, "cluster_thresh must be >= 2");
    Tree *t = nullptr;
    if (int rc = tree_build_device(xs, ys, zs, n, thresh, device, &t)) return rc;
    sal_tree *s = new sal_tree();
    static_cast<Tree &>(*s) = std::move(*t);
    delete t;
    *out = s;
    return SAL_OK;
}

extern "C" int sal_dual_tree_traversal_device(const sal_tree *t, double theta, int32_t thresh, int32_t device,
                                              int32_t **list, int64_t *count) {
    if (!t || !list || !count) return set_error(SAL_EINVAL, "null argument");
    std::vector<int32_t> L;
    if (int rc = dual_tree_traversal_device(*t, theta, thresh, device, &L)) return rc;
    *list = copy_out(L);
    if (!*list) return set_error(SAL_ENOMEM, "out of host memory");
    *count = (int64_t)(L.size() / 3);
    return SAL_OK;
}

extern "C" int sal_single_tree_traversal(const sal_tree *t, double theta, int32_t thresh, const double *xs,
                                         const double *ys, const double *zs, int32_t own, int32_t **pc,
                                         int64_t *npc, int32_t **pp, int64_t *npp) {
    if (!t || !xs || !ys || !zs || !pc || !npc || !pp || !npp) return set_error(SAL_EINVAL, "null argument");
    std::vector<int32_t> a, b;
    single_tree_traversal(*t, theta, thresh, xs, ys, zs, own, &a, &b);
    *pc = copy_out(a);
    *pp = copy_out(b);
    if (!*pc || !*pp) return set_error(SAL_ENOMEM, "out of host memory");
    *npc = (int64_t)(a.size() / 2);
    *npp = (int64_t)(b.size() / 2);
    return SAL_OK;
}

extern "C" int sal_assign_points_to_panels(const sal_tree *t, const double *xs, const double *ys, const double *zs,
                                           int32_t own, int32_t *pp, int32_t nlev) {
    if (!t || !xs || !ys || !zs || !pp) return set_error(SAL_EINVAL, "null argument");
    for (int64_t i = 0; i < (int64_t)own * nlev; ++i) pp[i] = -1;
    int rc = assign_points_to_panels(*t, xs, ys, zs, own, pp, nlev);
    if (rc) return set_error(SAL_EINVAL, "point " + std::to_string(-rc) + " lies in no panel");
    return SAL_OK;
}
