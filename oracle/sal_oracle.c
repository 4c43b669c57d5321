/*
 * sal_oracle.c -- CPU restatement of cygnari/sal-fort's SAL-gradient treecode.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA product path:
 * it is called from tests/, from __graft_entry__.smoke() and from bench.py's
 * cpu_baseline leg, and nothing in the product links or executes it.
 *
 * Parity status: UNPINNED against the reference's own outputs.  The reference
 * ships no tests, fixtures or golden vectors, and it is Fortran 90 + MPI, for
 * which no compiler exists in this image.  This restatement is pinned instead by
 * mathematical known-answer tests (geometry round trips, BLI polynomial
 * exactness), by an FP64 direct O(N^2) sum, and by convergence of the treecode to
 * that direct sum.
 *
 * Every routine follows the reference's operation order literally (left-to-right
 * Fortran evaluation, no FMA contraction: build with -O2 -ffp-contract=off
 * -fno-fast-math), so that the singular self pair (s == t) rounds exactly as the
 * reference's does.  Indices stored in panels, lists and points_panels are
 * 1-based, as in the Fortran; C arrays of point data are 0-based.
 *
 * Deviations from the reference, all of them bounds fixes that do not change a
 * result the reference produces without overflowing:
 *   - tree_traverse's panel array, the DTT queue and the STT temp list grow on
 *     demand instead of being sized N, 64*npanels and 128*N without checks
 *     (tree_module.f90:72, :288-290, :414);
 *   - assign_points_to_panels stops with an error instead of running past the
 *     panel array when a point lies in no panel (tree_module.f90:260-271);
 *   - tree_traverse stops refining at level 40 (identical points would refine
 *     forever in the reference, tree_module.f90:127-130).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define OR_MAX_LEVEL 40

/* ------------------------------------------------------------------------- */
/* cube_sphere_module.f90                                                     */
/* ------------------------------------------------------------------------- */

/* face_from_xyz, cube_sphere_module.f90:7-35: argmax |coord| with sign, ties
 * to x then y. */
int or_face_from_xyz(double x, double y, double z)
{
    double ax = fabs(x), ay = fabs(y), az = fabs(z);
    if (ax >= ay && ax >= az) return (x >= 0) ? 1 : 3;
    if (ay >= ax && ay >= az) return (y >= 0) ? 2 : 4;
    return (z >= 0) ? 5 : 6;
}

/* xieta_from_xyz, cube_sphere_module.f90:38-61 (face always supplied). */
void or_xieta_from_xyz(double x, double y, double z, double *xi, double *eta, int face)
{
    if (face == 1) { *xi = atan(y / x); *eta = atan(z / x); }
    else if (face == 2) { *xi = atan(-x / y); *eta = atan(z / y); }
    else if (face == 3) { *xi = atan(y / x); *eta = atan(-z / x); }
    else if (face == 4) { *xi = atan(-x / y); *eta = atan(-z / y); }
    else if (face == 5) { *xi = atan(y / z); *eta = atan(-x / z); }
    else if (face == 6) { *xi = atan(-y / z); *eta = atan(-x / z); }
}

/* xyz_from_xieta, cube_sphere_module.f90:64-95. */
void or_xyz_from_xieta(double *x, double *y, double *z, double xi, double eta, int face)
{
    double ax = tan(xi), ay = tan(eta);
    if (face == 1) { *x = 1.0 / sqrt(1 + ax * ax + ay * ay); *y = ax * *x; *z = ay * *x; }
    else if (face == 2) { *y = 1.0 / sqrt(1 + ax * ax + ay * ay); *x = -ax * *y; *z = ay * *y; }
    else if (face == 3) { *x = -1.0 / sqrt(1 + ax * ax + ay * ay); *y = ax * *x; *z = -ay * *x; }
    else if (face == 4) { *y = -1.0 / sqrt(1 + ax * ax + ay * ay); *x = -ax * *y; *z = -ay * *y; }
    else if (face == 5) { *z = 1.0 / sqrt(1 + ax * ax + ay * ay); *x = -ay * *z; *y = ax * *z; }
    else { *z = -1.0 / sqrt(1 + ax * ax + ay * ay); *x = -ay * *z; *y = -ax * *z; }
}

/* ------------------------------------------------------------------------- */
/* bli_module.f90                                                             */
/* ------------------------------------------------------------------------- */

/* bli_coeffs, bli_module.f90:6-26. */
static void bli_coeffs(double *c, int degree)
{
    if (degree == 0) { c[0] = 1.0; return; }
    for (int i = 1; i <= degree + 1; ++i) {
        double s = ((i + 1) % 2 == 0) ? 1.0 : -1.0; /* (-1)**(i+1) */
        if (i == 1) c[i - 1] = 0.5;
        else if (i == degree + 1) c[i - 1] = 0.5 * s;
        else c[i - 1] = s;
    }
}

/* bli_interp_points_shift, bli_module.f90:28-48: Chebyshev 2nd-kind nodes,
 * descending from max_x to min_x. */
void or_bli_interp_points_shift(double *pts, double min_x, double max_x, int degree)
{
    double pi = 4.0 * atan(1.0);
    double x_range = 0.5 * (max_x - min_x);
    double x_shift = 0.5 * (max_x + min_x);
    if (degree == 0) { pts[0] = x_shift; return; }
    for (int i = 1; i <= degree + 1; ++i)
        pts[i - 1] = cos(pi / degree * (double)(i - 1)) * x_range + x_shift;
}

/* interp_vals_bli, bli_module.f90:50-113.  vals is (d+1)x(d+1) column-major:
 * vals[i + j*(d+1)] = vals(i+1, j+1) = xi_basis(i+1) * eta_basis(j+1). */
void or_interp_vals_bli(double *vals, double xi, double eta, double min_xi, double max_xi,
                        double min_eta, double max_eta, int degree)
{
    int n = degree + 1;
    double xs[64], es[64], cf[64], fx[64], fe[64];
    or_bli_interp_points_shift(xs, min_xi, max_xi, degree);
    or_bli_interp_points_shift(es, min_eta, max_eta, degree);
    bli_coeffs(cf, degree);
    for (int i = 0; i < n; ++i) { fx[i] = 0.0; fe[i] = 0.0; }
    int found_xi = 0, found_eta = 0;
    for (int i = 0; i < n; ++i) {
        if (fabs(xi - xs[i]) < 1.0e-16) { found_xi = 1; fx[i] = 1.0; }
        if (fabs(eta - es[i]) < 1.0e-16) { found_eta = 1; fe[i] = 1.0; }
    }
    if (!found_xi) {
        double denom = 0.0;
        for (int i = 0; i < n; ++i) { double v = cf[i] / (xi - xs[i]); fx[i] = v; denom = denom + v; }
        for (int i = 0; i < n; ++i) fx[i] = fx[i] / denom;
    }
    if (!found_eta) {
        double denom = 0.0;
        for (int i = 0; i < n; ++i) { double v = cf[i] / (eta - es[i]); fe[i] = v; denom = denom + v; }
        for (int i = 0; i < n; ++i) fe[i] = fe[i] / denom;
    }
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) vals[i + j * n] = fx[i] * fe[j];
}

/* ------------------------------------------------------------------------- */
/* fast_sum_module.f90:9-31 -- the SAL Green's-function gradient              */
/* ------------------------------------------------------------------------- */

void or_sal_grad_gfunc(double tx, double ty, double tz, double sx, double sy, double sz,
                       double *sal_x, double *sal_y)
{
    double cons = -2.343256857908601e-9;
    *sal_x = 0.0;
    *sal_y = 0.0;
    if ((fabs(tz - 1.0) > 1e-15) && (fabs(tz + 1.0) > 1e-15)) {
        double g = tx * sx + ty * sy + tz * sz;
        g = g < 1.0 ? g : 1.0;      /* MIN(.,1) */
        g = g > -1.0 ? g : -1.0;    /* MAX(.,-1) */
        double mp = 2.0 - 2.0 * g;
        double sqp = sqrt(mp);
        double p1 = (1.0 - 6.21196) / (sqp * mp + 1e-16);
        double p2 = (2.7 + 6.0) * (2.0 * g + sqp) / (2.0 * (g * g - 1.0) + 1e-16);
        double val = (p1 + p2) * cons;
        double x32 = tz * tz;
        double mp2 = sqrt(1.0 - x32);
        *sal_y = (sz * (1.0 - x32) - tz * (tx * sx + ty * sy)) / mp2 * val;
        *sal_x = (tx * sy - ty * sx) / mp2 * val;
    }
}

/* ------------------------------------------------------------------------- */
/* tree_module.f90 -- cube_panel and the cubed-sphere quadtree                */
/* ------------------------------------------------------------------------- */

typedef struct {
    int level, is_leaf, id, parent, child[4], face;
    double min_xi, mid_xi, max_xi, min_eta, mid_eta, max_eta, radius;
    int *pts;  /* points_inside, 1-based point ids */
    int count; /* panel_point_count */
} or_panel;

typedef struct {
    int np, cap;
    or_panel *p; /* p[k] is panel id k+1 */
    int error;
} or_tree;

static or_panel *tree_push(or_tree *t)
{
    if (t->np == t->cap) {
        int nc = t->cap ? 2 * t->cap : 64;
        t->p = (or_panel *)realloc(t->p, (size_t)nc * sizeof(or_panel));
        t->cap = nc;
    }
    or_panel *q = &t->p[t->np++];
    memset(q, 0, sizeof(*q));
    q->is_leaf = 1;
    q->parent = -1;
    q->child[0] = q->child[1] = q->child[2] = q->child[3] = -1;
    return q;
}

/* contains_point, tree_module.f90:39-56. */
static int contains_point(const or_panel *p, double x, double y, double z)
{
    int face = or_face_from_xyz(x, y, z);
    if (face != p->face) return 0;
    double xi, eta;
    or_xieta_from_xyz(x, y, z, &xi, &eta, face);
    return (xi >= p->min_xi) && (xi < p->max_xi) && (eta >= p->min_eta) && (eta < p->max_eta);
}

/* tree_traverse, tree_module.f90:59-246.  xs/ys/zs are 0-based arrays of n
 * points; panels store 1-based point ids. */
or_tree *or_tree_traverse(int n, const double *xs, const double *ys, const double *zs, int cluster_thresh)
{
    or_tree *t = (or_tree *)calloc(1, sizeof(or_tree));
    double pi = 4.0 * atan(1.0);
    for (int i = 1; i <= 6; ++i) { /* :76-88 */
        or_panel *p = tree_push(t);
        p->id = i; p->face = i;
        p->min_xi = -pi / 4.0; p->mid_xi = 0.0; p->max_xi = pi / 4.0;
        p->min_eta = -pi / 4.0; p->mid_eta = 0.0; p->max_eta = pi / 4.0;
        p->pts = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
        p->count = 0;
    }
    for (int i = 1; i <= n; ++i) { /* :93-101 */
        int face = or_face_from_xyz(xs[i - 1], ys[i - 1], zs[i - 1]);
        or_panel *p = &t->p[face - 1];
        p->pts[p->count++] = i;
    }
    int i = 1; /* :126-220 */
    while (i <= t->np) {
        int count = t->p[i - 1].count;
        if (count >= cluster_thresh && t->p[i - 1].is_leaf && t->p[i - 1].level < OR_MAX_LEVEL) {
            int pc = t->np;
            for (int j = 0; j < 4; ++j) tree_push(t);
            or_panel *par = &t->p[i - 1]; /* re-fetch after realloc */
            par->is_leaf = 0;
            double min_xi = par->min_xi, mid_xi = par->mid_xi, max_xi = par->max_xi;
            double min_eta = par->min_eta, mid_eta = par->mid_eta, max_eta = par->max_eta;
            for (int j = 1; j <= 4; ++j) {
                or_panel *c = &t->p[pc + j - 1];
                c->parent = i; c->level = par->level + 1; c->face = par->face; c->id = pc + j;
                c->pts = (int *)malloc(sizeof(int) * (size_t)count);
                c->count = 0;
            }
            or_panel *c1 = &t->p[pc], *c2 = &t->p[pc + 1], *c3 = &t->p[pc + 2], *c4 = &t->p[pc + 3];
            c1->min_xi = min_xi; c1->min_eta = min_eta; c1->max_xi = mid_xi; c1->max_eta = mid_eta;
            c1->mid_xi = 0.5 * (min_xi + mid_xi); c1->mid_eta = 0.5 * (min_eta + mid_eta);
            c2->min_xi = mid_xi; c2->min_eta = min_eta; c2->max_xi = max_xi; c2->max_eta = mid_eta;
            c2->mid_xi = 0.5 * (mid_xi + max_xi); c2->mid_eta = 0.5 * (min_eta + mid_eta);
            c3->min_xi = mid_xi; c3->min_eta = mid_eta; c3->max_xi = max_xi; c3->max_eta = max_eta;
            c3->mid_xi = 0.5 * (mid_xi + max_xi); c3->mid_eta = 0.5 * (mid_eta + max_eta);
            c4->min_xi = min_xi; c4->min_eta = mid_eta; c4->max_xi = mid_xi; c4->max_eta = max_eta;
            c4->mid_xi = 0.5 * (min_xi + mid_xi); c4->mid_eta = 0.5 * (mid_eta + max_eta);
            for (int j = 0; j < 4; ++j) par->child[j] = pc + j + 1;
            for (int j = 0; j < par->count; ++j) { /* :175-197 */
                int idx = par->pts[j];
                double xi, eta;
                or_xieta_from_xyz(xs[idx - 1], ys[idx - 1], zs[idx - 1], &xi, &eta, par->face);
                int which;
                if (xi < mid_xi) which = (eta < mid_eta) ? 1 : 4;
                else which = (eta < mid_eta) ? 2 : 3;
                or_panel *c = &t->p[pc + which - 1];
                c->pts[c->count++] = idx;
            }
        }
        ++i;
    }
    for (int k = 0; k < t->np; ++k) { /* :224-244 */
        or_panel *p = &t->p[k];
        double x1, x2, x3, y1, y2, y3, d1, d2, d3, d4, v;
        or_xyz_from_xieta(&x1, &x2, &x3, p->mid_xi, p->mid_eta, p->face);
        or_xyz_from_xieta(&y1, &y2, &y3, p->min_xi, p->min_eta, p->face);
        v = x1 * y1 + x2 * y2 + x3 * y3; v = v < 1.0 ? v : 1.0; v = v > -1.0 ? v : -1.0; d1 = acos(v);
        or_xyz_from_xieta(&y1, &y2, &y3, p->min_xi, p->max_eta, p->face);
        v = x1 * y1 + x2 * y2 + x3 * y3; v = v < 1.0 ? v : 1.0; v = v > -1.0 ? v : -1.0; d2 = acos(v);
        or_xyz_from_xieta(&y1, &y2, &y3, p->max_xi, p->max_eta, p->face);
        v = x1 * y1 + x2 * y2 + x3 * y3; v = v < 1.0 ? v : 1.0; v = v > -1.0 ? v : -1.0; d3 = acos(v);
        or_xyz_from_xieta(&y1, &y2, &y3, p->max_xi, p->min_eta, p->face);
        v = x1 * y1 + x2 * y2 + x3 * y3; v = v < 1.0 ? v : 1.0; v = v > -1.0 ? v : -1.0; d4 = acos(v);
        double r = d1;
        if (d2 > r) r = d2;
        if (d3 > r) r = d3;
        if (d4 > r) r = d4;
        p->radius = r;
    }
    return t;
}

void or_tree_free(or_tree *t)
{
    if (!t) return;
    for (int k = 0; k < t->np; ++k) free(t->p[k].pts);
    free(t->p);
    free(t);
}

int or_tree_npanels(const or_tree *t) { return t->np; }

/* Flattened export.  ints: 9 per panel (level, is_leaf, id, parent, child1..4,
 * face); dbl: 7 per panel (min_xi, mid_xi, max_xi, min_eta, mid_eta, max_eta,
 * radius); pt_off: np+1 offsets into pt_idx (1-based point ids). */
long long or_tree_total_points(const or_tree *t)
{
    long long s = 0;
    for (int k = 0; k < t->np; ++k) s += t->p[k].count;
    return s;
}

void or_tree_export(const or_tree *t, int *ints, double *dbl, long long *pt_off, int *pt_idx)
{
    long long off = 0;
    for (int k = 0; k < t->np; ++k) {
        const or_panel *p = &t->p[k];
        int *I = ints + 9 * k;
        I[0] = p->level; I[1] = p->is_leaf; I[2] = p->id; I[3] = p->parent;
        I[4] = p->child[0]; I[5] = p->child[1]; I[6] = p->child[2]; I[7] = p->child[3]; I[8] = p->face;
        double *D = dbl + 7 * k;
        D[0] = p->min_xi; D[1] = p->mid_xi; D[2] = p->max_xi;
        D[3] = p->min_eta; D[4] = p->mid_eta; D[5] = p->max_eta; D[6] = p->radius;
        pt_off[k] = off;
        if (pt_idx) memcpy(pt_idx + off, p->pts, sizeof(int) * (size_t)p->count);
        off += p->count;
    }
    pt_off[t->np] = off;
}

/* ------------------------------------------------------------------------- */
/* Interaction lists                                                          */
/* ------------------------------------------------------------------------- */

typedef struct { int n, cap; int *v; } ivec;
static void iv_push(ivec *a, int x)
{
    if (a->n == a->cap) { a->cap = a->cap ? 2 * a->cap : 1024; a->v = (int *)realloc(a->v, sizeof(int) * (size_t)a->cap); }
    a->v[a->n++] = x;
}

/* dual_tree_traversal, tree_module.f90:277-398.  Returns the list as triplets
 * (index_target, index_source, interact_type); *out must be freed with
 * or_free. */
int or_dual_tree_traversal(const or_tree *t, double theta, int thresh, int **out)
{
    ivec tq = {0, 0, 0}, sq = {0, 0, 0}, L = {0, 0, 0};
    for (int i = 1; i <= 6; ++i)
        for (int j = 1; j <= 6; ++j) { iv_push(&tq, i); iv_push(&sq, j); }
    int cur = 0;
    while (cur < tq.n) {
        int it = tq.v[cur], is = sq.v[cur];
        const or_panel *T = &t->p[it - 1], *S = &t->p[is - 1];
        int ct = T->count, cs = S->count;
        if (ct > 0 && cs > 0) {
            double x1t, x2t, x3t, x1s, x2s, x3s;
            or_xyz_from_xieta(&x1t, &x2t, &x3t, T->mid_xi, T->mid_eta, T->face);
            or_xyz_from_xieta(&x1s, &x2s, &x3s, S->mid_xi, S->mid_eta, S->face);
            double v = x1t * x1s + x2t * x2s + x3t * x3s;
            v = v > -1.0 ? v : -1.0; v = v < 1.0 ? v : 1.0;
            double dist = acos(v);
            double sep = (T->radius + S->radius) / dist;
            if (dist > 0 && sep < theta) {
                int ty = 0;
                if (ct > thresh) ty += 2;
                if (cs > thresh) ty += 1;
                iv_push(&L, it); iv_push(&L, is); iv_push(&L, ty);
            } else if (ct < thresh && cs < thresh) {
                iv_push(&L, it); iv_push(&L, is); iv_push(&L, 0);
            } else if (T->is_leaf && S->is_leaf) {
                iv_push(&L, it); iv_push(&L, is); iv_push(&L, 0);
            } else if (T->is_leaf) {
                for (int c = 0; c < 4; ++c) { iv_push(&tq, it); iv_push(&sq, S->child[c]); }
            } else if (S->is_leaf) {
                for (int c = 0; c < 4; ++c) { iv_push(&sq, is); iv_push(&tq, T->child[c]); }
            } else if (ct >= cs) {
                for (int c = 0; c < 4; ++c) { iv_push(&sq, is); iv_push(&tq, T->child[c]); }
            } else {
                for (int c = 0; c < 4; ++c) { iv_push(&tq, it); iv_push(&sq, S->child[c]); }
            }
        }
        ++cur;
    }
    free(tq.v); free(sq.v);
    *out = L.v;
    return L.n / 3;
}

/* single_tree_traversal, tree_module.f90:401-487.  Produces the pc and pp
 * lists as pairs (index_target = point id, index_source = panel id). */
void or_single_tree_traversal(const or_tree *t, double theta, int thresh, const double *xs,
                              const double *ys, const double *zs, int own_points,
                              int **pc_out, int *npc, int **pp_out, int *npp)
{
    (void)thresh;
    ivec PC = {0, 0, 0}, PP = {0, 0, 0};
    int *q = (int *)malloc(sizeof(int) * (size_t)(t->np + 8));
    for (int i = 1; i <= own_points; ++i) {
        int n = 6;
        for (int j = 0; j < 6; ++j) q[j] = j + 1;
        int cur = 0;
        double x1t = xs[i - 1], x2t = ys[i - 1], x3t = zs[i - 1];
        while (cur < n) {
            int is = q[cur];
            const or_panel *S = &t->p[is - 1];
            if (S->count > 0) {
                double x1s, x2s, x3s;
                or_xyz_from_xieta(&x1s, &x2s, &x3s, S->mid_xi, S->mid_eta, S->face);
                double v = x1t * x1s + x2t * x2s + x3t * x3s;
                v = v > -1.0 ? v : -1.0; v = v < 1.0 ? v : 1.0;
                double dist = acos(v);
                double sep = S->radius / dist;
                int ws = (dist > 0) && (sep < theta);
                if (ws) { iv_push(&PC, i); iv_push(&PC, is); }
                else if (S->is_leaf) { iv_push(&PP, i); iv_push(&PP, is); }
                else { for (int c = 0; c < 4; ++c) q[n++] = S->child[c]; }
            }
            ++cur;
        }
    }
    free(q);
    *pc_out = PC.v; *npc = PC.n / 2;
    *pp_out = PP.v; *npp = PP.n / 2;
}

/* assign_points_to_panels, tree_module.f90:249-273.  points_panels is
 * (nlev x own_points) column-major, filled by the caller with -1.  Returns 0,
 * or -i when point i lies in no panel (the reference runs off the array). */
int or_assign_points_to_panels(const or_tree *t, const double *xs, const double *ys, const double *zs,
                               int own_points, int *points_panels, int nlev)
{
    for (int i = 1; i <= own_points; ++i) {
        int level = 1, j = 1;
        for (;;) {
            if (j == -1) break;
            if (j > t->np || level > nlev) return -i;
            if (contains_point(&t->p[j - 1], xs[i - 1], ys[i - 1], zs[i - 1])) {
                points_panels[(size_t)(level - 1) + (size_t)nlev * (size_t)(i - 1)] = j;
                ++level;
                j = t->p[j - 1].child[0];
            } else {
                ++j;
            }
        }
    }
    return 0;
}

void or_free(void *p) { free(p); }

/* ------------------------------------------------------------------------- */
/* fast_sum_module.f90 -- the DTT evaluator                                   */
/* ------------------------------------------------------------------------- */

/* pp_interact, fast_sum_module.f90:33-73. */
static void pp_interact(double *slon, double *slat, const or_panel *T, const or_panel *S, const double *xs,
                        const double *ys, const double *zs, const double *area, const double *ssh)
{
    for (int i = 0; i < T->count; ++i) {
        int ti = T->pts[i] - 1;
        double tx = xs[ti], ty = ys[ti], tz = zs[ti];
        for (int j = 0; j < S->count; ++j) {
            int sj = S->pts[j] - 1;
            double sx, sy;
            or_sal_grad_gfunc(tx, ty, tz, xs[sj], ys[sj], zs[sj], &sx, &sy);
            slon[ti] = slon[ti] + sx * area[sj] * ssh[sj];
            slat[ti] = slat[ti] + sy * area[sj] * ssh[sj];
        }
    }
}

/* Proxy weights of a source panel: the loop at fast_sum_module.f90:99-111
 * (identical in cc_interact :229-241).  W is (d+1)x(d+1) column-major. */
static void source_weights(double *W, const or_panel *S, const double *xs, const double *ys, const double *zs,
                           const double *area, const double *ssh, int d)
{
    int n = d + 1;
    double bv[64 * 64];
    for (int k = 0; k < n * n; ++k) W[k] = 0.0;
    for (int i = 0; i < S->count; ++i) {
        int sj = S->pts[i] - 1;
        double xi, eta;
        or_xieta_from_xyz(xs[sj], ys[sj], zs[sj], &xi, &eta, S->face);
        or_interp_vals_bli(bv, xi, eta, S->min_xi, S->max_xi, S->min_eta, S->max_eta, d);
        for (int k = 0; k < n; ++k)
            for (int j = 0; j < n; ++j) W[j + k * n] = W[j + k * n] + bv[j + k * n] * area[sj] * ssh[sj];
    }
}

/* pc_interact, fast_sum_module.f90:75-131. */
static void pc_interact(double *slon, double *slat, const or_panel *T, const or_panel *S, const double *xs,
                        const double *ys, const double *zs, const double *area, const double *ssh, int d)
{
    int n = d + 1;
    double cx_[64], ce_[64], W[64 * 64];
    or_bli_interp_points_shift(cx_, S->min_xi, S->max_xi, d);
    or_bli_interp_points_shift(ce_, S->min_eta, S->max_eta, d);
    source_weights(W, S, xs, ys, zs, area, ssh, d);
    for (int i = 0; i < T->count; ++i) {
        int ti = T->pts[i] - 1;
        double tx = xs[ti], ty = ys[ti], tz = zs[ti];
        for (int k = 0; k < n; ++k) {
            double eta = ce_[k];
            for (int j = 0; j < n; ++j) {
                double cx, cy, cz, sx, sy;
                or_xyz_from_xieta(&cx, &cy, &cz, cx_[j], eta, S->face);
                or_sal_grad_gfunc(tx, ty, tz, cx, cy, cz, &sx, &sy);
                slon[ti] = slon[ti] + sx * W[j + k * n];
                slat[ti] = slat[ti] + sy * W[j + k * n];
            }
        }
    }
}

/* Interpolation from target-panel proxies to target points, the loop at
 * fast_sum_module.f90:186-199 (identical in cc_interact :274-287). */
static void interp_to_targets(double *slon, double *slat, const or_panel *T, const double *xs, const double *ys,
                              const double *zs, const double *Px, const double *Py, int d)
{
    int n = d + 1;
    double bv[64 * 64];
    for (int i = 0; i < T->count; ++i) {
        int ti = T->pts[i] - 1;
        double xi, eta;
        or_xieta_from_xyz(xs[ti], ys[ti], zs[ti], &xi, &eta, T->face);
        or_interp_vals_bli(bv, xi, eta, T->min_xi, T->max_xi, T->min_eta, T->max_eta, d);
        for (int k = 0; k < n; ++k)
            for (int j = 0; j < n; ++j) {
                slon[ti] = slon[ti] + bv[j + k * n] * Px[j + k * n];
                slat[ti] = slat[ti] + bv[j + k * n] * Py[j + k * n];
            }
    }
}

/* cp_interact, fast_sum_module.f90:133-201. */
static void cp_interact(double *slon, double *slat, const or_panel *T, const or_panel *S, const double *xs,
                        const double *ys, const double *zs, const double *area, const double *ssh, int d)
{
    int n = d + 1;
    double cx_[64], ce_[64], Px[64 * 64], Py[64 * 64];
    or_bli_interp_points_shift(cx_, T->min_xi, T->max_xi, d);
    or_bli_interp_points_shift(ce_, T->min_eta, T->max_eta, d);
    for (int k = 0; k < n * n; ++k) { Px[k] = 0.0; Py[k] = 0.0; }
    for (int j = 0; j < n; ++j) {
        double eta = ce_[j];
        for (int i = 0; i < n; ++i) {
            double cx, cy, cz;
            or_xyz_from_xieta(&cx, &cy, &cz, cx_[i], eta, T->face);
            for (int k = 0; k < S->count; ++k) {
                int sj = S->pts[k] - 1;
                double sx, sy;
                or_sal_grad_gfunc(cx, cy, cz, xs[sj], ys[sj], zs[sj], &sx, &sy);
                Px[i + j * n] = Px[i + j * n] + sx * area[sj] * ssh[sj];
                Py[i + j * n] = Py[i + j * n] + sy * area[sj] * ssh[sj];
            }
        }
    }
    interp_to_targets(slon, slat, T, xs, ys, zs, Px, Py, d);
}

/* cc_interact, fast_sum_module.f90:204-288. */
static void cc_interact(double *slon, double *slat, const or_panel *T, const or_panel *S, const double *xs,
                        const double *ys, const double *zs, const double *area, const double *ssh, int d)
{
    int n = d + 1;
    double sxn[64], sen[64], txn[64], ten[64], W[64 * 64], Px[64 * 64], Py[64 * 64];
    or_bli_interp_points_shift(sxn, S->min_xi, S->max_xi, d);
    or_bli_interp_points_shift(sen, S->min_eta, S->max_eta, d);
    source_weights(W, S, xs, ys, zs, area, ssh, d);
    or_bli_interp_points_shift(txn, T->min_xi, T->max_xi, d);
    or_bli_interp_points_shift(ten, T->min_eta, T->max_eta, d);
    for (int k = 0; k < n * n; ++k) { Px[k] = 0.0; Py[k] = 0.0; }
    for (int j = 0; j < n; ++j) {
        for (int i = 0; i < n; ++i) {
            double cxt, cyt, czt;
            or_xyz_from_xieta(&cxt, &cyt, &czt, txn[i], ten[j], T->face);
            for (int l = 0; l < n; ++l) {
                for (int k = 0; k < n; ++k) {
                    double cxs, cys, czs, sx, sy;
                    or_xyz_from_xieta(&cxs, &cys, &czs, sxn[k], sen[l], S->face);
                    or_sal_grad_gfunc(cxt, cyt, czt, cxs, cys, czs, &sx, &sy);
                    Px[i + j * n] = Px[i + j * n] + sx * W[k + l * n];
                    Py[i + j * n] = Py[i + j * n] + sy * W[k + l * n];
                }
            }
        }
    }
    interp_to_targets(slon, slat, T, xs, ys, zs, Px, Py, d);
}

/* fast_sum, fast_sum_module.f90:291-332.  list holds ninter triplets
 * (target, source, type).  nranks > 1 emulates the MOD(i,P)==rank split with
 * one OpenMP thread per rank, each accumulating into a private copy, then a
 * sum in rank order (the Sum_Array step, code.f90:99-100).  Outputs are added
 * into slon/slat (intent(inout)). */
void or_fast_sum(double *slon, double *slat, const int *list, int ninter, const or_tree *t, const double *xs,
                 const double *ys, const double *zs, const double *area, const double *ssh, int n, int d,
                 int nranks)
{
    if (nranks < 1) nranks = 1;
    double *priv = NULL;
    if (nranks > 1) priv = (double *)calloc((size_t)nranks * 2 * (size_t)n, sizeof(double));
#pragma omp parallel for num_threads(nranks) schedule(static, 1) if (nranks > 1)
    for (int r = 0; r < nranks; ++r) {
        double *lon = nranks > 1 ? priv + (size_t)r * 2 * (size_t)n : slon;
        double *lat = nranks > 1 ? lon + n : slat;
        for (int i = 1; i <= ninter; ++i) {
            if (i % nranks != r) continue;
            int it = list[3 * (i - 1)], is = list[3 * (i - 1) + 1], ty = list[3 * (i - 1) + 2];
            const or_panel *T = &t->p[it - 1], *S = &t->p[is - 1];
            if (ty == 0) pp_interact(lon, lat, T, S, xs, ys, zs, area, ssh);
            else if (ty == 1) pc_interact(lon, lat, T, S, xs, ys, zs, area, ssh, d);
            else if (ty == 2) cp_interact(lon, lat, T, S, xs, ys, zs, area, ssh, d);
            else if (ty == 3) cc_interact(lon, lat, T, S, xs, ys, zs, area, ssh, d);
        }
    }
    if (nranks > 1) {
        for (int r = 0; r < nranks; ++r) {
            const double *lon = priv + (size_t)r * 2 * (size_t)n, *lat = lon + n;
            for (int k = 0; k < n; ++k) { slon[k] += lon[k]; slat[k] += lat[k]; }
        }
        free(priv);
    }
}


/* ------------------------------------------------------------------------- */
/* Cartesian target-side interpolation (the accuracy mode of the DTT path)    */
/* ------------------------------------------------------------------------- */

/* The reference kernel factors as G(t,s) = val(t.s) * [e_lon(t).s, e_lat(t).s]
 * with e_lon = (-ty, tx, 0)/sqrt(1-tz^2) and e_lat = (-tz tx, -tz ty,
 * 1-tz^2)/sqrt(1-tz^2) (fast_sum_module.f90:26-29).  cp_interact and
 * cc_interact evaluate G at target proxy nodes and interpolate the east/north
 * components, which lie in the proxies' own frames; near the poles those frames
 * rotate across a panel and the interpolant loses accuracy.  This mode instead
 * interpolates the frame-free vector u(x) = sum val(x.s) (s - x) w and projects
 * it onto the real target's frame.  cart_val is the scalar val of the kernel. */
static double cart_val(double tx, double ty, double tz, double sx, double sy, double sz)
{
    /* val of fast_sum_module.f90:20-25 with the removable singularity at the
     * antipode cancelled: with q = sqrt(mp) = |t - s|,
     *   2g + q = (2 - q)(1 + q)  and  2(g^2 - 1) = -q^2 (2 - q)(2 + q) / 2,
     * so p2 = -2 * 8.7 * (1 + q) / (q^2 (2 + q)).  p1 keeps its +1e-16. */
    double cons = -2.343256857908601e-9;
    double dx = sx - tx, dy = sy - ty, dz = sz - tz;
    double mp = dx * dx + dy * dy + dz * dz;
    double q = sqrt(mp);
    double p1 = (1.0 - 6.21196) / (q * mp + 1e-16);
    double p2 = -2.0 * (2.7 + 6.0) * (1.0 + q) / (mp * (2.0 + q) + 1e-16);
    return (p1 + p2) * cons;
}

static void cart_project_add(double *slon, double *slat, int ti, double tx, double ty, double tz,
                             double ux, double uy, double uz)
{
    if (!((fabs(tz - 1.0) > 1e-15) && (fabs(tz + 1.0) > 1e-15))) return;
    double x32 = tz * tz;
    double mp2 = sqrt(1.0 - x32);
    slon[ti] = slon[ti] + (tx * uy - ty * ux) / mp2;
    slat[ti] = slat[ti] + (uz * (1.0 - x32) - tz * (tx * ux + ty * uy)) / mp2;
}

static void cart_interp_to_targets(double *slon, double *slat, const or_panel *T, const double *xs,
                                   const double *ys, const double *zs, const double *U, int d)
{
    int n = d + 1;
    double bv[64 * 64];
    for (int i = 0; i < T->count; ++i) {
        int ti = T->pts[i] - 1;
        double xi, eta, ux = 0, uy = 0, uz = 0;
        or_xieta_from_xyz(xs[ti], ys[ti], zs[ti], &xi, &eta, T->face);
        or_interp_vals_bli(bv, xi, eta, T->min_xi, T->max_xi, T->min_eta, T->max_eta, d);
        for (int k = 0; k < n * n; ++k) {
            ux += bv[k] * U[3 * k]; uy += bv[k] * U[3 * k + 1]; uz += bv[k] * U[3 * k + 2];
        }
        cart_project_add(slon, slat, ti, xs[ti], ys[ti], zs[ti], ux, uy, uz);
    }
}

static void cp_interact_cart(double *slon, double *slat, const or_panel *T, const or_panel *S, const double *xs,
                             const double *ys, const double *zs, const double *area, const double *ssh, int d)
{
    int n = d + 1;
    double cx_[64], ce_[64], U[3 * 64 * 64];
    or_bli_interp_points_shift(cx_, T->min_xi, T->max_xi, d);
    or_bli_interp_points_shift(ce_, T->min_eta, T->max_eta, d);
    for (int k = 0; k < 3 * n * n; ++k) U[k] = 0.0;
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            double cx, cy, cz;
            or_xyz_from_xieta(&cx, &cy, &cz, cx_[i], ce_[j], T->face);
            double *u = U + 3 * (i + j * n);
            for (int k = 0; k < S->count; ++k) {
                int sj = S->pts[k] - 1;
                double v = cart_val(cx, cy, cz, xs[sj], ys[sj], zs[sj]) * (area[sj] * ssh[sj]);
                u[0] += v * (xs[sj] - cx); u[1] += v * (ys[sj] - cy); u[2] += v * (zs[sj] - cz);
            }
        }
    cart_interp_to_targets(slon, slat, T, xs, ys, zs, U, d);
}

static void cc_interact_cart(double *slon, double *slat, const or_panel *T, const or_panel *S, const double *xs,
                             const double *ys, const double *zs, const double *area, const double *ssh, int d)
{
    int n = d + 1;
    double sxn[64], sen[64], txn[64], ten[64], W[64 * 64], U[3 * 64 * 64];
    or_bli_interp_points_shift(sxn, S->min_xi, S->max_xi, d);
    or_bli_interp_points_shift(sen, S->min_eta, S->max_eta, d);
    source_weights(W, S, xs, ys, zs, area, ssh, d);
    or_bli_interp_points_shift(txn, T->min_xi, T->max_xi, d);
    or_bli_interp_points_shift(ten, T->min_eta, T->max_eta, d);
    for (int k = 0; k < 3 * n * n; ++k) U[k] = 0.0;
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            double cxt, cyt, czt;
            or_xyz_from_xieta(&cxt, &cyt, &czt, txn[i], ten[j], T->face);
            double *u = U + 3 * (i + j * n);
            for (int l = 0; l < n; ++l)
                for (int k = 0; k < n; ++k) {
                    double cxs, cys, czs;
                    or_xyz_from_xieta(&cxs, &cys, &czs, sxn[k], sen[l], S->face);
                    double v = cart_val(cxt, cyt, czt, cxs, cys, czs) * W[k + l * n];
                    u[0] += v * (cxs - cxt); u[1] += v * (cys - cyt); u[2] += v * (czs - czt);
                }
        }
    cart_interp_to_targets(slon, slat, T, xs, ys, zs, U, d);
}

/* fast_sum with CP/CC in the Cartesian form; PP and PC as the reference. */
void or_fast_sum_cart(double *slon, double *slat, const int *list, int ninter, const or_tree *t, const double *xs,
                      const double *ys, const double *zs, const double *area, const double *ssh, int n, int d,
                      int nthreads)
{
    if (nthreads < 1) nthreads = 1;
    double *priv = (double *)calloc((size_t)nthreads * 2 * (size_t)n, sizeof(double));
#pragma omp parallel for num_threads(nthreads) schedule(static, 1)
    for (int r = 0; r < nthreads; ++r) {
        double *lon = priv + (size_t)r * 2 * (size_t)n, *lat = lon + n;
        for (int i = 1; i <= ninter; ++i) {
            if (i % nthreads != r) continue;
            int it = list[3 * (i - 1)], is = list[3 * (i - 1) + 1], ty = list[3 * (i - 1) + 2];
            const or_panel *T = &t->p[it - 1], *S = &t->p[is - 1];
            if (ty == 0) pp_interact(lon, lat, T, S, xs, ys, zs, area, ssh);
            else if (ty == 1) pc_interact(lon, lat, T, S, xs, ys, zs, area, ssh, d);
            else if (ty == 2) cp_interact_cart(lon, lat, T, S, xs, ys, zs, area, ssh, d);
            else if (ty == 3) cc_interact_cart(lon, lat, T, S, xs, ys, zs, area, ssh, d);
        }
    }
    for (int r = 0; r < nthreads; ++r) {
        const double *lon = priv + (size_t)r * 2 * (size_t)n, *lat = lon + n;
        for (int k = 0; k < n; ++k) { slon[k] += lon[k]; slat[k] += lat[k]; }
    }
    free(priv);
}

/* ------------------------------------------------------------------------- */
/* mom6_fast_sum_module.f90 -- the STT evaluator                              */
/* ------------------------------------------------------------------------- */

/* proxy_source_compute, mom6_fast_sum_module.f90:33-74.  transposed=1 stores
 * basis_vals(k,l) at offset (k-1)(d+1)+l exactly as the reference (:63-70),
 * which pc_interact (:95-105) then reads as the weight of node (xi_l, eta_k)
 * -- a transpose.  transposed=0 stores basis_vals(l,k) there instead, the
 * orientation pc_interact expects.  Adds into weights (P*npanels). */
void or_proxy_source_compute(double *weights, const or_tree *t, const int *points_panels, int nlev,
                             const double *xs, const double *ys, const double *zs, const double *sshs,
                             const double *areas, int d, int point_count, int transposed, int nthreads)
{
    int n = d + 1;
    if (nthreads < 1) nthreads = 1;
    /* Threads own disjoint panel-id ranges (the panels' weights they write);
     * each walks every point in order, so every weight sums its points in the
     * reference's order whatever the thread count. */
#pragma omp parallel num_threads(nthreads)
    {
    int nth = omp_get_num_threads(), me = omp_get_thread_num();
    int lo = (int)((long long)t->np * me / nth) + 1, hi = (int)((long long)t->np * (me + 1) / nth);
    double bv[64 * 64];
    for (int i = 1; i <= point_count; ++i) {
        double x = xs[i - 1], y = ys[i - 1], z = zs[i - 1], a = areas[i - 1], h = sshs[i - 1];
        for (int j = 1; j <= nlev; ++j) {
            int it = points_panels[(size_t)(j - 1) + (size_t)nlev * (size_t)(i - 1)];
            if (it == -1) break;
            if (it < lo || it > hi) continue;
            const or_panel *P = &t->p[it - 1];
            size_t shift = (size_t)(it - 1) * (size_t)(n * n);
            double xi, eta;
            or_xieta_from_xyz(x, y, z, &xi, &eta, P->face);
            or_interp_vals_bli(bv, xi, eta, P->min_xi, P->max_xi, P->min_eta, P->max_eta, d);
            int offset = 0;
            for (int k = 1; k <= n; ++k)
                for (int l = 1; l <= n; ++l) {
                    offset = offset + 1;
                    double b = transposed ? bv[(k - 1) + (l - 1) * n] : bv[(l - 1) + (k - 1) * n];
                    weights[shift + offset - 1] = weights[shift + offset - 1] + b * a * h;
                }
        }
    }
    }
}

/* pc_compute + pc_interact, mom6_fast_sum_module.f90:153-174, :76-107.
 * pc holds npc pairs (target point id, source panel id). */
void or_pc_compute(double *slon, double *slat, const int *pc, int npc, const or_tree *t, const double *xs,
                   const double *ys, const double *zs, int d, const double *weights, int npoints, int nthreads)
{
    int n = d + 1;
    if (nthreads < 1) nthreads = 1;
    /* Threads own disjoint target-point ranges, as MPI ranks own points in
     * mom6_code.f90; each walks the whole list in order, so every target sums
     * its entries in list order whatever the thread count. */
#pragma omp parallel num_threads(nthreads)
    {
    int nth = omp_get_num_threads(), me = omp_get_thread_num();
    int lo = (int)((long long)npoints * me / nth) + 1, hi = (int)((long long)npoints * (me + 1) / nth);
    for (int e = 0; e < npc; ++e) {
        int it = pc[2 * e], is = pc[2 * e + 1];
        if (it < lo || it > hi) continue;
        const or_panel *S = &t->p[is - 1];
        const double *W = weights + (size_t)(is - 1) * (size_t)(n * n);
        double cxn[64], cen[64];
        or_bli_interp_points_shift(cxn, S->min_xi, S->max_xi, d);
        or_bli_interp_points_shift(cen, S->min_eta, S->max_eta, d);
        double x = xs[it - 1], y = ys[it - 1], z = zs[it - 1];
        int offset = 0;
        for (int j = 0; j < n; ++j) {
            double eta = cen[j];
            for (int i = 0; i < n; ++i) {
                double cx, cy, cz, sx, sy;
                or_xyz_from_xieta(&cx, &cy, &cz, cxn[i], eta, S->face);
                or_sal_grad_gfunc(x, y, z, cx, cy, cz, &sx, &sy);
                offset = offset + 1;
                slon[it - 1] = slon[it - 1] + sx * W[offset - 1];
                slat[it - 1] = slat[it - 1] + sy * W[offset - 1];
            }
        }
    }
    }
}

/* pp_compute + pp_interact, mom6_fast_sum_module.f90:177-192, :109-150, at one
 * rank (relabeled_points_inside == points_inside, no halo points). */
void or_pp_compute(double *slon, double *slat, const int *pp, int npp, const or_tree *t, const double *xs,
                   const double *ys, const double *zs, const double *areas, const double *sshs, int npoints,
                   int nthreads)
{
    if (nthreads < 1) nthreads = 1;
    /* target-point ownership per thread, as in or_pc_compute */
#pragma omp parallel num_threads(nthreads)
    {
    int nth = omp_get_num_threads(), me = omp_get_thread_num();
    int lo = (int)((long long)npoints * me / nth) + 1, hi = (int)((long long)npoints * (me + 1) / nth);
    for (int e = 0; e < npp; ++e) {
        int it = pp[2 * e], is = pp[2 * e + 1];
        if (it < lo || it > hi) continue;
        const or_panel *S = &t->p[is - 1];
        double tx = xs[it - 1], ty = ys[it - 1], tz = zs[it - 1];
        for (int i = 0; i < S->count; ++i) {
            int s = S->pts[i] - 1;
            double sx, sy;
            or_sal_grad_gfunc(tx, ty, tz, xs[s], ys[s], zs[s], &sx, &sy);
            slon[it - 1] = slon[it - 1] + sshs[s] * areas[s] * sx;
            slat[it - 1] = slat[it - 1] + sshs[s] * areas[s] * sy;
        }
    }
    }
}

/* ------------------------------------------------------------------------- */
/* FP64 direct O(N^2) sum -- the accuracy judge for both paths                */
/* ------------------------------------------------------------------------- */

/* For each sampled target (0-based point index), sums G(t,s)*area*ssh over all
 * n sources in index order, with the pp_interact multiplication order
 * (fast_sum_module.f90:69-70).  Includes s == t, as the treecode does. */
void or_direct_sum(const double *xs, const double *ys, const double *zs, const double *area, const double *ssh,
                   int n, const int *targets, int nt, double *out_x, double *out_y, int nthreads)
{
    if (nthreads < 1) nthreads = 1;
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 4)
    for (int k = 0; k < nt; ++k) {
        int ti = targets[k];
        double tx = xs[ti], ty = ys[ti], tz = zs[ti], ax = 0.0, ay = 0.0;
        for (int s = 0; s < n; ++s) {
            double sx, sy;
            or_sal_grad_gfunc(tx, ty, tz, xs[s], ys[s], zs[s], &sx, &sy);
            ax = ax + sx * area[s] * ssh[s];
            ay = ay + sy * area[s] * ssh[s];
        }
        out_x[k] = ax;
        out_y[k] = ay;
    }
}

/* Interaction work counters for a DTT list: kernel pairs by type and the
 * number of points touched by proxy-weight and interpolation loops. */
void or_dtt_work(const or_tree *t, const int *list, int ninter, int d, double *pairs4, double *macs)
{
    double P = (double)(d + 1) * (d + 1);
    for (int k = 0; k < 4; ++k) pairs4[k] = 0;
    *macs = 0;
    for (int i = 0; i < ninter; ++i) {
        const or_panel *T = &t->p[list[3 * i] - 1], *S = &t->p[list[3 * i + 1] - 1];
        int ty = list[3 * i + 2];
        double ct = T->count, cs = S->count;
        if (ty == 0) pairs4[0] += ct * cs;
        else if (ty == 1) { pairs4[1] += ct * P; *macs += cs * P; }
        else if (ty == 2) { pairs4[2] += P * cs; *macs += ct * P; }
        else { pairs4[3] += P * P; *macs += (cs + ct) * P; }
    }
}
