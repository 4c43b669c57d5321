// Internal host-side types of libsalgpu: the cubed-sphere tree, interaction
// lists and the flattened device work plan.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace sal {

// One panel of the cubed-sphere quadtree (tree_module.f90:5-28).  Panels live
// in BFS order with children contiguous, so panel id k (1-based, as in the
// reference) is Tree::p[k-1].  Instead of a points_inside array per panel,
// every panel owns the contiguous range [begin, end) of Tree::order: the tree
// builder partitions points stably, so a leaf's range lists its points in the
// reference's points_inside order, and an internal panel's range holds the same
// set as its points_inside.
struct Panel {
    int32_t level = 0, is_leaf = 1, id = 0, parent = -1;
    int32_t child[4] = {-1, -1, -1, -1};
    int32_t face = 0;
    double min_xi = 0, mid_xi = 0, max_xi = 0, min_eta = 0, mid_eta = 0, max_eta = 0, radius = 0;
    int64_t begin = 0, end = 0;
    int64_t count() const { return end - begin; }
};

struct Tree {
    int32_t n = 0;                 // points
    std::vector<Panel> p;          // p[k] = panel id k+1
    std::vector<int32_t> order;    // order[pos] = 0-based point index; panels own ranges of it
    std::vector<double> xi, eta;   // per point (0-based), on the point's own face
    std::vector<int8_t> face;      // per point
    std::vector<double> cx, cy, cz; // per panel: xyz of (mid_xi, mid_eta), the MAC centre
    int32_t max_level() const;
    // Reference points_inside of panel id k (1-based ids, index-sorted).
    std::vector<int32_t> points_inside(int32_t k) const;
};

// tree_module.f90 restated for the host.
void face_xieta(double x, double y, double z, int face, double *xi, double *eta);
void xyz_from_xieta(double xi, double eta, int face, double *x, double *y, double *z);
int face_from_xyz(double x, double y, double z);
void cheb_nodes(double min_x, double max_x, int degree, double *out);
void bli_basis_host(double x, const double *nodes, int n, double *f);

Tree *tree_build(const double *xs, const double *ys, const double *zs, int32_t n, int32_t thresh);
Tree *tree_import(int32_t npanels, const int32_t *ints9, const double *dbl7, const int64_t *pt_off,
                  const int32_t *pt_idx, int32_t n, const double *xs, const double *ys, const double *zs,
                  std::string *err);
void tree_set_points(Tree *t, const double *xs, const double *ys, const double *zs);
void tree_finish_panels(Tree *t);   // radii and MAC centres from the panel bounds
int dtt_decide(const Tree &t, int32_t it, int32_t is, double theta, int32_t thresh);
std::vector<int32_t> dual_tree_traversal(const Tree &t, double theta, int32_t thresh);
// The same two builds on a CUDA device (tree_dev.cu); SAL_* status codes.
int tree_build_device(const double *xs, const double *ys, const double *zs, int32_t n, int32_t thresh, int device,
                      Tree **out);
int dual_tree_traversal_device(const Tree &t, double theta, int32_t thresh, int device, std::vector<int32_t> *L);
void single_tree_traversal(const Tree &t, double theta, int32_t thresh, const double *xs, const double *ys,
                           const double *zs, int32_t own, std::vector<int32_t> *pc, std::vector<int32_t> *pp);
int assign_points_to_panels(const Tree &t, const double *xs, const double *ys, const double *zs, int32_t own,
                            int32_t *points_panels, int32_t nlev);

// ---------------------------------------------------------------- work plan
// Item of a target group's work list.  kind 0 (PP) / 1 (PC): sources are pool
// entries [off, off+cnt) (points / proxies); kind 2 (DOWN): interpolation from
// the potentials of target slot `off`.  mask: word offset of the per-target
// bitmask (STT), or -1.
struct Item {
    int32_t off, cnt, mask, kind;
};

struct Group {           // a set of targets with one work list
    int32_t tgt;         // first target: pool position (leaf) or target-proxy slot (proxy group)
    int32_t nt;          // number of targets
    int32_t ib, ie;      // item range
    int32_t out;         // partial-output slot (proxy groups) or unused
    int32_t pad0, pad1, pad2;
};

struct UpUnit {          // upward-pass work unit
    int32_t slot, beg, end, panel;
};

// Target group of the batched (mixed-precision) kernels: at most 64 targets
// (four 16-row tensor-core tiles) with a local coordinate origin (cx, cy, cz)
// near them.  row0: first target row of the group within its panel (proxy
// groups) or 0.
struct MixGroup {
    int32_t tgt, nt, ib, ie, out, row0, pad0, pad1;
    double cx, cy, cz, pad2;
};

// Item of the tcgen05 leaf pass.  kind & 3 = 0 / 1: sources are pool rows
// [off, off + cnt); kind & 3 = 2: rows [row0, row0 + cnt) of target slot
// off's Cartesian potentials.  kind & kTcFlush: the tensor-core accumulator
// chain ends after this item (its sum is folded into the running sum with
// round-to-nearest adds).  kb: first k-step (8 rows) of the item in the split
// weight store.  (dx, dy, dz): centre of the source panel minus centre of the
// target leaf (kinds 0, 1), so that source coordinates stored relative to
// their own panel centre become coordinates relative to the target leaf.
constexpr int32_t kTcFlush = 4;
struct TcItem {
    int32_t off, cnt, kb, kind;
    float dx, dy, dz;
    int32_t row0;
};

// Runtime choices of the batched form's tcgen05 passes: the search space of
// the autotuner (sal_grid_autotune).  Changing them re-cuts the tcgen05 part
// of the plan; the FP64 plan is unaffected.
struct TcOptions {
    int32_t chain_ksteps = 32;          // k-steps an accumulator chain reaches before it is folded
    int32_t tree_passes = 1;            // 1: leaf-level upward + child-to-parent transfers, parent-to-child
                                        //    transfers + one DOWN item per leaf; 0: direct per-slot passes
    int32_t up_chunk = 4096;            // direct upward pass: points per work unit at least
    int32_t proxy_unit_kpairs = 648;    // proxy pass: kernel pairs of a work unit, in units of 1024
    int32_t cta_groups = 1;             // tcgen05 launches: groups a CTA walks at most
    int32_t f16 = 0;                    // leaf pass: 1: FP16 hi/lo operands (kind::f16, 16 sources per MMA)
                                        //    with power-of-two scales; 0: TF32 hi/lo (8 sources per MMA)
    int32_t tile_store = 0;             // FP16 leaf pass: 1: its kernel tiles are kept in device memory
                                        //    (recorded by the first solve, replayed after); m > 1: one item in
                                        //    m is kept and replayed, the producers compute the others; the
                                        //    plan is the same either way
};

struct Plan {
    int32_t n = 0, d = 0, P = 0, mode = 0, npanels = 0, nleaves = 0;
    // point data in pool order (leaf-contiguous DFS)
    std::vector<int32_t> perm;       // pos -> caller index
    std::vector<double> px, py, pz, parea, pxi, peta;
    // source proxy slots
    std::vector<int32_t> src_slot_panel;          // slot -> panel index (0-based)
    std::vector<double> src_proxy_xyz;            // slot*P*3
    std::vector<UpUnit> up_units;
    std::vector<int32_t> up_unit_beg;             // slot -> first unit (size nslots+1)
    // target proxy slots (DTT CP/CC targets)
    std::vector<int32_t> tgt_slot_panel;
    std::vector<double> tgt_proxy_xyz;            // slot*P*3
    std::vector<double> tgt_nodes;                // slot*2*(d+1): xi nodes then eta nodes
    std::vector<double> tgt_box;                  // slot*4: min_xi,max_xi,min_eta,max_eta
    std::vector<double> src_nodes, src_box;       // same for source slots (upward)
    std::vector<Group> proxy_groups;              // work units of target slots, sorted by cost
    std::vector<int32_t> proxy_unit_beg;          // tgt slot -> first unit (nslots+1); units in proxy_groups order by slot
    std::vector<Item> proxy_items;
    std::vector<Group> leaf_groups;               // one per leaf with targets, sorted by cost
    std::vector<Item> leaf_items;
    std::vector<uint32_t> masks;                  // STT per-target bitmasks
    // batched form: items of at most kMixStage sources (DOWN items: rows of
    // a target slot's potentials, off = slot, cnt = rows, mask = first row)
    std::vector<MixGroup> mix_leaf_groups, mix_proxy_groups, mix_up_groups;
    bool mix_built = false;                       // the three above and their items (plan_build_mix)
    std::vector<int32_t> leaf_panel;              // leaf index (leaf_groups[].out) -> panel index
    // tcgen05 leaf pass: groups of at most kTcRows targets in pool order, their
    // items and the row map of the split weight store (per store row: wF row
    // if >= 0, phiF row -2-v if <= -2, zero row if -1; every leaf, source
    // slot and target slot starts on a multiple of 8 rows).
    std::vector<MixGroup> tc_leaf_groups;
    // FP16 kernel-tile store: per leaf group the byte offset of its stored
    // tiles (ngroups + 1 entries; the last is the store's size), for the
    // current sal_tune.tile_store (plan_tile_offsets)
    std::vector<int64_t> tc_tile_off;
    std::vector<TcItem> tc_items;
    // tcgen05 proxy pass: per proxy unit, row chunks of at most kTcProxyRows
    // target proxies (row0 = first proxy, out = unit), and their items
    std::vector<MixGroup> tc_proxy_groups;
    std::vector<TcItem> tc_proxy_items;
    // tcgen05 upward pass: units of whole leaves of a source slot's panel
    // (tgt = slot, row0 = first proxy, out = unit), items over their points
    // (row0 = first k-step of the item in the basis store), the first unit
    // of every slot (nsrc + 1), and per basis k-step (slot, first pool row,
    // rows) for building the store of per-point BLI factors
    std::vector<MixGroup> tc_up_groups;
    std::vector<TcItem> tc_up_items;
    std::vector<int32_t> tc_up_unit_beg;
    std::vector<int32_t> tc_bas;                  // 3 per basis k-step
    int64_t tc_pt_ksteps = 0;                     // k-steps of the store holding points
    std::vector<int32_t> bsrc;
    int64_t tc_src_ksteps = 0;                    // k-steps of the store holding sources (points, proxies)
    // pool row ranges (begin, end) of every leaf and every source slot's
    // proxies, with the centre (x, y, z) of the range's panel
    std::vector<int32_t> sloc_ranges;
    std::vector<double> sloc_centres;
    std::vector<Item> mix_leaf_items, mix_proxy_items;
    std::vector<int32_t> proxy_slot_items;        // tgt slot -> first item in proxy_items (ntgt + 1)
    // tcgen05 proxy pass units: the plan's own cut of each target slot's
    // items (tc_proxy_unit_beg: tgt slot -> first unit, ntgt + 1)
    std::vector<int32_t> tc_proxy_unit_beg;
    int32_t tc_nproxy_units = 0;
    // tree passes of the batched form.  Proxy-weight slots ("wslots"): the
    // source slots, then every other panel with points below a source slot;
    // potential slots ("dslots"): the target slots, then every other panel
    // with points below a target slot.  Nodes per slot: 2(d+1) (xi, then eta).
    TcOptions tc_opt;
    int32_t n_wslots = 0, n_dslots = 0;
    std::vector<double> tc_up_nodes, tc_down_nodes;
    std::vector<int32_t> m2m_tasks;               // per refined up panel: parent wslot, 4 child wslots (-1: none),
                                                  // the children's halves (2 bits each: xi, eta upper)
    std::vector<int32_t> m2m_level_beg;           // task ranges per level, deepest first
    std::vector<int32_t> l2l_tasks;               // per down panel under another: child dslot, parent dslot, own,
                                                  // the child's halves
    std::vector<int32_t> l2l_level_beg;           // task ranges per level, top first
    std::vector<double> tc_transfer;              // [half][j][i]: parent basis j at node i of its lower / upper half
    double tc_macs_up = 0, tc_macs_down = 0;      // per field: basis MACs of the batched form's upward / DOWN work
    double pairs[4] = {0, 0, 0, 0};               // PP, PC, CP, CC evaluations per field
    double macs_up = 0, macs_down = 0;
    int32_t max_nt = 0;
};

// Builds the plan of a DTT list (triplets) or STT lists (pairs).
bool plan_build(const Tree &t, int d, int mode, const int32_t *list, int64_t nlist, const int32_t *pc, int64_t npc,
                const int32_t *pp, int64_t npp, Plan *plan, std::string *err);
// (Re)builds the tcgen05 part of a DTT plan for the given options.
bool plan_build_tc(const Tree &t, Plan *plan, const TcOptions &opt, std::string *err);
// the kernel-tile store's per-group offsets for one stored item in `every`
void plan_tile_offsets(Plan *plan, int every);
// The 32-field (mma.sync) groups of the batched form, from a built plan.
void plan_build_mix(const Tree &t, Plan *plan);

constexpr int kMaxStage = 256;   // sources staged per item (items are split to fit)
constexpr int kMixStage = 64;    // sources (or DOWN rows) staged per batched item
constexpr int kMixRows = 64;     // targets per batched CTA
constexpr int kTcRows = 128;     // targets per tcgen05 leaf group (the MMA's M)
constexpr int kTcChunk = 64;     // sources (or DOWN rows) per tcgen05 item
constexpr int kTcProxyRows = 85;   // target proxies per tcgen05 proxy group: 3 x 85 <= 256
constexpr int kMaxDegree = 14;   // a DOWN record (4(d+1)^2 + 2(d+1) doubles) fits one 8 KB stage
constexpr int kMaxTreeDegree = 10;  // tree transfers of the batched form: their tiles fit shared memory up to here
constexpr int kMaxTreeP = (kMaxTreeDegree + 1) * (kMaxTreeDegree + 1);

}  // namespace sal
