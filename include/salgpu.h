/*
 * salgpu.h -- C ABI of the B200 SAL-gradient treecode (libsalgpu.so).
 *
 * Drop-in boundary for cygnari/sal-fort's fast-sum entry points.  The reference
 * is Fortran; its callers bind these functions with ISO_C_BINDING (the
 * interface block is in sal-fort_b200/fortran/salgpu_mod.f90).  Signatures use
 * plain pointers and sizes only.
 *
 * Conventions
 *   - Panel ids, point ids and interaction-list entries are 1-based, exactly as
 *     the reference's Fortran arrays hold them (tree_module.f90:5-34).
 *   - Point arrays (xs, ys, zs, areas, sshs, outputs) are 0-based C arrays of
 *     point_count doubles in the caller's point order.
 *   - Every function returns SAL_OK (0) or a negative SAL_E* code;
 *     sal_last_error() gives the message of the last failure on this thread.
 *   - Functions whose names end in _host take host pointers and are synchronous.
 *     sal_solve and sal_direct_sum take device pointers and a cudaStream_t
 *     (passed as void*) and are asynchronous on that stream.
 *   - There is no CPU fallback: without a usable CUDA device every device entry
 *     point returns SAL_ENODEV.
 */
#ifndef SALGPU_H
#define SALGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SAL_OK 0
#define SAL_EINVAL (-1)
#define SAL_ENOMEM (-2)
#define SAL_ECUDA (-3)
#define SAL_ETIMEOUT (-4)
#define SAL_ENODEV (-5)
#define SAL_ETREE (-6)   /* panels given without points_inside differ from the tree of the coordinates */

/* Evaluator families.  DTT is the code.f90 path (fast_sum_module.f90); the two
 * STT modes are the mom6_code.f90 path (mom6_fast_sum_module.f90). */
#define SAL_MODE_DTT 0               /* dual tree traversal, PP/PC/CP/CC */
#define SAL_MODE_STT_REF_COMPAT 1    /* single tree traversal, proxy weights stored transposed as the reference does */
#define SAL_MODE_STT_CORRECT 2       /* single tree traversal, proxy weights in the orientation pc_interact reads */

/* Arithmetic forms of a solve. */
#define SAL_FORM_REF 0       /* FP64, the reference's kernel and interpolation operation for operation */
#define SAL_FORM_ACCURATE 1  /* FP64; CP/CC interpolate the frame-free Cartesian sum and use the antipode-stable kernel */
#define SAL_FORM_MIXED 2     /* ACCURATE's algorithm with FP32 kernel tiles and tensor-core contractions; FP64 self/near pairs */

typedef struct sal_tree sal_tree;  /* host cubed-sphere quadtree (tree_module.f90 cube_panel array) */
typedef struct sal_grid sal_grid;  /* device-resident grid: points, panels, lists, work plan */

/* ------------------------------------------------------------------ errors */
const char *sal_last_error(void);
void sal_free(void *p);  /* frees arrays returned by the list builders below */

/* ------------------------------------------------------------------ host setup
 * These mirror tree_module.f90 for callers that build the tree in C/C++.  A
 * Fortran caller keeps its own tree_traverse/dual_tree_traversal and passes the
 * flattened result to sal_tree_import instead. */

/* tree_traverse, tree_module.f90:59-246. */
int sal_tree_traverse(const double *xs, const double *ys, const double *zs, int32_t point_count,
                      int32_t cluster_thresh, sal_tree **out);

/* Import a cube_panel array flattened by the caller (tree_module.f90:5-28)
 * together with the points it was built from.
 * ints9: per panel level, is_leaf, id, parent, child1..child4, face.
 * dbl7:  per panel min_xi, mid_xi, max_xi, min_eta, mid_eta, max_eta, radius.
 * pt_off (npanels+1) / pt_idx: CSR of points_inside (1-based point ids).
 * Every leaf's points_inside together must be a partition of 1..point_count,
 * and every panel's count must equal the sum of its children's. */
int sal_tree_import(int32_t npanels, const int32_t *ints9, const double *dbl7, const int64_t *pt_off,
                    const int32_t *pt_idx, int32_t point_count, const double *xs, const double *ys,
                    const double *zs, sal_tree **out);

/* Sizes of a tree: panel count, total length of all points_inside arrays, deepest level. */
int sal_tree_info(const sal_tree *t, int32_t *npanels, int64_t *points_inside_total, int32_t *max_level);

/* Export in the sal_tree_import layout (pt_idx may be NULL). */
int sal_tree_export(const sal_tree *t, int32_t *ints9, double *dbl7, int64_t *pt_off, int32_t *pt_idx);

int sal_tree_destroy(sal_tree *t);

/* dual_tree_traversal, tree_module.f90:277-398.  *list receives count triplets
 * (index_target, index_source, interact_type 0..3); free with sal_free. */
int sal_dual_tree_traversal(const sal_tree *t, double theta, int32_t cluster_thresh, int32_t **list,
                            int64_t *count);

/* tree_traverse and dual_tree_traversal with the refinement and the pair
 * traversal on CUDA device `device`, for fast admission of new grids (no
 * counterpart in the reference, which builds both on the host).  Results and
 * order equal sal_tree_traverse and sal_dual_tree_traversal bit for bit: the
 * per-point (xi, eta) and the panel radii and centres are computed with the
 * host's libm, and MAC ratios within 1e-12 of theta are decided on the host.
 * sal_dual_tree_traversal_device takes any tree (host- or device-built).  Both
 * are synchronous.  Their device scratch comes from a memory pool of the
 * library's own per device, which keeps up to 1 GiB between calls (a few
 * hundred MB after a 2.3M-cell build) until the process exits. */
int sal_tree_traverse_device(const double *xs, const double *ys, const double *zs, int32_t point_count,
                             int32_t cluster_thresh, int32_t device, sal_tree **out);
int sal_dual_tree_traversal_device(const sal_tree *t, double theta, int32_t cluster_thresh, int32_t device,
                                   int32_t **list, int64_t *count);

/* single_tree_traversal, tree_module.f90:401-487.  *pc and *pp receive pairs
 * (index_target = point id, index_source = panel id); free with sal_free. */
int sal_single_tree_traversal(const sal_tree *t, double theta, int32_t cluster_thresh, const double *xs,
                              const double *ys, const double *zs, int32_t own_points, int32_t **pc,
                              int64_t *npc, int32_t **pp, int64_t *npp);

/* assign_points_to_panels, tree_module.f90:249-273.  points_panels is
 * (nlev x own_points) column-major and is filled with -1 first. */
int sal_assign_points_to_panels(const sal_tree *t, const double *xs, const double *ys, const double *zs,
                                int32_t own_points, int32_t *points_panels, int32_t nlev);

/* ------------------------------------------------------------------ device grid */
typedef struct {
    int32_t point_count;
    const double *xs, *ys, *zs, *areas;  /* host, caller's order */
    int32_t interp_degree;               /* namelist interp_degree (code.f90:14) */
    int32_t mode;                        /* SAL_MODE_* */
    /* DTT: list_count triplets (target panel, source panel, type). */
    const int32_t *list;
    int64_t list_count;
    /* STT: pairs (target point, source panel). */
    const int32_t *pc_list;
    int64_t pc_count;
    const int32_t *pp_list;
    int64_t pp_count;
    int32_t max_fields;  /* fields per batched block: <= 32 sizes the batched buffers for 32, else 64 */
    int32_t device;      /* CUDA device ordinal */
} sal_grid_desc;

typedef struct {
    int32_t point_count, npanels, nleaves, degree, mode;
    int64_t list_count;
    double pairs_pp, pairs_pc, pairs_cp, pairs_cc;  /* kernel evaluations per field per solve */
    double macs_up, macs_down;                       /* proxy multiply-adds per field per solve */
    int64_t device_bytes;                            /* resident device memory of the grid */
    double setup_seconds;                            /* plan build + upload */
    int64_t mixed_bytes;                             /* device memory the batched form adds on its first solve */
    double macs_up_batched, macs_down_batched;       /* the batched form's basis multiply-adds per field: the
                                                        leaf-level upward and DOWN work of its tree passes (or the
                                                        direct ones, as macs_up / macs_down, when those are off) */
    int64_t launches_batched;                        /* kernel launches of one batched block under the current
                                                        choices (sal_tune) */
    int64_t tile_store_bytes;                        /* device bytes of the FP16 leaf pass's kernel-tile store under
                                                        the current plan (allocated only with sal_tune.tile_store) */
} sal_grid_stats;

/* Runtime choices of the batched form's tcgen05 passes (no counterpart in the
 * reference): the search space of sal_grid_autotune. */
typedef struct {
    int32_t chain_ksteps;       /* k-steps (8 sources) an accumulator chain reaches before it is folded into the
                                   running sums: longer chains fold less often, shorter ones round less (the tensor
                                   cores accumulate with truncation) */
    int32_t tree_passes;        /* 1: leaf-level upward pass plus child-to-parent transfers, parent-to-child
                                   transfers plus one DOWN item per leaf; 0: the direct per-slot passes
                                   (degrees above 10 always use the direct passes) */
    int32_t up_chunk;           /* direct upward pass: points per work unit at least */
    int32_t proxy_unit_kpairs;  /* proxy pass: kernel pairs per work unit, in units of 1024 */
    int32_t cta_groups;         /* tcgen05 launches: target groups one CTA walks at most */
    int32_t field_block;        /* fields per block: 64 (tcgen05 passes) or 32 (mma.sync passes) */
    int32_t f16;                /* 64-field leaf pass: 1 FP16 hi/lo operands (16 sources per MMA), scaled per field and
                                   per target by powers of two; 0 TF32 hi/lo (8 sources per MMA) */
    int32_t tile_store;         /* FP16 leaf pass: 1 keeps its kernel tiles (the near-field and proxy kernel values and
                                   DOWN interpolation rows, FP16 hi/lo, which depend on the grid alone) in device
                                   memory, sal_grid_stats.tile_store_bytes of it: the first solve records them, later
                                   solves read them instead of computing them, with the same results bit for bit.
                                   m > 1 keeps one item in m of each leaf group (about 1/m of the bytes); later
                                   solves copy those and compute the others.  Allocated with the batched buffers;
                                   ignored with f16 = 0 or 32-field blocks */
} sal_tune;

/* Flattens the tree and lists into device-resident arrays (once per grid). */
int sal_grid_create(const sal_tree *t, const sal_grid_desc *desc, sal_grid **out);
int sal_grid_stats_get(const sal_grid *g, sal_grid_stats *s);

/* The batched form's current choices; setting them re-cuts its plan and
 * frees its buffers (allocated again by the next batched solve, so the
 * grid's work on its streams must be finished).  SAL_MODE_DTT grids only. */
int sal_grid_tune_get(const sal_grid *g, sal_tune *t);
int sal_grid_tune_set(sal_grid *g, const sal_tune *t);

/* Autotuner of the batched form (no counterpart in the reference).  Times
 * SAL_FORM_MIXED solves of the caller's nfields device fields (column f at
 * ssh + f * ld_ssh, caller's order, nfields <= 64) for candidate sal_tune
 * settings, by coordinate descent from the current setting over each
 * choice's candidates (the leaf pass's chain length, operand precision and
 * groups per CTA a second time at the end), with CUDA events on the grid's
 * stream and a 256 MB
 * L2 flush before each timed solve.  A candidate counts only if the
 * relative L2 error of its first field, at ntargets evenly spaced points,
 * against the FP64 direct sum stays <= max_rel_err.  The fastest is set on
 * the grid and returned in *best; *ms_best and *ms_start (may be NULL)
 * receive its time and the starting setting's.  Synchronous; allocates
 * scratch for the check and the flush. */
int sal_grid_autotune(sal_grid *g, const double *ssh, int32_t nfields, int64_t ld_ssh, int32_t ntargets,
                      double max_rel_err, sal_tune *best, double *ms_best, double *ms_start);

/* Waits for the grid's work on stream (NULL: the grid's own stream) and
 * returns SAL_ETIMEOUT if a device-side staging wait gave up since the last
 * check. */
int sal_grid_sync(sal_grid *g, void *stream);

/* Fault injection for tests of the device-side time-outs (no counterpart in
 * the reference).  polls > 0: in the next FP64 solve on the grid, the leaf
 * pass leaves the last staging copy of every target group unissued and bounds
 * each staging wait to `polls` polls, so every group's last wait runs out
 * with no copy in flight.  That solve's outputs are undefined, and the next
 * sal_grid_sync (or the host entry point that ran the solve) returns
 * SAL_ETIMEOUT and clears the flag; later solves are unaffected.  polls = 0
 * cancels a pending injection. */
int sal_grid_inject_timeout(sal_grid *g, int32_t polls);

/* Per-pass device timers.  enable = 1 turns them on (each FP64 solve then
 * records CUDA events on its stream around three passes and waits for the
 * last), 0 turns them off, -1 leaves them as they are; 1 and 0 also reset the
 * sums.  phase_ms (4 doubles, may be NULL) receives the summed milliseconds of
 * prep+upward, proxy potentials, leaf evaluation and their total; solves the
 * number of solves summed. */
int sal_grid_timing(sal_grid *g, int32_t enable, double *phase_ms, int64_t *solves);

/* CUDA graphs of batched solves (no counterpart in the reference, which
 * solves one field per run).  enable = 1: the second SAL_FORM_MIXED sal_solve
 * of a call shape (field and output pointers, nfields, leading dimensions) on
 * a non-NULL stream runs as usual and is then captured into a graph, on a
 * stream of the caller stream's priority; later solves of that shape launch
 * the graph on their stream.  Graphs therefore pay off only for callers that
 * reuse their buffers.  The grid keeps up to 128 graphs, dropping the oldest.
 * 0 frees them and solves launch kernel by kernel again.  Graphs are not used
 * while the per-pass timers are on.  The graph cache has a lock of its own;
 * other state of a grid (its batched buffers) is shared by its solves, so one
 * grid's solves must not run concurrently on different streams. */
int sal_grid_set_graphs(sal_grid *g, int32_t enable);

/* Throughput of the FP64 (precision 64) or FP32 (precision 32) fused
 * multiply-add pipe of the current device, measured by a dependent-chain
 * microbenchmark: *tflops receives the achieved TFLOP/s (2 flops per FMA). */
int sal_fma_peak(int32_t precision, double *tflops);
int sal_grid_destroy(sal_grid *g);

/* Batched solve on device buffers.  ssh: nfields columns of point_count
 * doubles, column f at ssh + f*ld_ssh, caller's point order.  Outputs likewise
 * (overwritten, not accumulated).  form is SAL_FORM_*; SAL_FORM_REF supports
 * nfields == 1 per column loop.  Asynchronous on stream (NULL: the CUDA
 * default stream). */
int sal_solve(sal_grid *g, const double *ssh, int32_t nfields, int64_t ld_ssh, double *out_x, double *out_y,
              int64_t ld_out, int32_t form, void *stream);

/* Batched solves of several grids whose leaf passes share one launch (no
 * counterpart in the reference): the grids' smaller passes run one after
 * another on stream, then one tcgen05 leaf pass walks the target groups of
 * all of them, so grids of uneven size fill the GPU together instead of each
 * leaving it idle at its launch's tail.  SAL_FORM_MIXED; per grid k, nfields[k]
 * (1..64) fields at ssh[k] (column f at ssh[k] + f * ld_ssh[k]) and outputs at
 * out_x[k] / out_y[k] (leading dimension ld_out[k]).  At most 8 distinct
 * SAL_MODE_DTT grids of one device and one degree, each created with
 * max_fields > 32.  Results equal those of separate sal_solve calls bit for
 * bit.  A device-side time-out is reported by sal_grid_sync of grids[0].
 * Asynchronous on stream; a caller may capture it into a CUDA graph. */
int sal_solve_joint(sal_grid *const *grids, int32_t ngrids, const double *const *ssh, const int32_t *nfields,
                    const int64_t *ld_ssh, double *const *out_x, double *const *out_y, const int64_t *ld_out,
                    void *stream);

/* sal_solve on host buffers: copies the fields to the device, solves, copies
 * both components back and waits (outputs overwritten).  Device staging is
 * allocated on the first call and kept by the grid. */
int sal_solve_host(sal_grid *g, const double *ssh, int32_t nfields, int64_t ld_ssh, double *out_x, double *out_y,
                   int64_t ld_out, int32_t form);

/* Pipelined sal_solve_host.  No counterpart in the reference: it serves callers
 * that solve one batch after another from host memory.  The call enqueues the
 * copy of the fields to the device, the solve and the copy of both components
 * back, and returns without waiting.  The grid alternates two device staging
 * slots and copies on two streams of its own.  So one call's copies overlap the
 * neighbouring calls' solves, and its copy back overlaps the next copy in.
 * Host buffers must be pinned (cudaHostAlloc or cudaHostRegister) for the
 * copies to be asynchronous.  They must stay valid and unmodified until
 * sal_solve_host_wait returns.  Arguments and results as in sal_solve_host. */
int sal_solve_host_async(sal_grid *g, const double *ssh, int32_t nfields, int64_t ld_ssh, double *out_x,
                         double *out_y, int64_t ld_out, int32_t form);

/* Waits for every sal_solve_host_async call on the grid; reports a device-side
 * error of any of them (SAL_ETIMEOUT, ...). */
int sal_solve_host_wait(sal_grid *g);

/* fast_sum, fast_sum_module.f90:291-332: adds the SAL gradient of one field
 * into host arrays sal_longrad/sal_latgrad (intent(inout)).  The grid must be
 * SAL_MODE_DTT.  form as in sal_solve. */
int sal_fast_sum_host(sal_grid *g, const double *ssh, double *sal_longrad, double *sal_latgrad, int32_t form);

/* proxy_source_compute, mom6_fast_sum_module.f90:33-74: adds the proxy source
 * weights of every panel into proxy_source_weights ((d+1)^2 * npanels,
 * panel-major, the reference's flat layout; transposed in
 * SAL_MODE_STT_REF_COMPAT). */
int sal_proxy_source_compute_host(sal_grid *g, const double *sshs, double *proxy_source_weights);

/* pc_compute, mom6_fast_sum_module.f90:153-174: adds the far field computed
 * from proxy_weights (as returned above, possibly summed across ranks). */
int sal_pc_compute_host(sal_grid *g, const double *proxy_weights, double *sal_x, double *sal_y);

/* pp_compute, mom6_fast_sum_module.f90:177-192 (one rank, no halo points). */
int sal_pp_compute_host(sal_grid *g, const double *sshs, double *sal_x, double *sal_y);

/* ------------------------------------------------------------------ reference-signature entry points
 * The four hot routines with the reference's argument lists, for a Fortran
 * ISO_C_BINDING front end that changes nothing in code.f90 / mom6_code.f90
 * but their `use` lines.  Fortran derived types are not interoperable, so the
 * cube_panel array arrives flattened as in sal_tree_import (npanels, ints9,
 * dbl7, pt_off); pt_idx (points_inside) may be NULL, in which case the tree is
 * rebuilt from the coordinates and must equal the given panels (else
 * SAL_ETREE: pass pt_idx).  interaction_pair lists arrive as int32 tuples.
 * Each call hashes its set-up arguments (coordinates, areas, panels, list,
 * degree) and reuses the device grid it built for the same contents; any
 * change builds a new grid.  The library keeps up to four grids per entry
 * point, least recently used dropped.  Outputs are added into the caller's
 * arrays (intent(inout)), on the current CUDA device, synchronously.  The
 * calls serialise on one process-wide lock. */

/* fast_sum, fast_sum_module.f90:291-332 (list: list_count triplets target
 * panel, source panel, type).  Only interactions i (1-based) with
 * MOD(i, process_count) == rank are evaluated, as in the reference
 * (:303-304), so the caller's Sum_Array still completes the sum.  Arithmetic
 * form: sal_dropin_config (SAL_FORM_REF unless changed). */
int sal_fast_sum(double *sal_longrad, double *sal_latgrad, const int32_t *interaction_list, int64_t list_count,
                 int32_t npanels, const int32_t *ints9, const double *dbl7, const int64_t *pt_off,
                 const int32_t *pt_idx, const double *xs, const double *ys, const double *zs, const double *area,
                 const double *ssh, int32_t point_count, int32_t interp_degree, int32_t rank, int32_t process_count);

/* proxy_source_compute, mom6_fast_sum_module.f90:33-74: adds the proxy
 * source weights ((d+1)^2 * npanels, panel-major) into
 * proxy_source_weights.  points_panels is (nlev x point_count) column-major,
 * as assign_points_to_panels fills it (tree_module.f90:249-273); it must
 * match the panels.  Weight orientation: sal_dropin_config (the reference's
 * transposed store unless changed). */
int sal_mom6_proxy_source_compute(double *proxy_source_weights, int32_t npanels, const int32_t *ints9,
                                  const double *dbl7, const int64_t *pt_off, const int32_t *pt_idx,
                                  const int32_t *points_panels, int32_t nlev, const double *xs, const double *ys,
                                  const double *zs, const double *sshs, const double *areas, int32_t interp_degree,
                                  int32_t point_count);

/* pc_compute, mom6_fast_sum_module.f90:153-174 (list: pc_count pairs target
 * point, source panel; point_count = size(xs)). */
int sal_mom6_pc_compute(double *sal_longrad, double *sal_latgrad, const int32_t *pc_interaction_list, int64_t pc_count,
                        int32_t npanels, const int32_t *ints9, const double *dbl7, const int64_t *pt_off,
                        const int32_t *pt_idx, const double *xs, const double *ys, const double *zs,
                        int32_t point_count, int32_t interp_degree, const double *proxy_weights);

/* pp_compute, mom6_fast_sum_module.f90:177-192 (list: pp_count pairs target
 * point, source panel).  One rank: the halo arrays e_* of other ranks' points
 * must be empty (extra_count 0), else SAL_EINVAL. */
int sal_mom6_pp_compute(double *sal_longrad, double *sal_latgrad, const int32_t *pp_interaction_list, int64_t pp_count,
                        int32_t npanels, const int32_t *ints9, const double *dbl7, const int64_t *pt_off,
                        const int32_t *pt_idx, const double *xs, const double *ys, const double *zs,
                        const double *areas, const double *sshs, const double *e_xs, const double *e_ys,
                        const double *e_zs, const double *e_areas, const double *e_sshs, int32_t extra_count,
                        int32_t own_points);

/* Settings of the four entry points above (no counterpart in the reference):
 * form is SAL_FORM_REF (default) or SAL_FORM_ACCURATE for sal_fast_sum;
 * mom6_mode is SAL_MODE_STT_REF_COMPAT (default, the reference's transposed
 * weights) or SAL_MODE_STT_CORRECT for sal_mom6_proxy_source_compute. */
int sal_dropin_config(int32_t form, int32_t mom6_mode);

/* Frees every grid the four entry points above keep. */
int sal_dropin_release(void);

/* ------------------------------------------------------------------ grid ingestion
 * code.f90:36-56 (and mom6_code.f90:95-117) read five files of point_count
 * values, one per line, with list-directed READs.  sal_read_values reads the
 * first count values of such a file (E, D or Q exponents, blank lines
 * skipped) with every host thread, or, for a name ending in ".f64", count
 * raw little-endian float64 values as sal_write_values writes them.  Fewer
 * values than count, or a line that is not a number, returns SAL_EINVAL. */
int sal_read_values(const char *path, int64_t count, double *out);
int sal_write_values(const char *path, int64_t count, const double *values);

/* FP64 direct O(N^2) sum at nt targets (0-based indices into the sources),
 * with the reference kernel in its own operation order.  Device pointers;
 * w = area * ssh per source.  Overwrites out_x/out_y (nt each). */
int sal_direct_sum(const double *xs, const double *ys, const double *zs, const double *w, int32_t n,
                   const int32_t *targets, int32_t nt, double *out_x, double *out_y, void *stream);

/* Size of the fixed device scratch array behind sal_direct_sum_noalloc, in
 * doubles (2 MiB): one call handles at most SAL_NOALLOC_SCRATCH_DOUBLES / 2
 * targets. */
#define SAL_NOALLOC_SCRATCH_DOUBLES (1 << 18)

/* sal_direct_sum without any device allocation.  No counterpart in the
 * reference: it exists for callers that cannot call cudaMalloc -- for example a
 * thread running while another framework's caching allocator already holds the
 * device's memory, or code that cannot accept the device-wide synchronisation
 * cudaMalloc/cudaFree may cause.  Arguments and results are those of
 * sal_direct_sum; the partial sums live in a fixed 2 MiB array in the
 * library's device memory that every GPU loading the library keeps until the
 * process exits.  nt above SAL_NOALLOC_SCRATCH_DOUBLES / 2 returns SAL_EINVAL.
 * The first call on a device looks up that array's device address (make it
 * before any stream capture) and keeps it for the rest of the process: after
 * a cudaDeviceReset of that device the kept address is stale, so do not reset
 * a device between calls.  All calls share the array: calls whose work
 * overlaps on the GPU race and must be ordered by the caller (one stream, or
 * events). */
int sal_direct_sum_noalloc(const double *xs, const double *ys, const double *zs, const double *w, int32_t n,
                           const int32_t *targets, int32_t nt, double *out_x, double *out_y, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* SALGPU_H */
