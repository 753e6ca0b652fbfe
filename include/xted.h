/*
 * xted.h -- C ABI of the B200-native tree edit distance library (the
 * reference's unit cost by default, general edit costs as an option).
 *
 * Drop-in for the reference X-TED entry point
 *   int standard_ted(vector<string>& x_node, vector<vector<int>>& x_adj,
 *                    vector<string>& y_node, vector<vector<int>>& y_adj,
 *                    int num_threads, int parallel_version)
 * (X-TED_CPU/TED.cpp:177, declared X-TED_CPU/TED_C++.h:21; GPU twin
 * X-TED_GPU/TED.cu:116, X-TED_GPU/TED_C++.h:28), re-expressed as plain C:
 * pointers and sizes only. A C++ wrapper with the reference's exact signature
 * is in include/xted.hpp.
 *
 * Trees are ordered, labelled and numbered in preorder (root = 0), the
 * reference's input contract (README.md:31-44). Children of node v are
 * child_idx[child_off[v] .. child_off[v+1]) in left-to-right order. Labels
 * are int32 ids; the reference only tests label strings for equality
 * (X-TED_CPU/TED.cpp:153-159), so interning strings to ids is exact.
 * Unlike the reference (which clears the caller's label vectors,
 * X-TED_CPU/TED.cpp:160-161) the library never writes to caller input.
 *
 * Every function returns 0 on success or a negative XTED_E* code; none
 * throws or exits. A context is not thread-safe: use one per host thread, or
 * lock around calls.
 */
#ifndef XTED_H
#define XTED_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define XTED_OK 0
#define XTED_EINVAL (-1)   /* malformed tree, bad size or argument        */
#define XTED_ENOMEM (-2)   /* device or host allocation failed / over limit */
#define XTED_ETIMEOUT (-3) /* a bounded device wait ran out               */
#define XTED_ECUDA (-4)    /* a CUDA runtime call failed                  */
#define XTED_ENODEV (-5)   /* no usable sm_100 device                     */
#define XTED_ENOTFOUND (-6) /* unknown serving ticket                     */
#define XTED_EAGAIN (-7)   /* serving queue full; retry later             */
#define XTED_ETOOBIG (-8)  /* pair exceeds xted_distance_noalloc's arena   */

/* Largest tree accepted (nodes). Bounds the int32 key arithmetic of the
 * row scan and keeps the per-pair distance table addressable. */
#define XTED_MAX_NODES 65535

typedef struct xted_tree {
    const int32_t *labels;    /* [n] label ids                              */
    const int32_t *child_off; /* [n+1] CSR offsets, child_off[0] == 0       */
    const int32_t *child_idx; /* [n-1] children in preorder, left to right  */
    int32_t n;                /* number of nodes (0 = empty tree)           */
} xted_tree;

/* Decomposition of the keyroot tables. The distance is identical for all
 * three (tree edit distance is invariant under mirroring both trees); only
 * the amount of work differs. */
#define XTED_ORIENT_AUTO 0  /* per pair, the cheaper of the two            */
#define XTED_ORIENT_RIGHT 1 /* right-path keyroots, X-TED_CPU's choice      */
#define XTED_ORIENT_LEFT 2  /* left-path keyroots (classic Zhang-Shasha)    */

typedef struct xted_opts {
    int32_t device;         /* CUDA device ordinal                          */
    int32_t orientation;    /* XTED_ORIENT_*                                */
    int32_t narrow_width;   /* widest column chunk run by one warp (1..256);
                               0 runs every chunk on a whole thread block   */
    int32_t run_rows;       /* target rows per row run (>= 1)               */
    int32_t ctas_per_sm;    /* persistent blocks per SM (0 = occupancy max) */
    int32_t wide_rows;      /* > 0: a narrow chunk's unit whose row run is
                               longer than this runs on the whole block
                               (shortens critical paths, costs throughput);
                               <= 0: never (default)                        */
    int32_t half_width;     /* chunks wider than narrow_width up to this
                               width (at most 1024) run on half a block, two
                               at a time; 0 = 512 (fastest on the mixed
                               batch), < 0: none                            */
    int32_t tuned;          /* nonzero (default): run_rows, narrow_width and
                               half_width come per tree from the autotuned
                               size-bucket table; 0: the fields above apply
                               to every tree                                */
    double wait_timeout_s;  /* bound on every device-side wait              */
    int64_t mem_limit;      /* device bytes the context may hold (0 = none) */
    int64_t stripe_min_cells; /* a table whose column segment is wider than
                               2,048 and whose unit has at least this many
                               cells runs in column stripes of 512 columns
                               (wider past 128 stripes), each stripe a task
                               that any block may run (0 = 2^20; < 0: the
                               whole table on one block)                    */
    int32_t cost_del;       /* edit costs (integers >= 0): deleting a node of */
    int32_t cost_ins;       /* the first tree, inserting a node of the second */
    int32_t cost_ren;       /* tree, and mapping two nodes whose labels differ
                               (equal labels map at 0). 1, 1, 1 (the default,
                               and what 0, 0, 0 means) is the reference's unit
                               cost (X-TED_CPU/parallel_computing.cpp:17-39),
                               bit-exact with it. A pair of m and n nodes is
                               accepted while cost_del*m + cost_ins*n <
                               XTED_COST_BOUND (the row scan's key range),
                               else the call returns XTED_EINVAL. The
                               allocation-free entry point is unit-cost only. */
    int32_t pad_;
} xted_opts;

/* Bound on cost_del * m + cost_ins * n for a pair of m and n nodes. */
#define XTED_COST_BOUND (1 << 17)

typedef struct xted_ctx xted_ctx;

/* Statistics of the last distance/batch call. */
typedef struct xted_stats {
    int64_t pairs;
    int64_t cells;          /* interior forest-table cells executed          */
    int64_t cells_right;    /* cells X-TED's right-path decomposition needs  */
    int64_t tasks;          /* block-level tasks in the device queue         */
    int64_t units;          /* warp/block work units                         */
    int64_t h2d_bytes, d2h_bytes;
    double host_plan_ms;    /* host planning time                            */
    double device_ms;       /* device time of one run: counter reset, DP launch
                               and gather (CUDA events on the launch stream) */
    double total_ms;        /* wall time of the call                         */
    int32_t levels_max;     /* deepest keyroot-level count of any pair        */
    int32_t grid;           /* persistent blocks launched                    */
    double dp_ms;           /* device time of the DP kernel alone            */
    int32_t graph;          /* 1 if the step replayed its captured CUDA graph */
    int32_t pad;
} xted_stats;

void xted_opts_default(xted_opts *opts);
const char *xted_strerror(int code);

int xted_create(xted_ctx **ctx, const xted_opts *opts);
int xted_destroy(xted_ctx *ctx);

/* One pair; synchronous. Matches standard_ted, including its empty-tree
 * rules (m == 0 -> n, n == 0 -> m; X-TED_CPU/TED.cpp:181-186). */
int xted_distance(xted_ctx *ctx, const xted_tree *a, const xted_tree *b, int32_t *out);

/* npairs pairs (a[i], b[i]) in one persistent device launch; synchronous. */
int xted_distance_batch(xted_ctx *ctx, const xted_tree *a, const xted_tree *b, int32_t npairs,
                        int32_t *out);

/* Plans npairs pairs and uploads everything the device needs; the inputs then
 * stay resident in HBM. xted_run_prepared recomputes that batch from the
 * resident inputs (repeated evaluation; device-only timing). The prepared
 * batch lives until the next prepare or batch call on the context. */
int xted_prepare_batch(xted_ctx *ctx, const xted_tree *a, const xted_tree *b, int32_t npairs);
int xted_run_prepared(xted_ctx *ctx, int32_t *out);

int xted_last_stats(const xted_ctx *ctx, xted_stats *out);

/* Replaces, for this context, the size-bucket granularity table compiled
 * into the library (the autotuner's output) with nrows rows of four int32:
 * max_n (> 0, strictly increasing), run_rows (>= 1), narrow_width (0..256)
 * and half_width (-1..1024). Row k applies to trees with fewer than max_n
 * nodes, the last row to all larger trees. nrows == 0 restores the compiled
 * table. Applies, while the `tuned` option is set, to batches planned and
 * corpora loaded after the call; a prepared batch keeps its plan. At most 8
 * rows; a malformed table returns XTED_EINVAL and changes nothing. The
 * autotuner uses it to time a whole table on mixed batches without a
 * rebuild. */
int xted_set_tune_table(xted_ctx *ctx, const int32_t *rows, int32_t nrows);

/* All pairs of ntrees trees: out[i*ntrees + j] = TED(trees[i], trees[j]),
 * symmetric with a zero diagonal. The reference harness allocates this
 * matrix but fills only pair (0, 1) (X-TED_CPU/TED_test.cpp:26-47); here the
 * ntrees(ntrees-1)/2 pairs (every ordered pair when cost_del != cost_ins,
 * which makes TED asymmetric) run through the batch path in chunks whose
 * distance tables fit in pair_budget int32 elements (0: 2^30, or a quarter of
 * the context's mem_limit). Synchronous. */
int xted_distance_matrix(xted_ctx *ctx, const xted_tree *trees, int32_t ntrees, int64_t pair_budget, int32_t *out);

/* Cell count of a pair under each decomposition, without computing it:
 * out[0] = right path (X-TED), out[1] = left path, out[2] = the chosen one. */
int xted_pair_cells(const xted_tree *a, const xted_tree *b, int32_t orientation, int64_t *out3);

/* Checks that a tree is a well-formed preorder CSR. */
int xted_validate(const xted_tree *t);

/* Seeded synthetic trees (the benchmark workloads). shape: 0 random
 * recursive, 1 wide-shallow, 2 deep-narrow, 3 caterpillar. label_kind: 0
 * uniform over `alphabet` ids, 1 Zipf(s = 1.1) over `alphabet` ids. Writes
 * n labels, n+1 offsets and n-1 children into caller buffers. */
int xted_gen_tree(int32_t shape, int32_t n, uint64_t seed, int32_t label_kind, int32_t alphabet,
                  int32_t *labels, int32_t *child_off, int32_t *child_idx);

/* ---- dataset text formats (large corpora) ----
 *
 * xted_parse_adjacency: one line of the reference's adjacency files,
 * "[[1, 2], [], ...]" (grammar of X-TED_CPU/dataset_preprocess.cpp:7-66),
 * into CSR: child_off[n+1], child_idx[nchildren]. XTED_ENOMEM if the caps
 * are too small, XTED_EINVAL on text outside the grammar.
 * xted_parse_bracket: one tree in bracket notation, "{a{b}{c{d}}}" (the
 * format of the reference's Sampled_Dataset_Extra_Large_Trees/synthetic/
 * synthetic_tree_*.txt, which its code never reads), into preorder CSR plus
 * each node's label as a span of the input (label_at, label_len; backslash
 * escapes left in place). *end_out = index just past the tree. */
int xted_parse_adjacency(const char *line, int64_t len, int32_t cap_nodes, int32_t cap_children, int32_t *child_off,
                         int32_t *child_idx, int32_t *n_out, int32_t *nchildren_out);
int xted_parse_bracket(const char *s, int64_t len, int32_t cap_nodes, int32_t *child_off, int32_t *child_idx,
                       int64_t *label_at, int32_t *label_len, int32_t *n_out, int64_t *end_out);

/* ---- allocation-free single pair ----
 *
 * No counterpart in the reference. For callers that cannot allocate device
 * memory when they need a distance: a process whose HBM is already handed to
 * another allocator's pool, a checker running after an allocation failed, or
 * a latency-bound caller that cannot take the device-wide synchronisation a
 * cudaFree implies. The pair is computed in a fixed arena of
 * XTED_NOALLOC_ARENA_BYTES that is part of the loaded library module; the
 * call makes no device or pinned-host allocation and needs no context.
 * Limit: with m and n the tree sizes, the inputs, their metadata
 * (about 8(m + n) ints), the m x n tree-distance matrix and at least one
 * (m + 1) x (n + 1) forest table must fit in the arena (a pair of two
 * 1400-node trees fits); larger pairs return XTED_ETOOBIG. Synchronous. Every
 * call on a device shares the one arena, which keeps the last call's
 * contents (each call clears its status words and overwrites everything else
 * it reads): calls that overlap on the GPU (two host threads at once) race,
 * so serialise them. The first call on a device does the set-up: it checks
 * the device and looks up the arena's device address with that device
 * current; make that first call before any stream capture. CUDA loads
 * modules lazily by default (since CUDA 12.2), so that first lookup is also
 * what loads the library's module onto the device and commits the arena's
 * XTED_NOALLOC_ARENA_BYTES of device memory: "allocates nothing" holds from
 * the second call on. Make one warm-up call (any small pair) at start-up,
 * before handing device memory to another allocator's pool. The call makes
 * `device` current while it works and restores the calling thread's current
 * device before it returns. Same results and empty-tree rules as
 * xted_distance. */
#define XTED_NOALLOC_ARENA_BYTES (16 << 20)
int xted_distance_noalloc(const xted_tree *a, const xted_tree *b, int32_t device, int32_t *out);

/* ---- serving: a resident corpus and exact top-k queries ----
 *
 * No counterpart in the reference (its harness computes one pair). A
 * corpus stays resident on the device with its keyroot metadata; each query
 * is planned against every corpus tree and fed into the running persistent
 * DP launch as soon as one of XTED_SERVE_SLOTS slots and enough device
 * memory for its distance tables are free (continuous batching: queries
 * overlap on the device, earlier queries take priority). A worker thread of
 * the context drives the loop; these calls are thread-safe with respect to
 * each other. Batch calls on the same context wait while a serving launch
 * is running. */
#define XTED_SERVE_SLOTS_MAX 16
#define XTED_SERVE_MAX_QUERY 8192 /* nodes of one query tree */

/* Uploads a corpus (replacing any previous one, after finishing its queries)
 * and precomputes its keyroot metadata. */
int xted_corpus_load(xted_ctx *ctx, const xted_tree *trees, int32_t ntrees);

/* Queues a query for the k nearest corpus trees by TED. Returns at once;
 * XTED_EAGAIN when the queue is full, XTED_EINVAL for a malformed tree or
 * one larger than XTED_SERVE_MAX_QUERY. */
int xted_query_submit(xted_ctx *ctx, const xted_tree *q, int32_t k, uint64_t *ticket);

/* Reports a query. *done = 1 when ids/dists (k entries each, ascending
 * distance, ties by lower corpus index; -1 past the corpus size) are final;
 * the ticket is then released. A failed query returns its error code. */
int xted_query_poll(xted_ctx *ctx, uint64_t ticket, int32_t *ids, int32_t *dists, int32_t *done);

/* As xted_query_poll, and on completion the time from submission to
 * admission (queue_ms) and to completion (total_ms). Either may be NULL. */
int xted_query_poll_timed(xted_ctx *ctx, uint64_t ticket, int32_t *ids, int32_t *dists, int32_t *done,
                          double *queue_ms, double *total_ms);

/* Blocks until every submitted query is finished; returns the first device
 * error seen since the last drain, else 0. */
int xted_serve_drain(xted_ctx *ctx);

/* Writes the first n of: persistent launches made, queries served, pairs
 * computed, cells computed, pairs pruned (answered by the lower bound
 * without computing), queries that needed a second round, and the host
 * microseconds spent computing bounds and planning. */
int xted_serve_stats(xted_ctx *ctx, int64_t *out, int32_t n);

/* Exact top-k pruning by a lower bound of TED, per corpus tree:
 *   prune = 1: labels, max(m, n) - min(m, n, I), I the size of the two
 *              label multisets' intersection;
 *   prune = 2 (default): the Levenshtein distance of the two preorder label
 *              sequences (an edit mapping keeps preorder), which is never
 *              below the label bound;
 *   prune = 0: no pruning, every pair computed in one round.
 * Round 1 computes the max(first_round, 4k) trees of lowest (bound, index)
 * (first_round 0: 32); round 2 computes only the trees whose (bound, index)
 * still beats the k-th (distance, index) found. The answer equals the
 * unpruned one. Applies to queries admitted later. */
int xted_serve_options(xted_ctx *ctx, int32_t prune, int32_t first_round);

/* ---- failure injection for tests ----
 *
 * No counterpart in the reference, whose error handling prints CUDA errors and
 * carries on or exits the process (X-TED_GPU/utils/cuda_utils.h:35-41,
 * X-TED_GPU/help.h:6-14) and whose spin barriers wait without bound
 * (X-TED_GPU/parallel_X_TED.cu:68-91, 128-157). This hook lets a test check
 * that a failure here is bounded, reported and survivable, without faulting
 * or hanging anything: it arms one host-side fault for the next
 * xted_distance_batch / xted_distance call or the next serving query posted
 * to the device, then disarms itself.
 *   XTED_FAULT_HOLD_PAIR: level 0 of one computed pair (the batch's pair 0,
 *     or the query's first computed corpus tree) is never published into the
 *     ready queue, so its tables never become ready. A batch then ends when
 *     the persistent launch's bounded idle wait (wait_timeout_s) runs out and
 *     returns XTED_ETIMEOUT; a serving launch goes idle and ends, and the
 *     query fails with XTED_ETIMEOUT. The context stays usable. */
#define XTED_FAULT_NONE 0
#define XTED_FAULT_HOLD_PAIR 1
int xted_test_fault(xted_ctx *ctx, int32_t kind);

#ifdef __cplusplus
}
#endif

#endif /* XTED_H */
