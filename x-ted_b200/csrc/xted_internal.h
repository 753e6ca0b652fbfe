// xted_internal.h -- data layout shared by the host planner and the kernels.
//
// Terminology (reference names in brackets):
//   row tree A (m nodes) and column tree B (n nodes) of one pair;
//   orl(v)      rightmost leaf of v's subtree = v + size(v) - 1
//               [outermost_right_leaves, X-TED_CPU/TED.cpp:21-42];
//   keyroot     root or a node that is not the last child of its parent
//               [key_roots, X-TED_CPU/TED.cpp:46-77];
//   kdepth(k)   keyroot level: 1 + max kdepth of keyroots strictly inside
//               sub(k), 0 if none [X-TED_CPU/parallel_computing.cpp:93-119];
//   table (i0,j0) the forest-distance table of one keyroot pair, whose level
//               is kdepth(i0) + kdepth(j0) [parallel_computing.cpp:121-123].
//
// Work decomposition. All keyroots of B with the same kdepth have disjoint
// subtrees ("segments"); their columns are concatenated per depth into one
// column list. A *chunk* is a run of whole segments of one depth. A *row run*
// is a run of whole keyroots of A of one depth. A *unit* = (row run, chunk):
// every table (i0, j0) with i0 in the run and j0 in the chunk, computed row by
// row (rows descending, a min-plus suffix scan across the chunk's columns).
// A *task* is what one thread block claims from the device queue: one wide
// unit (chunk wider than a warp can hold) or up to XTED_TASK_UNITS narrow
// units that the block's warps claim one at a time, all of one pair and one
// level.
#pragma once

#include <stdint.h>
#include <vector_types.h>  // int2, int4 (CUDA toolkit header, host-includable)

#define XTED_CTA_THREADS 256
#define XTED_WARPS (XTED_CTA_THREADS / 32)
#define XTED_NARROW_MAX 256       // widest chunk one warp holds in registers (8 per lane)
#define XTED_WIDE_REG_MAX 2048    // widest chunk one block holds in registers (8 per thread)
#define XTED_KEY_BIG (1 << 17)    // key step between segments of one chunk
#define XTED_INF 0x3fffffff

// rowinfo.y bit layout: orl in the low 20 bits.
#define XTED_ROW_ORL_MASK 0x000fffff
#define XTED_ROW_ISKR (1u << 29)     // node is a keyroot
#define XTED_ROW_PREVLEAF (1u << 30) // node i-1 is a leaf

// Per-column state derived in the kernels (the wide generic path keeps it in
// scratch as int4: x = node j, y = label(j), z = foff | flags, w = dend):
// foff = orl(j) + 1 - j (low 20 bits), dend = je - j with je = orl(j0) + 1 for
// the segment's keyroot j0.
#define XTED_COL_FOFF_MASK 0x000fffff
#define XTED_COL_FARCOL (1u << 30)   // column j-1 is a leaf inside the segment: a far column

// Node record (both trees use the same pool): x = label, y = orl | flags.

// Granularity of one tree-size bucket: trees with fewer than max_n nodes use
// this row-run length and these narrow / half-block chunk limits.
#define XTED_TUNE_ROWS 8
struct XTuneRow {
    int32_t max_n, run_rows, narrow_width, half_width;
};

struct XRun {      // a run of keyroots of one depth of a row tree
    int32_t kr_lo; // index into the keyroot pool (global)
    int32_t kr_hi;
    int32_t rows;  // total rows = sum of subtree sizes
    int32_t depth;
};

struct XChunk {     // a run of whole segments of one depth of a column tree
    int32_t k_lo;   // keyroot-pool index of its first segment
    int32_t width;
    int32_t depth;
    int32_t nseg;
};

struct XPair {
    int64_t dt_off;   // element offset of this pair's m x n distance table
    int32_t m, n;     // rows (A) and columns (B)
    int32_t row_base; // index of A's node 0 in the node-record pool
    int32_t col_base; // index of B's node 0 in the node-record pool
};

struct XUnit {
    int32_t run;   // global run index (row tree)
    int32_t chunk; // global chunk index (column tree)
};

#define XTED_TASK_WIDE 0x80000000u  // one unit run by the whole block
#define XTED_TASK_STRIPED 0x20000000u  // (with WIDE) one column stripe of a striped unit
// Striped units: a single column segment wider than the register paths
// (XTED_WIDE_REG_MAX columns) is split into column stripes of 256 * sww
// columns, and every stripe is a task of its own: kind_n = WIDE | STRIPED |
// (stripe << XTED_STRIPE_SHIFT) | 1, unit_lo = the striped unit's index in
// XKernelParams::stripes. The K stripes of a unit are consecutive tasks of
// its level, rightmost first, and blocks claim a level's tasks in index order:
// the stripe a block waits for (its right neighbour, which passes it the row
// carries) has always been claimed before, by a block that is running it or
// has finished it. Any block runs any stripe, one block runs them all in turn.
#define XTED_STRIPE_SHIFT 16
#define XTED_STRIPE_MASK 0xfffu
#define XTED_STRIPE 2048        // widest stripe (8 columns per thread)
#define XTED_STRIPE_MIN_W 2     // narrowest stripe: 2 columns per thread (512 columns)
#define XTED_STRIPES_MAX 128    // stripes of one unit: a wider segment takes wider stripes
#define XTED_STRIPE_PIPE_ROWS 32  // 512-column stripes of a unit with R >= this * K rows pipeline the hand-off
#define XTED_STRIPE_MIN_CELLS_DEFAULT ((int64_t)1 << 20)

struct XStripe {       // a striped unit
    int32_t unit;      // its unit
    int32_t K;         // stripes
    int32_t sww;       // columns per thread: a stripe is 256 * sww columns
    int32_t X;         // far columns read across a stripe boundary (exported on every pushed row)
    int32_t w, R;      // width (one segment) and rows
    int32_t pair, pad;
    int64_t map_off;   // its export map (w ints): column -> export index, or -1
    int64_t buf_off;   // carries [K][R], first columns [K][R], exports [R][X]: 64-bit tagged words
};
#define XTED_TASK_HALF 0x40000000u  // units run by the block's two halves (4 warps each)
#define XTED_HALF_MAX 1024          // widest chunk one half block holds in registers (8 per thread)
#define XTED_HALF_DEFAULT 512       // default limit: wider chunks run faster on the whole block
// Per-block scratch ints of a wide unit on the generic path (one segment of
// w > XTED_WIDE_REG_MAX columns, far-row stack of sr rows): rows padded to
// whole columns per thread, prev | loc | column records (int4) | stack.
static inline int64_t xted_wide_big_scratch(int64_t w, int64_t sr) {
    const int64_t wp = (w + XTED_CTA_THREADS - 1) / XTED_CTA_THREADS * XTED_CTA_THREADS;
    return ((2 * wp + 4) & ~(int64_t)3) + 4 * wp + sr * wp;
}

#ifndef XTED_TASK_UNITS
#define XTED_TASK_UNITS 32   // narrow units per task (claimed by the block's warps dynamically)
#endif
#define XTED_PREFETCH 2      // rows of tree distances in flight per unit (cp.async ring depth; 2 measured
                             // faster than 4 or 8 on the mixed batch: the smaller ring leaves more L1)

struct XTask {
    int32_t pair;
    int32_t entry;    // its (pair, level) entry
    uint32_t kind_n;  // XTED_TASK_WIDE | number of units
    int32_t unit_lo;  // first unit
};

// Ready queue. Every (pair, level) is an entry whose tasks are contiguous.
// An entry is published into the ready queue of its priority bucket when the
// last task of the pair's previous level finishes (level 0 at launch), so a
// block only ever claims tasks whose tables' inputs are complete; the
// reference instead runs one host-synchronised level at a time
// (X-TED_CPU/parallel_computing.cpp:155-182, X-TED_GPU/parallel_X_TED.cu:312-387).
#define XTED_BUCKETS 16
// Every bucket has two rings: one for the narrow tasks of its entries (run by
// single warps, a block's warps independently) and one for their group tasks
// (half- and whole-block units, striped units), so that a block busy with
// narrow units can keep claiming narrow work instead of stopping all its
// warps for a group task. Ring index = kind * XTED_BUCKETS + bucket.
#define XTED_KIND_NARROW 0
#define XTED_KIND_GROUP 1
#define XTED_RINGS (2 * XTED_BUCKETS)
// entry_state words per entry: narrow tasks claimed, group tasks claimed, tasks done
#define XTED_ESTATE 3

struct XEntry {
    int32_t task_off;  // first task
    int32_t ntasks;
    int32_t bucket;    // priority: larger = longer remaining critical path of the pair
    int32_t next;      // entry of the pair's next level, -1 after the last level
    int32_t nnarrow;   // tasks [task_off, task_off + nnarrow) are narrow, the rest group tasks
    int32_t pad;
};

struct XKernelParams {
    const int2 *rowinfo;  // node records of every oriented tree
    const int32_t *krd;   // keyroots grouped by depth (node ids within their tree)
    const int32_t *cumw;  // position of each keyroot's segment in its depth's column list
    const XRun *runs;
    const XChunk *chunks;
    const XPair *pairs;
    const XUnit *units;
    const XTask *tasks;
    const XEntry *entries;
    const int32_t *first;  // [npairs] level-0 entry of every pair, -1 for pairs with an empty tree
    int32_t *dt;          // all distance tables
    int32_t *scratch;     // per-block far-row stacks (and wide generic rows)
    int64_t scratch_per_cta; // int32 elements
    int32_t stack_rows;   // stack capacity in rows
    int32_t ntasks;
    int32_t nentries, npairs;
    int32_t *entry_state; // [XTED_ESTATE * nentries]: narrow claimed, group claimed, done
    // Ring g's slots are rq[g << rq_log2 ...]; queue position pos lives in
    // slot pos & (2^rq_log2 - 1) as (pos << 32 | entry), so a reader knows a
    // slot holds position pos and not an older or not-yet-written one.
    unsigned long long *rq;
    int32_t rq_log2;
    int32_t *rq_ctl;      // [2 * XTED_RINGS]: head, tail of each ring (unsigned positions), then counters
    int32_t *done_total;  // finished tasks
    int32_t *error;       // 0 = ok; else an XTED error code
    int32_t *error_info;  // [4] diagnostics of the first error
    uint64_t timeout_ns;  // bound on every idle wait
    unsigned long long *trace; // optional, 4 words per task: claim ns, start ns, end ns, info
    // ---- striped units (nstriped = 0: none) ----
    const XStripe *stripes;
    const int32_t *smap;        // export maps
    unsigned long long *sbuf;   // carries, first columns, exports (zeroed per run)
    int64_t sbuf_words;
    int32_t nstriped;
    // ---- serving session (serve = 1); a batch launch leaves these zero ----
    int32_t serve;
    int32_t serve_pairs;    // pairs per query slot (the corpus size)
    uint64_t idle_exit_ns;  // a block with no work for this long leaves the launch
    int32_t *mbox;          // XTED_MBOX_* words and records, device memory
    int32_t *slot_done;     // [XTED_SERVE_SLOTS] pairs finished in the slot's current query
    const int32_t *slot_need, *slot_gen;  // pairs to finish, generation to report
    int32_t *results;       // [slots * serve_pairs] distances, mapped host memory
    int32_t *flags;         // [XTED_SERVE_SLOTS] generation of the last finished query, mapped host memory
    // ---- test hook (xted_test_fault): level 0 of this pair is never published; -1: none ----
    int32_t hold_pair;
    // ---- edit costs: delete a row-tree node, insert a column-tree node, change a label ----
    int32_t c_del, c_ins, c_ren;
};

// Serving mailbox in device memory. The host writes records and then the
// posted count with stream-ordered copies; blocks claim records in order and
// publish level 0 of the record's pairs into the running launch's ready queue.
#define XTED_SERVE_SLOTS 16
#define XTED_SERVE_RECS 64
#define XTED_MBOX_POSTED 0    // records posted (host)
#define XTED_MBOX_STOP 1      // nonzero: blocks leave when idle (host)
#define XTED_MBOX_CONSUMED 2  // records claimed (device), | XTED_MBOX_CLOSED once the launch leaves
#define XTED_MBOX_CLOSED (1 << 30)  // set by the block that ends the launch: no record is claimed after it
#define XTED_MBOX_TOP 3       // bucket of the oldest query in flight (host)
#define XTED_MBOX_REC 4       // records: 4 ints each {slot, pair_lo, npairs, 0}
#define XTED_MBOX_INTS (XTED_MBOX_REC + 4 * XTED_SERVE_RECS)
