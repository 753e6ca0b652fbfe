// plan_core.h -- keyroot preprocessing and work decomposition, as functions of
// one tree, one pair or one level so they run one-per-thread on the device
// (prep.cu) and sequentially on the host in the planner's CPU test.
//
// Reference counterparts:
//   orl(v) = v + size(v) - 1                  X-TED_CPU/TED.cpp:21-42
//   keyroots = root + non-last children       X-TED_CPU/TED.cpp:46-77 (topmost node per orl)
//   kdepth: bottom-up over parent pointers    X-TED_CPU/parallel_computing.cpp:93-119
//   level of table (i0,j0) = kdepth(i0)+kdepth(j0)   parallel_computing.cpp:121-123
// The left-path decomposition is the right-path one on the mirrored tree
// (children reversed), whose preorder id of node v is n-1-post(v) with
// post(v) = v - depth(v) + size(v) - 1.
#pragma once

#include <stdint.h>

#include "xted_internal.h"

#ifdef __CUDACC__
#define XT_HD __host__ __device__
#else
#define XT_HD
#endif

namespace xted {

// One input tree. Raw preorder CSR in the flat input buffer:
// labels at raw, child_off at raw + n, child_idx at raw + 2n + 1.
struct DTree {
    int32_t n;
    int32_t raw;
    int32_t nbase;  // prefix sum of n over trees (node pools)
    int32_t t;      // tree index
    int64_t S[2];   // keyroot subtree-size sums: right-path, left-path
};

// One depth level of one oriented tree.
struct DDepth {
    int32_t krd_lo, krd_hi;       // keyroots of this depth (pool indices, preorder)
    int32_t run_lo, run_hi;       // row runs
    int32_t chunk_lo, nnarrow, nwide;  // chunks: narrow, then half-block, then whole-block ones
    int32_t maxrows, maxw_n, maxw_w;   // largest run and chunk widths (cost estimates)
    int32_t nhalf, maxw_h;
};

// One tree in one orientation (index 2 * tree + o; o = 1 mirrored).
struct DOTree {
    int32_t n, D, maxka, maxw_wide;
    int32_t node_base;   // rowinfo/krd/cumw/runs/chunks pool base (capacity n each)
    int32_t depth_base;  // DDepth pool base (capacity n + 1)
    int64_t S;
};

struct DPair {
    int32_t ta, tb;      // input trees
    int32_t o;           // orientation: 0 right path, 1 left path (mirrored)
    int32_t L;           // levels (0 for a pair with an empty tree)
    int32_t lvl_base;    // first level entry
    int32_t trivial;     // distance of a pair with an empty tree, else -1
    int64_t dt_off;
    int64_t cells;
};

struct DLevel {
    int32_t pair, level;
    int32_t nwide, nnarrow, nhalf;
    int32_t ntasks, entry;  // tasks at this level; this entry's index
    int32_t nntasks;        // its narrow tasks (the first ones of its range)
    int32_t task_off, unit_off;
    int32_t nstriped, nstripes;    // striped units, and their stripes (tasks)
    int32_t stripe_off;            // its first striped unit
    int64_t key;            // estimate, then the earliest start of the level (see k_pair_rank)
};

struct PlanPools {
    const int32_t *raw;   // input trees
    const DTree *trees;
    int32_t ntrees;
    // per input tree node scratch (original numbering)
    int32_t *size, *depth, *parent;
    // per oriented tree node pools (capacity 2 * sum n)
    int2 *node;           // rowinfo: label, orl | flags
    int32_t *krd, *cumw;  // keyroots by depth, their column-list position within the depth
    XRun *runs;
    XChunk *chunks;
    int32_t *opar, *okd, *oka;  // orientation scratch
    DDepth *depths;       // capacity 2 * (sum n + ntrees)
    DOTree *otrees;
    int32_t run_rows, narrow_width;
    int32_t half_width;   // chunks wider than narrow_width up to this run on half a block
    // per tree-size bucket granularity (autotuned); ntune == 0: the three fields above
    int32_t ntune;
    XTuneRow tune[XTED_TUNE_ROWS];
};

// The granularity a tree of n nodes is planned with.
XT_HD inline void tree_granularity(const PlanPools &P, int n, int *run_rows, int *narrow_width, int *half_width) {
    *run_rows = P.run_rows;
    *narrow_width = P.narrow_width;
    *half_width = P.half_width;
    for (int k = 0; k < P.ntune; k++)
        if (n < P.tune[k].max_n || k == P.ntune - 1) {
            *run_rows = P.tune[k].run_rows;
            *narrow_width = P.tune[k].narrow_width;
            *half_width = P.tune[k].half_width;
            return;
        }
}

XT_HD inline int32_t mirror_id(int32_t v, int32_t n, const int32_t *size, const int32_t *depth) {
    return n - 1 - (v - depth[v] + size[v] - 1);
}

// Sizes, depths, parents and both keyroot-size sums of input tree t.
XT_HD inline void tree_basic(const PlanPools &P, int t, DTree *trees_out) {
    DTree T = P.trees[t];
    const int n = T.n;
    const int32_t *off = P.raw + T.raw + n;
    const int32_t *idx = P.raw + T.raw + 2 * n + 1;
    int32_t *size = P.size + T.nbase, *depth = P.depth + T.nbase, *par = P.parent + T.nbase;
    T.S[0] = T.S[1] = 0;
    if (n > 0) {
        par[0] = -1;
        depth[0] = 0;
        for (int v = 0; v < n; v++)
            for (int32_t e = off[v]; e < off[v + 1]; e++) {
                par[idx[e]] = v;
                depth[idx[e]] = depth[v] + 1;
            }
        for (int v = n - 1; v >= 0; v--) {
            int32_t s = 1;
            for (int32_t e = off[v]; e < off[v + 1]; e++) s += size[idx[e]];
            size[v] = s;
        }
        int64_t sr = size[0], sl = size[0];
        for (int v = 0; v < n; v++) {
            const int32_t lo = off[v], hi = off[v + 1];
            for (int32_t e = lo; e < hi; e++) {
                if (e != hi - 1) sr += size[idx[e]];
                if (e != lo) sl += size[idx[e]];
            }
        }
        T.S[0] = sr;
        T.S[1] = sl;
    }
    trees_out[t] = T;
}

// Cycles one row of a unit takes under full load (fitted to per-task traces
// of the mixed batch): a warp's narrow row, a block's wide row.
XT_HD inline double row_cost_est(bool wide, int width) {
    if (width <= 0) return 0.0;
    if (!wide) return 2800.0 + 6.0 * width;
    return 1300.0 + 0.7 * width;
}
XT_HD inline double row_cost_half(int width) { return width <= 0 ? 0.0 : 1600.0 + 1.4 * width; }

// Half-block units of one level are bundled into tasks of this many units
// (the block's two halves claim them one at a time).
XT_HD inline int32_t level_bundle_half(int64_t nhalf) {
    int64_t b = (nhalf + 15) / 16;
    if (b < 2) b = 2;
    if (b > 8) b = 8;
    return (int32_t)b;
}

// Narrow units of one level are bundled into tasks of this many units (the
// block's 8 warps claim them one at a time): small bundles when the level has
// few units, so its units spread over several blocks and the level (often on
// a pair's critical path) finishes sooner; up to XTED_TASK_UNITS when there
// are plenty, to keep per-task overhead low.
#ifndef XTED_BUNDLE_MIN
#define XTED_BUNDLE_MIN XTED_WARPS
#endif
#ifndef XTED_BUNDLE_DIV
#define XTED_BUNDLE_DIV 16
#endif
XT_HD inline int32_t level_bundle(int64_t nnarrow) {
    int64_t b = (nnarrow + XTED_BUNDLE_DIV - 1) / XTED_BUNDLE_DIV;
    if (b < XTED_BUNDLE_MIN) b = XTED_BUNDLE_MIN;
    if (b > XTED_TASK_UNITS) b = XTED_TASK_UNITS;
    return (int32_t)b;
}

// Narrow units of a run longer than this many rows are tasks of one unit
// each: a bundle of them would run its units a few at a time on one block's
// warps (4 rounds for 32 units on 8 warps), while single-unit tasks spread
// over the warps of several blocks. Such runs are the few big keyroots of
// large trees, whose levels are short of parallel work.
#ifndef XTED_LONG_RUN_ROWS
#define XTED_LONG_RUN_ROWS 4096
#endif
XT_HD inline bool long_run_rows(int32_t rows) { return rows > XTED_LONG_RUN_ROWS; }

// Builds oriented tree ot = 2 t + o: node records, keyroot depths, keyroots
// grouped by depth, column-list positions, row runs and column chunks.
XT_HD inline void orient_tree(const PlanPools &P, int ot) {
    const int t = ot >> 1, o = ot & 1;
    const DTree T = P.trees[t];
    const int n = T.n;
    DOTree O;
    O.n = n;
    O.node_base = 2 * T.nbase + o * n;
    O.depth_base = 2 * (T.nbase + t) + o * (n + 1);
    O.D = -1;
    O.maxka = 0;
    O.maxw_wide = 0;
    O.S = T.S[o];
    if (n == 0) {
        P.otrees[ot] = O;
        return;
    }
    const int32_t *lab = P.raw + T.raw;
    const int32_t *off = P.raw + T.raw + n;
    const int32_t *idx = P.raw + T.raw + 2 * n + 1;
    const int32_t *size = P.size + T.nbase, *depth = P.depth + T.nbase, *par = P.parent + T.nbase;
    int2 *node = P.node + O.node_base;
    int32_t *opar = P.opar + O.node_base, *okd = P.okd + O.node_base, *oka = P.oka + O.node_base;
    // node records in this orientation
    for (int v = 0; v < n; v++) {
        const int32_t u = o ? mirror_id(v, n, size, depth) : v;
        bool kr = true;
        if (v > 0) {
            const int32_t p = par[v];
            kr = o ? idx[off[p]] != v : idx[off[p + 1] - 1] != v;
            opar[u] = o ? mirror_id(p, n, size, depth) : p;
        } else {
            opar[u] = -1;
        }
        node[u].x = lab[v];
        node[u].y = (int32_t)((uint32_t)(u + size[v] - 1) | (kr ? XTED_ROW_ISKR : 0u));
    }
    for (int u = 1; u < n; u++) {
        const int32_t prev_orl = node[u - 1].y & XTED_ROW_ORL_MASK;
        if (prev_orl == u - 1) node[u].y = (int32_t)((uint32_t)node[u].y | XTED_ROW_PREVLEAF);
    }
    // keyroot depth bottom-up: oka[u] collects the max over u's children of
    // f(child) = max kdepth of keyroots in the child's subtree (-1 if none)
    for (int u = 0; u < n; u++) oka[u] = -1;
    for (int u = n - 1; u >= 0; u--) {
        const bool kr = (node[u].y & XTED_ROW_ISKR) != 0;
        const int32_t f = kr ? oka[u] + 1 : oka[u];
        okd[u] = kr ? f : -1;
        if (u > 0 && f > oka[opar[u]]) oka[opar[u]] = f;
    }
    O.D = okd[0];
    // keyroots on each root path
    int32_t maxka = 1;
    oka[0] = 1;
    for (int u = 1; u < n; u++) {
        oka[u] = oka[opar[u]] + ((node[u].y & XTED_ROW_ISKR) ? 1 : 0);
        if (oka[u] > maxka) maxka = oka[u];
    }
    O.maxka = maxka;
    // keyroots grouped by depth (counting sort, preorder inside a depth)
    DDepth *dep = P.depths + O.depth_base;
    const int D = O.D;
    for (int d = 0; d <= D; d++) {
        dep[d].krd_lo = 0;
        dep[d].krd_hi = 0;
    }
    for (int u = 0; u < n; u++)
        if (okd[u] >= 0) dep[okd[u]].krd_hi++;
    int32_t acc = O.node_base;
    for (int d = 0; d <= D; d++) {
        const int32_t c = dep[d].krd_hi;
        dep[d].krd_lo = acc;
        dep[d].krd_hi = acc;  // fill cursor
        acc += c;
    }
    for (int u = 0; u < n; u++)
        if (okd[u] >= 0) P.krd[dep[okd[u]].krd_hi++] = u;
    // column-list positions, row runs and chunks per depth
    int run_rows, nw, hw;
    tree_granularity(P, n, &run_rows, &nw, &hw);
    const int group_w = nw > 0 ? nw : XTED_NARROW_MAX;
    const int half_w = hw > nw ? (hw < XTED_HALF_MAX ? hw : XTED_HALF_MAX) : nw;
    int32_t run_cur = O.node_base, chunk_cur = O.node_base;
    for (int d = 0; d <= D; d++) {
        DDepth &dd = dep[d];
        int32_t pos = 0;
        dd.maxrows = 0;
        // runs
        dd.run_lo = run_cur;
        XRun r{-1, -1, 0, d};
        for (int32_t k = dd.krd_lo; k < dd.krd_hi; k++) {
            const int32_t u = P.krd[k];
            const int32_t sz = (node[u].y & XTED_ROW_ORL_MASK) - u + 1;
            P.cumw[k] = pos;
            pos += sz;
            if (r.kr_lo >= 0 && r.rows + sz > run_rows) {
                if (r.rows > dd.maxrows) dd.maxrows = r.rows;
                P.runs[run_cur++] = r;
                r = XRun{-1, -1, 0, d};
            }
            if (r.kr_lo < 0) r.kr_lo = k;
            r.kr_hi = k + 1;
            r.rows += sz;
        }
        if (r.kr_lo >= 0) {
            if (r.rows > dd.maxrows) dd.maxrows = r.rows;
            P.runs[run_cur++] = r;
        }
        dd.run_hi = run_cur;
        // chunks: three passes, narrow chunks first, then half-block ones, then whole-block ones
        dd.chunk_lo = chunk_cur;
        dd.nnarrow = dd.nwide = dd.nhalf = 0;
        dd.maxw_n = dd.maxw_w = dd.maxw_h = 0;
        for (int pass = 0; pass < 3; pass++) {
            XChunk c{-1, 0, d, 0};
            for (int32_t k = dd.krd_lo; k <= dd.krd_hi; k++) {
                int32_t w = 0;
                if (k < dd.krd_hi) {
                    const int32_t u = P.krd[k];
                    w = (node[u].y & XTED_ROW_ORL_MASK) - u + 1;
                }
                const bool flush = c.nseg > 0 && (k == dd.krd_hi || c.width + w > group_w);
                if (flush) {
                    const int kind = c.width <= nw ? 0 : (c.width <= half_w ? 1 : 2);
                    if (kind == pass) {
                        P.chunks[chunk_cur++] = c;
                        if (kind == 2) {
                            dd.nwide++;
                            if (c.width > dd.maxw_w) dd.maxw_w = c.width;
                        } else if (kind == 1) {
                            dd.nhalf++;
                            if (c.width > dd.maxw_h) dd.maxw_h = c.width;
                        } else {
                            dd.nnarrow++;
                            if (c.width > dd.maxw_n) dd.maxw_n = c.width;
                        }
                    }
                    c = XChunk{-1, 0, d, 0};
                }
                if (k == dd.krd_hi) break;
                if (c.nseg == 0) c.k_lo = k;  // first segment (keyroot pool index)
                c.width += w;
                c.nseg += 1;
            }
        }
        if (dd.maxw_h > O.maxw_wide) O.maxw_wide = dd.maxw_h;
        if (dd.maxw_w > O.maxw_wide) O.maxw_wide = dd.maxw_w;
    }
    P.otrees[ot] = O;
}

// Orientation, level count and table offset of pair p.
XT_HD inline void pair_setup(const DTree *trees, const DOTree *ot, const int32_t *pair_trees, int orientation,
                             int p, DPair *pairs) {
    DPair q;
    q.ta = pair_trees[2 * p];
    q.tb = pair_trees[2 * p + 1];
    const DTree &A = trees[q.ta], &B = trees[q.tb];
    q.trivial = -1;
    q.o = 0;
    q.L = 0;
    q.cells = 0;
    q.dt_off = 0;
    q.lvl_base = 0;
    if (A.n == 0 || B.n == 0) {  // X-TED_CPU/TED.cpp:181-186
        q.trivial = A.n == 0 ? B.n : A.n;
    } else {
        const int64_t cr = A.S[0] * B.S[0], cl = A.S[1] * B.S[1];
        q.o = orientation == XTED_ORIENT_LEFT || (orientation == XTED_ORIENT_AUTO && cl < cr);
        q.cells = q.o ? cl : cr;
        q.L = ot[2 * q.ta + q.o].D + ot[2 * q.tb + q.o].D + 1;
    }
    pairs[p] = q;
}

struct LevelCtx {
    const DOTree *ot;
    const DDepth *depths;
    const XRun *runs;
    const XChunk *chunks;
    const DPair *pairs;
    int32_t narrow_width;
    int32_t wide_rows;  // narrow-chunk units of runs longer than this are wide tasks (< 0: none)
    int64_t stripe_min_cells = 0;  // > 0: wide single-segment units with this many cells run in stripes
};

// A unit of a narrow chunk whose run is long (one big keyroot) would keep a
// whole block waiting on one warp; it runs on the whole block instead.
XT_HD inline bool big_run(const LevelCtx &C, int32_t run) {
    return C.wide_rows >= 0 && C.runs[run].rows > C.wide_rows;
}

// Columns per thread of a striped segment of w columns: the narrowest stripes
// (512 columns) unless that makes more than XTED_STRIPES_MAX of them. Narrow
// stripes run a table's rows on more blocks at once; a stripe row costs
// little more at 512 columns than at 2,048.
XT_HD inline int32_t stripe_sww(int32_t w) {
    int32_t sww = XTED_STRIPE_MIN_W;
    while (sww < XTED_STRIPE / XTED_CTA_THREADS &&
           (w + XTED_CTA_THREADS * sww - 1) / (XTED_CTA_THREADS * sww) > XTED_STRIPES_MAX)
        sww *= 2;
    return sww;
}
XT_HD inline int32_t stripe_count(int32_t w) {
    const int32_t sw = XTED_CTA_THREADS * stripe_sww(w);
    return (w + sw - 1) / sw;
}
// A whole-block unit of `rows` rows over one segment of w columns runs in
// column stripes (else on one block, the generic wide path).
#ifndef XTED_STRIPE_MIN_WIDTH
#define XTED_STRIPE_MIN_WIDTH XTED_WIDE_REG_MAX  // (tests of the plan's layout build with less)
#endif
XT_HD inline bool striped_unit(const LevelCtx &C, int32_t rows, int32_t w) {
    return C.stripe_min_cells > 0 && w > XTED_STRIPE_MIN_WIDTH && stripe_count(w) <= XTED_STRIPES_MAX &&
           (int64_t)rows * w >= C.stripe_min_cells;
}

// Units and tasks of level entry e (pair, level) and its time estimate.
XT_HD inline void level_count(const LevelCtx &C, DLevel &E, double *est_out) {
    const DPair &q = C.pairs[E.pair];
    const DOTree &A = C.ot[2 * q.ta + q.o], &B = C.ot[2 * q.tb + q.o];
    const DDepth *da = C.depths + A.depth_base, *db = C.depths + B.depth_base;
    const int d = E.level;
    int64_t wide = 0, narrow = 0, half = 0, nlong = 0, nstriped = 0, nstripes = 0, nhlong = 0;
    const int lo = d - B.D > 0 ? d - B.D : 0, hi = A.D < d ? A.D : d;
    int32_t small_max[64];  // longest bundled run per depth (the first 64 depths; more use maxrows)
    int32_t long_max[64];   // longest run of single-unit narrow tasks (or paired half units) per depth
    int32_t half_max[64];   // longest run of bundled half units per depth
    for (int al = lo; al <= hi; al++) {
        const DDepth &ra = da[al], &cb = db[d - al];
        const int64_t nr = ra.run_hi - ra.run_lo;
        int64_t nbig = 0, nl = 0, nlh = 0;
        int32_t sm = 0, lm = 0, hm = 0;
        if (cb.nnarrow > 0 || cb.nhalf > 0)
            for (int32_t r = ra.run_lo; r < ra.run_hi; r++) {
                const int32_t rows = C.runs[r].rows;
                const bool lr = long_run_rows(rows);
                if (lr && rows > lm) lm = rows;
                if (lr) nlh++;
                else if (rows > hm) hm = rows;
                if (big_run(C, r)) nbig++;
                else if (lr) nl++;
                else if (rows > sm) sm = rows;
            }
        if (al - lo < 64) {
            small_max[al - lo] = sm;
            long_max[al - lo] = lm;
            half_max[al - lo] = hm;
        }
        nhlong += nlh * cb.nhalf;
        wide += nr * cb.nwide + nbig * cb.nnarrow;
        half += nr * cb.nhalf;
        if (C.stripe_min_cells > 0 && cb.maxw_w > XTED_STRIPE_MIN_WIDTH) {
            const int32_t cw_lo = cb.chunk_lo + cb.nnarrow + cb.nhalf;
            for (int32_t r = ra.run_lo; r < ra.run_hi; r++)
                for (int32_t c = cw_lo; c < cw_lo + cb.nwide; c++)
                    if (striped_unit(C, C.runs[r].rows, C.chunks[c].width)) {
                        nstriped++;
                        nstripes += stripe_count(C.chunks[c].width);
                    }
        }
        narrow += (nr - nbig) * cb.nnarrow;
        nlong += nl * cb.nnarrow;
    }
    const int32_t bundle = level_bundle(narrow);
    const int rounds = (bundle + XTED_WARPS - 1) / XTED_WARPS;  // units a warp runs in one task
    const int32_t bundle_h = level_bundle_half(half);
    const int rounds_h = (bundle_h + 1) / 2;                     // units a half block runs in one task
    // the level's longest task: its largest run against its widest chunk
    double est = 0.0;
    for (int al = lo; al <= hi; al++) {
        const DDepth &ra = da[al], &cb = db[d - al];
        double e = 0.0;
        if (cb.nnarrow > 0) {
            const int32_t sm = al - lo < 64 ? small_max[al - lo] : ra.maxrows;
            const int32_t lm = al - lo < 64 ? long_max[al - lo] : ra.maxrows;
            e = rounds * sm * row_cost_est(false, cb.maxw_n);
            const double el = lm * row_cost_est(false, cb.maxw_n);
            if (el > e) e = el;
            if (C.wide_rows >= 0 && ra.maxrows > C.wide_rows) {
                const double eb = ra.maxrows * row_cost_est(true, cb.maxw_n);
                if (eb > e) e = eb;
            }
        }
        if (cb.nhalf > 0) {
            const int32_t hm = al - lo < 64 ? half_max[al - lo] : ra.maxrows;
            const int32_t lm = al - lo < 64 ? long_max[al - lo] : ra.maxrows;
            const double eh = rounds_h * hm * row_cost_half(cb.maxw_h), el = lm * row_cost_half(cb.maxw_h);
            if (eh > e) e = eh;
            if (el > e) e = el;
        }
        if (cb.nwide > 0) {
            const double ew = ra.maxrows * row_cost_est(true, cb.maxw_w);
            if (ew > e) e = ew;
        }
        if (e > est) est = e;
    }
    E.nwide = (int32_t)wide;
    E.nnarrow = (int32_t)narrow;
    E.nhalf = (int32_t)half;
    E.nntasks = (int32_t)((narrow - nlong + bundle - 1) / bundle + nlong);
    E.nstriped = (int32_t)nstriped;
    E.nstripes = (int32_t)nstripes;
    // half units of long runs go two to a task (one per half), the others in bundles
    E.ntasks = (int32_t)(wide - nstriped + nstripes + E.nntasks + (nhlong + 1) / 2 +
                         (half - nhlong + bundle_h - 1) / bundle_h);
    *est_out = est;
}

// Ready-queue bucket of a level whose pair has `remaining` estimated time left
// (this level included) when the longest pair of the batch has `chain_max`.
// Half-octave scale: bucket 15 holds the levels within a factor sqrt(2) of
// the longest chain, each bucket below another factor sqrt(2) less, so pairs
// with mid-length chains keep priority over the many short ones instead of
// sharing the lowest bucket with them.
XT_HD inline int32_t level_bucket(int64_t remaining, int64_t chain_max) {
    double x = remaining > 0 ? (double)remaining : 1.0;
    const double lim = (double)chain_max;
    int32_t b = XTED_BUCKETS - 1;
    while (b > 0 && x * 1.4142135623730951 < lim) {
        x *= 1.4142135623730951;
        b--;
    }
    return b;
}

// Writes the units and tasks of level entry E (offsets already assigned).
XT_HD inline void level_fill(const LevelCtx &C, const DLevel &E, XUnit *units, XTask *tasks,
                             XStripe *stripes = nullptr) {
    const DPair &q = C.pairs[E.pair];
    const DOTree &A = C.ot[2 * q.ta + q.o], &B = C.ot[2 * q.tb + q.o];
    const DDepth *da = C.depths + A.depth_base, *db = C.depths + B.depth_base;
    const int d = E.level;
    int32_t u = E.unit_off, t = E.task_off, so = E.stripe_off;
    const int32_t per_task = level_bundle(E.nnarrow);
    int32_t bundle = 0, bundle_lo = u;
    const int lo = d - B.D > 0 ? d - B.D : 0, hi = A.D < d ? A.D : d;
    for (int al = lo; al <= hi; al++) {
        const DDepth &ra = da[al], &cb = db[d - al];
        for (int32_t r = ra.run_lo; r < ra.run_hi; r++) {
            if (big_run(C, r) || long_run_rows(C.runs[r].rows)) continue;
            for (int32_t c = cb.chunk_lo; c < cb.chunk_lo + cb.nnarrow; c++) {
                if (bundle == 0) bundle_lo = u;
                units[u++] = XUnit{r, c};
                if (++bundle == per_task) {
                    tasks[t++] = XTask{E.pair, E.entry, (uint32_t)bundle, bundle_lo};
                    bundle = 0;
                }
            }
        }
    }
    if (bundle > 0) tasks[t++] = XTask{E.pair, E.entry, (uint32_t)bundle, bundle_lo};
    // Long runs, half-block and whole-block units are laid out from the row
    // tree's deepest keyroots down (most rows first): claimers take a level's
    // tasks of a kind in index order, so the longest units start first.
    for (int al = hi; al >= lo; al--) {  // long runs: a narrow task per unit
        const DDepth &ra = da[al], &cb = db[d - al];
        for (int32_t r = ra.run_lo; r < ra.run_hi; r++) {
            if (big_run(C, r) || !long_run_rows(C.runs[r].rows)) continue;
            for (int32_t c = cb.chunk_lo; c < cb.chunk_lo + cb.nnarrow; c++) {
                units[u] = XUnit{r, c};
                tasks[t++] = XTask{E.pair, E.entry, 1u, u};
                u++;
            }
        }
    }
    // half-block units: those of runs over XTED_LONG_RUN_ROWS rows two to a task
    // (one per half, so the level's longest units do not queue behind each
    // other in one block), then the rest in bundles
    const int32_t per_half = level_bundle_half(E.nhalf);
    bundle = 0;
    for (int al = hi; al >= lo; al--) {
        const DDepth &ra = da[al], &cb = db[d - al];
        for (int32_t r = ra.run_lo; r < ra.run_hi; r++) {
            if (!long_run_rows(C.runs[r].rows)) continue;
            for (int32_t c = cb.chunk_lo + cb.nnarrow; c < cb.chunk_lo + cb.nnarrow + cb.nhalf; c++) {
                if (bundle == 0) bundle_lo = u;
                units[u++] = XUnit{r, c};
                if (++bundle == 2) {
                    tasks[t++] = XTask{E.pair, E.entry, XTED_TASK_HALF | 2u, bundle_lo};
                    bundle = 0;
                }
            }
        }
    }
    if (bundle > 0) tasks[t++] = XTask{E.pair, E.entry, XTED_TASK_WIDE | 1u, bundle_lo};  // a lone one: the whole block
    bundle = 0;
    for (int al = hi; al >= lo; al--) {
        const DDepth &ra = da[al], &cb = db[d - al];
        for (int32_t r = ra.run_lo; r < ra.run_hi; r++) {
            if (long_run_rows(C.runs[r].rows)) continue;
            for (int32_t c = cb.chunk_lo + cb.nnarrow; c < cb.chunk_lo + cb.nnarrow + cb.nhalf; c++) {
                if (bundle == 0) bundle_lo = u;
                units[u++] = XUnit{r, c};
                if (++bundle == per_half) {
                    tasks[t++] = XTask{E.pair, E.entry, XTED_TASK_HALF | (uint32_t)bundle, bundle_lo};
                    bundle = 0;
                }
            }
        }
    }
    // a last task of one half-block unit would leave the block's other half
    // idle for the whole unit: it runs on the whole block instead
    if (bundle > 0)
        tasks[t++] = XTask{E.pair, E.entry, (bundle == 1 ? XTED_TASK_WIDE : XTED_TASK_HALF) | (uint32_t)bundle,
                           bundle_lo};
    for (int al = hi; al >= lo; al--) {
        const DDepth &ra = da[al], &cb = db[d - al];
        const int32_t cw_lo = cb.chunk_lo + cb.nnarrow + cb.nhalf, cw_hi = cw_lo + cb.nwide;
        for (int32_t r = ra.run_lo; r < ra.run_hi; r++) {
            if (big_run(C, r))
                for (int32_t c = cb.chunk_lo; c < cb.chunk_lo + cb.nnarrow; c++) {
                    units[u] = XUnit{r, c};
                    tasks[t++] = XTask{E.pair, E.entry, XTED_TASK_WIDE | 1u, u};
                    u++;
                }
            for (int32_t c = cw_lo; c < cw_hi; c++) {
                units[u] = XUnit{r, c};
                const int32_t w = C.chunks[c].width, rows = C.runs[r].rows;
                if (stripes && striped_unit(C, rows, w)) {
                    // one task per stripe, rightmost first
                    const int32_t K = stripe_count(w);
                    XStripe X;
                    X.unit = u;
                    X.K = K;
                    X.sww = stripe_sww(w);
                    X.X = 0;
                    X.w = w;
                    X.R = rows;
                    X.pair = E.pair;
                    X.pad = 0;
                    X.map_off = 0;
                    X.buf_off = 0;
                    stripes[so] = X;
                    for (int32_t k = K - 1; k >= 0; k--)
                        tasks[t++] = XTask{E.pair, E.entry,
                                           XTED_TASK_WIDE | XTED_TASK_STRIPED | ((uint32_t)k << XTED_STRIPE_SHIFT) | 1u, so};
                    so++;
                } else {
                    tasks[t++] = XTask{E.pair, E.entry, XTED_TASK_WIDE | 1u, u};
                }
                u++;
            }
        }
    }
}

}  // namespace xted
