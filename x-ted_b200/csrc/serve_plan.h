// serve_plan.h -- host-side planning of serving queries against a resident
// corpus (no CUDA runtime calls; the CPU emulation test includes it too).
//
// Pool layout: the corpus trees first (planned once, both orientations),
// then one fixed region per query slot sized for XTED_SERVE_MAX_QUERY nodes.
// A query is planned into its slot's region with the batch planner's own
// functions (plan_core.h): every (corpus tree, query) pair, the corpus tree
// as the row tree, so the far-row stack depth of every pair is bounded by a
// corpus property known at load time.
#pragma once

#include <algorithm>
#include <climits>
#include <cstring>
#include <vector>

#include "../../include/xted.h"
#include "plan_core.h"

namespace xted {

struct ServePools {
    int T = 0, S = 0, Qmax = 0;
    int64_t N = 0, R = 0;  // corpus nodes and raw ints
    std::vector<int32_t> raw;
    std::vector<DTree> trees;  // T corpus trees, then S slot trees
    std::vector<int32_t> size, depth, parent, krd, cumw, opar, okd, oka;
    std::vector<int2> node;
    std::vector<XRun> runs;
    std::vector<XChunk> chunks;
    std::vector<DDepth> depths;
    std::vector<DOTree> otrees;
    PlanPools P{};
    int32_t stack_rows = 1;  // far-row stack rows any pair needs (corpus rows)
};

// A planned query. Offsets are relative (pairs from 0, entries, units and
// tasks from 0, tables from 0) until serve_fixup moves them to the slot's
// device ranges.
struct QPlan {
    std::vector<XPair> pairs;     // [T]
    std::vector<int32_t> first;   // [T] level-0 entry, -1 for an empty-tree pair
    std::vector<int32_t> trivial; // [T] distance of an empty-tree pair, else -1
    std::vector<XEntry> entries;
    std::vector<XUnit> units;
    std::vector<XTask> tasks;
    int64_t dt_elems = 0, cells = 0;
    int32_t need = 0;             // pairs the device computes
};

// Lays out the pools and plans the corpus. The trees must be valid.
inline void serve_pools_build(ServePools &s, const xted_tree *tr, int T, int S, int Qmax, int run_rows,
                              int narrow_width, int half_width, const XTuneRow *tune = nullptr, int ntune = 0) {
    s.T = T;
    s.S = S;
    s.Qmax = Qmax;
    int64_t N = 0, R = 0;
    for (int t = 0; t < T; t++) {
        N += tr[t].n;
        R += 3 * (int64_t)tr[t].n + 1;
    }
    s.N = N;
    s.R = R;
    const int64_t Nall = N + (int64_t)S * Qmax;
    s.raw.assign((size_t)(R + (int64_t)S * (3 * Qmax + 1)), 0);
    s.trees.resize((size_t)(T + S));
    int64_t rpos = 0, nb = 0;
    for (int t = 0; t < T; t++) {
        DTree &d = s.trees[(size_t)t];
        const int n = tr[t].n;
        d.n = n;
        d.raw = (int32_t)rpos;
        d.nbase = (int32_t)nb;
        d.t = t;
        d.S[0] = d.S[1] = 0;
        if (n > 0) {
            std::memcpy(&s.raw[(size_t)rpos], tr[t].labels, 4 * (size_t)n);
            std::memcpy(&s.raw[(size_t)rpos + n], tr[t].child_off, 4 * ((size_t)n + 1));
            if (n > 1) std::memcpy(&s.raw[(size_t)rpos + 2 * n + 1], tr[t].child_idx, 4 * ((size_t)n - 1));
        }
        rpos += 3 * (int64_t)n + 1;
        nb += n;
    }
    for (int i = 0; i < S; i++) {
        DTree &d = s.trees[(size_t)(T + i)];
        d.n = 0;
        d.raw = (int32_t)(R + (int64_t)i * (3 * Qmax + 1));
        d.nbase = (int32_t)(N + (int64_t)i * Qmax);
        d.t = T + i;
        d.S[0] = d.S[1] = 0;
    }
    const size_t n1 = (size_t)std::max<int64_t>(Nall, 1), n2 = 2 * n1;
    s.size.assign(n1, 0);
    s.depth.assign(n1, 0);
    s.parent.assign(n1, 0);
    s.node.assign(n2, int2{0, 0});
    s.krd.assign(n2, 0);
    s.cumw.assign(n2, 0);
    s.opar.assign(n2, 0);
    s.okd.assign(n2, 0);
    s.oka.assign(n2, 0);
    s.runs.assign(n2, XRun{0, 0, 0, 0});
    s.chunks.assign(n2, XChunk{0, 0, 0, 0});
    s.depths.assign(2 * (n1 + (size_t)(T + S)), DDepth{});
    s.otrees.assign(2 * (size_t)(T + S), DOTree{});
    PlanPools &P = s.P;
    P.raw = s.raw.data();
    P.trees = s.trees.data();
    P.ntrees = T + S;
    P.size = s.size.data();
    P.depth = s.depth.data();
    P.parent = s.parent.data();
    P.node = s.node.data();
    P.krd = s.krd.data();
    P.cumw = s.cumw.data();
    P.runs = s.runs.data();
    P.chunks = s.chunks.data();
    P.opar = s.opar.data();
    P.okd = s.okd.data();
    P.oka = s.oka.data();
    P.depths = s.depths.data();
    P.otrees = s.otrees.data();
    P.run_rows = run_rows;
    P.narrow_width = narrow_width;
    P.half_width = half_width;
    P.ntune = 0;
    for (int k = 0; k < ntune && k < XTED_TUNE_ROWS; k++) P.tune[P.ntune++] = tune[k];
    s.stack_rows = 1;
    for (int t = 0; t < T; t++) {
        tree_basic(P, t, s.trees.data());
        orient_tree(P, 2 * t);
        orient_tree(P, 2 * t + 1);
        for (int o = 0; o < 2; o++) s.stack_rows = std::max(s.stack_rows, s.otrees[2 * (size_t)t + o].maxka + 1);
    }
}

// Plans query (lab, off, idx, n <= Qmax, valid) in slot `slot`: the tree into
// the slot's region, then every (corpus tree, query) pair as the batch
// planner does (k_pair_setup ... k_level_fill in prep.cu); with `include`,
// only the pairs of the corpus trees it marks (pairs with an empty tree are
// always answered on the host).
inline void serve_plan_query(ServePools &s, int slot, const int32_t *lab, const int32_t *off, const int32_t *idx,
                             int n, int orientation, int narrow_width, int wide_rows, QPlan &out,
                             const uint8_t *include = nullptr) {
    const int T = s.T, tq = T + slot;
    DTree &Q = s.trees[(size_t)tq];
    Q.n = n;
    int32_t *r = s.raw.data() + Q.raw;
    if (n > 0) {
        std::memcpy(r, lab, 4 * (size_t)n);
        std::memcpy(r + n, off, 4 * ((size_t)n + 1));
        if (n > 1) std::memcpy(r + 2 * n + 1, idx, 4 * ((size_t)n - 1));
    } else {
        r[0] = 0;
    }
    tree_basic(s.P, tq, s.trees.data());
    orient_tree(s.P, 2 * tq);
    orient_tree(s.P, 2 * tq + 1);

    out = QPlan{};
    std::vector<DPair> dp((size_t)T);
    out.pairs.resize((size_t)T);
    out.first.assign((size_t)T, -1);
    out.trivial.assign((size_t)T, -1);
    std::vector<DLevel> lv;
    int64_t dt = 0;
    for (int t = 0; t < T; t++) {
        const int32_t pt[2] = {t, tq};
        pair_setup(s.trees.data(), s.otrees.data(), pt, orientation, 0, &dp[(size_t)t]);
        DPair &d = dp[(size_t)t];
        XPair &x = out.pairs[(size_t)t];
        std::memset(&x, 0, sizeof(x));
        if (d.trivial >= 0) {
            out.trivial[(size_t)t] = d.trivial;
            continue;
        }
        if (include && !include[t]) continue;  // not computed in this round (first = -1)
        x.dt_off = dt;
        x.m = s.trees[(size_t)t].n;
        x.n = n;
        x.row_base = s.otrees[2 * (size_t)t + d.o].node_base;
        x.col_base = s.otrees[2 * (size_t)tq + d.o].node_base;
        dt += (int64_t)x.m * x.n;
        d.lvl_base = (int32_t)lv.size();
        out.first[(size_t)t] = d.lvl_base;
        for (int l = 0; l < d.L; l++) {
            DLevel E{};
            E.pair = t;
            E.level = l;
            lv.push_back(E);
        }
        out.cells += d.cells;
        out.need++;
    }
    out.dt_elems = dt;
    LevelCtx C;
    C.ot = s.otrees.data();
    C.depths = s.depths.data();
    C.runs = s.runs.data();
    C.chunks = s.chunks.data();
    C.pairs = dp.data();
    C.narrow_width = narrow_width;
    C.wide_rows = wide_rows;
    int64_t nu = 0, nt = 0;
    for (size_t e = 0; e < lv.size(); e++) {
        double est;
        level_count(C, lv[e], &est);
        lv[e].unit_off = (int32_t)nu;
        lv[e].task_off = (int32_t)nt;
        lv[e].entry = (int32_t)e;
        nu += (int64_t)lv[e].nwide + lv[e].nnarrow + lv[e].nhalf;
        nt += lv[e].ntasks;
    }
    out.units.resize((size_t)nu);
    out.tasks.resize((size_t)nt);
    out.entries.resize(lv.size());
    for (size_t e = 0; e < lv.size(); e++) {
        const DLevel &E = lv[e];
        level_fill(C, E, out.units.data(), out.tasks.data());
        XEntry &X = out.entries[e];
        X.task_off = E.task_off;
        X.ntasks = E.ntasks;
        X.bucket = 0;
        X.next = E.level + 1 < dp[(size_t)E.pair].L ? (int32_t)e + 1 : -1;
        X.nnarrow = E.nntasks;
        X.pad = 0;
    }
}

// ---- exact top-k pruning ---------------------------------------------------
//
// Unit-cost lower bound of TED(a, b) from the sorted label lists of the two
// trees: an edit mapping M costs (m - |M|) deletions + (n - |M|) insertions
// + its renames, and at most I (the size of the label multisets'
// intersection) of its pairs keep their label, so
//   TED >= m + n - 2|M| + max(0, |M| - I),
// which falls as |M| grows; at |M| = min(m, n) it is max(m, n) - min(m, n, I).
// The same bound under edit costs cd (delete a node of the query, m nodes),
// ci (insert a node of the corpus tree, n nodes) and cr (label change): a
// mapping M costs cd (m - |M|) + ci (n - |M|) + cr max(0, |M| - I), piecewise
// linear in |M|, so its minimum over 0 <= |M| <= min(m, n) is at 0, at
// min(I, m, n) or at min(m, n).
inline int64_t label_common(const int32_t *a, int m, const int32_t *b, int n) {
    int i = 0, j = 0;
    int64_t common = 0;
    while (i < m && j < n) {
        if (a[i] < b[j]) i++;
        else if (b[j] < a[i]) j++;
        else {
            common++;
            i++;
            j++;
        }
    }
    return common;
}
inline int32_t label_lower_bound_cost(int64_t common, int m, int n, int cd, int ci, int cr) {
    const int64_t mn = std::min(m, n), I = std::min<int64_t>(common, mn);
    auto cost = [&](int64_t M) { return (int64_t)cd * (m - M) + (int64_t)ci * (n - M) + (int64_t)cr * std::max<int64_t>(0, M - I); };
    return (int32_t)std::min(cost(0), std::min(cost(I), cost(mn)));
}

inline int32_t label_lower_bound(const int32_t *a, int m, const int32_t *b, int n) {
    int i = 0, j = 0, common = 0;
    while (i < m && j < n) {
        if (a[i] < b[j]) i++;
        else if (b[j] < a[i]) j++;
        else {
            common++;
            i++;
            j++;
        }
    }
    return std::max(m, n) - std::min(std::min(m, n), common);
}

// Preorder bound (S. Guha, H. V. Jagadish, N. Koudas, D. Srivastava, T. Yu,
// SIGMOD 2002): an edit mapping keeps preorder, so its pairs align the two
// trees' preorder label sequences at the same unit cost, and the sequences'
// Levenshtein distance is a lower bound of TED. It dominates the label bound.
//
// Computed with Myers' bit-vector algorithm (G. Myers, J. ACM 46(3), 1999),
// global-distance form (H. Hyyrö, 2003), in 64-row blocks: the pattern's
// column of vertical deltas is held as bit vectors Pv (+1) and Mv (-1), one
// text symbol advances every block by a few word operations, and the score
// D[m][j] follows the horizontal delta leaving the last row.
struct SeqBits {
    int m = 0, W = 0;
    std::vector<uint64_t> peq;  // [rows][W]: bit i of row r set where a[i] is symbol r
    std::vector<int32_t> row;   // dense symbol -> row of peq, -1 where the pattern lacks it

    // a: m dense symbols in [0, alphabet), or -1 for symbols that match nothing
    void build(const int32_t *a, int m_, int alphabet) {
        m = m_;
        W = (m + 63) / 64;
        row.assign((size_t)std::max(alphabet, 1), -1);
        peq.clear();
        for (int i = 0; i < m; i++) {
            if (a[i] < 0) continue;
            int32_t &r = row[(size_t)a[i]];
            if (r < 0) {
                r = (int32_t)(peq.size() / (size_t)W);
                peq.resize(peq.size() + (size_t)W, 0);
            }
            peq[(size_t)r * W + (size_t)(i >> 6)] |= 1ull << (i & 63);
        }
    }

    // Levenshtein distance of the pattern and text b[0..n) (dense symbols or -1).
    int32_t distance(const int32_t *b, int n, std::vector<uint64_t> &work) const {
        if (m == 0) return n;
        work.assign(2 * (size_t)W, 0);
        uint64_t *Pv = work.data(), *Mv = Pv + W;
        for (int w = 0; w < W; w++) Pv[w] = ~0ull;  // D[i][0] = i
        const uint64_t last = 1ull << ((m - 1) & 63);
        int32_t score = m;
        for (int j = 0; j < n; j++) {
            const int32_t r = b[j] >= 0 && b[j] < (int32_t)row.size() ? row[(size_t)b[j]] : -1;
            const uint64_t *E = r >= 0 ? &peq[(size_t)r * W] : nullptr;
            int hin = 1;  // D[0][j] = j: the top row always steps up by one
            for (int w = 0; w < W; w++) {
                uint64_t eq = E ? E[w] : 0;
                const uint64_t pv = Pv[w], mv = Mv[w];
                const uint64_t xv = eq | mv;
                if (hin < 0) eq |= 1;
                const uint64_t xh = (((eq & pv) + pv) ^ pv) | eq;
                uint64_t ph = mv | ~(xh | pv);
                uint64_t mh = pv & xh;
                const uint64_t high = w == W - 1 ? last : (1ull << 63);
                const int hout = (ph & high) ? 1 : ((mh & high) ? -1 : 0);
                ph <<= 1;
                mh <<= 1;
                if (hin < 0) mh |= 1;
                else if (hin > 0) ph |= 1;
                Pv[w] = mh | ~(xv | ph);
                Mv[w] = ph & xv;
                hin = hout;
            }
            score += hin;
        }
        return score;
    }
};

// (distance or bound, corpus index) order: ties go to the lower index.
inline bool key_less(int32_t dx, int32_t x, int32_t dy, int32_t y) { return dx != dy ? dx < dy : x < y; }

// Round 1: of the trees whose distance is unknown (dist < 0), the `want`
// lowest (bound, index); all of them when prune is off or few are unknown.
inline void prune_round1(const std::vector<int32_t> &lb, const std::vector<int32_t> &dist, size_t want, bool prune,
                         std::vector<uint8_t> &inc) {
    const size_t T = lb.size();
    inc.assign(T, 0);
    std::vector<int32_t> order;
    for (size_t t = 0; t < T; t++)
        if (dist[t] < 0) order.push_back((int32_t)t);
    if (prune && order.size() > want) {
        std::nth_element(order.begin(), order.begin() + (long)want, order.end(), [&](int32_t x, int32_t y) {
            return key_less(lb[(size_t)x], x, lb[(size_t)y], y);
        });
        order.resize(want);
    }
    for (int32_t t : order) inc[(size_t)t] = 1;
}

// Round 2: the unknown trees whose (bound, index) beats the k-th smallest
// known (distance, index) -- every unknown tree when fewer than k are known.
// The others cannot enter the top k. Returns false when none is left.
inline bool prune_round2(const std::vector<int32_t> &lb, const std::vector<int32_t> &dist, int k,
                         std::vector<uint8_t> &inc) {
    const size_t T = lb.size();
    std::vector<int32_t> known;
    for (size_t t = 0; t < T; t++)
        if (dist[t] >= 0) known.push_back((int32_t)t);
    int32_t dk = INT32_MAX, ik = INT32_MAX;
    if ((int)known.size() >= k) {
        std::nth_element(known.begin(), known.begin() + (k - 1), known.end(), [&](int32_t x, int32_t y) {
            return key_less(dist[(size_t)x], x, dist[(size_t)y], y);
        });
        ik = known[(size_t)(k - 1)];
        dk = dist[(size_t)ik];
    }
    inc.assign(T, 0);
    bool any = false;
    for (size_t t = 0; t < T; t++)
        if (dist[t] < 0 && key_less(lb[t], (int32_t)t, dk, ik)) {
            inc[t] = 1;
            any = true;
        }
    return any;
}

// The k smallest (distance, index) among the known distances; -1 past them.
inline void topk_known(const std::vector<int32_t> &dist, int k, int32_t *ids, int32_t *dists) {
    std::vector<int32_t> order;
    for (size_t t = 0; t < dist.size(); t++)
        if (dist[t] >= 0) order.push_back((int32_t)t);
    const int kk = std::min<int>(k, (int)order.size());
    std::partial_sort(order.begin(), order.begin() + kk, order.end(), [&](int32_t x, int32_t y) {
        return key_less(dist[(size_t)x], x, dist[(size_t)y], y);
    });
    for (int i = 0; i < k; i++) {
        ids[i] = i < kk ? order[(size_t)i] : -1;
        dists[i] = i < kk ? dist[(size_t)order[(size_t)i]] : -1;
    }
}

// Moves a plan to its device ranges: pairs of slot `slot` start at slot * T,
// tables at dt_off, units at u_off, tasks at t_off, entries at e_off; every
// entry goes to ready-queue bucket `bucket`.
inline void serve_fixup(QPlan &p, int slot, int T, int64_t dt_off, int64_t u_off, int64_t t_off, int64_t e_off,
                        int32_t bucket) {
    const int32_t pair_base = (int32_t)((int64_t)slot * T);
    for (XPair &x : p.pairs) x.dt_off += dt_off;
    for (int32_t &f : p.first)
        if (f >= 0) f += (int32_t)e_off;
    for (XEntry &X : p.entries) {
        X.task_off += (int32_t)t_off;
        X.bucket = bucket;
        if (X.next >= 0) X.next += (int32_t)e_off;
    }
    for (XTask &t : p.tasks) {
        t.pair += pair_base;
        t.entry += (int32_t)e_off;
        t.unit_lo += (int32_t)u_off;
    }
}

}  // namespace xted
