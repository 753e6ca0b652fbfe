// plan_emu.cpp -- TEST INFRASTRUCTURE: checks the batch planner on the CPU.
//
// Runs the planner's per-tree / per-pair / per-level functions (plan_core.h,
// the same code the device planning kernels run one-per-thread) sequentially,
// orders the level entries by their keys, and executes every unit with the row
// formulation of the kernels (columns derived from node records, row scan with
// segment keys, far-row stack), task by task in queue order. It checks the
// plan's invariants (dependency order, single write of every tree cell, every
// read cell already written, stack discipline, unit coverage) and the distances
// against the oracle's restatement of X-TED_CPU.
//   usage: plan_emu <iterations> <max_nodes> <seed> [stack window rows, default 8]
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <numeric>
#include <random>
#include <vector>

#include "../../include/xted.h"
#include "../../x-ted_b200/csrc/plan_core.h"
#include "emu_unit.h"

extern "C" int xo_distance_cost(int m, const int32_t *la, const int32_t *aoff, const int32_t *aidx, int n,
                                const int32_t *lb, const int32_t *boff, const int32_t *bidx, int cd, int ci, int cr);
using namespace xted;

struct HostPlan {
    std::vector<int32_t> raw, pair_trees;
    std::vector<DTree> trees;
    std::vector<int32_t> size, depth, parent, krd, cumw, opar, okd, oka;
    std::vector<int2> node;
    std::vector<XRun> runs;
    std::vector<XChunk> chunks;
    std::vector<DDepth> depths;
    std::vector<DOTree> ot;
    std::vector<DPair> pairs;
    std::vector<DLevel> lv;
    std::vector<XEntry> entries;
    std::vector<XUnit> units;
    std::vector<XTask> tasks;
    std::vector<XStripe> stripes;
    int stack_rows = 1;
};

static bool g_table = false;
// striped units: built with -DXTED_STRIPE_MIN_WIDTH=<small>, wide units of
// every size are planned as stripe tasks, whose layout the run checks
#ifdef XTED_STRIPE_MIN_WIDTH
static const bool g_stripes = true;
#else
static const bool g_stripes = false;
#endif

static void plan(const std::vector<std::vector<int32_t>> &L, const std::vector<std::vector<int32_t>> &O,
                 const std::vector<std::vector<int32_t>> &I, const std::vector<int> &nn,
                 const std::vector<int32_t> &pair_trees, int orientation, int narrow_width, int run_rows,
                 int wide_rows, int half_width, HostPlan &H) {
    const int T = (int)nn.size();
    int64_t N = 0;
    H.trees.resize((size_t)T);
    for (int t = 0; t < T; t++) {
        DTree &d = H.trees[(size_t)t];
        d.n = nn[(size_t)t];
        d.raw = (int32_t)H.raw.size();
        d.nbase = (int32_t)N;
        d.t = t;
        const int n = d.n;
        for (int k = 0; k < n; k++) H.raw.push_back(L[(size_t)t][(size_t)k]);
        for (int k = 0; k <= n; k++) H.raw.push_back(O[(size_t)t][(size_t)k]);
        for (int k = 0; k + 1 < n; k++) H.raw.push_back(I[(size_t)t][(size_t)k]);
        H.raw.push_back(0);
        N += n;
    }
    const size_t N2 = 2 * (size_t)std::max<int64_t>(N, 1);
    H.size.assign((size_t)N + 1, 0);
    H.depth.assign((size_t)N + 1, 0);
    H.parent.assign((size_t)N + 1, 0);
    H.node.assign(N2, int2{0, 0});
    H.krd.assign(N2, 0);
    H.cumw.assign(N2, 0);
    H.opar.assign(N2, 0);
    H.okd.assign(N2, 0);
    H.oka.assign(N2, 0);
    H.runs.assign(N2, XRun{});
    H.chunks.assign(N2, XChunk{});
    H.depths.assign(N2 + 2 * (size_t)T, DDepth{});
    H.ot.assign(2 * (size_t)T, DOTree{});
    PlanPools P;
    P.raw = H.raw.data();
    P.trees = H.trees.data();
    P.ntrees = T;
    P.size = H.size.data();
    P.depth = H.depth.data();
    P.parent = H.parent.data();
    P.node = H.node.data();
    P.krd = H.krd.data();
    P.cumw = H.cumw.data();
    P.runs = H.runs.data();
    P.chunks = H.chunks.data();
    P.opar = H.opar.data();
    P.okd = H.okd.data();
    P.oka = H.oka.data();
    P.depths = H.depths.data();
    P.otrees = H.ot.data();
    P.run_rows = run_rows;
    P.narrow_width = narrow_width;
    P.half_width = half_width;
    P.ntune = 0;
    if (g_table) {  // per tree-size granularity, as the autotuned table gives it
        P.tune[P.ntune++] = XTuneRow{40, 5, 32, 100};
        P.tune[P.ntune++] = XTuneRow{150, 64, 7, -1};
        P.tune[P.ntune++] = XTuneRow{1 << 30, 17, 256, 512};
    }
    for (int t = 0; t < T; t++) tree_basic(P, t, H.trees.data());
    for (int o = 0; o < 2 * T; o++) orient_tree(P, o);
    const int np = (int)pair_trees.size() / 2;
    H.pairs.resize((size_t)np);
    int64_t dt = 0, ent = 0;
    for (int p = 0; p < np; p++) {
        pair_setup(H.trees.data(), H.ot.data(), pair_trees.data(), orientation, p, H.pairs.data());
        DPair &q = H.pairs[(size_t)p];
        q.lvl_base = (int32_t)ent;
        q.dt_off = dt;
        ent += q.L;
        if (q.trivial < 0) {
            dt += (int64_t)H.trees[(size_t)q.ta].n * H.trees[(size_t)q.tb].n;
            H.stack_rows = std::max(H.stack_rows, H.ot[2 * (size_t)q.ta + q.o].maxka + 1);
        }
    }
    H.lv.resize((size_t)ent);
    LevelCtx C{H.ot.data(), H.depths.data(), H.runs.data(), H.chunks.data(), H.pairs.data(), narrow_width,
               wide_rows};
    C.stripe_min_cells = g_stripes ? 1 : 0;
    std::vector<int64_t> chain((size_t)np, 0);
    int64_t chain_max = 0;
    for (int p = 0; p < np; p++) {
        const DPair &q = H.pairs[(size_t)p];
        int64_t acc = 0;
        for (int d = 0; d < q.L; d++) {
            DLevel &E = H.lv[(size_t)(q.lvl_base + d)];
            E.pair = p;
            E.level = d;
            double est;
            level_count(C, E, &est);
            const int64_t e = (int64_t)(est / 64.0) + 1;
            E.key = acc;
            acc += e;
        }
        chain[(size_t)p] = acc;
        chain_max = std::max(chain_max, acc);
    }
    int64_t toff = 0, uoff = 0, soff = 0, poff = 0;
    H.entries.resize(H.lv.size());
    for (size_t e = 0; e < H.lv.size(); e++) {
        DLevel &E = H.lv[e];
        E.task_off = (int32_t)toff;
        E.unit_off = (int32_t)uoff;
        E.stripe_off = (int32_t)soff;
        E.entry = (int32_t)e;
        toff += E.ntasks;
        uoff += (int64_t)E.nwide + E.nnarrow + E.nhalf;
        soff += E.nstriped;
        poff += E.nstripes;
        XEntry &X = H.entries[e];
        X.task_off = E.task_off;
        X.ntasks = E.ntasks;
        X.bucket = level_bucket(chain[(size_t)E.pair] - E.key, chain_max);
        X.next = E.level + 1 < H.pairs[(size_t)E.pair].L ? (int32_t)e + 1 : -1;
        X.nnarrow = E.nntasks;
        X.pad = 0;
    }
    H.units.assign((size_t)uoff, XUnit{-1, -1});
    H.tasks.assign((size_t)toff, XTask{-1, -1, 0, -1});
    H.stripes.assign((size_t)soff + 1, XStripe{});
    for (auto &E : H.lv) level_fill(C, E, H.units.data(), H.tasks.data(), H.stripes.data());
    // stripes: every striped unit recorded, its stripes counted as planned
    int64_t pcheck = 0;
    for (int64_t i = 0; i < soff; i++) {
        const XStripe &S = H.stripes[(size_t)i];
        if (S.K != stripe_count(S.w) || S.unit < 0 || S.unit >= uoff)
            FAIL("striped unit %lld: unit %d, %d stripes", (long long)i, S.unit, S.K);
        pcheck += S.K;
    }
    if (pcheck != poff) FAIL("stripes %lld, planned %lld", (long long)pcheck, (long long)poff);
}

static void gen(int n, std::mt19937_64 &g, int alpha, int shape, std::vector<int32_t> &lab,
                std::vector<int32_t> &off, std::vector<int32_t> &idx) {
    lab.clear();
    off.assign(1, 0);
    idx.clear();
    if (n == 0) return;
    std::vector<std::vector<int>> ch((size_t)n);
    for (int i = 1; i < n; i++) {
        int p;
        if (shape == 0) p = (int)(g() % (uint64_t)i);                                   // random recursive
        else if (shape == 1) p = i < 6 ? 0 : (int)(g() % (uint64_t)std::min(i, 20));   // bushy
        else if (shape == 2) p = i - 1 - (int)(g() % (uint64_t)std::min(i, 3));        // deep
        else p = std::max(0, i - 1 - (int)(g() % 2));                                  // path-like
        if (g() % 2) ch[(size_t)p].insert(ch[(size_t)p].begin(), i);
        else ch[(size_t)p].push_back(i);
    }
    std::vector<int> order, st{0};
    while (!st.empty()) {
        int v = st.back();
        st.pop_back();
        order.push_back(v);
        for (int k = (int)ch[(size_t)v].size() - 1; k >= 0; k--) st.push_back(ch[(size_t)v][(size_t)k]);
    }
    std::vector<int> nid((size_t)n);
    for (int k = 0; k < n; k++) nid[(size_t)order[(size_t)k]] = k;
    lab.assign((size_t)n, 0);
    off.assign((size_t)n + 1, 0);
    for (int k = 0; k < n; k++) {
        lab[(size_t)k] = (int32_t)(g() % (uint64_t)alpha);
        for (int c : ch[(size_t)order[(size_t)k]]) idx.push_back(nid[(size_t)c]);
        off[(size_t)k + 1] = (int32_t)idx.size();
    }
}

int main(int argc, char **argv) {
    const int iters = argc > 1 ? std::atoi(argv[1]) : 200;
    if (argc > 4) emu::g_cache = std::atoi(argv[4]);
    const int maxn = argc > 2 ? std::atoi(argv[2]) : 300;
    std::mt19937_64 g(argc > 3 ? (uint64_t)std::atoll(argv[3]) : 12345);
    int64_t pairs_checked = 0;
    int64_t stripes_checked = 0;
    const int nws[4] = {0, 7, 64, XTED_NARROW_MAX};
    for (int it = 0; it < iters; it++) {
        const int ntrees = 1 + (int)(g() % 8);
        std::vector<std::vector<int32_t>> L((size_t)ntrees), O((size_t)ntrees), I((size_t)ntrees);
        std::vector<int> nn((size_t)ntrees);
        for (int t = 0; t < ntrees; t++) {
            nn[(size_t)t] = (g() % 4 == 0) ? (int)(g() % 9) : 1 + (int)(g() % (uint64_t)maxn);
            gen(nn[(size_t)t], g, 1 + (int)(g() % 6), (int)(g() % 4), L[(size_t)t], O[(size_t)t], I[(size_t)t]);
        }
        const int npairs = 1 + (int)(g() % 6);
        std::vector<int32_t> pt;
        for (int p = 0; p < 2 * npairs; p++) pt.push_back((int32_t)(g() % (uint64_t)ntrees));
        const int orient = it % 3, nw = nws[it % 4], rr = 1 + (int)(g() % 100);
        const int wrs[4] = {256, -1, 4, 40};
        const int wr = wrs[(it / 4) % 4];
        const int hws[3] = {XTED_HALF_MAX, -1, 100};
        const int hw = hws[(it / 16) % 3];
        g_table = it % 5 == 4;
        // edit costs: the reference's unit costs on two iterations of three,
        // else random delete / insert / rename costs (0 to 4)
        if (it % 3 == 2) {
            emu::g_cd = (int)(g() % 5);
            emu::g_ci = (int)(g() % 5);
            emu::g_cr = (int)(g() % 5);
        } else {
            emu::g_cd = emu::g_ci = emu::g_cr = 1;
        }
        HostPlan H;
        plan(L, O, I, nn, pt, orient, nw, rr, wr, hw, H);
        int64_t dts = 0;
        for (auto &q : H.pairs)
            if (q.trivial < 0) dts += (int64_t)H.trees[(size_t)q.ta].n * H.trees[(size_t)q.tb].n;
        std::vector<int32_t> dt((size_t)std::max<int64_t>(dts, 1), -1);
        // ready queue: level 0 of every pair, then each level once its predecessor is done;
        // highest bucket first, tasks of an entry in a shuffled order
        std::vector<std::vector<int32_t>> bucket(XTED_BUCKETS);
        for (auto &q : H.pairs)
            if (q.L > 0) bucket[(size_t)H.entries[(size_t)q.lvl_base].bucket].push_back(q.lvl_base);
        std::vector<size_t> head(XTED_BUCKETS, 0);
        std::vector<int> level_done((size_t)npairs, -1);
        std::vector<int> unit_seen(H.units.size(), 0);
        for (;;) {
            int e = -1;
            for (int b = XTED_BUCKETS - 1; b >= 0 && e < 0; b--)
                if (head[(size_t)b] < bucket[(size_t)b].size()) e = bucket[(size_t)b][head[(size_t)b]++];
            if (e < 0) break;
            const XEntry &X = H.entries[(size_t)e];
            const DLevel &E = H.lv[(size_t)e];
            if (level_done[(size_t)E.pair] != E.level - 1) FAIL("level published before its predecessor finished");
            std::vector<int> order((size_t)X.ntasks);
            std::iota(order.begin(), order.end(), 0);
            std::shuffle(order.begin(), order.end(), g);
            int lone_seen = 0;
            for (int k : order) {
                const XTask &t = H.tasks[(size_t)(X.task_off + k)];
                if (t.pair != E.pair || t.entry != e) FAIL("task of another entry in the range");
                if (t.kind_n & XTED_TASK_STRIPED) {
                    // stripe s of striped unit t.unit_lo: the unit's stripes are consecutive tasks,
                    // rightmost first; the unit runs once, at its rightmost stripe
                    const int si = t.unit_lo, s = (int)((t.kind_n >> XTED_STRIPE_SHIFT) & XTED_STRIPE_MASK);
                    if (!(t.kind_n & XTED_TASK_WIDE) || (t.kind_n & 0xffff) != 1 || si < E.stripe_off ||
                        si >= E.stripe_off + E.nstriped)
                        FAIL("stripe task %d of entry %d: striped unit %d", k, e, si);
                    const XStripe &S = H.stripes[(size_t)si];
                    if (s >= S.K) FAIL("stripe %d of %d", s, S.K);
                    const int first = X.task_off + k - (S.K - 1 - s);  // the task of stripe K - 1
                    const XTask &t0 = H.tasks[(size_t)first];
                    if (!(t0.kind_n & XTED_TASK_STRIPED) || t0.unit_lo != si ||
                        (int)((t0.kind_n >> XTED_STRIPE_SHIFT) & XTED_STRIPE_MASK) != S.K - 1)
                        FAIL("stripes of unit %d not consecutive from the rightmost", si);
                    if (s != S.K - 1) continue;
                    const XUnit &U = H.units[(size_t)S.unit];
                    if (H.runs[(size_t)U.run].rows != S.R || H.chunks[(size_t)U.chunk].width != S.w)
                        FAIL("striped unit %d: rows %d width %d", si, S.R, S.w);
                    const DPair &q = H.pairs[(size_t)t.pair];
                    XPair x;
                    x.dt_off = q.dt_off;
                    x.m = H.trees[(size_t)q.ta].n;
                    x.n = H.trees[(size_t)q.tb].n;
                    x.row_base = H.ot[2 * (size_t)q.ta + q.o].node_base;
                    x.col_base = H.ot[2 * (size_t)q.tb + q.o].node_base;
                    const emu::Pools EP{H.node.data(), H.krd.data(), H.cumw.data(), H.runs.data(), H.chunks.data(),
                                        H.stack_rows};
                    unit_seen[(size_t)S.unit]++;
                    emu::run_unit(EP, x, U, dt, nw, true);
                    stripes_checked++;
                    continue;
                }
                const int nu = (int)(t.kind_n & 0xffff);
                const bool full = (t.kind_n & XTED_TASK_WIDE) != 0, half = (t.kind_n & XTED_TASK_HALF) != 0;
                // the narrow tasks of a level are the first X.nnarrow of its range (two claim rings)
                if ((k < X.nnarrow) != !(full || half)) FAIL("task %d of a level out of its kind's range", k);
                const bool wide = full || half;
                if (nu < 1 || nu > XTED_TASK_UNITS || (full && nu != 1) || (half && nu > 8)) FAIL("bad unit count %d", nu);
                for (int u = 0; u < nu && !g_table; u++) {
                    const int w = H.chunks[(size_t)H.units[(size_t)(t.unit_lo + u)].chunk].width;
                    if (half && (w <= nw || w > XTED_HALF_MAX || w > hw)) FAIL("half unit of width %d", w);
                    // a half-width unit alone in its task runs on the whole block: at most the
                    // last of the paired units of long runs and the last of the bundled ones
                    if (full && w <= XTED_HALF_MAX && w > nw && hw >= w && ++lone_seen > 2)
                        FAIL("whole-block unit of width %d", w);
                }
                const DPair &q = H.pairs[(size_t)t.pair];
                XPair x;
                x.dt_off = q.dt_off;
                x.m = H.trees[(size_t)q.ta].n;
                x.n = H.trees[(size_t)q.tb].n;
                x.row_base = H.ot[2 * (size_t)q.ta + q.o].node_base;
                x.col_base = H.ot[2 * (size_t)q.tb + q.o].node_base;
                const emu::Pools EP{H.node.data(), H.krd.data(), H.cumw.data(), H.runs.data(), H.chunks.data(),
                                    H.stack_rows};
                for (int u = 0; u < nu; u++) {
                    const int ui = t.unit_lo + u;
                    unit_seen[(size_t)ui]++;
                    const XUnit &U = H.units[(size_t)ui];
                    const XChunk &UC = H.chunks[(size_t)U.chunk];
                    // every fourth single-segment unit is also computed in column stripes
                    // (multi-block path) on a copy of the pair's table: same tree distances
                    std::vector<int32_t> alt;
                    if (UC.nseg == 1 && UC.width >= 4 && ui % 4 == 0) {
                        alt.assign(dt.begin() + x.dt_off, dt.begin() + x.dt_off + (int64_t)x.m * x.n);
                        XPair x0 = x;
                        x0.dt_off = 0;
                        static const int kStripe[4] = {2, 3, 5, 16};
                        emu::run_unit_striped(EP, x0, U, alt, kStripe[(ui / 4) % 4]);
                        stripes_checked++;
                    }
                    emu::run_unit(EP, x, U, dt, g_table ? XTED_NARROW_MAX : nw, wide);
                    if (!alt.empty() && !std::equal(alt.begin(), alt.end(), dt.begin() + x.dt_off))
                        FAIL("striped unit %d (width %d) differs from the one-block unit", ui, UC.width);
                }
            }
            level_done[(size_t)E.pair] = E.level;
            if (X.next >= 0) bucket[(size_t)H.entries[(size_t)X.next].bucket].push_back(X.next);
        }
        for (int p = 0; p < npairs; p++)
            if (level_done[(size_t)p] != H.pairs[(size_t)p].L - 1) FAIL("pair %d did not finish its levels", p);
        for (int v : unit_seen)
            if (v != 1) FAIL("unit covered %d times", v);
        for (int p = 0; p < npairs; p++) {
            const DPair &q = H.pairs[(size_t)p];
            const int a = pt[2 * (size_t)p], b = pt[2 * (size_t)p + 1];
            // an empty-tree pair: the gather kernel's rule (insert or delete the other tree)
            const int got = q.trivial >= 0 ? (nn[(size_t)a] == 0 ? nn[(size_t)b] * emu::g_ci : nn[(size_t)a] * emu::g_cd)
                                           : dt[(size_t)q.dt_off];
            const int32_t z = 0;
            const int want = xo_distance_cost(nn[(size_t)a], nn[(size_t)a] ? L[(size_t)a].data() : &z,
                                              O[(size_t)a].data(), I[(size_t)a].empty() ? &z : I[(size_t)a].data(),
                                              nn[(size_t)b], nn[(size_t)b] ? L[(size_t)b].data() : &z,
                                              O[(size_t)b].data(), I[(size_t)b].empty() ? &z : I[(size_t)b].data(),
                                              emu::g_cd, emu::g_ci, emu::g_cr);
            if (got != want)
                FAIL("distance mismatch it=%d pair=%d m=%d n=%d got=%d want=%d", it, p, nn[(size_t)a],
                     nn[(size_t)b], got, want);
            pairs_checked++;
        }
    }
    std::printf("ok %lld pairs, %lld striped units\n", (long long)pairs_checked, (long long)stripes_checked);
    return 0;
}
