// serve_emu.cpp -- TEST INFRASTRUCTURE: checks the serving planner on the CPU.
//
// Builds a corpus with the library's serving planner (serve_plan.h), plans
// rounds of queries into the query slots, moves each plan to scattered
// device-style offsets (serve_fixup), and runs all queries of a round
// interleaved the way the serving launch does: level 0 of every pair
// published from `first`, the oldest query's bucket first, a pair's next level
// once its current one is done, every unit computed with the kernels' row
// math (emu_unit.h). Checks every index against its pool and every distance
// against the oracle's restatement of X-TED_CPU.
//   usage: serve_emu <rounds> <max_nodes> <seed>
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <deque>
#include <random>
#include <vector>

#include "../../include/xted.h"
#include "../../x-ted_b200/csrc/serve_plan.h"
#include "emu_unit.h"

extern "C" int xo_distance(int m, const int32_t *la, const int32_t *aoff, const int32_t *aidx, int n,
                           const int32_t *lb, const int32_t *boff, const int32_t *bidx);
using namespace xted;

struct HTree {
    std::vector<int32_t> lab, off, idx;
    int n = 0;
};

static HTree gen(int n, std::mt19937_64 &g, int alpha, int shape) {
    HTree t;
    t.n = n;
    t.off.assign(1, 0);
    if (n == 0) return t;
    std::vector<std::vector<int>> ch((size_t)n);
    for (int i = 1; i < n; i++) {
        int p;
        if (shape == 0) p = (int)(g() % (uint64_t)i);
        else if (shape == 1) p = i < 6 ? 0 : (int)(g() % (uint64_t)std::min(i, 20));
        else if (shape == 2) p = i - 1 - (int)(g() % (uint64_t)std::min(i, 3));
        else p = std::max(0, i - 1 - (int)(g() % 2));
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
    t.lab.assign((size_t)n, 0);
    t.off.assign((size_t)n + 1, 0);
    for (int k = 0; k < n; k++) {
        t.lab[(size_t)k] = (int32_t)(g() % (uint64_t)alpha);
        for (int c : ch[(size_t)order[(size_t)k]]) t.idx.push_back(nid[(size_t)c]);
        t.off[(size_t)k + 1] = (int32_t)t.idx.size();
    }
    return t;
}

static int oracle(const HTree &a, const HTree &b) {
    const int32_t z = 0;
    return xo_distance(a.n, a.n ? a.lab.data() : &z, a.off.data(), a.idx.empty() ? &z : a.idx.data(), b.n,
                       b.n ? b.lab.data() : &z, b.off.data(), b.idx.empty() ? &z : b.idx.data());
}

// The bit-vector Levenshtein distance equals the textbook dynamic program
// (lengths across the 64-row block edges, symbols absent from the pattern).
static int64_t check_seq_distance(std::mt19937_64 &g) {
    int64_t checked = 0;
    for (int it = 0; it < 300; it++) {
        const int m = (int)(g() % 260), n = (int)(g() % 260), alpha = 1 + (int)(g() % 6);
        std::vector<int32_t> a((size_t)m), b((size_t)n);
        for (int32_t &x : a) x = (int32_t)(g() % (uint64_t)(alpha + 1)) - 1;
        for (int32_t &x : b) x = (int32_t)(g() % (uint64_t)(alpha + 1)) - 1;
        std::vector<int32_t> prev((size_t)n + 1), cur((size_t)n + 1);
        for (int j = 0; j <= n; j++) prev[(size_t)j] = j;
        for (int i = 1; i <= m; i++) {
            cur[0] = i;
            for (int j = 1; j <= n; j++) {
                const int sub = prev[(size_t)j - 1] + ((a[(size_t)i - 1] == b[(size_t)j - 1] && a[(size_t)i - 1] >= 0) ? 0 : 1);
                cur[(size_t)j] = std::min(sub, std::min(prev[(size_t)j], cur[(size_t)j - 1]) + 1);
            }
            std::swap(prev, cur);
        }
        SeqBits P;
        P.build(a.data(), m, alpha);
        std::vector<uint64_t> work;
        const int32_t got = P.distance(b.data(), n, work);
        if (got != prev[(size_t)n]) FAIL("sequence distance m=%d n=%d: got %d want %d", m, n, got, prev[(size_t)n]);
        checked++;
    }
    return checked;
}

// Exact top-k pruning (serve_plan.h): the label and preorder bounds never
// exceed the oracle distance, and the two rounds return the unpruned top k.
static int64_t check_pruning(std::mt19937_64 &g, int maxn) {
    const int T = 40 + (int)(g() % 60);
    std::vector<HTree> corpus((size_t)T);
    std::vector<std::vector<int32_t>> sl((size_t)T);
    const int alpha = 2 + (int)(g() % 40);
    for (int t = 0; t < T; t++) {
        const int n = (g() % 10 == 0) ? (int)(g() % 2) : 1 + (int)(g() % (uint64_t)maxn);
        corpus[(size_t)t] = gen(n, g, alpha, (int)(g() % 4));
        sl[(size_t)t] = corpus[(size_t)t].lab;
        std::sort(sl[(size_t)t].begin(), sl[(size_t)t].end());
    }
    int64_t checked = 0;
    for (int qi = 0; qi < 6; qi++) {
        const HTree q = (qi == 0) ? corpus[(size_t)(g() % (uint64_t)T)]  // an exact match is in the corpus
                                  : gen((g() % 12 == 0) ? 0 : 1 + (int)(g() % (uint64_t)maxn), g, alpha, (int)(g() % 4));
        std::vector<int32_t> ql(q.lab);
        std::sort(ql.begin(), ql.end());
        std::vector<int32_t> full((size_t)T), lb((size_t)T), dist((size_t)T, -1);
        SeqBits P;
        P.build(q.lab.data(), q.n, alpha);
        std::vector<uint64_t> work;
        for (int t = 0; t < T; t++) {
            full[(size_t)t] = oracle(corpus[(size_t)t], q);
            const int32_t l1 = label_lower_bound(ql.data(), q.n, sl[(size_t)t].data(), (int)sl[(size_t)t].size());
            const int32_t l2 = P.distance(corpus[(size_t)t].lab.data(), corpus[(size_t)t].n, work);
            if (l2 < l1) FAIL("preorder bound %d below the label bound %d", l2, l1);
            lb[(size_t)t] = (g() % 2) ? l2 : l1;
            if (l2 > full[(size_t)t]) FAIL("bound %d above the distance %d", l2, full[(size_t)t]);
            if (q.n == 0 || corpus[(size_t)t].n == 0) dist[(size_t)t] = full[(size_t)t];
        }
        const int k = 1 + (int)(g() % 12);
        std::vector<uint8_t> inc;
        prune_round1(lb, dist, 1 + (size_t)(g() % (uint64_t)(2 * k)), true, inc);
        for (int t = 0; t < T; t++)
            if (inc[(size_t)t]) {
                if (dist[(size_t)t] >= 0) FAIL("round 1 picked a known pair");
                dist[(size_t)t] = full[(size_t)t];
            }
        if (prune_round2(lb, dist, k, inc))
            for (int t = 0; t < T; t++)
                if (inc[(size_t)t]) {
                    if (dist[(size_t)t] >= 0) FAIL("round 2 picked a known pair");
                    dist[(size_t)t] = full[(size_t)t];
                }
        std::vector<int32_t> id1((size_t)k), d1((size_t)k), id2((size_t)k), d2((size_t)k);
        topk_known(dist, k, id1.data(), d1.data());
        topk_known(full, k, id2.data(), d2.data());
        if (id1 != id2 || d1 != d2) FAIL("pruned top-%d differs from the unpruned one", k);
        checked += T;
    }
    return checked;
}

int main(int argc, char **argv) {
    const int rounds = argc > 1 ? std::atoi(argv[1]) : 10;
    const int maxn = argc > 2 ? std::atoi(argv[2]) : 120;
    std::mt19937_64 g(argc > 3 ? (uint64_t)std::atoll(argv[3]) : 7);
    const int T = 2 + (int)(g() % 9), S = 4, Qmax = maxn;
    std::vector<HTree> corpus((size_t)T);
    std::vector<xted_tree> ct((size_t)T);
    for (int t = 0; t < T; t++) {
        const int n = (g() % 6 == 0) ? (int)(g() % 3) : 1 + (int)(g() % (uint64_t)maxn);
        corpus[(size_t)t] = gen(n, g, 1 + (int)(g() % 5), (int)(g() % 4));
        const HTree &h = corpus[(size_t)t];
        ct[(size_t)t] = xted_tree{h.lab.data(), h.off.data(), h.idx.data(), h.n};
    }
    int64_t checked = 0;
    for (int r = 0; r < rounds; r++) {
        const int narrow = r % 3 == 0 ? XTED_NARROW_MAX : (r % 3 == 1 ? 7 : 0);
        const int run_rows = 1 + (int)(g() % 80), orient = r % 3;
        ServePools H;
        serve_pools_build(H, ct.data(), T, S, Qmax, run_rows, narrow, (r % 4 == 3) ? -1 : XTED_HALF_MAX);
        // device-style pools; plans land at scattered offsets
        const int64_t UC = 1 << 22, TC = 1 << 21, EC = 1 << 18;
        std::vector<XPair> pairs((size_t)S * T);
        std::vector<int32_t> first((size_t)S * T, -7);
        std::vector<XEntry> entries((size_t)EC);
        std::vector<XUnit> units((size_t)UC, XUnit{-1, -1});
        std::vector<XTask> tasks((size_t)TC, XTask{-1, -1, 0, -1});
        int64_t u_at = 0, t_at = 0, e_at = 0, dt_at = 0;
        const int nq = 1 + (int)(g() % S);
        std::vector<HTree> qs((size_t)nq);
        std::vector<QPlan> plans((size_t)nq);
        std::vector<int64_t> dt_base((size_t)nq);
        std::vector<std::vector<uint8_t>> incs((size_t)nq);
        for (int q = 0; q < nq; q++) {
            const int n = (g() % 8 == 0) ? 0 : 1 + (int)(g() % (uint64_t)Qmax);
            qs[(size_t)q] = gen(n, g, 1 + (int)(g() % 5), (int)(g() % 4));
            const HTree &h = qs[(size_t)q];
            std::vector<uint8_t> inc((size_t)T, 1);
            if (r % 4 == 1)  // a pruned round: a random subset of the corpus
                for (int t = 0; t < T; t++) inc[(size_t)t] = (uint8_t)(g() % 2);
            incs[(size_t)q] = inc;
            serve_plan_query(H, q, h.lab.data(), h.off.data(), h.idx.data(), h.n, orient, narrow,
                             (r % 2) ? 5 : 256, plans[(size_t)q], inc.data());
            QPlan &p = plans[(size_t)q];
            u_at += (int64_t)(g() % 1000);
            t_at += (int64_t)(g() % 1000);
            e_at += (int64_t)(g() % 100);
            dt_at += (int64_t)(g() % 5000);
            dt_base[(size_t)q] = dt_at;
            serve_fixup(p, q, T, dt_at, u_at, t_at, e_at, (int32_t)((-q) & (XTED_BUCKETS - 1)));
            if (u_at + (int64_t)p.units.size() > UC || t_at + (int64_t)p.tasks.size() > TC ||
                e_at + (int64_t)p.entries.size() > EC)
                FAIL("test pools too small");
            std::copy(p.units.begin(), p.units.end(), units.begin() + u_at);
            std::copy(p.tasks.begin(), p.tasks.end(), tasks.begin() + t_at);
            std::copy(p.entries.begin(), p.entries.end(), entries.begin() + e_at);
            std::copy(p.pairs.begin(), p.pairs.end(), pairs.begin() + (int64_t)q * T);
            std::copy(p.first.begin(), p.first.end(), first.begin() + (int64_t)q * T);
            u_at += (int64_t)p.units.size();
            t_at += (int64_t)p.tasks.size();
            e_at += (int64_t)p.entries.size();
            dt_at += p.dt_elems;
        }
        std::vector<int32_t> dt((size_t)std::max<int64_t>(dt_at, 1), -1);
        const emu::Pools EP{H.node.data(), H.krd.data(), H.cumw.data(), H.runs.data(), H.chunks.data(),
                            H.stack_rows};
        const int64_t npool = (int64_t)H.node.size();
        // ready queue by query age (bucket of query q = (-q) & 15, oldest first)
        std::vector<std::deque<int32_t>> bucket(XTED_BUCKETS);
        std::vector<int32_t> result((size_t)S * T, -1);
        auto publish = [&](int32_t e, int pair) {
            while (e >= 0) {
                if (e >= (int64_t)entries.size()) FAIL("entry index out of range");
                if (entries[(size_t)e].ntasks > 0) {
                    bucket[(size_t)entries[(size_t)e].bucket].push_back(e);
                    return;
                }
                e = entries[(size_t)e].next;
            }
            const XPair &x = pairs[(size_t)pair];
            result[(size_t)pair] = dt[(size_t)x.dt_off];
        };
        for (int q = 0; q < nq; q++)
            for (int t = 0; t < T; t++) {
                const int p = q * T + t;
                if (first[(size_t)p] >= 0) publish(first[(size_t)p], p);
            }
        int top = 0;
        for (;;) {
            int e = -1;
            for (int i = 0; i < XTED_BUCKETS && e < 0; i++) {
                auto &B = bucket[(size_t)((top - i) & (XTED_BUCKETS - 1))];
                if (!B.empty()) {
                    // interleave: take a random live entry of the bucket
                    const size_t k = (size_t)(g() % B.size());
                    e = B[k];
                    B.erase(B.begin() + (long)k);
                }
            }
            if (e < 0) break;
            const XEntry X = entries[(size_t)e];
            int pair = -1;
            for (int k = 0; k < X.ntasks; k++) {
                if (X.task_off + k >= TC) FAIL("task index out of range");
                const XTask &t = tasks[(size_t)(X.task_off + k)];
                if (t.entry != e) FAIL("task of another entry in the range");
                if (t.pair < 0 || t.pair >= S * T) FAIL("task pair out of range");
                if (pair >= 0 && t.pair != pair) FAIL("tasks of one entry from two pairs");
                pair = t.pair;
                const XPair &x = pairs[(size_t)t.pair];
                if (x.row_base < 0 || x.row_base + x.m > npool || x.col_base < 0 || x.col_base + x.n > npool)
                    FAIL("pair node ranges outside the pools");
                if (x.dt_off < 0 || x.dt_off + (int64_t)x.m * x.n > dt_at) FAIL("pair table outside the pool");
                const int nu = (int)(t.kind_n & 0xffff);
                const bool full = (t.kind_n & XTED_TASK_WIDE) != 0, half = (t.kind_n & XTED_TASK_HALF) != 0;
                const bool wide = full || half;
                if (nu < 1 || nu > XTED_TASK_UNITS || (full && nu != 1) || (half && nu > 8)) FAIL("bad unit count %d", nu);
                for (int u = 0; u < nu; u++) {
                    if (t.unit_lo + u >= UC) FAIL("unit index out of range");
                    const XUnit &U = units[(size_t)(t.unit_lo + u)];
                    if (U.run < 0 || U.run >= npool || U.chunk < 0 || U.chunk >= npool) FAIL("unit outside the pools");
                    emu::run_unit(EP, x, U, dt, narrow, wide);
                }
            }
            publish(X.next, pair);
            top = (top - (int)(g() % 2)) & (XTED_BUCKETS - 1);  // the oldest query changes as queries finish
        }
        for (int q = 0; q < nq; q++) {
            const QPlan &p = plans[(size_t)q];
            int need = 0;
            for (int t = 0; t < T; t++) {
                const int pi = q * T + t;
                if (p.trivial[(size_t)t] < 0 && !incs[(size_t)q][(size_t)t]) {
                    if (p.first[(size_t)t] != -1 || result[(size_t)pi] != -1) FAIL("excluded pair was computed");
                    continue;
                }
                const int got = p.trivial[(size_t)t] >= 0 ? p.trivial[(size_t)t] : result[(size_t)pi];
                if (p.trivial[(size_t)t] < 0) need++;
                const int want = oracle(corpus[(size_t)t], qs[(size_t)q]);
                if (got != want)
                    FAIL("round %d query %d corpus tree %d (m=%d n=%d): got %d want %d", r, q, t, corpus[(size_t)t].n,
                         qs[(size_t)q].n, got, want);
                checked++;
            }
            if (need != p.need) FAIL("need count %d != %d", p.need, need);
        }
    }
    int64_t pruned = check_seq_distance(g);
    for (int r = 0; r < std::max(1, rounds / 2); r++) pruned += check_pruning(g, std::min(maxn, 40));
    std::printf("ok %lld pairs, %lld pruning pairs\n", (long long)checked, (long long)pruned);
    return 0;
}
