// plan_emu.cpp -- TEST INFRASTRUCTURE: checks the host planner on the CPU.
//
// Builds plans for random batches with the product planner (plan.cpp) and
// executes every unit with the same row formulation the kernels use (row
// scan with segment keys, far-row stack), sequentially in queue order. It
// checks the plan's invariants (dependency order, single write of every
// tree cell, every read cell already written, stack discipline) and the
// distances against the oracle's restatement of X-TED_CPU.
//   usage: plan_emu <iterations> <max_nodes> <seed>
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "../../include/xted.h"
#include "../../x-ted_b200/csrc/plan.h"

extern "C" int xo_distance(int m, const int32_t *la, const int32_t *aoff, const int32_t *aidx, int n,
                           const int32_t *lb, const int32_t *boff, const int32_t *bidx);
using namespace xted;

#define FAIL(...)                     \
    do {                              \
        std::printf(__VA_ARGS__);     \
        std::printf("\n");            \
        std::exit(1);                 \
    } while (0)

static void run_unit(const Plan &P, const XPair &pr, const XUnit &u, std::vector<int32_t> &dtv) {
    int32_t *dt = dtv.data() + pr.dt_off;
    const XRun run = P.runs[(size_t)u.run];
    const XChunk ch = P.chunks[(size_t)u.chunk];
    const int W = ch.width, n = pr.n;
    std::vector<int> node(W), lab(W), foff(W), dend(W), key(W);
    std::vector<char> far(W);
    int seg = 0;
    for (int c = 0; c < W; c++) {
        const int4h ci = P.colinfo[(size_t)(ch.col_lo + c)];
        node[c] = ci.x;
        lab[c] = ci.y;
        foff[c] = ci.z & XTED_COL_FOFF_MASK;
        far[c] = (ci.z & XTED_COL_FARCOL) != 0;
        dend[c] = ci.w;
        key[c] = c + XTED_KEY_BIG * seg;
        if (dend[c] == 1) seg++;
    }
    if (seg != ch.nseg) FAIL("chunk segment count %d != %d", seg, ch.nseg);
    std::vector<std::vector<int>> stk((size_t)P.stack_rows, std::vector<int>((size_t)W, -777));
    std::vector<int> prev(W), cur(W), loc(W);
    for (int kr = run.kr_lo; kr < run.kr_hi; kr++) {
        const int i0 = P.krd[(size_t)kr];
        const int imax = (P.rowinfo[(size_t)(pr.row_base + i0)].y & XTED_ROW_ORL_MASK) + 1;
        for (int c = 0; c < W; c++) prev[c] = dend[c];
        int sp = 0;
        for (int i = imax - 1; i >= i0; i--) {
            const int2h ri = P.rowinfo[(size_t)(pr.row_base + i)];
            const int ro = ri.y & XTED_ROW_ORL_MASK;
            const bool trow = ro == imax - 1;
            const int bord = imax - i, rowfar = imax - ro - 1;
            int runmin = XTED_INF;
            for (int c = W - 1; c >= 0; c--) {
                const bool se = dend[c] == 1;
                const int diag = se ? bord - 1 : prev[(size_t)c + 1];
                const bool tcol = foff[c] == dend[c];
                int a;
                if (trow && tcol) {
                    a = diag + (ri.x != lab[c]);
                } else {
                    int fv;
                    if (trow) fv = dend[c] - foff[c];
                    else if (tcol) fv = rowfar;
                    else {
                        if (sp < 1) FAIL("far-row stack underflow");
                        fv = stk[(size_t)sp - 1][(size_t)(c + foff[c])];
                        if (fv == -777) FAIL("far value never pushed");
                    }
                    const int dv = dt[(size_t)i * n + node[c]];
                    if (dv < 0) FAIL("tree distance (%d,%d) read before it was written", i, node[c]);
                    a = dv + fv;
                }
                int A = std::min(a, prev[c] + 1);
                if (se) A = std::min(A, bord + 1);
                runmin = std::min(runmin, A + key[c]);
                loc[c] = runmin;
            }
            for (int c = 0; c < W; c++) {
                cur[c] = loc[c] - key[c];
                if (trow && foff[c] == dend[c]) {
                    int32_t &slot = dt[(size_t)i * n + node[c]];
                    if (slot >= 0) FAIL("tree distance (%d,%d) written twice", i, node[c]);
                    slot = cur[c];
                }
                prev[c] = cur[c];
            }
            if (i != i0 && (ri.y & XTED_ROW_ISKR)) sp--;
            if (i > i0 && (ri.y & XTED_ROW_PREVLEAF)) {
                if (sp >= P.stack_rows) FAIL("far-row stack overflow (%d rows)", P.stack_rows);
                for (int c = 0; c < W; c++) stk[(size_t)sp][(size_t)c] = far[c] ? prev[c] : -777;
                sp++;
            }
        }
        if (sp != 0) FAIL("far-row stack not empty at table end (%d)", sp);
    }
}

static void gen(int n, std::mt19937_64 &g, int alpha, int shape, std::vector<int32_t> &lab,
                std::vector<int32_t> &off, std::vector<int32_t> &idx) {
    if (n == 0) {
        lab.assign(1, 0);
        off.assign(1, 0);
        idx.assign(1, 0);
        return;
    }
    std::vector<std::vector<int>> ch((size_t)n);
    for (int i = 1; i < n; i++) {
        int p;
        if (shape == 0) p = (int)(g() % (uint64_t)i);                      // random recursive
        else if (shape == 1) p = i < 6 ? 0 : (int)(g() % (uint64_t)std::min(i, 20));  // bushy
        else if (shape == 2) p = i - 1 - (int)(g() % (uint64_t)std::min(i, 3));       // deep
        else p = std::max(0, i - 1 - (int)(g() % 2));                      // path-like
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
    idx.clear();
    for (int k = 0; k < n; k++) {
        lab[(size_t)k] = (int32_t)(g() % (uint64_t)alpha);
        for (int c : ch[(size_t)order[(size_t)k]]) idx.push_back(nid[(size_t)c]);
        off[(size_t)k + 1] = (int32_t)idx.size();
    }
    if (idx.empty()) idx.push_back(0);
}

int main(int argc, char **argv) {
    const int iters = argc > 1 ? std::atoi(argv[1]) : 200;
    const int maxn = argc > 2 ? std::atoi(argv[2]) : 300;
    std::mt19937_64 g(argc > 3 ? (uint64_t)std::atoll(argv[3]) : 12345);
    int64_t pairs_checked = 0;
    for (int it = 0; it < iters; it++) {
        const int npairs = 1 + (int)(g() % 5);
        std::vector<std::vector<int32_t>> L((size_t)2 * npairs), O((size_t)2 * npairs), I((size_t)2 * npairs);
        std::vector<TreeView> A((size_t)npairs), B((size_t)npairs);
        for (int p = 0; p < npairs; p++)
            for (int s = 0; s < 2; s++) {
                const size_t k = (size_t)(2 * p + s);
                const int n = (g() % 4 == 0) ? (int)(g() % 9) : 1 + (int)(g() % (uint64_t)maxn);
                gen(n, g, 1 + (int)(g() % 6), (int)(g() % 4), L[k], O[k], I[k]);
                TreeView t{n, L[k].data(), O[k].data(), I[k].data()};
                (s ? B : A)[(size_t)p] = t;
            }
        if (npairs > 1 && g() % 3 == 0) B[0] = A[1];  // shared tree objects
        PlanOptions opt;
        opt.orientation = it % 3;
        const int nws[4] = {0, 7, 64, XTED_NARROW_MAX};
        opt.narrow_width = nws[it % 4];
        opt.run_rows = 1 + (int)(g() % 100);
        Plan P;
        const int rc = make_plan(A.data(), B.data(), npairs, opt, P);
        if (rc) FAIL("make_plan returned %d", rc);
        std::vector<int32_t> dt((size_t)std::max<int64_t>(P.dt_elems, 1), -1);
        std::vector<int> fin((size_t)npairs, 0);
        for (const XTask &t : P.tasks) {
            if (fin[(size_t)t.pair] < t.need) FAIL("task queued before its dependencies");
            const int nu = (int)(t.kind_n & 0xffff);
            if (nu < 1 || nu > XTED_WARPS) FAIL("bad unit count %d", nu);
            for (int u = 0; u < nu; u++) {
                const XUnit &un = P.units[(size_t)(t.unit_lo + u)];
                const int w = P.chunks[(size_t)un.chunk].width;
                const bool wide = (t.kind_n & XTED_TASK_WIDE) != 0;
                if (!wide && w > opt.narrow_width) FAIL("narrow unit wider than the narrow limit");
                run_unit(P, P.pairs[(size_t)t.pair], un, dt);
            }
            fin[(size_t)t.pair]++;
        }
        for (int p = 0; p < npairs; p++) {
            const int got = P.trivial[(size_t)p] >= 0 ? P.trivial[(size_t)p] : dt[(size_t)P.pairs[(size_t)p].dt_off];
            const int want = xo_distance(A[(size_t)p].n, A[(size_t)p].labels, A[(size_t)p].off, A[(size_t)p].idx,
                                         B[(size_t)p].n, B[(size_t)p].labels, B[(size_t)p].off, B[(size_t)p].idx);
            if (got != want)
                FAIL("distance mismatch it=%d pair=%d m=%d n=%d got=%d want=%d", it, p, A[(size_t)p].n,
                     B[(size_t)p].n, got, want);
            pairs_checked++;
        }
    }
    std::printf("ok %lld pairs\n", (long long)pairs_checked);
    return 0;
}
