// emu_unit.h -- TEST INFRASTRUCTURE: one DP unit computed on the CPU exactly
// as the kernels compute it (columns derived like load_cols, row scan with
// segment keys, far-row stack with its shared-memory window), with checks of
// the plan's invariants. Shared by the batch and serving planner emulations.
#pragma once

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "../../x-ted_b200/csrc/plan_core.h"

#define FAIL(...)                 \
    do {                          \
        std::printf(__VA_ARGS__); \
        std::printf("\n");        \
        std::exit(1);             \
    } while (0)

namespace emu {

using namespace xted;

struct Pools {
    const int2 *node;
    const int32_t *krd, *cumw;
    const XRun *runs;
    const XChunk *chunks;
    int stack_rows;
};

inline int g_cache = 8;  // shared-memory window of the far-row stack (the kernels use 8)
// edit costs of the emulated launch: delete a row-tree node, insert a
// column-tree node, change a label (the reference's unit costs by default)
inline int g_cd = 1, g_ci = 1, g_cr = 1;

// Unit u of pair pr; the pair's m x n tree-distance table is dtv[pr.dt_off ...].
inline void run_unit(const Pools &H, const XPair &pr, const XUnit &u, std::vector<int32_t> &dtv, int narrow_width,
                     bool wide_task) {
    int32_t *dt = dtv.data() + pr.dt_off;
    const XRun run = H.runs[(size_t)u.run];
    const XChunk ch = H.chunks[(size_t)u.chunk];
    if (!wide_task && ch.width > narrow_width) FAIL("narrow unit wider than the narrow limit");
    (void)wide_task;  // a wide task may hold a narrow chunk (a long run); the row math is the same
    const int W = ch.width, n = pr.n;
    const int2 *cn = H.node + pr.col_base;
    const int2 *rn = H.node + pr.row_base;
    std::vector<int> node(W), lab(W), foff(W), dend(W), key(W);
    std::vector<char> far(W);
    int seg = 0, s = ch.k_lo;
    int j0 = H.krd[(size_t)s], je = (cn[j0].y & XTED_ROW_ORL_MASK) + 1, j = j0;
    if (H.cumw[(size_t)s] + W > H.cumw[(size_t)(ch.k_lo + ch.nseg - 1)] +
                                    ((cn[H.krd[(size_t)(ch.k_lo + ch.nseg - 1)]].y & XTED_ROW_ORL_MASK) + 1 -
                                     H.krd[(size_t)(ch.k_lo + ch.nseg - 1)]))
        FAIL("chunk width exceeds its segments");
    for (int c = 0; c < W; c++) {
        if (j >= je) {
            s++;
            j0 = H.krd[(size_t)s];
            je = (cn[j0].y & XTED_ROW_ORL_MASK) + 1;
            j = j0;
        }
        node[c] = j;
        lab[c] = cn[j].x;
        foff[c] = (cn[j].y & XTED_ROW_ORL_MASK) + 1 - j;
        dend[c] = je - j;
        far[c] = j > j0 && (cn[j].y & XTED_ROW_PREVLEAF);
        key[c] = c * g_ci + XTED_KEY_BIG * seg;
        if (dend[c] == 1) seg++;
        j++;
    }
    if (seg != ch.nseg || s != ch.k_lo + ch.nseg - 1) FAIL("chunk segment count mismatch");
    // global stack (written only when units can nest deeper than the window) and the window
    const bool deep = run.depth > g_cache;  // the kernels' rule: depth-d tables nest <= d rows
    std::vector<std::vector<int>> stk((size_t)H.stack_rows, std::vector<int>((size_t)W, -777));
    std::vector<std::vector<int>> cache((size_t)g_cache, std::vector<int>((size_t)W, -777));
    std::vector<int> prev(W), cur(W), loc(W);
    for (int kr = run.kr_lo; kr < run.kr_hi; kr++) {
        const int i0 = H.krd[(size_t)kr];
        const int imax = (rn[i0].y & XTED_ROW_ORL_MASK) + 1;
        for (int c = 0; c < W; c++) prev[c] = dend[c] * g_ci;
        int sp = 0, lo = 0;
        for (auto &row : cache) std::fill(row.begin(), row.end(), -777);
        for (auto &row : stk) std::fill(row.begin(), row.end(), -777);
        for (int i = imax - 1; i >= i0; i--) {
            const int2 ri = rn[i];
            const int ro = ri.y & XTED_ROW_ORL_MASK;
            const bool trow = ro == imax - 1;
            const int bord = (imax - i) * g_cd, rowfar = (imax - ro - 1) * g_cd;
            int runmin = XTED_INF;
            for (int c = W - 1; c >= 0; c--) {
                const bool se = dend[c] == 1;
                const int diag = se ? bord - g_cd : prev[(size_t)c + 1];
                const bool tcol = foff[c] == dend[c];
                int a;
                if (trow && tcol) {
                    a = diag + (ri.x != lab[c] ? g_cr : 0);
                } else {
                    int fv;
                    if (trow) fv = (dend[c] - foff[c]) * g_ci;
                    else if (tcol) fv = rowfar;
                    else {
                        if (sp < 1) FAIL("far-row stack underflow");
                        if (sp - 1 < lo) FAIL("stack top outside the shared window");
                        fv = cache[(size_t)((sp - 1) % g_cache)][(size_t)(c + foff[c])];
                        if (fv == -777) FAIL("far value never pushed");
                    }
                    const int dv = dt[(size_t)i * n + node[c]];
                    if (dv < 0) FAIL("tree distance (%d,%d) read before it was written", i, node[c]);
                    a = dv + fv;
                }
                int Av = std::min(a, prev[c] + g_cd);
                if (se) Av = std::min(Av, bord + g_ci);
                runmin = std::min(runmin, Av + key[c]);
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
            if (i != i0 && (ri.y & XTED_ROW_ISKR)) {
                sp--;
                if (sp > 0 && sp - 1 < lo) {
                    if (!deep) FAIL("window reload in a shallow unit");
                    for (int c = 0; c < W; c++)
                        if (far[c]) cache[(size_t)((sp - 1) % g_cache)][(size_t)c] = stk[(size_t)sp - 1][(size_t)c];
                    lo = sp - 1;
                }
            }
            if (i > i0 && (ri.y & XTED_ROW_PREVLEAF)) {
                if (sp >= H.stack_rows) FAIL("far-row stack overflow (%d rows)", H.stack_rows);
                for (int c = 0; c < W; c++)
                    if (far[c]) {
                        cache[(size_t)(sp % g_cache)][(size_t)c] = prev[c];
                        if (deep) stk[(size_t)sp][(size_t)c] = prev[c];
                    }
                sp++;
                if (sp > run.depth) FAIL("stack depth %d above the run's keyroot depth %d", sp, run.depth);
                if (sp - lo > g_cache) lo = sp - g_cache;
            }
        }
        if (sp != 0) FAIL("far-row stack not empty at table end (%d)", sp);
    }
}

// The same unit (one column segment) computed in column stripes of S columns
// the way the kernels' multi-block path does it: stripes right to left, each
// with its own rows and far-row stack, the row's suffix minimum continued
// from the stripe to the right (its carry per row), the tree rows' diagonal at
// a stripe's last column from the right stripe's first column one row below,
// and far columns owned by a stripe to the right read from that stripe's
// values kept per pushed row. Writes the unit's tree distances into dtv.
inline void run_unit_striped(const Pools &H, const XPair &pr, const XUnit &u, std::vector<int32_t> &dtv, int S) {
    int32_t *dt = dtv.data() + pr.dt_off;
    const XRun run = H.runs[(size_t)u.run];
    const XChunk ch = H.chunks[(size_t)u.chunk];
    if (ch.nseg != 1) FAIL("striped unit with %d segments", ch.nseg);
    const int W = ch.width, n = pr.n;
    const int2 *cn = H.node + pr.col_base;
    const int2 *rn = H.node + pr.row_base;
    const int j0 = H.krd[(size_t)ch.k_lo];
    std::vector<int> node(W), lab(W), foff(W), dend(W);
    for (int c = 0; c < W; c++) {
        const int j = j0 + c;
        node[c] = j;
        lab[c] = cn[j].x;
        foff[c] = (cn[j].y & XTED_ROW_ORL_MASK) + 1 - j;
        dend[c] = W - c;
    }
    const int K = (W + S - 1) / S, R = run.rows;
    // exported columns: far columns of some column in a stripe further left
    std::vector<char> exported(W, 0);
    for (int c = 0; c < W; c++) {
        const int f = c + foff[c];
        if (f < W && f / S != c / S) exported[f] = 1;
    }
    std::vector<std::vector<int>> CR((size_t)K, std::vector<int>((size_t)R, -999)), FC = CR;
    std::vector<std::vector<int>> E((size_t)R, std::vector<int>((size_t)W, -999));
    for (int st = K - 1; st >= 0; st--) {
        const int C0 = st * S, C1 = std::min(C0 + S, W), w = C1 - C0;
        const bool right = st + 1 < K;
        std::vector<int> prev(w), loc(w);
        int tflat = 0;
        for (int kr = run.kr_lo; kr < run.kr_hi; kr++) {
            const int i0 = H.krd[(size_t)kr];
            const int imax = (rn[i0].y & XTED_ROW_ORL_MASK) + 1;
            const int tbase = tflat;
            for (int c = 0; c < w; c++) prev[c] = dend[C0 + c] * g_ci;
            int edge = right ? dend[C1] * g_ci : 0;  // D[i+1][C1]: the bottom border first
            std::vector<std::vector<int>> stk;
            for (int i = imax - 1; i >= i0; i--, tflat++) {
                const int2 ri = rn[i];
                const int ro = ri.y & XTED_ROW_ORL_MASK;
                const bool trow = ro == imax - 1;
                const int bord = (imax - i) * g_cd, rowfar = (imax - ro - 1) * g_cd;
                int runmin = XTED_INF;
                for (int lc = w - 1; lc >= 0; lc--) {
                    const int c = C0 + lc;
                    const bool se = dend[c] == 1;
                    const int diag = se ? bord - g_cd : (lc + 1 < w ? prev[lc + 1] : edge);
                    const bool tcol = foff[c] == dend[c];
                    int a;
                    if (trow && tcol) {
                        a = diag + (ri.x != lab[c] ? g_cr : 0);
                    } else {
                        int fv;
                        if (trow) fv = (dend[c] - foff[c]) * g_ci;
                        else if (tcol) fv = rowfar;
                        else {
                            const int f = c + foff[c];
                            if (f < C1) {
                                if (stk.empty()) FAIL("stripe stack underflow");
                                fv = stk.back()[(size_t)(f - C0)];
                            } else {
                                if (!exported[f]) FAIL("far column %d not exported", f);
                                fv = E[(size_t)(tbase + (imax - 1 - (ro + 1)))][(size_t)f];
                                if (fv == -999) FAIL("exported far value read before it was written");
                            }
                        }
                        const int dv = dt[(size_t)i * n + node[c]];
                        if (dv < 0) FAIL("tree distance (%d,%d) read before it was written", i, node[c]);
                        a = dv + fv;
                    }
                    int Av = std::min(a, prev[lc] + g_cd);
                    if (se) Av = std::min(Av, bord + g_ci);
                    runmin = std::min(runmin, Av + c * g_ci);
                    loc[lc] = runmin;
                }
                int carry = XTED_INF;
                if (right) {
                    carry = CR[(size_t)st + 1][(size_t)tflat];
                    if (carry == -999) FAIL("carry of the right stripe missing");
                }
                for (int lc = 0; lc < w; lc++) {
                    const int c = C0 + lc;
                    prev[lc] = std::min(loc[lc], carry) - c * g_ci;
                    if (trow && foff[c] == dend[c]) {
                        int32_t &slot = dt[(size_t)i * n + node[c]];
                        if (slot >= 0) FAIL("tree distance (%d,%d) written twice", i, node[c]);
                        slot = prev[lc];
                    }
                }
                CR[(size_t)st][(size_t)tflat] = prev[0] + C0 * g_ci;
                FC[(size_t)st][(size_t)tflat] = prev[0];
                if (right) edge = FC[(size_t)st + 1][(size_t)tflat];
                if (i != i0 && (ri.y & XTED_ROW_ISKR)) stk.pop_back();
                if (i > i0 && (ri.y & XTED_ROW_PREVLEAF)) {
                    stk.push_back(prev);
                    for (int lc = 0; lc < w; lc++)
                        if (exported[C0 + lc]) E[(size_t)tflat][(size_t)(C0 + lc)] = prev[lc];
                }
            }
            if (!stk.empty()) FAIL("stripe stack not empty at table end");
        }
    }
}

}  // namespace emu
