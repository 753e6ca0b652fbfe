// plan.cpp -- host-side preprocessing and work decomposition.
//
// Per tree (reference counterparts):
//   orl(v) = v + size(v) - 1            X-TED_CPU/TED.cpp:21-42 (here O(n) from sizes)
//   keyroots: root and non-last children X-TED_CPU/TED.cpp:46-77 (the topmost node of
//             every distinct orl value is exactly that set)
//   kdepth: one bottom-up pass          X-TED_CPU/parallel_computing.cpp:93-119 (O(K^2) there)
// Per pair: every keyroot table (i0, j0) of level kdepth(i0) + kdepth(j0)
// (parallel_computing.cpp:121-123) is covered by exactly one unit, and a unit
// only runs after every unit of a lower level of its pair has finished, which
// is the reference's level order (parallel_computing.cpp:132-182).
#include "plan.h"

#include <algorithm>
#include <array>
#include <memory>
#include <cstring>
#include <unordered_map>

#include "../../include/xted.h"

namespace xted {

int validate_tree(const TreeView &t) {
    if (t.n < 0 || t.n > XTED_MAX_NODES) return XTED_EINVAL;
    if (t.n == 0) return XTED_OK;
    if (!t.labels || !t.off || (t.n > 1 && !t.idx)) return XTED_EINVAL;
    const int n = t.n;
    if (t.off[0] != 0 || t.off[n] != n - 1) return XTED_EINVAL;
    for (int v = 0; v < n; v++)
        if (t.off[v + 1] < t.off[v]) return XTED_EINVAL;
    // The k-th node of an iterative preorder walk must be node k.
    std::vector<int32_t> stack;
    stack.reserve(64);
    stack.push_back(0);
    int32_t expect = 0;
    while (!stack.empty()) {
        int32_t v = stack.back();
        stack.pop_back();
        if (v != expect) return XTED_EINVAL;
        expect++;
        for (int32_t e = t.off[v + 1] - 1; e >= t.off[v]; e--) {
            int32_t c = t.idx[e];
            if (c <= v || c >= n) return XTED_EINVAL;
            stack.push_back(c);
        }
    }
    return expect == n ? XTED_OK : XTED_EINVAL;
}

static void subtree_sizes(const TreeView &t, std::vector<int32_t> &size) {
    size.assign((size_t)t.n, 1);
    for (int v = t.n - 1; v >= 0; v--)
        for (int32_t e = t.off[v]; e < t.off[v + 1]; e++) size[(size_t)v] += size[(size_t)t.idx[e]];
}

void keyroot_sums(const TreeView &t, int64_t S[2]) {
    S[0] = S[1] = 0;
    if (t.n == 0) return;
    std::vector<int32_t> size;
    subtree_sizes(t, size);
    S[0] = S[1] = size[0];
    for (int v = 0; v < t.n; v++) {
        int32_t lo = t.off[v], hi = t.off[v + 1];
        for (int32_t e = lo; e < hi; e++) {
            int32_t s = size[(size_t)t.idx[e]];
            if (e != hi - 1) S[0] += s;  // right-path keyroots: not the last child
            if (e != lo) S[1] += s;      // left-path keyroots: not the first child
        }
    }
}

void build_otree(const TreeView &t0, bool mirrored, OTree &o) {
    const int n = t0.n;
    o = OTree();
    o.n = n;
    if (n == 0) return;
    // Oriented CSR (mirrored: children reversed, renumbered in preorder).
    std::vector<int32_t> lab((size_t)n), off((size_t)n + 1), idx((size_t)std::max(n - 1, 1));
    if (!mirrored) {
        std::memcpy(lab.data(), t0.labels, sizeof(int32_t) * (size_t)n);
        std::memcpy(off.data(), t0.off, sizeof(int32_t) * ((size_t)n + 1));
        if (n > 1) std::memcpy(idx.data(), t0.idx, sizeof(int32_t) * ((size_t)n - 1));
    } else {
        std::vector<int32_t> order, stack, newid((size_t)n);
        order.reserve((size_t)n);
        stack.push_back(0);
        while (!stack.empty()) {
            int32_t v = stack.back();
            stack.pop_back();
            order.push_back(v);
            for (int32_t e = t0.off[v]; e < t0.off[v + 1]; e++) stack.push_back(t0.idx[e]);
        }
        for (int k = 0; k < n; k++) newid[(size_t)order[(size_t)k]] = k;
        off[0] = 0;
        int32_t pos = 0;
        for (int k = 0; k < n; k++) {
            int32_t v = order[(size_t)k];
            lab[(size_t)k] = t0.labels[v];
            for (int32_t e = t0.off[v + 1] - 1; e >= t0.off[v]; e--) idx[(size_t)pos++] = newid[(size_t)t0.idx[e]];
            off[(size_t)k + 1] = pos;
        }
    }
    TreeView t;
    t.n = n;
    t.labels = lab.data();
    t.off = off.data();
    t.idx = idx.data();

    std::vector<int32_t> size;
    subtree_sizes(t, size);
    o.label = lab;
    o.orl.resize((size_t)n);
    o.leaf.assign((size_t)n, 0);
    o.kr.assign((size_t)n, 1);
    for (int v = 0; v < n; v++) {
        o.orl[(size_t)v] = v + size[(size_t)v] - 1;
        o.leaf[(size_t)v] = off[(size_t)v + 1] == off[(size_t)v];
        if (!o.leaf[(size_t)v]) o.kr[(size_t)idx[(size_t)off[(size_t)v + 1] - 1]] = 0;
    }
    // Keyroot depth bottom-up: f(v) = max kdepth of keyroots in sub(v), -1 if none.
    o.kdep.assign((size_t)n, -1);
    std::vector<int32_t> f((size_t)n, -1);
    for (int v = n - 1; v >= 0; v--) {
        int32_t mc = -1;
        for (int32_t e = off[(size_t)v]; e < off[(size_t)v + 1]; e++) mc = std::max(mc, f[(size_t)idx[(size_t)e]]);
        if (o.kr[(size_t)v]) {
            o.kdep[(size_t)v] = mc + 1;
            f[(size_t)v] = mc + 1;
        } else {
            f[(size_t)v] = mc;
        }
    }
    o.D = o.kdep[0];
    // keyroots on each root path (bounds the far-row stack)
    std::vector<int32_t> ka((size_t)n, 0);
    ka[0] = 1;
    o.maxka = 1;
    for (int v = 0; v < n; v++)
        for (int32_t e = off[(size_t)v]; e < off[(size_t)v + 1]; e++) {
            int32_t c = idx[(size_t)e];
            ka[(size_t)c] = ka[(size_t)v] + o.kr[(size_t)c];
            o.maxka = std::max(o.maxka, ka[(size_t)c]);
        }
    // keyroots grouped by depth, preorder within a depth
    o.krd_off.assign((size_t)o.D + 2, 0);
    for (int v = 0; v < n; v++)
        if (o.kr[(size_t)v]) o.krd_off[(size_t)o.kdep[(size_t)v] + 1]++;
    for (int d = 0; d <= o.D; d++) o.krd_off[(size_t)d + 1] += o.krd_off[(size_t)d];
    o.krd.resize((size_t)o.krd_off[(size_t)o.D + 1]);
    {
        std::vector<int32_t> fill(o.krd_off.begin(), o.krd_off.end() - 1);
        for (int v = 0; v < n; v++)
            if (o.kr[(size_t)v]) o.krd[(size_t)fill[(size_t)o.kdep[(size_t)v]]++] = v;
    }
    // column lists per depth: the concatenated subtrees of that depth's keyroots
    o.S = 0;
    o.seg_w.resize(o.krd.size());
    for (size_t k = 0; k < o.krd.size(); k++) {
        o.seg_w[k] = size[(size_t)o.krd[k]];
        o.S += o.seg_w[k];
    }
    o.cols.resize((size_t)o.S);
    o.col_off.assign((size_t)o.D + 2, 0);
    int64_t p = 0;
    for (int d = 0; d <= o.D; d++) {
        o.col_off[(size_t)d] = (int32_t)p;
        for (int32_t k = o.krd_off[(size_t)d]; k < o.krd_off[(size_t)d + 1]; k++) {
            int32_t j0 = o.krd[(size_t)k];
            int32_t je = o.orl[(size_t)j0] + 1;
            for (int32_t j = j0; j < je; j++) {
                int4h c;
                c.x = j;
                c.y = lab[(size_t)j];
                uint32_t z = (uint32_t)(o.orl[(size_t)j] + 1 - j);
                if (j > j0 && o.leaf[(size_t)j - 1]) z |= XTED_COL_FARCOL;
                c.z = (int32_t)z;
                c.w = je - j;
                o.cols[(size_t)p++] = c;
            }
        }
    }
    o.col_off[(size_t)o.D + 1] = (int32_t)p;
}

namespace {

struct TreeKey {
    const int32_t *l, *o, *i;
    int32_t n;
    bool operator==(const TreeKey &k) const { return l == k.l && o == k.o && i == k.i && n == k.n; }
};
struct TreeKeyHash {
    size_t operator()(const TreeKey &k) const {
        size_t h = (size_t)k.l * 0x9e3779b97f4a7c15ull;
        h ^= (size_t)k.o + 0x7f4a7c15 + (h << 6) + (h >> 2);
        h ^= (size_t)k.i + 0x165667b1 + (h << 6) + (h >> 2);
        h ^= (size_t)k.n;
        return h;
    }
};

// An oriented tree plus where its data sits in the plan's pools.
struct Slot {
    OTree t;
    bool row_done = false, col_done = false;
    int32_t row_base = 0;
    std::vector<int32_t> run_off;    // [D+2] global run indices by depth
    std::vector<int32_t> chunk_off;  // [D+2] global chunk indices by depth
};

// Estimated block-cycles per row of a unit (used only to order tasks).
inline double row_cost(bool wide, int width) {
    if (!wide) return 64.0 + 16.0 * ((width + 31) / 32);
    return 280.0 + 16.0 * ((width + XTED_CTA_THREADS - 1) / XTED_CTA_THREADS);
}

}  // namespace

int make_plan(const TreeView *a, const TreeView *b, int32_t npairs, const PlanOptions &opt,
              Plan &P) {
    P = Plan();
    if (npairs < 0) return XTED_EINVAL;
    const int nw = std::max(0, std::min(opt.narrow_width, XTED_NARROW_MAX));
    const int group_w = nw > 0 ? nw : XTED_NARROW_MAX;
    const int run_rows = std::max(1, opt.run_rows);

    std::unordered_map<TreeKey, int, TreeKeyHash> tid;
    std::vector<TreeView> uniq;
    std::vector<std::array<int64_t, 2>> sums;
    auto tree_id = [&](const TreeView &t) -> int {
        TreeKey k{t.labels, t.off, t.idx, t.n};
        auto it = tid.find(k);
        if (it != tid.end()) return it->second;
        int id = (int)uniq.size();
        tid.emplace(k, id);
        uniq.push_back(t);
        return id;
    };
    std::vector<int> pa((size_t)npairs), pb((size_t)npairs);
    for (int p = 0; p < npairs; p++) {
        pa[(size_t)p] = tree_id(a[p]);
        pb[(size_t)p] = tree_id(b[p]);
    }
    sums.resize(uniq.size());
    for (size_t u = 0; u < uniq.size(); u++) {
        int rc = validate_tree(uniq[u]);
        if (rc) return rc;
        int64_t S[2];
        keyroot_sums(uniq[u], S);
        sums[u] = {S[0], S[1]};
    }

    std::unordered_map<int64_t, int> slot_of;  // (tree id, mirrored) -> slot
    std::vector<std::unique_ptr<Slot>> slots;
    auto get_slot = [&](int u, bool mir) -> Slot & {
        int64_t key = (int64_t)u * 2 + (mir ? 1 : 0);
        auto it = slot_of.find(key);
        if (it != slot_of.end()) return *slots[(size_t)it->second];
        slots.emplace_back(new Slot());
        build_otree(uniq[(size_t)u], mir, slots.back()->t);
        slot_of.emplace(key, (int)slots.size() - 1);
        return *slots.back();
    };
    auto add_rows = [&](Slot &s) {
        if (s.row_done) return;
        s.row_done = true;
        const OTree &t = s.t;
        s.row_base = (int32_t)P.rowinfo.size();
        for (int v = 0; v < t.n; v++) {
            uint32_t y = (uint32_t)t.orl[(size_t)v];
            if (t.kr[(size_t)v]) y |= XTED_ROW_ISKR;
            if (v > 0 && t.leaf[(size_t)v - 1]) y |= XTED_ROW_PREVLEAF;
            P.rowinfo.push_back({t.label[(size_t)v], (int32_t)y});
        }
        const int32_t kbase = (int32_t)P.krd.size();
        P.krd.insert(P.krd.end(), t.krd.begin(), t.krd.end());
        s.run_off.assign((size_t)t.D + 2, 0);
        for (int d = 0; d <= t.D; d++) {
            s.run_off[(size_t)d] = (int32_t)P.runs.size();
            XRun r{-1, -1, 0, d};
            for (int32_t k = t.krd_off[(size_t)d]; k < t.krd_off[(size_t)d + 1]; k++) {
                int32_t sz = t.seg_w[(size_t)k];
                if (r.kr_lo >= 0 && r.rows + sz > run_rows) {
                    P.runs.push_back(r);
                    r = XRun{-1, -1, 0, d};
                }
                if (r.kr_lo < 0) r.kr_lo = kbase + k;
                r.kr_hi = kbase + k + 1;
                r.rows += sz;
            }
            if (r.kr_lo >= 0) P.runs.push_back(r);
        }
        s.run_off[(size_t)t.D + 1] = (int32_t)P.runs.size();
        P.stack_rows = std::max(P.stack_rows, t.maxka + 1);
    };
    auto add_cols = [&](Slot &s) {
        if (s.col_done) return;
        s.col_done = true;
        const OTree &t = s.t;
        const int32_t cbase = (int32_t)P.colinfo.size();
        P.colinfo.insert(P.colinfo.end(), t.cols.begin(), t.cols.end());
        s.chunk_off.assign((size_t)t.D + 2, 0);
        for (int d = 0; d <= t.D; d++) {
            s.chunk_off[(size_t)d] = (int32_t)P.chunks.size();
            int32_t pos = cbase + t.col_off[(size_t)d];
            XChunk c{pos, 0, d, 0};
            for (int32_t k = t.krd_off[(size_t)d]; k < t.krd_off[(size_t)d + 1]; k++) {
                int32_t w = t.seg_w[(size_t)k];
                if (c.nseg > 0 && c.width + w > group_w) {
                    P.chunks.push_back(c);
                    c = XChunk{pos, 0, d, 0};
                }
                c.width += w;
                c.nseg += 1;
                pos += w;
            }
            if (c.nseg > 0) P.chunks.push_back(c);
        }
        s.chunk_off[(size_t)t.D + 1] = (int32_t)P.chunks.size();
    };

    P.pairs.resize((size_t)npairs);
    P.trivial.assign((size_t)npairs, -1);
    // Per pair, per level: the estimated time of its slowest task.
    struct PendingTask { XTask t; int level; double est; };
    std::vector<PendingTask> all;
    std::vector<double> level_est;
    std::vector<std::pair<double, XUnit>> narrow;

    for (int p = 0; p < npairs; p++) {
        const TreeView &A0 = uniq[(size_t)pa[(size_t)p]];
        const TreeView &B0 = uniq[(size_t)pb[(size_t)p]];
        XPair &pr = P.pairs[(size_t)p];
        pr.m = A0.n;
        pr.n = B0.n;
        pr.dt_off = P.dt_elems;
        pr.row_base = 0;
        pr.pad = 0;
        if (A0.n == 0 || B0.n == 0) {  // X-TED_CPU/TED.cpp:181-186
            P.trivial[(size_t)p] = A0.n == 0 ? B0.n : A0.n;
            continue;
        }
        const auto &sa = sums[(size_t)pa[(size_t)p]], &sb = sums[(size_t)pb[(size_t)p]];
        const int64_t cr = sa[0] * sb[0], cl = sa[1] * sb[1];
        bool mir = opt.orientation == XTED_ORIENT_LEFT ||
                   (opt.orientation == XTED_ORIENT_AUTO && cl < cr);
        P.cells += mir ? cl : cr;
        P.cells_right += cr;
        Slot &SA = get_slot(pa[(size_t)p], mir);
        Slot &SB = get_slot(pb[(size_t)p], mir);
        add_rows(SA);
        add_cols(SB);
        pr.row_base = SA.row_base;
        P.dt_elems += (int64_t)A0.n * (int64_t)B0.n;
        const OTree &A = SA.t, &B = SB.t;
        const int L = A.D + B.D;
        P.levels_max = std::max(P.levels_max, L + 1);
        level_est.assign((size_t)L + 1, 0.0);
        const size_t first = all.size();
        int32_t need = 0;
        for (int d = 0; d <= L; d++) {
            const int32_t level_first = (int32_t)(all.size() - first);
            narrow.clear();
            for (int al = std::max(0, d - B.D); al <= std::min(A.D, d); al++) {
                const int de = d - al;
                for (int32_t r = SA.run_off[(size_t)al]; r < SA.run_off[(size_t)al + 1]; r++) {
                    const int rows = P.runs[(size_t)r].rows;
                    for (int32_t c = SB.chunk_off[(size_t)de]; c < SB.chunk_off[(size_t)de + 1]; c++) {
                        const int w = P.chunks[(size_t)c].width;
                        const bool wide = w > nw;
                        const double est = rows * row_cost(wide, w);
                        if (wide) {
                            XTask t;
                            t.pair = p;
                            t.need = need;
                            t.kind_n = XTED_TASK_WIDE | 1u;
                            t.unit_lo = (int32_t)P.units.size();
                            P.units.push_back({r, c});
                            all.push_back({t, d, est});
                            P.max_wide = std::max(P.max_wide, w);
                        } else {
                            narrow.push_back({est, XUnit{r, c}});
                        }
                    }
                }
            }
            std::sort(narrow.begin(), narrow.end(),
                      [](const std::pair<double, XUnit> &x, const std::pair<double, XUnit> &y) {
                          return x.first > y.first;
                      });
            for (size_t i = 0; i < narrow.size(); i += XTED_WARPS) {
                size_t cnt = std::min((size_t)XTED_WARPS, narrow.size() - i);
                XTask t;
                t.pair = p;
                t.need = need;
                t.kind_n = (uint32_t)cnt;
                t.unit_lo = (int32_t)P.units.size();
                for (size_t k = 0; k < cnt; k++) P.units.push_back(narrow[i + k].second);
                all.push_back({t, d, narrow[i].first});
            }
            for (size_t k = first + (size_t)level_first; k < all.size(); k++)
                level_est[(size_t)d] = std::max(level_est[(size_t)d], all[k].est);
            need = (int32_t)(all.size() - first);
        }
        // Highest-level-first priority: remaining critical path from this level.
        std::vector<double> rank((size_t)L + 2, 0.0);
        for (int d = L; d >= 0; d--) rank[(size_t)d] = rank[(size_t)d + 1] + level_est[(size_t)d] + 1.0;
        for (size_t k = first; k < all.size(); k++) all[k].est = rank[(size_t)all[k].level];
    }
    // Global queue order: larger remaining critical path first. Every task's
    // dependencies (lower levels of its pair) have a strictly larger rank, so
    // they precede it and the queue can never wait on an unclaimed task.
    std::vector<int32_t> order(all.size());
    for (size_t k = 0; k < order.size(); k++) order[k] = (int32_t)k;
    std::stable_sort(order.begin(), order.end(), [&](int32_t x, int32_t y) {
        return all[(size_t)x].est > all[(size_t)y].est;
    });
    P.tasks.resize(all.size());
    for (size_t k = 0; k < order.size(); k++) P.tasks[k] = all[(size_t)order[k]].t;
    return XTED_OK;
}

}  // namespace xted
