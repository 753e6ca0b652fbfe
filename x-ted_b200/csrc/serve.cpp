// serve.cpp -- a resident corpus and exact top-k TED queries, with continuous
// batching into one running persistent DP launch.
//
// Nothing in the reference serves queries (its only caller computes one pair,
// X-TED_CPU/TED_test.cpp:26-47); the per-pair work is the same keyroot-table
// DP as the batch path (X-TED_CPU/parallel_computing.cpp:4-182).
//
// Layout. The corpus trees are planned once (both orientations) on the host
// with the batch planner's own functions (plan_core.h) and stay resident on
// the device. A query is one more tree planned into one of XTED_SERVE_SLOTS
// slots: its node pools, its pairs (query x every corpus tree, the corpus
// tree as the row tree so the far-row stack depth is a corpus property),
// their level entries, units and tasks. Distance tables come from a pool of
// device memory; a query is admitted when a slot is free and its tables,
// units, tasks and entries fit ("DP scratch bytes"), in arrival order.
//
// Continuous batching. An admitted query's plan is copied to the device on a
// copy stream, followed by a mailbox record and the posted count. The DP
// kernel, launched once and kept running while there is work, claims the
// record, publishes level 0 of the query's pairs into its ready queue and
// runs them beside the queries already in flight. Each query owns one
// priority bucket (by arrival), and blocks probe the oldest query's bucket
// first, so earlier queries finish first while later ones fill idle blocks.
// A finished pair writes its distance into pinned host memory; the last pair
// of a query raises the slot's flag. Blocks leave the launch after an idle
// spell; a worker thread relaunches when new work arrives.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <climits>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/xted.h"
#include "ctx.h"
#include "plan.h"
#include "plan_core.h"
#include "serve_plan.h"

namespace xted {
cudaError_t launch_dp(const XKernelParams &P, int grid, cudaStream_t s);
}

static_assert(XTED_SERVE_SLOTS == XTED_SERVE_SLOTS_MAX, "slot count of the ABI and the kernels");
static_assert(XTED_SERVE_SLOTS <= XTED_BUCKETS, "one ready-queue bucket per query in flight");

namespace xted {

namespace {

double now_ms() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

// Allocator over [0, cap) (elements): first fit, or next fit from a cursor
// that follows the last allocation (freed ranges are then reused only after
// the cursor has gone round the whole pool).
class Extents {
public:
    void reset(int64_t cap, bool next_fit = false) {
        free_.clear();
        if (cap > 0) free_[0] = cap;
        cap_ = cap;
        next_fit_ = next_fit;
        cursor_ = 0;
    }
    int64_t cap() const { return cap_; }
    bool alloc(int64_t n, int64_t *off) {
        n = std::max<int64_t>(n, 1);
        auto take = [&](std::map<int64_t, int64_t>::iterator it, int64_t at) {
            // [at, at + n) lies inside the free range it
            const int64_t lo = it->first, len = it->second;
            free_.erase(it);
            if (at > lo) free_[lo] = at - lo;
            if (lo + len > at + n) free_[at + n] = lo + len - (at + n);
            *off = at;
            cursor_ = at + n;
        };
        if (next_fit_) {
            // a free range holding the cursor, then ranges after it, then from the start
            auto it = free_.upper_bound(cursor_);
            if (it != free_.begin()) {
                auto pv = std::prev(it);
                if (pv->first + pv->second >= cursor_ + n) {
                    take(pv, std::max(pv->first, cursor_));
                    return true;
                }
            }
            for (auto jt = it; jt != free_.end(); ++jt)
                if (jt->second >= n) {
                    take(jt, jt->first);
                    return true;
                }
        }
        for (auto it = free_.begin(); it != free_.end(); ++it)
            if (it->second >= n) {
                take(it, it->first);
                return true;
            }
        return false;
    }
    // n = 0: nothing is held (a slot whose extents were already released)
    void release(int64_t off, int64_t n) {
        if (n <= 0) return;
        auto it = free_.emplace(off, n).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }

private:
    std::map<int64_t, int64_t> free_;
    int64_t cap_ = 0, cursor_ = 0;
    bool next_fit_ = false;
};

struct Query {
    std::vector<int32_t> lab, off, idx;
    int32_t n = 0, k = 0;
    std::vector<int32_t> lb, dist;  // per corpus tree: label lower bound; distance once known (-1 before)
    int state = 0;  // 0 queued, 1 admitted, 2 done, < 0 error code
    std::vector<int32_t> ids, dists;
    double t_submit = 0, t_admit = 0, t_done = 0;
};

struct Slot {
    bool busy = false;
    bool planned = false;
    int round = 1;               // 1: the most promising corpus trees; 2: what may still beat them
    bool need_post = false;      // a planned next round waits for device room
    std::vector<uint8_t> inc;    // corpus trees computed in this round
    uint64_t ticket = 0;
    int64_t seq = 0;
    int32_t gen = 0;
    int32_t rec = -1;            // mailbox record of the posted round
    int64_t dt_off = 0, dt_n = 0, u_off = 0, u_n = 0, t_off = 0, t_n = 0, e_off = 0, e_n = 0;
    QPlan plan;
};

}  // namespace

struct ServeState {
    xted_ctx *c = nullptr;
    int T = 0, S = XTED_SERVE_SLOTS, Qmax = XTED_SERVE_MAX_QUERY;  // XTED_SERVE_SLOTS == XTED_SERVE_SLOTS_MAX
    int32_t max_tree = 0;  // largest corpus tree
    int64_t Nc_nonempty = 0;
    ServePools pools;  // host planning pools: the corpus, then one region per slot
    // device
    std::vector<void *> dev_allocs;
    int2 *d_node = nullptr;
    int32_t *d_krd = nullptr, *d_cumw = nullptr, *d_first = nullptr, *d_state = nullptr, *d_ctl = nullptr,
            *d_mbox = nullptr, *d_slot = nullptr, *d_err = nullptr, *d_scratch = nullptr, *d_dt = nullptr;
    XRun *d_runs = nullptr;
    XChunk *d_chunks = nullptr;
    XPair *d_pairs = nullptr;
    XEntry *d_entries = nullptr;
    XUnit *d_units = nullptr;
    XTask *d_tasks = nullptr;
    unsigned long long *d_rq = nullptr;
    int32_t *h_results = nullptr, *h_flags = nullptr;  // mapped pinned host memory
    Extents dt_ext, u_ext, t_ext, e_ext;
    int rq_log2 = 12;
    XKernelParams K{};
    cudaStream_t ks = nullptr, cs = nullptr;
    cudaEvent_t kev = nullptr;
    bool running = false;
    int32_t posted = 0;
    int32_t top_written = -1;
    // requests
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<uint64_t> pending;
    std::unordered_map<uint64_t, Query> queries;
    uint64_t next_ticket = 1;
    int64_t next_seq = 0;
    int32_t next_gen = 1;
    Slot slots[XTED_SERVE_SLOTS];
    int error = 0;
    bool stop = false;
    std::thread worker;
    // counters
    int64_t launches = 0, served = 0, pairs_served = 0, cells_served = 0, pairs_pruned = 0, second_rounds = 0;
    int64_t bound_us = 0, plan_us = 0;  // host time spent on bounds and on planning
    // exact top-k pruning by lower bounds: 0 off, 1 label multisets, 2 preorder sequences
    int prune = 2;
    int first_round = 32;                            // at least this many trees, and 4k, in round 1
    std::vector<std::vector<int32_t>> sorted_labels;  // per corpus tree
    std::unordered_map<int32_t, int32_t> dense;       // corpus label -> dense symbol
    std::vector<std::vector<int32_t>> dense_seq;      // per corpus tree: preorder dense symbols
};

namespace {

constexpr int kMaxPending = 1 << 16;
constexpr int64_t kUnitCap = 24 << 20, kTaskCap = 12 << 20, kEntryCap = 2 << 20;
constexpr int64_t kDtCapMax = (int64_t)4 << 30;  // int32 elements (16 GiB)

template <class T>
int dev_alloc(ServeState *s, T **p, size_t count) {
    void *q = nullptr;
    if (cudaMalloc(&q, sizeof(T) * std::max<size_t>(count, 1)) != cudaSuccess) {
        cudaGetLastError();
        return XTED_ENOMEM;
    }
    s->dev_allocs.push_back(q);
    *p = (T *)q;
    return XTED_OK;
}

int upload(void *dst, const void *src, size_t bytes, cudaStream_t st) {
    if (bytes == 0) return XTED_OK;
    return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st) == cudaSuccess ? XTED_OK : XTED_ECUDA;
}

void free_all(ServeState *s) {
    for (void *p : s->dev_allocs) cudaFree(p);
    s->dev_allocs.clear();
    if (s->h_results) cudaFreeHost(s->h_results);
    if (s->h_flags) cudaFreeHost(s->h_flags);
    s->h_results = s->h_flags = nullptr;
    if (s->kev) cudaEventDestroy(s->kev);
    if (s->ks) cudaStreamDestroy(s->ks);
    if (s->cs) cudaStreamDestroy(s->cs);
    s->kev = nullptr;
    s->ks = s->cs = nullptr;
}

// Reserves device room for a planned query; false if it does not fit now.
bool reserve(ServeState *s, Slot &sl) {
    const QPlan &p = sl.plan;
    sl.dt_n = std::max<int64_t>(p.dt_elems, 1);
    sl.u_n = std::max<int64_t>((int64_t)p.units.size(), 1);
    sl.t_n = std::max<int64_t>((int64_t)p.tasks.size(), 1);
    sl.e_n = std::max<int64_t>((int64_t)p.entries.size(), 1);
    if (!s->dt_ext.alloc(sl.dt_n, &sl.dt_off)) return false;
    if (!s->u_ext.alloc(sl.u_n, &sl.u_off)) {
        s->dt_ext.release(sl.dt_off, sl.dt_n);
        return false;
    }
    if (!s->t_ext.alloc(sl.t_n, &sl.t_off)) {
        s->dt_ext.release(sl.dt_off, sl.dt_n);
        s->u_ext.release(sl.u_off, sl.u_n);
        return false;
    }
    if (!s->e_ext.alloc(sl.e_n, &sl.e_off)) {
        s->dt_ext.release(sl.dt_off, sl.dt_n);
        s->u_ext.release(sl.u_off, sl.u_n);
        s->t_ext.release(sl.t_off, sl.t_n);
        return false;
    }
    return true;
}

bool never_fits(ServeState *s, const QPlan &p) {
    return p.dt_elems > s->dt_ext.cap() || (int64_t)p.units.size() > s->u_ext.cap() ||
           (int64_t)p.tasks.size() > s->t_ext.cap() || (int64_t)p.entries.size() > s->e_ext.cap();
}

void release_extents(ServeState *s, Slot &sl) {
    s->dt_ext.release(sl.dt_off, sl.dt_n);
    s->u_ext.release(sl.u_off, sl.u_n);
    s->t_ext.release(sl.t_off, sl.t_n);
    s->e_ext.release(sl.e_off, sl.e_n);
    sl.dt_n = sl.u_n = sl.t_n = sl.e_n = 0;
}

void release(ServeState *s, Slot &sl) {
    s->dt_ext.release(sl.dt_off, sl.dt_n);
    s->u_ext.release(sl.u_off, sl.u_n);
    s->t_ext.release(sl.t_off, sl.t_n);
    s->e_ext.release(sl.e_off, sl.e_n);
    sl = Slot{};
}

// Fixes the plan up to its device offsets and copies it, its slot words and
// a mailbox record to the device, in that order, on the copy stream.
int post(ServeState *s, int slot, Slot &sl) {
    QPlan &p = sl.plan;
    const int T = s->T;
    const int64_t pair_base = (int64_t)slot * T;
    serve_fixup(p, slot, T, sl.dt_off, sl.u_off, sl.t_off, sl.e_off, (int32_t)((-sl.seq) & (XTED_BUCKETS - 1)));
    const ServePools &H = s->pools;
    const DTree &Q = H.trees[(size_t)(T + slot)];
    const size_t nb = 2 * (size_t)Q.nbase, n2 = 2 * (size_t)Q.n;
    cudaStream_t st = s->cs;
    const std::vector<int32_t> zeros(XTED_ESTATE * p.entries.size(), 0);
    std::vector<int32_t> first_held;  // test hook: one computed pair's level 0 is never published
    if (s->c->fault == XTED_FAULT_HOLD_PAIR) {
        first_held = p.first;
        for (int32_t &f : first_held)
            if (f >= 0) {
                f = -1;
                break;
            }
        s->c->fault = 0;
    }
    const std::vector<int32_t> &first = first_held.empty() ? p.first : first_held;
    const int32_t words[2] = {p.need, sl.gen};
    const int32_t rec[4] = {slot, (int32_t)pair_base, T, 0};
    const int32_t posted = s->posted + 1;
    int rc = XTED_OK;
    rc |= upload(s->d_node + nb, H.node.data() + nb, n2 * sizeof(int2), st);
    rc |= upload(s->d_krd + nb, H.krd.data() + nb, n2 * 4, st);
    rc |= upload(s->d_cumw + nb, H.cumw.data() + nb, n2 * 4, st);
    rc |= upload(s->d_runs + nb, H.runs.data() + nb, n2 * sizeof(XRun), st);
    rc |= upload(s->d_chunks + nb, H.chunks.data() + nb, n2 * sizeof(XChunk), st);
    rc |= upload(s->d_pairs + pair_base, p.pairs.data(), p.pairs.size() * sizeof(XPair), st);
    rc |= upload(s->d_first + pair_base, first.data(), first.size() * 4, st);
    rc |= upload(s->d_entries + sl.e_off, p.entries.data(), p.entries.size() * sizeof(XEntry), st);
    rc |= upload(s->d_state + XTED_ESTATE * sl.e_off, zeros.data(), zeros.size() * 4, st);
    rc |= upload(s->d_units + sl.u_off, p.units.data(), p.units.size() * sizeof(XUnit), st);
    rc |= upload(s->d_tasks + sl.t_off, p.tasks.data(), p.tasks.size() * sizeof(XTask), st);
    rc |= upload(s->d_slot + XTED_SERVE_SLOTS + slot, &words[0], 4, st);      // slot_need
    rc |= upload(s->d_slot + 2 * XTED_SERVE_SLOTS + slot, &words[1], 4, st);  // slot_gen
    rc |= upload(s->d_mbox + XTED_MBOX_REC + 4 * (s->posted & (XTED_SERVE_RECS - 1)), rec, sizeof(rec), st);
    rc |= upload(s->d_mbox + XTED_MBOX_POSTED, &posted, 4, st);
    if (rc) return XTED_ECUDA;
    sl.rec = s->posted;
    s->posted = posted;
    return XTED_OK;
}

// Finishes a query from its known distances: every corpus tree not computed
// has a bound that cannot beat the k-th of them (prune_round2 saw to it).
void finish_query(ServeState *s, Query &q) {
    q.ids.assign((size_t)q.k, -1);
    q.dists.assign((size_t)q.k, -1);
    topk_known(q.dist, q.k, q.ids.data(), q.dists.data());
    for (int32_t d : q.dist) s->pairs_pruned += d < 0;
    q.state = 2;
    q.t_done = now_ms();
}

// Round 1 of a query: the bound of every corpus tree (host threads), the
// distances of empty-tree pairs, and the trees computed first.
void first_round(ServeState *s, const Query &q, std::vector<int32_t> &lb, std::vector<int32_t> &dist,
                 std::vector<uint8_t> &inc) {
    const int T = s->T, level = s->prune;
    // distances are TED(query, corpus tree): deleting a query node costs
    // cost_del, inserting a corpus node cost_ins
    const xted_opts &o = s->c->opts;
    const bool unit = o.cost_del == 1 && o.cost_ins == 1 && o.cost_ren == 1;
    lb.assign((size_t)T, 0);
    dist.assign((size_t)T, -1);
    for (int t = 0; t < T; t++) {
        const int32_t ct = (int32_t)s->sorted_labels[(size_t)t].size();
        if (q.n == 0) dist[(size_t)t] = ct * o.cost_ins;  // X-TED_CPU/TED.cpp:181-186, with costs
        else if (ct == 0) dist[(size_t)t] = q.n * o.cost_del;
    }
    if (!unit && level > 0) {
        // weighted bounds: the label bound under the costs, and the unit
        // Levenshtein bound times the cheapest operation (an alignment of
        // distance L makes at least L operations)
        std::vector<int32_t> ql(q.lab);
        std::sort(ql.begin(), ql.end());
        std::vector<int32_t> qd;
        SeqBits P;
        if (level >= 2 && q.n > 0) {
            qd.resize((size_t)q.n);
            for (int v = 0; v < q.n; v++) {
                auto it = s->dense.find(q.lab[(size_t)v]);
                qd[(size_t)v] = it == s->dense.end() ? -1 : it->second;
            }
            P.build(qd.data(), q.n, (int)s->dense.size());
        }
        const int cmin = std::min(o.cost_del, std::min(o.cost_ins, o.cost_ren));
        parallel_for(T, 16, [&](int64_t lo, int64_t hi) {
            std::vector<uint64_t> work;
            for (int64_t t = lo; t < hi; t++) {
                if (dist[(size_t)t] >= 0) continue;
                const std::vector<int32_t> &tl = s->sorted_labels[(size_t)t];
                int32_t b = label_lower_bound_cost(label_common(ql.data(), q.n, tl.data(), (int)tl.size()), q.n,
                                                   (int)tl.size(), o.cost_del, o.cost_ins, o.cost_ren);
                if (level >= 2) {
                    const std::vector<int32_t> &sq = s->dense_seq[(size_t)t];
                    b = std::max<int32_t>(b, cmin * P.distance(sq.data(), (int)sq.size(), work));
                }
                lb[(size_t)t] = b;
            }
        });
    } else if (level == 1) {
        std::vector<int32_t> ql(q.lab);
        std::sort(ql.begin(), ql.end());
        parallel_for(T, 64, [&](int64_t lo, int64_t hi) {
            for (int64_t t = lo; t < hi; t++) {
                const std::vector<int32_t> &tl = s->sorted_labels[(size_t)t];
                lb[(size_t)t] = label_lower_bound(ql.data(), q.n, tl.data(), (int)tl.size());
            }
        });
    } else if (level >= 2 && q.n > 0) {
        std::vector<int32_t> qd((size_t)q.n);
        for (int v = 0; v < q.n; v++) {
            auto it = s->dense.find(q.lab[(size_t)v]);
            qd[(size_t)v] = it == s->dense.end() ? -1 : it->second;
        }
        SeqBits P;
        P.build(qd.data(), q.n, (int)s->dense.size());
        parallel_for(T, 16, [&](int64_t lo, int64_t hi) {
            std::vector<uint64_t> work;
            for (int64_t t = lo; t < hi; t++) {
                const std::vector<int32_t> &sq = s->dense_seq[(size_t)t];
                if (dist[(size_t)t] < 0) lb[(size_t)t] = P.distance(sq.data(), (int)sq.size(), work);
            }
        });
    }
    prune_round1(lb, dist, std::max<size_t>((size_t)s->first_round, 4 * (size_t)q.k), level > 0, inc);
}

int64_t oldest_seq(ServeState *s) {
    int64_t o = INT64_MAX;
    for (const Slot &sl : s->slots)
        if (sl.busy && sl.planned) o = std::min(o, sl.seq);  // between rounds too: its bucket stays its own
    return o;
}

void fail_inflight(ServeState *s, int code) {
    for (int i = 0; i < s->S; i++) {
        Slot &sl = s->slots[i];
        if (!sl.busy) continue;
        auto it = s->queries.find(sl.ticket);
        if (it != s->queries.end()) it->second.state = code;
        release(s, sl);
    }
}

// One pass of the serving loop (called with the lock held; drops it while planning).
bool step(ServeState *s, std::unique_lock<std::mutex> &lk) {
    bool progress = false;
    const int T = s->T;
    // 1. completions
    for (int i = 0; i < s->S; i++) {
        Slot &sl = s->slots[i];
        if (!sl.busy || sl.gen == 0) continue;
        if (((volatile int32_t *)s->h_flags)[i] != sl.gen) continue;
        std::atomic_thread_fence(std::memory_order_acquire);
        s->pairs_served += sl.plan.need;
        s->cells_served += sl.plan.cells;
        progress = true;
        auto it = s->queries.find(sl.ticket);
        if (it == s->queries.end()) {
            release(s, sl);
            continue;
        }
        Query &q = it->second;
        const int32_t *res = s->h_results + (size_t)i * T;
        for (int t = 0; t < T; t++)
            if (sl.plan.trivial[(size_t)t] < 0 && sl.inc[(size_t)t]) q.dist[(size_t)t] = res[t];
        if (sl.round == 1 && s->prune > 0) {
            std::vector<uint8_t> inc2;
            if (prune_round2(q.lb, q.dist, q.k, inc2)) {  // plan round 2 in the same slot (its bucket stays reserved)
                release_extents(s, sl);
                sl.gen = 0;
                sl.round = 2;
                sl.inc = std::move(inc2);
                Query qcopy = q;
                const int wr = s->c->opts.wide_rows;
                lk.unlock();
                const double t1 = now_ms();
                serve_plan_query(s->pools, i, qcopy.lab.data(), qcopy.off.data(), qcopy.idx.data(), qcopy.n,
                                 s->c->opts.orientation, s->c->opts.narrow_width, wr > 0 ? wr : -1, sl.plan,
                                 sl.inc.data());
                const double t2 = now_ms();
                lk.lock();
                s->plan_us += (int64_t)((t2 - t1) * 1e3);
                s->second_rounds++;
                if (never_fits(s, sl.plan)) {  // round 2 covers more trees than round 1 did
                    q.state = XTED_ENOMEM;
                    release(s, sl);
                    continue;
                }
                sl.need_post = true;
                continue;
            }
        }
        finish_query(s, q);
        s->served++;
        release(s, sl);
    }
    // next rounds waiting for device room
    for (int i = 0; i < s->S; i++) {
        Slot &sl = s->slots[i];
        if (!sl.busy || !sl.need_post || !reserve(s, sl)) continue;
        sl.need_post = false;
        sl.gen = s->next_gen++;
        if (s->next_gen <= 0) s->next_gen = 1;
        auto it = s->queries.find(sl.ticket);
        if (post(s, i, sl) != XTED_OK) {
            if (it != s->queries.end()) it->second.state = XTED_ECUDA;
            release(s, sl);
        }
        progress = true;
    }
    if (progress) s->cv_done.notify_all();
    // 2. the launch: notice its end (and any error), relaunch for work in flight.
    // One query: the launch may end between two of them.
    const cudaError_t kq = s->running ? cudaEventQuery(s->kev) : cudaErrorNotReady;
    if (s->running && kq == cudaSuccess) {
        s->running = false;
        int32_t err = 0, cons = 0;
        if (cudaMemcpy(&err, s->d_err, 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(&cons, s->d_mbox + XTED_MBOX_CONSUMED, 4, cudaMemcpyDeviceToHost) != cudaSuccess)
            err = XTED_ECUDA;
        int32_t consumed = cons & ~XTED_MBOX_CLOSED;
        if (err != 0) {
            s->error = err;
            fail_inflight(s, err);
            cudaMemset(s->d_err, 0, 8 * sizeof(int32_t));
            cudaMemset(s->d_slot, 0, XTED_SERVE_SLOTS * sizeof(int32_t));
            // records of the failed queries are void: the next launch starts after them
            cudaStreamSynchronize(s->cs);
            consumed = s->posted;
            s->cv_done.notify_all();
            progress = true;
        } else {
            // Every query whose record this launch claimed has finished: a
            // launch leaves only when all of its blocks are idle. One that
            // has not (its work was lost) fails instead of waiting forever.
            for (int i = 0; i < s->S; i++) {
                Slot &sl = s->slots[i];
                if (!sl.busy || sl.gen == 0 || sl.rec < 0 || sl.rec >= consumed) continue;
                if (((volatile int32_t *)s->h_flags)[i] == sl.gen) continue;  // done: step 1 takes it
                if (std::getenv("XTED_SERVE_DEBUG")) {
                    int32_t done = -1;
                    cudaMemcpy(&done, s->d_slot + i, 4, cudaMemcpyDeviceToHost);
                    std::fprintf(stderr,
                                 "xted serve: launch %lld ended with slot %d unfinished: round %d gen %d rec %d "
                                 "consumed %d posted %d need %d done %d flag %d\n",
                                 (long long)s->launches, i, sl.round, sl.gen, sl.rec, consumed, s->posted,
                                 sl.plan.need, done, ((volatile int32_t *)s->h_flags)[i]);
                }
                auto it = s->queries.find(sl.ticket);
                if (it != s->queries.end()) it->second.state = XTED_ETIMEOUT;
                s->error = XTED_ETIMEOUT;
                const int32_t zero = 0;  // the slot's finished-pair count restarts for its next query
                if (cudaMemcpy(s->d_slot + i, &zero, 4, cudaMemcpyHostToDevice) != cudaSuccess) cudaGetLastError();
                release(s, sl);
                s->cv_done.notify_all();
                progress = true;
            }
        }
        // reopen the claim word for the next launch
        if (cons != consumed &&
            cudaMemcpy(s->d_mbox + XTED_MBOX_CONSUMED, &consumed, 4, cudaMemcpyHostToDevice) != cudaSuccess) {
            cudaGetLastError();
            s->error = XTED_ECUDA;
            fail_inflight(s, XTED_ECUDA);
            s->cv_done.notify_all();
        }
    } else if (s->running && kq != cudaErrorNotReady) {
        cudaGetLastError();
        s->running = false;
        s->error = XTED_ECUDA;
        fail_inflight(s, XTED_ECUDA);
        s->cv_done.notify_all();
    }
    // 3. admission, in arrival order
    while (!s->pending.empty()) {
        const uint64_t ticket = s->pending.front();
        auto it = s->queries.find(ticket);
        if (it == s->queries.end()) {
            s->pending.pop_front();
            continue;
        }
        Query &q = it->second;
        int slot = -1;
        for (int i = 0; i < s->S; i++)
            if (s->slots[i].busy && s->slots[i].ticket == ticket) slot = i;
        if (slot < 0) {
            const int64_t seq = s->next_seq;
            const int64_t old = oldest_seq(s);
            if (old != INT64_MAX && seq - old >= XTED_BUCKETS) break;  // keep buckets distinct by age
            for (int i = 0; i < s->S && slot < 0; i++)
                if (!s->slots[i].busy) slot = i;
            if (slot < 0) break;
            Slot &sl = s->slots[slot];
            sl.busy = true;
            sl.ticket = ticket;
            sl.seq = seq;
            s->next_seq++;
            Query qcopy = q;  // plan outside the lock
            lk.unlock();
            const double t0 = now_ms();
            std::vector<int32_t> lb, dist;
            std::vector<uint8_t> inc;
            first_round(s, qcopy, lb, dist, inc);
            const double t1 = now_ms();
            const int wr = s->c->opts.wide_rows;
            serve_plan_query(s->pools, slot, qcopy.lab.data(), qcopy.off.data(), qcopy.idx.data(), qcopy.n,
                             s->c->opts.orientation, s->c->opts.narrow_width, wr > 0 ? wr : -1,
                             sl.plan, inc.data());
            const double t2 = now_ms();
            lk.lock();
            s->bound_us += (int64_t)((t1 - t0) * 1e3);
            s->plan_us += (int64_t)((t2 - t1) * 1e3);
            if (s->stop || !sl.busy || sl.ticket != ticket) break;  // shut down meanwhile
            q.lb = std::move(lb);
            q.dist = std::move(dist);
            sl.inc = std::move(inc);
            sl.round = 1;
            sl.planned = true;
            progress = true;
        }
        Slot &sl = s->slots[slot];
        if (never_fits(s, sl.plan)) {
            q.state = XTED_ENOMEM;
            sl = Slot{};
            s->pending.pop_front();
            s->cv_done.notify_all();
            continue;
        }
        if (sl.plan.need == 0) {  // empty query or empty corpus trees only
            finish_query(s, q);
            sl = Slot{};
            s->pending.pop_front();
            s->cv_done.notify_all();
            progress = true;
            continue;
        }
        if (!reserve(s, sl)) break;  // wait for memory to free up
        sl.gen = s->next_gen++;
        if (s->next_gen <= 0) s->next_gen = 1;
        const int rc = post(s, slot, sl);
        s->pending.pop_front();
        if (rc) {
            q.state = rc;
            release(s, sl);
            s->cv_done.notify_all();
            continue;
        }
        q.state = 1;
        q.t_admit = now_ms();
        progress = true;
    }
    // 4. priority: the oldest query in flight goes first
    const int64_t old = oldest_seq(s);
    if (old != INT64_MAX) {
        const int32_t top = (int32_t)((-old) & (XTED_BUCKETS - 1));
        if (top != s->top_written) {
            s->top_written = top;
            cudaMemcpyAsync(s->d_mbox + XTED_MBOX_TOP, &top, 4, cudaMemcpyHostToDevice, s->cs);
        }
    }
    // 5. keep a launch running while queries are in flight
    bool inflight = false;
    for (const Slot &sl : s->slots) inflight |= sl.busy && sl.gen != 0;
    if (inflight && !s->running && s->stop) {
        // shutting down: a query whose record no launch claimed is not started again
        for (int i = 0; i < s->S; i++) {
            Slot &sl = s->slots[i];
            if (!sl.busy || sl.gen == 0) continue;
            if (((volatile int32_t *)s->h_flags)[i] == sl.gen) continue;  // done: step 1 takes it
            auto it = s->queries.find(sl.ticket);
            if (it != s->queries.end()) it->second.state = XTED_ETIMEOUT;
            release(s, sl);
        }
        s->cv_done.notify_all();
        return true;
    }
    if (inflight && !s->running) {
        // every earlier launch ended with all of its work done: start from empty rings
        cudaStreamSynchronize(s->cs);
        bool ok = cudaMemsetAsync(s->d_rq, 0xff, ((size_t)XTED_RINGS << s->rq_log2) * 8, s->ks) == cudaSuccess &&
                  cudaMemsetAsync(s->d_ctl, 0, (2 * XTED_RINGS + 8) * 4, s->ks) == cudaSuccess &&
                  launch_dp(s->K, s->c->grid, s->ks) == cudaSuccess &&
                  cudaEventRecord(s->kev, s->ks) == cudaSuccess;
        if (!ok) {
            cudaGetLastError();
            s->error = XTED_ECUDA;
            fail_inflight(s, XTED_ECUDA);
            s->cv_done.notify_all();
        } else {
            s->running = true;
            s->launches++;
        }
        progress = true;
    }
    return progress;
}

void worker_main(ServeState *s) {
    cudaSetDevice(s->c->opts.device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        const bool progress = step(s, lk);
        bool inflight = false;
        for (const Slot &sl : s->slots) inflight |= sl.busy;
        if (s->stop && !inflight && s->pending.empty() && !s->running) break;
        if (!progress) s->cv_work.wait_for(lk, std::chrono::microseconds(inflight || s->running ? 50 : 2000));
    }
}

void stop_worker(ServeState *s) {
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->stop = true;
        for (uint64_t t : s->pending) {
            auto it = s->queries.find(t);
            if (it != s->queries.end() && it->second.state == 0) it->second.state = XTED_EINVAL;
        }
        s->pending.clear();
        for (Slot &sl : s->slots)
            if (sl.busy && sl.gen == 0) sl = Slot{};  // planned but never posted
        const int32_t one = 1;
        if (s->cs) cudaMemcpyAsync(s->d_mbox + XTED_MBOX_STOP, &one, 4, cudaMemcpyHostToDevice, s->cs);
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
}

int load(xted_ctx *c, ServeState *s, const xted_tree *tr, int32_t ntrees) {
    s->c = c;
    s->T = ntrees;
    const int T = ntrees, S = s->S, Qm = s->Qmax;
    int64_t N = 0, R = 0, nonempty = 0;
    for (int t = 0; t < T; t++) {
        TreeView tv{tr[t].n, tr[t].labels, tr[t].child_off, tr[t].child_idx};
        const int rc = validate_tree(tv);
        if (rc) return rc;
        N += tr[t].n;
        s->max_tree = std::max(s->max_tree, tr[t].n);
        R += 3 * (int64_t)tr[t].n + 1;
        nonempty += tr[t].n;
    }
    const int64_t Nall = N + (int64_t)S * Qm;
    if (2 * Nall + 2 * (int64_t)(T + S) >= INT32_MAX / 2 || (int64_t)S * T >= INT32_MAX / 2) return XTED_ENOMEM;
    s->Nc_nonempty = nonempty;
    s->sorted_labels.resize((size_t)T);
    s->dense_seq.resize((size_t)T);
    for (int t = 0; t < T; t++) {
        std::vector<int32_t> &v = s->sorted_labels[(size_t)t];
        v.assign(tr[t].labels, tr[t].labels + tr[t].n);
        std::sort(v.begin(), v.end());
        std::vector<int32_t> &d = s->dense_seq[(size_t)t];
        d.resize((size_t)tr[t].n);
        for (int v2 = 0; v2 < tr[t].n; v2++)
            d[(size_t)v2] = s->dense.emplace(tr[t].labels[v2], (int32_t)s->dense.size()).first->second;
    }
    int ntune = 0;
    const XTuneRow *tune = ctx_tune_table(c, &ntune);
    serve_pools_build(s->pools, tr, T, S, Qm, c->opts.run_rows, c->opts.narrow_width,
                      c->opts.half_width == 0 ? XTED_HALF_DEFAULT : c->opts.half_width,
                      c->opts.tuned ? tune : nullptr, c->opts.tuned ? ntune : 0);
    const ServePools &H = s->pools;
    const size_t n2 = H.node.size();
    // device memory
    int rq_log2 = 12;
    while (((int64_t)1 << rq_log2) < 4 * (int64_t)XTED_SERVE_SLOTS * std::max(T, 1)) rq_log2++;
    s->rq_log2 = rq_log2;
    int64_t dt_cap = std::min<int64_t>(kDtCapMax, (int64_t)S * Qm * std::max<int64_t>(nonempty, 1));
    if (c->opts.mem_limit > 0) dt_cap = std::min<int64_t>(dt_cap, c->opts.mem_limit / 8);  // half of the limit
    dt_cap = std::max<int64_t>(dt_cap, 1);
    int rc = XTED_OK;
    rc |= dev_alloc(s, &s->d_node, n2);
    rc |= dev_alloc(s, &s->d_krd, n2);
    rc |= dev_alloc(s, &s->d_cumw, n2);
    rc |= dev_alloc(s, &s->d_runs, n2);
    rc |= dev_alloc(s, &s->d_chunks, n2);
    rc |= dev_alloc(s, &s->d_pairs, (size_t)S * T);
    rc |= dev_alloc(s, &s->d_first, (size_t)S * T);
    rc |= dev_alloc(s, &s->d_entries, (size_t)kEntryCap);
    rc |= dev_alloc(s, &s->d_state, XTED_ESTATE * (size_t)kEntryCap);
    rc |= dev_alloc(s, &s->d_units, (size_t)kUnitCap);
    rc |= dev_alloc(s, &s->d_tasks, (size_t)kTaskCap);
    rc |= dev_alloc(s, &s->d_rq, (size_t)XTED_RINGS << rq_log2);
    rc |= dev_alloc(s, &s->d_ctl, 2 * XTED_RINGS + 8);
    rc |= dev_alloc(s, &s->d_mbox, XTED_MBOX_INTS);
    rc |= dev_alloc(s, &s->d_slot, 3 * XTED_SERVE_SLOTS);
    rc |= dev_alloc(s, &s->d_err, 8);
    rc |= dev_alloc(s, &s->d_dt, (size_t)dt_cap);
    // per-block scratch: far-row stacks, and rows of the wide paths for queries up to Qmax columns
    const int64_t sr = H.stack_rows;
    int64_t per = sr * (XTED_WARPS * XTED_NARROW_MAX);
    per = std::max<int64_t>(per, sr * std::min(Qm, XTED_WIDE_REG_MAX));
    if (Qm > XTED_WIDE_REG_MAX) per = std::max<int64_t>(per, xted_wide_big_scratch(Qm, sr));
    per = (per + 63) / 64 * 64;
    rc |= dev_alloc(s, &s->d_scratch, (size_t)per * (size_t)c->grid);
    if (rc) return XTED_ENOMEM;
    if (cudaHostAlloc((void **)&s->h_results, sizeof(int32_t) * std::max<size_t>((size_t)S * T, 1),
                      cudaHostAllocMapped) != cudaSuccess ||
        cudaHostAlloc((void **)&s->h_flags, sizeof(int32_t) * XTED_SERVE_SLOTS, cudaHostAllocMapped) != cudaSuccess) {
        cudaGetLastError();
        return XTED_ENOMEM;
    }
    std::memset(s->h_flags, 0, sizeof(int32_t) * XTED_SERVE_SLOTS);
    int32_t *d_results = nullptr, *d_flags = nullptr;
    if (cudaHostGetDevicePointer((void **)&d_results, s->h_results, 0) != cudaSuccess ||
        cudaHostGetDevicePointer((void **)&d_flags, s->h_flags, 0) != cudaSuccess ||
        cudaStreamCreateWithFlags(&s->ks, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&s->cs, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->kev, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        return XTED_ECUDA;
    }
    const size_t ncorp = 2 * (size_t)N;
    if (upload(s->d_node, H.node.data(), ncorp * sizeof(int2), s->cs) ||
        upload(s->d_krd, H.krd.data(), ncorp * 4, s->cs) || upload(s->d_cumw, H.cumw.data(), ncorp * 4, s->cs) ||
        upload(s->d_runs, H.runs.data(), ncorp * sizeof(XRun), s->cs) ||
        upload(s->d_chunks, H.chunks.data(), ncorp * sizeof(XChunk), s->cs) ||
        cudaMemsetAsync(s->d_mbox, 0, XTED_MBOX_INTS * 4, s->cs) != cudaSuccess ||
        cudaMemsetAsync(s->d_slot, 0, 3 * XTED_SERVE_SLOTS * 4, s->cs) != cudaSuccess ||
        cudaMemsetAsync(s->d_err, 0, 8 * 4, s->cs) != cudaSuccess || cudaStreamSynchronize(s->cs) != cudaSuccess) {
        cudaGetLastError();
        return XTED_ECUDA;
    }
    s->dt_ext.reset(dt_cap);
    s->u_ext.reset(kUnitCap);
    s->t_ext.reset(kTaskCap);
    s->e_ext.reset(kEntryCap, true);  // entry ids: reused as late as possible
    XKernelParams &K = s->K;
    std::memset(&K, 0, sizeof(K));
    K.rowinfo = s->d_node;
    K.krd = s->d_krd;
    K.cumw = s->d_cumw;
    K.runs = s->d_runs;
    K.chunks = s->d_chunks;
    K.pairs = s->d_pairs;
    K.units = s->d_units;
    K.tasks = s->d_tasks;
    K.entries = s->d_entries;
    K.first = s->d_first;
    K.dt = s->d_dt;
    K.scratch = s->d_scratch;
    K.scratch_per_cta = per;
    K.stack_rows = H.stack_rows;
    K.ntasks = INT32_MAX;
    K.nentries = (int32_t)kEntryCap;
    K.npairs = S * T;
    K.entry_state = s->d_state;
    K.rq = s->d_rq;
    K.rq_log2 = rq_log2;
    K.rq_ctl = s->d_ctl;
    K.done_total = s->d_ctl + 2 * XTED_RINGS;
    K.error = s->d_err;
    K.error_info = s->d_err + 1;
    K.timeout_ns = (uint64_t)(c->opts.wait_timeout_s * 1e9);
    K.trace = nullptr;
    K.serve = 1;
    K.serve_pairs = T;
    K.idle_exit_ns = 2000000;  // 2 ms
    K.mbox = s->d_mbox;
    K.slot_done = s->d_slot;
    K.slot_need = s->d_slot + XTED_SERVE_SLOTS;
    K.slot_gen = s->d_slot + 2 * XTED_SERVE_SLOTS;
    K.results = d_results;
    K.flags = d_flags;
    K.hold_pair = -1;
    // the kernel's row tree is the corpus tree and its column tree the query:
    // TED(query, corpus tree) deletes query nodes and inserts corpus nodes,
    // so the kernel's row deletions cost cost_ins and its column insertions cost_del
    K.c_del = c->opts.cost_ins;
    K.c_ins = c->opts.cost_del;
    K.c_ren = c->opts.cost_ren;
    s->worker = std::thread(worker_main, s);
    return XTED_OK;
}

}  // namespace

std::mutex &serve_mutex(xted_ctx *c) { return c->serve->mu; }

void serve_shutdown(xted_ctx *c) {
    ServeState *s = c->serve;
    if (!s) return;
    stop_worker(s);
    if (s->ks) cudaStreamSynchronize(s->ks);
    if (s->cs) cudaStreamSynchronize(s->cs);
    free_all(s);
    delete s;
    c->serve = nullptr;
}

}  // namespace xted

using namespace xted;

extern "C" {

int xted_corpus_load(xted_ctx *c, const xted_tree *trees, int32_t ntrees) {
    if (!c || ntrees < 1 || !trees) return XTED_EINVAL;
    if (cudaSetDevice(c->opts.device) != cudaSuccess) return XTED_ECUDA;
    serve_shutdown(c);
    ServeState *s = new (std::nothrow) ServeState();
    if (!s) return XTED_ENOMEM;
    const int rc = load(c, s, trees, ntrees);
    if (rc) {
        if (s->worker.joinable()) stop_worker(s);
        free_all(s);
        delete s;
        return rc;
    }
    c->serve = s;
    return XTED_OK;
}

int xted_query_submit(xted_ctx *c, const xted_tree *q, int32_t k, uint64_t *ticket) {
    if (!c || !q || !ticket || k < 1) return XTED_EINVAL;
    ServeState *s = c->serve;
    if (!s) return XTED_EINVAL;
    if (q->n > s->Qmax) return XTED_EINVAL;
    // every pair must fit the row scan's key range: the corpus tree is the
    // row tree (deleted at cost_ins), the query the column tree (cost_del)
    if ((int64_t)c->opts.cost_ins * s->max_tree + (int64_t)c->opts.cost_del * q->n >= XTED_COST_BOUND)
        return XTED_EINVAL;
    const int rc = validate_tree(TreeView{q->n, q->labels, q->child_off, q->child_idx});
    if (rc) return rc;
    Query Q;
    Q.n = q->n;
    Q.k = k;
    Q.lab.assign(q->labels, q->labels + q->n);
    Q.off.assign((size_t)q->n + 1, 0);
    if (q->n > 0) Q.off.assign(q->child_off, q->child_off + q->n + 1);
    if (q->n > 1) Q.idx.assign(q->child_idx, q->child_idx + q->n - 1);
    Q.t_submit = now_ms();
    {
        std::lock_guard<std::mutex> g(s->mu);
        if (s->stop) return XTED_EINVAL;
        if ((int)s->pending.size() >= kMaxPending) return XTED_EAGAIN;
        const uint64_t t = s->next_ticket++;
        s->queries.emplace(t, std::move(Q));
        s->pending.push_back(t);
        *ticket = t;
    }
    s->cv_work.notify_all();
    return XTED_OK;
}

int xted_query_poll_timed(xted_ctx *c, uint64_t ticket, int32_t *ids, int32_t *dists, int32_t *done,
                          double *queue_ms, double *total_ms) {
    if (!c || !done) return XTED_EINVAL;
    ServeState *s = c->serve;
    if (!s) return XTED_EINVAL;
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->queries.find(ticket);
    if (it == s->queries.end()) return XTED_ENOTFOUND;
    Query &q = it->second;
    *done = 0;
    if (q.state < 0) {
        const int code = q.state;
        s->queries.erase(it);
        return code;
    }
    if (q.state != 2) return XTED_OK;
    if (ids) std::memcpy(ids, q.ids.data(), 4 * q.ids.size());
    if (dists) std::memcpy(dists, q.dists.data(), 4 * q.dists.size());
    if (queue_ms) *queue_ms = q.t_admit > 0 ? q.t_admit - q.t_submit : 0.0;
    if (total_ms) *total_ms = q.t_done - q.t_submit;
    *done = 1;
    s->queries.erase(it);
    return XTED_OK;
}

int xted_query_poll(xted_ctx *c, uint64_t ticket, int32_t *ids, int32_t *dists, int32_t *done) {
    return xted_query_poll_timed(c, ticket, ids, dists, done, nullptr, nullptr);
}

int xted_serve_drain(xted_ctx *c) {
    if (!c) return XTED_EINVAL;
    ServeState *s = c->serve;
    if (!s) return XTED_EINVAL;
    std::unique_lock<std::mutex> lk(s->mu);
    s->cv_work.notify_all();
    // bounded: XTED_ETIMEOUT once no query has finished, failed or been
    // admitted for 4 x wait_timeout_s (at least 30 s)
    const double limit_ms = 1e3 * std::max(30.0, 4.0 * s->c->opts.wait_timeout_s);
    int64_t mark = -1;
    double since = now_ms();
    for (;;) {
        int64_t busy = (int64_t)s->pending.size();
        for (const Slot &sl : s->slots) busy += sl.busy;
        if (busy == 0) break;
        const int64_t m = s->served + s->pairs_served + (int64_t)s->pending.size() + 1000003 * busy;
        if (m != mark) {
            mark = m;
            since = now_ms();
        } else if (now_ms() - since > limit_ms) {
            return XTED_ETIMEOUT;
        }
        s->cv_done.wait_for(lk, std::chrono::milliseconds(5));
    }
    const int e = s->error;
    s->error = 0;
    return e;
}

int xted_serve_stats(xted_ctx *c, int64_t *out, int32_t n) {
    if (!c || !out || n < 0) return XTED_EINVAL;
    ServeState *s = c->serve;
    if (!s) return XTED_EINVAL;
    std::lock_guard<std::mutex> g(s->mu);
    const int64_t v[8] = {s->launches,     s->served,        s->pairs_served, s->cells_served,
                          s->pairs_pruned, s->second_rounds, s->bound_us,     s->plan_us};
    for (int k = 0; k < n && k < 8; k++) out[k] = v[k];
    return XTED_OK;
}

int xted_serve_options(xted_ctx *c, int32_t prune, int32_t first_round) {
    if (!c || first_round < 0) return XTED_EINVAL;
    ServeState *s = c->serve;
    if (!s) return XTED_EINVAL;
    std::lock_guard<std::mutex> g(s->mu);
    if (prune < 0 || prune > 2) return XTED_EINVAL;
    s->prune = prune;
    s->first_round = first_round > 0 ? first_round : 32;
    return XTED_OK;
}

}  // extern "C"
