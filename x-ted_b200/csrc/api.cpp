// api.cpp -- the C ABI (include/xted.h): context, device memory, launches.
//
// xted_distance / xted_distance_batch replace the reference's
// standard_ted (X-TED_CPU/TED.cpp:177-190; X-TED_GPU/TED.cu:116-128): the
// planner (plan.cpp) lays out every keyroot table of every pair as device
// tasks, one cooperative launch of the persistent DP kernel (kernels.cu)
// drains them, and a gather kernel reads Dtree[0][0] of each pair
// (X-TED_CPU/TED.cpp:188). Errors are returned, never printed or exited on
// (the reference prints CUDA errors and continues, X-TED_GPU/utils/cuda_utils.h:35-41,
// or exits, X-TED_GPU/help.h:6-14).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/xted.h"
#include "ctx.h"
#include "plan.h"
#include "tune_table.h"

namespace xted {
int dp_occupancy(int *blocks_per_sm);
cudaError_t launch_dp(const XKernelParams &P, int grid, cudaStream_t s);
cudaError_t launch_rq_init(const XKernelParams &P, cudaStream_t s);
cudaError_t launch_gather(const XPair *pairs, const int32_t *trivial, const int32_t *dt, int npairs,
                          int32_t *out, int c_del, int c_ins, cudaStream_t s);
}  // namespace xted

using namespace xted;

namespace {

inline double now_ms() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

}  // namespace

namespace xted {

bool costs_fit(const xted_opts &o, int64_t m, int64_t n) {
    return (int64_t)o.cost_del * m + (int64_t)o.cost_ins * n < XTED_COST_BOUND;
}

int ctx_dev_reserve(xted_ctx *c, DevBuf &b, size_t bytes) {
    if (b.cap >= bytes) return XTED_OK;
    size_t want = align_up(std::max(bytes, b.cap + b.cap / 2), (size_t)2 << 20);
    if (c->opts.mem_limit > 0) {
        const int64_t limit = c->opts.mem_limit;
        if (c->held - (int64_t)b.cap + (int64_t)want > limit) want = align_up(bytes, 256);
        if (c->held - (int64_t)b.cap + (int64_t)want > limit) return XTED_ENOMEM;
    }
    if (b.p) {
        cudaFree(b.p);
        c->held -= (int64_t)b.cap;
        b.p = nullptr;
        b.cap = 0;
    }
    void *p = nullptr;
    if (cudaMalloc(&p, want) != cudaSuccess) {
        cudaGetLastError();
        return XTED_ENOMEM;
    }
    b.p = p;
    b.cap = want;
    c->held += (int64_t)want;
    return XTED_OK;
}

int ctx_host_reserve(HostBuf &b, size_t bytes) {
    if (b.cap >= bytes) return XTED_OK;
    size_t want = align_up(std::max(bytes, b.cap + b.cap / 2), (size_t)1 << 20);
    if (b.p) cudaFreeHost(b.p);
    b.p = nullptr;
    b.cap = 0;
    if (cudaHostAlloc(&b.p, want, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        b.p = nullptr;
        return XTED_ENOMEM;
    }
    b.cap = want;
    return XTED_OK;
}

// Plans a batch on the device (prep.cu) and sizes every buffer the DP launch
// needs; the kernel parameters stay in the context so the batch can be run
// repeatedly from device-resident inputs.
int ctx_prepare(xted_ctx *c, const xted_tree *a, const xted_tree *b, int32_t npairs) {
    c->prepared = false;
    ctx_drop_graph(c);  // the graph holds the previous plan's buffers and sizes
    for (int32_t p = 0; p < npairs; p++)
        if (!costs_fit(c->opts, a[p].n, b[p].n)) return XTED_EINVAL;
    XKernelParams &K = c->kp;
    int rc = dev_plan(c, a, b, npairs, K);
    if (rc) return rc;
    K.c_del = c->opts.cost_del;
    K.c_ins = c->opts.cost_ins;
    K.c_ren = c->opts.cost_ren;
    rc = ctx_dev_reserve(c, c->dt, (size_t)std::max<int64_t>(c->plan_dt_elems, 1) * sizeof(int32_t));
    if (rc) return rc;
    const int64_t stack_rows = c->plan_stack_rows, max_wide = c->plan_max_wide;
    // per-block scratch: far-row stacks (+ rows of the generic wide path)
    int64_t per = stack_rows * (XTED_WARPS * XTED_NARROW_MAX);
    if (max_wide > 0 && max_wide <= XTED_WIDE_REG_MAX) per = std::max<int64_t>(per, stack_rows * max_wide);
    if (max_wide > XTED_WIDE_REG_MAX) per = std::max<int64_t>(per, xted_wide_big_scratch(max_wide, stack_rows));
    per = (int64_t)align_up((size_t)per, 64);
    rc = ctx_dev_reserve(c, c->scratch, (size_t)per * (size_t)c->grid * sizeof(int32_t));
    if (rc) return rc;
    // counters: [1] error, [2..5] error info, then out[npairs]
    rc = ctx_dev_reserve(c, c->counters, (8 + 2 * (size_t)npairs) * sizeof(int32_t));
    if (rc) return rc;
    rc = ctx_host_reserve(c->result, ((size_t)npairs + 8) * sizeof(int32_t));
    if (rc) return rc;
    int32_t *cnt = (int32_t *)c->counters.p;
    K.dt = (int32_t *)c->dt.p;
    K.scratch = (int32_t *)c->scratch.p;
    K.scratch_per_cta = per;
    K.stack_rows = (int32_t)stack_rows;
    K.error = cnt + 1;
    K.error_info = cnt + 2;
    K.timeout_ns = (uint64_t)(c->opts.wait_timeout_s * 1e9);
    // Optional per-task trace (XTED_TRACE=<file>): timestamps of every task,
    // written as raw uint64 quadruples after each run.
    const char *tr = std::getenv("XTED_TRACE");
    K.trace = nullptr;
    if (tr && *tr && K.ntasks > 0) {
        rc = ctx_dev_reserve(c, c->trace, (size_t)K.ntasks * 4 * sizeof(unsigned long long));
        if (rc) return rc;
        K.trace = (unsigned long long *)c->trace.p;
    }
    c->npairs = npairs;
    c->prepared = true;
    return XTED_OK;
}

// Runs the prepared plan: counter reset, the persistent DP launch, the
// gather, and the copy of results + error word to pinned memory. Synchronous.
// One step of the prepared plan, enqueued on the context's stream: counter
// reset, the ready queue's level 0, the persistent DP launch, the gather, and
// the copy of results + error word to pinned memory.
static int enqueue_step(xted_ctx *c, bool events) {
    const XKernelParams &K = c->kp;
    const int npairs = c->npairs;
    int32_t *cnt = (int32_t *)c->counters.p;
    int32_t *d_out = cnt + 8 + npairs;
    int32_t *hres = (int32_t *)c->result.p;
    const size_t res_bytes = (size_t)npairs * sizeof(int32_t);
    if (events && cudaEventRecord(c->ev0, c->stream) != cudaSuccess) return XTED_ECUDA;
    // per-run reset of the error words and the ready queue, then level 0 of every pair
    const size_t ne = (size_t)K.nentries;
    if (cudaMemsetAsync(cnt, 0, 8 * sizeof(int32_t), c->stream) != cudaSuccess ||
        (K.ntasks > 0 &&
         (cudaMemsetAsync(K.entry_state, 0, XTED_ESTATE * ne * sizeof(int32_t), c->stream) != cudaSuccess ||
          cudaMemsetAsync(K.rq, 0xff, ((size_t)XTED_RINGS << K.rq_log2) * sizeof(unsigned long long),
                          c->stream) != cudaSuccess ||
          cudaMemsetAsync(K.rq_ctl, 0, (2 * XTED_RINGS + 8) * sizeof(int32_t), c->stream) != cudaSuccess ||
          (K.nstriped > 0 &&
           cudaMemsetAsync(K.sbuf, 0, (size_t)K.sbuf_words * sizeof(unsigned long long), c->stream) != cudaSuccess) ||
          launch_rq_init(K, c->stream) != cudaSuccess)))
        return XTED_ECUDA;
    if (events && cudaEventRecord(c->evk0, c->stream) != cudaSuccess) return XTED_ECUDA;
    if (K.ntasks > 0 && launch_dp(K, c->grid, c->stream) != cudaSuccess) return XTED_ECUDA;
    if (events && cudaEventRecord(c->evk1, c->stream) != cudaSuccess) return XTED_ECUDA;
    if (launch_gather(K.pairs, c->d_trivial, K.dt, npairs, d_out, K.c_del, K.c_ins, c->stream) != cudaSuccess)
        return XTED_ECUDA;
    if ((events && cudaEventRecord(c->ev1, c->stream) != cudaSuccess) ||
        cudaMemcpyAsync(hres, cnt, 8 * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
        (npairs && cudaMemcpyAsync(hres + 8, d_out, res_bytes, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess))
        return XTED_ECUDA;
    return XTED_OK;
}

void ctx_drop_graph(xted_ctx *c) {
    if (c->step_graph) cudaGraphExecDestroy(c->step_graph);
    c->step_graph = nullptr;
    c->runs_prepared = 0;
}

// Captures the step into a graph; false (and no graph is tried again for this
// context) if the runtime refuses any part of it.
static bool capture_step(xted_ctx *c) {
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    const int rc = enqueue_step(c, false);  // events recorded inside a graph cannot be timed
    const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    bool ok = rc == XTED_OK && e == cudaSuccess && g != nullptr &&
              cudaGraphInstantiate(&c->step_graph, g, 0) == cudaSuccess;
    if (g) cudaGraphDestroy(g);
    if (!ok) {
        cudaGetLastError();
        c->step_graph = nullptr;
    }
    return ok;
}

// Runs the prepared plan. Synchronous. With allow_graph, the second and later
// runs of one prepared plan replay a CUDA graph of the step (one launch of
// the whole sequence instead of eleven enqueues).
int ctx_run(xted_ctx *c, int32_t *out, bool allow_graph) {
    if (!c->prepared) return XTED_EINVAL;
    const XKernelParams &K = c->kp;
    const int npairs = c->npairs;
    int32_t *hres = (int32_t *)c->result.p;
    const size_t res_bytes = (size_t)npairs * sizeof(int32_t);
    bool replay = false;
    if (allow_graph && !K.trace && !c->graph_failed && c->runs_prepared >= 1) {
        if (!c->step_graph && !capture_step(c)) c->graph_failed = true;
        replay = c->step_graph != nullptr;
    }
    c->runs_prepared++;
    if (replay) {
        // timed from outside: the DP time of a replay includes the step's
        // small kernels (ready-queue init and gather, a few microseconds)
        if (cudaEventRecord(c->ev0, c->stream) != cudaSuccess || cudaEventRecord(c->evk0, c->stream) != cudaSuccess ||
            cudaGraphLaunch(c->step_graph, c->stream) != cudaSuccess ||
            cudaEventRecord(c->evk1, c->stream) != cudaSuccess || cudaEventRecord(c->ev1, c->stream) != cudaSuccess) {
            cudaGetLastError();
            return XTED_ECUDA;
        }
    } else {
        const int rc = enqueue_step(c, true);
        if (rc) {
            cudaGetLastError();
            return rc;
        }
    }
    c->stats.graph = replay ? 1 : 0;
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) {
        cudaGetLastError();
        return XTED_ECUDA;
    }
    float ms = 0.f, kms = 0.f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    cudaEventElapsedTime(&kms, c->evk0, c->evk1);
    cudaGetLastError();  // a failed timing read must not surface in a later call
    c->stats.device_ms = ms;
    c->stats.dp_ms = kms;
    c->stats.h2d_bytes = c->h2d_bytes;
    c->stats.d2h_bytes = (int64_t)(res_bytes + 8 * sizeof(int32_t));
    c->stats.grid = c->grid;
    std::memcpy(c->err_info, hres + 2, sizeof(c->err_info));
    if (K.trace) {
        std::vector<unsigned long long> tr((size_t)K.ntasks * 4);
        if (cudaMemcpy(tr.data(), K.trace, tr.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost) ==
            cudaSuccess) {
            if (FILE *f = std::fopen(std::getenv("XTED_TRACE"), "wb")) {
                std::fwrite(tr.data(), sizeof(unsigned long long), tr.size(), f);
                std::fclose(f);
            }
            // the plan beside it: tasks (pair, entry, kind, first unit) and entries
            std::vector<XTask> tk((size_t)K.ntasks);
            std::vector<XEntry> en((size_t)K.nentries);
            const std::string base = std::getenv("XTED_TRACE");
            if (cudaMemcpy(tk.data(), K.tasks, tk.size() * sizeof(XTask), cudaMemcpyDeviceToHost) == cudaSuccess &&
                cudaMemcpy(en.data(), K.entries, en.size() * sizeof(XEntry), cudaMemcpyDeviceToHost) == cudaSuccess) {
                if (FILE *f = std::fopen((base + ".tasks").c_str(), "wb")) {
                    std::fwrite(tk.data(), sizeof(XTask), tk.size(), f);
                    std::fclose(f);
                }
                if (FILE *f = std::fopen((base + ".entries").c_str(), "wb")) {
                    std::fwrite(en.data(), sizeof(XEntry), en.size(), f);
                    std::fclose(f);
                }
            }
        }
    }
    if (hres[1] != 0) return hres[1];
    if (npairs) std::memcpy(out, hres + 8, res_bytes);
    return XTED_OK;
}

const XTuneRow *ctx_tune_table(const xted_ctx *c, int *nrows) {
    if (c->ntune > 0) {
        *nrows = c->ntune;
        return c->tune;
    }
    *nrows = kTuneRows;
    return kTuneTable;
}

void fill_stats(xted_ctx *c, double plan_ms) {
    c->stats.pairs = c->npairs;
    c->stats.cells = c->plan_cells;
    c->stats.cells_right = c->plan_cells_right;
    c->stats.tasks = c->kp.ntasks;
    c->stats.units = c->plan_units;
    c->stats.levels_max = c->plan_levels_max;
    c->stats.host_plan_ms = plan_ms;
}

}  // namespace xted

extern "C" {

void xted_opts_default(xted_opts *o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->device = 0;
    o->orientation = XTED_ORIENT_AUTO;
    o->narrow_width = XTED_NARROW_MAX;
    o->run_rows = 64;
    o->ctas_per_sm = 0;
    o->wide_rows = 0;
    o->half_width = 0;
    o->tuned = 1;
    o->wait_timeout_s = 20.0;
    o->mem_limit = 0;
    o->stripe_min_cells = 0;
    o->cost_del = o->cost_ins = o->cost_ren = 1;
}

const char *xted_strerror(int code) {
    switch (code) {
        case XTED_OK: return "ok";
        case XTED_EINVAL: return "invalid argument or malformed tree";
        case XTED_ENOMEM: return "out of memory (device, host or the context's limit)";
        case XTED_ETIMEOUT: return "a bounded device wait timed out";
        case XTED_ECUDA: return "CUDA runtime error";
        case XTED_ENODEV: return "no usable sm_100 CUDA device";
        case XTED_ENOTFOUND: return "unknown ticket";
        case XTED_EAGAIN: return "serving queue full";
        case XTED_ETOOBIG: return "pair does not fit the fixed arena of xted_distance_noalloc";
        default: return "unknown error";
    }
}

int xted_create(xted_ctx **out, const xted_opts *opts) {
    if (!out) return XTED_EINVAL;
    *out = nullptr;
    xted_opts o;
    if (opts) o = *opts;
    else xted_opts_default(&o);
    if (o.narrow_width < 0 || o.narrow_width > XTED_NARROW_MAX || o.run_rows < 1 ||
        o.orientation < 0 || o.orientation > 2 || o.wait_timeout_s <= 0 || o.ctas_per_sm < 0 ||
        o.cost_del < 0 || o.cost_ins < 0 || o.cost_ren < 0 || o.cost_del >= XTED_COST_BOUND ||
        o.cost_ins >= XTED_COST_BOUND || o.cost_ren >= XTED_COST_BOUND)
        return XTED_EINVAL;
    if (o.cost_del == 0 && o.cost_ins == 0 && o.cost_ren == 0) o.cost_del = o.cost_ins = o.cost_ren = 1;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || o.device < 0 || o.device >= ndev) {
        cudaGetLastError();
        return XTED_ENODEV;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, o.device) != cudaSuccess || prop.major != 10) return XTED_ENODEV;
    if (cudaSetDevice(o.device) != cudaSuccess) return XTED_ECUDA;
    xted_ctx *c = new (std::nothrow) xted_ctx();
    if (!c) return XTED_ENOMEM;
    c->opts = o;
    c->sms = prop.multiProcessorCount;
    int occ = 0;
    if (dp_occupancy(&occ) != 0 || occ < 1) {
        delete c;
        return XTED_ECUDA;
    }
    if (o.ctas_per_sm > 0) occ = std::min(occ, o.ctas_per_sm);
    c->grid = occ * c->sms;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess ||
        cudaEventCreate(&c->evk0) != cudaSuccess || cudaEventCreate(&c->evk1) != cudaSuccess) {
        delete c;
        return XTED_ECUDA;
    }
    *out = c;
    return XTED_OK;
}

int xted_destroy(xted_ctx *c) {
    if (!c) return XTED_OK;
    cudaSetDevice(c->opts.device);
    xted::serve_shutdown(c);
    cudaStreamSynchronize(c->stream);
    ctx_drop_graph(c);
    for (DevBuf *b : {&c->meta, &c->levels, &c->work, &c->dt, &c->scratch, &c->counters, &c->trace, &c->smap, &c->sbuf})
        if (b->p) cudaFree(b->p);
    for (HostBuf *b : {&c->stage, &c->result, &c->summary})
        if (b->p) cudaFreeHost(b->p);
    for (cudaEvent_t e : {c->ev0, c->ev1, c->evk0, c->evk1})
        if (e) cudaEventDestroy(e);
    cudaStreamDestroy(c->stream);
    delete c;
    return XTED_OK;
}

int xted_distance_batch(xted_ctx *c, const xted_tree *a, const xted_tree *b, int32_t npairs,
                        int32_t *out) {
    if (!c || npairs < 0 || (npairs > 0 && (!a || !b || !out))) return XTED_EINVAL;
    const double t0 = now_ms();
    if (cudaSetDevice(c->opts.device) != cudaSuccess) return XTED_ECUDA;
    int rc = ctx_prepare(c, a, b, npairs);
    const double t1 = now_ms();
    std::memset(&c->stats, 0, sizeof(c->stats));
    if (rc) return rc;
    const bool hold = c->fault == XTED_FAULT_HOLD_PAIR && npairs > 0;
    if (hold) {  // test hook: pair 0's level 0 is never published
        c->fault = 0;
        c->kp.hold_pair = 0;
    }
    rc = ctx_run(c, out, false);
    c->kp.hold_pair = -1;
    fill_stats(c, t1 - t0);
    c->stats.total_ms = now_ms() - t0;
    return rc;
}

int xted_prepare_batch(xted_ctx *c, const xted_tree *a, const xted_tree *b, int32_t npairs) {
    if (!c || npairs < 0 || (npairs > 0 && (!a || !b))) return XTED_EINVAL;
    if (cudaSetDevice(c->opts.device) != cudaSuccess) return XTED_ECUDA;
    const double t0 = now_ms();
    int rc = ctx_prepare(c, a, b, npairs);
    std::memset(&c->stats, 0, sizeof(c->stats));
    if (rc) return rc;
    c->prep_ms = now_ms() - t0;
    c->stats.host_plan_ms = c->prep_ms;
    return cudaStreamSynchronize(c->stream) == cudaSuccess ? XTED_OK : XTED_ECUDA;
}

int xted_run_prepared(xted_ctx *c, int32_t *out) {
    if (!c || !out) return XTED_EINVAL;
    if (cudaSetDevice(c->opts.device) != cudaSuccess) return XTED_ECUDA;
    const int rc = ctx_run(c, out, true);
    fill_stats(c, c->prep_ms);
    return rc;
}

int xted_distance(xted_ctx *c, const xted_tree *a, const xted_tree *b, int32_t *out) {
    return xted_distance_batch(c, a, b, 1, out);
}

int xted_distance_matrix(xted_ctx *c, const xted_tree *trees, int32_t ntrees, int64_t pair_budget, int32_t *out) {
    if (!c || ntrees < 0 || (ntrees > 0 && (!trees || !out)) || pair_budget < 0) return XTED_EINVAL;
    int64_t budget = pair_budget > 0 ? pair_budget
                                     : (c->opts.mem_limit > 0 ? c->opts.mem_limit / 16 : (int64_t)1 << 30);
    const int64_t max_pairs = (int64_t)1 << 20;
    // TED is symmetric when deleting and inserting cost the same: each
    // unordered pair once, mirrored; else both orders
    const bool sym = c->opts.cost_del == c->opts.cost_ins;
    std::vector<xted_tree> A, B;
    std::vector<int64_t> at;  // i * ntrees + j of each pair in the chunk
    std::vector<int32_t> res;
    auto flush = [&]() -> int {
        if (A.empty()) return XTED_OK;
        res.resize(A.size());
        const int rc = xted_distance_batch(c, A.data(), B.data(), (int32_t)A.size(), res.data());
        if (rc) return rc;
        for (size_t k = 0; k < A.size(); k++) {
            const int64_t i = at[k] / ntrees, j = at[k] % ntrees;
            out[i * ntrees + j] = res[k];
            if (sym) out[j * ntrees + i] = res[k];
        }
        A.clear();
        B.clear();
        at.clear();
        return XTED_OK;
    };
    int64_t cells = 0;
    for (int32_t i = 0; i < ntrees; i++) {
        out[(int64_t)i * ntrees + i] = 0;
        for (int32_t j = sym ? i + 1 : 0; j < ntrees; j++) {
            if (j == i) continue;
            const int64_t c2 = (int64_t)std::max(trees[i].n, 1) * std::max(trees[j].n, 1);
            if (!A.empty() && (cells + c2 > budget || (int64_t)A.size() >= max_pairs)) {
                const int rc = flush();
                if (rc) return rc;
                cells = 0;
            }
            A.push_back(trees[i]);
            B.push_back(trees[j]);
            at.push_back((int64_t)i * ntrees + j);
            cells += c2;
        }
    }
    return flush();
}

int xted_test_fault(xted_ctx *c, int32_t kind) {
    if (!c || kind < 0 || kind > XTED_FAULT_HOLD_PAIR) return XTED_EINVAL;
    if (c->serve) {
        std::lock_guard<std::mutex> g(serve_mutex(c));
        c->fault = kind;
    } else {
        c->fault = kind;
    }
    return XTED_OK;
}

int xted_last_stats(const xted_ctx *c, xted_stats *out) {
    if (!c || !out) return XTED_EINVAL;
    *out = c->stats;
    return XTED_OK;
}

int xted_set_tune_table(xted_ctx *c, const int32_t *rows, int32_t nrows) {
    if (!c || nrows < 0 || nrows > XTED_TUNE_ROWS || (nrows > 0 && !rows)) return XTED_EINVAL;
    for (int k = 0; k < nrows; k++) {
        const int32_t *r = rows + 4 * k;
        if (r[0] <= 0 || (k > 0 && r[0] <= rows[4 * (k - 1)]) || r[1] < 1 || r[2] < 0 || r[2] > XTED_NARROW_MAX ||
            r[3] < -1 || r[3] > XTED_HALF_MAX)
            return XTED_EINVAL;
    }
    for (int k = 0; k < nrows; k++) c->tune[k] = XTuneRow{rows[4 * k], rows[4 * k + 1], rows[4 * k + 2], rows[4 * k + 3]};
    c->ntune = nrows > 0 ? nrows : -1;
    return XTED_OK;
}

int xted_pair_cells(const xted_tree *a, const xted_tree *b, int32_t orientation, int64_t *out3) {
    if (!a || !b || !out3 || orientation < 0 || orientation > 2) return XTED_EINVAL;
    TreeView A{a->n, a->labels, a->child_off, a->child_idx};
    TreeView B{b->n, b->labels, b->child_off, b->child_idx};
    int rc = validate_tree(A);
    if (!rc) rc = validate_tree(B);
    if (rc) return rc;
    int64_t sa[2], sb[2];
    keyroot_sums(A, sa);
    keyroot_sums(B, sb);
    out3[0] = sa[0] * sb[0];
    out3[1] = sa[1] * sb[1];
    out3[2] = orientation == XTED_ORIENT_RIGHT ? out3[0]
              : orientation == XTED_ORIENT_LEFT ? out3[1]
                                                : std::min(out3[0], out3[1]);
    return XTED_OK;
}

int xted_validate(const xted_tree *t) {
    if (!t) return XTED_EINVAL;
    return validate_tree(TreeView{t->n, t->labels, t->child_off, t->child_idx});
}

}  // extern "C"
