// ctx.h -- the library context behind the opaque xted_ctx handle.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "../../include/xted.h"
#include "plan.h"
#include "plan_core.h"

namespace xted {

struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
};

struct HostBuf {
    void *p = nullptr;
    size_t cap = 0;
};

struct ServeState;  // serve.cpp
struct DTree;       // plan_core.h

}  // namespace xted

struct xted_ctx {
    xted_opts opts;
    int sms = 0;
    int grid = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, evk0 = nullptr, evk1 = nullptr;
    xted::DevBuf meta, levels, work, dt, scratch, counters, trace, smap, sbuf;
    xted::HostBuf stage, result, summary;
    const int32_t *d_trivial = nullptr;
    int64_t held = 0;  // device bytes held by this context
    xted_stats stats{};
    int32_t err_info[4] = {0, 0, 0, 0};
    int32_t fault = 0;  // armed test fault (xted_test_fault), taken by the next batch or posted query
    // size-bucket granularity set by xted_set_tune_table (ntune < 0: the compiled table)
    XTuneRow tune[XTED_TUNE_ROWS] = {};
    int32_t ntune = -1;
    xted::ServeState *serve = nullptr;  // owned; released by serve_shutdown
    // device planning: host-side bookkeeping of the current batch
    std::unordered_map<xted::TreeKey, int, xted::TreeKeyHash> tree_ids;
    std::vector<xted::TreeView> uniq;
    std::vector<int32_t> pair_trees;
    std::vector<xted::DTree> htrees;
    int64_t plan_dt_elems = 0, plan_cells = 0, plan_cells_right = 0, plan_units = 0;
    int32_t plan_stack_rows = 1, plan_max_wide = 0, plan_levels_max = 0;
    // the prepared plan (xted_prepare_batch / every batch call)
    XKernelParams kp{};
    int32_t npairs = 0;
    int64_t h2d_bytes = 0;
    double prep_ms = 0;
    bool prepared = false;
    // the prepared step captured as a CUDA graph (from its second run on)
    cudaGraphExec_t step_graph = nullptr;
    int32_t runs_prepared = 0;
    bool graph_failed = false;
};

namespace xted {

int ctx_dev_reserve(xted_ctx *c, DevBuf &b, size_t bytes);
// A pair of m and n nodes fits the row scan's key range under the context's costs.
bool costs_fit(const xted_opts &o, int64_t m, int64_t n);
int ctx_host_reserve(HostBuf &b, size_t bytes);
int ctx_prepare(xted_ctx *c, const xted_tree *a, const xted_tree *b, int32_t npairs);
int dev_plan(xted_ctx *c, const xted_tree *a, const xted_tree *b, int32_t npairs, XKernelParams &K);
int ctx_run(xted_ctx *c, int32_t *out, bool allow_graph);
void ctx_drop_graph(xted_ctx *c);
void fill_stats(xted_ctx *c, double plan_ms);
// The size-bucket granularity table the context plans with: the one set by
// xted_set_tune_table, else the autotuned table compiled into the library.
const XTuneRow *ctx_tune_table(const xted_ctx *c, int *nrows);
void serve_shutdown(xted_ctx *c);
std::mutex &serve_mutex(xted_ctx *c);  // the serving state's lock (c->serve must be set)

}  // namespace xted
