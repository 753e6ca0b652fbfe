// ctx.h -- the library context behind the opaque xted_ctx handle.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>

#include "../../include/xted.h"
#include "plan.h"

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

}  // namespace xted

struct xted_ctx {
    xted_opts opts;
    int sms = 0;
    int grid = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, evk0 = nullptr, evk1 = nullptr;
    xted::DevBuf meta, dt, scratch, counters, trace;
    xted::HostBuf stage, result;
    const int32_t *d_trivial = nullptr;
    int64_t held = 0;  // device bytes held by this context
    xted::Plan plan;
    xted_stats stats{};
    int32_t err_info[4] = {0, 0, 0, 0};
    xted::ServeState *serve = nullptr;  // owned; released by serve_shutdown
    // the prepared plan (xted_prepare_batch / every batch call)
    XKernelParams kp{};
    int32_t npairs = 0;
    int64_t h2d_bytes = 0;
    bool prepared = false;
};

namespace xted {

int ctx_dev_reserve(xted_ctx *c, DevBuf &b, size_t bytes);
int ctx_host_reserve(HostBuf &b, size_t bytes);
int ctx_prepare(xted_ctx *c, const Plan &P);
int ctx_run(xted_ctx *c, int32_t *out);
void serve_shutdown(xted_ctx *c);

}  // namespace xted
