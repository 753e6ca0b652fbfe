// serve.cpp -- resident corpus and exact top-k queries (placeholder; filled in next).
#include "ctx.h"

namespace xted {
struct ServeState {};
void serve_shutdown(xted_ctx *c) {
    delete c->serve;
    c->serve = nullptr;
}
}  // namespace xted

extern "C" {
int xted_corpus_load(xted_ctx *, const xted_tree *, int32_t) { return XTED_EINVAL; }
int xted_query_submit(xted_ctx *, const xted_tree *, int32_t, uint64_t *) { return XTED_EINVAL; }
int xted_query_poll(xted_ctx *, uint64_t, int32_t *, int32_t *, int32_t *) { return XTED_EINVAL; }
int xted_serve_drain(xted_ctx *) { return XTED_EINVAL; }
}
