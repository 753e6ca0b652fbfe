// xted.hpp -- header-only C++ wrapper with the reference's exact entry point.
//
//   int standard_ted(vector<string>& x_node, vector<vector<int>>& x_adj,
//                    vector<string>& y_node, vector<vector<int>>& y_adj,
//                    int num_threads, int parallel_version);
// (X-TED_CPU/TED.cpp:177, X-TED_CPU/TED_C++.h:21; X-TED_GPU/TED.cu:116,
// X-TED_GPU/TED_C++.h:28). A caller of the reference switches by including
// this header and linking libxted.so. Label strings are interned to int32 ids
// (exact: the reference only compares them for equality), the adjacency is
// turned into preorder CSR, and the pair runs through xted_distance.
//
// Differences, all deliberate: the label vectors are NOT cleared (the
// reference clears them, X-TED_CPU/TED.cpp:160-161); malformed input or a
// device failure throws std::runtime_error (the reference's behaviour is
// undefined or it exits); num_threads and parallel_version are ignored, as
// X-TED_GPU ignores them (X-TED_GPU/test_TED.cu:50). The wrapper keeps one
// context per thread on device 0 (thread_local), created on first use.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "xted.h"

namespace xted_cpp {

struct TreeCSR {
    std::vector<int32_t> labels, off, idx;
    xted_tree view() const {
        xted_tree t;
        t.labels = labels.data();
        t.child_off = off.data();
        t.child_idx = idx.data();
        t.n = (int32_t)labels.size();
        return t;
    }
};

inline TreeCSR to_csr(const std::vector<std::string> &node, const std::vector<std::vector<int>> &adj,
                      std::unordered_map<std::string, int32_t> &ids) {
    if (node.size() != adj.size()) throw std::runtime_error("xted: label count differs from adjacency size");
    TreeCSR t;
    t.labels.reserve(node.size());
    for (const std::string &s : node) {
        auto it = ids.emplace(s, (int32_t)ids.size()).first;
        t.labels.push_back(it->second);
    }
    t.off.assign(adj.size() + 1, 0);
    for (size_t v = 0; v < adj.size(); v++) {
        t.off[v + 1] = t.off[v] + (int32_t)adj[v].size();
        for (int c : adj[v]) t.idx.push_back(c);
    }
    if (t.idx.empty()) t.idx.push_back(0);
    return t;
}

class Context {
public:
    explicit Context(int device = 0) {
        xted_opts o;
        xted_opts_default(&o);
        o.device = device;
        int rc = xted_create(&ctx_, &o);
        if (rc) throw std::runtime_error(std::string("xted_create: ") + xted_strerror(rc));
    }
    ~Context() { xted_destroy(ctx_); }
    Context(const Context &) = delete;
    Context &operator=(const Context &) = delete;
    xted_ctx *get() const { return ctx_; }

private:
    xted_ctx *ctx_ = nullptr;
};

inline Context &thread_context() {
    thread_local Context ctx(0);
    return ctx;
}

inline int standard_ted(std::vector<std::string> &x_node, std::vector<std::vector<int>> &x_adj,
                        std::vector<std::string> &y_node, std::vector<std::vector<int>> &y_adj,
                        int num_threads, int parallel_version) {
    (void)num_threads;
    (void)parallel_version;
    const int m = (int)x_adj.size(), n = (int)y_adj.size();
    if (m == 0) return n;  // X-TED_CPU/TED.cpp:181-183
    if (n == 0) return m;  // X-TED_CPU/TED.cpp:184-186
    std::unordered_map<std::string, int32_t> ids;
    TreeCSR a = to_csr(x_node, x_adj, ids), b = to_csr(y_node, y_adj, ids);
    xted_tree ta = a.view(), tb = b.view();
    int32_t d = 0;
    int rc = xted_distance(thread_context().get(), &ta, &tb, &d);
    if (rc) throw std::runtime_error(std::string("xted_distance: ") + xted_strerror(rc));
    return d;
}

}  // namespace xted_cpp
