// plan.cpp -- host-side input checks: preorder validation of a caller's tree
// (the reference assumes valid preorder input and never checks it,
// README.md:31-44) and the keyroot-size sums that price each decomposition.
#include "plan.h"

#include <algorithm>
#include <cstring>

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

}  // namespace xted
