// plan.h -- host-side checks of caller trees (planning itself runs on the device, prep.cu).
#pragma once

#include <cstdint>
#include <vector>

#include "xted_internal.h"

namespace xted {

struct int4h { int32_t x, y, z, w; };
struct int2h { int32_t x, y; };

// A tree in preorder CSR as the C ABI passes it (not owned).
struct TreeView {
    int32_t n = 0;
    const int32_t *labels = nullptr, *off = nullptr, *idx = nullptr;
};

// Sum of keyroot subtree sizes for right-path (S[0]) and left-path (S[1])
// keyroots, straight from the CSR (O(n), no tree is built).
void keyroot_sums(const TreeView &t, int64_t S[2]);

// Validates a preorder CSR tree. Returns 0 or XTED_EINVAL.
int validate_tree(const TreeView &t);

// Identity of a caller's tree (its pointers and size): the same tree passed in
// several pairs is preprocessed once.
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

}  // namespace xted
