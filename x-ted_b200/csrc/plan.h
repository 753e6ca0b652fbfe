// plan.h -- host-side checks of caller trees (planning itself runs on the device, prep.cu).
#pragma once

#include <algorithm>
#include <cstdint>
#include <system_error>
#include <thread>
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

// Runs f(lo, hi) over [0, n) split across host threads, at least `grain`
// items per thread (inline when that leaves one thread, or when threads
// cannot be started).
template <class F>
void parallel_for(int64_t n, int64_t grain, F &&f) {
    unsigned hw = std::thread::hardware_concurrency();
    const int64_t nt = std::min<int64_t>(std::max(1u, std::min(hw, 32u)), (n + grain - 1) / std::max<int64_t>(grain, 1));
    if (nt <= 1) {
        f((int64_t)0, n);
        return;
    }
    const int64_t per = (n + nt - 1) / nt;
    std::vector<std::thread> th;
    int64_t done_inline = 0;
    for (int64_t k = 1; k < nt; k++) {
        const int64_t lo = k * per, hi = std::min(n, lo + per);
        if (lo >= hi) break;
        try {
            th.emplace_back(f, lo, hi);
        } catch (const std::system_error &) {
            done_inline = lo;  // run the rest here
            break;
        }
    }
    f((int64_t)0, std::min(n, per));
    if (done_inline > 0) f(done_inline, n);
    for (std::thread &t : th) t.join();
}

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
