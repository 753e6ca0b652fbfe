// plan.h -- host-side planning of keyroot-table work for a batch of pairs.
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

// One tree in one orientation, with everything the kernels need about it.
// Right-path orientation is the tree as given; left-path orientation is the
// mirrored tree (children reversed, renumbered in preorder).
struct OTree {
    int32_t n = 0;
    std::vector<int32_t> label, orl;
    std::vector<uint8_t> leaf, kr;
    std::vector<int32_t> kdep;   // keyroot depth, -1 for non-keyroots
    int32_t D = 0;               // max keyroot depth (= kdep of the root)
    int64_t S = 0;               // sum of keyroot subtree sizes
    int32_t maxka = 0;           // max keyroots on any root path (stack bound)
    std::vector<int32_t> krd;    // keyroots ordered by (depth, preorder)
    std::vector<int32_t> krd_off;  // [D+2]
    std::vector<int4h> cols;     // column lists of every depth, concatenated
    std::vector<int32_t> col_off;  // [D+2]
    std::vector<int32_t> seg_w;    // segment widths in krd order (= subtree sizes)
};

// Builds an oriented tree. mirrored = false: as given (right-path
// keyroots, X-TED_CPU's decomposition); true: children reversed.
void build_otree(const TreeView &t, bool mirrored, OTree &out);

// Sum of keyroot subtree sizes for right-path (S[0]) and left-path (S[1])
// keyroots, straight from the CSR (O(n), no tree is built).
void keyroot_sums(const TreeView &t, int64_t S[2]);

// Validates a preorder CSR tree. Returns 0 or XTED_EINVAL.
int validate_tree(const TreeView &t);

struct PlanOptions {
    int orientation = 0;   // XTED_ORIENT_*
    int narrow_width = XTED_NARROW_MAX;
    int run_rows = 64;
};

// The device-bound plan of one batch. All index fields are global indices
// into the pools below.
struct Plan {
    std::vector<int2h> rowinfo;
    std::vector<int4h> colinfo;
    std::vector<int32_t> krd;
    std::vector<XRun> runs;
    std::vector<XChunk> chunks;
    std::vector<XPair> pairs;
    std::vector<XUnit> units;
    std::vector<XTask> tasks;
    std::vector<int32_t> trivial;   // per pair: -1 = computed on device, else the distance
    int64_t dt_elems = 0;
    int32_t stack_rows = 1;
    int32_t max_wide = 0;           // widest wide chunk
    int64_t cells = 0, cells_right = 0;
    int32_t levels_max = 0;
};

// Plans npairs pairs. Trees that are the same object (same pointers and n)
// are preprocessed once. Returns 0 or an XTED_* error.
int make_plan(const TreeView *a, const TreeView *b, int32_t npairs, const PlanOptions &opt,
              Plan &plan);

}  // namespace xted
