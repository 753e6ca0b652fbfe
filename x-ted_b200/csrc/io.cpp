// io.cpp -- dataset text formats, parsed at C speed for large corpora.
//
// * Adjacency lines of the reference's dataset files, "[[1, 2], [], ...]":
//   one list per node in preorder, children in order. The reference splits
//   the line at '[' ... ']' groups and each group at ',' with spaces ignored
//   (X-TED_CPU/dataset_preprocess.cpp:7-66); this parser reads the same
//   grammar in one pass and returns CSR.
// * Bracket notation, "{a{b}{c{d}}}": a node is '{' label children '}', its
//   children in order; the reference ships one file of it
//   (Sampled_Dataset_Extra_Large_Trees/synthetic/*/synthetic_tree_*.txt) and
//   reads it nowhere. Labels may contain '\{', '\}' and '\\' escapes.
// Both return the tree in preorder CSR; neither validates beyond the grammar
// (xted_validate checks the tree).
#include <cstdint>
#include <vector>

#include "../../include/xted.h"

extern "C" {

int xted_parse_adjacency(const char *line, int64_t len, int32_t cap_nodes, int32_t cap_children, int32_t *child_off,
                         int32_t *child_idx, int32_t *n_out, int32_t *nchildren_out) {
    if (!line || len < 0 || !child_off || !n_out || !nchildren_out || cap_nodes < 0 || cap_children < 0)
        return XTED_EINVAL;
    int64_t i = 0;
    while (i < len && line[i] != '[') i++;
    if (i == len) return XTED_EINVAL;
    i++;  // the outer '['
    int32_t n = 0, e = 0;
    child_off[0] = 0;
    for (;;) {
        while (i < len && (line[i] == ' ' || line[i] == ',' || line[i] == '\r')) i++;
        if (i >= len) return XTED_EINVAL;
        if (line[i] == ']') break;  // the outer ']'
        if (line[i] != '[') return XTED_EINVAL;
        i++;
        if (n >= cap_nodes) return XTED_ENOMEM;
        bool have = false;
        int64_t v = 0;
        for (;; i++) {
            if (i >= len) return XTED_EINVAL;
            const char ch = line[i];
            if (ch >= '0' && ch <= '9') {
                v = v * 10 + (ch - '0');
                if (v > XTED_MAX_NODES) return XTED_EINVAL;
                have = true;
            } else if (ch == ',' || ch == ']') {
                if (have) {
                    if (e >= cap_children || !child_idx) return XTED_ENOMEM;
                    child_idx[e++] = (int32_t)v;
                } else if (ch == ',') {
                    return XTED_EINVAL;
                }
                have = false;
                v = 0;
                if (ch == ']') {
                    i++;
                    break;
                }
            } else if (ch != ' ') {
                return XTED_EINVAL;
            }
        }
        n++;
        child_off[n] = e;
    }
    *n_out = n;
    *nchildren_out = e;
    return XTED_OK;
}

int xted_parse_bracket(const char *s, int64_t len, int32_t cap_nodes, int32_t *child_off, int32_t *child_idx,
                       int64_t *label_at, int32_t *label_len, int32_t *n_out, int64_t *end_out) {
    if (!s || len < 0 || !child_off || !label_at || !label_len || !n_out || cap_nodes < 0) return XTED_EINVAL;
    // pass 1: parent of every node in preorder, label spans
    std::vector<int32_t> parent, stack;
    int64_t i = 0;
    while (i < len && s[i] != '{') i++;
    if (i == len) return XTED_EINVAL;
    int32_t n = 0;
    for (;;) {
        if (i < len && s[i] == '{') {
            if (n >= cap_nodes) return XTED_ENOMEM;
            parent.push_back(stack.empty() ? -1 : stack.back());
            stack.push_back(n);
            i++;
            label_at[n] = i;
            while (i < len && s[i] != '{' && s[i] != '}') i += (s[i] == '\\' && i + 1 < len) ? 2 : 1;
            label_len[n] = (int32_t)(i - label_at[n]);
            n++;
        } else if (i < len && s[i] == '}') {
            stack.pop_back();
            i++;
            if (stack.empty()) break;
            while (i < len && (s[i] == ' ' || s[i] == '\n' || s[i] == '\r' || s[i] == '\t')) i++;
        } else {
            return XTED_EINVAL;  // unbalanced or stray text
        }
    }
    // pass 2: children lists (a node's children follow it in preorder, in order)
    std::vector<int32_t> cnt((size_t)n + 1, 0);
    for (int32_t v = 1; v < n; v++) cnt[(size_t)parent[(size_t)v]]++;
    child_off[0] = 0;
    for (int32_t v = 0; v < n; v++) child_off[v + 1] = child_off[v] + cnt[(size_t)v];
    if (n > 1 && !child_idx) return XTED_EINVAL;
    std::vector<int32_t> fill(child_off, child_off + n);
    for (int32_t v = 1; v < n; v++) child_idx[fill[(size_t)parent[(size_t)v]]++] = v;
    *n_out = n;
    if (end_out) *end_out = i;
    return XTED_OK;
}

}  // extern "C"
