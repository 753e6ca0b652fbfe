// hpp_check.cpp -- TEST INFRASTRUCTURE: compiles include/xted.hpp and checks
// its host-side conversion (no GPU needed).
//
// xted_cpp::to_csr turns the reference's input (vector<string> labels and a
// preorder vector<vector<int>> adjacency, X-TED_CPU/TED.cpp:177) into the C
// ABI's CSR tree. Checked here: labels interned to ids shared across the two
// trees of a pair (equal strings, equal ids), offsets and children as the
// adjacency lists them, the tree accepted by xted_validate, the single-node
// and label-count-mismatch cases, and the cell counts of xted_pair_cells for
// a hand-computed pair. Prints "ok" and exits 0 on success.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "xted.hpp"

#define CHECK(c)                                                   \
    do {                                                           \
        if (!(c)) {                                                \
            std::printf("FAILED %s:%d: %s\n", __FILE__, __LINE__, #c); \
            std::exit(1);                                          \
        }                                                          \
    } while (0)

int main() {
    std::unordered_map<std::string, int32_t> ids;
    // a(b(d) c) and x(a b): preorder 0 1 2 3
    std::vector<std::string> l1 = {"a", "b", "d", "c"}, l2 = {"x", "a", "b"};
    std::vector<std::vector<int>> a1 = {{1, 3}, {2}, {}, {}}, a2 = {{1, 2}, {}, {}};
    xted_cpp::TreeCSR t1 = xted_cpp::to_csr(l1, a1, ids), t2 = xted_cpp::to_csr(l2, a2, ids);
    CHECK((t1.labels == std::vector<int32_t>{0, 1, 2, 3}));
    CHECK((t2.labels == std::vector<int32_t>{4, 0, 1}));  // "a", "b" keep their ids across trees
    CHECK((t1.off == std::vector<int32_t>{0, 2, 3, 3, 3}));
    CHECK((t1.idx == std::vector<int32_t>{1, 3, 2}));
    CHECK((t2.off == std::vector<int32_t>{0, 2, 2, 2}));
    xted_tree v1 = t1.view(), v2 = t2.view();
    CHECK(v1.n == 4 && v2.n == 3);
    CHECK(xted_validate(&v1) == XTED_OK && xted_validate(&v2) == XTED_OK);
    // keyroots (right path): t1 {0, 1}, sizes 4 + 2 = 6; t2 {0, 1}, 3 + 1 = 4
    int64_t cells[3] = {0, 0, 0};
    CHECK(xted_pair_cells(&v1, &v2, XTED_ORIENT_RIGHT, cells) == XTED_OK);
    CHECK(cells[0] == 24 && cells[2] == 24);
    // one node: no children, a placeholder child array that is never read
    std::vector<std::string> l3 = {"q"};
    std::vector<std::vector<int>> a3 = {{}};
    xted_cpp::TreeCSR t3 = xted_cpp::to_csr(l3, a3, ids);
    xted_tree v3 = t3.view();
    CHECK(v3.n == 1 && t3.off == (std::vector<int32_t>{0, 0}) && xted_validate(&v3) == XTED_OK);
    // a child listed before its parent's earlier subtree ends is not preorder
    std::vector<std::vector<int>> bad = {{2, 1}, {}, {}};
    xted_cpp::TreeCSR t4 = xted_cpp::to_csr(l2, bad, ids);
    xted_tree v4 = t4.view();
    CHECK(xted_validate(&v4) == XTED_EINVAL);
    bool threw = false;
    try {
        std::vector<std::string> short_labels = {"a"};
        xted_cpp::to_csr(short_labels, a1, ids);
    } catch (const std::runtime_error &) {
        threw = true;
    }
    CHECK(threw);
    // empty trees follow standard_ted's rules without touching a device
    std::vector<std::string> e;
    std::vector<std::vector<int>> ea;
    CHECK(xted_cpp::standard_ted(e, ea, l1, a1, 8, 1) == 4);
    CHECK(xted_cpp::standard_ted(l2, a2, e, ea, 8, 1) == 3);
    std::printf("ok\n");
    return 0;
}
