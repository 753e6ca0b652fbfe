// dropin_standard_ted.cpp -- TEST INFRASTRUCTURE: the reference's own caller
// on this library.
//
// The reference's harness (X-TED_CPU/main.cpp, X-TED_CPU/TED_test.cpp and its
// parsers X-TED_CPU/dataset_preprocess.cpp) is compiled unmodified, where it
// lies, and linked against this file instead of the reference's TED.cpp and
// parallel_computing.cpp. This file defines the one function the harness
// calls, the global
//   int standard_ted(vector<string>&, vector<vector<int>>&,
//                    vector<string>&, vector<vector<int>>&, int, int)
// declared by the reference header X-TED_CPU/TED_C++.h:21 (included here, so
// the signature is checked against the reference's own declaration) and
// called at X-TED_CPU/TED_test.cpp:43. It forwards to xted_cpp::standard_ted
// of include/xted.hpp, which is what a C++ caller of the reference switches
// to. Built by tests/cpp/Makefile (target `dropin`).
#include "TED_C++.h"

#include "xted.hpp"

int standard_ted(vector<string> &x_node, vector<vector<int>> &x_adj, vector<string> &y_node,
                 vector<vector<int>> &y_adj, int num_threads, int parallel_version) {
    return xted_cpp::standard_ted(x_node, x_adj, y_node, y_adj, num_threads, parallel_version);
}
