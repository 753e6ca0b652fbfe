// ref_harness.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A C-ABI shim linked together with the reference X-TED_CPU sources
// (TED.cpp, parallel_computing.cpp, dataset_preprocess.cpp, compiled where
// they lie by oracle/Makefile into oracle/_ref/libxted_ref.so). It calls the
// reference's own entry point
//   int standard_ted(vector<string>&, vector<vector<int>>&,
//                    vector<string>&, vector<vector<int>>&, int, int)
// (X-TED_CPU/TED.cpp:177) once per pair, so goldens and the CPU baseline come
// from the unmodified reference code path rather than a restatement.
// The reference prints "Total Time for Parallel Computing = X ms" to cout
// (X-TED_CPU/parallel_computing.cpp:184); the shim captures it and returns X.
#include "TED_C++.h"

#include <cstdint>
#include <cstdlib>
#include <sstream>

namespace {

vector<vector<int>> csr_to_adj(int n, const int32_t *off, const int32_t *idx) {
    vector<vector<int>> adj((size_t)n);
    for (int v = 0; v < n; v++)
        for (int32_t e = off[v]; e < off[v + 1]; e++) adj[(size_t)v].push_back(idx[e]);
    return adj;
}

double parse_total_ms(const std::string &s) {
    const std::string key = "Total Time for Parallel Computing = ";
    size_t p = s.rfind(key);
    if (p == std::string::npos) return -1.0;
    return std::atof(s.c_str() + p + key.size());
}

}  // namespace

extern "C" {

// Labels given as C strings (exactly what the reference reads from its files).
int xr_standard_ted_str(int m, const char *const *la, const int32_t *aoff, const int32_t *aidx,
                        int n, const char *const *lb, const int32_t *boff, const int32_t *bidx,
                        int num_threads, double *level_ms) {
    vector<string> xn, yn;
    for (int i = 0; i < m; i++) xn.emplace_back(la[i]);
    for (int i = 0; i < n; i++) yn.emplace_back(lb[i]);
    vector<vector<int>> xa = csr_to_adj(m, aoff, aidx), ya = csr_to_adj(n, boff, bidx);
    std::stringstream cap;
    std::streambuf *old = std::cout.rdbuf(cap.rdbuf());
    int d = standard_ted(xn, xa, yn, ya, num_threads, 1);
    std::cout.rdbuf(old);
    if (level_ms) *level_ms = parse_total_ms(cap.str());
    return d;
}

// Labels given as int32 ids, rendered as decimal strings for the reference.
int xr_standard_ted_int(int m, const int32_t *la, const int32_t *aoff, const int32_t *aidx,
                        int n, const int32_t *lb, const int32_t *boff, const int32_t *bidx,
                        int num_threads, double *level_ms) {
    vector<string> xn, yn;
    for (int i = 0; i < m; i++) xn.push_back(std::to_string(la[i]));
    for (int i = 0; i < n; i++) yn.push_back(std::to_string(lb[i]));
    vector<vector<int>> xa = csr_to_adj(m, aoff, aidx), ya = csr_to_adj(n, boff, bidx);
    std::stringstream cap;
    std::streambuf *old = std::cout.rdbuf(cap.rdbuf());
    int d = standard_ted(xn, xa, yn, ya, num_threads, 1);
    std::cout.rdbuf(old);
    if (level_ms) *level_ms = parse_total_ms(cap.str());
    return d;
}

}  // extern "C"
