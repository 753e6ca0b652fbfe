// gen.cpp -- seeded synthetic trees for the benchmark workloads.
//
// Shapes (all relabelled to preorder; children keep their creation order):
//   0 random recursive: node i > 0 picks its parent uniformly in 0..i-1.
//   1 wide-shallow:     root fanout 40, every other node at depth < 4 has a
//                       geometric fanout of mean 4 (support 1, 2, ...), filled
//                       breadth first and truncated at n nodes; if the depth-4
//                       frontier is exhausted first, the rest become extra last
//                       children of uniformly drawn nodes at depth < 4.
//   2 deep-narrow:      a spine (chain) of min(100, ceil(n/2)) nodes, then
//                       breadth-first fill from the spine: every node gets a
//                       fanout uniform in 1..3 (a spine node's spine child
//                       counts as one), new children at uniform positions.
//   3 caterpillar:      a spine of ceil(n/10) nodes, each carrying 9 leaves
//                       followed by its spine child as the LAST child.
// Labels: uniform over `alphabet` ids, or Zipf(s = 1.1) over `alphabet` ids.
// The random stream is xoshiro256** seeded through splitmix64.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <deque>
#include <vector>

#include "../../include/xted.h"

namespace {

struct Rng {
    uint64_t s[4];
    explicit Rng(uint64_t seed) {
        for (int i = 0; i < 4; i++) {
            seed += 0x9e3779b97f4a7c15ull;
            uint64_t z = seed;
            z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
            z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
            s[i] = z ^ (z >> 31);
        }
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {
        const uint64_t r = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
    uint32_t below(uint32_t k) { return (uint32_t)(((unsigned __int128)next() * k) >> 64); }
    double unit() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

void to_csr(const std::vector<std::vector<int32_t>> &ch, int32_t *off, int32_t *idx,
            std::vector<int32_t> &order) {
    const int n = (int)ch.size();
    std::vector<int32_t> stack{0}, newid((size_t)n);
    order.clear();
    order.reserve((size_t)n);
    while (!stack.empty()) {
        int32_t v = stack.back();
        stack.pop_back();
        order.push_back(v);
        for (auto it = ch[(size_t)v].rbegin(); it != ch[(size_t)v].rend(); ++it) stack.push_back(*it);
    }
    for (int k = 0; k < n; k++) newid[(size_t)order[(size_t)k]] = k;
    off[0] = 0;
    int32_t pos = 0;
    for (int k = 0; k < n; k++) {
        for (int32_t c : ch[(size_t)order[(size_t)k]]) idx[pos++] = newid[(size_t)c];
        off[k + 1] = pos;
    }
}

}  // namespace

extern "C" int xted_gen_tree(int32_t shape, int32_t n, uint64_t seed, int32_t label_kind,
                             int32_t alphabet, int32_t *labels, int32_t *off, int32_t *idx) {
    if (n < 0 || n > XTED_MAX_NODES || shape < 0 || shape > 3 || alphabet < 1 || label_kind < 0 ||
        label_kind > 1 || (n > 0 && (!labels || !off || (n > 1 && !idx))))
        return XTED_EINVAL;
    if (n == 0) {
        if (off) off[0] = 0;
        return XTED_OK;
    }
    Rng g(seed);
    std::vector<std::vector<int32_t>> ch((size_t)n);
    if (shape == 0) {
        for (int i = 1; i < n; i++) ch[g.below((uint32_t)i)].push_back(i);
    } else if (shape == 1) {
        std::vector<int32_t> depth((size_t)n, 0);
        std::deque<int32_t> q{0};
        int cnt = 1;
        while (cnt < n && !q.empty()) {
            int32_t v = q.front();
            q.pop_front();
            if (depth[(size_t)v] >= 4) continue;
            int f = 40;
            if (v != 0) {
                f = 1;
                while (g.unit() >= 0.25) f++;
            }
            for (int k = 0; k < f && cnt < n; k++) {
                ch[(size_t)v].push_back(cnt);
                depth[(size_t)cnt] = depth[(size_t)v] + 1;
                q.push_back(cnt);
                cnt++;
            }
        }
        if (cnt < n) {
            std::vector<int32_t> cand;
            for (int v = 0; v < cnt; v++)
                if (depth[(size_t)v] < 4) cand.push_back(v);
            while (cnt < n) {
                int32_t v = cand[g.below((uint32_t)cand.size())];
                ch[(size_t)v].push_back(cnt);
                depth[(size_t)cnt] = depth[(size_t)v] + 1;
                cnt++;
            }
        }
    } else if (shape == 2) {
        const int spine = std::min(100, std::max(1, (n + 1) / 2));
        for (int i = 1; i < spine; i++) ch[(size_t)i - 1].push_back(i);
        std::deque<int32_t> q;
        for (int i = 0; i < spine; i++) q.push_back(i);
        int cnt = spine;
        while (cnt < n && !q.empty()) {
            int32_t v = q.front();
            q.pop_front();
            int f = 1 + (int)g.below(3);
            int extra = f - (int)ch[(size_t)v].size();
            for (int k = 0; k < extra && cnt < n; k++) {
                auto &c = ch[(size_t)v];
                uint32_t pos = g.below((uint32_t)c.size() + 1);
                c.insert(c.begin() + pos, cnt);
                q.push_back(cnt);
                cnt++;
            }
            if (q.empty() && cnt < n) q.push_back(cnt - 1);
        }
    } else {
        const int spine = (n + 9) / 10;
        int cnt = spine;
        for (int s = 0; s < spine; s++) {
            for (int k = 0; k < 9 && cnt < n; k++) ch[(size_t)s].push_back(cnt++);
            if (s + 1 < spine) ch[(size_t)s].push_back(s + 1);
        }
        while (cnt < n) ch[(size_t)spine - 1].push_back(cnt++);
    }
    std::vector<int32_t> order;
    to_csr(ch, off, idx, order);
    if (label_kind == 0) {
        for (int k = 0; k < n; k++) labels[k] = (int32_t)g.below((uint32_t)alphabet);
    } else {
        std::vector<double> cdf((size_t)alphabet);
        double s = 0;
        for (int r = 0; r < alphabet; r++) {
            s += 1.0 / std::pow((double)(r + 1), 1.1);
            cdf[(size_t)r] = s;
        }
        for (int k = 0; k < n; k++) {
            double u = g.unit() * s;
            int lo = 0, hi = alphabet - 1;
            while (lo < hi) {
                int mid = (lo + hi) / 2;
                if (cdf[(size_t)mid] < u) lo = mid + 1;
                else hi = mid;
            }
            labels[k] = lo;
        }
    }
    return XTED_OK;
}
