// prep.cu -- device-side preprocessing and work decomposition of a batch.
//
// The reference computes orl, keyroots and keyroot depths on the host, then
// for every depth level fetches, sizes, sorts and bins tables with host
// round trips (X-TED_CPU/TED.cpp:163-166, X-TED_GPU/parallel_X_TED.cu:184-224,
// 304-387). Here the raw trees go up once and everything else is built on the
// device, one warp per tree / oriented tree, one thread per pair / (pair, level):
//
//   k_tree_basic_warp  sizes, depths, parents, keyroot-size sums (both decompositions)
//   k_orient_warp  per orientation: node records, kdepth, keyroots by depth,
//                  column-list positions, row runs, column chunks (the records
//                  plan_core.h's orient_tree builds for the host planners)
//   k_pair_setup   decomposition choice, level count
//   k_level_*      unit/task counts and estimates per (pair, level), ready-
//                  queue priority, then the units and tasks themselves
//
// Each (pair, level) entry gets a ready-queue priority bucket from the pair's
// remaining estimated critical path; the DP kernel publishes an entry when the
// previous level of its pair has finished (see xted_internal.h).
// Two small device-to-host reads size the buffers (entries; tasks and units).
#include <cuda_runtime.h>

#include <cstring>

#include "ctx.h"
#include "plan_core.h"

namespace xted {

namespace {

// The outputs of tree_basic (plan_core.h: sizes, depths and parents of every
// node, the keyroot-size sums of both decompositions) with a warp per tree
// and the work spread over its lanes instead of one thread walking the tree:
// parents straight from the child lists; each node's orl (rightmost leaf) by
// pointer jumping along last children, its size orl - v + 1; depths as a
// prefix sum of +1 at every node and -1 just past its subtree (u is an
// ancestor of v exactly when u <= v <= orl(u)); the sums as lane sums. One
// thread per tree waited on a dependent global load per node visited.
__global__ void k_tree_basic_warp(PlanPools P, DTree *trees_out) {
    const int lane = threadIdx.x & 31;
    const int t = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (t >= P.ntrees) return;  // whole warps: t is the same in every lane
    DTree T = P.trees[t];
    const int n = T.n;
    const int32_t *off = P.raw + T.raw + n, *idx = P.raw + T.raw + 2 * n + 1;
    int32_t *size = P.size + T.nbase, *depth = P.depth + T.nbase, *par = P.parent + T.nbase;
    int32_t *jump = P.opar + 2 * (int64_t)T.nbase;  // scratch: this tree's orientation pool, unused until k_orient_warp
    T.S[0] = T.S[1] = 0;
    if (n > 0) {
        for (int v = lane; v < n; v += 32) {
            const int32_t lo = off[v], hi = off[v + 1];
            for (int32_t e = lo; e < hi; e++) par[idx[e]] = v;
            size[v] = hi > lo ? idx[hi - 1] : v;  // last child, or the node itself for a leaf
        }
        if (lane == 0) par[0] = -1;
        __syncwarp();
        int32_t *cur = size, *nxt = jump;
        for (int round = 0; round < 32; round++) {
            bool changed = false;
            for (int v = lane; v < n; v += 32) {
                const int32_t a = cur[v], b = cur[a];
                nxt[v] = b;
                changed |= b != a;
            }
            __syncwarp();
            int32_t *tmp = cur;
            cur = nxt;
            nxt = tmp;
            if (!__any_sync(0xffffffffu, changed)) break;
        }
        // cur[v] = orl(v). Depth: +1 at every u, -1 at orl(u) + 1, then an inclusive prefix sum
        for (int v = lane; v < n; v += 32) depth[v] = 0;
        __syncwarp();
        for (int u = lane; u < n; u += 32) {
            atomicAdd(&depth[u], 1);
            const int32_t o1 = cur[u] + 1;
            if (o1 < n) atomicSub(&depth[o1], 1);
        }
        __syncwarp();
        const int per = (n + 31) / 32, a0 = min(lane * per, n), a1 = min(a0 + per, n);
        int32_t sum = 0;
        for (int v = a0; v < a1; v++) sum += depth[v];
        int32_t incl = sum;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int32_t o = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += o;
        }
        int32_t run = incl - sum;
        for (int v = a0; v < a1; v++) {
            run += depth[v];
            depth[v] = run - 1;
        }
        __syncwarp();
        for (int v = lane; v < n; v += 32) size[v] = cur[v] - v + 1;
        __syncwarp();
        int64_t sr = 0, sl = 0;
        for (int v = lane; v < n; v += 32) {
            const int32_t lo = off[v], hi = off[v + 1];
            for (int32_t e = lo; e < hi; e++) {
                const int64_t z = size[idx[e]];
                if (e != hi - 1) sr += z;
                if (e != lo) sl += z;
            }
        }
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) {
            sr += __shfl_down_sync(0xffffffffu, sr, d);
            sl += __shfl_down_sync(0xffffffffu, sl, d);
        }
        T.S[0] = sr + size[0];
        T.S[1] = sl + size[0];
    }
    if (lane == 0) trees_out[t] = T;
}

__device__ __forceinline__ int warp_incl_sum(int v, int lane) {
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int o = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= d) v += o;
    }
    return v;
}

// One warp per oriented tree: the same records as orient_tree (plan_core.h,
// which the host planners run), with its passes spread over the lanes (a
// thread per oriented tree took 10 ms for the 8,192 trees of the 4,096-pair
// batch, its passes waiting on one global load after another; this takes 1.8).
//   * node records and the previous-node-is-leaf flags: one node per lane;
//   * A(x), the keyroots on x's root path (x included): a prefix sum over
//     preorder of +1 at each keyroot and -1 just past its subtree;
//   * keyroot depth kd(u) = (max of A over u's subtree) - A(u), the height of u
//     among the keyroots nested in it: each lane scans the subtrees of its
//     keyroots (the keyroot-size sum of the tree in all);
//   * keyroots grouped by depth in preorder: a counting sort, 32 nodes at a time,
//     lanes of one depth ranked by lane;
//   * row runs and column chunks per depth: sizes and column positions loaded
//     and summed 32 keyroots at a time, the greedy packing then decided by the
//     whole warp from shuffled sizes (every lane holds the same packing state).
__global__ void k_orient_warp(PlanPools P) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int ot = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (ot >= 2 * P.ntrees) return;  // whole warps
    const int t = ot >> 1, o = ot & 1;
    const DTree T = P.trees[t];
    const int n = T.n;
    DOTree O;
    O.n = n;
    O.node_base = 2 * T.nbase + o * n;
    O.depth_base = 2 * (T.nbase + t) + o * (n + 1);
    O.D = -1;
    O.maxka = 0;
    O.maxw_wide = 0;
    O.S = T.S[o];
    if (n == 0) {
        if (lane == 0) P.otrees[ot] = O;
        return;
    }
    const int32_t *lab = P.raw + T.raw;
    const int32_t *off = P.raw + T.raw + n;
    const int32_t *idx = P.raw + T.raw + 2 * n + 1;
    const int32_t *size = P.size + T.nbase, *depth = P.depth + T.nbase, *par = P.parent + T.nbase;
    int2 *node = P.node + O.node_base;
    int32_t *opar = P.opar + O.node_base, *okd = P.okd + O.node_base, *oka = P.oka + O.node_base;
    // node records in this orientation
    for (int v = lane; v < n; v += 32) {
        const int32_t u = o ? mirror_id(v, n, size, depth) : v;
        bool kr = true;
        if (v > 0) {
            const int32_t p = par[v];
            kr = o ? idx[off[p]] != v : idx[off[p + 1] - 1] != v;
            opar[u] = o ? mirror_id(p, n, size, depth) : p;
        } else {
            opar[u] = -1;
        }
        node[u].x = lab[v];
        node[u].y = (int32_t)((uint32_t)(u + size[v] - 1) | (kr ? XTED_ROW_ISKR : 0u));
        oka[u] = 0;
    }
    __syncwarp();
    for (int u = 1 + lane; u < n; u += 32) {
        const int32_t prev_orl = node[u - 1].y & XTED_ROW_ORL_MASK;  // (its flag bits may change meanwhile)
        if (prev_orl == u - 1) node[u].y = (int32_t)((uint32_t)node[u].y | XTED_ROW_PREVLEAF);
    }
    // A(x): +1 at a keyroot, -1 just past its subtree, summed over preorder
    for (int u = lane; u < n; u += 32) {
        const int32_t y = node[u].y;
        if (y & XTED_ROW_ISKR) {
            atomicAdd(&oka[u], 1);
            const int e = (y & XTED_ROW_ORL_MASK) + 1;
            if (e < n) atomicSub(&oka[e], 1);
        }
    }
    __syncwarp();
    int carry = 0, maxa = 1;
    for (int base = 0; base < n; base += 32) {
        const int x = base + lane;
        const int dv = x < n ? __ldcg(&oka[x]) : 0;
        const int a = carry + warp_incl_sum(dv, lane);
        if (x < n) {
            oka[x] = a;
            maxa = max(maxa, a);
        }
        carry = __shfl_sync(FULL, a, 31);
    }
    for (int d = 16; d > 0; d >>= 1) maxa = max(maxa, __shfl_xor_sync(FULL, maxa, d));
    O.maxka = maxa;
    __syncwarp();
    // keyroot depths
    for (int u = lane; u < n; u += 32) {
        const int32_t y = node[u].y;
        int kd = -1;
        if (y & XTED_ROW_ISKR) {
            const int e = y & XTED_ROW_ORL_MASK, au = oka[u];
            int m = au;
            for (int x = u + 1; x <= e; x++) m = max(m, oka[x]);
            kd = m - au;
        }
        okd[u] = kd;
    }
    __syncwarp();
    const int D = okd[0];  // the root is a keyroot
    O.D = D;
    // keyroots grouped by depth (counting sort, preorder inside a depth)
    DDepth *dep = P.depths + O.depth_base;
    for (int d = lane; d <= D; d += 32) {
        dep[d].krd_lo = 0;
        dep[d].krd_hi = 0;
    }
    __syncwarp();
    for (int u = lane; u < n; u += 32)
        if (okd[u] >= 0) atomicAdd(&dep[okd[u]].krd_hi, 1);
    __syncwarp();
    carry = O.node_base;
    for (int base = 0; base <= D; base += 32) {
        const int d = base + lane;
        const int c = d <= D ? __ldcg(&dep[d].krd_hi) : 0;
        const int incl = warp_incl_sum(c, lane);
        if (d <= D) {
            dep[d].krd_lo = carry + incl - c;
            dep[d].krd_hi = carry + incl - c;  // fill cursor
        }
        carry += __shfl_sync(FULL, incl, 31);
    }
    __syncwarp();
    const unsigned below = (1u << lane) - 1u;
    for (int base = 0; base < n; base += 32) {
        const int u = base + lane;
        const int kd = u < n ? okd[u] : -1;
        const unsigned same = __match_any_sync(FULL, kd);  // lanes holding keyroots of this depth
        if (kd >= 0) {
            const int leader = __ffs(same) - 1;
            int at = 0;
            if (lane == leader) {
                at = dep[kd].krd_hi;
                dep[kd].krd_hi = at + __popc(same);
            }
            at = __shfl_sync(same, at, leader);
            P.krd[at + __popc(same & below)] = u;
        }
        __syncwarp();
    }
    // column-list positions, row runs and chunks per depth
    int run_rows, nw, hw;
    tree_granularity(P, n, &run_rows, &nw, &hw);
    const int group_w = nw > 0 ? nw : XTED_NARROW_MAX;
    const int half_w = hw > nw ? (hw < XTED_HALF_MAX ? hw : XTED_HALF_MAX) : nw;
    int32_t run_cur = O.node_base, chunk_cur = O.node_base;
    for (int d = 0; d <= D; d++) {
        DDepth dd = dep[d];  // krd_lo, krd_hi
        const int klo = dd.krd_lo, khi = dd.krd_hi;
        // runs
        dd.run_lo = run_cur;
        dd.maxrows = 0;
        int pos = 0, r_lo = -1, r_hi = -1, r_rows = 0;
        for (int kb = klo; kb < khi; kb += 32) {
            const int k = kb + lane;
            int sz = 0;
            if (k < khi) {
                const int32_t u = P.krd[k];
                sz = (node[u].y & XTED_ROW_ORL_MASK) - u + 1;
            }
            const int incl = warp_incl_sum(sz, lane);
            if (k < khi) P.cumw[k] = pos + incl - sz;
            pos += __shfl_sync(FULL, incl, 31);
            const int cnt = min(32, khi - kb);
            for (int j = 0; j < cnt; j++) {
                const int szj = __shfl_sync(FULL, sz, j);
                if (r_lo >= 0 && r_rows + szj > run_rows) {
                    if (r_rows > dd.maxrows) dd.maxrows = r_rows;
                    if (lane == 0) P.runs[run_cur] = XRun{r_lo, r_hi, r_rows, d};
                    run_cur++;
                    r_lo = -1;
                    r_rows = 0;
                }
                if (r_lo < 0) r_lo = kb + j;
                r_hi = kb + j + 1;
                r_rows += szj;
            }
        }
        if (r_lo >= 0) {
            if (r_rows > dd.maxrows) dd.maxrows = r_rows;
            if (lane == 0) P.runs[run_cur] = XRun{r_lo, r_hi, r_rows, d};
            run_cur++;
        }
        dd.run_hi = run_cur;
        // chunks: three passes, narrow chunks first, then half-block ones, then whole-block ones
        dd.chunk_lo = chunk_cur;
        dd.nnarrow = dd.nwide = dd.nhalf = 0;
        dd.maxw_n = dd.maxw_w = dd.maxw_h = 0;
        for (int pass = 0; pass < 3; pass++) {
            int c_lo = -1, c_w = 0, c_n = 0;
            bool done = false;
            for (int kb = klo; kb <= khi && !done; kb += 32) {
                const int k = kb + lane;
                int w = 0;
                if (k < khi) {
                    const int32_t u = P.krd[k];
                    w = (node[u].y & XTED_ROW_ORL_MASK) - u + 1;
                }
                const int cnt = min(32, khi + 1 - kb);
                for (int j = 0; j < cnt; j++) {
                    const int kk = kb + j;
                    const int wj = __shfl_sync(FULL, w, j);
                    const bool flush = c_n > 0 && (kk == khi || c_w + wj > group_w);
                    if (flush) {
                        const int kind = c_w <= nw ? 0 : (c_w <= half_w ? 1 : 2);
                        if (kind == pass) {
                            if (lane == 0) P.chunks[chunk_cur] = XChunk{c_lo, c_w, d, c_n};
                            chunk_cur++;
                            if (kind == 2) {
                                dd.nwide++;
                                if (c_w > dd.maxw_w) dd.maxw_w = c_w;
                            } else if (kind == 1) {
                                dd.nhalf++;
                                if (c_w > dd.maxw_h) dd.maxw_h = c_w;
                            } else {
                                dd.nnarrow++;
                                if (c_w > dd.maxw_n) dd.maxw_n = c_w;
                            }
                        }
                        c_lo = -1;
                        c_w = 0;
                        c_n = 0;
                    }
                    if (kk == khi) {
                        done = true;
                        break;
                    }
                    if (c_n == 0) c_lo = kk;  // first segment (keyroot pool index)
                    c_w += wj;
                    c_n += 1;
                }
            }
        }
        if (dd.maxw_h > O.maxw_wide) O.maxw_wide = dd.maxw_h;
        if (dd.maxw_w > O.maxw_wide) O.maxw_wide = dd.maxw_w;
        if (lane == 0) dep[d] = dd;
        __syncwarp();
    }
    if (lane == 0) P.otrees[ot] = O;
}

__global__ void k_pair_setup(const DTree *trees, const DOTree *ot, const int32_t *pair_trees, int orientation,
                             int npairs, DPair *pairs, int64_t *L, int64_t *cells) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npairs) return;
    pair_setup(trees, ot, pair_trees, orientation, p, pairs);
    L[p] = pairs[p].L;
    cells[p] = pairs[p].trivial >= 0 ? 0 : (int64_t)trees[pairs[p].ta].n * trees[pairs[p].tb].n;
}

// Exclusive scan of n int64 values in one block; out[n] = total. Optional
// permutation: scans v[perm[i]] in the order i and writes out[i].
__global__ void k_scan64(const int64_t *v, const int32_t *perm, int n, int64_t *out) {
    __shared__ int64_t part[1024];
    const int tid = threadIdx.x, nt = blockDim.x;
    const int per = (n + nt - 1) / nt;
    const int lo = tid * per, hi = min(lo + per, n);
    int64_t s = 0;
    for (int i = lo; i < hi; i++) s += v[perm ? perm[i] : i];
    part[tid] = s;
    __syncthreads();
    for (int d = 1; d < nt; d <<= 1) {
        int64_t x = tid >= d ? part[tid - d] : 0;
        __syncthreads();
        part[tid] += x;
        __syncthreads();
    }
    int64_t run = part[tid] - s;
    for (int i = lo; i < hi; i++) {
        out[i] = run;
        run += v[perm ? perm[i] : i];
    }
    if (tid == nt - 1) out[n] = part[nt - 1];
}

struct Summary {
    int64_t entries, dt_elems;
    int64_t tasks, units;
    int64_t nstriped, nstripes;  // striped units and their stripes
    int64_t stripe_buf;          // 64-bit words of the striped units' buffers
    int32_t stack_rows, max_wide;
    int64_t cells, cells_right;
    int32_t levels_max, pad;
    int64_t chain_max;
};

__global__ void k_pair_offsets(DPair *pairs, const DTree *trees, const DOTree *ot, int npairs, const int64_t *Lscan,
                               const int64_t *dtscan, Summary *sum) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p == 0) {
        sum->entries = Lscan[npairs];
        sum->dt_elems = dtscan[npairs];
    }
    if (p >= npairs) return;
    DPair &q = pairs[p];
    q.lvl_base = (int32_t)Lscan[p];
    q.dt_off = dtscan[p];
    if (q.trivial < 0) {
        const DOTree &A = ot[2 * q.ta + q.o], &B = ot[2 * q.tb + q.o];
        atomicMax(&sum->stack_rows, A.maxka + 1);
        atomicMax(&sum->max_wide, B.maxw_wide);
        atomicMax(&sum->levels_max, q.L);
        atomicAdd((unsigned long long *)&sum->cells, (unsigned long long)q.cells);
        atomicAdd((unsigned long long *)&sum->cells_right,
                  (unsigned long long)(trees[q.ta].S[0] * trees[q.tb].S[0]));
    }
}

__global__ void k_level_expand(const DPair *pairs, int npairs, DLevel *lv) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npairs) return;
    const DPair q = pairs[p];
    for (int d = 0; d < q.L; d++) {
        DLevel &E = lv[q.lvl_base + d];
        E.pair = p;
        E.level = d;
    }
}

__global__ void k_level_count(LevelCtx C, DLevel *lv, int64_t nent, int64_t *units, int64_t *tasks,
                              int64_t *striped, int64_t *stripes) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nent) return;
    DLevel E = lv[e];
    double est;
    level_count(C, E, &est);
    E.key = (int64_t)(est / 64.0) + 1;  // >= 1: strictly decreasing ranks below
    lv[e] = E;
    units[e] = (int64_t)E.nwide + E.nnarrow + E.nhalf;
    tasks[e] = E.ntasks;
    striped[e] = E.nstriped;
    stripes[e] = E.nstripes;
}

// Per pair: est(d) is the estimated time of level d's slowest task; EST(d) =
// sum of est below d; the pair's chain C = sum of all est. A level's ready-
// queue bucket grows with the pair's remaining chain C - EST(d) relative to
// the longest chain of the batch.
__global__ void k_pair_rank(const DPair *pairs, int npairs, DLevel *lv, int64_t *chain, Summary *sum) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npairs) return;
    const DPair q = pairs[p];
    int64_t acc = 0;
    for (int d = 0; d < q.L; d++) {
        DLevel &E = lv[q.lvl_base + d];
        const int64_t est = E.key;
        E.key = acc;
        acc += est;
    }
    chain[p] = acc;
    atomicMax((unsigned long long *)&sum->chain_max, (unsigned long long)acc);
}

__global__ void k_level_offsets(DLevel *lv, int64_t nent, const int64_t *task_scan, const int64_t *unit_scan,
                                const int64_t *striped_scan, const int64_t *stripes_scan, const int64_t *chain,
                                const DPair *pairs, XEntry *entries, Summary *sum) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e == 0) {
        sum->tasks = task_scan[nent];
        sum->units = unit_scan[nent];
        sum->nstriped = striped_scan[nent];
        sum->nstripes = stripes_scan[nent];
    }
    if (e >= nent) return;
    DLevel &E = lv[e];
    E.task_off = (int32_t)task_scan[e];
    E.unit_off = (int32_t)unit_scan[e];
    E.stripe_off = (int32_t)striped_scan[e];
    E.entry = (int32_t)e;
    XEntry X;
    X.task_off = E.task_off;
    X.ntasks = E.ntasks;
    X.bucket = level_bucket(chain[E.pair] - E.key, sum->chain_max);
    X.next = E.level + 1 < pairs[E.pair].L ? (int32_t)e + 1 : -1;
    X.nnarrow = E.nntasks;
    X.pad = 0;
    entries[e] = X;
}

__global__ void k_level_fill(LevelCtx C, const DLevel *lv, int64_t nent, XUnit *units, XTask *tasks,
                             XStripe *stripes) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < nent) level_fill(C, lv[e], units, tasks, stripes);
}

// One block per striped unit: its export map, the far columns that a stripe
// reads from a stripe to its right (f = orl(j) + 1 in another stripe), numbered
// in column order (-1 elsewhere), and the words its buffer needs: carries and
// first columns of every stripe and row, and the exported values of every row.
__global__ void k_stripe_prep(XStripe *stripes, int32_t *smap, int64_t map_stride, const XUnit *units,
                              const XChunk *chunks, const XPair *pairs, const int2 *rowinfo, const int32_t *krd,
                              int64_t *need) {
    __shared__ int ends[XTED_WARPS];
    const int i = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const XStripe S = stripes[i];
    const XChunk ch = chunks[units[S.unit].chunk];
    const XPair pr = pairs[S.pair];
    const int w = S.w, SW = XTED_CTA_THREADS * S.sww;
    int32_t *expmap = smap + (int64_t)i * map_stride;
    for (int c = tid; c < w; c += XTED_CTA_THREADS) expmap[c] = 0;
    __syncthreads();
    const int2 *nodes = rowinfo + pr.col_base;
    const int j0 = krd[ch.k_lo];
    for (int c = tid; c < w; c += XTED_CTA_THREADS) {
        const int j = j0 + c;
        const int f = c + ((nodes[j].y & XTED_ROW_ORL_MASK) + 1 - j);
        if (f < w && f / SW != c / SW) expmap[f] = 1;
    }
    __syncthreads();
    const int per = (w + XTED_CTA_THREADS - 1) / XTED_CTA_THREADS;
    const int a0 = min(tid * per, w), a1 = min(a0 + per, w);
    int cnt = 0;
    for (int c = a0; c < a1; c++) cnt += expmap[c];
    int incl = cnt;
    for (int d = 1; d < 32; d <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += y;
    }
    if (lane == 31) ends[warp] = incl;
    __syncthreads();
    int before = incl - cnt, total = 0;
    for (int q = 0; q < XTED_WARPS; q++) {
        if (q < warp) before += ends[q];
        total += ends[q];
    }
    for (int c = a0; c < a1; c++) {
        const int m = expmap[c];
        expmap[c] = m ? before : -1;
        before += m;
    }
    if (tid == 0) {
        stripes[i].X = total;
        stripes[i].map_off = (int64_t)i * map_stride;
        need[i] = (2 * (int64_t)S.K * S.R + (int64_t)S.R * total + 15) & ~(int64_t)15;
    }
}

__global__ void k_stripe_bufoff(XStripe *stripes, int64_t n, const int64_t *scan, Summary *sum) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) sum->stripe_buf = scan[n];
    if (i < n) stripes[i].buf_off = scan[i];
}

__global__ void k_pair_finalize(const DPair *pairs, const DTree *trees, const DOTree *ot, int npairs, XPair *xp,
                                int32_t *trivial, int32_t *first) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npairs) return;
    const DPair q = pairs[p];
    first[p] = q.L > 0 ? q.lvl_base : -1;
    XPair x;
    x.dt_off = q.dt_off;
    x.m = trees[q.ta].n;
    x.n = trees[q.tb].n;
    x.row_base = ot[2 * q.ta + q.o].node_base;
    x.col_base = ot[2 * q.tb + q.o].node_base;
    xp[p] = x;
    trivial[p] = q.trivial;
}

inline unsigned blocks_for(int64_t n, int bs) { return (unsigned)((n + bs - 1) / bs); }

}  // namespace

// Carves a device buffer into aligned sections.
struct Carver {
    char *base;
    size_t off = 0;
    template <class T>
    T *take(size_t count) {
        off = (off + 255) & ~(size_t)255;
        T *p = (T *)(base + off);
        off += sizeof(T) * (count > 0 ? count : 1);
        return p;
    }
};

int dev_plan(xted_ctx *c, const xted_tree *a, const xted_tree *b, int32_t npairs, XKernelParams &K) {
    cudaStream_t s = c->stream;
    // ---- host: unique trees, flat raw input, pair list ----
    c->tree_ids.clear();
    c->uniq.clear();
    std::vector<int32_t> &pt = c->pair_trees;
    pt.resize(2 * (size_t)npairs);
    int64_t N = 0, R = 0;
    for (int p = 0; p < npairs; p++) {
        for (int side = 0; side < 2; side++) {
            const xted_tree &t = side ? b[p] : a[p];
            TreeKey key{t.labels, t.child_off, t.child_idx, t.n};
            auto it = c->tree_ids.find(key);
            int id;
            if (it == c->tree_ids.end()) {
                id = (int)c->uniq.size();
                c->tree_ids.emplace(key, id);
                if (t.n < 0 || t.n > XTED_MAX_NODES) return XTED_EINVAL;
                c->uniq.push_back(TreeView{t.n, t.labels, t.child_off, t.child_idx});
                N += t.n;
                R += 3 * (int64_t)t.n + 1;
            } else {
                id = it->second;
            }
            pt[2 * (size_t)p + side] = id;
        }
    }
    const int T = (int)c->uniq.size();
    if (N > (int64_t)1 << 30) return XTED_ENOMEM;
    {   // every unique tree is checked before anything reads it (host threads for big batches)
        std::vector<int> bad((size_t)std::max(T, 1), 0);
        parallel_for(T, 512, [&](int64_t lo, int64_t hi) {
            for (int64_t t = lo; t < hi; t++) bad[(size_t)t] = validate_tree(c->uniq[(size_t)t]);
        });
        for (int t = 0; t < T; t++)
            if (bad[(size_t)t]) return bad[(size_t)t];
    }
    std::vector<DTree> &ht = c->htrees;
    ht.resize((size_t)T);
    // staging: raw trees | DTree[T] | pair_trees
    const size_t raw_bytes = (size_t)R * 4, tr_bytes = sizeof(DTree) * (size_t)T,
                 pt_bytes = 8 * (size_t)npairs;
    const size_t stage_bytes = raw_bytes + tr_bytes + pt_bytes + 1024;
    int rc = ctx_host_reserve(c->stage, stage_bytes);
    if (rc) return rc;
    char *h = (char *)c->stage.p;
    int32_t *hraw = (int32_t *)h;
    {
        int64_t rpos = 0, nb = 0;
        for (int t = 0; t < T; t++) {
            const TreeView &tv = c->uniq[(size_t)t];
            DTree &d = ht[(size_t)t];
            d.n = tv.n;
            d.raw = (int32_t)rpos;
            d.nbase = (int32_t)nb;
            d.t = t;
            d.S[0] = d.S[1] = 0;
            rpos += 3 * (int64_t)tv.n + 1;
            nb += tv.n;
        }
        parallel_for(T, 512, [&](int64_t lo, int64_t hi) {
            for (int64_t t = lo; t < hi; t++) {
                const TreeView &tv = c->uniq[(size_t)t];
                int32_t *dst = hraw + ht[(size_t)t].raw;
                const int n = tv.n;
                if (n > 0) {
                    std::memcpy(dst, tv.labels, 4 * (size_t)n);
                    std::memcpy(dst + n, tv.off, 4 * ((size_t)n + 1));
                    if (n > 1) std::memcpy(dst + 2 * n + 1, tv.idx, 4 * ((size_t)n - 1));
                } else {
                    dst[0] = 0;  // child_off[0]
                }
            }
        });
    }
    size_t hoff = (raw_bytes + 255) & ~(size_t)255;
    std::memcpy(h + hoff, ht.data(), tr_bytes);
    const size_t hoff_pt = (hoff + tr_bytes + 255) & ~(size_t)255;
    std::memcpy(h + hoff_pt, pt.data(), pt_bytes);
    const size_t upload = hoff_pt + pt_bytes;

    // ---- device buffer A: input + per-tree pools (sizes known from N, T, npairs) ----
    const size_t N2 = 2 * (size_t)std::max<int64_t>(N, 1);
    size_t need = upload + 4096;
    need += 3 * sizeof(int32_t) * (size_t)std::max<int64_t>(N, 1);  // size, depth, parent
    need += N2 * (sizeof(int2) + 2 * sizeof(int32_t) + sizeof(XRun) + sizeof(XChunk) + 3 * sizeof(int32_t));
    need += sizeof(DDepth) * (N2 + 2 * (size_t)T) + sizeof(DOTree) * 2 * (size_t)T + sizeof(DTree) * (size_t)T;
    need += (size_t)npairs * (sizeof(DPair) + sizeof(XPair) + 4 + 5 * 8) + 20 * 256 + sizeof(Summary);
    rc = ctx_dev_reserve(c, c->meta, need);
    if (rc) return rc;
    Carver cv{(char *)c->meta.p};
    char *d_in = cv.take<char>(upload);
    if (cudaMemcpyAsync(d_in, h, upload, cudaMemcpyHostToDevice, s) != cudaSuccess) return XTED_ECUDA;
    c->h2d_bytes = (int64_t)upload;
    PlanPools P;
    P.raw = (const int32_t *)d_in;
    DTree *d_trees = (DTree *)(d_in + hoff);
    P.trees = d_trees;
    const int32_t *d_pt = (const int32_t *)(d_in + hoff_pt);
    P.ntrees = T;
    P.size = cv.take<int32_t>((size_t)N);
    P.depth = cv.take<int32_t>((size_t)N);
    P.parent = cv.take<int32_t>((size_t)N);
    P.node = cv.take<int2>(N2);
    P.krd = cv.take<int32_t>(N2);
    P.cumw = cv.take<int32_t>(N2);
    P.runs = cv.take<XRun>(N2);
    P.chunks = cv.take<XChunk>(N2);
    P.opar = cv.take<int32_t>(N2);
    P.okd = cv.take<int32_t>(N2);
    P.oka = cv.take<int32_t>(N2);
    P.depths = cv.take<DDepth>(N2 + 2 * (size_t)T);
    P.otrees = cv.take<DOTree>(2 * (size_t)T);
    P.run_rows = c->opts.run_rows;
    P.narrow_width = c->opts.narrow_width;
    P.half_width = c->opts.half_width == 0 ? XTED_HALF_DEFAULT : c->opts.half_width;
    P.ntune = 0;
    if (c->opts.tuned) {
        int nt = 0;
        const XTuneRow *tt = ctx_tune_table(c, &nt);
        for (int k = 0; k < nt && k < XTED_TUNE_ROWS; k++) P.tune[P.ntune++] = tt[k];
    }
    DPair *d_pairs = cv.take<DPair>((size_t)npairs);
    XPair *d_xpairs = cv.take<XPair>((size_t)npairs);
    int32_t *d_trivial = cv.take<int32_t>((size_t)npairs);
    int64_t *d_L = cv.take<int64_t>((size_t)npairs + 1);
    int64_t *d_chain = cv.take<int64_t>((size_t)npairs + 1);
    int64_t *d_cells = cv.take<int64_t>((size_t)npairs + 1);
    int64_t *d_Ls = cv.take<int64_t>((size_t)npairs + 1);
    int64_t *d_dts = cv.take<int64_t>((size_t)npairs + 1);
    Summary *d_sum = cv.take<Summary>(1);
    if (cv.off > c->meta.cap) return XTED_ENOMEM;

    const int BS = 128;
    cudaMemsetAsync(d_sum, 0, sizeof(Summary), s);
    k_tree_basic_warp<<<blocks_for(32 * (int64_t)T, BS), BS, 0, s>>>(P, d_trees);
    k_orient_warp<<<blocks_for(64 * (int64_t)T, BS), BS, 0, s>>>(P);
    k_pair_setup<<<blocks_for(npairs, BS), BS, 0, s>>>(d_trees, P.otrees, d_pt, c->opts.orientation, npairs,
                                                       d_pairs, d_L, d_cells);
    k_scan64<<<1, 1024, 0, s>>>(d_L, nullptr, npairs, d_Ls);
    k_scan64<<<1, 1024, 0, s>>>(d_cells, nullptr, npairs, d_dts);
    k_pair_offsets<<<blocks_for(std::max(npairs, 1), BS), BS, 0, s>>>(d_pairs, d_trees, P.otrees, npairs, d_Ls,
                                                                      d_dts, d_sum);
    rc = ctx_host_reserve(c->summary, sizeof(Summary));
    if (rc) return rc;
    Summary *hs = (Summary *)c->summary.p;
    cudaMemcpyAsync(hs, d_sum, sizeof(Summary), cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) {
        cudaGetLastError();
        return XTED_ECUDA;
    }
    const int64_t nent = hs->entries;
    if (nent > INT32_MAX / XTED_BUCKETS) return XTED_ENOMEM;
    // ---- buffer B: level entries and scans ----
    const size_t E1 = (size_t)nent + 1;
    size_t needB = sizeof(DLevel) * E1 + sizeof(XEntry) * E1 + 8 * 8 * E1 + 16 * 256;
    rc = ctx_dev_reserve(c, c->levels, needB);
    if (rc) return rc;
    Carver cb{(char *)c->levels.p};
    DLevel *d_lv = cb.take<DLevel>(E1);
    XEntry *d_entries = cb.take<XEntry>(E1);
    int64_t *d_units = cb.take<int64_t>(E1), *d_tasks = cb.take<int64_t>(E1);
    int64_t *d_uscan = cb.take<int64_t>(E1), *d_tscan = cb.take<int64_t>(E1);
    int64_t *d_striped = cb.take<int64_t>(E1), *d_stripes = cb.take<int64_t>(E1);
    int64_t *d_sdscan = cb.take<int64_t>(E1), *d_spscan = cb.take<int64_t>(E1);
    LevelCtx C;
    C.ot = P.otrees;
    C.depths = P.depths;
    C.runs = P.runs;
    C.chunks = P.chunks;
    C.pairs = d_pairs;
    C.narrow_width = c->opts.narrow_width;
    C.wide_rows = c->opts.wide_rows > 0 ? c->opts.wide_rows : -1;
    C.stripe_min_cells = c->opts.stripe_min_cells < 0 ? 0
                         : (c->opts.stripe_min_cells > 0 ? c->opts.stripe_min_cells : XTED_STRIPE_MIN_CELLS_DEFAULT);
    if (nent > 0) {
        k_level_expand<<<blocks_for(npairs, BS), BS, 0, s>>>(d_pairs, npairs, d_lv);
        k_level_count<<<blocks_for(nent, BS), BS, 0, s>>>(C, d_lv, nent, d_units, d_tasks, d_striped, d_stripes);
        k_pair_rank<<<blocks_for(npairs, BS), BS, 0, s>>>(d_pairs, npairs, d_lv, d_chain, d_sum);
        k_scan64<<<1, 1024, 0, s>>>(d_tasks, nullptr, (int)nent, d_tscan);
        k_scan64<<<1, 1024, 0, s>>>(d_units, nullptr, (int)nent, d_uscan);
        k_scan64<<<1, 1024, 0, s>>>(d_striped, nullptr, (int)nent, d_sdscan);
        k_scan64<<<1, 1024, 0, s>>>(d_stripes, nullptr, (int)nent, d_spscan);
        k_level_offsets<<<blocks_for(nent, BS), BS, 0, s>>>(d_lv, nent, d_tscan, d_uscan, d_sdscan, d_spscan,
                                                              d_chain, d_pairs, d_entries, d_sum);
    }
    cudaMemcpyAsync(hs, d_sum, sizeof(Summary), cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) {
        cudaGetLastError();
        return XTED_ECUDA;
    }
    const int64_t ntasks = nent > 0 ? hs->tasks : 0, nunits = nent > 0 ? hs->units : 0;
    const int64_t nstriped = nent > 0 ? hs->nstriped : 0, nstripes = nent > 0 ? hs->nstripes : 0;
    if (ntasks > INT32_MAX / 2 || nunits > INT32_MAX / 2 || nstripes > INT32_MAX / 2) return XTED_ENOMEM;
    // ---- buffer C: units, tasks and the ready queue's state ----
    int rq_log2 = 0;
    while (((int64_t)1 << rq_log2) < (int64_t)E1) rq_log2++;
    const size_t rq_slots = (size_t)XTED_RINGS << rq_log2;
    rc = ctx_dev_reserve(c, c->work, sizeof(XUnit) * (size_t)(nunits + 1) + sizeof(XTask) * (size_t)(ntasks + 1) +
                                         8 * rq_slots + 4 * (XTED_ESTATE * E1 + (size_t)npairs + 2 * XTED_RINGS + 8) +
                                         sizeof(XStripe) * (size_t)(nstriped + 1) + 8 * 2 * (size_t)(nstriped + 1) +
                                         12 * 256);
    if (rc) return rc;
    Carver cw{(char *)c->work.p};
    XUnit *d_units_out = cw.take<XUnit>((size_t)nunits);
    XTask *d_tasks_out = cw.take<XTask>((size_t)ntasks);
    int32_t *d_first = cw.take<int32_t>((size_t)npairs);
    int32_t *d_state = cw.take<int32_t>(XTED_ESTATE * E1);  // narrow claimed, group claimed, done per entry
    unsigned long long *d_rq = cw.take<unsigned long long>(rq_slots);
    int32_t *d_ctl = cw.take<int32_t>(2 * XTED_RINGS + 8);  // heads/tails, then the done counter
    XStripe *d_st = cw.take<XStripe>((size_t)nstriped + 1);
    int64_t *d_need = cw.take<int64_t>((size_t)nstriped + 1), *d_needscan = cw.take<int64_t>((size_t)nstriped + 1);
    if (nent > 0)
        k_level_fill<<<blocks_for(nent, 64), 64, 0, s>>>(C, d_lv, nent, d_units_out, d_tasks_out, d_st);
    k_pair_finalize<<<blocks_for(std::max(npairs, 1), BS), BS, 0, s>>>(d_pairs, d_trees, P.otrees, npairs, d_xpairs,
                                                                       d_trivial, d_first);
    if (cudaGetLastError() != cudaSuccess) return XTED_ECUDA;
    // striped units: export maps (one stride of the widest segment each), then
    // the buffers, whose sizes the maps give
    int64_t stripe_buf = 0;
    if (nstriped > 0) {
        const int64_t map_stride = ((int64_t)hs->max_wide + 31) & ~(int64_t)31;
        rc = ctx_dev_reserve(c, c->smap, (size_t)(nstriped * map_stride) * sizeof(int32_t));
        if (rc) return rc;
        k_stripe_prep<<<(unsigned)nstriped, XTED_CTA_THREADS, 0, s>>>(d_st, (int32_t *)c->smap.p, map_stride,
                                                                      d_units_out, P.chunks, d_xpairs, P.node,
                                                                      P.krd, d_need);
        k_scan64<<<1, 1024, 0, s>>>(d_need, nullptr, (int)nstriped, d_needscan);
        k_stripe_bufoff<<<blocks_for(nstriped, BS), BS, 0, s>>>(d_st, nstriped, d_needscan, d_sum);
        cudaMemcpyAsync(hs, d_sum, sizeof(Summary), cudaMemcpyDeviceToHost, s);
        if (cudaStreamSynchronize(s) != cudaSuccess) {
            cudaGetLastError();
            return XTED_ECUDA;
        }
        stripe_buf = hs->stripe_buf;
        rc = ctx_dev_reserve(c, c->sbuf, (size_t)std::max<int64_t>(stripe_buf, 1) * sizeof(unsigned long long));
        if (rc) return rc;
    }

    std::memset(&K, 0, sizeof(K));
    K.rowinfo = P.node;
    K.krd = P.krd;
    K.cumw = P.cumw;
    K.runs = P.runs;
    K.chunks = P.chunks;
    K.pairs = d_xpairs;
    K.units = d_units_out;
    K.tasks = d_tasks_out;
    K.entries = d_entries;
    K.first = d_first;
    K.ntasks = (int32_t)ntasks;
    K.nentries = (int32_t)nent;
    K.npairs = npairs;
    K.entry_state = d_state;
    K.rq = d_rq;
    K.rq_log2 = rq_log2;
    K.rq_ctl = d_ctl;
    K.done_total = d_ctl + 2 * XTED_RINGS;
    K.stripes = d_st;
    K.nstriped = (int32_t)nstriped;
    K.smap = nstriped > 0 ? (const int32_t *)c->smap.p : nullptr;
    K.sbuf = nstriped > 0 ? (unsigned long long *)c->sbuf.p : nullptr;
    K.sbuf_words = stripe_buf;
    K.hold_pair = -1;
    c->d_trivial = d_trivial;
    c->plan_dt_elems = hs->dt_elems;
    c->plan_stack_rows = std::max(hs->stack_rows, 1);
    c->plan_max_wide = hs->max_wide;
    c->plan_cells = hs->cells;
    c->plan_cells_right = hs->cells_right;
    c->plan_levels_max = hs->levels_max;
    c->plan_units = nunits;
    return XTED_OK;
}

}  // namespace xted
