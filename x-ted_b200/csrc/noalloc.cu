// Allocation-free single-pair distance: xted_distance_noalloc.
//
// Some callers cannot allocate device memory at the moment they need a
// distance: a process whose HBM is already handed out to another allocator's
// pool (a serving process that reserved its memory up front), a checker that
// runs after an allocation has failed, or a latency-bound caller that cannot
// take the device-wide synchronisation that freeing memory implies. For them
// this file computes one pair entirely inside a fixed scratch arena that is
// part of the loaded module: no cudaMalloc, no cudaFree, no pinned host
// buffer, no host heap.
//
// The arena is shared by every call in the process on a device and keeps the
// last call's contents; a call clears only its status words and writes every
// other cell before reading it. The entry point is synchronous, so calls made
// one after another from one host thread are safe; calls that overlap on the
// GPU (two host threads at once) race on the arena and must be serialised by
// the caller. The first call on a device checks the device and looks up the
// arena's device address (the array's name is only a stand-in in host code),
// so that first call belongs before any stream capture. With CUDA's lazy
// module loading (the default since CUDA 12.2) that lookup is also what loads
// this module onto the device and commits the arena's 16 MiB, so "allocates
// nothing" holds from the second call on: a caller that hands its memory to a
// pool makes one warm-up call at start-up, before it does so. The caller's
// current device is restored before every return.
//
// Algorithm: the same right-path keyroot decomposition as the batched path
// (orl(v) = v + size(v) - 1 in preorder; keyroots = root and every child that
// is not a last child), tables processed by keyroot level
// kd(i0) + kd(j0) so that every tree-distance entry a table reads was written
// at a lower level. One block; each warp fills whole tables row by row, the
// in-row dependency resolved by a warp prefix-min scan.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>

#include "xted.h"

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kHeaderInts = 64;  // [0] status (0 = not finished, 1 = ok, <0 error), [1] distance
constexpr int64_t kArenaInts = (int64_t)XTED_NOALLOC_ARENA_BYTES / 4;
constexpr int kMaxDevices = 64;
constexpr int kInf = 0x3fffffff;

// The scratch arena: inputs, per-tree metadata, the tree-distance matrix and
// one forest table per active warp. Nothing in it needs to start at zero
// except the status word, which the host clears before each launch.
__device__ __align__(256) int32_t g_noalloc_arena[kArenaInts];

// Offsets (in int32 elements) of one tree's regions inside the arena.
struct TreeRegs {
    int64_t lab, off, idx;  // input copy
    int64_t size, inner, kf, krs, doff;  // derived
    int32_t n;
};

struct Layout {
    TreeRegs t[2];
    int64_t dt, tables, table_ints, end;
    int32_t warps;
};

int64_t align64(int64_t x) { return (x + 63) & ~(int64_t)63; }

// Lays out a pair (m, n >= 1) and picks how many warps get a forest table.
// Returns false when even one table does not fit.
bool plan_layout(int32_t m, int32_t n, Layout *L) {
    int64_t p = kHeaderInts;
    const int32_t sz[2] = {m, n};
    for (int s = 0; s < 2; s++) {
        TreeRegs &r = L->t[s];
        const int64_t k = sz[s];
        r.n = sz[s];
        r.lab = p; p = align64(p + k);
        r.off = p; p = align64(p + k + 1);
        r.idx = p; p = align64(p + std::max<int64_t>(k - 1, 1));
        r.size = p; p = align64(p + k);
        r.inner = p; p = align64(p + k);
        r.kf = p; p = align64(p + k);
        r.krs = p; p = align64(p + k);
        r.doff = p; p = align64(p + k + 3);
    }
    L->dt = p;
    p = align64(p + (int64_t)m * n);
    L->tables = p;
    L->table_ints = align64(((int64_t)m + 1) * ((int64_t)n + 1));
    const int64_t room = kArenaInts - p;
    if (room < L->table_ints) return false;
    L->warps = (int32_t)std::min<int64_t>(kWarps, room / L->table_ints);
    L->end = p + L->warps * L->table_ints;
    return true;
}

// Validates one preorder CSR tree and derives its metadata with one thread.
// A tree is accepted when its offsets are monotone with off[0] = 0,
// off[n] = n - 1, and the children of every node tile the node's preorder
// interval in order (first child v + 1, next child = previous + its size).
// Every index is range-checked before it is used. Writes size, inner (one
// less than the keyroot depth of a keyroot: the largest keyroot depth found
// strictly below the node, -1 if none), kf (keyroot flag) and the keyroots
// bucketed by depth (krs, doff). Returns the largest keyroot depth, or -1
// for a malformed tree.
__device__ int derive_tree(int32_t *A, const TreeRegs &r) {
    const int n = r.n;
    const int32_t *off = A + r.off, *idx = A + r.idx;
    int32_t *size = A + r.size, *inner = A + r.inner, *kf = A + r.kf, *krs = A + r.krs, *doff = A + r.doff;
    if (off[0] != 0 || off[n] != n - 1) return -1;
    for (int v = 0; v < n; v++)
        if (off[v + 1] < off[v]) return -1;
    for (int v = n - 1; v >= 0; v--) {
        int next = v + 1, best = -1;
        const int lo = off[v], hi = off[v + 1];
        for (int e = lo; e < hi; e++) {
            const int c = idx[e];
            if (c != next || c >= n) return -1;
            const bool last = e == hi - 1;
            kf[c] = last ? 0 : 1;
            best = max(best, last ? inner[c] : inner[c] + 1);
            next = c + size[c];
            if (next > n) return -1;
        }
        size[v] = next - v;
        inner[v] = best;
    }
    if (size[0] != n) return -1;
    kf[0] = 1;
    int maxd = 0;
    for (int v = 0; v < n; v++)
        if (kf[v]) maxd = max(maxd, inner[v] + 1);
    // counting sort by depth d = inner + 1: count at d + 2, inclusive prefix
    // (doff[d + 1] = start of depth d), scatter advancing doff[d + 1] to the
    // end of depth d, leaving doff[d] .. doff[d + 1] as depth d's range
    for (int d = 0; d <= maxd + 2; d++) doff[d] = 0;
    for (int v = 0; v < n; v++)
        if (kf[v]) doff[inner[v] + 3]++;
    for (int d = 1; d <= maxd + 2; d++) doff[d] += doff[d - 1];
    for (int v = 0; v < n; v++)
        if (kf[v]) krs[doff[inner[v] + 2]++] = v;
    return maxd;
}

// Forest table of the keyroot pair (i0, j0), rows from the bottom up.
// D is the warp's table: (size(i0) + 1) x (size(j0) + 1), local coordinates.
__device__ void fill_table(int32_t *A, const Layout &L, int i0, int j0, int32_t *D, int lane) {
    const TreeRegs &ra = L.t[0], &rb = L.t[1];
    const int32_t *szA = A + ra.size, *szB = A + rb.size, *la = A + ra.lab, *lb = A + rb.lab;
    int32_t *Dt = A + L.dt;
    const int n = rb.n;
    const int si = szA[i0], sj = szB[j0], ld = sj + 1;
    const int oi = i0 + si - 1, oj = j0 + sj - 1;
    for (int c = lane; c <= sj; c += 32) D[(int64_t)si * ld + c] = sj - c;
    for (int r = lane; r < si; r += 32) D[(int64_t)r * ld + sj] = si - r;
    __syncwarp();
    for (int r = si - 1; r >= 0; r--) {
        const int i = i0 + r;
        const int orl_i = i + szA[i] - 1;
        const bool left_i = orl_i == oi;
        const int lab_i = la[i];
        const int32_t *below = D + (int64_t)(r + 1) * ld;
        const int32_t *far = D + (int64_t)(orl_i + 1 - i0) * ld;
        int32_t *row = D + (int64_t)r * ld;
        int carry = (si - r) + sj;  // D[r][sj] + sj
        for (int chi = sj - 1; chi >= 0; chi -= 32) {
            const int c = chi - lane;
            int key = kInf;
            bool both = false;
            if (c >= 0) {
                const int j = j0 + c;
                const int orl_j = j + szB[j] - 1;
                both = left_i && orl_j == oj;
                int a = below[c] + 1;
                if (both) a = min(a, below[c + 1] + (lab_i != lb[j] ? 1 : 0));
                else a = min(a, Dt[(int64_t)i * n + j] + far[orl_j + 1 - j0]);
                key = a + c;
            }
            // lanes hold columns chi, chi-1, ...: a prefix over lanes is a suffix over columns
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, key, o);
                if (lane >= o) key = min(key, t);
            }
            if (c >= 0) {
                const int v = min(key, carry) - c;
                row[c] = v;
                if (both) Dt[(int64_t)i * n + j0 + c] = v;
            }
            carry = min(carry, __shfl_sync(0xffffffffu, key, 31));
        }
        __syncwarp();
    }
}

__global__ void __launch_bounds__(kThreads) xted_noalloc_kernel(int32_t *A, Layout L) {
    __shared__ int s_maxd[2], s_next, s_total;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (lane == 0 && warp < 2) s_maxd[warp] = derive_tree(A, L.t[warp]);
    __syncthreads();
    if (s_maxd[0] < 0 || s_maxd[1] < 0) {
        if (tid == 0) A[0] = XTED_EINVAL;
        return;
    }
    const int mA = s_maxd[0], mB = s_maxd[1];
    const int32_t *dA = A + L.t[0].doff, *dB = A + L.t[1].doff;
    const int32_t *kA = A + L.t[0].krs, *kB = A + L.t[1].krs;
    int32_t *D = A + L.tables + (int64_t)warp * L.table_ints;
    for (int lvl = 0; lvl <= mA + mB; lvl++) {
        const int a_lo = max(0, lvl - mB), a_hi = min(mA, lvl);
        if (tid == 0) {
            int total = 0;
            for (int a = a_lo; a <= a_hi; a++)
                total += (dA[a + 1] - dA[a]) * (dB[lvl - a + 1] - dB[lvl - a]);
            s_total = total;
            s_next = 0;
        }
        __syncthreads();
        if (warp < L.warps) {
            for (;;) {
                int k = 0;
                if (lane == 0) k = atomicAdd(&s_next, 1);
                k = __shfl_sync(0xffffffffu, k, 0);
                if (k >= s_total) break;
                int a = a_lo, na = 0, nb = 0;
                for (; a <= a_hi; a++) {
                    na = dA[a + 1] - dA[a];
                    nb = dB[lvl - a + 1] - dB[lvl - a];
                    if (k < na * nb) break;
                    k -= na * nb;
                }
                fill_table(A, L, kA[dA[a] + k / nb], kB[dB[lvl - a] + k % nb], D, lane);
            }
        }
        __syncthreads();
    }
    if (tid == 0) {
        A[1] = A[L.dt];  // the root pair's entry: Dt[0][0]
        A[0] = 1;
    }
}

// Per-device arena address, looked up once with that device current.
std::mutex g_setup_mu;
int32_t *g_arena_ptr[kMaxDevices];

int arena_for(int device, int32_t **out) {
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_arena_ptr[device]) {
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10) {
            cudaGetLastError();
            return XTED_ENODEV;
        }
        if (cudaSetDevice(device) != cudaSuccess) return XTED_ECUDA;
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_arena) != cudaSuccess || !p) {
            cudaGetLastError();
            return XTED_ECUDA;
        }
        g_arena_ptr[device] = (int32_t *)p;
    }
    *out = g_arena_ptr[device];
    return XTED_OK;
}

int copy_tree(int32_t *A, const TreeRegs &r, const xted_tree &t, cudaStream_t s) {
    const size_t n = (size_t)t.n;
    bool ok = cudaMemcpyAsync(A + r.lab, t.labels, 4 * n, cudaMemcpyHostToDevice, s) == cudaSuccess &&
              cudaMemcpyAsync(A + r.off, t.child_off, 4 * (n + 1), cudaMemcpyHostToDevice, s) == cudaSuccess;
    if (ok && n > 1) ok = cudaMemcpyAsync(A + r.idx, t.child_idx, 4 * (n - 1), cudaMemcpyHostToDevice, s) == cudaSuccess;
    return ok ? XTED_OK : XTED_ECUDA;
}

// Restores the calling thread's current device on scope exit (the entry
// point makes `device` current for its work, and must not leave it so).
struct DeviceRestore {
    int prev = -1;
    DeviceRestore() {
        if (cudaGetDevice(&prev) != cudaSuccess) {
            cudaGetLastError();
            prev = -1;
        }
    }
    ~DeviceRestore() {
        if (prev >= 0 && cudaSetDevice(prev) != cudaSuccess) cudaGetLastError();
    }
};

}  // namespace

extern "C" int xted_distance_noalloc(const xted_tree *a, const xted_tree *b, int32_t device, int32_t *out) {
    if (!a || !b || !out) return XTED_EINVAL;
    for (const xted_tree *t : {a, b}) {
        if (t->n < 0 || t->n > XTED_MAX_NODES) return XTED_EINVAL;
        if (t->n > 0 && (!t->labels || !t->child_off || (t->n > 1 && !t->child_idx))) return XTED_EINVAL;
    }
    Layout L;
    if (a->n > 0 && b->n > 0 && !plan_layout(a->n, b->n, &L)) return XTED_ETOOBIG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev || device >= kMaxDevices) {
        cudaGetLastError();
        return XTED_ENODEV;
    }
    const DeviceRestore restore;
    int32_t *A = nullptr;
    int rc = arena_for(device, &A);
    if (rc) return rc;
    // Empty trees follow standard_ted's rules (the distance is the other
    // tree's size); a non-empty partner is still validated, by running it
    // against a one-node tree.
    if (a->n == 0 || b->n == 0) {
        if (a->n == 0 && b->n == 0) {
            *out = 0;
            return XTED_OK;
        }
        const xted_tree *t = a->n ? a : b;
        const int32_t lab0 = 0, off1[2] = {0, 0};
        const xted_tree single{&lab0, off1, nullptr, 1};
        if (!plan_layout(t->n, 1, &L)) return XTED_ETOOBIG;
        int32_t d = 0;
        rc = xted_distance_noalloc(t, &single, device, &d);
        if (rc) return rc;
        *out = t->n;
        return XTED_OK;
    }
    if (cudaSetDevice(device) != cudaSuccess) return XTED_ECUDA;
    cudaGetLastError();  // drop a non-sticky error left by an earlier, unrelated runtime call on this thread
    cudaStream_t s = cudaStreamPerThread;
    if (cudaMemsetAsync(A, 0, 4 * kHeaderInts, s) != cudaSuccess) return XTED_ECUDA;
    rc = copy_tree(A, L.t[0], *a, s);
    if (!rc) rc = copy_tree(A, L.t[1], *b, s);
    if (rc) return rc;
    void *args[] = {&A, &L};
    if (cudaLaunchKernel((const void *)xted_noalloc_kernel, dim3(1), dim3(kThreads), args, 0, s) != cudaSuccess) {
        cudaGetLastError();
        return XTED_ECUDA;
    }
    int32_t res[2] = {0, 0};
    if (cudaMemcpyAsync(res, A, sizeof(res), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
        cudaGetLastError();
        return XTED_ECUDA;
    }
    if (res[0] == 1) {
        *out = res[1];
        return XTED_OK;
    }
    return res[0] < 0 ? res[0] : XTED_ECUDA;
}
