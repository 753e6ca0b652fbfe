// kernels.cu -- the keyroot-table dynamic program on sm_100a.
//
// One persistent kernel drains a device ready queue of tasks (see xted_internal.h).
// A task is one wide unit run by the whole 256-thread block, or up to eight
// narrow units, one per warp. A unit computes the forest tables of a run of
// A-keyroots against a chunk of B-segments, row by row from the bottom:
//
//   reference recurrence (X-TED_CPU/parallel_computing.cpp:17-43), with the
//   unit costs there generalised to del (a row-tree node), ins (a column-tree
//   node) and ren (a label change); the reference's costs are 1, 1, 1:
//     tree cell   D[i][j] = min(D[i+1][j+1] + ren*(l(i) != l(j)), D[i+1][j] + del,
//                               D[i][j+1] + ins),  Dtree[i][j] = D[i][j]
//     forest cell D[i][j] = min(Dtree[i][j] + D[orl(i)+1][orl(j)+1], D[i+1][j] + del,
//                               D[i][j+1] + ins)
//   with borders D[i][je] = (imax - i) del and D[imax][j] = (je - j) ins.
//
// Row formulation: with A[j] = min(first term, D[i+1][j] + del), row i is the
// min-plus suffix scan D[i][j] = min_{k >= j} (A[k] + (k - j) ins) closed by
// the border D[i][je]. Every column carries a key ins*c + BIG*seg, so one
// unsegmented suffix-min of A + key over a whole chunk yields every segment
// (table) at once: values from a later segment are at least BIG too large
// (the host admits a pair only while del*m + ins*n, a bound of every table
// value, stays below BIG).
// The row above (D[i+1][*]) lives in registers; rows that later rows will use
// as D[orl(i)+1][*] are pushed on a per-warp stack in global scratch (its
// depth is the number of keyroots on a root path). Dtree is read with
// ld.global.cg (L2), because other blocks write it during the launch.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/xted.h"
#include "xted_internal.h"

namespace xted {

#define FULLMASK 0xffffffffu

__device__ __forceinline__ int ld_acquire(const int32_t *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void set_error(const XKernelParams &P, int code, int a, int b, int c) {
    if (atomicCAS(P.error, 0, code) == 0) {
        P.error_info[0] = a;
        P.error_info[1] = b;
        P.error_info[2] = c;
    }
}

// Edit costs of a launch (XKernelParams c_del, c_ins, c_ren). The DP kernel
// is compiled twice more for them: UC (unit cost, the reference's) makes them
// compile-time ones, so the default path carries no cost registers.
struct Costs {
    int del, ins, ren;
};
template <bool UC>
__device__ __forceinline__ Costs costs_of(const XKernelParams &P) {
    return UC ? Costs{1, 1, 1} : Costs{P.c_del, P.c_ins, P.c_ren};
}

// Inclusive suffix minimum over the warp (lane l: min over lanes >= l). A lane
// whose source is out of range gets its own value back from shfl.down, which
// leaves the minimum unchanged, so no bounds test is needed.
__device__ __forceinline__ int warp_suffix_min(int v, int lane) {
    (void)lane;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) v = min(v, __shfl_down_sync(FULLMASK, v, d));
    return v;
}

__device__ __forceinline__ int warp_prefix_sum(int v, int lane) {
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        int o = __shfl_up_sync(FULLMASK, v, d);
        if (lane >= d) v += o;
    }
    return v;
}

// Shared rows (ring slots and stack rows) store column c at pad(c) = c + c/32:
// a thread owning W consecutive columns then reads and writes its k-th column
// in a different bank from every other lane of its warp (the plain layout put
// lanes W columns apart, a W-way bank conflict on every access).
__device__ __forceinline__ int pad(int c) { return c + (c >> 5); }

// Per-column state of one thread: W consecutive columns of the chunk.
// Columns past the chunk's end are inert: key KEY_INVALID lifts their scan
// values above every real one, and their inputs (zeroed shared memory or old
// distances, never negative) keep them bounded.
#define KEY_INVALID 0x20000000
#define NOSEG 0x40000000
template <int W>
struct Cols {
    int node[W], lab[W], key[W];
    int fb[W];      // je - orl(j) - 1: far value on the table's right path (0: a tree column)
    int fidx[W];    // padded stack index of the far column orl(j)+1
    int segor[W];   // 0 at a segment's last column, NOSEG elsewhere (min(A, (bord+1) | segor))
    int dend[W];    // je - j: the table's bottom border, the first row above
    unsigned far;   // bit k: column k is a far column (pushed with stack rows)
    unsigned tcol;  // bit k: column k is on its segment's right path
    unsigned valid; // bit k: column k exists
};

// Loads the thread's columns [c0, c0+W) of a chunk: finds the segment of
// column c0 by binary search over the segments' column positions, then walks
// the keyroots' subtrees, deriving each column from the column tree's node
// records (label, orl, previous-node-is-leaf flag).
template <int W>
__device__ __forceinline__ void load_cols(const XKernelParams &P, const XPair &pr, const XChunk &ch, int c0,
                                          Cols<W> &C, int row_max) {
    C.far = 0;
    C.tcol = 0;
    C.valid = 0;
    const int2 *nodes = P.rowinfo + pr.col_base;
    int s = ch.k_lo, j = 0, j0 = 0, je = 0;
    if (c0 < ch.width) {
        const int32_t pos0 = P.cumw[ch.k_lo] + c0;
        int lo = ch.k_lo, hi = ch.k_lo + ch.nseg - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (P.cumw[mid] <= pos0) lo = mid;
            else hi = mid - 1;
        }
        s = lo;
        j0 = P.krd[s];
        je = (nodes[j0].y & XTED_ROW_ORL_MASK) + 1;
        j = j0 + (pos0 - P.cumw[s]);
    }
#pragma unroll
    for (int k = 0; k < W; k++) {
        const int c = c0 + k;
        if (c < ch.width) {
            if (j >= je) {
                s++;
                j0 = P.krd[s];
                je = (nodes[j0].y & XTED_ROW_ORL_MASK) + 1;
                j = j0;
            }
            const int2 nd = nodes[j];
            const int foff = (nd.y & XTED_ROW_ORL_MASK) + 1 - j;
            C.node[k] = j;
            C.lab[k] = nd.x;
            C.dend[k] = je - j;
            C.fb[k] = je - j - foff;
            C.fidx[k] = pad(min(c + foff, row_max));
            C.segor[k] = je - j == 1 ? 0 : NOSEG;
            if (j > j0 && (nd.y & XTED_ROW_PREVLEAF)) C.far |= 1u << k;
            if (je - j == foff) C.tcol |= 1u << k;
            C.valid |= 1u << k;
            j++;
        } else {
            C.node[k] = 0;
            C.lab[k] = 0;
            C.dend[k] = 2;
            C.fb[k] = 1;
            C.fidx[k] = pad(min(c, row_max));
            C.segor[k] = NOSEG;
        }
    }
}

template <int W>
__device__ __forceinline__ int count_ends(const Cols<W> &C) {
    int e = 0;
#pragma unroll
    for (int k = 0; k < W; k++) e += ((C.valid >> k) & 1u) && C.segor[k] == 0;
    return e;
}

template <int W>
__device__ __forceinline__ void set_keys(Cols<W> &C, int c0, int before, int ins) {
    int seg = before;
#pragma unroll
    for (int k = 0; k < W; k++) {
        const bool v = (C.valid >> k) & 1u;
        C.key[k] = v ? (c0 + k) * ins + XTED_KEY_BIG * seg : KEY_INVALID;
        if (v && C.segor[k] == 0) seg++;
    }
}

// Row step, forest rows (row i off its table's right path: the common case).
// Every cell is a forest cell: a = Dtree + far value, far from the stack top
// (or the table's border row for a column on its segment's right path).
// Returns the thread's suffix minimum; loc[k] = minimum over its columns >= k.
template <int W>
__device__ __forceinline__ int row_forest(const Cols<W> &C, const int (&prev)[W], const int32_t *slot,
                                          const int32_t *top, int bord1, int rowfar, int del, int (&loc)[W]) {
    int cur[W], farv[W];
#pragma unroll
    for (int k = 0; k < W; k++) {
        cur[k] = slot[k];
        farv[k] = top[C.fidx[k]];
    }
    int run = XTED_INF;
#pragma unroll
    for (int k = W - 1; k >= 0; k--) {
        const int far = ((C.tcol >> k) & 1u) ? rowfar : farv[k];
        int A = __viaddmin_s32(prev[k], del, cur[k] + far);  // min(up + del, forest term)
        A = min(A, bord1 | C.segor[k]);                       // a segment's last column meets the border
        run = __viaddmin_s32(A, C.key[k], run);             // min(A + key, run)
        loc[k] = run;
    }
    return run;
}

// Row step, tree-path rows (row i on its table's right path): tree cells on
// the segments' right paths, forest cells elsewhere with the far value of the
// table's bottom border. bord = D[i][je] = (imax - i) del.
template <int W>
__device__ __forceinline__ int row_tree(const Cols<W> &C, const int (&prev)[W], const int32_t *slot, int dnext,
                                        int rl, int bord, Costs K, int (&loc)[W]) {
    int cur[W];
#pragma unroll
    for (int k = 0; k < W; k++) cur[k] = slot[k];
    const int bord1 = bord + K.ins;
    int run = XTED_INF;
#pragma unroll
    for (int k = W - 1; k >= 0; k--) {
        const int diag = C.segor[k] == 0 ? bord - K.del : ((k == W - 1) ? dnext : prev[k + 1]);
        const int a = ((C.tcol >> k) & 1u) ? diag + (rl != C.lab[k] ? K.ren : 0) : cur[k] + C.fb[k] * K.ins;
        int A = __viaddmin_s32(prev[k], K.del, a);
        A = min(A, bord1 | C.segor[k]);
        run = __viaddmin_s32(A, C.key[k], run);
        loc[k] = run;
    }
    return run;
}

// ---------------------------------------------------------------------------
// Row prefetch. Tree distances of the rows a unit will reach next do not
// depend on the unit's own work (they were written at lower levels), so each
// thread keeps XTED_PREFETCH rows of its columns in flight with cp.async into
// a shared-memory ring, plus the row's node record (copied by one thread).
// L1-allocating copies are safe here: every task starts after an acquire of
// its pair's counter and a block barrier, the pattern grid-wide sync relies on.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async4(int32_t *smem, const int32_t *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Far-row stack: the top XTED_STACK_CACHE rows of every unit's stack live in
// shared memory (a ring indexed by stack position); rows are also written to
// the global stack only when a unit can nest deeper than that, and a row that
// falls out of the window is reloaded from there when the stack unwinds.
#define XTED_STACK_CACHE 8
#define NARROW_ROW (XTED_NARROW_MAX + XTED_NARROW_MAX / 32)     // 264 ints
#define WIDE_ROW (XTED_WIDE_REG_MAX + XTED_WIDE_REG_MAX / 32)   // 2112 ints
#define NARROW_SLOT (NARROW_ROW + 8)  // ring slot: padded columns, then the row record (8-byte aligned)
#define WIDE_SLOT (WIDE_ROW + 8)
#define RING_INTS ((XTED_WARPS * XTED_PREFETCH * NARROW_SLOT) > (XTED_PREFETCH * WIDE_SLOT) \
                       ? (XTED_WARPS * XTED_PREFETCH * NARROW_SLOT)                          \
                       : (XTED_PREFETCH * WIDE_SLOT))
#define CACHE_INTS (XTED_STACK_CACHE * WIDE_ROW)  // = warps x depth x padded narrow row
static_assert(CACHE_INTS == XTED_WARPS * XTED_STACK_CACHE * NARROW_ROW, "stack cache split");
#define CNODE_INTS XTED_WIDE_REG_MAX  // = warps x narrow width: node ids of the unit's columns
#define DP_SMEM_BYTES ((RING_INTS + CACHE_INTS + CNODE_INTS) * 4)

// Issues the copies of row r. Copies are coalesced: thread `me` of `nthr`
// copies columns me, me + nthr, ... (node ids from the unit's shared column
// table), so consecutive lanes read consecutive tree distances; one thread
// also copies the row's node record. The thread that computes a column is not
// the one that copied it, so a row is read only after a barrier that follows
// every copier's wait. (Each thread copying its own W columns, from node ids
// in registers, issues fewer instructions but makes each warp-wide copy touch
// W lines instead of one; it measured 4% slower on the mixed batch.)
template <int W>
__device__ __forceinline__ void issue_row(const int32_t *cnode, int width, const int32_t *dt, int n,
                                          const int2 *rows, int r, int32_t *slot, int rec_at, int me, int nthr,
                                          bool rec) {
    const int32_t *drow = dt + (int64_t)r * n;
#pragma unroll
    for (int j = 0; j < W; j++) {
        const int c = me + j * nthr;
        if (c < width) cp_async4(slot + pad(c), drow + cnode[c]);
    }
    if (rec) cp_async8(slot + rec_at, rows + r);
}

// The same copies with the thread's copy plan held in registers for the whole
// unit: cpn[j] is the column tree's node of column me + nthr j (nthr = 32 G,
// G warps), bit j of cpm says that column exists, and the column's padded
// place in the slot is pbase + (nthr + G) j with pbase = pad(me). Per row this
// leaves one address and one copy per column.
template <int W, int G>
__device__ __forceinline__ void issue_row_planned(const int (&cpn)[W], unsigned cpm, int pbase, const int32_t *dt,
                                                  int n, const int2 *rows, int r, int32_t *slot, int rec_at,
                                                  bool rec) {
    const int32_t *drow = dt + (int64_t)r * n;
#pragma unroll
    for (int j = 0; j < W; j++)
        if ((cpm >> j) & 1u) cp_async4(slot + pbase + (32 * G + G) * j, drow + cpn[j]);
    if (rec) cp_async8(slot + rec_at, rows + r);
}

// ---------------------------------------------------------------------------
// Narrow unit: one warp, chunk width <= 32*W.
// ---------------------------------------------------------------------------
// Keyroots [kr_start, run end) of the unit. With `yield` set, the warp stops
// between two keyroot tables once *yield is no longer FLOW_RUN (its block is
// gathering for a group task) and returns the next keyroot; the tables of a
// run are independent, so the rest runs later from there. Returns -1 when
// the unit is done.
template <int W, bool UC>
__device__ int run_narrow(const XKernelParams &P, const XPair &pr, const XUnit &u, int lane, int32_t *stk,
                          int32_t *ring, int32_t *cache, int32_t *cnode, int kr_start, const volatile int *yield) {
    const XRun run = P.runs[u.run];
    const XChunk ch = P.chunks[u.chunk];
    const int c0 = lane * W;
    const int width = ch.width;
    const Costs K = costs_of<UC>(P);
    Cols<W> C;
    // the stack window holds rows of 32 W columns (padded: 33 W ints), so
    // narrower units keep more rows of it in the warp's shared memory
    constexpr int CROW = 33 * W, SC0 = XTED_STACK_CACHE * NARROW_ROW / CROW;
    constexpr int SC = SC0 >= 32 ? 32 : SC0 >= 16 ? 16 : XTED_STACK_CACHE;
    static_assert(SC * CROW <= XTED_STACK_CACHE * NARROW_ROW, "narrow stack window");
    load_cols<W>(P, pr, ch, c0, C, 32 * W - 1);
    __syncwarp();  // the previous unit's copies have drained (cp_async_wait<0> at its end)
#pragma unroll
    for (int k = 0; k < W; k++)
        if ((C.valid >> k) & 1u) cnode[c0 + k] = C.node[k];
    __syncwarp();
    // this lane's copy plan (nodes of columns lane + 32 j) in registers; the
    // widest units keep reading it from the shared column table (registers)
    constexpr bool PLAN = W <= 4;
    int cpn[W];
    unsigned cpm = 0;
#pragma unroll
    for (int j = 0; j < W && PLAN; j++) {
        const int c = lane + 32 * j;
        cpn[j] = c < width ? cnode[c] : 0;
        if (c < width) cpm |= 1u << j;
    }
    {
        const int e = count_ends<W>(C);
        const int incl = warp_prefix_sum(e, lane);
        set_keys<W>(C, c0, incl - e, K.ins);
    }
    const int n = pr.n;
    const int32_t *dt_in = P.dt + pr.dt_off;
    int32_t *dt_out = P.dt + pr.dt_off;
    const int2 *rows = P.rowinfo + pr.row_base;
    const int stride = XTED_NARROW_MAX;
    const int pbase = pad(c0);  // pad(c0 + k) == pbase + k for k < W (W divides 32)
    constexpr int PF = XTED_PREFETCH;
    // a table at keyroot depth d nests at most d stack rows (nested keyroots have
    // strictly smaller depths), so only deep runs need the global copy of the stack
    const bool deep = run.depth > SC;
    const int stack_rows = P.stack_rows;

    for (int kr = kr_start < 0 ? run.kr_lo : kr_start; kr < run.kr_hi; kr++) {
        if (yield && kr > run.kr_lo && kr != kr_start) {
            int y = 0;
            if (lane == 0) y = *yield != 0;  // FLOW_RUN == 0
            if (__shfl_sync(FULLMASK, y, 0)) {
                cp_async_wait<0>();
                return kr;
            }
        }
        const int i0 = P.krd[kr];
        const int imax = (rows[i0].y & XTED_ROW_ORL_MASK) + 1;
        int prev[W];
#pragma unroll
        for (int k = 0; k < W; k++) prev[k] = C.dend[k] * K.ins;
        int sp = 0, lo = 0;  // stack depth; lowest position held in the shared window
        __syncwarp();  // the ring's previous readers are done
#pragma unroll
        for (int q = 0; q < PF - 1; q++) {
            const int r = imax - 1 - q;
            if (r >= i0) {
                if (PLAN)
                    issue_row_planned<W, 1>(cpn, cpm, lane, dt_in, n, rows, r, ring + (r & (PF - 1)) * NARROW_SLOT,
                                            NARROW_ROW, lane == 0);
                else
                    issue_row<W>(cnode, width, dt_in, n, rows, r, ring + (r & (PF - 1)) * NARROW_SLOT, NARROW_ROW,
                                 lane, 32, lane == 0);
            }
            cp_async_commit();
        }
        for (int i = imax - 1; i >= i0; i--) {
            {
                const int r = i - (PF - 1);
                if (r >= i0) {
                    if (PLAN)
                        issue_row_planned<W, 1>(cpn, cpm, lane, dt_in, n, rows, r,
                                                ring + (r & (PF - 1)) * NARROW_SLOT, NARROW_ROW, lane == 0);
                    else
                        issue_row<W>(cnode, width, dt_in, n, rows, r, ring + (r & (PF - 1)) * NARROW_SLOT,
                                     NARROW_ROW, lane, 32, lane == 0);
                }
                cp_async_commit();
            }
            cp_async_wait<PF - 1>();
            __syncwarp();
            const int32_t *slot = ring + (i & (PF - 1)) * NARROW_SLOT;
            const int2 ri = *(const int2 *)(slot + NARROW_ROW);
            const int ro = ri.y & XTED_ROW_ORL_MASK;
            const bool trow = ro == imax - 1;
            const int bord = (imax - i) * K.del;
            int loc[W];
            int mine;
            if (!trow) {
                const int32_t *top = cache + ((sp > 0 ? sp - 1 : 0) & (SC - 1)) * CROW;
                mine = row_forest<W>(C, prev, slot + pbase, top, bord + K.ins, (imax - ro - 1) * K.del, K.del, loc);
            } else {
                const int dnext = __shfl_down_sync(FULLMASK, prev[0], 1);
                mine = row_tree<W>(C, prev, slot + pbase, dnext, ri.x, bord, K, loc);
            }
            const int incl = warp_suffix_min(mine, lane);
            int carry = __shfl_down_sync(FULLMASK, incl, 1);
            if (lane == 31) carry = XTED_INF;
#pragma unroll
            for (int k = 0; k < W; k++) prev[k] = min(loc[k], carry) - C.key[k];
            if (trow) {
                int32_t *orow = dt_out + (int64_t)i * n;
#pragma unroll
                for (int k = 0; k < W; k++)
                    if ((C.tcol >> k) & 1u) orow[C.node[k]] = prev[k];
            }
            // every lane has read this row's stack top (its values fed the scan above)
            if (i != i0 && (ri.y & XTED_ROW_ISKR)) {
                sp--;
                if (sp > 0 && sp - 1 < lo) {  // the new top left the window: reload it
                    const int32_t *src = stk + (sp - 1) * stride + c0;
                    int32_t *dst = cache + ((sp - 1) & (SC - 1)) * CROW + pbase;
#pragma unroll
                    for (int k = 0; k < W; k++) dst[k] = src[k];
                    lo = sp - 1;
                }
            }
            if (i > i0 && (ri.y & XTED_ROW_PREVLEAF)) {
                if (sp < stack_rows) {
                    // whole rows: only far columns are ever read back, and the
                    // others (inert ones included) hold this row's bounded values
                    int32_t *dst = cache + (sp & (SC - 1)) * CROW + pbase;
#pragma unroll
                    for (int k = 0; k < W; k++) dst[k] = prev[k];
                    if (deep) {
                        int32_t *g = stk + sp * stride + c0;
#pragma unroll
                        for (int k = 0; k < W; k++) g[k] = prev[k];
                    }
                } else if (lane == 0) {
                    set_error(P, XTED_ENOMEM, 1, sp, stack_rows);
                }
                sp++;
                if (sp - lo > SC) lo = sp - SC;
            }
            __syncwarp();
        }
    }
    cp_async_wait<0>();
    return -1;
}

// ---------------------------------------------------------------------------
// Group unit: G warps (a half block, G = 4, or the whole block, G = 8), chunk
// width <= 32*G*W. The group's threads hold W consecutive columns each; a row
// is a suffix scan within each warp, then across the group's warps through
// shared memory, with the group's own named barrier.
// ---------------------------------------------------------------------------
struct __align__(16) WideShared {
    int wtot[XTED_WARPS];       // per-warp suffix minima of the current row
    int first[XTED_WARPS + 1];  // prev[0] of lane 0 of each warp (cross-warp diagonal)
    int ends[XTED_WARPS];
    int cin;                    // stripes: the right neighbour's carry for the current row
    int cinb[2], fcb[2];        // pipelined stripes: its carry and first column, by flat-row parity
};
static_assert(XTED_WARPS <= 32, "the warp minima are read one per lane");

template <int G>
__device__ __forceinline__ void group_sync(int gid) {
    if (G == XTED_WARPS) {
        __syncthreads();
    } else {
        // immediate barrier ids: the kernel then reserves only barriers 0-2
        if (gid == 0) asm volatile("bar.sync 1, %0;" ::"n"(32 * G) : "memory");
        else asm volatile("bar.sync 2, %0;" ::"n"(32 * G) : "memory");
    }
}

template <int W, int G, bool UC>
__device__ void run_group(const XKernelParams &P, const XPair &pr, const XUnit &u, int32_t *stk, WideShared &S,
                          int32_t *ring, int32_t *cache, int32_t *cnode, int gtid, int gid) {
    constexpr int GROW = 256 * G + 8 * G;  // padded row of 256*G columns
    constexpr int GSLOT = GROW + 8;        // ring slot: the row, then its record
    const int lane = gtid & 31, warp = gtid >> 5;
    const XRun run = P.runs[u.run];
    const XChunk ch = P.chunks[u.chunk];
    const int c0 = gtid * W;
    const int stride = ch.width;
    const int width = ch.width;
    const int pbase = pad(c0);  // pad(c0 + k) == pbase + k for k < W (W divides 32)
    constexpr int PF = XTED_PREFETCH;
    // stack window rows of 32 G W columns (33 G W ints padded): narrower units
    // keep more rows of it in the group's shared memory
    constexpr int CROW = 33 * G * W, SC0 = XTED_STACK_CACHE * GROW / CROW;
    constexpr int SC = SC0 >= 32 ? 32 : SC0 >= 16 ? 16 : XTED_STACK_CACHE;
    static_assert(SC * CROW <= XTED_STACK_CACHE * GROW, "group stack window");
    const bool deep = run.depth > SC;  // see run_narrow
    const int stack_rows = P.stack_rows;
    const Costs K = costs_of<UC>(P);
    Cols<W> C;
    load_cols<W>(P, pr, ch, c0, C, 32 * G * W - 1);
    group_sync<G>(gid);  // the group's previous unit is done with cnode and S
#pragma unroll
    for (int k = 0; k < W; k++)
        if ((C.valid >> k) & 1u) cnode[c0 + k] = C.node[k];
    group_sync<G>(gid);  // the whole column table is written
    // this thread's copy plan (nodes of columns gtid + 32 G j) in registers;
    // the widest units keep reading it from the shared column table
    constexpr bool PLAN = W <= 4;
    int cpn[W];
    unsigned cpm = 0;
#pragma unroll
    for (int j = 0; j < W && PLAN; j++) {
        const int c = gtid + 32 * G * j;
        cpn[j] = c < width ? cnode[c] : 0;
        if (c < width) cpm |= 1u << j;
    }
    {
        const int e = count_ends<W>(C);
        const int incl = warp_prefix_sum(e, lane);
        if (lane == 31) S.ends[warp] = incl;
        group_sync<G>(gid);
        int before = incl - e;
        for (int w = 0; w < warp; w++) before += S.ends[w];
        set_keys<W>(C, c0, before, K.ins);
    }
    const int n = pr.n;
    const int32_t *dt_in = P.dt + pr.dt_off;
    int32_t *dt_out = P.dt + pr.dt_off;
    const int2 *rows = P.rowinfo + pr.row_base;

    for (int kr = run.kr_lo; kr < run.kr_hi; kr++) {
        const int i0 = P.krd[kr];
        const int imax = (rows[i0].y & XTED_ROW_ORL_MASK) + 1;
        int prev[W];
#pragma unroll
        for (int k = 0; k < W; k++) prev[k] = C.dend[k] * K.ins;
        int sp = 0, lo = 0;  // stack depth; lowest position held in the shared window
        group_sync<G>(gid);  // the ring's and S.first's previous readers are done
        if (lane == 0) S.first[warp] = prev[0];
        if (gtid == 0) S.first[G] = 0;
#pragma unroll
        for (int q = 0; q < PF - 1; q++) {
            const int r = imax - 1 - q;
            if (r >= i0) {
                if (PLAN)
                    issue_row_planned<W, G>(cpn, cpm, gtid + warp, dt_in, n, rows, r, ring + (r & (PF - 1)) * GSLOT,
                                            GROW, gtid == 0);
                else
                    issue_row<W>(cnode, width, dt_in, n, rows, r, ring + (r & (PF - 1)) * GSLOT, GROW, gtid, 32 * G,
                                 gtid == 0);
            }
            cp_async_commit();
        }
        cp_async_wait<PF - 2>();
        group_sync<G>(gid);
        for (int i = imax - 1; i >= i0; i--) {
            {
                const int r = i - (PF - 1);
                if (r >= i0) {
                    if (PLAN)
                        issue_row_planned<W, G>(cpn, cpm, gtid + warp, dt_in, n, rows, r,
                                                ring + (r & (PF - 1)) * GSLOT, GROW, gtid == 0);
                    else
                        issue_row<W>(cnode, width, dt_in, n, rows, r, ring + (r & (PF - 1)) * GSLOT, GROW, gtid,
                                     32 * G, gtid == 0);
                }
                cp_async_commit();
            }
            const int32_t *slot = ring + (i & (PF - 1)) * GSLOT;
            const int2 ri = *(const int2 *)(slot + GROW);
            const int ro = ri.y & XTED_ROW_ORL_MASK;
            const bool trow = ro == imax - 1;
            const int bord = (imax - i) * K.del;
            int loc[W];
            int mine;
            if (!trow) {
                const int32_t *top = cache + ((sp > 0 ? sp - 1 : 0) & (SC - 1)) * CROW;
                mine = row_forest<W>(C, prev, slot + pbase, top, bord + K.ins, (imax - ro - 1) * K.del, K.del, loc);
            } else {
                int dnext = __shfl_down_sync(FULLMASK, prev[0], 1);
                if (lane == 31) dnext = S.first[warp + 1];
                mine = row_tree<W>(C, prev, slot + pbase, dnext, ri.x, bord, K, loc);
            }
            const int incl = warp_suffix_min(mine, lane);
            if (lane == 0) S.wtot[warp] = incl;
            group_sync<G>(gid);
            int carry = __shfl_down_sync(FULLMASK, incl, 1);
            if (lane == 31) carry = XTED_INF;
            {
                // minimum of the warps to the right: lane w reads warp w's row
                // minimum, then one warp-wide reduction
                const int mv = (lane > warp && lane < G) ? S.wtot[lane] : XTED_INF;
                carry = min(carry, __reduce_min_sync(FULLMASK, mv));
            }
            int32_t *orow = dt_out + (int64_t)i * n;
#pragma unroll
            for (int k = 0; k < W; k++) prev[k] = min(loc[k], carry) - C.key[k];
            if (trow) {
#pragma unroll
                for (int k = 0; k < W; k++)
                    if ((C.tcol >> k) & 1u) orow[C.node[k]] = prev[k];
            }
            if (lane == 0) S.first[warp] = prev[0];
            if (i != i0 && (ri.y & XTED_ROW_ISKR)) {
                sp--;
                if (sp > 0 && sp - 1 < lo) {  // the new top left the window: reload it
                    const int32_t *src = stk + (int64_t)(sp - 1) * stride + c0;
                    int32_t *dst = cache + ((sp - 1) & (SC - 1)) * CROW + pbase;
#pragma unroll
                    for (int k = 0; k < W; k++)
                        if ((C.far >> k) & 1u) dst[k] = src[k];
                    lo = sp - 1;
                }
            }
            if (i > i0 && (ri.y & XTED_ROW_PREVLEAF)) {
                if (sp < stack_rows) {
                    int32_t *dst = cache + (sp & (SC - 1)) * CROW + pbase;
#pragma unroll
                    for (int k = 0; k < W; k++) dst[k] = prev[k];  // whole rows in shared memory, as in run_narrow
                    if (deep) {
                        int32_t *g = stk + (int64_t)sp * stride + c0;
#pragma unroll
                        for (int k = 0; k < W; k++)
                            if ((C.far >> k) & 1u) g[k] = prev[k];
                    }
                } else if (gtid == 0) {
                    set_error(P, XTED_ENOMEM, 2, sp, stack_rows);
                }
                sp++;
                if (sp - lo > SC) lo = sp - SC;
            }
            cp_async_wait<PF - 2>();  // row i-1 has landed (this thread's copies)
            group_sync<G>(gid);       // ... and everyone's, the record and the stack push
        }
    }
    cp_async_wait<0>();
}

// ---------------------------------------------------------------------------
// Stripe s of a striped unit: columns [C0, C1) = [SW s, min(SW (s+1), w)),
// SW = 256 W, of a single column segment of width w, on the whole block (W
// columns per thread), concurrently with the unit's other stripes on other
// blocks (or after them on this one). It is run_group's row step with three
// additions:
//   * the row's suffix minimum continues from the right: before the scan
//     barrier the block waits for its right neighbour to finish the row and
//     takes that stripe's carry (its minimum of A[k] + k over k >= C1);
//   * a far column to the right of the stripe (f = orl(j)+1 >= C1) is read
//     from the exported values of its owner, kept per pushed row (the owner
//     is ahead, and its stack slot may since hold another row);
//   * the tree rows' diagonal at the last column is the right neighbour's
//     first column one row below.
// Everything a stripe hands to another is a 64-bit word (flat row + 1) << 32
// | value, written with one relaxed store: its carry and first column per row
// (for the stripe to its left), and its exported columns on pushed rows (for
// any stripe to its left). A reader checks the tag, so it needs no fence and
// no progress counter: it loads the word early (the latency hides behind the
// row's own work) and waits only if the tag is not there yet. The unit's
// buffer is zeroed before every run. A stripe waits only for stripes to its
// right, claimed before it (stripes are tasks, rightmost first), which wait
// for nobody to their left; the waits are bounded by the launch's timeout.
// PIPED (tables with many rows per stripe): thread 0 loads the neighbour's
// words of the NEXT flat row when a row starts and takes them at its end
// (into S.cinb / S.fcb by row parity), so the round trip of the load leaves
// the row's critical path; a stripe then stays a row behind its neighbour,
// and a thread whose far column is exported by a stripe to the right loads
// the next row's value after the scan barrier, a row before it is used. The
// cost is a row of pipeline fill per stripe, which short tables do not repay.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long ld_tagged(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ void st_tagged(unsigned long long *p, unsigned tag, int value) {
    asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(((unsigned long long)tag << 32) | (unsigned)value));
}
// The value of the word at p once it carries `tag` (XTED_INF after an error
// or the timeout); called only when an early load missed.
__device__ __forceinline__ int wait_tagged(const XKernelParams &P, const unsigned long long *p, unsigned tag) {
    const uint64_t t0 = global_ns();
    for (long it = 0; it < (1L << 26); it++) {
        const unsigned long long v = ld_tagged(p);
        if ((unsigned)(v >> 32) == tag) return (int)(unsigned)v;
        if (*(volatile int32_t *)P.error != 0) return XTED_INF;
        if (global_ns() - t0 > P.timeout_ns) break;
        __nanosleep(32);
    }
    set_error(P, XTED_ETIMEOUT, 10, (int)tag, 0);
    return XTED_INF;
}
__device__ __forceinline__ int tagged_value(const XKernelParams &P, const unsigned long long *p, unsigned long long v,
                                            unsigned tag) {
    return (unsigned)(v >> 32) == tag ? (int)(unsigned)v : wait_tagged(P, p, tag);
}

template <int W, bool UC, bool PIPED>
__device__ void run_stripe(const XKernelParams &P, const XPair &pr, const XUnit &u, int32_t *stk, WideShared &S,
                           int32_t *ring, int32_t *cache, int32_t *cnode, int s, int K, int X, int R,
                           const int32_t *expmap, unsigned long long *CR, unsigned long long *FC,
                           unsigned long long *E) {
    constexpr int G = XTED_WARPS, SW = XTED_CTA_THREADS * W;  // stripe width: W columns per thread
    // the ring and the stack window hold stripe rows only (SW columns):
    // narrow stripes keep more rows in the same shared memory (at 512 columns
    // 8 rows in flight and a 32-row window of the far-row stack, so a deep
    // table rarely reloads a stack row from global memory)
    constexpr int SROW = SW + SW / 32, SSLOT = SROW + 8;
    constexpr int PF = 8 * SSLOT <= RING_INTS ? 8 : 4 * SSLOT <= RING_INTS ? 4 : 2;
    static_assert(PF * SSLOT <= RING_INTS, "stripe ring");
    constexpr int SC = 32 * SROW <= CACHE_INTS ? 32 : 16 * SROW <= CACHE_INTS ? 16 : XTED_STACK_CACHE;
    static_assert(SC * SROW <= CACHE_INTS, "stripe stack window");
    // the exported-value prefetch reads the next row's record, so rows i and
    // i-1 must have landed when row i runs: one row less in flight
    constexpr bool XPF = PIPED && PF >= 4;
    constexpr int WAITN = XPF ? PF - 3 : PF - 2;
    const int gtid = threadIdx.x, lane = gtid & 31, warp = gtid >> 5;
    const XRun run = P.runs[u.run];
    const XChunk ch = P.chunks[u.chunk];
    const int w = ch.width;
    const int C0 = s * SW, C1 = min(C0 + SW, w);
    const bool right = s + 1 < K, left = s > 0;
    const int lc0 = gtid * W, c0 = C0 + lc0;  // this thread's first column: local, in the segment
    const int pbase = pad(lc0);
    const bool deep = run.depth > SC;
    const int stack_rows = P.stack_rows;
    const Costs KC = costs_of<UC>(P);
    Cols<W> C;
    load_cols<W>(P, pr, ch, c0, C, w - 1);
    // this thread's columns that stripes to the left read as far columns, and
    // the export index of the first of them (exports are numbered in column
    // order, so the k-th is ebase + the exported columns before it)
    unsigned expm = 0;
    int ebase = -1;
#pragma unroll
    for (int k = 0; k < W; k++) {
        const int c = c0 + k;
        if (c >= C1) {  // past the stripe: an inert column
            C.valid &= ~(1u << k);
            C.far &= ~(1u << k);
            C.tcol &= ~(1u << k);
            C.node[k] = 0;
            C.lab[k] = 0;
            C.dend[k] = 2;
            C.fb[k] = 1;
            C.segor[k] = NOSEG;
            C.fidx[k] = pad(min(lc0 + k, SW - 1));
        } else {
            const int f = c + (C.dend[k] - C.fb[k]);  // orl(j)+1 in segment columns
            if (f >= w) C.fidx[k] = pad(lc0 + k);     // the border: a tree-path column (rowfar)
            else if (f < C1) C.fidx[k] = pad(f - C0);
            else C.fidx[k] = -1 - __ldcg(&expmap[f]);  // exported by a stripe to the right
            const int ex = __ldcg(&expmap[c]);
            if (ex >= 0) {
                if (ebase < 0) ebase = ex;
                expm |= 1u << k;
            }
        }
    }
    unsigned xfar = 0;  // bit k: column k's far column is exported by a stripe to the right (prefetched)
#pragma unroll
    for (int k = 0; k < W; k++)
        if (XPF && !((C.tcol >> k) & 1u) && C.fidx[k] < 0) xfar |= 1u << k;
    __syncthreads();  // the block's previous unit is done with cnode and S
#pragma unroll
    for (int k = 0; k < W; k++)
        if ((C.valid >> k) & 1u) cnode[lc0 + k] = C.node[k];
    set_keys<W>(C, c0, 0, KC.ins);  // one segment: key = ins * segment column
    // this thread's copy plan: one segment, so column c is node j0 + C0 + c
    constexpr bool PLAN = W <= 4;
    int cpn[W];
    unsigned cpm = 0;
    {
        const int jc = P.krd[ch.k_lo] + C0;
#pragma unroll
        for (int j = 0; j < W && PLAN; j++) {
            const int c = gtid + SW * j / W;  // columns gtid + 256 j
            cpn[j] = jc + c;
            if (c < C1 - C0) cpm |= 1u << j;
        }
    }
    const int n = pr.n;
    const int32_t *dt_in = P.dt + pr.dt_off;
    int32_t *dt_out = P.dt + pr.dt_off;
    const int2 *rows = P.rowinfo + pr.row_base;
    const unsigned long long *cr_right = CR + (int64_t)(s + 1) * R, *fc_right = FC + (int64_t)(s + 1) * R;
    unsigned long long *cr_mine = CR + (int64_t)s * R, *fc_mine = FC + (int64_t)s * R;
    int tflat = 0, fc_next = 0;
    if (PIPED && gtid == 0) {  // flat row 0's words; the rightmost stripe's carry stays infinite
        S.cinb[0] = right ? wait_tagged(P, cr_right, 1u) : XTED_INF;
        S.cinb[1] = XTED_INF;
        S.fcb[0] = right ? wait_tagged(P, fc_right, 1u) : 0;
    }
    for (int kr = run.kr_lo; kr < run.kr_hi; kr++) {
        const int i0 = P.krd[kr];
        const int imax = (rows[i0].y & XTED_ROW_ORL_MASK) + 1;
        const int tbase = tflat;
        int prev[W];
#pragma unroll
        for (int k = 0; k < W; k++) prev[k] = C.dend[k] * KC.ins;
        int sp = 0, lo = 0;
        int pf_efl = -1;  // flat far row whose exported values pfw holds
        unsigned long long pfw[W];
#pragma unroll
        for (int k = 0; k < W; k++) pfw[k] = 0;
        __syncthreads();  // the ring's and S's previous readers are done
        if (lane == 0) S.first[warp] = prev[0];
        if (gtid == 0) S.first[G] = right ? (w - C1) * KC.ins : 0;  // D[imax][C1]: the bottom border
#pragma unroll
        for (int q = 0; q < PF - 1; q++) {
            const int r = imax - 1 - q;
            if (r >= i0) {
                if (PLAN)
                    issue_row_planned<W, G>(cpn, cpm, gtid + warp, dt_in, n, rows, r, ring + (r & (PF - 1)) * SSLOT,
                                            SROW, gtid == 0);
                else
                    issue_row<W>(cnode, C1 - C0, dt_in, n, rows, r, ring + (r & (PF - 1)) * SSLOT, SROW, gtid,
                                 32 * G, gtid == 0);
            }
            cp_async_commit();
        }
        cp_async_wait<WAITN>();
        __syncthreads();
        for (int i = imax - 1; i >= i0; i--, tflat++) {
            {
                const int r = i - (PF - 1);
                if (r >= i0) {
                    if (PLAN)
                        issue_row_planned<W, G>(cpn, cpm, gtid + warp, dt_in, n, rows, r,
                                                ring + (r & (PF - 1)) * SSLOT, SROW, gtid == 0);
                    else
                        issue_row<W>(cnode, C1 - C0, dt_in, n, rows, r, ring + (r & (PF - 1)) * SSLOT, SROW, gtid,
                                     32 * G, gtid == 0);
                }
                cp_async_commit();
            }
            // thread 0: the right neighbour's carry and first column of this
            // row, checked at the scan barrier (PIPED: of the next row, taken
            // at the end of this one)
            unsigned long long cw = 0, fw = 0;
            if (gtid == 0 && right && (!PIPED || tflat + 1 < R)) {
                cw = ld_tagged(cr_right + tflat + (PIPED ? 1 : 0));
                fw = ld_tagged(fc_right + tflat + (PIPED ? 1 : 0));
            }
            const int32_t *slot = ring + (i & (PF - 1)) * SSLOT;
            const int2 ri = *(const int2 *)(slot + SROW);
            const int ro = ri.y & XTED_ROW_ORL_MASK;
            const bool trow = ro == imax - 1;
            const int bord = (imax - i) * KC.del;
            int loc[W];
            int mine;
            if (!trow) {
                // forest row: far values from the stack top, or exported by the stripe that owns them
                const int32_t *top = cache + ((sp > 0 ? sp - 1 : 0) & (SC - 1)) * SROW;
                const int efl = tbase + (imax - 1 - (ro + 1));  // flat row of the far row
                const unsigned long long *erow = E + (int64_t)efl * X;
                const int32_t *cur = slot + pbase;
                const int rowfar = (imax - ro - 1) * KC.del, bord1 = bord + KC.ins;
                int run_min = XTED_INF;
#pragma unroll
                for (int k = W - 1; k >= 0; k--) {
                    int far;
                    if ((C.tcol >> k) & 1u) far = rowfar;
                    else if (C.fidx[k] >= 0) far = top[C.fidx[k]];
                    else {
                        const unsigned long long *ep = erow + (-1 - C.fidx[k]);
                        const unsigned long long v = ((xfar >> k) & 1u) && pf_efl == efl ? pfw[k] : ld_tagged(ep);
                        far = tagged_value(P, ep, v, (unsigned)efl + 1);
                    }
                    int A = __viaddmin_s32(prev[k], KC.del, cur[k] + far);
                    A = min(A, bord1 | C.segor[k]);
                    run_min = __viaddmin_s32(A, C.key[k], run_min);
                    loc[k] = run_min;
                }
                mine = run_min;
            } else {
                int dnext = __shfl_down_sync(FULLMASK, prev[0], 1);
                if (lane == 31) dnext = S.first[warp + 1];
                mine = row_tree<W>(C, prev, slot + pbase, dnext, ri.x, bord, KC, loc);
            }
            const int incl = warp_suffix_min(mine, lane);
            if (lane == 0) S.wtot[warp] = incl;
            if (!PIPED && gtid == 0) {
                int cin = XTED_INF;
                if (right) {
                    cin = tagged_value(P, cr_right + tflat, cw, (unsigned)tflat + 1);
                    fc_next = tagged_value(P, fc_right + tflat, fw, (unsigned)tflat + 1);
                }
                S.cin = cin;
            }
            __syncthreads();
            int carry = __shfl_down_sync(FULLMASK, incl, 1);
            if (lane == 31) carry = XTED_INF;
            {
                // minimum of the warps to the right (one warp-wide reduction) and
                // of the stripe to the right
                const int mv = (lane > warp && lane < G) ? S.wtot[lane] : XTED_INF;
                carry = min(carry, min(PIPED ? S.cinb[tflat & 1] : S.cin, __reduce_min_sync(FULLMASK, mv)));
            }
            if (XPF && xfar && i > i0) {  // the next row's exported far values (its record has landed)
                const int ron = ((const int2 *)(ring + ((i - 1) & (PF - 1)) * SSLOT + SROW))->y & XTED_ROW_ORL_MASK;
                if (ron != imax - 1) {
                    pf_efl = tbase + (imax - 1 - (ron + 1));
                    const unsigned long long *prow = E + (int64_t)pf_efl * X;
#pragma unroll
                    for (int k = 0; k < W; k++)
                        if ((xfar >> k) & 1u) pfw[k] = ld_tagged(prow + (-1 - C.fidx[k]));
                }
            }
            int32_t *orow = dt_out + (int64_t)i * n;
#pragma unroll
            for (int k = 0; k < W; k++) prev[k] = min(loc[k], carry) - C.key[k];
            if (trow) {
#pragma unroll
                for (int k = 0; k < W; k++)
                    if ((C.tcol >> k) & 1u) orow[C.node[k]] = prev[k];
            }
            if (lane == 0) S.first[warp] = prev[0];
            if (gtid == 0 && left) {  // for the left neighbour: carry at C0 and D[i][C0]
                st_tagged(cr_mine + tflat, (unsigned)tflat + 1, prev[0] + C.key[0]);
                st_tagged(fc_mine + tflat, (unsigned)tflat + 1, prev[0]);
            }
            if (i != i0 && (ri.y & XTED_ROW_ISKR)) {
                sp--;
                if (sp > 0 && sp - 1 < lo) {  // the new top left the window: reload it
                    const int32_t *src = stk + (int64_t)(sp - 1) * SW + lc0;
                    int32_t *dst = cache + ((sp - 1) & (SC - 1)) * SROW + pbase;
#pragma unroll
                    for (int k = 0; k < W; k++) dst[k] = src[k];
                    lo = sp - 1;
                }
            }
            if (i > i0 && (ri.y & XTED_ROW_PREVLEAF)) {
                if (sp < stack_rows) {
                    int32_t *dst = cache + (sp & (SC - 1)) * SROW + pbase;
#pragma unroll
                    for (int k = 0; k < W; k++) dst[k] = prev[k];
                    if (deep) {
                        int32_t *g = stk + (int64_t)sp * SW + lc0;
#pragma unroll
                        for (int k = 0; k < W; k++) g[k] = prev[k];
                    }
                } else if (gtid == 0) {
                    set_error(P, XTED_ENOMEM, 11, sp, stack_rows);
                }
                if (expm) {  // a pushed row is a far row: export the columns stripes to the left read
                    unsigned long long *erow = E + (int64_t)tflat * X;
#pragma unroll
                    for (int k = 0; k < W; k++)
                        if ((expm >> k) & 1u)
                            st_tagged(erow + ebase + __popc(expm & ((1u << k) - 1)), (unsigned)tflat + 1, prev[k]);
                }
                sp++;
                if (sp - lo > SC) lo = sp - SC;
            }
            // the next row's diagonal at C1: the right neighbour's first column of this row
            if (gtid == 0 && right) {
                if (!PIPED) {
                    S.first[G] = fc_next;
                } else {  // this row's first column, then the next row's words (slot (t+1)&1 is unread now)
                    S.first[G] = S.fcb[tflat & 1];
                    if (tflat + 1 < R) {
                        S.cinb[(tflat + 1) & 1] = tagged_value(P, cr_right + tflat + 1, cw, (unsigned)tflat + 2);
                        S.fcb[(tflat + 1) & 1] = tagged_value(P, fc_right + tflat + 1, fw, (unsigned)tflat + 2);
                    }
                }
            }
            cp_async_wait<WAITN>();  // row i-1 (with the prefetch: and i-2) has landed (this thread's copies)
            __syncthreads();         // ... and everyone's, the records and the stack push
        }
    }
    cp_async_wait<0>();
}

// A stripe task: stripe s of striped unit T.unit_lo, on the whole block. The
// unit's buffer holds every stripe's carries and first columns per row, then
// the exported far values per row, as tagged words.
template <bool UC>
__device__ void run_striped(const XKernelParams &P, const XPair &pr, const XTask &T, int32_t *stk, WideShared &S,
                            int32_t *ring, int32_t *cache, int32_t *cnode) {
    const XStripe X = P.stripes[T.unit_lo];
    const int s = (int)((T.kind_n >> XTED_STRIPE_SHIFT) & XTED_STRIPE_MASK);
    const XUnit u = P.units[X.unit];
    const int32_t *expmap = P.smap + X.map_off;
    unsigned long long *CR = P.sbuf + X.buf_off;
    unsigned long long *FC = CR + (int64_t)X.K * X.R;
    unsigned long long *E = FC + (int64_t)X.K * X.R;
    // a table with many rows per stripe pipelines the hand-off (a row of fill per stripe)
    if (X.sww == 2 && X.R >= XTED_STRIPE_PIPE_ROWS * X.K)
        run_stripe<2, UC, true>(P, pr, u, stk, S, ring, cache, cnode, s, X.K, X.X, X.R, expmap, CR, FC, E);
    else if (X.sww == 2)
        run_stripe<2, UC, false>(P, pr, u, stk, S, ring, cache, cnode, s, X.K, X.X, X.R, expmap, CR, FC, E);
    else if (X.sww == 4)
        run_stripe<4, UC, false>(P, pr, u, stk, S, ring, cache, cnode, s, X.K, X.X, X.R, expmap, CR, FC, E);
    else if (X.sww == 8)
        run_stripe<8, UC, false>(P, pr, u, stk, S, ring, cache, cnode, s, X.K, X.X, X.R, expmap, CR, FC, E);
    else if (threadIdx.x == 0)
        set_error(P, XTED_EINVAL, 13, X.sww, s);
}

template <bool UC>
__device__ int dispatch_narrow(const XKernelParams &P, const XPair &pr, const XUnit &u, int lane, int32_t *stk,
                               int32_t *ring, int32_t *cache, int32_t *cnode, int kr_start,
                               const volatile int *yield) {
    // Two columns per lane at the least: a one-column row loop would be one more
    // instantiation competing for the instruction cache for little gain.
    const int width = P.chunks[u.chunk].width;
    if (width <= 64) return run_narrow<2, UC>(P, pr, u, lane, stk, ring, cache, cnode, kr_start, yield);
    if (width <= 128) return run_narrow<4, UC>(P, pr, u, lane, stk, ring, cache, cnode, kr_start, yield);
    return run_narrow<8, UC>(P, pr, u, lane, stk, ring, cache, cnode, kr_start, yield);
}

// ---------------------------------------------------------------------------
// Wide unit wider than the register path (one segment of > 2048 columns):
// the same row step with the row above, the local minima and the far-row
// stack in block-private global scratch, on one block. Each thread owns
// `per` consecutive columns; the scratch rows are stored interleaved (a
// thread's k-th column at k * 256 + thread), so every access of the block's
// threads to their k-th columns is one coalesced line instead of 32 lines
// `per` columns apart.
// Scratch layout (Wp = per * 256): prev[Wp + 1] | loc[Wp] | column records
// (int4)[Wp] | stack[stack_rows][Wp]; the size is xted_wide_big_scratch().
// The segment's tree distances of a row (contiguous nodes) are staged in the
// block's shared memory by coalesced cp.async, the next row's while this one
// is computed when two rows fit, else row by row; wider segments read them
// straight from global memory.
// ---------------------------------------------------------------------------
template <bool UC>
__device__ void run_wide_big(const XKernelParams &P, const XPair &pr, const XUnit &u, int32_t *scr,
                             WideShared &S, int32_t *smem) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const XRun run = P.runs[u.run];
    const XChunk ch = P.chunks[u.chunk];
    const Costs K = costs_of<UC>(P);
    const int width = ch.width;
    const int per = (width + XTED_CTA_THREADS - 1) / XTED_CTA_THREADS;
    const int64_t Wp = (int64_t)per * XTED_CTA_THREADS;
    const int c0 = min(tid * per, width);
    const int c1 = min(c0 + per, width);
    const int nk = c1 - c0;  // this thread's columns (0 for threads past the end)
    int32_t *prevb = scr;    // prevb[Wp]: D[i+1][width] (0)
    int32_t *locb = scr + Wp + 1;
    int4 *cols = (int4 *)(scr + ((2 * Wp + 4) & ~3));
    int32_t *stk = (int32_t *)(cols + Wp);
    // interleaved index of column f (any thread's)
    auto ix = [&](int f) -> int64_t {
        const int t = f / per;
        return (int64_t)(f - t * per) * XTED_CTA_THREADS + t;
    };
    {   // derive this thread's columns once per unit (single segment: keyroot k_lo)
        const int2 *nodes = P.rowinfo + pr.col_base;
        const int j0 = P.krd[ch.k_lo];
        const int je = j0 + width;
        for (int k = 0; k < nk; k++) {
            const int c = c0 + k;
            const int j = j0 + c;
            const int2 nd = nodes[j];
            uint32_t z = (uint32_t)((nd.y & XTED_ROW_ORL_MASK) + 1 - j);
            if (j > j0 && (nd.y & XTED_ROW_PREVLEAF)) z |= XTED_COL_FARCOL;
            cols[(int64_t)k * XTED_CTA_THREADS + tid] = make_int4(j, nd.x, (int)z, je - j);
        }
    }
    const int n = pr.n;
    const int32_t *dt_in = P.dt + pr.dt_off;
    int32_t *dt_out = P.dt + pr.dt_off;
    const int2 *rows = P.rowinfo + pr.row_base;
    const int stack_rows = P.stack_rows;
    // the next thread's first column (the diagonal of this thread's last one)
    const int64_t next_ix = c1 < width ? (int64_t)tid + 1 : Wp;
    const int j0s = P.krd[ch.k_lo];  // the segment's first node: row slice drow[j0s, j0s + width)
    constexpr int kStageInts = DP_SMEM_BYTES / 4;
    const bool staged = width <= kStageInts, dbl = 2 * width <= kStageInts;
    auto stage_row = [&](int r, int32_t *dst) {
        const int32_t *src = dt_in + (int64_t)r * n + j0s;
        for (int c = tid; c < width; c += XTED_CTA_THREADS) cp_async4(dst + c, src + c);
        cp_async_commit();
    };
    // single segment: key = column index
    for (int kr = run.kr_lo; kr < run.kr_hi; kr++) {
        const int i0 = P.krd[kr];
        const int imax = (rows[i0].y & XTED_ROW_ORL_MASK) + 1;
        for (int k = 0; k < nk; k++)
            prevb[(int64_t)k * XTED_CTA_THREADS + tid] = cols[(int64_t)k * XTED_CTA_THREADS + tid].w * K.ins;
        if (tid == 0) prevb[Wp] = 0;
        int sp = 0;
        __syncthreads();
        if (staged && dbl) stage_row(imax - 1, smem + ((imax - 1) & 1) * width);
        for (int i = imax - 1; i >= i0; i--) {
            const int32_t *srow = nullptr;
            if (staged) {
                if (dbl) {
                    srow = smem + (i & 1) * width;
                    if (i - 1 >= i0) {
                        stage_row(i - 1, smem + ((i - 1) & 1) * width);  // its buffer's last readers passed the row-end barrier
                        cp_async_wait<1>();
                    } else {
                        cp_async_wait<0>();
                    }
                } else {
                    srow = smem;
                    stage_row(i, smem);
                    cp_async_wait<0>();
                }
                __syncthreads();  // every thread's copies of row i have landed
            }
            const int2 ri = rows[i];
            const int ro = ri.y & XTED_ROW_ORL_MASK;
            const bool trow = ro == imax - 1;
            const int bord = (imax - i) * K.del;
            const int rowfar = (imax - ro - 1) * K.del;
            const int32_t *top = stk + (int64_t)(sp > 0 ? sp - 1 : 0) * Wp;
            const int32_t *drow = dt_in + (int64_t)i * n;
            int run_min = XTED_INF;
            int diag_next = nk > 0 ? prevb[next_ix] : 0;  // D[i+1][c1]
            for (int k = nk - 1; k >= 0; k--) {
                const int c = c0 + k;
                const int64_t at = (int64_t)k * XTED_CTA_THREADS + tid;
                const int4 ci = cols[at];
                const int foff = ci.z & XTED_COL_FOFF_MASK, dend = ci.w;
                const int up = prevb[at];
                int diag = diag_next;
                diag_next = up;
                const bool segend = dend == 1;
                if (segend) diag = bord - K.del;
                const bool tcol = foff == dend;
                int a;
                if (trow && tcol) {
                    a = diag + (ri.x != ci.y ? K.ren : 0);
                } else {
                    int far;
                    if (trow) far = (dend - foff) * K.ins;
                    else if (tcol) far = rowfar;
                    else {
                        const int f = c + foff;
                        far = top[k + foff < nk ? (int64_t)(k + foff) * XTED_CTA_THREADS + tid : ix(f)];
                    }
                    a = (staged ? srow[c] : __ldcg(drow + ci.x)) + far;
                }
                int A = min(a, up + K.del);
                if (segend) A = min(A, bord + K.ins);
                run_min = min(run_min, A + c * K.ins);
                locb[at] = run_min;
            }
            const int incl = warp_suffix_min(run_min, lane);
            if (lane == 0) S.wtot[warp] = incl;
            __syncthreads();
            int carry = __shfl_down_sync(FULLMASK, incl, 1);
            if (lane == 31) carry = XTED_INF;
            for (int w = warp + 1; w < XTED_WARPS; w++) carry = min(carry, S.wtot[w]);
            int32_t *orow = dt_out + (int64_t)i * n;
            const bool pop = i != i0 && (ri.y & XTED_ROW_ISKR);
            const bool push = i > i0 && (ri.y & XTED_ROW_PREVLEAF);
            const int spush = pop ? sp - 1 : sp;
            if (push && spush >= stack_rows && tid == 0) set_error(P, XTED_ENOMEM, 3, spush, stack_rows);
            for (int k = 0; k < nk; k++) {
                const int c = c0 + k;
                const int64_t at = (int64_t)k * XTED_CTA_THREADS + tid;
                const int4 ci = cols[at];
                const int d = min(locb[at], carry) - c * K.ins;
                prevb[at] = d;
                if (trow && (ci.z & XTED_COL_FOFF_MASK) == ci.w) orow[ci.x] = d;
                if (push && spush < stack_rows && (ci.z & XTED_COL_FARCOL)) stk[(int64_t)spush * Wp + at] = d;
            }
            sp = push ? spush + 1 : spush;
            __syncthreads();
        }
    }
}

template <bool UC>
__device__ void dispatch_wide(const XKernelParams &P, const XPair &pr, const XUnit &u, int32_t *stk,
                              WideShared &S, int32_t *ring, int32_t *cache, int32_t *cnode) {
    const int width = P.chunks[u.chunk].width;
    const int tid = threadIdx.x;
    if (width <= 512) run_group<2, XTED_WARPS, UC>(P, pr, u, stk, S, ring, cache, cnode, tid, 0);
    else if (width <= 1024) run_group<4, XTED_WARPS, UC>(P, pr, u, stk, S, ring, cache, cnode, tid, 0);
    else if (width <= XTED_WIDE_REG_MAX) run_group<8, XTED_WARPS, UC>(P, pr, u, stk, S, ring, cache, cnode, tid, 0);
    else if (P.chunks[u.chunk].nseg == 1) run_wide_big<UC>(P, pr, u, stk, S, ring);
    else if (tid == 0) set_error(P, XTED_EINVAL, 4, width, P.chunks[u.chunk].nseg);
}

// Half-block unit: group gid (warps 4*gid .. 4*gid+3), chunk width <= XTED_HALF_MAX.
template <bool UC>
__device__ void dispatch_half(const XKernelParams &P, const XPair &pr, const XUnit &u, int32_t *stk, WideShared &S,
                              int32_t *ring, int32_t *cache, int32_t *cnode, int gtid, int gid) {
    const int width = P.chunks[u.chunk].width;
    if (width <= 256) run_group<2, 4, UC>(P, pr, u, stk, S, ring, cache, cnode, gtid, gid);
    else if (width <= 512) run_group<4, 4, UC>(P, pr, u, stk, S, ring, cache, cnode, gtid, gid);
    else if (width <= XTED_HALF_MAX) run_group<8, 4, UC>(P, pr, u, stk, S, ring, cache, cnode, gtid, gid);
    else if (gtid == 0) set_error(P, XTED_EINVAL, 6, width, 0);
}

// ---------------------------------------------------------------------------
// Ready queue (see xted_internal.h). Entries are appended to their bucket's
// list; blocks claim tasks from the oldest unexhausted entry of the highest
// non-empty bucket. An entry is only published after every task of the
// previous level of its pair has finished, so claimed tasks never wait.
// ---------------------------------------------------------------------------
// A field of a ready-queue entry, read through L2: P.entries[e].f. A serving
// session hands the entry ids of a finished query (or of its first round) to
// the next plan while the kernel runs, and a claimer reads the entry straight
// after the ring slot that names it, before any acquire: a copy of the old
// entry left in this SM's L1 would give the wrong task range and move the
// ring's head past a live entry. Only the fields a caller uses are loaded.
__device__ __forceinline__ int32_t entry_ld(const int32_t &f) { return __ldcg(&f); }

// Appends entry e at the tail of ring g.
__device__ __forceinline__ void ring_push(const XKernelParams &P, int g, int e) {
    const unsigned pos = (unsigned)atomicAdd(&P.rq_ctl[2 * g + 1], 1);
    const unsigned head = *(volatile unsigned *)&P.rq_ctl[2 * g];
    if (pos - head >= (1u << P.rq_log2)) {  // ring full: never overwrite a live slot
        set_error(P, XTED_ENOMEM, 5, g, (int)pos);
        return;
    }
    const unsigned long long v = ((unsigned long long)pos << 32) | (unsigned)e;
    ((volatile unsigned long long *)P.rq)[((int64_t)g << P.rq_log2) + (pos & ((1u << P.rq_log2) - 1))] = v;
}

// Publishes entry e (or, past levels without tasks, the first later level that
// has some): its narrow tasks into its bucket's narrow ring, its group tasks
// into its bucket's group ring. Returns false when the pair has no level
// left, i.e. the pair is finished.
__device__ bool rq_publish(const XKernelParams &P, int e) {
    while (e >= 0) {
        const XEntry &X = P.entries[e];
        const int nt = entry_ld(X.ntasks);
        if (nt > 0) {
            const int nn = entry_ld(X.nnarrow), b = entry_ld(X.bucket);
            if (nn > 0) ring_push(P, XTED_KIND_NARROW * XTED_BUCKETS + b, e);
            if (nt > nn) ring_push(P, XTED_KIND_GROUP * XTED_BUCKETS + b, e);
            return true;
        }
        e = entry_ld(X.next);  // a level without tasks: go on to the next one
    }
    return false;
}

// Entry held by ring position pos of ring g, or -1 if that position is not
// written yet.
__device__ __forceinline__ int rq_entry(const XKernelParams &P, int g, unsigned pos) {
    const unsigned long long v =
        ((volatile const unsigned long long *)P.rq)[((int64_t)g << P.rq_log2) + (pos & ((1u << P.rq_log2) - 1))];
    return (unsigned)(v >> 32) == pos ? (int)(unsigned)v : -1;
}

// Longest sleeps between polls (ns; a sleep lasts anywhere up to twice the
// request): a claimer polling the ready queue, and a warp waiting for its
// block's claimer.
#ifndef XTED_CLAIM_SLEEP_MAX
#define XTED_CLAIM_SLEEP_MAX 1024
#endif
#ifndef XTED_IDLE_SLEEP_MAX
#define XTED_IDLE_SLEEP_MAX 2048
#endif
#define CLAIM_EXIT (-1)
#define CLAIM_RECORD (-2)
#define CLAIM_NONE (-3)

// Returns a task index (and its entry), CLAIM_EXIT when the launch is over
// (all tasks done, an error, or in a serving session the stop word or an
// idle spell), or CLAIM_RECORD with *entry = a mailbox record this block
// claimed and must publish. Buckets are probed from the most urgent: bucket
// 15 down in a batch, the oldest query's bucket onwards in a serving session.
// Within a bucket entries are served first in, first out: a block claims the
// next task of the entry at the bucket's head, and whoever finds that entry
// exhausted moves the head on. Idle polling is bounded by time and by
// iterations. With wait = false (the block still has units in flight, whose
// completions may publish work) one pass is made and CLAIM_NONE returned if it
// finds nothing; only a block with nothing in flight waits, counts as idle in
// a serving session, or ends the launch.
// Kinds: a bit mask of XTED_KIND_* rings the claim may take from, and the
// kind preferred within a bucket; buckets keep their priority order across
// kinds. A block that has narrow units in flight claims narrow tasks only (a
// group task would stop its warps until every unit in flight had finished).
// Serving: rq_ctl words after the done counter.
#define CTL_IDLE (2 * XTED_RINGS + 1)     // blocks currently idle (or gone)
#define CTL_LEAVING (2 * XTED_RINGS + 2)  // nonzero once blocks have started to leave
#define KINDS_NARROW 1u
#define KINDS_ANY 3u

__device__ int claim_task(const XKernelParams &P, int *entry, bool wait, int lane, unsigned kinds, int prefer) {
    // Called by a whole warp; lane 0 claims, the warp reads every bucket's
    // head and tail in one coalesced load so that only non-empty buckets are
    // probed. Returns the same result in every lane.
    volatile int32_t *ctl = P.rq_ctl;
    volatile int32_t *state = P.entry_state;
    volatile int32_t *mbox = P.mbox;
    unsigned ns = 32;
    uint64_t t0 = 0;
    bool idle_counted = false;  // serving: this block is counted in CTL_IDLE
    static_assert(2 * XTED_BUCKETS == 32, "one lane per bucket head or tail of each kind");
    for (long it = 0; it < (1L << 28); it++) {
        int res = CLAIM_NONE, e_out = -1, top = XTED_BUCKETS - 1;
        if (lane == 0) {
            if (*(volatile int32_t *)P.error != 0) {
                res = CLAIM_EXIT;
            } else if (P.serve) {
                // admit posted queries first: their level-0 entries go to the new
                // query's own (least urgent) bucket, and a busy launch would
                // otherwise only look at the mailbox once it ran out of work
                // a record is claimed only while the launch is open (no CLOSED
                // bit): the claim and the closing are CAS on the same word
                int cons = mbox[XTED_MBOX_CONSUMED];
                while (!(cons & XTED_MBOX_CLOSED) && cons < mbox[XTED_MBOX_POSTED]) {
                    if (atomicCAS(&P.mbox[XTED_MBOX_CONSUMED], cons, cons + 1) == cons) {
                        __threadfence();  // acquire: the record and its query's plan are visible from here on
                        if (idle_counted) atomicSub(&P.rq_ctl[CTL_IDLE], 1);
                        e_out = cons;
                        res = CLAIM_RECORD;
                        break;
                    }
                    cons = mbox[XTED_MBOX_CONSUMED];
                }
                top = mbox[XTED_MBOX_TOP];
            }
        }
        res = __shfl_sync(FULLMASK, res, 0);
        if (res != CLAIM_NONE) {
            *entry = __shfl_sync(FULLMASK, e_out, 0);
            return res;
        }
        top = __shfl_sync(FULLMASK, top, 0);
        // snapshot: lane 2b holds bucket b's narrow-ring head, lane 2b+1 its
        // tail; the same lanes read the group rings' words 32 further on
        const int v0 = ctl[lane], v1 = ctl[2 * XTED_BUCKETS + lane];
        const int tl0 = __shfl_down_sync(FULLMASK, v0, 1), tl1 = __shfl_down_sync(FULLMASK, v1, 1);
        const unsigned ne0 = __ballot_sync(FULLMASK, (lane & 1) == 0 && (int)((unsigned)tl0 - (unsigned)v0) > 0);
        const unsigned ne1 = __ballot_sync(FULLMASK, (lane & 1) == 0 && (int)((unsigned)tl1 - (unsigned)v1) > 0);
        if (lane == 0) {
            for (int i = 0; i < XTED_BUCKETS && res == CLAIM_NONE; i++) {
                const int b = (top - i) & (XTED_BUCKETS - 1);
                for (int pass = 0; pass < 2 && res == CLAIM_NONE; pass++) {
                    const int kind = pass == 0 ? prefer : 1 - prefer;
                    if (!((kinds >> kind) & 1u)) continue;
                    if (!(((kind ? ne1 : ne0) >> (2 * b)) & 1u)) continue;  // empty when looked at
                    const int g = kind * XTED_BUCKETS + b;
                    for (int guard = 0; guard < 256; guard++) {
                        const unsigned h = (unsigned)ctl[2 * g];
                        if ((int)((unsigned)ctl[2 * g + 1] - h) <= 0) break;  // empty
                        const int e = rq_entry(P, g, h);
                        if (e < 0) break;  // the head position is reserved but not yet written
                        const XEntry &X = P.entries[e];
                        const int nn = entry_ld(X.nnarrow);
                        const int lim = kind == XTED_KIND_NARROW ? nn : entry_ld(X.ntasks) - nn;
                        if (state[XTED_ESTATE * e + kind] < lim) {
                            const int k = atomicAdd(&P.entry_state[XTED_ESTATE * e + kind], 1);
                            if (k < lim) {
                                __threadfence();  // acquire: the level's inputs are visible from here on
                                if (idle_counted) atomicSub(&P.rq_ctl[CTL_IDLE], 1);
                                e_out = e;
                                res = entry_ld(X.task_off) + (kind == XTED_KIND_NARROW ? 0 : nn) + k;
                                break;
                            }
                        }
                        atomicCAS((int32_t *)&ctl[2 * g], (int)h, (int)(h + 1));  // exhausted: next entry
                    }
                }
            }
            if (res == CLAIM_NONE && wait) {
                if (P.serve) {
                    // A block leaves a serving launch only once every block has been
                    // idle (then the others follow as soon as they are idle too), so
                    // the launch never runs on a few blocks while work arrives; the
                    // host relaunches when the last one is gone and work is posted.
                    if (!idle_counted) {
                        atomicAdd(&P.rq_ctl[CTL_IDLE], 1);
                        idle_counted = true;
                    }
                    if (mbox[XTED_MBOX_STOP] != 0 || ctl[CTL_LEAVING] != 0 ||
                        (mbox[XTED_MBOX_CONSUMED] & XTED_MBOX_CLOSED))
                        res = CLAIM_EXIT;
                } else if (ld_acquire(P.done_total) >= P.ntasks) {
                    res = CLAIM_EXIT;
                }
                if (res == CLAIM_NONE) {
                    const uint64_t now = global_ns();
                    if (t0 == 0) {
                        t0 = now;
                    } else if (P.serve) {
                        // Idle everywhere: close the launch to new records and
                        // leave (the host relaunches on new work). Closing is a
                        // CAS on the claim word, so no block can claim a record
                        // after it and then run that query alone while the
                        // others leave; a record posted meanwhile stays for
                        // the next launch.
                        if (now - t0 > P.idle_exit_ns && ctl[CTL_IDLE] >= (int)gridDim.x) {
                            const int cons = mbox[XTED_MBOX_CONSUMED];
                            if (!(cons & XTED_MBOX_CLOSED) && cons >= mbox[XTED_MBOX_POSTED] &&
                                atomicCAS(&P.mbox[XTED_MBOX_CONSUMED], cons, cons | XTED_MBOX_CLOSED) == cons) {
                                atomicExch(&P.rq_ctl[CTL_LEAVING], 1);
                                res = CLAIM_EXIT;
                            }
                        }
                    } else if (now - t0 > P.timeout_ns) {
                        set_error(P, XTED_ETIMEOUT, 0, 0, 0);
                        res = CLAIM_EXIT;
                    }
                }
            }
        }
        res = __shfl_sync(FULLMASK, res, 0);
        if (res != CLAIM_NONE || !wait) {
            *entry = __shfl_sync(FULLMASK, e_out, 0);
            return res;
        }
        __nanosleep(ns);
        __syncwarp();
        if (ns < XTED_CLAIM_SLEEP_MAX) ns <<= 1;
    }
    if (lane == 0) set_error(P, XTED_ETIMEOUT, 1, 0, 0);
    return CLAIM_EXIT;
}

// A serving pair is finished: its distance goes to the host-visible result
// array, and the last pair of a query raises the slot's flag to the query's
// generation (the host polls it).
__device__ void finish_served_pair(const XKernelParams &P, int pair, int bucket) {
    const int d = __ldcg(P.dt + __ldcg(&P.pairs[pair].dt_off));
    ((volatile int32_t *)P.results)[pair] = d;
    __threadfence_system();
    const int s = pair / P.serve_pairs;
    const int n = atomicAdd(&P.slot_done[s], 1) + 1;
    if (n == __ldcg(&P.slot_need[s])) {
        P.slot_done[s] = 0;
        // Every position left in the query's bucket (both its rings) names
        // one of its own, now exhausted, entries (a bucket serves one query at
        // a time). Move the heads past them before the host may hand those
        // entry ids to a new query: a claimer must never find an old position
        // whose entry id has been reused.
        for (int kind = 0; kind < 2; kind++) {
            const int rg = kind * XTED_BUCKETS + bucket;
            volatile int32_t *ctl = P.rq_ctl + 2 * rg;
            const unsigned tl = (unsigned)ctl[1];
            for (int g = 0; g < 1024; g++) {
                const unsigned h = (unsigned)ctl[0];
                if ((int)(tl - h) <= 0) break;
                atomicCAS((int32_t *)&P.rq_ctl[2 * rg], (int)h, (int)tl);
            }
        }
        __threadfence_system();
        ((volatile int32_t *)P.flags)[s] = __ldcg(&P.slot_gen[s]);
    }
}

// After a task (all its writes fenced and the block synchronised).
__device__ void complete_task(const XKernelParams &P, int e, int pair) {
    const XEntry &X = P.entries[e];
    const int done = atomicAdd(&P.entry_state[XTED_ESTATE * e + 2], 1) + 1;
    if (done == entry_ld(X.ntasks)) {
        __threadfence();  // acquire the level's other tasks, release to the next level's claimers
        if (!rq_publish(P, entry_ld(X.next)) && P.serve) finish_served_pair(P, pair, entry_ld(X.bucket));
    }
    __threadfence();
    atomicAdd(P.done_total, 1);
}

// A warp publishes level 0 of every pair of mailbox record r (claimed, and
// acquired, by its lane 0).
__device__ void publish_record(const XKernelParams &P, int r, int lane) {
    int lo = 0, n = 0;
    if (lane == 0) {
        const volatile int32_t *rec = P.mbox + XTED_MBOX_REC + 4 * (r & (XTED_SERVE_RECS - 1));
        lo = rec[1];
        n = rec[2];
    }
    lo = __shfl_sync(FULLMASK, lo, 0);
    n = __shfl_sync(FULLMASK, n, 0);
    __threadfence();
    for (int p = lo + lane; p < lo + n; p += 32) {
        const int e = __ldcg(&P.first[p]);
        if (e >= 0 && p != P.hold_pair && !rq_publish(P, e)) finish_served_pair(P, p, entry_ld(P.entries[e].bucket));
    }
    __syncwarp();
}

__global__ void xted_rq_init_kernel(XKernelParams P) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < P.npairs && P.first[p] >= 0 && p != P.hold_pair) rq_publish(P, P.first[p]);
}

// Trace record of a finished task (XTED_TRACE): end time and
// group(1) | units(7) | sm(8) | widest chunk(16) | cells(32).
__device__ void trace_task_end(const XKernelParams &P, int t) {
    const XTask T = P.tasks[t];
    unsigned sm;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(sm));
    const int nu = (int)(T.kind_n & 0xffff);
    unsigned long long cells = 0, wmax = 0;
    if (T.kind_n & XTED_TASK_STRIPED) {  // this stripe's columns of its unit
        const XStripe X = P.stripes[T.unit_lo];
        const int sw = XTED_CTA_THREADS * X.sww, s = (int)((T.kind_n >> XTED_STRIPE_SHIFT) & XTED_STRIPE_MASK);
        wmax = (unsigned long long)min(sw, X.w - s * sw);
        cells = wmax * (unsigned)X.R;
    } else {
        for (int k = 0; k < nu; k++) {
            const XUnit u = P.units[T.unit_lo + k];
            const unsigned long long w = (unsigned)P.chunks[u.chunk].width;
            cells += w * (unsigned)P.runs[u.run].rows;
            if (w > wmax) wmax = w;
        }
    }
    P.trace[4 * (int64_t)t + 2] = global_ns();
    P.trace[4 * (int64_t)t + 3] = ((T.kind_n & (XTED_TASK_WIDE | XTED_TASK_HALF)) ? 1ull : 0ull) |
                                  ((unsigned long long)(nu & 127) << 1) | ((unsigned long long)(sm & 255) << 8) |
                                  ((wmax & 0xffff) << 16) | ((cells & 0xffffffffull) << 32);
}

// Narrow tasks open in a block. The block's warps take units one at a time
// from any open task and never wait for each other: the warp that finishes a
// task's last unit completes the task, and a warp that finds no unit left
// claims the next task (one claimer at a time). A group task (half or whole
// block) gathers every warp at a block barrier once they are between units.
#define FLOW_SLOTS 16  // > warps + 1: every open task has a unit running or unclaimed
#define FLOW_RUN 0  // zero: run_narrow's yield test reads "mode != 0"
#define FLOW_GROUP 1
#define FLOW_EXIT 2
// A slot's units are handed out through one word, (units << 8) | handed out:
// a warp's atomicAdd on it yields a unit index and the unit count of the same
// filling, so a warp racing with the slot's reuse never takes a unit of the
// old task by the new one's count. A free slot holds 0 units.
struct FlowSlot {
    int word;  // (units << 8) | next unit; units == 0: free
    int done;  // units finished
    int task, entry, pair, unit_lo;
    int pad[2];
};
static_assert(XTED_TASK_UNITS + XTED_WARPS < 256, "unit counter of a flow slot");
#define CHAIN_MAX 2  // group tasks run back to back while narrow units wait
#define PARK_SLOTS 16  // parked narrow units (at most one per warp is ever in flight; spare room for races)

// The persistent DP kernel. Two instantiations per cost model: without
// striped units (every batch whose column segments fit the register paths:
// the stripe code is left out of the hot loop entirely), and with them.
template <bool STRIPES, bool UC>
__device__ __forceinline__ void dp_main(const XKernelParams &P) {
    __shared__ int s_next, s_k[2];
    __shared__ int s_mode, s_lock, s_gtask, s_gentry, s_progress, s_epoch, s_chain;
    __shared__ int s_role;  // XTED_KIND_* the block last claimed: the kind it prefers when idle
    __shared__ FlowSlot s_fs[FLOW_SLOTS];
    // narrow units parked between two keyroot tables while the block ran a
    // group task: x flow slot, y unit, z pair, w next keyroot
    __shared__ int s_park[4 * PARK_SLOTS];
    __shared__ unsigned s_park_full, s_park_held;
    __shared__ WideShared S[2];
    extern __shared__ __align__(16) int32_t s_dyn[];  // ring | stack cache | column nodes (DP_SMEM_BYTES)
    int32_t *s_ring = s_dyn;
    int32_t *s_cache = s_dyn + RING_INTS;
    int32_t *s_cnode = s_cache + CACHE_INTS;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // columns past a chunk's end read ring and stack cells nobody writes for
    // that unit: start them at zero so those inert columns stay non-negative
    for (int x = tid; x < RING_INTS + CACHE_INTS; x += XTED_CTA_THREADS) s_dyn[x] = 0;
    if (tid < FLOW_SLOTS) {
        s_fs[tid].word = 0;
        s_fs[tid].done = 0;
        s_fs[tid].task = -1;
    }
    if (tid == 0) {
        s_park_full = 0;
        s_park_held = 0;
        s_chain = 0;
        s_role = (blockIdx.x & 1) ? XTED_KIND_NARROW : XTED_KIND_GROUP;
        s_mode = FLOW_RUN;
        s_lock = -1;
        s_progress = 0;
        s_epoch = 0;
    }
    __syncthreads();
    volatile int *vmode = &s_mode, *vlock = &s_lock, *vprog = &s_progress, *vepoch = &s_epoch;
    volatile FlowSlot *vfs = s_fs;
    int32_t *scratch = P.scratch + (int64_t)blockIdx.x * P.scratch_per_cta;
    // this warp's regions for narrow units
    int32_t *n_stk = scratch + (int64_t)warp * P.stack_rows * XTED_NARROW_MAX;
    int32_t *n_ring = s_ring + warp * (XTED_PREFETCH * NARROW_SLOT);
    int32_t *n_cache = s_cache + warp * (XTED_STACK_CACHE * NARROW_ROW);
    int32_t *n_cnode = s_cnode + warp * XTED_NARROW_MAX;
    // A warp without work either is the block's claimer (one at a time: it
    // polls the ready queue, its waits bounded inside claim_task) or sleeps
    // until the block's epoch moves (a task opened, the mode changed, the
    // claimer left). As a guard, a warp that sees its block make no progress
    // for far longer than any claim may wait gives up.
    const uint64_t idle_limit = (P.serve ? 16ull : 2ull) * P.timeout_ns;
    for (;;) {
        // one read per warp, broadcast: every lane takes the same branch
        // (lanes woken from a sleep one by one could otherwise read two modes)
        int mode = 0, epoch = 0;
        if (lane == 0) {
            epoch = *vepoch;  // before the slot scan: a task opened later moves it
            mode = *vmode;
        }
        mode = __shfl_sync(FULLMASK, mode, 0);
        epoch = __shfl_sync(FULLMASK, epoch, 0);
        if (mode == FLOW_EXIT) break;
        if (mode == FLOW_GROUP) {
            __syncwarp();
            __syncthreads();  // every warp is between units
            const int t = s_gtask;
            const XTask T = P.tasks[t];
            const XPair pr = P.pairs[T.pair];
            if (P.trace && tid == 0) P.trace[4 * (int64_t)t + 1] = global_ns();
            if (STRIPES && (T.kind_n & XTED_TASK_STRIPED)) {
                run_striped<UC>(P, pr, T, scratch, S[0], s_ring, s_cache, s_cnode);
            } else if (T.kind_n & XTED_TASK_WIDE) {
                dispatch_wide<UC>(P, pr, P.units[T.unit_lo], scratch, S[0], s_ring, s_cache, s_cnode);
            } else {
                // the block's two halves take the task's units one at a time
                const int nu = (int)(T.kind_n & 0xffff);
                const int gid = warp >> 2, gtid = tid & 127;
                int32_t *stk = scratch + (int64_t)gid * P.stack_rows * XTED_HALF_MAX;
                int32_t *ring = s_ring + gid * (4 * XTED_PREFETCH * NARROW_SLOT);
                int32_t *cache = s_cache + gid * (4 * XTED_STACK_CACHE * NARROW_ROW);
                int32_t *cnode = s_cnode + gid * (4 * XTED_NARROW_MAX);
                for (;;) {
                    if (gtid == 0) s_k[gid] = atomicAdd(&s_next, 1);
                    group_sync<4>(gid);
                    const int k = s_k[gid];
                    group_sync<4>(gid);  // every thread of the half has read s_k before its next claim
                    if (k >= nu) break;
                    dispatch_half<UC>(P, pr, P.units[T.unit_lo + k], stk, S[gid], ring, cache, cnode, gtid, gid);
                }
            }
            __threadfence();
            __syncthreads();
            if (warp == 0) {
                // Every warp waits at the barrier below, so the block looks for
                // its next task now: another group task (a stripe among them)
                // then runs without gathering the warps again,
                // which costs them the tail of whatever they were running. A
                // narrow task found here is opened as usual. While parked or
                // open narrow units wait, at most CHAIN_MAX group tasks chain.
                int nt = CLAIM_NONE, ne = -1, allow = 0;
                if (lane == 0) {
                    complete_task(P, s_gentry, T.pair);
                    if (P.trace) trace_task_end(P, t);
                    s_progress++;
                    bool waiting = *(volatile unsigned *)&s_park_full != 0, room = false;
                    for (int q = 0; q < FLOW_SLOTS; q++) {
                        const int w = vfs[q].word;
                        if ((w & 255) < (w >> 8)) waiting = true;
                        if ((w >> 8) == 0) room = true;
                    }
                    allow = room && (!waiting || s_chain < CHAIN_MAX);
                }
                if (__shfl_sync(FULLMASK, allow, 0))
                    nt = claim_task(P, &ne, false, lane, KINDS_ANY, XTED_KIND_GROUP);
                if (lane == 0) {
                    bool stay = false;
                    if (nt >= 0) {
                        const XTask T2 = P.tasks[nt];
                        if (P.trace) P.trace[4 * (int64_t)nt] = global_ns();
                        if (T2.kind_n & (XTED_TASK_WIDE | XTED_TASK_HALF)) {
                            s_gtask = nt;
                            s_gentry = ne;
                            s_next = 0;
                            stay = true;
                        } else {
                            s_role = XTED_KIND_NARROW;
                            int q = 0;
                            while (q < FLOW_SLOTS - 1 && (vfs[q].word >> 8) != 0) q++;  // room was seen
                            vfs[q].task = nt;
                            vfs[q].entry = ne;
                            vfs[q].pair = T2.pair;
                            vfs[q].unit_lo = T2.unit_lo;
                            vfs[q].done = 0;
                            __threadfence_block();
                            atomicExch(&s_fs[q].word, (int)(T2.kind_n & 0xffff) << 8);
                            if (P.trace) P.trace[4 * (int64_t)nt + 1] = global_ns();
                        }
                    }
                    s_chain = stay ? s_chain + 1 : 0;
                    __threadfence_block();
                    *vmode = nt == CLAIM_EXIT ? FLOW_EXIT : (stay ? FLOW_GROUP : FLOW_RUN);
                }
                nt = __shfl_sync(FULLMASK, nt, 0);
                ne = __shfl_sync(FULLMASK, ne, 0);
                if (nt == CLAIM_RECORD) publish_record(P, ne, lane);
            }
            __syncthreads();
            continue;
        }
        // a parked unit first (it holds a slot's task open), else a new unit of an open narrow task
        int slot = -1, k = 0, kr0 = -1, upark = 0, ppark = 0;
        if (lane == 0) {
            for (unsigned f = *(volatile unsigned *)&s_park_full; f != 0 && slot < 0;
                 f = *(volatile unsigned *)&s_park_full) {
                const unsigned bit = f & (0u - f);
                if (atomicAnd(&s_park_full, ~bit) & bit) {
                    const int i = __ffs(bit) - 1;
                    const volatile int *pk = s_park + 4 * i;
                    slot = pk[0];
                    upark = pk[1];
                    ppark = pk[2];
                    kr0 = pk[3];
                    __threadfence_block();
                    atomicAnd(&s_park_held, ~bit);  // the entry may be reused
                }
            }
            for (int q = 0; q < FLOW_SLOTS && slot < 0; q++) {
                const int w = vfs[q].word;
                if ((w & 255) < (w >> 8)) {
                    const int got = atomicAdd(&s_fs[q].word, 1);
                    if ((got & 255) < (got >> 8)) {
                        slot = q;
                        k = got & 255;
                    }
                }
            }
        }
        slot = __shfl_sync(FULLMASK, slot, 0);
        if (slot >= 0) {
            int pair = 0, ulo = 0;
            if (lane == 0) {
                pair = kr0 >= 0 ? ppark : vfs[slot].pair;
                ulo = kr0 >= 0 ? upark : vfs[slot].unit_lo + k;
            }
            pair = __shfl_sync(FULLMASK, pair, 0);
            ulo = __shfl_sync(FULLMASK, ulo, 0);
            kr0 = __shfl_sync(FULLMASK, kr0, 0);
            __threadfence();  // acquire: the task's inputs, seen by the claimer, are visible here too
            const XPair pr = P.pairs[pair];
            // with no room to park (never expected), the unit runs on to its end
            bool parked = false;
            for (const volatile int *yield = vmode;; yield = nullptr) {
                const int next = dispatch_narrow<UC>(P, pr, P.units[ulo], lane, n_stk, n_ring, n_cache, n_cnode, kr0,
                                                     yield);
                if (next < 0) break;
                // the block gathers for a group task: park the rest of the unit
                int ok = 0;
                if (lane == 0) {
                    for (int i = 0; i < PARK_SLOTS && !ok; i++) {
                        const unsigned bit = 1u << i;
                        if (!(atomicOr(&s_park_held, bit) & bit)) {
                            volatile int *pk = s_park + 4 * i;
                            pk[0] = slot;
                            pk[1] = ulo;
                            pk[2] = pair;
                            pk[3] = next;
                            __threadfence_block();
                            atomicOr(&s_park_full, bit);
                            ok = 1;
                        }
                    }
                }
                kr0 = next;
                if (__shfl_sync(FULLMASK, ok, 0)) {
                    parked = true;
                    break;
                }
            }
            if (parked) {
                __syncwarp();
                continue;
            }
            __threadfence();  // release this unit's writes before it is counted done
            __syncwarp();
            if (lane == 0) {
                if (atomicAdd(&s_fs[slot].done, 1) + 1 == (vfs[slot].word >> 8)) {
                    const int e = vfs[slot].entry, t = vfs[slot].task;
                    __threadfence();  // acquire the task's other units
                    complete_task(P, e, pair);
                    if (P.trace) trace_task_end(P, t);
                    atomicExch(&s_fs[slot].word, 0);  // free (every unit was handed out)
                    atomicAdd(&s_progress, 1);
                }
            }
            __syncwarp();
            continue;
        }
        // no unit left: claim the next task (one warp of the block at a time)
        int t = CLAIM_NONE, e = -1;
        int seat = 0;
        if (lane == 0) seat = *vlock < 0 && atomicCAS(&s_lock, -1, warp) == -1;
        if (__shfl_sync(FULLMASK, seat, 0)) {
            unsigned ns = 64;
            const uint64_t c0 = global_ns();
            const int pg0 = *vprog;
            for (;;) {
                // a slot stays filled until its last unit is done: no filled
                // slot, no unit of this block in flight
                int busy = 0, stop = 0;
                if (lane == 0) {
                    bool room = false, open = false;
                    for (int q = 0; q < FLOW_SLOTS; q++) {
                        const int w = vfs[q].word;
                        if ((w >> 8) != 0) {
                            busy = 1;
                            if ((w & 255) < (w >> 8)) open = true;
                        } else {
                            room = true;
                        }
                    }
                    stop = *vmode != FLOW_RUN || open || !room || *(volatile unsigned *)&s_park_full != 0;
                    if (!stop && busy && *vprog == pg0 && global_ns() - c0 > idle_limit) {
                        set_error(P, XTED_ETIMEOUT, 8, warp, pg0);
                        stop = 2;
                    }
                }
                stop = __shfl_sync(FULLMASK, stop, 0);
                busy = __shfl_sync(FULLMASK, busy, 0);
                if (stop == 2) t = CLAIM_EXIT;
                if (stop) break;
                // narrow units in flight: narrow tasks only; an idle block takes
                // either kind, its role's first within a bucket
                t = claim_task(P, &e, !busy, lane, busy ? KINDS_NARROW : KINDS_ANY,
                                        busy ? XTED_KIND_NARROW : *(volatile int *)&s_role);
                if (t != CLAIM_NONE) break;
                __nanosleep(ns);  // nothing ready while units of this block run: poll again soon
                __syncwarp();
                if (ns < XTED_CLAIM_SLEEP_MAX) ns <<= 1;
            }
            if (lane == 0) {
                if (t >= 0) {
                    atomicAdd(&s_progress, 1);
                    const XTask T = P.tasks[t];
                    if (P.trace) P.trace[4 * (int64_t)t] = global_ns();
                    if (T.kind_n & (XTED_TASK_WIDE | XTED_TASK_HALF)) {
                        s_gtask = t;
                        s_gentry = e;
                        s_next = 0;
                        s_role = XTED_KIND_GROUP;
                        __threadfence_block();
                        *vmode = FLOW_GROUP;
                    } else {
                        s_role = XTED_KIND_NARROW;
                        int q = 0;
                        while (q < FLOW_SLOTS - 1 && (vfs[q].word >> 8) != 0) q++;  // room was seen; only the claimer fills
                        vfs[q].task = t;
                        vfs[q].entry = e;
                        vfs[q].pair = T.pair;
                        vfs[q].unit_lo = T.unit_lo;
                        vfs[q].done = 0;
                        __threadfence_block();
                        atomicExch(&s_fs[q].word, (int)(T.kind_n & 0xffff) << 8);  // open: units handed out from here
                        if (P.trace) P.trace[4 * (int64_t)t + 1] = global_ns();
                    }
                } else if (t == CLAIM_EXIT) {
                    atomicCAS(&s_mode, FLOW_RUN, FLOW_EXIT);
                }
                if (t != CLAIM_RECORD) {
                    __threadfence_block();
                    *vlock = -1;
                    atomicAdd(&s_epoch, 1);  // wake the sleepers: a task, a mode change, or a free claimer seat
                }
            }
        }
        t = __shfl_sync(FULLMASK, t, 0);
        e = __shfl_sync(FULLMASK, e, 0);
        if (t == CLAIM_RECORD) {
            publish_record(P, e, lane);
            if (lane == 0) {
                __threadfence_block();
                *vlock = -1;
                atomicAdd(&s_epoch, 1);
            }
            __syncwarp();
            continue;
        }
        if (t != CLAIM_NONE) continue;  // claimed (or ended), or left the claimer seat with units open
        // another warp is the claimer: sleep until the block's epoch moves
        if (lane == 0) {
            unsigned ns = 128;
            const uint64_t i0 = global_ns();
            int pg = *vprog;
            uint64_t p0 = i0;
            for (long it = 0; *vepoch == epoch; it++) {
                __nanosleep(ns);
                if (ns < XTED_IDLE_SLEEP_MAX) ns <<= 1;
                const uint64_t now = global_ns();
                const int pg2 = *vprog;
                if (pg2 != pg) {
                    pg = pg2;
                    p0 = now;
                } else if (now - p0 > idle_limit || it > (1L << 28)) {
                    set_error(P, XTED_ETIMEOUT, 7, warp, pg);
                    atomicCAS(&s_mode, FLOW_RUN, FLOW_EXIT);  // never while a group task gathers the block
                    break;
                }
            }
        }
        __syncwarp();
    }
    cp_async_wait<0>();
}

// Four instantiations: with or without striped units, unit or general costs.
__global__ void __launch_bounds__(XTED_CTA_THREADS, 2) xted_dp_kernel(XKernelParams P) { dp_main<false, true>(P); }
__global__ void __launch_bounds__(XTED_CTA_THREADS, 2) xted_dp_kernel_striped(XKernelParams P) {
    dp_main<true, true>(P);
}
__global__ void __launch_bounds__(XTED_CTA_THREADS, 2) xted_dp_kernel_costs(XKernelParams P) {
    dp_main<false, false>(P);
}
__global__ void __launch_bounds__(XTED_CTA_THREADS, 2) xted_dp_kernel_striped_costs(XKernelParams P) {
    dp_main<true, false>(P);
}

// Result of pair p: Dtree[0][0] of its table (X-TED_CPU/TED.cpp:188), or for
// a pair with an empty tree the cost of inserting (m = 0) or deleting (n = 0)
// the other one (TED.cpp:181-186, with unit costs there).
__global__ void xted_gather_kernel(const XPair *pairs, const int32_t *trivial, const int32_t *dt,
                                   int npairs, int32_t *out, int c_del, int c_ins) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npairs) return;
    const int tv = trivial[p];
    out[p] = tv >= 0 ? (pairs[p].m == 0 ? pairs[p].n * c_ins : pairs[p].m * c_del) : __ldcg(dt + pairs[p].dt_off);
}

// ---- host-side launch helpers ----
int dp_occupancy(int *blocks_per_sm) {
    cudaError_t e = cudaFuncSetAttribute(xted_dp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, DP_SMEM_BYTES);
    if (e != cudaSuccess) return (int)e;
    int least = 1 << 30;
    for (const void *k : {(const void *)xted_dp_kernel_striped, (const void *)xted_dp_kernel_costs,
                          (const void *)xted_dp_kernel_striped_costs, (const void *)xted_dp_kernel}) {
        e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, DP_SMEM_BYTES);
        if (e != cudaSuccess) return (int)e;
        int occ = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, XTED_CTA_THREADS, DP_SMEM_BYTES);
        if (e != cudaSuccess) return (int)e;
        least = occ < least ? occ : least;  // one grid size for every instantiation
    }
    *blocks_per_sm = least;
    return (int)e;
}

// Cooperative launch (every block resident at once), expressed as a launch
// attribute so that the same call also records into a CUDA graph.
cudaError_t launch_dp(const XKernelParams &P, int grid, cudaStream_t s) {
    XKernelParams p = P;
    void *args[] = {&p};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(XTED_CTA_THREADS);
    cfg.dynamicSmemBytes = DP_SMEM_BYTES;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const bool unit = P.c_del == 1 && P.c_ins == 1 && P.c_ren == 1;
    const void *k = P.nstriped > 0 ? (unit ? (const void *)xted_dp_kernel_striped : (const void *)xted_dp_kernel_striped_costs)
                                      : (unit ? (const void *)xted_dp_kernel : (const void *)xted_dp_kernel_costs);
    return cudaLaunchKernelExC(&cfg, k, args);
}

cudaError_t launch_rq_init(const XKernelParams &P, cudaStream_t s) {
    if (P.npairs <= 0) return cudaSuccess;
    xted_rq_init_kernel<<<(P.npairs + 255) / 256, 256, 0, s>>>(P);
    return cudaGetLastError();
}

cudaError_t launch_gather(const XPair *pairs, const int32_t *trivial, const int32_t *dt, int npairs,
                          int32_t *out, int c_del, int c_ins, cudaStream_t s) {
    if (npairs <= 0) return cudaSuccess;
    xted_gather_kernel<<<(npairs + 255) / 256, 256, 0, s>>>(pairs, trivial, dt, npairs, out, c_del, c_ins);
    return cudaGetLastError();
}

}  // namespace xted
