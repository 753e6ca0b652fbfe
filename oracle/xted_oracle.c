/*
 * xted_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference X-TED_CPU tree edit distance
 * (Davis-Fan/X-TED). It is the checker for the CUDA path: only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg may load it.
 * The product library never links or calls this file.
 *
 * Parity of this restatement is pinned against golden distances produced by
 * running the reference X-TED_CPU itself (compiled from its own sources by
 * oracle/Makefile into oracle/_ref/), see tests/golden/.
 *
 * Trees are preorder CSR: labels[n], child_off[n+1], child_idx[n-1]; the
 * children of node v are child_idx[child_off[v] .. child_off[v+1]) in order.
 * Labels are int32 ids; the reference compares label strings for equality
 * only (X-TED_CPU/TED.cpp:153-159), so interned ids are exact.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>

/* X-TED_CPU/TED.cpp:3-17 min3 */
static inline int xo_min3(int a, int b, int c) {
    int t = a < b ? a : b;
    return t < c ? t : c;
}

/* X-TED_CPU/TED.cpp:21-42 outermost_right_leaves: follow last children,
 * memoised on already-resolved nodes. */
static void xo_orl(int n, const int32_t *off, const int32_t *idx, int32_t *orl) {
    for (int i = 0; i < n; i++) orl[i] = -1;
    for (int i = 0; i < n; i++) {
        int r = i;
        for (;;) {
            if (off[r + 1] == off[r]) { orl[i] = r; break; }
            if (orl[r] >= 0) { orl[i] = orl[r]; break; }
            r = idx[off[r + 1] - 1];
        }
    }
}

static int xo_cmp_desc(const void *a, const void *b) {
    int x = *(const int *)a, y = *(const int *)b;
    return (x < y) - (x > y);
}

/* X-TED_CPU/TED.cpp:46-77 key_roots: the smallest preorder node of every
 * distinct orl value, sorted in descending order. Returns K. */
static int xo_keyroots(int n, const int32_t *orl, int32_t *kr) {
    int32_t *view = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i < n; i++) view[i] = -1;
    int K = 0;
    for (int i = 0; i < n; i++) {
        int r = orl[i];
        if (view[r] < 0) { view[r] = i; K++; }
    }
    int k = 0;
    for (int r = 0; r < n; r++) if (view[r] >= 0) kr[k++] = view[r];
    qsort(kr, (size_t)K, sizeof(int32_t), xo_cmp_desc);
    free(view);
    return K;
}

/* X-TED_CPU/parallel_computing.cpp:93-107 keyroot depth: 0 for a leaf or a
 * node whose orl is node+1, else 1 + max depth of keyroots inside its
 * subtree (keyroots are visited in the same descending order). */
static void xo_kr_depth(int K, const int32_t *kr, const int32_t *orl, int32_t *d) {
    for (int i = 0; i < K; i++) {
        int node = kr[i];
        d[i] = 0;
        if (node == orl[node] || node == orl[node] - 1) continue;
        for (int j = 0; j < i; j++) {
            int node2 = kr[j];
            if (node <= node2 && orl[node] >= node2) {
                int c = d[j] + 1;
                if (c > d[i]) d[i] = c;
            }
        }
    }
}

/* X-TED_CPU/parallel_computing.cpp:4-45 compute: the forest table of the
 * keyroot pair (k,l), filled from high indices to low. D is (m+1)x(n+1),
 * Dt is m x n, both row-major. The reference's unit costs (its literal 1s
 * at :17-25 and :31-39, and the label test) are the parameters cd (delete
 * a node of the first tree), ci (insert a node of the second) and cr
 * (label change); cd = ci = cr = 1 is the reference exactly. */
static void xo_table(int i0, int j0, const int32_t *xorl, const int32_t *yorl,
                     const int32_t *la, const int32_t *lb, int n,
                     int32_t *D, int32_t *Dt, int cd, int ci, int cr) {
    const size_t ld = (size_t)n + 1;
    int imax = xorl[i0] + 1, jmax = yorl[j0] + 1;
    D[imax * ld + jmax] = 0;
    for (int i = imax - 1; i > i0 - 1; i--) D[i * ld + jmax] = cd + D[(i + 1) * ld + jmax];
    for (int j = jmax - 1; j > j0 - 1; j--) D[imax * ld + j] = ci + D[imax * ld + j + 1];
    for (int i = imax - 1; i > i0 - 1; i--) {
        for (int j = jmax - 1; j > j0 - 1; j--) {
            if ((xorl[i] == xorl[i0]) & (yorl[j] == yorl[j0])) {
                int cost = la[i] != lb[j] ? cr : 0;
                int v = xo_min3(cost + D[(i + 1) * ld + j + 1], cd + D[(i + 1) * ld + j],
                                ci + D[i * ld + j + 1]);
                D[i * ld + j] = v;
                Dt[(size_t)i * n + j] = v;
            } else {
                D[i * ld + j] = xo_min3(Dt[(size_t)i * n + j] + D[(xorl[i] + 1) * ld + yorl[j] + 1],
                                        cd + D[(i + 1) * ld + j], ci + D[i * ld + j + 1]);
            }
        }
    }
}

/* Per-tree preprocessing shared by every table of a pair. */
typedef struct { int32_t *orl, *kr, *dep; int K, maxd; } xo_prep;

static void xo_prep_tree(int n, const int32_t *off, const int32_t *idx, xo_prep *p) {
    p->orl = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
    p->kr = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
    p->dep = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
    xo_orl(n, off, idx, p->orl);
    p->K = xo_keyroots(n, p->orl, p->kr);
    xo_kr_depth(p->K, p->kr, p->orl, p->dep);
    p->maxd = 0;
    for (int i = 0; i < p->K; i++) if (p->dep[i] > p->maxd) p->maxd = p->dep[i];
}

static void xo_prep_free(xo_prep *p) { free(p->orl); free(p->kr); free(p->dep); }

/*
 * X-TED_CPU/TED.cpp:177-190 standard_ted (+ standard_ted_1 :145-174 and the
 * level loop of parallel_computing.cpp:121-182, run sequentially here: any
 * order that finishes every lower level first gives the same table values).
 * Returns the distance, or -1 on allocation failure. With edit costs cd
 * (delete), ci (insert), cr (rename); the empty-tree rules become n * ci and
 * m * cd.
 */
int xo_distance_cost(int m, const int32_t *la, const int32_t *aoff, const int32_t *aidx,
                     int n, const int32_t *lb, const int32_t *boff, const int32_t *bidx,
                     int cd, int ci, int cr) {
    if (m == 0) return n * ci;
    if (n == 0) return m * cd;
    xo_prep A, B;
    xo_prep_tree(m, aoff, aidx, &A);
    xo_prep_tree(n, boff, bidx, &B);
    int32_t *D = (int32_t *)malloc(sizeof(int32_t) * (size_t)(m + 1) * (size_t)(n + 1));
    int32_t *Dt = (int32_t *)malloc(sizeof(int32_t) * (size_t)m * (size_t)n);
    int result = -1;
    if (D && Dt) {
        int maxlev = A.maxd + B.maxd;
        for (int lev = 0; lev <= maxlev; lev++)
            for (int k = 0; k < A.K; k++) {
                int dl = lev - A.dep[k];
                if (dl < 0 || dl > B.maxd) continue;
                for (int l = 0; l < B.K; l++)
                    if (B.dep[l] == dl)
                        xo_table(A.kr[k], B.kr[l], A.orl, B.orl, la, lb, n, D, Dt, cd, ci, cr);
            }
        result = Dt[0];
    }
    free(D);
    free(Dt);
    xo_prep_free(&A);
    xo_prep_free(&B);
    return result;
}

/* The reference's unit-cost distance (X-TED_CPU/TED.cpp:177-190). */
int xo_distance(int m, const int32_t *la, const int32_t *aoff, const int32_t *aidx,
                int n, const int32_t *lb, const int32_t *boff, const int32_t *bidx) {
    return xo_distance_cost(m, la, aoff, aidx, n, lb, boff, bidx, 1, 1, 1);
}

/* Keyroot statistics used by tests: K, max keyroot depth and the sum of
 * keyroot subtree sizes (the per-tree factor of the cell count). */
void xo_tree_stats(int n, const int32_t *off, const int32_t *idx, int64_t *out4) {
    if (n == 0) { out4[0] = out4[1] = out4[2] = out4[3] = 0; return; }
    xo_prep A;
    xo_prep_tree(n, off, idx, &A);
    int64_t s = 0;
    for (int k = 0; k < A.K; k++) s += A.orl[A.kr[k]] - A.kr[k] + 1;
    out4[0] = A.K;
    out4[1] = A.maxd;
    out4[2] = s;
    out4[3] = 0;
    xo_prep_free(&A);
}

/* ---- pair-parallel batch (one pair per worker thread) ---- */
typedef struct {
    int npairs;
    const int32_t *m, *n;                /* sizes per pair */
    const int64_t *a_lab, *a_off, *a_idx; /* offsets into the flat arrays */
    const int64_t *b_lab, *b_off, *b_idx;
    const int32_t *flat;                 /* all int32 data */
    int32_t *out;
    int next;
    pthread_mutex_t mu;
} xo_batch;

static void *xo_worker(void *arg) {
    xo_batch *b = (xo_batch *)arg;
    for (;;) {
        pthread_mutex_lock(&b->mu);
        int p = b->next++;
        pthread_mutex_unlock(&b->mu);
        if (p >= b->npairs) break;
        const int32_t *f = b->flat;
        b->out[p] = xo_distance(b->m[p], f + b->a_lab[p], f + b->a_off[p], f + b->a_idx[p],
                                b->n[p], f + b->b_lab[p], f + b->b_off[p], f + b->b_idx[p]);
    }
    return NULL;
}

/* Distances of npairs pairs with nthreads worker threads (pairs in parallel).
 * Tree data lives in one flat int32 array; the *_lab/_off/_idx arrays hold
 * element offsets into it. */
int xo_distance_batch(int npairs, const int32_t *m, const int32_t *n, const int32_t *flat,
                      const int64_t *a_lab, const int64_t *a_off, const int64_t *a_idx,
                      const int64_t *b_lab, const int64_t *b_off, const int64_t *b_idx,
                      int nthreads, int32_t *out) {
    xo_batch b;
    b.npairs = npairs; b.m = m; b.n = n; b.flat = flat;
    b.a_lab = a_lab; b.a_off = a_off; b.a_idx = a_idx;
    b.b_lab = b_lab; b.b_off = b_off; b.b_idx = b_idx;
    b.out = out; b.next = 0;
    pthread_mutex_init(&b.mu, NULL);
    if (nthreads < 1) nthreads = 1;
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)nthreads);
    for (int t = 0; t < nthreads; t++) pthread_create(&th[t], NULL, xo_worker, &b);
    for (int t = 0; t < nthreads; t++) pthread_join(th[t], NULL);
    free(th);
    pthread_mutex_destroy(&b.mu);
    return 0;
}
