/*
 * UMFPACK-ABI shim for the oracle (test infrastructure only).
 *
 * The reference hot path factors and solves its CSC Jacobian through
 * SuiteSparse UMFPACK (pgabor/sdddst src/simulation.cpp:83,386-396:
 * umfpack_di_symbolic / numeric / solve(UMFPACK_A) / free_*).  UMFPACK is not
 * vendored by the reference and is not installed here, and no version is
 * pinned (cmake/FindUmfpack.cmake:9-22 discovers whatever the system has).
 * This file supplies the same five entry points with a project-written direct
 * solver:
 *   - symbolic: reverse Cuthill-McKee ordering of the symmetrised pattern,
 *   - numeric : banded LU with row partial pivoting on the permuted matrix
 *               (the classic column-major band layout with kl extra rows for
 *               pivoting fill),
 *   - solve   : forward/back substitution followed by up to two steps of
 *               iterative refinement against the original CSC matrix
 *               (UMFPACK's own default is two refinement steps).
 * Any correct LU solve agrees with UMFPACK to about cond(J)*eps; the
 * Jacobians of the implicit scheme are I + O(h) and well conditioned at the
 * adaptive step sizes, so the shim is an adequate stand-in for parity work.
 *
 * Nothing in the product library links this file.
 */
#include "umfpack.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    int n;
    int *perm;  /* perm[new] = old */
    int *iperm; /* iperm[old] = new */
    int kl;     /* half bandwidth of the permuted pattern */
} shim_symbolic;

typedef struct {
    int n, kl, ku, kv, ldab;
    double *ab;
    int *ipiv;
    int *perm, *iperm;
    int singular;
} shim_numeric;

/* ---------------------------------------------------------------- RCM --- */

typedef struct {
    int n;
    int *ptr;
    int *adj;
    int *deg;
} sym_graph;

static int build_sym_graph(int n, const int *Ap, const int *Ai, sym_graph *g)
{
    int *cnt = (int *)calloc((size_t)n + 1, sizeof(int));
    if (!cnt) return -1;
    for (int j = 0; j < n; ++j)
        for (int p = Ap[j]; p < Ap[j + 1]; ++p) {
            int i = Ai[p];
            if (i == j || i < 0 || i >= n) continue;
            cnt[i]++;
            cnt[j]++;
        }
    int *ptr = (int *)malloc(((size_t)n + 1) * sizeof(int));
    ptr[0] = 0;
    for (int i = 0; i < n; ++i) ptr[i + 1] = ptr[i] + cnt[i];
    int *adj = (int *)malloc((size_t)(ptr[n] > 0 ? ptr[n] : 1) * sizeof(int));
    int *fill = (int *)malloc((size_t)n * sizeof(int));
    for (int i = 0; i < n; ++i) fill[i] = ptr[i];
    for (int j = 0; j < n; ++j)
        for (int p = Ap[j]; p < Ap[j + 1]; ++p) {
            int i = Ai[p];
            if (i == j || i < 0 || i >= n) continue;
            adj[fill[i]++] = j;
            adj[fill[j]++] = i;
        }
    /* de-duplicate each list in place */
    int *mark = fill; /* reuse */
    for (int i = 0; i < n; ++i) mark[i] = -1;
    int *deg = (int *)malloc((size_t)n * sizeof(int));
    int w = 0;
    int *nptr = cnt; /* reuse as new ptr */
    for (int i = 0; i < n; ++i) {
        int start = w;
        for (int p = ptr[i]; p < ptr[i + 1]; ++p) {
            int v = adj[p];
            if (mark[v] == i) continue;
            mark[v] = i;
            adj[w++] = v;
        }
        nptr[i] = start;
        deg[i] = w - start;
    }
    nptr[n] = w;
    free(ptr);
    free(fill);
    g->n = n;
    g->ptr = nptr;
    g->adj = adj;
    g->deg = deg;
    return 0;
}

static void free_sym_graph(sym_graph *g)
{
    free(g->ptr);
    free(g->adj);
    free(g->deg);
}

/* BFS from root over unvisited-by-component nodes; returns number of levels,
 * writes the visit order to q (length = component size) and the start of the
 * last level to *last_start. */
static int bfs_levels(const sym_graph *g, int root, int *q, int *lvl, int stamp,
                      int *seen, int *qlen, int *last_start)
{
    int head = 0, tail = 0;
    q[tail++] = root;
    seen[root] = stamp;
    lvl[root] = 0;
    int maxl = 0;
    *last_start = 0;
    while (head < tail) {
        int u = q[head++];
        for (int p = g->ptr[u]; p < g->ptr[u + 1]; ++p) {
            int v = g->adj[p];
            if (seen[v] == stamp) continue;
            seen[v] = stamp;
            lvl[v] = lvl[u] + 1;
            if (lvl[v] > maxl) {
                maxl = lvl[v];
                *last_start = tail;
            }
            q[tail++] = v;
        }
    }
    *qlen = tail;
    return maxl;
}

static int cmp_deg_ctx_deg;
static const int *cmp_deg_arr;
static int cmp_by_degree(const void *a, const void *b)
{
    int da = cmp_deg_arr[*(const int *)a], db = cmp_deg_arr[*(const int *)b];
    if (da != db) return da < db ? -1 : 1;
    return (*(const int *)a) - (*(const int *)b);
}

static void rcm_order(const sym_graph *g, int *perm)
{
    int n = g->n;
    int *visited = (int *)calloc((size_t)n, sizeof(int));
    int *seen = (int *)malloc((size_t)n * sizeof(int));
    int *q = (int *)malloc((size_t)n * sizeof(int));
    int *lvl = (int *)malloc((size_t)n * sizeof(int));
    int *nb = (int *)malloc((size_t)(n > 0 ? n : 1) * sizeof(int));
    for (int i = 0; i < n; ++i) seen[i] = -1;
    int stamp = 0;
    int out = 0;
    cmp_deg_arr = g->deg;
    (void)cmp_deg_ctx_deg;
    for (;;) {
        /* minimum-degree unvisited node starts the next component */
        int root = -1;
        for (int i = 0; i < n; ++i)
            if (!visited[i] && (root < 0 || g->deg[i] < g->deg[root])) root = i;
        if (root < 0) break;
        /* pseudo-peripheral node search (George & Liu) */
        int qlen, last_start;
        int ecc = bfs_levels(g, root, q, lvl, stamp++, seen, &qlen, &last_start);
        for (int it = 0; it < 8; ++it) {
            int cand = q[last_start];
            for (int t = last_start; t < qlen; ++t)
                if (g->deg[q[t]] < g->deg[cand]) cand = q[t];
            int ql2, ls2;
            int e2 = bfs_levels(g, cand, q, lvl, stamp++, seen, &ql2, &ls2);
            if (e2 > ecc) {
                ecc = e2;
                root = cand;
                qlen = ql2;
                last_start = ls2;
            } else {
                break;
            }
        }
        /* Cuthill-McKee from root, neighbours by increasing degree */
        int head = out;
        perm[out++] = root;
        visited[root] = 1;
        while (head < out) {
            int u = perm[head++];
            int k = 0;
            for (int p = g->ptr[u]; p < g->ptr[u + 1]; ++p) {
                int v = g->adj[p];
                if (!visited[v]) {
                    visited[v] = 1;
                    nb[k++] = v;
                }
            }
            qsort(nb, (size_t)k, sizeof(int), cmp_by_degree);
            for (int t = 0; t < k; ++t) perm[out++] = nb[t];
        }
    }
    /* reverse */
    for (int i = 0, j = n - 1; i < j; ++i, --j) {
        int t = perm[i];
        perm[i] = perm[j];
        perm[j] = t;
    }
    free(visited);
    free(seen);
    free(q);
    free(lvl);
    free(nb);
}

/* ------------------------------------------------------ UMFPACK ABI ---- */

int umfpack_di_symbolic(int n_row, int n_col, const int Ap[], const int Ai[],
                        const double Ax[], void **Symbolic,
                        const double Control[], double Info[])
{
    (void)Ax;
    (void)Control;
    (void)Info;
    if (!Symbolic) return -5;
    *Symbolic = NULL;
    if (n_row != n_col || n_row <= 0) return -8;
    int n = n_row;
    shim_symbolic *s = (shim_symbolic *)calloc(1, sizeof(shim_symbolic));
    if (!s) return UMFPACK_ERROR_out_of_memory;
    s->n = n;
    s->perm = (int *)malloc((size_t)n * sizeof(int));
    s->iperm = (int *)malloc((size_t)n * sizeof(int));
    sym_graph g;
    if (build_sym_graph(n, Ap, Ai, &g)) return UMFPACK_ERROR_out_of_memory;
    rcm_order(&g, s->perm);
    for (int i = 0; i < n; ++i) s->iperm[s->perm[i]] = i;
    int kl = 0;
    for (int u = 0; u < n; ++u)
        for (int p = g.ptr[u]; p < g.ptr[u + 1]; ++p) {
            int d = s->iperm[u] - s->iperm[g.adj[p]];
            if (d < 0) d = -d;
            if (d > kl) kl = d;
        }
    s->kl = kl;
    free_sym_graph(&g);
    *Symbolic = s;
    return UMFPACK_OK;
}

#define AB(r, c) nm->ab[(size_t)(nm->kv + (r) - (c)) + (size_t)(c) * (size_t)nm->ldab]

int umfpack_di_numeric(const int Ap[], const int Ai[], const double Ax[],
                       void *Symbolic, void **Numeric,
                       const double Control[], double Info[])
{
    (void)Control;
    (void)Info;
    if (!Numeric || !Symbolic) return -5;
    *Numeric = NULL;
    shim_symbolic *s = (shim_symbolic *)Symbolic;
    int n = s->n;
    shim_numeric *nm = (shim_numeric *)calloc(1, sizeof(shim_numeric));
    if (!nm) return UMFPACK_ERROR_out_of_memory;
    nm->n = n;
    nm->kl = s->kl;
    nm->ku = s->kl;
    nm->kv = nm->kl + nm->ku;
    nm->ldab = 2 * nm->kl + nm->ku + 1;
    nm->ab = (double *)calloc((size_t)nm->ldab * (size_t)n, sizeof(double));
    nm->ipiv = (int *)malloc((size_t)n * sizeof(int));
    nm->perm = (int *)malloc((size_t)n * sizeof(int));
    nm->iperm = (int *)malloc((size_t)n * sizeof(int));
    if (!nm->ab || !nm->ipiv || !nm->perm || !nm->iperm) return UMFPACK_ERROR_out_of_memory;
    memcpy(nm->perm, s->perm, (size_t)n * sizeof(int));
    memcpy(nm->iperm, s->iperm, (size_t)n * sizeof(int));
    for (int j = 0; j < n; ++j)
        for (int p = Ap[j]; p < Ap[j + 1]; ++p) {
            int r = s->iperm[Ai[p]], c = s->iperm[j];
            AB(r, c) += Ax[p];
        }
    /* banded LU with partial pivoting (right-looking, unblocked) */
    int kl = nm->kl, ku = nm->ku;
    int ju = 0;
    for (int j = 0; j < n; ++j) {
        int km = kl < n - 1 - j ? kl : n - 1 - j;
        int jp = 0;
        double best = fabs(AB(j, j));
        for (int t = 1; t <= km; ++t) {
            double a = fabs(AB(j + t, j));
            if (a > best) {
                best = a;
                jp = t;
            }
        }
        nm->ipiv[j] = j + jp;
        if (AB(j + jp, j) == 0.0) {
            nm->singular = 1;
            continue;
        }
        int hi = j + ku + jp;
        if (hi > n - 1) hi = n - 1;
        if (hi > ju) ju = hi;
        if (jp != 0)
            for (int c = j; c <= ju; ++c) {
                double t = AB(j, c);
                AB(j, c) = AB(j + jp, c);
                AB(j + jp, c) = t;
            }
        if (km > 0) {
            double piv = AB(j, j);
            for (int t = 1; t <= km; ++t) AB(j + t, j) /= piv;
            for (int c = j + 1; c <= ju; ++c) {
                double a = AB(j, c);
                if (a == 0.0) continue;
                double *col = &AB(j, c);
                const double *l = &AB(j, j);
                /* rows j+1..j+km of column c sit at col[1..km] */
                for (int t = 1; t <= km; ++t) col[t] -= l[t] * a;
            }
        }
    }
    *Numeric = nm;
    return nm->singular ? UMFPACK_WARNING_singular_matrix : UMFPACK_OK;
}

static void band_solve(const shim_numeric *nm, double *b)
{
    int n = nm->n, kl = nm->kl, kv = nm->kv;
    for (int j = 0; j < n - 1; ++j) {
        int lm = kl < n - 1 - j ? kl : n - 1 - j;
        int l = nm->ipiv[j];
        if (l != j) {
            double t = b[l];
            b[l] = b[j];
            b[j] = t;
        }
        double bj = b[j];
        if (bj != 0.0) {
            const double *lcol = &AB(j, j);
            for (int t = 1; t <= lm; ++t) b[j + t] -= lcol[t] * bj;
        }
    }
    for (int j = n - 1; j >= 0; --j) {
        double d = AB(j, j);
        if (d != 0.0) b[j] /= d;
        double bj = b[j];
        if (bj == 0.0) continue;
        int i0 = j - kv > 0 ? j - kv : 0;
        for (int i = i0; i < j; ++i) b[i] -= bj * AB(i, j);
    }
}

int umfpack_di_solve(int sys, const int Ap[], const int Ai[], const double Ax[],
                     double X[], const double B[], void *Numeric,
                     const double Control[], double Info[])
{
    (void)Control;
    (void)Info;
    if (sys != UMFPACK_A) return UMFPACK_ERROR_invalid_system;
    shim_numeric *nm = (shim_numeric *)Numeric;
    if (!nm) return -5;
    int n = nm->n;
    double *w = (double *)malloc((size_t)n * sizeof(double));
    double *r = (double *)malloc((size_t)n * sizeof(double));
    for (int i = 0; i < n; ++i) w[i] = B[nm->perm[i]];
    band_solve(nm, w);
    for (int i = 0; i < n; ++i) X[nm->perm[i]] = w[i];
    /* iterative refinement: r = B - A X, solve, correct (at most two steps,
     * stop when the residual no longer shrinks) */
    double prev = HUGE_VAL;
    for (int step = 0; step < 2; ++step) {
        for (int i = 0; i < n; ++i) r[i] = B[i];
        for (int j = 0; j < n; ++j) {
            double xj = X[j];
            for (int p = Ap[j]; p < Ap[j + 1]; ++p) r[Ai[p]] -= Ax[p] * xj;
        }
        double nr = 0.0;
        for (int i = 0; i < n; ++i) nr = fmax(nr, fabs(r[i]));
        if (!(nr < 0.5 * prev) || nr == 0.0) break;
        prev = nr;
        for (int i = 0; i < n; ++i) w[i] = r[nm->perm[i]];
        band_solve(nm, w);
        for (int i = 0; i < n; ++i) X[nm->perm[i]] += w[i];
    }
    free(w);
    free(r);
    return nm->singular ? UMFPACK_WARNING_singular_matrix : UMFPACK_OK;
}

void umfpack_di_free_symbolic(void **Symbolic)
{
    if (!Symbolic || !*Symbolic) return;
    shim_symbolic *s = (shim_symbolic *)*Symbolic;
    free(s->perm);
    free(s->iperm);
    free(s);
    *Symbolic = NULL;
}

void umfpack_di_free_numeric(void **Numeric)
{
    if (!Numeric || !*Numeric) return;
    shim_numeric *nm = (shim_numeric *)*Numeric;
    free(nm->ab);
    free(nm->ipiv);
    free(nm->perm);
    free(nm->iperm);
    free(nm);
    *Numeric = NULL;
}

/* Half bandwidth chosen by the last symbolic analysis (diagnostics only). */
int sdddst_shim_bandwidth(void *Symbolic)
{
    return Symbolic ? ((shim_symbolic *)Symbolic)->kl : -1;
}
