/*
 * pf_oracle.c -- CPU restatement of lightsim2grid's AC Newton-Raphson power-flow path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle for the CUDA engine in
 * lightsim2grid_b200/: only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline legs may load it.  The product never links or calls it.
 *
 * What is restated (file:line of the reference project, lightsim2grid 0.13.1):
 *   - mismatch F            src/powerflow_algorithm/BaseAlgo.cpp:30-54 (single slack),
 *                           :56-118 (distributed slack)
 *   - convergence test      BaseAlgo.cpp:120-129 (||F||_inf < tol, strict)
 *   - dS/dVm, dS/dVa        src/powerflow_algorithm/BaseNRAlgo.tpp:202-260
 *   - J pattern + value map BaseNRSingleSlackAlgo.tpp:247-447 (single slack),
 *                           BaseNRAlgo.tpp:396-635 (distributed slack)
 *   - NR driver             BaseNRSingleSlackAlgo.tpp:12-183, BaseNRAlgo.tpp:14-186
 *   - N-1 loop              src/batch_algorithm/ContingencyAnalysis.cpp:14-45 (islanding BFS),
 *                           :112-164 (remove / re-add Ybus coefficients), :166-233 (loop)
 *   - time-series loop      src/batch_algorithm/TimeSeries.cpp:14-109,
 *                           BaseBatchSolverSynch.cpp:14-43, BaseBatchSolverSynch.hpp:277-321
 *
 * The reference factorises J with SuiteSparse KLU (src/linear_solvers/KLUSolver.cpp:24-69),
 * an un-vendored submodule absent from the reference checkout.  KLU's published method
 * (Davis & Palamadai Natarajan, ACM TOMS 37(3), 2010) is a fill-reducing column ordering
 * followed by a left-looking Gilbert-Peierls LU (Gilbert & Peierls, SIAM J. Sci. Stat.
 * Comput. 9(5), 1988) with threshold partial pivoting that prefers the diagonal; later
 * calls refactorise with the pivots of the first factorisation.  This file writes that
 * method from the papers: a minimum-degree ordering (Tinney scheme 2 / Rose 1972) on the
 * pattern of J + J^T, GP factorisation with a 1e-3 diagonal-preference threshold, and a
 * fixed-pivot refactorisation.  KLU's block-triangular pre-ordering is not restated; for
 * the irreducible power-flow Jacobians here it is the identity.
 *
 * Error codes equal the reference's ErrorType ordinals (src/Utils.hpp:47-56).
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef double _Complex cplx;

enum {
    E_NoError = 0,
    E_SingularMatrix = 1,
    E_TooManyIterations = 2,
    E_InifiniteValue = 3,
    E_SolverAnalyze = 4,
    E_SolverFactor = 5,
    E_SolverReFactor = 6,
    E_SolverSolve = 7,
    E_NotInitError = 8,
    E_LicenseError = 9
};

/* ------------------------------------------------------------------------- */
/* small helpers                                                             */
/* ------------------------------------------------------------------------- */

static void *xmalloc(size_t n) {
    void *p = malloc(n ? n : 1);
    if (!p) abort();
    return p;
}
static void *xcalloc(size_t n, size_t s) {
    void *p = calloc(n ? n : 1, s ? s : 1);
    if (!p) abort();
    return p;
}
static void *xrealloc(void *p, size_t n) {
    void *q = realloc(p, n ? n : 1);
    if (!q) abort();
    return q;
}

/* ------------------------------------------------------------------------- */
/* minimum-degree ordering on the pattern of A + A^T (diagonal ignored)      */
/* ------------------------------------------------------------------------- */

typedef struct {
    int *v;
    int n, cap;
} ivec;

static void iv_push(ivec *a, int x) {
    if (a->n == a->cap) {
        a->cap = a->cap ? 2 * a->cap : 8;
        a->v = (int *)xrealloc(a->v, sizeof(int) * (size_t)a->cap);
    }
    a->v[a->n++] = x;
}

/* min-heap of 64-bit keys degree << 31 | label (smaller key: smaller degree, then label) */
typedef struct {
    long long *v;
    int n, cap;
} mdheap;

static long long md_key(int deg, int label) { return ((long long)deg << 31) | (long long)label; }

static void mdh_push(mdheap *h, long long key) {
    if (h->n == h->cap) {
        h->cap = h->cap ? 2 * h->cap : 64;
        h->v = (long long *)xrealloc(h->v, sizeof(long long) * (size_t)h->cap);
    }
    int i = h->n++;
    while (i > 0) {
        const int p = (i - 1) / 2;
        if (h->v[p] <= key) break;
        h->v[i] = h->v[p];
        i = p;
    }
    h->v[i] = key;
}

static long long mdh_pop(mdheap *h) {
    const long long top = h->v[0];
    const long long last = h->v[--h->n];
    int i = 0;
    for (;;) {
        int c = 2 * i + 1;
        if (c >= h->n) break;
        if (c + 1 < h->n && h->v[c + 1] < h->v[c]) ++c;
        if (h->v[c] >= last) break;
        h->v[i] = h->v[c];
        i = c;
    }
    if (h->n > 0) h->v[i] = last;
    return top;
}

static void md_order(int m, const int *Ap, const int *Ai, int *order) {
    ivec *adj = (ivec *)xcalloc((size_t)m, sizeof(ivec));
    int *mark = (int *)xmalloc(sizeof(int) * (size_t)m);
    char *dead = (char *)xcalloc((size_t)m, 1);
    int stamp = 0;
    for (int i = 0; i < m; ++i) mark[i] = -1;
    /* symmetric adjacency, deduplicated */
    for (int j = 0; j < m; ++j) {
        for (int p = Ap[j]; p < Ap[j + 1]; ++p) {
            int i = Ai[p];
            if (i == j) continue;
            iv_push(&adj[i], j);
            iv_push(&adj[j], i);
        }
    }
    for (int i = 0; i < m; ++i) {
        ++stamp;
        int w = 0;
        for (int t = 0; t < adj[i].n; ++t) {
            int u = adj[i].v[t];
            if (mark[u] == stamp) continue;
            mark[u] = stamp;
            adj[i].v[w++] = u;
        }
        adj[i].n = w;
    }
    ivec nb = {0, 0, 0};
    /* the live vertex of least degree, ties to the lowest label: a binary heap of (degree,
       label) keys with lazy deletion (an entry whose degree is no longer current is skipped;
       each degree change pushes a fresh entry), O(fill log m) instead of a scan per pivot */
    mdheap H = {0, 0, 0};
    for (int i = 0; i < m; ++i) mdh_push(&H, md_key(adj[i].n, i));
    for (int k = 0; k < m; ++k) {
        int v = -1;
        while (H.n > 0) {
            const long long top = mdh_pop(&H);
            const int i = (int)(top & 0x7fffffff), d = (int)(top >> 31);
            if (dead[i] || adj[i].n != d) continue;
            v = i;
            break;
        }
        if (v < 0) abort();
        order[k] = v;
        dead[v] = 1;
        nb.n = 0;
        for (int t = 0; t < adj[v].n; ++t) iv_push(&nb, adj[v].v[t]);
        /* every neighbour of v becomes adjacent to every other neighbour of v */
        for (int t = 0; t < nb.n; ++t) {
            int u = nb.v[t];
            ++stamp;
            ivec na = {0, 0, 0};
            mark[u] = stamp;
            mark[v] = stamp;
            for (int s = 0; s < adj[u].n; ++s) {
                int z = adj[u].v[s];
                if (mark[z] == stamp || dead[z]) continue;
                mark[z] = stamp;
                iv_push(&na, z);
            }
            for (int s = 0; s < nb.n; ++s) {
                int z = nb.v[s];
                if (mark[z] == stamp || dead[z]) continue;
                mark[z] = stamp;
                iv_push(&na, z);
            }
            free(adj[u].v);
            adj[u] = na;
            mdh_push(&H, md_key(adj[u].n, u));
        }
        free(adj[v].v);
        adj[v].v = NULL;
        adj[v].n = adj[v].cap = 0;
    }
    free(nb.v);
    free(H.v);
    for (int i = 0; i < m; ++i) free(adj[i].v);
    free(adj);
    free(mark);
    free(dead);
}

/* ------------------------------------------------------------------------- */
/* Gilbert-Peierls sparse LU with threshold partial pivoting and fixed-pivot */
/* refactorisation                                                           */
/* ------------------------------------------------------------------------- */

typedef struct {
    int m;
    int ready;
    int *q;      /* step k factorises column q[k] of A                         */
    int *prow;   /* prow[k] = row of A chosen as pivot at step k               */
    int *pinv;   /* inverse of prow                                            */
    int *Lp, *Li; /* unit-lower L, column k: rows (step numbering) > k         */
    double *Lx;
    int *Up, *Ui; /* U(:,k) off-diagonal entries (steps < k), topological order */
    double *Ux;
    double *Ud;  /* diagonal of U                                              */
    double *x;   /* dense work vector (length m)                               */
    int *xi;     /* DFS work (2m)                                              */
} olu;

static void olu_free(olu *F) {
    free(F->q); free(F->prow); free(F->pinv);
    free(F->Lp); free(F->Li); free(F->Lx);
    free(F->Up); free(F->Ui); free(F->Ux); free(F->Ud);
    free(F->x); free(F->xi);
    memset(F, 0, sizeof(*F));
}

static int olu_factor(olu *F, int m, const int *Ap, const int *Ai, const double *Ax, double thresh) {
    olu_free(F);
    F->m = m;
    F->q = (int *)xmalloc(sizeof(int) * (size_t)m);
    F->prow = (int *)xmalloc(sizeof(int) * (size_t)m);
    F->pinv = (int *)xmalloc(sizeof(int) * (size_t)m);
    F->x = (double *)xcalloc((size_t)m, sizeof(double));
    F->xi = (int *)xmalloc(sizeof(int) * 2 * (size_t)m);
    F->Ud = (double *)xmalloc(sizeof(double) * (size_t)m);
    md_order(m, Ap, Ai, F->q);
    for (int i = 0; i < m; ++i) F->pinv[i] = -1;

    size_t lcap = (size_t)Ap[m] * 2 + (size_t)m, ucap = lcap, ln = 0, un = 0;
    F->Lp = (int *)xmalloc(sizeof(int) * (size_t)(m + 1));
    F->Up = (int *)xmalloc(sizeof(int) * (size_t)(m + 1));
    F->Li = (int *)xmalloc(sizeof(int) * lcap);
    F->Lx = (double *)xmalloc(sizeof(double) * lcap);
    F->Ui = (int *)xmalloc(sizeof(int) * ucap);
    F->Ux = (double *)xmalloc(sizeof(double) * ucap);

    int *visited = (int *)xmalloc(sizeof(int) * (size_t)m);
    int *head = (int *)xmalloc(sizeof(int) * (size_t)m);
    for (int i = 0; i < m; ++i) visited[i] = -1;
    double *x = F->x;
    int *xi = F->xi, *stack = F->xi + m;
    int status = E_NoError;

    for (int k = 0; k < m; ++k) {
        F->Lp[k] = (int)ln;
        F->Up[k] = (int)un;
        int j = F->q[k];
        /* reach: DFS from each row of A(:,j); L rows are stored in A-row numbering */
        int top = m;
        for (int p = Ap[j]; p < Ap[j + 1]; ++p) {
            int r0 = Ai[p];
            if (visited[r0] == k) continue;
            int sp = 0;
            stack[0] = r0;
            visited[r0] = k;
            head[r0] = -1;
            while (sp >= 0) {
                int r = stack[sp];
                int c = F->pinv[r];
                if (head[r] < 0) head[r] = (c >= 0) ? F->Lp[c] : 0;
                int done = 1;
                if (c >= 0) {
                    int end = F->Lp[c + 1];
                    for (int t = head[r]; t < end; ++t) {
                        int r2 = F->Li[t];
                        if (visited[r2] == k) continue;
                        head[r] = t + 1;
                        visited[r2] = k;
                        head[r2] = -1;
                        stack[++sp] = r2;
                        done = 0;
                        break;
                    }
                }
                if (done) {
                    --sp;
                    xi[--top] = r;
                }
            }
        }
        /* numeric: x = L \ A(:,j) on the reach */
        for (int t = top; t < m; ++t) x[xi[t]] = 0.0;
        for (int p = Ap[j]; p < Ap[j + 1]; ++p) x[Ai[p]] = Ax[p];
        for (int t = top; t < m; ++t) {
            int r = xi[t];
            int c = F->pinv[r];
            if (c < 0) continue;
            double xr = x[r];
            for (int s = F->Lp[c]; s < F->Lp[c + 1]; ++s) x[F->Li[s]] -= F->Lx[s] * xr;
        }
        /* pivot: diagonal row j if |x_j| >= thresh * max, else the largest candidate */
        int piv = -1;
        double amax = -1.0;
        for (int t = top; t < m; ++t) {
            int r = xi[t];
            if (F->pinv[r] >= 0) continue;
            double a = fabs(x[r]);
            if (a > amax) {
                amax = a;
                piv = r;
            }
        }
        if (piv < 0 || amax <= 0.0 || !isfinite(amax)) {
            status = E_SolverFactor;
            break;
        }
        if (visited[j] == k && F->pinv[j] < 0 && fabs(x[j]) >= thresh * amax) piv = j;
        double pivot = x[piv];
        F->Ud[k] = pivot;
        F->pinv[piv] = k;
        F->prow[k] = piv;
        /* U(:,k) in topological order, L(:,k) scaled */
        for (int t = top; t < m; ++t) {
            int r = xi[t];
            int c = F->pinv[r];
            if (r == piv) continue;
            if (c >= 0) {
                if (un == ucap) {
                    ucap *= 2;
                    F->Ui = (int *)xrealloc(F->Ui, sizeof(int) * ucap);
                    F->Ux = (double *)xrealloc(F->Ux, sizeof(double) * ucap);
                }
                F->Ui[un] = c;
                F->Ux[un] = x[r];
                ++un;
            } else {
                if (ln == lcap) {
                    lcap *= 2;
                    F->Li = (int *)xrealloc(F->Li, sizeof(int) * lcap);
                    F->Lx = (double *)xrealloc(F->Lx, sizeof(double) * lcap);
                }
                F->Li[ln] = r;
                F->Lx[ln] = x[r] / pivot;
                ++ln;
            }
        }
    }
    F->Lp[m] = (int)ln;
    F->Up[m] = (int)un;
    free(visited);
    free(head);
    if (status != E_NoError) {
        olu_free(F);
        return status;
    }
    /* L rows to step numbering */
    for (size_t t = 0; t < ln; ++t) F->Li[t] = F->pinv[F->Li[t]];
    F->ready = 1;
    return E_NoError;
}

/* numeric refactorisation with the pivots and patterns of the last olu_factor */
static int olu_refactor(olu *F, const int *Ap, const int *Ai, const double *Ax) {
    int m = F->m;
    double *x = F->x;
    for (int k = 0; k < m; ++k) {
        int j = F->q[k];
        for (int t = F->Up[k]; t < F->Up[k + 1]; ++t) x[F->Ui[t]] = 0.0;
        x[k] = 0.0;
        for (int t = F->Lp[k]; t < F->Lp[k + 1]; ++t) x[F->Li[t]] = 0.0;
        for (int p = Ap[j]; p < Ap[j + 1]; ++p) x[F->pinv[Ai[p]]] = Ax[p];
        for (int t = F->Up[k]; t < F->Up[k + 1]; ++t) {
            int c = F->Ui[t];
            double u = x[c];
            F->Ux[t] = u;
            for (int s = F->Lp[c]; s < F->Lp[c + 1]; ++s) x[F->Li[s]] -= F->Lx[s] * u;
        }
        double pivot = x[k];
        if (pivot == 0.0) return E_SolverReFactor;
        F->Ud[k] = pivot;
        for (int t = F->Lp[k]; t < F->Lp[k + 1]; ++t) F->Lx[t] = x[F->Li[t]] / pivot;
    }
    return E_NoError;
}

/* solve A x = b in place */
static void olu_solve(olu *F, double *b) {
    int m = F->m;
    double *y = F->x;
    for (int k = 0; k < m; ++k) y[k] = b[F->prow[k]];
    for (int k = 0; k < m; ++k) {
        double yk = y[k];
        for (int t = F->Lp[k]; t < F->Lp[k + 1]; ++t) y[F->Li[t]] -= F->Lx[t] * yk;
    }
    for (int k = m - 1; k >= 0; --k) {
        double yk = y[k] / F->Ud[k];
        y[k] = yk;
        for (int t = F->Up[k]; t < F->Up[k + 1]; ++t) y[F->Ui[t]] -= F->Ux[t] * yk;
    }
    for (int k = 0; k < m; ++k) b[F->q[k]] = y[k];
}

/* ------------------------------------------------------------------------- */
/* Newton-Raphson solver object                                              */
/* ------------------------------------------------------------------------- */

typedef struct {
    int distributed;      /* 0: KLUSolverSingleSlack semantics, 1: KLUSolver   */
    int n;                /* buses                                             */
    int nnzY;             /* pattern of the Ybus the J pattern was built from  */
    int *Yp, *Yi;         /* copy of that pattern, to detect a change          */
    int npv, npq;         /* as in the last build (npv includes extra slacks)  */
    int *pvpq_key;        /* pv, pq used for the last build                    */
    int slack0;
    /* J (CSC) and its value map */
    int mJ;
    int *Jp, *Ji;
    double *Jx;
    int *map_src;         /* index into dS arrays (Ybus nnz order), -1: constant */
    unsigned char *map_kind; /* 0 Re dVa, 1 Im dVa, 2 Re dVm, 3 Im dVm          */
    cplx *dVm, *dVa;
    olu lu;
    int need_factorize;
    /* state */
    cplx *V;
    double *Vm, *Va;
    int nr_iter;
    int err;
} onr;

static void onr_free_pattern(onr *S) {
    free(S->Yp); free(S->Yi); free(S->pvpq_key);
    free(S->Jp); free(S->Ji); free(S->Jx);
    free(S->map_src); free(S->map_kind);
    free(S->dVm); free(S->dVa);
    S->Yp = S->Yi = S->pvpq_key = NULL;
    S->Jp = S->Ji = NULL;
    S->Jx = NULL;
    S->map_src = NULL;
    S->map_kind = NULL;
    S->dVm = S->dVa = NULL;
    S->mJ = 0;
}

void *oracle_solver_create(int distributed) {
    onr *S = (onr *)xcalloc(1, sizeof(onr));
    S->distributed = distributed ? 1 : 0;
    S->need_factorize = 1;
    S->err = E_NotInitError;
    return S;
}

void oracle_solver_reset(void *h) {
    onr *S = (onr *)h;
    onr_free_pattern(S);
    olu_free(&S->lu);
    free(S->V); free(S->Vm); free(S->Va);
    S->V = NULL; S->Vm = S->Va = NULL;
    S->n = 0;
    S->need_factorize = 1;
    S->nr_iter = 0;
    S->err = E_NotInitError;
}

void oracle_solver_destroy(void *h) {
    oracle_solver_reset(h);
    free(h);
}

/* Ibus = Ybus * V (column-major accumulation, as Eigen's sparse*dense product) */
static void spmv_csc(int n, const int *Yp, const int *Yi, const cplx *Yx, const cplx *V, cplx *out) {
    for (int i = 0; i < n; ++i) out[i] = 0.0;
    for (int c = 0; c < n; ++c) {
        cplx vc = V[c];
        for (int p = Yp[c]; p < Yp[c + 1]; ++p) out[Yi[p]] += Yx[p] * vc;
    }
}

static int all_finite(const double *F, int m) {
    for (int i = 0; i < m; ++i)
        if (!isfinite(F[i])) return 0;
    return 1;
}

static double norm_inf(const double *F, int m) {
    double r = 0.0;
    for (int i = 0; i < m; ++i) {
        double a = fabs(F[i]);
        if (a > r || isnan(a)) r = a;
    }
    return r;
}

/* BaseAlgo.cpp:30-54 and :56-118 */
static void eval_Fx(const onr *S, const int *Yp, const int *Yi, const cplx *Yx, const cplx *V,
                    const cplx *Sbus, const int *mypv, int npv, const int *pq, int npq,
                    double slack_absorbed, const double *w, int slack0, double *F, cplx *work) {
    int n = S->n;
    spmv_csc(n, Yp, Yi, Yx, V, work);
    for (int i = 0; i < n; ++i) {
        cplx mis = V[i] * conj(work[i]) - Sbus[i];
        if (S->distributed) mis += slack_absorbed * w[i];
        work[i] = mis;
    }
    int off = S->distributed ? 1 : 0;
    for (int t = 0; t < npv; ++t) F[off + t] = creal(work[mypv[t]]);
    for (int t = 0; t < npq; ++t) F[off + npv + t] = creal(work[pq[t]]);
    for (int t = 0; t < npq; ++t) F[off + npv + npq + t] = cimag(work[pq[t]]);
    if (S->distributed) F[0] = creal(work[slack0]);
}

/* BaseNRAlgo.tpp:202-260 */
static void dSbus_dV(onr *S, const int *Yp, const int *Yi, const cplx *Yx, const cplx *V, cplx *Ibus) {
    int n = S->n;
    spmv_csc(n, Yp, Yi, Yx, V, Ibus);
    for (int c = 0; c < n; ++c) {
        cplx vnorm_c = V[c] / cabs(V[c]);
        for (int p = Yp[c]; p < Yp[c + 1]; ++p) {
            int r = Yi[p];
            cplx y = Yx[p];
            cplx dvm = conj(y * vnorm_c) * V[r];
            cplx dva = y * V[c];
            if (r == c) {
                cplx vnorm_r = V[r] / cabs(V[r]);
                dvm += conj(Ibus[r]) * vnorm_r;
                dva -= Ibus[r];
            }
            dva = conj(-dva) * (I * V[r]);
            S->dVm[p] = dvm;
            S->dVa[p] = dva;
        }
    }
}

typedef struct {
    int row, col, src;
    unsigned char kind;
    double val;
} jtrip;

static int jtrip_cmp(const void *a, const void *b) {
    const jtrip *x = (const jtrip *)a, *y = (const jtrip *)b;
    if (x->col != y->col) return x->col < y->col ? -1 : 1;
    if (x->row != y->row) return x->row < y->row ? -1 : 1;
    return 0;
}

/* J pattern and value map: BaseNRSingleSlackAlgo.tpp:247-447, BaseNRAlgo.tpp:396-635 */
static void build_J(onr *S, const int *Yp, const int *Yi, const int *pvpq, int npvpq, const int *pq, int npq,
                    const int *pvpq_inv, const int *pq_inv, const double *w, int slack0) {
    int n = S->n;
    int off = S->distributed ? 1 : 0;
    int mJ = npvpq + npq + off;
    size_t cap = (size_t)4 * (size_t)Yp[n] + (size_t)n + 8, nt = 0;
    jtrip *T = (jtrip *)xmalloc(sizeof(jtrip) * cap);
    for (int c = 0; c < npvpq; ++c) {
        int bus = pvpq[c];
        for (int p = Yp[bus]; p < Yp[bus + 1]; ++p) {
            int r = Yi[p];
            if (pvpq_inv[r] >= 0) T[nt++] = (jtrip){pvpq_inv[r] + off, c + off, p, 0, 0.0};
        }
        for (int p = Yp[bus]; p < Yp[bus + 1]; ++p) {
            int r = Yi[p];
            if (pq_inv[r] >= 0) T[nt++] = (jtrip){npvpq + pq_inv[r] + off, c + off, p, 1, 0.0};
        }
    }
    for (int c = 0; c < npq; ++c) {
        int bus = pq[c];
        for (int p = Yp[bus]; p < Yp[bus + 1]; ++p) {
            int r = Yi[p];
            if (pvpq_inv[r] >= 0) T[nt++] = (jtrip){pvpq_inv[r] + off, npvpq + c + off, p, 2, 0.0};
        }
        for (int p = Yp[bus]; p < Yp[bus + 1]; ++p) {
            int r = Yi[p];
            if (pq_inv[r] >= 0) T[nt++] = (jtrip){npvpq + pq_inv[r] + off, npvpq + c + off, p, 3, 0.0};
        }
    }
    if (S->distributed) {
        /* slack-bus row (row 0): BaseNRAlgo.tpp:520-540 */
        for (int c = 0; c < n; ++c) {
            if (pvpq_inv[c] < 0) continue;
            for (int p = Yp[c]; p < Yp[c + 1]; ++p)
                if (Yi[p] == slack0) T[nt++] = (jtrip){0, pvpq_inv[c] + 1, p, 0, 0.0};
        }
        for (int c = 0; c < n; ++c) {
            if (pq_inv[c] < 0) continue;
            for (int p = Yp[c]; p < Yp[c + 1]; ++p)
                if (Yi[p] == slack0) T[nt++] = (jtrip){0, npvpq + pq_inv[c] + 1, p, 2, 0.0};
        }
        /* weight column (column 0): BaseNRAlgo.tpp:542-552 */
        T[nt++] = (jtrip){0, 0, -1, 0, w[slack0]};
        for (int t = 0; t < npvpq; ++t) {
            double sw = w[pvpq[t]];
            if (fabs(sw) > 1e-7) T[nt++] = (jtrip){t + 1, 0, -1, 0, sw};
        }
    }
    qsort(T, nt, sizeof(jtrip), jtrip_cmp);
    S->mJ = mJ;
    S->Jp = (int *)xcalloc((size_t)mJ + 1, sizeof(int));
    S->Ji = (int *)xmalloc(sizeof(int) * nt);
    S->Jx = (double *)xcalloc(nt, sizeof(double));
    S->map_src = (int *)xmalloc(sizeof(int) * nt);
    S->map_kind = (unsigned char *)xmalloc(nt);
    for (size_t t = 0; t < nt; ++t) {
        S->Jp[T[t].col + 1]++;
        S->Ji[t] = T[t].row;
        S->map_src[t] = T[t].src;
        S->map_kind[t] = T[t].kind;
        S->Jx[t] = T[t].val;
    }
    for (int c = 0; c < mJ; ++c) S->Jp[c + 1] += S->Jp[c];
    free(T);
}

static void fill_J_values(onr *S) {
    int nz = S->Jp[S->mJ];
    for (int t = 0; t < nz; ++t) {
        int src = S->map_src[t];
        if (src < 0) continue; /* constant weight column */
        switch (S->map_kind[t]) {
            case 0: S->Jx[t] = creal(S->dVa[src]); break;
            case 1: S->Jx[t] = cimag(S->dVa[src]); break;
            case 2: S->Jx[t] = creal(S->dVm[src]); break;
            default: S->Jx[t] = cimag(S->dVm[src]); break;
        }
    }
}

static int same_pattern(const onr *S, int n, const int *Yp, const int *Yi, const int *mypv, int npv,
                        const int *pq, int npq, int slack0) {
    if (!S->Jp || S->n != n || S->npv != npv || S->npq != npq || S->slack0 != slack0) return 0;
    if (S->nnzY != Yp[n]) return 0;
    if (memcmp(S->Yp, Yp, sizeof(int) * (size_t)(n + 1))) return 0;
    if (memcmp(S->Yi, Yi, sizeof(int) * (size_t)Yp[n])) return 0;
    if (npv && memcmp(S->pvpq_key, mypv, sizeof(int) * (size_t)npv)) return 0;
    if (npq && memcmp(S->pvpq_key + npv, pq, sizeof(int) * (size_t)npq)) return 0;
    return 1;
}

/*
 * compute_pf: BaseNRSingleSlackAlgo.tpp:12-183 (distributed == 0) or BaseNRAlgo.tpp:14-186.
 * Ybus is CSC (n x n) with complex values stored as interleaved (re, im) doubles.
 * V is the start point (not modified); the result is read back with oracle_solver_get_V.
 * Returns 1 when converged, 0 otherwise; -1 on size errors.
 */
int oracle_solver_compute_pf(void *h, int n, const int *Yp, const int *Yi, const double *Yx_ri,
                             const double *V_ri, const double *Sbus_ri, const int *slack_ids, int nslack,
                             const double *slack_weights, const int *pv, int npv_in, const int *pq, int npq,
                             int max_iter, double tol) {
    onr *S = (onr *)h;
    const cplx *Yx = (const cplx *)Yx_ri;
    const cplx *Sbus = (const cplx *)Sbus_ri;
    if (n <= 0 || nslack <= 0) return -1;
    S->err = E_NoError;
    int slack0 = slack_ids[0];
    /* retrieve_pv_with_slack: BaseAlgo.hpp:201-216 (distributed only) */
    int extra = (S->distributed && nslack > 1) ? nslack - 1 : 0;
    int npv = npv_in + extra;
    int *mypv = (int *)xmalloc(sizeof(int) * (size_t)(npv + 1));
    for (int t = 0; t < extra; ++t) mypv[t] = slack_ids[t + 1];
    for (int t = 0; t < npv_in; ++t) mypv[extra + t] = pv[t];
    int npvpq = npv + npq;
    int *pvpq = (int *)xmalloc(sizeof(int) * (size_t)(npvpq + 1));
    memcpy(pvpq, mypv, sizeof(int) * (size_t)npv);
    memcpy(pvpq + npv, pq, sizeof(int) * (size_t)npq);
    int *pvpq_inv = (int *)xmalloc(sizeof(int) * (size_t)n);
    int *pq_inv = (int *)xmalloc(sizeof(int) * (size_t)n);
    for (int i = 0; i < n; ++i) pvpq_inv[i] = pq_inv[i] = -1;
    for (int t = 0; t < npvpq; ++t) pvpq_inv[pvpq[t]] = t;
    for (int t = 0; t < npq; ++t) pq_inv[pq[t]] = t;

    if (!same_pattern(S, n, Yp, Yi, mypv, npv, pq, npq, slack0)) {
        /* a new problem: drop the J pattern, the value map and the factorisation */
        onr_free_pattern(S);
        olu_free(&S->lu);
        S->need_factorize = 1;
        S->n = n;
        S->npv = npv;
        S->npq = npq;
        S->slack0 = slack0;
        S->nnzY = Yp[n];
        S->Yp = (int *)xmalloc(sizeof(int) * (size_t)(n + 1));
        S->Yi = (int *)xmalloc(sizeof(int) * (size_t)(Yp[n] + 1));
        memcpy(S->Yp, Yp, sizeof(int) * (size_t)(n + 1));
        memcpy(S->Yi, Yi, sizeof(int) * (size_t)Yp[n]);
        S->pvpq_key = (int *)xmalloc(sizeof(int) * (size_t)(npvpq + 1));
        memcpy(S->pvpq_key, pvpq, sizeof(int) * (size_t)npvpq);
        S->dVm = (cplx *)xcalloc((size_t)Yp[n] + 1, sizeof(cplx));
        S->dVa = (cplx *)xcalloc((size_t)Yp[n] + 1, sizeof(cplx));
        build_J(S, Yp, Yi, pvpq, npvpq, pq, npq, pvpq_inv, pq_inv, slack_weights, slack0);
        free(S->V); free(S->Vm); free(S->Va);
        S->V = (cplx *)xmalloc(sizeof(cplx) * (size_t)n);
        S->Vm = (double *)xmalloc(sizeof(double) * (size_t)n);
        S->Va = (double *)xmalloc(sizeof(double) * (size_t)n);
    }
    cplx *V = S->V;
    double *Vm = S->Vm, *Va = S->Va;
    memcpy(V, V_ri, sizeof(cplx) * (size_t)n);
    for (int i = 0; i < n; ++i) {
        Vm[i] = cabs(V[i]);
        Va[i] = carg(V[i]);
    }
    int mF = S->mJ;
    double *F = (double *)xmalloc(sizeof(double) * (size_t)mF);
    cplx *work = (cplx *)xmalloc(sizeof(cplx) * (size_t)n);
    double slack_absorbed = 0.0;
    if (S->distributed) {
        for (int i = 0; i < n; ++i) slack_absorbed += creal(Sbus[i]);
    }
    eval_Fx(S, Yp, Yi, Yx, V, Sbus, mypv, npv, pq, npq, slack_absorbed, slack_weights, slack0, F, work);
    int converged = norm_inf(F, mF) < tol;
    S->nr_iter = 0;
    int res = 1;
    int off = S->distributed ? 1 : 0;
    while (!converged && S->nr_iter < max_iter) {
        S->nr_iter++;
        dSbus_dV(S, Yp, Yi, Yx, V, work);
        fill_J_values(S);
        if (S->need_factorize) {
            int st = olu_factor(&S->lu, S->mJ, S->Jp, S->Ji, S->Jx, 1e-3);
            if (st != E_NoError) {
                S->err = st;
                res = 0;
                break;
            }
            S->need_factorize = 0;
        } else {
            int st = olu_refactor(&S->lu, S->Jp, S->Ji, S->Jx);
            if (st != E_NoError) {
                S->err = st;
                res = 0;
                break;
            }
        }
        olu_solve(&S->lu, F);
        if (S->distributed) {
            slack_absorbed -= F[0];
        } else {
            for (int i = 0; i < n; ++i) {
                Vm[i] = cabs(V[i]);
                Va[i] = carg(V[i]);
            }
        }
        for (int t = 0; t < npv; ++t) Va[mypv[t]] -= F[off + t];
        for (int t = 0; t < npq; ++t) Va[pq[t]] -= F[off + npv + t];
        for (int t = 0; t < npq; ++t) Vm[pq[t]] -= F[off + npv + npq + t];
        double vmin = INFINITY;
        for (int i = 0; i < n; ++i) {
            V[i] = Vm[i] * (cos(Va[i]) + I * sin(Va[i]));
            if (Vm[i] < vmin) vmin = Vm[i];
        }
        if (vmin < 0.0) {
            for (int i = 0; i < n; ++i) {
                Vm[i] = cabs(V[i]);
                Va[i] = carg(V[i]);
            }
        }
        eval_Fx(S, Yp, Yi, Yx, V, Sbus, mypv, npv, pq, npq, slack_absorbed, slack_weights, slack0, F, work);
        if (!all_finite(F, mF)) {
            S->err = E_InifiniteValue;
            break;
        }
        converged = norm_inf(F, mF) < tol;
    }
    if (!converged) {
        if (S->err == E_NoError) S->err = E_TooManyIterations;
        res = 0;
    }
    for (int i = 0; i < n; ++i) {
        Vm[i] = cabs(V[i]);
        Va[i] = carg(V[i]);
    }
    free(F); free(work); free(mypv); free(pvpq); free(pvpq_inv); free(pq_inv);
    return res;
}

void oracle_solver_get_V(void *h, double *V_ri) { onr *S = (onr *)h; memcpy(V_ri, S->V, sizeof(cplx) * (size_t)S->n); }
void oracle_solver_get_Vm(void *h, double *out) { onr *S = (onr *)h; memcpy(out, S->Vm, sizeof(double) * (size_t)S->n); }
void oracle_solver_get_Va(void *h, double *out) { onr *S = (onr *)h; memcpy(out, S->Va, sizeof(double) * (size_t)S->n); }
int oracle_solver_get_nb_iter(void *h) { return ((onr *)h)->nr_iter; }
int oracle_solver_get_error(void *h) { return ((onr *)h)->err; }
int oracle_solver_get_n(void *h) { return ((onr *)h)->n; }

/* J of the last iteration (CSC).  Call with NULL buffers to get sizes. */
int oracle_solver_get_J(void *h, int *m, int *Jp, int *Ji, double *Jx) {
    onr *S = (onr *)h;
    if (!S->Jp) return -1;
    int nz = S->Jp[S->mJ];
    if (m) *m = S->mJ;
    if (Jp) memcpy(Jp, S->Jp, sizeof(int) * (size_t)(S->mJ + 1));
    if (Ji) memcpy(Ji, S->Ji, sizeof(int) * (size_t)nz);
    if (Jx) memcpy(Jx, S->Jx, sizeof(double) * (size_t)nz);
    return nz;
}

/* number of stored entries of L and U of the current factorisation (diagnostics) */
int oracle_solver_lu_nnz(void *h) {
    onr *S = (onr *)h;
    if (!S->lu.ready) return -1;
    return S->lu.Lp[S->lu.m] + S->lu.Up[S->lu.m] + S->lu.m;
}

/* ------------------------------------------------------------------------- */
/* batch drivers                                                             */
/* ------------------------------------------------------------------------- */

/* ContingencyAnalysis.cpp:14-45: BFS from bus 0 over entries with |y| > 1e-8 */
static int check_invertible(int n, const int *Yp, const int *Yi, const cplx *Yx, char *visited, char *added, int *queue) {
    memset(visited, 0, (size_t)n);
    memset(added, 0, (size_t)n);
    int qh = 0, qt = 0;
    int col = 0;
    for (;;) {
        visited[col] = 1;
        for (int p = Yp[col]; p < Yp[col + 1]; ++p) {
            int r = Yi[p];
            if (!visited[r] && !added[r] && cabs(Yx[p]) > 1e-8) {
                queue[qt++] = r;
                added[r] = 1;
            }
        }
        if (qh == qt) break;
        col = queue[qh++];
    }
    for (int i = 0; i < n; ++i)
        if (!visited[i]) return 0;
    return 1;
}

static int find_pos(const int *Yp, const int *Yi, int row, int col) {
    for (int p = Yp[col]; p < Yp[col + 1]; ++p)
        if (Yi[p] == row) return p;
    return -1;
}

/*
 * N-1 / N-k batch: ContingencyAnalysis::compute (ContingencyAnalysis.cpp:166-233) with the
 * solver state semantics of BaseBatchSolverSynch::_finish_preprocessing (.hpp:277-321).
 * Each case c removes the coefficients coef_{row,col,val}[cptr[c]..cptr[c+1]) from Ybus
 * (Ybus(row,col) -= val, pattern kept), runs the islanding check, solves from Vinit, and
 * adds them back.  Vout is (ncases x n) complex, zero for skipped / diverged cases.
 * conv[c]: 1 converged, 0 not; iters[c], errs[c]: per case (-1 / NotInitError if islanded).
 * Returns 1 if the base (N) power flow converged, 0 otherwise (then nothing is computed).
 */
int oracle_contingency_analysis(int distributed, int n, const int *Yp, const int *Yi, const double *Yx_ri,
                                const double *Sbus_ri, const double *Vinit_ri, const int *slack_ids, int nslack,
                                const double *w, const int *pv, int npv, const int *pq, int npq, int max_iter,
                                double tol, double sn_mva, int init_from_n, int ncases, const int *cptr,
                                const int *crow, const int *ccol, const double *cval_ri, double *Vout_ri,
                                int *conv, int *iters, int *errs) {
    void *S = oracle_solver_create(distributed);
    int nz = Yp[n];
    cplx *Yx = (cplx *)xmalloc(sizeof(cplx) * (size_t)(nz + 1));
    memcpy(Yx, Yx_ri, sizeof(cplx) * (size_t)nz);
    const cplx *cval = (const cplx *)cval_ri;
    cplx *Vinit = (cplx *)xmalloc(sizeof(cplx) * (size_t)n);
    memcpy(Vinit, Vinit_ri, sizeof(cplx) * (size_t)n);
    memset(Vout_ri, 0, sizeof(cplx) * (size_t)n * (size_t)ncases);
    for (int c = 0; c < ncases; ++c) {
        conv[c] = 0;
        iters[c] = 0;
        errs[c] = E_NotInitError;
    }
    int ok_n = oracle_solver_compute_pf(S, n, Yp, Yi, (const double *)Yx, (const double *)Vinit, Sbus_ri, slack_ids,
                                        nslack, w, pv, npv, pq, npq, max_iter, tol);
    if (ok_n == 1 && init_from_n) oracle_solver_get_V(S, (double *)Vinit);
    if (ok_n != 1) {
        oracle_solver_destroy(S);
        free(Yx);
        free(Vinit);
        return 0;
    }
    char *visited = (char *)xmalloc((size_t)n), *added = (char *)xmalloc((size_t)n);
    int *queue = (int *)xmalloc(sizeof(int) * (size_t)n);
    int *pos = (int *)xmalloc(sizeof(int) * 64);
    cplx *Vc = (cplx *)xmalloc(sizeof(cplx) * (size_t)n);
    for (int c = 0; c < ncases; ++c) {
        int k0 = cptr[c], k1 = cptr[c + 1];
        int nk = k1 - k0;
        if (nk > 64) nk = 64;
        for (int t = 0; t < nk; ++t) {
            int p = find_pos(Yp, Yi, crow[k0 + t], ccol[k0 + t]);
            pos[t] = p;
            if (p >= 0) Yx[p] -= cval[k0 + t];
        }
        int inv = check_invertible(n, Yp, Yi, Yx, visited, added, queue);
        if (inv) {
            int ok = oracle_solver_compute_pf(S, n, Yp, Yi, (const double *)Yx, (const double *)Vinit, Sbus_ri,
                                              slack_ids, nslack, w, pv, npv, pq, npq, max_iter, tol / sn_mva);
            iters[c] = oracle_solver_get_nb_iter(S);
            errs[c] = oracle_solver_get_error(S);
            if (ok == 1) {
                conv[c] = 1;
                oracle_solver_get_V(S, (double *)Vc);
                memcpy(Vout_ri + (size_t)2 * n * c, Vc, sizeof(cplx) * (size_t)n);
            }
        }
        for (int t = 0; t < nk; ++t)
            if (pos[t] >= 0) Yx[pos[t]] += cval[k0 + t];
    }
    free(visited); free(added); free(queue); free(pos); free(Vc);
    oracle_solver_destroy(S);
    free(Yx);
    free(Vinit);
    return 1;
}

/*
 * Time series: TimeSeries::compute_Vs (TimeSeries.cpp:14-109).  Sbus is (nsteps x n)
 * complex, already divided by sn_mva.  Step i starts from step i-1's solution (warm
 * start); the loop stops at the first divergence.  Returns the status (1 all converged,
 * 0 otherwise); Vout rows of steps not solved stay zero.
 */
int oracle_time_series(int distributed, int n, const int *Yp, const int *Yi, const double *Yx_ri,
                       const double *Sbus0_ri, const double *Sbuses_ri, int nsteps, const double *Vinit_ri,
                       const int *slack_ids, int nslack, const double *w, const int *pv, int npv, const int *pq,
                       int npq, int max_iter, double tol, double sn_mva, int init_from_n, double *Vout_ri,
                       int *conv, int *iters, int *errs) {
    void *S = oracle_solver_create(distributed);
    cplx *V = (cplx *)xmalloc(sizeof(cplx) * (size_t)n);
    memcpy(V, Vinit_ri, sizeof(cplx) * (size_t)n);
    memset(Vout_ri, 0, sizeof(cplx) * (size_t)n * (size_t)nsteps);
    for (int s = 0; s < nsteps; ++s) {
        conv[s] = 0;
        iters[s] = 0;
        errs[s] = E_NotInitError;
    }
    int ok_n = oracle_solver_compute_pf(S, n, Yp, Yi, Yx_ri, (const double *)V, Sbus0_ri, slack_ids, nslack, w, pv,
                                        npv, pq, npq, max_iter, tol);
    if (ok_n != 1) {
        oracle_solver_destroy(S);
        free(V);
        return 0;
    }
    if (init_from_n) oracle_solver_get_V(S, (double *)V);
    int status = 1;
    for (int s = 0; s < nsteps; ++s) {
        const double *Sb = Sbuses_ri + (size_t)2 * n * s;
        int ok = oracle_solver_compute_pf(S, n, Yp, Yi, Yx_ri, (const double *)V, Sb, slack_ids, nslack, w, pv, npv,
                                          pq, npq, max_iter, tol / sn_mva);
        iters[s] = oracle_solver_get_nb_iter(S);
        errs[s] = oracle_solver_get_error(S);
        if (ok != 1) {
            status = 0;
            break;
        }
        conv[s] = 1;
        oracle_solver_get_V(S, (double *)V);
        memcpy(Vout_ri + (size_t)2 * n * s, V, sizeof(cplx) * (size_t)n);
    }
    oracle_solver_destroy(S);
    free(V);
    return status;
}
