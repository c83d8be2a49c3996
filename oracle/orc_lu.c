/*
 * TEST INFRASTRUCTURE (oracle), not product code. See espice_oracle.h.
 *
 * Pattern freeze, BTF+AMD column ordering, Gilbert-Peierls sparse LU with
 * threshold pivoting, numeric refactor and the direct.Solver policy,
 * restated in C from the reference:
 *   src/device/Circuit.zig:77-167, src/device/abi.zig:428-457
 *   src/solver/order.zig:78-224 (order), :225-281 (cholCount), :348-680 (amd)
 *   src/solver/sparse_lu.zig:260-622 (factor), :900-1024 (refactor),
 *                            :1140-1224 (solve, solveT)
 *   src/solver/direct.zig:228-383 (factor policy), :486-560 (probe)
 * Compiled with -ffp-contract=off: every a -= b*c rounds twice, as Zig's
 * strict float mode does.
 */
#include "orc_internal.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ */
/* growable arrays                                                     */

void vu_push(vec_u32 *v, uint32_t x) {
    if (v->len == v->cap) {
        v->cap = v->cap ? 2 * v->cap : 64;
        v->a = (uint32_t *)realloc(v->a, v->cap * sizeof(uint32_t));
    }
    v->a[v->len++] = x;
}

void vd_push(vec_f64 *v, double x) {
    if (v->len == v->cap) {
        v->cap = v->cap ? 2 * v->cap : 64;
        v->a = (double *)realloc(v->a, v->cap * sizeof(double));
    }
    v->a[v->len++] = x;
}

uint64_t bits_of(double x) {
    uint64_t u;
    memcpy(&u, &x, 8);
    return u;
}

double of_bits(uint64_t u) {
    double x;
    memcpy(&x, &u, 8);
    return x;
}

/* num.normInf: max of |x_i| by bit pattern, NaN winning. */
double norm_inf(const double *x, size_t n) {
    uint64_t m = 0;
    for (size_t i = 0; i < n; i++) {
        uint64_t b = bits_of(fabs(x[i]));
        if (b > m) m = b;
    }
    return of_bits(m);
}

/* Zig's @max on floats: the non-NaN operand when one is NaN. */
static double zmax(double a, double b) { return fmax(a, b); }

/* ------------------------------------------------------------------ */
/* pattern: abi.PatternBuilder + Circuit.freeze                        */

static int cmp_u64(const void *a, const void *b) {
    uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
    return x < y ? -1 : x > y;
}

typedef struct {
    uint64_t *k;
    size_t len, cap;
} keys_t;

static void key_add(keys_t *k, uint32_t row, uint32_t col) {
    if (row == 0 || col == 0) return; /* ground entries land in the trash slot */
    if (k->len == k->cap) {
        k->cap = k->cap ? 2 * k->cap : 256;
        k->k = (uint64_t *)realloc(k->k, k->cap * sizeof(uint64_t));
    }
    k->k[k->len++] = ((uint64_t)col << 32) | row;
}

int64_t orc_pattern(const orc_circuit *c, uint32_t *col_ptr, uint32_t *row_idx, size_t cap) {
    keys_t k = {0};
    uint32_t n = c->n;
    /* Every diagonal first, ground's included (Circuit.zig:96). */
    for (uint32_t i = 0; i < n; i++) {
        if (k.len == k.cap) {
            k.cap = k.cap ? 2 * k.cap : 256;
            k.k = (uint64_t *)realloc(k.k, k.cap * sizeof(uint64_t));
        }
        k.k[k.len++] = ((uint64_t)i << 32) | i;
    }
    for (uint32_t b = 0; b < c->n_batches; b++) {
        const orc_batch *bt = &c->batches[b];
        int nt = orc_nodes_per(bt->type);
        for (uint32_t id = 0; id < bt->count; id++) {
            const uint32_t *nd = bt->nodes + (size_t)id * nt;
            uint32_t rows[2 * ORC_MAX_E], cols[2 * ORC_MAX_E];
            int ne = dev_pattern(bt->type, nd, bt->params + (size_t)id * orc_params_per(bt->type),
                                 rows, cols);
            for (int e = 0; e < ne; e++) key_add(&k, rows[e], cols[e]);
        }
    }
    qsort(k.k, k.len, sizeof(uint64_t), cmp_u64);
    size_t nnz = 0;
    for (uint32_t j = 0; j <= n; j++) col_ptr[j] = 0;
    uint64_t last = ~(uint64_t)0;
    for (size_t i = 0; i < k.len; i++) {
        if (k.k[i] == last) continue;
        last = k.k[i];
        if (nnz >= cap) {
            free(k.k);
            return -1;
        }
        row_idx[nnz++] = (uint32_t)(last & 0xffffffffu);
        col_ptr[(last >> 32) + 1]++;
    }
    for (uint32_t j = 0; j < n; j++) col_ptr[j + 1] += col_ptr[j];
    free(k.k);
    return (int64_t)nnz;
}

uint32_t find_slot(const uint32_t *col_ptr, const uint32_t *row_idx, uint32_t nnz,
                   uint32_t row, uint32_t col) {
    if (row == 0 || col == 0) return nnz; /* trash */
    uint32_t lo = col_ptr[col], hi = col_ptr[col + 1];
    while (lo < hi) {
        uint32_t mid = lo + (hi - lo) / 2;
        if (row_idx[mid] < row) lo = mid + 1;
        else hi = mid;
    }
    if (lo < col_ptr[col + 1] && row_idx[lo] == row) return lo;
    return nnz;
}

/* ------------------------------------------------------------------ */
/* order.zig                                                           */

static int cmp_u32(const void *a, const void *b) {
    uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
    return x < y ? -1 : x > y;
}

/* order.zig:225-281 cholCount: |L| of the symmetrized pattern in `perm`. */
static uint64_t chol_count(uint32_t n, const uint32_t *cp, const uint32_t *ri, const uint32_t *perm) {
    uint32_t nnz = cp[n];
    uint32_t *pinv = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
    uint32_t *ptr = (uint32_t *)calloc(n + 1, sizeof(uint32_t));
    uint32_t *lst = (uint32_t *)malloc(sizeof(uint32_t) * (nnz ? nnz : 1));
    uint32_t *fill = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
    uint32_t *parent = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
    for (uint32_t k = 0; k < n; k++) pinv[perm[k]] = k;
    for (uint32_t j = 0; j < n; j++)
        for (uint32_t p = cp[j]; p < cp[j + 1]; p++) {
            uint32_t a = pinv[ri[p]], b = pinv[j];
            if (a != b) ptr[(a > b ? a : b) + 1] += 1;
        }
    for (uint32_t k = 1; k <= n; k++) ptr[k] += ptr[k - 1];
    memcpy(fill, ptr, sizeof(uint32_t) * n);
    for (uint32_t j = 0; j < n; j++)
        for (uint32_t p = cp[j]; p < cp[j + 1]; p++) {
            uint32_t a = pinv[ri[p]], b = pinv[j];
            if (a == b) continue;
            uint32_t hi = a > b ? a : b;
            lst[fill[hi]++] = a > b ? b : a;
        }
    uint32_t *anc = fill;
    for (uint32_t k = 0; k < n; k++) {
        parent[k] = NONE;
        anc[k] = NONE;
        for (uint32_t t = ptr[k]; t < ptr[k + 1]; t++) {
            uint32_t i = lst[t];
            while (i != NONE && i < k) {
                uint32_t next = anc[i];
                anc[i] = k;
                if (next == NONE) parent[i] = k;
                i = next;
            }
        }
    }
    uint32_t *flag = anc;
    uint64_t count = 0;
    for (uint32_t k = 0; k < n; k++) {
        flag[k] = k;
        count++;
        for (uint32_t t = ptr[k]; t < ptr[k + 1]; t++) {
            uint32_t i = lst[t];
            while (flag[i] != k) {
                flag[i] = k;
                count++;
                i = parent[i];
            }
        }
    }
    free(pinv);
    free(ptr);
    free(lst);
    free(fill);
    free(parent);
    return count;
}

/* Degree lists (order.zig DegLists). */
typedef struct {
    uint32_t *head, *next, *prev;
} deglists;

static void dl_insert(deglists *s, uint32_t d, uint32_t i) {
    s->next[i] = s->head[d];
    s->prev[i] = NONE;
    if (s->head[d] != NONE) s->prev[s->head[d]] = i;
    s->head[d] = i;
}

static void dl_remove(deglists *s, uint32_t d, uint32_t i) {
    if (s->prev[i] != NONE) s->next[s->prev[i]] = s->next[i];
    else s->head[d] = s->next[i];
    if (s->next[i] != NONE) s->prev[s->next[i]] = s->prev[i];
}

/* Growable slab for the variable and element adjacency spans. `compact`
 * in the reference only slides live spans left and keeps their order, so
 * growing the slab instead yields the same lists. */
typedef struct {
    uint32_t *a;
    size_t cap;
} slab;

static void slab_need(slab *s, size_t need) {
    if (need <= s->cap) return;
    size_t c = s->cap ? s->cap : 64;
    while (c < need) c *= 2;
    s->a = (uint32_t *)realloc(s->a, c * sizeof(uint32_t));
    s->cap = c;
}

static int same_adj(const uint32_t *va, const uint32_t *va_pe, const uint32_t *va_len,
                    const uint32_t *ea, const uint32_t *ea_pe, const uint32_t *ea_len,
                    uint32_t *mark, uint32_t *era, uint32_t i, uint32_t j) {
    if (va_len[i] != va_len[j] || ea_len[i] != ea_len[j]) return 0;
    for (int pass = 0; pass < 2; pass++) {
        const uint32_t *adj = pass == 0 ? va : ea;
        const uint32_t *pos = pass == 0 ? va_pe : ea_pe;
        const uint32_t *len = pass == 0 ? va_len : ea_len;
        *era += 1;
        uint32_t m = *era;
        for (uint32_t t = 0; t < len[i]; t++) mark[adj[pos[i] + t]] = m;
        for (uint32_t t = 0; t < len[j]; t++)
            if (mark[adj[pos[j] + t]] != m) return 0;
    }
    return 1;
}

static uint32_t isqrt_u32(uint32_t n) {
    uint32_t r = (uint32_t)sqrt((double)n);
    while ((uint64_t)r * r > n) r--;
    while ((uint64_t)(r + 1) * (r + 1) <= n) r++;
    return r;
}

/* order.zig:348-680 amd. */
static void amd(uint32_t n, const uint32_t *cp, const uint32_t *ri, uint32_t *q) {
    if (n == 0) return;
    uint32_t nnz = cp[n];
    slab va = {0}, ea = {0};
    slab_need(&va, 4 * (size_t)nnz + 4 * (size_t)n + 16);
    slab_need(&ea, 8 * (size_t)n + nnz);
#define A(name) uint32_t *name = (uint32_t *)malloc(sizeof(uint32_t) * n)
    A(va_pe); A(va_len); A(ea_pe); A(ea_lim); A(esize); A(deg); A(w_buf);
    A(hkey); A(hnext); A(hbuckets); A(lp_buf); A(touched);
#undef A
    uint32_t *ea_len = (uint32_t *)calloc(n, sizeof(uint32_t));
    uint32_t *nv = (uint32_t *)malloc(sizeof(uint32_t) * n);
    uint32_t *elem_alive = (uint32_t *)calloc(n, sizeof(uint32_t));
    uint32_t *mark = (uint32_t *)calloc(n, sizeof(uint32_t));
    uint32_t *wmark = (uint32_t *)calloc(n, sizeof(uint32_t));
    uint32_t *hhead = (uint32_t *)malloc(sizeof(uint32_t) * n);
    uint32_t *mlink = (uint32_t *)malloc(sizeof(uint32_t) * n);
    deglists dl;
    dl.head = (uint32_t *)malloc(sizeof(uint32_t) * (n + 1));
    dl.next = (uint32_t *)malloc(sizeof(uint32_t) * n);
    dl.prev = (uint32_t *)malloc(sizeof(uint32_t) * n);
    for (uint32_t i = 0; i < n; i++) {
        nv[i] = 1;
        hhead[i] = NONE;
        mlink[i] = NONE;
    }
    for (uint32_t i = 0; i <= n; i++) dl.head[i] = NONE;
    uint32_t era = 0, erw = 0;

    memset(deg, 0, sizeof(uint32_t) * n);
    for (uint32_t j = 0; j < n; j++)
        for (uint32_t p = cp[j]; p < cp[j + 1]; p++) {
            uint32_t r = ri[p];
            if (r == j) continue;
            deg[j]++;
            deg[r]++;
        }
    size_t va_free = 0;
    for (uint32_t i = 0; i < n; i++) {
        va_pe[i] = (uint32_t)va_free;
        va_free += deg[i];
    }
    memset(deg, 0, sizeof(uint32_t) * n);
    for (uint32_t j = 0; j < n; j++)
        for (uint32_t p = cp[j]; p < cp[j + 1]; p++) {
            uint32_t r = ri[p];
            if (r == j) continue;
            va.a[va_pe[j] + deg[j]] = r;
            deg[j]++;
            va.a[va_pe[r] + deg[r]] = j;
            deg[r]++;
        }
    memcpy(va_len, deg, sizeof(uint32_t) * n);
    for (uint32_t i = 0; i < n; i++) {
        era++;
        uint32_t wp = 0, s = va_pe[i];
        for (uint32_t t = 0; t < va_len[i]; t++) {
            uint32_t v = va.a[s + t];
            if (mark[v] != era) {
                mark[v] = era;
                va.a[s + wp++] = v;
            }
        }
        va_len[i] = wp;
    }

    uint32_t isq = isqrt_u32(n);
    uint32_t dense_thresh = 10 * isq > 16 ? 10 * isq : 16;
    uint32_t ndense = 0;
    for (uint32_t i = 0; i < n; i++)
        if (va_len[i] >= dense_thresh) ndense++;
    uint32_t dense_start = n - ndense;
    {
        uint32_t di = 0;
        for (uint32_t i = 0; i < n; i++)
            if (va_len[i] >= dense_thresh) {
                nv[i] = 0;
                lp_buf[dense_start + di++] = i;
            }
    }
    if (ndense > 0) {
        for (uint32_t i = 0; i < n; i++) {
            if (nv[i] == 0) continue;
            uint32_t wp = 0, s = va_pe[i];
            for (uint32_t t = 0; t < va_len[i]; t++) {
                uint32_t v = va.a[s + t];
                if (nv[v] != 0) va.a[s + wp++] = v;
            }
            va_len[i] = wp;
        }
    }
    size_t ea_free = 0;
    for (uint32_t i = 0; i < n; i++) {
        ea_pe[i] = (uint32_t)ea_free;
        ea_lim[i] = 4;
        ea_free += 4;
    }
    slab_need(&ea, ea_free);
    for (uint32_t i = 0; i < n; i++) {
        if (nv[i] == 0) continue;
        deg[i] = va_len[i];
        dl_insert(&dl, deg[i], i);
    }

    uint32_t n_amd = n - ndense, mindeg = 0, k = 0;
    while (k < n_amd) {
        while (dl.head[mindeg] == NONE) mindeg++;
        uint32_t p = dl.head[mindeg];
        dl_remove(&dl, deg[p], p);

        era++;
        mark[p] = era;
        uint32_t nlp = 0;
        for (uint32_t t = 0; t < va_len[p]; t++) {
            uint32_t v = va.a[va_pe[p] + t];
            if (nv[v] != 0 && mark[v] != era) {
                mark[v] = era;
                lp_buf[nlp++] = v;
            }
        }
        for (uint32_t t = 0; t < ea_len[p]; t++) {
            uint32_t e = ea.a[ea_pe[p] + t];
            if (elem_alive[e] == 0) continue;
            for (uint32_t u = 0; u < va_len[e]; u++) {
                uint32_t v = va.a[va_pe[e] + u];
                if (nv[v] != 0 && mark[v] != era) {
                    mark[v] = era;
                    lp_buf[nlp++] = v;
                }
            }
            elem_alive[e] = 0;
        }
        uint32_t nvpiv = nv[p];
        nv[p] = 0;
        elem_alive[p] = 1;

        slab_need(&va, va_free + nlp);
        va_pe[p] = (uint32_t)va_free;
        va_len[p] = nlp;
        memcpy(va.a + va_free, lp_buf, sizeof(uint32_t) * nlp);
        va_free += nlp;

        uint32_t lpsize = 0;
        for (uint32_t t = 0; t < nlp; t++) lpsize += nv[lp_buf[t]];
        esize[p] = lpsize;
        for (uint32_t t = 0; t < nlp; t++) dl_remove(&dl, deg[lp_buf[t]], lp_buf[t]);

        erw++;
        uint32_t ntouched = 0;
        for (uint32_t t = 0; t < nlp; t++) {
            uint32_t i = lp_buf[t];
            for (uint32_t u = 0; u < ea_len[i]; u++) {
                uint32_t e = ea.a[ea_pe[i] + u];
                if (elem_alive[e] == 0) continue;
                if (wmark[e] != erw) {
                    wmark[e] = erw;
                    w_buf[e] = esize[e];
                    touched[ntouched++] = e;
                }
                w_buf[e] -= w_buf[e] < nv[i] ? w_buf[e] : nv[i];
            }
        }
        for (uint32_t t = 0; t < ntouched; t++)
            if (w_buf[touched[t]] == 0) elem_alive[touched[t]] = 0;

        for (uint32_t t = 0; t < nlp; t++) {
            uint32_t i = lp_buf[t];
            uint32_t esum = 0, ewp = 0;
            for (uint32_t u = 0; u < ea_len[i]; u++) {
                uint32_t e = ea.a[ea_pe[i] + u];
                if (elem_alive[e] != 0 && e != p) {
                    ea.a[ea_pe[i] + ewp++] = e;
                    esum += w_buf[e];
                }
            }
            if (ewp < ea_lim[i]) {
                ea.a[ea_pe[i] + ewp] = p;
            } else {
                uint32_t nc = (ewp + 1) * 2;
                slab_need(&ea, ea_free + nc);
                memmove(ea.a + ea_free, ea.a + ea_pe[i], sizeof(uint32_t) * ewp);
                ea.a[ea_free + ewp] = p;
                ea_pe[i] = (uint32_t)ea_free;
                ea_lim[i] = nc;
                ea_free += nc;
            }
            ea_len[i] = ewp + 1;

            uint32_t asum = 0, vwp = 0;
            for (uint32_t u = 0; u < va_len[i]; u++) {
                uint32_t v = va.a[va_pe[i] + u];
                if (nv[v] != 0 && mark[v] != era) {
                    va.a[va_pe[i] + vwp++] = v;
                    asum += nv[v];
                }
            }
            va_len[i] = vwp;
            uint32_t capd = n_amd - k - nvpiv;
            uint32_t d = asum + (lpsize - nv[i]) + esum;
            deg[i] = d < capd ? d : capd;
        }

        uint32_t nhb = 0;
        for (uint32_t t = 0; t < nlp; t++) {
            uint32_t i = lp_buf[t];
            if (nv[i] == 0) continue;
            uint32_t h = 0;
            for (uint32_t u = 0; u < va_len[i]; u++) h += va.a[va_pe[i] + u];
            for (uint32_t u = 0; u < ea_len[i]; u++) h += ea.a[ea_pe[i] + u];
            hkey[i] = h;
            uint32_t b = h % n;
            if (hhead[b] == NONE) hbuckets[nhb++] = b;
            hnext[i] = hhead[b];
            hhead[b] = i;
        }
        for (uint32_t t = 0; t < nhb; t++) {
            uint32_t b = hbuckets[t];
            for (uint32_t i = hhead[b]; i != NONE; i = hnext[i]) {
                if (nv[i] == 0) continue;
                for (uint32_t j = hnext[i]; j != NONE; j = hnext[j]) {
                    if (nv[j] == 0 || hkey[j] != hkey[i]) continue;
                    if (!same_adj(va.a, va_pe, va_len, ea.a, ea_pe, ea_len, mark, &era, i, j)) continue;
                    deg[i] -= deg[i] < nv[j] ? deg[i] : nv[j];
                    nv[i] += nv[j];
                    nv[j] = 0;
                    uint32_t tail = j;
                    while (mlink[tail] != NONE) tail = mlink[tail];
                    mlink[tail] = mlink[i];
                    mlink[i] = j;
                }
            }
            hhead[b] = NONE;
        }
        for (uint32_t t = 0; t < nlp; t++) {
            uint32_t i = lp_buf[t];
            if (nv[i] == 0) continue;
            dl_insert(&dl, deg[i], i);
            if (deg[i] < mindeg) mindeg = deg[i];
        }
        q[k++] = p;
        for (uint32_t mb = mlink[p]; mb != NONE; mb = mlink[mb]) q[k++] = mb;
    }
    memcpy(q + k, lp_buf + dense_start, sizeof(uint32_t) * ndense);

    free(va.a); free(ea.a); free(va_pe); free(va_len); free(ea_pe); free(ea_lim);
    free(esize); free(deg); free(w_buf); free(hkey); free(hnext); free(hbuckets);
    free(lp_buf); free(touched); free(ea_len); free(nv); free(elem_alive); free(mark);
    free(wmark); free(hhead); free(mlink); free(dl.head); free(dl.next); free(dl.prev);
}

/* order.zig:78-224: Tarjan BTF, sink block first, AMD or natural per block. */
int orc_order(uint32_t n, const uint32_t *cp, const uint32_t *ri, uint32_t *q) {
    if (n == 0) return 0;
#define A(name) uint32_t *name = (uint32_t *)malloc(sizeof(uint32_t) * (n + 1))
    A(num); A(low); A(on); A(scc); A(fv); A(fp); A(emit); A(bptr); A(blk_of); A(loc);
#undef A
    for (uint32_t i = 0; i < n; i++) {
        num[i] = NONE;
        on[i] = 0;
    }
    uint32_t sp = 0, fpn = 0, counter = 0, no = 0, nb = 0;
    bptr[0] = 0;
    for (uint32_t root = 0; root < n; root++) {
        if (num[root] != NONE) continue;
        num[root] = counter;
        low[root] = counter;
        counter++;
        scc[sp++] = root;
        on[root] = 1;
        fv[fpn] = root;
        fp[fpn] = cp[root];
        fpn++;
        while (fpn > 0) {
            uint32_t v = fv[fpn - 1];
            if (fp[fpn - 1] < cp[v + 1]) {
                uint32_t child = ri[fp[fpn - 1]];
                fp[fpn - 1]++;
                if (child == v) continue;
                if (num[child] == NONE) {
                    num[child] = counter;
                    low[child] = counter;
                    counter++;
                    scc[sp++] = child;
                    on[child] = 1;
                    fv[fpn] = child;
                    fp[fpn] = cp[child];
                    fpn++;
                } else if (on[child]) {
                    if (num[child] < low[v]) low[v] = num[child];
                }
                continue;
            }
            if (low[v] == num[v]) {
                for (;;) {
                    sp--;
                    uint32_t m = scc[sp];
                    on[m] = 0;
                    emit[no++] = m;
                    if (m == v) break;
                }
                nb++;
                bptr[nb] = no;
            }
            fpn--;
            if (fpn > 0) {
                uint32_t u = fv[fpn - 1];
                if (low[v] < low[u]) low[u] = low[v];
            }
        }
    }
    for (uint32_t b = 0; b < nb; b++)
        for (uint32_t i = bptr[b], li = 0; i < bptr[b + 1]; i++, li++) {
            blk_of[emit[i]] = b;
            loc[emit[i]] = li;
        }
    for (uint32_t b = 0; b < nb; b++) {
        uint32_t lo = bptr[b], hi = bptr[b + 1], bs = hi - lo;
        const uint32_t *verts = emit + lo;
        if (bs == 1) {
            q[lo] = verts[0];
            continue;
        }
        uint32_t *sub_cp = (uint32_t *)malloc(sizeof(uint32_t) * (bs + 1));
        uint32_t sub_nnz = 0;
        sub_cp[0] = 0;
        for (uint32_t j = 0; j < bs; j++) {
            uint32_t v = verts[j];
            for (uint32_t p = cp[v]; p < cp[v + 1]; p++)
                if (blk_of[ri[p]] == b) sub_nnz++;
            sub_cp[j + 1] = sub_nnz;
        }
        uint32_t *sub_ri = (uint32_t *)malloc(sizeof(uint32_t) * (sub_nnz ? sub_nnz : 1));
        uint32_t w = 0;
        for (uint32_t j = 0; j < bs; j++) {
            uint32_t v = verts[j];
            for (uint32_t p = cp[v]; p < cp[v + 1]; p++)
                if (blk_of[ri[p]] == b) sub_ri[w++] = loc[ri[p]];
        }
        uint32_t *sub_q = (uint32_t *)malloc(sizeof(uint32_t) * bs);
        amd(bs, sub_cp, sub_ri, sub_q);
        uint32_t *nat = (uint32_t *)malloc(sizeof(uint32_t) * bs);
        memcpy(nat, verts, sizeof(uint32_t) * bs);
        qsort(nat, bs, sizeof(uint32_t), cmp_u32);
        for (uint32_t i = 0; i < bs; i++) nat[i] = loc[nat[i]];
        const uint32_t *ord = chol_count(bs, sub_cp, sub_ri, nat) < chol_count(bs, sub_cp, sub_ri, sub_q) ? nat : sub_q;
        for (uint32_t i = 0; i < bs; i++) q[lo + i] = verts[ord[i]];
        free(sub_cp);
        free(sub_ri);
        free(sub_q);
        free(nat);
    }
    free(num); free(low); free(on); free(scc); free(fv); free(fp); free(emit); free(bptr);
    free(blk_of); free(loc);
    return 0;
}

/* ------------------------------------------------------------------ */
/* sparse_lu.zig SparseLu                                              */

void slu_init(slu_t *s, uint32_t n, const uint32_t *cp, const uint32_t *ri, const uint32_t *q) {
    memset(s, 0, sizeof(*s));
    s->n = n;
    s->nnz = cp[n];
    s->cp = cp;
    s->ri = ri;
    s->q = q;
    size_t nn = n ? n : 1;
    s->pinv = (uint32_t *)malloc(sizeof(uint32_t) * nn);
    s->lp = (uint32_t *)calloc(n + 1, sizeof(uint32_t));
    s->up = (uint32_t *)calloc(n + 1, sizeof(uint32_t));
    s->udiag = (double *)calloc(nn, sizeof(double));
    s->prow = (uint32_t *)malloc(sizeof(uint32_t) * (s->nnz ? s->nnz : 1));
    s->void_col = (uint8_t *)calloc(nn, 1);
    s->scaled = (uint8_t *)calloc(nn, 1);
    s->w = (double *)calloc(nn, sizeof(double));
    s->y = (double *)calloc(nn, sizeof(double));
    s->rscale = (double *)calloc(nn, sizeof(double));
    s->prev = (uint32_t *)calloc(nn, sizeof(uint32_t));
    s->want = (uint32_t *)malloc(sizeof(uint32_t) * nn);
    s->want_of = (uint32_t *)malloc(sizeof(uint32_t) * nn);
    s->flag = (uint32_t *)malloc(sizeof(uint32_t) * nn);
    s->topo = (uint32_t *)malloc(sizeof(uint32_t) * nn);
    s->stack = (uint32_t *)malloc(sizeof(uint32_t) * nn);
    s->pstack = (uint32_t *)malloc(sizeof(uint32_t) * nn);
}

void slu_free(slu_t *s) {
    free(s->pinv); free(s->lp); free(s->up); free(s->udiag); free(s->prow);
    free(s->void_col); free(s->scaled); free(s->w); free(s->y); free(s->rscale);
    free(s->prev); free(s->want); free(s->want_of); free(s->flag); free(s->topo);
    free(s->stack); free(s->pstack);
    free(s->li.a); free(s->lx.a); free(s->ui.a); free(s->ux.a); free(s->void_slots.a);
    memset(s, 0, sizeof(*s));
}

/* sparse_lu.zig voidUnknown. */
static int void_unknown(const slu_t *s, const double *vals, uint32_t c) {
    if (s->pinv[c] != NONE) return 0;
    for (uint32_t p = s->cp[c]; p < s->cp[c + 1]; p++)
        if (vals[p] != 0) return 0;
    for (uint32_t j = 0; j < s->n; j++) {
        if (j == c) continue;
        for (uint32_t p = s->cp[j]; p < s->cp[j + 1]; p++)
            if (s->ri[p] == c && vals[p] != 0) return 0;
    }
    return 1;
}

enum { FP_OK = 0, FP_SINGULAR = 1, FP_CAPPED = 2 };

/* sparse_lu.zig factorPass. The reference switches to a supernodal copy of
 * the loop once an L column reaches 32 rows; its `lend` shortcut only skips
 * rows the DFS has already marked, and its panel updates subtract in the
 * same order per row (`panelRun`'s own contract), so the plain column loop
 * below gives the same pattern, pivots and values. */
static int factor_pass(slu_t *s, const double *vals, double pivot_tol, size_t cap, int keep_prev) {
    uint32_t n = s->n;
    const uint32_t *cp = s->cp, *ri = s->ri;
    s->factored = 0;
    for (uint32_t i = 0; i < n; i++) {
        s->pinv[i] = NONE;
        s->flag[i] = 0;
        s->void_col[i] = 0;
        s->scaled[i] = 0;
    }
    s->li.len = s->lx.len = s->ui.len = s->ux.len = s->void_slots.len = 0;
    int has_void = 0;
    for (uint32_t i = 0; i < n; i++) s->rscale[i] = 0;
    if (!(norm_inf(vals, s->nnz) <= 1.7976931348623157e308)) return FP_SINGULAR;
    for (uint32_t j = 0; j < n; j++)
        for (uint32_t p = cp[j]; p < cp[j + 1]; p++)
            s->rscale[ri[p]] = zmax(s->rscale[ri[p]], fabs(vals[p]));
    for (uint32_t i = 0; i < n; i++) {
        double v = s->rscale[i];
        s->rscale[i] = (v > 0 && isfinite(v)) ? 1 / v : 1;
    }
    uint32_t *pinv = s->pinv, *flag = s->flag, *stack = s->stack, *pstack = s->pstack;
    uint32_t *topo = s->topo, *lp = s->lp, *want = s->want, *want_of = s->want_of;
    double *w = s->w;
    uint64_t nonfinite = 0;
    for (uint32_t i = 0; i < n; i++) want[i] = keep_prev ? s->prev[i] : i;
    for (uint32_t c = 0; c < n; c++) want_of[want[c]] = c;

    for (uint32_t k = 0; k < n; k++) {
        uint32_t c = s->q[k];
        lp[k] = (uint32_t)s->li.len;
        s->up[k] = (uint32_t)s->ui.len;
        uint32_t mark = k + 1;
        uint32_t nt = 0;
        for (uint32_t p = cp[c]; p < cp[c + 1]; p++) {
            uint32_t r = ri[p];
            if (flag[r] == mark) continue;
            uint32_t sp = 0;
            stack[0] = r;
            pstack[0] = pinv[r] == NONE ? 0 : lp[pinv[r]];
            flag[r] = mark;
            for (;;) {
                r = stack[sp];
                uint32_t kc = pinv[r];
                uint32_t end = kc == NONE ? 0 : lp[kc + 1];
                uint32_t pos = pstack[sp];
                int descended = 0;
                while (pos < end) {
                    uint32_t child = s->li.a[pos++];
                    if (flag[child] != mark) {
                        pstack[sp] = pos;
                        flag[child] = mark;
                        sp++;
                        stack[sp] = child;
                        pstack[sp] = pinv[child] == NONE ? 0 : lp[pinv[child]];
                        descended = 1;
                        break;
                    }
                }
                if (descended) continue;
                topo[nt++] = r;
                if (sp == 0) break;
                sp--;
            }
        }
        for (uint32_t p = cp[c]; p < cp[c + 1]; p++) w[ri[p]] = vals[p];
        for (uint32_t idx = nt; idx > 0;) {
            idx--;
            uint32_t r = topo[idx];
            uint32_t kc = pinv[r];
            if (kc == NONE) continue;
            double ukr = w[r];
            vu_push(&s->ui, kc);
            vd_push(&s->ux, ukr);
            for (uint32_t t = lp[kc]; t < lp[kc + 1]; t++) w[s->li.a[t]] -= s->lx.a[t] * ukr;
        }
        double amax = 0, smax = 0;
        uint32_t piv = NONE;
        for (uint32_t t = 0; t < nt; t++) {
            uint32_t r = topo[t];
            if (pinv[r] != NONE) continue;
            double a = fabs(w[r]);
            if (a > amax) {
                amax = a;
                piv = r;
            }
            smax = zmax(smax, a * s->rscale[r]);
        }
        if (piv == NONE || amax == 0 || !isfinite(amax)) {
            if (!void_unknown(s, vals, c)) {
                for (uint32_t t = 0; t < nt; t++) w[topo[t]] = 0;
                return FP_SINGULAR;
            }
            s->void_col[k] = 1;
            has_void = 1;
            s->udiag[k] = 1;
            pinv[c] = k;
            for (uint32_t t = 0; t < nt; t++) w[topo[t]] = 0;
            continue;
        }
        uint32_t pr = want[c];
        if (pinv[pr] == NONE) {
            double dmag = fabs(w[pr]);
            if (keep_prev) {
                if (dmag > 0 && dmag >= s->keep_min * amax) piv = pr;
            } else if (dmag > 0 && dmag >= pivot_tol * amax) {
                piv = pr;
            } else if (dmag > 0 && dmag * s->rscale[pr] >= pivot_tol * smax) {
                piv = pr;
                s->scaled[k] = 1;
            }
        }
        if (piv != pr) {
            uint32_t c2 = want_of[piv];
            want[c2] = pr;
            want_of[pr] = c2;
        }
        double d = w[piv];
        s->udiag[k] = d;
        pinv[piv] = k;
        for (uint32_t t = 0; t < nt; t++) {
            uint32_t r = topo[t];
            double v = w[r];
            nonfinite |= bits_of(v - v);
            if (pinv[r] == NONE) {
                double l = v / d;
                nonfinite |= bits_of(l - l);
                vu_push(&s->li, r);
                vd_push(&s->lx, l);
            }
            w[r] = 0;
        }
        if (s->li.len + s->ui.len > cap) return FP_CAPPED;
    }
    lp[n] = (uint32_t)s->li.len;
    s->up[n] = (uint32_t)s->ui.len;
    if (nonfinite != 0) return FP_SINGULAR;
    for (size_t t = 0; t < s->li.len; t++) s->li.a[t] = pinv[s->li.a[t]];
    for (uint32_t p = 0; p < s->nnz; p++) s->prow[p] = pinv[ri[p]];
    if (has_void) {
        for (uint32_t j = 0; j < n; j++) {
            uint32_t c = s->q[j];
            for (uint32_t p = cp[c]; p < cp[c + 1]; p++)
                if (s->void_col[j] || s->void_col[s->prow[p]]) vu_push(&s->void_slots, p);
        }
    }
    s->epoch++;
    s->factored = 1;
    return FP_OK;
}

/* sparse_lu.zig factor. 0 ok, 1 singular. */
int slu_factor(slu_t *s, const double *vals, double pivot_tol) {
    int repivot = s->factored && s->fill_cap > 0 && s->base_lu > 0;
    size_t cap = (size_t)-1;
    if (repivot) {
        for (uint32_t r = 0; r < s->n; r++) s->prev[s->q[s->pinv[r]]] = r;
        double cf = s->fill_cap * (double)s->base_lu;
        if (cf > 1e18) cf = 1e18;
        cap = (size_t)cf;
    }
    int rc = factor_pass(s, vals, pivot_tol, cap, 0);
    if (rc == FP_CAPPED) rc = factor_pass(s, vals, pivot_tol, (size_t)-1, 1);
    if (rc != FP_OK) {
        s->factored = 0;
        return 1;
    }
    if (!repivot) s->base_lu = s->li.len + s->ui.len;
    return 0;
}

/* sparse_lu.zig refactor + refactorColumns. 0 ok, 1 singular. */
int slu_refactor(slu_t *s, const double *vals, double growth) {
    for (size_t t = 0; t < s->void_slots.len; t++)
        if (vals[s->void_slots.a[t]] != 0) return 1;
    uint32_t n = s->n;
    const uint32_t *li = s->li.a, *ui = s->ui.a, *lp = s->lp, *up = s->up;
    double *lx = s->lx.a, *ux = s->ux.a, *w = s->w;
    uint64_t nonfinite = 0;
    for (uint32_t k = 0; k < n; k++) {
        uint32_t c = s->q[k];
        for (uint32_t p = s->cp[c]; p < s->cp[c + 1]; p++) w[s->prow[p]] = vals[p];
        for (uint32_t p = up[k]; p < up[k + 1]; p++) {
            uint32_t i = ui[p];
            double uki = w[i];
            w[i] = 0;
            ux[p] = uki;
            nonfinite |= bits_of(uki - uki);
            for (uint32_t t = lp[i]; t < lp[i + 1]; t++) w[li[t]] -= lx[t] * uki;
        }
        if (s->void_col[k]) {
            s->udiag[k] = 1;
            for (uint32_t p = lp[k]; p < lp[k + 1]; p++) {
                lx[p] = 0;
                w[li[p]] = 0;
            }
            w[k] = 0;
            for (uint32_t p = up[k]; p < up[k + 1]; p++) {
                uint32_t i = ui[p];
                for (uint32_t t = lp[i]; t < lp[i + 1]; t++) w[li[t]] = 0;
            }
            continue;
        }
        double d = w[k];
        w[k] = 0;
        if (d == 0 || !isfinite(d)) {
            for (uint32_t p = lp[k]; p < lp[k + 1]; p++) w[li[p]] = 0;
            return 1;
        }
        s->udiag[k] = d;
        if (growth > 0 && !s->scaled[k]) {
            uint64_t cbits = bits_of(fabs(d));
            for (uint32_t p = lp[k]; p < lp[k + 1]; p++) {
                uint32_t r = li[p];
                double v = w[r];
                w[r] = 0;
                uint64_t b = bits_of(fabs(v));
                if ((int64_t)b > (int64_t)cbits) cbits = b;
                lx[p] = v / d;
            }
            double cmax = of_bits(cbits);
            if (!(fabs(d) >= growth * cmax)) return 1;
        } else {
            for (uint32_t p = lp[k]; p < lp[k + 1]; p++) {
                uint32_t r = li[p];
                double l = w[r] / d;
                nonfinite |= bits_of(l - l);
                lx[p] = l;
                w[r] = 0;
            }
        }
    }
    return nonfinite != 0;
}

/* sparse_lu.zig solve (x may alias b). */
void slu_solve(slu_t *s, const double *b, double *x) {
    uint32_t n = s->n;
    double *y = s->y;
    for (uint32_t r = 0; r < n; r++) y[s->pinv[r]] = b[r];
    for (uint32_t k = 0; k < n; k++) {
        double yk = y[k];
        if (yk == 0) continue;
        for (uint32_t p = s->lp[k]; p < s->lp[k + 1]; p++) y[s->li.a[p]] -= s->lx.a[p] * yk;
    }
    for (uint32_t k = n; k > 0;) {
        k--;
        double zk = y[k] / s->udiag[k];
        y[k] = zk;
        if (zk == 0) continue;
        for (uint32_t p = s->up[k]; p < s->up[k + 1]; p++) y[s->ui.a[p]] -= s->ux.a[p] * zk;
    }
    for (uint32_t j = 0; j < n; j++) x[s->q[j]] = y[j];
}

/* sparse_lu.zig solveT. */
void slu_solve_t(slu_t *s, const double *b, double *x) {
    uint32_t n = s->n;
    double *y = s->y;
    for (uint32_t k = 0; k < n; k++) y[k] = b[s->q[k]];
    for (uint32_t k = 0; k < n; k++) {
        double yk = y[k];
        for (uint32_t p = s->up[k]; p < s->up[k + 1]; p++) yk -= s->ux.a[p] * y[s->ui.a[p]];
        y[k] = yk / s->udiag[k];
    }
    for (uint32_t k = n; k > 0;) {
        k--;
        double yk = y[k];
        for (uint32_t p = s->lp[k]; p < s->lp[k + 1]; p++) yk -= s->lx.a[p] * y[s->li.a[p]];
        y[k] = yk;
    }
    for (uint32_t r = 0; r < n; r++) x[r] = y[s->pinv[r]];
}

/* ------------------------------------------------------------------ */
/* direct.zig Solver (general sparse LU engine)                        */

void dsv_init(dsv_t *d, uint32_t n, const uint32_t *cp, const uint32_t *ri) {
    memset(d, 0, sizeof(*d));
    d->n = n;
    d->cp = cp;
    d->ri = ri;
    d->q = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
    orc_order(n, cp, ri, d->q);
    slu_init(&d->lu, n, cp, ri, d->q);
    d->vcopy = (double *)calloc(cp[n] ? cp[n] : 1, sizeof(double));
    d->probe = (double *)calloc(3 * (size_t)(n ? n : 1), sizeof(double));
}

void dsv_free(dsv_t *d) {
    slu_free(&d->lu);
    free(d->q);
    free(d->vcopy);
    free(d->probe);
    memset(d, 0, sizeof(*d));
}

/* direct.zig maxMultiplier. */
static double max_multiplier(const slu_t *lu) {
    double all = norm_inf(lu->lx.a, lu->lx.len);
    int any_scaled = 0;
    for (uint32_t k = 0; k < lu->n; k++) any_scaled |= lu->scaled[k];
    if (isnan(all) || !any_scaled) return all;
    double m = 0;
    for (uint32_t k = 0; k < lu->n; k++) {
        if (lu->scaled[k]) continue;
        m = zmax(m, norm_inf(lu->lx.a + lu->lp[k], lu->lp[k + 1] - lu->lp[k]));
    }
    return m;
}

static void probe_rhs(double *b, uint32_t n) {
    double den = (double)((n > 2 ? n : 2) - 1);
    for (uint32_t i = 0; i < n; i++) {
        double mag = 1 + (double)i / den;
        b[i] = i % 2 == 0 ? mag : -mag;
    }
}

/* direct.zig replayHolds. */
static int replay_holds(dsv_t *d, const double *vals) {
    slu_t *lu = &d->lu;
    if (max_multiplier(lu) <= 1 / PIVOT_TOL) return 1;
    uint32_t n = d->n;
    double *x = d->probe, *r = d->probe + n, *rows = d->probe + 2 * (size_t)n;
    memset(rows, 0, sizeof(double) * n);
    double norm_1 = 0;
    for (uint32_t j = 0; j < n; j++) {
        double col = 0;
        for (uint32_t p = d->cp[j]; p < d->cp[j + 1]; p++) {
            double a = fabs(vals[p]);
            rows[d->ri[p]] += a;
            col += a;
        }
        norm_1 = zmax(norm_1, col);
    }
    double norm_infv = norm_inf(rows, n);
    double nf = (double)n;
    for (int transpose = 0; transpose < 2; transpose++) {
        probe_rhs(r, n);
        if (transpose) slu_solve_t(lu, r, x);
        else slu_solve(lu, r, x);
        probe_rhs(r, n);
        for (uint32_t j = 0; j < n; j++)
            for (uint32_t p = d->cp[j]; p < d->cp[j + 1]; p++) {
                uint32_t i = d->ri[p];
                if (transpose) r[j] -= vals[p] * x[i];
                else r[i] -= vals[p] * x[j];
            }
        double a_norm = transpose ? norm_1 : norm_infv;
        double ratio = norm_inf(r, n) / (a_norm * norm_inf(x, n) * nf * 2.220446049250313e-16);
        if (!(ratio <= REPLAY_RATIO_MAX / PIVOT_TOL)) return 0;
    }
    return 1;
}

/* direct.zig Solver.factor. 0 ok, 1 singular. */
int dsv_factor(dsv_t *d, const double *vals) {
    uint32_t nnz = d->cp[d->n];
    if (nnz != 0 && d->factored) {
        int same = 1;
        for (uint32_t p = 0; p < nnz; p++)
            if (!(d->vcopy[p] == vals[p])) {
                same = 0;
                break;
            }
        if (same) {
            d->bypassed++;
            return 0;
        }
    }
    slu_t *lu = &d->lu;
    lu->fill_cap = REPIVOT_FILL_CAP;
    lu->keep_min = GROWTH_LIMIT;
    int done = 0;
    if (d->factored) {
        if (slu_refactor(lu, vals, GROWTH_LIMIT) == 0) {
            if (replay_holds(d, vals)) done = 1;
            else d->probed_out++;
        }
        if (!done) d->factored = 0;
    }
    if (!done) {
        if (slu_factor(lu, vals, PIVOT_TOL) != 0) {
            d->factored = 0;
            return 1;
        }
        d->full_factors++;
    }
    d->factored = 1;
    memcpy(d->vcopy, vals, sizeof(double) * nnz);
    return 0;
}

/* direct.zig solveNeg: x = -A^-1 rhs. */
void dsv_solve_neg(dsv_t *d, const double *rhs, double *x) {
    for (uint32_t i = 0; i < d->n; i++) x[i] = -rhs[i];
    slu_solve(&d->lu, x, x);
}
