/*
 * TEST INFRASTRUCTURE (oracle), not product code. See espice_oracle.h.
 *
 * The circuit planes and the Newton loop, restated from the reference:
 *   src/analysis/Circuit.zig:570-636 (stamp, ground pin), :845-863 (limits,
 *     junction seeds), src/device/eval.zig:782-922 (stamp order)
 *   src/solver/converger.zig:199-315 (newtonLanes at W = 1), :321-346
 *     (loadExtras, residualGate), :377-384 (plausibleLimit), :454-522
 *     (finalizeStep), :657-694 (run), :794-819 (updateAndNorm)
 *   src/analysis/sweep/lanes.zig:34-80 (independent sweep points)
 *   src/analysis/dc/dc.zig:22-46, :309-385 (sequential .dc sweep)
 *   src/analysis/dc/op.zig:24-140 (cold start, plain rung)
 */
#include "orc_internal.h"
#include "orc_ckt.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ */
/* circuit runtime                                                     */

int ckt_init(ckt_t *k, const orc_circuit *c) {
    memset(k, 0, sizeof(*k));
    k->c = c;
    k->n = c->n;
    uint32_t n = c->n;
    size_t cap = (size_t)n + 64;
    for (uint32_t b = 0; b < c->n_batches; b++) cap += (size_t)c->batches[b].count * ORC_MAX_E * 2;
    k->cp = (uint32_t *)malloc(sizeof(uint32_t) * (n + 1));
    k->ri = (uint32_t *)malloc(sizeof(uint32_t) * cap);
    int64_t nnz = orc_pattern(c, k->cp, k->ri, cap);
    if (nnz < 0) return 1;
    k->nnz = (uint32_t)nnz;
    k->diag = (uint32_t *)malloc(sizeof(uint32_t) * n);
    for (uint32_t i = 0; i < n; i++) k->diag[i] = find_slot(k->cp, k->ri, k->nnz, i, i);
    /* the ground diagonal is slot 0 (column 0 holds only it) */
    k->diag[0] = k->cp[0];
    k->nb = c->n_batches;
    k->bt = (bat_t *)calloc(k->nb ? k->nb : 1, sizeof(bat_t));
    uint32_t lim_off = 0, st_off = 0;
    for (uint32_t b = 0; b < k->nb; b++) {
        const orc_batch *src = &c->batches[b];
        bat_t *bt = &k->bt[b];
        bt->type = src->type;
        bt->count = src->count;
        bt->nt = orc_nodes_per(src->type);
        bt->np = orc_params_per(src->type);
        bt->nodes = src->nodes;
        bt->prm = (double *)malloc(sizeof(double) * ((size_t)src->count * bt->np + 1));
        memcpy(bt->prm, src->params, sizeof(double) * (size_t)src->count * bt->np);
        bt->der = (double *)calloc((size_t)src->count * ORC_NDER + 1, sizeof(double));
        bt->lay = (layout_t *)malloc(sizeof(layout_t) * (src->count ? src->count : 1));
        bt->slot = (uint32_t *)malloc(sizeof(uint32_t) * ((size_t)src->count * ORC_MAX_E + 1));
        bt->qslot = (uint32_t *)malloc(sizeof(uint32_t) * ((size_t)src->count * ORC_MAX_E + 1));
        bt->lim_off = lim_off;
        bt->st_off = st_off;
        for (uint32_t id = 0; id < src->count; id++) {
            const uint32_t *nd = bt->nodes + (size_t)id * bt->nt;
            layout_t *l = &bt->lay[id];
            dev_layout(bt->type, bt->prm + (size_t)id * bt->np, l);
            dev_derive(bt->type, bt->prm + (size_t)id * bt->np, bt->der + (size_t)id * ORC_NDER);
            for (int e = 0; e < l->nj; e++)
                bt->slot[(size_t)id * ORC_MAX_E + e] = find_slot(k->cp, k->ri, k->nnz, nd[l->jac[e].ru], nd[l->jac[e].cu]);
            for (int e = 0; e < l->nq; e++)
                bt->qslot[(size_t)id * ORC_MAX_E + e] = find_slot(k->cp, k->ri, k->nnz, nd[l->qjac[e].ru], nd[l->qjac[e].cu]);
            lim_off += (uint32_t)l->nlim;
            st_off += (uint32_t)dev_nstate(bt->type);
        }
    }
    k->nlim = lim_off;
    k->nst = st_off;
    k->lim = (double *)calloc(lim_off + 1, sizeof(double));
    k->lim_new = (double *)calloc(lim_off + 1, sizeof(double));
    k->st = (double *)calloc(2 * (size_t)st_off + 2, sizeof(double));
    k->g = (double *)calloc(k->nnz + 1, sizeof(double));
    k->cv = (double *)calloc(k->nnz + 1, sizeof(double));
    k->rhs = (double *)calloc(n + 1, sizeof(double));
    k->q = (double *)calloc(n + 1, sizeof(double));
    k->dx = (double *)calloc(n + 1, sizeof(double));
    k->x_old = (double *)calloc(n + 1, sizeof(double));
    k->av = (double *)calloc(k->nnz + 1, sizeof(double));
    k->sim.kind = 0;
    k->sim.src_scale = 1.0;
    k->sim.gmin = -1.0;
    k->sim.iteration = 1;
    dsv_init(&k->dsv, n, k->cp, k->ri);
    return 0;
}

void ckt_free(ckt_t *k) {
    for (uint32_t b = 0; b < k->nb; b++) {
        free(k->bt[b].prm);
        free(k->bt[b].der);
        free(k->bt[b].lay);
        free(k->bt[b].slot);
        free(k->bt[b].qslot);
    }
    free(k->bt);
    free(k->cp); free(k->ri); free(k->diag); free(k->lim); free(k->lim_new); free(k->st);
    free(k->g); free(k->cv); free(k->rhs); free(k->q); free(k->dx); free(k->x_old); free(k->av);
    free(k->gst);
    dsv_free(&k->dsv);
    memset(k, 0, sizeof(*k));
}

/* Installs one swept value and re-derives the instance (Circuit.recompute). */
void ckt_set(ckt_t *k, orc_slot s, double v) {
    bat_t *bt = &k->bt[s.batch];
    bt->prm[(size_t)s.inst * bt->np + s.param] = v;
    dev_derive(bt->type, bt->prm + (size_t)s.inst * bt->np, bt->der + (size_t)s.inst * ORC_NDER);
}

/* Circuit.stamp (.full): clear the planes, every batch in order, then the
 * ground pin g[diag0] += 1, rhs[0] += x[0] (Circuit.zig:570-573). */
void ckt_assemble(ckt_t *k, const double *x) {
    memset(k->g, 0, sizeof(double) * (k->nnz + 1));
    memset(k->cv, 0, sizeof(double) * (k->nnz + 1));
    memset(k->rhs, 0, sizeof(double) * (k->n + 1));
    memset(k->q, 0, sizeof(double) * (k->n + 1));
    devout_t o;
    for (uint32_t b = 0; b < k->nb; b++) {
        bat_t *bt = &k->bt[b];
        uint32_t lo = bt->lim_off;
        for (uint32_t id = 0; id < bt->count; id++) {
            const uint32_t *nd = bt->nodes + (size_t)id * bt->nt;
            const layout_t *l = &bt->lay[id];
            const double *lim = (l->nlim && k->lim_active) ? k->lim + lo : NULL;
            const double *st = dev_nstate(bt->type) ? k->st + bt->st_off + (size_t)id * dev_nstate(bt->type) : NULL;
            dev_eval(bt->type, nd, bt->prm + (size_t)id * bt->np, bt->der + (size_t)id * ORC_NDER, x, lim, st, &k->sim, &o);
            const uint32_t *sl = bt->slot + (size_t)id * ORC_MAX_E;
            int e = 0;
            for (int ru = 0; ru < l->nu; ru++) {
                if (l->res_row[ru]) {
                    uint32_t row = nd[ru];
                    k->rhs[row == 0 ? k->n : row] += o.f[ru];
                }
                for (; e < l->nj && l->jac[e].ru == ru; e++) k->g[sl[e]] += o.J[ru][l->jac[e].cu];
            }
            const uint32_t *qs = bt->qslot + (size_t)id * ORC_MAX_E;
            e = 0;
            for (int ru = 0; ru < l->nu; ru++) {
                if (l->q_row[ru]) {
                    uint32_t row = nd[ru];
                    k->q[row == 0 ? k->n : row] += o.q[ru];
                }
                for (; e < l->nq && l->qjac[e].ru == ru; e++) k->cv[qs[e]] += o.C[ru][l->qjac[e].cu];
            }
            lo += (uint32_t)l->nlim;
        }
    }
    k->g[k->diag[0]] += 1.0;
    k->rhs[0] += x[0];
}

/* Circuit.applyLimits: every limited instance against its image (or x_old
 * before the first pass); returns 1 when any device limited. */
int ckt_apply_limits(ckt_t *k, const double *x, const double *x_old) {
    int any = 0;
    for (uint32_t b = 0; b < k->nb; b++) {
        bat_t *bt = &k->bt[b];
        uint32_t lo = bt->lim_off;
        for (uint32_t id = 0; id < bt->count; id++) {
            const layout_t *l = &bt->lay[id];
            if (l->nlim) {
                const uint32_t *nd = bt->nodes + (size_t)id * bt->nt;
                int lm = dev_limit(bt->type, nd, bt->prm + (size_t)id * bt->np,
                                   bt->der + (size_t)id * ORC_NDER, x, x_old,
                                   k->lim_active ? k->lim + lo : NULL, k->lim_new + lo);
                any |= lm;
            }
            lo += (uint32_t)l->nlim;
        }
    }
    memcpy(k->lim, k->lim_new, sizeof(double) * k->nlim);
    if (k->nlim) k->lim_active = 1;
    return any;
}

void ckt_seed(ckt_t *k, double *x) {
    int any = 0;
    for (uint32_t b = 0; b < k->nb; b++) {
        bat_t *bt = &k->bt[b];
        uint32_t lo = bt->lim_off;
        for (uint32_t id = 0; id < bt->count; id++) {
            const layout_t *l = &bt->lay[id];
            if (l->nlim) {
                const uint32_t *nd = bt->nodes + (size_t)id * bt->nt;
                any |= dev_seed(bt->type, nd, bt->prm + (size_t)id * bt->np,
                                bt->der + (size_t)id * ORC_NDER, x, k->lim + lo);
            }
            lo += (uint32_t)l->nlim;
        }
    }
    if (any) k->lim_active = 1;
}

/* op.zig coldStart: zero x, then the junction seeds. */
void ckt_cold_start(ckt_t *k, double *x) {
    memset(x, 0, sizeof(double) * k->n);
    ckt_seed(k, x);
}

/* ------------------------------------------------------------------ */
/* converger.zig                                                       */

static double plausible_limit(const ckt_t *k, const double *x, const double *f, const double *v) {
    double g = 1;
    for (uint32_t i = 0; i < k->n; i++) g = fmax(g, fabs(v[k->diag[i]]));
    double scale = fmin(fmax(norm_inf(x, k->n), norm_inf(f, k->n) * g), 1e18);
    return !(1e3 * scale > X_PLAUSIBLE) ? X_PLAUSIBLE : 1e3 * scale;
}

double update_and_norm(uint32_t n, double *x, const double *dx, double *x_old, const uint8_t *cur,
                       double reltol, double abstol, double vntol) {
    int64_t worst = 0;
    for (uint32_t i = 0; i < n; i++) {
        double xo = x[i];
        double d = dx[i];
        double xn = xo + d;
        x_old[i] = xo;
        x[i] = xn;
        double tol = reltol * fmax(fabs(xn), fabs(xo)) + (cur[i] ? abstol : vntol);
        int finite = fabs(xn) < INFINITY && fabs(d) < INFINITY;
        double q = fabs(d) / tol;
        double score = !finite ? INFINITY : (q == q ? q : 0);
        int64_t b = (int64_t)bits_of(score);
        if (b > worst) worst = b;
    }
    return of_bits((uint64_t)worst);
}

static double residual_gate(const orc_newton_opts *o, double diag, double xi) {
    double scale = fabs(diag);
    double s = scale == 0 ? 1.0 : scale;
    return fmax(o->residual_tol, 10.0 * s * (o->reltol * fabs(xi) + o->vntol));
}

/* converger.newton (newtonLanes at W = 1) with direct.Solver as the engine.
 * Returns 0 converged, 1 not converged, 2 singular. */
int ckt_newton(ckt_t *k, double *x, const orc_newton_opts *opts, int init_fix, uint32_t *iters) {
    uint32_t n = k->n;
    uint32_t max_iter = opts->max_iter < 100 ? 100 : opts->max_iter;
    if (k->iter_cap && k->iter_cap < max_iter) max_iter = k->iter_cap;
    double limit = X_PLAUSIBLE;
    k->sim.iteration = 1;
    for (uint32_t iter = 0; iter < max_iter; iter++) {
        if (iter != 0) k->sim.iteration++;
        ckt_assemble(k, x);
        double *v = k->g;
        if (k->tran) {
            /* integrator.zig companionAt(accumulate) and Circuit.combineGC */
            for (uint32_t j = 0; j < n; j++) {
                double d = k->ag0 * (k->q[j] - k->q1[j]);
                double base = k->rhs[j] + d;
                k->rhs[j] = k->trap ? base - k->ag1 * k->ip[j] : base;
            }
            for (uint32_t s = 0; s < k->nnz; s++) k->av[s] = k->g[s] + k->ag0 * k->cv[s];
            v = k->av;
        }
        if (opts->gmin > 0) {
            for (uint32_t i = 0; i < n; i++) v[k->diag[i]] += opts->gmin;
            for (uint32_t i = 0; i < n; i++) k->rhs[i] += opts->gmin * x[i];
        }
        if (k->gs > 0) {
            /* converger.loadGmin with gmin_stamps (converger.zig:696-713) */
            for (uint32_t e = 0; e < k->n_gst; e++) v[k->gst[3 * e]] += k->gs;
            for (uint32_t e = 0; e < k->n_gst; e++) k->rhs[k->gst[3 * e + 1]] += k->gs * x[k->gst[3 * e + 2]];
        }
        if (iter == 0) limit = plausible_limit(k, x, k->rhs, v);
        if (dsv_factor(&k->dsv, v) != 0) {
            *iters = iter + 1;
            return 2;
        }
        dsv_solve_neg(&k->dsv, k->rhs, k->dx);
        /* finalizeStep */
        double scaled = update_and_norm(n, x, k->dx, k->x_old, k->c->current_row,
                                        opts->reltol, opts->abstol, opts->vntol);
        int limited = ckt_apply_limits(k, x, k->x_old);
        int ok = !limited;
        if (ok && iter == 0) ok = 0;
        if (ok && scaled >= 1.0) ok = 0;
        if (ok) {
            for (uint32_t i = 0; i < n; i++)
                if (!(fabs(x[i]) <= limit)) {
                    ok = 0;
                    break;
                }
        }
        if (ok) {
            for (uint32_t i = 0; i < n; i++)
                if (!(fabs(k->rhs[i]) <= residual_gate(opts, v[k->diag[i]], x[i]))) {
                    ok = 0;
                    break;
                }
        }
        k->last_scaled = scaled;
        if (k->trace && iter < k->trace_cap) {
            /* the gate inputs of this iterate: the delta score, the largest
               |rhs_i| / residual gate, whether a junction was limited */
            double worst_res = 0;
            for (uint32_t i = 0; i < n; i++) {
                double r = fabs(k->rhs[i]) / residual_gate(opts, v[k->diag[i]], x[i]);
                if (r > worst_res || r != r) worst_res = r;
            }
            k->trace[3 * iter] = scaled;
            k->trace[3 * iter + 1] = worst_res;
            k->trace[3 * iter + 2] = limited;
        }
        if (ok) {
            if (init_fix) {
                init_fix = 0;
            } else {
                memcpy(x, k->x_old, sizeof(double) * n);
                *iters = iter + 1;
                return 0;
            }
        }
    }
    *iters = max_iter;
    return 1;
}

/* The charge states of every instance at raw x, in batch/instance order. */
uint32_t ckt_qtape(ckt_t *k, const double *x, double *out) {
    uint32_t m = 0;
    for (uint32_t b = 0; b < k->nb; b++) {
        bat_t *bt = &k->bt[b];
        for (uint32_t id = 0; id < bt->count; id++) {
            const uint32_t *nd = bt->nodes + (size_t)id * bt->nt;
            double tmp[4];
            int c = dev_qtape(bt->type, nd, bt->prm + (size_t)id * bt->np, bt->der + (size_t)id * ORC_NDER, x, tmp);
            for (int i = 0; i < c; i++) {
                if (out) out[m] = tmp[i];
                m++;
            }
        }
    }
    return m;
}

/* converger.run: newton, then clearLimits. */
int ckt_run(ckt_t *k, double *x, const orc_newton_opts *opts, int init_fix, uint32_t *iters) {
    int rc = ckt_newton(k, x, opts, init_fix, iters);
    k->lim_active = 0;
    return rc;
}

/* ------------------------------------------------------------------ */
/* the operating-point ladder (op.zig solveLadder / afterPlain)        */

#define LADDER_GMIN_START 1e-2   /* Tolerances.gmin_start (numerics.zig:389) */
#define LADDER_GMIN_TARGET 1e-12 /* Tolerances.gmin */
#define LADDER_ITL2 50u          /* Tolerances.itl2 */

/* CountTwins of op.zig gminStamps (:560-575): in column position j, the
 * +-1 entries (ground row skipped) whose transposed entry, row j at
 * original column perm[r], is +-1 too; counting stops at two. */
static uint32_t count_twins(const ckt_t *k, const uint32_t *perm, uint32_t j, uint32_t *twin) {
    uint32_t col = perm[j], count = 0;
    for (uint32_t p = k->cp[col]; p < k->cp[col + 1]; p++) {
        uint32_t r = k->ri[p];
        if (r == 0 || fabs(k->g[p]) != 1.0) continue;
        uint32_t q = find_slot(k->cp, k->ri, k->nnz, j, perm[r]);
        if (q == k->nnz || fabs(k->g[q]) != 1.0) continue;
        count++;
        if (count == 1) *twin = r;
        else break;
    }
    return count;
}

/* op.zig gminStamps (:531-608): ngspice's diagonal-gmin placement. Rows
 * whose unknown is a branch current with nothing on the diagonal (G and C
 * both zero in the current planes) have no diagonal; spMNA_Preorder swaps
 * such a column with the twin of a +-1 pair, lone twins first, then the
 * first column with several. Writes (slot, row, col) triples for rows 1..n-1
 * that end with a diagonal; returns their count. */
uint32_t ckt_gmin_stamps(const ckt_t *k, uint32_t *out) {
    const uint32_t n = k->n, none = 0xffffffffu;
    uint32_t *perm = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
    uint32_t *dcol = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
    for (uint32_t i = 0; i < n; i++) {
        uint32_t d = k->diag[i];
        perm[i] = i;
        dcol[i] = (k->c->current_row[i] && k->g[d] == 0.0 && k->cv[d] == 0.0) ? none : i;
    }
    uint32_t start = 1;
    for (;;) {
        int swapped = 0, again = 0;
        for (uint32_t j = start; j < n; j++) {
            if (dcol[j] != none) continue;
            uint32_t r = 0, t = count_twins(k, perm, j, &r);
            if (t == 1) {
                dcol[j] = perm[r]; dcol[r] = perm[j];
                uint32_t tmp = perm[j]; perm[j] = perm[r]; perm[r] = tmp;
                swapped = 1;
            } else if (t > 1 && !again) {
                again = 1;
                start = j;
            }
        }
        if (!again) break;
        for (uint32_t j = start; !swapped && j < n; j++) {
            if (dcol[j] != none) continue;
            uint32_t r = 0, t = count_twins(k, perm, j, &r);
            if (t > 0) {
                dcol[j] = perm[r]; dcol[r] = perm[j];
                uint32_t tmp = perm[j]; perm[j] = perm[r]; perm[r] = tmp;
                swapped = 1;
            }
        }
        if (!swapped) break;
    }
    uint32_t m = 0;
    for (uint32_t i = 1; i < n; i++) {
        if (dcol[i] == none) continue;
        out[3 * m] = find_slot(k->cp, k->ri, k->nnz, i, dcol[i]);
        out[3 * m + 1] = i;
        out[3 * m + 2] = dcol[i];
        m++;
    }
    free(perm);
    free(dcol);
    return m;
}

/* op.zig newtonRun: one converger.run with the rung's gmin stamps, source
 * factor and Newton cap; a singular Jacobian is a failed solve of zero
 * iterations. Returns 1 converged. */
static int ladder_run(ckt_t *k, double *x, const orc_newton_opts *opts, uint32_t max_iter, double gs,
                      double src, int init_fix, uint32_t *iters) {
    orc_newton_opts o = *opts;
    o.gmin = 0.0;
    o.max_iter = max_iter;
    k->gs = gs;
    k->sim.gmin = gs > 0 ? gs : -1.0;
    k->sim.src_scale = src;
    uint32_t it = 0;
    int rc = ckt_run(k, x, &o, init_fix, &it);
    k->gs = 0.0;
    k->sim.gmin = -1.0;
    k->sim.src_scale = 1.0;
    *iters = rc == 2 ? 0 : it;
    return rc == 0;
}

static uint32_t sat_add16(uint32_t a, uint32_t b) {
    uint32_t s = a + b;
    return s > 65535u ? 65535u : s;
}

/* op.zig solveLadder from a cold start, without holds: rung 1 plain Newton
 * (MODEINITFIX), rung 2 dynamic gmin stepping (cktop.c dynamic_gmin: the
 * descent, the 4th-root back-off toward the last good gmin, the clean solve
 * at the target), rung 3 adaptive source stepping, then the full-source
 * Newton. Rungs 4 (JFNK) and 5 (OPtran) are not restated: a point that
 * needs them reads not converged. `x` holds the cold start. Returns 1
 * converged; *iters the plain run's iterations, or the sum over every run
 * (saturating at 65535) once the ladder is entered; *rung the rung that
 * converged (0 plain, 1 gmin, 2 source; 3 none). */
int ckt_ladder(ckt_t *k, double *x, const orc_newton_opts *opts, uint32_t *iters, uint32_t *rung) {
    const uint32_t n = k->n;
    const uint32_t itl1 = opts->max_iter, itl2 = LADDER_ITL2;
    uint32_t it = 0;
    *rung = 0;
    if (ladder_run(k, x, opts, itl1, 0.0, 1.0, 1, &it)) {
        *iters = it;
        return 1;
    }
    uint32_t total = it;
    double *x_good = (double *)malloc(sizeof(double) * (n ? n : 1));
    if (!k->gst) k->gst = (uint32_t *)malloc(sizeof(uint32_t) * 3 * (n ? n : 1));
    k->n_gst = ckt_gmin_stamps(k, k->gst);

    /* rung 2: dynamic gmin stepping (op.zig:158-227) */
    {
        ckt_cold_start(k, x);
        double factor = 10.0, good = LADDER_GMIN_START, g = good / factor;
        int have_good = 0;
        for (uint32_t solves = 0; solves < 100; solves++) {
            int conv = ladder_run(k, x, opts, itl2, g, 1.0, !have_good, &it);
            total = sat_add16(total, it);
            if (conv) {
                if (g <= LADDER_GMIN_TARGET) {
                    conv = ladder_run(k, x, opts, itl1, 0.0, 1.0, 0, &it);
                    total = sat_add16(total, it);
                    if (conv) {
                        free(x_good);
                        *iters = total;
                        *rung = 1;
                        return 1;
                    }
                    break;
                }
                memcpy(x_good, x, sizeof(double) * n);
                have_good = 1;
                good = g;
                if (it <= itl2 / 4) {
                    double f = factor * sqrt(factor);
                    factor = f < 10.0 ? f : 10.0;
                } else if (it > 3 * itl2 / 4) {
                    double f = sqrt(factor);
                    factor = f > 1.00005 ? f : 1.00005;
                }
                if (g < factor * LADDER_GMIN_TARGET) {
                    factor = g / LADDER_GMIN_TARGET;
                    g = LADDER_GMIN_TARGET;
                } else {
                    g = g / factor;
                }
            } else {
                if (factor < 1.00005) break;
                factor = sqrt(sqrt(factor));
                g = good / factor;
                if (have_good) memcpy(x, x_good, sizeof(double) * n);
                else ckt_cold_start(k, x);
            }
        }
    }

    /* rung 3: source stepping (op.zig:229-279) */
    ckt_cold_start(k, x);
    {
        double lambda = 0.0, lambda_good = -1.0, delta = 0.25;
        for (uint32_t solves = 0; solves < 100; solves++) {
            int conv = ladder_run(k, x, opts, itl2, 0.0, lambda, lambda_good < 0.0, &it);
            total = sat_add16(total, it);
            if (conv) {
                if (lambda >= 1.0) break;
                lambda_good = lambda;
                memcpy(x_good, x, sizeof(double) * n);
                delta *= 1.5;
                lambda = lambda + delta < 1.0 ? lambda + delta : 1.0;
            } else {
                delta *= 0.5;
                if (delta < 1e-4) break;
                if (lambda_good < 0.0) break;
                memcpy(x, x_good, sizeof(double) * n);
                lambda = lambda_good + delta < 1.0 ? lambda_good + delta : 1.0;
            }
        }
    }
    int conv = ladder_run(k, x, opts, itl1, 0.0, 1.0, 0, &it);
    total = sat_add16(total, it);
    free(x_good);
    *iters = total;
    *rung = conv ? 2 : 3;
    return conv;
}

/* ------------------------------------------------------------------ */
/* entry points                                                        */

int orc_dc_points(const orc_circuit *c, const orc_slot *slots, uint32_t n_slots,
                  const double *values, uint32_t n_lanes, const double *warm,
                  const orc_newton_opts *opts, double *x_out, uint32_t *iters,
                  uint8_t *conv) {
    uint32_t n = c->n;
    for (uint32_t l = 0; l < n_lanes; l++) {
        /* Each lane is its own circuit with its own direct.Solver
         * (sweep/lanes.zig runBatch: one RunCtx circuit per lane row). */
        ckt_t k;
        if (ckt_init(&k, c)) return 1;
        for (uint32_t s = 0; s < n_slots; s++) ckt_set(&k, slots[s], values[(size_t)l * n_slots + s]);
        double *x = x_out + (size_t)l * n;
        if (warm) memcpy(x, warm, sizeof(double) * n);
        else ckt_cold_start(&k, x);
        uint32_t it = 0;
        int rc = ckt_run(&k, x, opts, 0, &it);
        conv[l] = rc == 0;
        iters[l] = rc == 2 ? 0 : it;
        ckt_free(&k);
    }
    return 0;
}

/* orc_dc_points with each lane's gate inputs per iterate: trace
 * [n_lanes][cap][3] = (delta score, max |rhs_i| / residual gate, limited),
 * NaN past the lane's last iterate. */
int orc_dc_points_trace(const orc_circuit *c, const orc_slot *slots, uint32_t n_slots,
                        const double *values, uint32_t n_lanes, const double *warm,
                        const orc_newton_opts *opts, double *x_out, uint32_t *iters,
                        uint8_t *conv, double *trace, uint32_t cap) {
    uint32_t n = c->n;
    for (size_t i = 0; i < (size_t)n_lanes * cap * 3; i++) trace[i] = NAN;
    for (uint32_t l = 0; l < n_lanes; l++) {
        ckt_t k;
        if (ckt_init(&k, c)) return 1;
        k.trace = trace + (size_t)l * cap * 3;
        k.trace_cap = cap;
        for (uint32_t s = 0; s < n_slots; s++) ckt_set(&k, slots[s], values[(size_t)l * n_slots + s]);
        double *x = x_out + (size_t)l * n;
        if (warm) memcpy(x, warm, sizeof(double) * n);
        else ckt_cold_start(&k, x);
        uint32_t it = 0;
        int rc = ckt_run(&k, x, opts, 0, &it);
        conv[l] = rc == 0;
        iters[l] = rc == 2 ? 0 : it;
        k.trace = NULL;
        ckt_free(&k);
    }
    return 0;
}

/* Operating-point lanes: every lane's parameters installed, then op.zig's
 * ladder from the cold start (ckt_ladder), each lane with its own solver.
 * iter_cap (0: none) caps every Newton run of the ladder, as the lanes'
 * iter_cap option does. */
int orc_op_points(const orc_circuit *c, const orc_slot *slots, uint32_t n_slots, const double *values,
                  uint32_t n_lanes, const orc_newton_opts *opts, uint32_t iter_cap, double *x_out,
                  uint32_t *iters, uint8_t *conv, uint8_t *rung) {
    uint32_t n = c->n;
    for (uint32_t l = 0; l < n_lanes; l++) {
        ckt_t k;
        if (ckt_init(&k, c)) return 1;
        k.iter_cap = iter_cap;
        for (uint32_t s = 0; s < n_slots; s++) ckt_set(&k, slots[s], values[(size_t)l * n_slots + s]);
        double *x = x_out + (size_t)l * n;
        ckt_cold_start(&k, x);
        uint32_t it = 0, r = 0;
        conv[l] = (uint8_t)ckt_ladder(&k, x, opts, &it, &r);
        iters[l] = it;
        rung[l] = (uint8_t)r;
        ckt_free(&k);
    }
    return 0;
}

/* op.solve without holds: the ladder from the cold start. Returns 0
 * converged, 1 not. */
int orc_op(const orc_circuit *c, const orc_newton_opts *opts, double *x_out, uint32_t *iters) {
    ckt_t k;
    if (ckt_init(&k, c)) return -1;
    ckt_cold_start(&k, x_out);
    uint32_t rung = 0;
    int conv = ckt_ladder(&k, x_out, opts, iters, &rung);
    ckt_free(&k);
    return conv ? 0 : 1;
}

/* One sequential sweep on an initialized circuit (dc.zig Sweep :163-386). */
static void sweep_run(ckt_t *kp, orc_slot slot, const double *values, uint32_t n_pts,
                      const orc_newton_opts *opts, double *x_out, uint32_t *iters, uint8_t *conv) {
    ckt_t k = *kp;
    uint32_t n = k.n;
    double *sol = (double *)calloc(n, sizeof(double));
    double *prev = (double *)calloc(n, sizeof(double));
    int cold = 1;
    for (uint32_t pt = 0; pt < n_pts; pt++) {
        ckt_set(&k, slot, values[pt]);
        /* MODEINITPRED predictor: 2 * last - prev (dc.zig:330-337). */
        for (uint32_t i = 0; i < n; i++) {
            double last = sol[i];
            sol[i] = 2.0 * last - prev[i];
            prev[i] = last;
        }
        int converged = 0;
        uint32_t it_total = 0;
        if (!cold) {
            /* prepareWarm: limit the predictor against the last point. */
            ckt_apply_limits(&k, sol, prev);
            uint32_t it = 0;
            int rc = ckt_run(&k, sol, opts, 0, &it);
            it_total += it;
            converged = rc == 0;
        }
        if (!converged) {
            /* dc.zig endPoint: the cold ladder (op.nodesetLadder, no
             * nodesets) at the deck's itl1 */
            ckt_cold_start(&k, sol);
            orc_newton_opts cold_opts = *opts;
            cold_opts.max_iter = 100;
            uint32_t it = 0, rung = 0;
            converged = ckt_ladder(&k, sol, &cold_opts, &it, &rung);
            it_total += it;
        }
        memcpy(x_out + (size_t)pt * n, sol, sizeof(double) * n);
        iters[pt] = it_total;
        conv[pt] = (uint8_t)converged;
        if (converged) {
            cold = 0;
            if (pt == 0) memcpy(prev, sol, sizeof(double) * n);
        } else {
            cold = 1;
        }
    }
    free(sol);
    free(prev);
    *kp = k;
}

int orc_dc_sweep(const orc_circuit *c, orc_slot slot, const double *values,
                 uint32_t n_pts, const orc_newton_opts *opts, double *x_out,
                 uint32_t *iters, uint8_t *conv) {
    ckt_t k;
    if (ckt_init(&k, c)) return -1;
    sweep_run(&k, slot, values, n_pts, opts, x_out, iters, conv);
    ckt_free(&k);
    return 0;
}

/* One sequential sweep per lane, each lane first setting its own slots
 * (esl_dc_sweep_device's semantics). x_out [lanes][n_pts][n]. */
int orc_dc_sweep_lanes(const orc_circuit *c, const orc_slot *slots, uint32_t n_slots,
                       const double *lane_values, uint32_t n_lanes, orc_slot sweep,
                       const double *values, uint32_t n_pts, const orc_newton_opts *opts,
                       double *x_out, uint32_t *iters, uint8_t *conv) {
    for (uint32_t l = 0; l < n_lanes; l++) {
        ckt_t k;
        if (ckt_init(&k, c)) return -1;
        for (uint32_t s = 0; s < n_slots; s++) ckt_set(&k, slots[s], lane_values[(size_t)l * n_slots + s]);
        const size_t at = (size_t)l * n_pts;
        sweep_run(&k, sweep, values, n_pts, opts, x_out + at * c->n, iters + at, conv + at);
        ckt_free(&k);
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* LU-level entry points for the kernel parity tests                   */

int orc_factor_tape(uint32_t n, const uint32_t *cp, const uint32_t *ri, const double *vals,
                    uint32_t *q, uint32_t *pinv, uint32_t *lp, uint32_t *li, double *lx,
                    uint32_t *up, uint32_t *ui, double *ux, double *udiag, uint8_t *flags,
                    uint32_t *counts, size_t cap) {
    dsv_t d;
    dsv_init(&d, n, cp, ri);
    int rc = dsv_factor(&d, vals);
    slu_t *s = &d.lu;
    if (counts) {
        counts[0] = (uint32_t)s->li.len;
        counts[1] = (uint32_t)s->ui.len;
        counts[2] = (uint32_t)s->void_slots.len;
    }
    if (rc == 0 && s->li.len <= cap && s->ui.len <= cap) {
        if (q) memcpy(q, d.q, sizeof(uint32_t) * n);
        if (pinv) memcpy(pinv, s->pinv, sizeof(uint32_t) * n);
        if (lp) memcpy(lp, s->lp, sizeof(uint32_t) * (n + 1));
        if (up) memcpy(up, s->up, sizeof(uint32_t) * (n + 1));
        if (li) memcpy(li, s->li.a, sizeof(uint32_t) * s->li.len);
        if (ui) memcpy(ui, s->ui.a, sizeof(uint32_t) * s->ui.len);
        if (lx) memcpy(lx, s->lx.a, sizeof(double) * s->lx.len);
        if (ux) memcpy(ux, s->ux.a, sizeof(double) * s->ux.len);
        if (udiag) memcpy(udiag, s->udiag, sizeof(double) * n);
        if (flags)
            for (uint32_t k = 0; k < n; k++) flags[k] = (uint8_t)(s->void_col[k] | (s->scaled[k] << 1));
    }
    dsv_free(&d);
    return rc;
}

/* lane_kernels.zig Bodies.refactor + solveNeg for every lane on the tape a
 * full factor of `lead` made (the host oracle of the device kernel). */
int orc_lane_refactor_solve(uint32_t n, const uint32_t *cp, const uint32_t *ri,
                            const double *lead, uint32_t n_lanes, const double *vals,
                            const double *rhs, double *dx, double *lx_out, double *ux_out,
                            double *udiag_out, uint8_t *bad) {
    dsv_t d;
    dsv_init(&d, n, cp, ri);
    if (dsv_factor(&d, lead) != 0) {
        dsv_free(&d);
        return 1;
    }
    slu_t *s = &d.lu;
    uint32_t nnz = cp[n];
    for (uint32_t l = 0; l < n_lanes; l++) {
        const double *a = vals + (size_t)l * nnz;
        int b = 0;
        for (size_t t = 0; t < s->void_slots.len; t++)
            if (a[s->void_slots.a[t]] != 0) b = 1;
        uint64_t nonfinite = 0;
        double *w = s->w;
        for (uint32_t k = 0; k < n && !b; k++) {
            uint32_t c = s->q[k];
            for (uint32_t p = cp[c]; p < cp[c + 1]; p++) w[s->prow[p]] = a[p];
            for (uint32_t p = s->up[k]; p < s->up[k + 1]; p++) {
                uint32_t i = s->ui.a[p];
                double uki = w[i];
                w[i] = 0;
                s->ux.a[p] = uki;
                nonfinite |= bits_of(uki - uki);
                for (uint32_t t = s->lp[i]; t < s->lp[i + 1]; t++) w[s->li.a[t]] -= s->lx.a[t] * uki;
            }
            if (s->void_col[k]) {
                s->udiag[k] = 1;
                for (uint32_t p = s->lp[k]; p < s->lp[k + 1]; p++) {
                    s->lx.a[p] = 0;
                    w[s->li.a[p]] = 0;
                }
                w[k] = 0;
                for (uint32_t p = s->up[k]; p < s->up[k + 1]; p++) {
                    uint32_t i = s->ui.a[p];
                    for (uint32_t t = s->lp[i]; t < s->lp[i + 1]; t++) w[s->li.a[t]] = 0;
                }
                continue;
            }
            double dd = w[k];
            w[k] = 0;
            int dead = dd == 0 || !(fabs(dd) < INFINITY);
            if (dead) {
                b = 1;
                dd = 1;
            }
            s->udiag[k] = dd;
            if (GROWTH_LIMIT > 0 && !s->scaled[k]) {
                uint64_t cbits = bits_of(fabs(dd));
                for (uint32_t p = s->lp[k]; p < s->lp[k + 1]; p++) {
                    uint32_t r = s->li.a[p];
                    double v = w[r];
                    w[r] = 0;
                    uint64_t bb = bits_of(fabs(v));
                    if ((int64_t)bb > (int64_t)cbits) cbits = bb;
                    s->lx.a[p] = v / dd;
                }
                if (!(fabs(dd) >= GROWTH_LIMIT * of_bits(cbits))) b = 1;
            } else {
                for (uint32_t p = s->lp[k]; p < s->lp[k + 1]; p++) {
                    uint32_t r = s->li.a[p];
                    double lv = w[r] / dd;
                    nonfinite |= bits_of(lv - lv);
                    s->lx.a[p] = lv;
                    w[r] = 0;
                }
            }
        }
        for (uint32_t i = 0; i < n; i++) w[i] = 0;
        if (nonfinite) b = 1;
        if (!b) {
            uint64_t worst = 0;
            for (uint32_t k = 0; k < n; k++) {
                if (s->scaled[k]) continue;
                for (uint32_t p = s->lp[k]; p < s->lp[k + 1]; p++) {
                    uint64_t bb = bits_of(fabs(s->lx.a[p]));
                    if (bb > worst) worst = bb;
                }
            }
            if (!(of_bits(worst) <= 1 / PIVOT_TOL)) b = 1;
        }
        bad[l] = (uint8_t)b;
        if (lx_out) memcpy(lx_out + (size_t)l * s->lx.len, s->lx.a, sizeof(double) * s->lx.len);
        if (ux_out) memcpy(ux_out + (size_t)l * s->ux.len, s->ux.a, sizeof(double) * s->ux.len);
        if (udiag_out) memcpy(udiag_out + (size_t)l * n, s->udiag, sizeof(double) * n);
        if (dx) {
            double *o = dx + (size_t)l * n;
            const double *r = rhs + (size_t)l * n;
            for (uint32_t i = 0; i < n; i++) o[i] = -r[i];
            slu_solve(s, o, o);
        }
    }
    dsv_free(&d);
    return 0;
}

int orc_solver_rounds(uint32_t n, const uint32_t *cp, const uint32_t *ri, uint32_t rounds,
                      uint32_t n_lanes, const double *vals, const double *rhs, double *dx,
                      uint8_t *status) {
    uint32_t nnz = cp[n];
    dsv_t *d = (dsv_t *)malloc(sizeof(dsv_t) * (n_lanes ? n_lanes : 1));
    for (uint32_t l = 0; l < n_lanes; l++) dsv_init(&d[l], n, cp, ri);
    for (uint32_t r = 0; r < rounds; r++)
        for (uint32_t l = 0; l < n_lanes; l++) {
            size_t at = (size_t)r * n_lanes + l;
            int rc = dsv_factor(&d[l], vals + at * nnz);
            status[at] = (uint8_t)rc;
            if (rc == 0) dsv_solve_neg(&d[l], rhs + at * n, dx + at * n);
        }
    for (uint32_t l = 0; l < n_lanes; l++) dsv_free(&d[l]);
    free(d);
    return 0;
}
