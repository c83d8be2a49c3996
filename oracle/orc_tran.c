/*
 * TEST INFRASTRUCTURE (oracle), not product code. See espice_oracle.h.
 *
 * Transient, restated from the reference's step control:
 *   src/analysis/tran/tran.zig:672-689   first step (dctran.c:134, :578-586)
 *   src/analysis/tran/tran.zig:728-806   Sim.begin: predictor, limits, Newton
 *                                        options (itl4, no residual gate)
 *   src/analysis/tran/tran.zig:808-1064  Sim.end: Newton reject (dt/8, order
 *                                        1), LTE reject, growth cap, order
 *                                        promotion, history advance,
 *                                        breakpoint landing and clamping
 *   src/analysis/tran/integrator.zig:40-53 coeffs, :166-212 companionAt,
 *                                        :348-424 stepBound / minDel (CKTterr)
 *   models/vsource.va:133-200            PULSE corners as periodic timers,
 *                                        PWL corners as one-shot timers
 * Left out (no device on this path uses them): uic, VPI callbacks, state
 * flips and reject_at, bound_step, stateful-charge rebase, delay-line
 * echoes, gear orders above 2 and tangents. Measures (orc_meas.c) are fed
 * every recorded row, with the early stop of tran.zig:1057-1064. The
 * operating point is the plain Newton rung from a cold start.
 */
#include "orc_internal.h"
#include "orc_ckt.h"
#include "orc_meas.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* integrator.lteCoeff: trapCoeff[1], gearCoeff[0] */
#define LTE_BE 0.5
#define LTE_TRAP 0.08333333333

typedef struct {
    double start, per; /* per 0: a one-shot timer */
} timer_t_;

/* The corner timers of the circuit's sources (vsource.va / isource.va):
 * the 4 periodic PULSE corners of each PULSE source (:133-136), and for a
 * PWL source one one-shot timer per table time plus TD, and TD itself when
 * the table leaves slots unused (their times read 0). Timers at or before
 * the first step never act (breakpoints are sought after t + min_break). */
static uint32_t source_timers(const ckt_t *k, timer_t_ *out, uint32_t cap) {
    uint32_t m = 0;
    for (uint32_t b = 0; b < k->nb; b++) {
        const bat_t *bt = &k->bt[b];
        if (bt->type != ORC_V && bt->type != ORC_I) continue;
        for (uint32_t id = 0; id < bt->count; id++) {
            const double *p = bt->prm + (size_t)id * bt->np;
            if (p[1] == 4.0) {
                const int len = (int)p[2];
                for (int j = 0; j < len && m < cap; j++) {
                    out[m].start = p[ORC_SRC_PWL_T + j] + p[4];
                    out[m].per = 0.0;
                    m++;
                }
                if (len < ORC_PWL_MAX && m < cap) {
                    out[m].start = 0.0 + p[4];
                    out[m].per = 0.0;
                    m++;
                }
                continue;
            }
            if (p[1] != 1.0) continue;
            double tr = p[5] > 1.0e-12 ? p[5] : 1.0e-12;
            double tf = p[6] > 1.0e-12 ? p[6] : 1.0e-12;
            double pw = (p[7] > 0.0 ? p[7] : 0.0) + (-p[7] > 0.0 ? -p[7] : 0.0) * 1.0e30;
            double per = p[8];
            double per_min = tr + pw + tf + 1.0e-12;
            if (per < per_min) per = per_min;
            double td = p[4];
            double s[4] = {td, td + tr, td + tr + pw, td + tr + pw + tf};
            for (int i = 0; i < 4 && m < cap; i++) {
                out[m].start = s[i];
                out[m].per = per;
                m++;
            }
        }
    }
    return m;
}

/* The first timer event at or after `after` (tran.zig nextBp). */
static int next_bp(const timer_t_ *tm, uint32_t nt, double after, double *bp) {
    double best = INFINITY;
    for (uint32_t i = 0; i < nt; i++) {
        double t = tm[i].start;
        if (t < after) {
            if (tm[i].per == 0.0) continue;
            double kk = ceil((after - tm[i].start) / tm[i].per);
            t = tm[i].start + kk * tm[i].per;
            if (t < after) t += tm[i].per;
        }
        if (t < best) best = t;
    }
    if (best == INFINITY) return 0;
    *bp = best;
    return 1;
}

static int almost_equal_ulps(double a, double b, int64_t ulps) {
    if (a == b) return 1;
    if ((a < 0) != (b < 0)) return 0;
    int64_t ia = (int64_t)bits_of(a), ib = (int64_t)bits_of(b);
    int64_t d = ia - ib;
    return (d < 0 ? -d : d) <= ulps;
}

/* tran.zig atStop */
static int at_stop(double t, double t_stop) { return almost_equal_ulps(t, t_stop, 100); }

/* integrator.minDel at w = 1 over the charge states, then the order-2 root:
 * CKTterr's bound for `method` (1 BE, 2 trap) after a step integrated with
 * `cur` (1 BE, 2 trap). NaN when a read entry is NaN or inf. */
static double step_bound(int method, int cur, uint32_t m, double *const q[4], const double *ip,
                         double ag0, double ag1, double dt, double dt1, double dt2, const orc_tran_opts *o) {
    const double sum01 = dt + dt1, sum12 = dt1 + dt2, sum012 = dt + (dt1 + dt2);
    const double coeff = method == 1 ? LTE_BE : LTE_TRAP;
    double vmin = INFINITY, poison = 0.0;
    for (uint32_t j = 0; j < m; j++) {
        const double qc = q[0][j], qp = q[1][j], qp2 = q[2][j], ipj = ip[j];
        double i_new = cur == 2 ? ag0 * (qc - qp) - ag1 * ipj : ag0 * (qc - qp);
        double volttol = o->abstol + o->reltol * fmax(fabs(i_new), fabs(ipj));
        double chargetol = o->reltol * fmax(fmax(fabs(qc), fabs(qp)), o->chgtol) / dt;
        double tol = fmax(volttol, chargetol);
        poison += (qc - qc) + (qp - qp) + (qp2 - qp2) + (ipj - ipj);
        double f12 = (qp - qp2) / dt1;
        double dd = ((qc - qp) / dt - f12) / sum01;
        if (method != 1) {
            const double qp3 = q[3][j];
            poison += qp3 - qp3;
            double f123 = (f12 - (qp2 - qp3) / dt2) / sum12;
            dd = (dd - f123) / sum012;
        }
        double del = o->trtol * tol / fmax(o->abstol, coeff * fabs(dd));
        poison += del == del ? 0.0 : del;
        vmin = fmin(vmin, del);
    }
    if (isnan(poison)) return NAN;
    return method == 1 ? vmin : sqrt(vmin);
}

/* integrator.advanceCurrent: i <- ag0*(q0 - q1) (- ag1*i for trap). */
static void advance_current(int trap, double *i, const double *q0, const double *q1, uint32_t m, double ag0,
                            double ag1) {
    for (uint32_t j = 0; j < m; j++) {
        double d = ag0 * (q0[j] - q1[j]);
        i[j] = trap ? d - ag1 * i[j] : d;
    }
}

static void rotate4(double *r[4]) {
    double *t = r[3];
    r[3] = r[2];
    r[2] = r[1];
    r[1] = r[0];
    r[0] = t;
}

typedef struct {
    uint32_t n_probes, max_pts, n_pts;
    const uint32_t *probes;
    double *out_t, *out_v;
    const orc_measure *meas;
    uint32_t n_meas;
    int early_stop;
    orc_meas_state *ms;
} rec_t;

/* Records the row (t, x) and feeds it to the measures; returns the cards
 * still open. */
static int record(rec_t *r, double t, const double *x) {
    int open = r->n_meas ? meas_feed(r->ms, r->meas, r->n_meas, t, x) : 1;
    if (!r->out_t || r->n_pts >= r->max_pts) return open;
    r->out_t[r->n_pts] = t;
    for (uint32_t p = 0; p < r->n_probes; p++) r->out_v[(size_t)r->n_pts * r->n_probes + p] = x[r->probes[p]];
    r->n_pts++;
    return open;
}

/* One lane: operating point, then the step loop. */
static void tran_lane(ckt_t *k, const orc_tran_opts *o, rec_t *rec, uint32_t *st, double *x_final) {
    const uint32_t n = k->n;
    double *cur = (double *)calloc(n, sizeof(double));
    double *prev = (double *)calloc(n, sizeof(double));
    double *trial = (double *)calloc(n, sizeof(double));
    memset(st, 0, sizeof(uint32_t) * ORC_TS_N);

    /* operating point, cold start: the transient's own operating point
       evaluates the source waves at t = 0 (vsource.va:214-219, the ic phase
       where analysis("tran") is true), so a PULSE source with an explicit DC
       value biases at its first level, not at DC */
    orc_newton_opts op = {o->reltol, o->abstol, o->vntol, 1e-9, 0.0, 100};
    k->sim.kind = 2;
    k->sim.t = 0.0;
    k->tran = 0;
    ckt_cold_start(k, cur);
    uint32_t it = 0, rung = 0;
    /* op.solve with tran_op: the ladder from the cold start */
    if (!ckt_ladder(k, cur, &op, &it, &rung)) {
        st[ORC_TS_STATUS] = 2;
        st[ORC_TS_OP_ITERS] = it;
        memcpy(x_final, cur, sizeof(double) * n);
        free(cur); free(prev); free(trial);
        return;
    }
    st[ORC_TS_OP_ITERS] = it;
    memcpy(prev, cur, sizeof(double) * n);

    /* charge histories: rows (companion) and states (LTE), flat at q(x_op) */
    k->sim.kind = 1;
    k->sim.t = 0.0;
    ckt_assemble(k, cur);
    int has_charge = 0;
    for (uint32_t j = 0; j <= n; j++) has_charge |= k->q[j] != 0.0;
    for (uint32_t s = 0; s <= k->nnz; s++) has_charge |= k->cv[s] != 0.0;
    uint32_t m = ckt_qtape(k, cur, NULL);
    double *qh[4], *qt[4];
    for (int i = 0; i < 4; i++) {
        qh[i] = (double *)calloc(n + 1, sizeof(double));
        qt[i] = (double *)calloc(m + 1, sizeof(double));
    }
    double *ip_row = (double *)calloc(n + 1, sizeof(double));
    double *ip_st = (double *)calloc(m + 1, sizeof(double));
    for (int i = 1; i < 4; i++) {
        memcpy(qh[i], k->q, sizeof(double) * n);
        ckt_qtape(k, cur, qt[i]);
    }

    /* src/frontend/analyses.zig:534: DELMAX, else min(tstep, span / 50) */
    const double dt_max = o->tmax > 0 ? o->tmax : fmin(o->tstep, o->tstop / 50.0);
    const double delmin = 1e-11 * dt_max;
    const double min_break = 10.0 * delmin;
    uint32_t cap_tm = 0;
    for (uint32_t b = 0; b < k->nb; b++)
        if (k->bt[b].type == ORC_V || k->bt[b].type == ORC_I) cap_tm += k->bt[b].count * (ORC_PWL_MAX + 4);
    timer_t_ *tm = (timer_t_ *)calloc(cap_tm + 1, sizeof(timer_t_));
    uint32_t nt = source_timers(k, tm, cap_tm);
    double dt = fmin(fmin(o->tstep, o->tstop / 100.0) / 10.0, dt_max);
    double bp0;
    if (next_bp(tm, nt, min_break, &bp0)) dt = fmin(dt, 0.1 * bp0);
    dt /= 10.0;
    double dt_old[6] = {dt_max, dt_max, dt_max, dt_max, dt_max, dt_max};
    double t = 0.0;
    int order = 1;
    uint32_t steps = 0;
    int have_bp = 0, bp_clamped = 0;
    double bp_next = 0.0, bp_save_dt = o->tstop / 50.0;
    record(rec, 0.0, cur);

    orc_newton_opts nr = {o->reltol, o->abstol, o->vntol, INFINITY, 0.0, 100};
    for (;;) {
        if (!(t < o->tstop && !at_stop(t, o->tstop) && steps < o->max_steps)) break;
        const double t_dev = t + dt;
        k->sim.kind = 1;
        k->sim.t = t_dev;
        k->sim.initial_tran = steps == 0;
        const int trap = order == 2;
        /* integrator.coeffs: BE 1/dt; trap at xmu = 0.5: (1/dt)/0.5, ag1 1 */
        const double ag0 = trap ? 1.0 / dt / (1.0 - 0.5) : 1.0 / dt;
        const double ag1 = trap ? 0.5 / (1.0 - 0.5) : 1.0;
        /* attempt: predictor, then limits against the accepted point */
        const double xfact = dt / dt_old[0];
        for (uint32_t i = 0; i < n; i++) trial[i] = cur[i] + xfact * (cur[i] - prev[i]);
        k->lim_active = 0;
        ckt_apply_limits(k, trial, cur);
        k->tran = 1;
        k->trap = trap;
        k->ag0 = ag0;
        k->ag1 = ag1;
        k->q1 = qh[1];
        k->ip = ip_row;
        uint32_t iters = 0;
        int rc = ckt_run(k, trial, &nr, 0, &iters);
        k->tran = 0;
        st[ORC_TS_ATTEMPTS]++;
        st[ORC_TS_NR_ITERS] += iters;
        if (rc != 0) {
            st[ORC_TS_REJ_NEWTON]++;
            order = 1;
            dt = dt / 8.0;
            if (dt < o->dt_min) {
                st[ORC_TS_STATUS] = 1;
                break;
            }
            continue;
        }
        double dt_next = steps == 0 ? dt : fmin(dt * 2.0, dt_max);
        /* charges re-read at the solution */
        if (has_charge) {
            ckt_assemble(k, trial);
            memcpy(qh[0], k->q, sizeof(double) * n);
            ckt_qtape(k, trial, qt[0]);
        }
        const double dt1 = dt_old[0], dt2 = dt_old[1];
        if (has_charge && steps > 0) {
            double del = step_bound(trap ? 2 : 1, trap ? 2 : 1, m, qt, ip_st, ag0, ag1, dt, dt1, dt2, o);
            if (!(del >= 0.9 * dt)) {
                st[ORC_TS_REJ_LTE]++;
                if (isnan(del)) {
                    order = 1;
                    dt = dt / 8.0;
                } else {
                    dt = del;
                }
                if (dt < o->dt_min) {
                    st[ORC_TS_STATUS] = 1;
                    break;
                }
                continue;
            }
            dt_next = fmin(fmin(fmax(del, o->dt_min), 2.0 * dt), dt_max);
        }
        if (has_charge) {
            if (steps > 0 && order == 1) {
                double trial_del = step_bound(2, 1, m, qt, ip_st, ag0, ag1, dt, dt1, dt2, o);
                if (!isnan(trial_del)) {
                    double nd2 = fmin(2.0 * dt, trial_del);
                    if (nd2 > 1.05 * dt) order = 2;
                    dt_next = fmin(fmax(nd2, o->dt_min), dt_max);
                }
            }
            advance_current(trap, ip_row, qh[0], qh[1], n, ag0, ag1);
            advance_current(trap, ip_st, qt[0], qt[1], m, ag0, ag1);
            rotate4(qh);
            rotate4(qt);
        }
        for (int i = 5; i > 0; i--) dt_old[i] = dt_old[i - 1];
        dt_old[0] = dt;
        double *stale = prev;
        prev = cur;
        cur = trial;
        trial = stale;
        t = t + dt;
        steps++;
        st[ORC_TS_ACCEPTED]++;
        const double t_new = t;
        if (have_bp) {
            int landed = bp_clamped ? fabs(t_new - bp_next) <= min_break
                                    : (bp_next - t_new <= delmin || almost_equal_ulps(t_new, bp_next, 100));
            if (landed) {
                st[ORC_TS_BP_LANDINGS]++;
                order = 1;
                double shrink = bp_save_dt, nb;
                if (next_bp(tm, nt, t_new + min_break, &nb)) shrink = fmin(shrink, nb - t_new);
                dt_next = fmin(dt_next, 0.1 * shrink);
            }
            have_bp = 0;
        }
        const int open = record(rec, t_new, cur);
        if (rec->early_stop && rec->n_meas && open == 0) {
            st[ORC_TS_STATUS] = ORC_TRAN_RESOLVED;
            break;
        }
        have_bp = next_bp(tm, nt, t_new + min_break, &bp_next);
        bp_clamped = 0;
        if (have_bp) {
            double dt_to_bp = bp_next - t_new;
            if (dt_to_bp < dt_next) {
                bp_save_dt = dt_next;
                dt_next = dt_to_bp;
                bp_clamped = 1;
            }
        }
        dt = dt_next;
        if (t_new + dt > o->tstop) dt = o->tstop - t_new;
    }
    if (st[ORC_TS_STATUS] == 0 && steps >= o->max_steps && !(t >= o->tstop || at_stop(t, o->tstop)))
        st[ORC_TS_STATUS] = 3;
    memcpy(x_final, cur, sizeof(double) * n);
    for (int i = 0; i < 4; i++) {
        free(qh[i]);
        free(qt[i]);
    }
    free(ip_row); free(ip_st); free(cur); free(prev); free(trial);
    free(tm);
}

/* MOS1 with TOX given carries the bias-dependent Meyer halves and their
 * $prev averaging (mos1.va:351-441), which this restatement leaves out: a
 * transient of such a circuit is refused (DC runs, TOX affecting only the
 * KP default there). */
static int orc_tran_supported(const orc_circuit *c) {
    for (uint32_t b = 0; b < c->n_batches; b++) {
        const orc_batch *bt = &c->batches[b];
        if (bt->type != ORC_M) continue;
        for (uint32_t id = 0; id < bt->count; id++)
            if (!orc_mos1_supported(bt->params + (size_t)id * ORC_M_NP)) return 0;
    }
    return 1;
}

int orc_tran(const orc_circuit *c, const orc_slot *slots, uint32_t n_slots,
             const double *values, uint32_t n_lanes, const orc_tran_opts *topts,
             const uint32_t *probe_nodes, uint32_t n_probes, uint32_t max_pts,
             double *out_t, double *out_v, uint32_t *n_pts_out, uint32_t *stats,
             double *x_final) {
    ckt_t k;
    if (!orc_tran_supported(c)) return -2;
    if (ckt_init(&k, c) != 0) return -1;
    for (uint32_t l = 0; l < n_lanes; l++) {
        for (uint32_t s = 0; s < n_slots; s++) ckt_set(&k, slots[s], values[(size_t)l * n_slots + s]);
        rec_t r = {n_probes, max_pts, 0, probe_nodes,
                   out_t ? out_t + (size_t)l * max_pts : NULL,
                   out_v ? out_v + (size_t)l * max_pts * n_probes : NULL, NULL, 0, 0, NULL};
        k.lim_active = 0;
        tran_lane(&k, topts, &r, stats + (size_t)l * ORC_TS_N, x_final + (size_t)l * k.n);
        if (n_pts_out) n_pts_out[l] = r.n_pts;
    }
    ckt_free(&k);
    return 0;
}

int orc_tran_meas(const orc_circuit *c, const orc_slot *slots, uint32_t n_slots,
                  const double *values, uint32_t n_lanes, const orc_tran_opts *topts,
                  const orc_measure *meas, uint32_t n_meas, int early_stop, double *meas_out,
                  uint32_t *stats, double *x_final) {
    ckt_t k;
    if (!orc_tran_supported(c)) return -2;
    if (ckt_init(&k, c) != 0) return -1;
    orc_meas_state *ms = (orc_meas_state *)calloc(n_meas ? n_meas : 1, sizeof(orc_meas_state));
    for (uint32_t l = 0; l < n_lanes; l++) {
        for (uint32_t s = 0; s < n_slots; s++) ckt_set(&k, slots[s], values[(size_t)l * n_slots + s]);
        meas_init(ms, meas, n_meas);
        rec_t r = {0, 0, 0, NULL, NULL, NULL, meas, n_meas, early_stop, ms};
        k.lim_active = 0;
        tran_lane(&k, topts, &r, stats + (size_t)l * ORC_TS_N, x_final + (size_t)l * k.n);
        meas_results(ms, meas, n_meas, meas_out + (size_t)l * n_meas);
    }
    free(ms);
    ckt_free(&k);
    return 0;
}
