/*
 * TEST INFRASTRUCTURE (oracle), not product code. See espice_oracle.h.
 *
 * Streaming transient measures, restated from the reference's .meas
 * evaluation (src/output/measure.zig, a port of ngspice com_measure2.c):
 *   measure.zig:1269-1365  Cross: RISE/FALL/CROSS event counting from the
 *                          second sample, the level crossing interpolated
 *                          on the last segment, LAST counts, TD, FROM/TO
 *   measure.zig:1379-1398  At: FIND .. AT=, the first segment holding AT
 *   measure.zig:1401-1449  Extremum: MIN/MAX (the last sample reaching
 *                          the extreme), AVG (trapezoids over the samples'
 *                          span), inside FROM..TO, without interpolated ends
 *   measure.zig:575-650    TRIG/TARG (targ - trig), WHEN, FIND AT, MIN,
 *                          MAX, AVG, PP (max - min)
 *   tran.zig:1057-1064     feeding accepted rows and the early stop once
 *                          every card has resolved
 * Only WHEN, TRIG/TARG (each clause its own TD), FIND AT, MIN, MAX, AVG and
 * PP are restated, with VAL levels (no vector levels), as the device
 * streams them.
 */
#include "orc_meas.h"

#include <math.h>
#include <string.h>

void meas_init(orc_meas_state *s, const orc_measure *m, uint32_t n_meas) {
    memset(s, 0, sizeof(*s) * n_meas);
    for (uint32_t c = 0; c < n_meas; c++) {
        for (int k = 0; k < 2; k++) {
            const orc_meas_clause *cl = k ? &m[c].b : &m[c].a;
            orc_cross *x = &s[c].x[k];
            x->td = cl->td;
            x->want_rise = cl->rise;
            x->want_fall = cl->fall;
            x->want_cross = cl->cross;
            x->last = NAN;
            x->hit = NAN;
            if (m[c].kind >= ORC_MEAS_MIN) {
                x->hit = 0.0;  /* Extremum's m */
                x->td = 0.0;   /* its span */
            }
        }
    }
}

/* measure.zig Cross.feed for one event (times.len = 1); 1 once the scan
 * is over (its event found, or past TO). */
static int cross_feed(orc_cross *s, const orc_meas_clause *c, double xv, double v) {
    if (s->over) return 1;
    if (xv < s->td) return 0;
    if (xv < c->from) return 0;
    if (c->to != 0 && xv > c->to) {
        s->over = 1;
        return 1;
    }
    const double level = c->val, prev_level = c->val;
    if (s->first == 1) {
        s->cross = 0;
        s->above = !(v < level);
        if (!s->above && s->prev >= prev_level) {
            s->fall = 1;
            s->cross = 1;
        } else if (s->above && s->prev < prev_level) {
            s->rise = 1;
            s->cross = 1;
        }
    }
    if (s->first > 1) {
        if (!s->above && v >= level) {
            s->above = 1;
            s->cross += 1;
            s->rise += 1;
            if (c->fall != ORC_MEAS_LAST) s->pending = 1;
        } else if (s->above && v <= level) {
            s->above = 0;
            s->cross += 1;
            s->fall += 1;
            if (c->rise != ORC_MEAS_LAST) s->pending = 1;
        }
        const double hit = s->prev_x + (prev_level - s->prev) * (xv - s->prev_x) / (v - s->prev - level + prev_level);
        if (s->cross == s->want_cross || s->rise == s->want_rise || s->fall == s->want_fall) {
            s->hit = hit;
            s->found = 1;
            s->over = 1;
            return 1;
        }
        if (s->pending) {
            if (c->cross == ORC_MEAS_UNSET && c->rise == ORC_MEAS_UNSET && c->fall == ORC_MEAS_UNSET) {
                s->hit = hit;
                s->found = 1;
                s->over = 1;
                return 1;
            }
            if (c->cross == ORC_MEAS_LAST || c->rise == ORC_MEAS_LAST || c->fall == ORC_MEAS_LAST) s->last = hit;
            s->pending = 0;
        }
    }
    s->first += 1;
    s->prev = v;
    s->prev_x = xv;
    return 0;
}

/* measure.zig At.feed (not DC, value). */
static int at_feed(orc_cross *s, const orc_meas_clause *c, double xv, double v) {
    if (s->over) return 1;
    if (s->first > 0 && s->prev_x <= c->at && xv >= c->at) {
        s->hit = s->prev + (c->at - s->prev_x) * (v - s->prev) / (xv - s->prev_x);
        s->found = 1;
        s->over = 1;
        return 1;
    }
    s->first += 1;
    s->prev_x = xv;
    s->prev = v;
    return 0;
}

/* measure.zig Extremum.feed (not DC): op 0 min, 1 max, 2 avg; hit holds
 * m, prev/prev_x the last sample, td the span; 1 once past TO. */
static int ext_feed(orc_cross *s, const orc_meas_clause *c, int op, double xv, double v) {
    if (s->over) return 1;
    if (xv < c->from) return 0;
    if (c->to != 0 && xv > c->to) {
        s->over = 1;
        return 1;
    }
    if (!s->first) {
        s->first = 1;
        s->hit = op == 2 ? 0.0 : v;
        s->prev = v;
        s->prev_x = xv;
        return 0;
    }
    if (op == 0) {
        if (v <= s->hit) s->hit = v;
    } else if (op == 1) {
        if (v >= s->hit) s->hit = v;
    } else {
        s->hit += 0.5 * (v + s->prev) * (xv - s->prev_x);
        s->td += xv - s->prev_x;
        s->prev = v;
        s->prev_x = xv;
    }
    return 0;
}

int meas_feed(orc_meas_state *s, const orc_measure *m, uint32_t n_meas, double t, const double *x) {
    int open = 0;
    for (uint32_t c = 0; c < n_meas; c++) {
        const orc_measure *mc = &m[c];
        int done;
        if (mc->kind == ORC_MEAS_FIND_AT) {
            done = at_feed(&s[c].x[0], &mc->a, t, x[mc->a.unknown]);
        } else if (mc->kind == ORC_MEAS_MIN || mc->kind == ORC_MEAS_MAX || mc->kind == ORC_MEAS_AVG) {
            done = ext_feed(&s[c].x[0], &mc->a, (int)(mc->kind - ORC_MEAS_MIN), t, x[mc->a.unknown]);
        } else if (mc->kind == ORC_MEAS_PP) {
            const int d0 = ext_feed(&s[c].x[0], &mc->a, 0, t, x[mc->a.unknown]);
            const int d1 = ext_feed(&s[c].x[1], &mc->a, 1, t, x[mc->a.unknown]);
            done = d0 && d1;
        } else if (mc->kind == ORC_MEAS_WHEN) {
            done = cross_feed(&s[c].x[0], &mc->a, t, x[mc->a.unknown]);
        } else {
            const int da = cross_feed(&s[c].x[0], &mc->a, t, x[mc->a.unknown]);
            const int db = cross_feed(&s[c].x[1], &mc->b, t, x[mc->b.unknown]);
            done = da && db;
        }
        open += !done;
    }
    return open;
}

/* A clause's event time at the end of its data: the event found, else the
 * last event of a LAST count, else NaN (Cross.finish). */
static double cross_result(const orc_cross *s) {
    if (s->found) return s->hit;
    return s->last;
}

void meas_results(const orc_meas_state *s, const orc_measure *m, uint32_t n_meas, double *out) {
    for (uint32_t c = 0; c < n_meas; c++) {
        const orc_measure *mc = &m[c];
        double v;
        if (mc->kind == ORC_MEAS_FIND_AT) {
            v = s[c].x[0].found ? s[c].x[0].hit : NAN;
        } else if (mc->kind == ORC_MEAS_MIN || mc->kind == ORC_MEAS_MAX) {
            v = s[c].x[0].hit;  /* 0 when no sample fell in the window */
        } else if (mc->kind == ORC_MEAS_AVG) {
            v = s[c].x[0].hit / (s[c].x[0].first ? s[c].x[0].td : 1.0);
        } else if (mc->kind == ORC_MEAS_PP) {
            v = s[c].x[1].hit - s[c].x[0].hit;
        } else if (mc->kind == ORC_MEAS_WHEN) {
            v = cross_result(&s[c].x[0]);
        } else {
            const double trig = cross_result(&s[c].x[0]), targ = cross_result(&s[c].x[1]);
            v = isfinite(trig) && isfinite(targ) ? targ - trig : NAN;
        }
        out[c] = isfinite(v) ? v : NAN;
    }
}
