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
 *   measure.zig:1515-1595  Integ: INTEGRAL and RMS over FROM..TO, ends
 *                          interpolated, panels by Simpson's 3/8 rule,
 *                          Simpson's rule or the trapezoid as the spacing
 *                          of the next points allows (ngspice
 *                          measure_rms_integral)
 *   measure.zig:1380-1398  At with slope: DERIV .. AT=, the slope of the
 *                          first segment holding AT
 * Only WHEN, TRIG/TARG (each clause its own TD), FIND AT, MIN, MAX, AVG,
 * PP, INTEGRAL, RMS and DERIV AT are restated, with VAL levels (no vector
 * levels), as the device streams them.
 */
#include "orc_meas.h"

#include <math.h>
#include <stdint.h>
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

/* measure.zig At.feed with slope (DERIV .. AT=). */
static int slope_feed(orc_cross *s, const orc_meas_clause *c, double xv, double v) {
    if (s->over) return 1;
    if (s->first > 0 && s->prev_x <= c->at && xv >= c->at) {
        s->hit = (v - s->prev) / (xv - s->prev_x);
        s->found = 1;
        s->over = 1;
        return 1;
    }
    s->first += 1;
    s->prev_x = xv;
    s->prev = v;
    return 0;
}

/* measure.zig almostEqualUlps (:1699-1708): within 100 units in the last
 * place, on the doubles' order-preserving integer images. */
static int almost_equal_ulps(double a, double b) {
    if (a == b) return 1;
    int64_t ia, ib;
    memcpy(&ia, &a, 8);
    memcpy(&ib, &b, 8);
    if (ia < 0) ia = INT64_MIN - ia;
    if (ib < 0) ib = INT64_MIN - ib;
    const uint64_t d = (uint64_t)ia - (uint64_t)ib;
    const uint64_t mag = (int64_t)d < 0 ? (uint64_t)0 - d : d;
    return mag <= 100;
}

/* measure.zig line (:1257-1261). */
static double line_at(double x0, double y0, double x1, double y1, double at) {
    const double slope = (y1 - y0) / (x1 - x0);
    const double intercept = y0 - slope * x0;
    return slope * at + intercept;
}

/* Integ.panel: folds the oldest points into one panel; `avail` of p are
 * points, the rest read zero, a spacing past them zero. */
static void integ_panel(orc_integ *s, uint32_t avail) {
    double p[4][2];
    memcpy(p, s->p, sizeof(p));
    for (uint32_t j = avail; j < 4; j++) p[j][0] = p[j][1] = 0.0;
    double w[3];
    for (uint32_t j = 0; j < 3; j++) w[j] = j + 1 < avail ? p[j + 1][0] - p[j][0] : 0.0;
    uint32_t used;
    if (almost_equal_ulps(w[0], w[1]) && almost_equal_ulps(w[0], w[2])) {
        s->sum[0] += 3 * w[0] * (p[0][1] + 3 * (p[1][1] + p[2][1]) + p[3][1]) / 8.0;
        used = 3;
    } else if (almost_equal_ulps(w[0], w[1])) {
        s->sum[1] += w[0] * (p[0][1] + 4 * p[1][1] + p[2][1]) / 3.0;
        used = 2;
    } else {
        s->sum[2] += w[0] * (p[0][1] + p[1][1]) / 2;
        used = 1;
    }
    s->np = avail > used ? avail - used : 0;
    memmove(s->p, s->p + (avail - s->np), sizeof(double) * 2 * s->np);
}

/* Integ.feed; 1 once past a nonzero TO. */
static int integ_feed(orc_integ *s, const orc_meas_clause *c, int rms, double xv, double v) {
    if (s->over) return 1;
    int ret = 0;
    if (!s->inside && xv < c->from) goto done;
    s->inside = 1;
    s->cut = c->to != 0 && xv > c->to;
    double pt[2] = {xv, v};
    if (s->cut) {
        if (s->rows > 0 && !almost_equal_ulps(xv, c->to)) {
            pt[0] = c->to;
            pt[1] = line_at(s->px, s->py, xv, v, c->to);
        }
    } else if (s->count == 0 && c->from != 0 && s->rows > 0 && !almost_equal_ulps(xv, c->from)) {
        pt[0] = c->from;
        pt[1] = line_at(s->px, s->py, xv, v, c->from);
    }
    if (rms) pt[1] = pt[1] * pt[1];
    if (s->count == 0) s->first_x = pt[0];
    if (s->cut) s->cut_x = pt[0];
    s->count += 1;
    s->p[s->np][0] = pt[0];
    s->p[s->np][1] = pt[1];
    s->np += 1;
    if (s->np == 4) integ_panel(s, s->np);
    ret = s->cut;
    if (ret) s->over = 1;
done:
    s->rows += 1;
    s->px = xv;
    s->py = v;
    return ret;
}

/* Integ.result. */
static double integ_result(orc_integ s, int rms) {
    if (s.rows == 0) return NAN;
    while (s.np > 1) integ_panel(&s, s.np);
    const double from = s.count > (uint32_t)(s.cut ? 1 : 0) ? s.first_x : NAN;
    const double to = s.cut ? s.cut_x : s.px;
    const double total = s.sum[0] + s.sum[1] + s.sum[2];
    return rms ? sqrt(total / (to - from)) : total;
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
        } else if (mc->kind == ORC_MEAS_DERIV) {
            done = slope_feed(&s[c].x[0], &mc->a, t, x[mc->a.unknown]);
        } else if (mc->kind == ORC_MEAS_INTEG || mc->kind == ORC_MEAS_RMS) {
            done = integ_feed(&s[c].g, &mc->a, mc->kind == ORC_MEAS_RMS, t, x[mc->a.unknown]);
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
        if (mc->kind == ORC_MEAS_FIND_AT || mc->kind == ORC_MEAS_DERIV) {
            v = s[c].x[0].found ? s[c].x[0].hit : NAN;
        } else if (mc->kind == ORC_MEAS_INTEG || mc->kind == ORC_MEAS_RMS) {
            v = integ_result(s[c].g, mc->kind == ORC_MEAS_RMS);
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
