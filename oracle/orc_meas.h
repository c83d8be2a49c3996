/* TEST INFRASTRUCTURE (oracle), not product code: streaming transient
 * measures (see orc_meas.c). */
#ifndef ORC_MEAS_H
#define ORC_MEAS_H
#include "espice_oracle.h"

typedef struct {
    double td, prev, prev_x, last, hit;
    int32_t want_rise, want_fall, want_cross;
    int32_t rise, fall, cross;
    uint32_t first;
    int32_t above, pending, found, over;
} orc_cross;

/* measure.zig Integ: the window's points not folded into a panel yet
 * (scale, value or value squared), the three rules' sums, the last raw
 * sample and the window's ends. */
typedef struct {
    double p[4][2];
    double sum[3];
    double px, py, first_x, cut_x;
    uint32_t rows, np, count, inside, cut, over;
} orc_integ;

typedef struct {
    orc_cross x[2];
    orc_integ g;
} orc_meas_state;

void meas_init(orc_meas_state *s, const orc_measure *m, uint32_t n_meas);
/* Feeds the accepted row (t, x); returns the cards still open. */
int meas_feed(orc_meas_state *s, const orc_measure *m, uint32_t n_meas, double t, const double *x);
void meas_results(const orc_meas_state *s, const orc_measure *m, uint32_t n_meas, double *out);
#endif
