/* TEST INFRASTRUCTURE (oracle), not product code. Circuit runtime. */
#ifndef ORC_CKT_H
#define ORC_CKT_H

#include "orc_internal.h"

typedef struct {
    uint32_t type, count, nt, np;
    const uint32_t *nodes;
    double *prm;        /* mutable copy: swept slots land here */
    double *der;        /* ORC_NDER per instance */
    layout_t *lay;
    uint32_t *slot;     /* jac entry -> CSC slot (nnz = trash) */
    uint32_t *qslot;
    uint32_t lim_off, st_off;
} bat_t;

typedef struct {
    const orc_circuit *c;
    uint32_t n, nnz, nb, nlim, nst;
    uint32_t *cp, *ri, *diag;
    bat_t *bt;
    double *g, *cv, *rhs, *q;   /* planes: nnz + 1 / n + 1 (trash last) */
    double *lim, *lim_new;
    int lim_active;
    double *st;                 /* committed state, then staged state */
    double *dx, *x_old;
    double last_scaled;
    double *trace;              /* optional per-iterate gate inputs (orc_dc_points_trace) */
    uint32_t trace_cap;
    sim_t sim;
    dsv_t dsv;
    /* transient companion hook (integrator.zig Hook): when `tran`, the
     * residual gains ag0*(q - q1) (- ag1*ip for trap) and the matrix is
     * G + ag0*C in av */
    int tran, trap;
    double ag0, ag1;
    const double *q1, *ip;
    double *av;
    /* op.zig gmin stepping: gmin `gs` loaded at the n_gst stamps
     * (slot, row, col) instead of every diagonal, when gs > 0 */
    double gs;
    uint32_t iter_cap;          /* 0, or a cap on every Newton run below max_iter */
    uint32_t n_gst;
    uint32_t *gst;
} ckt_t;

int ckt_init(ckt_t *k, const orc_circuit *c);
void ckt_free(ckt_t *k);
void ckt_set(ckt_t *k, orc_slot s, double v);
void ckt_assemble(ckt_t *k, const double *x);
int ckt_apply_limits(ckt_t *k, const double *x, const double *x_old);
void ckt_seed(ckt_t *k, double *x);
void ckt_cold_start(ckt_t *k, double *x);
int ckt_newton(ckt_t *k, double *x, const orc_newton_opts *opts, int init_fix, uint32_t *iters);
uint32_t ckt_qtape(ckt_t *k, const double *x, double *out);
int ckt_run(ckt_t *k, double *x, const orc_newton_opts *opts, int init_fix, uint32_t *iters);
uint32_t ckt_gmin_stamps(const ckt_t *k, uint32_t *out);
int ckt_ladder(ckt_t *k, double *x, const orc_newton_opts *opts, uint32_t *iters, uint32_t *rung);
double update_and_norm(uint32_t n, double *x, const double *dx, double *x_old, const uint8_t *cur,
                       double reltol, double abstol, double vntol);

#endif
