/* TEST INFRASTRUCTURE (oracle), not product code. Internal declarations. */
#ifndef ORC_INTERNAL_H
#define ORC_INTERNAL_H

#include "espice_oracle.h"

/* exp, log, pow and sin of the model code: the functions the CUDA
 * kernels use (espice_b200/csrc/esl_math.h), so that the oracle's model
 * evaluations are bitwise the device's. Built with ORC_LIBM_TRANSCENDENTALS
 * (liboracle_libm.so) they are the host C library's instead, which shows
 * what the choice changes: only last-ulp differences that move a Newton
 * gate sitting at its threshold. */
#ifdef ORC_LIBM_TRANSCENDENTALS
#include <math.h>
#define esl_exp exp
#define esl_log log
#define esl_pow pow
#define esl_sin sin
#else
#include "../espice_b200/csrc/esl_math.h"
#endif

#define NONE 0xffffffffu
#define ORC_MAX_U 6
#define ORC_MAX_E 40
#define ORC_MAX_LIM 4

/* direct.zig:32-35,43-54,542 */
#define PIVOT_TOL 1e-3
#define REPIVOT_FILL_CAP 3.0
#define GROWTH_LIMIT 1e-12
#define REPLAY_RATIO_MAX 30.0
/* converger.zig:366 */
#define X_PLAUSIBLE 1e9

typedef struct {
    uint32_t *a;
    size_t len, cap;
} vec_u32;
typedef struct {
    double *a;
    size_t len, cap;
} vec_f64;

void vu_push(vec_u32 *v, uint32_t x);
void vd_push(vec_f64 *v, double x);
uint64_t bits_of(double x);
double of_bits(uint64_t u);
double norm_inf(const double *x, size_t n);

typedef struct {
    uint32_t n, nnz;
    const uint32_t *cp, *ri, *q;
    uint32_t *pinv, *lp, *up, *prow;
    vec_u32 li, ui, void_slots;
    vec_f64 lx, ux;
    double *udiag, *w, *y, *rscale;
    uint8_t *void_col, *scaled;
    uint32_t *want, *want_of, *prev, *flag, *topo, *stack, *pstack;
    size_t base_lu;
    double fill_cap, keep_min;
    int factored;
    uint32_t epoch;
} slu_t;

void slu_init(slu_t *s, uint32_t n, const uint32_t *cp, const uint32_t *ri, const uint32_t *q);
void slu_free(slu_t *s);
int slu_factor(slu_t *s, const double *vals, double pivot_tol);
int slu_refactor(slu_t *s, const double *vals, double growth);
void slu_solve(slu_t *s, const double *b, double *x);
void slu_solve_t(slu_t *s, const double *b, double *x);

typedef struct {
    uint32_t n;
    const uint32_t *cp, *ri;
    uint32_t *q;
    slu_t lu;
    double *vcopy, *probe;
    int factored;
    uint32_t bypassed, probed_out, full_factors;
} dsv_t;

void dsv_init(dsv_t *d, uint32_t n, const uint32_t *cp, const uint32_t *ri);
void dsv_free(dsv_t *d);
int dsv_factor(dsv_t *d, const double *vals);
void dsv_solve_neg(dsv_t *d, const double *rhs, double *x);

uint32_t find_slot(const uint32_t *col_ptr, const uint32_t *row_idx, uint32_t nnz,
                   uint32_t row, uint32_t col);

/* ------------------------------------------------------------------ */
/* devices                                                             */

typedef struct {
    int kind;          /* 0 static (.op/.dc), 1 transient, 2 transient op (ic) */
    double t;
    double src_scale;
    double gmin;        /* $simparam("gmin") read in an analog block (BSIM3's
                           junction gminx): the gmin-stepping rung's value,
                           negative for the card's */
    uint32_t iteration; /* $simparam("iteration"), 1 on a solve's first */
    int initial_tran;   /* first transient step (MODEINITTRAN) */
} sim_t;

typedef struct {
    uint8_t ru, cu;
} ent_t;

/* Local stamp layout of one instance: the residual rows it writes, its
 * Jacobian entries (row-major, columns ascending), and the same for charge. */
typedef struct {
    int nu;
    uint8_t res_row[ORC_MAX_U];
    int nj;
    ent_t jac[ORC_MAX_E];
    uint8_t q_row[ORC_MAX_U];
    int nq;
    ent_t qjac[ORC_MAX_E];
    int nlim; /* limited images per instance */
} layout_t;

#define ORC_NDER 96 /* derived (bias-independent) values per instance */

typedef struct {
    double f[ORC_MAX_U];
    double J[ORC_MAX_U][ORC_MAX_U];
    double q[ORC_MAX_U];
    double C[ORC_MAX_U][ORC_MAX_U];
} devout_t;

void dev_layout(uint32_t type, const double *prm, layout_t *lay);
int dev_pattern(uint32_t type, const uint32_t *nodes, const double *prm, uint32_t *rows, uint32_t *cols);
void dev_derive(uint32_t type, const double *prm, double *der);
/* lim: this instance's images when lim_active, else NULL. st: state words. */
void dev_eval(uint32_t type, const uint32_t *nd, const double *prm, const double *der,
              const double *x, const double *lim, const double *st, const sim_t *sim,
              devout_t *out);
/* Limit pass: images from x (new) against old (images when active, else
 * x_old); returns 1 when any image moved off its raw value. */
int dev_limit(uint32_t type, const uint32_t *nd, const double *prm, const double *der,
              const double *x, const double *x_old, const double *lim_old, double *lim_new);
/* MODEINITJCT seeds into the lim images; returns 1 when the type seeds. */
int dev_seed(uint32_t type, const uint32_t *nd, const double *prm, const double *der,
             const double *x, double *lim);
int dev_nstate(uint32_t type);
/* The instance's charge states that join the LTE (one per ddt() site the
 * model keeps in the truncation-error test), at raw x; returns the count. */
int dev_qtape(uint32_t type, const uint32_t *nd, const double *prm, const double *der,
              const double *x, double *out);
int mos1_qtape(const uint32_t *nd, const double *der, const double *x, double *out);
/* Stage accepted-step state ($prev latches) from x; `static_` at an OP. */
void dev_stage(uint32_t type, const uint32_t *nd, const double *prm, const double *der,
               const double *x, const double *lim, const sim_t *sim, double *staged);

double source_value(const double *p, const sim_t *sim);
void mos1_derive(const double *prm, double *der);
void mos1_eval(const uint32_t *nd, const double *prm, const double *der, const double *x,
               const double *lim, const double *st, const sim_t *sim, devout_t *o);
void bsim3_derive(const double *prm, double *der);
void bsim3_eval(const uint32_t *nd, const double *der, const double *x, const double *lim, double gmin,
                devout_t *o);
int bsim3_limit(const uint32_t *nd, const double *der, const double *x, const double *x_old,
                const double *lim_old, double *lim_new);
int bsim3_seed(const double *der, double *lim);
int mos1_limit(const uint32_t *nd, const double *prm, const double *der, const double *x,
               const double *x_old, const double *lim_old, double *lim_new);
int mos1_seed(const uint32_t *nd, const double *prm, const double *der, const double *x, double *lim);
int mos1_has_charge(const double *der);
int orc_mos1_supported(const double *prm);

double pnjlim(double vnew, double vold, double vt, double vcrit, int *lim);
double fetlim(double vnew, double vold, double vto);
double limvds(double vnew, double vold);

#endif
