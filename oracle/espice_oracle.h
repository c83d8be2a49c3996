/*
 * TEST INFRASTRUCTURE, NOT PRODUCT CODE.
 *
 * CPU oracle for the sweep-lane Newton path: a plain C (FP64, no FMA
 * contraction) restatement of the reference's CPU algorithm, used only by
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg to check
 * and time the CUDA library. Nothing in espice_b200/ links or imports it.
 *
 * Reference files restated (paths inside the ESPice project):
 *   src/device/Circuit.zig:77-167            frozen CSC pattern, ground row 0
 *   src/solver/order.zig                     BTF (Tarjan) + AMD + natural fallback
 *   src/solver/sparse_lu.zig:260-1224        Gilbert-Peierls factor/refactor/solve
 *   src/solver/direct.zig:32-55,228-383      bypass, refactor, replayHolds, re-pivot
 *   src/solver/converger.zig:85-122,199-522,794-819   Newton gates
 *   src/device/eval.zig:782-922              stamp, limiting correction
 *   models/{resistor,capacitor,vsource,isource,diode,mos1}.va
 *   src/analysis/dc/dc.zig:163-386           sequential .dc sweep
 *   src/analysis/sweep/lanes.zig:34-92       independent sweep points
 *   src/analysis/tran/{integrator,tran}.zig  trapezoidal transient + LTE
 *
 * Parity pinning: the reference cannot be built here (Zig 0.18-dev and its
 * un-vendored VerA/Gompute dependencies are absent). The oracle is pinned
 * against the reference's own ngspice-44.2 golden fixtures (DC rtol 1e-6,
 * transient rtol 1e-3) committed under tests/golden/, and against the
 * reference's bitwise self-consistency properties (lane == scalar).
 */
#ifndef ESPICE_ORACLE_H
#define ESPICE_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Device types and their per-instance layouts (node count, param count). */
enum {
    ORC_R = 0,  /* nodes p n;          params r                          */
    ORC_C = 1,  /* nodes p n;          params c                          */
    ORC_V = 2,  /* nodes p n br;       params: the source layout below   */
    ORC_I = 3,  /* nodes p n;          params: the source layout below   */
    ORC_D = 4,  /* nodes a c ai;       params see ORC_D_* (ai == a: RS collapsed) */
    ORC_M = 5,  /* nodes d g s b di si; params see ORC_M_*               */
    ORC_B3 = 6, /* nodes d g s b di si; params see ORC_B3_* (BSIM3v3 DC) */
    ORC_NTYPES = 7
};

/* Diode parameter slots (models/diode.va). */
enum {
    ORC_D_IS = 0, ORC_D_N, ORC_D_RS, ORC_D_BV, ORC_D_IBV, ORC_D_CJO, ORC_D_VJ,
    ORC_D_M, ORC_D_FC, ORC_D_TT, ORC_D_AREA, ORC_D_GMIN, ORC_D_XTI, ORC_D_EG,
    ORC_D_TNOM, ORC_D_TEMP, ORC_D_NP
};

/* MOS1 parameter slots (models/mos1.va). TYPE = +1 NMOS, -1 PMOS. */
enum {
    ORC_M_TYPE = 0, ORC_M_VTO, ORC_M_KP, ORC_M_GAMMA, ORC_M_PHI, ORC_M_LAMBDA,
    ORC_M_RD, ORC_M_RS, ORC_M_CBD, ORC_M_CBS, ORC_M_IS, ORC_M_PB, ORC_M_CGSO,
    ORC_M_CGDO, ORC_M_CGBO, ORC_M_CJ, ORC_M_MJ, ORC_M_CJSW, ORC_M_MJSW,
    ORC_M_TOX, ORC_M_LD, ORC_M_U0, ORC_M_FC, ORC_M_W, ORC_M_L, ORC_M_AD,
    ORC_M_AS, ORC_M_PD, ORC_M_PS, ORC_M_DELVTO, ORC_M_M, ORC_M_GMIN,
    ORC_M_TNOM, ORC_M_TEMP, ORC_M_NP
};

/* BSIM3v3 DC-core parameter slots (models/bsim3.va:26-138, model card then
 * instance). A NaN value means "not given": the slots whose defaults depend
 * on $param_given (TOXM, NCH, GAMMA1, GAMMA2, VBX, K1, K2, VTH0, VFB, DSUB,
 * UC, UC1, U0) take their derived defaults then. */
enum {
    ORC_B3_TYPE = 0, ORC_B3_MOBMOD, ORC_B3_TNOM, ORC_B3_TOX, ORC_B3_TOXM, ORC_B3_XJ,
    ORC_B3_NCH, ORC_B3_NSUB, ORC_B3_NGATE, ORC_B3_GAMMA1, ORC_B3_GAMMA2, ORC_B3_XT,
    ORC_B3_VBX, ORC_B3_VBM, ORC_B3_K1, ORC_B3_K2, ORC_B3_K3, ORC_B3_K3B, ORC_B3_W0,
    ORC_B3_NLX, ORC_B3_VTH0, ORC_B3_VFB, ORC_B3_DVT0, ORC_B3_DVT1, ORC_B3_DVT2,
    ORC_B3_DVT0W, ORC_B3_DVT1W, ORC_B3_DVT2W, ORC_B3_DROUT, ORC_B3_DSUB, ORC_B3_NFACTOR,
    ORC_B3_CDSC, ORC_B3_CDSCB, ORC_B3_CDSCD, ORC_B3_CIT, ORC_B3_VSAT, ORC_B3_AT,
    ORC_B3_A0, ORC_B3_AGS, ORC_B3_A1, ORC_B3_A2, ORC_B3_KETA, ORC_B3_UA, ORC_B3_UA1,
    ORC_B3_UB, ORC_B3_UB1, ORC_B3_UC, ORC_B3_UC1, ORC_B3_U0, ORC_B3_UTE, ORC_B3_VOFF,
    ORC_B3_DELTA, ORC_B3_RDSW, ORC_B3_PRWG, ORC_B3_PRWB, ORC_B3_PRT, ORC_B3_WR,
    ORC_B3_ETA0, ORC_B3_ETAB, ORC_B3_PCLM, ORC_B3_PDIBLC1, ORC_B3_PDIBLC2,
    ORC_B3_PDIBLCB, ORC_B3_PSCBE1, ORC_B3_PSCBE2, ORC_B3_PVAG, ORC_B3_DWG, ORC_B3_DWB,
    ORC_B3_B0, ORC_B3_B1, ORC_B3_ALPHA0, ORC_B3_ALPHA1, ORC_B3_BETA0, ORC_B3_KT1,
    ORC_B3_KT1L, ORC_B3_KT2, ORC_B3_LINT, ORC_B3_LL, ORC_B3_LLN, ORC_B3_LW, ORC_B3_LWN,
    ORC_B3_LWL, ORC_B3_WINT, ORC_B3_WL, ORC_B3_WLN, ORC_B3_WW, ORC_B3_WWN, ORC_B3_WWL,
    ORC_B3_XL, ORC_B3_XW, ORC_B3_JS, ORC_B3_JSW, ORC_B3_NJ, ORC_B3_XTI, ORC_B3_IJTH,
    ORC_B3_RSH, ORC_B3_L, ORC_B3_W, ORC_B3_AD, ORC_B3_AS, ORC_B3_PD, ORC_B3_PS,
    ORC_B3_NRD, ORC_B3_NRS, ORC_B3_M, ORC_B3_DELVTO, ORC_B3_MULU0, ORC_B3_GMIN,
    ORC_B3_TEMP, ORC_B3_NP
};

typedef struct {
    uint32_t type;
    uint32_t count;
    const uint32_t *nodes;  /* count * nodes_per_type */
    const double *params;   /* count * params_per_type */
} orc_batch;

typedef struct {
    uint32_t n;             /* unknowns, ground row 0 included */
    uint32_t n_batches;
    const orc_batch *batches;
    const uint8_t *current_row; /* n: 1 for a branch-current unknown */
} orc_circuit;

/* One swept parameter slot: batch, instance, param index. */
typedef struct {
    uint32_t batch, inst, param;
} orc_slot;

typedef struct {
    double reltol, abstol, vntol, residual_tol, gmin;
    uint32_t max_iter;      /* before the max(itl, 100) raise */
} orc_newton_opts;

/* V and I source parameters (models/vsource.va, isource.va): dc, wave
 * (0 DC, 1 PULSE, 2 SIN, 3 EXP, 4 PWL), the wave's eight parameters (PULSE
 * v1 v2 td tr tf pw per phase; SIN vo va freq td theta phase; EXP v1 v2 td1
 * tau1 td2 tau2; PWL len repeat td), then the PWL table: 64 times, 64
 * values. */
#define ORC_SRC_NP 138
#define ORC_SRC_PWL_T 10
#define ORC_SRC_PWL_V 74
#define ORC_PWL_MAX 64
int orc_nodes_per(uint32_t type);
int orc_params_per(uint32_t type);
/* One instance's static stamp at local voltages xloc[nodes_per(type)] (node
 * k of the instance is xloc[k]), no limiting: residuals f[6] and Jacobian
 * J[6][6] over its local nodes, row-major. A test hook for the models'
 * derivatives. Returns 0, or 1 for an unknown type. */
/* The model code's exp (which 0), log (1) or pow (2) over n arguments. */
void orc_math(int which, uint32_t n, const double *x, const double *y, double *out);
int orc_dev_stamp(uint32_t type, const double *prm, const double *xloc, double *f, double *J);

/* Pattern (Circuit.freeze): CSC with every diagonal, rows ascending.
 * col_ptr has n + 1 entries; row_idx capacity is given; returns nnz or -1. */
int64_t orc_pattern(const orc_circuit *c, uint32_t *col_ptr, uint32_t *row_idx, size_t cap);

/* Column order (order.zig `order`). 0 on success. */
int orc_order(uint32_t n, const uint32_t *col_ptr, const uint32_t *row_idx, uint32_t *q);

/* Full factor of one matrix (direct.Solver.factor from a fresh solver),
 * exporting the pivot tape. Sizes out: counts[0] = nnz_L, counts[1] = nnz_U.
 * Any output pointer may be NULL. Returns 0, or 1 for a singular matrix. */
int orc_factor_tape(uint32_t n, const uint32_t *col_ptr, const uint32_t *row_idx,
                    const double *vals, uint32_t *q, uint32_t *pinv,
                    uint32_t *lp, uint32_t *li, double *lx,
                    uint32_t *up, uint32_t *ui, double *ux, double *udiag,
                    uint8_t *flags, uint32_t *counts, size_t cap);

/* Refactor of `vals` on the tape a full factor of `lead` made, then
 * dx = -A^-1 rhs; `bad` = the lane kernel's peel verdict (pivot test,
 * growth, non-finite, wide multiplier). Bitwise the reference's
 * lane_kernels.Bodies.refactor + solveNeg on the host. */
int orc_lane_refactor_solve(uint32_t n, const uint32_t *col_ptr, const uint32_t *row_idx,
                            const double *lead, uint32_t n_lanes, const double *vals,
                            const double *rhs, double *dx, double *lx_out, double *ux_out,
                            double *udiag_out, uint8_t *bad);

/* Each lane a direct.Solver of its own: factor (bypass / refactor+replayHolds
 * / full factor) then solveNeg, over `rounds` rounds of values per lane.
 * vals [rounds][n_lanes][nnz], rhs [rounds][n_lanes][n] -> dx same shape,
 * status [rounds][n_lanes] (0 ok, 1 singular). */
int orc_solver_rounds(uint32_t n, const uint32_t *col_ptr, const uint32_t *row_idx,
                      uint32_t rounds, uint32_t n_lanes, const double *vals,
                      const double *rhs, double *dx, uint8_t *status);

/* Independent DC sweep points (sweep/lanes.zig solveLanes): each lane
 * installs its slot values, starts from `warm` (n values) or cold, and
 * runs converger.run. x_out [n_lanes][n], iters, conv per lane. */
int orc_dc_points(const orc_circuit *c, const orc_slot *slots, uint32_t n_slots,
                  const double *values, uint32_t n_lanes, const double *warm,
                  const orc_newton_opts *opts, double *x_out, uint32_t *iters,
                  uint8_t *conv);
/* orc_dc_points recording each lane's gate inputs per iterate: trace
 * [n_lanes][cap][3] = (delta score, max |rhs_i| / residual gate, limited
 * flag), NaN past the lane's last iterate. */
int orc_dc_points_trace(const orc_circuit *c, const orc_slot *slots, uint32_t n_slots,
                        const double *values, uint32_t n_lanes, const double *warm,
                        const orc_newton_opts *opts, double *x_out, uint32_t *iters,
                        uint8_t *conv, double *trace, uint32_t cap);

/* Sequential .dc sweep (dc.zig Sweep): point 0 cold, later points warm
 * from the 2*last - prev predictor limited against the last point; a failed
 * warm point takes the plain cold rung. x_out [n_pts][n]. */
int orc_dc_sweep(const orc_circuit *c, orc_slot slot, const double *values,
                 uint32_t n_pts, const orc_newton_opts *opts, double *x_out,
                 uint32_t *iters, uint8_t *conv);

/* One sequential sweep per lane, each lane first setting slots[] to its row
 * of lane_values [n_lanes][n_slots]; x_out [n_lanes][n_pts][n], iters and
 * conv [n_lanes][n_pts]. */
int orc_dc_sweep_lanes(const orc_circuit *c, const orc_slot *slots, uint32_t n_slots,
                       const double *lane_values, uint32_t n_lanes, orc_slot sweep,
                       const double *values, uint32_t n_pts, const orc_newton_opts *opts,
                       double *x_out, uint32_t *iters, uint8_t *conv);

/* Operating point (op.zig solve, plain rung, cold start). */
/* Operating points of independent lanes through op.zig's ladder (plain,
 * gmin stepping, source stepping) from the cold start; rung per lane: 0
 * plain, 1 gmin, 2 source, 3 not converged. iter_cap (0: none) caps every
 * Newton run. */
int orc_op_points(const orc_circuit *c, const orc_slot *slots, uint32_t n_slots, const double *values,
                  uint32_t n_lanes, const orc_newton_opts *opts, uint32_t iter_cap, double *x_out,
                  uint32_t *iters, uint8_t *conv, uint8_t *rung);
int orc_op(const orc_circuit *c, const orc_newton_opts *opts, double *x_out,
           uint32_t *iters);

/* Transient (src/analysis/tran/tran.zig Sim.begin/end with HostOps,
 * integrator.zig): each lane its own operating point (cold start, plain
 * Newton), then BE-started trapezoidal steps with LTE control on the
 * devices' charge states, order promotion, Newton rejection (dt / 8) and
 * PULSE-corner breakpoints. Lanes are independent, each with its slot
 * values. Records (t, x[probes]) at t = 0 and every accepted step:
 * out_t [n_lanes][max_pts], out_v [n_lanes][max_pts][n_probes], rows
 * written per lane in n_pts_out (recording stops at max_pts). stats
 * [n_lanes][ORC_TS_N]; x_final [n_lanes][n] the last accepted solution. */
typedef struct {
    double tstop, tstep, tmax;  /* .tran tstep tstop; tmax <= 0: min(tstep, tstop / 50) */
    double reltol, abstol, vntol, chgtol, trtol, dt_min;
    uint32_t max_steps;
} orc_tran_opts;

enum {
    ORC_TS_STATUS,      /* 0 reached tstop, 1 dt underflow, 2 OP failed, 3 max_steps */
    ORC_TS_ACCEPTED,
    ORC_TS_ATTEMPTS,
    ORC_TS_NR_ITERS,
    ORC_TS_REJ_NEWTON,
    ORC_TS_REJ_LTE,
    ORC_TS_BP_LANDINGS,
    ORC_TS_OP_ITERS,
    ORC_TS_N
};

/* Streamed transient measures (src/output/measure.zig): WHEN (the time of
 * a clause's event), TRIG/TARG (targ - trig, each clause its own TD) and
 * FIND .. AT= (the value at a time), and MIN, MAX, AVG (trapezoidal mean)
 * and PP over the FROM..TO window of clause a. A clause: the probed unknown, the level
 * VAL, RISE/FALL/CROSS counts (ORC_MEAS_UNSET, ORC_MEAS_LAST or k >= 1),
 * TD, FROM, TO (0: none) and AT. */
enum { ORC_MEAS_WHEN = 0, ORC_MEAS_TRIG_TARG = 1, ORC_MEAS_FIND_AT = 2,
       ORC_MEAS_MIN = 3, ORC_MEAS_MAX = 4, ORC_MEAS_AVG = 5, ORC_MEAS_PP = 6,
       ORC_MEAS_INTEG = 7, ORC_MEAS_RMS = 8, ORC_MEAS_DERIV = 9 };
enum { ORC_MEAS_UNSET = -1, ORC_MEAS_LAST = -2 };
typedef struct {
    uint32_t unknown;
    int32_t rise, fall, cross;
    double val, td, from, to, at;
} orc_meas_clause;
typedef struct {
    uint32_t kind, pad;
    orc_meas_clause a, b;
} orc_measure;

/* orc_tran with measures: meas [n_meas] cards fed every recorded row (t = 0
 * and every accepted step); values [n_lanes][n_meas] (NaN: unresolved);
 * with early_stop a lane ends its transient once every card has resolved
 * (status ORC_TRAN_RESOLVED). */
enum { ORC_TRAN_RESOLVED = 5 };
int orc_tran_meas(const orc_circuit *c, const orc_slot *slots, uint32_t n_slots,
                  const double *values, uint32_t n_lanes, const orc_tran_opts *topts,
                  const orc_measure *meas, uint32_t n_meas, int early_stop, double *meas_out,
                  uint32_t *stats, double *x_final);

int orc_tran(const orc_circuit *c, const orc_slot *slots, uint32_t n_slots,
             const double *values, uint32_t n_lanes, const orc_tran_opts *topts,
             const uint32_t *probe_nodes, uint32_t n_probes, uint32_t max_pts,
             double *out_t, double *out_v, uint32_t *n_pts_out, uint32_t *stats,
             double *x_final);

#ifdef __cplusplus
}
#endif
#endif
