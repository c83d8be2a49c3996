/*
 * espice_lanes.h: C ABI of the B200 sweep-lane Newton library
 * (libespice_lanes.so). Plain C types only; all device memory is owned by
 * the context.
 *
 * The reference reaches this path through Gompute raw kernels driven by
 * src/analysis/gpu_lanes.zig (GpuLanes.init / newton / deinit,
 * gpu_lanes.zig:349-845) under tran.runGpuLanes (tran.zig:1654) and, on the
 * CPU, sweep/lanes.solveBatch (sweep/lanes.zig:186-233). A Zig host would
 * call these entry points where gpu_lanes.zig launches its kernels, through
 * an `extern` block that declares them with the same C types.
 *
 * Threading: calls on one context must be serialized (the rule of
 * include/espice.h:139-156 for a problem handle). Each context owns one CUDA
 * stream on one device; contexts are independent.
 */
#ifndef ESPICE_LANES_H
#define ESPICE_LANES_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes (int32). The reference's outcomes they map to: */
enum {
    ESL_OK = 0,
    ESL_INVALID_ARGUMENT = 1, /* espice.h ESPICE_INVALID_ARGUMENT */
    ESL_OUT_OF_MEMORY = 3,    /* OutOfMemory */
    ESL_NOT_ELIGIBLE = 4,     /* tran.zig:1612 gpuLaneRefusal: run on the CPU */
    ESL_NO_DEVICE = 5,        /* no CUDA device / image: run on the CPU */
    ESL_DEVICE_FAULT = 6,     /* a driver error mid-run: QueryCancelled (tran.zig:1824) */
    ESL_TIMEOUT = 7           /* a bounded device wait ran out */
};

/* Device types and per-instance layouts (unknown indices; 0 is ground). */
enum {
    ESL_R = 0, /* nodes p n;          params r                               */
    ESL_C = 1, /* nodes p n;          params c                               */
    ESL_V = 2, /* nodes p n br;       params: ESL_SRC_PARAMS (below)         */
    ESL_I = 3, /* nodes p n;          params: ESL_SRC_PARAMS (below)         */
    ESL_D = 4, /* nodes a c ai;       params is n rs bv ibv cjo vj m fc tt area gmin xti eg tnom temp */
    ESL_M = 5, /* nodes d g s b di si; params (MOS1, models/mos1.va; kp NaN =
                  not given: u0 * Cox' with tox > 0, else 2e-5; a circuit with
                  tox > 0 runs DC only, its transients ESL_NOT_ELIGIBLE)    */
    ESL_B3 = 6 /* nodes d g s b di si; params (BSIM3v3 DC core, models/bsim3.va) */
};

/* ESL_V and ESL_I parameters (models/vsource.va, isource.va): dc; wave (0
 * DC, 1 PULSE, 2 SIN, 3 EXP, 4 PWL); the wave's eight parameters (PULSE v1
 * v2 td tr tf pw per phase, the -1 sentinels of the .va for tr tf pw per;
 * SIN vo va freq td theta phase; EXP v1 v2 td1 tau1 td2 tau2; PWL len
 * repeat td, repeat < 0 for none); then the PWL table: ESL_PWL_MAX times
 * (non-decreasing) and ESL_PWL_MAX values. Static analyses bias at dc, the
 * transient and its operating point at the wave; PULSE and PWL corners are
 * breakpoints of the transient. */
#define ESL_PWL_MAX 64
#define ESL_SRC_PARAMS 138

/* ESL_B3 parameter slots: the model card of models/bsim3.va:26-138 in its
 * order (type mobmod tnom tox toxm xj nch nsub ngate gamma1 gamma2 xt vbx
 * vbm k1 k2 k3 k3b w0 nlx vth0 vfb dvt0 dvt1 dvt2 dvt0w dvt1w dvt2w drout
 * dsub nfactor cdsc cdscb cdscd cit vsat at a0 ags a1 a2 keta ua ua1 ub ub1
 * uc uc1 u0 ute voff delta rdsw prwg prwb prt wr eta0 etab pclm pdiblc1
 * pdiblc2 pdiblcb pscbe1 pscbe2 pvag dwg dwb b0 b1 alpha0 alpha1 beta0 kt1
 * kt1l kt2 lint ll lln lw lwn lwl wint wl wln ww wwn wwl xl xw js jsw nj xti
 * ijth rsh), then the instance (l w ad as pd ps nrd nrs m delvto mulu0),
 * then gmin and the device temperature in K: ESL_B3_PARAMS doubles. type is
 * +1 NMOS, -1 PMOS. A NaN slot is a parameter left off the card: toxm, nch,
 * gamma1, gamma2, vbx, k1, k2, vth0, vfb, dsub, uc, uc1 and u0 then take the
 * defaults the model derives ($param_given). The DC core has no charges. */
#define ESL_B3_PARAMS 109

/* Per-lane outcome (esl_lane_result.status). */
enum {
    ESL_LANE_CONVERGED = 1,
    ESL_LANE_MAX_ITER = 2, /* Newton ran out of iterations (non-converged point) */
    ESL_LANE_SINGULAR = 3, /* the lane's own factor failed (SingularMatrix) */
    ESL_LANE_NEED_SOLVE = 4 /* left the lead tape; only esl_dc_solve_device_static leaves it */
};

typedef struct {
    uint32_t type;
    uint32_t count;
    const uint32_t *nodes;  /* count * nodes-per-type */
    const double *params;   /* count * params-per-type */
} esl_batch;

/* A frozen circuit (src/device/Circuit.zig:77-167): n unknowns, ground is
 * row/column 0 held by a unit pin, device batches in stamp order. */
typedef struct {
    uint32_t n;
    uint32_t n_batches;
    const esl_batch *batches;
    const uint8_t *current_row; /* n: 1 for a branch-current unknown */
} esl_circuit;

/* One swept parameter of a lane: batch, instance, parameter index. */
typedef struct {
    uint32_t batch, inst, param;
} esl_slot;

/* converger.Options (converger.zig:99-122) for one solve. */
typedef struct {
    double reltol, abstol, vntol, residual_tol, gmin;
    uint32_t max_iter;   /* raised to at least 100, as optionsFromTolerances does */
    uint32_t init_fix;   /* MODEINITFIX: publish the second passing iterate */
    uint32_t iter_cap;   /* 0, or a hard cap on Newton iterations below max_iter (a learned
                            warm start's budget before its nominal fallback) */
} esl_newton_opts;

typedef struct {
    int device;               /* CUDA ordinal */
    uint32_t lanes_per_block; /* warps per CTA; 0 picks the tuned value */
} esl_options;

typedef struct esl_ctx esl_ctx;

typedef struct {
    uint32_t lanes;        /* lanes solved */
    uint32_t converged;    /* lanes that converged */
    uint32_t peeled;       /* lanes that paused for a host factor at least once */
    uint32_t host_solves;  /* host factor+solve calls (lane_solver.zig peels) */
    uint32_t launches;     /* kernel launches in the call */
    double kernel_ms;      /* device time of the Newton launches */
    uint32_t path;         /* the lanes that ran: ESL_PATH_WARP or ESL_PATH_BLOCK */
    uint32_t refinements;  /* mixed precision: FP64 refinement corrections, all lanes */
} esl_stats;

/* How a context's DC solves run (esl_set_mode). No reference counterpart:
 * the reference's lane LU is FP64 and one thread per lane.
 *
 * precision: ESL_PREC_FP64 (the default), or ESL_PREC_MIXED: the refactor
 * and the triangular solves in FP32 on the same pivot tape, each Newton step
 * then refined in FP64 (residual -F - J dx from the FP64 Jacobian, the
 * correction solved on the FP32 factors) until max |res| <= refine_tol *
 * max |F| or refine_max corrections; device evaluation, assembly, the
 * update and the Newton gates stay FP64. A lane the FP32 factors cannot
 * stand in for (the pivot tests on them) takes the host's FP64 factor.
 * path: ESL_PATH_AUTO picks the warp lanes (a warp per lane, its working
 * set in shared memory) for FP64 when the tape fits them, else the block
 * lanes (a CTA per lane, block_threads wide: 256, or 0 for 256; the
 * working set in shared memory when it fits, else in global memory, for any
 * circuit size); ESL_PATH_WARP / ESL_PATH_BLOCK force one (the warp lanes
 * are FP64 only). refine_tol 0 takes 1e-12, refine_max 0 takes 6.
 * refine_skip > 0 (mixed precision): a Newton step whose FP32 solution is
 * still more than refine_skip times its convergence tolerance (the delta
 * score, max |dx_i| / (reltol max(|x_i|, |x_i + dx_i|) + vntol or abstol))
 * is taken unrefined, as an inexact Newton step; the steps nearer
 * convergence, the accepted one among them, are refined. 0: every step is
 * refined. */
enum { ESL_PREC_FP64 = 0, ESL_PREC_MIXED = 1 };
enum { ESL_PATH_AUTO = 0, ESL_PATH_WARP = 1, ESL_PATH_BLOCK = 2 };
typedef struct {
    uint32_t precision;
    uint32_t path;
    uint32_t block_threads;
    uint32_t refine_max;
    double refine_tol;
    uint32_t profile;  /* != 0: block-lane solves count their phase cycles (esl_block_profile) */
    uint32_t pad;
    double refine_skip;
} esl_solve_mode;

/* Builds the pattern, column order and stamp tables of `circuit` on
 * `opts->device` (NULL: device 0). Replaces GpuLanes.init's pattern and
 * table work (gpu_lanes.zig:349-622). */
int32_t esl_create(const esl_circuit *circuit, const esl_options *opts, esl_ctx **out);

/* Frees every device buffer of the context (GpuLanes.deinit,
 * gpu_lanes.zig:626-662). NULL is a no-op. */
int32_t esl_destroy(esl_ctx *ctx);

/* The last error's text on this context ("" when none). */
const char *esl_last_error(const esl_ctx *ctx);

/* Matrix dimension n and pattern size nnz of the context's circuit. */
int32_t esl_dims(const esl_ctx *ctx, uint32_t *n, uint32_t *nnz);

/* Installs n_lanes lanes: lane l sets slots[s] to values[l * n_slots + s]
 * on the nominal circuit (the per-lane params of sweep/lanes.zig install,
 * :96-100), derives each lane's device records and uploads them. */
int32_t esl_set_lanes(esl_ctx *ctx, const esl_slot *slots, uint32_t n_slots,
                      const double *values, uint32_t n_lanes);

/* esl_set_lanes with the values of a lane's live parameters: values is
 * [n_lanes][n_cols] row-major and slot s takes column cols[s] (cols[s] <
 * n_cols), so one parameter can set many device fields, as a live .param
 * (include/espice.h:99,310-312, espice_append_points' [count]
 * [live_param_count] rows) sets every instance that names it. The host
 * uploads n_lanes * n_cols values; the device expands them while it derives
 * the records. INVALID_ARGUMENT for a column out of range. */
int32_t esl_set_lanes_cols(esl_ctx *ctx, const esl_slot *slots, uint32_t n_slots,
                           const uint32_t *cols, const double *values, uint32_t n_cols,
                           uint32_t n_lanes);

/* DC Newton for every lane, each bitwise its own converger.run on its own
 * direct solver (sweep/lanes.zig solveBatch, :186-233). Host buffers:
 * x0 [n_lanes][n] start points (NULL: cold, op.zig coldStart), x_out
 * [n_lanes][n], iters and status [n_lanes] (ESL_LANE_*). The call copies
 * the start points in and the results out. */
int32_t esl_dc_solve(esl_ctx *ctx, const esl_newton_opts *opts, const double *x0,
                     double *x_out, uint32_t *iters, uint32_t *status, esl_stats *stats);

/* esl_dc_solve on device buffers: d_x [n_lanes][n] start points in place of
 * x0 (overwritten with the solutions), d_iters/d_status device arrays.
 * cold != 0 seeds the junctions and starts from zero. Returns once the
 * lanes are done (host peels included). Runs on the warp or the block lanes
 * in the context's precision (esl_set_mode). */
int32_t esl_dc_solve_device(esl_ctx *ctx, const esl_newton_opts *opts, double *d_x, int cold,
                            uint32_t *d_iters, uint32_t *d_status, esl_stats *stats);

/* Operating-point lanes: every lane's operating point from the cold start
 * through op.zig's continuation ladder (src/analysis/dc/op.zig:84-320,
 * solveLadder and afterPlain), the batched form of op.solve without holds.
 * Rung 1 is plain Newton with MODEINITFIX (opts->init_fix is implied);
 * a lane it leaves unconverged goes on, on the device and without the
 * host, to dynamic gmin stepping (gmin from 1e-2 down to 1e-12 at ngspice's
 * diagonal placement, the BSIM3 junction gmin following it; a clean solve
 * at the end) and then source stepping (V and I sources scaled by an
 * adaptive lambda) and the full-source Newton. Each stepping run has a
 * cap of max(itl2, 100) = 100 iterations, the others opts->max_iter (at
 * least 100); opts->iter_cap caps every run. Rungs 4 (JFNK) and 5 (OPtran)
 * are not built: a lane that needs them reads ESL_LANE_MAX_ITER. iters:
 * the plain run's iterations, or the sum over every run once the lane
 * entered the ladder (saturating at 65535, op.zig's u16); rung: 0 plain,
 * 1 gmin stepping, 2 source stepping, 3 not converged. Lanes whose factor
 * leaves the lead tape pause for the host's factor as in esl_dc_solve. */
int32_t esl_op_solve(esl_ctx *ctx, const esl_newton_opts *opts, double *x_out, uint32_t *iters,
                     uint32_t *status, uint32_t *rung, esl_stats *stats);

/* esl_op_solve on device buffers: d_x [n_lanes][n] (the solutions out),
 * d_iters, d_status and d_rung [n_lanes]. */
int32_t esl_op_solve_device(esl_ctx *ctx, const esl_newton_opts *opts, double *d_x, uint32_t *d_iters,
                            uint32_t *d_status, uint32_t *d_rung, esl_stats *stats);

/* esl_dc_solve_device without allocating. No counterpart in the reference:
 * its lane solver allocates its lane planes per call.
 *
 * For callers that cannot allocate device memory while they solve: a
 * process whose device memory is held by a pool sized at start-up, and any
 * caller that keeps work in flight on other streams, where cudaMalloc and
 * cudaFree would synchronise the whole device. The call allocates no device
 * memory: the per-lane Newton state and the paused-lane buffers live in one
 * fixed 16 MiB device array in the library, and the lane start state is set
 * by a kernel. Per lane it needs 8 * (nnz + 3 n + max(nlim, 1) + 1) + 8
 * bytes (each plane rounded up to 256 bytes, plus 256 for a counter); more
 * lanes than fit are refused with ESL_INVALID_ARGUMENT before any launch.
 *
 * Set-up: the first call on a device looks up the array's address, and the
 * first call on a context reserves its error-message buffer; make that
 * first call before any stream capture begins. The address is kept for the
 * life of the process: a cudaDeviceReset on that device (which also frees
 * every context's device memory) is not supported while the library is
 * loaded. Each call waits for its stream before it returns (it reads the
 * paused-lane count back to the host). The context needs its pivot
 * tape (one esl_dc_solve_device call on it first) and its lanes (esl_set_lanes).
 * Nothing has to start at zero: the call writes every lane's start state and
 * clears the counter itself. Calls overlapping in time on one device (any
 * contexts, streams or host threads) share the array and race: serialise them.
 *
 * Same arguments and results as esl_dc_solve_device, except that lanes that
 * leave the lead pivot tape are not served on the host (that needs memory):
 * they are left with status ESL_LANE_NEED_SOLVE, their count goes to
 * *n_paused (may be NULL) and the call returns ESL_NOT_ELIGIBLE. */
int32_t esl_dc_solve_device_static(esl_ctx *ctx, const esl_newton_opts *opts, double *d_x,
                                   int cold, uint32_t *d_iters, uint32_t *d_status,
                                   uint32_t *n_paused);

/* Transient options (src/core/query.zig Tran with Tolerances). t_max <= 0
 * takes min(t_step, t_stop / 50) (src/frontend/analyses.zig:534); dt_min <= 0
 * takes 1e-18; max_steps 0 means unbounded. */
typedef struct {
    double t_stop, t_step, t_max;
    double reltol, abstol, vntol, chgtol, trtol, dt_min;
    uint32_t max_steps;
} esl_tran_opts;

/* Per-lane transient statistics, uint32 [n_lanes][ESL_TS_N]. */
enum {
    ESL_TS_STATUS = 0,      /* ESL_TRAN_* */
    ESL_TS_ACCEPTED = 1,
    ESL_TS_ATTEMPTS = 2,
    ESL_TS_NR_ITERS = 3,
    ESL_TS_REJ_NEWTON = 4,
    ESL_TS_REJ_LTE = 5,
    ESL_TS_BP_LANDINGS = 6,
    ESL_TS_OP_ITERS = 7,
    ESL_TS_N = 8
};
enum {
    ESL_TRAN_DONE = 0,       /* reached t_stop */
    ESL_TRAN_UNDERFLOW = 1,  /* TimestepTooSmall */
    ESL_TRAN_OP_FAILED = 2,  /* the operating point did not converge */
    ESL_TRAN_MAX_STEPS = 3,
    ESL_TRAN_LEFT_TAPE = 4   /* a block lane whose factor left the lead tape (the warp lanes peel instead) */
};

/* Monte-Carlo transient lanes (tran.runGpuLanes, tran.zig:1654, driving
 * gpu_lanes.zig predictRound/newton/apply per tick): each lane solves its
 * operating point from a cold start, then steps trapezoidally (BE first
 * step, order promotion, LTE control over the charge states, Newton
 * rejection, PULSE and PWL breakpoints) to t_stop, all inside one launch.
 * A lane whose factor leaves the lead pivot tape pauses, takes a factor
 * of its own on the host (lane_solver.zig's peel) and resumes where it
 * stopped, in a further launch (esl_peel_counts). Host
 * buffers: x_out [n_lanes][n] the last accepted solution, stats
 * [n_lanes][ESL_TS_N]; with max_pts > 0, probes [n_probes] unknowns
 * recorded at t = 0 and every accepted step into t_out [n_lanes][max_pts],
 * v_out [n_lanes][max_pts][n_probes], rows per lane in n_pts. ms: the
 * kernel's device time (may be NULL).
 *
 * Lane shape (esl_set_mode): the warp lanes for FP64 when the run fits a
 * warp's share of shared memory, else (or with ESL_PATH_BLOCK, or with
 * ESL_PREC_MIXED) the block lanes, a CTA per lane. The block lanes stream
 * no measures and do not peel: a lane whose factor leaves the lead tape
 * stops with ESL_TRAN_LEFT_TAPE. Their mixed form refactors and solves in
 * FP32 and refines every Newton step in FP64 on the FP64 residual as the DC
 * block lanes do (refine_tol, refine_max, refine_skip); evaluation,
 * assembly, the companion, the Newton gates and the LTE control stay FP64
 * (esl_tran_refinements counts the corrections). */
int32_t esl_tran(esl_ctx *ctx, const esl_tran_opts *opts, const uint32_t *probes,
                 uint32_t n_probes, uint32_t max_pts, double *t_out, double *v_out,
                 uint32_t *n_pts, uint32_t *stats, double *x_out, float *ms);

/* esl_tran on device buffers (d_x, d_stats; the trace buffers may be NULL
 * when max_pts is 0). */
int32_t esl_tran_device(esl_ctx *ctx, const esl_tran_opts *opts, double *d_x, uint32_t *d_stats,
                        const uint32_t *d_probes, uint32_t n_probes, uint32_t max_pts,
                        double *d_t, double *d_v, uint32_t *d_n_pts, float *ms);

/* Streamed transient measures (.meas tran, src/output/measure.zig, a port
 * of ngspice com_measure2.c): every recorded row (t = 0 and each accepted
 * step) feeds each card. WHEN: the time of a clause's event; TRIG/TARG:
 * targ - trig (each clause with its own TD); FIND .. AT=: the value at a
 * time; MIN, MAX, AVG (trapezoidal mean) and PP of clause a's unknown over
 * its FROM..TO window (the samples inside it, ends not interpolated; MIN
 * and MAX read 0 when no sample falls inside, as the reference's do);
 * INTEG and RMS of clause a's unknown over FROM..TO with interpolated ends,
 * by Simpson's 3/8 rule, Simpson's rule or the trapezoid panel by panel as
 * the sample spacing allows (measure.zig Integ, ngspice
 * measure_rms_integral); DERIV .. AT=: the slope of the first segment
 * holding AT (measure.zig At with slope). A
 * clause: the probed unknown, the level VAL, RISE/FALL/CROSS counts
 * (ESL_MEAS_UNSET, ESL_MEAS_LAST or k >= 1), TD, FROM, TO (0: none), AT. An
 * event is counted from the clause's second sample and its time is the
 * level crossing interpolated on the last segment, as ngspice does. */
enum { ESL_MEAS_WHEN = 0, ESL_MEAS_TRIG_TARG = 1, ESL_MEAS_FIND_AT = 2,
       ESL_MEAS_MIN = 3, ESL_MEAS_MAX = 4, ESL_MEAS_AVG = 5, ESL_MEAS_PP = 6,
       ESL_MEAS_INTEG = 7, ESL_MEAS_RMS = 8, ESL_MEAS_DERIV = 9 };
enum { ESL_MEAS_UNSET = -1, ESL_MEAS_LAST = -2 };
typedef struct {
    uint32_t unknown;
    int32_t rise, fall, cross;
    double val, td, from, to, at;
} esl_meas_clause;
typedef struct {
    uint32_t kind, pad;
    esl_meas_clause a, b;  /* b: TRIG/TARG's target */
} esl_measure;
enum { ESL_TRAN_RESOLVED = 5 };

/* esl_tran_device (no trace) with up to 32 measure cards: d_values
 * [n_lanes][n_meas] the cards' values (NaN: unresolved). With early_stop a
 * lane ends its transient once every card has resolved (tran.zig:1057-1064,
 * `early_stop`), with status ESL_TRAN_RESOLVED. */
int32_t esl_tran_meas_device(esl_ctx *ctx, const esl_tran_opts *opts, const esl_measure *meas, uint32_t n_meas,
                             int early_stop, double *d_x, uint32_t *d_stats, double *d_values, float *ms);

/* Sequential .dc sweeps, one per lane (dc.zig Sweep :163-386; the
 * reference's `.dc` path, which the oracle's orc_dc_sweep restates): every
 * lane (its own parameters from esl_set_lanes) sweeps the DC value of one V
 * or I source (`slot`, parameter 0) through values[0 .. n_pts). Per point: the
 * MODEINITPRED predictor 2 last - prev, limited against the last point, a
 * warm Newton; on its failure, or before a point has converged, a cold start
 * with MODEINITFIX at 100 iterations (op.zig's plain rung). Device buffers:
 * d_x [n_lanes][n_pts][n], d_iters [n_lanes][n_pts] (both solves of a
 * point), d_conv [n_lanes][n_pts], d_status [n_lanes] (ESL_SWEEP_DONE). A
 * lane whose factor leaves the lead pivot tape pauses and takes the host's
 * factor on its own direct solver, then continues where it stopped, until
 * its own factor is the lead tape again (lane_solver.zig peels); the call
 * returns once every lane's sweep is done. ESL_NOT_ELIGIBLE for a slot that
 * is not a source's DC value. ms: the device time of the launches (may be
 * NULL). ESL_SWEEP_LEFT_TAPE is not returned since the peels. */
int32_t esl_dc_sweep_device(esl_ctx *ctx, const esl_slot *slot, const double *values, uint32_t n_pts,
                            const esl_newton_opts *opts, double *d_x, uint32_t *d_iters, uint8_t *d_conv,
                            uint32_t *d_status, float *ms);

/* Uneven batching: the DC solves of n_ctx contexts (circuits of any sizes,
 * one device) in one launch, each context's lanes with its own topology and
 * tape; per context its device buffers as esl_dc_solve_device takes them,
 * cold[c] (NULL: all warm) and stats[c] (may be NULL). Lanes that leave
 * their tape are served per context afterwards. No reference counterpart:
 * the reference's lanes run one topology per round (gpu_lanes.zig:349). */
int32_t esl_group_dc_solve_device(esl_ctx *const *ctxs, uint32_t n_ctx, const esl_newton_opts *opts,
                                  double *const *d_x, const int *cold, uint32_t *const *d_iters,
                                  uint32_t *const *d_status, esl_stats *stats);

/* Sets how the context's later DC solves (esl_dc_solve, esl_dc_solve_device)
 * run. */
int32_t esl_set_mode(esl_ctx *ctx, const esl_solve_mode *mode);

/* The block lanes' programs and working set for the context's tape (after
 * its first solve): rows of `width` ops in programs A (refactor + forward
 * solve, a_levels its longest dependence chain), B and F; the tape's
 * values and ops; per precision (0 FP64, 1 mixed) a lane's working-set
 * bytes in shared memory (all of it, or its hot part when split), whether
 * it sits in shared memory, CTAs per SM, and whether it is split (its
 * previous iterate and staging cells, cold_bytes, in global memory). */
typedef struct {
    uint32_t width, a_rows, b_rows, f_rows, a_levels, a_nops, b_nops, ntv, warp_ok;
    uint32_t lane_bytes[2], in_smem[2], ctas_per_sm[2], split[2], cold_bytes[2];
    uint32_t gather_terms, gather_cells; /* the assembly's terms and cells a thread walks */
} esl_block_info_t;
int32_t esl_block_info(esl_ctx *ctx, esl_block_info_t *info);

/* The SM cycles of the last block-lane solve by phase, summed over its
 * CTAs (each CTA's thread 0 reads clock64 between phases), when the mode
 * asked for a profile: cycles[0] device evaluation, [1] assembly, [2]
 * refactor + forward solve, [3] back solve and step, [4] mixed refinement,
 * [5] update, limiting and gates, [6] the Newton iterations counted. */
int32_t esl_block_profile(esl_ctx *ctx, uint64_t *cycles);

/* The peels of the context's last transient (esl_tran*, esl_tran_meas_device)
 * or sequential sweep (esl_dc_sweep_device) call: lanes that paused for a
 * host factor at least once, host factor + solve calls, and kernel launches
 * (the first and every resume). Any pointer may be NULL. */
int32_t esl_peel_counts(const esl_ctx *ctx, uint32_t *lanes, uint32_t *host_solves, uint32_t *launches);

/* The FP64 refinement corrections of the context's last transient call on
 * the block lanes in mixed precision, summed over its lanes (0 after an
 * FP64 or warp-lane transient). No counterpart in the reference, whose
 * lane solver is FP64 only. */
int32_t esl_tran_refinements(const esl_ctx *ctx, uint64_t *corrections);

/* Picks the context's lanes per CTA (1, 2, 4 or 8, as shared memory allows)
 * by timing its DC solve from x0 (NULL: cold) on its current lanes; keeps
 * the fastest for later launches and returns it in *lanes_per_block. */
int32_t esl_autotune(esl_ctx *ctx, const esl_newton_opts *opts, const double *x0,
                     uint32_t *lanes_per_block);

/* The lead lane's pivot tape after the last solve (buildTab,
 * lane_kernels.zig:321-345): q[n], pinv[n]; counts[0] = |L|, counts[1] = |U|,
 * counts[2] = refactor levels, counts[3] = solve levels. */
int32_t esl_tape(const esl_ctx *ctx, uint32_t *q, uint32_t *pinv, uint32_t *counts);

/* Standalone lane refactor + solve on the lead tape (arp_lane_refactor +
 * arp_lane_solve, lane_device.zig:26-38): device buffers a [n_lanes][nnz]
 * (pattern order), rhs [n_lanes][n] -> dx [n_lanes][n] = -A^-1 rhs and
 * bad [n_lanes] (1: pivot failure, growth, non-finite entry or a multiplier
 * past 1/pivot_tol: the lane must peel). tv [n_lanes][ntv] receives the
 * tape values (U, diagonal, L) when not NULL; ntv via esl_tape_size.
 * The tape is built from `lead` (host, nnz values) on the first call. */
int32_t esl_lu_replay_device(esl_ctx *ctx, const double *lead, uint32_t n_lanes,
                             const double *d_a, const double *d_rhs, double *d_dx,
                             uint8_t *d_bad, double *d_tv, float *ms);

/* esl_lu_replay_device on lane-interleaved planes, one thread per lane (the
 * reference's own layout: a [nnz][n_lanes], rhs and dx [n][n_lanes], tv
 * [ntv][n_lanes], lane_kernels.zig:49-143). Same results, bitwise; for lane
 * counts that fill the GPU many times over. ESL_NOT_ELIGIBLE when a warp's
 * 32 lanes of tape values exceed shared memory. */
int32_t esl_lu_lanes_device(esl_ctx *ctx, const double *lead, uint32_t n_lanes, const double *d_a,
                            const double *d_rhs, double *d_dx, uint8_t *d_bad, double *d_tv, float *ms);

/* esl_lu_lanes_device with the tape compiled into code: on its first call
 * the lead tape becomes one straight-line sm_100a kernel (each op one
 * statement on values held in registers, A and rhs read at first use, tape
 * values written to their plane as they become final and re-read from it
 * when next needed far off, dx written after its last update), built with
 * NVRTC and kept for the context's tape. With d_tv NULL a context-owned
 * plane stands in. Same arguments and results, bitwise;
 * ESL_NOT_ELIGIBLE when NVRTC is missing or the tape is too long to
 * compile (the interpreted esl_lu_lanes_device serves it). */
int32_t esl_lu_lanes_compiled_device(esl_ctx *ctx, const double *lead, uint32_t n_lanes,
                                     const double *d_a, const double *d_rhs, double *d_dx,
                                     uint8_t *d_bad, double *d_tv, float *ms);

/* Host-only: the CUDA source esl_lu_lanes_compiled_device compiles for the
 * tape of `lead` on this pattern (NUL-terminated in buf when cap > 0; *len
 * = its length without the NUL). resident: the register budget in values;
 * beyond it the final tape values needed farthest ahead are re-read from
 * their plane at their next use (0: the library's default, 48). */
int32_t esl_lu_compiled_source(uint32_t n, const uint32_t *col_ptr, const uint32_t *row_idx,
                               const double *lead, uint32_t resident, char *buf, size_t cap,
                               size_t *len);

/* esl_lu_lanes_mixed_device with the tape compiled into code (NVRTC, first
 * call): FP32 factors and solves in registers (an FP32 factor plane, owned
 * by the context, holds the values let go and serves the corrections), then
 * the same FP64 refinement on the residual -rhs - A dx until it falls below
 * 1e-12 of rhs, at most 6 corrections. Same arguments as
 * esl_lu_lanes_mixed_device; ESL_NOT_ELIGIBLE without NVRTC. */
int32_t esl_lu_lanes_mixed_compiled_device(esl_ctx *ctx, const double *lead, uint32_t n_lanes,
                                           const double *d_a, const double *d_rhs, double *d_dx,
                                           uint8_t *d_bad, uint8_t *d_refine, float *ms);

/* Host-only: the mixed form's CUDA source (as esl_lu_compiled_source). */
int32_t esl_lu_compiled_mixed_source(uint32_t n, const uint32_t *col_ptr, const uint32_t *row_idx,
                                     const double *lead, char *buf, size_t cap, size_t *len);

/* The compiler's log of the context's compiled LU (ptxas register and spill
 * lines), "" before the first esl_lu_lanes_compiled_device call. */
const char *esl_lu_compiled_log(const esl_ctx *ctx);

/* esl_lu_lanes_device in mixed precision: the refactor and the triangular
 * solves in FP32 on the same tape, then FP64 iterative refinement (residual
 * -rhs - A dx in FP64 from the FP64 planes, corrections solved on the FP32
 * factors) until the residual falls below 1e-12 of rhs, at most 6
 * corrections. dx [n][n_lanes] is FP64; refine [n_lanes] (may be NULL)
 * receives each lane's number of corrections; bad as the FP64 kernel's
 * tests, taken on the FP32 factors. */
int32_t esl_lu_lanes_mixed_device(esl_ctx *ctx, const double *lead, uint32_t n_lanes,
                                  const double *d_a, const double *d_rhs, double *d_dx,
                                  uint8_t *d_bad, uint8_t *d_refine, float *ms);

int32_t esl_tape_size(const esl_ctx *ctx, uint32_t *nu, uint32_t *nl, uint32_t *ntv);

/* Host-only symbolic stage (no device needed). */

/* The frozen CSC pattern of `circuit` (Circuit.freeze, Circuit.zig:77-167):
 * col_ptr [n + 1], row_idx [cap]; *nnz set even when cap is short. */
int32_t esl_pattern(const esl_circuit *circuit, uint32_t *col_ptr, uint32_t *row_idx,
                    size_t cap, uint32_t *nnz);

typedef struct {
    uint32_t nu, nl, ntv;        /* |U|, |L|, tape values (nu + n + nl + 1) */
    uint32_t n_fill;             /* tape values no pattern slot writes */
    uint32_t a_rows, a_levels, a_nops; /* program A (refactor + forward solve) */
    uint32_t b_rows, b_levels, b_nops; /* program B (back solve) */
    uint64_t flops;              /* refactor multiply-subtracts */
    uint32_t has_void;           /* a fabricated pivot (not run on the device) */
} esl_tape_info;

/* Orders the pattern (order.zig), factors `lead` with threshold pivoting
 * (sparse_lu.zig factor, pivot_tol 1e-3) and compiles the tape into the
 * warp programs the kernels run (buildTab's role, lane_kernels.zig:321-345):
 * rows of 32 ops, two u32 words per op, over v = [tape values | y]. Any
 * output array may be NULL; sizes come from info. */
int32_t esl_compile_tape(uint32_t n, const uint32_t *col_ptr, const uint32_t *row_idx,
                         const double *lead, esl_tape_info *info, uint32_t *q, uint32_t *pinv,
                         uint32_t *amap, uint32_t *fill, uint32_t *a_ops, uint32_t *b_ops,
                         uint8_t *l_scaled);

#ifdef __cplusplus
}
#endif
#endif
