// Device-side tables of one topology and of a lane batch, passed to the
// kernels by value. A lane is one sweep point (or one Monte-Carlo sample):
// one warp owns it, and its working values live in shared memory for the
// whole Newton solve; the tables below are read-only and shared by every
// lane of the topology (broadcast through L1/L2).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../common.h"

namespace esl {

struct BatchDev {
  uint32_t type, count, nt;     // device type, instances, unknowns per instance
  uint32_t stage_base, stride;  // staging cells: stage_base + inst * stride
  uint32_t rec_off;             // record block offset (fields x count, field-major)
  uint32_t lim_off;             // limited images: lim_off + lim_count(type) * inst
  const uint32_t* nodes;        // count * nt unknown indices
  uint32_t qt_off, qt_sites;    // LTE charge states: qt_off + inst * qt_sites + k
  uint32_t src_off;             // V and I sources: the lane's cached value at src_off + inst
};

struct TopoDev {
  uint32_t n, nnz, nu, nl, ntv;   // unknowns, pattern, |U|, |L|, tape values (nu + n + nl + 1)
  uint32_t nv;                    // program value space: ntv + n (y) + 3 (0.0, 1.0, sink)
  uint32_t n_stage, nlim, rec_size;
  uint32_t n_batches;
  BatchDev b[kMaxBatches];
  // Residual gather: row i sums rhs_src[rhs_ptr[i] .. rhs_ptr[i + 1]).
  const uint32_t* rhs_ptr;
  const uint32_t* rhs_src;
  // Matrix gather: pattern slot p sums a_src[a_ptr[p] ..) into tape value
  // amap[p]; slot_row[p] = i when p is row i's diagonal.
  const uint32_t* a_ptr;
  const uint32_t* a_src;
  const uint32_t* amap;
  const uint32_t* slot_row;
  // Tape values no pattern slot writes (fill-in): zeroed per iteration.
  const uint32_t* fill;
  uint32_t n_fill;
  // The warp programs live in one 16-byte-aligned blob, staged into each
  // CTA's shared memory: A = refactor + forward solve and B = back solve,
  // rows of 32 ops over v = [tape values | y | 0.0 | 1.0 | sink], each row
  // divisions only or multiply-subtracts only (every op word carries its
  // kind); the assembly as one segmented gather: g_nseg segments of
  // kGatherBlock g_seg_blocks terms, thread t summing term k of its column at
  // src[k * 32 + t] (lane-block indices) and, at a segment's end where its
  // destination triple (dst[(3 s + i) * 32 + t]) carries kGatherEnd,
  // writing the sum to the first two places and its negation to the third
  // and starting over (residual rows, pattern slots into tape values, the
  // diagonal copy and y = P(-rhs); fill-in tape values sum +0.0); and the
  // transient companion's gather program in groups of 32 cells, cell t of
  // group g summing src[off[g] + k * 32 + t] for k < depth[g]: the rows with
  // charge cells (groups 0 .. n_kr_groups - 1; dst pair: the row, or kNone
  // on padding, and its y value), then the pattern slots with capacitance
  // cells (dst pair: the tape value, the diagonal copy or the sink).
  // Offsets in bytes.
  const unsigned char* prog;
  uint32_t prog_bytes;
  uint32_t o_a_ops, o_b_ops, o_g_src, o_g_dst;
  uint32_t a_rows, b_rows, g_nseg, g_seg_blocks;
  uint32_t o_k_depth, o_k_off, o_k_src, o_k_dst;
  uint32_t n_kr_groups, n_ks_groups;
  // L tape values whose column passed on the row-scaled test (no wide test).
  const uint8_t* l_scaled;
  // y[pinv[r]] = -rhs[r] before program A; dx[q[j]] = y[j] after program B.
  const uint32_t* pinv;
  const uint32_t* qcol;
  const uint8_t* cur_row;
  uint32_t smem_doubles;  // per lane
  // Transient planes: row i's charge sums q_src[q_ptr[i] ..), slot p's
  // capacitance sums c_src[c_ptr[p] ..) (staging cells, stamp order); the
  // LTE charge states number n_qt.
  const uint32_t* q_ptr;
  const uint32_t* q_src;
  const uint32_t* c_ptr;
  const uint32_t* c_src;
  uint32_t n_qt;
  uint32_t n_src;         // V and I source instances (the cached source values)
  uint32_t tran_doubles;  // per lane, transient kernel
  // The pattern by rows (the refinement's residual): row i's entries
  // row_ptr[i] .. row_ptr[i + 1], each its pattern slot and column.
  const uint32_t* row_ptr;
  const uint32_t* row_slot;
  const uint32_t* row_col;
  // The gmin-stepping rung's loads (op.zig gminStamps): n_gst triples
  // (pattern slot, row, column); gmin goes on the slot and gmin x[column]
  // on the row's residual.
  const uint32_t* gst;
  uint32_t n_gst;
};

// One transient over every lane (tran.zig Sim): options, the probe trace
// and the per-lane step statistics.
// A streamed transient measure card (esl_measure's layout): WHEN, TRIG/TARG
// or FIND AT over clauses of one probed unknown each.
struct MeasClauseDev {
  uint32_t unknown;
  int32_t rise, fall, cross;  // -1 unset, -2 LAST, else the event count
  double val, td, from, to, at;
};
struct MeasDev {
  uint32_t kind, pad;
  MeasClauseDev a, b;
};
// One clause's scan state (measure.zig Cross / At), in the lane's shared
// memory: kMeasDoubles per card (two clauses).
struct CrossDev {
  double td, prev, prev_x, last, hit;
  int32_t want_rise, want_fall, want_cross;
  int32_t rise, fall, cross;
  uint32_t first;
  int32_t above, pending, found, over;
  int32_t pad;
};
constexpr uint32_t kMeasDoubles = 2 * sizeof(CrossDev) / sizeof(double);
// INTEG and RMS (measure.zig Integ) in the same card state: the window's
// points not folded into a panel yet, the three rules' sums, the last raw
// sample and the window's ends.
struct IntegDev {
  double p[4][2];
  double sum[3];
  double px, py, first_x, cut_x;
  uint32_t rows, np, count, inside, cut, over;
};
static_assert(sizeof(IntegDev) <= 2 * sizeof(CrossDev), "a card's state holds INTEG");

struct TranDev {
  double t_stop, t_step, dt_max, dt_min;
  double reltol, abstol, vntol, chgtol, trtol;
  uint32_t max_steps;
  uint32_t n_probes, max_pts;
  const uint32_t* probes;  // [n_probes] unknowns recorded
  double* out_t;           // [lane][max_pts] accepted times (null: no trace)
  double* out_v;           // [lane][max_pts][n_probes]
  uint32_t* n_pts;         // [lane] rows recorded
  uint32_t* stats;         // [lane][kTsN]
  const MeasDev* meas;     // [n_meas] cards fed every recorded row (null: none)
  uint32_t n_meas, early_stop;
  double* meas_out;        // [lane][n_meas] card values (NaN: unresolved)
  uint32_t* next_lane;     // the lane-refill counter, zero at launch
  // A lane paused for a host factor (LaneDev's pause protocol): its state
  // words [lane][kTranStateN] and its shared memory and double state
  // [lane][tran_doubles + kMeasDoubles n_meas + kTranSaveRegs].
  uint32_t* tstate;
  double* tsave;
};
// A paused transient lane's state words.
enum TranStateWord : uint32_t {
  kTrPhase = 0,      // 1 paused in the operating point, 2 in a step
  kTrIter = 1,       // the Newton iteration it paused in
  kTrInitFix = 2,
  kTrOrder = 3,
  kTrSteps = 4,
  kTrHaveBp = 5,
  kTrBpClamped = 6,
  kTrHb = 7,         // the charge rings' base slot
  kTrNRec = 8,       // rows recorded
  kTrLimActive = 9,
  kTrStat = 10,      // kTsN step statistics
  kTranStateN = 10 + kTsN
};
constexpr uint32_t kTranSaveRegs = 10;  // t, dt, the breakpoint and its saved step, six past steps

// Sequential .dc sweeps, one per lane (dc.zig Sweep): the swept source
// (its index among the V and I sources' cached values) takes values[pt] at
// point pt; per lane and point the solution, the Newton iterations and
// whether it converged; per lane a status (kSweepDone, kSweepLeftTape).
struct SweepDev {
  const double* values;  // [n_pts]
  uint32_t n_pts;
  uint32_t src;
  double* x_out;     // [lane][n_pts][n]
  uint32_t* iters;   // [lane][n_pts]
  uint8_t* conv;     // [lane][n_pts]
  uint32_t* status;  // [lane]
  uint32_t* next_lane;  // the lane-refill counter, zero at launch
  // A lane paused for a host factor (LaneDev's pause protocol): where its
  // sweep stands, [lane][kSweepStateN] words, and its predictor rows, the
  // last solution and the one before, [lane][2 n].
  uint32_t* state;
  double* rows;
};

// A paused sweep lane's state words.
enum SweepStateWord : uint32_t {
  kSwPoint, kSwPhase, kSwItTotal, kSwCold, kSwIter, kSwInitFix, kSwLimActive, kSweepStateN
};

// A Newton solve's loop state across a pause (sweep lanes): the iteration
// reached, the runaway bound, the INITFIX flag; on resume, whether the
// host's step (in y, permuted) or its singular verdict stands for the
// iteration, and whether every factor of the lane is the host's.
struct NewtonCarry {
  uint32_t iter;
  double limit;
  uint32_t init_fix;
  uint32_t resume;     // 0 none, 1 the host's step, 2 the host's factor was singular
  uint32_t host_mode;  // the lane's factor left the lead tape: pause before every factor
};

// Shared-memory doubles per lane of sweep_kernel: the lane working set,
// then the sweep's solution and previous point, then the cached sources.
__host__ __device__ inline uint32_t sweep_doubles(const TopoDev& T) {
  return (T.smem_doubles + 2 * T.n + T.n_src + 1) & ~1u;
}

// An operating-point lane's place on op.zig's ladder (solveLadder /
// afterPlain), in global memory across Newton runs and pauses: the rung of
// the run in flight, the runs of the stepping loop, the iterations summed
// over every run, and the stepping state (the gmin descent and the source
// factor with their last good values).
struct LadderDev {
  uint32_t rung;       // LadderRung of the run in flight
  uint32_t solves;     // runs of the current stepping loop
  uint32_t total;      // iterations over every run, saturating at 65535
  uint32_t have_good;  // the gmin loop has a converged point in x_good
  double factor, good_gmin, gmin_val;
  double lambda, lambda_good, delta;
};
enum LadderRung : uint32_t {
  kRungPlain = 0,   // rung 1: plain Newton from the cold start (MODEINITFIX)
  kRungGmin = 1,    // rung 2: a gmin-stepping run
  kRungClean = 2,   // rung 2's last run, without the shunt
  kRungSource = 3,  // rung 3: a source-stepping run
  kRungFinal = 4,   // the full-source Newton after rung 3
  kRungDone = 5
};

struct LaneDev {
  uint32_t n_lanes;
  uint32_t resume;        // 1: lanes paused at the solve take the host's dx
  const double* rec;      // [lane][rec_size]
  double* x;              // [lane][n]: start in, solution out
  double* lim;            // [lane][nlim]
  uint32_t* lim_active;   // [lane]
  uint32_t* status;       // [lane] LaneStatus
  uint32_t* iters;        // [lane]
  uint32_t* flags;        // [lane] bit 0 INITFIX pending, bit 1 every solve on the host,
                          // bit 2 the lane's solver factored in an earlier run
  double* limit;          // [lane] runaway bound of this solve
  double* xo;             // [lane][n]  (pause state)
  double* a_vals;         // [lane][nnz] (pause: matrix for the host factor)
  double* rhs;            // [lane][n]   (pause: residual; resume: gate input)
  double* dx;             // [lane][n]   (resume: the host's step)
  double* diag;           // [lane][n]   (pause: assembled diagonal for the gate)
  uint32_t* n_paused;     // device counter
  LadderDev* ladder;      // [lane] operating-point lanes: the ladder's state
  double* x_good;         // [lane][n] its last converged stepping point
  uint32_t* rung_out;     // [lane] the rung that converged (0 plain, 1 gmin, 2 source; 3 none)
};

}  // namespace esl
