// Structures shared by the host runtime and the CUDA kernels of the
// sweep-lane library. Plain C++ (no CUDA types) so both compilers read it.
#pragma once

#include <cstdint>

namespace esl {

// Device types, numbered as the C ABI numbers them (include/espice_lanes.h).
enum DevType : uint32_t { kR = 0, kC = 1, kV = 2, kI = 3, kD = 4, kM = 5, kB3 = 6, kNumTypes = 7 };

constexpr int kMaxBatches = 8;

// Fixed per-type staging layout: the cells one instance's eval writes, in
// this order. The host's gather lists reference these positions.
//   R: f0 f1 J00 J01 J10 J11
//   C: q0 q1 C00 C01 C10 C11
//   V: f0 f1 f2 J02 J12 J20 J21
//   I: f0 f1
//   D: f0 f1 f2 J00 J02 J11 J12 J20 J21 J22 | q1 q2 C11 C12 C21 C22
//   M (local unknowns 0 d, 1 g, 2 s, 3 b, 4 di, 5 si):
//      f0 f2 f3 f4 f5 | J00 J04 J22 J25 J33 J34 J35 J40 J41 J43 J44 J45 J51 J52 J53 J54 J55
//      | q1 q3 q4 q5 | C11 C13 C14 C15 C31 C33 C34 C35 C41 C43 C44 C51 C53 C55
//   B3 (BSIM3 DC core, the MOS1 node set; the substrate current adds J31):
//      f0 f2 f3 f4 f5 | J00 J04 J22 J25 J31 J33 J34 J35 J40 J41 J43 J44 J45 J51 J52 J53 J54 J55
constexpr int kStageR = 6, kStageC = 6, kStageV = 7, kStageI = 2, kStageD = 16, kStageM = 40, kStageB3 = 23;
// A MOS1 batch without any charge keeps only the residual and Jacobian cells.
constexpr int kStageMNoQ = 22;

// Per-instance record fields (doubles, field-major per batch in a lane's
// record block). Diode fields follow the bias-independent part of
// models/diode.va.
enum DiodeField {
  kDVte, kDIs, kDVcrit, kDRs, kDGmin, kDBv, kDXbv, kDVtebrk, kDCjo, kDVj, kDMt, kDFc, kDTt,
  kDHasRs, kDHasQ, kDiodeFields
};
constexpr int kRFields = 1, kCFields = 1;
// V and I sources (models/vsource.va, isource.va): the parameters as given,
// one record field each: dc, wave (kWave*), the wave's eight parameters at
// kSrcShape (PULSE v1 v2 td tr tf pw per phase; SIN vo va freq td theta
// phase; EXP v1 v2 td1 tau1 td2 tau2; PWL len repeat td), then the PWL table,
// kPwlMax times at kSrcPwlT and values at kSrcPwlV.
enum SourceWave { kWaveDc = 0, kWavePulse = 1, kWaveSin = 2, kWaveExp = 3, kWavePwl = 4 };
constexpr int kPwlMax = 64;
constexpr int kSrcShape = 2, kSrcPwlT = 10, kSrcPwlV = kSrcPwlT + kPwlMax;
constexpr int kSrcParams = kSrcPwlV + kPwlMax;
constexpr int kVFields = kSrcParams, kIFields = kSrcParams;

// MOS1 record fields: the bias-independent part of models/mos1.va
// (temperature, geometry, junction sizing), in the type frame.
enum MosField {
  kMType, kMVt, kMVbit, kMGamma, kMPhit, kMBeta, kMLambda, kMIsats, kMIsatd, kMVcrits, kMVcritd,
  kMGdrain, kMGsource, kMCzbd, kMCzbs, kMCzbdsw, kMCzbssw, kMPbt, kMMj, kMMjsw, kMFc, kMF2d, kMF3d,
  kMF4d, kMF2s, kMF3s, kMF4s, kMCgs, kMCgd, kMCgb, kMGmin, kMHasQ, kMSeedVgs, kMosFields
};
constexpr int kMosParams = 34;
constexpr int kMParamRd = 6, kMParamRs = 7, kMParamTox = 19;

// BSIM3v3 record fields: the bias-independent part of models/bsim3.va
// (b3temp.c: temperature, geometry, parameter defaulting, junction sizing)
// and the card values the bias-dependent chain reads, in the type frame.
enum B3Field {
  kB3Type, kB3Mobmod, kB3Vt, kB3Tratio1, kB3Vth0i, kB3Isats, kB3Isatd, kB3Nvtmj, kB3Vjsm, kB3Isevjsm,
  kB3Vjdm, kB3Isevjdm, kB3Ijth, kB3Gmin, kB3Vbsc, kB3Phi, kB3Sqrtphi, kB3Phis3, kB3Xdep0, kB3Factor1,
  kB3Dvt2, kB3Dvt2w, kB3Dvt1, kB3Dvt1w, kB3Dvt0, kB3Dvt0w, kB3Leff, kB3Weff, kB3Vbi, kB3Nlx, kB3K1x,
  kB3K1ox, kB3K2ox, kB3Kt1, kB3Kt1l, kB3Kt2, kB3Tox, kB3W0, kB3K3, kB3K3b, kB3Eta0, kB3Etab,
  kB3Theta0vb0, kB3Nfactor, kB3Cdsc, kB3Cdscb, kB3Cdscd, kB3Cit, kB3Cox, kB3Vfbi, kB3Ngate, kB3Voff,
  kB3Cdep0, kB3Dwg, kB3Dwb, kB3Rds0, kB3Prwg, kB3Prwb, kB3Xj, kB3A0, kB3B0, kB3B1, kB3Ags, kB3Keta,
  kB3Ua, kB3Ub, kB3Uc, kB3U0temp, kB3Vsattemp, kB3A1, kB3A2, kB3Delta, kB3Pclm, kB3Litl,
  kB3Thetarout, kB3Pdiblcb, kB3Pvag, kB3Pscbe1, kB3Pscbe2, kB3Alpha0, kB3Alpha1, kB3Beta0, kB3M,
  kB3Gdrain, kB3Gsource, kB3Vt0, kB3Vcrit, kB3SeedVgs, kB3Fields
};
// Card slots (models/bsim3.va:26-138, then gmin and the temperature in K);
// NaN marks a parameter whose default the model derives ($param_given).
constexpr int kB3Params = 109;
constexpr int kB3ParamRsh = 95, kB3ParamNrd = 102, kB3ParamNrs = 103;

// Limited images per instance: a diode's junction voltage; a MOSFET's
// vgs, vds, vbs in the type frame.
constexpr uint32_t lim_count(uint32_t type) { return type == kD ? 1u : (type == kM || type == kB3) ? 3u : 0u; }

// Special gather sources beside staging positions.
constexpr uint32_t kSrcOne = 0xfffffffeu;    // + 1.0 (the ground pin on g)
constexpr uint32_t kSrcX0 = 0xfffffffdu;     // + x[0] (the ground pin on rhs)
constexpr uint32_t kNoDiag = 0xffffffffu;
constexpr uint32_t kGatherEnd = 0x80000000u;  // a segmented gather's cell ends at this segment
constexpr int kGatherBlock = 8;                // terms per pipelined block of the segmented gather

// One op of a warp program over a lane's shared-memory values v (the tape
// values, then the permuted right-hand side y). word0 = dst | (kind << 28);
// word1 = a | (b << 16).
enum OpKind : uint32_t {
  kOpFlop = 0,       // v[dst] -= v[a] * v[b]
  kOpDivGrowth = 1,  // v[dst] = v[b] / v[a]; peel unless |v[a]| >= growth * |v[b]|
  kOpDivScaled = 2,  // v[dst] = v[b] / v[a]; peel on a non-finite quotient
  kOpSubNz = 3,      // v[dst] -= v[a] * v[b] when v[b] != 0 (the solves' zero skip)
  kOpDivY = 4,       // v[dst] = v[b] / v[a]   (b = dst for a real op)
  kOpNop = 7,
};

// Per-lane transient statistics (the same fields, in the same order, as the
// oracle's step counters), and the run's status word.
enum TranStat : uint32_t {
  kTsStatus, kTsAccepted, kTsAttempts, kTsNrIters, kTsRejNewton, kTsRejLte, kTsBpLandings, kTsOpIters,
  kTsN
};
enum SweepStatus : uint32_t {
  kSweepDone = 0,      // every point ran (each point's convergence is its own flag)
  kSweepLeftTape = 4,  // a factor left the lead pivot tape: the rest of the sweep is the CPU's
};
// Streamed measure cards and clause counts (esl_measure).
enum MeasKind : uint32_t {
  kMeasWhen = 0, kMeasTrigTarg = 1, kMeasFindAt = 2, kMeasMin = 3, kMeasMax = 4, kMeasAvg = 5, kMeasPp = 6,
  kMeasInteg = 7, kMeasRms = 8, kMeasDeriv = 9
};
constexpr int32_t kMeasUnset = -1;
constexpr int32_t kMeasLast = -2;
constexpr uint32_t kMaxMeas = 32;  // one warp thread per card

enum TranStatus : uint32_t {
  kTranDone = 0,       // reached t_stop
  kTranUnderflow = 1,  // dt fell below dt_min
  kTranOpFailed = 2,   // the operating point did not converge
  kTranMaxSteps = 3,
  kTranLeftTape = 4,   // a factor left the lead pivot tape (needs a host factor)
  kTranResolved = 5,   // every measure card resolved and the run stopped early
};

// LTE charge states per instance: one per ddt() site kept in the
// truncation-error test (capacitor; diode junction; MOS1 qgs, qgd, qgb).
constexpr uint32_t qt_count(uint32_t type) { return type == kC ? 1u : type == kD ? 1u : type == kM ? 3u : 0u; }

struct LaneOpts {
  double reltol, abstol, vntol, residual_tol, gmin;
  uint32_t max_iter;
  uint32_t init_fix;
  uint32_t iter_cap;  // 0 or a hard cap below max_iter
  uint32_t ladder;    // 1: operating-point lanes, op.zig's ladder between Newton runs
  double gstamp;      // lane_newton: the gmin-stepping rung's gmin at the stamps (0: none)
};

// Lane status words (device -> host).
enum LaneStatus : uint32_t {
  kRunning = 0,
  kConverged = 1,
  kMaxIter = 2,
  kSingular = 3,
  kNeedSolve = 4,   // paused at the linear solve: the host factors this lane
};

}  // namespace esl
