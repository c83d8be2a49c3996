// Host-side sparse machinery of the sweep-lane library: the frozen CSC
// pattern, BTF + AMD column ordering, the threshold-pivoting Gilbert-Peierls
// factor that lays down the lead lane's pivot tape, the numeric refactor on a
// frozen tape, and the per-lane direct-solver policy a peeled lane runs on.
//
// Semantics follow the reference's CPU solver:
//   src/solver/order.zig            (BTF by Tarjan, AMD per block, natural fallback)
//   src/solver/sparse_lu.zig:260-1224 (factor, refactor, solve, solveT)
//   src/solver/direct.zig:228-383   (bypass, refactor + replayHolds, re-pivot)
// All arithmetic is compiled without FMA contraction so a host peel is
// bitwise the device replay and the reference's strict-float code.
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

namespace esl {

constexpr uint32_t kNone = 0xffffffffu;
constexpr double kPivotTol = 1e-3;        // direct.zig:32
constexpr double kRepivotFillCap = 3.0;   // direct.zig:35
constexpr double kGrowthLimit = 1e-12;    // direct.zig:53
constexpr double kReplayRatioMax = 30.0;  // direct.zig:542

struct Csc {
  uint32_t n = 0;
  std::vector<uint32_t> col_ptr, row_idx;
  uint32_t nnz() const { return col_ptr.empty() ? 0 : col_ptr[n]; }
  // CSC slot of (row, col); nnz (the trash slot) when absent or on ground.
  uint32_t slot(uint32_t row, uint32_t col) const;
};

// Column order q[k] = column eliminated at step k (order.zig `order`).
std::vector<uint32_t> order_columns(const Csc& a);

// The gmin-stepping rung's loads (op.zig gminStamps): (slot, row, column)
// triples for rows 1 .. n-1 after ngspice's spMNA_Preorder, from the
// pattern, the current-row flags and an assembled G.
std::vector<uint32_t> gmin_stamps(const Csc& a, const std::vector<uint8_t>& cur_row, const double* g);

// One sparse LU (sparse_lu.zig SparseLu). L row indices are pivot steps once
// a factor returns; U columns keep the order the triangular solve visited.
struct SparseLu {
  const Csc* a = nullptr;
  std::vector<uint32_t> q, pinv, lp, li, up, ui, prow, void_slots;
  std::vector<double> lx, ux, udiag;
  std::vector<uint8_t> void_col, scaled;
  size_t base_lu = 0;
  double fill_cap = 0, keep_min = 0;
  bool factored = false;
  uint32_t epoch = 0;

  void init(const Csc* pattern, std::vector<uint32_t> order);
  bool factor(const double* vals, double pivot_tol);     // false: singular
  bool refactor(const double* vals, double growth);      // false: singular
  void solve(const double* b, double* x) const;          // x may alias b
  void solve_t(const double* b, double* x) const;
  bool same_tape(const SparseLu& o) const;

 private:
  enum Pass { kOk, kSingular, kCapped };
  Pass factor_pass(const double* vals, double pivot_tol, size_t cap, bool keep_prev);
  bool void_unknown(const double* vals, uint32_t c) const;
  std::vector<double> w_, rscale_;
  mutable std::vector<double> y_;
  std::vector<uint32_t> want_, want_of_, prev_, flag_, topo_, stack_, pstack_;
};

// One lane's own direct solver (direct.zig Solver on the general LU).
struct DirectSolver {
  SparseLu lu;
  std::vector<double> vcopy;
  bool factored = false;
  uint32_t full_factors = 0, bypassed = 0;

  void init(const Csc* pattern, std::vector<uint32_t> order);
  // Adopts an already factored lead LU (its tape and values) as this lane's
  // last factor of `vals`.
  void adopt(const SparseLu& lead, const double* vals);
  bool factor(const double* vals);                        // false: singular
  void solve_neg(const double* rhs, double* x) const;

 private:
  bool replay_holds(const double* vals);
};

// num.normInf: max |x_i| by bit pattern, NaN winning.
double norm_inf(const double* x, size_t n);

}  // namespace esl
