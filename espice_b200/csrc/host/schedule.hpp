// Compiles the lead lane's pivot tape (a factored SparseLu) into the warp
// programs the kernels run. One value space per lane: the tape values (U
// entries, the diagonal, L entries, one discard slot, as the reference's
// refactor tape lays them out, sparse_lu.zig buildTape :1041-1082) followed
// by the n entries of the permuted right-hand side y.
//
// Program A is the refactor with the forward substitution through unit L
// merged in (a column's forward updates run as soon as its L entries and
// y entry are final, overlapping later columns' refactor); program B is the
// back substitution through U. Each is list-scheduled into rows of 32 ops,
// one op per thread of the lane's warp, padded with no-ops; a row holds
// divisions only or multiply-subtracts only, so the kernel's branch between
// the two is uniform across the warp.
#pragma once

#include <cstdint>
#include <vector>

#include "sparse.hpp"

namespace esl {

struct Op {
  uint32_t w0, w1;  // see common.h OpKind
};

struct Programs {
  uint32_t nu = 0, nl = 0, ntv = 0, n = 0;
  uint32_t nv = 0;                 // value space: ntv + n (y) + 0.0, 1.0, sink
  std::vector<uint32_t> amap;      // pattern slot -> tape value
  std::vector<uint32_t> fill;      // tape values no pattern slot writes
  std::vector<Op> a_ops;           // rows x 32: refactor + forward solve
  std::vector<Op> b_ops;           // rows x 32: back solve
  std::vector<Op> a_list, b_list;  // the same ops in the replay's sequential order (column by column)
  uint32_t a_rows = 0, b_rows = 0, a_levels = 0, b_levels = 0;  // levels: longest chain
  uint32_t a_nops = 0, b_nops = 0; // real ops (no padding)
  std::vector<uint8_t> l_scaled;   // per L entry: its column took the row-scaled pivot
  uint64_t flops = 0;              // refactor multiply-subtracts (the census F)
  bool has_void = false;
};

// Every op reads final operands and every value's updates keep their
// sequential order, so the programs are bitwise the column replay and the
// sparse triangular solves.
Programs compile_tape(const SparseLu& lu);

constexpr uint32_t kRow = 32;

}  // namespace esl
