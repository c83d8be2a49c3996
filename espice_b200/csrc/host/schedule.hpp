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

// A block-lane op: w0 = dst | (kind << 28), then the two sources as full
// 32-bit value indices (any tape size), 16 bytes for one vector load.
struct Op4 {
  uint32_t w0, a, b, pad;
};

struct Programs {
  uint32_t nu = 0, nl = 0, ntv = 0, n = 0;
  uint32_t nv = 0;                 // value space: ntv + n (y) + 0.0, 1.0, sink
  std::vector<uint32_t> amap;      // pattern slot -> tape value
  std::vector<uint32_t> fill;      // tape values no pattern slot writes
  std::vector<Op> a_ops;           // rows x 32: refactor + forward solve
  std::vector<Op> b_ops;           // rows x 32: back solve
  std::vector<Op> a_list, b_list;  // the same ops in the replay's sequential order (column by column)
  std::vector<Op4> a_seq, b_seq;   // the same, with 32-bit indices (any value space)
  uint32_t a_rows = 0, b_rows = 0, a_levels = 0, b_levels = 0;  // levels: longest chain
  uint32_t a_nops = 0, b_nops = 0; // real ops (no padding)
  std::vector<uint8_t> l_scaled;   // per L entry: its column took the row-scaled pivot
  uint64_t flops = 0;              // refactor multiply-subtracts (the census F)
  bool has_void = false;
};

// The programs of a block lane: the same dependences list-scheduled into
// rows of `width` ops (one per thread of the lane's CTA, a barrier between
// rows), padding as no-ops, plus program F, the forward substitution alone
// (the mixed form's refinement solves on finished factors).
struct BlockPrograms {
  uint32_t width = 0;  // ops a row: row_k * the CTA's threads
  uint32_t row_k = 1;  // ops a thread a row
  std::vector<Op4> a_ops, b_ops, f_ops;
  uint32_t a_rows = 0, b_rows = 0, f_rows = 0, a_levels = 0;
};

// Every op reads final operands and every value's updates keep their
// sequential order, so the programs are bitwise the column replay and the
// sparse triangular solves.
Programs compile_tape(const SparseLu& lu);

// Rows of `width` for the block lanes (the warp programs, a_ops and b_ops,
// exist only when the value space fits 16-bit indices: nv < 65536).
BlockPrograms compile_block(const Programs& P, uint32_t width);

constexpr uint32_t kRow = 32;

}  // namespace esl
