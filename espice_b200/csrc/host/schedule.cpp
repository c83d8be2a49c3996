// See schedule.hpp.
#include "schedule.hpp"

#include <algorithm>

#include "../common.h"

namespace esl {

namespace {

struct SeqOp {
  uint32_t kind, dst, a, b;  // a, b: value sources (kNone when unused)
};

Op encode(uint32_t kind, uint32_t dst, uint32_t a, uint32_t b) {
  Op o;
  o.w0 = dst | (kind << 28);
  o.w1 = (a == kNone ? 0 : a) | ((b == kNone ? 0 : b) << 16);
  return o;
}

bool is_div(uint32_t kind) { return kind == kOpDivGrowth || kind == kOpDivScaled || kind == kOpDivY; }

// Dependences: an op follows the last write of each value it reads, the
// last write of its destination (a value's updates keep their sequential
// order, so every sum rounds as in the column replay), and every read of its
// destination since that write (no value is overwritten before it is read).
// The ops are then list-scheduled into rows of kRow ops (one per thread),
// each row one class, the divisions or the multiply-subtracts (the kernel's
// two warp-uniform paths; the checks inside a path are per op): row by row,
// the class of the ready op with the longest path to the end of the program,
// then up to kRow ready ops of that class, longest paths first. An op's
// successors become ready only for a later row. `n_levels` is the longest
// dependence chain, the least number of rows any packing can have.
// Padding ops write the sink slot (space - 1) from the constants 1.0
// (space - 2) and 0.0 (space - 3): 1.0 / 1.0 in a division row, a
// zero-skipped 1.0 * 0.0 in a multiply-subtract row.
template <class Enc, class OpT>
void pack_rows(const std::vector<SeqOp>& seq, uint32_t space, uint32_t width, Enc enc, const OpT& pad_div,
               const OpT& pad_flop, std::vector<OpT>& rows, uint32_t& n_rows, uint32_t& n_levels) {
  const size_t n = seq.size();
  std::vector<int32_t> last_write(space, -1);
  std::vector<std::vector<uint32_t>> readers(space);
  std::vector<uint32_t> succ_ptr(n + 1, 0), n_pred(n, 0);
  std::vector<std::pair<uint32_t, uint32_t>> edges;  // (pred, succ)
  std::vector<uint32_t> preds;
  for (size_t i = 0; i < n; ++i) {
    const SeqOp& s = seq[i];
    preds.clear();
    for (uint32_t src : {s.a, s.b})
      if (src != kNone && last_write[src] >= 0) preds.push_back(uint32_t(last_write[src]));
    if (last_write[s.dst] >= 0) preds.push_back(uint32_t(last_write[s.dst]));
    for (uint32_t r : readers[s.dst])
      if (r != i) preds.push_back(r);
    std::sort(preds.begin(), preds.end());
    preds.erase(std::unique(preds.begin(), preds.end()), preds.end());
    for (uint32_t p : preds) edges.push_back({p, uint32_t(i)});
    n_pred[i] = uint32_t(preds.size());
    last_write[s.dst] = int32_t(i);
    readers[s.dst].clear();
    for (uint32_t src : {s.a, s.b})
      if (src != kNone) readers[src].push_back(uint32_t(i));
  }
  for (const auto& e : edges) ++succ_ptr[e.first + 1];
  for (size_t i = 0; i < n; ++i) succ_ptr[i + 1] += succ_ptr[i];
  std::vector<uint32_t> succ(edges.size()), fill(succ_ptr.begin(), succ_ptr.end() - 1);
  for (const auto& e : edges) succ[fill[e.first]++] = e.second;
  // height: ops on the longest path from this op to the end, inclusive
  std::vector<uint32_t> height(n, 1);
  uint32_t top = 0;
  for (size_t i = n; i-- > 0;) {
    for (uint32_t e = succ_ptr[i]; e < succ_ptr[i + 1]; ++e) height[i] = std::max(height[i], height[succ[e]] + 1);
    top = std::max(top, height[i]);
  }
  n_levels = top;
  // ready queues per class, longest path first, then sequence order
  auto later = [&](uint32_t x, uint32_t y) { return height[x] != height[y] ? height[x] < height[y] : x > y; };
  std::vector<uint32_t> ready[2];
  for (size_t i = 0; i < n; ++i)
    if (n_pred[i] == 0) ready[is_div(seq[i].kind)].push_back(uint32_t(i));
  for (auto& q : ready) std::make_heap(q.begin(), q.end(), later);
  rows.clear();
  n_rows = 0;
  std::vector<uint32_t> row;
  while (!ready[0].empty() || !ready[1].empty()) {
    int c;
    if (ready[0].empty()) c = 1;
    else if (ready[1].empty()) c = 0;
    else c = later(ready[0].front(), ready[1].front()) ? 1 : 0;
    auto& q = ready[c];
    row.clear();
    while (!q.empty() && row.size() < width) {
      std::pop_heap(q.begin(), q.end(), later);
      row.push_back(q.back());
      q.pop_back();
    }
    for (uint32_t t = 0; t < width; ++t) {
      if (t < row.size()) rows.push_back(enc(seq[row[t]]));
      else rows.push_back(c ? pad_div : pad_flop);
    }
    ++n_rows;
    for (uint32_t i : row)
      for (uint32_t e = succ_ptr[i]; e < succ_ptr[i + 1]; ++e) {
        const uint32_t j = succ[e];
        if (--n_pred[j] == 0) {
          auto& qj = ready[is_div(seq[j].kind)];
          qj.push_back(j);
          std::push_heap(qj.begin(), qj.end(), later);
        }
      }
  }
}

void pack(const std::vector<SeqOp>& seq, uint32_t space, std::vector<Op>& rows, uint32_t& n_rows,
          uint32_t& n_levels) {
  auto enc = [](const SeqOp& s) { return encode(s.kind, s.dst, s.a, s.b); };
  pack_rows(seq, space, kRow, enc, encode(kOpDivY, space - 1, space - 2, space - 2),
            encode(kOpSubNz, space - 1, space - 2, space - 3), rows, n_rows, n_levels);
}

// Block-lane ops: 32-bit value indices, padding as no-ops.
Op4 encode4(const SeqOp& s) {
  return Op4{s.dst | (s.kind << 28), s.a == kNone ? 0u : s.a, s.b == kNone ? 0u : s.b, 0u};
}

}  // namespace

Programs compile_tape(const SparseLu& lu) {
  Programs P;
  const Csc& A = *lu.a;
  const uint32_t n = A.n;
  P.n = n;
  P.nu = uint32_t(lu.ui.size());
  P.nl = uint32_t(lu.li.size());
  const uint32_t lx0 = P.nu + n;
  const uint32_t discard = lx0 + P.nl;
  P.ntv = discard + 1;
  const uint32_t y0 = P.ntv;  // y[k] lives at y0 + k
  for (auto v : lu.void_col) P.has_void |= v != 0;

  // buildTape's slot map: per column k, its U rows, the diagonal, its L rows.
  std::vector<uint32_t> pos(n, kNone);
  P.amap.assign(A.nnz(), discard);
  std::vector<SeqOp> a;
  for (uint32_t k = 0; k < n; ++k) {
    const bool void_k = lu.void_col[k] != 0;
    for (uint32_t p = lu.up[k]; p < lu.up[k + 1]; ++p) pos[lu.ui[p]] = p;
    pos[k] = P.nu + k;
    for (uint32_t q = lu.lp[k]; q < lu.lp[k + 1]; ++q) pos[lu.li[q]] = lx0 + q;
    for (uint32_t p = lu.up[k]; p < lu.up[k + 1]; ++p) {
      const uint32_t i = lu.ui[p];
      for (uint32_t q = lu.lp[i]; q < lu.lp[i + 1]; ++q) {
        const uint32_t r = lu.li[q];
        a.push_back({kOpFlop, (void_k && r > k) ? discard : pos[r], lx0 + q, p});
        ++P.flops;
      }
    }
    const uint32_t c = lu.q[k];
    for (uint32_t e = A.col_ptr[c]; e < A.col_ptr[c + 1]; ++e) {
      const uint32_t r = lu.prow[e];
      P.amap[e] = (void_k && r > k) ? discard : pos[r];
    }
    const uint32_t div = lu.scaled[k] ? kOpDivScaled : kOpDivGrowth;
    for (uint32_t q = lu.lp[k]; q < lu.lp[k + 1]; ++q) a.push_back({div, lx0 + q, P.nu + k, lx0 + q});
    // Forward substitution of column k (sparse_lu.zig solve): y[li] -= l * y[k].
    for (uint32_t q = lu.lp[k]; q < lu.lp[k + 1]; ++q) a.push_back({kOpSubNz, y0 + lu.li[q], lx0 + q, y0 + k});
  }
  P.nv = P.ntv + n + 3;
  for (const SeqOp& s : a) {
    P.a_list.push_back(encode(s.kind, s.dst, s.a, s.b));
    P.a_seq.push_back(Op4{s.dst | (s.kind << 28), s.a == kNone ? 0u : s.a, s.b == kNone ? 0u : s.b, 0u});
  }
  if (P.nv < 65536) pack(a, P.nv, P.a_ops, P.a_rows, P.a_levels);
  P.a_nops = uint32_t(a.size());

  std::vector<uint8_t> written(P.ntv, 0);
  for (uint32_t e = 0; e < A.nnz(); ++e) written[P.amap[e]] = 1;
  for (uint32_t s = 0; s < P.ntv; ++s)
    if (!written[s]) P.fill.push_back(s);

  P.l_scaled.assign(P.nl, 0);
  for (uint32_t k = 0; k < n; ++k)
    for (uint32_t q = lu.lp[k]; q < lu.lp[k + 1]; ++q) P.l_scaled[q] = lu.scaled[k];

  // Back substitution through U: the diagonal division first in each column.
  std::vector<SeqOp> b;
  for (uint32_t k = n; k-- > 0;) {
    b.push_back({kOpDivY, y0 + k, P.nu + k, y0 + k});
    for (uint32_t p = lu.up[k]; p < lu.up[k + 1]; ++p) b.push_back({kOpSubNz, y0 + lu.ui[p], p, y0 + k});
  }
  for (const SeqOp& s : b) {
    P.b_list.push_back(encode(s.kind, s.dst, s.a, s.b));
    P.b_seq.push_back(Op4{s.dst | (s.kind << 28), s.a, s.b, 0u});
  }
  if (P.nv < 65536) pack(b, P.nv, P.b_ops, P.b_rows, P.b_levels);
  P.b_nops = uint32_t(b.size());
  return P;
}

}  // namespace esl

namespace esl {

namespace {

std::vector<SeqOp> unpack(const std::vector<Op4>& ops) {
  std::vector<SeqOp> out;
  out.reserve(ops.size());
  for (const Op4& o : ops) {
    const uint32_t kind = o.w0 >> 28;
    // a multiply-subtract reads a and b; a division reads a (divisor) and b
    out.push_back(SeqOp{kind, o.w0 & 0x0fffffffu, o.a, o.b});
  }
  return out;
}

}  // namespace

BlockPrograms compile_block(const Programs& P, uint32_t width) {
  BlockPrograms B;
  B.width = width;
  const Op4 nop{uint32_t(kOpNop) << 28, 0u, 0u, 0u};
  const std::vector<SeqOp> a = unpack(P.a_seq), b = unpack(P.b_seq);
  uint32_t lv = 0;
  pack_rows(a, P.nv, width, encode4, nop, nop, B.a_ops, B.a_rows, B.a_levels);
  pack_rows(b, P.nv, width, encode4, nop, nop, B.b_ops, B.b_rows, lv);
  // the forward substitution alone (program A's solve ops), for the mixed
  // form's refinement corrections on the finished factors
  std::vector<SeqOp> f;
  for (const SeqOp& s : a)
    if (s.kind == kOpSubNz) f.push_back(s);
  pack_rows(f, P.nv, width, encode4, nop, nop, B.f_ops, B.f_rows, lv);
  return B;
}

}  // namespace esl
