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

// Levels: an op runs after the last write of each value it reads, after
// the last write of its destination, and after every earlier read of its
// destination by another op (no value is overwritten before it is read).
// Each level is then packed into rows of kRow ops (one per thread) of one
// kind.
// Padding ops keep the row's kind and write the sink slot (space - 1) from
// the constants 1.0 (space - 2) and 0.0 (space - 3): a multiply-subtract of
// 1.0 * 0.0, or 1.0 / 1.0 (divisions read their dividend at b).
void pack(const std::vector<SeqOp>& seq, uint32_t space, std::vector<Op>& rows,
          std::vector<uint32_t>& kinds, uint32_t& n_rows, uint32_t& n_levels) {
  std::vector<int32_t> lw(space, -1), lr(space, -1), level(seq.size());
  int32_t top = -1;
  for (size_t i = 0; i < seq.size(); ++i) {
    const SeqOp& s = seq[i];
    int32_t l = std::max(lw[s.dst], lr[s.dst]) + 1;
    if (s.a != kNone) l = std::max(l, lw[s.a] + 1);
    if (s.b != kNone) l = std::max(l, lw[s.b] + 1);
    level[i] = l;
    lw[s.dst] = l;
    if (s.a != kNone) lr[s.a] = std::max(lr[s.a], l);
    if (s.b != kNone) lr[s.b] = std::max(lr[s.b], l);
    top = std::max(top, l);
  }
  n_levels = uint32_t(top + 1);
  std::vector<std::vector<uint32_t>> by(n_levels);
  for (size_t i = 0; i < seq.size(); ++i) by[level[i]].push_back(uint32_t(i));
  rows.clear();
  kinds.clear();
  n_rows = 0;
  for (auto& ids : by) {
    std::stable_sort(ids.begin(), ids.end(), [&](uint32_t x, uint32_t y) { return seq[x].kind < seq[y].kind; });
    for (size_t at = 0; at < ids.size();) {
      const uint32_t kind = seq[ids[at]].kind;
      size_t end = at;
      while (end < ids.size() && end - at < kRow && seq[ids[end]].kind == kind) ++end;
      for (uint32_t t = 0; t < kRow; ++t) {
        if (at + t < end) {
          const SeqOp& s = seq[ids[at + t]];
          rows.push_back(encode(s.kind, s.dst, s.a, s.b));
        } else {
          const bool div = kind == kOpDivGrowth || kind == kOpDivScaled || kind == kOpDivY;
          rows.push_back(encode(kind, space - 1, space - 2, div ? space - 2 : space - 3));
        }
      }
      kinds.push_back(kind);
      ++n_rows;
      at = end;
    }
  }
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
  pack(a, P.nv, P.a_ops, P.a_kind, P.a_rows, P.a_levels);
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
  pack(b, P.nv, P.b_ops, P.b_kind, P.b_rows, P.b_levels);
  P.b_nops = uint32_t(b.size());
  return P;
}

}  // namespace esl
