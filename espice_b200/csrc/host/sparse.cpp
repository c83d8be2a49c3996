// See sparse.hpp. Reference semantics: src/solver/order.zig,
// src/solver/sparse_lu.zig:260-1224, src/solver/direct.zig:228-383.
#include "sparse.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>

namespace esl {

namespace {

uint64_t bits(double x) {
  uint64_t u;
  std::memcpy(&u, &x, 8);
  return u;
}
double from_bits(uint64_t u) {
  double x;
  std::memcpy(&x, &u, 8);
  return x;
}

// ---------------------------------------------------------------------------
// order.zig cholCount: |L| (diagonal included) of the symmetrized pattern
// eliminated in `perm`, by Liu's elimination tree with path compression.
uint64_t chol_count(uint32_t n, const std::vector<uint32_t>& cp, const std::vector<uint32_t>& ri,
                    const std::vector<uint32_t>& perm) {
  std::vector<uint32_t> pinv(n), ptr(n + 1, 0), lst(cp[n] ? cp[n] : 1), fill(n), parent(n);
  for (uint32_t k = 0; k < n; ++k) pinv[perm[k]] = k;
  for (uint32_t j = 0; j < n; ++j)
    for (uint32_t p = cp[j]; p < cp[j + 1]; ++p) {
      uint32_t a = pinv[ri[p]], b = pinv[j];
      if (a != b) ptr[std::max(a, b) + 1]++;
    }
  for (uint32_t k = 1; k <= n; ++k) ptr[k] += ptr[k - 1];
  std::copy(ptr.begin(), ptr.begin() + n, fill.begin());
  for (uint32_t j = 0; j < n; ++j)
    for (uint32_t p = cp[j]; p < cp[j + 1]; ++p) {
      uint32_t a = pinv[ri[p]], b = pinv[j];
      if (a == b) continue;
      lst[fill[std::max(a, b)]++] = std::min(a, b);
    }
  std::vector<uint32_t>& anc = fill;
  for (uint32_t k = 0; k < n; ++k) {
    parent[k] = kNone;
    anc[k] = kNone;
    for (uint32_t t = ptr[k]; t < ptr[k + 1]; ++t) {
      for (uint32_t i = lst[t]; i != kNone && i < k;) {
        uint32_t next = anc[i];
        anc[i] = k;
        if (next == kNone) parent[i] = k;
        i = next;
      }
    }
  }
  std::vector<uint32_t>& flag = anc;
  uint64_t count = 0;
  for (uint32_t k = 0; k < n; ++k) {
    flag[k] = k;
    ++count;
    for (uint32_t t = ptr[k]; t < ptr[k + 1]; ++t)
      for (uint32_t i = lst[t]; flag[i] != k; i = parent[i]) {
        flag[i] = k;
        ++count;
      }
  }
  return count;
}

// Approximate minimum degree on the symmetrized block pattern
// (order.zig amd): quotient graph, approximate external degrees, aggressive
// absorption, hashed supervariables, dense rows (degree >= max(16,
// 10 sqrt(n))) ordered last. Per-variable lists grow in place of the
// reference's slab compaction, which only moves spans and keeps their order.
class Amd {
 public:
  Amd(uint32_t n, const std::vector<uint32_t>& cp, const std::vector<uint32_t>& ri)
      : n_(n), cp_(cp), ri_(ri) {}

  std::vector<uint32_t> run() {
    const uint32_t n = n_;
    std::vector<uint32_t> q(n);
    if (n == 0) return q;
    va_.assign(4 * size_t(cp_[n]) + 4 * size_t(n) + 16, 0);
    ea_.assign(8 * size_t(n) + cp_[n], 0);
    va_pe_.assign(n, 0);
    va_len_.assign(n, 0);
    ea_pe_.assign(n, 0);
    ea_len_.assign(n, 0);
    ea_lim_.assign(n, 0);
    nv_.assign(n, 1);
    alive_.assign(n, 0);
    esize_.assign(n, 0);
    deg_.assign(n, 0);
    wbuf_.assign(n, 0);
    mark_.assign(n, 0);
    wmark_.assign(n, 0);
    hkey_.assign(n, 0);
    hhead_.assign(n, kNone);
    hnext_.assign(n, 0);
    mlink_.assign(n, kNone);
    head_.assign(n + 1, kNone);
    next_.assign(n, 0);
    prev_.assign(n, 0);
    std::vector<uint32_t> lp(n), touched(n), hbuckets(n);

    for (uint32_t j = 0; j < n; ++j)
      for (uint32_t p = cp_[j]; p < cp_[j + 1]; ++p)
        if (ri_[p] != j) {
          deg_[j]++;
          deg_[ri_[p]]++;
        }
    size_t va_free = 0;
    for (uint32_t i = 0; i < n; ++i) {
      va_pe_[i] = uint32_t(va_free);
      va_free += deg_[i];
    }
    std::fill(deg_.begin(), deg_.end(), 0u);
    for (uint32_t j = 0; j < n; ++j)
      for (uint32_t p = cp_[j]; p < cp_[j + 1]; ++p) {
        uint32_t r = ri_[p];
        if (r == j) continue;
        va_[va_pe_[j] + deg_[j]++] = r;
        va_[va_pe_[r] + deg_[r]++] = j;
      }
    va_len_ = deg_;
    for (uint32_t i = 0; i < n; ++i) {
      ++era_;
      uint32_t wp = 0;
      for (uint32_t t = 0; t < va_len_[i]; ++t) {
        uint32_t v = va_[va_pe_[i] + t];
        if (mark_[v] != era_) {
          mark_[v] = era_;
          va_[va_pe_[i] + wp++] = v;
        }
      }
      va_len_[i] = wp;
    }
    uint32_t isq = uint32_t(std::sqrt(double(n)));
    while (uint64_t(isq) * isq > n) --isq;
    while (uint64_t(isq + 1) * (isq + 1) <= n) ++isq;
    const uint32_t dense = std::max<uint32_t>(16, 10 * isq);
    uint32_t ndense = 0;
    for (uint32_t i = 0; i < n; ++i) ndense += va_len_[i] >= dense;
    const uint32_t dense_start = n - ndense;
    for (uint32_t i = 0, di = 0; i < n; ++i)
      if (va_len_[i] >= dense) {
        nv_[i] = 0;
        lp[dense_start + di++] = i;
      }
    if (ndense)
      for (uint32_t i = 0; i < n; ++i) {
        if (!nv_[i]) continue;
        uint32_t wp = 0;
        for (uint32_t t = 0; t < va_len_[i]; ++t) {
          uint32_t v = va_[va_pe_[i] + t];
          if (nv_[v]) va_[va_pe_[i] + wp++] = v;
        }
        va_len_[i] = wp;
      }
    size_t ea_free = 0;
    for (uint32_t i = 0; i < n; ++i) {
      ea_pe_[i] = uint32_t(ea_free);
      ea_lim_[i] = 4;
      ea_free += 4;
    }
    need(ea_, ea_free);
    for (uint32_t i = 0; i < n; ++i)
      if (nv_[i]) {
        deg_[i] = va_len_[i];
        insert(deg_[i], i);
      }

    const uint32_t n_amd = n - ndense;
    uint32_t mindeg = 0, k = 0;
    while (k < n_amd) {
      while (head_[mindeg] == kNone) ++mindeg;
      const uint32_t p = head_[mindeg];
      remove(deg_[p], p);
      ++era_;
      mark_[p] = era_;
      uint32_t nlp = 0;
      for (uint32_t t = 0; t < va_len_[p]; ++t) {
        uint32_t v = va_[va_pe_[p] + t];
        if (nv_[v] && mark_[v] != era_) {
          mark_[v] = era_;
          lp[nlp++] = v;
        }
      }
      for (uint32_t t = 0; t < ea_len_[p]; ++t) {
        uint32_t e = ea_[ea_pe_[p] + t];
        if (!alive_[e]) continue;
        for (uint32_t u = 0; u < va_len_[e]; ++u) {
          uint32_t v = va_[va_pe_[e] + u];
          if (nv_[v] && mark_[v] != era_) {
            mark_[v] = era_;
            lp[nlp++] = v;
          }
        }
        alive_[e] = 0;
      }
      const uint32_t nvpiv = nv_[p];
      nv_[p] = 0;
      alive_[p] = 1;
      need(va_, va_free + nlp);
      va_pe_[p] = uint32_t(va_free);
      va_len_[p] = nlp;
      std::copy(lp.begin(), lp.begin() + nlp, va_.begin() + va_free);
      va_free += nlp;
      uint32_t lpsize = 0;
      for (uint32_t t = 0; t < nlp; ++t) lpsize += nv_[lp[t]];
      esize_[p] = lpsize;
      for (uint32_t t = 0; t < nlp; ++t) remove(deg_[lp[t]], lp[t]);

      ++erw_;
      uint32_t ntouched = 0;
      for (uint32_t t = 0; t < nlp; ++t) {
        const uint32_t i = lp[t];
        for (uint32_t u = 0; u < ea_len_[i]; ++u) {
          uint32_t e = ea_[ea_pe_[i] + u];
          if (!alive_[e]) continue;
          if (wmark_[e] != erw_) {
            wmark_[e] = erw_;
            wbuf_[e] = esize_[e];
            touched[ntouched++] = e;
          }
          wbuf_[e] -= std::min(wbuf_[e], nv_[i]);
        }
      }
      for (uint32_t t = 0; t < ntouched; ++t)
        if (wbuf_[touched[t]] == 0) alive_[touched[t]] = 0;

      for (uint32_t t = 0; t < nlp; ++t) {
        const uint32_t i = lp[t];
        uint32_t esum = 0, ewp = 0;
        for (uint32_t u = 0; u < ea_len_[i]; ++u) {
          uint32_t e = ea_[ea_pe_[i] + u];
          if (alive_[e] && e != p) {
            ea_[ea_pe_[i] + ewp++] = e;
            esum += wbuf_[e];
          }
        }
        if (ewp < ea_lim_[i]) {
          ea_[ea_pe_[i] + ewp] = p;
        } else {
          const uint32_t nc = (ewp + 1) * 2;
          need(ea_, ea_free + nc);
          std::memmove(&ea_[ea_free], &ea_[ea_pe_[i]], sizeof(uint32_t) * ewp);
          ea_[ea_free + ewp] = p;
          ea_pe_[i] = uint32_t(ea_free);
          ea_lim_[i] = nc;
          ea_free += nc;
        }
        ea_len_[i] = ewp + 1;
        uint32_t asum = 0, vwp = 0;
        for (uint32_t u = 0; u < va_len_[i]; ++u) {
          uint32_t v = va_[va_pe_[i] + u];
          if (nv_[v] && mark_[v] != era_) {
            va_[va_pe_[i] + vwp++] = v;
            asum += nv_[v];
          }
        }
        va_len_[i] = vwp;
        const uint32_t cap = n_amd - k - nvpiv;
        deg_[i] = std::min(asum + (lpsize - nv_[i]) + esum, cap);
      }

      uint32_t nhb = 0;
      for (uint32_t t = 0; t < nlp; ++t) {
        const uint32_t i = lp[t];
        if (!nv_[i]) continue;
        uint32_t h = 0;
        for (uint32_t u = 0; u < va_len_[i]; ++u) h += va_[va_pe_[i] + u];
        for (uint32_t u = 0; u < ea_len_[i]; ++u) h += ea_[ea_pe_[i] + u];
        hkey_[i] = h;
        const uint32_t b = h % n;
        if (hhead_[b] == kNone) hbuckets[nhb++] = b;
        hnext_[i] = hhead_[b];
        hhead_[b] = i;
      }
      for (uint32_t t = 0; t < nhb; ++t) {
        const uint32_t b = hbuckets[t];
        for (uint32_t i = hhead_[b]; i != kNone; i = hnext_[i]) {
          if (!nv_[i]) continue;
          for (uint32_t j = hnext_[i]; j != kNone; j = hnext_[j]) {
            if (!nv_[j] || hkey_[j] != hkey_[i] || !same_adj(i, j)) continue;
            deg_[i] -= std::min(deg_[i], nv_[j]);
            nv_[i] += nv_[j];
            nv_[j] = 0;
            uint32_t tail = j;
            while (mlink_[tail] != kNone) tail = mlink_[tail];
            mlink_[tail] = mlink_[i];
            mlink_[i] = j;
          }
        }
        hhead_[b] = kNone;
      }
      for (uint32_t t = 0; t < nlp; ++t) {
        const uint32_t i = lp[t];
        if (!nv_[i]) continue;
        insert(deg_[i], i);
        mindeg = std::min(mindeg, deg_[i]);
      }
      q[k++] = p;
      for (uint32_t mb = mlink_[p]; mb != kNone; mb = mlink_[mb]) q[k++] = mb;
    }
    std::copy(lp.begin() + dense_start, lp.begin() + n, q.begin() + k);
    return q;
  }

 private:
  static void need(std::vector<uint32_t>& v, size_t size) {
    if (v.size() < size) v.resize(std::max(size, 2 * v.size()));
  }
  void insert(uint32_t d, uint32_t i) {
    next_[i] = head_[d];
    prev_[i] = kNone;
    if (head_[d] != kNone) prev_[head_[d]] = i;
    head_[d] = i;
  }
  void remove(uint32_t d, uint32_t i) {
    if (prev_[i] != kNone) next_[prev_[i]] = next_[i];
    else head_[d] = next_[i];
    if (next_[i] != kNone) prev_[next_[i]] = prev_[i];
  }
  bool same_adj(uint32_t i, uint32_t j) {
    if (va_len_[i] != va_len_[j] || ea_len_[i] != ea_len_[j]) return false;
    for (int pass = 0; pass < 2; ++pass) {
      const auto& adj = pass ? ea_ : va_;
      const auto& pe = pass ? ea_pe_ : va_pe_;
      const auto& len = pass ? ea_len_ : va_len_;
      const uint32_t m = ++era_;
      for (uint32_t t = 0; t < len[i]; ++t) mark_[adj[pe[i] + t]] = m;
      for (uint32_t t = 0; t < len[j]; ++t)
        if (mark_[adj[pe[j] + t]] != m) return false;
    }
    return true;
  }

  uint32_t n_;
  const std::vector<uint32_t>& cp_;
  const std::vector<uint32_t>& ri_;
  std::vector<uint32_t> va_, ea_, va_pe_, va_len_, ea_pe_, ea_len_, ea_lim_, nv_, alive_, esize_,
      deg_, wbuf_, mark_, wmark_, hkey_, hhead_, hnext_, mlink_, head_, next_, prev_;
  uint32_t era_ = 0, erw_ = 0;
};

}  // namespace

double norm_inf(const double* x, size_t n) {
  uint64_t m = 0;
  for (size_t i = 0; i < n; ++i) m = std::max(m, bits(std::fabs(x[i])));
  return from_bits(m);
}

uint32_t Csc::slot(uint32_t row, uint32_t col) const {
  if (row == 0 || col == 0) return nnz();
  auto b = row_idx.begin() + col_ptr[col], e = row_idx.begin() + col_ptr[col + 1];
  auto it = std::lower_bound(b, e, row);
  return (it != e && *it == row) ? uint32_t(it - row_idx.begin()) : nnz();
}

// op.zig gminStamps (:531-608): LoadGmin adds gmin to the diagonal that
// Sparse holds after spMNA_Preorder, which gives each branch-current column
// without a diagonal (its row's G and C both zero: no device here stamps a
// capacitance there, so G decides) the position of a +-1 twin: the column
// is exchanged with the row r whose entry (r, column) and transposed entry
// (column's position, column r) are both +-1, single twins first, then the
// first column with several. The ground row takes no load.
std::vector<uint32_t> gmin_stamps(const Csc& a, const std::vector<uint8_t>& cur_row, const double* g) {
  const uint32_t n = a.n, none = ~0u;
  std::vector<uint32_t> perm(n), dcol(n);
  for (uint32_t i = 0; i < n; ++i) {
    perm[i] = i;
    const uint32_t d = a.slot(i, i);
    const bool zero = d == a.nnz() || g[d] == 0.0;
    dcol[i] = (i != 0 && cur_row[i] && zero) ? none : i;
  }
  // the twins of column position j: how many (stopping at two) and the first
  auto twins = [&](uint32_t j, uint32_t& first) {
    uint32_t count = 0;
    const uint32_t col = perm[j];
    for (uint32_t p = a.col_ptr[col]; p < a.col_ptr[col + 1]; ++p) {
      const uint32_t r = a.row_idx[p];
      if (r == 0 || std::fabs(g[p]) != 1.0) continue;
      const uint32_t q = a.slot(j, perm[r]);
      if (q == a.nnz() || std::fabs(g[q]) != 1.0) continue;
      if (++count == 1)
        first = r;
      else
        break;
    }
    return count;
  };
  auto exchange = [&](uint32_t j, uint32_t r) {
    dcol[j] = perm[r];
    dcol[r] = perm[j];
    std::swap(perm[j], perm[r]);
  };
  uint32_t start = 1;
  for (;;) {
    bool swapped = false, again = false;
    for (uint32_t j = start; j < n; ++j) {
      if (dcol[j] != none) continue;
      uint32_t r = 0;
      const uint32_t t = twins(j, r);
      if (t == 1) {
        exchange(j, r);
        swapped = true;
      } else if (t > 1 && !again) {
        again = true;
        start = j;
      }
    }
    if (!again) break;
    for (uint32_t j = start; !swapped && j < n; ++j) {
      if (dcol[j] != none) continue;
      uint32_t r = 0;
      if (twins(j, r) > 0) {
        exchange(j, r);
        swapped = true;
      }
    }
    if (!swapped) break;
  }
  std::vector<uint32_t> out;
  for (uint32_t i = 1; i < n; ++i)
    if (dcol[i] != none) out.insert(out.end(), {a.slot(i, dcol[i]), i, dcol[i]});
  return out;
}

// order.zig order: Tarjan SCCs of j -> i for A(i, j) != 0 (sink block
// first), each non-singleton block in AMD or natural order, whichever gives
// the smaller Cholesky factor of the block's A + A^T.
std::vector<uint32_t> order_columns(const Csc& a) {
  const uint32_t n = a.n;
  const auto& cp = a.col_ptr;
  const auto& ri = a.row_idx;
  std::vector<uint32_t> q(n);
  if (n == 0) return q;
  std::vector<uint32_t> num(n, kNone), low(n), scc(n), fv(n), fp(n), emit(n), bptr(n + 1), blk(n), loc(n);
  std::vector<uint8_t> on(n, 0);
  uint32_t sp = 0, top = 0, counter = 0, no = 0, nb = 0;
  for (uint32_t root = 0; root < n; ++root) {
    if (num[root] != kNone) continue;
    num[root] = low[root] = counter++;
    scc[sp++] = root;
    on[root] = 1;
    fv[top] = root;
    fp[top++] = cp[root];
    while (top > 0) {
      const uint32_t v = fv[top - 1];
      if (fp[top - 1] < cp[v + 1]) {
        const uint32_t child = ri[fp[top - 1]++];
        if (child == v) continue;
        if (num[child] == kNone) {
          num[child] = low[child] = counter++;
          scc[sp++] = child;
          on[child] = 1;
          fv[top] = child;
          fp[top++] = cp[child];
        } else if (on[child]) {
          low[v] = std::min(low[v], num[child]);
        }
        continue;
      }
      if (low[v] == num[v]) {
        for (;;) {
          const uint32_t m = scc[--sp];
          on[m] = 0;
          emit[no++] = m;
          if (m == v) break;
        }
        bptr[++nb] = no;
      }
      if (--top > 0) low[fv[top - 1]] = std::min(low[fv[top - 1]], low[v]);
    }
  }
  for (uint32_t b = 0; b < nb; ++b)
    for (uint32_t i = bptr[b], li = 0; i < bptr[b + 1]; ++i, ++li) {
      blk[emit[i]] = b;
      loc[emit[i]] = li;
    }
  for (uint32_t b = 0; b < nb; ++b) {
    const uint32_t lo = bptr[b], bs = bptr[b + 1] - lo;
    const uint32_t* verts = emit.data() + lo;
    if (bs == 1) {
      q[lo] = verts[0];
      continue;
    }
    std::vector<uint32_t> scp(bs + 1, 0), sri;
    for (uint32_t j = 0; j < bs; ++j) {
      for (uint32_t p = cp[verts[j]]; p < cp[verts[j] + 1]; ++p)
        if (blk[ri[p]] == b) sri.push_back(loc[ri[p]]);
      scp[j + 1] = uint32_t(sri.size());
    }
    std::vector<uint32_t> sq = Amd(bs, scp, sri).run();
    std::vector<uint32_t> nat(verts, verts + bs);
    std::sort(nat.begin(), nat.end());
    for (auto& v : nat) v = loc[v];
    const auto& ord = chol_count(bs, scp, sri, nat) < chol_count(bs, scp, sri, sq) ? nat : sq;
    for (uint32_t i = 0; i < bs; ++i) q[lo + i] = verts[ord[i]];
  }
  return q;
}

// ---------------------------------------------------------------------------
// SparseLu

void SparseLu::init(const Csc* pattern, std::vector<uint32_t> order) {
  a = pattern;
  const uint32_t n = a->n;
  q = std::move(order);
  pinv.assign(n, kNone);
  lp.assign(n + 1, 0);
  up.assign(n + 1, 0);
  udiag.assign(n, 0);
  prow.assign(a->nnz(), 0);
  void_col.assign(n, 0);
  scaled.assign(n, 0);
  w_.assign(n, 0);
  y_.assign(n, 0);
  rscale_.assign(n, 0);
  want_.assign(n, 0);
  want_of_.assign(n, 0);
  prev_.assign(n, 0);
  flag_.assign(n, 0);
  topo_.assign(n, 0);
  stack_.assign(n, 0);
  pstack_.assign(n, 0);
  factored = false;
  base_lu = 0;
}

bool SparseLu::void_unknown(const double* vals, uint32_t c) const {
  if (pinv[c] != kNone) return false;
  const auto& cp = a->col_ptr;
  for (uint32_t p = cp[c]; p < cp[c + 1]; ++p)
    if (vals[p] != 0) return false;
  for (uint32_t j = 0; j < a->n; ++j) {
    if (j == c) continue;
    for (uint32_t p = cp[j]; p < cp[j + 1]; ++p)
      if (a->row_idx[p] == c && vals[p] != 0) return false;
  }
  return true;
}

// One full factor (sparse_lu.zig factorPass, plain column loop: the
// reference's supernodal copy of the loop skips only rows its DFS has
// marked and subtracts panel rows in step order, so it lays down the same
// pattern, pivots and values).
SparseLu::Pass SparseLu::factor_pass(const double* vals, double pivot_tol, size_t cap, bool keep_prev) {
  const uint32_t n = a->n;
  const auto& cp = a->col_ptr;
  const auto& ri = a->row_idx;
  factored = false;
  std::fill(pinv.begin(), pinv.end(), kNone);
  std::fill(flag_.begin(), flag_.end(), 0u);
  std::fill(void_col.begin(), void_col.end(), 0);
  std::fill(scaled.begin(), scaled.end(), 0);
  li.clear();
  lx.clear();
  ui.clear();
  ux.clear();
  void_slots.clear();
  bool has_void = false;
  std::fill(rscale_.begin(), rscale_.end(), 0.0);
  if (!(norm_inf(vals, a->nnz()) <= std::numeric_limits<double>::max())) return kSingular;
  for (uint32_t j = 0; j < n; ++j)
    for (uint32_t p = cp[j]; p < cp[j + 1]; ++p) rscale_[ri[p]] = std::fmax(rscale_[ri[p]], std::fabs(vals[p]));
  for (auto& s : rscale_) s = (s > 0 && std::isfinite(s)) ? 1 / s : 1;
  uint64_t nonfinite = 0;
  for (uint32_t i = 0; i < n; ++i) want_[i] = keep_prev ? prev_[i] : i;
  for (uint32_t c = 0; c < n; ++c) want_of_[want_[c]] = c;
  double* w = w_.data();

  for (uint32_t k = 0; k < n; ++k) {
    const uint32_t c = q[k];
    lp[k] = uint32_t(li.size());
    up[k] = uint32_t(ui.size());
    const uint32_t mark = k + 1;
    uint32_t nt = 0;
    // Reach of A[:, c] through the graph of L, in finish order.
    for (uint32_t p0 = cp[c]; p0 < cp[c + 1]; ++p0) {
      uint32_t r = ri[p0];
      if (flag_[r] == mark) continue;
      uint32_t sp = 0;
      stack_[0] = r;
      pstack_[0] = pinv[r] == kNone ? 0 : lp[pinv[r]];
      flag_[r] = mark;
      for (;;) {
        r = stack_[sp];
        const uint32_t kc = pinv[r];
        const uint32_t end = kc == kNone ? 0 : lp[kc + 1];
        uint32_t pos = pstack_[sp];
        bool descended = false;
        while (pos < end) {
          const uint32_t child = li[pos++];
          if (flag_[child] != mark) {
            pstack_[sp] = pos;
            flag_[child] = mark;
            stack_[++sp] = child;
            pstack_[sp] = pinv[child] == kNone ? 0 : lp[pinv[child]];
            descended = true;
            break;
          }
        }
        if (descended) continue;
        topo_[nt++] = r;
        if (sp == 0) break;
        --sp;
      }
    }
    for (uint32_t p = cp[c]; p < cp[c + 1]; ++p) w[ri[p]] = vals[p];
    // Sparse triangular solve in reverse finish order.
    for (uint32_t idx = nt; idx-- > 0;) {
      const uint32_t r = topo_[idx];
      const uint32_t kc = pinv[r];
      if (kc == kNone) continue;
      const double ukr = w[r];
      ui.push_back(kc);
      ux.push_back(ukr);
      for (uint32_t t = lp[kc]; t < lp[kc + 1]; ++t) w[li[t]] -= lx[t] * ukr;
    }
    double amax = 0, smax = 0;
    uint32_t piv = kNone;
    for (uint32_t t = 0; t < nt; ++t) {
      const uint32_t r = topo_[t];
      if (pinv[r] != kNone) continue;
      const double av = std::fabs(w[r]);
      if (av > amax) {
        amax = av;
        piv = r;
      }
      smax = std::fmax(smax, av * rscale_[r]);
    }
    if (piv == kNone || amax == 0 || !std::isfinite(amax)) {
      if (!void_unknown(vals, c)) {
        for (uint32_t t = 0; t < nt; ++t) w[topo_[t]] = 0;
        return kSingular;
      }
      void_col[k] = 1;
      has_void = true;
      udiag[k] = 1;
      pinv[c] = k;
      for (uint32_t t = 0; t < nt; ++t) w[topo_[t]] = 0;
      continue;
    }
    // Diagonal-preferred threshold pivot with the row-scaled second chance.
    const uint32_t pr = want_[c];
    if (pinv[pr] == kNone) {
      const double dmag = std::fabs(w[pr]);
      if (keep_prev) {
        if (dmag > 0 && dmag >= keep_min * amax) piv = pr;
      } else if (dmag > 0 && dmag >= pivot_tol * amax) {
        piv = pr;
      } else if (dmag > 0 && dmag * rscale_[pr] >= pivot_tol * smax) {
        piv = pr;
        scaled[k] = 1;
      }
    }
    if (piv != pr) {  // hand the row c gave up to the column that wanted piv
      const uint32_t c2 = want_of_[piv];
      want_[c2] = pr;
      want_of_[pr] = c2;
    }
    const double d = w[piv];
    udiag[k] = d;
    pinv[piv] = k;
    for (uint32_t t = 0; t < nt; ++t) {
      const uint32_t r = topo_[t];
      const double v = w[r];
      nonfinite |= bits(v - v);
      if (pinv[r] == kNone) {
        const double l = v / d;
        nonfinite |= bits(l - l);
        li.push_back(r);
        lx.push_back(l);
      }
      w[r] = 0;
    }
    if (li.size() + ui.size() > cap) return kCapped;
  }
  lp[n] = uint32_t(li.size());
  up[n] = uint32_t(ui.size());
  if (nonfinite) return kSingular;
  for (auto& r : li) r = pinv[r];
  for (uint32_t p = 0; p < a->nnz(); ++p) prow[p] = pinv[ri[p]];
  if (has_void)
    for (uint32_t j = 0; j < n; ++j)
      for (uint32_t p = cp[q[j]]; p < cp[q[j] + 1]; ++p)
        if (void_col[j] || void_col[prow[p]]) void_slots.push_back(p);
  ++epoch;
  factored = true;
  return kOk;
}

bool SparseLu::factor(const double* vals, double pivot_tol) {
  const bool repivot = factored && fill_cap > 0 && base_lu > 0;
  size_t cap = std::numeric_limits<size_t>::max();
  if (repivot) {
    for (uint32_t r = 0; r < a->n; ++r) prev_[q[pinv[r]]] = r;
    cap = size_t(std::fmin(fill_cap * double(base_lu), 1e18));
  }
  Pass rc = factor_pass(vals, pivot_tol, cap, false);
  if (rc == kCapped) rc = factor_pass(vals, pivot_tol, std::numeric_limits<size_t>::max(), true);
  if (rc != kOk) {
    factored = false;
    return false;
  }
  if (!repivot) base_lu = li.size() + ui.size();
  return true;
}

// sparse_lu.zig refactorColumns: the frozen pattern and pivot sequence on
// new values; false on a dead or non-finite pivot, growth below `growth`
// times the column max (scaled pivots excepted), a non-finite L/U entry, or
// a nonzero fabricated-pivot slot.
bool SparseLu::refactor(const double* vals, double growth) {
  for (uint32_t p : void_slots)
    if (vals[p] != 0) return false;
  const uint32_t n = a->n;
  const auto& cp = a->col_ptr;
  double* w = w_.data();
  uint64_t nonfinite = 0;
  for (uint32_t k = 0; k < n; ++k) {
    const uint32_t c = q[k];
    for (uint32_t p = cp[c]; p < cp[c + 1]; ++p) w[prow[p]] = vals[p];
    for (uint32_t p = up[k]; p < up[k + 1]; ++p) {
      const uint32_t i = ui[p];
      const double uki = w[i];
      w[i] = 0;
      ux[p] = uki;
      nonfinite |= bits(uki - uki);
      for (uint32_t t = lp[i]; t < lp[i + 1]; ++t) w[li[t]] -= lx[t] * uki;
    }
    if (void_col[k]) {
      udiag[k] = 1;
      for (uint32_t p = lp[k]; p < lp[k + 1]; ++p) {
        lx[p] = 0;
        w[li[p]] = 0;
      }
      w[k] = 0;
      for (uint32_t p = up[k]; p < up[k + 1]; ++p)
        for (uint32_t t = lp[ui[p]]; t < lp[ui[p] + 1]; ++t) w[li[t]] = 0;
      continue;
    }
    const double d = w[k];
    w[k] = 0;
    if (d == 0 || !std::isfinite(d)) {
      for (uint32_t p = lp[k]; p < lp[k + 1]; ++p) w[li[p]] = 0;
      return false;
    }
    udiag[k] = d;
    if (growth > 0 && !scaled[k]) {
      uint64_t cbits = bits(std::fabs(d));
      for (uint32_t p = lp[k]; p < lp[k + 1]; ++p) {
        const double v = w[li[p]];
        w[li[p]] = 0;
        cbits = std::max(cbits, bits(std::fabs(v)));
        lx[p] = v / d;
      }
      if (!(std::fabs(d) >= growth * from_bits(cbits))) return false;
    } else {
      for (uint32_t p = lp[k]; p < lp[k + 1]; ++p) {
        const double l = w[li[p]] / d;
        nonfinite |= bits(l - l);
        lx[p] = l;
        w[li[p]] = 0;
      }
    }
  }
  return nonfinite == 0;
}

void SparseLu::solve(const double* b, double* x) const {
  const uint32_t n = a->n;
  double* y = y_.data();
  for (uint32_t r = 0; r < n; ++r) y[pinv[r]] = b[r];
  for (uint32_t k = 0; k < n; ++k) {
    const double yk = y[k];
    if (yk == 0) continue;
    for (uint32_t p = lp[k]; p < lp[k + 1]; ++p) y[li[p]] -= lx[p] * yk;
  }
  for (uint32_t k = n; k-- > 0;) {
    const double zk = y[k] / udiag[k];
    y[k] = zk;
    if (zk == 0) continue;
    for (uint32_t p = up[k]; p < up[k + 1]; ++p) y[ui[p]] -= ux[p] * zk;
  }
  for (uint32_t j = 0; j < n; ++j) x[q[j]] = y[j];
}

void SparseLu::solve_t(const double* b, double* x) const {
  const uint32_t n = a->n;
  double* y = y_.data();
  for (uint32_t k = 0; k < n; ++k) y[k] = b[q[k]];
  for (uint32_t k = 0; k < n; ++k) {
    double yk = y[k];
    for (uint32_t p = up[k]; p < up[k + 1]; ++p) yk -= ux[p] * y[ui[p]];
    y[k] = yk / udiag[k];
  }
  for (uint32_t k = n; k-- > 0;) {
    double yk = y[k];
    for (uint32_t p = lp[k]; p < lp[k + 1]; ++p) yk -= lx[p] * y[li[p]];
    y[k] = yk;
  }
  for (uint32_t r = 0; r < n; ++r) x[r] = y[pinv[r]];
}

// lane_solver.zig sameTape: same ordering, pivots, L/U structure and flags.
bool SparseLu::same_tape(const SparseLu& o) const {
  return q == o.q && pinv == o.pinv && lp == o.lp && li == o.li && up == o.up && ui == o.ui &&
         void_col == o.void_col && scaled == o.scaled;
}

// ---------------------------------------------------------------------------
// DirectSolver

void DirectSolver::init(const Csc* pattern, std::vector<uint32_t> order) {
  lu.init(pattern, std::move(order));
  vcopy.assign(pattern->nnz(), 0.0);
  factored = false;
}

void DirectSolver::adopt(const SparseLu& lead, const double* vals) {
  lu = lead;
  // Without the last values no bypass can match: a NaN copy never equals.
  if (vals) vcopy.assign(vals, vals + lead.a->nnz());
  else vcopy.assign(lead.a->nnz(), std::numeric_limits<double>::quiet_NaN());
  factored = true;
}

// direct.zig maxMultiplier.
static double max_multiplier(const SparseLu& lu) {
  const double all = norm_inf(lu.lx.data(), lu.lx.size());
  bool any_scaled = false;
  for (auto s : lu.scaled) any_scaled |= s != 0;
  if (std::isnan(all) || !any_scaled) return all;
  double m = 0;
  for (uint32_t k = 0; k < lu.a->n; ++k)
    if (!lu.scaled[k]) m = std::fmax(m, norm_inf(lu.lx.data() + lu.lp[k], lu.lp[k + 1] - lu.lp[k]));
  return m;
}

// direct.zig replayHolds: a replay whose multipliers stay within
// 1/pivot_tol holds; otherwise Higham's alternating probe must solve both
// ways within replay_ratio_max / pivot_tol of LAWN 41's bar.
bool DirectSolver::replay_holds(const double* vals) {
  if (max_multiplier(lu) <= 1 / kPivotTol) return true;
  const uint32_t n = lu.a->n;
  const auto& cp = lu.a->col_ptr;
  const auto& ri = lu.a->row_idx;
  std::vector<double> x(n), r(n), rows(n, 0.0);
  double norm_1 = 0;
  for (uint32_t j = 0; j < n; ++j) {
    double col = 0;
    for (uint32_t p = cp[j]; p < cp[j + 1]; ++p) {
      rows[ri[p]] += std::fabs(vals[p]);
      col += std::fabs(vals[p]);
    }
    norm_1 = std::fmax(norm_1, col);
  }
  const double norm_infv = norm_inf(rows.data(), n);
  auto probe = [n](std::vector<double>& b) {
    const double den = double(std::max<uint32_t>(n, 2) - 1);
    for (uint32_t i = 0; i < n; ++i) {
      const double mag = 1 + double(i) / den;
      b[i] = i % 2 == 0 ? mag : -mag;
    }
  };
  for (int transpose = 0; transpose < 2; ++transpose) {
    probe(r);
    if (transpose) lu.solve_t(r.data(), x.data());
    else lu.solve(r.data(), x.data());
    probe(r);
    for (uint32_t j = 0; j < n; ++j)
      for (uint32_t p = cp[j]; p < cp[j + 1]; ++p) {
        if (transpose) r[j] -= vals[p] * x[ri[p]];
        else r[ri[p]] -= vals[p] * x[j];
      }
    const double anorm = transpose ? norm_1 : norm_infv;
    const double ratio = norm_inf(r.data(), n) / (anorm * norm_inf(x.data(), n) * double(n) * 2.220446049250313e-16);
    if (!(ratio <= kReplayRatioMax / kPivotTol)) return false;
  }
  return true;
}

// direct.zig Solver.factor: bypass on unchanged values, else refactor and
// keep it when replayHolds, else a full (re-)pivoting factor.
bool DirectSolver::factor(const double* vals) {
  const uint32_t nnz = lu.a->nnz();
  if (nnz && factored) {
    bool same = true;
    for (uint32_t p = 0; p < nnz && same; ++p) same = vcopy[p] == vals[p];
    if (same) {
      ++bypassed;
      return true;
    }
  }
  lu.fill_cap = kRepivotFillCap;
  lu.keep_min = kGrowthLimit;
  bool done = false;
  if (factored) {
    if (lu.refactor(vals, kGrowthLimit) && replay_holds(vals)) done = true;
    factored = false;
  }
  if (!done) {
    if (!lu.factor(vals, kPivotTol)) return false;
    ++full_factors;
  }
  factored = true;
  std::copy(vals, vals + nnz, vcopy.begin());
  return true;
}

void DirectSolver::solve_neg(const double* rhs, double* x) const {
  for (uint32_t i = 0; i < lu.a->n; ++i) x[i] = -rhs[i];
  lu.solve(x, x);
}

}  // namespace esl
