// C ABI of the sweep-lane library (include/espice_lanes.h): the host half
// of the reference's GpuLanes (src/analysis/gpu_lanes.zig:349-1027) for DC
// sweep lanes. It freezes the pattern, orders it, builds the stamp gather
// tables, factors the lead lane's first Jacobian into the pivot tape,
// compiles that tape into warp programs, and runs the fused Newton kernel;
// lanes the frozen tape cannot stand in for pause and take a host factor
// on their own direct solver (lane_solver.zig:76-131), then resume.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <thread>
#include <limits>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../../include/espice_lanes.h"
#include "../kernels/block.h"
#include "../kernels/launch.h"
#include "../kernels/derive.h"
#include "lu_jit.hpp"
#include "records.hpp"
#include "schedule.hpp"
#include "sparse.hpp"

using namespace esl;

namespace {

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  cudaError_t ensure(size_t b) {
    if (b <= bytes && p) return cudaSuccess;
    release();
    bytes = b ? b : 8;
    return cudaMalloc(&p, bytes);
  }
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

struct HostBatch {
  uint32_t type = 0, count = 0, nt = 0, np = 0;
  uint32_t stage_base = 0, stride = 0, rec_off = 0, nfields = 0, lim_off = 0;
  uint32_t qt_off = 0, qt_sites = 0;
  std::vector<uint32_t> nodes;
  std::vector<double> params;
};

uint32_t stage_stride(uint32_t type) {
  switch (type) {
    case kR: return kStageR;
    case kC: return kStageC;
    case kV: return kStageV;
    case kI: return kStageI;
    case kD: return kStageD;
    case kM: return kStageM;
    case kB3: return kStageB3;
    default: return 0;
  }
}

// The cells one instance writes, in stamp order: its residual rows (local
// row, staging position) and its Jacobian entries (local row, local column,
// staging position), as src/device/eval.zig:864-895 orders them. Charge
// entries are the transient planes' and are not gathered for DC.
struct Entry {
  uint8_t ru, cu, pos;
};
struct InstLayout {
  std::vector<Entry> res, jac, q, qjac;
};

InstLayout layout_of(uint32_t type, const double* prm) {
  InstLayout L;
  switch (type) {
    case kR:
      L.res = {{0, 0, 0}, {1, 0, 1}};
      L.jac = {{0, 0, 2}, {0, 1, 3}, {1, 0, 4}, {1, 1, 5}};
      break;
    case kC:
      L.q = {{0, 0, 0}, {1, 0, 1}};
      L.qjac = {{0, 0, 2}, {0, 1, 3}, {1, 0, 4}, {1, 1, 5}};
      break;
    case kV:
      L.res = {{0, 0, 0}, {1, 0, 1}, {2, 0, 2}};
      L.jac = {{0, 2, 3}, {1, 2, 4}, {2, 0, 5}, {2, 1, 6}};
      break;
    case kI:
      L.res = {{0, 0, 0}, {1, 0, 1}};
      break;
    case kD: {
      const bool rs = prm[2] > 0;
      if (rs) L.res.push_back({0, 0, 0});
      L.res.push_back({1, 0, 1});
      L.res.push_back({2, 0, 2});
      if (rs) {
        L.jac.push_back({0, 0, 3});
        L.jac.push_back({0, 2, 4});
      }
      L.jac.push_back({1, 1, 5});
      L.jac.push_back({1, 2, 6});
      if (rs) L.jac.push_back({2, 0, 7});
      L.jac.push_back({2, 1, 8});
      L.jac.push_back({2, 2, 9});
      if (prm[5] > 0 || prm[9] > 0) {
        L.q = {{1, 0, 10}, {2, 0, 11}};
        L.qjac = {{1, 1, 12}, {1, 2, 13}, {2, 1, 14}, {2, 2, 15}};
      }
      break;
    }
    case kM: {  // d g s b di si (models/mos1.va contributions)
      const bool rd = prm[kMParamRd] > 0, rs = prm[kMParamRs] > 0;
      if (rd) L.res.push_back({0, 0, 0});
      if (rs) L.res.push_back({2, 0, 1});
      L.res.push_back({3, 0, 2});
      L.res.push_back({4, 0, 3});
      L.res.push_back({5, 0, 4});
      if (rd) {
        L.jac.push_back({0, 0, 5});
        L.jac.push_back({0, 4, 6});
      }
      if (rs) {
        L.jac.push_back({2, 2, 7});
        L.jac.push_back({2, 5, 8});
      }
      L.jac.push_back({3, 3, 9});
      L.jac.push_back({3, 4, 10});
      L.jac.push_back({3, 5, 11});
      if (rd) L.jac.push_back({4, 0, 12});
      L.jac.push_back({4, 1, 13});
      L.jac.push_back({4, 3, 14});
      L.jac.push_back({4, 4, 15});
      L.jac.push_back({4, 5, 16});
      L.jac.push_back({5, 1, 17});
      if (rs) L.jac.push_back({5, 2, 18});
      L.jac.push_back({5, 3, 19});
      L.jac.push_back({5, 4, 20});
      L.jac.push_back({5, 5, 21});
      double rec[kMosFields];
      derive_instance(kM, prm, rec, 1);
      if (rec[kMHasQ] != 0.0) {
        L.q = {{1, 0, 22}, {3, 0, 23}, {4, 0, 24}, {5, 0, 25}};
        L.qjac = {{1, 1, 26}, {1, 3, 27}, {1, 4, 28}, {1, 5, 29}, {3, 1, 30}, {3, 3, 31}, {3, 4, 32},
                  {3, 5, 33}, {4, 1, 34}, {4, 3, 35}, {4, 4, 36}, {5, 1, 37}, {5, 3, 38}, {5, 5, 39}};
      }
      break;
    }
    case kB3: {  // d g s b di si (models/bsim3.va:613-624); the DC core has no charges
      const double rsh = prm[kB3ParamRsh];
      const bool rd = rsh > 0 && prm[kB3ParamNrd] > 0, rs = rsh > 0 && prm[kB3ParamNrs] > 0;
      if (rd) L.res.push_back({0, 0, 0});
      if (rs) L.res.push_back({2, 0, 1});
      L.res.push_back({3, 0, 2});
      L.res.push_back({4, 0, 3});
      L.res.push_back({5, 0, 4});
      if (rd) {
        L.jac.push_back({0, 0, 5});
        L.jac.push_back({0, 4, 6});
      }
      if (rs) {
        L.jac.push_back({2, 2, 7});
        L.jac.push_back({2, 5, 8});
      }
      L.jac.push_back({3, 1, 9});
      L.jac.push_back({3, 3, 10});
      L.jac.push_back({3, 4, 11});
      L.jac.push_back({3, 5, 12});
      if (rd) L.jac.push_back({4, 0, 13});
      L.jac.push_back({4, 1, 14});
      L.jac.push_back({4, 3, 15});
      L.jac.push_back({4, 4, 16});
      L.jac.push_back({4, 5, 17});
      L.jac.push_back({5, 1, 18});
      if (rs) L.jac.push_back({5, 2, 19});
      L.jac.push_back({5, 3, 20});
      L.jac.push_back({5, 4, 21});
      L.jac.push_back({5, 5, 22});
      break;
    }
    default:
      break;
  }
  return L;
}

template <class T>
cudaError_t upload(DevBuf& b, const std::vector<T>& v, cudaStream_t s) {
  cudaError_t e = b.ensure(v.size() * sizeof(T));
  if (e != cudaSuccess || v.empty()) return e;
  return cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s);
}

}  // namespace

struct esl_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::string err;
  uint32_t lanes_per_block = 0;  // 0: as many as the lane count spreads over the SMs
  uint32_t lanes_eff = 4;  // lanes per CTA that fit beside the staged programs
  uint32_t tran_lanes_eff = 0;  // the same for the transient kernel (0: does not fit)
  int sms = 148;

  Csc pat;
  std::vector<uint8_t> cur;
  std::vector<uint32_t> order;
  std::vector<HostBatch> bats;
  uint32_t n_stage = 0, rec_size = 0, nlim = 0;
  std::vector<uint32_t> rhs_ptr, rhs_src, a_ptr, a_src, slot_row;
  std::vector<uint32_t> gst;  // gmin-stepping stamps (slot, row, column)
  std::vector<uint32_t> q_ptr, q_src, c_ptr, c_src;  // transient charge rows, capacitance slots
  uint32_t n_qt = 0;
  std::vector<double> rec_nominal;

  uint32_t n_lanes = 0;
  std::vector<double> rec_lane0;   // lane 0's records (the lead lane's, for the host-side tape builds)
  std::vector<uint32_t> prm_off;   // each batch's first parameter in d_params
  DevBuf d_rec_nominal, d_params, d_derive_items, d_derive_slots, d_values;

  bool have_tape = false;
  bool warp_ok = false;    // the tape's warp programs fit (16-bit value indices, a warp's shared memory)
  bool has_meyer = false;  // a MOS1 instance gives TOX: DC only
  // Block lanes (block.cu): the solve mode, the block programs of the
  // current tape and their device copies, the per-CTA working-set slab.
  uint32_t precision = ESL_PREC_FP64;
  uint32_t path = ESL_PATH_AUTO;
  uint32_t block_width = 256;
  double refine_tol = 1e-12;
  uint32_t refine_max = 6;
  double refine_skip = 0.0;  // mixed: steps above this many tolerances go unrefined (0: none)
  bool have_block = false;
  bool profile = false;  // block lanes: accumulate the phase cycles (esl_solve_mode.profile)
  BlockPrograms bprog;
  uint32_t block_op_bytes = 8;     // 8: 16-bit value indices; 16: 32-bit
  uint32_t block_g_len = 0, block_g_ncells = 0;
  DevBuf d_ba, d_bb, d_bf, d_slab, d_refine, d_prof, d_bg_terms, d_bg_cells;
  SparseLu lead;
  Programs prog;

  DevBuf d_nodes[kMaxBatches], d_rhs_ptr, d_rhs_src, d_a_ptr, d_a_src, d_slot_row, d_cur;
  DevBuf d_q_ptr, d_q_src, d_c_ptr, d_c_src, d_probes, d_tran_t, d_tran_v, d_tran_n, d_tran_stats;
  DevBuf d_amap, d_fill, d_prog, d_l_scaled, d_pinv, d_q, d_seq, d_sweep_values, d_meas, d_next_lane;
  DevBuf d_sweep_state, d_sweep_rows;  // paused sweep lanes' state
  DevBuf d_tran_state, d_tran_save;    // paused transient lanes' state
  esl_stats last_peels{};              // the last call's peel counts (esl_peel_stats)
  uint64_t last_tran_refinements = 0;  // the last block transient's FP64 corrections (mixed)
  uint32_t n_seq_a = 0, n_seq = 0, seq_warps = 0;  // lane-interleaved op list
  uint32_t n_seq_f = 0, mixed_warps = 0;            // its forward-only tail, the mixed kernel's warps
  LuJitKernels lu_jit;                               // the tape-compiled lane LU of the current tape
  DevBuf d_lu_scratch;                               // its tape-value plane when the caller passes none
  LuJitKernels lu_jit_mixed;                         // the compiled mixed-precision form
  int lu_jit_mixed_state = 0;
  DevBuf d_lu_scratch32;                             // its FP32 factor plane
  int lu_jit_state = 0;                              // 0 not built, 1 built, -1 failed
  DevBuf d_row_ptr, d_row_slot, d_row_col;
  DevBuf d_group_topo, d_group_lanes, d_group_cta_ctx, d_group_cta_first, d_group_lpb;  // a group launch's tables
  DevBuf d_group_blocks, d_group_items, d_group_slab;  // a block-lane group launch's tables and slabs
  DevBuf d_rec, d_lim, d_lim_active, d_status, d_iters, d_flags, d_limit, d_a_vals, d_rhs, d_dx,
      d_diag, d_paused, d_x;
  DevBuf d_gst, d_ladder, d_x_good;  // operating-point lanes: stamps, ladder states, stepping points
  DevBuf d_tran_slab;                // block transient lanes: each CTA's run state
  TopoDev topo{};

  std::unordered_map<uint32_t, DirectSolver> peel;

  int32_t fail(int32_t code, const std::string& what) {
    err = what;
    return code;
  }
  int32_t cuda_fail(cudaError_t e, const char* where) {
    err = std::string(where) + ": " + cudaGetErrorString(e);
    return ESL_DEVICE_FAULT;
  }
};

#define ESL_CUDA(call)                                   \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return ctx->cuda_fail(e_, #call); \
  } while (0)

namespace {

// Pattern (Circuit.freeze): every diagonal, then every device entry off
// ground; CSC with rows ascending.
Csc build_pattern(const std::vector<HostBatch>& bats, uint32_t n) {
  std::vector<uint64_t> keys;
  for (uint32_t i = 0; i < n; ++i) keys.push_back((uint64_t(i) << 32) | i);
  for (const auto& B : bats)
    for (uint32_t id = 0; id < B.count; ++id) {
      const uint32_t* nd = &B.nodes[size_t(id) * B.nt];
      InstLayout L = layout_of(B.type, &B.params[size_t(id) * B.np]);
      for (auto* list : {&L.jac, &L.qjac})
        for (const Entry& e : *list) {
          const uint32_t r = nd[e.ru], c = nd[e.cu];
          if (r != 0 && c != 0) keys.push_back((uint64_t(c) << 32) | r);
        }
    }
  std::sort(keys.begin(), keys.end());
  keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
  Csc pat;
  pat.n = n;
  pat.col_ptr.assign(n + 1, 0);
  for (uint64_t k : keys) {
    pat.row_idx.push_back(uint32_t(k & 0xffffffffu));
    pat.col_ptr[(k >> 32) + 1]++;
  }
  for (uint32_t j = 0; j < n; ++j) pat.col_ptr[j + 1] += pat.col_ptr[j];
  return pat;
}

// Copies a C-ABI circuit into host batches; false on a bad table.
bool read_circuit(const esl_circuit* c, std::vector<HostBatch>& bats) {
  uint32_t stage = 0, rec = 0, lim = 0;
  for (uint32_t b = 0; b < c->n_batches; ++b) {
    const esl_batch& src = c->batches[b];
    if (src.type >= kNumTypes) return false;
    HostBatch B;
    B.type = src.type;
    B.count = src.count;
    B.nt = node_count(src.type);
    B.np = param_count(src.type);
    B.nodes.assign(src.nodes, src.nodes + size_t(src.count) * B.nt);
    B.params.assign(src.params, src.params + size_t(src.count) * B.np);
    for (uint32_t v : B.nodes)
      if (v >= c->n) return false;
    B.stride = stage_stride(src.type);
    if (src.type == kM) {
      bool any = false;
      for (uint32_t id = 0; id < B.count && !any; ++id) {
        double r[kMosFields];
        derive_instance(kM, &B.params[size_t(id) * B.np], r, 1);
        any = r[kMHasQ] != 0.0;
      }
      if (!any) B.stride = kStageMNoQ;
    }
    B.stage_base = stage;
    stage += B.stride * B.count;
    B.nfields = record_fields(src.type);
    B.rec_off = rec;
    rec += B.nfields * B.count;
    B.lim_off = lim;
    lim += lim_count(src.type) * B.count;
    bats.push_back(std::move(B));
  }
  return true;
}

// Gather lists: for each residual row and pattern slot, its staging cells
// in stamp order, then the ground pin on row 0 and slot (0, 0).
void build_gather(esl_ctx* ctx) {
  const uint32_t n = ctx->pat.n, nnz = ctx->pat.nnz();
  std::vector<std::vector<uint32_t>> rows(n), slots(nnz), qrows(n), cslots(nnz);
  for (const auto& B : ctx->bats)
    for (uint32_t id = 0; id < B.count; ++id) {
      const uint32_t* nd = &B.nodes[size_t(id) * B.nt];
      InstLayout L = layout_of(B.type, &B.params[size_t(id) * B.np]);
      const uint32_t base = B.stage_base + id * B.stride;
      for (const Entry& e : L.res)
        if (nd[e.ru] != 0) rows[nd[e.ru]].push_back(base + e.pos);
      for (const Entry& e : L.jac) {
        const uint32_t s = ctx->pat.slot(nd[e.ru], nd[e.cu]);
        if (s != nnz) slots[s].push_back(base + e.pos);
      }
      for (const Entry& e : L.q)
        if (nd[e.ru] != 0) qrows[nd[e.ru]].push_back(base + e.pos);
      for (const Entry& e : L.qjac) {
        const uint32_t s = ctx->pat.slot(nd[e.ru], nd[e.cu]);
        if (s != nnz) cslots[s].push_back(base + e.pos);
      }
    }
  rows[0].push_back(kSrcX0);
  slots[ctx->pat.col_ptr[0]].push_back(kSrcOne);
  auto flatten = [](const std::vector<std::vector<uint32_t>>& v, std::vector<uint32_t>& ptr,
                    std::vector<uint32_t>& src) {
    ptr.assign(v.size() + 1, 0);
    src.clear();
    for (size_t i = 0; i < v.size(); ++i) {
      src.insert(src.end(), v[i].begin(), v[i].end());
      ptr[i + 1] = uint32_t(src.size());
    }
  };
  flatten(rows, ctx->rhs_ptr, ctx->rhs_src);
  flatten(slots, ctx->a_ptr, ctx->a_src);
  flatten(qrows, ctx->q_ptr, ctx->q_src);
  flatten(cslots, ctx->c_ptr, ctx->c_src);
  ctx->slot_row.assign(nnz, kNoDiag);
  for (uint32_t i = 0; i < n; ++i) {
    const uint32_t s = i == 0 ? ctx->pat.col_ptr[0] : ctx->pat.slot(i, i);
    ctx->slot_row[s] = i;
  }
}

int32_t upload_topology(esl_ctx* ctx) {
  cudaStream_t s = ctx->stream;
  TopoDev& T = ctx->topo;
  T.n = ctx->pat.n;
  T.nnz = ctx->pat.nnz();
  T.n_stage = ctx->n_stage;
  T.nlim = ctx->nlim;
  T.rec_size = ctx->rec_size;
  T.n_batches = uint32_t(ctx->bats.size());
  T.n_src = 0;
  for (size_t b = 0; b < ctx->bats.size(); ++b) {
    const HostBatch& B = ctx->bats[b];
    ESL_CUDA(upload(ctx->d_nodes[b], B.nodes, s));
    T.b[b] = BatchDev{B.type, B.count, B.nt, B.stage_base, B.stride, B.rec_off, B.lim_off,
                      ctx->d_nodes[b].as<uint32_t>(), B.qt_off, B.qt_sites, T.n_src};
    if (B.type == kV || B.type == kI) T.n_src += B.count;
  }
  ESL_CUDA(upload(ctx->d_q_ptr, ctx->q_ptr, s));
  ESL_CUDA(upload(ctx->d_q_src, ctx->q_src, s));
  ESL_CUDA(upload(ctx->d_c_ptr, ctx->c_ptr, s));
  ESL_CUDA(upload(ctx->d_c_src, ctx->c_src, s));
  T.q_ptr = ctx->d_q_ptr.as<uint32_t>();
  T.q_src = ctx->d_q_src.as<uint32_t>();
  T.c_ptr = ctx->d_c_ptr.as<uint32_t>();
  T.c_src = ctx->d_c_src.as<uint32_t>();
  T.n_qt = ctx->n_qt;
  {
    // the pattern by rows, for the refinement's residual
    const uint32_t n = ctx->pat.n;
    std::vector<std::vector<std::pair<uint32_t, uint32_t>>> rows(n);
    for (uint32_t j = 0; j < n; ++j)
      for (uint32_t p = ctx->pat.col_ptr[j]; p < ctx->pat.col_ptr[j + 1]; ++p) rows[ctx->pat.row_idx[p]].push_back({p, j});
    std::vector<uint32_t> rp(n + 1, 0), rs, rc;
    for (uint32_t i = 0; i < n; ++i) {
      for (auto& e : rows[i]) {
        rs.push_back(e.first);
        rc.push_back(e.second);
      }
      rp[i + 1] = uint32_t(rs.size());
    }
    ESL_CUDA(upload(ctx->d_row_ptr, rp, s));
    ESL_CUDA(upload(ctx->d_row_slot, rs, s));
    ESL_CUDA(upload(ctx->d_row_col, rc, s));
    T.row_ptr = ctx->d_row_ptr.as<uint32_t>();
    T.row_slot = ctx->d_row_slot.as<uint32_t>();
    T.row_col = ctx->d_row_col.as<uint32_t>();
  }
  ESL_CUDA(upload(ctx->d_rhs_ptr, ctx->rhs_ptr, s));
  ESL_CUDA(upload(ctx->d_rhs_src, ctx->rhs_src, s));
  ESL_CUDA(upload(ctx->d_a_ptr, ctx->a_ptr, s));
  ESL_CUDA(upload(ctx->d_a_src, ctx->a_src, s));
  ESL_CUDA(upload(ctx->d_slot_row, ctx->slot_row, s));
  ESL_CUDA(upload(ctx->d_cur, ctx->cur, s));
  T.rhs_ptr = ctx->d_rhs_ptr.as<uint32_t>();
  T.rhs_src = ctx->d_rhs_src.as<uint32_t>();
  T.a_ptr = ctx->d_a_ptr.as<uint32_t>();
  T.a_src = ctx->d_a_src.as<uint32_t>();
  T.slot_row = ctx->d_slot_row.as<uint32_t>();
  T.cur_row = ctx->d_cur.as<uint8_t>();
  return ESL_OK;
}

// One lane's shared block, in doubles (newton.cu carves the same layout):
// x | xo | rhs | diag | v = [tape values | y | 0.0 | 1.0 | sink] |
// staging | limited images.
struct LaneLayout {
  uint32_t x, xo, rhs, diag, tv, y, zero, one, sink, st, lim, total;
};

LaneLayout lane_layout(uint32_t n, uint32_t ntv, uint32_t n_stage, uint32_t nlim) {
  LaneLayout L;
  L.x = 0;
  L.xo = n;
  L.rhs = 2 * n;
  L.diag = 3 * n;
  L.tv = 4 * n;
  L.y = L.tv + ntv;
  L.zero = L.y + n;
  L.one = L.zero + 1;
  L.sink = L.zero + 2;
  L.st = L.zero + 3;
  L.lim = L.st + n_stage;
  L.total = (L.lim + nlim + 1) & ~1u;
  return L;
}

struct GatherProgram {
  std::vector<uint32_t> depth, off, src, dst;
};

// Assembly cells: every residual row, every pattern slot and every fill-in
// tape value, each summing its staging cells in stamp order.
struct AsmCell {
  std::vector<uint32_t> src;
  uint32_t d0, d1, d2;
};

std::vector<AsmCell> assembly_cells(const esl_ctx* ctx, const Programs& P, const LaneLayout& L) {
  const uint32_t n = ctx->pat.n, nnz = ctx->pat.nnz();
  std::vector<AsmCell> cells;
  auto remap = [&](uint32_t s) { return s == kSrcOne ? L.one : s == kSrcX0 ? L.x : L.st + s; };
  for (uint32_t i = 0; i < n; ++i) {
    AsmCell c;
    for (uint32_t e = ctx->rhs_ptr[i]; e < ctx->rhs_ptr[i + 1]; ++e) c.src.push_back(remap(ctx->rhs_src[e]));
    c.d0 = L.rhs + i;
    c.d1 = L.sink;
    c.d2 = L.y + ctx->lead.pinv[i];
    cells.push_back(std::move(c));
  }
  for (uint32_t p = 0; p < nnz; ++p) {
    AsmCell c;
    for (uint32_t e = ctx->a_ptr[p]; e < ctx->a_ptr[p + 1]; ++e) c.src.push_back(remap(ctx->a_src[e]));
    c.d0 = L.tv + P.amap[p];
    c.d1 = ctx->slot_row[p] != kNoDiag ? L.diag + ctx->slot_row[p] : L.sink;
    c.d2 = L.sink;
    cells.push_back(std::move(c));
  }
  for (uint32_t f : P.fill) cells.push_back(AsmCell{{}, L.tv + f, L.sink, L.sink});
  return cells;
}

// The assembly as one segmented gather: the warp walks nseg segments of
// seg_len terms (a multiple of kGatherBlock), thread t summing term k of its column at
// src[k * 32 + t]; at each segment's end every thread whose cell ends there
// stores its sum (twice, and the negation) to that segment's destination
// triple for it (dst[(3 s + i) * 32 + t], kGatherEnd on the first word) and
// starts over from +0.0. A cell spans ceil(len / seg_len) consecutive
// segments of one column, its terms at the end of that span and +0.0 before
// them (a sum that starts at +0.0 is never -0.0, so a +0.0 term changes no
// bit). Cells go to the least loaded column, longest first, and seg_len is
// the multiple of kGatherBlock that minimises the segments walked times (seg_len +
// the boundary's cost): one long sum (a supply node's row, a term per device
// on the node) then runs beside all the short ones instead of after them.
struct GatherSegments {
  std::vector<uint32_t> src, dst;
  uint32_t nseg = 0, seg_len = kGatherBlock;
};

GatherSegments build_gather_segments(const esl_ctx* ctx, const Programs& P) {
  const LaneLayout L = lane_layout(ctx->pat.n, P.ntv, ctx->n_stage, ctx->nlim);
  std::vector<AsmCell> cells = assembly_cells(ctx, P, L);
  std::stable_sort(cells.begin(), cells.end(),
                   [](const AsmCell& a, const AsmCell& b) { return a.src.size() > b.src.size(); });
  const size_t longest = cells.empty() ? 0 : cells.front().src.size();
  constexpr size_t kBoundaryCost = 8;  // terms' worth of time per segment boundary
  auto place = [&](uint32_t seg_len, uint32_t* column) {
    std::vector<uint32_t> load(32, 0);
    for (size_t c = 0; c < cells.size(); ++c) {
      const uint32_t segs = std::max<uint32_t>(1, uint32_t((cells[c].src.size() + seg_len - 1) / seg_len));
      const uint32_t t = uint32_t(std::min_element(load.begin(), load.end()) - load.begin());
      if (column) column[c] = t;
      load[t] += segs;
    }
    return *std::max_element(load.begin(), load.end());
  };
  const uint32_t gb = kGatherBlock;
  uint32_t best_len = gb, best_nseg = place(gb, nullptr);
  for (uint32_t len = 2 * gb; len <= std::max<size_t>(gb, (longest + gb - 1) / gb * gb); len += gb) {
    const uint32_t nseg = place(len, nullptr);
    if (size_t(nseg) * (len + kBoundaryCost) < size_t(best_nseg) * (best_len + kBoundaryCost)) {
      best_len = len;
      best_nseg = nseg;
    }
  }
  std::vector<uint32_t> column(cells.size());
  place(best_len, column.data());
  GatherSegments G;
  G.seg_len = best_len;
  G.nseg = best_nseg;
  G.src.assign(size_t(G.nseg) * G.seg_len * 32, L.zero);
  // one sink triple past the last segment: the kernel loads a triple ahead
  G.dst.assign(size_t(G.nseg + 1) * 3 * 32, L.sink);
  std::vector<uint32_t> at(32, 0);  // next free segment per column
  for (size_t c = 0; c < cells.size(); ++c) {
    const uint32_t t = column[c];
    const size_t len = cells[c].src.size();
    const uint32_t segs = std::max<uint32_t>(1, uint32_t((len + G.seg_len - 1) / G.seg_len));
    const size_t end = size_t(at[t] + segs) * G.seg_len;  // one past the cell's last term
    for (size_t k = 0; k < len; ++k) G.src[(end - len + k) * 32 + t] = cells[c].src[k];
    const size_t s = at[t] + segs - 1;
    G.dst[(3 * s + 0) * 32 + t] = cells[c].d0 | kGatherEnd;
    G.dst[(3 * s + 1) * 32 + t] = cells[c].d1;
    G.dst[(3 * s + 2) * 32 + t] = cells[c].d2;
    at[t] += segs;
  }
  return G;
}

// The transient companion's cells (integrator.zig Hook): every row with
// charge cells (its charge sum; dst pair: the row, its y value) and then
// every pattern slot with capacitance cells (its capacitance sum; dst pair:
// the tape value, the diagonal copy or the sink), each part sorted by list
// length. Rows and slots without such cells are left out: their companion
// terms are exactly zero and their values, sums from +0.0, are never -0.0,
// so adding the zero terms would change no bit.
GatherProgram build_companion_program(const esl_ctx* ctx, const Programs& P, uint32_t& n_row_groups) {
  const uint32_t n = ctx->pat.n, nnz = ctx->pat.nnz();
  const LaneLayout L = lane_layout(n, P.ntv, ctx->n_stage, ctx->nlim);
  struct Cell {
    std::vector<uint32_t> src;
    uint32_t d0, d1;
  };
  auto by_len = [](const Cell& a, const Cell& b) { return a.src.size() > b.src.size(); };
  std::vector<Cell> rows, slots;
  for (uint32_t i = 0; i < n; ++i) {
    if (ctx->q_ptr[i + 1] == ctx->q_ptr[i]) continue;
    Cell c{{}, i, L.y + ctx->lead.pinv[i]};
    for (uint32_t e = ctx->q_ptr[i]; e < ctx->q_ptr[i + 1]; ++e) c.src.push_back(L.st + ctx->q_src[e]);
    rows.push_back(std::move(c));
  }
  for (uint32_t p = 0; p < nnz; ++p) {
    if (ctx->c_ptr[p + 1] == ctx->c_ptr[p]) continue;
    Cell c{{}, L.tv + P.amap[p], ctx->slot_row[p] != kNoDiag ? L.diag + ctx->slot_row[p] : L.sink};
    for (uint32_t e = ctx->c_ptr[p]; e < ctx->c_ptr[p + 1]; ++e) c.src.push_back(L.st + ctx->c_src[e]);
    slots.push_back(std::move(c));
  }
  std::stable_sort(rows.begin(), rows.end(), by_len);
  std::stable_sort(slots.begin(), slots.end(), by_len);
  GatherProgram K;
  auto pack = [&](const std::vector<Cell>& cells, uint32_t pad0) {
    for (size_t g0 = 0; g0 < cells.size(); g0 += 32) {
      uint32_t depth = 0;
      for (size_t t = 0; t < 32 && g0 + t < cells.size(); ++t)
        depth = std::max<uint32_t>(depth, cells[g0 + t].src.size());
      K.depth.push_back(depth);
      K.off.push_back(uint32_t(K.src.size()));
      for (uint32_t k = 0; k < depth; ++k)
        for (size_t t = 0; t < 32; ++t) {
          const bool live = g0 + t < cells.size() && k < cells[g0 + t].src.size();
          K.src.push_back(live ? cells[g0 + t].src[k] : L.zero);
        }
      for (size_t t = 0; t < 32; ++t) {
        const bool live = g0 + t < cells.size();
        K.dst.push_back(live ? cells[g0 + t].d0 : pad0);  // kNone: the kernel's kNoDiag
        K.dst.push_back(live ? cells[g0 + t].d1 : L.sink);
      }
    }
  };
  pack(rows, kNone);
  n_row_groups = uint32_t(K.depth.size());
  pack(slots, L.sink);
  return K;
}

// The sequential op list of the lane-interleaved kernels: the programs'
// real ops in row order (padding writes the sink, nv - 1), then a copy of
// program A's forward-solve ops (the mixed kernel's correction solves).
std::vector<Op> lane_sequence(const Programs& P, uint32_t& n_a, uint32_t& n_all, uint32_t& n_f) {
  std::vector<Op> seq;
  for (const Op& o : P.a_ops)
    if ((o.w0 & 0x0fffffffu) != P.nv - 1) seq.push_back(o);
  n_a = uint32_t(seq.size());
  for (const Op& o : P.b_ops)
    if ((o.w0 & 0x0fffffffu) != P.nv - 1) seq.push_back(o);
  n_all = uint32_t(seq.size());
  for (uint32_t k = 0; k < n_a; ++k)
    if ((seq[k].w0 >> 28) == kOpSubNz) seq.push_back(seq[k]);
  n_f = uint32_t(seq.size()) - n_all;
  return seq;
}

// The compiled lane LU's source for a factored lead tape: the ops in the
// replay's own sequential order (column by column; every value's updates in
// the same order as the warp programs', so the same bits), which keeps
// fewer values live at once than the programs' level-packed rows.
std::string compiled_lu_source(uint32_t nnz, const SparseLu& lu, const Programs& P, uint32_t resident = 0,
                               bool mixed = false) {
  std::vector<Op> seq = P.a_list;
  const uint32_t n_a = uint32_t(seq.size());
  seq.insert(seq.end(), P.b_list.begin(), P.b_list.end());
  const uint32_t n_all = uint32_t(seq.size());
  LuJitInput in;
  in.n = P.n;
  in.nnz = nnz;
  in.nu = P.nu;
  in.nl = P.nl;
  in.ntv = P.ntv;
  in.nv = P.nv;
  in.amap = &P.amap;
  in.fill = &P.fill;
  std::vector<uint32_t> pinv(lu.pinv.begin(), lu.pinv.begin() + P.n);
  in.pinv = &pinv;
  in.qcol = &lu.q;
  in.l_scaled = &P.l_scaled;
  in.seq = &seq;
  in.n_seq_a = n_a;
  in.n_seq = n_all;
  in.mixed = mixed;
  in.col_ptr = &lu.a->col_ptr;
  in.row_idx = &lu.a->row_idx;
  if (mixed) in.resident_values = 48;  // the refinement loop needs the registers (more spilled)
  if (resident) in.resident_values = resident;
  return lu_jit_source(in);
}

// The lead lane's pivot tape, compiled and uploaded.
int32_t upload_tape(esl_ctx* ctx) {
  cudaStream_t s = ctx->stream;
  TopoDev& T = ctx->topo;
  Programs& P = ctx->prog;
  if (P.has_void) return ctx->fail(ESL_NOT_ELIGIBLE, "the lead factor fabricated a pivot for a void unknown");
  ESL_CUDA(upload(ctx->d_amap, P.amap, s));
  ESL_CUDA(upload(ctx->d_fill, P.fill, s));
  ESL_CUDA(upload(ctx->d_l_scaled, P.l_scaled, s));
  ESL_CUDA(upload(ctx->d_pinv, ctx->lead.pinv, s));
  ESL_CUDA(upload(ctx->d_q, ctx->lead.q, s));
  T.nu = P.nu;
  T.nl = P.nl;
  T.ntv = P.ntv;
  T.nv = P.nv;
  T.amap = ctx->d_amap.as<uint32_t>();
  T.fill = ctx->d_fill.as<uint32_t>();
  T.n_fill = uint32_t(P.fill.size());
  T.l_scaled = ctx->d_l_scaled.as<uint8_t>();
  T.pinv = ctx->d_pinv.as<uint32_t>();
  T.qcol = ctx->d_q.as<uint32_t>();
  ctx->have_block = false;  // a new tape needs its own block programs
  lu_jit_release(ctx->lu_jit);  // and its own compiled LU
  ctx->lu_jit_state = 0;
  lu_jit_release(ctx->lu_jit_mixed);
  ctx->lu_jit_mixed_state = 0;
  ctx->have_tape = true;
  // The warp lanes: programs with 16-bit value indices, the programs and one
  // lane's working set in a CTA's shared memory. A tape beyond them runs on
  // the block lanes only.
  ctx->warp_ok = false;
  if (P.nv >= 65536) return ESL_OK;
  {
    // One blob: A ops, B ops, gather depth/off/src/dst, each section
    // 16-byte aligned.
    GatherSegments G = build_gather_segments(ctx, P);
    std::vector<unsigned char> blob;
    auto put = [&blob](const void* p, size_t bytes) {
      const uint32_t at = uint32_t(blob.size());
      blob.insert(blob.end(), static_cast<const unsigned char*>(p), static_cast<const unsigned char*>(p) + bytes);
      blob.resize((blob.size() + 15) & ~size_t(15), 0);
      return at;
    };
    T.o_a_ops = put(P.a_ops.data(), P.a_ops.size() * sizeof(Op));
    T.o_b_ops = put(P.b_ops.data(), P.b_ops.size() * sizeof(Op));
    T.o_g_src = put(G.src.data(), G.src.size() * 4);
    T.o_g_dst = put(G.dst.data(), G.dst.size() * 4);
    uint32_t n_kr = 0;
    GatherProgram K = build_companion_program(ctx, P, n_kr);
    T.o_k_depth = put(K.depth.data(), K.depth.size() * 4);
    T.o_k_off = put(K.off.data(), K.off.size() * 4);
    T.o_k_src = put(K.src.data(), K.src.size() * 4);
    T.o_k_dst = put(K.dst.data(), K.dst.size() * 4);
    T.n_kr_groups = n_kr;
    T.n_ks_groups = uint32_t(K.depth.size()) - n_kr;
    ESL_CUDA(upload(ctx->d_prog, blob, s));
    T.prog = ctx->d_prog.as<unsigned char>();
    T.prog_bytes = uint32_t(blob.size());
    T.a_rows = P.a_rows;
    T.b_rows = P.b_rows;
    T.g_nseg = G.nseg;
    T.g_seg_blocks = G.seg_len / kGatherBlock;
  }
  T.smem_doubles = lane_layout(T.n, T.ntv, T.n_stage, T.nlim).total;
  // Every CTA stages the programs; as many lanes per CTA as fit beside them.
  const size_t lane_bytes = size_t(T.smem_doubles) * 8;
  const size_t room = size_t(227) * 1024;
  if (T.prog_bytes + lane_bytes > room) return ESL_OK;
  ctx->lanes_eff = std::max<uint32_t>(1, std::min<uint32_t>(8, uint32_t((room - T.prog_bytes) / lane_bytes)));
  // Transient lanes add the accepted points, the charge rings and dynamic
  // currents over the rows and the LTE states: cur | prev | q[4] | ip over
  // n, then q[4] | ip over n_qt, then the V and I sources' values at the
  // current time point and the PULSE corner timers (4 start/period pairs
  // per source).
  T.tran_doubles = (T.smem_doubles + 7 * T.n + 5 * T.n_qt + 9 * T.n_src + 1) & ~1u;
  const size_t tran_bytes = size_t(T.tran_doubles) * 8;
  ctx->tran_lanes_eff = T.prog_bytes + tran_bytes > room
                            ? 0
                            : std::max<uint32_t>(1, std::min<uint32_t>(8, uint32_t((room - T.prog_bytes) / tran_bytes)));
  // The sequential op list of the lane-interleaved kernel: the programs'
  // real ops in row order (padding writes the sink, nv - 1).
  {
    std::vector<Op> seq = lane_sequence(P, ctx->n_seq_a, ctx->n_seq, ctx->n_seq_f);
    ESL_CUDA(upload(ctx->d_seq, seq, s));
    ctx->mixed_warps = 0;
    for (uint32_t w = 8; w >= 1; --w)
      if (lu_lanes_mixed_smem(T, ctx->n_seq + ctx->n_seq_f, w) <= room) {
        ctx->mixed_warps = w;
        break;
      }
    ctx->seq_warps = 0;
    for (uint32_t w = 8; w >= 1; --w)
      if (lu_lanes_smem(T, ctx->n_seq, w) <= room) {
        ctx->seq_warps = w;
        break;
      }
  }
  ctx->warp_ok = true;
  return ESL_OK;
}

// The block lanes' program rows in their device format: 8-byte words
// {dst | kind << 28, a | b << 16} when the value space has 16-bit indices,
// else the 16-byte words as built.
std::vector<uint32_t> block_words(const std::vector<Op4>& ops, bool short_ops) {
  std::vector<uint32_t> w;
  w.reserve(ops.size() * (short_ops ? 2 : 4));
  for (const Op4& o : ops) {
    if (short_ops) {
      w.push_back(o.w0);
      w.push_back(o.a | (o.b << 16));
    } else {
      w.push_back(o.w0);
      w.push_back(o.a);
      w.push_back(o.b);
      w.push_back(0u);
    }
  }
  return w;
}

// The block lanes' assembly streams (block.cu block_assemble): every
// residual row and pattern slot is a cell summing its staging terms in list
// order; cells go to the CTA's threads longest first, each to the least
// loaded thread; a thread's terms follow one another in its stream
// (terms[k * W + t]), the last term of each cell flagged, and its cells'
// destinations in its cell stream (cells[c * W + t]).
void build_block_gather(const esl_ctx* ctx, uint32_t W, std::vector<uint32_t>& terms, std::vector<uint32_t>& cells,
                        uint32_t& len, uint32_t& ncells) {
  struct Cell {
    std::vector<uint32_t> src;
    uint32_t w0, w1, w2, w3;
  };
  const uint32_t ns = ctx->n_stage;
  auto code = [ns](uint32_t s) { return s == kSrcOne ? ns + kGCellOne : s == kSrcX0 ? ns + kGCellX0 : s; };
  std::vector<Cell> all;
  const uint32_t n = ctx->pat.n, nnz = ctx->pat.nnz();
  // the gmin-stepping stamps: the column + 1 on a stamped row, 1 on a
  // stamped slot (block.cu gather_store)
  std::vector<uint32_t> row_w(n, 0u), slot_w(nnz, 0u);
  for (size_t k = 0; k + 2 < ctx->gst.size(); k += 3) {
    slot_w[ctx->gst[k]] = 1u;
    row_w[ctx->gst[k + 1]] = ctx->gst[k + 2] + 1u;
  }
  for (uint32_t i = 0; i < n; ++i) {
    Cell c{{}, i | kGCellRow, ctx->lead.pinv[i], 0u, row_w[i]};
    for (uint32_t e = ctx->rhs_ptr[i]; e < ctx->rhs_ptr[i + 1]; ++e) c.src.push_back(code(ctx->rhs_src[e]));
    all.push_back(std::move(c));
  }
  for (uint32_t p = 0; p < nnz; ++p) {
    Cell c{{}, p, ctx->prog.amap[p], ctx->slot_row[p], slot_w[p]};
    for (uint32_t e = ctx->a_ptr[p]; e < ctx->a_ptr[p + 1]; ++e) c.src.push_back(code(ctx->a_src[e]));
    all.push_back(std::move(c));
  }
  for (Cell& c : all) {
    if (c.src.empty()) c.src.push_back(ns + kGCellZero);
    c.src.back() |= kGTermEnd;
  }
  std::stable_sort(all.begin(), all.end(), [](const Cell& a, const Cell& b) { return a.src.size() > b.src.size(); });
  std::vector<std::vector<uint32_t>> t_terms(W), t_cells(W);
  std::vector<size_t> load(W, 0);
  for (const Cell& c : all) {
    const uint32_t t = uint32_t(std::min_element(load.begin(), load.end()) - load.begin());
    t_terms[t].insert(t_terms[t].end(), c.src.begin(), c.src.end());
    t_cells[t].insert(t_cells[t].end(), {c.w0, c.w1, c.w2, c.w3});
    load[t] += c.src.size();
  }
  len = 0;
  ncells = 0;
  for (uint32_t t = 0; t < W; ++t) {
    len = std::max(len, uint32_t(t_terms[t].size()));
    ncells = std::max(ncells, uint32_t(t_cells[t].size() / 4));
  }
  terms.assign(size_t(std::max(len, 1u)) * W, ns + kGCellZero);
  cells.assign(size_t(std::max(ncells, 1u)) * W * 4, 0u);
  for (uint32_t t = 0; t < W; ++t) {
    for (size_t k = 0; k < t_terms[t].size(); ++k) terms[k * W + t] = t_terms[t][k];
    for (size_t c = 0; c < t_cells[t].size() / 4; ++c)
      for (int j = 0; j < 4; ++j) cells[(c * W + t) * 4 + j] = t_cells[t][4 * c + j];
  }
}

void block_layout(const TopoDev& T, uint32_t nv, bool mixed, bool split, BlockDev& D);
uint32_t block_ring_bytes(uint32_t op_bytes, uint32_t row_k);
constexpr size_t kBlockSmemRoom = size_t(227) * 1024 - 256;

// Ops a thread a program row: kSlabRowOps when no placement of the working
// set (whole or its hot part, FP64 or mixed) fits a CTA's shared memory
// beside the op ring, so that the lanes run from the slab; 1 otherwise.
uint32_t block_row_k(const TopoDev& T, uint32_t op_bytes) {
  BlockDev D{};
  for (int mixed = 0; mixed < 2; ++mixed)
    for (int split = 0; split < 2; ++split) {
      block_layout(T, T.nv, mixed != 0, split != 0, D);
      if (D.lane_bytes + block_ring_bytes(op_bytes, 1) <= kBlockSmemRoom) return 1;
    }
  return kSlabRowOps;
}

// The block programs at rows of k ops a thread, uploaded in the context's
// op format.
int32_t set_block_programs(esl_ctx* ctx, uint32_t k) {
  cudaStream_t s = ctx->stream;
  const bool short_ops = ctx->block_op_bytes == 8;
  ctx->bprog = compile_block(ctx->prog, k * kBlockThreads);
  ctx->bprog.row_k = k;
  ESL_CUDA(upload(ctx->d_ba, block_words(ctx->bprog.a_ops, short_ops), s));
  ESL_CUDA(upload(ctx->d_bb, block_words(ctx->bprog.b_ops, short_ops), s));
  ESL_CUDA(upload(ctx->d_bf, block_words(ctx->bprog.f_ops, short_ops), s));
  return ESL_OK;
}

// The block lanes' programs and assembly streams of the current tape.
int32_t ensure_block(esl_ctx* ctx) {
  if (ctx->have_block) return ESL_OK;
  cudaStream_t s = ctx->stream;
  ctx->block_op_bytes = ctx->prog.nv < 65536 ? 8 : 16;
  if (int32_t rc = set_block_programs(ctx, block_row_k(ctx->topo, ctx->block_op_bytes))) return rc;
  std::vector<uint32_t> terms, cells;
  build_block_gather(ctx, kBlockThreads, terms, cells, ctx->block_g_len, ctx->block_g_ncells);
  ESL_CUDA(upload(ctx->d_bg_terms, terms, s));
  ESL_CUDA(upload(ctx->d_bg_cells, cells, s));
  ctx->have_block = true;
  return ESL_OK;
}

// The op ring a block-lane CTA streams its programs through (block.cu
// block_rows_k): kDepth + 1 slots of row_k op words per thread, 4 rows
// ahead for rows of one op a thread, 2 for rows of kSlabRowOps.
uint32_t block_ring_bytes(uint32_t op_bytes, uint32_t row_k) {
  return (row_k == 1 ? 5u : 3u) * row_k * kBlockThreads * op_bytes;
}

// A block lane's working set (block.cu carves the same): the hot part x,
// rhs, diag, dx (FP64, n each), limited images, the FP64 matrix (mixed
// form), the value space (nv values, FP64 or FP32); the cold part xo and
// the staging cells; each 16-byte aligned. split: the cold part's offsets
// start again from 0 (it lives in the CTA's slab).
void block_layout(const TopoDev& T, uint32_t nv, bool mixed, bool split, BlockDev& D) {
  size_t at = 0;
  auto take = [&at](size_t bytes) {
    const size_t o = at;
    at += (bytes + 15) & ~size_t(15);
    return uint32_t(o);
  };
  D.o_x = take(8 * size_t(T.n));
  D.o_rhs = take(8 * size_t(T.n));
  D.o_diag = take(8 * size_t(T.n));
  D.o_dx = take(8 * size_t(T.n));
  D.o_lim = take(8 * size_t(std::max<uint32_t>(T.nlim, 1)));
  D.o_a64 = take(mixed ? 8 * size_t(T.nnz) : 0);
  D.o_v = take(size_t(mixed ? 4 : 8) * nv);
  const size_t hot = at;
  if (split) at = 0;
  D.o_xo = take(8 * size_t(T.n));
  D.o_st = take(8 * size_t(T.n_stage + kGConstCells));
  D.split = split ? 1u : 0u;
  D.lane_bytes = uint32_t(split ? hot : at);
  D.cold_bytes = uint32_t(split ? at : 0);
}

// Shared memory a block lane may take (kBlockSmemRoom: a CTA's 227 KB, less
// the static reduction words).

// The launch view of the block lanes for n_lanes lanes: programs, layout,
// where the working set lives, the persistent grid and its slab.
int32_t block_view(esl_ctx* ctx, bool mixed, uint32_t n_lanes, BlockDev& D) {
  if (int32_t rc = ensure_block(ctx)) return rc;
  const TopoDev& T = ctx->topo;
  D = BlockDev{};
  D.T = T;
  D.a_ops = ctx->d_ba.p;
  D.b_ops = ctx->d_bb.p;
  D.f_ops = ctx->d_bf.p;
  D.a_rows = ctx->bprog.a_rows;
  D.b_rows = ctx->bprog.b_rows;
  D.f_rows = ctx->bprog.f_rows;
  D.op_bytes = ctx->block_op_bytes;
  D.row_k = ctx->bprog.row_k;
  D.ring_bytes = block_ring_bytes(D.op_bytes, D.row_k);
  D.g_terms = ctx->d_bg_terms.as<uint32_t>();
  D.g_cells = ctx->d_bg_cells.as<uint4>();
  D.g_len = ctx->block_g_len;
  D.g_ncells = ctx->block_g_ncells;
  // The placement with the most CTAs an SM: the whole working set in shared
  // memory, its hot part there (the cold part in the slab), or all of it in
  // the slab; on a tie, the most in shared memory.
  const bool long_ops = D.op_bytes == 16, b3 = topo_has_b3(T);
  int best = -1;
  uint32_t place = 2;
  for (uint32_t p = 0; p < 3; ++p) {
    block_layout(T, T.nv, mixed, p == 1, D);
    if (p < 2 && D.lane_bytes + D.ring_bytes > kBlockSmemRoom) continue;
    const int per_sm = block_occupancy(mixed, long_ops, b3, (p < 2 ? D.lane_bytes : 0) + D.ring_bytes);
    if (per_sm > best) {
      best = per_sm;
      place = p;
    }
  }
  block_layout(T, T.nv, mixed, place == 1, D);
  D.in_smem = place < 2;
  const uint32_t cap = uint32_t(ctx->sms) * uint32_t(std::max(best, 1));
  D.grid = std::max<uint32_t>(1, std::min(n_lanes, cap));
  ESL_CUDA(ctx->d_slab.ensure(size_t(D.in_smem && !D.split ? 1 : D.grid) * (D.split ? D.cold_bytes : D.lane_bytes)));
  D.slab = ctx->d_slab.as<unsigned char>();
  D.refine_tol = ctx->refine_tol;
  D.refine_max = ctx->refine_max;
  D.refine_skip = ctx->refine_skip;
  ESL_CUDA(ctx->d_refine.ensure(size_t(n_lanes) * 4));
  D.refine_out = mixed ? ctx->d_refine.as<uint32_t>() : nullptr;
  D.prof = nullptr;
  if (ctx->profile) {
    ESL_CUDA(ctx->d_prof.ensure(kBlockPhases * sizeof(unsigned long long)));
    D.prof = ctx->d_prof.as<unsigned long long>();
  }
  return ESL_OK;
}

// Whether a DC solve of this context runs on the block lanes: asked for,
// mixed precision (the warp lanes are FP64), or a tape beyond the warp
// lanes.
bool use_block(const esl_ctx* ctx) {
  return ctx->path == ESL_PATH_BLOCK || ctx->precision == ESL_PREC_MIXED || !ctx->warp_ok;
}

// The lead lane's first Jacobian in pattern order: the warp assembly kernel
// when its working set fits a CTA's shared memory, else the block lanes'
// (global scratch). The same gathers in the same order: the same bits.
cudaError_t lead_jacobian(esl_ctx* ctx, const LaneDev& L, double* out) {
  const TopoDev& T = ctx->topo;
  const size_t smem = size_t(4 * T.n + T.nv + T.n_stage + T.nlim + 2) * sizeof(double);
  if (smem <= size_t(227) * 1024) return launch_assemble(T, L, 0, out, ctx->stream);
  BlockDev D{};
  D.T = T;
  block_layout(T, 0, false, false, D);
  cudaError_t e = ctx->d_slab.ensure(D.lane_bytes);
  if (e != cudaSuccess) return e;
  D.slab = ctx->d_slab.as<unsigned char>();
  return launch_block_lead(D, L, 0, out, topo_has_b3(T), ctx->stream);
}

int32_t warp_only(esl_ctx* ctx) {
  if (ctx->warp_ok) return ESL_OK;
  return ctx->fail(ESL_NOT_ELIGIBLE,
                   "the circuit's tape exceeds the warp lanes (16-bit value indices or a warp's shared memory); "
                   "its DC solves run on the block lanes, this call has no block form");
}

int32_t build_tape_from(esl_ctx* ctx, const double* lead_vals) {
  ctx->lead.init(&ctx->pat, ctx->order);
  ctx->lead.fill_cap = kRepivotFillCap;
  ctx->lead.keep_min = kGrowthLimit;
  if (!ctx->lead.factor(lead_vals, kPivotTol))
    return ctx->fail(ESL_NOT_ELIGIBLE, "the lead lane's first Jacobian is singular");
  ctx->prog = compile_tape(ctx->lead);
  if (int32_t rc = upload_tape(ctx)) return rc;
  // The gmin-stepping rung's stamps: the V-source incidence (+-1) and the
  // zero branch diagonals decide them, the same in every lane.
  ctx->gst = gmin_stamps(ctx->pat, ctx->cur, lead_vals);
  ESL_CUDA(upload(ctx->d_gst, ctx->gst, ctx->stream));
  ctx->topo.gst = ctx->d_gst.as<uint32_t>();
  ctx->topo.n_gst = uint32_t(ctx->gst.size() / 3);
  return ESL_OK;
}

// Lanes per CTA for a launch over n_lanes: the caller's choice when given,
// else enough that the lanes spread over every SM once (each lane is a
// latency-bound warp; fewer, fuller CTAs would leave SMs idle), at most what
// shared memory fits.
uint32_t lanes_per_cta(const esl_ctx* ctx, uint32_t n_lanes, uint32_t fit) {
  uint32_t want = ctx->lanes_per_block;
  if (want == 0) want = (n_lanes + uint32_t(ctx->sms) - 1) / uint32_t(ctx->sms);
  return std::max<uint32_t>(1, std::min<uint32_t>(want, fit));
}

LaneDev lane_view(esl_ctx* ctx, uint32_t resume) {
  LaneDev L{};
  L.n_lanes = ctx->n_lanes;
  L.resume = resume;
  L.rec = ctx->d_rec.as<double>();
  L.x = ctx->d_x.as<double>();
  L.lim = ctx->d_lim.as<double>();
  L.lim_active = ctx->d_lim_active.as<uint32_t>();
  L.status = ctx->d_status.as<uint32_t>();
  L.iters = ctx->d_iters.as<uint32_t>();
  L.flags = ctx->d_flags.as<uint32_t>();
  L.limit = ctx->d_limit.as<double>();
  L.a_vals = ctx->d_a_vals.as<double>();
  L.rhs = ctx->d_rhs.as<double>();
  L.dx = ctx->d_dx.as<double>();
  L.diag = ctx->d_diag.as<double>();
  L.n_paused = ctx->d_paused.as<uint32_t>();
  return L;
}

int32_t ensure_lane_buffers(esl_ctx* ctx) {
  const size_t N = ctx->n_lanes, n = ctx->pat.n, nnz = ctx->pat.nnz();
  ESL_CUDA(ctx->d_x.ensure(N * n * 8));
  ESL_CUDA(ctx->d_lim.ensure(N * std::max<size_t>(ctx->nlim, 1) * 8));
  ESL_CUDA(ctx->d_lim_active.ensure(N * 4));
  ESL_CUDA(ctx->d_status.ensure(N * 4));
  ESL_CUDA(ctx->d_iters.ensure(N * 4));
  ESL_CUDA(ctx->d_flags.ensure(N * 4));
  ESL_CUDA(ctx->d_limit.ensure(N * 8));
  ESL_CUDA(ctx->d_a_vals.ensure(N * nnz * 8));
  ESL_CUDA(ctx->d_rhs.ensure(N * n * 8));
  ESL_CUDA(ctx->d_dx.ensure(N * n * 8));
  ESL_CUDA(ctx->d_diag.ensure(N * n * 8));
  ESL_CUDA(ctx->d_paused.ensure(4));
  return ESL_OK;
}

// Host factor + solve of the paused lanes (lane_solver.zig peel), then
// resume. A lane's first host factor is its own fresh factor when it paused
// at its first iterate; later it continues the lead tape's replay history.
// The status and iteration words are the launch's own (L.status, L.iters:
// the caller's device arrays for esl_dc_solve_device), the other hand-off
// planes the context's.
int32_t serve_pauses(esl_ctx* ctx, const LaneDev& L, esl_stats* st, bool* any) {
  cudaStream_t s = ctx->stream;
  uint32_t paused = 0;
  ESL_CUDA(cudaMemcpyAsync(&paused, ctx->d_paused.p, 4, cudaMemcpyDeviceToHost, s));
  ESL_CUDA(cudaStreamSynchronize(s));
  *any = paused != 0;
  if (!paused) return ESL_OK;
  const uint32_t N = ctx->n_lanes, n = ctx->pat.n, nnz = ctx->pat.nnz();
  std::vector<uint32_t> status(N), iters(N), flags(N);
  ESL_CUDA(cudaMemcpyAsync(status.data(), L.status, N * 4, cudaMemcpyDeviceToHost, s));
  ESL_CUDA(cudaMemcpyAsync(iters.data(), L.iters, N * 4, cudaMemcpyDeviceToHost, s));
  ESL_CUDA(cudaMemcpyAsync(flags.data(), ctx->d_flags.p, N * 4, cudaMemcpyDeviceToHost, s));
  ESL_CUDA(cudaStreamSynchronize(s));
  std::vector<double> a(nnz), r(n), dx(n);
  for (uint32_t l = 0; l < N; ++l) {
    if (status[l] != kNeedSolve) continue;
    ESL_CUDA(cudaMemcpy(a.data(), ctx->d_a_vals.as<double>() + size_t(l) * nnz, nnz * 8, cudaMemcpyDeviceToHost));
    ESL_CUDA(cudaMemcpy(r.data(), ctx->d_rhs.as<double>() + size_t(l) * n, n * 8, cudaMemcpyDeviceToHost));
    auto it = ctx->peel.find(l);
    if (it == ctx->peel.end()) {
      DirectSolver ds;
      ds.init(&ctx->pat, ctx->order);
      // a lane that factored before (an earlier iteration, or an earlier
      // run of the ladder) holds the lead tape in its solver
      if (iters[l] != 0 || (flags[l] & 4u)) ds.adopt(ctx->lead, nullptr);
      it = ctx->peel.emplace(l, std::move(ds)).first;
      it->second.lu.a = &ctx->pat;
      if (st) st->peeled++;
    }
    DirectSolver& ds = it->second;
    if (st) st->host_solves++;
    if (!ds.factor(a.data())) {
      status[l] = kSingular;
      iters[l] = 0;
      continue;
    }
    ds.solve_neg(r.data(), dx.data());
    ESL_CUDA(cudaMemcpy(ctx->d_dx.as<double>() + size_t(l) * n, dx.data(), n * 8, cudaMemcpyHostToDevice));
    if (ds.lu.same_tape(ctx->lead)) flags[l] &= ~2u;
  }
  ESL_CUDA(cudaMemcpyAsync(L.status, status.data(), N * 4, cudaMemcpyHostToDevice, s));
  ESL_CUDA(cudaMemcpyAsync(L.iters, iters.data(), N * 4, cudaMemcpyHostToDevice, s));
  ESL_CUDA(cudaMemcpyAsync(ctx->d_flags.p, flags.data(), N * 4, cudaMemcpyHostToDevice, s));
  ESL_CUDA(cudaMemsetAsync(ctx->d_paused.p, 0, 4, s));
  return ESL_OK;
}

}  // namespace

extern "C" {

int32_t esl_create(const esl_circuit* circuit, const esl_options* opts, esl_ctx** out) {
  if (!circuit || !out || circuit->n == 0 || circuit->n_batches > kMaxBatches) return ESL_INVALID_ARGUMENT;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return ESL_NO_DEVICE;
  auto ctx = std::make_unique<esl_ctx>();
  ctx->device = opts ? opts->device : 0;
  if (opts && opts->lanes_per_block) ctx->lanes_per_block = std::min<uint32_t>(opts->lanes_per_block, 8);
  cudaDeviceGetAttribute(&ctx->sms, cudaDevAttrMultiProcessorCount, ctx->device);
  if (cudaSetDevice(ctx->device) != cudaSuccess) return ESL_NO_DEVICE;
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) return ESL_DEVICE_FAULT;
  cudaEventCreate(&ctx->ev0);
  cudaEventCreate(&ctx->ev1);
  const uint32_t n = circuit->n;
  ctx->cur.assign(circuit->current_row, circuit->current_row + n);
  if (!read_circuit(circuit, ctx->bats)) return ESL_INVALID_ARGUMENT;
  for (const auto& B : ctx->bats) {
    if (B.type == kM)
      for (uint32_t id = 0; id < B.count; ++id)
        if (B.params[size_t(id) * B.np + kMParamTox] > 0.0) ctx->has_meyer = true;
    ctx->n_stage += B.stride * B.count;
    ctx->rec_size += B.nfields * B.count;
    ctx->nlim += lim_count(B.type) * B.count;
  }
  // LTE charge states: a batch keeps its sites when any instance has the
  // charge (capacitors always; diodes with CJO or TT; MOSFETs with overlap
  // capacitance).
  for (auto& B : ctx->bats) {
    bool any = B.type == kC;
    for (uint32_t id = 0; id < B.count && !any; ++id) {
      const double* p = &B.params[size_t(id) * B.np];
      if (B.type == kD) any = p[5] > 0 || p[9] > 0;
      if (B.type == kM) any = p[12] != 0 || p[13] != 0 || p[14] != 0;
    }
    B.qt_sites = any ? qt_count(B.type) : 0;
    B.qt_off = ctx->n_qt;
    ctx->n_qt += B.qt_sites * B.count;
  }
  const uint32_t rec = ctx->rec_size;
  ctx->pat = build_pattern(ctx->bats, n);
  build_gather(ctx.get());
  ctx->order = order_columns(ctx->pat);
  ctx->rec_nominal.assign(rec, 0.0);
  std::vector<double> params;
  for (const auto& B : ctx->bats) {
    ctx->prm_off.push_back(uint32_t(params.size()));
    params.insert(params.end(), B.params.begin(), B.params.end());
    for (uint32_t id = 0; id < B.count; ++id)
      derive_instance(B.type, &B.params[size_t(id) * B.np], &ctx->rec_nominal[B.rec_off + id], B.count);
  }
  ctx->rec_lane0 = ctx->rec_nominal;
  if (cudaError_t e = upload(ctx->d_rec_nominal, ctx->rec_nominal, ctx->stream)) {
    *out = ctx.release();
    return (*out)->cuda_fail(e, "nominal records");
  }
  if (cudaError_t e = upload(ctx->d_params, params, ctx->stream)) {
    *out = ctx.release();
    return (*out)->cuda_fail(e, "nominal parameters");
  }
  if (int32_t rc = upload_topology(ctx.get())) {
    *out = ctx.release();
    return rc;
  }
  *out = ctx.release();
  return ESL_OK;
}

int32_t esl_destroy(esl_ctx* ctx) {
  if (!ctx) return ESL_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  lu_jit_release(ctx->lu_jit);
  lu_jit_release(ctx->lu_jit_mixed);
  cudaStream_t s = ctx->stream;
  delete ctx;
  if (s) cudaStreamDestroy(s);
  return ESL_OK;
}

const char* esl_last_error(const esl_ctx* ctx) { return ctx ? ctx->err.c_str() : "no context"; }

int32_t esl_dims(const esl_ctx* ctx, uint32_t* n, uint32_t* nnz) {
  if (!ctx) return ESL_INVALID_ARGUMENT;
  if (n) *n = ctx->pat.n;
  if (nnz) *nnz = ctx->pat.nnz();
  return ESL_OK;
}

int32_t esl_set_lanes(esl_ctx* ctx, const esl_slot* slots, uint32_t n_slots, const double* values,
                      uint32_t n_lanes) {
  return esl_set_lanes_cols(ctx, slots, n_slots, nullptr, values, n_slots, n_lanes);
}

int32_t esl_set_lanes_cols(esl_ctx* ctx, const esl_slot* slots, uint32_t n_slots, const uint32_t* cols,
                           const double* values, uint32_t n_cols, uint32_t n_lanes) {
  if (!ctx || n_lanes == 0 || (n_slots && (!slots || !values || n_cols == 0))) return ESL_INVALID_ARGUMENT;
  for (uint32_t k = 0; k < n_slots; ++k) {
    if (slots[k].batch >= ctx->bats.size()) return ESL_INVALID_ARGUMENT;
    const HostBatch& B = ctx->bats[slots[k].batch];
    if (slots[k].inst >= B.count || slots[k].param >= B.np) return ESL_INVALID_ARGUMENT;
    if ((cols ? cols[k] : k) >= n_cols) return ESL_INVALID_ARGUMENT;
  }
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  ctx->n_lanes = n_lanes;
  const size_t R = ctx->rec_size;
  // The instances the slots touch, each with its slots: a lane re-derives
  // every touched instance once, with all of its overrides in place; the
  // device derives every lane's (derive.cu) from the nominal records.
  std::vector<DeriveItem> items;
  std::vector<DeriveSlot> dslots;
  {
    std::vector<std::pair<uint64_t, uint32_t>> keyed;  // (batch, inst) key, slot
    for (uint32_t k = 0; k < n_slots; ++k) keyed.push_back({(uint64_t(slots[k].batch) << 32) | slots[k].inst, k});
    std::stable_sort(keyed.begin(), keyed.end(),
                     [](const auto& a, const auto& b) { return a.first < b.first; });
    for (size_t i = 0; i < keyed.size();) {
      const uint32_t b = uint32_t(keyed[i].first >> 32), inst = uint32_t(keyed[i].first);
      const HostBatch& B = ctx->bats[b];
      DeriveItem it{};
      it.type = B.type;
      it.np = B.np;
      it.rec_at = B.rec_off + inst;
      it.stride = B.count;
      it.prm_at = ctx->prm_off[b] + inst * B.np;
      it.slot0 = uint32_t(dslots.size());
      for (; i < keyed.size() && keyed[i].first == ((uint64_t(b) << 32) | inst); ++i)
        dslots.push_back({slots[keyed[i].second].param, cols ? cols[keyed[i].second] : keyed[i].second});
      it.slot1 = uint32_t(dslots.size());
      items.push_back(it);
    }
  }
  ESL_CUDA(ctx->d_rec.ensure(size_t(n_lanes) * R * 8));
  if (!items.empty()) {
    ESL_CUDA(upload(ctx->d_derive_items, items, s));
    ESL_CUDA(upload(ctx->d_derive_slots, dslots, s));
    ESL_CUDA(ctx->d_values.ensure(size_t(n_lanes) * n_cols * 8));
    ESL_CUDA(cudaMemcpyAsync(ctx->d_values.p, values, size_t(n_lanes) * n_cols * 8, cudaMemcpyHostToDevice, s));
  }
  ESL_CUDA(launch_derive_lanes(ctx->d_rec_nominal.as<double>(), uint32_t(R), ctx->d_derive_items.as<DeriveItem>(),
                               uint32_t(items.size()), ctx->d_derive_slots.as<DeriveSlot>(),
                               ctx->d_params.as<double>(), ctx->d_values.as<double>(), n_cols, n_lanes,
                               ctx->d_rec.as<double>(), s));
  ctx->rec_lane0.resize(R);
  ESL_CUDA(cudaMemcpyAsync(ctx->rec_lane0.data(), ctx->d_rec.p, R * 8, cudaMemcpyDeviceToHost, s));
  ESL_CUDA(cudaStreamSynchronize(s));
  ctx->topo.rec_size = ctx->rec_size;
  ctx->peel.clear();
  return ensure_lane_buffers(ctx);
}

namespace {

// Every lane's start state (cold: zero with the junction seeds, op.zig
// coldStart; warm: x with limiting off) and, on a context's first solve,
// the lead tape from lane 0's first Jacobian. Leaves the lane view in L.
int32_t prepare_dc(esl_ctx* ctx, const esl_newton_opts* opts, double* d_x, int cold, uint32_t* d_iters,
                   uint32_t* d_status, esl_stats* st, LaneDev& L, uint32_t* d_rung = nullptr) {
  cudaStream_t s = ctx->stream;
  if (st) std::memset(st, 0, sizeof(*st));
  // Per-lane start state, set on the device (lane_init_kernel): cold lanes
  // start at zero with the junction seeds (op.zig coldStart), warm lanes at
  // x with limiting off; operating-point lanes (d_rung given) on the
  // ladder's first rung.
  ctx->peel.clear();
  L = lane_view(ctx, 0);
  L.x = d_x;
  L.iters = d_iters;
  L.status = d_status;
  if (d_rung) {
    const size_t N = ctx->n_lanes;
    ESL_CUDA(ctx->d_ladder.ensure(N * sizeof(LadderDev)));
    ESL_CUDA(ctx->d_x_good.ensure(N * ctx->pat.n * 8));
    L.ladder = ctx->d_ladder.as<LadderDev>();
    L.x_good = ctx->d_x_good.as<double>();
    L.rung_out = d_rung;
  }
  ESL_CUDA(launch_lane_init(ctx->topo, L, cold != 0, opts->init_fix != 0, s));
  if (!ctx->have_tape) {
    // The lead lane's first Jacobian, factored on the host into the tape.
    ESL_CUDA(lead_jacobian(ctx, L, ctx->d_a_vals.as<double>()));
    std::vector<double> a0(ctx->pat.nnz());
    ESL_CUDA(cudaMemcpyAsync(a0.data(), ctx->d_a_vals.p, a0.size() * 8, cudaMemcpyDeviceToHost, s));
    ESL_CUDA(cudaStreamSynchronize(s));
    if (int32_t rc = build_tape_from(ctx, a0.data())) return rc;
  }
  return ESL_OK;
}

}  // namespace

}  // extern "C"

namespace {

// The DC lanes' solve: every lane's Newton run (a plain DC solve), or every
// lane's operating point through op.zig's ladder (d_rung given), with the
// host serving the lanes that pause for a factor of their own.
int32_t dc_solve(esl_ctx* ctx, const esl_newton_opts* opts, double* d_x, int cold, uint32_t* d_iters,
                 uint32_t* d_status, uint32_t* d_rung, esl_stats* st) {
  cudaStream_t s = ctx->stream;
  const uint32_t N = ctx->n_lanes;
  LaneDev L;
  if (int32_t rc = prepare_dc(ctx, opts, d_x, cold, d_iters, d_status, st, L, d_rung)) return rc;
  LaneOpts o{opts->reltol, opts->abstol, opts->vntol, opts->residual_tol, opts->gmin, opts->max_iter, opts->init_fix,
             opts->iter_cap, d_rung ? 1u : 0u};
  // operating-point lanes run the FP64 form (warp or block lanes)
  const bool block = d_rung ? (ctx->path == ESL_PATH_BLOCK || !ctx->warp_ok) : use_block(ctx);
  if (!block && !ctx->warp_ok) return warp_only(ctx);
  if (ctx->path == ESL_PATH_WARP && block)
    return ctx->fail(ESL_NOT_ELIGIBLE, ctx->warp_ok ? "the warp lanes solve in FP64 only" : "the tape exceeds the warp lanes");
  const bool mixed = ctx->precision == ESL_PREC_MIXED && !d_rung;
  BlockDev D{};
  if (block) {
    if (int32_t rc = block_view(ctx, mixed, N, D)) return rc;
    if (D.refine_out) ESL_CUDA(cudaMemsetAsync(D.refine_out, 0, size_t(N) * 4, s));
    if (D.prof) ESL_CUDA(cudaMemsetAsync(D.prof, 0, kBlockPhases * sizeof(unsigned long long), s));
  }
  const bool b3 = topo_has_b3(ctx->topo);
  auto launch = [&](const LaneDev& LL) {
    return block ? launch_dc_block(D, LL, o, mixed, b3, s)
                 : launch_dc_newton(ctx->topo, LL, o, lanes_per_cta(ctx, N, ctx->lanes_eff), s);
  };
  ESL_CUDA(cudaEventRecord(ctx->ev0, s));
  ESL_CUDA(launch(L));
  uint32_t launches = 1;
  for (;;) {
    bool any = false;
    if (int32_t rc = serve_pauses(ctx, L, st, &any)) return rc;
    if (!any) break;
    LaneDev R = L;
    R.resume = 1;
    ESL_CUDA(launch(R));
    ++launches;
  }
  ESL_CUDA(cudaEventRecord(ctx->ev1, s));
  ESL_CUDA(cudaEventSynchronize(ctx->ev1));
  if (st) {
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    st->kernel_ms = ms;
    st->launches = launches;
    st->lanes = N;
    st->path = block ? ESL_PATH_BLOCK : ESL_PATH_WARP;
    std::vector<uint32_t> status(N);
    ESL_CUDA(cudaMemcpy(status.data(), d_status, N * 4, cudaMemcpyDeviceToHost));
    for (uint32_t v : status) st->converged += v == kConverged;
    if (D.refine_out) {
      std::vector<uint32_t> ref(N);
      ESL_CUDA(cudaMemcpy(ref.data(), D.refine_out, N * 4, cudaMemcpyDeviceToHost));
      for (uint32_t v : ref) st->refinements += v;
    }
  }
  return ESL_OK;
}

}  // namespace

extern "C" {

int32_t esl_dc_solve_device(esl_ctx* ctx, const esl_newton_opts* opts, double* d_x, int cold,
                            uint32_t* d_iters, uint32_t* d_status, esl_stats* st) {
  if (!ctx || !opts || !d_x || ctx->n_lanes == 0) return ESL_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  return dc_solve(ctx, opts, d_x, cold, d_iters, d_status, nullptr, st);
}

int32_t esl_op_solve_device(esl_ctx* ctx, const esl_newton_opts* opts, double* d_x, uint32_t* d_iters,
                            uint32_t* d_status, uint32_t* d_rung, esl_stats* st) {
  if (!ctx || !opts || !d_x || !d_iters || !d_status || !d_rung || ctx->n_lanes == 0) return ESL_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  // the plain rung is a cold operating point: MODEINITJCT seeds, then INITFIX
  esl_newton_opts o = *opts;
  o.init_fix = 1;
  return dc_solve(ctx, &o, d_x, 1, d_iters, d_status, d_rung, st);
}

int32_t esl_op_solve(esl_ctx* ctx, const esl_newton_opts* opts, double* x_out, uint32_t* iters,
                     uint32_t* status, uint32_t* rung, esl_stats* st) {
  if (!ctx || !opts || !x_out || ctx->n_lanes == 0) return ESL_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  const size_t N = ctx->n_lanes, n = ctx->pat.n;
  if (int32_t rc = ensure_lane_buffers(ctx)) return rc;
  DevBuf d_rung;
  ESL_CUDA(d_rung.ensure(N * 4));
  if (int32_t rc = esl_op_solve_device(ctx, opts, ctx->d_x.as<double>(), ctx->d_iters.as<uint32_t>(),
                                       ctx->d_status.as<uint32_t>(), d_rung.as<uint32_t>(), st))
    return rc;
  ESL_CUDA(cudaMemcpyAsync(x_out, ctx->d_x.p, N * n * 8, cudaMemcpyDeviceToHost, ctx->stream));
  if (iters) ESL_CUDA(cudaMemcpyAsync(iters, ctx->d_iters.p, N * 4, cudaMemcpyDeviceToHost, ctx->stream));
  if (status) ESL_CUDA(cudaMemcpyAsync(status, ctx->d_status.p, N * 4, cudaMemcpyDeviceToHost, ctx->stream));
  if (rung) ESL_CUDA(cudaMemcpyAsync(rung, d_rung.p, N * 4, cudaMemcpyDeviceToHost, ctx->stream));
  ESL_CUDA(cudaStreamSynchronize(ctx->stream));
  return ESL_OK;
}

// Allocation-free variant of esl_dc_solve_device: the same fused kernel, with
// the per-lane Newton state and hand-off buffers carved from the fixed device
// array of newton.cu instead of the context's allocations, and the lane start
// state written by a kernel instead of host vectors. Error text goes into the
// context's message buffer, reserved on the first call.
int32_t esl_dc_solve_device_static(esl_ctx* ctx, const esl_newton_opts* opts, double* d_x, int cold,
                                   uint32_t* d_iters, uint32_t* d_status, uint32_t* n_paused) {
  if (!ctx) return ESL_INVALID_ARGUMENT;
  constexpr size_t kErrCap = 256;
  if (ctx->err.capacity() < kErrCap) ctx->err.reserve(kErrCap);
  char msg[kErrCap];
  auto fail = [&](int32_t code, const char* text) {
    ctx->err.assign(text, std::min(std::strlen(text), kErrCap - 1));
    return code;
  };
  auto cuda = [&](cudaError_t e, const char* where) {
    std::snprintf(msg, sizeof msg, "%s: %s", where, cudaGetErrorString(e));
    return fail(ESL_DEVICE_FAULT, msg);
  };
  if (n_paused) *n_paused = 0;
  if (!opts || !d_x || !d_iters || !d_status || ctx->n_lanes == 0)
    return fail(ESL_INVALID_ARGUMENT, "null argument or no lanes set");
  if (!ctx->have_tape)
    return fail(ESL_NOT_ELIGIBLE, "no pivot tape yet: the first solve of a context must be esl_dc_solve_device");
  if (!ctx->warp_ok || use_block(ctx))
    return fail(ESL_NOT_ELIGIBLE, "the allocation-free entry runs the warp lanes in FP64 only");
  if (cudaError_t e = cudaSetDevice(ctx->device)) return cuda(e, "cudaSetDevice");
  void* base = nullptr;
  if (cudaError_t e = static_scratch(&base)) return cuda(e, "cudaGetSymbolAddress(lane scratch)");

  // Carve: the paused-lane counter, then each per-lane plane on 256 bytes.
  const size_t N = ctx->n_lanes, n = ctx->pat.n, nnz = ctx->pat.nnz();
  const size_t nlim = std::max<size_t>(ctx->nlim, 1);
  size_t at = 256;
  auto carve = [&](size_t bytes) {
    const size_t off = at;
    at += (bytes + 255) & ~size_t(255);
    return static_cast<unsigned char*>(base) + off;
  };
  LaneDev L{};
  L.n_lanes = ctx->n_lanes;
  L.rec = ctx->d_rec.as<double>();
  L.x = d_x;
  L.iters = d_iters;
  L.status = d_status;
  L.n_paused = static_cast<uint32_t*>(base);
  L.a_vals = reinterpret_cast<double*>(carve(N * nnz * 8));
  L.rhs = reinterpret_cast<double*>(carve(N * n * 8));
  L.dx = reinterpret_cast<double*>(carve(N * n * 8));
  L.diag = reinterpret_cast<double*>(carve(N * n * 8));
  L.lim = reinterpret_cast<double*>(carve(N * nlim * 8));
  L.limit = reinterpret_cast<double*>(carve(N * 8));
  L.flags = reinterpret_cast<uint32_t*>(carve(N * 4));
  L.lim_active = reinterpret_cast<uint32_t*>(carve(N * 4));
  if (at > kStaticScratchBytes) {
    std::snprintf(msg, sizeof msg,
                  "%zu lanes need %zu bytes of lane scratch, above the fixed %zu bytes: use fewer lanes per call",
                  N, at, kStaticScratchBytes);
    return fail(ESL_INVALID_ARGUMENT, msg);
  }
  const LaneOpts o{opts->reltol, opts->abstol, opts->vntol, opts->residual_tol, opts->gmin, opts->max_iter,
                   opts->init_fix, opts->iter_cap};
  cudaStream_t s = ctx->stream;
  if (cudaError_t e = launch_lane_init(ctx->topo, L, cold != 0, opts->init_fix != 0, s))
    return cuda(e, "lane_init_kernel");
  if (cudaError_t e = launch_dc_newton(ctx->topo, L, o, lanes_per_cta(ctx, N, ctx->lanes_eff), s)) return cuda(e, "dc_newton_kernel");
  uint32_t paused = 0;
  if (cudaError_t e = cudaMemcpyAsync(&paused, L.n_paused, 4, cudaMemcpyDeviceToHost, s))
    return cuda(e, "read paused-lane count");
  if (cudaError_t e = cudaStreamSynchronize(s)) return cuda(e, "cudaStreamSynchronize");
  if (n_paused) *n_paused = paused;
  if (paused) {
    std::snprintf(msg, sizeof msg,
                  "%u lanes left the lead pivot tape (status ESL_LANE_NEED_SOLVE); their host factor "
                  "needs memory: solve those points with esl_dc_solve_device",
                  paused);
    return fail(ESL_NOT_ELIGIBLE, msg);
  }
  return ESL_OK;
}

namespace {

// The lead tape from lane 0's cold-start Jacobian (x = 0, junction seeds),
// as the first DC solve builds it.
int32_t ensure_tape_cold(esl_ctx* ctx) {
  if (ctx->have_tape) return ESL_OK;
  cudaStream_t s = ctx->stream;
  const uint32_t n = ctx->pat.n;
  std::vector<double> lim(std::max<uint32_t>(ctx->nlim, 1), 0.0);
  for (const auto& B : ctx->bats) {
    const double* rec = &ctx->rec_lane0[B.rec_off];
    if (B.type == kD)
      for (uint32_t i = 0; i < B.count; ++i) lim[B.lim_off + i] = rec[kDVcrit * B.count + i];
    if (B.type == kM)
      for (uint32_t i = 0; i < B.count; ++i) {
        lim[B.lim_off + 3 * i] = rec[kMSeedVgs * B.count + i];
        lim[B.lim_off + 3 * i + 1] = 0.0;
        lim[B.lim_off + 3 * i + 2] = -1.0;
      }
    if (B.type == kB3)
      for (uint32_t i = 0; i < B.count; ++i) {
        lim[B.lim_off + 3 * i] = rec[kB3SeedVgs * B.count + i];
        lim[B.lim_off + 3 * i + 1] = 0.1;
        lim[B.lim_off + 3 * i + 2] = 0.0;
      }
  }
  const uint32_t act = ctx->nlim ? 1u : 0u;
  ESL_CUDA(cudaMemsetAsync(ctx->d_x.p, 0, size_t(n) * 8, s));
  ESL_CUDA(cudaMemcpyAsync(ctx->d_lim.p, lim.data(), lim.size() * 8, cudaMemcpyHostToDevice, s));
  ESL_CUDA(cudaMemcpyAsync(ctx->d_lim_active.p, &act, 4, cudaMemcpyHostToDevice, s));
  LaneDev L = lane_view(ctx, 0);
  ESL_CUDA(lead_jacobian(ctx, L, ctx->d_a_vals.as<double>()));
  std::vector<double> a0(ctx->pat.nnz());
  ESL_CUDA(cudaMemcpyAsync(a0.data(), ctx->d_a_vals.p, a0.size() * 8, cudaMemcpyDeviceToHost, s));
  ESL_CUDA(cudaStreamSynchronize(s));
  return build_tape_from(ctx, a0.data());
}

int32_t tran_view(esl_ctx* ctx, const esl_tran_opts* o, TranDev& P, LaneOpts& lo) {
  if (!o || !(o->t_stop > 0) || !(o->t_step > 0)) return ctx->fail(ESL_INVALID_ARGUMENT, "t_stop and t_step must be positive");
  if (ctx->has_meyer)
    return ctx->fail(ESL_NOT_ELIGIBLE, "MOS1 with TOX: the bias-dependent Meyer gate capacitance is not built");
  P = TranDev{};
  P.t_stop = o->t_stop;
  P.t_step = o->t_step;
  // src/frontend/analyses.zig:534: DELMAX, else min(TSTEP, span / 50)
  P.dt_max = o->t_max > 0 ? o->t_max : std::min(o->t_step, o->t_stop / 50.0);
  P.dt_min = o->dt_min > 0 ? o->dt_min : 1e-18;
  P.reltol = o->reltol;
  P.abstol = o->abstol;
  P.vntol = o->vntol;
  P.chgtol = o->chgtol;
  P.trtol = o->trtol;
  P.max_steps = o->max_steps ? o->max_steps : 1000000000u;
  lo = LaneOpts{o->reltol, o->abstol, o->vntol, std::numeric_limits<double>::infinity(), 0.0, 100, 0, 0};
  return ESL_OK;
}

}  // namespace

}  // extern "C"

namespace {

// One transient launch over every lane, then the host factors of the lanes
// that paused (serve_pauses) and resume launches until none pauses.
// The transient on the block lanes (a CTA per lane, FP64 or mixed
// precision): one persistent launch, every lane's run state in the CTA's
// part of the transient slab. Lanes whose factor leaves the lead tape stop
// (kTranLeftTape): no host factor on this path.
int32_t run_tran_block(esl_ctx* ctx, LaneDev L, TranDev P, const LaneOpts& lo) {
  cudaStream_t s = ctx->stream;
  const uint32_t N = ctx->n_lanes;
  if (P.meas) return ctx->fail(ESL_NOT_ELIGIBLE, "the block transient lanes stream no measure cards");
  const bool mixed = ctx->precision == ESL_PREC_MIXED;
  BlockDev D{};
  if (int32_t rc = block_view(ctx, mixed, N, D)) return rc;
  if (mixed) ESL_CUDA(cudaMemsetAsync(D.refine_out, 0, size_t(N) * 4, s));
  ESL_CUDA(ctx->d_tran_slab.ensure(size_t(D.grid) * tran_block_slab(ctx->topo) * 8));
  ESL_CUDA(ctx->d_x_good.ensure(size_t(N) * ctx->topo.n * 8));
  L.x_good = ctx->d_x_good.as<double>();
  ESL_CUDA(cudaMemsetAsync(L.status, 0, size_t(N) * 4, s));
  std::memset(&ctx->last_peels, 0, sizeof(ctx->last_peels));
  ESL_CUDA(cudaEventRecord(ctx->ev0, s));
  ESL_CUDA(launch_tran_block(D, L, P, lo, mixed, topo_has_b3(ctx->topo), ctx->d_tran_slab.as<double>(), s));
  ctx->last_peels.launches = 1;
  ESL_CUDA(cudaEventRecord(ctx->ev1, s));
  ESL_CUDA(cudaEventSynchronize(ctx->ev1));
  ctx->last_tran_refinements = 0;
  if (mixed) {
    std::vector<uint32_t> ref(N);
    ESL_CUDA(cudaMemcpyAsync(ref.data(), D.refine_out, size_t(N) * 4, cudaMemcpyDeviceToHost, s));
    ESL_CUDA(cudaStreamSynchronize(s));
    for (uint32_t v : ref) ctx->last_tran_refinements += v;
  }
  return ESL_OK;
}

int32_t run_tran(esl_ctx* ctx, LaneDev L, TranDev P, const LaneOpts& lo, uint32_t lpb) {
  cudaStream_t s = ctx->stream;
  const uint32_t N = ctx->n_lanes;
  const size_t bd = size_t(ctx->topo.tran_doubles) + size_t(kMeasDoubles) * P.n_meas + kTranSaveRegs;
  ESL_CUDA(ctx->d_tran_state.ensure(size_t(N) * kTranStateN * 4));
  ESL_CUDA(ctx->d_tran_save.ensure(size_t(N) * bd * 8));
  P.tstate = ctx->d_tran_state.as<uint32_t>();
  P.tsave = ctx->d_tran_save.as<double>();
  // the operating point's ladder: its state across pauses, its last good point
  ESL_CUDA(ctx->d_ladder.ensure(size_t(N) * sizeof(LadderDev)));
  ESL_CUDA(ctx->d_x_good.ensure(size_t(N) * ctx->topo.n * 8));
  L.ladder = ctx->d_ladder.as<LadderDev>();
  L.x_good = ctx->d_x_good.as<double>();
  ESL_CUDA(cudaMemsetAsync(L.status, 0, size_t(N) * 4, s));
  ESL_CUDA(cudaMemsetAsync(L.flags, 0, size_t(N) * 4, s));
  ESL_CUDA(cudaMemsetAsync(L.n_paused, 0, 4, s));
  ctx->peel.clear();
  std::memset(&ctx->last_peels, 0, sizeof(ctx->last_peels));
  ESL_CUDA(ctx->d_next_lane.ensure(sizeof(uint32_t)));
  P.next_lane = ctx->d_next_lane.as<uint32_t>();
  ESL_CUDA(cudaEventRecord(ctx->ev0, s));
  ESL_CUDA(launch_tran(ctx->topo, L, P, lo, lpb, s));
  ctx->last_peels.launches = 1;
  for (;;) {
    bool any = false;
    if (int32_t rc = serve_pauses(ctx, L, &ctx->last_peels, &any)) return rc;
    if (!any) break;
    LaneDev R = L;
    R.resume = 1;
    ESL_CUDA(launch_tran(ctx->topo, R, P, lo, lpb, s));
    ++ctx->last_peels.launches;
  }
  ESL_CUDA(cudaEventRecord(ctx->ev1, s));
  ESL_CUDA(cudaEventSynchronize(ctx->ev1));
  return ESL_OK;
}

}  // namespace

extern "C" {

int32_t esl_tran_device(esl_ctx* ctx, const esl_tran_opts* opts, double* d_x, uint32_t* d_stats,
                        const uint32_t* d_probes, uint32_t n_probes, uint32_t max_pts, double* d_t,
                        double* d_v, uint32_t* d_n_pts, float* ms) {
  if (!ctx || !d_x || !d_stats || ctx->n_lanes == 0) return ESL_INVALID_ARGUMENT;
  if (max_pts && (!d_probes || !d_t || !d_v || !d_n_pts)) return ESL_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  TranDev P;
  LaneOpts lo;
  if (int32_t rc = tran_view(ctx, opts, P, lo)) return rc;
  if (int32_t rc = ensure_tape_cold(ctx)) return rc;
  // the block lanes when asked for, for mixed precision (the warp lanes are
  // FP64), or when a warp lane cannot hold the run
  const bool block = ctx->path == ESL_PATH_BLOCK || ctx->precision == ESL_PREC_MIXED || !ctx->warp_ok ||
                     ctx->tran_lanes_eff == 0;
  P.stats = d_stats;
  P.n_probes = max_pts ? n_probes : 0;
  P.max_pts = max_pts;
  P.probes = d_probes;
  P.out_t = max_pts ? d_t : nullptr;
  P.out_v = d_v;
  P.n_pts = max_pts ? d_n_pts : nullptr;
  LaneDev L = lane_view(ctx, 0);
  L.x = d_x;
  if (block) {
    if (int32_t rc = run_tran_block(ctx, L, P, lo)) return rc;
  } else if (int32_t rc = run_tran(ctx, L, P, lo, lanes_per_cta(ctx, ctx->n_lanes, ctx->tran_lanes_eff))) {
    return rc;
  }
  if (ms) cudaEventElapsedTime(ms, ctx->ev0, ctx->ev1);
  return ESL_OK;
}

int32_t esl_dc_sweep_device(esl_ctx* ctx, const esl_slot* slot, const double* values, uint32_t n_pts,
                            const esl_newton_opts* opts, double* d_x, uint32_t* d_iters, uint8_t* d_conv,
                            uint32_t* d_status, float* ms) {
  if (!ctx || !slot || !values || !opts || !d_x || !d_iters || !d_conv || !d_status || n_pts == 0 ||
      ctx->n_lanes == 0)
    return ESL_INVALID_ARGUMENT;
  if (slot->batch >= ctx->bats.size()) return ctx->fail(ESL_INVALID_ARGUMENT, "swept slot: no such batch");
  const HostBatch& SB = ctx->bats[slot->batch];
  if (slot->inst >= SB.count) return ctx->fail(ESL_INVALID_ARGUMENT, "swept slot: no such instance");
  if ((SB.type != kV && SB.type != kI) || slot->param != 0)
    return ctx->fail(ESL_NOT_ELIGIBLE, "a sweep lane sweeps a V or I source's DC value (parameter 0)");
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  if (!ctx->have_tape) {
    // The lead tape from lane 0's cold Jacobian at the sweep's first point
    // (the first Jacobian the sweep solves), its source set there for the
    // assembly and restored after.
    double* src = ctx->d_rec.as<double>() + SB.rec_off + slot->inst;
    const double first = values[0], keep = ctx->rec_lane0[SB.rec_off + slot->inst];
    ESL_CUDA(cudaMemcpyAsync(src, &first, 8, cudaMemcpyHostToDevice, s));
    const int32_t rc = ensure_tape_cold(ctx);
    ESL_CUDA(cudaMemcpyAsync(src, &keep, 8, cudaMemcpyHostToDevice, s));
    ESL_CUDA(cudaStreamSynchronize(s));
    if (rc) return rc;
  }
  if (int32_t rc = warp_only(ctx)) return rc;
  const TopoDev& T = ctx->topo;
  const size_t lane_bytes = size_t(sweep_doubles(T)) * 8, room = size_t(227) * 1024;
  if (T.prog_bytes + lane_bytes > room) return ctx->fail(ESL_NOT_ELIGIBLE, "a sweep lane exceeds a CTA's shared memory");
  const uint32_t fit = std::max<uint32_t>(1, std::min<uint32_t>(8, uint32_t((room - T.prog_bytes) / lane_bytes)));
  ESL_CUDA(ctx->d_sweep_values.ensure(size_t(n_pts) * 8));
  ESL_CUDA(cudaMemcpyAsync(ctx->d_sweep_values.p, values, size_t(n_pts) * 8, cudaMemcpyHostToDevice, s));
  SweepDev P{};
  P.values = ctx->d_sweep_values.as<double>();
  P.n_pts = n_pts;
  P.src = T.b[slot->batch].src_off + slot->inst;
  P.x_out = d_x;
  P.iters = d_iters;
  P.conv = d_conv;
  P.status = d_status;
  const LaneOpts o{opts->reltol, opts->abstol, opts->vntol, opts->residual_tol, opts->gmin, opts->max_iter, 0, 0};
  const uint32_t N = ctx->n_lanes;
  ESL_CUDA(ctx->d_sweep_state.ensure(size_t(N) * kSweepStateN * 4));
  ESL_CUDA(ctx->d_sweep_rows.ensure(size_t(N) * 2 * T.n * 8));
  P.state = ctx->d_sweep_state.as<uint32_t>();
  P.rows = ctx->d_sweep_rows.as<double>();
  // every lane running on the lead tape; lanes that pause are served on
  // the host (serve_pauses) and resumed where they stopped
  LaneDev L = lane_view(ctx, 0);
  ESL_CUDA(cudaMemsetAsync(L.status, 0, size_t(N) * 4, s));
  ESL_CUDA(cudaMemsetAsync(L.flags, 0, size_t(N) * 4, s));
  ESL_CUDA(cudaMemsetAsync(L.n_paused, 0, 4, s));
  // a cold point's ladder: its state across pauses, its last good point
  ESL_CUDA(ctx->d_ladder.ensure(size_t(N) * sizeof(LadderDev)));
  ESL_CUDA(ctx->d_x_good.ensure(size_t(N) * T.n * 8));
  L.ladder = ctx->d_ladder.as<LadderDev>();
  L.x_good = ctx->d_x_good.as<double>();
  ctx->peel.clear();
  ESL_CUDA(ctx->d_next_lane.ensure(sizeof(uint32_t)));
  P.next_lane = ctx->d_next_lane.as<uint32_t>();
  const uint32_t lpb = lanes_per_cta(ctx, N, fit);
  ESL_CUDA(cudaEventRecord(ctx->ev0, s));
  std::memset(&ctx->last_peels, 0, sizeof(ctx->last_peels));
  ESL_CUDA(launch_sweep(T, L, P, o, lpb, s));
  ctx->last_peels.launches = 1;
  for (;;) {
    bool any = false;
    if (int32_t rc = serve_pauses(ctx, L, &ctx->last_peels, &any)) return rc;
    if (!any) break;
    LaneDev R = L;
    R.resume = 1;
    ESL_CUDA(launch_sweep(T, R, P, o, lpb, s));
    ++ctx->last_peels.launches;
  }
  ESL_CUDA(cudaEventRecord(ctx->ev1, s));
  ESL_CUDA(cudaEventSynchronize(ctx->ev1));
  if (ms) cudaEventElapsedTime(ms, ctx->ev0, ctx->ev1);
  return ESL_OK;
}

static_assert(sizeof(esl_meas_clause) == sizeof(MeasClauseDev) && sizeof(esl_measure) == sizeof(MeasDev),
              "esl_measure and the device card share one layout");

int32_t esl_tran_meas_device(esl_ctx* ctx, const esl_tran_opts* opts, const esl_measure* meas, uint32_t n_meas,
                             int early_stop, double* d_x, uint32_t* d_stats, double* d_values, float* ms) {
  if (!ctx || !meas || !d_x || !d_stats || !d_values || n_meas == 0 || ctx->n_lanes == 0)
    return ESL_INVALID_ARGUMENT;
  if (n_meas > kMaxMeas) return ctx->fail(ESL_INVALID_ARGUMENT, "at most 32 measure cards");
  for (uint32_t c = 0; c < n_meas; ++c) {
    const esl_measure& m = meas[c];
    if (m.kind > ESL_MEAS_DERIV) return ctx->fail(ESL_INVALID_ARGUMENT, "unknown measure kind");
    if (m.a.unknown >= ctx->pat.n || (m.kind == ESL_MEAS_TRIG_TARG && m.b.unknown >= ctx->pat.n))
      return ctx->fail(ESL_INVALID_ARGUMENT, "measure probe out of range");
  }
  cudaSetDevice(ctx->device);
  TranDev P;
  LaneOpts lo;
  if (int32_t rc = tran_view(ctx, opts, P, lo)) return rc;
  if (int32_t rc = ensure_tape_cold(ctx)) return rc;
  if (int32_t rc = warp_only(ctx)) return rc;
  const TopoDev& T = ctx->topo;
  const size_t lane_bytes = (size_t(T.tran_doubles) + size_t(kMeasDoubles) * n_meas) * 8, room = size_t(227) * 1024;
  if (T.prog_bytes + lane_bytes > room) return ctx->fail(ESL_NOT_ELIGIBLE, "a transient lane exceeds a CTA's shared memory");
  const uint32_t fit = std::max<uint32_t>(1, std::min<uint32_t>(8, uint32_t((room - T.prog_bytes) / lane_bytes)));
  cudaStream_t s = ctx->stream;
  ESL_CUDA(ctx->d_meas.ensure(size_t(n_meas) * sizeof(esl_measure)));
  ESL_CUDA(cudaMemcpyAsync(ctx->d_meas.p, meas, size_t(n_meas) * sizeof(esl_measure), cudaMemcpyHostToDevice, s));
  P.stats = d_stats;
  P.meas = ctx->d_meas.as<MeasDev>();
  P.n_meas = n_meas;
  P.early_stop = early_stop ? 1u : 0u;
  P.meas_out = d_values;
  LaneDev L = lane_view(ctx, 0);
  L.x = d_x;
  if (int32_t rc = run_tran(ctx, L, P, lo, lanes_per_cta(ctx, ctx->n_lanes, fit))) return rc;
  if (ms) cudaEventElapsedTime(ms, ctx->ev0, ctx->ev1);
  return ESL_OK;
}

int32_t esl_tran(esl_ctx* ctx, const esl_tran_opts* opts, const uint32_t* probes, uint32_t n_probes,
                 uint32_t max_pts, double* t_out, double* v_out, uint32_t* n_pts, uint32_t* stats,
                 double* x_out, float* ms) {
  if (!ctx || !stats || !x_out || ctx->n_lanes == 0) return ESL_INVALID_ARGUMENT;
  if (max_pts && (!probes || !t_out || !v_out || !n_pts || n_probes == 0)) return ESL_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  const size_t N = ctx->n_lanes, n = ctx->pat.n;
  for (uint32_t k = 0; k < n_probes && max_pts; ++k)
    if (probes[k] >= n) return ctx->fail(ESL_INVALID_ARGUMENT, "probe index out of range");
  ESL_CUDA(ctx->d_tran_stats.ensure(N * kTsN * 4));
  if (max_pts) {
    ESL_CUDA(ctx->d_probes.ensure(size_t(n_probes) * 4));
    ESL_CUDA(ctx->d_tran_t.ensure(N * max_pts * 8));
    ESL_CUDA(ctx->d_tran_v.ensure(N * max_pts * n_probes * 8));
    ESL_CUDA(ctx->d_tran_n.ensure(N * 4));
    ESL_CUDA(cudaMemcpyAsync(ctx->d_probes.p, probes, size_t(n_probes) * 4, cudaMemcpyHostToDevice, s));
  }
  if (int32_t rc = esl_tran_device(ctx, opts, ctx->d_x.as<double>(), ctx->d_tran_stats.as<uint32_t>(),
                                   ctx->d_probes.as<uint32_t>(), n_probes, max_pts, ctx->d_tran_t.as<double>(),
                                   ctx->d_tran_v.as<double>(), ctx->d_tran_n.as<uint32_t>(), ms))
    return rc;
  ESL_CUDA(cudaMemcpyAsync(x_out, ctx->d_x.p, N * n * 8, cudaMemcpyDeviceToHost, s));
  ESL_CUDA(cudaMemcpyAsync(stats, ctx->d_tran_stats.p, N * kTsN * 4, cudaMemcpyDeviceToHost, s));
  if (max_pts) {
    ESL_CUDA(cudaMemcpyAsync(t_out, ctx->d_tran_t.p, N * max_pts * 8, cudaMemcpyDeviceToHost, s));
    ESL_CUDA(cudaMemcpyAsync(v_out, ctx->d_tran_v.p, N * max_pts * n_probes * 8, cudaMemcpyDeviceToHost, s));
    ESL_CUDA(cudaMemcpyAsync(n_pts, ctx->d_tran_n.p, N * 4, cudaMemcpyDeviceToHost, s));
  }
  ESL_CUDA(cudaStreamSynchronize(s));
  return ESL_OK;
}

namespace {

// Shared memory a topology's working set may take in a group launch (the
// group kernel keeps the work item's tables in static shared memory too).
constexpr size_t kGroupSmemRoom = size_t(227) * 1024 - 2048;

// The uneven batch on the block lanes: every context's lanes in one
// persistent launch (work items largest topology first), then each
// context's paused lanes served on the host and resumed on its own.
int32_t group_block(esl_ctx* const* ctxs, uint32_t n_ctx, const esl_newton_opts* opts,
                    const std::vector<LaneDev>& lanes, uint32_t* const* d_status, esl_stats* stats) {
  esl_ctx* c0 = ctxs[0];
  esl_ctx* ctx = c0;  // ESL_CUDA reports on the first context
  const bool mixed = c0->precision == ESL_PREC_MIXED;
  for (uint32_t c = 0; c < n_ctx; ++c)
    if ((ctxs[c]->precision == ESL_PREC_MIXED) != mixed || ctxs[c]->path == ESL_PATH_WARP)
      return c0->fail(ESL_INVALID_ARGUMENT, "a block-lane group runs every context in one precision");
  std::vector<BlockDev> Ds(n_ctx);
  bool b3 = false;
  size_t smem = 0, stride = 16;
  for (uint32_t c = 0; c < n_ctx; ++c) {
    esl_ctx* x = ctxs[c];
    // one op ring for the whole launch: rows of one op a thread for every
    // topology (a slab topology's wider rows would size every CTA's ring
    // for them); the context keeps these programs after the group
    if (int32_t rc = ensure_block(x)) return rc;
    if (x->bprog.row_k != 1) {
      if (int32_t rc = set_block_programs(x, 1)) return rc;
      ESL_CUDA(cudaStreamSynchronize(x->stream));
    }
    if (int32_t rc = block_view(x, mixed, x->n_lanes, Ds[c])) return rc;
    if (Ds[c].refine_out) ESL_CUDA(cudaMemsetAsync(Ds[c].refine_out, 0, size_t(x->n_lanes) * 4, x->stream));
    ESL_CUDA(cudaStreamSynchronize(x->stream));
    b3 |= topo_has_b3(x->topo);
  }
  // the group's own placement: the op ring of the widest op format after
  // the working sets that fit shared memory within the group room
  bool long_ops = false;
  for (uint32_t c = 0; c < n_ctx; ++c) long_ops |= Ds[c].op_bytes == 16;
  if (long_ops)
    for (uint32_t c = 0; c < n_ctx; ++c)
      if (Ds[c].op_bytes != 16) {
        // one op format per launch: the long words for every topology
        esl_ctx* x = ctxs[c];
        ESL_CUDA(upload(x->d_ba, block_words(x->bprog.a_ops, false), x->stream));
        ESL_CUDA(upload(x->d_bb, block_words(x->bprog.b_ops, false), x->stream));
        ESL_CUDA(upload(x->d_bf, block_words(x->bprog.f_ops, false), x->stream));
        ESL_CUDA(cudaStreamSynchronize(x->stream));
        x->block_op_bytes = 16;
        if (int32_t rc = block_view(x, mixed, x->n_lanes, Ds[c])) return rc;
      }
  uint32_t ring = 0;
  for (uint32_t c = 0; c < n_ctx; ++c) ring = std::max(ring, block_ring_bytes(long_ops ? 16 : 8, Ds[c].row_k));
  std::vector<BlockDev> Dg = Ds;
  for (uint32_t c = 0; c < n_ctx; ++c) {
    // each topology keeps its own placement (block_view's), the whole
    // working set in the CTA's slab when its shared part misses the room
    Dg[c].in_smem = Dg[c].in_smem && Dg[c].lane_bytes + ring <= kGroupSmemRoom;
    if (!Dg[c].in_smem && Dg[c].split) block_layout(ctxs[c]->topo, ctxs[c]->topo.nv, mixed, false, Dg[c]);
    if (Dg[c].in_smem) smem = std::max<size_t>(smem, Dg[c].lane_bytes);
    stride = std::max<size_t>(stride, Dg[c].split ? Dg[c].cold_bytes : Dg[c].in_smem ? 0 : Dg[c].lane_bytes);
  }
  const uint32_t ring_at = uint32_t((smem + 15) & ~size_t(15));
  smem = ring_at + ring;
  std::vector<uint32_t> order(n_ctx);
  for (uint32_t c = 0; c < n_ctx; ++c) order[c] = c;
  std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
    return ctxs[a]->prog.a_nops > ctxs[b]->prog.a_nops;
  });
  std::vector<uint2> items;
  for (uint32_t c : order)
    for (uint32_t l = 0; l < ctxs[c]->n_lanes; ++l) items.push_back(make_uint2(c, l));
  const int per_sm = block_group_occupancy(mixed, long_ops, b3, smem);
  const uint32_t grid = std::max<uint32_t>(1, std::min<uint32_t>(uint32_t(items.size()),
                                                                 uint32_t(c0->sms) * uint32_t(std::max(per_sm, 1))));
  cudaStream_t s = c0->stream;
  ESL_CUDA(upload(c0->d_group_blocks, Dg, s));
  ESL_CUDA(upload(c0->d_group_lanes, lanes, s));
  ESL_CUDA(upload(c0->d_group_items, items, s));
  ESL_CUDA(c0->d_next_lane.ensure(sizeof(uint32_t)));
  ESL_CUDA(c0->d_group_slab.ensure(size_t(grid) * stride));
  const LaneOpts o{opts->reltol, opts->abstol, opts->vntol, opts->residual_tol, opts->gmin, opts->max_iter,
                   opts->init_fix, opts->iter_cap};
  ESL_CUDA(cudaEventRecord(c0->ev0, s));
  ESL_CUDA(launch_dc_block_group(c0->d_group_blocks.as<BlockDev>(), c0->d_group_lanes.as<LaneDev>(),
                                 c0->d_group_items.as<uint2>(), uint32_t(items.size()),
                                 c0->d_next_lane.as<uint32_t>(), o, c0->d_group_slab.as<unsigned char>(), stride,
                                 smem, ring_at, grid, mixed, long_ops, b3, s));
  ESL_CUDA(cudaEventRecord(c0->ev1, s));
  ESL_CUDA(cudaEventSynchronize(c0->ev1));
  float ms = 0;
  cudaEventElapsedTime(&ms, c0->ev0, c0->ev1);
  for (uint32_t c = 0; c < n_ctx; ++c) {
    esl_ctx* x = ctxs[c];
    ctx = x;
    uint32_t launches = 1;
    for (;;) {
      bool any = false;
      if (int32_t rc = serve_pauses(x, lanes[c], stats ? &stats[c] : nullptr, &any)) return rc;
      if (!any) break;
      LaneDev R = lanes[c];
      R.resume = 1;
      ESL_CUDA(launch_dc_block(Ds[c], R, o, mixed, topo_has_b3(x->topo), x->stream));
      ++launches;
    }
    ESL_CUDA(cudaStreamSynchronize(x->stream));
    if (stats) {
      stats[c].kernel_ms = ms;
      stats[c].launches = launches;
      stats[c].lanes = x->n_lanes;
      stats[c].path = ESL_PATH_BLOCK;
      std::vector<uint32_t> status(x->n_lanes);
      ESL_CUDA(cudaMemcpy(status.data(), d_status[c], x->n_lanes * 4, cudaMemcpyDeviceToHost));
      for (uint32_t v : status) stats[c].converged += v == kConverged;
      if (Ds[c].refine_out) {
        std::vector<uint32_t> ref(x->n_lanes);
        ESL_CUDA(cudaMemcpy(ref.data(), Ds[c].refine_out, x->n_lanes * 4, cudaMemcpyDeviceToHost));
        for (uint32_t v : ref) stats[c].refinements += v;
      }
    }
  }
  return ESL_OK;
}

}  // namespace

int32_t esl_group_dc_solve_device(esl_ctx* const* ctxs, uint32_t n_ctx, const esl_newton_opts* opts,
                                  double* const* d_x, const int* cold, uint32_t* const* d_iters,
                                  uint32_t* const* d_status, esl_stats* stats) {
  if (!ctxs || n_ctx == 0 || !opts || !d_x || !d_iters || !d_status) return ESL_INVALID_ARGUMENT;
  esl_ctx* c0 = ctxs[0];
  for (uint32_t c = 0; c < n_ctx; ++c) {
    if (!ctxs[c] || ctxs[c]->n_lanes == 0 || !d_x[c] || !d_iters[c] || !d_status[c]) return ESL_INVALID_ARGUMENT;
    if (ctxs[c]->device != c0->device) return c0->fail(ESL_INVALID_ARGUMENT, "a group's contexts share one device");
  }
  cudaSetDevice(c0->device);
  esl_ctx* ctx = c0;  // ESL_CUDA reports on the first context
  std::vector<LaneDev> lanes(n_ctx);
  std::vector<TopoDev> topos(n_ctx);
  std::vector<uint32_t> cta_ctx, cta_first, lpb(n_ctx);
  size_t smem = 0;
  uint32_t max_lpb = 1;
  bool block = false;
  for (uint32_t c = 0; c < n_ctx; ++c) {
    esl_ctx* x = ctxs[c];
    if (int32_t rc = prepare_dc(x, opts, d_x[c], cold ? cold[c] : 0, d_iters[c], d_status[c],
                                stats ? &stats[c] : nullptr, lanes[c]))
      return rc;
    ESL_CUDA(cudaStreamSynchronize(x->stream));
    block |= use_block(x);
  }
  if (block) return group_block(ctxs, n_ctx, opts, lanes, d_status, stats);
  for (uint32_t c = 0; c < n_ctx; ++c) {
    esl_ctx* x = ctxs[c];
    if (int32_t rc = warp_only(x)) return rc;
    topos[c] = x->topo;
    lpb[c] = lanes_per_cta(x, x->n_lanes, x->lanes_eff);
    max_lpb = std::max(max_lpb, lpb[c]);
    smem = std::max(smem, size_t(x->topo.prog_bytes) + size_t(lpb[c]) * x->topo.smem_doubles * 8);
    for (uint32_t f = 0; f < x->n_lanes; f += lpb[c]) {
      cta_ctx.push_back(c);
      cta_first.push_back(f);
    }
  }
  if (smem > size_t(227) * 1024) return c0->fail(ESL_NOT_ELIGIBLE, "a group CTA exceeds shared memory");
  cudaStream_t s = c0->stream;
  ESL_CUDA(upload(c0->d_group_topo, topos, s));
  ESL_CUDA(upload(c0->d_group_lanes, lanes, s));
  ESL_CUDA(upload(c0->d_group_cta_ctx, cta_ctx, s));
  ESL_CUDA(upload(c0->d_group_cta_first, cta_first, s));
  ESL_CUDA(upload(c0->d_group_lpb, lpb, s));
  const LaneOpts o{opts->reltol, opts->abstol, opts->vntol, opts->residual_tol, opts->gmin, opts->max_iter,
                   opts->init_fix, opts->iter_cap};
  ESL_CUDA(cudaEventRecord(c0->ev0, s));
  ESL_CUDA(launch_dc_newton_group(c0->d_group_topo.as<TopoDev>(), c0->d_group_lanes.as<LaneDev>(),
                                  c0->d_group_cta_ctx.as<uint32_t>(), c0->d_group_cta_first.as<uint32_t>(),
                                  c0->d_group_lpb.as<uint32_t>(), uint32_t(cta_ctx.size()), max_lpb, smem, o,
                                  std::any_of(topos.begin(), topos.end(), topo_has_b3), s));
  ESL_CUDA(cudaEventRecord(c0->ev1, s));
  ESL_CUDA(cudaEventSynchronize(c0->ev1));
  float ms = 0;
  cudaEventElapsedTime(&ms, c0->ev0, c0->ev1);
  // lanes that left their tape: each context's host peels, then its own resume launches
  for (uint32_t c = 0; c < n_ctx; ++c) {
    esl_ctx* x = ctxs[c];
    ctx = x;
    uint32_t launches = 1;
    for (;;) {
      bool any = false;
      if (int32_t rc = serve_pauses(x, lanes[c], stats ? &stats[c] : nullptr, &any)) return rc;
      if (!any) break;
      LaneDev R = lanes[c];
      R.resume = 1;
      ESL_CUDA(launch_dc_newton(x->topo, R, o, lanes_per_cta(x, x->n_lanes, x->lanes_eff), x->stream));
      ++launches;
    }
    ESL_CUDA(cudaStreamSynchronize(x->stream));
    if (stats) {
      stats[c].kernel_ms = ms;
      stats[c].launches = launches;
      stats[c].lanes = x->n_lanes;
      std::vector<uint32_t> status(x->n_lanes);
      ESL_CUDA(cudaMemcpy(status.data(), d_status[c], x->n_lanes * 4, cudaMemcpyDeviceToHost));
      for (uint32_t v : status) stats[c].converged += v == kConverged;
    }
  }
  return ESL_OK;
}

int32_t esl_set_mode(esl_ctx* ctx, const esl_solve_mode* mode) {
  if (!ctx || !mode) return ESL_INVALID_ARGUMENT;
  if (mode->precision > ESL_PREC_MIXED || mode->path > ESL_PATH_BLOCK)
    return ctx->fail(ESL_INVALID_ARGUMENT, "unknown precision or path");
  const uint32_t width = mode->block_threads ? mode->block_threads : kBlockThreads;
  if (width != kBlockThreads) return ctx->fail(ESL_INVALID_ARGUMENT, "block_threads: 256 (or 0)");
  ctx->precision = mode->precision;
  ctx->path = mode->path;
  ctx->block_width = width;
  ctx->refine_tol = mode->refine_tol > 0.0 ? mode->refine_tol : 1e-12;
  ctx->refine_max = mode->refine_max ? mode->refine_max : 6;
  ctx->refine_skip = mode->refine_skip > 0.0 ? mode->refine_skip : 0.0;
  ctx->profile = mode->profile != 0;
  return ESL_OK;
}

int32_t esl_peel_counts(const esl_ctx* ctx, uint32_t* lanes, uint32_t* host_solves, uint32_t* launches) {
  if (!ctx) return ESL_INVALID_ARGUMENT;
  if (lanes) *lanes = ctx->last_peels.peeled;
  if (host_solves) *host_solves = ctx->last_peels.host_solves;
  if (launches) *launches = ctx->last_peels.launches;
  return ESL_OK;
}

int32_t esl_tran_refinements(const esl_ctx* ctx, uint64_t* corrections) {
  if (!ctx || !corrections) return ESL_INVALID_ARGUMENT;
  *corrections = ctx->last_tran_refinements;
  return ESL_OK;
}

int32_t esl_block_profile(esl_ctx* ctx, uint64_t* cycles) {
  if (!ctx || !cycles) return ESL_INVALID_ARGUMENT;
  if (!ctx->profile || !ctx->d_prof.p) return ctx->fail(ESL_INVALID_ARGUMENT, "no profiled block-lane solve yet");
  cudaSetDevice(ctx->device);
  ESL_CUDA(cudaMemcpy(cycles, ctx->d_prof.p, kBlockPhases * sizeof(uint64_t), cudaMemcpyDeviceToHost));
  return ESL_OK;
}

int32_t esl_block_info(esl_ctx* ctx, esl_block_info_t* info) {
  if (!ctx || !info || !ctx->have_tape) return ESL_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  if (int32_t rc = ensure_block(ctx)) return rc;
  std::memset(info, 0, sizeof(*info));
  info->width = kBlockThreads;
  info->a_rows = ctx->bprog.a_rows;
  info->b_rows = ctx->bprog.b_rows;
  info->f_rows = ctx->bprog.f_rows;
  info->a_levels = ctx->bprog.a_levels;
  info->a_nops = ctx->prog.a_nops;
  info->b_nops = ctx->prog.b_nops;
  info->ntv = ctx->prog.ntv;
  info->warp_ok = ctx->warp_ok;
  for (int m = 0; m < 2; ++m) {
    BlockDev D{};
    if (int32_t rc = block_view(ctx, m == 1, ctx->n_lanes ? ctx->n_lanes : 1, D)) return rc;
    info->lane_bytes[m] = D.lane_bytes;
    info->in_smem[m] = D.in_smem;
    info->ctas_per_sm[m] = uint32_t(std::max(
        0, block_occupancy(m == 1, D.op_bytes == 16, topo_has_b3(ctx->topo),
                           (D.in_smem ? D.lane_bytes : 0) + D.ring_bytes)));
    info->split[m] = D.split;
    info->cold_bytes[m] = D.cold_bytes;
    info->gather_terms = D.g_len;
    info->gather_cells = D.g_ncells;
  }
  return ESL_OK;
}

int32_t esl_autotune(esl_ctx* ctx, const esl_newton_opts* opts, const double* x0, uint32_t* lanes_per_block) {
  if (!ctx || !opts || ctx->n_lanes == 0) return ESL_INVALID_ARGUMENT;
  const size_t N = ctx->n_lanes, n = ctx->pat.n;
  std::vector<double> x(N * n);
  std::vector<uint32_t> it(N), st(N);
  esl_stats stats;
  // the first solve builds the tape (and fixes the lanes that fit per CTA)
  ctx->lanes_per_block = 0;
  if (int32_t rc = esl_dc_solve(ctx, opts, x0, x.data(), it.data(), st.data(), &stats)) return rc;
  uint32_t best = 0;
  float best_ms = 0;
  for (uint32_t cand : {1u, 2u, 4u, 8u}) {
    if (cand > ctx->lanes_eff) break;
    ctx->lanes_per_block = cand;
    float t = 0;
    for (int rep = 0; rep < 2; ++rep) {
      if (int32_t rc = esl_dc_solve(ctx, opts, x0, x.data(), it.data(), st.data(), &stats)) return rc;
      t = rep == 0 ? float(stats.kernel_ms) : std::min(t, float(stats.kernel_ms));
    }
    if (best == 0 || t < best_ms) {
      best = cand;
      best_ms = t;
    }
  }
  ctx->lanes_per_block = best;
  if (lanes_per_block) *lanes_per_block = best;
  return ESL_OK;
}

int32_t esl_dc_solve(esl_ctx* ctx, const esl_newton_opts* opts, const double* x0, double* x_out,
                     uint32_t* iters, uint32_t* status, esl_stats* st) {
  if (!ctx || !opts || !x_out || ctx->n_lanes == 0) return ESL_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  const size_t N = ctx->n_lanes, n = ctx->pat.n;
  if (x0) ESL_CUDA(cudaMemcpyAsync(ctx->d_x.p, x0, N * n * 8, cudaMemcpyHostToDevice, ctx->stream));
  if (int32_t rc = esl_dc_solve_device(ctx, opts, ctx->d_x.as<double>(), x0 == nullptr,
                                       ctx->d_iters.as<uint32_t>(), ctx->d_status.as<uint32_t>(), st))
    return rc;
  ESL_CUDA(cudaMemcpyAsync(x_out, ctx->d_x.p, N * n * 8, cudaMemcpyDeviceToHost, ctx->stream));
  if (iters) ESL_CUDA(cudaMemcpyAsync(iters, ctx->d_iters.p, N * 4, cudaMemcpyDeviceToHost, ctx->stream));
  if (status) ESL_CUDA(cudaMemcpyAsync(status, ctx->d_status.p, N * 4, cudaMemcpyDeviceToHost, ctx->stream));
  ESL_CUDA(cudaStreamSynchronize(ctx->stream));
  return ESL_OK;
}

int32_t esl_pattern(const esl_circuit* circuit, uint32_t* col_ptr, uint32_t* row_idx, size_t cap,
                    uint32_t* nnz) {
  if (!circuit || !col_ptr || !nnz) return ESL_INVALID_ARGUMENT;
  std::vector<HostBatch> bats;
  if (!read_circuit(circuit, bats)) return ESL_INVALID_ARGUMENT;
  Csc pat = build_pattern(bats, circuit->n);
  *nnz = pat.nnz();
  std::copy(pat.col_ptr.begin(), pat.col_ptr.end(), col_ptr);
  if (row_idx && cap >= pat.nnz()) std::copy(pat.row_idx.begin(), pat.row_idx.end(), row_idx);
  return cap >= pat.nnz() ? ESL_OK : ESL_INVALID_ARGUMENT;
}

int32_t esl_compile_tape(uint32_t n, const uint32_t* col_ptr, const uint32_t* row_idx, const double* lead,
                         esl_tape_info* info, uint32_t* q, uint32_t* pinv, uint32_t* amap, uint32_t* fill,
                         uint32_t* a_ops, uint32_t* b_ops, uint8_t* l_scaled) {
  if (!col_ptr || !row_idx || !lead || !info || n == 0) return ESL_INVALID_ARGUMENT;
  Csc pat;
  pat.n = n;
  pat.col_ptr.assign(col_ptr, col_ptr + n + 1);
  pat.row_idx.assign(row_idx, row_idx + col_ptr[n]);
  SparseLu lu;
  lu.init(&pat, order_columns(pat));
  lu.fill_cap = kRepivotFillCap;
  lu.keep_min = kGrowthLimit;
  if (!lu.factor(lead, kPivotTol)) return ESL_NOT_ELIGIBLE;
  Programs P = compile_tape(lu);
  info->nu = P.nu;
  info->nl = P.nl;
  info->ntv = P.ntv;
  info->n_fill = uint32_t(P.fill.size());
  info->a_rows = P.a_rows;
  info->a_levels = P.a_levels;
  info->a_nops = P.a_nops;
  info->b_rows = P.b_rows;
  info->b_levels = P.b_levels;
  info->b_nops = P.b_nops;
  info->flops = P.flops;
  info->has_void = P.has_void;
  if (q) std::copy(lu.q.begin(), lu.q.end(), q);
  if (pinv) std::copy(lu.pinv.begin(), lu.pinv.end(), pinv);
  if (amap) std::copy(P.amap.begin(), P.amap.end(), amap);
  if (fill) std::copy(P.fill.begin(), P.fill.end(), fill);
  auto words = [](const std::vector<Op>& ops, uint32_t* out) {
    for (size_t i = 0; i < ops.size(); ++i) {
      out[2 * i] = ops[i].w0;
      out[2 * i + 1] = ops[i].w1;
    }
  };
  if (a_ops) words(P.a_ops, a_ops);
  if (b_ops) words(P.b_ops, b_ops);
  if (l_scaled) std::copy(P.l_scaled.begin(), P.l_scaled.end(), l_scaled);
  return ESL_OK;
}

int32_t esl_lu_compiled_source(uint32_t n, const uint32_t* col_ptr, const uint32_t* row_idx, const double* lead,
                               uint32_t resident, char* buf, size_t cap, size_t* len) {
  if (!col_ptr || !row_idx || !lead || !len || n == 0) return ESL_INVALID_ARGUMENT;
  Csc pat;
  pat.n = n;
  pat.col_ptr.assign(col_ptr, col_ptr + n + 1);
  pat.row_idx.assign(row_idx, row_idx + col_ptr[n]);
  SparseLu lu;
  lu.init(&pat, order_columns(pat));
  lu.fill_cap = kRepivotFillCap;
  lu.keep_min = kGrowthLimit;
  if (!lu.factor(lead, kPivotTol)) return ESL_NOT_ELIGIBLE;
  Programs P = compile_tape(lu);
  if (P.has_void) return ESL_NOT_ELIGIBLE;
  const std::string src = compiled_lu_source(col_ptr[n], lu, P, resident);
  *len = src.size();
  if (buf && cap > 0) {
    const size_t k = std::min(cap - 1, src.size());
    std::memcpy(buf, src.data(), k);
    buf[k] = '\0';
  }
  return ESL_OK;
}

int32_t esl_tape(const esl_ctx* ctx, uint32_t* q, uint32_t* pinv, uint32_t* counts) {
  if (!ctx || !ctx->have_tape) return ESL_INVALID_ARGUMENT;
  const uint32_t n = ctx->pat.n;
  if (q) std::copy(ctx->lead.q.begin(), ctx->lead.q.end(), q);
  if (pinv) std::copy(ctx->lead.pinv.begin(), ctx->lead.pinv.begin() + n, pinv);
  if (counts) {
    counts[0] = ctx->prog.nl;
    counts[1] = ctx->prog.nu;
    counts[2] = ctx->prog.a_levels;
    counts[3] = ctx->prog.b_levels;
  }
  return ESL_OK;
}

int32_t esl_lu_lanes_device(esl_ctx* ctx, const double* lead, uint32_t n_lanes, const double* d_a,
                            const double* d_rhs, double* d_dx, uint8_t* d_bad, double* d_tv, float* ms) {
  if (!ctx || !d_a || !d_rhs || !d_dx || !d_bad || n_lanes == 0) return ESL_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  if (!ctx->have_tape) {
    if (!lead) return ESL_INVALID_ARGUMENT;
    if (int32_t rc = build_tape_from(ctx, lead)) return rc;
  }
  if (int32_t rc = warp_only(ctx)) return rc;
  if (ctx->seq_warps == 0) return ctx->fail(ESL_NOT_ELIGIBLE, "a warp's interleaved lane values exceed shared memory");
  ESL_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
  ESL_CUDA(launch_lu_lanes(ctx->topo, ctx->d_seq.as<uint2>(), ctx->n_seq_a, ctx->n_seq, n_lanes, d_a, d_rhs, d_tv,
                           d_dx, d_bad, ctx->seq_warps, ctx->stream));
  ESL_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
  ESL_CUDA(cudaEventSynchronize(ctx->ev1));
  if (ms) cudaEventElapsedTime(ms, ctx->ev0, ctx->ev1);
  return ESL_OK;
}

// Tapes beyond this many ops compile slowly and gain nothing over the
// interpreted kernel (their lanes no longer fit registers either).
constexpr uint32_t kLuJitMaxOps = 60000;

int32_t esl_lu_lanes_compiled_device(esl_ctx* ctx, const double* lead, uint32_t n_lanes, const double* d_a,
                                     const double* d_rhs, double* d_dx, uint8_t* d_bad, double* d_tv, float* ms) {
  if (!ctx || !d_a || !d_rhs || !d_dx || !d_bad || n_lanes == 0) return ESL_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  if (!ctx->have_tape) {
    if (!lead) return ESL_INVALID_ARGUMENT;
    if (int32_t rc = build_tape_from(ctx, lead)) return rc;
  }
  if (int32_t rc = warp_only(ctx)) return rc;
  if (ctx->lu_jit_state == 0) {
    ctx->lu_jit_state = -1;
    if (ctx->prog.a_nops + ctx->prog.b_nops > kLuJitMaxOps)
      return ctx->fail(ESL_NOT_ELIGIBLE, "the tape is too long to compile");
    const std::string src = compiled_lu_source(ctx->topo.nnz, ctx->lead, ctx->prog);
    if (!lu_jit_build(src, ctx->lu_jit))
      return ctx->fail(ESL_NOT_ELIGIBLE, "compiling the tape failed: " + ctx->lu_jit.log);
    ctx->lu_jit_state = 1;
  }
  if (ctx->lu_jit_state < 0) return ctx->fail(ESL_NOT_ELIGIBLE, "the tape could not be compiled");
  if (!d_tv) {
    ESL_CUDA(ctx->d_lu_scratch.ensure(size_t(ctx->prog.ntv) * n_lanes * 8));
    d_tv = ctx->d_lu_scratch.as<double>();
  }
  ESL_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
  ESL_CUDA(lu_jit_launch(ctx->lu_jit, n_lanes, d_a, d_rhs, d_tv, d_dx, d_bad, ctx->stream));
  ESL_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
  ESL_CUDA(cudaEventSynchronize(ctx->ev1));
  if (ms) cudaEventElapsedTime(ms, ctx->ev0, ctx->ev1);
  return ESL_OK;
}

int32_t esl_lu_lanes_mixed_compiled_device(esl_ctx* ctx, const double* lead, uint32_t n_lanes, const double* d_a,
                                           const double* d_rhs, double* d_dx, uint8_t* d_bad, uint8_t* d_refine,
                                           float* ms) {
  if (!ctx || !d_a || !d_rhs || !d_dx || !d_bad || n_lanes == 0) return ESL_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  if (!ctx->have_tape) {
    if (!lead) return ESL_INVALID_ARGUMENT;
    if (int32_t rc = build_tape_from(ctx, lead)) return rc;
  }
  if (int32_t rc = warp_only(ctx)) return rc;
  if (ctx->lu_jit_mixed_state == 0) {
    ctx->lu_jit_mixed_state = -1;
    if (ctx->prog.a_nops + ctx->prog.b_nops > kLuJitMaxOps)
      return ctx->fail(ESL_NOT_ELIGIBLE, "the tape is too long to compile");
    const std::string src = compiled_lu_source(ctx->topo.nnz, ctx->lead, ctx->prog, 0, true);
    if (!lu_jit_build(src, ctx->lu_jit_mixed, "lu_tape_mixed"))
      return ctx->fail(ESL_NOT_ELIGIBLE, "compiling the tape failed: " + ctx->lu_jit_mixed.log);
    ctx->lu_jit_mixed_state = 1;
  }
  if (ctx->lu_jit_mixed_state < 0) return ctx->fail(ESL_NOT_ELIGIBLE, "the tape could not be compiled");
  ESL_CUDA(ctx->d_lu_scratch32.ensure(size_t(ctx->prog.ntv) * n_lanes * 4));
  ESL_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
  ESL_CUDA(lu_jit_launch_mixed(ctx->lu_jit_mixed, n_lanes, d_a, d_rhs, ctx->d_lu_scratch32.as<float>(), d_dx, d_bad,
                               d_refine, ctx->stream));
  ESL_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
  ESL_CUDA(cudaEventSynchronize(ctx->ev1));
  if (ms) cudaEventElapsedTime(ms, ctx->ev0, ctx->ev1);
  return ESL_OK;
}

int32_t esl_lu_compiled_mixed_source(uint32_t n, const uint32_t* col_ptr, const uint32_t* row_idx,
                                     const double* lead, char* buf, size_t cap, size_t* len) {
  if (!col_ptr || !row_idx || !lead || !len || n == 0) return ESL_INVALID_ARGUMENT;
  Csc pat;
  pat.n = n;
  pat.col_ptr.assign(col_ptr, col_ptr + n + 1);
  pat.row_idx.assign(row_idx, row_idx + col_ptr[n]);
  SparseLu lu;
  lu.init(&pat, order_columns(pat));
  lu.fill_cap = kRepivotFillCap;
  lu.keep_min = kGrowthLimit;
  if (!lu.factor(lead, kPivotTol)) return ESL_NOT_ELIGIBLE;
  Programs P = compile_tape(lu);
  if (P.has_void) return ESL_NOT_ELIGIBLE;
  const std::string src = compiled_lu_source(col_ptr[n], lu, P, 0, true);
  *len = src.size();
  if (buf && cap > 0) {
    const size_t k = std::min(cap - 1, src.size());
    std::memcpy(buf, src.data(), k);
    buf[k] = '\0';
  }
  return ESL_OK;
}

const char* esl_lu_compiled_log(const esl_ctx* ctx) {
  return ctx && ctx->lu_jit_state == 1 ? ctx->lu_jit.log.c_str() : "";
}

int32_t esl_lu_lanes_mixed_device(esl_ctx* ctx, const double* lead, uint32_t n_lanes, const double* d_a,
                                  const double* d_rhs, double* d_dx, uint8_t* d_bad, uint8_t* d_refine, float* ms) {
  if (!ctx || !d_a || !d_rhs || !d_dx || !d_bad || n_lanes == 0) return ESL_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  if (!ctx->have_tape) {
    if (!lead) return ESL_INVALID_ARGUMENT;
    if (int32_t rc = build_tape_from(ctx, lead)) return rc;
  }
  if (int32_t rc = warp_only(ctx)) return rc;
  if (ctx->mixed_warps == 0) return ctx->fail(ESL_NOT_ELIGIBLE, "a warp's interleaved lane values exceed shared memory");
  ESL_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
  ESL_CUDA(launch_lu_lanes_mixed(ctx->topo, ctx->d_seq.as<uint2>(), ctx->n_seq_a, ctx->n_seq, ctx->n_seq_f, n_lanes,
                                 d_a, d_rhs, d_dx, d_bad, d_refine, ctx->mixed_warps, ctx->stream));
  ESL_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
  ESL_CUDA(cudaEventSynchronize(ctx->ev1));
  if (ms) cudaEventElapsedTime(ms, ctx->ev0, ctx->ev1);
  return ESL_OK;
}

int32_t esl_tape_size(const esl_ctx* ctx, uint32_t* nu, uint32_t* nl, uint32_t* ntv) {
  if (!ctx || !ctx->have_tape) return ESL_INVALID_ARGUMENT;
  if (nu) *nu = ctx->prog.nu;
  if (nl) *nl = ctx->prog.nl;
  if (ntv) *ntv = ctx->prog.ntv;
  return ESL_OK;
}

int32_t esl_lu_replay_device(esl_ctx* ctx, const double* lead, uint32_t n_lanes, const double* d_a,
                             const double* d_rhs, double* d_dx, uint8_t* d_bad, double* d_tv, float* ms) {
  if (!ctx || !d_a || !d_rhs || !d_dx || !d_bad || n_lanes == 0) return ESL_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  if (!ctx->have_tape) {
    if (!lead) return ESL_INVALID_ARGUMENT;
    if (int32_t rc = build_tape_from(ctx, lead)) return rc;
  }
  if (int32_t rc = warp_only(ctx)) return rc;
  ESL_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
  ESL_CUDA(launch_lu_replay(ctx->topo, n_lanes, d_a, d_rhs, d_tv, d_dx, d_bad, lanes_per_cta(ctx, n_lanes, ctx->lanes_eff), ctx->stream));
  ESL_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
  ESL_CUDA(cudaEventSynchronize(ctx->ev1));
  if (ms) cudaEventElapsedTime(ms, ctx->ev0, ctx->ev1);
  return ESL_OK;
}

}  // extern "C"
