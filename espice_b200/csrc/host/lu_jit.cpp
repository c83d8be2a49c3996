// Tape-compiled lane LU (see lu_jit.hpp).
//
// The interpreted lane-interleaved kernel keeps every lane's tape values in
// shared memory and reads an op word per op, so its occupancy is bound by
// shared memory (58.6 KB per warp on the ring's tape: 3 warps per SM) and
// each op costs a decode, three shared-memory round trips and a store. Here
// the tape is known when the context builds it, so it becomes code: each op
// is one statement on local variables that the compiler keeps in registers,
// A and rhs are read from their [entry][lane] planes at their first use and
// the tape values and dx are written after their last update, all
// coalesced across the warp. The ops run in the warp programs' order with
// the same roundings (__ddiv_rn, __dmul_rn, __dsub_rn) and the same peel
// tests, so every lane's values are bitwise those of the interpreted kernel
// and of the CPU replay.
#include "lu_jit.hpp"

#include <dlfcn.h>

#include <algorithm>

#include <cstdio>
#include <mutex>
#include <sstream>

#include "../common.h"

namespace esl {

namespace {

// 128 threads, at least 4 CTAs per SM: 128 registers a thread, 16 warps
// per SM. On the B200 this beat the unbounded form (about 240 registers,
// 8 warps) by 20% on the ring's tape and the grid's, and an L2 prefetch of
// every A row at the start gained nothing.
constexpr uint32_t kThreads = 128;
constexpr uint32_t kMinBlocks = 4;
// The A and rhs entries a lane reads arrive through shared memory in
// stages of kStage entries in first-use order, two stages in flight
// (cp.async into a per-thread double buffer: 2 x 24 x 128 x 8 B = 48 KB a
// CTA), so each warp keeps dozens of loads outstanding without holding
// registers for them: the kernel was bound by load latency, with about 2.4
// MB in flight over the GPU at 16 warps per SM.
constexpr uint32_t kStage = 24;

struct Gen {
  const LuJitInput& in;
  std::ostringstream os;
  std::vector<uint8_t> defined;
  std::vector<int64_t> slot_of;  // tape value -> the last pattern slot that loads it, -1 none
  std::vector<int64_t> row_of;   // y value -> its rhs row, -1 none
  // Register residency. Every value has a home in HBM: a tape value its
  // entry of the tape-value plane, y[j] its dx entry (the final dx store
  // overwrites it). The first pass records every use of every value; the
  // second keeps a model of which values sit in registers. Over the budget,
  // the value whose next use is farthest ahead leaves (Belady): written home
  // first when its home is stale, re-read at its next use. A tape value is
  // written home once anyway when final, so most evictions cost no store.
  std::vector<std::vector<uint32_t>> uses;
  std::vector<uint32_t> next;
  std::vector<uint8_t> resident, clean;
  uint32_t uc = 0, n_res = 0;
  // staging: the loaded values (A or rhs) in first-use order, recorded by the
  // first pass; each value's position in it; the stage being read
  bool record = true;
  std::vector<uint32_t> order;
  std::vector<int64_t> pos;
  int64_t cur_stage = -1;
  uint32_t n_stages = 0;

  explicit Gen(const LuJitInput& i) : in(i) {
    defined.assign(in.nv, 0);
    slot_of.assign(in.nv, -1);
    row_of.assign(in.nv, -1);
    pos.assign(in.nv, -1);
    uses.assign(in.nv, {});
    next.assign(in.nv, 0);
    resident.assign(in.nv, 0);
    clean.assign(in.nv, 0);
    for (uint32_t p = 0; p < in.nnz; ++p) slot_of[(*in.amap)[p]] = p;
    for (uint32_t r = 0; r < in.n; ++r) row_of[in.ntv + (*in.pinv)[r]] = r;
  }

  // FP64 form (double values, __d*_rn) or mixed form (float factors and y,
  // __f*_rn, FP32 peel tests as the interpreted mixed kernel takes them)
  const char* ty() const { return in.mixed ? "float" : "double"; }
  const char* sub_rn() const { return in.mixed ? "__fsub_rn" : "__dsub_rn"; }
  const char* mul_rn() const { return in.mixed ? "__fmul_rn" : "__dmul_rn"; }
  const char* div_rn() const { return in.mixed ? "__fdiv_rn" : "__ddiv_rn"; }
  const char* zero() const { return in.mixed ? "0.0f" : "0.0"; }

  static constexpr uint32_t kNever = 0xffffffffu;
  uint32_t next_use(uint32_t v) const { return next[v] < uses[v].size() ? uses[v][next[v]] : kNever; }
  bool constant(uint32_t v) const { return v >= in.nv - 3; }

  // The home of value v, as an expression for this lane.
  std::string home(uint32_t v) const {
    std::ostringstream h;
    if (v < in.ntv) h << "tl[" << v << " * N]";
    else h << "dx[" << (*in.qcol)[v - in.ntv] << " * N + lane]";
    return h.str();
  }

  // The residency model's bookkeeping for one reference at position u.
  void touch(uint32_t v) {
    if (!resident[v]) {
      resident[v] = 1;
      ++n_res;
    }
    ++next[v];
    if (next_use(v) == kNever) {  // dead after this reference
      resident[v] = 0;
      --n_res;
    }
  }

  // A read of value v: its start at first use (A, -rhs for y = P(-rhs), the
  // constants 0.0 and 1.0, a fill-in zero), or a reload from its home when
  // the model let it go.
  void use(uint32_t v) {
    const uint32_t u = uc++;
    if (record) {
      uses[v].push_back(u);
    } else if (!constant(v)) {
      if (defined[v] && !resident[v]) os << "  v" << v << " = __ldcg(&" << home(v) << ");\n";
      touch(v);
    }
    if (!defined[v]) {
      defined[v] = 1;
      const bool loaded = !constant(v) && (slot_of[v] >= 0 || row_of[v] >= 0);
      if (loaded && record) {
        pos[v] = int64_t(order.size());
        order.push_back(v);
      }
      if (loaded && !record) enter_stage(uint32_t(pos[v] / kStage));
      os << "  " << ty() << " v" << v << " = ";
      if (v == in.nv - 2) os << (in.mixed ? "1.0f" : "1.0");
      else if (constant(v)) os << zero();
      else if (loaded)
        os << (in.mixed ? "float(" : "") << (slot_of[v] >= 0 ? "" : "-") << "stage_read(sb, " << (pos[v] / kStage) % 2
           << ", " << pos[v] % kStage << ")" << (in.mixed ? ")" : "");
      else os << zero();  // fill-in (and an entry no slot or op sets)
      os << ";\n";
    }
  }

  // A write of value d by the current op (its home is now stale).
  void wrote(uint32_t d) {
    clean[d] = 0;
    if (record) return;
  }

  // After each op: back under the register budget.
  void settle() {
    if (record) return;
    while (n_res > in.resident_values) {
      uint32_t best = kNever, far = 0;
      for (uint32_t v = 0; v < in.nv - 3; ++v)
        if (resident[v] && next_use(v) >= far && (next_use(v) > far || clean[v])) {
          far = next_use(v);
          best = v;
        }
      if (best == kNever) return;
      if (!clean[best]) {
        os << "  " << home(best) << " = v" << best << ";\n";
        clean[best] = 1;
      }
      resident[best] = 0;
      --n_res;
    }
  }

  // Stage t's copies into buffer t % 2, as one commit group.
  void issue(uint32_t t) {
    for (uint32_t j = t * kStage; j < std::min<uint32_t>(uint32_t(order.size()), (t + 1) * kStage); ++j) {
      const uint32_t v = order[j];
      os << "  stage_copy(sb, " << t % 2 << ", " << j % kStage << ", ";
      if (slot_of[v] >= 0) os << "al + " << slot_of[v] << " * N);\n";
      else os << "rl + " << row_of[v] << " * N);\n";
    }
    os << "  stage_commit();\n";
  }

  // The first read of stage s: stage s - 1 is consumed, so stage s + 1 goes
  // into its buffer; then wait until stage s has landed.
  void enter_stage(uint32_t s) {
    if (int64_t(s) == cur_stage) return;
    cur_stage = s;
    if (s >= 1 && s + 1 < n_stages) issue(s + 1);
    os << "  stage_wait<" << (s + 1 < n_stages ? 1 : 0) << ">();\n";
  }

  void op(uint32_t k, const Op& o) {
    const uint32_t kind = o.w0 >> 28, d = o.w0 & 0x0fffffffu, a = o.w1 & 0xffffu, b = o.w1 >> 16;
    if (kind == kOpNop) return;
    use(a);
    use(b);
    if (kind == kOpFlop || kind == kOpSubNz) {
      use(d);
      if (kind == kOpSubNz) os << "  if (v" << b << " != " << zero() << ")";
      os << "  v" << d << " = " << sub_rn() << "(v" << d << ", " << mul_rn() << "(v" << a << ", v" << b << "));\n";
      wrote(d);
      return;
    }
    os << "  const " << ty() << " q" << k << " = " << div_rn() << "(v" << b << ", v" << a << ");\n";
    if (kind == kOpDivGrowth) {
      if (in.mixed) os << "  bad |= !(fabsf(v" << a << ") >= __fmul_rn(1e-12f, fabsf(v" << b << ")));\n";
      else os << "  bad |= !(fabs(v" << a << ") >= __dmul_rn(1e-12, fabs(v" << b << ")));\n";
    }
    if (kind == kOpDivScaled) os << "  bad |= !(fabs(q" << k << ") < kInf);\n";
    if (defined[d]) {
      os << "  v" << d << " = q" << k << ";\n";
    } else {
      defined[d] = 1;
      os << "  " << ty() << " v" << d << " = q" << k << ";\n";
    }
    // a division's destination is a new value in a register: counted as a
    // reference, with no load
    const uint32_t u = uc++;
    if (record) uses[d].push_back(u);
    else touch(d);
    wrote(d);
  }

  // A tape value is final: out to its plane, then the refactor's peel test
  // on it (a non-finite U entry, a dead or non-finite pivot, an unscaled L
  // multiplier past 1 / pivot_tol).
  void finish(uint32_t v) {
    if (v >= in.ntv - 1) return;  // the discard entry holds nothing
    use(v);
    os << "  " << home(v) << " = v" << v << ";\n";
    clean[v] = 1;
    if (in.mixed) {  // the interpreted mixed kernel's FP32 tests
      if (v < in.nu) os << "  bad |= !(fabsf(v" << v << ") < kInf);\n";
      else if (v < in.nu + in.n) os << "  bad |= v" << v << " == 0.0f || !(fabsf(v" << v << ") < kInf);\n";
      else if (!(*in.l_scaled)[v - in.nu - in.n]) os << "  bad |= !(fabsf(v" << v << ") <= 1e3f);\n";
      return;
    }
    if (v < in.nu) {
      os << "  bad |= __double_as_longlong(v" << v << " - v" << v << ") != 0;\n";
    } else if (v < in.nu + in.n) {
      os << "  bad |= v" << v << " == 0.0 || !(fabs(v" << v << ") < kInf);\n";
    } else if (!(*in.l_scaled)[v - in.nu - in.n]) {
      os << "  bad |= !(fabs(v" << v << ") <= 1e3);\n";
    }
  }

  // y[j] is final: out to dx (its home).
  void store_dx(uint32_t j) {
    use(in.ntv + j);
    os << "  " << home(in.ntv + j) << " = v" << (in.ntv + j) << ";\n";
    clean[in.ntv + j] = 1;
  }
};

}  // namespace

// The mixed form's FP64 refinement, after dx = the FP32 solve: the residual
// res = -rhs - A dx in FP64 (A and rhs re-read, the pattern by rows, columns
// ascending), then, unless max |res| <= 1e-12 max |rhs| or 6 corrections
// are done, the correction solved on the FP32 factors (the forward
// substitution's ops of program A, then program B, all in their sequential
// order, the factors read from their FP32 plane) and added to dx, as the
// interpreted mixed kernel does it.
static void refinement(const LuJitInput& in, std::ostringstream& os) {
  const std::vector<Op>& seq = *in.seq;
  std::vector<std::vector<std::pair<uint32_t, uint32_t>>> rows(in.n);
  for (uint32_t j = 0; j < in.n; ++j)
    for (uint32_t p = (*in.col_ptr)[j]; p < (*in.col_ptr)[j + 1]; ++p) rows[(*in.row_idx)[p]].push_back({p, j});
  auto y = [&](uint32_t v) { return "r" + std::to_string(v - in.ntv); };
  auto fac = [&](uint32_t v) { return "__ldcg(&tl[" + std::to_string(v) + " * N])"; };
  os << "  unsigned char refined = 0;\n"
     << "  #pragma unroll 1\n"
     << "  for (int it = 0; it <= 6; ++it) {\n"
     << "    double rmax = 0.0, bmax = 0.0;\n    float";
  for (uint32_t j = 0; j < in.n; ++j) os << (j ? ", r" : " r") << j;
  os << ";\n";
  for (uint32_t i = 0; i < in.n; ++i) {
    os << "    {\n      const double b = __ldg(rl + " << i << " * N);\n      double res = -b;\n";
    for (const auto& e : rows[i])
      os << "      res = __dsub_rn(res, __dmul_rn(__ldg(al + " << e.first << " * N), __ldcg(&dx[" << e.second
         << " * N + lane])));\n";
    os << "      rmax = fmax(rmax, fabs(res));\n      bmax = fmax(bmax, fabs(b));\n"
       << "      r" << (*in.pinv)[i] << " = float(res);\n    }\n";
  }
  os << "    if (!(rmax > 1e-12 * bmax) || it == 6) break;\n";
  for (uint32_t k = 0; k < in.n_seq_a; ++k) {
    const Op& o = seq[k];
    if ((o.w0 >> 28) != kOpSubNz) continue;
    const uint32_t d = o.w0 & 0x0fffffffu, a = o.w1 & 0xffffu, b = o.w1 >> 16;
    os << "    if (" << y(b) << " != 0.0f) " << y(d) << " = __fsub_rn(" << y(d) << ", __fmul_rn(" << fac(a) << ", " << y(b)
       << "));\n";
  }
  for (uint32_t k = in.n_seq_a; k < in.n_seq; ++k) {
    const Op& o = seq[k];
    const uint32_t kind = o.w0 >> 28, d = o.w0 & 0x0fffffffu, a = o.w1 & 0xffffu, b = o.w1 >> 16;
    if (kind == kOpNop) continue;
    if (kind == kOpSubNz)
      os << "    if (" << y(b) << " != 0.0f) " << y(d) << " = __fsub_rn(" << y(d) << ", __fmul_rn(" << fac(a) << ", "
         << y(b) << "));\n";
    else  // the back substitution's divisions (kOpDivY)
      os << "    " << y(d) << " = __fdiv_rn(" << y(b) << ", " << fac(a) << ");\n";
  }
  for (uint32_t j = 0; j < in.n; ++j)
    os << "    dx[" << (*in.qcol)[j] << " * N + lane] = __ldcg(&dx[" << (*in.qcol)[j] << " * N + lane]) + double(r" << j
       << ");\n";
  os << "    ++refined;\n  }\n"
     << "  if (refine_out) refine_out[lane] = refined;\n";
}

std::string lu_jit_source(const LuJitInput& in) {
  const std::vector<Op>& seq = *in.seq;
  // the last op that writes each value, per program
  std::vector<int64_t> last_a(in.nv, -1), last_all(in.nv, -1);
  for (uint32_t k = 0; k < in.n_seq; ++k) {
    const uint32_t kind = seq[k].w0 >> 28, d = seq[k].w0 & 0x0fffffffu;
    if (kind == kOpNop) continue;
    if (k < in.n_seq_a) last_a[d] = k;
    last_all[d] = k;
  }
  // The op stream: tape values (U, diagonal, L) are final after their last
  // update in program A (at once when program A never writes them); dx is
  // final after its last update (a y entry no op writes goes out as loaded).
  auto walk = [&](Gen& g) {
    for (uint32_t v = 0; v + 1 < in.ntv; ++v)
      if (last_a[v] < 0) {
        g.finish(v);
        g.settle();
      }
    for (uint32_t k = 0; k < in.n_seq_a; ++k) {
      g.op(k, seq[k]);
      const uint32_t d = seq[k].w0 & 0x0fffffffu;
      if (last_a[d] == int64_t(k) && d < in.ntv) g.finish(d);
      g.settle();
    }
    for (uint32_t k = in.n_seq_a; k < in.n_seq; ++k) {
      g.op(k, seq[k]);
      const uint32_t d = seq[k].w0 & 0x0fffffffu;
      if (d >= in.ntv && d < in.ntv + in.n && last_all[d] == int64_t(k)) g.store_dx(d - in.ntv);
      g.settle();
    }
    for (uint32_t j = 0; j < in.n; ++j)
      if (last_all[in.ntv + j] < int64_t(in.n_seq_a)) {
        g.store_dx(j);
        g.settle();
      }
  };
  // pass 1: the loaded values' first-use order
  Gen first(in);
  walk(first);
  Gen g(in);
  g.record = false;
  g.order = first.order;
  g.pos = first.pos;
  g.uses = first.uses;
  g.n_stages = uint32_t((g.order.size() + kStage - 1) / kStage);
  std::ostringstream& os = g.os;
  os << "// generated: the lane refactor + solve of one pivot tape (" << in.n << " unknowns, " << in.ntv
     << " tape values, " << in.n_seq << " ops)\n"
     << "#ifndef ESL_LU_HOST_EMULATION\n"
     << "__device__ __forceinline__ void stage_copy(unsigned sb, unsigned b, unsigned i, const double* src) {\n"
     << "  asm volatile(\"cp.async.ca.shared.global [%0], [%1], 8;\" :: \"r\"(sb + (b * " << kStage << "u + i) * "
     << kThreads * 8 << "u), \"l\"(src) : \"memory\");\n"
     << "}\n"
     << "__device__ __forceinline__ void stage_commit() { asm volatile(\"cp.async.commit_group;\" ::: \"memory\"); }\n"
     << "template <int P> __device__ __forceinline__ void stage_wait() {\n"
     << "  asm volatile(\"cp.async.wait_group %0;\" :: \"n\"(P) : \"memory\");\n"
     << "}\n"
     << "__device__ __forceinline__ double stage_read(unsigned sb, unsigned b, unsigned i) {\n"
     << "  double v;\n"
     << "  asm volatile(\"ld.shared.f64 %0, [%1];\" : \"=d\"(v) : \"r\"(sb + (b * " << kStage << "u + i) * "
     << kThreads * 8 << "u) : \"memory\");\n"
     << "  return v;\n"
     << "}\n"
     << "#endif\n";
  if (in.mixed)
    os << "extern \"C\" __global__ void __launch_bounds__(" << kThreads << ", " << kMinBlocks << ") lu_tape_mixed(\n"
       << "    const double* __restrict__ a, const double* __restrict__ rhs, float* __restrict__ tv,\n"
       << "    double* __restrict__ dx, unsigned char* __restrict__ bad_out, unsigned char* __restrict__ refine_out,\n"
       << "    unsigned n_lanes) {\n";
  else
    os << "extern \"C\" __global__ void __launch_bounds__(" << kThreads << ", " << kMinBlocks << ") lu_tape(\n"
       << "    const double* __restrict__ a, const double* __restrict__ rhs, double* __restrict__ tv,\n"
       << "    double* __restrict__ dx, unsigned char* __restrict__ bad_out, unsigned n_lanes) {\n";
  os
     << "  __shared__ __align__(16) double stage_buf[2 * " << kStage << " * " << kThreads << "];\n"
     << "  const unsigned lane = blockIdx.x * " << kThreads << "u + threadIdx.x;\n"
     << "  if (lane >= n_lanes) return;\n"
     << "  const size_t N = n_lanes;\n"
     << "  const double* al = a + lane;\n"
     << "  const double* rl = rhs + lane;\n"
     << "  " << g.ty() << "* tl = tv + lane;\n"
     << "  const unsigned sb = unsigned(__cvta_generic_to_shared(stage_buf + threadIdx.x));\n"
     << (in.mixed ? "  const float kInf = __int_as_float(0x7f800000);\n"
                  : "  const double kInf = __longlong_as_double(0x7ff0000000000000ll);\n")
     << "  bool bad = false;\n";
  // the first two stages in flight before any op
  if (g.n_stages > 0) g.issue(0);
  if (g.n_stages > 1) g.issue(1);
  walk(g);
  if (in.mixed) refinement(in, os);
  os << "  bad_out[lane] = bad;\n"
     << "}\n";
  return os.str();
}

namespace {

// NVRTC through dlopen: the library carries no link-time dependency on it,
// and a machine without it reports "not eligible" instead of failing to load.
struct Nvrtc {
  using Prog = void*;
  int (*create)(Prog*, const char*, const char*, int, const char* const*, const char* const*) = nullptr;
  int (*compile)(Prog, int, const char* const*) = nullptr;
  int (*log_size)(Prog, size_t*) = nullptr;
  int (*log)(Prog, char*) = nullptr;
  int (*cubin_size)(Prog, size_t*) = nullptr;
  int (*cubin)(Prog, char*) = nullptr;
  int (*destroy)(Prog*) = nullptr;
  bool ok = false;
};

const Nvrtc& nvrtc() {
  static Nvrtc n;
  static std::once_flag once;
  std::call_once(once, [] {
    void* h = dlopen("libnvrtc.so.12", RTLD_NOW | RTLD_LOCAL);
    if (!h) h = dlopen("libnvrtc.so", RTLD_NOW | RTLD_LOCAL);
    if (!h) return;
    auto sym = [h](const char* s) { return dlsym(h, s); };
    n.create = reinterpret_cast<decltype(n.create)>(sym("nvrtcCreateProgram"));
    n.compile = reinterpret_cast<decltype(n.compile)>(sym("nvrtcCompileProgram"));
    n.log_size = reinterpret_cast<decltype(n.log_size)>(sym("nvrtcGetProgramLogSize"));
    n.log = reinterpret_cast<decltype(n.log)>(sym("nvrtcGetProgramLog"));
    n.cubin_size = reinterpret_cast<decltype(n.cubin_size)>(sym("nvrtcGetCUBINSize"));
    n.cubin = reinterpret_cast<decltype(n.cubin)>(sym("nvrtcGetCUBIN"));
    n.destroy = reinterpret_cast<decltype(n.destroy)>(sym("nvrtcDestroyProgram"));
    n.ok = n.create && n.compile && n.log_size && n.log && n.cubin_size && n.cubin && n.destroy;
  });
  return n;
}

}  // namespace

bool lu_jit_build(const std::string& src, LuJitKernels& out, const char* name) {
  const Nvrtc& nv = nvrtc();
  if (!nv.ok) {
    out.log = "NVRTC (libnvrtc.so.12) is not available";
    return false;
  }
  Nvrtc::Prog prog = nullptr;
  if (nv.create(&prog, src.c_str(), "lu_tape.cu", 0, nullptr, nullptr) != 0) {
    out.log = "nvrtcCreateProgram failed";
    return false;
  }
  const char* opts[] = {"--gpu-architecture=sm_100a", "--fmad=false", "-std=c++17", "--ptxas-options=-v"};
  const int rc = nv.compile(prog, 4, opts);
  size_t ls = 0;
  nv.log_size(prog, &ls);
  std::string log(ls, '\0');
  if (ls) nv.log(prog, &log[0]);
  out.log = log;
  if (rc != 0) {
    nv.destroy(&prog);
    return false;
  }
  size_t cs = 0;
  nv.cubin_size(prog, &cs);
  std::vector<char> cubin(cs);
  nv.cubin(prog, cubin.data());
  nv.destroy(&prog);
  if (cudaLibraryLoadData(&out.lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0) != cudaSuccess) {
    cudaGetLastError();
    out.log += "\ncudaLibraryLoadData failed";
    out.lib = nullptr;
    return false;
  }
  if (cudaLibraryGetKernel(&out.kernel, out.lib, name) != cudaSuccess) {
    cudaGetLastError();
    out.log += "\ncudaLibraryGetKernel failed";
    lu_jit_release(out);
    return false;
  }
  return true;
}

void lu_jit_release(LuJitKernels& k) {
  if (k.lib) cudaLibraryUnload(k.lib);
  k.lib = nullptr;
  k.kernel = nullptr;
}

cudaError_t lu_jit_launch(const LuJitKernels& k, uint32_t n_lanes, const double* a, const double* rhs, double* tv,
                          double* dx, uint8_t* bad, cudaStream_t s) {
  void* args[] = {&a, &rhs, &tv, &dx, &bad, &n_lanes};
  const void* fn = reinterpret_cast<const void*>(k.kernel);
  return cudaLaunchKernel(fn, dim3((n_lanes + kThreads - 1) / kThreads), dim3(kThreads), args, 0, s);
}

}  // namespace esl

namespace esl {

cudaError_t lu_jit_launch_mixed(const LuJitKernels& k, uint32_t n_lanes, const double* a, const double* rhs,
                                float* tf, double* dx, uint8_t* bad, uint8_t* refine, cudaStream_t s) {
  void* args[] = {&a, &rhs, &tf, &dx, &bad, &refine, &n_lanes};
  return cudaLaunchKernel(reinterpret_cast<const void*>(k.kernel), dim3((n_lanes + kThreads - 1) / kThreads),
                          dim3(kThreads), args, 0, s);
}

}  // namespace esl
