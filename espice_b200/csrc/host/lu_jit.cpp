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

struct Gen {
  const LuJitInput& in;
  std::ostringstream os;
  std::vector<uint8_t> defined;
  std::vector<int64_t> slot_of;  // tape value -> the last pattern slot that loads it, -1 none
  std::vector<int64_t> row_of;   // y value -> its rhs row, -1 none
  std::vector<int64_t> last_ref; // statement of each value's latest reference
  std::vector<uint8_t> stored;   // written to the tape-value plane (final)
  int64_t at = 0;                // the current statement

  explicit Gen(const LuJitInput& i) : in(i) {
    defined.assign(in.nv, 0);
    slot_of.assign(in.nv, -1);
    row_of.assign(in.nv, -1);
    last_ref.assign(in.nv, -1);
    stored.assign(in.nv, 0);
    for (uint32_t p = 0; p < in.nnz; ++p) slot_of[(*in.amap)[p]] = p;
    for (uint32_t r = 0; r < in.n; ++r) row_of[in.ntv + (*in.pinv)[r]] = r;
  }

  // A reference to value v: its start at first use (A, -rhs for y = P(-rhs),
  // the constants 0.0 and 1.0, a fill-in zero), or, for a final tape value
  // last touched long ago, a reload from the tape-value plane, so that the
  // register file holds the values in use and not every value still needed.
  void use(uint32_t v) {
    if (!defined[v]) {
      defined[v] = 1;
      os << "  double v" << v << " = ";
      if (v == in.nv - 2) os << "1.0";
      else if (v >= in.nv - 3) os << "0.0";
      else if (slot_of[v] >= 0) os << "__ldg(al + " << slot_of[v] << " * N)";
      else if (row_of[v] >= 0) os << "-__ldg(rl + " << row_of[v] << " * N)";
      else os << "0.0";  // fill-in (and an entry no slot or op sets)
      os << ";\n";
    } else if (stored[v] && at - last_ref[v] > int64_t(in.reload_gap)) {
      os << "  v" << v << " = __ldcg(tl + " << v << " * N);\n";
    }
    last_ref[v] = at;
  }

  void op(uint32_t k, const Op& o) {
    const uint32_t kind = o.w0 >> 28, d = o.w0 & 0x0fffffffu, a = o.w1 & 0xffffu, b = o.w1 >> 16;
    if (kind == kOpNop) return;
    ++at;
    use(a);
    use(b);
    if (kind == kOpFlop || kind == kOpSubNz) {
      use(d);
      if (kind == kOpSubNz) os << "  if (v" << b << " != 0.0)";
      os << "  v" << d << " = __dsub_rn(v" << d << ", __dmul_rn(v" << a << ", v" << b << "));\n";
      return;
    }
    os << "  const double q" << k << " = __ddiv_rn(v" << b << ", v" << a << ");\n";
    if (kind == kOpDivGrowth)
      os << "  bad |= !(fabs(v" << a << ") >= __dmul_rn(1e-12, fabs(v" << b << ")));\n";
    if (kind == kOpDivScaled) os << "  bad |= !(fabs(q" << k << ") < kInf);\n";
    if (defined[d]) {
      os << "  v" << d << " = q" << k << ";\n";
    } else {
      defined[d] = 1;
      os << "  double v" << d << " = q" << k << ";\n";
    }
    last_ref[d] = at;
  }

  // A tape value is final: out to its plane, then the refactor's peel test
  // on it (a non-finite U entry, a dead or non-finite pivot, an unscaled L
  // multiplier past 1 / pivot_tol).
  void finish(uint32_t v) {
    if (v >= in.ntv - 1) return;  // the discard entry holds nothing
    use(v);
    os << "  tl[" << v << " * N] = v" << v << ";\n";
    stored[v] = 1;
    if (v < in.nu) {
      os << "  bad |= __double_as_longlong(v" << v << " - v" << v << ") != 0;\n";
    } else if (v < in.nu + in.n) {
      os << "  bad |= v" << v << " == 0.0 || !(fabs(v" << v << ") < kInf);\n";
    } else if (!(*in.l_scaled)[v - in.nu - in.n]) {
      os << "  bad |= !(fabs(v" << v << ") <= 1e3);\n";
    }
  }
};

}  // namespace

std::string lu_jit_source(const LuJitInput& in) {
  Gen g(in);
  const std::vector<Op>& seq = *in.seq;
  // the last op that writes each value, per program
  std::vector<int64_t> last_a(in.nv, -1), last_all(in.nv, -1);
  for (uint32_t k = 0; k < in.n_seq; ++k) {
    const uint32_t kind = seq[k].w0 >> 28, d = seq[k].w0 & 0x0fffffffu;
    if (kind == kOpNop) continue;
    if (k < in.n_seq_a) last_a[d] = k;
    last_all[d] = k;
  }
  std::ostringstream& os = g.os;
  os << "// generated: the lane refactor + solve of one pivot tape (" << in.n << " unknowns, " << in.ntv
     << " tape values, " << in.n_seq << " ops)\n"
     << "extern \"C\" __global__ void __launch_bounds__(" << kThreads << ", " << kMinBlocks << ") lu_tape(\n"
     << "    const double* __restrict__ a, const double* __restrict__ rhs, double* __restrict__ tv,\n"
     << "    double* __restrict__ dx, unsigned char* __restrict__ bad_out, unsigned n_lanes) {\n"
     << "  const unsigned lane = blockIdx.x * " << kThreads << "u + threadIdx.x;\n"
     << "  if (lane >= n_lanes) return;\n"
     << "  const size_t N = n_lanes;\n"
     << "  const double* al = a + lane;\n"
     << "  const double* rl = rhs + lane;\n"
     << "  double* tl = tv + lane;\n"
     << "  const double kInf = __longlong_as_double(0x7ff0000000000000ll);\n"
     << "  bool bad = false;\n";
  // tape values (U, diagonal, L) are final after their last update in
  // program A (at once when program A never writes them)
  for (uint32_t v = 0; v + 1 < in.ntv; ++v)
    if (last_a[v] < 0) g.finish(v);
  for (uint32_t k = 0; k < in.n_seq_a; ++k) {
    g.op(k, seq[k]);
    const uint32_t d = seq[k].w0 & 0x0fffffffu;
    if (last_a[d] == int64_t(k) && d < in.ntv) g.finish(d);
  }
  // dx is final after its last update; a y entry no op writes goes out as loaded
  auto store_dx = [&](uint32_t j) {
    os << "  dx[" << (*in.qcol)[j] << " * N + lane] = v" << (in.ntv + j) << ";\n";
  };
  for (uint32_t k = in.n_seq_a; k < in.n_seq; ++k) {
    g.op(k, seq[k]);
    const uint32_t d = seq[k].w0 & 0x0fffffffu;
    if (d >= in.ntv && d < in.ntv + in.n && last_all[d] == int64_t(k)) store_dx(d - in.ntv);
  }
  for (uint32_t j = 0; j < in.n; ++j)
    if (last_all[in.ntv + j] < int64_t(in.n_seq_a)) {
      g.use(in.ntv + j);
      store_dx(j);
    }
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

bool lu_jit_build(const std::string& src, LuJitKernels& out) {
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
  if (cudaLibraryGetKernel(&out.kernel, out.lib, "lu_tape") != cudaSuccess) {
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
