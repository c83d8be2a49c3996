// Block lanes (block.cu): one CTA per lane for circuits too large for a
// warp's share of shared memory. The host builds a BlockDev per context and
// precision; the launchers below run the persistent DC kernel.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "lanes.cuh"

namespace esl {

// Threads of a block lane's CTA (its program rows are this wide).
constexpr uint32_t kBlockThreads = 256;
// Ops per thread in a program row of a working set that lives in the CTA's
// global slab (rows of kSlabRowOps * kBlockThreads ops); 1 in shared memory.
constexpr uint32_t kSlabRowOps = 4;

// The block lanes' assembly streams (see block_assemble): a term word is a
// staging index, with kGTermEnd on a cell's last term. Three cells past the
// device stamps hold constants, so every term is a plain load: n_stage +
// kGCellZero (+0.0: a cell without terms, padding), + kGCellOne (1.0: the
// ground pin on g) and + kGCellX0 (x[0]: the ground pin on rhs, refreshed
// each iteration). A cell word {index | kGCellRow, tape value or y index,
// diagonal row or kNoDiag, 0} is a pattern slot (index p) or, with
// kGCellRow, a residual row (index i).
constexpr uint32_t kGTermEnd = 0x80000000u;
constexpr uint32_t kGCellZero = 0, kGCellOne = 1, kGCellX0 = 2, kGConstCells = 3;
constexpr uint32_t kGCellRow = 0x80000000u;

struct BlockDev {
  TopoDev T;  // the topology's tables (pattern, gathers, tape maps, batches)
  // Programs A (refactor + forward solve), B (back solve) and F (forward
  // solve alone), rows of row_k * kBlockThreads ops (row_k 1 or
  // kSlabRowOps), op_bytes each: 8 {dst | kind << 28, a | b << 16} (value
  // space below 65,536) or 16 {dst | kind << 28, a, b, 0}; ring_bytes: the
  // per-CTA ring the ops stream through.
  const void* a_ops;
  const void* b_ops;
  const void* f_ops;
  uint32_t a_rows, b_rows, f_rows, op_bytes, ring_bytes, row_k;
  // The assembly: term stream [g_len][kBlockThreads], cell stream
  // [g_ncells][kBlockThreads] (uint4).
  const uint32_t* g_terms;
  const uint4* g_cells;
  uint32_t g_len, g_ncells;
  // A lane's working set, byte offsets: the hot part x, rhs, diag, dx (FP64,
  // n each), limited images, the FP64 matrix (mixed form: nnz), the value
  // space v (FP64, or FP32 in the mixed form); then the cold part xo (n) and
  // the staging cells. Split: the cold part lives apart, in the CTA's slab
  // (its offsets from there), so that more CTAs fit an SM's shared memory.
  uint32_t o_x, o_xo, o_rhs, o_diag, o_dx, o_st, o_lim, o_a64, o_v;
  uint32_t lane_bytes;  // the working set (split: its hot part), 16-byte aligned
  uint32_t in_smem;     // 1: (the hot part) in the CTA's shared memory; 0: all in its slab of `slab`
  uint32_t split;       // 1: the cold part in the CTA's slab, cold_bytes each
  uint32_t cold_bytes;
  uint32_t grid;        // CTAs of a launch (persistent)
  unsigned char* slab;  // per CTA: the working set (in_smem 0) or its cold part (split), and the lead assembly's scratch
  // Mixed form: refinement stops at max |res| <= refine_tol * max |rhs| or
  // after refine_max corrections; refine_out [lane] accumulates them.
  double refine_tol;
  uint32_t refine_max;
  uint32_t* refine_out;
  // Mixed form: a step whose FP32 solution scores above refine_skip
  // tolerances (the Newton delta score) is taken unrefined (0: never).
  double refine_skip;
  // Optional phase profile (null: off): thread 0 of each CTA adds the SM
  // cycles (clock64) of each phase of each Newton iteration to
  // prof[kBlockPhase*], and counts the iterations in prof[kBlockPhaseIters].
  unsigned long long* prof;
};

enum BlockPhase : uint32_t {
  kBlockPhaseEval = 0,     // device evaluation into the staging cells
  kBlockPhaseAssemble = 1, // gathers into the tape values, rhs and y
  kBlockPhaseRefactor = 2, // program A (refactor + forward solve) and the peel tests
  kBlockPhaseSolve = 3,    // program B (back solve) and the step
  kBlockPhaseRefine = 4,   // the mixed form's refinement
  kBlockPhaseGates = 5,    // update, limiting and the Newton gates
  kBlockPhaseIters = 6,    // Newton iterations counted
  kBlockPhases = 7
};

// The DC Newton solve of every lane of L (the block counterpart of
// launch_dc_newton; same lane state and pause protocol). mixed: FP32 tape
// values with FP64 refinement; has_b3: the BSIM3 instantiation.
cudaError_t launch_dc_block(const BlockDev& D, const LaneDev& L, const LaneOpts& o, bool mixed, bool has_b3,
                            cudaStream_t s);
// CTAs per SM of the DC kernel at this precision, op format and dynamic shared memory.
int block_occupancy(bool mixed, bool long_ops, bool has_b3, size_t smem);
// Uneven batching: the lanes of several topologies (device arrays of their
// BlockDev and LaneDev) in one persistent launch over work items (topology,
// lane), taken from the counter d_next in order; smem: the largest working
// set of the topologies that keep theirs in shared memory; slab_stride: the
// largest of the others (each CTA's slab at slab + blockIdx.x * stride);
// ring_at: the op ring's offset in dynamic shared memory. Every topology
// of a group has the same op format.
cudaError_t launch_dc_block_group(const BlockDev* d_Ds, const LaneDev* d_Ls, const uint2* d_items, uint32_t n_items,
                                  uint32_t* d_next, const LaneOpts& o, unsigned char* slab, size_t slab_stride,
                                  size_t smem, uint32_t ring_at, uint32_t grid, bool mixed, bool long_ops, bool has_b3,
                                  cudaStream_t s);
int block_group_occupancy(bool mixed, bool long_ops, bool has_b3, size_t smem);

// Transient block lanes: every lane's operating point and whole transient
// (the warp lanes' tran_kernel run, no measure cards) on a CTA per lane,
// FP64 or mixed precision (FP32 refactor and solves, the step refined in
// FP64 as the DC block lanes refine it; D.refine_out[lane] gets the lane's
// corrections); tslab: the run state, tran_block_slab(T) doubles per CTA of
// the launch (D.grid, or fewer when there are fewer lanes). A lane whose
// factor leaves the lead tape stops with kTranLeftTape.
size_t tran_block_slab(const TopoDev& T);
cudaError_t launch_tran_block(const BlockDev& D, const LaneDev& L, const TranDev& P, const LaneOpts& o, bool mixed,
                              bool has_b3, double* tslab, cudaStream_t s);

// The lead lane's first Jacobian in pattern order (D.slab as scratch).
cudaError_t launch_block_lead(const BlockDev& D, const LaneDev& L, uint32_t lane, double* out, bool has_b3,
                              cudaStream_t s);

}  // namespace esl
