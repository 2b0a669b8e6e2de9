// lbx_internal.h -- the domain handle's layout, shared by the library's
// translation units (not part of the ABI).
#pragma once

#include "lbx.h"

#include <cuda_runtime.h>

#include <vector>

struct lbx_domain {
  lbx_params p;
  int Q = 0, D = 0;
  long long N = 0;
  size_t real_size = 0;
  void* f = nullptr;          // [nsubs][Q][N] dense (the exchange format)
  void* fc = nullptr;         // [nsubs][Q][P] compact layout
  int* fidx = nullptr;        // [N] dense -> compact (-1 solid)
  int* fnode = nullptr;       // [F] compact -> dense
  uint2* frm = nullptr;       // [ceil(N/32) + 2] fluid bitmask with word ranks, guard word each end
  long long P = 0;            // compact plane stride: fluid rounded up to 32
  int layout = LBX_LAYOUT_DENSE;
  bool dense_stale = false;   // compact state newer than the dense array
  void* mv = nullptr;         // [nsubs][1+D][N]
  uint8_t* solids = nullptr;  // [N] as given (device rule: == 1)
  uint8_t* cls = nullptr;     // [N]
  uint32_t* nbm = nullptr;    // [N]
  void* red = nullptr;        // reduction partials
  int red_blocks = 0;
  cudaStream_t stream = nullptr;      // stream all work is queued on
  cudaStream_t own_stream = nullptr;  // the library's stream
  // with z faces in the compact layout: the face planes' launch runs on
  // `side` beside the interior launches, forked from and joined back into
  // `stream` by the two events
  cudaStream_t side = nullptr;
  cudaEvent_t side_fork = nullptr, side_join = nullptr;
  std::vector<double> n_table, s_table;
  long long fluid = 0;
  bool faces_active = false;  // any 2D face boundary configured
  bool faces_fused = false;   // fused into the step kernels
  bool faces3_active = false; // any 3D z-face boundary configured
  bool faces3_fuse_odd = false;  // z faces exact inside odd compact steps (fluid upstream)
  std::vector<long long> plane_fluid;  // fluid nodes per plane (k in 3D, j in 2D)
  void* ubuf = nullptr;        // [3][P or N] flow velocity for the solute launch
  void* prof_t = nullptr;      // [LX*LY] constant-concentration profiles (real)
  void* prof_b = nullptr;
  void* ns = nullptr;        // Walsh fraction per node, [N] in the run's precision
  // plane record (lbx_btc_*)
  double* btc_vals = nullptr;  // [2][plane nodes]: C and u_x this step
  double* btc_rec = nullptr;   // [btc_cap][2] means
  int* btc_slot = nullptr;     // steps recorded
  double* btc_part = nullptr;  // [kBtcMaxBlocks][2] block partials of one step
  unsigned* btc_ticket = nullptr;  // blocks done this step (reset by the last)
  int btc_cap = 0;
  int btc_lo = 0, btc_hi = 0;  // node (dense) or slot (compact) range
  int btc_plane = 0;
  void* fout = nullptr;        // set only while recomputing states (OOP step)
  void* adj = nullptr;         // adjoint checkpoints and objective (lbx_adjoint.cu)
  void* frames = nullptr;      // frame statistics and snapshots (lbx_frames.cu)
  void* pest = nullptr;        // PEST point samples (lbx_pest.cu)
  int parity = 0;             // 0: natural order (next step odd); 1: swapped
  long long launches = 0;
  // graph replay of frame-free, time-invariant runs: one captured AA pair
  cudaGraphExec_t graph = nullptr;
  cudaGraphExec_t graph_multi = nullptr;   // the same pair repeated (replay_pairs)
  cudaStream_t graph_stream = nullptr;   // stream the pair was captured on
  unsigned char graph_key[2 * 640];      // keys of the odd and the even step
  size_t graph_key_len = 0;
  long long graph_launches = 0;          // kernels one replay of the graph runs
  // temporal blocking of small 2D lattices (lbx_tiled.cu)
  int run_mode = LBX_RUN_AUTO;
  void* tiled_scratch = nullptr;         // a second population array for its rounds
  int* tiled_flags = nullptr;            // per-tile round counters, then a status word
  int4* tiled_plan = nullptr;            // per tile: x, y, height
  int* tiled_nbrs = nullptr;             // per tile: the tiles its halo reads
  int tiled_ntiles = 0;
  bool tiled_local = false;              // tiles wait for their neighbours only
  int tiled_base = 0;                    // counter value the next launch starts from
  int tiled_grid = 0;                    // resident blocks of the tiled kernel (-1: none)
};

namespace lbx { template <typename T> struct StepArgs; }

// Hidden helpers of the library's translation units (not exported).
#define LBX_HIDDEN __attribute__((visibility("hidden")))
LBX_HIDDEN lbx_status lbx_internal_fail(lbx_status code, const char* msg);
LBX_HIDDEN lbx_status lbx_internal_step_into(lbx_domain* d, int t, void* src, void* dst);
LBX_HIDDEN void lbx_internal_adjoint_free(lbx_domain* d);
LBX_HIDDEN void lbx_internal_frames_free(lbx_domain* d);
LBX_HIDDEN void lbx_internal_drop_graphs(lbx_domain* d);
// PEST sampling: whether a sample is due at time t (the step then writes
// the macro variables), the gather after that step, and the release.
LBX_HIDDEN bool lbx_internal_pest_due(const lbx_domain* d, int t);
LBX_HIDDEN lbx_status lbx_internal_pest_after(lbx_domain* d, int t);
LBX_HIDDEN void lbx_internal_pest_free(lbx_domain* d);
// Temporal blocking: steps one round advances, and `rounds` (even) rounds
// with the launch arguments A of every step, from the state after an even
// step.
LBX_HIDDEN int lbx_internal_tiled_steps_per_round(const lbx_domain* d);
template <typename T>
LBX_HIDDEN lbx_status lbx_internal_tiled_run(lbx_domain* d, const lbx::StepArgs<T>& A, int rounds);
LBX_HIDDEN void lbx_internal_tiled_free(lbx_domain* d);
// LBX_OK, or the error of a tiled launch whose bounded wait ran out (then
// cleared); synchronous.
LBX_HIDDEN lbx_status lbx_internal_tiled_status(lbx_domain* d);
