// lbx_abi.cu -- the C ABI (include/lbx.h) over the sm_100a kernels.
//
// Host-side restatement of the reference's device orchestration:
//   construct_lattice device part   src/latman.c:147-376, :461-493
//   solid upload                    src/lbgpu_prime.cu:170-257
//   per-step order                  src/lbgpu_prime.cu:369-915
//   face schedule (bcs_1 / bcs_2)   src/bcs.c:226-558, :1179-1506
// No CPU compute path exists here: every step is a CUDA launch, and a
// failed launch is an error returned to the caller.
#include "lbx.h"
#include "lbx_internal.h"
#include "lbx_kernels.cuh"

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

using namespace lbx;

namespace {

thread_local std::string g_err;

lbx_status fail(lbx_status code, const char* fmt, ...)
    __attribute__((format(printf, 2, 3)));

lbx_status fail(lbx_status code, const char* fmt, ...)
{
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

}  // namespace

// For the library's other translation units; hidden, so not an entry point.
__attribute__((visibility("hidden"))) lbx_status lbx_internal_fail(lbx_status code,
                                                                    const char* msg)
{
  g_err = msg;
  return code;
}

// Drops the cached step graphs (their launch arguments no longer hold).
__attribute__((visibility("hidden"))) void lbx_internal_drop_graphs(lbx_domain* d)
{
  if (d->graph) cudaGraphExecDestroy(d->graph);
  if (d->graph_multi) cudaGraphExecDestroy(d->graph_multi);
  d->graph = nullptr;
  d->graph_multi = nullptr;
}

namespace {

#define CK(call)                                                              \
  do {                                                                        \
    cudaError_t e_ = (call);                                                  \
    if (e_ != cudaSuccess)                                                    \
      return fail(e_ == cudaErrorMemoryAllocation ? LBX_ERR_NOMEM             \
                                                  : LBX_ERR_CUDA,             \
                  "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__,  \
                  __LINE__);                                                  \
  } while (0)

}  // namespace


namespace {

template <typename T>
T face_rho(const lbx_domain* d, int s, int t, int in_kind, bool is_in,
           const std::vector<double>& table)
{
  // src/bcs.c:286-322 (and the three sibling faces), in the run's `real`.
  const lbx_params& p = d->p;
  T rho;
  if (is_in && in_kind == 2)
    rho = (T)p.pfadd + (T)p.pfmul * (T)table[t % (int)table.size()];
  else
    rho = is_in ? (T)p.rho_in : (T)p.rho_out;
  if (p.bc_ramp_start >= 0 && p.bc_ramp_stop >= 0) {
    if (t < p.bc_ramp_start) {
      rho = (T)p.rho_A[s];
    } else if (t < p.bc_ramp_stop) {
      T ramp = ((T)(t - p.bc_ramp_start)) / ((T)(p.bc_ramp_stop - p.bc_ramp_start));
      rho *= ramp;
      rho = (T)((double)rho + (1. - (double)ramp) * (double)(T)p.rho_A[s]);
    }
  }
  return rho;
}

// A step with the solute off still runs the solute's face operations: the
// reference launches its face kernels whatever sigma_t_on/off say
// (src/bcs.c:503-541, :1453-1491), and their deposits change the idle
// solute's slots.  The fused face paths apply the rules only to the
// substances a step updates, so such steps take the stand-alone face kernels.
bool solute_faces_idle(const lbx_domain* d, int t)
{
  const lbx_params& p = d->p;
  if (p.nsubs != 2 || (t >= p.sigma_t_on && t <= p.sigma_t_off)) return false;
  return p.zeroconcgrad_n || p.zeroconcgrad_s || p.pressure_n_in[1] || p.pressure_n_out[1] ||
         p.pressure_s_in[1] || p.pressure_s_out[1] || p.constcon_t_in || p.constcon_b_in ||
         p.zeroconcgrad_t || p.zeroconcgrad_b || p.pressure_t_in[1] || p.pressure_t_out[1] ||
         p.pressure_b_in[1] || p.pressure_b_out[1] || p.velocity_t_in[1] ||
         p.velocity_t_out[1] || p.velocity_b_in[1] || p.velocity_b_out[1];
}

template <typename T>
void fill_args(const lbx_domain* d, int t, unsigned flags, StepArgs<T>& A)
{
  const lbx_params& p = d->p;
  std::memset(&A, 0, sizeof A);   // padding included: args are compared as bytes
  A.f = (T*)(d->layout == LBX_LAYOUT_COMPACT ? d->fc : d->f);
  A.mv = (T*)d->mv;
  A.cls = d->cls;
  A.nbm = d->nbm;
  A.LX = p.LX; A.LY = p.LY; A.LZ = p.LZ;
  A.N = d->N;
  for (int s = 0; s < 2; ++s) {
    const T tau = (T)p.tau[s];
    const T itau = (T)(1. / tau);
    A.sc[s].itau = itau;
    A.sc[s].omc = (T)(1. - itau);
    A.sc[s].rhoA = (T)p.rho_A[s];
    for (int c = 0; c < 3; ++c) A.sc[s].tg[c] = tau * (T)p.gaccel[s * 3 + c];
  }
  A.sink1 = (T)(1.0 - (T)p.sink * (T)p.tau[1]);
  A.write_mv = (flags & LBX_WRITE_MV) ? 1 : 0;
  A.solute_on = (t >= p.sigma_t_on && t <= p.sigma_t_off) ? 1 : 0;
  A.kahan = p.kahan ? 1 : 0;
  A.ubuf = (T*)d->ubuf;
  A.fout = (T*)d->fout;
  A.ustride = d->layout == LBX_LAYOUT_COMPACT ? d->P : d->N;
  if (d->ns) {
    A.ns = (const T*)d->ns;
    for (int s = 0; s < 2; ++s) {
      A.wtau[s] = (double)(T)p.tau[s];
      for (int c = 0; c < 3; ++c) A.wg[s * 3 + c] = (double)(T)p.gaccel[s * 3 + c];
    }
  }
  if (d->btc_vals) {
    A.btc = d->btc_vals;
    A.btc_lo = d->btc_lo;
    A.btc_hi = d->btc_hi;
  }
  if (d->faces_fused && !solute_faces_idle(d, t)) {
    for (int s = 0; s < p.nsubs; ++s) {
      // last active boundary on each face wins (see FaceKind)
      if (s == 1 && p.nsubs == 2 && p.zeroconcgrad_n) A.face_n[s] = FACE_ZEROGRAD;
      else if (p.pressure_n_out[s]) { A.face_n[s] = FACE_PRESSURE; A.rho_n[s] = face_rho<T>(d, s, t, 0, false, d->n_table); }
      else if (p.pressure_n_in[s]) { A.face_n[s] = FACE_PRESSURE; A.rho_n[s] = face_rho<T>(d, s, t, p.pressure_n_in[s], true, d->n_table); }
      if (s == 1 && p.nsubs == 2 && p.zeroconcgrad_s) A.face_s[s] = FACE_ZEROGRAD;
      else if (p.pressure_s_out[s]) { A.face_s[s] = FACE_PRESSURE; A.rho_s[s] = face_rho<T>(d, s, t, 0, false, d->s_table); }
      else if (p.pressure_s_in[s]) { A.face_s[s] = FACE_PRESSURE; A.rho_s[s] = face_rho<T>(d, s, t, p.pressure_s_in[s], true, d->s_table); }
    }
    for (int s = 0; s < p.nsubs; ++s) {
      A.drho_n[s] = (T)((double)A.rho_n[s] - (double)A.sc[s].rhoA);
      A.drho_s[s] = (T)((double)A.rho_s[s] - (double)A.sc[s].rhoA);
    }
  }
}

template <typename T>
StepArgs<T> make_args(const lbx_domain* d, int t, unsigned flags)
{
  StepArgs<T> A;
  fill_args<T>(d, t, flags, A);
  return A;
}

// The compact kernels' arguments for one step.
template <typename T>
CompactArgs<T> make_compact(const lbx_domain* d, const StepArgs<T>& A)
{
  CompactArgs<T> C;
  std::memset(&C, 0, sizeof C);
  C.s = A;
  C.fidx = d->fidx;
  C.fnode = d->fnode;
  C.frm = d->frm + 1;   // past the front guard word
  C.F = (int)d->fluid;
  C.P = (int)d->P;
  C.div_plane = make_fastdiv((unsigned)(A.LX * A.LY));
  C.div_lx = make_fastdiv((unsigned)A.LX);
  C.faces = d->faces_fused ? 1 : 0;
  C.m_base = 0;
  C.m_skip = 0x7fffffff;
  C.m_jump = 0;
  C.m_end = C.F;
  return C;
}

// The fluid nodes of the two z-face planes (compact [0, lo_end) and
// [hi_start, F)) with their face operations applied in registers, every
// substance in one launch (flow, then solute, per node).  The interior
// between them runs in the ordinary step launches, so the face code's
// registers do not weigh on the bulk of the nodes.
template <typename T, int Q, int NS, int MODEL>
void launch_face_nodes(lbx_domain* d, const StepArgs<T>& A, bool odd, const Face3Fused<T>& f3,
                       cudaStream_t stream)
{
  if constexpr (Q == 19) {
    CompactArgs<T> C = make_compact<T>(d, A);
    C.f3 = f3;
    C.m_base = 0;
    C.m_skip = f3.lo_end;
    C.m_jump = f3.hi_start - f3.lo_end;
    const long long count = (long long)f3.lo_end + (d->fluid - f3.hi_start);
    const unsigned blocks = (unsigned)((count + 255) / 256);
    if (blocks == 0) return;
    const bool idx32 = (unsigned long long)Q * (unsigned long long)d->P < (1ull << 32);
    auto go = [&](auto odd_c, auto idx_c) {
      aa_step_compact<T, Q, NS, MODEL, decltype(odd_c)::value, PART_ALL, decltype(idx_c)::value,
                      false, true><<<blocks, 256, 0, stream>>>(C);
    };
    using TT = std::true_type;
    using FF = std::false_type;
    if (idx32) { if (odd) go(TT{}, TT{}); else go(FF{}, TT{}); }
    else { if (odd) go(TT{}, FF{}); else go(FF{}, FF{}); }
    d->launches++;
  }
}

template <typename T, int Q, int NS, int MODEL, int PART>
void launch_part(lbx_domain* d, const StepArgs<T>& A, bool odd, const Face3Fused<T>* f3)
{
  if (d->layout == LBX_LAYOUT_COMPACT) {
    CompactArgs<T> C = make_compact<T>(d, A);
    if (f3) {   // the interior only; launch_face_nodes takes the two planes
      C.m_base = f3->lo_end;
      C.m_end = f3->hi_start;
    }
    const unsigned blocks = (unsigned)((C.m_end - C.m_base + 255) / 256);
    if (C.m_end <= C.m_base) return;
    const bool idx32 = (unsigned long long)Q * (unsigned long long)d->P < (1ull << 32);
    auto go = [&](auto odd_c, auto idx_c, auto oop_c) {
      aa_step_compact<T, Q, NS, MODEL, decltype(odd_c)::value, PART, decltype(idx_c)::value,
                      decltype(oop_c)::value><<<blocks, 256, 0, d->stream>>>(C);
    };
    using TT = std::true_type;
    using FF = std::false_type;
    if (A.fout) {
      if (idx32) { if (odd) go(TT{}, TT{}, TT{}); else go(FF{}, TT{}, TT{}); }
      else { if (odd) go(TT{}, FF{}, TT{}); else go(FF{}, FF{}, TT{}); }
    } else {
      if (idx32) { if (odd) go(TT{}, TT{}, FF{}); else go(FF{}, TT{}, FF{}); }
      else { if (odd) go(TT{}, FF{}, FF{}); else go(FF{}, FF{}, FF{}); }
    }
    d->launches++;
    return;
  }
  dim3 block(128, 1, 1);
  dim3 grid((A.LX + 127) / 128, A.LY, A.LZ);
  if (A.ns) {
    if (odd) aa_step<T, Q, NS, MODEL, true, PART, true><<<grid, block, 0, d->stream>>>(A);
    else aa_step<T, Q, NS, MODEL, false, PART, true><<<grid, block, 0, d->stream>>>(A);
  } else {
    if (odd) aa_step<T, Q, NS, MODEL, true, PART><<<grid, block, 0, d->stream>>>(A);
    else aa_step<T, Q, NS, MODEL, false, PART><<<grid, block, 0, d->stream>>>(A);
  }
  d->launches++;
}

// One step: a single launch for the flow alone; for two substances, an odd
// step of the compact layout is one launch too (per node the flow, then the
// solute from the slots the flow's pulls found, its u in registers; written
// out of place, for the adjoint's recomputation, it also stores u), and an
// even step is a flow launch that hands u to a solute launch (the solute
// launch only while the solute is active; fused, the even step spilled and
// ran slower).
// With the z faces fused, the face planes' nodes run in a launch of their
// own on the side stream, beside the interior launches: in an AA step every
// node reads and writes only its own set of population slots, the face
// launch carries the flow's u to the solute in registers (it reads no
// handoff value of the interior's), and node-indexed outputs (macro
// variables, plane-record values) are disjoint, so the two touch no common
// location.  Returns true when the face launch went to the side stream: the
// caller joins it back into the step's stream (step_t).
template <typename T, int Q, int NS, int MODEL>
bool launch_aa(lbx_domain* d, const StepArgs<T>& A, bool odd, const Face3Fused<T>* f3)
{
  const bool beside = f3 && d->side;
  if (beside) {
    cudaEventRecord(d->side_fork, d->stream);
    cudaStreamWaitEvent(d->side, d->side_fork, 0);
    launch_face_nodes<T, Q, NS, MODEL>(d, A, odd, *f3, d->side);
  }
  if constexpr (NS == 1) {
    launch_part<T, Q, NS, MODEL, PART_ALL>(d, A, odd, f3);
  } else if (odd && d->layout == LBX_LAYOUT_COMPACT) {
    launch_part<T, Q, NS, MODEL, PART_ALL>(d, A, odd, f3);
  } else {
    launch_part<T, Q, NS, MODEL, PART_FLOW>(d, A, odd, f3);
    if (A.solute_on) launch_part<T, Q, NS, MODEL, PART_SOLUTE>(d, A, odd, f3);
  }
  if (f3 && !beside) launch_face_nodes<T, Q, NS, MODEL>(d, A, odd, *f3, d->stream);
  return beside;
}

template <typename T, int Q, int NS>
bool launch_model(lbx_domain* d, const StepArgs<T>& A, bool odd,
                  const Face3Fused<T>* f3 = nullptr)
{
  const int model = d->p.accurate ? (d->p.compressible ? SHIFTED_COMP : SHIFTED_INC)
                                  : PLAIN_COMP;
  if (model == SHIFTED_INC) return launch_aa<T, Q, NS, SHIFTED_INC>(d, A, odd, f3);
  if (model == PLAIN_COMP) return launch_aa<T, Q, NS, PLAIN_COMP>(d, A, odd, f3);
  return launch_aa<T, Q, NS, SHIFTED_COMP>(d, A, odd, f3);
}

// The stand-alone face kernels, in the order of bcs_1 / bcs_2.
template <typename T>
void launch_faces_exact(lbx_domain* d, int t, bool second)
{
  const lbx_params& p = d->p;
  dim3 block(128), grid((p.LX + 127) / 128);
  for (int s = 0; s < p.nsubs; ++s) {
    const bool compact = d->layout == LBX_LAYOUT_COMPACT;
    T* fs = compact ? (T*)d->fc + (long long)s * d->Q * d->P
                    : (T*)d->f + (long long)s * d->Q * d->N;
    const int shifted = p.accurate && !(s == 1 && p.nsubs == 2);
    const T rhoA = (T)p.rho_A[s];
    auto run = [&](int north, int kind, T rho) {
      const T drho = (T)((double)rho - (double)rhoA);
      if (compact)
        face_row_compact<T><<<grid, block, 0, d->stream>>>(fs, d->fidx, p.LX, p.LY,
                                                           (int)d->P, north, kind,
                                                           second ? 1 : 0, rho, rhoA,
                                                           drho, shifted);
      else
        face_row<T><<<grid, block, 0, d->stream>>>(fs, d->solids, p.LX, p.LY, d->N,
                                                   north, kind, second ? 1 : 0, rho,
                                                   rhoA, drho, shifted);
      d->launches++;
    };
    if (p.pressure_n_in[s]) run(1, FACE_PRESSURE, face_rho<T>(d, s, t, p.pressure_n_in[s], true, d->n_table));
    if (p.pressure_n_out[s]) run(1, FACE_PRESSURE, face_rho<T>(d, s, t, 0, false, d->n_table));
    if (p.pressure_s_in[s]) run(0, FACE_PRESSURE, face_rho<T>(d, s, t, p.pressure_s_in[s], true, d->s_table));
    if (p.pressure_s_out[s]) run(0, FACE_PRESSURE, face_rho<T>(d, s, t, 0, false, d->s_table));
    if (s == 1 && p.nsubs == 2 && p.zeroconcgrad_n) run(1, FACE_ZEROGRAD, T(0));
    if (s == 1 && p.nsubs == 2 && p.zeroconcgrad_s) run(0, FACE_ZEROGRAD, T(0));
  }
}

// The z-face operations of step t in their fixed order (t_in, t_out, b_in,
// b_out per substance, then the solute's constcon t/b and zeroconcgrad t/b),
// as (top, kind, substance, drho) tuples; `run` is called for each.
template <typename T, typename F>
void for_each_face3(const lbx_domain* d, int t, F&& run)
{
  const lbx_params& p = d->p;
  for (int s = 0; s < p.nsubs; ++s) {
    const bool shifted = p.accurate && !(s == 1 && p.nsubs == 2);
    const double rA = shifted ? (double)(T)p.rho_A[s] : 0.0;
    auto dr = [&](bool in) {
      return (T)((double)face_rho<T>(d, s, t, in ? 1 : 0, in, d->n_table) - rA);
    };
    if (p.pressure_t_in[s]) run(1, FACE_PRESSURE, s, dr(true));
    if (p.pressure_t_out[s]) run(1, FACE_PRESSURE, s, dr(false));
    if (p.pressure_b_in[s]) run(0, FACE_PRESSURE, s, dr(true));
    if (p.pressure_b_out[s]) run(0, FACE_PRESSURE, s, dr(false));
    if (p.velocity_t_in[s]) run(1, FACE_VELOCITY, s, (T)p.uz_in);
    if (p.velocity_t_out[s]) run(1, FACE_VELOCITY, s, (T)p.uz_out);
    if (p.velocity_b_in[s]) run(0, FACE_VELOCITY, s, (T)p.uz_in);
    if (p.velocity_b_out[s]) run(0, FACE_VELOCITY, s, (T)p.uz_out);
    if (s == 1 && p.nsubs == 2) {
      if (p.constcon_t_in) run(1, FACE_CONSTCON, s, T(0));
      if (p.constcon_b_in) run(0, FACE_CONSTCON, s, T(0));
      if (p.zeroconcgrad_t) run(1, FACE_ZEROGRAD, s, T(0));
      if (p.zeroconcgrad_b) run(0, FACE_ZEROGRAD, s, T(0));
    }
  }
}

// The face operations of step t grouped by (face, substance), each group in
// the configured order.
template <typename T>
FaceOps<T> face3_table(const lbx_domain* d, int t)
{
  struct Op { int kind; T drho, shift; const T* profile; };
  std::vector<Op> group[4];
  int gtop[4] = {0, 0, 0, 0}, gsubs[4] = {0, 0, 0, 0}, ng = 0;
  for_each_face3<T>(d, t, [&](int top, int kind, int s, T drho) {
    int g = 0;
    while (g < ng && !(gtop[g] == top && gsubs[g] == s)) ++g;
    if (g == ng) { gtop[g] = top; gsubs[g] = s; ++ng; }
    const bool shifted = d->p.accurate && !(s == 1 && d->p.nsubs == 2);
    Op op;
    op.kind = kind;
    op.drho = drho;
    op.shift = kind == FACE_VELOCITY && shifted ? (T)d->p.rho_A[s] : T(0);
    op.profile = kind == FACE_CONSTCON ? (const T*)(top ? d->prof_t : d->prof_b) : nullptr;
    group[g].push_back(op);
  });
  FaceOps<T> ops;
  std::memset(&ops, 0, sizeof ops);
  ops.conc = (T)d->p.rho_sigma_in;
  int q = 0;
  for (int g = 0; g < ng; ++g) {
    ops.top[g] = gtop[g]; ops.subs[g] = gsubs[g];
    ops.first[g] = q;
    ops.count[g] = (int)group[g].size();
    for (const Op& op : group[g]) {
      ops.kind[q] = op.kind; ops.drho[q] = op.drho; ops.shift[q] = op.shift;
      ops.profile[q] = op.profile;
      ++q;
    }
  }
  ops.ngroups = ng;
  return ops;
}

// The same operations for the step kernels (FACES3): per substance and face.
template <typename T>
Face3Fused<T> face3_fused(const lbx_domain* d, int t)
{
  Face3Fused<T> f;
  std::memset(&f, 0, sizeof f);
  f.lo_end = (int)d->plane_fluid[0];
  f.hi_start = (int)(d->fluid - d->plane_fluid[d->p.LZ - 1]);
  f.conc = (T)d->p.rho_sigma_in;
  for_each_face3<T>(d, t, [&](int top, int kind, int s, T drho) {
    int& n = f.nops[s][top];
    const bool shifted = d->p.accurate && !(s == 1 && d->p.nsubs == 2);
    f.kind[s][top][n] = kind;
    f.drho[s][top][n] = drho;
    f.shift[s][top][n] = kind == FACE_VELOCITY && shifted ? (T)d->p.rho_A[s] : T(0);
    f.profile[s][top][n] = kind == FACE_CONSTCON ? (const T*)(top ? d->prof_t : d->prof_b)
                                                 : nullptr;
    ++n;
  });
  return f;
}

template <typename T>
void launch_faces3(lbx_domain* d, int t, bool second)
{
  const lbx_params& p = d->p;
  const bool compact = d->layout == LBX_LAYOUT_COMPACT;
  const long long stride = compact ? d->P : d->N;
  const FaceOps<T> ops = face3_table<T>(d, t);
  if (ops.ngroups == 0) return;
  dim3 block(128), grid((p.LX + 127) / 128, p.LY, ops.ngroups);
  T* f = (T*)(compact ? d->fc : d->f);
  if (compact)
    face_plane<T, true><<<grid, block, 0, d->stream>>>(f, nullptr, d->fidx, p.LX, p.LY, p.LZ,
                                                        stride, second ? 1 : 0, ops);
  else
    face_plane<T, false><<<grid, block, 0, d->stream>>>(f, d->solids, nullptr, p.LX, p.LY, p.LZ,
                                                         stride, second ? 1 : 0, ops);
  d->launches++;
}

template <typename T>
lbx_status step_t(lbx_domain* d, int t, unsigned flags)
{
  const bool odd = (t % 2) != 0;
  const bool idle = solute_faces_idle(d, t);
  if (d->faces_active && (!d->faces_fused || idle)) launch_faces_exact<T>(d, t, !odd);
  // z faces inside the compact step kernel where that is exact (before an
  // even step always, before an odd step with fluid upstream planes); never
  // while recomputing stored states, which keep the stand-alone deposits
  const bool f3_fused = d->faces3_active && d->layout == LBX_LAYOUT_COMPACT && !d->fout &&
                        (!odd || d->faces3_fuse_odd) && !idle;
  if (d->faces3_active && !f3_fused) launch_faces3<T>(d, t, !odd);
  Face3Fused<T> f3;
  if (f3_fused) f3 = face3_fused<T>(d, t);
  StepArgs<T> A = make_args<T>(d, t, flags);
  bool beside = false;   // the face planes' launch is on the side stream
  if (d->Q == 9) {
    if (d->p.nsubs == 1) launch_model<T, 9, 1>(d, A, odd);
    else launch_model<T, 9, 2>(d, A, odd);
  } else {
    if (d->p.nsubs == 1) beside = launch_model<T, 19, 1>(d, A, odd, f3_fused ? &f3 : nullptr);
    else beside = launch_model<T, 19, 2>(d, A, odd, f3_fused ? &f3 : nullptr);
  }
  // a record of a face plane reads values only the face launch wrote: its
  // reduction follows that launch on the side stream, beside the interior
  const bool record_beside = beside && d->btc_vals &&
                             (d->btc_hi <= f3.lo_end || d->btc_lo >= f3.hi_start);
  if (beside && !record_beside) {
    cudaEventRecord(d->side_join, d->side);
    cudaStreamWaitEvent(d->stream, d->side_join, 0);
  }
  if (d->btc_vals) {
    const bool compact = d->layout == LBX_LAYOUT_COMPACT;
    const int count = d->btc_hi - d->btc_lo;
    const int nb = std::max(1, std::min(kBtcMaxBlocks, (count + 1023) / 1024));
    btc_reduce<<<nb, kBtcThreads, 0, record_beside ? d->side : d->stream>>>(
        d->btc_vals, count, compact ? nullptr : d->solids + d->btc_lo,
        (double)d->plane_fluid[d->btc_plane], d->p.nsubs == 2 && A.solute_on, d->btc_rec,
        d->btc_slot, d->btc_cap, d->btc_part, d->btc_ticket);
    d->launches++;
  }
  if (record_beside) {
    cudaEventRecord(d->side_join, d->side);
    cudaStreamWaitEvent(d->stream, d->side_join, 0);
  }
  CK(cudaGetLastError());
  return LBX_OK;
}

lbx_status check_params(const lbx_params* p)
{
  if (!p) return fail(LBX_ERR_INVALID, "params is NULL");
  if (p->dims != 2 && p->dims != 3) return fail(LBX_ERR_INVALID, "dims must be 2 or 3");
  if (p->LX < 1 || p->LY < 1 || p->LZ < 1)
    return fail(LBX_ERR_INVALID, "lattice extents must be positive");
  if (p->dims == 2 && p->LZ != 1) return fail(LBX_ERR_INVALID, "LZ must be 1 in 2D");
  if (p->LY > 65535 || p->LZ > 65535)
    return fail(LBX_ERR_INVALID, "LY and LZ are limited to 65535");
  if ((long long)p->LX * p->LY * p->LZ >= (1LL << 31))
    return fail(LBX_ERR_INVALID, "a domain holds fewer than 2^31 nodes");
  if (p->nsubs != 1 && p->nsubs != 2) return fail(LBX_ERR_INVALID, "nsubs must be 1 or 2");
  if (p->precision != 4 && p->precision != 8)
    return fail(LBX_ERR_INVALID, "precision must be 4 or 8");
  if (p->layout < LBX_LAYOUT_AUTO || p->layout > LBX_LAYOUT_COMPACT)
    return fail(LBX_ERR_INVALID, "layout must be one of LBX_LAYOUT_*");
  if (!p->accurate && !p->compressible)
    return fail(LBX_ERR_INVALID,
                "accurate=0 requires compressible=1 (the reference does not "
                "build ACCURATE 0, COMPRESSIBLE 0)");
  for (int s = 0; s < p->nsubs; ++s)
    if (!(p->tau[s] > 0.5)) return fail(LBX_ERR_INVALID, "tau[%d] must exceed 0.5", s);
  bool faces = false;
  for (int s = 0; s < p->nsubs; ++s)
    faces |= p->pressure_n_in[s] || p->pressure_s_in[s] || p->pressure_n_out[s] ||
             p->pressure_s_out[s];
  faces |= p->nsubs == 2 && (p->zeroconcgrad_n || p->zeroconcgrad_s);
  if (faces && p->dims != 2)
    return fail(LBX_ERR_INVALID, "north/south face boundaries exist for 2D runs only");
  bool faces3 = false, vel3 = false;
  for (int s = 0; s < p->nsubs; ++s) {
    faces3 |= p->pressure_t_in[s] || p->pressure_b_in[s] || p->pressure_t_out[s] ||
              p->pressure_b_out[s];
    vel3 |= p->velocity_t_in[s] || p->velocity_b_in[s] || p->velocity_t_out[s] ||
            p->velocity_b_out[s];
  }
  faces3 |= vel3;
  if (vel3 && !(std::fabs(p->uz_in) < 1. && std::fabs(p->uz_out) < 1.))
    return fail(LBX_ERR_INVALID, "velocity faces need |uz_in|, |uz_out| < 1");
  faces3 |= p->nsubs == 2 && (p->constcon_t_in || p->constcon_b_in || p->zeroconcgrad_t ||
                              p->zeroconcgrad_b);
  if (faces3 && p->dims != 3)
    return fail(LBX_ERR_INVALID, "top/bottom face boundaries exist for 3D runs only");
  if (faces3 && p->LZ < 3) return fail(LBX_ERR_INVALID, "top/bottom faces need LZ >= 3");
  if (p->walsh && (faces || faces3))
    return fail(LBX_ERR_INVALID, "Walsh runs take no face boundaries");
  if (p->walsh && p->layout == LBX_LAYOUT_COMPACT)
    return fail(LBX_ERR_INVALID, "Walsh runs update every node: dense layout only");
  if (faces && p->LY < 3) return fail(LBX_ERR_INVALID, "face boundaries need LY >= 3");
  for (int s = 0; s < p->nsubs; ++s) {
    if (p->pressure_n_in[s] == 2 && (!p->pressure_n_table || p->pressure_n_len < 1))
      return fail(LBX_ERR_INVALID, "pressure_n_in == 2 needs pressure_n_table");
    if (p->pressure_s_in[s] == 2 && (!p->pressure_s_table || p->pressure_s_len < 1))
      return fail(LBX_ERR_INVALID, "pressure_s_in == 2 needs pressure_s_table");
  }
  return LBX_OK;
}

// Fused faces are exact when every configured face node pulls its unknowns
// from a fluid (wrapped) upstream node: then the reference's deposit lands on
// exactly the slot the node pulls and overwrites in the same step.
bool faces_fusable(const lbx_params& p, const uint8_t* sol)
{
  auto solid = [&](int i, int j) {
    i = (i + p.LX) % p.LX; j = (j + p.LY) % p.LY;
    return sol[(long long)i + (long long)p.LX * j] == 1;
  };
  bool north = false, south = false;
  for (int s = 0; s < p.nsubs; ++s) {
    north |= p.pressure_n_in[s] || p.pressure_n_out[s];
    south |= p.pressure_s_in[s] || p.pressure_s_out[s];
  }
  if (p.nsubs == 2) { north |= p.zeroconcgrad_n != 0; south |= p.zeroconcgrad_s != 0; }
  for (int i = 0; i < p.LX; ++i) {
    if (north && !solid(i, p.LY - 1))
      if (solid(i, 0) || solid(i + 1, 0) || solid(i - 1, 0)) return false;
    if (south && !solid(i, 0))
      if (solid(i, p.LY - 1) || solid(i - 1, p.LY - 1) || solid(i + 1, p.LY - 1)) return false;
  }
  return true;
}

// The z faces' deposits before an odd step land only in slots their own
// face node pulls when every upstream node n - c_a of every unknown
// direction a of every fluid node of a configured face is fluid: the
// planes across the periodic z wrap, shifted by the unknowns' in-plane c.
bool faces3_fusable_odd(const lbx_params& p, const uint8_t* sol)
{
  bool top = false, bot = false;
  for (int s = 0; s < p.nsubs; ++s) {
    top |= p.pressure_t_in[s] || p.pressure_t_out[s] || p.velocity_t_in[s] || p.velocity_t_out[s];
    bot |= p.pressure_b_in[s] || p.pressure_b_out[s] || p.velocity_b_in[s] || p.velocity_b_out[s];
  }
  if (p.nsubs == 2) {
    top |= p.constcon_t_in || p.zeroconcgrad_t;
    bot |= p.constcon_b_in || p.zeroconcgrad_b;
  }
  auto solid = [&](int i, int j, int k) {
    i = (i + p.LX) % p.LX; j = (j + p.LY) % p.LY; k = (k + p.LZ) % p.LZ;
    return sol[(long long)i + (long long)p.LX * ((long long)j + (long long)p.LY * k)] == 1;
  };
  // in-plane parts of the unknowns (cz = +1 at the bottom, -1 at the top):
  // (0,0), (+-1,0), (0,+-1)
  const int ux[5] = {0, 1, -1, 0, 0}, uy[5] = {0, 0, 0, 1, -1};
  for (int j = 0; j < p.LY; ++j)
    for (int i = 0; i < p.LX; ++i)
      for (int q = 0; q < 5; ++q) {
        if (bot && !solid(i, j, 0) && solid(i - ux[q], j - uy[q], -1)) return false;
        if (top && !solid(i, j, p.LZ - 1) && solid(i - ux[q], j - uy[q], p.LZ)) return false;
      }
  return true;
}

void release(lbx_domain* d)
{
  lbx_internal_drop_graphs(d);
  cudaFree(d->fc); cudaFree(d->fidx); cudaFree(d->fnode); cudaFree(d->frm);
  cudaFree(d->f); cudaFree(d->mv); cudaFree(d->solids); cudaFree(d->cls);
  cudaFree(d->nbm); cudaFree(d->red);
  cudaFree(d->btc_vals); cudaFree(d->btc_rec); cudaFree(d->btc_slot);
  cudaFree(d->btc_part); cudaFree(d->btc_ticket);
  cudaFree(d->ubuf); cudaFree(d->prof_t); cudaFree(d->prof_b); cudaFree(d->ns);
  lbx_internal_adjoint_free(d);
  lbx_internal_frames_free(d);
  lbx_internal_pest_free(d);
  lbx_internal_tiled_free(d);
  if (d->side) cudaStreamDestroy(d->side);
  if (d->side_fork) cudaEventDestroy(d->side_fork);
  if (d->side_join) cudaEventDestroy(d->side_join);
  if (d->own_stream) cudaStreamDestroy(d->own_stream);
}

lbx_status check_subs(lbx_domain* d, int subs)
{
  if (!d) return fail(LBX_ERR_INVALID, "domain is NULL");
  if (subs < 0 || subs >= d->p.nsubs) return fail(LBX_ERR_INVALID, "subs out of range");
  return LBX_OK;
}

lbx_status do_step(lbx_domain* d, int t, unsigned flags)
{
  const int want_odd = d->parity == 0;
  if (t < 1) return fail(LBX_ERR_INVALID, "time must be >= 1");
  if (((t % 2) != 0) != (want_odd != 0))
    return fail(LBX_ERR_STATE, "step at time %d out of AA order: expected an %s time", t,
                want_odd ? "odd" : "even");
  // a due PEST sample needs the macro variables of this step
  const bool pest = lbx_internal_pest_due(d, t);
  if (pest) flags |= LBX_WRITE_MV;
  lbx_status st = d->real_size == 8 ? step_t<double>(d, t, flags) : step_t<float>(d, t, flags);
  if (st == LBX_OK) {
    d->parity ^= 1;
    if (d->layout == LBX_LAYOUT_COMPACT) d->dense_stale = true;
    if (pest) st = lbx_internal_pest_after(d, t);
  }
  return st;
}

}  // namespace

// The step at time t on the compact state `src` (its face operations in
// place), writing the result to `dst`; no plane record.  Used to recompute
// stored forward states for the adjoint.
lbx_status lbx_internal_step_into(lbx_domain* d, int t, void* src, void* dst)
{
  if (d->layout != LBX_LAYOUT_COMPACT) return fail(LBX_ERR_INVALID, "compact layout required");
  void* fc = d->fc;
  double* bv = d->btc_vals;
  d->fc = src; d->fout = dst; d->btc_vals = nullptr;
  lbx_status st = d->real_size == 8 ? step_t<double>(d, t, 0) : step_t<float>(d, t, 0);
  d->fc = fc; d->fout = nullptr; d->btc_vals = bv;
  return st;
}

namespace {

// The launch arguments of the step at time t, as bytes (for comparing steps:
// two steps with equal bytes launch identical work).
constexpr size_t kKey = 640;   // one step's key: StepArgs bytes + face densities
constexpr int kKeyFaces = 16;  // 2D: 4 per substance; 3D: 4 per substance
static_assert(sizeof(StepArgs<double>) + kKeyFaces * sizeof(double) <= kKey &&
              sizeof(StepArgs<float>) + kKeyFaces * sizeof(double) <= kKey, "step key size");

// The launch arguments of the step at time t, as bytes, followed by the
// densities of every configured face (the stand-alone face kernels take
// them as arguments): two steps with equal keys launch identical work.
size_t step_key(const lbx_domain* d, int t, unsigned char* out)
{
  std::memset(out, 0, kKey);
  size_t len;
  if (d->real_size == 8) {
    fill_args<double>(d, t, 0, *reinterpret_cast<StepArgs<double>*>(out));
    len = sizeof(StepArgs<double>);
  } else {
    fill_args<float>(d, t, 0, *reinterpret_cast<StepArgs<float>*>(out));
    len = sizeof(StepArgs<float>);
  }
  double rho[kKeyFaces] = {0};
  const lbx_params& p = d->p;
  if (d->faces_active) {
    for (int s = 0; s < p.nsubs; ++s) {
      if (p.pressure_n_in[s]) rho[4 * s + 0] = face_rho<double>(d, s, t, p.pressure_n_in[s], true, d->n_table);
      if (p.pressure_n_out[s]) rho[4 * s + 1] = face_rho<double>(d, s, t, 0, false, d->n_table);
      if (p.pressure_s_in[s]) rho[4 * s + 2] = face_rho<double>(d, s, t, p.pressure_s_in[s], true, d->s_table);
      if (p.pressure_s_out[s]) rho[4 * s + 3] = face_rho<double>(d, s, t, 0, false, d->s_table);
    }
  }
  if (d->faces3_active) {
    for (int s = 0; s < p.nsubs; ++s) {
      if (p.pressure_t_in[s] || p.pressure_b_in[s]) rho[8 + 4 * s + 0] = face_rho<double>(d, s, t, 1, true, d->n_table);
      if (p.pressure_t_out[s] || p.pressure_b_out[s]) rho[8 + 4 * s + 1] = face_rho<double>(d, s, t, 0, false, d->n_table);
    }
  }
  std::memcpy(out + len, rho, sizeof rho);
  return len + sizeof rho;
}

// Replay `pairs` AA pairs starting at odd time t from one captured pair.
// Only called when every step of the stretch has the launch arguments of
// the first pair (checked by the caller) and the stream is capturable.
// Captures `npairs` repetitions of the pair (t, t+1) into one graph.
lbx_status capture_pairs(lbx_domain* d, int t, int npairs, cudaGraphExec_t* out,
                         long long* nlaunch)
{
  cudaGraph_t g = nullptr;
  CK(cudaStreamBeginCapture(d->stream, cudaStreamCaptureModeThreadLocal));
  const long long before = d->launches;
  lbx_status st = LBX_OK;
  for (int r = 0; r < npairs && st == LBX_OK; ++r) {
    st = d->real_size == 8 ? step_t<double>(d, t, 0) : step_t<float>(d, t, 0);
    if (st == LBX_OK)
      st = d->real_size == 8 ? step_t<double>(d, t + 1, 0) : step_t<float>(d, t + 1, 0);
  }
  cudaError_t e = cudaStreamEndCapture(d->stream, &g);
  *nlaunch = d->launches - before;
  d->launches = before;
  if (st != LBX_OK) { if (g) cudaGraphDestroy(g); return st; }
  if (e != cudaSuccess) return fail(LBX_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
  e = cudaGraphInstantiate(out, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    *out = nullptr;
    return fail(LBX_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
  }
  return LBX_OK;
}

// `pairs` AA pairs with the launch arguments of the pair at t, replayed from
// graphs of one pair and of kGraphPairs pairs (fewer graph launches, and
// the kernels of a multi-pair graph follow each other without the host).
constexpr int kGraphPairs = 8;

lbx_status replay_pairs(lbx_domain* d, int t, int pairs)
{
  alignas(16) unsigned char key[2 * kKey];
  const size_t k1 = step_key(d, t, key);
  const size_t k2 = step_key(d, t + 1, key + kKey);
  std::memmove(key + k1, key + kKey, k2);
  const size_t klen = k1 + k2;
  if (!d->graph || d->graph_stream != d->stream || d->graph_key_len != klen ||
      std::memcmp(d->graph_key, key, klen) != 0) {
    // both graphs at once, so a later, longer stretch does not pay a capture
    lbx_internal_drop_graphs(d);
    if (lbx_status st = capture_pairs(d, t, 1, &d->graph, &d->graph_launches)) return st;
    long long n = 0;
    if (lbx_status st = capture_pairs(d, t, kGraphPairs, &d->graph_multi, &n)) {
      lbx_internal_drop_graphs(d);
      return st;
    }
    d->graph_stream = d->stream;
    std::memcpy(d->graph_key, key, klen);
    d->graph_key_len = klen;
  }
  // the graphs hold every kernel of their steps (faces and records included)
  for (int r = 0; r < pairs / kGraphPairs; ++r) {
    CK(cudaGraphLaunch(d->graph_multi, d->stream));
    d->launches += kGraphPairs * d->graph_launches;
  }
  for (int r = 0; r < pairs % kGraphPairs; ++r) {
    CK(cudaGraphLaunch(d->graph, d->stream));
    d->launches += d->graph_launches;
  }
  if (d->layout == LBX_LAYOUT_COMPACT) d->dense_stale = true;
  return LBX_OK;
}

// LBX_RUN_AUTO takes the tiled path where every 32 x 16 tile of the
// lattice can have a block (an SM) of its own: there it beat the per-step
// path (D2Q9 FP64 128^2 and 256^2: 1.7x and 1.5x); at 512^2 blocks take
// several tiles each, meet at grid barriers, and lose to it (3x slower).
bool tiled_applies(const lbx_domain* d)
{
  const lbx_params& p = d->p;
  if (d->run_mode == LBX_RUN_STEPS || d->tiled_grid < 0) return false;
  if (p.dims != 2 || p.nsubs != 1 || d->ns || d->btc_vals || d->fout) return false;
  if (d->faces_active && !d->faces_fused) return false;
  if (d->run_mode == LBX_RUN_TILED) return true;
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, p.device) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return (long long)((p.LX + 31) / 32) * ((p.LY + 15) / 16) <= sms;
}

// The tiled path over as many whole, even-numbered rounds as `pairs` AA
// pairs starting at odd time t hold; returns the pairs it advanced.
lbx_status tiled_pairs(lbx_domain* d, int t, int pairs, int* done)
{
  *done = 0;
  const int K = lbx_internal_tiled_steps_per_round(d);
  int rounds = (2 * pairs) / K;
  rounds -= rounds % 2;
  if (rounds < 2) return LBX_OK;
  lbx_status st;
  if (d->real_size == 8) st = lbx_internal_tiled_run<double>(d, make_args<double>(d, t, 0), rounds);
  else st = lbx_internal_tiled_run<float>(d, make_args<float>(d, t, 0), rounds);
  if (st != LBX_OK) return st;
  if (d->layout == LBX_LAYOUT_COMPACT) d->dense_stale = true;
  *done = rounds * K / 2;
  return LBX_OK;
}

// Dense exchange array <-> compact populations.
lbx_status exchange(lbx_domain* d, bool to_compact)
{
  if (d->layout != LBX_LAYOUT_COMPACT || d->fluid == 0) return LBX_OK;
  const int planes = d->p.nsubs * d->Q;
  const long long total = d->fluid * planes;
  const unsigned blocks = (unsigned)((total + 255) / 256);
  if (d->real_size == 8) {
    if (to_compact) gather_compact<double><<<blocks, 256, 0, d->stream>>>((double*)d->fc, (const double*)d->f, d->fnode, (int)d->fluid, (int)d->P, d->N, planes);
    else scatter_compact<double><<<blocks, 256, 0, d->stream>>>((double*)d->f, (const double*)d->fc, d->fnode, (int)d->fluid, (int)d->P, d->N, planes);
  } else {
    if (to_compact) gather_compact<float><<<blocks, 256, 0, d->stream>>>((float*)d->fc, (const float*)d->f, d->fnode, (int)d->fluid, (int)d->P, d->N, planes);
    else scatter_compact<float><<<blocks, 256, 0, d->stream>>>((float*)d->f, (const float*)d->fc, d->fnode, (int)d->fluid, (int)d->P, d->N, planes);
  }
  d->launches++;
  CK(cudaGetLastError());
  if (!to_compact) d->dense_stale = false;
  return LBX_OK;
}

}  // namespace

extern "C" {

void lbx_params_default(lbx_params* p)
{
  std::memset(p, 0, sizeof *p);
  p->dims = 3; p->LX = p->LY = p->LZ = 1; p->nsubs = 1; p->precision = 8;
  p->accurate = 1; p->compressible = 0;
  p->tau[0] = p->tau[1] = 1.0; p->rho_A[0] = p->rho_A[1] = 1.0;
  p->sigma_t_on = 0; p->sigma_t_off = -1;
  p->rho_in = p->rho_out = 1.0; p->pfadd = 1.0; p->pfmul = 0.1;
  p->bc_ramp_start = p->bc_ramp_stop = -1;
  p->rho_sigma_in = 1.0;
}

lbx_status lbx_create(const lbx_params* p, const uint8_t* solids, lbx_domain** out)
{
  if (!out) return fail(LBX_ERR_INVALID, "out is NULL");
  *out = nullptr;
  lbx_status st = check_params(p);
  if (st) return st;
  if (!solids) return fail(LBX_ERR_INVALID, "solids is NULL");
  CK(cudaSetDevice(p->device));
  lbx_domain* d = new lbx_domain();
  d->p = *p;
  d->p.pressure_n_table = nullptr; d->p.pressure_s_table = nullptr;
  if (p->pressure_n_table) d->n_table.assign(p->pressure_n_table, p->pressure_n_table + p->pressure_n_len);
  if (p->pressure_s_table) d->s_table.assign(p->pressure_s_table, p->pressure_s_table + p->pressure_s_len);
  d->Q = p->dims == 2 ? 9 : 19;
  d->D = p->dims;
  d->N = (long long)p->LX * p->LY * p->LZ;
  d->real_size = (size_t)p->precision;
  for (int s = 0; s < p->nsubs; ++s)
    d->faces_active |= p->pressure_n_in[s] || p->pressure_s_in[s] || p->pressure_n_out[s] ||
                       p->pressure_s_out[s];
  d->faces_active |= p->nsubs == 2 && (p->zeroconcgrad_n || p->zeroconcgrad_s);
  d->faces_fused = d->faces_active && faces_fusable(*p, solids);
  for (int s = 0; s < p->nsubs; ++s)
    d->faces3_active |= p->pressure_t_in[s] || p->pressure_b_in[s] || p->pressure_t_out[s] ||
                        p->pressure_b_out[s] || p->velocity_t_in[s] || p->velocity_b_in[s] ||
                        p->velocity_t_out[s] || p->velocity_b_out[s];
  d->faces3_active |= p->nsubs == 2 && (p->constcon_t_in || p->constcon_b_in ||
                                        p->zeroconcgrad_t || p->zeroconcgrad_b);
  d->faces3_fuse_odd = d->faces3_active && faces3_fusable_odd(*p, solids);
  {
    const int planes = p->dims == 2 ? p->LY : p->LZ;
    const long long per = d->N / planes;
    d->plane_fluid.assign(planes, 0);
    for (long long n = 0; n < d->N; ++n) d->plane_fluid[n / per] += solids[n] != 1;
    for (int q = 0; q < planes; ++q) d->fluid += d->plane_fluid[q];
  }
  d->layout = p->layout == LBX_LAYOUT_AUTO
                  ? ((d->N - d->fluid) * 20 >= d->N && !p->walsh ? LBX_LAYOUT_COMPACT
                                                                 : LBX_LAYOUT_DENSE)
                  : p->layout;

  auto bail = [&](lbx_status s) { release(d); delete d; return s; };
  cudaError_t e;
#define CKD(call)                                                                  \
  if ((e = (call)) != cudaSuccess)                                                 \
    return bail(fail(e == cudaErrorMemoryAllocation ? LBX_ERR_NOMEM : LBX_ERR_CUDA, \
                     "%s: %s", #call, cudaGetErrorString(e)));
  CKD(cudaStreamCreateWithFlags(&d->own_stream, cudaStreamNonBlocking));
  d->stream = d->own_stream;
  if (d->faces3_active && d->layout == LBX_LAYOUT_COMPACT) {
    CKD(cudaStreamCreateWithFlags(&d->side, cudaStreamNonBlocking));
    CKD(cudaEventCreateWithFlags(&d->side_fork, cudaEventDisableTiming));
    CKD(cudaEventCreateWithFlags(&d->side_join, cudaEventDisableTiming));
  }
  const size_t fbytes = (size_t)p->nsubs * d->Q * d->N * d->real_size;
  const size_t mvbytes = (size_t)p->nsubs * (1 + d->D) * d->N * d->real_size;
  CKD(cudaMalloc(&d->f, fbytes));
  CKD(cudaMalloc(&d->mv, mvbytes));
  CKD(cudaMalloc(&d->solids, d->N));
  CKD(cudaMalloc(&d->cls, d->N));
  CKD(cudaMalloc(&d->nbm, d->N * sizeof(uint32_t)));
  d->red_blocks = 2 * 148;
  CKD(cudaMalloc(&d->red, d->red_blocks * sizeof(RedPartial)));
  if (d->layout == LBX_LAYOUT_COMPACT) {
    std::vector<int> fidx(d->N), fnode(d->fluid > 0 ? d->fluid : 1);
    int m = 0;
    for (long long n = 0; n < d->N; ++n) {
      if (solids[n] == 1) fidx[n] = -1;
      else { fidx[n] = m; fnode[m++] = (int)n; }
    }
    d->P = (d->fluid + 31) / 32 * 32;
    CKD(cudaMalloc(&d->fc, std::max<size_t>(1, (size_t)p->nsubs * d->Q * d->P * d->real_size)));
    CKD(cudaMalloc(&d->fidx, d->N * sizeof(int)));
    CKD(cudaMalloc(&d->fnode, fnode.size() * sizeof(int)));
    CKD(cudaMemcpy(d->fidx, fidx.data(), d->N * sizeof(int), cudaMemcpyHostToDevice));
    CKD(cudaMemcpy(d->fnode, fnode.data(), fnode.size() * sizeof(int), cudaMemcpyHostToDevice));
    {
      // the fluid bitmask in 32-node words, each with the number of fluid
      // nodes before it: the compact index of fluid node n is the word's
      // rank plus the fluid bits below n.  A guard word with no fluid bits
      // on either side (ranks 0 and F) lets the odd step read the words
      // around node 0 and node N - 1 without bounds checks.
      const long long W = (d->N + 31) / 32;
      std::vector<uint2> frm((size_t)W + 2);
      unsigned rank = 0;
      frm[0] = make_uint2(0u, 0u);
      for (long long w = 0; w < W; ++w) {
        unsigned bits = 0;
        for (int b = 0; b < 32; ++b) {
          const long long n = w * 32 + b;
          if (n < d->N && solids[n] != 1) bits |= 1u << b;
        }
        frm[(size_t)w + 1] = make_uint2(rank, bits);
        rank += (unsigned)__builtin_popcount(bits);
      }
      frm[(size_t)W + 1] = make_uint2(rank, 0u);
      CKD(cudaMalloc(&d->frm, ((size_t)W + 2) * sizeof(uint2)));
      CKD(cudaMemcpy(d->frm, frm.data(), ((size_t)W + 2) * sizeof(uint2),
                     cudaMemcpyHostToDevice));
    }
    CKD(cudaMemsetAsync(d->fc, 0, std::max<size_t>(1, (size_t)p->nsubs * d->Q * d->P * d->real_size), d->stream));
  }
  if (p->nsubs == 2) {
    const long long us = d->layout == LBX_LAYOUT_COMPACT ? d->P : d->N;
    CKD(cudaMalloc(&d->ubuf, std::max<size_t>(1, (size_t)3 * us * d->real_size)));
  }
  if (p->walsh) {
    CKD(cudaMalloc(&d->ns, d->N * d->real_size));
    CKD(cudaMemsetAsync(d->ns, 0, d->N * d->real_size, d->stream));
  }
  CKD(cudaMemsetAsync(d->f, 0, fbytes, d->stream));
  CKD(cudaMemsetAsync(d->mv, 0, mvbytes, d->stream));
  CKD(cudaMemcpyAsync(d->solids, solids, d->N, cudaMemcpyHostToDevice, d->stream));
  {
    dim3 block(128), grid((p->LX + 127) / 128, p->LY, p->LZ);
    if (d->Q == 9) classify<9><<<grid, block, 0, d->stream>>>(d->solids, d->cls, d->nbm, p->LX, p->LY, p->LZ);
    else classify<19><<<grid, block, 0, d->stream>>>(d->solids, d->cls, d->nbm, p->LX, p->LY, p->LZ);
    d->launches++;
  }
  CKD(cudaGetLastError());
  CKD(cudaStreamSynchronize(d->stream));
#undef CKD
  *out = d;
  return LBX_OK;
}

lbx_status lbx_destroy(lbx_domain* d)
{
  if (!d) return LBX_OK;
  if (d->stream) cudaStreamSynchronize(d->stream);
  release(d);
  delete d;
  return LBX_OK;
}

lbx_status lbx_upload_f(lbx_domain* d, int subs, const void* f_host)
{
  if (lbx_status st = check_subs(d, subs)) return st;
  if (!f_host) return fail(LBX_ERR_INVALID, "f_host is NULL");
  const size_t bytes = (size_t)d->Q * d->N * d->real_size;
  // the other substance's dense copy must be current before the gather; a
  // single substance is overwritten whole, so its stale copy is not brought
  // back first
  if (d->dense_stale && d->p.nsubs > 1) {
    if (lbx_status st = exchange(d, false)) return st;
  }
  CK(cudaMemcpyAsync((char*)d->f + subs * bytes, f_host, bytes, cudaMemcpyHostToDevice,
                     d->stream));
  if (lbx_status st = exchange(d, true)) return st;
  CK(cudaStreamSynchronize(d->stream));
  d->dense_stale = false;   // the compact state was just gathered from it
  d->parity = 0;
  return LBX_OK;
}

lbx_status lbx_download_f(lbx_domain* d, int subs, void* f_host)
{
  if (lbx_status st = check_subs(d, subs)) return st;
  if (!f_host) return fail(LBX_ERR_INVALID, "f_host is NULL");
  const size_t bytes = (size_t)d->Q * d->N * d->real_size;
  if (d->dense_stale) { if (lbx_status st = exchange(d, false)) return st; }
  CK(cudaMemcpyAsync(f_host, (char*)d->f + subs * bytes, bytes, cudaMemcpyDeviceToHost,
                     d->stream));
  CK(cudaStreamSynchronize(d->stream));
  return LBX_OK;
}

lbx_status lbx_upload_mv(lbx_domain* d, int subs, const void* mv_host)
{
  if (lbx_status st = check_subs(d, subs)) return st;
  if (!mv_host) return fail(LBX_ERR_INVALID, "mv_host is NULL");
  const size_t bytes = (size_t)(1 + d->D) * d->N * d->real_size;
  CK(cudaMemcpyAsync((char*)d->mv + subs * bytes, mv_host, bytes, cudaMemcpyHostToDevice,
                     d->stream));
  CK(cudaStreamSynchronize(d->stream));
  return LBX_OK;
}

lbx_status lbx_download_mv(lbx_domain* d, int subs, void* rho, void* ux, void* uy, void* uz)
{
  if (lbx_status st = check_subs(d, subs)) return st;
  const size_t plane = (size_t)d->N * d->real_size;
  char* base = (char*)d->mv + (size_t)subs * (1 + d->D) * plane;
  void* dst[4] = {rho, ux, uy, uz};
  for (int c = 0; c <= d->D; ++c)
    if (dst[c])
      CK(cudaMemcpyAsync(dst[c], base + c * plane, plane, cudaMemcpyDeviceToHost, d->stream));
  CK(cudaStreamSynchronize(d->stream));
  return LBX_OK;
}

lbx_status lbx_init_equilibrium(lbx_domain* d, int subs, const void* rho, const void* ux,
                                const void* uy, const void* uz)
{
  if (lbx_status st = check_subs(d, subs)) return st;
  if (!rho) return fail(LBX_ERR_INVALID, "rho is required");
  // as in lbx_upload_f: the other substance's dense copy must be current
  // before the gather; a single substance is overwritten whole, so its
  // stale copy is not brought back first
  if (d->dense_stale && d->p.nsubs > 1) {
    if (lbx_status st = exchange(d, false)) return st;
  }
  // the fields land in the substance's macro variables, where the
  // reference's init_problem leaves them (src/latman.c:1302-1780), and the
  // populations are formed from there: no staging allocation.  A velocity
  // component given as NULL is zero, filled on the device (init_problem
  // always starts at rest, so only rho need cross the host link)
  const size_t plane = (size_t)d->N * d->real_size;
  char* t = (char*)d->mv + (size_t)subs * (1 + d->D) * plane;
  const void* src[4] = {rho, ux, uy, uz};
  cudaError_t e = cudaSuccess;
  for (int c = 0; c <= d->D && e == cudaSuccess; ++c)
    e = src[c] ? cudaMemcpyAsync(t + c * plane, src[c], plane, cudaMemcpyHostToDevice, d->stream)
               : cudaMemsetAsync(t + c * plane, 0, plane, d->stream);
  if (e == cudaSuccess) {
    const int shifted = d->p.accurate && subs == 0;
    const unsigned blocks = (unsigned)((d->N + 255) / 256);
    if (d->real_size == 8) {
      double* fs = (double*)d->f + (long long)subs * d->Q * d->N;
      const double* uzp = d->D == 3 ? (const double*)(t + 3 * plane) : nullptr;
      if (d->Q == 9) init_feq<double, 9><<<blocks, 256, 0, d->stream>>>(fs, (double*)t, (double*)(t + plane), (double*)(t + 2 * plane), uzp, d->N, shifted);
      else init_feq<double, 19><<<blocks, 256, 0, d->stream>>>(fs, (double*)t, (double*)(t + plane), (double*)(t + 2 * plane), uzp, d->N, shifted);
    } else {
      float* fs = (float*)d->f + (long long)subs * d->Q * d->N;
      const float* uzp = d->D == 3 ? (const float*)(t + 3 * plane) : nullptr;
      if (d->Q == 9) init_feq<float, 9><<<blocks, 256, 0, d->stream>>>(fs, (float*)t, (float*)(t + plane), (float*)(t + 2 * plane), uzp, d->N, shifted);
      else init_feq<float, 19><<<blocks, 256, 0, d->stream>>>(fs, (float*)t, (float*)(t + plane), (float*)(t + 2 * plane), uzp, d->N, shifted);
    }
    d->launches++;
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && d->layout == LBX_LAYOUT_COMPACT) {
    if (exchange(d, true) != LBX_OK) e = cudaErrorUnknown;
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(d->stream);
  if (e != cudaSuccess) return fail(LBX_ERR_CUDA, "init_equilibrium: %s", cudaGetErrorString(e));
  d->dense_stale = false;   // the compact state was just gathered from it
  d->parity = 0;
  return LBX_OK;
}

lbx_status lbx_step(lbx_domain* d, int time, unsigned flags)
{
  if (!d) return fail(LBX_ERR_INVALID, "domain is NULL");
  return do_step(d, time, flags);
}

lbx_status lbx_step_pair(lbx_domain* d, int time, unsigned flags)
{
  if (!d) return fail(LBX_ERR_INVALID, "domain is NULL");
  if (lbx_status st = do_step(d, time, flags)) return st;
  return do_step(d, time + 1, flags);
}

lbx_status lbx_run(lbx_domain* d, int t0, int nsteps, int frame_rate)
{
  if (!d) return fail(LBX_ERR_INVALID, "domain is NULL");
  if (nsteps < 0) return fail(LBX_ERR_INVALID, "nsteps must be >= 0");
  const int tend = t0 + nsteps;
  int t = t0 + 1;
  alignas(16) unsigned char k_odd[kKey], k_even[kKey], k[kKey];
  while (t <= tend) {
    const bool frame = frame_rate > 0 && t % frame_rate == 0;
    // a stretch of >= 4 frame-free steps starting on an odd time, with the
    // launch arguments of its first pair throughout, is replayed from a graph
    if (!frame && (t % 2) == 1 && d->parity == 0 && d->stream != nullptr && tend - t + 1 >= 4) {
      const size_t ko = step_key(d, t, k_odd), ke = step_key(d, t + 1, k_even);
      int pairs = 0;
      for (int u = t; u + 1 <= tend; u += 2) {
        if (frame_rate > 0 && (u % frame_rate == 0 || (u + 1) % frame_rate == 0)) break;
        if (lbx_internal_pest_due(d, u) || lbx_internal_pest_due(d, u + 1)) break;
        if (pairs > 0 && (step_key(d, u, k) != ko || std::memcmp(k, k_odd, ko) ||
                          step_key(d, u + 1, k) != ke || std::memcmp(k, k_even, ke)))
          break;
        ++pairs;
      }
      if (pairs >= 2) {
        int done = 0;
        if (tiled_applies(d)) {
          if (lbx_status st = tiled_pairs(d, t, pairs, &done)) return st;
          t += 2 * done;
          pairs -= done;
        }
        if (pairs > 0) {
          if (lbx_status st = replay_pairs(d, t, pairs)) return st;
          t += 2 * pairs;
        }
        continue;
      }
    }
    if (lbx_status st = do_step(d, t, frame ? LBX_WRITE_MV : 0u)) return st;
    ++t;
  }
  return LBX_OK;
}

lbx_status lbx_set_run_mode(lbx_domain* d, int mode)
{
  if (!d) return fail(LBX_ERR_INVALID, "domain is NULL");
  if (mode != LBX_RUN_AUTO && mode != LBX_RUN_STEPS && mode != LBX_RUN_TILED)
    return fail(LBX_ERR_INVALID, "unknown run mode %d", mode);
  d->run_mode = mode;
  return LBX_OK;
}

lbx_status lbx_set_stream(lbx_domain* d, void* stream)
{
  if (!d) return fail(LBX_ERR_INVALID, "domain is NULL");
  CK(cudaStreamSynchronize(d->stream));
  d->stream = (cudaStream_t)stream;
  return LBX_OK;
}

lbx_status lbx_sync(lbx_domain* d)
{
  if (!d) return fail(LBX_ERR_INVALID, "domain is NULL");
  CK(cudaStreamSynchronize(d->stream));
  CK(cudaGetLastError());
  return lbx_internal_tiled_status(d);
}

lbx_status lbx_reduce(lbx_domain* d, lbx_reductions* out)
{
  if (!d || !out) return fail(LBX_ERR_INVALID, "NULL argument");
  const int nb = d->red_blocks;
  RedPartial* red = (RedPartial*)d->red;
  if (d->real_size == 8) {
    if (d->D == 2) reduce_mv<double, 2><<<nb, 256, 0, d->stream>>>((const double*)d->mv, d->solids, d->N, d->p.nsubs, red);
    else reduce_mv<double, 3><<<nb, 256, 0, d->stream>>>((const double*)d->mv, d->solids, d->N, d->p.nsubs, red);
  } else {
    if (d->D == 2) reduce_mv<float, 2><<<nb, 256, 0, d->stream>>>((const float*)d->mv, d->solids, d->N, d->p.nsubs, red);
    else reduce_mv<float, 3><<<nb, 256, 0, d->stream>>>((const float*)d->mv, d->solids, d->N, d->p.nsubs, red);
  }
  d->launches++;
  CK(cudaGetLastError());
  std::vector<RedPartial> h(nb);
  CK(cudaMemcpyAsync(h.data(), red, nb * sizeof(RedPartial), cudaMemcpyDeviceToHost, d->stream));
  CK(cudaStreamSynchronize(d->stream));
  std::memset(out, 0, sizeof *out);
  out->rho_min = 1e300; out->rho_max = -1e300;
  unsigned long long fl = 0, nf = 0;
  for (const RedPartial& r : h) {
    out->mass += r.mass; out->solute_mass += r.solute;
    for (int c = 0; c < 3; ++c) { out->momentum[c] += r.mom[c]; out->u_sum[c] += r.usum[c]; }
    out->rho_min = r.rmin < out->rho_min ? r.rmin : out->rho_min;
    out->rho_max = r.rmax > out->rho_max ? r.rmax : out->rho_max;
    fl += r.fluid; nf += r.nonfinite;
  }
  out->fluid_nodes = (long long)fl;
  out->nonfinite = (int)nf;
  if (nf) return fail(LBX_ERR_NUMERIC, "%llu fluid nodes hold non-finite macro variables", nf);
  return LBX_OK;
}

lbx_status lbx_device_f(lbx_domain* d, void** ptr)
{
  if (!d || !ptr) return fail(LBX_ERR_INVALID, "NULL argument");
  if (d->dense_stale) { if (lbx_status st = exchange(d, false)) return st; }
  CK(cudaStreamSynchronize(d->stream));
  *ptr = d->f;
  return LBX_OK;
}

lbx_status lbx_device_mv(lbx_domain* d, void** ptr)
{
  if (!d || !ptr) return fail(LBX_ERR_INVALID, "NULL argument");
  *ptr = d->mv;
  return LBX_OK;
}

lbx_status lbx_info(lbx_domain* d, long long* fluid_nodes, int* faces_fused, int* layout)
{
  if (!d) return fail(LBX_ERR_INVALID, "domain is NULL");
  if (fluid_nodes) *fluid_nodes = d->fluid;
  if (faces_fused) *faces_fused = d->faces_fused ? 1 : 0;
  if (layout) *layout = d->layout;
  return LBX_OK;
}

long long lbx_launch_count(lbx_domain* d) { return d ? d->launches : -1; }

lbx_status lbx_btc_stop(lbx_domain* d)
{
  if (!d) return fail(LBX_ERR_INVALID, "domain is NULL");
  if (d->btc_vals) {
    CK(cudaStreamSynchronize(d->stream));
    lbx_internal_drop_graphs(d);
  }
  cudaFree(d->btc_vals); cudaFree(d->btc_rec); cudaFree(d->btc_slot);
  cudaFree(d->btc_part); cudaFree(d->btc_ticket);
  d->btc_vals = nullptr; d->btc_rec = nullptr; d->btc_slot = nullptr;
  d->btc_part = nullptr; d->btc_ticket = nullptr;
  d->btc_cap = 0;
  return LBX_OK;
}

lbx_status lbx_btc_start(lbx_domain* d, int plane, int capacity)
{
  if (!d) return fail(LBX_ERR_INVALID, "domain is NULL");
  const int planes = d->p.dims == 2 ? d->p.LY : d->p.LZ;
  if (plane < 0 || plane >= planes) return fail(LBX_ERR_INVALID, "plane %d out of range", plane);
  if (capacity < 1) return fail(LBX_ERR_INVALID, "capacity must be positive");
  lbx_status st = lbx_btc_stop(d);
  if (st) return st;
  const long long per = d->N / planes;
  long long lo, hi;
  if (d->layout == LBX_LAYOUT_COMPACT) {
    lo = 0;
    for (int q = 0; q < plane; ++q) lo += d->plane_fluid[q];
    hi = lo + d->plane_fluid[plane];
  } else {
    lo = per * plane;
    hi = lo + per;
  }
  d->btc_lo = (int)lo; d->btc_hi = (int)hi;
  d->btc_plane = plane;
  d->btc_cap = capacity;
  CK(cudaMalloc(&d->btc_vals, 2 * std::max<long long>(1, hi - lo) * sizeof(double)));
  CK(cudaMalloc(&d->btc_rec, (size_t)capacity * 2 * sizeof(double)));
  CK(cudaMalloc(&d->btc_slot, sizeof(int)));
  CK(cudaMalloc(&d->btc_part, 2 * kBtcMaxBlocks * sizeof(double)));
  CK(cudaMalloc(&d->btc_ticket, sizeof(unsigned)));
  CK(cudaMemsetAsync(d->btc_slot, 0, sizeof(int), d->stream));
  CK(cudaMemsetAsync(d->btc_ticket, 0, sizeof(unsigned), d->stream));
  // the step arguments changed: a captured pair no longer matches
  if (d->graph) { CK(cudaStreamSynchronize(d->stream)); lbx_internal_drop_graphs(d); }
  return LBX_OK;
}

lbx_status lbx_btc_read(lbx_domain* d, double* c_out, double* ux_out, int max,
                        long long* count)
{
  if (!d || (!c_out && !ux_out && max > 0)) return fail(LBX_ERR_INVALID, "NULL argument");
  if (!d->btc_slot) return fail(LBX_ERR_STATE, "no plane record started");
  int slot = 0;
  CK(cudaMemcpyAsync(&slot, d->btc_slot, sizeof(int), cudaMemcpyDeviceToHost, d->stream));
  CK(cudaStreamSynchronize(d->stream));
  const int n = std::min(std::min(slot, d->btc_cap), std::max(max, 0));
  if (n > 0) {
    std::vector<double> rec((size_t)2 * n);
    CK(cudaMemcpyAsync(rec.data(), d->btc_rec, rec.size() * sizeof(double),
                       cudaMemcpyDeviceToHost, d->stream));
    CK(cudaStreamSynchronize(d->stream));
    for (int q = 0; q < n; ++q) {
      if (c_out) c_out[q] = rec[2 * q];
      if (ux_out) ux_out[q] = rec[2 * q + 1];
    }
  }
  if (count) *count = slot;
  return LBX_OK;
}

lbx_status lbx_set_face_profile(lbx_domain* d, int top, const double* conc)
{
  if (!d) return fail(LBX_ERR_INVALID, "domain is NULL");
  void*& dst = top ? d->prof_t : d->prof_b;
  CK(cudaStreamSynchronize(d->stream));
  lbx_internal_drop_graphs(d);
  if (!conc) { cudaFree(dst); dst = nullptr; return LBX_OK; }
  const size_t n = (size_t)d->p.LX * d->p.LY;
  if (!dst) CK(cudaMalloc(&dst, n * d->real_size));
  if (d->real_size == 8) {
    CK(cudaMemcpy(dst, conc, n * sizeof(double), cudaMemcpyHostToDevice));
  } else {
    std::vector<float> h(conc, conc + n);
    CK(cudaMemcpy(dst, h.data(), n * sizeof(float), cudaMemcpyHostToDevice));
  }
  return LBX_OK;
}

lbx_status lbx_set_ns(lbx_domain* d, const double* ns)
{
  if (!d) return fail(LBX_ERR_INVALID, "domain is NULL");
  if (!d->ns) return fail(LBX_ERR_STATE, "domain was created without walsh");
  if (!ns) return fail(LBX_ERR_INVALID, "ns is NULL");
  for (long long n = 0; n < d->N; ++n)
    if (!(ns[n] >= 0. && ns[n] <= 1.))
      return fail(LBX_ERR_INVALID, "ns[%lld] = %g is outside [0, 1]", n, ns[n]);
  CK(cudaStreamSynchronize(d->stream));
  if (d->real_size == 8) {
    CK(cudaMemcpy(d->ns, ns, d->N * sizeof(double), cudaMemcpyHostToDevice));
  } else {
    std::vector<float> h(ns, ns + d->N);
    CK(cudaMemcpy(d->ns, h.data(), d->N * sizeof(float), cudaMemcpyHostToDevice));
  }
  return LBX_OK;
}

const char* lbx_last_error(void) { return g_err.c_str(); }

}  // extern "C"
