// lbx_adjoint.cu -- discrete adjoint of the compact AA step (reverse
// stream-collide) with checkpointing, for gradients of plane objectives with
// respect to the body force, tau, tau_solute and a constant-concentration
// face profile.  No counterpart in the reference.
//
// Forward step t (lbx_step): the face operations of step t on the memory
// state, then the AA kernel (odd: pull, collide, push; even: swapped local
// load, collide, natural store).  Per node the AA kernel reads each slot of
// its own exclusive slot set once and writes each once, so its adjoint has
// the same access pattern with reads and writes exchanged and runs in place:
// the adjoint of the slot node n wrote d'_a to is read, the collision's
// transposed Jacobian applied, and the result written to the slot d_a was
// read from.
//
// Collision adjoints (shifted incompressible flow, omega = 1/tau):
//   d'_a = (1-w) d_a + w W_a drho + w W_a rho_A P_a(u),
//   P_a = 3 c_a.u + 4.5 (c_a.u)^2 - 1.5 u.u,  u = sum_b c_b d_b / rho_A + tau g,
//   lam_b = (1-w) lam'_b + w sum_a W_a lam'_a + c_b . mu / rho_A,
//   mu = w rho_A sum_a lam'_a W_a (3 c_a + 9 (c_a.u) c_a - 3 u) + mu_ext,
//   dJ/dg += tau mu,  dJ/dtau += sum_a lam'_a (d_a - deq_a) / tau^2 + mu . g;
// solute (Inamuro sigma, C_eff = C s1^k, s1 = 1 - sink tau_s, k = 1 odd /
// 2 even):
//   g'_a = (1-w_s) g_a + w_s W_a C_eff (1 + 3 c_a.u),
//   B = w_s sum_a lam'_a W_a (1 + 3 c_a.u) + dJ/dC_eff,
//   lam_b = (1-w_s) lam'_b + s1^k B,  mu_ext(flow) = w_s C_eff sum_a lam'_a W_a 3 c_a,
//   dJ/dtau_s += sum_a lam'_a (g_a - W_a C_eff (1+3 c_a.u)) / tau_s^2 + B dC_eff/dtau_s.
// The solute's adjoint runs first (it hands mu_ext to the flow's), mirroring
// the forward split.  Adjoint populations are in the run's precision; every
// parameter-gradient sum is FP64.
//
// Checkpoints: lbx_adjoint_forward stores the state every K steps; the
// backward sweep restores one, recomputes its K steps out of place into K+1
// stored states, and runs the adjoint steps back through them.
#include "lbx.h"
#include "lbx_internal.h"
#include "lbx_kernels.cuh"

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <type_traits>
#include <vector>

using namespace lbx;

namespace {

lbx_status afail(lbx_status code, const char* fmt, ...)
{
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  return lbx_internal_fail(code, buf);
}

#define ACK(call)                                                               \
  do {                                                                          \
    cudaError_t e_ = (call);                                                    \
    if (e_ != cudaSuccess)                                                      \
      return afail(e_ == cudaErrorMemoryAllocation ? LBX_ERR_NOMEM : LBX_ERR_CUDA, \
                   "%s: %s", #call, cudaGetErrorString(e_));                    \
  } while (0)

template <typename T>
struct AdjArgs {
  const T* S;              // forward state before the step's AA kernel [nsubs][Q][P]
  T* L;                    // adjoint state [nsubs][Q][P], updated in place
  const T* uhist;          // [3][P]: the flow's u of this step (solute kernel)
  const int* fidx;
  const int* fnode;
  int F, P, LX, LY, LZ;
  FastDiv div_plane, div_lx;
  SubsConst<T> sc[2];
  T sink1;
  double tau[2], g[3], sink;
  int obj_lo, obj_hi;      // compact range of the objective plane's nodes
  T wc, wu;                // this step's seeds: dJ/dC_eff, dJ/du_x per plane node
  double* acc;             // [blocks][5]: per-block sums of dJ/dg_x, dJ/dg_y,
                           // dJ/dg_z, dJ/dtau, dJ/dtau_s over all steps
  // the solute's z-face adjoint applied in the step kernel (see adj_face_local)
  int face_on;             // 1: apply it at this step's face-plane nodes
  int face_lo_end, face_hi_start;   // face planes: compact [0, lo_end), [hi_start, F)
  int face_kind[2];        // bottom, top: 0, FACE_CONSTCON or FACE_ZEROGRAD
  double* face_dprof[2];   // bottom, top: constant-concentration profile gradient
};

// The adjoint of the solute's face operation of a face node, applied to the
// adjoints the step kernel is about to store at the node's slots (l[a] at
// the slot it loaded d_a from).  Where the faces fuse into the step (every
// unknown's upstream node fluid before an odd step; always before an even
// one), the forward deposited the unknowns in slots the node itself then
// read, and every slot the adjoint of the face operation touches is one of
// the node's own: the same arithmetic, in the same order, as adj_face_plane
// on the stored values, without a launch of its own.  TOP is a compile-time
// constant so that l stays in registers.
template <typename T, int Q, bool TOP>
__device__ __forceinline__ void adj_face_local(T (&l)[Q], int kind, double* dprof, int ij)
{
  if constexpr (Q == 19) {
    T wsum = wgt<T, 19>(face3_unknown(TOP, 0));
#pragma unroll
    for (int q = 1; q < 5; ++q) wsum = wsum + wgt<T, 19>(face3_unknown(TOP, q));
    T Ax = T(0);
#pragma unroll
    for (int q = 0; q < 5; ++q) Ax += wgt<T, 19>(face3_unknown(TOP, q)) * l[face3_unknown(TOP, q)];
    const T ax = Ax / wsum;
#pragma unroll
    for (int q = 0; q < 5; ++q) l[face3_unknown(TOP, q)] = T(0);
    if (kind == FACE_ZEROGRAD) {
#pragma unroll
      for (int a = 0; a < 19; ++a)
        if (cz(a) == (TOP ? 1 : -1)) l[a] = l[a] + ax;
    } else {
#pragma unroll
      for (int a = 0; a < 19; ++a)
        if (cz(a) != (TOP ? -1 : 1)) l[a] = l[a] - ax;
      if (dprof) dprof[ij] += (double)ax;
    }
  }
}

// Sum of v over the block, added by one thread to this block's own row of
// partial sums (out[q], q < NV).  A block index covers the same nodes in
// every step, so rows need no atomics, and the final sum over rows (on the
// host, in block order) is reproducible.
template <int NV>
__device__ __forceinline__ void block_add(double (&v)[NV], double* out)
{
  __shared__ double part[NV][8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    double x = v[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) part[q][warp] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      double x = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) x += part[q][w];
      out[q] += x;
    }
  }
}

// Adjoint of one AA kernel launch on the compact layout: the solute's
// (WITH_SOLUTE, first, as the forward's solute depends on the flow's u) and
// then the flow's, handing dJ/du between them in registers.  256 threads per block, every thread reaches the block reduction.
// The slots come from a shared-memory table filled once per node (as in
// the forward kernel); lam' is loaded first and the forward populations
// stream through running sums, so one 19-value array is live at a time.
// The solute reads the flow's u of the step from the recompute pass.
// Resident 256-thread blocks: in FP32 four (64 registers), with or without
// the solute phase: with the slot table neither spills there (cfg5's
// backward 3 % faster than at three blocks; five blocks spill and lose);
// FP64 keeps about its natural register count (lower caps spill).
template <typename T, bool WITH_SOLUTE>
constexpr int adj_min_blocks() { return sizeof(T) == 4 ? 4 : 2; }

template <typename T, int Q, bool ODD, bool WITH_SOLUTE, bool IDX32>
__global__ void __launch_bounds__(256, (adj_min_blocks<T, WITH_SOLUTE>()))
adj_step(AdjArgs<T> A)
{
  constexpr int D = (Q == 9) ? 2 : 3;
  using Idx = typename std::conditional<IDX32, unsigned, size_t>::type;
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = m < A.F;
  double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  if (live) {
    const Idx F = (Idx)A.P;
    int n = 0, xm = 0, xp = 0, ym = 0, yp = 0, zm = 0, zp = 0;
    if (ODD) {
      const int plane = A.LX * A.LY;
      n = A.fnode[m];
      const int k = fast_div(n, A.div_plane);
      const int r = n - k * plane;
      const int j = fast_div(r, A.div_lx);
      const int i = r - j * A.LX;
      xm = (i == 0) ? A.LX - 1 : -1; xp = (i == A.LX - 1) ? 1 - A.LX : 1;
      ym = (j == 0) ? plane - A.LX : -A.LX; yp = (j == A.LY - 1) ? A.LX - plane : A.LX;
      if (D == 3) {
        const int tot = plane * A.LZ;
        zm = (k == 0) ? tot - plane : -plane;
        zp = (k == A.LZ - 1) ? plane - tot : plane;
      }
    }
    auto off = [&](int a) -> int {
      return (cx(a) < 0 ? xm : (cx(a) > 0 ? xp : 0)) + (cy(a) < 0 ? ym : (cy(a) > 0 ? yp : 0)) +
             (cz(a) < 0 ? zm : (cz(a) > 0 ? zp : 0));
    };
    const int* const fidx_n = A.fidx + n;
    int mm = m;   // laundered between phases so slot addresses are not kept live
    // The slot the forward read d_a from (odd step: slot a of the upstream
    // node n - c_a, or the node's own opp(a) behind a solid), once per node
    // into this thread's column of a shared-memory table; the slot it wrote
    // d'_a to is the one it read d_opp(a) from (the AA pairing), so the table
    // gives both.  Looked up at every use instead (114 index loads per node
    // over the two phases), the lookups' instructions dominated the kernel.
    __shared__ Idx slot_tab[ODD ? Q : 1][256];
    if (ODD) {
#pragma unroll
      for (int a = 0; a < Q; ++a) {
        Idx v = (Idx)opp(a) * F + (Idx)m;
        if (a != 0) {
          const int up = fidx_n[off(opp(a))];
          if (up >= 0) v = (Idx)a * F + (Idx)up;
        }
        slot_tab[a][threadIdx.x] = v;
      }
    }
    auto src = [&](int a) -> Idx {
      if (!ODD) return (Idx)opp(a) * F + (Idx)mm;
      return slot_tab[a][threadIdx.x];
    };
    auto dst = [&](int a) -> Idx {
      if (!ODD) return (Idx)a * F + (Idx)mm;
      return slot_tab[opp(a)][threadIdx.x];
    };
    auto launder = [&]() {
      xm = opaque(xm); xp = opaque(xp); ym = opaque(ym); yp = opaque(yp);
      if (D == 3) { zm = opaque(zm); zp = opaque(zp); }
      mm = opaque(mm);
    };
    // dJ/du at this node from the solute phase (and the objective)
    T mux = T(0), muy = T(0), muz = T(0);
    if (WITH_SOLUTE) {
      // sum lam'(g - W C_eff q) = sum lam' g - C_eff sum lam' W q
      const T* Ss = A.S + (size_t)Q * A.P;
      T* Ls = A.L + (size_t)Q * A.P;
      const SubsConst<T>& cs = A.sc[1];
      T u[3];
      u[0] = A.uhist[m];
      u[1] = A.uhist[(Idx)A.P + m];
      u[2] = (D == 3) ? A.uhist[2 * (Idx)A.P + m] : T(0);
      T lam[Q];
#pragma unroll
      for (int a = 0; a < Q; ++a) lam[a] = Ls[dst(a)];
      launder();
      T C = T(0);
      double sLG = 0.0;
#pragma unroll
      for (int a = 0; a < Q; ++a) {
        const T ga = Ss[src(a)];
        C = (a == 0) ? ga : C + ga;
        sLG += (double)lam[a] * (double)ga;
      }
      T Ce = C;
      if (!ODD) Ce *= A.sink1;
      Ce *= A.sink1;
      const T s1k = ODD ? A.sink1 : A.sink1 * A.sink1;
      const T w = cs.itau;
      T Bs = T(0), M0 = T(0), M1 = T(0), M2 = T(0);
#pragma unroll
      for (int a = 0; a < Q; ++a) {
        const T W = wgt<T, Q>(a);
        const T cu = T(cx(a)) * u[0] + T(cy(a)) * u[1] + (D == 3 ? T(cz(a)) * u[2] : T(0));
        const T wl = W * lam[a];
        Bs += wl * (T(1) + T(3) * cu);
        M0 += wl * T(cx(a));
        M1 += wl * T(cy(a));
        if (D == 3) M2 += wl * T(cz(a));
      }
      const double dt = sLG - (double)Ce * (double)Bs;
      T B = w * Bs;
      if (m >= A.obj_lo && m < A.obj_hi) B += A.wc;
      const T omw = cs.omc;
      const T sB = s1k * B;
      launder();
#pragma unroll
      for (int b = 0; b < Q; ++b) lam[b] = omw * lam[b] + sB;
      if (A.face_on && (m < A.face_lo_end || m >= A.face_hi_start)) {
        const bool top = m >= A.face_hi_start;
        const int kind = top ? A.face_kind[1] : A.face_kind[0];
        if (kind) {
          const int nn = ODD ? n : A.fnode[m];
          const int ij = nn - (top ? (A.LZ - 1) * A.LX * A.LY : 0);
          if (top) adj_face_local<T, Q, true>(lam, kind, A.face_dprof[1], ij);
          else adj_face_local<T, Q, false>(lam, kind, A.face_dprof[0], ij);
        }
      }
#pragma unroll
      for (int b = 0; b < Q; ++b) Ls[src(b)] = lam[b];
      const T k3 = T(3) * w * Ce;
      mux = k3 * M0;
      muy = k3 * M1;
      muz = (D == 3) ? k3 * M2 : T(0);
      const double taus = A.tau[1];
      // dC_eff/dtau_s through s1 = 1 - sink tau_s
      const double dce = -A.sink * (double)C * (ODD ? 1.0 : 2.0 * (double)A.sink1);
      acc[4] = dt / (taus * taus) + (double)B * dce;
      launder();
      asm volatile("" ::: "memory");
    }
    {
      // sum lam'(d - deq) = sum lam' d - rho S0 - rho_A sum lam' W P(u)
      const T* Sf = A.S;
      T* Lf = A.L;
      const SubsConst<T>& cf = A.sc[0];
      T lam[Q];
#pragma unroll
      for (int a = 0; a < Q; ++a) lam[a] = Lf[dst(a)];
      launder();
      T rho = T(0), m0 = T(0), m1 = T(0), m2 = T(0);
      double sLD = 0.0;
#pragma unroll
      for (int a = 0; a < Q; ++a) {
        const T da = Sf[src(a)];
        rho = (a == 0) ? da : rho + da;
        if (cx(a) > 0) m0 += da; else if (cx(a) < 0) m0 -= da;
        if (cy(a) > 0) m1 += da; else if (cy(a) < 0) m1 -= da;
        if (D == 3) { if (cz(a) > 0) m2 += da; else if (cz(a) < 0) m2 -= da; }
        sLD += (double)lam[a] * (double)da;
      }
      T u[3];
      u[0] = add_(m0 / cf.rhoA, cf.tg[0]);
      u[1] = add_(m1 / cf.rhoA, cf.tg[1]);
      u[2] = (D == 3) ? add_(m2 / cf.rhoA, cf.tg[2]) : T(0);
      const T w = cf.itau;
      const T rA = cf.rhoA;
      if (m >= A.obj_lo && m < A.obj_hi) mux += A.wu;
      const T usq = u[0] * u[0] + u[1] * u[1] + (D == 3 ? u[2] * u[2] : T(0));
      T S0 = T(0), V0 = T(0), V1 = T(0), V2 = T(0), SP = T(0);
#pragma unroll
      for (int a = 0; a < Q; ++a) {
        const T W = wgt<T, Q>(a);
        const T cu = T(cx(a)) * u[0] + T(cy(a)) * u[1] + (D == 3 ? T(cz(a)) * u[2] : T(0));
        const T wl = W * lam[a];
        S0 += wl;
        const T k3 = T(3) + T(9) * cu;
        V0 += wl * (k3 * T(cx(a)) - T(3) * u[0]);
        V1 += wl * (k3 * T(cy(a)) - T(3) * u[1]);
        if (D == 3) V2 += wl * (k3 * T(cz(a)) - T(3) * u[2]);
        SP += wl * (T(3) * cu + T(4.5) * cu * cu - T(1.5) * usq);
      }
      const double dt = sLD - (double)rho * (double)S0 - (double)rA * (double)SP;
      mux += w * rA * V0;
      muy += w * rA * V1;
      if (D == 3) muz += w * rA * V2;
      const T omw = cf.omc;
      const T iA = T(1) / rA;
      const T wS0 = w * S0;
      launder();
#pragma unroll
      for (int b = 0; b < Q; ++b) {
        const T cm = T(cx(b)) * mux + T(cy(b)) * muy + (D == 3 ? T(cz(b)) * muz : T(0));
        Lf[src(b)] = omw * lam[b] + wS0 + cm * iA;
      }
      const double tau = A.tau[0];
      acc[0] = tau * (double)mux;
      acc[1] = tau * (double)muy;
      acc[2] = tau * (double)muz;
      acc[3] = dt / (tau * tau) + (double)mux * A.g[0] + (double)muy * A.g[1] +
               (double)muz * A.g[2];
    }
  }
  block_add<5>(acc, A.acc + (size_t)blockIdx.x * 5);
}

// Adjoint of the solute's face operations of one step (the effective one
// on each face, one per blockIdx.z), compact layout, one thread per (i, j).
// The forward overwrote the five unknown slots with W_u X: their adjoints
// feed X and are cleared first, then X's adjoint goes to the slots X was
// computed from (and, for a constant concentration, to the face's
// concentration profile).
struct AdjFaceOps {
  int n;
  int top[2], kind[2];
  double* dprof[2];
};

// Node (i, j) of the top (TOP, a compile-time constant so that the
// per-direction arrays are indexed by constants and stay in registers) or
// bottom plane, compact slot `self`.
template <typename T, bool TOP>
__device__ __forceinline__ void adj_face_node(T* Ls, const int* fidx, int LX, int LY, int LZ,
                                              long long stride, int second, int kind,
                                              double* dprof, int i, int j, int self)
{
  const int k = TOP ? LZ - 1 : 0;
  const int plane = LX * LY;
  // Every slot address first, then every value, then every store: written
  // as read-modify-writes in order, each access waited for the one before
  // it (the compiler cannot tell the slots apart), a chain of ~19 memory
  // round trips per thread.  Slots of distinct directions are distinct,
  // except that a known slot can be the very slot an unknown was deposited
  // in (solids on both sides: the own-slot fallback of the load and of the
  // deposit); there the known's old value is the cleared unknown's, 0.
  constexpr bool tp = TOP;
  int up[19];
#pragma unroll
  for (int a = 1; a < 19; ++a) {
    if (second) { up[a] = -1; continue; }
    int ii = i - cx(a), jj = j - cy(a), kk = k - cz(a);
    ii = ii < 0 ? LX - 1 : (ii == LX ? 0 : ii);
    jj = jj < 0 ? LY - 1 : (jj == LY ? 0 : jj);
    kk = kk < 0 ? LZ - 1 : (kk == LZ ? 0 : kk);
    up[a] = fidx[ii + LX * jj + plane * kk];
  }
  up[0] = self;
  auto rslot = [&](int a) -> long long {   // where the forward loaded d_a
    if (second) return (long long)opp(a) * stride + self;
    return up[a] < 0 ? (long long)opp(a) * stride + self : (long long)a * stride + up[a];
  };
  auto wslot = [&](int a) -> long long {   // where it stored unknown a
    if (second) return (long long)opp(a) * stride + self;
    return (long long)a * stride + (up[a] < 0 ? self : up[a]);
  };
  T wsum = wgt<T, 19>(face3_unknown(tp, 0));
#pragma unroll
  for (int q = 1; q < 5; ++q) wsum = wsum + wgt<T, 19>(face3_unknown(tp, q));
  long long ws[5];
  T lu[5];
#pragma unroll
  for (int q = 0; q < 5; ++q) ws[q] = wslot(face3_unknown(tp, q));
#pragma unroll
  for (int q = 0; q < 5; ++q) lu[q] = Ls[ws[q]];
  // the knowns the adjoint of X goes to: the five opposite the unknowns
  // (zero gradient: in D3Q19 exactly the directions of the other c_z) or
  // every direction but the unknowns (the rest)
  const bool zg = kind == FACE_ZEROGRAD;
  long long rs[19];
  T lk[19];
#pragma unroll
  for (int a = 0; a < 19; ++a) {
    const bool known = zg ? cz(a) == (tp ? 1 : -1) : cz(a) != (tp ? -1 : 1);
    rs[a] = known ? rslot(a) : -1;
  }
#pragma unroll
  for (int a = 0; a < 19; ++a) lk[a] = rs[a] >= 0 ? Ls[rs[a]] : T(0);
  T Ax = T(0);
#pragma unroll
  for (int q = 0; q < 5; ++q) Ax += wgt<T, 19>(face3_unknown(tp, q)) * lu[q];
  const T ax = Ax / wsum;
#pragma unroll
  for (int q = 0; q < 5; ++q) Ls[ws[q]] = T(0);
#pragma unroll
  for (int a = 0; a < 19; ++a) {
    if (rs[a] < 0) continue;
    T old = lk[a];
#pragma unroll
    for (int q = 0; q < 5; ++q) old = rs[a] == ws[q] ? T(0) : old;
    Ls[rs[a]] = zg ? old + ax : old - ax;
  }
  if (!zg && dprof) dprof[i + LX * j] += (double)ax;
}

template <typename T>
__global__ void adj_face_plane(T* Ls, const int* fidx, int LX, int LY, int LZ,
                               long long stride, int second, AdjFaceOps ops)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= LX) return;
  const int j = blockIdx.y;
  // the group's entries by select: indexing the parameter arrays by
  // blockIdx.z would copy them to local memory
  const bool g1 = blockIdx.z != 0;
  const int top = g1 ? ops.top[1] : ops.top[0];
  const int kind = g1 ? ops.kind[1] : ops.kind[0];
  double* const dprof = g1 ? ops.dprof[1] : ops.dprof[0];
  const int n = i + LX * j + LX * LY * (top ? LZ - 1 : 0);
  const int self = fidx[n];
  if (self < 0) return;
  if (top) adj_face_node<T, true>(Ls, fidx, LX, LY, LZ, stride, second, kind, dprof, i, j, self);
  else adj_face_node<T, false>(Ls, fidx, LX, LY, LZ, stride, second, kind, dprof, i, j, self);
}

struct AdjState {
  int t0 = 0, nsteps = 0, K = 0;
  lbx_objective obj{};
  std::vector<void*> ckpt;
  double J = 0.0;
  size_t state_bytes = 0;
  // backward workspace, allocated with the checkpoints and kept for later
  // runs of the same shape
  std::vector<void*> snap;     // K+1 recomputed states
  void* L = nullptr;           // adjoint state
  void* uh = nullptr;          // [K+1][3][P] the flow's u per recomputed step
  double* acc = nullptr;       // [blocks][5] gradient rows
  double* dpb = nullptr;       // [LX*LY] profile gradients
  double* dpt = nullptr;
  size_t nblk = 0;
};

void free_state(AdjState* st)
{
  for (void* c : st->ckpt) cudaFree(c);
  for (void* c : st->snap) cudaFree(c);
  cudaFree(st->L); cudaFree(st->uh);
  cudaFree(st->acc); cudaFree(st->dpb); cudaFree(st->dpt);
  st->ckpt.clear(); st->snap.clear();
  st->L = st->uh = nullptr;
  st->acc = st->dpb = st->dpt = nullptr;
}

// Checkpoints for nseg segments of K steps.
lbx_status alloc_checkpoints(AdjState* st, int nseg)
{
  st->ckpt.assign(nseg, nullptr);
  cudaError_t e = cudaSuccess;
  for (int q = 0; q < nseg && e == cudaSuccess; ++q) e = cudaMalloc(&st->ckpt[q], st->state_bytes);
  if (e != cudaSuccess) {
    free_state(st);
    return afail(LBX_ERR_NOMEM, "adjoint checkpoints: %s", cudaGetErrorString(e));
  }
  return LBX_OK;
}

// The backward sweep's workspace, allocated by its first call and kept.
lbx_status alloc_workspace(const lbx_domain* d, AdjState* st)
{
  if (st->L) return LBX_OK;
  const lbx_params& p = d->p;
  const size_t plane2 = (size_t)p.LX * p.LY;
  const size_t ustep = (size_t)3 * d->P * d->real_size;
  st->nblk = std::max<size_t>(1, (size_t)((d->fluid + 255) / 256));
  st->snap.assign(st->K + 1, nullptr);
  cudaError_t e = cudaSuccess;
  for (int q = 0; q <= st->K && e == cudaSuccess; ++q) e = cudaMalloc(&st->snap[q], st->state_bytes);
  if (e == cudaSuccess) e = cudaMalloc(&st->L, st->state_bytes);
  if (e == cudaSuccess && p.nsubs == 2) e = cudaMalloc(&st->uh, (size_t)(st->K + 1) * ustep);
  if (e == cudaSuccess) e = cudaMalloc(&st->acc, st->nblk * 5 * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&st->dpb, plane2 * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&st->dpt, plane2 * sizeof(double));
  if (e != cudaSuccess) {
    for (void* c : st->snap) cudaFree(c);
    cudaFree(st->L); cudaFree(st->uh);
    cudaFree(st->acc); cudaFree(st->dpb); cudaFree(st->dpt);
    st->snap.clear();
    st->L = st->uh = nullptr;
    st->acc = st->dpb = st->dpt = nullptr;
    return afail(LBX_ERR_NOMEM, "adjoint workspace: %s", cudaGetErrorString(e));
  }
  return LBX_OK;
}

bool solute_on(const lbx_params& p, int t) { return t >= p.sigma_t_on && t <= p.sigma_t_off; }

lbx_status check_adjoint(const lbx_domain* d)
{
  const lbx_params& p = d->p;
  if (p.walsh) return afail(LBX_ERR_INVALID, "the adjoint has no Walsh partial bounce-back");
  if (d->layout != LBX_LAYOUT_COMPACT)
    return afail(LBX_ERR_INVALID, "the adjoint runs on the compact layout");
  if (!p.accurate || p.compressible)
    return afail(LBX_ERR_INVALID, "the adjoint covers the shifted incompressible model");
  if (d->faces_active) return afail(LBX_ERR_INVALID, "the adjoint has no 2D face boundaries");
  if ((p.constcon_t_in && p.zeroconcgrad_t) || (p.constcon_b_in && p.zeroconcgrad_b))
    return afail(LBX_ERR_INVALID, "the adjoint takes one solute operation per face");
  for (int s = 0; s < p.nsubs; ++s)
    if (p.pressure_t_in[s] || p.pressure_b_in[s] || p.pressure_t_out[s] || p.pressure_b_out[s])
      return afail(LBX_ERR_INVALID, "the adjoint has no pressure faces");
    else if (p.velocity_t_in[s] || p.velocity_b_in[s] || p.velocity_t_out[s] ||
             p.velocity_b_out[s])
      return afail(LBX_ERR_INVALID, "the adjoint has no velocity faces");
  return LBX_OK;
}

template <typename T>
AdjArgs<T> make_adj(const lbx_domain* d, const void* S, void* L, double* acc)
{
  const lbx_params& p = d->p;
  AdjArgs<T> A;
  std::memset(&A, 0, sizeof A);
  A.S = (const T*)S; A.L = (T*)L;
  A.fidx = d->fidx; A.fnode = d->fnode;
  A.F = (int)d->fluid; A.P = (int)d->P;
  A.LX = p.LX; A.LY = p.LY; A.LZ = p.LZ;
  A.div_plane = make_fastdiv((unsigned)(p.LX * p.LY));
  A.div_lx = make_fastdiv((unsigned)p.LX);
  for (int s = 0; s < 2; ++s) {
    const T tau = (T)p.tau[s];
    const T itau = (T)(1. / tau);
    A.sc[s].itau = itau;
    A.sc[s].omc = (T)(1. - itau);
    A.sc[s].rhoA = (T)p.rho_A[s];
    for (int c = 0; c < 3; ++c) A.sc[s].tg[c] = tau * (T)p.gaccel[s * 3 + c];
    A.tau[s] = (double)(T)p.tau[s];
  }
  for (int c = 0; c < 3; ++c) A.g[c] = (double)(T)p.gaccel[c];
  A.sink1 = (T)(1.0 - (T)p.sink * (T)p.tau[1]);
  A.sink = (double)(T)p.sink;
  A.acc = acc;
  return A;
}

template <typename T, int Q>
void launch_adj(lbx_domain* d, bool odd, bool solute, const AdjArgs<T>& A)
{
  const unsigned blocks = (unsigned)((d->fluid + 255) / 256);
  if (blocks == 0) return;
  const bool idx32 = (unsigned long long)Q * (unsigned long long)d->P < (1ull << 32);
  auto go = [&](auto o, auto s, auto i) {
    adj_step<T, Q, decltype(o)::value, decltype(s)::value, decltype(i)::value>
        <<<blocks, 256, 0, d->stream>>>(A);
  };
  using TT = std::true_type;
  using FF = std::false_type;
  if (idx32) {
    if (solute) { if (odd) go(TT{}, TT{}, TT{}); else go(FF{}, TT{}, TT{}); }
    else { if (odd) go(TT{}, FF{}, TT{}); else go(FF{}, FF{}, TT{}); }
  } else {
    if (solute) { if (odd) go(TT{}, TT{}, FF{}); else go(FF{}, TT{}, FF{}); }
    else { if (odd) go(TT{}, FF{}, FF{}); else go(FF{}, FF{}, FF{}); }
  }
  d->launches++;
}

// Adjoint of the solute face operations of a step: at most one per face
// (check_adjoint rejects a face with both).
template <typename T>
void launch_adj_faces(lbx_domain* d, int t, T* L, double* dprof_t, double* dprof_b)
{
  const lbx_params& p = d->p;
  if (p.nsubs != 2 || d->p.dims != 3) return;
  AdjFaceOps ops;
  std::memset(&ops, 0, sizeof ops);
  auto add = [&](int top, bool cc, bool zg) {
    if (!cc && !zg) return;
    ops.top[ops.n] = top;
    ops.kind[ops.n] = zg ? FACE_ZEROGRAD : FACE_CONSTCON;
    ops.dprof[ops.n] = zg ? nullptr : (top ? dprof_t : dprof_b);
    ++ops.n;
  };
  add(1, p.constcon_t_in != 0, p.zeroconcgrad_t != 0);
  add(0, p.constcon_b_in != 0, p.zeroconcgrad_b != 0);
  if (ops.n == 0) return;
  const bool second = (t % 2) == 0;
  T* Ls = L + (size_t)d->Q * d->P;
  dim3 block(128), grid((p.LX + 127) / 128, p.LY, ops.n);
  adj_face_plane<T><<<grid, block, 0, d->stream>>>(Ls, d->fidx, p.LX, p.LY, p.LZ, d->P,
                                                   second ? 1 : 0, ops);
  d->launches++;
}

template <typename T>
lbx_status backward_t(lbx_domain* d, lbx_gradient* out, double* dprof_b, double* dprof_t)
{
  AdjState* st = (AdjState*)d->adj;
  const lbx_params& p = d->p;
  if (lbx_status rc0 = alloc_workspace(d, st)) return rc0;
  const size_t sb = st->state_bytes;
  const int K = st->K;
  const size_t plane2 = (size_t)p.LX * p.LY;
  const size_t ustep = (size_t)3 * d->P;
  const size_t nblk = st->nblk;
  std::vector<void*>& snap = st->snap;
  void* L = st->L;
  T* uh = (T*)st->uh;
  double* acc = st->acc;
  lbx_status rc = LBX_OK;
  ACK(cudaMemsetAsync(L, 0, sb, d->stream));
  ACK(cudaMemsetAsync(acc, 0, nblk * 5 * sizeof(double), d->stream));
  ACK(cudaMemsetAsync(st->dpb, 0, plane2 * sizeof(double), d->stream));
  ACK(cudaMemsetAsync(st->dpt, 0, plane2 * sizeof(double), d->stream));

  // objective plane and seeds
  const lbx_objective& ob = st->obj;
  long long lo = 0;
  for (int q = 0; q < ob.plane; ++q) lo += d->plane_fluid[q];
  const long long hi = lo + d->plane_fluid[ob.plane];
  const int t_first = std::max(ob.t_first, st->t0 + 1);
  const int t_last = std::min(ob.t_last, st->t0 + st->nsteps);
  const double nwin = (double)std::max(0, t_last - t_first + 1);
  const double nout = (double)std::max<long long>(1, hi - lo);

  // the solute's adjoint stays exactly zero until the first C seed (going
  // back in time); until then its kernels are skipped
  bool solute_live = false;
  const int nseg = (int)st->ckpt.size();
  for (int seg = nseg - 1; seg >= 0; --seg) {
    const int tc = st->t0 + seg * K;
    const int len = std::min(K, st->t0 + st->nsteps - tc);
    ACK(cudaMemcpyAsync(snap[0], st->ckpt[seg], sb, cudaMemcpyDeviceToDevice, d->stream));
    void* ubuf = d->ubuf;
    for (int q = 1; q <= len; ++q) {
      if (uh) d->ubuf = uh + (size_t)q * ustep;
      rc = lbx_internal_step_into(d, tc + q, snap[q - 1], snap[q]);
      if (rc) { d->ubuf = ubuf; return rc; }
    }
    d->ubuf = ubuf;
    for (int q = len; q >= 1; --q) {
      const int t = tc + q;
      const bool odd = (t % 2) != 0;
      AdjArgs<T> A = make_adj<T>(d, snap[q - 1], L, acc);
      A.uhist = uh ? uh + (size_t)q * ustep : nullptr;
      A.obj_lo = (int)lo; A.obj_hi = (int)hi;
      const bool in_win = nwin > 0 && t >= t_first && t <= t_last;
      A.wc = in_win ? (T)(ob.w_c / (nwin * nout)) : T(0);
      A.wu = in_win ? (T)(ob.w_ux / (nwin * nout)) : T(0);
      solute_live = solute_live || (p.nsubs == 2 && A.wc != T(0));
      const bool sol = p.nsubs == 2 && solute_on(p, t) && solute_live;
      // the adjoint of the solute's face operations inside the step kernel
      // where the z faces fuse (adj_face_local), else its own launch
      const bool face_fused = sol && d->Q == 19 && d->faces3_active &&
                              (!odd || d->faces3_fuse_odd);
      if (face_fused) {
        A.face_on = 1;
        A.face_lo_end = (int)d->plane_fluid[0];
        A.face_hi_start = (int)(d->fluid - d->plane_fluid[p.LZ - 1]);
        A.face_kind[0] = p.zeroconcgrad_b ? FACE_ZEROGRAD : (p.constcon_b_in ? FACE_CONSTCON : 0);
        A.face_kind[1] = p.zeroconcgrad_t ? FACE_ZEROGRAD : (p.constcon_t_in ? FACE_CONSTCON : 0);
        A.face_dprof[0] = A.face_kind[0] == FACE_CONSTCON ? st->dpb : nullptr;
        A.face_dprof[1] = A.face_kind[1] == FACE_CONSTCON ? st->dpt : nullptr;
      }
      if (d->Q == 19) launch_adj<T, 19>(d, odd, sol, A);
      else launch_adj<T, 9>(d, odd, sol, A);
      if (solute_live && !face_fused) launch_adj_faces<T>(d, t, (T*)L, st->dpt, st->dpb);
      ACK(cudaGetLastError());
    }
  }
  std::vector<double> rows(nblk * 5);
  ACK(cudaMemcpyAsync(rows.data(), acc, rows.size() * sizeof(double), cudaMemcpyDeviceToHost,
                      d->stream));
  if (dprof_b) ACK(cudaMemcpyAsync(dprof_b, st->dpb, plane2 * sizeof(double), cudaMemcpyDeviceToHost, d->stream));
  if (dprof_t) ACK(cudaMemcpyAsync(dprof_t, st->dpt, plane2 * sizeof(double), cudaMemcpyDeviceToHost, d->stream));
  ACK(cudaStreamSynchronize(d->stream));
  double h[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (size_t b = 0; b < nblk; ++b)
    for (int q = 0; q < 5; ++q) h[q] += rows[b * 5 + q];
  out->J = st->J;
  for (int c = 0; c < 3; ++c) out->d_gaccel[c] = h[c];
  out->d_tau = h[3];
  out->d_tau_s = h[4];
  return LBX_OK;
}

}  // namespace

void lbx_internal_adjoint_free(lbx_domain* d)
{
  AdjState* st = (AdjState*)d->adj;
  if (!st) return;
  cudaStreamSynchronize(d->stream);
  free_state(st);
  delete st;
  d->adj = nullptr;
}

extern "C" {

lbx_status lbx_adjoint_forward(lbx_domain* d, int t0, int nsteps, int checkpoint_every,
                               const lbx_objective* obj, double* J)
{
  if (!d || !obj) return afail(LBX_ERR_INVALID, "NULL argument");
  lbx_status rc = check_adjoint(d);
  if (rc) return rc;
  if (nsteps < 1 || checkpoint_every < 1)
    return afail(LBX_ERR_INVALID, "nsteps and checkpoint_every must be positive");
  if (t0 < 0 || t0 % 2 != 0 || d->parity != 0)
    return afail(LBX_ERR_STATE, "the adjoint run starts from the natural-order state at an even time");
  const int planes = d->p.dims == 2 ? d->p.LY : d->p.LZ;
  if (obj->plane < 0 || obj->plane >= planes) return afail(LBX_ERR_INVALID, "objective plane out of range");
  const size_t sbytes = (size_t)d->p.nsubs * d->Q * d->P * d->real_size;
  const int nseg = (nsteps + checkpoint_every - 1) / checkpoint_every;
  AdjState* st = (AdjState*)d->adj;
  if (st && (st->K != checkpoint_every || (int)st->ckpt.size() != nseg ||
             st->state_bytes != sbytes)) {
    lbx_internal_adjoint_free(d);
    st = nullptr;
  }
  if (!st) {
    st = new AdjState();
    st->K = checkpoint_every;
    st->state_bytes = sbytes;
    rc = alloc_checkpoints(st, nseg);
    if (rc) { delete st; return rc; }
    d->adj = st;
  }
  st->t0 = t0; st->nsteps = nsteps; st->obj = *obj;
  // plane means are recorded over the objective's steps only
  const int t_first = std::max(obj->t_first, t0 + 1);
  const int t_last = std::min(obj->t_last, t0 + nsteps);
  const int nwin = std::max(0, t_last - t_first + 1);
  bool recording = false;
  for (int q = 0; q < nseg; ++q) {
    const int tc = t0 + q * checkpoint_every;
    const int te = std::min(tc + checkpoint_every, t0 + nsteps);
    ACK(cudaMemcpyAsync(st->ckpt[q], d->fc, st->state_bytes, cudaMemcpyDeviceToDevice, d->stream));
    int t = tc;
    while (t < te) {
      if (!recording && nwin > 0 && t == t_first - 1) {
        rc = lbx_btc_start(d, obj->plane, nwin);
        if (rc) { lbx_internal_adjoint_free(d); return rc; }
        recording = true;
        continue;
      }
      int stop = te;
      if (!recording && nwin > 0 && t < t_first - 1 && t_first - 1 < te) stop = t_first - 1;
      rc = lbx_run(d, t, stop - t, 0);
      if (rc) { lbx_internal_adjoint_free(d); return rc; }
      t = stop;
    }
  }
  st->J = 0.0;
  if (recording) {
    std::vector<double> c(nwin), ux(nwin);
    long long cnt = 0;
    rc = lbx_btc_read(d, c.data(), ux.data(), nwin, &cnt);
    lbx_btc_stop(d);
    if (rc) { lbx_internal_adjoint_free(d); return rc; }
    double sc = 0.0, su = 0.0;
    for (int q = 0; q < nwin; ++q) {
      if (obj->w_c != 0.0) sc += c[q];
      su += ux[q];
    }
    st->J = obj->w_c * (sc / nwin) + obj->w_ux * (su / nwin);
  }
  if (J) *J = st->J;
  return LBX_OK;
}

lbx_status lbx_adjoint_backward(lbx_domain* d, lbx_gradient* out, double* d_profile_b,
                                double* d_profile_t)
{
  if (!d || !out) return afail(LBX_ERR_INVALID, "NULL argument");
  if (!d->adj) return afail(LBX_ERR_STATE, "lbx_adjoint_forward has not run");
  std::memset(out, 0, sizeof *out);
  return d->real_size == 8 ? backward_t<double>(d, out, d_profile_b, d_profile_t)
                           : backward_t<float>(d, out, d_profile_b, d_profile_t);
}

}  // extern "C"
