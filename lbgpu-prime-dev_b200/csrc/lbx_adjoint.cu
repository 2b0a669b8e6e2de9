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
  T* mu;                   // [3][P]: dJ/du from the solute, for the flow
  const int* fidx;
  const int* fnode;
  int F, P, LX, LY, LZ;
  FastDiv div_plane, div_lx;
  SubsConst<T> sc[2];
  T sink1;
  double tau[2], g[3], sink;
  int obj_lo, obj_hi;      // compact range of the objective plane's nodes
  T wc, wu;                // this step's seeds: dJ/dC_eff, dJ/du_x per plane node
  int mu_in;               // flow: add the solute's mu
  double* acc;             // [5]: dJ/dg_x, dJ/dg_y, dJ/dg_z, dJ/dtau, dJ/dtau_s
};

// Sum of v over the block, added to *out by one thread.
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
      if (x != 0.0) atomicAdd(out + q, x);
    }
  }
}

// Adjoint of one AA kernel launch for one substance (SOLUTE) on the compact
// layout.  256 threads per block, every thread reaches the block reduction.
template <typename T, int Q, bool ODD, bool SOLUTE>
__global__ void __launch_bounds__(256)
adj_step(AdjArgs<T> A)
{
  constexpr int D = (Q == 9) ? 2 : 3;
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = m < A.F;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  if (live) {
    const size_t F = (size_t)A.P;
    // neighbour slots exactly as the forward step forms them
    int nb[Q];
    nb[0] = m;
    if (ODD) {
      const int plane = A.LX * A.LY;
      const int n = A.fnode[m];
      const int k = fast_div(n, A.div_plane);
      const int r = n - k * plane;
      const int j = fast_div(r, A.div_lx);
      const int i = r - j * A.LX;
      const int xm = (i == 0) ? A.LX - 1 : -1, xp = (i == A.LX - 1) ? 1 - A.LX : 1;
      const int ym = (j == 0) ? plane - A.LX : -A.LX, yp = (j == A.LY - 1) ? A.LX - plane : A.LX;
      int zm = 0, zp = 0;
      if (D == 3) {
        const int tot = plane * A.LZ;
        zm = (k == 0) ? tot - plane : -plane;
        zp = (k == A.LZ - 1) ? plane - tot : plane;
      }
#pragma unroll
      for (int a = 1; a < Q; ++a) {
        const int o = (cx(a) < 0 ? xm : (cx(a) > 0 ? xp : 0)) +
                      (cy(a) < 0 ? ym : (cy(a) > 0 ? yp : 0)) +
                      (cz(a) < 0 ? zm : (cz(a) > 0 ? zp : 0));
        nb[a] = A.fidx[n + o];     // compact index of n + c_a, -1 if solid
      }
    }
    // slot the forward read d_a from / wrote d'_a to
    auto src = [&](int a) -> size_t {
      if (!ODD) return (size_t)opp(a) * F + m;
      const int up = nb[opp(a)];
      return up >= 0 ? (size_t)a * F + (size_t)up : (size_t)opp(a) * F + m;
    };
    auto dst = [&](int a) -> size_t {
      if (!ODD) return (size_t)a * F + m;
      const int dn = nb[a];
      return dn >= 0 ? (size_t)opp(a) * F + (size_t)dn : (size_t)a * F + m;
    };
    // the flow's velocity at this node (the forward collide's u)
    const T* Sf = A.S;
    const SubsConst<T>& cf = A.sc[0];
    T u[3] = {T(0), T(0), T(0)};
    {
      T d[Q];
#pragma unroll
      for (int a = 0; a < Q; ++a) d[a] = Sf[src(a)];
      T m0 = T(0), m1 = T(0), m2 = T(0);
#pragma unroll
      for (int a = 0; a < Q; ++a) {
        if (cx(a) > 0) m0 += d[a]; else if (cx(a) < 0) m0 -= d[a];
        if (cy(a) > 0) m1 += d[a]; else if (cy(a) < 0) m1 -= d[a];
        if (D == 3) { if (cz(a) > 0) m2 += d[a]; else if (cz(a) < 0) m2 -= d[a]; }
      }
      u[0] = add_(m0 / cf.rhoA, cf.tg[0]);
      u[1] = add_(m1 / cf.rhoA, cf.tg[1]);
      u[2] = (D == 3) ? add_(m2 / cf.rhoA, cf.tg[2]) : T(0);
      if (!SOLUTE) {
        // flow adjoint
        T rho = d[0];
#pragma unroll
        for (int a = 1; a < Q; ++a) rho += d[a];
        const T w = cf.itau;
        const T rA = cf.rhoA;
        T lam[Q];
#pragma unroll
        for (int a = 0; a < Q; ++a) lam[a] = A.L[dst(a)];
        T mux = T(0), muy = T(0), muz = T(0);
        if (A.mu_in) {
          mux = A.mu[m];
          muy = A.mu[F + m];
          if (D == 3) muz = A.mu[2 * F + m];
        }
        if (m >= A.obj_lo && m < A.obj_hi) mux += A.wu;
        const T usq = u[0] * u[0] + u[1] * u[1] + (D == 3 ? u[2] * u[2] : T(0));
        T S0 = T(0), V0 = T(0), V1 = T(0), V2 = T(0);
        double dt = 0.0;
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
          const T deq = W * rho + W * rA * (T(3) * cu + T(4.5) * cu * cu - T(1.5) * usq);
          dt += (double)lam[a] * ((double)d[a] - (double)deq);
        }
        mux += w * rA * V0;
        muy += w * rA * V1;
        if (D == 3) muz += w * rA * V2;
        const T omw = cf.omc;
        const T iA = T(1) / rA;
#pragma unroll
        for (int b = 0; b < Q; ++b) {
          const T cm = T(cx(b)) * mux + T(cy(b)) * muy + (D == 3 ? T(cz(b)) * muz : T(0));
          A.L[src(b)] = omw * lam[b] + w * S0 + cm * iA;
        }
        const double tau = A.tau[0];
        acc[0] = tau * (double)mux;
        acc[1] = tau * (double)muy;
        acc[2] = tau * (double)muz;
        acc[3] = dt / (tau * tau) + (double)mux * A.g[0] + (double)muy * A.g[1] +
                 (double)muz * A.g[2];
      }
    }
    if (SOLUTE) {
      const T* Ss = A.S + (size_t)Q * F;
      T* Ls = A.L + (size_t)Q * F;
      const SubsConst<T>& cs = A.sc[1];
      T g[Q];
#pragma unroll
      for (int a = 0; a < Q; ++a) g[a] = Ss[src(a)];
      T C = g[0];
#pragma unroll
      for (int a = 1; a < Q; ++a) C += g[a];
      T Ce = C;
      if (!ODD) Ce *= A.sink1;
      Ce *= A.sink1;
      const T s1k = ODD ? A.sink1 : A.sink1 * A.sink1;
      const T w = cs.itau;
      T lam[Q];
#pragma unroll
      for (int a = 0; a < Q; ++a) lam[a] = Ls[dst(a)];
      T Bs = T(0), M0 = T(0), M1 = T(0), M2 = T(0);
      double dt = 0.0;
#pragma unroll
      for (int a = 0; a < Q; ++a) {
        const T W = wgt<T, Q>(a);
        const T cu = T(cx(a)) * u[0] + T(cy(a)) * u[1] + (D == 3 ? T(cz(a)) * u[2] : T(0));
        const T wl = W * lam[a];
        Bs += wl * (T(1) + T(3) * cu);
        M0 += wl * T(cx(a));
        M1 += wl * T(cy(a));
        if (D == 3) M2 += wl * T(cz(a));
        dt += (double)lam[a] * ((double)g[a] - (double)(W * Ce * (T(1) + T(3) * cu)));
      }
      T B = w * Bs;
      if (m >= A.obj_lo && m < A.obj_hi) B += A.wc;
      const T omw = cs.omc;
#pragma unroll
      for (int b = 0; b < Q; ++b) Ls[src(b)] = omw * lam[b] + s1k * B;
      const T k3 = T(3) * w * Ce;
      A.mu[m] = k3 * M0;
      A.mu[F + m] = k3 * M1;
      if (D == 3) A.mu[2 * F + m] = k3 * M2;
      const double taus = A.tau[1];
      // dC_eff/dtau_s through s1 = 1 - sink tau_s
      const double dce = -A.sink * (double)C * (ODD ? 1.0 : 2.0 * (double)A.sink1);
      acc[3] = dt / (taus * taus) + (double)B * dce;
    }
  }
  if (SOLUTE) {
    double v[1] = {acc[3]};
    block_add<1>(v, A.acc + 4);
  } else {
    block_add<4>(acc, A.acc);
  }
}

// Adjoint of one solute face operation (zero gradient or constant
// concentration) on the compact layout, one thread per (i, j).  The forward
// overwrote the five unknown slots with W_u X: their adjoints feed X and are
// cleared first, then X's adjoint goes to the slots X was computed from (and,
// for a constant concentration, to the face's concentration profile).
template <typename T>
__global__ void adj_face_plane(T* Ls, const int* fidx, int LX, int LY, int LZ,
                               long long stride, int top, int kind, int second,
                               double* dprof)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= LX) return;
  const int j = blockIdx.y;
  const int k = top ? LZ - 1 : 0;
  const int plane = LX * LY;
  const int n = i + LX * j + plane * k;
  const int self = fidx[n];
  if (self < 0) return;
  auto upstream = [&](int a) -> int {
    int ii = i - cx(a), jj = j - cy(a), kk = k - cz(a);
    ii = ii < 0 ? LX - 1 : (ii == LX ? 0 : ii);
    jj = jj < 0 ? LY - 1 : (jj == LY ? 0 : jj);
    kk = kk < 0 ? LZ - 1 : (kk == LZ ? 0 : kk);
    return fidx[ii + LX * jj + plane * kk];
  };
  auto rslot = [&](int a) -> long long {   // where the forward loaded d_a
    if (second) return (long long)opp(a) * stride + self;
    const int up = upstream(a);
    return up < 0 ? (long long)opp(a) * stride + self : (long long)a * stride + up;
  };
  auto wslot = [&](int a) -> long long {   // where it stored unknown a
    if (second) return (long long)opp(a) * stride + self;
    const int up = upstream(a);
    return (long long)a * stride + (up < 0 ? self : up);
  };
  const bool tp = top != 0;
  T wsum = wgt<T, 19>(face3_unknown(tp, 0));
#pragma unroll
  for (int q = 1; q < 5; ++q) wsum = wsum + wgt<T, 19>(face3_unknown(tp, q));
  T Ax = T(0);
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    const int a = face3_unknown(tp, q);
    const long long s = wslot(a);
    Ax += wgt<T, 19>(a) * Ls[s];
    Ls[s] = T(0);
  }
  const T ax = Ax / wsum;
  if (kind == FACE_ZEROGRAD) {
#pragma unroll
    for (int q = 0; q < 5; ++q) Ls[rslot(opp(face3_unknown(tp, q)))] += ax;
  } else {
#pragma unroll
    for (int a = 0; a < 19; ++a)
      if (cz(a) != (tp ? -1 : 1)) Ls[rslot(a)] -= ax;
    if (dprof) dprof[i + LX * j] += (double)ax;
  }
}

struct AdjState {
  int t0 = 0, nsteps = 0, K = 0;
  lbx_objective obj{};
  std::vector<void*> ckpt;
  double J = 0.0;
  size_t state_bytes = 0;
};

bool solute_on(const lbx_params& p, int t) { return t >= p.sigma_t_on && t <= p.sigma_t_off; }

lbx_status check_adjoint(const lbx_domain* d)
{
  const lbx_params& p = d->p;
  if (d->layout != LBX_LAYOUT_COMPACT)
    return afail(LBX_ERR_INVALID, "the adjoint runs on the compact layout");
  if (!p.accurate || p.compressible)
    return afail(LBX_ERR_INVALID, "the adjoint covers the shifted incompressible model");
  if (d->faces_active) return afail(LBX_ERR_INVALID, "the adjoint has no 2D face boundaries");
  for (int s = 0; s < p.nsubs; ++s)
    if (p.pressure_t_in[s] || p.pressure_b_in[s] || p.pressure_t_out[s] || p.pressure_b_out[s])
      return afail(LBX_ERR_INVALID, "the adjoint has no pressure faces");
  return LBX_OK;
}

template <typename T>
AdjArgs<T> make_adj(const lbx_domain* d, const void* S, void* L, void* mu, double* acc)
{
  const lbx_params& p = d->p;
  AdjArgs<T> A;
  std::memset(&A, 0, sizeof A);
  A.S = (const T*)S; A.L = (T*)L; A.mu = (T*)mu;
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
  if (solute) {
    if (odd) adj_step<T, Q, true, true><<<blocks, 256, 0, d->stream>>>(A);
    else adj_step<T, Q, false, true><<<blocks, 256, 0, d->stream>>>(A);
  } else {
    if (odd) adj_step<T, Q, true, false><<<blocks, 256, 0, d->stream>>>(A);
    else adj_step<T, Q, false, false><<<blocks, 256, 0, d->stream>>>(A);
  }
  d->launches++;
}

// Adjoint of the solute face operations of step t, in reverse order.
template <typename T>
void launch_adj_faces(lbx_domain* d, int t, T* L, double* dprof_t, double* dprof_b)
{
  const lbx_params& p = d->p;
  if (p.nsubs != 2 || d->p.dims != 3) return;
  const bool second = (t % 2) == 0;
  T* Ls = L + (size_t)d->Q * d->P;
  dim3 block(128), grid((p.LX + 127) / 128, p.LY);
  auto run = [&](int top, int kind, double* dp) {
    adj_face_plane<T><<<grid, block, 0, d->stream>>>(Ls, d->fidx, p.LX, p.LY, p.LZ, d->P, top,
                                                     kind, second ? 1 : 0, dp);
    d->launches++;
  };
  if (p.zeroconcgrad_b) run(0, FACE_ZEROGRAD, nullptr);
  if (p.zeroconcgrad_t) run(1, FACE_ZEROGRAD, nullptr);
  if (p.constcon_b_in) run(0, FACE_CONSTCON, dprof_b);
  if (p.constcon_t_in) run(1, FACE_CONSTCON, dprof_t);
}

template <typename T>
lbx_status backward_t(lbx_domain* d, lbx_gradient* out, double* dprof_b, double* dprof_t)
{
  AdjState* st = (AdjState*)d->adj;
  const lbx_params& p = d->p;
  const size_t sb = st->state_bytes;
  const int K = st->K;
  std::vector<void*> snap(K + 1, nullptr);
  void *L = nullptr, *mu = nullptr;
  double *acc = nullptr, *dpb = nullptr, *dpt = nullptr;
  const size_t plane2 = (size_t)p.LX * p.LY;
  lbx_status rc = LBX_OK;
  auto cleanup = [&]() {
    for (void* s : snap) cudaFree(s);
    cudaFree(L); cudaFree(mu); cudaFree(acc); cudaFree(dpb); cudaFree(dpt);
  };
#define BCK(call)                                                                 \
  do {                                                                            \
    cudaError_t e_ = (call);                                                      \
    if (e_ != cudaSuccess) {                                                      \
      rc = afail(e_ == cudaErrorMemoryAllocation ? LBX_ERR_NOMEM : LBX_ERR_CUDA,  \
                 "%s: %s", #call, cudaGetErrorString(e_));                        \
      cleanup();                                                                  \
      return rc;                                                                  \
    }                                                                             \
  } while (0)
  for (int q = 0; q <= K; ++q) BCK(cudaMalloc(&snap[q], sb));
  BCK(cudaMalloc(&L, sb));
  BCK(cudaMalloc(&mu, std::max<size_t>(1, (size_t)3 * d->P * sizeof(T))));
  BCK(cudaMalloc(&acc, 5 * sizeof(double)));
  BCK(cudaMalloc(&dpb, plane2 * sizeof(double)));
  BCK(cudaMalloc(&dpt, plane2 * sizeof(double)));
  BCK(cudaMemsetAsync(L, 0, sb, d->stream));
  BCK(cudaMemsetAsync(mu, 0, (size_t)3 * d->P * sizeof(T), d->stream));
  BCK(cudaMemsetAsync(acc, 0, 5 * sizeof(double), d->stream));
  BCK(cudaMemsetAsync(dpb, 0, plane2 * sizeof(double), d->stream));
  BCK(cudaMemsetAsync(dpt, 0, plane2 * sizeof(double), d->stream));

  // objective plane and seeds
  const lbx_objective& ob = st->obj;
  long long lo = 0;
  for (int q = 0; q < ob.plane; ++q) lo += d->plane_fluid[q];
  const long long hi = lo + d->plane_fluid[ob.plane];
  const int t_first = std::max(ob.t_first, st->t0 + 1);
  const int t_last = std::min(ob.t_last, st->t0 + st->nsteps);
  const double nwin = (double)std::max(0, t_last - t_first + 1);
  const double nout = (double)std::max<long long>(1, hi - lo);

  const int nseg = (int)st->ckpt.size();
  for (int seg = nseg - 1; seg >= 0; --seg) {
    const int tc = st->t0 + seg * K;
    const int len = std::min(K, st->t0 + st->nsteps - tc);
    BCK(cudaMemcpyAsync(snap[0], st->ckpt[seg], sb, cudaMemcpyDeviceToDevice, d->stream));
    for (int q = 1; q <= len; ++q) {
      rc = lbx_internal_step_into(d, tc + q, snap[q - 1], snap[q]);
      if (rc) { cleanup(); return rc; }
    }
    for (int q = len; q >= 1; --q) {
      const int t = tc + q;
      const bool odd = (t % 2) != 0;
      AdjArgs<T> A = make_adj<T>(d, snap[q - 1], L, mu, acc);
      A.obj_lo = (int)lo; A.obj_hi = (int)hi;
      const bool in_win = nwin > 0 && t >= t_first && t <= t_last;
      A.wc = in_win ? (T)(ob.w_c / (nwin * nout)) : T(0);
      A.wu = in_win ? (T)(ob.w_ux / (nwin * nout)) : T(0);
      const bool sol = p.nsubs == 2 && solute_on(p, t);
      if (sol) {
        if (d->Q == 19) launch_adj<T, 19>(d, odd, true, A);
        else launch_adj<T, 9>(d, odd, true, A);
      }
      A.mu_in = sol ? 1 : 0;
      if (d->Q == 19) launch_adj<T, 19>(d, odd, false, A);
      else launch_adj<T, 9>(d, odd, false, A);
      launch_adj_faces<T>(d, t, (T*)L, dpt, dpb);
      BCK(cudaGetLastError());
    }
  }
  double h[5];
  BCK(cudaMemcpyAsync(h, acc, sizeof h, cudaMemcpyDeviceToHost, d->stream));
  if (dprof_b) BCK(cudaMemcpyAsync(dprof_b, dpb, plane2 * sizeof(double), cudaMemcpyDeviceToHost, d->stream));
  if (dprof_t) BCK(cudaMemcpyAsync(dprof_t, dpt, plane2 * sizeof(double), cudaMemcpyDeviceToHost, d->stream));
  BCK(cudaStreamSynchronize(d->stream));
#undef BCK
  out->J = st->J;
  for (int c = 0; c < 3; ++c) out->d_gaccel[c] = h[c];
  out->d_tau = h[3];
  out->d_tau_s = h[4];
  cleanup();
  return LBX_OK;
}

}  // namespace

void lbx_internal_adjoint_free(lbx_domain* d)
{
  AdjState* st = (AdjState*)d->adj;
  if (!st) return;
  for (void* c : st->ckpt) cudaFree(c);
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
  lbx_internal_adjoint_free(d);
  AdjState* st = new AdjState();
  d->adj = st;
  st->t0 = t0; st->nsteps = nsteps; st->K = checkpoint_every; st->obj = *obj;
  st->state_bytes = (size_t)d->p.nsubs * d->Q * d->P * d->real_size;
  const int nseg = (nsteps + checkpoint_every - 1) / checkpoint_every;
  st->ckpt.assign(nseg, nullptr);
  for (int q = 0; q < nseg; ++q) {
    cudaError_t e = cudaMalloc(&st->ckpt[q], st->state_bytes);
    if (e != cudaSuccess) {
      lbx_internal_adjoint_free(d);
      return afail(LBX_ERR_NOMEM, "adjoint checkpoints: %s", cudaGetErrorString(e));
    }
  }
  rc = lbx_btc_start(d, obj->plane, nsteps);
  if (rc) { lbx_internal_adjoint_free(d); return rc; }
  for (int q = 0; q < nseg; ++q) {
    const int tc = t0 + q * checkpoint_every;
    const int len = std::min(checkpoint_every, t0 + nsteps - tc);
    ACK(cudaMemcpyAsync(st->ckpt[q], d->fc, st->state_bytes, cudaMemcpyDeviceToDevice, d->stream));
    rc = lbx_run(d, tc, len, 0);
    if (rc) { lbx_internal_adjoint_free(d); return rc; }
  }
  std::vector<double> c(nsteps), ux(nsteps);
  long long cnt = 0;
  rc = lbx_btc_read(d, c.data(), ux.data(), nsteps, &cnt);
  lbx_btc_stop(d);
  if (rc) { lbx_internal_adjoint_free(d); return rc; }
  const int t_first = std::max(obj->t_first, t0 + 1);
  const int t_last = std::min(obj->t_last, t0 + nsteps);
  double sc = 0.0, su = 0.0;
  int nw = 0;
  for (int t = t_first; t <= t_last; ++t, ++nw) {
    if (obj->w_c != 0.0) sc += c[t - t0 - 1];
    su += ux[t - t0 - 1];
  }
  st->J = nw ? (obj->w_c * (sc / nw) + obj->w_ux * (su / nw)) : 0.0;
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
