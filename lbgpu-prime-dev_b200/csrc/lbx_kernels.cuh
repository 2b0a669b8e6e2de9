// lbx_kernels.cuh -- sm_100a device code for the AA-pattern LBM hot path.
//
// One thread per lattice node, x fastest, so every population access of a
// warp is one contiguous run of 32 reals in one direction's plane of the SoA
// array [subs][a][n].  The step is HBM-bound (19 loads + 19 stores of
// populations per fluid node and one byte of node class), so there is no
// shared-memory staging of populations and no tensor-core work: the only
// per-node state is the Q populations, held in registers.
//
// Reference semantics restated here (file:line in the reference tree):
//   odd step   src/k_stream_collide_stream.c:15-423  (pull, collide, push)
//   even step  src/k_collide.c:17-416                (swapped local update)
//   helpers    src/lattice.c:2660-2944               (bounce-back, BGK)
//   faces      src/system_boundary_kernels.c:5-831   (Zou-He, zero gradient)
#pragma once

#include <cstdint>
#include <type_traits>
#include <cuda_runtime.h>

namespace lbx {

// ---- lattice tables --------------------------------------------------------
// Direction order of the reference (src/lbgpu_prime.h:82-84): opposites are
// adjacent (a odd <-> a+1) and D2Q9 is the first nine directions.
__host__ __device__ constexpr int cx(int a) {
  return (a == 1 || a == 5 || a == 8 || a == 11 || a == 14) ? 1
       : (a == 2 || a == 6 || a == 7 || a == 12 || a == 13) ? -1 : 0;
}
__host__ __device__ constexpr int cy(int a) {
  return (a == 3 || a == 5 || a == 7 || a == 15 || a == 18) ? 1
       : (a == 4 || a == 6 || a == 8 || a == 16 || a == 17) ? -1 : 0;
}
__host__ __device__ constexpr int cz(int a) {
  return (a == 9 || a == 11 || a == 13 || a == 15 || a == 17) ? 1
       : (a == 10 || a == 12 || a == 14 || a == 16 || a == 18) ? -1 : 0;
}
__host__ __device__ constexpr int opp(int a) {
  return a == 0 ? 0 : ((a & 1) ? a + 1 : a - 1);
}
// Weights (src/latman.c:161-192), rounded to T as the reference's `real`.
template <typename T, int Q>
__host__ __device__ constexpr T wgt(int a) {
  return Q == 9
    ? (a == 0 ? T(4. / 9.) : (a < 5 ? T(1. / 9.) : T(1. / 36.)))
    : (a == 0 ? T(1. / 3.)
       : (a < 5 ? T(1. / 18.)
          : (a < 9 ? T(1. / 36.) : (a < 11 ? T(1. / 18.) : T(1. / 36.)))));
}

enum Dir2 { DC = 0, DE, DW, DN, DS, DNE, DSW, DNW, DSE };

// FP64 arithmetic without contraction: every product and sum is rounded as
// written (the intrinsics are never fused into FMAs), so the FP64 kernels
// compute the reference's C arithmetic, in its operation order, bit for bit.
// FP32 uses plain operators and lets the compiler form FMAs.
__device__ __forceinline__ double mul_(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add_(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub_(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float mul_(float a, float b) { return a * b; }
__device__ __forceinline__ float add_(float a, float b) { return a + b; }
__device__ __forceinline__ float sub_(float a, float b) { return a - b; }

// A load the compiler may neither merge with an earlier load of the same
// address nor hoist: used to re-read small index arrays (L1 hits) instead of
// holding them in registers across the collision.
__device__ __forceinline__ int ld_reload(const int* p)
{
  int v;
  asm volatile("ld.global.nc.b32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}

// An opaque copy: stops the compiler from proving two address expressions
// equal and keeping the first set of addresses live in registers.
__device__ __forceinline__ int opaque(int x)
{
  int v;
  asm volatile("mov.b32 %0, %1;" : "=r"(v) : "r"(x));
  return v;
}

template <typename P>
__device__ __forceinline__ P* opaque(P* x)
{
  P* v;
  asm volatile("mov.b64 %0, %1;" : "=l"(v) : "l"(x));
  return v;
}

// Division of a node index by a lattice extent without a hardware divide:
// q = umulhi(n, m) >> s with l = ceil(log2 d), m = ceil(2^(31+l) / d),
// s = l - 1, exact for 0 <= n < 2^31 (Granlund & Montgomery, "Division by
// invariant integers using multiplication", PLDI 1994, Theorem 4.2 with
// N = 31).  d == 1 is the identity (s = -1).
struct FastDiv {
  unsigned m;
  int s;
};

inline FastDiv make_fastdiv(unsigned d)
{
  FastDiv f{0u, -1};
  if (d <= 1) return f;
  int l = 0;
  while ((1ull << l) < d) ++l;                       // ceil(log2 d)
  const unsigned long long num = 1ull << (31 + l);
  f.m = (unsigned)((num + d - 1) / d);
  f.s = l - 1;
  return f;
}

__device__ __forceinline__ int fast_div(int n, FastDiv f)
{
  return f.s < 0 ? n : (int)(__umulhi((unsigned)n, f.m) >> f.s);
}

// Node class byte, built once per domain from the solids mask.
enum : uint8_t {
  CLS_SOLID = 1,      // byte == 1 in the reference's mask
  CLS_NEAR = 2,       // fluid with at least one solid neighbour: read nbm[n]
  CLS_NORTH = 4,      // 2D: row j = LY-1
  CLS_SOUTH = 8       // 2D: row j = 0
};

// Collision models: the reference's ACCURATE / COMPRESSIBLE flag pairs.
enum Model { SHIFTED_INC = 0, PLAIN_COMP = 1, SHIFTED_COMP = 2 };

// Face action per substance.  2D fused faces: what the last active boundary
// on that face does (boundaries on one face all rewrite the same three
// unknowns from the same knowns, and fusing requires fluid upstream nodes,
// so the last one in the reference's order decides); 3D z faces apply every
// configured operation in order (FaceOps).
enum FaceKind { FACE_NONE = 0, FACE_PRESSURE = 1, FACE_ZEROGRAD = 2, FACE_CONSTCON = 3,
                FACE_VELOCITY = 4 };

template <typename T>
struct SubsConst {
  T omc;     // 1 - 1/tau
  T itau;    // 1/tau
  T rhoA;    // rho_A
  T tg[3];   // tau * g  (velocity shift of the body force)
};

template <typename T>
struct StepArgs {
  T* f;                  // [nsubs][Q][N]
  T* mv;                 // [nsubs][1+D][N]
  const uint8_t* cls;    // [N]
  const uint32_t* nbm;   // [N]: bit a set iff node n + c_a is solid
  int LX, LY, LZ;
  long long N;
  SubsConst<T> sc[2];
  T sink1;               // (1 - sink * tau[1]) for the solute
  int write_mv;
  int solute_on;
  int kahan;                  // compensated density sums (flow lattice)
  int face_n[2], face_s[2];   // FaceKind per substance (2D, fused path)
  T rho_n[2], rho_s[2];       // face densities this step
  T drho_n[2], drho_s[2];     // face density minus rho_A, formed in double
  double* btc;                // plane record: [0][.] C, [1][.] u_x of the nodes [btc_lo, btc_hi)
  int btc_lo, btc_hi;         // node (dense) or slot (compact) range of the plane
  T* ubuf;                    // [3][stride]: the flow's u, handed to the solute
  long long ustride;          // N (dense) or P (compact)
  T* fout;                    // compact, OOP kernels: where the step's result goes
  // Walsh partial bounce-back (dense layout only): per-node fraction ns[N],
  // and tau and g as the reference's double-precision force term uses them
  const T* ns;
  double wtau[2];
  double wg[6];
};

// Which substances one launch of a step kernel advances.  Two-substance
// steps run as two launches: the flow (PART_FLOW), which also stores its
// post-force u, then the solute (PART_SOLUTE), which reads it.  One fused
// body holding both substances needs about twice the registers of either
// alone (halving occupancy); the split costs 24 B per FP32 node instead.
enum StepPart { PART_ALL = 0, PART_FLOW = 1, PART_SOLUTE = 2 };

// ---- per-node collision ---------------------------------------------------
// d[] holds the node's incoming populations of substance s; u carries the
// fluid velocity to the solute as the reference's per-thread scratch does.
// sinks: the solute sink applies once on odd steps and twice on even steps
// (src/k_stream_collide_stream.c:254-256; src/k_collide.c:96-97, :261-262).
// Returns the node's density (the solute's C), the value stored as rho.
// WALSH: partial bounce-back with the node's fraction ns (WALSH_NS_ON,
// src/k_stream_collide_stream.c:129-215, :363-386; src/lattice.c:2936-2939):
// the momentum is scaled by (1 - ns) before the division, the force term by
// (1 - ns), and each collided population is blended with the opposite
// incoming one, f_a <- f_a (1 - ns) + ns f_opp(a).  The factor 1 - ns is a
// double (the reference writes `1.`), so those products round once from
// double in FP32 as well.
// FP32 collision by opposite pairs (a, a+1) (same weight, opposite c): the
// moments come from pair sums and differences, the symmetric part of each
// pair's equilibrium (w rho / tau + w rq (4.5 (c.u)^2 - 1.5 u^2) / tau, or
// the solute's w C / tau) is formed once and the antisymmetric part
// (3 c.u times the same weight) is added to one population and subtracted
// from the other, and the three divisions of u by the density become one
// reciprocal: about a third fewer instructions than the per-direction form.
// A step run for seconds draws the B200's 1000 W cap and its SM clock falls
// to ~1.6 GHz, where the odd step's instruction count shows; sustained 256^3
// FP32 steps run 3% faster this way (0.196 vs 0.203 ms; a short burst at
// full clock gains under 1%).  The sums round in another order, which moves
// FP32 results by a few ulps; FP64, Kahan sums and Walsh runs keep the
// reference's operation order.
template <int Q, int MODEL>
__device__ __forceinline__ float collide_pairs(const StepArgs<float>& A, int s, bool solute,
                                               int sinks, float (&d)[Q], float (&u)[3],
                                               long long n)
{
  constexpr int D = (Q == 9) ? 2 : 3;
  constexpr int NP = (Q - 1) / 2;
  const SubsConst<float>& c = A.sc[s];
  float rho = d[0];
  float dif[NP];
#pragma unroll
  for (int p = 0; p < NP; ++p) {
    rho += d[2 * p + 1] + d[2 * p + 2];
    dif[p] = d[2 * p + 1] - d[2 * p + 2];
  }
  if (solute) {
    if (sinks == 2) rho *= A.sink1;
    rho *= A.sink1;
  } else {
    float m0 = 0.f, m1 = 0.f, m2 = 0.f;
#pragma unroll
    for (int p = 0; p < NP; ++p) {
      const int a = 2 * p + 1;
      if (cx(a) > 0) m0 += dif[p]; else if (cx(a) < 0) m0 -= dif[p];
      if (cy(a) > 0) m1 += dif[p]; else if (cy(a) < 0) m1 -= dif[p];
      if (D == 3) { if (cz(a) > 0) m2 += dif[p]; else if (cz(a) < 0) m2 -= dif[p]; }
    }
    const float den = (MODEL == SHIFTED_INC) ? c.rhoA
                    : (MODEL == PLAIN_COMP) ? rho : (c.rhoA + rho);
    const float inv = 1.f / den;
    u[0] = m0 * inv + c.tg[0];
    u[1] = m1 * inv + c.tg[1];
    u[2] = (D == 3) ? m2 * inv + c.tg[2] : 0.f;
  }
  if (A.write_mv) {
    float* m = A.mv + (long long)s * (1 + D) * A.N;
    m[n] = (!solute && MODEL != PLAIN_COMP) ? rho + c.rhoA : rho;
    m[A.N + n] = u[0];
    m[2 * A.N + n] = u[1];
    if (D == 3) m[3 * A.N + n] = u[2];
  }
  auto cdotu = [&](int a) -> float {
    float r = 0.f;
    if (cx(a) > 0) r += u[0]; else if (cx(a) < 0) r -= u[0];
    if (cy(a) > 0) r += u[1]; else if (cy(a) < 0) r -= u[1];
    if (D == 3) { if (cz(a) > 0) r += u[2]; else if (cz(a) < 0) r -= u[2]; }
    return r;
  };
  if (solute) {
    const float ci = rho * c.itau;
    d[0] = fmaf(d[0], c.omc, wgt<float, Q>(0) * ci);
#pragma unroll
    for (int p = 0; p < NP; ++p) {
      const int a = 2 * p + 1;
      const float base = wgt<float, Q>(a) * ci;
      const float anti = (3.f * base) * cdotu(a);
      d[a] = fmaf(d[a], c.omc, base + anti);
      d[a + 1] = fmaf(d[a + 1], c.omc, base - anti);
    }
  } else {
    const float usq = u[0] * u[0] + u[1] * u[1] + (D == 3 ? u[2] * u[2] : 0.f);
    const float rq = (MODEL == SHIFTED_INC) ? c.rhoA
                   : (MODEL == PLAIN_COMP) ? rho : (c.rhoA + rho);
    const float ri = rho * c.itau, qi = rq * c.itau;
    const float k = -1.5f * usq;
    d[0] = fmaf(d[0], c.omc, fmaf(wgt<float, Q>(0) * qi, k, wgt<float, Q>(0) * ri));
#pragma unroll
    for (int p = 0; p < NP; ++p) {
      const int a = 2 * p + 1;
      const float cu = cdotu(a);
      const float wq = wgt<float, Q>(a) * qi;
      const float sym = fmaf(wq, fmaf(4.5f * cu, cu, k), wgt<float, Q>(a) * ri);
      const float anti = (3.f * wq) * cu;
      d[a] = fmaf(d[a], c.omc, sym + anti);
      d[a + 1] = fmaf(d[a + 1], c.omc, sym - anti);
    }
  }
  return rho;
}

// UNIT_DEN: the caller knows the divisor of the momentum is exactly 1
// (the shifted incompressible model with rho_A = 1), and m / 1 == m in
// IEEE arithmetic, so the divisions are left out with the same results.
template <typename T, int Q, int MODEL, bool WALSH = false, bool UNIT_DEN = false>
__device__ __forceinline__ T collide(const StepArgs<T>& A, int s, bool solute,
                                        int sinks, T (&d)[Q], T (&u)[3],
                                        long long n)
{
  if constexpr (sizeof(T) == 4 && !WALSH) {
    if (!A.kahan)
      return collide_pairs<Q, MODEL>(A, s, solute, sinks, reinterpret_cast<float (&)[Q]>(d),
                                     reinterpret_cast<float (&)[3]>(u), n);
  }
  constexpr int D = (Q == 9) ? 2 : 3;
  const SubsConst<T>& c = A.sc[s];
  T nsv = T(0), pre[WALSH ? Q : 1];
  double om = 1.;
  if (WALSH) {
    nsv = A.ns[n];
    om = __dsub_rn(1., (double)nsv);
#pragma unroll
    for (int a = 0; a < Q; ++a) pre[WALSH ? a : 0] = d[a];
  }
  T rho = d[0];
  if (A.kahan && !solute) {
    // compensated sum (KAHAN_SUMMATION: fk_add, src/lattice.c:3099-3114)
    T corr = T(0);
#pragma unroll
    for (int a = 1; a < Q; ++a) {
      const T next = sub_(d[a], corr);
      const T sum = add_(rho, next);
      corr = sub_(sub_(sum, rho), next);
      rho = sum;
    }
  } else {
#pragma unroll
    for (int a = 1; a < Q; ++a) rho += d[a];
  }
  if (solute) {
    if (sinks == 2) rho *= A.sink1;
    rho *= A.sink1;
  } else {
    T m0 = T(0), m1 = T(0), m2 = T(0);
#pragma unroll
    for (int a = 0; a < Q; ++a) {
      if (cx(a) > 0) m0 += d[a]; else if (cx(a) < 0) m0 -= d[a];
      if (cy(a) > 0) m1 += d[a]; else if (cy(a) < 0) m1 -= d[a];
      if (D == 3) { if (cz(a) > 0) m2 += d[a]; else if (cz(a) < 0) m2 -= d[a]; }
    }
    T den = (MODEL == SHIFTED_INC) ? c.rhoA
          : (MODEL == PLAIN_COMP) ? rho : (c.rhoA + rho);
    if (WALSH) {
      m0 = (T)__dmul_rn((double)m0, om);
      m1 = (T)__dmul_rn((double)m1, om);
      if (D == 3) m2 = (T)__dmul_rn((double)m2, om);
      // u += ((1 - ns) tau) g, formed in double
      const double ot = __dmul_rn(om, A.wtau[s]);
      u[0] = (T)__dadd_rn((double)(m0 / den), __dmul_rn(ot, A.wg[s * 3 + 0]));
      u[1] = (T)__dadd_rn((double)(m1 / den), __dmul_rn(ot, A.wg[s * 3 + 1]));
      u[2] = (D == 3) ? (T)__dadd_rn((double)(m2 / den), __dmul_rn(ot, A.wg[s * 3 + 2]))
                      : T(0);
    } else if (UNIT_DEN) {
      u[0] = add_(m0, c.tg[0]);
      u[1] = add_(m1, c.tg[1]);
      u[2] = (D == 3) ? add_(m2, c.tg[2]) : T(0);
    } else {
      u[0] = add_(m0 / den, c.tg[0]);
      u[1] = add_(m1 / den, c.tg[1]);
      u[2] = (D == 3) ? add_(m2 / den, c.tg[2]) : T(0);
    }
  }
  if (A.write_mv) {
    T* m = A.mv + (long long)s * (1 + D) * A.N;
    m[n] = (!solute && MODEL != PLAIN_COMP) ? rho + c.rhoA : rho;
    m[A.N + n] = u[0];
    m[2 * A.N + n] = u[1];
    if (D == 3) m[3 * A.N + n] = u[2];
  }
  if (solute) {
    // g_a <- g_a (1 - 1/tau_s) + w_a C (1 + 3 c.u) / tau_s  (src/lattice.c:2858-2875)
#pragma unroll
    for (int a = 0; a < Q; ++a) {
      T cu = T(cx(a)) * u[0] + T(cy(a)) * u[1] + (D == 3 ? T(cz(a)) * u[2] : T(0));
      d[a] = add_(mul_(d[a], c.omc),
                  mul_(mul_(mul_(wgt<T, Q>(a), rho), add_(T(1), mul_(T(3), cu))), c.itau));
    }
  } else {
    // BGK in shifted or plain form (src/lattice.c:2880-2919):
    // d (1 - 1/tau) + w drho / tau + w rq (3 cu + 4.5 cu^2 - 1.5 u^2) / tau
    T usq = add_(mul_(u[0], u[0]), mul_(u[1], u[1]));
    if (D == 3) usq = add_(usq, mul_(u[2], u[2]));
    T rq = (MODEL == SHIFTED_INC) ? c.rhoA
         : (MODEL == PLAIN_COMP) ? rho : (c.rhoA + rho);
#pragma unroll
    for (int a = 0; a < Q; ++a) {
      // c.u: products by -1, 0, 1 are exact, so contraction cannot change it
      T cu = T(cx(a)) * u[0] + T(cy(a)) * u[1] + (D == 3 ? T(cz(a)) * u[2] : T(0));
      T w = wgt<T, Q>(a);
      T poly = sub_(add_(mul_(T(3), cu), mul_(mul_(T(4.5), cu), cu)), mul_(T(1.5), usq));
      d[a] = add_(add_(mul_(d[a], c.omc), mul_(mul_(w, rho), c.itau)),
                  mul_(mul_(mul_(w, rq), poly), c.itau));
    }
  }
  if (WALSH) {
#pragma unroll
    for (int a = 0; a < Q; ++a)
      d[a] = add_((T)__dmul_rn((double)d[a], om), mul_(nsv, pre[WALSH ? opp(a) : 0]));
  }
  return rho;
}

// ---- fused 2D faces ---------------------------------------------------------
// Zou-He density on the north / south row in shifted or plain form
// (src/system_boundary_kernels.c:58-83, :282-307) and the solute
// zero-gradient rule (:503-521, :692-710), applied to the node's incoming
// populations in registers.  Valid only where the reference's deposit of the
// unknowns lands on the slot this node then pulls (the host checks that the
// wrapped upstream nodes of every face node are fluid, else it runs the
// stand-alone face kernels below).
// In FP32 the shifted density balance cancels at magnitude 1
// (sum - rho_bc + rho_A with rho_bc ~ 1), which costs ~1e-5 relative in the
// unknowns; there the host passes rho_bc - rho_A formed in double instead
// (`drho`), so X = sum - drho keeps float precision.  FP64 keeps the
// reference's operation order.
template <typename T>
__device__ __forceinline__ T face_balance(T sum, T rho_bc, T rhoA, T drho, bool shifted)
{
  if (sizeof(T) == 4 && shifted) return sum - drho;
  T X = sum - rho_bc;
  if (shifted) X += rhoA;
  return X;
}

template <typename T>
__device__ __forceinline__ void face_north(int kind, T rho_bc, T rhoA, T drho, bool shifted,
                                           T (&d)[9])
{
  if (kind == FACE_PRESSURE) {
    const T X = face_balance<T>(d[DC] + d[DE] + d[DW] + d[DN] + d[DN] + d[DNE] + d[DNE]
                                + d[DNW] + d[DNW], rho_bc, rhoA, drho, shifted);
    d[DS] = sub_(d[DN], mul_(T(2. / 3.), X));
    d[DSW] = sub_(add_(d[DNE], mul_(T(0.5), d[DE] - d[DW])), mul_(T(1. / 6.), X));
    d[DSE] = sub_(add_(d[DNW], mul_(T(0.5), d[DW] - d[DE])), mul_(T(1. / 6.), X));
  } else if (kind == FACE_ZEROGRAD) {
    T X = (d[DN] + d[DNE] + d[DNW]) / (wgt<T, 9>(DS) + wgt<T, 9>(DSW) + wgt<T, 9>(DSE));
    d[DS] = wgt<T, 9>(DS) * X;
    d[DSW] = wgt<T, 9>(DSW) * X;
    d[DSE] = wgt<T, 9>(DSE) * X;
  }
}

template <typename T>
__device__ __forceinline__ void face_south(int kind, T rho_bc, T rhoA, T drho, bool shifted,
                                           T (&d)[9])
{
  if (kind == FACE_PRESSURE) {
    // south balance is the negated north one: -(sum) + rho_bc - rho_A
    const T X = -face_balance<T>(d[DC] + d[DE] + d[DW] + d[DS] + d[DS] + d[DSE] + d[DSE]
                                 + d[DSW] + d[DSW], rho_bc, rhoA, drho, shifted);
    d[DN] = add_(d[DS], mul_(T(2. / 3.), X));
    d[DNE] = add_(add_(d[DSW], mul_(T(0.5), d[DW] - d[DE])), mul_(T(1. / 6.), X));
    d[DNW] = add_(add_(d[DSE], mul_(T(0.5), d[DE] - d[DW])), mul_(T(1. / 6.), X));
  } else if (kind == FACE_ZEROGRAD) {
    T X = (d[DS] + d[DSW] + d[DSE]) / (wgt<T, 9>(DN) + wgt<T, 9>(DNE) + wgt<T, 9>(DNW));
    d[DN] = wgt<T, 9>(DN) * X;
    d[DNE] = wgt<T, 9>(DNE) * X;
    d[DNW] = wgt<T, 9>(DNW) * X;
  }
}

// ---- the AA step kernel -----------------------------------------------------
// ODD: pull d_a from f[a][n - c_a] (own f[opp a][n] if that node is solid),
//      collide, push d_a to f[opp a][n + c_a] (own f[a][n] if solid).
// EVEN: d_a = f[opp a][n], collide, f[a][n] = d_a.
// Each node reads and writes one fixed slot set, disjoint from every other
// node's, so the update is in place with no ordering between threads.
// WALSH (partial bounce-back, COMPUTE_ON_SOLIDS): every node is updated and
// streams periodically with no solid checks (src/lattice.c:2704-2707,
// :2812-2815); the collision blends by ns (see collide).
template <typename T, int Q, int NS, int MODEL, bool ODD, int PART, bool WALSH = false>
__global__ void __launch_bounds__(128)
aa_step(StepArgs<T> A)
{
  constexpr int D = (Q == 9) ? 2 : 3;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.LX) return;
  const int j = blockIdx.y, k = blockIdx.z;
  const int LX = A.LX, LY = A.LY;
  // Node indices are 32-bit (the host rejects N >= 2^31); direction planes
  // are reached through 64-bit base pointers, which are uniform per warp.
  const int plane = LX * LY;
  const int n = i + LX * j + plane * k;
  const uint8_t cl = WALSH ? uint8_t(0) : A.cls[n];
  if (cl & CLS_SOLID) return;
  const uint32_t nb = (cl & CLS_NEAR) ? A.nbm[n] : 0u;

  // dense offsets to the neighbours along each axis (periodic on every
  // axis, a serial run's wrap); neighbour n + c_a = n + off(a)
  int xm = (i == 0) ? LX - 1 : -1, xp = (i == LX - 1) ? 1 - LX : 1;
  int ym = (j == 0) ? plane - LX : -LX, yp = (j == LY - 1) ? LX - plane : LX;
  int zm = 0, zp = 0;
  if (D == 3) {
    const int tot = plane * A.LZ;
    zm = (k == 0) ? tot - plane : -plane;
    zp = (k == A.LZ - 1) ? plane - tot : plane;
  }
  auto off = [&](int a) -> int {
    return (cx(a) < 0 ? xm : (cx(a) > 0 ? xp : 0)) + (cy(a) < 0 ? ym : (cy(a) > 0 ? yp : 0))
         + (cz(a) < 0 ? zm : (cz(a) > 0 ? zp : 0));
  };

  T u[3] = {T(0), T(0), T(0)};
  constexpr int S_BEGIN = (PART == PART_SOLUTE) ? 1 : 0;
  constexpr int S_END = (PART == PART_FLOW) ? 1 : NS;
  if (PART == PART_SOLUTE) {
#pragma unroll
    for (int c = 0; c < D; ++c) u[c] = A.ubuf[c * A.ustride + n];
  }
#pragma unroll
  for (int s = S_BEGIN; s < S_END; ++s) {
    const bool solute = (NS == 2 && s == 1);
    if (solute && !A.solute_on) break;
    if (s > 0) {
      // recompute the solute's neighbour addresses rather than keeping the
      // flow's live across the flow's collision and push, and start only
      // after the flow's stores are issued
      asm volatile("" ::: "memory");
      xm = opaque(xm); xp = opaque(xp); ym = opaque(ym); yp = opaque(yp);
      if (D == 3) { zm = opaque(zm); zp = opaque(zp); }
    }
    T* const fs = A.f + (size_t)s * Q * (size_t)A.N;
    const size_t N = (size_t)A.N;
    T d[Q];
    if (ODD) {
      // pull: d_a = f[a][n - c_a], or own f[opp a][n] behind a solid
#pragma unroll
      for (int a = 0; a < Q; ++a) {
        const size_t src = ((nb >> opp(a)) & 1u) ? (size_t)opp(a) * N + n
                                                 : (size_t)a * N + (size_t)(n + off(opp(a)));
        d[a] = fs[src];
      }
    } else {
#pragma unroll
      for (int a = 0; a < Q; ++a) d[a] = fs[opp(a) * N + n];
    }
    if (Q == 9 && (cl & (CLS_NORTH | CLS_SOUTH))) {
      T (&d9)[9] = reinterpret_cast<T (&)[9]>(d);
      const bool shifted = (MODEL != PLAIN_COMP) && !solute;
      if (cl & CLS_NORTH)
        face_north<T>(A.face_n[s], A.rho_n[s], A.sc[s].rhoA, A.drho_n[s], shifted, d9);
      if (cl & CLS_SOUTH)
        face_south<T>(A.face_s[s], A.rho_s[s], A.sc[s].rhoA, A.drho_s[s], shifted, d9);
    }
    const T rho = collide<T, Q, MODEL, WALSH>(A, s, solute, ODD ? 1 : 2, d, u, n);
    if (PART == PART_FLOW && A.solute_on) {
#pragma unroll
      for (int c = 0; c < D; ++c) A.ubuf[c * A.ustride + n] = u[c];
    }
    if (A.btc && n >= A.btc_lo && n < A.btc_hi) {
      if (NS == 2 && solute) A.btc[n - A.btc_lo] = (double)rho;
      else if (!solute) A.btc[(A.btc_hi - A.btc_lo) + (n - A.btc_lo)] = (double)u[0];
    }
    if (ODD) {
      // push: f[opp a][n + c_a] = d_a, or own f[a][n] in front of a solid
      // (offsets laundered so the pull addresses are not kept live)
      xm = opaque(xm); xp = opaque(xp); ym = opaque(ym); yp = opaque(yp);
      if (D == 3) { zm = opaque(zm); zp = opaque(zp); }
#pragma unroll
      for (int a = 0; a < Q; ++a) {
        const size_t dst = ((nb >> a) & 1u) ? (size_t)a * N + n
                                            : (size_t)opp(a) * N + (size_t)(n + off(a));
        fs[dst] = d[a];
      }
    } else {
      const int n2 = opaque(n);   // do not keep the load addresses live
#pragma unroll
      for (int a = 0; a < Q; ++a) fs[a * N + n2] = d[a];
    }
  }
}

// ---- the AA step on the compact fluid-only layout ---------------------------
// Populations are stored for fluid nodes only, [subs][a][F] in dense node
// order, so a warp's accesses in every direction plane cover only fluid
// data (with 60% solids a dense layout fetches ~2x the useful bytes at
// sector granularity).  fidx[n] maps a dense node to its compact index
// (-1: solid; the face kernels use it), fnode[m] maps back, and frm holds
// the fluid bitmask with word ranks the odd step finds neighbours in.  One
// thread per fluid node.
// The z-face operations of one step applied inside the compact step kernel
// (the FACES3 instantiations) instead of by the stand-alone face_plane
// kernel.  Exact wherever that kernel's deposit is read only by the face
// node itself: always before an even step (it works on the node's own
// slots), and before an odd step when every upstream node of every unknown
// direction of every fluid face node is fluid (the host checks; otherwise
// face_plane runs).  The bottom plane's fluid nodes are the compact indices
// [0, lo_end), the top plane's [hi_start, F).  Per substance and face, the
// operations in their configured order.
constexpr int kFace3PerGroup = 6;   // pressure in/out, velocity in/out, constcon, zero gradient

template <typename T>
struct Face3Fused {
  int lo_end, hi_start;
  int nops[2][2];                        // [substance][top]
  int kind[2][2][kFace3PerGroup];
  T drho[2][2][kFace3PerGroup];          // pressure: rho_bc - rA; velocity: u_z
  T shift[2][2][kFace3PerGroup];         // velocity: rA
  const T* profile[2][2][kFace3PerGroup];  // constant concentration per (i, j), or NULL
  T conc;
};

template <typename T>
__device__ __forceinline__ void face3_apply(T (&d)[19], bool top, int kind, T drho, T conc,
                                            T shift);

template <typename T>
struct CompactArgs {
  StepArgs<T> s;          // f = compact populations; N = dense node count
  const int* fidx;        // [N]
  const int* fnode;       // [F]
  const uint2* frm;       // [ceil(N/32)]: (fluid nodes before the word, fluid bits),
                          // with a guard word at [-1] (0, 0) and at [ceil(N/32)] (F, 0)
  int F;                  // fluid nodes
  int P;                  // plane stride of fc: F rounded up to 32 (aligned warps)
  FastDiv div_plane, div_lx;   // n / (LX*LY), r / LX
  int faces;              // 2D: fused face boundaries configured
  Face3Fused<T> f3;       // 3D: read by the FACES3 kernels only
  // the compact indices a launch covers: thread t takes m = t + m_base,
  // moved on by m_jump once it reaches m_skip, up to m_end (the whole range
  // [0, F), the interior between the z-face planes, or the two planes)
  int m_base, m_skip, m_jump, m_end;
};

// Resident 256-thread blocks asked of the compiler: six (40 registers) for
// the FP32 kernels, where that measured fastest (the solute kernel spills
// 12-16 bytes there and still runs 4% faster than at three blocks, its
// natural 85 registers); for FP64 the cap closest above the natural
// register count (flow 85, solute 128), since a lower cap spills more.
template <typename T, int PART>
constexpr int compact_min_blocks()
{
  return sizeof(T) == 4 ? 6 : (PART == PART_SOLUTE ? 2 : 3);
}

// The odd step of two substances in one launch (flow, then the solute from
// the flow's slot table): four resident blocks (64 registers) in FP32,
// where it runs without spills (at six blocks it spilled and ran no faster
// than the two launches it replaces); two (128) in FP64, which spills 4-12
// bytes there and 230-250 at three blocks.
template <typename T, int PART, int NS, bool FACES3>
constexpr int compact_step_min_blocks()
{
  return (PART == PART_ALL && NS == 2 && !FACES3) ? (sizeof(T) == 4 ? 4 : 2)
                                                  : compact_min_blocks<T, PART>();
}

// IDX32: population offsets within one substance's [Q][P] block fit in 32
// bits (Q * P < 2^32), so slot selects and address arithmetic stay 32-bit.
// OOP: write the step's result to C.s.fout instead of in place (used to
// recompute stored forward states for the adjoint).
// The update of fluid node m (compact index) by one block thread; the
// odd step's slot table is indexed by threadIdx.x, so a block's threads
// handle distinct nodes.
template <typename T, int Q, int NS, int MODEL, bool ODD, int PART, bool IDX32, bool OOP,
          bool FACES3 = false>
__device__ __forceinline__ void compact_node(const CompactArgs<T>& C, const int m)
{
  using Idx = typename std::conditional<IDX32, unsigned, size_t>::type;
  constexpr int D = (Q == 9) ? 2 : 3;
  const StepArgs<T>& A = C.s;
  const Idx F = (Idx)C.P;   // plane stride
  const int LX = A.LX, LY = A.LY;
  const int plane = LX * LY;
  const bool faces = (Q == 9) && C.faces;
  int n = 0, j = 0;
  // dense offsets to the neighbours along each axis (odd step)
  int xm = 0, xp = 0, ym = 0, yp = 0, zm = 0, zp = 0;
  if (ODD || A.write_mv || faces) {
    n = C.fnode[m];
    const int k = fast_div(n, C.div_plane);
    const int r = n - k * plane;
    j = fast_div(r, C.div_lx);
    const int i = r - j * LX;
    if (ODD) {
      xm = (i == 0) ? LX - 1 : -1; xp = (i == LX - 1) ? 1 - LX : 1;
      ym = (j == 0) ? plane - LX : -LX; yp = (j == LY - 1) ? LX - plane : LX;
      if (D == 3) {
        const int tot = plane * A.LZ;
        zm = (k == 0) ? tot - plane : -plane;
        zp = (k == A.LZ - 1) ? plane - tot : plane;
      }
    }
  }
  // dense offset of neighbour n + c_a
  auto off = [&](int a) -> int {
    return (cx(a) < 0 ? xm : (cx(a) > 0 ? xp : 0)) + (cy(a) < 0 ? ym : (cy(a) > 0 ? yp : 0))
         + (cz(a) < 0 ? zm : (cz(a) > 0 ? zp : 0));
  };
  // compact index of dense node q, -1 if solid: the fluid nodes before
  // its 32-node word plus the fluid bits below it in the word.
  // The table is 8 B per 32 nodes (4 MB at 256^3, resident in L2) where a
  // dense index array is 4 B per node.
  auto nb_at = [&](int qi) -> int {
    const unsigned q = (unsigned)qi;
    const uint2 w = __ldg(C.frm + (q >> 5));
    const unsigned b = q & 31u;
    const int idx = (int)(w.x + (unsigned)__popc(w.y & ((1u << b) - 1u)));
    return ((w.y >> b) & 1u) ? idx : -1;
  };
  // the three x neighbours q0 - 1, q0, q0 + 1 of an x row from one window
  // of the bitmask (the words holding q0 - 1 and the next; a guard word
  // on either side of the table keeps q0 = 0 and q0 = N - 1 in bounds):
  // one rank, then +1 per fluid bit.  Valid where the x offsets are -1 and
  // +1; a node on an x edge looks its wrapped neighbour up directly.
  // own >= 0: the row is the node's own (q0 = n), whose rank is own.
  auto row3 = [&](int q0, int own, int& im, int& i0, int& ip) {
    const int k = (q0 - 1) >> 5;          // -1 for q0 = 0: the front guard
    const unsigned p = (unsigned)(q0 - 1) & 31u;
    const uint2 w = __ldg(C.frm + k);
    const unsigned hi = __ldg(&C.frm[k + 1].y);
    const unsigned t = __funnelshift_r(w.y, hi, p);   // bits of q0-1, q0, q0+1
    // fluid nodes before q0
    const int rb = (own >= 0) ? own
                 : (int)(w.x + (unsigned)__popc(w.y & ((1u << p) - 1u)) + (t & 1u));
    im = (t & 1u) ? rb - 1 : -1;
    i0 = (t & 2u) ? rb : -1;
    ip = (t & 4u) ? rb + (int)((t >> 1) & 1u) : -1;
    if (xm != -1) im = nb_at(q0 + xm);
    if (xp != 1) ip = nb_at(q0 + xp);
  };
  T u[3] = {T(0), T(0), T(0)};
  constexpr int S_BEGIN = (PART == PART_SOLUTE) ? 1 : 0;
  constexpr int S_END = (PART == PART_FLOW) ? 1 : NS;
  if (PART == PART_SOLUTE) {
#pragma unroll
    for (int c = 0; c < D; ++c) u[c] = A.ubuf[c * A.ustride + m];
  }
#pragma unroll
  for (int s = S_BEGIN; s < S_END; ++s) {
    const bool solute = (NS == 2 && s == 1);
    if (solute && !A.solute_on) break;
    if (s > 0) {
      // the solute re-reads its neighbour indices (L1 hits) rather than
      // keeping the flow's live across the flow's collision and push, and
      // starts only after the flow's stores are issued
      asm volatile("" ::: "memory");
      xm = opaque(xm); xp = opaque(xp); ym = opaque(ym); yp = opaque(yp);
      if (D == 3) { zm = opaque(zm); zp = opaque(zp); }
    }
    T* const fs = A.f + (size_t)s * Q * F;
    T* const fo = (OOP ? A.fout : A.f) + (size_t)s * Q * F;
    // the odd step's pull slots: the push writes d_a back to the slot it
    // pulled d_opp(a) from (the AA pattern's in-place pairing), so the
    // push reads them here instead of repeating the 18 index lookups;
    // one column per thread, no barrier needed
    // (offsets in the kernel's index type: 64-bit above 2^32 slots)
    __shared__ Idx sslot[ODD ? Q : 1][256];
    T d[Q];
    if (ODD) {
      // pull: d_a = f[a][idx(n - c_a)], or own f[opp a] behind a solid; the
      // slot is chosen by integer select so every load issues unconditionally
      auto pull = [&](int a, int up) {
        const Idx src = (up >= 0) ? (Idx)a * F + (Idx)up : (Idx)opp(a) * F + (Idx)m;
        sslot[a][threadIdx.x] = src;
        d[a] = fs[src];
      };
      if (PART == PART_ALL && NS == 2 && s > 0) {
        // the solute's slots are the flow's (the same solids): read them from
        // the table the flow's pulls filled, this thread's column, instead of
        // repeating the upstream lookups
#pragma unroll
        for (int a = 0; a < Q; ++a) d[a] = fs[sslot[a][threadIdx.x]];
      } else if (NS == 1) {
        // one lookup per direction: measured faster than the row windows
        // below for the flow-only kernels (0.214 vs 0.218 ms at 256^3 FP32)
        pull(0, m);
#pragma unroll
        for (int a = 1; a < Q; ++a) pull(a, nb_at(n + off(opp(a))));
      } else {
        pull(0, m);
        // two substances: upstream neighbours n - c_a grouped by their (y, z)
        // row, three per window (the split flow + solute step pair 1.2%
        // faster at 256^3 FP32)
#pragma unroll
        for (int dz = (D == 3 ? -1 : 0); dz <= (D == 3 ? 1 : 0); ++dz) {
#pragma unroll
          for (int dy = -1; dy <= 1; ++dy) {
            bool any = false, anyx = false;
#pragma unroll
            for (int a = 1; a < Q; ++a)
              if (-cy(a) == dy && -cz(a) == dz) { any = true; anyx |= (cx(a) != 0); }
            if (!any) continue;
            const int q0 = n + (dy < 0 ? ym : (dy > 0 ? yp : 0)) + (dz < 0 ? zm : (dz > 0 ? zp : 0));
            if (!anyx) {
#pragma unroll
              for (int a = 1; a < Q; ++a)
                if (-cy(a) == dy && -cz(a) == dz) pull(a, nb_at(q0));
              continue;
            }
            int im, i0, ip;
            row3(q0, (dy == 0 && dz == 0) ? m : -1, im, i0, ip);
#pragma unroll
            for (int a = 1; a < Q; ++a)
              if (-cy(a) == dy && -cz(a) == dz)
                pull(a, cx(a) > 0 ? im : (cx(a) < 0 ? ip : i0));
          }
        }
      }
    } else {
#pragma unroll
      for (int a = 0; a < Q; ++a) d[a] = fs[opp(a) * F + m];
    }
    if constexpr (FACES3 && Q == 19) {
      // z faces: the stand-alone face_plane rules on the loaded populations
      const bool bot = m < C.f3.lo_end, top = m >= C.f3.hi_start;
      if (bot || top) {
        const int tp = top ? 1 : 0;
        const int cnt = C.f3.nops[s][tp];
        for (int q = 0; q < cnt; ++q) {
          T conc = C.f3.conc;
          const T* prof = C.f3.profile[s][tp][q];
          if (prof) {
            const int nd = (ODD || A.write_mv) ? n : C.fnode[m];
            conc = prof[nd - (top ? (A.LZ - 1) * plane : 0)];
          }
          face3_apply<T>(reinterpret_cast<T (&)[19]>(d), top, C.f3.kind[s][tp][q],
                         C.f3.drho[s][tp][q], conc, C.f3.shift[s][tp][q]);
        }
      }
    }
    if (faces && (j == 0 || j == LY - 1)) {
      T (&d9)[9] = reinterpret_cast<T (&)[9]>(d);
      const bool shifted = (MODEL != PLAIN_COMP) && !solute;
      if (j == LY - 1)
        face_north<T>(A.face_n[s], A.rho_n[s], A.sc[s].rhoA, A.drho_n[s], shifted, d9);
      if (j == 0)
        face_south<T>(A.face_s[s], A.rho_s[s], A.sc[s].rhoA, A.drho_s[s], shifted, d9);
    }
    const T rho = collide<T, Q, MODEL>(A, s, solute, ODD ? 1 : 2, d, u, n);
    // the flow's u for the solute launch, or, written out of place by the
    // joint launch (the adjoint's recomputation), kept for the adjoint
    if ((PART == PART_FLOW || (PART == PART_ALL && NS == 2 && OOP && s == 0)) && A.solute_on) {
#pragma unroll
      for (int c = 0; c < D; ++c) A.ubuf[c * A.ustride + m] = u[c];
    }
    if (A.btc && m >= A.btc_lo && m < A.btc_hi) {
      if (NS == 2 && solute) A.btc[m - A.btc_lo] = (double)rho;
      else if (!solute) A.btc[(A.btc_hi - A.btc_lo) + (m - A.btc_lo)] = (double)u[0];
    }
    if (ODD) {
      // push: f[opp a][idx(n + c_a)] = d_a, or own f[a] in front of a solid;
      // the neighbour indices are re-read rather than kept in registers
      xm = opaque(xm); xp = opaque(xp); ym = opaque(ym); yp = opaque(yp);
      if (D == 3) { zm = opaque(zm); zp = opaque(zp); }
#pragma unroll
      for (int a = 0; a < Q; ++a) fo[sslot[opp(a)][threadIdx.x]] = d[a];
    } else {
      const int m2 = opaque(m);   // do not keep the load addresses live
#pragma unroll
      for (int a = 0; a < Q; ++a) fo[a * F + m2] = d[a];
    }
  }
}

template <typename T, int Q, int NS, int MODEL, bool ODD, int PART, bool IDX32, bool OOP,
          bool FACES3 = false>
__global__ void __launch_bounds__(256, (compact_step_min_blocks<T, PART, NS, FACES3>()))
aa_step_compact(CompactArgs<T> C)
{
  int m = blockIdx.x * blockDim.x + threadIdx.x + C.m_base;
  if (m >= C.m_skip) m += C.m_jump;
  if (m >= C.m_end) return;
  compact_node<T, Q, NS, MODEL, ODD, PART, IDX32, OOP, FACES3>(C, m);
}

// Dense <-> compact exchange of all substances' populations.
template <typename T>
__global__ void gather_compact(T* fc, const T* fdense, const int* fnode, int F, int P,
                               long long N, int planes)
{
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)F * planes) return;
  const int pl = (int)(t / F), m = (int)(t - (long long)pl * F);
  fc[(long long)pl * P + m] = fdense[(long long)pl * N + fnode[m]];
}

template <typename T>
__global__ void scatter_compact(T* fdense, const T* fc, const int* fnode, int F, int P,
                                long long N, int planes)
{
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)F * planes) return;
  const int pl = (int)(t / F), m = (int)(t - (long long)pl * F);
  fdense[(long long)pl * N + fnode[m]] = fc[(long long)pl * P + m];
}

// Stand-alone face kernel on the compact layout: the same deposits as
// face_row, with each fluid node's slot reached through fidx.
template <typename T>
__global__ void face_row_compact(T* fs, const int* fidx, int LX, int LY, int F,
                                 int north, int kind, int second, T rho_bc, T rhoA,
                                 T drho, int shifted)  // F: plane stride of fs
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= LX) return;
  const int j = north ? LY - 1 : 0;
  const int m = fidx[i + LX * j];
  if (m < 0) return;
  auto cidx = [&](int ii, int jj) -> int {
    ii = ii < 0 ? ii + LX : (ii == LX ? 0 : ii);
    jj = jj < 0 ? jj + LY : (jj == LY ? 0 : jj);
    return fidx[ii + LX * jj];
  };
  const size_t P = (size_t)F;
  T d[9];
#pragma unroll
  for (int a = 0; a < 9; ++a) {
    if (second) {
      d[a] = fs[opp(a) * P + m];
    } else {
      const int up = cidx(i - cx(a), j - cy(a));
      d[a] = (up < 0) ? fs[opp(a) * P + m] : fs[a * P + up];
    }
  }
  if (north) face_north<T>(kind, rho_bc, rhoA, drho, shifted != 0, d);
  else face_south<T>(kind, rho_bc, rhoA, drho, shifted != 0, d);
  const int unk[3] = {north ? DS : DN, north ? DSE : DNW, north ? DSW : DNE};
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const int a = unk[q];
    if (second) {
      fs[opp(a) * P + m] = d[a];
    } else {
      const int up = cidx(i - cx(a), j - cy(a));
      if (up < 0) fs[a * P + m] = d[a];
      else fs[a * P + up] = d[a];
    }
  }
}

// ---- stand-alone 2D face kernels (exact reference semantics) ----------------
// One thread per node of the row.  `_1` form (before an odd step): pull the
// node's populations through bounce-back, compute the unknowns, deposit each
// into slot a of the upstream node n - c_a, or into the node's own slot a if
// that node is solid (set_f1d_d with offset -c_a).  `_2` form (before an even
// step): swapped own-slot load, unknown a stored in own slot opp(a).
template <typename T>
__global__ void face_row(T* fs, const uint8_t* solids, int LX, int LY,
                         long long N, int north, int kind, int second, T rho_bc,
                         T rhoA, T drho, int shifted)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= LX) return;
  const int j = north ? LY - 1 : 0;
  const long long n = (long long)i + (long long)LX * j;
  if (solids[n] == 1) return;
  auto wrap = [&](int ii, int jj) -> long long {
    ii = ii < 0 ? ii + LX : (ii == LX ? 0 : ii);
    jj = jj < 0 ? jj + LY : (jj == LY ? 0 : jj);
    return (long long)ii + (long long)LX * jj;
  };
  T d[9];
#pragma unroll
  for (int a = 0; a < 9; ++a) {
    if (second) {
      d[a] = fs[(long long)opp(a) * N + n];
    } else {
      const long long up = wrap(i - cx(a), j - cy(a));
      d[a] = (solids[up] == 1) ? fs[(long long)opp(a) * N + n]
                               : fs[(long long)a * N + up];
    }
  }
  if (north) face_north<T>(kind, rho_bc, rhoA, drho, shifted != 0, d);
  else face_south<T>(kind, rho_bc, rhoA, drho, shifted != 0, d);
  const int u0 = north ? DS : DN, u1 = north ? DSE : DNW, u2 = north ? DSW : DNE;
  const int unk[3] = {u0, u1, u2};
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const int a = unk[q];
    if (second) {
      fs[(long long)opp(a) * N + n] = d[a];
    } else {
      const long long up = wrap(i - cx(a), j - cy(a));
      if (solids[up] == 1) fs[(long long)a * N + n] = d[a];
      else fs[(long long)a * N + up] = d[a];
    }
  }
}

// ---- 3D z faces (stand-alone, before each step) ------------------------------
// top = plane k = LZ-1 (unknowns: the five cz = -1 directions), bottom =
// plane k = 0 (unknowns: cz = +1).  No reference device code exists for
// these faces: the rules are the 2D kernels' carried to z.  Zou-He density
// with zero tangential velocity (D3Q19 reconstruction as in the reference's
// CPU top/bottom code, src/bcs.c:596-870):
//   J = rho u_z from the density balance against drho (= rho_bc - rho_A in
//   shifted form, rho_bc otherwise, formed in double by the host), then
//   bottom: d_T = d_B + J/3, d_TE = d_BW + J/6 - Nx, d_TW = d_BE + J/6 + Nx,
//           d_TN = d_BS + J/6 - Ny, d_TS = d_BN + J/6 + Ny;
//   top:    d_B = d_T - J/3, d_BW = d_TE - J/6 + Nx, d_BE = d_TW - J/6 - Nx,
//           d_BS = d_TN - J/6 + Ny, d_BN = d_TS - J/6 - Ny,
// Nx, Ny half the in-plane x / y momentum.  Zero gradient: unknowns w_a X,
// X = (sum of the populations opposite them) / (sum of their weights), the
// rule of src/system_boundary_kernels.c:503-521.  Constant concentration:
// unknowns w_a X with X = (conc - sum of the known populations) / (sum of
// the unknowns' weights).  Operation order is fixed (FP64 is bit-compatible
// with the CPU restatement).
enum { D3T = 9, D3B, D3TE, D3BW, D3TW, D3BE, D3TN, D3BS, D3TS, D3BN };

__device__ __forceinline__ int face3_unknown(bool top, int q)
{
  return top ? D3B + 2 * q : D3T + 2 * q;   // B,BW,BE,BS,BN / T,TE,TW,TN,TS
}

// Velocity (the reference's CPU rule, src/bcs.c:764-862): rho =
// (S0 + 2 S_out + rA) / (1 + u) on the top, / (1 - u) on the bottom, formed
// in double as the reference's `1.` makes it in FP32 builds, and J = rho u;
// `drho` carries u and `shift` rA (rho_A for shifted populations, else 0).
template <typename T>
__device__ __forceinline__ T face3_velocity_J(T S0, T Sout, T u, T shift, bool top)
{
  const double s = __dadd_rn(__dadd_rn((double)S0, __dmul_rn(2., (double)Sout)), (double)shift);
  const double den = top ? __dadd_rn(1., (double)u) : __dsub_rn(1., (double)u);
  const T rho = (T)(s / den);
  return mul_(rho, u);
}

template <typename T>
__device__ __forceinline__ void face3_apply(T (&d)[19], bool top, int kind, T drho, T conc,
                                            T shift)
{
  if (kind == FACE_PRESSURE || kind == FACE_VELOCITY) {
    T S0 = d[DC];
#pragma unroll
    for (int a = 1; a < 9; ++a) S0 = add_(S0, d[a]);
    const T Nx = mul_(T(0.5), sub_(add_(add_(d[DE], d[DNE]), d[DSE]), add_(add_(d[DW], d[DSW]), d[DNW])));
    const T Ny = mul_(T(0.5), sub_(add_(add_(d[DN], d[DNE]), d[DNW]), add_(add_(d[DS], d[DSW]), d[DSE])));
    if (top) {
      const T Sp = add_(add_(add_(add_(d[D3T], d[D3TE]), d[D3TW]), d[D3TN]), d[D3TS]);
      const T J = kind == FACE_VELOCITY ? face3_velocity_J<T>(S0, Sp, drho, shift, true)
                                        : sub_(add_(S0, mul_(T(2), Sp)), drho);
      const T J3 = J / T(3), J6 = J / T(6);
      d[D3B] = sub_(d[D3T], J3);
      d[D3BW] = add_(sub_(d[D3TE], J6), Nx);
      d[D3BE] = sub_(sub_(d[D3TW], J6), Nx);
      d[D3BS] = add_(sub_(d[D3TN], J6), Ny);
      d[D3BN] = sub_(sub_(d[D3TS], J6), Ny);
    } else {
      const T Sm = add_(add_(add_(add_(d[D3B], d[D3BW]), d[D3BE]), d[D3BS]), d[D3BN]);
      const T J = kind == FACE_VELOCITY ? face3_velocity_J<T>(S0, Sm, drho, shift, false)
                                        : sub_(drho, add_(S0, mul_(T(2), Sm)));
      const T J3 = J / T(3), J6 = J / T(6);
      d[D3T] = add_(d[D3B], J3);
      d[D3TE] = sub_(add_(d[D3BW], J6), Nx);
      d[D3TW] = add_(add_(d[D3BE], J6), Nx);
      d[D3TN] = sub_(add_(d[D3BS], J6), Ny);
      d[D3TS] = add_(add_(d[D3BN], J6), Ny);
    }
  } else {
    T wsum = wgt<T, 19>(face3_unknown(top, 0));
#pragma unroll
    for (int q = 1; q < 5; ++q) wsum = add_(wsum, wgt<T, 19>(face3_unknown(top, q)));
    T X;
    if (kind == FACE_ZEROGRAD) {
      T num = d[opp(face3_unknown(top, 0))];
#pragma unroll
      for (int q = 1; q < 5; ++q) num = add_(num, d[opp(face3_unknown(top, q))]);
      X = num / wsum;
    } else {
      T known = d[0];
#pragma unroll
      for (int a = 1; a < 19; ++a)
        if (cz(a) != (top ? -1 : 1)) known = add_(known, d[a]);
      X = sub_(conc, known) / wsum;
    }
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      const int a = face3_unknown(top, q);
      d[a] = mul_(wgt<T, 19>(a), X);
    }
  }
}

// The face operations of one step, grouped by (face, substance) in their
// configured order.  For LZ >= 3 different groups touch disjoint slots, so
// the groups run side by side in one launch (blockIdx.z = group).  Within a
// group the operations run in order in each thread: an operation reads the
// known slots and rewrites the five unknowns, and at a face node with
// solids above and below a known slot of the node is also the slot its
// unknown is deposited in (the own-slot fallback on both sides), so a later
// operation can read an earlier one's result.  Every slot involved belongs
// to the thread's own node, so no other thread sees the intermediate.
constexpr int kFaceOpsMax = 24;   // 2 substances x 2 faces x 4 pressure/velocity + 4 solute ops

template <typename T>
struct FaceOps {
  int ngroups;
  int first[4], count[4];          // each group's operations: [first, first + count)
  int top[4], subs[4];             // each group's face and substance
  int kind[kFaceOpsMax];
  T drho[kFaceOpsMax];             // pressure: rho_bc - rA; velocity: u_z
  T shift[kFaceOpsMax];            // velocity: rA
  const T* profile[kFaceOpsMax];   // constant concentration per node, or NULL
  T conc;                          // constant concentration otherwise
};

// The face operations of group g at node (i, j) of the top (TOP) or bottom
// plane, whose populations are at slots `self` of fs (see face_plane).
template <typename T, bool COMPACT, bool TOP>
__device__ __forceinline__ void face_plane_node(T* fs, const uint8_t* solids, const int* fidx,
                                                int LX, int LY, int LZ, long long stride,
                                                int second, const FaceOps<T>& ops, int g,
                                                int i, int j, int self)
{
  const int k = TOP ? LZ - 1 : 0;
  const int plane = LX * LY;
  // slot of the upstream node n - c_a, -1 if it is solid, for every a
  // before any population moves: looked up between the stores, each lookup
  // waited for the store before it (the compiler cannot tell the arrays
  // apart).  TOP is a compile-time constant so that every index into the
  // per-direction arrays is one, and they stay in registers.
  int up[19];
#pragma unroll
  for (int a = 0; a < 19; ++a) {
    if (second || a == 0) { up[a] = self; continue; }
    int ii = i - cx(a), jj = j - cy(a), kk = k - cz(a);
    ii = ii < 0 ? LX - 1 : (ii == LX ? 0 : ii);
    jj = jj < 0 ? LY - 1 : (jj == LY ? 0 : jj);
    kk = kk < 0 ? LZ - 1 : (kk == LZ ? 0 : kk);
    const int q = ii + LX * jj + plane * kk;
    if (COMPACT) up[a] = fidx[q];
    else up[a] = solids[q] == 1 ? -1 : q;
  }
  // the group's operations in order; each loads only the populations its
  // rule reads: the knowns (cz != the unknowns'), or for the zero gradient
  // the five opposite the unknowns
  constexpr int cz_unknown = TOP ? -1 : 1;
  const int q_end = ops.first[g] + ops.count[g];
  for (int q0 = ops.first[g]; q0 < q_end; ++q0) {
    const int kind = ops.kind[q0];
    T d[19];
#pragma unroll
    for (int a = 0; a < 19; ++a) {
      const bool need = kind == FACE_ZEROGRAD ? cz(a) == -cz_unknown : cz(a) != cz_unknown;
      if (!need) { d[a] = T(0); continue; }
      if (second) d[a] = fs[opp(a) * stride + self];
      else d[a] = (up[a] < 0) ? fs[opp(a) * stride + self] : fs[a * stride + up[a]];
    }
    const T* prof = ops.profile[q0];
    face3_apply<T>(d, TOP, kind, ops.drho[q0], prof ? prof[i + LX * j] : ops.conc,
                   ops.shift[q0]);
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      const int a = face3_unknown(TOP, q);
      if (second) fs[opp(a) * stride + self] = d[a];
      else fs[a * stride + (up[a] < 0 ? self : up[a])] = d[a];
    }
  }
}

// One thread per (i, j) of one group.  `_1` form (second == 0, before
// an odd step): loads what the odd step will pull and deposits the unknowns
// where it will pull them from (slot a of the upstream node, or of the node
// itself behind a solid, as set_f1d_d does); `_2` form (before an even
// step): the node's own swapped slots.  The dense layout tests solids, the
// compact one maps nodes through fidx.  f is [nsubs][Q][stride].
template <typename T, bool COMPACT>
__global__ void face_plane(T* f, const uint8_t* solids, const int* fidx, int LX, int LY,
                           int LZ, long long stride, int second, FaceOps<T> ops)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= LX) return;
  const int j = blockIdx.y;
  const int g = blockIdx.z;
  const int top = ops.top[g];
  T* const fs = f + (long long)ops.subs[g] * 19 * stride;
  const int n = i + LX * j + LX * LY * (top ? LZ - 1 : 0);
  int self;
  if (COMPACT) { self = fidx[n]; if (self < 0) return; }
  else { if (solids[n] == 1) return; self = n; }
  if (top) face_plane_node<T, COMPACT, true>(fs, solids, fidx, LX, LY, LZ, stride, second, ops, g, i, j, self);
  else face_plane_node<T, COMPACT, false>(fs, solids, fidx, LX, LY, LZ, stride, second, ops, g, i, j, self);
}

// ---- plane record ---------------------------------------------------------------
// The means over the plane's fluid nodes of the recorded C (channel 0, when
// the solute was active) and u_x (channel 1) into rec[2 * slot + channel]
// (skipping solid nodes of a dense plane), then the slot advances.  Each
// block sums a fixed chunk of the plane; the block that finishes last (a
// ticket taken with an atomic counter, no waiting) adds the block partials
// in block order, so the record is reproducible, and resets the counter for
// the next step.
constexpr int kBtcThreads = 256;
constexpr int kBtcMaxBlocks = 64;

static __global__ void __launch_bounds__(kBtcThreads)
btc_reduce(const double* vals, int count, const uint8_t* plane_solids, double fluid,
           int on_c, double* rec, int* slot, int capacity, double* part, unsigned* ticket)
{
  __shared__ double sh[2][kBtcThreads];
  __shared__ int last;
  const int per = (count + gridDim.x - 1) / gridDim.x;
  const int q0 = blockIdx.x * per;
  const int q1 = min(count, q0 + per);
  double sc = 0.0, su = 0.0;
  for (int q = q0 + threadIdx.x; q < q1; q += kBtcThreads)
    if (!plane_solids || plane_solids[q] != 1) {
      if (on_c) sc += vals[q];
      su += vals[count + q];
    }
  sh[0][threadIdx.x] = sc;
  sh[1][threadIdx.x] = su;
  __syncthreads();
  for (int w = kBtcThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      sh[0][threadIdx.x] += sh[0][threadIdx.x + w];
      sh[1][threadIdx.x] += sh[1][threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = sh[0][0];
    part[2 * blockIdx.x + 1] = sh[1][0];
    __threadfence();
    last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    double c = 0.0, u = 0.0;
    for (int b = 0; b < (int)gridDim.x; ++b) {
      c += __ldcg(part + 2 * b);
      u += __ldcg(part + 2 * b + 1);
    }
    const int k = *slot;
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    if (k < capacity) {
      rec[2 * k] = (on_c && fluid > 0.0) ? c / fluid : nan;
      rec[2 * k + 1] = fluid > 0.0 ? u / fluid : nan;
    }
    *slot = k + 1;
    *ticket = 0u;
  }
}

// ---- node classification ----------------------------------------------------
template <int Q>
__global__ void classify(const uint8_t* solids, uint8_t* cls, uint32_t* nbm,
                         int LX, int LY, int LZ)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= LX) return;
  const int j = blockIdx.y, k = blockIdx.z;
  const long long n = (long long)i + (long long)LX * (j + (long long)LY * k);
  if (solids[n] == 1) { cls[n] = CLS_SOLID; nbm[n] = 0; return; }
  uint32_t m = 0;
#pragma unroll
  for (int a = 1; a < Q; ++a) {
    int ii = i + cx(a), jj = j + cy(a), kk = k + cz(a);
    ii = ii < 0 ? ii + LX : (ii == LX ? 0 : ii);
    jj = jj < 0 ? jj + LY : (jj == LY ? 0 : jj);
    kk = kk < 0 ? kk + LZ : (kk == LZ ? 0 : kk);
    const long long nn = (long long)ii + (long long)LX * (jj + (long long)LY * kk);
    if (solids[nn] == 1) m |= 1u << a;
  }
  uint8_t c = m ? CLS_NEAR : 0;
  if (Q == 9) {
    if (j == LY - 1) c |= CLS_NORTH;
    if (j == 0) c |= CLS_SOUTH;
  }
  cls[n] = c;
  nbm[n] = m;
}

// ---- equilibrium initial state (src/latman.c:1786-1840) --------------------
template <typename T, int Q>
__global__ void init_feq(T* fs, const T* rho, const T* ux, const T* uy,
                         const T* uz, long long N, int shifted)
{
  const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const T r = rho[n], x = ux[n], y = uy[n], z = uz ? uz[n] : T(0);
  const T usq = add_(add_(mul_(x, x), mul_(y, y)), mul_(z, z));
#pragma unroll
  for (int a = 0; a < Q; ++a) {
    const T cu = T(cx(a)) * x + T(cy(a)) * y + T(cz(a)) * z;
    const T wr = mul_(wgt<T, Q>(a), r);
    const T q = add_(mul_(T(3), cu), mul_(mul_(T(4.5), cu), cu));   // 3 cu + 4.5 cu^2
    T v;
    if (a == 0) v = shifted ? mul_(wr, mul_(T(-1.5), usq)) : mul_(wr, sub_(T(1), mul_(T(1.5), usq)));
    else if (shifted) v = mul_(wr, sub_(q, mul_(T(1.5), usq)));
    else v = mul_(wr, sub_(add_(add_(T(1), mul_(T(3), cu)), mul_(mul_(T(4.5), cu), cu)),
                           mul_(T(1.5), usq)));
    fs[(long long)a * N + n] = v;
  }
}

// ---- FP64 reductions over macro variables -----------------------------------
struct RedPartial {
  double mass, solute, mom[3], usum[3], rmin, rmax;
  unsigned long long fluid, nonfinite;
};

template <typename T, int D>
__global__ void reduce_mv(const T* mv, const uint8_t* solids, long long N, int nsubs,
                          RedPartial* out)
{
  RedPartial r;
  r.mass = r.solute = 0; r.mom[0] = r.mom[1] = r.mom[2] = 0;
  r.usum[0] = r.usum[1] = r.usum[2] = 0;
  r.rmin = 1e300; r.rmax = -1e300; r.fluid = 0; r.nonfinite = 0;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < N;
       n += (long long)gridDim.x * blockDim.x) {
    if (solids[n] == 1) continue;
    const double rho = (double)mv[n];
    double u[3] = {(double)mv[N + n], (double)mv[2 * N + n],
                   D == 3 ? (double)mv[3 * N + n] : 0.0};
    if (!isfinite(rho) || !isfinite(u[0]) || !isfinite(u[1]) || !isfinite(u[2])) {
      r.nonfinite++;
      continue;
    }
    r.fluid++;
    r.mass += rho;
    r.rmin = fmin(r.rmin, rho);
    r.rmax = fmax(r.rmax, rho);
    for (int c = 0; c < 3; ++c) { r.mom[c] += rho * u[c]; r.usum[c] += u[c]; }
    if (nsubs == 2) r.solute += (double)mv[(long long)(1 + D) * N + n];
  }
  // warp then block reduction
  for (int off = 16; off > 0; off >>= 1) {
    r.mass += __shfl_down_sync(0xffffffffu, r.mass, off);
    r.solute += __shfl_down_sync(0xffffffffu, r.solute, off);
    for (int c = 0; c < 3; ++c) {
      r.mom[c] += __shfl_down_sync(0xffffffffu, r.mom[c], off);
      r.usum[c] += __shfl_down_sync(0xffffffffu, r.usum[c], off);
    }
    r.rmin = fmin(r.rmin, __shfl_down_sync(0xffffffffu, r.rmin, off));
    r.rmax = fmax(r.rmax, __shfl_down_sync(0xffffffffu, r.rmax, off));
    r.fluid += __shfl_down_sync(0xffffffffu, r.fluid, off);
    r.nonfinite += __shfl_down_sync(0xffffffffu, r.nonfinite, off);
  }
  __shared__ RedPartial sh[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sh[wid] = r;
  __syncthreads();
  if (threadIdx.x == 0) {
    RedPartial t = sh[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
      t.mass += sh[w].mass; t.solute += sh[w].solute;
      for (int c = 0; c < 3; ++c) { t.mom[c] += sh[w].mom[c]; t.usum[c] += sh[w].usum[c]; }
      t.rmin = fmin(t.rmin, sh[w].rmin); t.rmax = fmax(t.rmax, sh[w].rmax);
      t.fluid += sh[w].fluid; t.nonfinite += sh[w].nonfinite;
    }
    out[blockIdx.x] = t;
  }
}

}  // namespace lbx
