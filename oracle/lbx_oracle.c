/*
 * lbx_oracle.c -- CPU restatement of the reference's GPU lattice-Boltzmann
 * hot path.  TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py may call it, as the checker; the product
 * (liblbx) never links it and has no CPU fallback.
 *
 * What it restates (file:line in the reference tree):
 *   - odd AA step   src/k_stream_collide_stream.c:15-423
 *   - even AA step  src/k_collide.c:17-416
 *   - device helpers src/lattice.c:2660-2944 (pull/push with halfway
 *     bounce-back, BGK in shifted or plain form, body force)
 *   - Zou-He pressure faces   src/system_boundary_kernels.c:5-451
 *   - solute zero gradient    src/system_boundary_kernels.c:455-831
 *   - BC order + density schedule src/bcs.c:278-558, :1231-1506
 *   - per-step order          src/lbgpu_prime.cu:369-915
 *   - equilibrium init        src/latman.c:1786-1840
 *   - weights                 src/latman.c:161-192
 *   - Kahan density sums      src/lattice.c:3099-3114 (KAHAN_SUMMATION)
 *   - Walsh partial bounce-back src/k_stream_collide_stream.c:129-215,
 *     :363-386, src/lattice.c:2704, :2812, :2936 (WALSH_NS_ON)
 *   - 3D z faces: no reference device code; the 2D rules above carried to
 *     the planes k = 0 / k = LZ-1, Zou-He reconstruction as in the
 *     reference's CPU top/bottom code (src/bcs.c:596-870) -- parity unpinned
 * Semantics are those of a serial run: periodic wrap on every axis using the
 * true solid flag of the wrapped node; a node is solid iff its byte == 1
 * (src/lattice.c:2291, :2314).
 *
 * Parity: pinned against the reference's own kernel sources compiled for the
 * CPU (oracle/refk_harness.c); the FP64 restatement is bit-identical to them
 * on the pinned cases (tests/test_oracle_pin.py).
 *
 * Arithmetic follows the reference's operation order and its C literal types
 * (double literals promote float expressions in the FP32 build), so the FP32
 * restatement reproduces the reference FP32 build's mixed rounding.
 *
 * Threads: plain pthreads over node ranges (no OpenMP runtime needed).
 *
 * Compiled three times by oracle/Makefile into one .so: REAL = double,
 * float (-DLBX_ORACLE_F32), and double _Complex (-DLBX_ORACLE_CPLX) for
 * complex-step differentiation (Squire & Trapp, SIAM Review 40, 1998):
 * with tau, g and the inlet profile given imaginary parts i h v, every
 * result's imaginary part is h times its directional derivative along v,
 * exact to rounding because no difference of nearby values is taken.  That
 * forward-mode (tangent) derivative of the FP64 discrete model is the
 * independent check of the product's discrete adjoint.  The arithmetic here
 * is analytic in those parameters (sums, products and divisions; no branch
 * depends on a value), which the method needs.
 */
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "lbx_oracle.h"

#ifdef LBX_ORACLE_F32
#define REAL float
#define SFX(name) name##_f32
#elif defined(LBX_ORACLE_CPLX)
#define REAL double _Complex
#define SFX(name) name##_cs
#else
#define REAL double
#define SFX(name) name##_f64
#endif

typedef REAL real_t;

/* Plane-record sums: FP64 in the real builds; complex in the complex-step
 * build, whose imaginary parts carry the derivative. */
#ifdef LBX_ORACLE_CPLX
typedef double _Complex acc_t;
#define ACC(x) (x)
#else
typedef double acc_t;
#define ACC(x) ((double)(x))
#endif

/* Direction order of the reference (src/lbgpu_prime.h:82-84). */
static const int CX[19] = { 0, 1,-1, 0, 0, 1,-1,-1, 1, 0, 0, 1,-1,-1, 1, 0, 0, 0, 0};
static const int CY[19] = { 0, 0, 0, 1,-1, 1,-1, 1,-1, 0, 0, 0, 0, 0, 0, 1,-1,-1, 1};
static const int CZ[19] = { 0, 0, 0, 0, 0, 0, 0, 0, 0, 1,-1, 1,-1, 1,-1, 1,-1, 1,-1};
enum { DC = 0, DE, DW, DN, DS, DNE, DSW, DNW, DSE };

static inline int opp(int a) { return a == 0 ? 0 : ((a & 1) ? a + 1 : a - 1); }

typedef struct {
  const orc_params* p;
  int Q, D, NS;
  long NN;
  real_t w[19];
  real_t tau[2], inv_tau[2], rho_A[2], g[6], sink;
} ctx_t;

static void make_ctx(ctx_t* c, const orc_params* p)
{
  int a, s;
  c->p = p;
  c->D = p->dims;
  c->Q = p->dims == 2 ? 9 : 19;
  c->NS = p->nsubs;
  c->NN = (long)p->LX * p->LY * p->LZ;
  /* src/latman.c:161-192: weights are computed in `real`. */
  {
    real_t W0, W1, W2;
    if (c->D == 2) { W0 = 4./9.; W1 = 1./9.; W2 = 1./36.; }
    else           { W0 = 1./3.; W1 = 1./18.; W2 = 1./36.; }
    c->w[0] = W0;
    for (a = 1; a < 5; a++) c->w[a] = W1;
    for (; a < 9; a++) c->w[a] = W2;
    for (; a < 11; a++) c->w[a] = (c->D == 2) ? (real_t)0. : W1;
    for (; a < 19; a++) c->w[a] = (c->D == 2) ? (real_t)0. : W2;
  }
  for (s = 0; s < 2; s++) {
#ifdef LBX_ORACLE_CPLX
    c->tau[s] = p->tau[s] + I * p->d_tau[s];
    c->inv_tau[s] = 1. / c->tau[s];
#else
    c->tau[s] = (real_t)p->tau[s];
    c->inv_tau[s] = 1. / (real_t)p->tau[s];   /* src/latman.c:232-235 */
#endif
    c->rho_A[s] = (real_t)p->rho_A[s];
  }
#ifdef LBX_ORACLE_CPLX
  for (a = 0; a < 6; a++) c->g[a] = p->gaccel[a] + I * p->d_gaccel[a];
#else
  for (a = 0; a < 6; a++) c->g[a] = (real_t)p->gaccel[a];
#endif
  c->sink = (real_t)p->sink;
}

static inline long node_of(const orc_params* p, int i, int j, int k)
{ return (long)i + (long)p->LX * ((long)j + (long)p->LY * k); }

/* Periodic neighbour n + (dx,dy,dz): src/lattice.c:2692-2699 (serial). */
static inline long wrap_nbr(const orc_params* p, int i, int j, int k,
                            int dx, int dy, int dz)
{
  int ii = i + dx, jj = j + dy, kk = k + dz;
  if (ii < 0) ii += p->LX; if (ii == p->LX) ii = 0;
  if (jj < 0) jj += p->LY; if (jj == p->LY) jj = 0;
  if (kk < 0) kk += p->LZ; if (kk == p->LZ) kk = 0;
  return node_of(p, ii, jj, kk);
}

static inline int is_solid(const uint8_t* sol, long n) { return sol[n] == 1; }

/* ---- per-node collision, shared by both AA half-steps -------------------
 * d[0..Q-1] holds the node's (incoming) populations of substance `s`;
 * uvec carries the fluid velocity from substance 0 to the solute, as the
 * kernels' per-thread scratch does (src/k_stream_collide_stream.c:76-77).
 * `sinks` is how many times the solute sink applies: once on odd steps
 * (:254-256), twice on even steps (src/k_collide.c:96-97 and :261-262). */
static void collide_node(const ctx_t* c, int s, real_t* d, real_t* uvec,
                         int sinks, int write_mv, real_t* mv, long n)
{
  const orc_params* p = c->p;
  const int Q = c->Q, D = c->D;
  int a;
  const real_t ns = p->walsh ? (real_t)p->ns[n] : (real_t)0;
  real_t pre[19];
  real_t rho = d[0];
  if (p->walsh)
    for (a = 0; a < Q; a++) pre[a] = d[a];
  if (p->kahan && !(s == 1 && p->nsubs == 2)) {
    /* compensated sum of fk_add (src/lattice.c:3099-3114) */
    real_t correction = 0.0, next, sum;
    for (a = 1; a < Q; a++) {
      next = d[a] - correction;
      sum = rho + next;
      correction = (sum - rho) - next;
      rho = sum;
    }
  } else {
    for (a = 1; a < Q; a++) rho += d[a];
  }
  if (s == 1 && p->nsubs == 2) {
    /* solute: C = sum g; velocity is the fluid's */
    if (sinks == 2) rho *= (1.0 - c->sink * c->tau[1]);
  } else {
    real_t u[3] = {0, 0, 0};
    for (a = 0; a < Q; a++) {
      u[0] += ((real_t)CX[a]) * d[a];
      u[1] += ((real_t)CY[a]) * d[a];
      if (D == 3) u[2] += ((real_t)CZ[a]) * d[a];
    }
    for (a = 0; a < D; a++) {
      if (p->walsh) u[a] *= (1. - ns);
      if (p->compressible) {
        if (p->accurate) u[a] /= (c->rho_A[s] + rho);
        else u[a] /= rho;
      } else {
        u[a] /= c->rho_A[s];
      }
    }
    uvec[0] = u[0]; uvec[1] = u[1]; uvec[2] = u[2];
  }
  /* body force (src/lattice.c:2928-2944) or solute sink */
  if (s == 1 && p->nsubs == 2) {
    rho *= (1.0 - c->sink * c->tau[1]);
  } else if (p->walsh) {
    for (a = 0; a < D; a++) uvec[a] += (1. - ns) * c->tau[s] * c->g[s * 3 + a];
  } else {
    for (a = 0; a < D; a++) uvec[a] += c->tau[s] * c->g[s * 3 + a];
  }
  if (write_mv) {
    long NN = c->NN;
    real_t* m = mv + (long)s * (1 + D) * NN;
    if (p->accurate && !(s == 1 && p->nsubs == 2)) m[n] = rho + c->rho_A[s];
    else m[n] = rho;
    for (a = 0; a < D; a++) m[(long)(a + 1) * NN + n] = uvec[a];
  }
  /* BGK (src/lattice.c:2850-2924) */
  {
    real_t usq = 0;
    if (!(s == 1 && p->nsubs == 2)) {
      usq = uvec[0] * uvec[0] + uvec[1] * uvec[1];
      if (D == 3) usq += uvec[2] * uvec[2];
    }
    for (a = 0; a < Q; a++) {
      real_t cu = ((real_t)CX[a]) * uvec[0] + ((real_t)CY[a]) * uvec[1];
      if (D == 3) cu += ((real_t)CZ[a]) * uvec[2];
      d[a] *= (1. - c->inv_tau[s]);
      if (s == 1 && p->nsubs == 2) {
        d[a] += c->w[a] * rho * (1. + 3. * cu) * c->inv_tau[s];
      } else if (p->accurate) {
        d[a] += c->w[a] * rho * c->inv_tau[s];
        if (p->compressible)
          d[a] += c->w[a] * (c->rho_A[s] + rho)
                * (3. * cu + 4.5 * cu * cu - 1.5 * usq) * c->inv_tau[s];
        else
          d[a] += c->w[a] * (c->rho_A[s])
                * (3. * cu + 4.5 * cu * cu - 1.5 * usq) * c->inv_tau[s];
      } else {
        d[a] += c->w[a] * rho * c->inv_tau[s];
        d[a] += c->w[a] * rho
              * (3. * cu + 4.5 * cu * cu - 1.5 * usq) * c->inv_tau[s];
      }
    }
    /* Walsh: blend with the opposite pre-collision population */
    if (p->walsh)
      for (a = 0; a < Q; a++) {
        d[a] *= 1. - ns;
        d[a] += ns * pre[opp(a)];
      }
  }
}

static int solute_on(const orc_params* p, int t)
{ return t >= p->sigma_t_on && t <= p->sigma_t_off; }

/* Odd step: pull through bounce-back, collide, push to the neighbours'
 * opposite slots (src/k_stream_collide_stream.c:46-67, :401-423;
 * src/lattice.c:2730-2741 and :2835-2844). */
static void odd_range(const ctx_t* c, real_t* f, const uint8_t* sol,
                      real_t* mv, int t, int write_mv, long n0, long n1)
{
  const orc_params* p = c->p;
  const long NN = c->NN;
  const int Q = c->Q;
  long n;
  for (n = n0; n < n1; n++) {
    int i = (int)(n % p->LX), j = (int)((n / p->LX) % p->LY);
    int k = (int)(n / ((long)p->LX * p->LY));
    real_t d[19], uvec[3] = {0, 0, 0};
    long nb[19];
    int a, s;
    const int wl = p->walsh;
    if (!wl && is_solid(sol, n)) continue;
    for (a = 0; a < Q; a++) nb[a] = wrap_nbr(p, i, j, k, CX[a], CY[a], CZ[a]);
    for (s = 0; s < c->NS; s++) {
      real_t* fs = f + (long)s * Q * NN;
      if (s == 1 && !solute_on(p, t)) continue;
      for (a = 0; a < Q; a++) {
        long up = nb[opp(a)];                /* n - c_a */
        d[a] = (!wl && is_solid(sol, up)) ? fs[(long)opp(a) * NN + n]
                                          : fs[(long)a * NN + up];
      }
      collide_node(c, s, d, uvec, 1, write_mv, mv, n);
      for (a = 0; a < Q; a++) {
        long dn = nb[a];                     /* n + c_a */
        if (!wl && is_solid(sol, dn)) fs[(long)a * NN + n] = d[a];
        else fs[(long)opp(a) * NN + dn] = d[a];
      }
    }
  }
}

/* Even step: local, swapped load and natural-order store
 * (src/k_collide.c:53-77, :408-416). */
static void even_range(const ctx_t* c, real_t* f, const uint8_t* sol,
                       real_t* mv, int t, int write_mv, long n0, long n1)
{
  const long NN = c->NN;
  const int Q = c->Q;
  long n;
  for (n = n0; n < n1; n++) {
    real_t d[19], uvec[3] = {0, 0, 0};
    int a, s;
    if (!c->p->walsh && is_solid(sol, n)) continue;
    for (s = 0; s < c->NS; s++) {
      real_t* fs = f + (long)s * Q * NN;
      if (s == 1 && !solute_on(c->p, t)) continue;
      for (a = 0; a < Q; a++) d[a] = fs[(long)opp(a) * NN + n];
      collide_node(c, s, d, uvec, 2, write_mv, mv, n);
      for (a = 0; a < Q; a++) fs[(long)a * NN + n] = d[a];
    }
  }
}

/* ---- threads --------------------------------------------------------------
 * Both half-steps touch a disjoint slot set per node, so any split of the
 * node range over threads gives the sequential result. */
typedef struct {
  const ctx_t* c; real_t* f; const uint8_t* sol; real_t* mv;
  int t, write_mv, odd; long n0, n1;
} job_t;

static void* run_job(void* arg)
{
  job_t* j = (job_t*)arg;
  if (j->odd) odd_range(j->c, j->f, j->sol, j->mv, j->t, j->write_mv, j->n0, j->n1);
  else even_range(j->c, j->f, j->sol, j->mv, j->t, j->write_mv, j->n0, j->n1);
  return NULL;
}

static void half_step(const ctx_t* c, real_t* f, const uint8_t* sol,
                      real_t* mv, int t, int write_mv, int odd, int nthreads)
{
  job_t jobs[256];
  pthread_t th[256];
  int i, nt = nthreads < 1 ? 1 : (nthreads > 256 ? 256 : nthreads);
  long chunk = (c->NN + nt - 1) / nt;
  for (i = 0; i < nt; i++) {
    jobs[i].c = c; jobs[i].f = f; jobs[i].sol = sol; jobs[i].mv = mv;
    jobs[i].t = t; jobs[i].write_mv = write_mv; jobs[i].odd = odd;
    jobs[i].n0 = (long)i * chunk;
    jobs[i].n1 = jobs[i].n0 + chunk < c->NN ? jobs[i].n0 + chunk : c->NN;
  }
  if (nt == 1) { run_job(&jobs[0]); return; }
  for (i = 1; i < nt; i++) pthread_create(&th[i], NULL, run_job, &jobs[i]);
  run_job(&jobs[0]);
  for (i = 1; i < nt; i++) pthread_join(th[i], NULL);
}

/* ---- 2D system boundaries ------------------------------------------------
 * A face is the row j = LY-1 (north) or j = 0 (south).  The `_1` form runs
 * before the odd step on pulled values and deposits the unknowns where the
 * odd step will pull them from; the `_2` form runs before the even step on
 * the node's own swapped slots.  Both read the node's pulled/unswapped
 * populations exactly as the odd/even steps would. */
static void face_load(const ctx_t* c, const real_t* fs, const uint8_t* sol,
                      int second, int i, int j, real_t* d)
{
  const orc_params* p = c->p;
  const long NN = c->NN;
  long n = node_of(p, i, j, 0);
  int a;
  for (a = 0; a < 9; a++) {
    if (second) {
      d[a] = fs[(long)opp(a) * NN + n];
    } else {
      long up = wrap_nbr(p, i, j, 0, -CX[a], -CY[a], 0);
      d[a] = is_solid(sol, up) ? fs[(long)opp(a) * NN + n]
                               : fs[(long)a * NN + up];
    }
  }
}

/* Store value `v` for unknown direction `a` (an incoming direction of the
 * face).  `_1`: into slot a of the upstream node n - c_a, or of the node
 * itself when that node is solid (set_f1d_d with offset -c_a, da = 0).
 * `_2`: into the node's own slot opp(a), which the even step loads as d_a. */
static void face_store(const ctx_t* c, real_t* fs, const uint8_t* sol,
                       int second, int i, int j, int a, real_t v)
{
  const orc_params* p = c->p;
  const long NN = c->NN;
  long n = node_of(p, i, j, 0);
  if (second) {
    fs[(long)opp(a) * NN + n] = v;
  } else {
    long up = wrap_nbr(p, i, j, 0, -CX[a], -CY[a], 0);
    if (is_solid(sol, up)) fs[(long)a * NN + n] = v;
    else fs[(long)a * NN + up] = v;
  }
}

/* Zou-He pressure on the north face in shifted form
 * (src/system_boundary_kernels.c:58-83). */
static void zou_he_north(const ctx_t* c, real_t* fs, const uint8_t* sol,
                         int s, int second, real_t rho_bc)
{
  const orc_params* p = c->p;
  int i, j = p->LY - 1;
  for (i = 0; i < p->LX; i++) {
    real_t d[9], X, vS, vSW, vSE;
    if (is_solid(sol, node_of(p, i, j, 0))) continue;
    face_load(c, fs, sol, second, i, j, d);
    X = d[DC] + d[DE] + d[DW] + d[DN] + d[DN] + d[DNE] + d[DNE]
      + d[DNW] + d[DNW];
    X -= rho_bc;
    if (p->accurate) X += c->rho_A[s];
    vS = d[DN] - (2. / 3.) * X;
    vSW = d[DNE] + (1. / 2.) * (d[DE] - d[DW]) - (1. / 6.) * X;
    vSE = d[DNW] + (1. / 2.) * (d[DW] - d[DE]) - (1. / 6.) * X;
    face_store(c, fs, sol, second, i, j, DS, vS);
    face_store(c, fs, sol, second, i, j, DSE, vSE);
    face_store(c, fs, sol, second, i, j, DSW, vSW);
  }
}

/* Zou-He pressure on the south face (src/system_boundary_kernels.c:282-307). */
static void zou_he_south(const ctx_t* c, real_t* fs, const uint8_t* sol,
                         int s, int second, real_t rho_bc)
{
  const orc_params* p = c->p;
  int i, j = 0;
  for (i = 0; i < p->LX; i++) {
    real_t d[9], X, vN, vNE, vNW;
    if (is_solid(sol, node_of(p, i, j, 0))) continue;
    face_load(c, fs, sol, second, i, j, d);
    X = -d[DC] - d[DE] - d[DW] - d[DS] - d[DS] - d[DSE] - d[DSE]
      - d[DSW] - d[DSW];
    X += rho_bc;
    if (p->accurate) X -= c->rho_A[s];
    vN = d[DS] + (2. / 3.) * X;
    vNE = d[DSW] + (1. / 2.) * (d[DW] - d[DE]) + (1. / 6.) * X;
    vNW = d[DSE] + (1. / 2.) * (d[DE] - d[DW]) + (1. / 6.) * X;
    face_store(c, fs, sol, second, i, j, DN, vN);
    face_store(c, fs, sol, second, i, j, DNW, vNW);
    face_store(c, fs, sol, second, i, j, DNE, vNE);
  }
}

/* Solute zero-concentration-gradient faces
 * (src/system_boundary_kernels.c:503-521 north, :692-710 south). */
static void zero_grad(const ctx_t* c, real_t* fs, const uint8_t* sol,
                      int north, int second)
{
  const orc_params* p = c->p;
  int i, j = north ? p->LY - 1 : 0;
  for (i = 0; i < p->LX; i++) {
    real_t d[9], X;
    if (is_solid(sol, node_of(p, i, j, 0))) continue;
    face_load(c, fs, sol, second, i, j, d);
    if (north) {
      X = (d[DN] + d[DNE] + d[DNW]) / (c->w[DS] + c->w[DSW] + c->w[DSE]);
      face_store(c, fs, sol, second, i, j, DS, c->w[DS] * X);
      face_store(c, fs, sol, second, i, j, DSE, c->w[DSE] * X);
      face_store(c, fs, sol, second, i, j, DSW, c->w[DSW] * X);
    } else {
      X = (d[DS] + d[DSW] + d[DSE]) / (c->w[DN] + c->w[DNE] + c->w[DNW]);
      face_store(c, fs, sol, second, i, j, DN, c->w[DN] * X);
      face_store(c, fs, sol, second, i, j, DNW, c->w[DNW] * X);
      face_store(c, fs, sol, second, i, j, DNE, c->w[DNE] * X);
    }
  }
}

/* Face density at `time` (src/bcs.c:286-322 and the three siblings). */
static real_t face_rho(const ctx_t* c, int s, int t, int in_kind, int is_in,
                       const double* table, int len)
{
  const orc_params* p = c->p;
  real_t rho, ramp;
  if (is_in && in_kind == 2)
    rho = (real_t)p->pfadd + (real_t)p->pfmul * (real_t)table[t % len];
  else
    rho = is_in ? (real_t)p->rho_in : (real_t)p->rho_out;
  if (p->bc_ramp_start >= 0 && p->bc_ramp_stop >= 0) {
    if (t < p->bc_ramp_start) {
      rho = c->rho_A[s];
    } else if (t < p->bc_ramp_stop) {
      ramp = ((real_t)(t - p->bc_ramp_start))
           / ((real_t)(p->bc_ramp_stop - p->bc_ramp_start));
      rho *= ramp;
      rho += (1. - ramp) * c->rho_A[s];
    }
  }
  return rho;
}

static void apply_bcs(const ctx_t* c, real_t* f, const uint8_t* sol, int t,
                      int second)
{
  const orc_params* p = c->p;
  int s;
  for (s = 0; s < c->NS; s++) {
    real_t* fs = f + (long)s * c->Q * c->NN;
    if (p->pressure_n_in[s])
      zou_he_north(c, fs, sol, s, second,
                   face_rho(c, s, t, p->pressure_n_in[s], 1,
                            p->pressure_n_table, p->pressure_n_len));
    if (p->pressure_n_out[s])
      zou_he_north(c, fs, sol, s, second, face_rho(c, s, t, 0, 0, 0, 0));
    if (p->pressure_s_in[s])
      zou_he_south(c, fs, sol, s, second,
                   face_rho(c, s, t, p->pressure_s_in[s], 1,
                            p->pressure_s_table, p->pressure_s_len));
    if (p->pressure_s_out[s])
      zou_he_south(c, fs, sol, s, second, face_rho(c, s, t, 0, 0, 0, 0));
    if (s == 1 && p->nsubs == 2 && p->zeroconcgrad_n)
      zero_grad(c, fs, sol, 1, second);
    if (s == 1 && p->nsubs == 2 && p->zeroconcgrad_s)
      zero_grad(c, fs, sol, 0, second);
  }
}

/* ---- 3D z faces (parity unpinned) ------------------------------------------
 * top = plane k = LZ-1 (unknowns: the five cz = -1 directions), bottom =
 * plane k = 0 (unknowns: cz = +1).  Load/store follow face_load/face_store
 * above: `_1` pulls as the odd step and deposits upstream, `_2` works on the
 * node's own swapped slots. */
enum { DT = 9, DB, DTE, DBW, DTW, DBE, DTN, DBS, DTS, DBN };

static void face3_load(const ctx_t* c, const real_t* fs, const uint8_t* sol,
                       int second, int i, int j, int k, real_t* d)
{
  const orc_params* p = c->p;
  const long NN = c->NN;
  long n = node_of(p, i, j, k);
  int a;
  for (a = 0; a < 19; a++) {
    if (second) {
      d[a] = fs[(long)opp(a) * NN + n];
    } else {
      long up = wrap_nbr(p, i, j, k, -CX[a], -CY[a], -CZ[a]);
      d[a] = is_solid(sol, up) ? fs[(long)opp(a) * NN + n]
                               : fs[(long)a * NN + up];
    }
  }
}

static void face3_store(const ctx_t* c, real_t* fs, const uint8_t* sol,
                        int second, int i, int j, int k, int a, real_t v)
{
  const orc_params* p = c->p;
  const long NN = c->NN;
  long n = node_of(p, i, j, k);
  if (second) {
    fs[(long)opp(a) * NN + n] = v;
  } else {
    long up = wrap_nbr(p, i, j, k, -CX[a], -CY[a], -CZ[a]);
    if (is_solid(sol, up)) fs[(long)a * NN + n] = v;
    else fs[(long)a * NN + up] = v;
  }
}

/* Unknown directions of a face, and the known directions opposite them. */
static const int UNK_TOP[5] = {DB, DBW, DBE, DBS, DBN};
static const int UNK_BOT[5] = {DT, DTE, DTW, DTN, DTS};

/* Zou-He density (Hecht & Harting's D3Q19 form, zero tangential velocity):
 * J = rho u_z from the density balance, then
 *   bottom: d_T = d_B + J/3, d_TE = d_BW + J/6 - Nx, d_TW = d_BE + J/6 + Nx,
 *           d_TN = d_BS + J/6 - Ny, d_TS = d_BN + J/6 + Ny;
 *   top:    d_B = d_T - J/3, d_BW = d_TE - J/6 + Nx, d_BE = d_TW - J/6 - Nx,
 *           d_BS = d_TN - J/6 + Ny, d_BN = d_TS - J/6 - Ny;
 * with Nx, Ny half the in-plane x / y momentum.  In shifted form the rho_A
 * weights cancel from every difference, and the balance uses rho_bc - rho_A
 * (`drho`, formed in double). */
/* Velocity form (vel != 0, the reference's CPU rule, src/bcs.c:764-862):
 * rho = (S0 + 2 S_out + rA) / (1 + u) at the top, / (1 - u) at the bottom,
 * with the `1.` of the reference (a double in FP32 builds too), J = rho u;
 * rA = rho_A puts the shifted sums back to full densities (the rho_A
 * weights of the summed directions add to 1), 0 for unshifted populations. */
static void zou_he_3d(real_t* d, int top, real_t drho, int vel, real_t u, real_t rA)
{
  real_t S0 = d[DC] + d[DE] + d[DW] + d[DN] + d[DS] + d[DNE] + d[DSW] + d[DNW] + d[DSE];
  real_t Nx = 0.5 * ((d[DE] + d[DNE] + d[DSE]) - (d[DW] + d[DSW] + d[DNW]));
  real_t Ny = 0.5 * ((d[DN] + d[DNE] + d[DNW]) - (d[DS] + d[DSW] + d[DSE]));
  real_t J;
  if (top) {
    real_t Sp = d[DT] + d[DTE] + d[DTW] + d[DTN] + d[DTS];
    if (vel) {
      real_t rho = ((S0 + 2. * Sp) + rA) / (1. + u);
      J = rho * u;
    } else {
      J = (S0 + 2. * Sp) - drho;
    }
    d[DB] = d[DT] - J / 3.;
    d[DBW] = d[DTE] - J / 6. + Nx;
    d[DBE] = d[DTW] - J / 6. - Nx;
    d[DBS] = d[DTN] - J / 6. + Ny;
    d[DBN] = d[DTS] - J / 6. - Ny;
  } else {
    real_t Sm = d[DB] + d[DBW] + d[DBE] + d[DBS] + d[DBN];
    if (vel) {
      real_t rho = ((S0 + 2. * Sm) + rA) / (1. - u);
      J = rho * u;
    } else {
      J = drho - (S0 + 2. * Sm);
    }
    d[DT] = d[DB] + J / 3.;
    d[DTE] = d[DBW] + J / 6. - Nx;
    d[DTW] = d[DBE] + J / 6. + Nx;
    d[DTN] = d[DBS] + J / 6. - Ny;
    d[DTS] = d[DBN] + J / 6. + Ny;
  }
}

enum { F3_PRESSURE = 1, F3_ZEROGRAD = 2, F3_CONSTCON = 3, F3_VELOCITY = 4 };

/* drho: pressure faces' rho_bc - rA; for velocity faces the velocity u_z,
 * with conc carrying rA */
static void face3(const ctx_t* c, real_t* fs, const uint8_t* sol, int top,
                  int kind, int second, real_t drho, real_t conc,
                  const double* profile, const double* dprofile)
{
  const orc_params* p = c->p;
  const int k = top ? p->LZ - 1 : 0;
  const int* unk = top ? UNK_TOP : UNK_BOT;
  int i, j, q;
  for (j = 0; j < p->LY; j++)
    for (i = 0; i < p->LX; i++) {
      real_t d[19];
      if (is_solid(sol, node_of(p, i, j, k))) continue;
      face3_load(c, fs, sol, second, i, j, k, d);
      if (kind == F3_PRESSURE) {
        zou_he_3d(d, top, drho, 0, 0, 0);
      } else if (kind == F3_VELOCITY) {
        zou_he_3d(d, top, 0, 1, drho, conc);
      } else {
        /* unknowns set to w_a X: zero gradient takes X from the outgoing
         * populations opposite the unknowns (the 2D rule of
         * src/system_boundary_kernels.c:503-521), constant concentration
         * from C minus the known populations */
        real_t wsum = c->w[unk[0]] + c->w[unk[1]] + c->w[unk[2]] + c->w[unk[3]] + c->w[unk[4]];
        real_t X;
        if (kind == F3_ZEROGRAD) {
          X = (d[opp(unk[0])] + d[opp(unk[1])] + d[opp(unk[2])] + d[opp(unk[3])]
               + d[opp(unk[4])]) / wsum;
        } else {
          real_t known = 0;
          int a;
          for (a = 0; a < 19; a++)
            if (CZ[a] != (top ? -1 : 1)) known += d[a];
          real_t cin = conc;
          if (profile) cin = (real_t)profile[i + (long)p->LX * j];
#ifdef LBX_ORACLE_CPLX
          if (profile && dprofile) cin += I * dprofile[i + (long)p->LX * j];
#else
          (void)dprofile;
#endif
          X = (cin - known) / wsum;
        }
        for (q = 0; q < 5; q++) d[unk[q]] = c->w[unk[q]] * X;
      }
      for (q = 0; q < 5; q++) face3_store(c, fs, sol, second, i, j, k, unk[q], d[unk[q]]);
    }
}

/* Order: pressure t_in, t_out, b_in, b_out per substance (as n/s in 2D),
 * velocity t_in, t_out, b_in, b_out, then the solute's
 * constant-concentration and zero-gradient faces. */
static void apply_bcs3(const ctx_t* c, real_t* f, const uint8_t* sol, int t,
                       int second)
{
  const orc_params* p = c->p;
  int s;
  for (s = 0; s < c->NS; s++) {
    real_t* fs = f + (long)s * c->Q * c->NN;
    const int shifted = p->accurate && !(s == 1 && p->nsubs == 2);
    const double rA = shifted ? (double)c->rho_A[s] : 0.;
    if (p->pressure_t_in[s])
      face3(c, fs, sol, 1, F3_PRESSURE, second,
            (real_t)((double)face_rho(c, s, t, 1, 1, 0, 0) - rA), 0, 0, 0);
    if (p->pressure_t_out[s])
      face3(c, fs, sol, 1, F3_PRESSURE, second,
            (real_t)((double)face_rho(c, s, t, 0, 0, 0, 0) - rA), 0, 0, 0);
    if (p->pressure_b_in[s])
      face3(c, fs, sol, 0, F3_PRESSURE, second,
            (real_t)((double)face_rho(c, s, t, 1, 1, 0, 0) - rA), 0, 0, 0);
    if (p->pressure_b_out[s])
      face3(c, fs, sol, 0, F3_PRESSURE, second,
            (real_t)((double)face_rho(c, s, t, 0, 0, 0, 0) - rA), 0, 0, 0);
    if (p->velocity_t_in[s])
      face3(c, fs, sol, 1, F3_VELOCITY, second, (real_t)p->uz_in, (real_t)rA, 0, 0);
    if (p->velocity_t_out[s])
      face3(c, fs, sol, 1, F3_VELOCITY, second, (real_t)p->uz_out, (real_t)rA, 0, 0);
    if (p->velocity_b_in[s])
      face3(c, fs, sol, 0, F3_VELOCITY, second, (real_t)p->uz_in, (real_t)rA, 0, 0);
    if (p->velocity_b_out[s])
      face3(c, fs, sol, 0, F3_VELOCITY, second, (real_t)p->uz_out, (real_t)rA, 0, 0);
    if (s == 1 && p->nsubs == 2) {
      if (p->constcon_t_in)
        face3(c, fs, sol, 1, F3_CONSTCON, second, 0, (real_t)p->rho_sigma_in,
              p->constcon_profile_t, p->d_profile_t);
      if (p->constcon_b_in)
        face3(c, fs, sol, 0, F3_CONSTCON, second, 0, (real_t)p->rho_sigma_in,
              p->constcon_profile_b, p->d_profile_b);
      if (p->zeroconcgrad_t) face3(c, fs, sol, 1, F3_ZEROGRAD, second, 0, 0, 0, 0);
      if (p->zeroconcgrad_b) face3(c, fs, sol, 0, F3_ZEROGRAD, second, 0, 0, 0, 0);
    }
  }
}

/* t0 even: f in natural order; t0 odd: f as the odd step at t0 left it
 * (swapped slots), so a run may stop after any step and continue. */
int SFX(orc_run)(const orc_params* p, REAL* f, const uint8_t* solids,
                 REAL* mv, int t0, int nsteps, int frame_rate, int nthreads)
{
  ctx_t c;
  int t;
  if (t0 < 0 || p->LX < 1 || p->LY < 1 || p->LZ < 1) return -1;
  if (p->dims == 2 && p->LZ != 1) return -1;
  make_ctx(&c, p);
  for (t = t0 + 1; t <= t0 + nsteps; t++) {
    int wmv = frame_rate > 0 && t % frame_rate == 0;
    int odd = (t % 2) == 1;
    if (p->dims == 2) apply_bcs(&c, f, solids, t, !odd);
    else apply_bcs3(&c, f, solids, t, !odd);
    half_step(&c, f, solids, mv, t, wmv, odd, nthreads);
  }
  return 0;
}

/* orc_run plus a plane record: btc[i] = mean over the fluid nodes of the
 * plane k = `plane` (3D) or row j = `plane` (2D) of the solute concentration
 * C computed by the step at time t0+1+i (FP64 sum in node order; NaN for
 * steps with no active solute), btc_ux[i] the same mean of the flow u_x. */
int SFX(orc_run_btc)(const orc_params* p, REAL* f, const uint8_t* solids,
                     REAL* mv, int t0, int nsteps, int frame_rate, int nthreads,
                     int plane, double* btc, double* btc_ux)
{
  ctx_t c;
  int t;
  long per, base, q, cnt = 0;
  REAL* scratch;
  if (t0 % 2 != 0 || p->LX < 1 || p->LY < 1 || p->LZ < 1) return -1;
  if (p->dims == 2 && p->LZ != 1) return -1;
  if (plane < 0 || plane >= (p->dims == 2 ? p->LY : p->LZ)) return -1;
  make_ctx(&c, p);
  per = p->dims == 2 ? (long)p->LX : (long)p->LX * p->LY;
  base = per * plane;
  for (q = 0; q < per; q++) cnt += !is_solid(solids, base + q);
  scratch = (REAL*)malloc(sizeof(REAL) * (size_t)p->nsubs * (1 + c.D) * c.NN);
  if (!scratch) return -2;
  for (t = t0 + 1; t <= t0 + nsteps; t++) {
    int wmv = frame_rate > 0 && t % frame_rate == 0;
    int odd = (t % 2) == 1;
    REAL* m = wmv ? mv : scratch;
    acc_t sc = 0, su = 0;
    if (p->dims == 2) apply_bcs(&c, f, solids, t, !odd);
    else apply_bcs3(&c, f, solids, t, !odd);
    half_step(&c, f, solids, m, t, 1, odd, nthreads);
    for (q = 0; q < per; q++)
      if (!is_solid(solids, base + q)) {
        su += ACC(m[c.NN + base + q]);                      /* subs 0, u_x */
        if (p->nsubs == 2) sc += ACC(m[(long)(1 + c.D) * c.NN + base + q]);
      }
    {
      const acc_t ux = cnt ? su / (double)cnt : 0. / 0.;
      const acc_t cc = (p->nsubs == 2 && t >= p->sigma_t_on && t <= p->sigma_t_off && cnt)
                           ? sc / (double)cnt : 0. / 0.;
#ifdef LBX_ORACLE_CPLX
      btc_ux[2 * (t - t0 - 1)] = creal(ux); btc_ux[2 * (t - t0 - 1) + 1] = cimag(ux);
      btc[2 * (t - t0 - 1)] = creal(cc); btc[2 * (t - t0 - 1) + 1] = cimag(cc);
#else
      btc_ux[t - t0 - 1] = ux;
      btc[t - t0 - 1] = cc;
#endif
    }
  }
  free(scratch);
  return 0;
}

/* Equilibrium initial state (src/latman.c:1786-1840): shifted deviations
 * d_a = w_a rho (3 c.u + 4.5 (c.u)^2 - 1.5 u^2) for the flow lattice of an
 * ACCURATE build, full feq for the solute and for plain builds.  All nodes,
 * solid ones included.  rho/u are [NumSubs][N]. */
int SFX(orc_init_feq)(const orc_params* p, const REAL* rho, const REAL* ux,
                      const REAL* uy, const REAL* uz, REAL* f)
{
  ctx_t c;
  long n;
  int s;
  make_ctx(&c, p);
  for (s = 0; s < c.NS; s++) {
    int shifted = p->accurate && (s == 0);
    real_t W[19];
    int a;
    for (a = 0; a < c.Q; a++) W[a] = c.w[a];
    for (n = 0; n < c.NN; n++) {
      real_t r = rho[(long)s * c.NN + n];
      real_t x = ux[(long)s * c.NN + n], y = uy[(long)s * c.NN + n];
      real_t z = uz ? uz[(long)s * c.NN + n] : 0;
      real_t usq = x * x + y * y + z * z;
      for (a = 0; a < c.Q; a++) {
        real_t cu = (real_t)CX[a] * x + (real_t)CY[a] * y + (real_t)CZ[a] * z;
        real_t v;
        if (a == 0)
          v = shifted ? W[0] * r * (-1.5 * usq) : W[0] * r * (1. - 1.5 * usq);
        else if (shifted)
          v = W[a] * r * (3. * cu + 4.5 * cu * cu - 1.5 * usq);
        else
          v = W[a] * r * (1. + 3. * cu + 4.5 * cu * cu - 1.5 * usq);
        f[((long)s * c.Q + a) * c.NN + n] = v;
      }
    }
  }
  return 0;
}
