/*
 * refk_harness.c -- runs the reference's own CUDA kernel sources on the CPU.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker's checker: it pins the
 * C restatement in oracle/lbx_oracle.c against the reference's own kernel
 * code.  Nothing in the product path links or calls it.
 *
 * Built by oracle/ref_build.py, which force-includes a variant of the
 * reference's src/flags.h and puts the reference's src/ on the include path.
 * The reference files are compiled where they lie; nothing is copied.
 *
 * How a launch is emulated: every kernel is launched with one-thread blocks
 * (BX=BY=BZ=1), so the per-thread shared-memory scratch `fptr` is one
 * (Q+D+1)-entry array, and the grid is walked block by block.  The reference
 * kernels are data-parallel with a disjoint read/write slot set per node
 * (src/k_stream_collide_stream.c:46-67 pulls and :401-423 pushes the same
 * slots; src/k_collide.c:53-77 and :408-416 touch only the node's own slots),
 * so the sequential walk computes what the GPU launch computes.
 *
 * The host orchestration that cannot be compiled here (src/bcs.c uses <<<>>>
 * launch syntax; src/lbgpu_prime.cu is the CUDA main) is restated below with
 * file:line citations: the per-step order of src/lbgpu_prime.cu:369-915 and
 * the density schedule of src/bcs.c:278-558 / :1231-1506.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <assert.h>
#include <time.h>
#include <pthread.h>

#ifndef CLK_TCK
#define CLK_TCK CLOCKS_PER_SEC   /* as src/lbgpu_prime.h:18-21 */
#endif

#if DP_ON
typedef double real;
#else
typedef float real;
#endif

/* CUDA keywords and built-ins for a host build. */
#define __global__
#define __device__
#define __constant__
#define __shared__ __thread   /* only `extern __shared__ real fptr[]` uses it */
#define __CUDACC__ 1
#define __CUDA_ARCH__ 1000
typedef struct { unsigned int x, y, z; } refk_dim3;
/* Thread-local, so host threads can each walk a part of the grid. */
static __thread refk_dim3 threadIdx, blockIdx, blockDim;

/* CUDA runtime names referenced by host code in src/lattice.c (never run). */
typedef int cudaError_t;
#define cudaSuccess 0
enum { cudaMemcpyHostToDevice = 1, cudaMemcpyDeviceToHost = 2,
       cudaMemcpyDeviceToDevice = 3 };
static int cudaGetLastError(void) { return 0; }
static const char* cudaGetErrorString(int e) { (void)e; return ""; }
static int cudaThreadSynchronize(void) { return 0; }
static int cudaMemcpy(void* d, const void* s, size_t n, int k)
{ (void)k; memcpy(d, s, n); return 0; }

/* Velocity table in the reference's order (src/lbgpu_prime.h:82-84):
   opposite directions adjacent (a odd <-> a+1), D2Q9 = the first nine. */
int vx[19] = { 0, 1,-1, 0, 0, 1,-1,-1, 1, 0, 0, 1,-1,-1, 1, 0, 0, 0, 0};
int vy[19] = { 0, 0, 0, 1,-1, 1,-1, 1,-1, 0, 0, 0, 0, 0, 0, 1,-1,-1, 1};
int vz[19] = { 0, 0, 0, 0, 0, 0, 0, 0, 0, 1,-1, 1,-1, 1,-1, 1,-1, 1,-1};
real wt[19];
int cumul_stride[20];
/* Direction names used by the boundary kernels (src/lbgpu_prime.h:91-109). */
#define C  0
#define E  1
#define W  2
#define N  3
#define S  4
#define NE 5
#define SW 6
#define NW 7
#define SE 8
#define T  9
#define B  10
#define TE 11
#define BW 12
#define TW 13
#define BE 14
#define TN 15
#define BS 16
#define TS 17
#define BN 18

#include "process.h"
#include "lattice.h"
#include "forward_declarations.h"
#include "lattice.c"
#include "params.h"
#include "process.c"
#include "lbio.c"
#include "compute.c"
/* init_problem and the PEST point sampling live in src/latman.c, whose
 * other functions set up the device; their CUDA calls compile to no-ops here
 * (never run), and a copy to a __constant__ symbol becomes a copy to the host
 * global. */
#define cudaMalloc(p, n) 0
#define cudaFree(p) 0
#define cudaFreeHost(p) 0
#define cudaMemcpyToSymbol(sym, src, n, ...) (memcpy(&(sym), (src), (n)), 0)
#define cudaMemcpyFromSymbol(dst, sym, n, ...) (memcpy((dst), &(sym), (n)), 0)
/* globals of src/lbgpu_prime.cu:17-24 that src/latman.c names */
int f_mem_size, mv_mem_size, solids_mem_size;
real *f_mem_d, *mv_mem_d, *ns_mem_d;
unsigned char* solids_mem_d;
#include "latman.c"
#include "system_boundary_kernels.c"
#include "k_stream_collide_stream.c"
#include "k_collide.c"
/* the reference's own CPU loops (its host-only build), timed as a cost
 * baseline; src/stream_collide_stream.c:2-240, src/collide.c:9-251 */
#include "stream_collide_stream.c"
#include "collide.c"

/* The dynamic shared-memory scratch of one one-thread block (per host
   thread). */
__thread real fptr[32];

#define EXPORT __attribute__((visibility("default")))

typedef struct {
  int LX, LY, LZ;
  double tau[2], rho_A[2], gaccel[6], sink;
  int sigma_t_on, sigma_t_off;
  /* 2D system boundaries (src/bcs.c GPU branches) */
  int pressure_n_in[2], pressure_s_in[2], pressure_n_out[2], pressure_s_out[2];
  int zeroconcgrad_n, zeroconcgrad_s;
  double rho_in, rho_out, pfadd, pfmul;
  int bc_ramp_start, bc_ramp_stop;
  const double* pressure_n_table; int pressure_n_len;   /* subs 0 */
  const double* pressure_s_table; int pressure_s_len;
} refk_params;

EXPORT int refk_real_size(void) { return (int)sizeof(real); }
EXPORT int refk_num_dims(void) { return NUM_DIMENSIONS; }
EXPORT int refk_num_subs(void) { return NUM_FLUID_COMPONENTS; }
EXPORT int refk_accurate(void) { return ACCURATE; }
EXPORT int refk_compressible(void) { return COMPRESSIBLE; }

/* Constant upload, as construct_lattice does it (src/latman.c:147-376) for
   a serial run: EndBoundSize = 0, so cumul_stride[a] = a*NumNodes. */
static void upload_constants(const refk_params* p)
{
  int a, s;
  int D = NUM_DIMENSIONS, Qd = 2 * D * D + 1, NS = NUM_FLUID_COMPONENTS;
  int NN = p->LX * p->LY * p->LZ;
  memcpy(vx_c, vx, sizeof vx); memcpy(vy_c, vy, sizeof vy);
  memcpy(vz_c, vz, sizeof vz);
  if (D == 2) {
    real W0 = 4./9., W1 = 1./9., W2 = 1./36.;
    wt[0] = W0;
    for (a = 1; a < 5; a++) wt[a] = W1;
    for (; a < 9; a++) wt[a] = W2;
    for (; a < 19; a++) wt[a] = 0.;
  } else {
    real W0 = 1./3., W1 = 1./18., W2 = 1./36.;
    wt[0] = W0;
    for (a = 1; a < 5; a++) wt[a] = W1;
    for (; a < 9; a++) wt[a] = W2;
    for (; a < 11; a++) wt[a] = W1;
    for (; a < 19; a++) wt[a] = W2;
  }
  for (a = 0; a <= Qd; a++) cumul_stride[a] = a * NN;
  memcpy(wt_c, wt, sizeof wt);
  memcpy(cumul_stride_c, cumul_stride, sizeof cumul_stride);
  for (s = 0; s < NS; s++) {
    tau_c[s] = (real)p->tau[s];
    inv_tau_c[s] = 1. / (real)p->tau[s];     /* src/latman.c:232-235 */
    rho_A_c[s] = (real)p->rho_A[s];
    for (a = 0; a < D; a++) gaccel_c[s * 3 + a] = (real)p->gaccel[s * 3 + a];
  }
  numsubs_c = NS; numdims_c = D; numdirs_c = Qd;
  numbounddirs_c = (D == 2) ? 6 : 10; numunbounddirs_c = Qd - numbounddirs_c;
  end_bound_c = 0; proc_id_c = 0; num_procs_c = 1;
  ni_c = p->LX; nj_c = p->LY; nk_c = p->LZ;
  kloop_c = 1; bixbj_c = 1; bixbk_c = 1; bjxbk_c = 1;
  nixnj_c = p->LX * p->LY; blocksize_c = 1; numnodes_c = NN;
  sink_c = (real)p->sink; pfmul_c = (real)p->pfmul; pfadd_c = (real)p->pfadd;
#if INAMURO_SIGMA_COMPONENT
  sigma_t_on_c = p->sigma_t_on; sigma_t_off_c = p->sigma_t_off;
#endif
  is_end_of_frame_mem_c = 0; pest_output_flag_c = 0;
}

typedef void (*refk_kernel)(real*, real*, unsigned char*, real*);
typedef void (*refk_bc_kernel)(real*, unsigned char*, real*);

typedef struct {
  refk_kernel k; int gx, gy, z0, z1; real* f; real* mv; unsigned char* sol;
} grid_job;

/* The per-node Walsh fraction n_s handed to the kernels as ns_mem_d
 * (WALSH_NS_ON builds; NULL otherwise, as the other builds never read it). */
static real* g_ns = NULL;

static void* grid_worker(void* arg)
{
  grid_job* g = (grid_job*)arg;
  unsigned x, y, z;
  blockDim.x = blockDim.y = blockDim.z = 1;
  threadIdx.x = threadIdx.y = threadIdx.z = 0;
  for (z = (unsigned)g->z0; z < (unsigned)g->z1; z++)
    for (y = 0; y < (unsigned)g->gy; y++)
      for (x = 0; x < (unsigned)g->gx; x++) {
        blockIdx.x = x; blockIdx.y = y; blockIdx.z = z;
        g->k(g->f, g->mv, g->sol, g_ns);
      }
  return NULL;
}

static void* grid_worker_rows(void* arg)
{
  grid_job* g = (grid_job*)arg;
  unsigned x, y;
  blockDim.x = blockDim.y = blockDim.z = 1;
  threadIdx.x = threadIdx.y = threadIdx.z = 0;
  blockIdx.z = 0;
  for (y = 0; y < (unsigned)g->gy; y++)
    for (x = 0; x < (unsigned)g->gx; x++) {
      blockIdx.x = x; blockIdx.y = (unsigned)g->z0 + y;
      g->k(g->f, g->mv, g->sol, g_ns);
    }
  return NULL;
}

static int g_threads = 1;
EXPORT void refk_set_threads(int n) { g_threads = n < 1 ? 1 : (n > 256 ? 256 : n); }

/* Walk the grid, split into slabs of z-planes (or y-rows in 2D) over
   g_threads host threads; the per-node slot sets are disjoint. */
static void launch_grid(refk_kernel k, int gx, int gy, int gz,
                        real* f, real* mv, unsigned char* sol)
{
  grid_job jobs[256];
  pthread_t th[256];
  int nt = g_threads, t;
  int split_y = (gz == 1);
  int extent = split_y ? gy : gz;
  if (nt > extent) nt = extent;
  for (t = 0; t < nt; t++) {
    int a = (int)((long)extent * t / nt), b = (int)((long)extent * (t + 1) / nt);
    jobs[t].k = k; jobs[t].f = f; jobs[t].mv = mv; jobs[t].sol = sol;
    jobs[t].gx = gx;
    if (split_y) { jobs[t].gy = b - a; jobs[t].z0 = 0; jobs[t].z1 = 1; }
    else { jobs[t].gy = gy; jobs[t].z0 = a; jobs[t].z1 = b; }
  }
  if (split_y) {
    /* rows: run a y-offset grid by shifting blockIdx.y inside the worker */
    for (t = 0; t < nt; t++) jobs[t].z0 = (int)((long)extent * t / nt);
  }
  if (nt == 1 && !split_y) { grid_worker(&jobs[0]); return; }
  for (t = 0; t < nt; t++)
    pthread_create(&th[t], NULL, split_y ? grid_worker_rows : grid_worker, &jobs[t]);
  for (t = 0; t < nt; t++) pthread_join(th[t], NULL);
}

static void launch_row(refk_bc_kernel k, int gx, real* f, unsigned char* sol)
{
  unsigned x;
  blockDim.x = blockDim.y = blockDim.z = 1;
  threadIdx.x = threadIdx.y = threadIdx.z = 0;
  blockIdx.y = blockIdx.z = 0;
  for (x = 0; x < (unsigned)gx; x++) { blockIdx.x = x; k(f, sol, NULL); }
}

/* Density for one pressure face at `time`: src/bcs.c:286-322 (north in),
   :345-371 (north out), :396-431 (south in), :458-484 (south out). */
static real face_rho(const refk_params* p, int subs, int time, int in_flag,
                     int is_in, const double* table, int len)
{
  real rho, ramp_factor;
  if (is_in && in_flag == 2)
    rho = (real)p->pfadd + (real)p->pfmul * (real)table[time % len];
  else
    rho = is_in ? (real)p->rho_in : (real)p->rho_out;
  if (p->bc_ramp_start >= 0 && p->bc_ramp_stop >= 0) {
    if (time < p->bc_ramp_start) {
      rho = (real)p->rho_A[subs];
    } else if (time < p->bc_ramp_stop) {
      ramp_factor = ((real)(time - p->bc_ramp_start))
                  / ((real)(p->bc_ramp_stop - p->bc_ramp_start));
      rho *= ramp_factor;
      rho += (1. - ramp_factor) * (real)p->rho_A[subs];
    }
  }
  return rho;
}

/* bcs_1 / bcs_2 (src/bcs.c:226-558, :1179-1506): per substance, north in,
   north out, south in, south out, then (solute only) zero-gradient N, S. */
static void bcs(const refk_params* p, int time, int second,
                real* f, unsigned char* sol)
{
  int subs;
  refk_bc_kernel pn = second ? k_sysbound_pressure_n_2 : k_sysbound_pressure_n_1;
  refk_bc_kernel ps = second ? k_sysbound_pressure_s_2 : k_sysbound_pressure_s_1;
  for (subs = 0; subs < NUM_FLUID_COMPONENTS; subs++) {
    subs_c = subs;
    if (p->pressure_n_in[subs]) {
      fixed_bound_var_c = face_rho(p, subs, time, p->pressure_n_in[subs], 1,
                                   p->pressure_n_table, p->pressure_n_len);
      launch_row(pn, p->LX, f, sol);
    }
    if (p->pressure_n_out[subs]) {
      fixed_bound_var_c = face_rho(p, subs, time, 0, 0, NULL, 0);
      launch_row(pn, p->LX, f, sol);
    }
    if (p->pressure_s_in[subs]) {
      fixed_bound_var_c = face_rho(p, subs, time, p->pressure_s_in[subs], 1,
                                   p->pressure_s_table, p->pressure_s_len);
      launch_row(ps, p->LX, f, sol);
    }
    if (p->pressure_s_out[subs]) {
      fixed_bound_var_c = face_rho(p, subs, time, 0, 0, NULL, 0);
      launch_row(ps, p->LX, f, sol);
    }
#if INAMURO_SIGMA_COMPONENT
    if (subs == 1 && p->zeroconcgrad_n)
      launch_row(second ? k_sysbound_zeroconcgrad_n_2
                        : k_sysbound_zeroconcgrad_n_1, p->LX, f, sol);
    if (subs == 1 && p->zeroconcgrad_s)
      launch_row(second ? k_sysbound_zeroconcgrad_s_2
                        : k_sysbound_zeroconcgrad_s_1, p->LX, f, sol);
#endif
  }
}

/*
 * Run lattice times t0+1 .. t0+nsteps (t0 even: an AA pair starts on an odd
 * time).  f is [NumSubs][Q][N] in the reference's serial layout, mv is
 * [NumSubs][1+D][N].  mv is written at the steps where t % frame_rate == 0
 * (frame_rate <= 0: never), exactly as is_end_of_frame_mem_c gates it.
 * Per step, src/lbgpu_prime.cu:369-915: set time_c; 2D only: bcs_1 (odd) or
 * bcs_2 (even); then k_stream_collide_stream (odd) or k_collide (even).
 */
/* Walsh builds: the per-node n_s (N reals, kept by the caller). */
EXPORT void refk_set_ns(real* ns) { g_ns = ns; }

EXPORT int refk_walsh(void) { return WALSH_NS_ON ? 1 : 0; }

#if PEST_OUTPUT_ON
/* The lattice of an open PEST sampling (refk_pest_begin .. refk_pest_end). */
static struct lattice_struct* g_pest;
#endif

EXPORT int refk_run(const refk_params* p, real* f, const unsigned char* solids,
                    real* mv, int t0, int nsteps, int frame_rate)
{
  int t;
  unsigned char* sol = (unsigned char*)solids;
  if (t0 % 2) return -1;
  upload_constants(p);
  for (t = t0 + 1; t <= t0 + nsteps; t++) {
#if INAMURO_SIGMA_COMPONENT
    time_c = t;
#endif
#if PEST_OUTPUT_ON
    /* before and after each kernel, src/lbgpu_prime.cu:515, :532, :739, :754 */
    if (g_pest) { g_pest->time = t; PEST_gpu_switch(&g_pest, mv, 0, NULL); }
#endif
    if (NUM_DIMENSIONS == 2) bcs(p, t, !(t % 2 == 1), f, sol);
    is_end_of_frame_mem_c = (frame_rate > 0 && t % frame_rate == 0);
    if (t % 2 == 1)
      launch_grid(k_stream_collide_stream, p->LX, p->LY, p->LZ, f, mv, sol);
    else
      launch_grid(k_collide, p->LX, p->LY, p->LZ, f, mv, sol);
    is_end_of_frame_mem_c = 0;
#if PEST_OUTPUT_ON
    if (g_pest) write_PEST_out_data(&g_pest, mv, 0, NULL);
#endif
  }
  return 0;
}

EXPORT int refk_pest(void) { return PEST_OUTPUT_ON ? 1 : 0; }

#if PEST_OUTPUT_ON
/* read_PEST_in_files (src/latman.c:899-1046) on ./in of the current
 * directory, for a lattice of the given extents whose macro variables the
 * sampling copies into; refk_run then samples as the reference's main does,
 * and refk_pest_end writes ./out/{conc_data,vel_data,conc_order}_proc0000.dat
 * (write_PEST_out_file, src/latman.c:1178-1232).  One entry past the kept
 * samples is set to time -1: the reference's sampling loop reads the entry
 * after the last kept sample, which holds stale data there.  Returns the
 * number of kept samples, or -1 when an input file is missing. */
EXPORT int refk_pest_begin(int LX, int LY, int LZ)
{
  struct lattice_struct* l = (struct lattice_struct*)calloc(1, sizeof *l);
  int s, c;
  const int D = NUM_DIMENSIONS, NN = LX * LY * LZ;
  l->param.LX = LX; l->param.LY = LY; l->param.LZ = LZ;
  l->NumNodes = NN;
  l->NumDims = D;
  l->NumSubs = NUM_FLUID_COMPONENTS;
  l->process.id = 0; l->process.num_procs = 1;
  l->vars = (struct vars_struct*)calloc(NUM_FLUID_COMPONENTS, sizeof *l->vars);
  for (s = 0; s < NUM_FLUID_COMPONENTS; s++) {
    l->vars[s].macrovars_memblock = (real*)calloc((size_t)NN * (1 + D), sizeof(real));
    l->vars[s].macrovars1d = (real**)malloc((1 + D) * sizeof(real*));
    for (c = 0; c <= D; c++) l->vars[s].macrovars1d[c] = l->vars[s].macrovars_memblock + (size_t)c * NN;
  }
  read_PEST_in_files(&l, 0, NULL);
  if (!l->concentration_data) return -1;
  l->concentration_data = (struct conc_data_struct*)realloc(
      l->concentration_data, (size_t)(l->conc_array_size + 1) * sizeof *l->concentration_data);
  memset(&l->concentration_data[l->conc_array_size], 0, sizeof *l->concentration_data);
  l->concentration_data[l->conc_array_size].timestep = -1;
  g_pest = l;
  return l->conc_array_size;
}

/* The kept samples of the open sampling: original index, time, x, y. */
EXPORT int refk_pest_samples(int* order, int* time, int* x, int* y)
{
  int k;
  if (!g_pest) return -1;
  for (k = 0; k < g_pest->conc_array_size; k++) {
    order[k] = g_pest->concentration_data[k].countervar;
    time[k] = g_pest->concentration_data[k].timestep;
    x[k] = g_pest->concentration_data[k].x_coord;
    y[k] = g_pest->concentration_data[k].y_coord;
  }
  return g_pest->conc_array_size;
}

EXPORT int refk_pest_end(void)
{
  struct lattice_struct* l = g_pest;
  int s;
  if (!l) return -1;
  write_PEST_out_file(&l, 0, NULL);
  for (s = 0; s < NUM_FLUID_COMPONENTS; s++) {
    free(l->vars[s].macrovars1d);
    free(l->vars[s].macrovars_memblock);
  }
  free(l->vars);
  free(l->concentration_data);
  free(l);
  g_pest = NULL;
  return 0;
}
#endif

/* ---- host-side input readers of the reference ------------------------------
 * read_params (src/params.h:40-660), spy_bmp (src/lbio.c:3073-3363) and
 * read_solids (src/lbio.c:507-629), run on a lattice struct the harness
 * fills itself (in a serial build the global extents they use are the
 * local ones, src/process.c:2115-2126). */
static struct lattice_struct* harness_lattice(int LX, int LY, int LZ)
{
  struct lattice_struct* l = (struct lattice_struct*)calloc(1, sizeof *l);
  l->param.LX = LX; l->param.LY = LY; l->param.LZ = LZ;
  l->NumNodes = LX * LY * LZ;
  l->process.id = 0; l->process.num_procs = 1;
  l->solids_memblock = (unsigned char*)calloc((size_t)(LX * LY * LZ), 1);
  return l;
}

/* out[0..9] = LX LY LZ NumFrames FrameRate initial_condition
 *             bc_ramp_start bc_ramp_stop pressure_n_in[0] pressure_s_in[0]
 * dout[0..7] = tau[0] rho_A[0] rho_B[0] rho_in rho_out sink gforce[0][0] pfmul */
EXPORT int refk_read_params(const char* path, int* iout, double* dout)
{
  struct lattice_struct* l = harness_lattice(1, 1, 1);
  read_params(l, path);
  iout[0] = l->param.LX; iout[1] = l->param.LY; iout[2] = l->param.LZ;
  iout[3] = l->param.NumFrames; iout[4] = l->param.FrameRate;
  iout[5] = l->param.initial_condition; iout[6] = l->param.bc_ramp_start;
  iout[7] = l->param.bc_ramp_stop; iout[8] = l->param.pressure_n_in[0];
  iout[9] = l->param.pressure_s_in[0];
  dout[0] = l->param.tau[0]; dout[1] = l->param.rho_A[0]; dout[2] = l->param.rho_B[0];
  dout[3] = l->param.rho_in; dout[4] = l->param.rho_out; dout[5] = l->param.sink;
  dout[6] = l->param.gforce[0][0]; dout[7] = l->param.pfmul;
  free(l->solids_memblock); free(l);
  return 0;
}

EXPORT int refk_read_bmp(const char* path, int LX, int LY, unsigned char* out)
{
  struct lattice_struct* l = harness_lattice(LX, LY, 1);
  int j, i;
  int** matrix = (int**)malloc((size_t)LY * sizeof(int*));
  for (j = 0; j < LY; j++) matrix[j] = (int*)calloc((size_t)LX, sizeof(int));
  spy_bmp(l, (char*)path, matrix);
  for (j = 0; j < LY; j++)
    for (i = 0; i < LX; i++) out[j * LX + i] = (unsigned char)matrix[j][i];
  for (j = 0; j < LY; j++) free(matrix[j]);
  free(matrix); free(l->solids_memblock); free(l);
  return 0;
}

EXPORT int refk_read_raw(const char* path, int LX, int LY, int LZ, unsigned char* out)
{
  struct lattice_struct* l = harness_lattice(LX, LY, LZ);
  read_solids(l, (char*)path);
  memcpy(out, l->solids_memblock, (size_t)(LX * LY * LZ));
  free(l->solids_memblock); free(l);
  return 0;
}

/* ---- the reference's frame output --------------------------------------------
 * output_frame (src/lbio.c:37-131): the frame statistics of src/compute.c:
 * 1159-1467, dump_frame_summary (src/lbio.c:140-290), dump_macro_vars (3D
 * .raw images and .dat files, src/lbio.c:300-420, src/lattice.c:1737-1900)
 * and write_{rho,u}_txt (src/lbio.c:2864-2973), run on a harness lattice
 * holding the macro variables mv ([subs][1+D][N], real) and the mask bytes
 * sol.  Files go to ./out of the current directory (get_out_path). */
EXPORT int refk_output_frame(int LX, int LY, int LZ, const real* mv, const unsigned char* sol,
                             int time, int frame, int frame_rate)
{
  struct lattice_struct* l = harness_lattice(LX, LY, LZ);
  const int D = NUM_DIMENSIONS, NN = LX * LY * LZ;
  int s, c;
  l->NumDims = D;
  l->NumSubs = NUM_FLUID_COMPONENTS;
  l->param.FrameRate = frame_rate > 0 ? frame_rate : 1;
  memcpy(l->solids_memblock, sol, (size_t)NN);
  l->vars = (struct vars_struct*)calloc(NUM_FLUID_COMPONENTS, sizeof *l->vars);
  for (s = 0; s < NUM_FLUID_COMPONENTS; s++) {
    l->vars[s].macrovars_memblock = (real*)malloc((size_t)NN * (1 + D) * sizeof(real));
    memcpy(l->vars[s].macrovars_memblock, mv + (size_t)s * (1 + D) * NN,
           (size_t)NN * (1 + D) * sizeof(real));
    l->vars[s].macrovars1d = (real**)malloc((1 + D) * sizeof(real*));
    for (c = 0; c <= D; c++) l->vars[s].macrovars1d[c] = l->vars[s].macrovars_memblock + (size_t)c * NN;
  }
  l->time = time;
  l->frame = frame;
  output_frame(l);
  for (s = 0; s < NUM_FLUID_COMPONENTS; s++) {
    free(l->vars[s].macrovars1d);
    free(l->vars[s].macrovars_memblock);
  }
  free(l->vars); free(l->solids_memblock); free(l);
  return 0;
}

/* ---- the reference's initial state -------------------------------------------
 * init_problem (src/latman.c:1270-2063) on a harness lattice: the density of
 * every node per initial_condition (0 uniform, 2 cube; the others exit, as
 * in the reference), u = 0, and f = feq (shifted for the flow lattice of an
 * ACCURATE build).  f ([subs][Q][N]) and mv ([subs][1+D][N]) are written. */
typedef struct {
  int initial_condition;
  double rho_A[2], rho_B[2], rho_sigma;
  int x1, x2, y1, y2, z1, z2;
} refk_init;

EXPORT int refk_init_problem(int LX, int LY, int LZ, const refk_init* ip, real* f, real* mv)
{
  struct lattice_struct* l = harness_lattice(LX, LY, LZ);
  const int D = NUM_DIMENSIONS, Qd = 2 * D * D + 1, NN = LX * LY * LZ;
  int s, a, c;
  if (ip->initial_condition != 0 && ip->initial_condition != 2) return -1;
  l->NumDims = D;
  l->NumSubs = NUM_FLUID_COMPONENTS;
  l->NumVelDirs = Qd;
  l->param.initial_condition = ip->initial_condition;
  for (s = 0; s < NUM_FLUID_COMPONENTS; s++) {   /* the arrays hold one entry per substance */
    l->param.rho_A[s] = (real)ip->rho_A[s];
    l->param.rho_B[s] = (real)ip->rho_B[s];
  }
#if INAMURO_SIGMA_COMPONENT
  l->param.rho_sigma = (real)ip->rho_sigma;
#endif
  l->param.x1 = ip->x1; l->param.x2 = ip->x2;
  l->param.y1 = ip->y1; l->param.y2 = ip->y2;
  l->param.z1 = ip->z1; l->param.z2 = ip->z2;
  l->vars = (struct vars_struct*)calloc(NUM_FLUID_COMPONENTS, sizeof *l->vars);
  for (s = 0; s < NUM_FLUID_COMPONENTS; s++) {
    l->vars[s].f1d = (real**)malloc((size_t)Qd * sizeof(real*));
    for (a = 0; a < Qd; a++) l->vars[s].f1d[a] = f + ((size_t)s * Qd + a) * NN;
    l->vars[s].macrovars1d = (real**)malloc((size_t)(1 + D) * sizeof(real*));
    for (c = 0; c <= D; c++) l->vars[s].macrovars1d[c] = mv + ((size_t)s * (1 + D) + c) * NN;
  }
  init_problem(l);
  for (s = 0; s < NUM_FLUID_COMPONENTS; s++) {
    free(l->vars[s].f1d);
    free(l->vars[s].macrovars1d);
  }
  free(l->vars); free(l->solids_memblock); free(l);
  return 0;
}

/* read_params (src/params.h:40-660, derived values and defaults included)
 * on `path`, then init_problem: the reference's whole start-up path.  The
 * caller sizes f ([subs][Q][N]) and mv ([subs][1+D][N]) from the file's
 * extents; `cap` is the N they hold (-2 if the file's lattice is larger;
 * -1 for an initial_condition the reference exits on). */
EXPORT int refk_init_from_params(const char* path, int cap, real* f, real* mv)
{
  struct lattice_struct* l = harness_lattice(1, 1, 1);
  const int D = NUM_DIMENSIONS, Qd = 2 * D * D + 1;
  int s, a, c, NN;
  read_params(l, (char*)path);
  NN = l->param.LX * l->param.LY * l->param.LZ;
  if (NN > cap) { free(l->solids_memblock); free(l); return -2; }
  if (l->param.initial_condition != 0 && l->param.initial_condition != 2) {
    free(l->solids_memblock); free(l); return -1;
  }
  free(l->solids_memblock);
  l->solids_memblock = (unsigned char*)calloc((size_t)NN, 1);
  l->NumNodes = NN;
  l->NumDims = D;
  l->NumSubs = NUM_FLUID_COMPONENTS;
  l->NumVelDirs = Qd;
  l->vars = (struct vars_struct*)calloc(NUM_FLUID_COMPONENTS, sizeof *l->vars);
  for (s = 0; s < NUM_FLUID_COMPONENTS; s++) {
    l->vars[s].f1d = (real**)malloc((size_t)Qd * sizeof(real*));
    for (a = 0; a < Qd; a++) l->vars[s].f1d[a] = f + ((size_t)s * Qd + a) * NN;
    l->vars[s].macrovars1d = (real**)malloc((size_t)(1 + D) * sizeof(real*));
    for (c = 0; c <= D; c++) l->vars[s].macrovars1d[c] = mv + ((size_t)s * (1 + D) + c) * NN;
  }
  init_problem(l);
  for (s = 0; s < NUM_FLUID_COMPONENTS; s++) {
    free(l->vars[s].f1d);
    free(l->vars[s].macrovars1d);
  }
  free(l->vars); free(l->solids_memblock); free(l);
  return 0;
}

/* The reference's CPU time loop (src/lbgpu_prime.cu:597, :818, the
 * non-CUDA branches): stream_collide_stream on odd steps, collide on even
 * ones, on a serial lattice with the given populations ([subs][Q][N]),
 * solids, tau and body force of substance 0.  A cost baseline: this is the
 * reference's host model, not the device arithmetic the oracle pins. */
EXPORT int refk_cpu_loops(int LX, int LY, int LZ, double tau, const double* g,
                          const unsigned char* solids, real* f, int t0, int nsteps)
{
  struct lattice_struct* l = harness_lattice(LX, LY, LZ);
  const int D = NUM_DIMENSIONS, Qd = 2 * D * D + 1, NN = LX * LY * LZ;
  int s, a, t;
  memcpy(l->solids_memblock, solids, (size_t)NN);
  l->NumDims = D;
  l->NumSubs = NUM_FLUID_COMPONENTS;
  l->NumVelDirs = Qd;
  for (s = 0; s < NUM_FLUID_COMPONENTS; s++) {
    l->param.tau[s] = (real)tau;
    for (a = 0; a < 3; a++) l->param.gforce[s][a] = (real)g[a];
  }
  real* mv = (real*)calloc((size_t)NUM_FLUID_COMPONENTS * (1 + D) * NN, sizeof(real));
  l->vars = (struct vars_struct*)calloc(NUM_FLUID_COMPONENTS, sizeof *l->vars);
  for (s = 0; s < NUM_FLUID_COMPONENTS; s++) {
    l->vars[s].f1d = (real**)malloc((size_t)Qd * sizeof(real*));
    for (a = 0; a < Qd; a++) l->vars[s].f1d[a] = f + ((size_t)s * Qd + a) * NN;
    /* collide stores rho and u of every node (set_rho / set_ux ...) */
    l->vars[s].macrovars1d = (real**)malloc((size_t)(1 + D) * sizeof(real*));
    for (a = 0; a <= D; a++) l->vars[s].macrovars1d[a] = mv + ((size_t)s * (1 + D) + a) * NN;
  }
  for (t = t0 + 1; t <= t0 + nsteps; t++) {
    if (t % 2) stream_collide_stream(l);
    else collide(l);
  }
  for (s = 0; s < NUM_FLUID_COMPONENTS; s++) {
    free(l->vars[s].f1d);
    free(l->vars[s].macrovars1d);
  }
  free(l->vars); free(mv); free(l->solids_memblock); free(l);
  return 0;
}
