/*
 * refgpu_harness.cu -- the reference's own CUDA step kernels on the GPU.
 *
 * TEST INFRASTRUCTURE ONLY.  Built by oracle/ref_build.py (the --gpu
 * targets) from the reference's sources where they lie, for sm_100a, with
 * an edited flags.h force-included; nothing is copied into the repository.
 * The product library never links it.  tests/test_gpu_reference_kernels.py
 * runs it to check the product's GPU results against the reference's GPU
 * results and to time the reference's kernels on the same device.
 *
 * What runs: k_stream_collide_stream (odd times) and k_collide (even times)
 * of src/k_stream_collide_stream.c and src/k_collide.c, unmodified, launched
 * as the reference's serial main launches them (src/lbgpu_prime.cu:144-147,
 * :517-527, :741-750): a grid of (LX/BX, LY/BY, LZ/BZ) blocks of
 * (BX, BY, BZ) threads with (Q + D + 1) reals of dynamic shared memory per
 * thread, after the constant upload of construct_lattice
 * (src/latman.c:147-376) for a serial run (EndBoundSize 0, so
 * cumul_stride[a] = a N).  One substance, periodic on every face, body
 * force, no face boundaries, no PEST sampling.  The host side (the
 * arguments, files, the step loop and its timing) is this harness's own.
 *
 * Usage: refgpu LX LY LZ BX BY BZ tau gx gy gz steps mask.raw f_in f_out [time]
 *   f_in / f_out: [Q][N] reals in the variant's precision ("-": start from
 *   zero populations / write nothing); the last step writes the macro
 *   variables too (is_end_of_frame).  With "time": two warm-up steps, then
 *   `steps` steps between CUDA events; prints one JSON line.
 */
#if DP_ON
typedef double real;
#else
typedef float real;
#endif

/* the device globals the reference's sources name (src/lbgpu_prime.cu:10-17) */
real* f_mem_d;
int f_mem_size;
real* mv_mem_d;
int mv_mem_size;
unsigned char* solids_mem_d;
real* ns_mem_d;
int solids_mem_size;
#if BOUNDARY_KERNEL
real* pos_dir_send_ptr_d;
real* pos_dir_recv_ptr_d;
real* neg_dir_send_ptr_d;
real* neg_dir_recv_ptr_d;
#endif

#include "lbgpu_prime.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static void refgpu_check(const char* what)
{
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    fprintf(stderr, "refgpu: %s: %s\n", what, cudaGetErrorString(e));
    exit(2);
  }
}

template <typename V>
static void refgpu_const(const V& sym, const void* src, size_t n)
{
  cudaMemcpyToSymbol(sym, src, n);
  refgpu_check("cudaMemcpyToSymbol");
}

int main(int argc, char** argv)
{
  if (argc < 15) {
    fprintf(stderr, "usage: refgpu LX LY LZ BX BY BZ tau gx gy gz steps mask f_in f_out [time]\n");
    return 1;
  }
  const int LX = atoi(argv[1]), LY = atoi(argv[2]), LZ = atoi(argv[3]);
  const int BX = atoi(argv[4]), BY = atoi(argv[5]), BZ = atoi(argv[6]);
  const double tau = atof(argv[7]);
  const double g[3] = {atof(argv[8]), atof(argv[9]), atof(argv[10])};
  const int steps = atoi(argv[11]);
  const char* mask_path = argv[12];
  const char* fin_path = argv[13];
  const char* fout_path = argv[14];
  const int timing = argc > 15 && strcmp(argv[15], "time") == 0;
  const int nd = NUM_DIMENSIONS, nq = (nd == 2) ? 9 : 19, nsub = NUM_FLUID_COMPONENTS;
  if (nsub != 1 || LX % BX || LY % BY || LZ % BZ || steps < 1) {
    fprintf(stderr, "refgpu: one substance, and block extents dividing the lattice\n");
    return 1;
  }
  const long long nnodes_ll = (long long)LX * LY * LZ;
  if (nnodes_ll * nq >= (1LL << 31)) {
    fprintf(stderr, "refgpu: the reference indexes populations with int\n");
    return 1;
  }
  const int nn = (int)nnodes_ll;

  /* constants, as construct_lattice uploads them for a serial run */
  {
    int a;
    real w[19], tr = (real)tau, itr = 1. / (real)tau, rA = 1.0, ga[6] = {0, 0, 0, 0, 0, 0};
    int cs[20];
    if (nd == 2) {
      real W0 = 4./9., W1 = 1./9., W2 = 1./36.;
      w[0] = W0;
      for (a = 1; a < 5; a++) w[a] = W1;
      for (; a < 9; a++) w[a] = W2;
      for (; a < 19; a++) w[a] = 0.;
    } else {
      real W0 = 1./3., W1 = 1./18., W2 = 1./36.;
      w[0] = W0;
      for (a = 1; a < 5; a++) w[a] = W1;
      for (; a < 9; a++) w[a] = W2;
      for (; a < 11; a++) w[a] = W1;
      for (; a < 19; a++) w[a] = W2;
    }
    for (a = 0; a < 20; a++) cs[a] = a * nn;
    for (a = 0; a < nd; a++) ga[a] = (real)g[a];
    const int nbd = (nd == 2) ? 6 : 10, nunb = nq - nbd, zero = 0, one = 1;
    const int bij = BX * BY, bik = BX * BZ, bjk = BY * BZ, nij = LX * LY, bs = BX * BY * BZ;
    refgpu_const(vx_c, vx, 19 * sizeof(int));
    refgpu_const(vy_c, vy, 19 * sizeof(int));
    refgpu_const(vz_c, vz, 19 * sizeof(int));
    refgpu_const(wt_c, w, 19 * sizeof(real));
    refgpu_const(cumul_stride_c, cs, 20 * sizeof(int));
    refgpu_const(tau_c, &tr, sizeof(real));
    refgpu_const(inv_tau_c, &itr, sizeof(real));
    refgpu_const(rho_A_c, &rA, sizeof(real));
    refgpu_const(gaccel_c, ga, 3 * sizeof(real));
    refgpu_const(numsubs_c, &nsub, sizeof(int));
    refgpu_const(numdims_c, &nd, sizeof(int));
    refgpu_const(numdirs_c, &nq, sizeof(int));
    refgpu_const(numbounddirs_c, &nbd, sizeof(int));
    refgpu_const(numunbounddirs_c, &nunb, sizeof(int));
    refgpu_const(end_bound_c, &zero, sizeof(int));
    refgpu_const(proc_id_c, &zero, sizeof(int));
    refgpu_const(num_procs_c, &one, sizeof(int));
    refgpu_const(ni_c, &LX, sizeof(int));
    refgpu_const(nj_c, &LY, sizeof(int));
    refgpu_const(nk_c, &LZ, sizeof(int));
    refgpu_const(kloop_c, &one, sizeof(int));
    refgpu_const(bixbj_c, &bij, sizeof(int));
    refgpu_const(bixbk_c, &bik, sizeof(int));
    refgpu_const(bjxbk_c, &bjk, sizeof(int));
    refgpu_const(nixnj_c, &nij, sizeof(int));
    refgpu_const(blocksize_c, &bs, sizeof(int));
    refgpu_const(numnodes_c, &nn, sizeof(int));
    refgpu_const(is_end_of_frame_mem_c, &zero, sizeof(int));
    refgpu_const(pest_output_flag_c, &zero, sizeof(int));
  }

  /* device arrays, sized as construct_lattice sizes them */
  const size_t fbytes = (size_t)nq * nn * sizeof(real);
  cudaMalloc((void**)&f_mem_d, fbytes);
  cudaMalloc((void**)&mv_mem_d, (size_t)(1 + nd) * nn * sizeof(real));
  cudaMalloc((void**)&solids_mem_d, (size_t)nn);
  refgpu_check("cudaMalloc");
  ns_mem_d = NULL;
  {
    unsigned char* sol = (unsigned char*)malloc((size_t)nn);
    FILE* fh = fopen(mask_path, "rb");
    if (!fh || fread(sol, 1, (size_t)nn, fh) != (size_t)nn) {
      fprintf(stderr, "refgpu: cannot read %s\n", mask_path);
      return 1;
    }
    fclose(fh);
    cudaMemcpy(solids_mem_d, sol, (size_t)nn, cudaMemcpyHostToDevice);
    free(sol);
  }
  {
    real* f = (real*)calloc((size_t)nq * nn, sizeof(real));
    if (strcmp(fin_path, "-") != 0) {
      FILE* fh = fopen(fin_path, "rb");
      if (!fh || fread(f, sizeof(real), (size_t)nq * nn, fh) != (size_t)nq * nn) {
        fprintf(stderr, "refgpu: cannot read %s\n", fin_path);
        return 1;
      }
      fclose(fh);
    }
    cudaMemcpy(f_mem_d, f, fbytes, cudaMemcpyHostToDevice);
    free(f);
  }
  cudaMemset(mv_mem_d, 0, (size_t)(1 + nd) * nn * sizeof(real));
  refgpu_check("upload");

  dim3 block(BX, BY, BZ), grid(LX / BX, LY / BY, LZ / BZ);
  const size_t smem = sizeof(real) * (nq + nd + 1) * BX * BY * BZ;
  auto step = [&](int t, int last) {
    const int eof = last ? 1 : 0;
    cudaMemcpyToSymbol(is_end_of_frame_mem_c, &eof, sizeof(int));
    if (t % 2) k_stream_collide_stream<<<grid, block, smem>>>(f_mem_d, mv_mem_d, solids_mem_d, ns_mem_d);
    else k_collide<<<grid, block, smem>>>(f_mem_d, mv_mem_d, solids_mem_d, ns_mem_d);
    refgpu_check("step launch");
  };

  int t = 0;
  if (timing) {
    step(++t, 0);
    step(++t, 0);
    cudaDeviceSynchronize();
    refgpu_check("warm-up");
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, 0);
    for (int s = 0; s < steps; ++s) step(++t, 0);
    cudaEventRecord(e1, 0);
    cudaEventSynchronize(e1);
    refgpu_check("timed steps");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    printf("{\"LX\": %d, \"LY\": %d, \"LZ\": %d, \"block\": [%d, %d, %d], \"real_bytes\": %d, "
           "\"steps\": %d, \"ms_per_step\": %.5f, \"mlups\": %.3f}\n",
           LX, LY, LZ, BX, BY, BZ, (int)sizeof(real), steps, ms / steps,
           (double)nn * steps / (ms * 1e-3) / 1e6);
  } else {
    for (int s = 1; s <= steps; ++s) step(++t, s == steps);
    cudaDeviceSynchronize();
    refgpu_check("steps");
  }
  if (strcmp(fout_path, "-") != 0) {
    real* f = (real*)malloc(fbytes);
    real* mv = (real*)malloc((size_t)(1 + nd) * nn * sizeof(real));
    cudaMemcpy(f, f_mem_d, fbytes, cudaMemcpyDeviceToHost);
    cudaMemcpy(mv, mv_mem_d, (size_t)(1 + nd) * nn * sizeof(real), cudaMemcpyDeviceToHost);
    refgpu_check("download");
    FILE* fh = fopen(fout_path, "wb");
    if (!fh) { fprintf(stderr, "refgpu: cannot write %s\n", fout_path); return 1; }
    fwrite(f, sizeof(real), (size_t)nq * nn, fh);
    fwrite(mv, sizeof(real), (size_t)(1 + nd) * nn, fh);
    fclose(fh);
    free(f);
    free(mv);
  }
  cudaFree(f_mem_d);
  cudaFree(mv_mem_d);
  cudaFree(solids_mem_d);
  return 0;
}
