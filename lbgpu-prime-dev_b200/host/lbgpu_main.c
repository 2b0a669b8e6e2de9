/*
 * lbgpu_main.c -- the host driver: the reference's main()
 * (src/lbgpu_prime.cu:82-940) with its device work done through the lbx C
 * ABI (include/lbx.h).
 *
 *   lbgpu_b200 [name] [--dims 2|3] [--subs 1|2] [--precision 4|8]
 *              [--model shifted|plain|shifted-compressible] [--device N]
 *              [--solid-rule device|nonzero] [--kahan] [--walsh]
 *
 * Reads ./in/params.in (./in_<name>/params.in with a name, src/latman.c:
 * 108-116), the mask ./in/<LX>x<LY>.bmp (2D) or ./in/<LX>x<LY>x<LZ>.raw (3D)
 * and, for pressure_{n,s}_in[0] == 2, ./in/pressure_{n,s}_in0.in; then runs
 * NumFrames*FrameRate steps in AA pairs and at every frame writes
 * ./out/cuda_{rho,u_x,u_y[,u_z]}<size>_frame<NNNN>[_subsNN].dat and appends
 * a line to ./out/cuda_frames<size>[_subsNN].dat.
 *
 * The build-time flags of the reference (NUM_DIMENSIONS, NUM_FLUID_COMPONENTS,
 * DP_ON, ACCURATE/COMPRESSIBLE, KAHAN_SUMMATION, WALSH_NS_ON with
 * COMPUTE_ON_SOLIDS) are the options above; the defaults are the reference's
 * shipped flags.h (2D, one substance, double, shifted).  --walsh takes its
 * fraction field from the mask and the params.in value `ns` (the field the
 * reference's 2D runs upload); a 3D run with ns_flag 1 reads
 * ./in/ns<LX>x<LY>x<LZ>.raw (byte / 255) instead, as read_ns does (the
 * reference's own 3D runs leave the uploaded field unset).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <time.h>

#include "lbh.h"
#include "lbx.h"

#define DIE(...) do { fprintf(stderr, "lbgpu_b200: " __VA_ARGS__); fputc('\n', stderr); exit(1); } while (0)
#define LBX(call) do { lbx_status st_ = (call); if (st_ != LBX_OK) \
  DIE("%s failed (%d): %s", #call, st_, lbx_last_error()); } while (0)

static double* read_table(const char* path, int* len)
{
  FILE* in = fopen(path, "r");
  double v, *t = NULL;
  int n = 0, cap = 0;
  if (!in) return NULL;
  while (fscanf(in, "%lf", &v) == 1) {
    if (n == cap) { cap = cap ? 2 * cap : 64; t = (double*)realloc(t, (size_t)cap * sizeof *t); }
    t[n++] = v;
  }
  fclose(in);
  *len = n;
  return t;
}

static double rv(const lbh_real* r, int prec) { return prec == 4 ? (double)r->f : r->d; }

typedef struct {
  lbh_params hp;
  int dims, nsubs, prec;
  uint8_t* mask;
  lbx_domain* dom;
  void* mv;       /* host copy of one substance's macro variables */
  char size[64];
} run_t;

static void output_frame(run_t* r, int time, int frame)
{
  const long long N = r->hp.NumNodes;
  const size_t plane = (size_t)N * (size_t)r->prec;
  char fn[1024];
  int s, c;
  lbx_reductions red;
  const char* names[4] = {"rho", "u_x", "u_y", "u_z"};
  lbx_status st = lbx_reduce(r->dom, &red);
  if (st != LBX_OK && st != LBX_ERR_NUMERIC) DIE("lbx_reduce: %s", lbx_last_error());
  for (s = 0; s < r->nsubs; s++) {
    char* base = (char*)r->mv;
    FILE* o;
    LBX(lbx_download_mv(r->dom, s, base, base + plane, base + 2 * plane,
                        r->dims == 3 ? base + 3 * plane : NULL));
    for (c = 0; c <= r->dims; c++) {
      lbh_frame_filename(fn, sizeof fn, "./out", names[c], r->dims, r->hp.LX, r->hp.LY,
                         r->hp.LZ, frame, r->nsubs, s, ".dat");
      if (lbh_write_dat(fn, base + c * plane, r->prec, N, r->mask)) DIE("cannot write %s", fn);
    }
    lbh_frame_filename(fn, sizeof fn, "./out", "frames", r->dims, r->hp.LX, r->hp.LY,
                       r->hp.LZ, -1, r->nsubs, s, ".dat");
    o = fopen(fn, time == 0 ? "w" : "a");
    if (!o) DIE("cannot write %s", fn);
    if (time == 0)
      fprintf(o, "# time frame fluid_nodes mass ave_u_x ave_u_y ave_u_z min_rho max_rho"
                 " solute_mass nonfinite\n");
    if (s == 0) {
      const double nf = red.fluid_nodes > 0 ? (double)red.fluid_nodes : 1.0;
      fprintf(o, "%d %d %lld %.17g %.10e %.10e %.10e %.17g %.17g %.17g %d\n", time, frame,
              red.fluid_nodes, red.mass, red.u_sum[0] / nf, red.u_sum[1] / nf,
              red.u_sum[2] / nf, red.rho_min, red.rho_max, red.solute_mass, red.nonfinite);
    } else {
      fprintf(o, "%d %d solute_mass %.17g\n", time, frame, red.solute_mass);
    }
    fclose(o);
  }
  printf("frame %d at time %d: mass %.12g, <ux> %.6e\n", frame, time, red.mass,
         red.fluid_nodes ? red.u_sum[0] / (double)red.fluid_nodes : 0.0);
}

int main(int argc, char** argv)
{
  run_t r;
  lbx_params p;
  char dir[512], path[1024], err[512];
  const char* name = NULL;
  const char* model = "shifted";
  const char* solid_rule = "device";
  int kahan = 0, walsh = 0;
  int device = 0, i, s, time, frame;
  double* ntab = NULL, *stab = NULL;
  int nlen = 0, slen = 0;
  memset(&r, 0, sizeof r);
  r.dims = 2; r.nsubs = 1; r.prec = 8;
  for (i = 1; i < argc; i++) {
    if (!strcmp(argv[i], "--dims") && i + 1 < argc) r.dims = atoi(argv[++i]);
    else if (!strcmp(argv[i], "--subs") && i + 1 < argc) r.nsubs = atoi(argv[++i]);
    else if (!strcmp(argv[i], "--precision") && i + 1 < argc) r.prec = atoi(argv[++i]);
    else if (!strcmp(argv[i], "--model") && i + 1 < argc) model = argv[++i];
    else if (!strcmp(argv[i], "--device") && i + 1 < argc) device = atoi(argv[++i]);
    else if (!strcmp(argv[i], "--solid-rule") && i + 1 < argc) solid_rule = argv[++i];
    else if (!strcmp(argv[i], "--kahan")) kahan = 1;
    else if (!strcmp(argv[i], "--walsh")) walsh = 1;
    else if (argv[i][0] != '-') name = argv[i];
    else DIE("unknown option %s", argv[i]);
  }
  snprintf(dir, sizeof dir, name ? "./in_%s" : "./in", name);
  snprintf(path, sizeof path, "%s/params.in", dir);
  if (lbh_read_params(path, r.dims, r.nsubs, &r.hp, err, sizeof err)) DIE("%s", err);

  /* mask (src/latman.c:389-428) */
  r.mask = (uint8_t*)malloc((size_t)r.hp.NumNodes);
  if (r.dims == 2) {
    snprintf(path, sizeof path, "./in/%dx%d.bmp", r.hp.LX, r.hp.LY);
    if (lbh_read_bmp_mask(path, r.hp.LX, r.hp.LY, r.mask, err, sizeof err)) DIE("%s", err);
  } else {
    snprintf(path, sizeof path, "./in/%dx%dx%d.raw", r.hp.LX, r.hp.LY, r.hp.LZ);
    if (lbh_read_raw_mask(path, r.hp.NumNodes, r.mask, err, sizeof err)) DIE("%s", err);
  }
  {
    const int rule = !strcmp(solid_rule, "nonzero") ? LBH_SOLID_NONZERO
                   : !strcmp(solid_rule, "device") ? LBH_SOLID_DEVICE : -1;
    long long odd;
    if (rule < 0) DIE("--solid-rule must be device or nonzero");
    odd = lbh_apply_solid_rule(r.mask, r.hp.NumNodes, rule);
    if (odd && rule == LBH_SOLID_DEVICE)
      fprintf(stderr, "warning: %lld mask bytes are neither 0 nor 1; the device rule "
              "runs them as fluid (--solid-rule nonzero makes them solid)\n", odd);
  }

  lbx_params_default(&p);
  p.dims = r.dims; p.LX = r.hp.LX; p.LY = r.hp.LY; p.LZ = r.hp.LZ;
  p.nsubs = r.nsubs; p.precision = r.prec; p.device = device;
  p.kahan = kahan;
  p.walsh = walsh;
  if (!strcmp(model, "shifted")) { p.accurate = 1; p.compressible = 0; }
  else if (!strcmp(model, "plain")) { p.accurate = 0; p.compressible = 1; }
  else if (!strcmp(model, "shifted-compressible")) { p.accurate = 1; p.compressible = 1; }
  else DIE("unknown model %s", model);
  for (s = 0; s < 2; s++) {
    int c;
    p.tau[s] = rv(&r.hp.tau[s], r.prec);
    p.rho_A[s] = rv(&r.hp.rho_A[s], r.prec);
    for (c = 0; c < 3; c++) p.gaccel[3 * s + c] = rv(&r.hp.gforce[s][c], r.prec);
    p.pressure_n_in[s] = r.hp.pressure_n_in[s];
    p.pressure_s_in[s] = r.hp.pressure_s_in[s];
    p.pressure_n_out[s] = r.hp.pressure_n_out[s];
    p.pressure_s_out[s] = r.hp.pressure_s_out[s];
  }
  if (r.nsubs == 1)
    for (s = 0; s < 2; s++) p.pressure_n_in[1] = p.pressure_s_in[1] = p.pressure_n_out[1] = p.pressure_s_out[1] = 0;
  if (r.dims == 3) {   /* the reference applies faces in 2D only (src/lbgpu_prime.cu:489-496) */
    for (s = 0; s < 2; s++) p.pressure_n_in[s] = p.pressure_s_in[s] = p.pressure_n_out[s] = p.pressure_s_out[s] = 0;
  }
  p.sink = rv(&r.hp.sink, r.prec);
  p.sigma_t_on = r.hp.sigma_t_on; p.sigma_t_off = r.hp.sigma_t_off;
  p.zeroconcgrad_n = r.dims == 2 ? r.hp.zeroconcgrad_n : 0;
  p.zeroconcgrad_s = r.dims == 2 ? r.hp.zeroconcgrad_s : 0;
  p.rho_in = rv(&r.hp.rho_in, r.prec); p.rho_out = rv(&r.hp.rho_out, r.prec);
  p.pfadd = rv(&r.hp.pfadd, r.prec); p.pfmul = rv(&r.hp.pfmul, r.prec);
  p.bc_ramp_start = r.hp.bc_ramp_start; p.bc_ramp_stop = r.hp.bc_ramp_stop;
  if (p.pressure_n_in[0] == 2) {
    if (!(ntab = read_table("./in/pressure_n_in0.in", &nlen)) || !nlen)
      DIE("pressure_n_in == 2 needs ./in/pressure_n_in0.in");
    p.pressure_n_table = ntab; p.pressure_n_len = nlen;
  }
  if (p.pressure_s_in[0] == 2) {
    if (!(stab = read_table("./in/pressure_s_in0.in", &slen)) || !slen)
      DIE("pressure_s_in == 2 needs ./in/pressure_s_in0.in");
    p.pressure_s_table = stab; p.pressure_s_len = slen;
  }
  LBX(lbx_create(&p, r.mask, &r.dom));
  if (walsh) {
    double* ns = (double*)malloc((size_t)r.hp.NumNodes * sizeof(double));
    const int src = r.dims == 3 && r.hp.ns_flag == 1 ? LBH_NS_FILE : LBH_NS_MASK;
    snprintf(path, sizeof path, "./in/ns%dx%dx%d.raw", r.hp.LX, r.hp.LY, r.hp.LZ);
    if (lbh_walsh_ns(rv(&r.hp.ns, r.prec), src, r.mask, r.hp.NumNodes, path, ns, err,
                     sizeof err))
      DIE("%s", err);
    LBX(lbx_set_ns(r.dom, ns));
    free(ns);
  }

  /* initial state (init_problem, src/latman.c:1270-1959): rho per
   * initial_condition, u = 0, f = feq; the same [rho, u] planes are the
   * macro variables frame 0 reports */
  {
    const long long N = r.hp.NumNodes;
    const size_t plane = (size_t)N * (size_t)r.prec;
    double* rho = (double*)malloc((size_t)N * sizeof(double));
    char* b = (char*)calloc(1 + (size_t)r.dims, plane);
    long long n;
    for (s = 0; s < r.nsubs; s++) {
      if (lbh_initial_rho(&r.hp, r.dims, r.nsubs, s, rho))
        DIE("initial_condition %d is not supported", r.hp.initial_condition);
      for (n = 0; n < N; n++) {
        if (r.prec == 8) ((double*)b)[n] = rho[n];
        else ((float*)b)[n] = (float)rho[n];
      }
      LBX(lbx_init_equilibrium(r.dom, s, b, b + plane, b + 2 * plane,
                               r.dims == 3 ? b + 3 * plane : NULL));
      LBX(lbx_upload_mv(r.dom, s, b));
    }
    free(rho);
    free(b);
  }
  mkdir("./out", 0755);
  r.mv = malloc((size_t)r.hp.NumNodes * (size_t)r.prec * (size_t)(1 + r.dims));
  output_frame(&r, 0, 0);

  /* the time loop of src/lbgpu_prime.cu:369-915: pairs of steps, frames at
   * multiples of FrameRate, stop after the final frame */
  {
    clock_t t0 = clock();
    for (frame = 0, time = 1; time <= r.hp.NumTimeSteps; time++) {
      int eof = (time % r.hp.FrameRate) == 0;
      LBX(lbx_step(r.dom, time, eof ? LBX_WRITE_MV : 0));
      if (eof) {
        LBX(lbx_sync(r.dom));
        output_frame(&r, time, ++frame);
        if (frame == r.hp.NumFrames) break;
      }
      time++;
      eof = (time % r.hp.FrameRate) == 0;
      LBX(lbx_step(r.dom, time, eof ? LBX_WRITE_MV : 0));
      if (eof) {
        LBX(lbx_sync(r.dom));
        output_frame(&r, time, ++frame);
      }
      if (frame >= r.hp.NumFrames) break;
    }
    LBX(lbx_sync(r.dom));
    printf("ran %d steps of %lld nodes in %.3f s\n", time, r.hp.NumNodes,
           (double)(clock() - t0) / CLOCKS_PER_SEC);
  }
  LBX(lbx_destroy(r.dom));
  free(r.mv); free(r.mask); free(ntab); free(stab);
  return 0;
}
