/*
 * lbgpu_main.c -- the host driver: the reference's main()
 * (src/lbgpu_prime.cu:82-940) with its device work done through the lbx C
 * ABI (include/lbx.h).
 *
 *   lbgpu_b200 [name] [--dims 2|3] [--subs 1|2] [--precision 4|8]
 *              [--model shifted|plain|shifted-compressible] [--device N]
 *              [--solid-rule device|nonzero] [--kahan] [--walsh] [--zfaces]
 *              [--frames summary,raw,dat,txt|all|none]
 *
 * Reads ./in/params.in (./in_<name>/params.in with a name, src/latman.c:
 * 108-116), the mask ./in/<LX>x<LY>.bmp (2D) or ./in/<LX>x<LY>x<LZ>.raw (3D)
 * and, for pressure_{n,s}_in[0] == 2, ./in/pressure_{n,s}_in0.in; then runs
 * NumFrames*FrameRate steps and at every frame writes the files of the
 * reference's output_frame into ./out: a line of cuda_frames<size>[_subsNN].dat
 * (summary), in 3D the byte images cuda_{rho,u,u_x,u_y,u_z}<size>_frameNNNN.raw
 * (raw), cuda_{rho,u_x,u_y[,u_z]}<size>_frameNNNN.dat (dat) and the text dumps
 * cuda_{rho,ux,uy,uz}<size>_frameNNNN.txt (txt); --frames selects the kinds
 * (default all, as the reference's build writes).  With
 * ./in/{timestep,x_coord,y_coord}_file.in present (and two substances) the
 * PEST point samples are taken and written at the end to
 * ./out/{conc_data,vel_data,conc_order}_proc0000.dat.
 *
 * The build-time flags of the reference (NUM_DIMENSIONS, NUM_FLUID_COMPONENTS,
 * DP_ON, ACCURATE/COMPRESSIBLE, KAHAN_SUMMATION, WALSH_NS_ON with
 * COMPUTE_ON_SOLIDS) are the options above; the defaults are the reference's
 * shipped flags.h (2D, one substance, double, shifted).  --walsh takes its
 * fraction field from the mask and the params.in value `ns` (the field the
 * reference's 2D runs upload); a 3D run with ns_flag 1 reads
 * ./in/ns<LX>x<LY>x<LZ>.raw (byte / 255) instead, as read_ns does (the
 * reference's own 3D runs leave the uploaded field unset).  --zfaces applies
 * the z-face boundaries of params.in in 3D (pressure_{t,b}_{in,out},
 * velocity_{t,b}_{in,out} with uz_in / uz_out, constcon_{t,b}_in and
 * zeroconcgrad_{t,b} for the solute), which the reference's device code
 * does not implement; without it a 3D run is periodic, as the reference's.
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
  unsigned frame_files;   /* LBH_FRAME_* kinds written per frame */
} run_t;

/* The files of output_frame (src/lbio.c:37-131) for one frame that
 * lbx_frame_wait returned: the summary line, the 3D byte images, the .dat
 * files and the text dumps, with the statistics computed on the device. */
static void write_frame(run_t* r, const lbx_frame* fr, int frame)
{
  lbh_frame_stats st[2];
  const void* mv[2] = {fr->mv[0], fr->mv[1]};
  int s, c;
  for (s = 0; s < fr->nsubs; s++) {
    st[s].nodes = fr->stats[s].nodes;
    st[s].max_rho = fr->stats[s].max_rho;
    st[s].min_rho = fr->stats[s].min_rho;
    st[s].ave_rho = fr->stats[s].ave_rho;
    for (c = 0; c < 3; c++) {
      st[s].max_u[c] = fr->stats[s].max_u[c];
      st[s].min_u[c] = fr->stats[s].min_u[c];
      st[s].ave_u[c] = fr->stats[s].ave_u[c];
    }
    if (st[s].ave_rho != st[s].ave_rho)
      fprintf(stderr, "warning: subs %d holds non-finite densities at time %d\n", s, fr->time);
  }
  if (lbh_write_frame("./out", r->dims, r->nsubs, r->hp.LX, r->hp.LY, r->hp.LZ, fr->time, frame,
                      r->prec, mv, st, r->mask, r->frame_files))
    DIE("cannot write the files of frame %d in ./out", frame);
  printf("frame %d (time %d): ave_rho = %.17g, ave_u = [ %g %g %g]\n", frame, fr->time,
         st[0].ave_rho, st[0].ave_u[0], st[0].ave_u[1], st[0].ave_u[2]);
}

static unsigned parse_frame_files(const char* list)
{
  unsigned f = 0;
  const char* p = list;
  while (*p) {
    size_t n = strcspn(p, ",");
    if (n == 7 && !strncmp(p, "summary", 7)) f |= LBH_FRAME_SUMMARY;
    else if (n == 3 && !strncmp(p, "raw", 3)) f |= LBH_FRAME_RAW;
    else if (n == 3 && !strncmp(p, "dat", 3)) f |= LBH_FRAME_DAT;
    else if (n == 3 && !strncmp(p, "txt", 3)) f |= LBH_FRAME_TXT;
    else if (n == 3 && !strncmp(p, "all", 3)) f |= LBH_FRAME_ALL;
    else if (n == 4 && !strncmp(p, "none", 4)) f |= 0;
    else DIE("--frames takes a comma list of summary, raw, dat, txt, all, none");
    p += n;
    if (*p == ',') p++;
  }
  return f;
}

int main(int argc, char** argv)
{
  run_t r;
  lbx_params p;
  char dir[512], path[1024], err[512];
  const char* name = NULL;
  const char* model = "shifted";
  const char* solid_rule = "device";
  int kahan = 0, walsh = 0, zfaces = 0;
  int pest_n = -1, pest_kept = 0;
  int *pest_order = NULL, *pest_time = NULL, *pest_node = NULL;
  const char* frames = "all";
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
    else if (!strcmp(argv[i], "--zfaces")) zfaces = 1;
    else if (!strcmp(argv[i], "--frames") && i + 1 < argc) frames = argv[++i];
    else if (argv[i][0] != '-') name = argv[i];
    else DIE("unknown option %s", argv[i]);
  }
  r.frame_files = parse_frame_files(frames);
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
    if (zfaces) {       /* the z faces of params.in, which the reference's device ignores */
      for (s = 0; s < r.nsubs; s++) {
        p.pressure_t_in[s] = r.hp.pressure_t_in[s];
        p.pressure_b_in[s] = r.hp.pressure_b_in[s];
        p.pressure_t_out[s] = r.hp.pressure_t_out[s];
        p.pressure_b_out[s] = r.hp.pressure_b_out[s];
        p.velocity_t_in[s] = r.hp.velocity_t_in[s];
        p.velocity_b_in[s] = r.hp.velocity_b_in[s];
        p.velocity_t_out[s] = r.hp.velocity_t_out[s];
        p.velocity_b_out[s] = r.hp.velocity_b_out[s];
      }
      p.uz_in = rv(&r.hp.uz_in, r.prec);
      p.uz_out = rv(&r.hp.uz_out, r.prec);
      if (r.nsubs == 2) {
        p.constcon_t_in = r.hp.constcon[0];    /* constcon_t_in, constcon_b_in */
        p.constcon_b_in = r.hp.constcon[1];
        p.zeroconcgrad_t = r.hp.zeroconcgrad_t;
        p.zeroconcgrad_b = r.hp.zeroconcgrad_b;
        p.rho_sigma_in = rv(&r.hp.rho_sigma_in, r.prec);
      }
    }
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
  /* PEST point samples (PEST_OUTPUT_ON): on when ./in/timestep_file.in exists */
  pest_n = lbh_pest_count("./in");
  if (pest_n >= 0 && r.nsubs != 2) {
    fprintf(stderr, "warning: PEST samples read the solute; a one-substance run skips them\n");
    pest_n = -1;
  }
  if (pest_n >= 0) {
    pest_order = (int*)malloc((size_t)(pest_n + 1) * sizeof(int));
    pest_time = (int*)malloc((size_t)(pest_n + 1) * sizeof(int));
    pest_node = (int*)malloc((size_t)(pest_n + 1) * sizeof(int));
    pest_kept = lbh_read_pest("./in", r.hp.LX, r.hp.LY, pest_n, pest_order, pest_time,
                              pest_node, err, sizeof err);
    if (pest_kept < 0) DIE("%s", err);
    LBX(lbx_pest_set(r.dom, pest_kept, pest_time, pest_node));
    printf("PEST: %d samples read, %d in the lattice\n", pest_n, pest_kept);
  }
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
   * initial_condition, u = 0 (NULL: filled on the device), f = feq; the
   * domain's macro variables then hold [rho, u], which frame 0 reports */
  {
    const long long N = r.hp.NumNodes;
    const size_t plane = (size_t)N * (size_t)r.prec;
    double* rho = (double*)malloc((size_t)N * sizeof(double));
    char* b = (char*)malloc(plane);
    long long n;
    for (s = 0; s < r.nsubs; s++) {
      if (lbh_initial_rho(&r.hp, r.dims, r.nsubs, s, rho))
        DIE("initial_condition %d is not supported", r.hp.initial_condition);
      for (n = 0; n < N; n++) {
        if (r.prec == 8) ((double*)b)[n] = rho[n];
        else ((float*)b)[n] = (float)rho[n];
      }
      LBX(lbx_init_equilibrium(r.dom, s, b, NULL, NULL, NULL));
    }
    free(rho);
    free(b);
  }
  mkdir("./out", 0755);
  {
    lbx_frame fr;
    struct timespec t0, t1;
    double secs;
    LBX(lbx_frame_enqueue(r.dom, 0));
    LBX(lbx_frame_wait(r.dom, &fr));
    write_frame(&r, &fr, 0);
    /* the time loop of src/lbgpu_prime.cu:369-915: NumFrames stretches of
     * FrameRate steps, the last of each writing the macro variables.  Each
     * frame is snapshotted on the device and copied to the host in the
     * background; its files are written while the next stretch runs. */
    clock_gettime(CLOCK_MONOTONIC, &t0);
    for (frame = 1; frame <= r.hp.NumFrames; frame++) {
      time = (frame - 1) * r.hp.FrameRate;
      LBX(lbx_run(r.dom, time, r.hp.FrameRate, r.hp.FrameRate));
      LBX(lbx_frame_enqueue(r.dom, time + r.hp.FrameRate));
      if (frame > 1) {
        LBX(lbx_frame_wait(r.dom, &fr));
        write_frame(&r, &fr, frame - 1);
      }
    }
    if (r.hp.NumFrames >= 1) {
      LBX(lbx_frame_wait(r.dom, &fr));
      write_frame(&r, &fr, r.hp.NumFrames);
    }
    LBX(lbx_sync(r.dom));
    clock_gettime(CLOCK_MONOTONIC, &t1);
    secs = (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
    printf("ran %d steps of %lld nodes in %.3f s (%.1f MLUPS with frame output)\n",
           r.hp.NumFrames * r.hp.FrameRate, r.hp.NumNodes, secs,
           secs > 0 ? (double)r.hp.NumNodes * r.hp.NumFrames * r.hp.FrameRate / secs * 1e-6 : 0.);
  }
  if (pest_n >= 0) {
    double* v = (double*)malloc((size_t)(3 * pest_kept + 3) * sizeof(double));
    int taken = 0;
    LBX(lbx_pest_read(r.dom, v, v + pest_kept, v + 2 * pest_kept, &taken));
    if (lbh_write_pest("./out", pest_kept, v, v + pest_kept, v + 2 * pest_kept, pest_order,
                       r.prec))
      DIE("cannot write the PEST files in ./out");
    if (taken < pest_kept)
      fprintf(stderr, "warning: %d of %d PEST samples were not reached\n", pest_kept - taken,
              pest_kept);
    free(v);
    free(pest_order); free(pest_time); free(pest_node);
  }
  LBX(lbx_destroy(r.dom));
  free(r.mask); free(ntab); free(stab);
  return 0;
}
