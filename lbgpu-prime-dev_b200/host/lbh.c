/*
 * lbh.c -- params.in reader, mask decoders, initial density and frame
 * writers for the host driver (see lbh.h).  Plain C99, no device code.
 */
#include "lbh.h"

#include <ctype.h>
#include <math.h>
#include <pthread.h>
#include <unistd.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>

static void seterr(char* err, int errlen, const char* msg, const char* path)
{
  if (err && errlen > 0) snprintf(err, (size_t)errlen, "%s: %s", path ? path : "", msg);
}

/* ---- params.in -------------------------------------------------------------
 * The file is positional: each line is "label value" or a bare value, and a
 * label is skipped up to its first space and the spaces after it
 * (skip_label, src/params.h:13-31), after which scanf reads the value. */
static void skip_label(FILE* in)
{
  int c = fgetc(in);
  if ((c >= '0' && c <= '9') || c == '-' || c == '.') {
    ungetc(c, in);
    return;
  }
  while (c != EOF && (c = fgetc(in)) != ' ') {}
  while (c != EOF && (c = fgetc(in)) == ' ') {}
  if (c != EOF) ungetc(c, in);
}

/* F_INTW: read with "%d ", which also eats the whitespace after the value
 * (and so changes where the next skip_label starts). */
enum { F_INT, F_INTW, F_REAL };
typedef struct { int kind; size_t off; const char* name; } field_t;

#define I(member) { F_INT, offsetof(lbh_params, member), #member }
#define IW(member) { F_INTW, offsetof(lbh_params, member), #member }
#define R(member) { F_REAL, offsetof(lbh_params, member), #member }

/* File order of src/params.h:40-660 (INTEGER_IC_BOUND build). */
static const field_t FIELDS[] = {
  I(LX), I(LY), I(LZ), I(BX), I(BY), I(BZ), I(length_scale), I(NumFrames), I(FrameRate),
  R(tau[0]), R(gforce[0][0]), R(gforce[0][1]), R(gforce[0][2]), I(end_grav[0]),
  R(tau[1]), R(gforce[1][0]), R(gforce[1][1]), R(gforce[1][2]), I(end_grav[1]),
  IW(buoyancy), IW(incompressible), IW(simple_diffusion),
  R(rho_A[0]), R(rho_B[0]),
  R(rho_sigma), R(rho_sigma_in), R(rho_sigma_out), R(u_sigma), R(u_sigma_in), R(u_sigma_out),
  IW(sigma_t_on), IW(sigma_t_off), IW(sigma_start), IW(sigma_stop), IW(sigma_btc_rate),
  IW(sigma_btc_spot),
  IW(GZL), IW(PressureBC), IW(AllBoundaryPeriodic),
  R(sink), R(pfmul), R(pfadd), R(rho_in), R(rho_out), R(ux_in), R(ux_out), R(uy_in),
  R(uy_out), R(uz_in), R(uz_out), R(big_V0), R(big_V0_solid[0]), R(big_V0_solid[1]),
  I(ns_flag), R(ns), I(ic_poisseuille), I(bc_poisseuille), I(bc_slip_north),
  I(bc_sigma_slip), I(bc_ramp_start), I(bc_ramp_stop),
#define SUBS_BLOCK(s) \
  I(pressure_t_in[s]), I(pressure_b_in[s]), I(pressure_t_out[s]), I(pressure_b_out[s]), \
  I(velocity_t_in[s]), I(velocity_b_in[s]), I(velocity_t_out[s]), I(velocity_b_out[s]), \
  I(pressure_n_in[s]), I(pressure_s_in[s]), I(pressure_n_out[s]), I(pressure_s_out[s]), \
  I(velocity_n_in[s]), I(velocity_s_in[s]), I(velocity_n_out[s]), I(velocity_s_out[s]), \
  I(pressure_e_in[s]), I(pressure_w_in[s]), I(pressure_e_out[s]), I(pressure_w_out[s]), \
  I(velocity_e_in[s]), I(velocity_w_in[s]), I(velocity_e_out[s]), I(velocity_w_out[s])
  SUBS_BLOCK(0), SUBS_BLOCK(1),
#undef SUBS_BLOCK
  I(constcon[0]), I(constcon[1]), I(constcon[2]), I(constcon[3]), I(constcon[4]),
  I(constcon[5]), I(constcon[6]), I(constcon[7]), I(constcon[8]), I(constcon[9]),
  I(constcon[10]), I(constcon[11]), I(constcon[12]), I(constcon[13]), I(constcon[14]),
  I(constcon[15]), I(constcon[16]), I(constcon[17]), I(constcon[18]), I(constcon[19]),
  I(constcon[20]), I(constcon[21]), I(constcon[22]), I(constcon[23]),
  I(zeroconcgrad_t), I(zeroconcgrad_b), I(zeroconcgrad_n), I(zeroconcgrad_s),
  I(zeroconcgrad_e), I(zeroconcgrad_w), I(zeroconcgrad_full),
  I(plot_scale_dynamic), I(use_colormap), I(initial_condition),
  I(x0), I(y0), I(z0), I(r0), R(cut), I(x1), I(x2), I(y1), I(y2), I(z1), I(z2),
  R(rel_x1), R(rel_x2), R(rel_y1), R(rel_y2), R(rel_z1), R(rel_z2),
  I(dump_rho), I(dump_u), I(dump_force), I(dump_vor),
};
#undef I
#undef IW
#undef R

int lbh_params_field_count(void) { return (int)(sizeof FIELDS / sizeof FIELDS[0]); }

const char* lbh_params_field(int k, int* is_real)
{
  if (k < 0 || k >= lbh_params_field_count()) return NULL;
  if (is_real) *is_real = FIELDS[k].kind == F_REAL;
  return FIELDS[k].name;
}

static int read_token(FILE* in, char* buf, int len)
{
  int c, n = 0;
  do { c = fgetc(in); } while (c != EOF && isspace(c));
  while (c != EOF && !isspace(c) && n < len - 1) { buf[n++] = (char)c; c = fgetc(in); }
  if (c != EOF) ungetc(c, in);
  buf[n] = '\0';
  return n;
}

int lbh_read_params(const char* path, int dims, int nsubs, lbh_params* out,
                    char* err, int errlen)
{
  FILE* in;
  size_t k;
  char tok[256];
  memset(out, 0, sizeof *out);
  if (!(in = fopen(path, "r"))) { seterr(err, errlen, "cannot open", path); return -1; }
  for (k = 0; k < sizeof FIELDS / sizeof FIELDS[0]; k++) {
    char* base = (char*)out + FIELDS[k].off;
    char* end = NULL;
    skip_label(in);
    if (!read_token(in, tok, sizeof tok)) {
      fclose(in);
      snprintf(tok, sizeof tok, "file ends before field %d", (int)k + 1);
      seterr(err, errlen, tok, path);
      return -1;
    }
    if (FIELDS[k].kind != F_REAL) {
      *(int*)base = (int)strtol(tok, &end, 10);
      if (*end != '\0') end = tok;   /* "1.5" for an integer: reject */
      if (FIELDS[k].kind == F_INTW) {
        int c;
        while ((c = fgetc(in)) != EOF && isspace(c)) {}
        if (c != EOF) ungetc(c, in);
      }
    } else {
      lbh_real* r = (lbh_real*)base;
      r->d = strtod(tok, &end);
      r->f = strtof(tok, NULL);
    }
    if (end == tok) {
      fclose(in);
      seterr(err, errlen, "malformed value", path);
      return -1;
    }
  }
  fclose(in);
  /* derived values and defaults (src/params.h:395-470) */
  if (dims == 2) out->LZ = 1;
  out->NumNodes = (long long)out->LX * out->LY * out->LZ;
  out->NumTimeSteps = out->NumFrames * out->FrameRate;
  if (nsubs == 2) {
    if (out->sigma_t_on < 0) out->sigma_t_on = 0;
    if (out->sigma_t_off < 0) out->sigma_t_off = out->NumTimeSteps;
    out->rho_A[1] = out->rho_B[0];
    out->rho_B[1] = out->rho_A[0];
  }
  if (out->x0 < 0) out->x0 = out->LX / 2;
  if (out->y0 < 0) out->y0 = out->LY / 2;
  if (out->z0 < 0) out->z0 = out->LZ / 2;
  if (out->r0 < 0) {
    int m = out->LX < out->LY ? out->LX : out->LY;
    out->r0 = m < out->LZ ? m : out->LZ;
  }
  if (out->cut.d < 0.) { out->cut.d = 0.3; out->cut.f = 0.3f; }
#define REL(v, rel, L, dflt) \
  if (out->v < 0) out->v = (out->rel.d < 0.) ? (dflt) : (int)llround(out->rel.d * (double)(L));
  REL(x1, rel_x1, out->LX, out->LX / 4)
  REL(x2, rel_x2, out->LX, out->LX / 2)
  REL(y1, rel_y1, out->LY, out->LY / 4)
  REL(y2, rel_y2, out->LY, out->LY / 2)
  REL(z1, rel_z1, out->LZ, out->LZ / 4)
  REL(z2, rel_z2, out->LZ, out->LZ / 2)
#undef REL
  if (out->LX < 1 || out->LY < 1 || out->LZ < 1) {
    seterr(err, errlen, "lattice extents must be positive", path);
    return -1;
  }
  return 0;
}

/* ---- masks --------------------------------------------------------------- */
static int le32(const unsigned char* p) { return (int)(p[0] | p[1] << 8 | p[2] << 16 | (unsigned)p[3] << 24); }
static int le16(const unsigned char* p) { return (short)(p[0] | p[1] << 8); }

int lbh_read_bmp_mask(const char* path, int LX, int LY, uint8_t* out, char* err, int errlen)
{
  FILE* in;
  unsigned char hdr[54];
  int w, h, bits, row, pad, i, j;
  unsigned char* line;
  if (!(in = fopen(path, "rb"))) { seterr(err, errlen, "cannot open", path); return -1; }
  if (fread(hdr, 1, 54, in) != 54 || hdr[0] != 'B' || hdr[1] != 'M') {
    fclose(in); seterr(err, errlen, "not a BMP file", path); return -1;
  }
  w = le32(hdr + 18); h = le32(hdr + 22); bits = le16(hdr + 28);
  if (le32(hdr + 30) != 0) { fclose(in); seterr(err, errlen, "compressed BMP", path); return -1; }
  if (w != LX || h != LY) { fclose(in); seterr(err, errlen, "BMP size differs from LX x LY", path); return -1; }
  if (bits != 24) { fclose(in); seterr(err, errlen, "only 24-bit BMP masks are read", path); return -1; }
  row = 3 * w;
  pad = (4 - row % 4) % 4;
  line = (unsigned char*)malloc((size_t)(row + pad));
  if (!line) { fclose(in); seterr(err, errlen, "out of host memory reading", path); return -1; }
  /* pixel data follows the 54-byte header; rows bottom-up as stored */
  for (j = 0; j < h; j++) {
    size_t got = fread(line, 1, (size_t)(row + pad), in);
    if (got < (size_t)row) memset(line + got, 0xff, (size_t)(row - got));
    for (i = 0; i < w; i++) {
      const unsigned char* px = line + 3 * i;
      out[(long long)j * LX + i] = (px[0] == 0 && px[1] == 0 && px[2] == 0) ? 1 : 0;
    }
  }
  free(line);
  fclose(in);
  return 0;
}

int lbh_read_raw_mask(const char* path, long long N, uint8_t* out, char* err, int errlen)
{
  FILE* in;
  if (!(in = fopen(path, "rb"))) { seterr(err, errlen, "cannot open", path); return -1; }
  if ((long long)fread(out, 1, (size_t)N, in) != N) {
    fclose(in); seterr(err, errlen, "file holds fewer than LX*LY*LZ bytes", path); return -1;
  }
  fclose(in);
  return 0;
}

static void put32(unsigned char* p, unsigned v) { p[0] = v; p[1] = v >> 8; p[2] = v >> 16; p[3] = v >> 24; }

int lbh_write_bmp_mask(const char* path, int LX, int LY, const uint8_t* mask)
{
  FILE* o;
  unsigned char hdr[54];
  int row = 3 * LX, pad = (4 - row % 4) % 4, i, j;
  unsigned char* line = (unsigned char*)calloc(1, (size_t)(row + pad));
  if (!line) return -1;
  memset(hdr, 0, sizeof hdr);
  hdr[0] = 'B'; hdr[1] = 'M';
  put32(hdr + 2, 54u + (unsigned)(row + pad) * (unsigned)LY);
  put32(hdr + 10, 54); put32(hdr + 14, 40);
  put32(hdr + 18, (unsigned)LX); put32(hdr + 22, (unsigned)LY);
  hdr[26] = 1; hdr[28] = 24;
  put32(hdr + 34, (unsigned)(row + pad) * (unsigned)LY);
  if (!(o = fopen(path, "wb"))) { free(line); return -1; }
  fwrite(hdr, 1, 54, o);
  for (j = 0; j < LY; j++) {
    for (i = 0; i < LX; i++) {
      unsigned char v = mask[(long long)j * LX + i] ? 0 : 255;
      line[3 * i] = line[3 * i + 1] = line[3 * i + 2] = v;
    }
    fwrite(line, 1, (size_t)(row + pad), o);
  }
  free(line);
  fclose(o);
  return 0;
}

int lbh_write_raw_mask(const char* path, long long N, const uint8_t* mask)
{
  FILE* o = fopen(path, "wb");
  if (!o) return -1;
  fwrite(mask, 1, (size_t)N, o);
  fclose(o);
  return 0;
}

/* ---- initial density (src/latman.c:1319-1632, serial build) -------------- */
/* Only the uniform (0) and cube (2) cases are compiled in the reference; its
 * random (1) and sphere (3) cases sit inside #if 0, so init_problem prints
 * "Unhandled case" and exits for them (src/latman.c:1340-1376, :1507-1630),
 * and so does this function return -1. */
int lbh_initial_rho(const lbh_params* p, int dims, int nsubs, int subs, double* rho)
{
  long long n;
  const int LX = p->LX, LY = p->LY;
  if (p->initial_condition != 0 && p->initial_condition != 2) return -1;
  for (n = 0; n < p->NumNodes; n++) {
    const int i = (int)(n % LX), j = (int)((n / LX) % LY), k = (int)(n / ((long long)LX * LY));
    const int in_box = i >= p->x1 && i <= p->x2 && j >= p->y1 && j <= p->y2 &&
                       (dims == 2 || (k >= p->z1 && k <= p->z2));
    if (p->initial_condition == 0)
      rho[n] = p->rho_A[subs].d;
    else if (nsubs == 1)
      rho[n] = in_box ? p->rho_B[0].d : p->rho_A[0].d;
    else if (subs == 0)
      rho[n] = p->rho_A[0].d;
    else
      rho[n] = in_box ? p->rho_sigma.d : 0.;
  }
  return 0;
}

/* ---- frame output --------------------------------------------------------- */
int lbh_write_dat(const char* path, const void* a, int real_size, long long N,
                  const uint8_t* mask)
{
  const size_t bytes = (size_t)(N > 0 ? N : 1) * (size_t)real_size;
  char* buf = (char*)malloc(bytes);
  FILE* o;
  long long n;
  int rc = 0;
  if (!buf) return -1;
  if (real_size == 8) {
    double* v = (double*)buf;
    for (n = 0; n < N; n++) v[n] = mask[n] ? 0. : ((const double*)a)[n];
  } else {
    float* v = (float*)buf;
    for (n = 0; n < N; n++) v[n] = mask[n] ? 0.f : ((const float*)a)[n];
  }
  if (!(o = fopen(path, "wb"))) { free(buf); return -1; }
  if (N > 0 && fwrite(buf, (size_t)real_size, (size_t)N, o) != (size_t)N) rc = -1;
  if (fclose(o)) rc = -1;
  free(buf);
  return rc;
}

void lbh_frame_filename(char* buf, int buflen, const char* outdir, const char* prefix,
                        int dims, int LX, int LY, int LZ, int frame, int nsubs, int subs,
                        const char* suffix)
{
  char size[64], fr[32], sb[32];
  (void)LZ;
  if (dims == 2) snprintf(size, sizeof size, "%dx%d", LX, LY);
  else snprintf(size, sizeof size, "%dx%dx%d", LX, LY, LY);   /* sic: LY twice */
  if (frame >= 0) snprintf(fr, sizeof fr, "_frame%04d", frame); else fr[0] = '\0';
  if (nsubs == 1) sb[0] = '\0'; else snprintf(sb, sizeof sb, "_subs%02d", subs);
  snprintf(buf, (size_t)buflen, "%s/cuda_%s%s%s%s%s", outdir, prefix, size, fr, sb, suffix);
}

/* ---- per-frame files ---------------------------------------------------- */
int lbh_write_frame_summary(const char* path, int time, int real_size,
                            const lbh_frame_stats* st)
{
  FILE* o;
  double r[4];
  int c;
  if (time == 0) {
    static const char* cols[21] = {
      "time", "|j|", "j_x", "j_y", "j_z", "min_u[x]", "min_u[y]", "min_u[z]",
      "max_u[x]", "max_u[y]", "max_u[z]", "ave_u[x]", "ave_u[y]", "ave_u[z]",
      "max/ave[x]", "max/ave[y]", "max/ave[z]", "min_rho", "max_rho", "ave_rho", "max/ave"};
    if (!(o = fopen(path, "w+"))) return -1;
    fprintf(o, "\n");
    for (c = 0; c < 21; c++) fprintf(o, "%12s ", cols[c]);
    fprintf(o, "\n");
    for (c = 0; c < 21; c++) fprintf(o, "------------ ");
    fprintf(o, "\n");
    fclose(o);
  }
  if (!(o = fopen(path, "a+"))) return -1;
  /* max / ave in the run's precision, +inf beyond 9999 */
  for (c = 0; c < 4; c++) {
    const double mx = c < 3 ? st->max_u[c] : st->max_rho;
    const double av = c < 3 ? st->ave_u[c] : st->ave_rho;
    double q;
    if (real_size == 4) q = (float)av != 0.f ? (double)((float)mx / (float)av) : 1.;
    else q = av != 0. ? mx / av : 1.;
    r[c] = fabs(q) <= 9999. ? q : HUGE_VAL;
  }
#define LBH_R(x) (real_size == 4 ? (double)(float)(x) : (x))
  fprintf(o,
          "%12d "
          "%12.7f %12.7f %12.7f %12.7f"
          "%12.7f %12.7f %12.7f "
          "%12.7f %12.7f %12.7f "
          "%12.7f %12.7f %12.7f "
          "%12.7f %12.7f %12.7f "
          "%12.7f %12.7f %12.7f "
          "%12.7f\n",
          time, 0., 0., 0., 0.,
          LBH_R(st->min_u[0]), LBH_R(st->min_u[1]), LBH_R(st->min_u[2]),
          LBH_R(st->max_u[0]), LBH_R(st->max_u[1]), LBH_R(st->max_u[2]),
          LBH_R(st->ave_u[0]), LBH_R(st->ave_u[1]), LBH_R(st->ave_u[2]),
          r[0], r[1], r[2],
          LBH_R(st->min_rho), LBH_R(st->max_rho), LBH_R(st->ave_rho), r[3]);
#undef LBH_R
  fclose(o);
  return 0;
}

typedef struct {
  const void* a;
  int real_size, LX, LY;
  long long r0, r1;      /* rows [r0, r1), row r = j + LY k */
  char* buf;
  size_t len, cap;
  int fail;
} txt_job;

static void txt_put(txt_job* t, const char* s, size_t n)
{
  if (t->fail) return;
  if (t->len + n > t->cap) {
    size_t cap = t->cap ? t->cap : 4096;
    char* b;
    while (cap < t->len + n) cap *= 2;
    if (!(b = (char*)realloc(t->buf, cap))) { t->fail = 1; return; }
    t->buf = b; t->cap = cap;
  }
  memcpy(t->buf + t->len, s, n);
  t->len += n;
}

static void* txt_rows(void* arg)
{
  txt_job* t = (txt_job*)arg;
  char tmp[512];
  long long r;
  int i;
  for (r = t->r0; r < t->r1; r++) {
    const long long base = r * t->LX;
    for (i = 0; i < t->LX; i++) {
      double v = 0.;
      int n;
      if (t->a) v = t->real_size == 4 ? (double)((const float*)t->a)[base + i]
                                      : ((const double*)t->a)[base + i];
      n = snprintf(tmp, sizeof tmp, " %18.16f", v);
      if (n < 0) { t->fail = 1; return NULL; }
      if ((size_t)n < sizeof tmp) txt_put(t, tmp, (size_t)n);
      else {   /* magnitudes beyond 1e490 do not occur in a lattice; format in full */
        char* big = (char*)malloc((size_t)n + 1);
        if (!big) { t->fail = 1; return NULL; }
        snprintf(big, (size_t)n + 1, " %18.16f", v);
        txt_put(t, big, (size_t)n);
        free(big);
      }
    }
    txt_put(t, "\n", 1);
    if ((r + 1) % t->LY == 0) txt_put(t, "\n", 1);
  }
  return NULL;
}

int lbh_write_txt(const char* path, const void* a, int real_size, int LX, int LY, int LZ)
{
  const long long rows = (long long)LY * LZ;
  long ncpu = sysconf(_SC_NPROCESSORS_ONLN);
  int nt = (int)(ncpu > 0 ? (ncpu < 64 ? ncpu : 64) : 1), k, rc = 0;
  txt_job* jobs;
  pthread_t* th;
  FILE* o;
  if (rows < 1 || LX < 1) return -1;
  if (nt > rows) nt = (int)rows;
  jobs = (txt_job*)calloc((size_t)nt, sizeof *jobs);
  th = (pthread_t*)calloc((size_t)nt, sizeof *th);
  if (!jobs || !th) { free(jobs); free(th); return -1; }
  for (k = 0; k < nt; k++) {
    jobs[k].a = a; jobs[k].real_size = real_size; jobs[k].LX = LX; jobs[k].LY = LY;
    jobs[k].r0 = rows * k / nt; jobs[k].r1 = rows * (k + 1) / nt;
  }
  for (k = 1; k < nt; k++)
    if (pthread_create(&th[k], NULL, txt_rows, &jobs[k])) { jobs[k].fail = 2; txt_rows(&jobs[k]); }
  txt_rows(&jobs[0]);
  for (k = 1; k < nt; k++)
    if (jobs[k].fail != 2) pthread_join(th[k], NULL);
  o = fopen(path, "w+");
  if (!o) rc = -1;
  for (k = 0; k < nt; k++) {
    if (jobs[k].fail == 1) rc = -1;
    if (o && rc == 0 && jobs[k].len && fwrite(jobs[k].buf, 1, jobs[k].len, o) != jobs[k].len) rc = -1;
    free(jobs[k].buf);
  }
  if (o && fclose(o)) rc = -1;
  free(jobs); free(th);
  return rc;
}

/* The reference stores (unsigned char)ROUND(x) with ROUND = floor; its
 * build converts through a 32-bit integer and keeps the low byte, and a
 * value outside the int range (or NaN) becomes INT_MIN, low byte 0. */
static unsigned char raw_byte(double x)
{
  const double f = floor(x);
  if (!(f >= -2147483648.0 && f <= 2147483647.0)) return 0;
  return (unsigned char)((unsigned int)(int)f & 0xffu);
}

int lbh_write_raw_image(const char* path, const void* a, int real_size, long long N,
                        const uint8_t* mask, double a_max, double a_min)
{
  unsigned char* px = (unsigned char*)malloc((size_t)(N > 0 ? N : 1));
  long long n;
  FILE* o;
  int rc = 0;
  if (!px) return -1;
  for (n = 0; n < N; n++) {
    if (mask[n]) { px[n] = 0; continue; }
    if (real_size == 4) {
      const float v = ((const float*)a)[n], lo = (float)a_min, hi = (float)a_max;
      px[n] = raw_byte(1. + 254. * (v - lo) / (hi - lo));
    } else {
      const double v = ((const double*)a)[n];
      px[n] = raw_byte(1. + 254. * (v - a_min) / (a_max - a_min));
    }
  }
  if (!(o = fopen(path, "w"))) { free(px); return -1; }
  if (N > 0 && fwrite(px, 1, (size_t)N, o) != (size_t)N) rc = -1;
  if (fclose(o)) rc = -1;
  free(px);
  return rc;
}

int lbh_write_raw_u(const char* path, const void* ux, const void* uy, const void* uz,
                    int real_size, int dims, long long N, const uint8_t* mask,
                    const double max_u[3], const double min_u[3])
{
  unsigned char* px = (unsigned char*)malloc((size_t)(N > 0 ? N : 1));
  long long n;
  FILE* o;
  int rc = 0;
  if (!px) return -1;
  if (real_size == 4) {
    const float* x = (const float*)ux, *y = (const float*)uy, *z = (const float*)uz;
    const float mx0 = (float)max_u[0], mx1 = (float)max_u[1], mx2 = (float)max_u[2];
    const float mn0 = (float)min_u[0], mn1 = (float)min_u[1], mn2 = (float)min_u[2];
    const float hi = (float)sqrt(mx0 * mx0 + mx1 * mx1 + mx2 * mx2);
    const float lo = (float)sqrt(mn0 * mn0 + mn1 * mn1 + mn2 * mn2);
    for (n = 0; n < N; n++) {
      float m;
      if (mask[n]) { px[n] = 0; continue; }
      m = (float)sqrt(x[n] * x[n] + y[n] * y[n] + (dims == 2 ? 0.f : z[n] * z[n]));
      px[n] = raw_byte(1. + 254. * (m - lo) / (hi - lo));
    }
  } else {
    const double* x = (const double*)ux, *y = (const double*)uy, *z = (const double*)uz;
    const double hi = sqrt(max_u[0] * max_u[0] + max_u[1] * max_u[1] + max_u[2] * max_u[2]);
    const double lo = sqrt(min_u[0] * min_u[0] + min_u[1] * min_u[1] + min_u[2] * min_u[2]);
    for (n = 0; n < N; n++) {
      double m;
      if (mask[n]) { px[n] = 0; continue; }
      m = sqrt(x[n] * x[n] + y[n] * y[n] + (dims == 2 ? 0. : z[n] * z[n]));
      px[n] = raw_byte(1. + 254. * (m - lo) / (hi - lo));
    }
  }
  if (!(o = fopen(path, "w"))) { free(px); return -1; }
  if (N > 0 && fwrite(px, 1, (size_t)N, o) != (size_t)N) rc = -1;
  if (fclose(o)) rc = -1;
  free(px);
  return rc;
}

/* One file of a frame, for the worker pool of lbh_write_frame. */
typedef struct {
  int kind;                 /* 0 .dat, 1 byte image, 2 |u| byte image */
  char path[1024];
  const void* a[3];
  double hi, lo;
  const double* max_u;
  const double* min_u;
} frame_job;

typedef struct {
  frame_job* jobs;
  int njobs, next, fail;
  int real_size, dims;
  long long N;
  const uint8_t* mask;
  pthread_mutex_t lock;
} frame_pool;

static void* frame_worker(void* arg)
{
  frame_pool* P = (frame_pool*)arg;
  for (;;) {
    int i, rc = 0;
    frame_job* j;
    pthread_mutex_lock(&P->lock);
    i = P->next++;
    pthread_mutex_unlock(&P->lock);
    if (i >= P->njobs) return NULL;
    j = &P->jobs[i];
    if (j->kind == 0) rc = lbh_write_dat(j->path, j->a[0], P->real_size, P->N, P->mask);
    else if (j->kind == 1)
      rc = lbh_write_raw_image(j->path, j->a[0], P->real_size, P->N, P->mask, j->hi, j->lo);
    else
      rc = lbh_write_raw_u(j->path, j->a[0], j->a[1], j->a[2], P->real_size, P->dims, P->N,
                           P->mask, j->max_u, j->min_u);
    if (rc) {
      pthread_mutex_lock(&P->lock);
      P->fail = 1;
      pthread_mutex_unlock(&P->lock);
    }
  }
}

int lbh_write_frame(const char* outdir, int dims, int nsubs, int LX, int LY, int LZ,
                    int time, int frame, int real_size, const void* const* mv,
                    const lbh_frame_stats* st, const uint8_t* mask, unsigned flags)
{
  const long long N = (long long)LX * LY * LZ;
  const size_t plane = (size_t)N * (size_t)real_size;
  char fn[1024];
  int s, c, k, nt;
  static const char* dat[4] = {"rho", "u_x", "u_y", "u_z"};
  static const char* txt[4] = {"rho", "ux", "uy", "uz"};
  frame_job jobs[2 * 9];
  frame_pool P;
  pthread_t th[18];
  long ncpu = sysconf(_SC_NPROCESSORS_ONLN);
  memset(&P, 0, sizeof P);
  P.jobs = jobs; P.real_size = real_size; P.dims = dims; P.N = N; P.mask = mask;
  for (s = 0; s < nsubs && s < 2; s++) {
    const char* base = (const char*)mv[s];
    if (flags & LBH_FRAME_SUMMARY) {
      lbh_frame_filename(fn, sizeof fn, outdir, "frames", dims, LX, LY, LZ, -1, nsubs, s, ".dat");
      if (lbh_write_frame_summary(fn, time, real_size, &st[s])) return -1;
    }
    if ((flags & LBH_FRAME_RAW) && dims == 3) {
      frame_job* j = &jobs[P.njobs++];
      memset(j, 0, sizeof *j);
      j->kind = 1; j->a[0] = base; j->hi = st[s].max_rho; j->lo = st[s].min_rho;
      lbh_frame_filename(j->path, sizeof j->path, outdir, "rho", dims, LX, LY, LZ, frame, nsubs, s, ".raw");
      j = &jobs[P.njobs++];
      memset(j, 0, sizeof *j);
      j->kind = 2; j->a[0] = base + plane; j->a[1] = base + 2 * plane; j->a[2] = base + 3 * plane;
      j->max_u = st[s].max_u; j->min_u = st[s].min_u;
      lbh_frame_filename(j->path, sizeof j->path, outdir, "u", dims, LX, LY, LZ, frame, nsubs, s, ".raw");
      for (c = 1; c <= 3; c++) {
        j = &jobs[P.njobs++];
        memset(j, 0, sizeof *j);
        j->kind = 1; j->a[0] = base + c * plane; j->hi = st[s].max_u[c - 1]; j->lo = st[s].min_u[c - 1];
        lbh_frame_filename(j->path, sizeof j->path, outdir, dat[c], dims, LX, LY, LZ, frame, nsubs, s, ".raw");
      }
    }
    if (flags & LBH_FRAME_DAT)
      for (c = 0; c <= dims; c++) {
        frame_job* j = &jobs[P.njobs++];
        memset(j, 0, sizeof *j);
        j->kind = 0; j->a[0] = base + c * plane;
        lbh_frame_filename(j->path, sizeof j->path, outdir, dat[c], dims, LX, LY, LZ, frame, nsubs, s, ".dat");
      }
  }
  /* the binary files, one per worker at a time */
  nt = (int)(ncpu > 1 ? ncpu : 1);
  if (nt > P.njobs) nt = P.njobs;
  pthread_mutex_init(&P.lock, NULL);
  for (k = 1; k < nt; k++)
    if (pthread_create(&th[k], NULL, frame_worker, &P)) { nt = k; break; }
  if (P.njobs > 0) frame_worker(&P);
  for (k = 1; k < nt; k++) pthread_join(th[k], NULL);
  pthread_mutex_destroy(&P.lock);
  if (P.fail) return -1;
  /* the text dumps, each formatted on all cores */
  if (flags & LBH_FRAME_TXT)
    for (s = 0; s < nsubs; s++)
      for (c = 0; c < 4; c++) {
        lbh_frame_filename(fn, sizeof fn, outdir, txt[c], dims, LX, LY, LZ, frame, nsubs, s, ".txt");
        if (lbh_write_txt(fn, c <= dims ? (const char*)mv[s] + c * plane : NULL, real_size, LX,
                          LY, LZ))
          return -1;
      }
  return 0;
}

/* ---- PEST samples ----------------------------------------------------------- */
static FILE* pest_open(const char* dir, const char* name)
{
  char path[1024];
  snprintf(path, sizeof path, "%s/%s", dir, name);
  return fopen(path, "r");
}

int lbh_pest_count(const char* dir)
{
  FILE* in = pest_open(dir, "timestep_file.in");
  int v, count = 0, r;
  if (!in) return -1;
  r = fscanf(in, "%d", &v);
  while (!feof(in)) {
    if (r != 1) { fclose(in); return -1; }   /* a non-integer: the reference loops forever */
    count++;
    r = fscanf(in, "%d", &v);
  }
  fclose(in);
  return count;
}

static int pest_ints(const char* dir, const char* name, int count, int* out, char* err,
                     int errlen)
{
  FILE* in = pest_open(dir, name);
  int k;
  if (!in) { snprintf(err, (size_t)errlen, "cannot open %s/%s", dir, name); return -1; }
  for (k = 0; k < count; k++)
    if (fscanf(in, "%d", &out[k]) != 1) {
      fclose(in);
      snprintf(err, (size_t)errlen, "%s/%s holds fewer than %d integers", dir, name, count);
      return -1;
    }
  fclose(in);
  return 0;
}

int lbh_read_pest(const char* dir, int LX, int LY, int count, int* order, int* time,
                  int* node, char* err, int errlen)
{
  int* t = (int*)malloc((size_t)(count > 0 ? count : 1) * sizeof(int));
  int* x = (int*)malloc((size_t)(count > 0 ? count : 1) * sizeof(int));
  int* y = (int*)malloc((size_t)(count > 0 ? count : 1) * sizeof(int));
  int k, kept = -1;
  if (!t || !x || !y) { snprintf(err, (size_t)errlen, "out of host memory"); goto done; }
  if (pest_ints(dir, "timestep_file.in", count, t, err, errlen)) goto done;
  for (k = 1; k < count; k++)
    if (t[k] < t[k - 1]) {
      snprintf(err, (size_t)errlen, "PEST sample times not in order (sample %d)", k);
      goto done;
    }
  if (pest_ints(dir, "x_coord_file.in", count, x, err, errlen)) goto done;
  if (pest_ints(dir, "y_coord_file.in", count, y, err, errlen)) goto done;
  kept = 0;
  for (k = 0; k < count; k++) {
    if (y[k] < 0 || y[k] > LY - 1 || x[k] < 0 || x[k] > LX - 1) continue;
    order[kept] = k;
    time[kept] = t[k];
    node[kept] = y[k] * LX + x[k];
    kept++;
  }
done:
  free(t); free(x); free(y);
  return kept;
}

int lbh_write_pest(const char* outdir, int count, const double* conc, const double* ux,
                   const double* uy, const int* order, int real_size)
{
  char path[1024];
  FILE* o;
  int k;
  snprintf(path, sizeof path, "%s/conc_data_proc%04d.dat", outdir, 0);
  if (!(o = fopen(path, "w+"))) return -1;
  for (k = 0; k < count; k++) fprintf(o, "%20.17f\n", conc[k] == conc[k] ? conc[k] : 0.);
  fclose(o);
  snprintf(path, sizeof path, "%s/vel_data_proc%04d.dat", outdir, 0);
  if (!(o = fopen(path, "w+"))) return -1;
  for (k = 0; k < count; k++) {
    double v = 0.;
    if (ux[k] == ux[k] && uy[k] == uy[k]) {
      if (real_size == 4) {
        const float fx = (float)ux[k], fy = (float)uy[k];
        const float s2 = fx * fx + fy * fy;
        v = sqrt((double)s2);
      } else {
        v = sqrt(ux[k] * ux[k] + uy[k] * uy[k]);
      }
    }
    fprintf(o, "%20.17f\n", v);
  }
  fclose(o);
  snprintf(path, sizeof path, "%s/conc_order_proc%04d.dat", outdir, 0);
  if (!(o = fopen(path, "w+"))) return -1;
  for (k = 0; k < count; k++) fprintf(o, "%d\n", order[k]);
  fclose(o);
  return 0;
}

int lbh_walsh_ns(double ns_value, int source, const uint8_t* mask, long long N,
                 const char* path, double* ns, char* err, int errlen)
{
  long long n;
  if (source == LBH_NS_MASK) {
    if (!(ns_value >= 0. && ns_value <= 1.)) {
      snprintf(err, (size_t)errlen, "ns = %g: should have 0 <= ns <= 1", ns_value);
      return -1;
    }
    for (n = 0; n < N; n++) ns[n] = mask[n] == 1 ? ns_value : 0.;
    return 0;
  }
  if (source == LBH_NS_FILE) {
    uint8_t* raw = (uint8_t*)malloc((size_t)(N > 0 ? N : 1));
    if (!raw) { snprintf(err, (size_t)errlen, "out of host memory"); return -1; }
    if (lbh_read_raw_mask(path, N, raw, err, errlen)) { free(raw); return -1; }
    for (n = 0; n < N; n++) ns[n] = raw[n] / 255.0;
    free(raw);
    return 0;
  }
  snprintf(err, (size_t)errlen, "unknown ns source %d", source);
  return -1;
}

long long lbh_apply_solid_rule(uint8_t* mask, long long N, int rule)
{
  long long n, odd = 0;
  for (n = 0; n < N; n++) {
    if (mask[n] > 1) {
      ++odd;
      if (rule == LBH_SOLID_NONZERO) mask[n] = 1;
    }
  }
  return odd;
}
