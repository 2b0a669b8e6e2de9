/*
 * lbh.c -- params.in reader, mask decoders, initial density and frame
 * writers for the host driver (see lbh.h).  Plain C99, no device code.
 */
#include "lbh.h"

#include <ctype.h>
#include <math.h>
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
int lbh_initial_rho(const lbh_params* p, int dims, int nsubs, int subs, double* rho)
{
  long long n;
  const int LX = p->LX, LY = p->LY;
  for (n = 0; n < p->NumNodes; n++) {
    const int i = (int)(n % LX), j = (int)((n / LX) % LY), k = (int)(n / ((long long)LX * LY));
    const int in_box = i >= p->x1 && i <= p->x2 && j >= p->y1 && j <= p->y2 &&
                       (dims == 2 || (k >= p->z1 && k <= p->z2));
    const long long dx = i - p->x0, dy = j - p->y0, dz = k - p->z0;
    const int in_ball = dx * dx + dy * dy + dz * dz <= (long long)p->r0 * p->r0;
    switch (p->initial_condition) {
      case 0:
        rho[n] = (nsubs == 2 && subs == 1) ? p->rho_A[1].d : p->rho_A[subs].d;
        break;
      case 2:
        if (nsubs == 1) rho[n] = in_box ? p->rho_B[0].d : p->rho_A[0].d;
        else if (subs == 0) rho[n] = p->rho_A[0].d;
        else rho[n] = in_box ? p->rho_sigma.d : 0.;
        break;
      case 3:
        rho[n] = in_ball ? p->rho_A[subs].d : p->rho_B[subs].d;
        break;
      default:
        return -1;
    }
  }
  return 0;
}

/* ---- frame output --------------------------------------------------------- */
int lbh_write_dat(const char* path, const void* a, int real_size, long long N,
                  const uint8_t* mask)
{
  FILE* o = fopen(path, "wb");
  long long n;
  if (!o) return -1;
  for (n = 0; n < N; n++) {
    if (real_size == 8) {
      double v = mask[n] ? 0. : ((const double*)a)[n];
      fwrite(&v, 8, 1, o);
    } else {
      float v = mask[n] ? 0.f : ((const float*)a)[n];
      fwrite(&v, 4, 1, o);
    }
  }
  fclose(o);
  return 0;
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
