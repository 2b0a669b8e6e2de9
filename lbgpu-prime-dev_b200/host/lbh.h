/*
 * lbh.h -- host-side C library that keeps the reference's input/output
 * interface around the lbx C ABI: the positional params.in reader, the
 * .bmp/.raw solid-mask decoders, the initial density field, and the frame
 * writers.  The driver in lbgpu_main.c strings them together exactly as the
 * reference's main() does (src/lbgpu_prime.cu:82-940), with every device
 * call going through include/lbx.h.
 */
#ifndef LBH_H
#define LBH_H

#include <stdint.h>
#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One real-valued parameter as read: the double value and the float value
 * parsed from the same text, so a float run rounds the text once, as the
 * reference's "%f" scanf of a float `real` does (src/params.h:55). */
typedef struct { double d; float f; } lbh_real;

/* Everything src/params.h:40-660 reads, in file order.  Fields the
 * reference discards for a build are still read (the file is positional). */
typedef struct lbh_params {
  int LX, LY, LZ, BX, BY, BZ, length_scale, NumFrames, FrameRate;
  lbh_real tau[2], gforce[2][3];
  int end_grav[2];
  int buoyancy, incompressible, simple_diffusion;
  lbh_real rho_A[2], rho_B[2];
  lbh_real rho_sigma, rho_sigma_in, rho_sigma_out, u_sigma, u_sigma_in, u_sigma_out;
  int sigma_t_on, sigma_t_off, sigma_start, sigma_stop, sigma_btc_rate, sigma_btc_spot;
  int GZL, PressureBC, AllBoundaryPeriodic;
  lbh_real sink, pfmul, pfadd, rho_in, rho_out, ux_in, ux_out, uy_in, uy_out, uz_in, uz_out;
  lbh_real big_V0, big_V0_solid[2];
  int ns_flag;
  lbh_real ns;
  int ic_poisseuille, bc_poisseuille, bc_slip_north, bc_sigma_slip;
  int bc_ramp_start, bc_ramp_stop;
  /* per substance: t b (in/out) n s e w, pressure and velocity */
  int pressure_t_in[2], pressure_b_in[2], pressure_t_out[2], pressure_b_out[2];
  int velocity_t_in[2], velocity_b_in[2], velocity_t_out[2], velocity_b_out[2];
  int pressure_n_in[2], pressure_s_in[2], pressure_n_out[2], pressure_s_out[2];
  int velocity_n_in[2], velocity_s_in[2], velocity_n_out[2], velocity_s_out[2];
  int pressure_e_in[2], pressure_w_in[2], pressure_e_out[2], pressure_w_out[2];
  int velocity_e_in[2], velocity_w_in[2], velocity_e_out[2], velocity_w_out[2];
  int constcon[24];          /* constcon/constflx t b n s e w in/out      */
  int zeroconcgrad_t, zeroconcgrad_b, zeroconcgrad_n, zeroconcgrad_s;
  int zeroconcgrad_e, zeroconcgrad_w, zeroconcgrad_full;
  int plot_scale_dynamic, use_colormap, initial_condition;
  int x0, y0, z0, r0;        /* INTEGER_IC_BOUND build (the default)      */
  lbh_real cut;
  int x1, x2, y1, y2, z1, z2;
  lbh_real rel_x1, rel_x2, rel_y1, rel_y2, rel_z1, rel_z2;
  int dump_rho, dump_u, dump_force, dump_vor;
  /* derived, as read_params sets them (src/params.h:395-470) */
  long long NumNodes;
  int NumTimeSteps;
} lbh_params;

/* Read a positional params.in for a run with `dims` dimensions and `nsubs`
 * substances (NUM_DIMENSIONS / NUM_FLUID_COMPONENTS of the reference build).
 * Returns 0, or -1 with a message in `err` (missing file, short file). */
int lbh_read_params(const char* path, int dims, int nsubs, lbh_params* out,
                    char* err, int errlen);

/* The positional layout itself: the number of fields, and the name (the
 * lbh_params member, e.g. "tau[1]") and kind of field k in file order. */
int lbh_params_field_count(void);
const char* lbh_params_field(int k, int* is_real);

/* 24-bit BMP mask, black pixel -> 1, anything else -> 0, rows in file order
 * (bottom-up), as spy_bmp does (src/lbio.c:3073-3363).  out: LX*LY bytes.
 * Returns 0, or -1 (unreadable, not "BM", compressed, size mismatch, or a
 * bit depth other than 24) with a message in `err`. */
int lbh_read_bmp_mask(const char* path, int LX, int LY, uint8_t* out,
                      char* err, int errlen);

/* Raw mask: exactly N bytes copied verbatim (src/lbio.c:507-559). */
int lbh_read_raw_mask(const char* path, long long N, uint8_t* out,
                      char* err, int errlen);

/* Solid-flag rule.  The reference's device treats a mask byte as solid iff
 * it equals 1 (src/lattice.c:2291, :2314) while its frame writer blanks every
 * non-zero byte (src/lbio.c:2530-2540): a RAW mask that marks solids with
 * 255 runs them as fluid yet zeroes them in the output frames.
 * LBH_SOLID_DEVICE leaves the bytes as they are (parity with the reference);
 * LBH_SOLID_NONZERO maps every non-zero byte to 1, so the device and the
 * writer agree.  Returns the number of bytes whose meaning differs between
 * the two rules (non-zero bytes other than 1), counted before any change. */
enum { LBH_SOLID_DEVICE = 0, LBH_SOLID_NONZERO = 1 };
long long lbh_apply_solid_rule(uint8_t* mask, long long N, int rule);

/* Walsh fraction field ns (N doubles) for a WALSH_NS_ON run.
 * LBH_NS_MASK: ns = the params.in value `ns` where the mask byte is 1, else
 *   0 (process_ns, src/latman.c:48-80: the field the reference's 2D runs
 *   upload, src/lbgpu_prime.cu:259-264).
 * LBH_NS_FILE: ns = byte / 255 of the N-byte file `path` (read_ns,
 *   src/lbio.c:694-743, ./in/ns<LX>x<LY>x<LZ>.raw).
 * The value `ns` must lie in [0, 1] (src/latman.c:677-689).  Returns 0, or
 * -1 with a message in err. */
enum { LBH_NS_MASK = 0, LBH_NS_FILE = 1 };
int lbh_walsh_ns(double ns_value, int source, const uint8_t* mask, long long N,
                 const char* path, double* ns, char* err, int errlen);

/* Write a 24-bit BMP / raw mask in the same conventions (for generators). */
int lbh_write_bmp_mask(const char* path, int LX, int LY, const uint8_t* mask);
int lbh_write_raw_mask(const char* path, long long N, const uint8_t* mask);

/* Initial density of substance `subs` per initial_condition 0 (uniform),
 * 2 (cube) or 3 (sphere) of init_problem (src/latman.c:1319-1632).
 * rho: N doubles.  Returns 0, or -1 for an unsupported condition. */
int lbh_initial_rho(const lbh_params* p, int dims, int nsubs, int subs,
                    double* rho);

/* Frame output: the reference's .dat writer (binary reals, zero where the
 * mask byte is non-zero -- the host rule of src/lbio.c:2530-2540) under its
 * file names (src/lattice.c:371-452). */
int lbh_write_dat(const char* path, const void* a, int real_size, long long N,
                  const uint8_t* mask);
void lbh_frame_filename(char* buf, int buflen, const char* outdir,
                        const char* prefix, int dims, int LX, int LY, int LZ,
                        int frame, int nsubs, int subs, const char* suffix);

#ifdef __cplusplus
}
#endif
#endif
