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

/* ---- the reference's per-frame files (output_frame, src/lbio.c:37-131) ----
 * Frame statistics of one substance as compute_{max,min,ave}_{u,rho}
 * (src/compute.c:1159-1416) define them, over the nodes whose mask byte is
 * 0 (is_not_solid, src/lattice.c:163-194).  The library's device reduction
 * (lbx_frame_stats) fills the same fields. */
typedef struct lbh_frame_stats {
  long long nodes;
  double max_rho, min_rho, ave_rho;
  double max_u[3], min_u[3], ave_u[3];
} lbh_frame_stats;

/* Append one line to <outdir>/cuda_frames<size>[_subsNN].dat in the layout
 * of dump_frame_summary (src/lbio.c:140-290): a new file with its header at
 * time 0.  The flux columns are 0 (compute_flux has no body in the
 * reference's build, src/compute.c:1418-1467); the max/ave ratios are
 * formed in the run's precision (real_size 4 or 8).  Returns 0 or -1. */
int lbh_write_frame_summary(const char* path, int time, int real_size,
                            const lbh_frame_stats* st);

/* rho / ux / uy / uz text dump (write_rho_txt, write_u_txt, src/lbio.c:
 * 2864-2973): " %18.16f" per node, a newline per row, a blank line per
 * plane, every node (no mask).  a = NULL writes zeros (u_z of a 2D run).
 * Rows are formatted on all host cores.  Returns 0 or -1. */
int lbh_write_txt(const char* path, const void* a, int real_size, int LX, int LY, int LZ);

/* 3D byte images (write_raw and write_raw_u, src/lbio.c:934-1061): byte =
 * floor(1 + 254 (a - a_min) / (a_max - a_min)) converted as the reference's
 * build converts it, 0 where the mask byte is non-zero.  a_max / a_min are
 * the frame statistics (max and min of |a|).  write_raw_u images |u| with
 * the limits |(max_u)| and |(min_u)|.  Returns 0 or -1. */
int lbh_write_raw_image(const char* path, const void* a, int real_size, long long N,
                        const uint8_t* mask, double a_max, double a_min);
int lbh_write_raw_u(const char* path, const void* ux, const void* uy, const void* uz,
                    int real_size, int dims, long long N, const uint8_t* mask,
                    const double max_u[3], const double min_u[3]);

/* Every file output_frame writes for one frame into outdir: the summary
 * line per substance, in 3D the byte images rho, u, u_x, u_y, u_z, the .dat
 * files rho, u_x, u_y (u_z in 3D) and the text dumps rho, ux, uy, uz, under
 * the reference's names (lbh_frame_filename).  mv[s] holds substance s's
 * [1+D][N] reals, st[s] its statistics.  flags select the kinds (all four
 * are the reference's default build).  Returns 0 or -1. */
enum { LBH_FRAME_SUMMARY = 1, LBH_FRAME_RAW = 2, LBH_FRAME_DAT = 4, LBH_FRAME_TXT = 8,
       LBH_FRAME_ALL = 15 };
int lbh_write_frame(const char* outdir, int dims, int nsubs, int LX, int LY, int LZ,
                    int time, int frame, int real_size, const void* const* mv,
                    const lbh_frame_stats* st, const uint8_t* mask, unsigned flags);

/* PEST inputs (read_PEST_in_files, src/latman.c:899-1046):
 * <dir>/timestep_file.in, x_coord_file.in and y_coord_file.in, integers.
 * lbh_pest_count gives the number of samples by the reference's rule (a
 * value counts when a read is attempted before end-of-file was seen, so a
 * last value with no newline after it is not counted); -1 when the file is
 * missing or holds a non-integer.  lbh_read_pest reads `count` samples,
 * keeps those with 0 <= x < LX and 0 <= y < LY in file order, and returns
 * how many: order[k] (the sample's index in the files), time[k] and
 * node[k] = y*LX + x; -1 with a message for a missing file, too few values
 * or times that decrease (the reference exits there). */
int lbh_pest_count(const char* dir);
int lbh_read_pest(const char* dir, int LX, int LY, int count, int* order, int* time,
                  int* node, char* err, int errlen);

/* PEST outputs (write_PEST_out_file, src/latman.c:1178-1232):
 * <outdir>/conc_data_proc0000.dat and vel_data_proc0000.dat ("%20.17f" per
 * line) and conc_order_proc0000.dat ("%d").  vel = sqrt(u_x^2 + u_y^2)
 * formed in the run's precision (real_size) as the reference forms it;
 * samples not taken (NaN) are written as 0.  Returns 0 or -1. */
int lbh_write_pest(const char* outdir, int count, const double* conc, const double* ux,
                   const double* uy, const int* order, int real_size);

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

/* Initial density of substance `subs` per initial_condition 0 (uniform) or
 * 2 (cube) of init_problem (src/latman.c:1319-1632).  rho: N doubles.
 * Returns 0, or -1 for any other condition (the reference compiles only
 * these two and exits on the others). */
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
