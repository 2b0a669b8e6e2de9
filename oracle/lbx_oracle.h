/*
 * lbx_oracle.h -- parameters of the CPU restatement in lbx_oracle.c.
 * TEST INFRASTRUCTURE ONLY (see lbx_oracle.c).
 *
 * Field meanings follow the reference's params.in (src/params.h:40-660) and
 * the __constant__ block its kernels read (src/lattice.c:2224-2268).
 */
#ifndef LBX_ORACLE_H
#define LBX_ORACLE_H
#include <stdint.h>

typedef struct {
  int dims;                 /* 2 (D2Q9) or 3 (D3Q19) */
  int LX, LY, LZ;           /* LZ == 1 for dims == 2 */
  int nsubs;                /* 1 = flow; 2 = flow + solute (Inamuro sigma) */
  int accurate;             /* 1 = shifted populations d = f - w rho_A */
  int compressible;         /* 0 = He-Luo incompressible */
  double tau[2], rho_A[2], gaccel[6], sink;
  int sigma_t_on, sigma_t_off;
  /* 2D Zou-He / zero-gradient faces (src/bcs.c GPU branches) */
  int pressure_n_in[2], pressure_s_in[2], pressure_n_out[2], pressure_s_out[2];
  int zeroconcgrad_n, zeroconcgrad_s;
  double rho_in, rho_out, pfadd, pfmul;
  int bc_ramp_start, bc_ramp_stop;
  const double* pressure_n_table; int pressure_n_len;
  const double* pressure_s_table; int pressure_s_len;
  /* 3D faces: top = plane k = LZ-1, bottom = plane k = 0.  The reference
   * reads these flags (src/params.h:191-198, :282-307) but has no device
   * code for them: the rules restated here are the 2D kernels carried to
   * the z faces (parity unpinned). */
  int pressure_t_in[2], pressure_b_in[2], pressure_t_out[2], pressure_b_out[2];
  int constcon_t_in, constcon_b_in;   /* solute: C = rho_sigma_in on the face */
  int zeroconcgrad_t, zeroconcgrad_b;
  double rho_sigma_in;
  /* per-node concentration of a constant-concentration face (LX*LY, i
   * fastest), used instead of rho_sigma_in when not NULL */
  const double* constcon_profile_t;
  const double* constcon_profile_b;
  /* KAHAN_SUMMATION (src/flags.h:46-49): the flow's density sum is
   * compensated (fk_add, src/lattice.c:3099-3114) */
  int kahan;
  /* WALSH_NS_ON with COMPUTE_ON_SOLIDS (src/flags.h:56-63): every node is
   * updated, streaming ignores the solid flags, and the collision blends
   * with the opposite populations by the node's fraction ns[n] (N values)
   * (src/k_stream_collide_stream.c:129-215, :363-386; src/lattice.c:2704,
   * :2812, :2936) */
  int walsh;
  const double* ns;
  /* Zou-He velocity on the z faces (the reference's CPU formula,
   * src/bcs.c:764-862): top / bottom plane, u_z = uz_in for the *_in faces
   * and uz_out for the *_out faces, per substance */
  int velocity_t_in[2], velocity_t_out[2], velocity_b_in[2], velocity_b_out[2];
  double uz_in, uz_out;
  /* Complex-step build only (orc_*_cs): imaginary parts added to tau,
   * gaccel and the constant-concentration profiles, so that the imaginary
   * part of every result is h times its derivative along that direction
   * (h the size of these parts).  Ignored by the real builds. */
  double d_tau[2], d_gaccel[6];
  const double* d_profile_t;
  const double* d_profile_b;
} orc_params;

int orc_run_f64(const orc_params*, double* f, const uint8_t* solids,
                double* mv, int t0, int nsteps, int frame_rate,
                int nthreads);
int orc_run_f32(const orc_params*, float* f, const uint8_t* solids,
                float* mv, int t0, int nsteps, int frame_rate,
                int nthreads);
int orc_run_btc_f64(const orc_params*, double* f, const uint8_t* solids,
                    double* mv, int t0, int nsteps, int frame_rate,
                    int nthreads, int plane, double* btc, double* btc_ux);
int orc_run_btc_f32(const orc_params*, float* f, const uint8_t* solids,
                    float* mv, int t0, int nsteps, int frame_rate,
                    int nthreads, int plane, double* btc, double* btc_ux);
int orc_init_feq_f64(const orc_params*, const double* rho, const double* ux,
                     const double* uy, const double* uz, double* f);
int orc_init_feq_f32(const orc_params*, const float* rho, const float* ux,
                     const float* uy, const float* uz, float* f);
#ifdef LBX_ORACLE_CPLX
#include <complex.h>
/* The forward run in complex arithmetic (complex-step differentiation): f
 * and mv complex; btc and btc_ux hold 2*nsteps doubles, (real, imaginary)
 * per step. */
int orc_run_btc_cs(const orc_params*, double _Complex* f, const uint8_t* solids,
                   double _Complex* mv, int t0, int nsteps, int frame_rate,
                   int nthreads, int plane, double* btc, double* btc_ux);
int orc_run_cs(const orc_params*, double _Complex* f, const uint8_t* solids,
               double _Complex* mv, int t0, int nsteps, int frame_rate, int nthreads);
int orc_init_feq_cs(const orc_params*, const double _Complex* rho,
                    const double _Complex* ux, const double _Complex* uy,
                    const double _Complex* uz, double _Complex* f);
#endif
#endif
