/*
 * lbx.h -- C ABI of the B200-native lattice-Boltzmann hot path.
 *
 * This is the drop-in boundary for the reference's device path: the
 * in-place two-kernel (AA-pattern) update of src/k_stream_collide_stream.c
 * (odd times) and src/k_collide.c (even times), with halfway bounce-back at
 * solid nodes, the Zou-He pressure faces and the solute zero-gradient faces
 * of src/system_boundary_kernels.c, for D2Q9 and D3Q19 BGK flow and the
 * coupled solute (Inamuro sigma) lattice.
 *
 * Conventions (same as the reference's device data):
 *   - node index  n = i + LX*(j + LY*k)            (x fastest)
 *   - populations [subs][a][n], a in the reference's direction order
 *     (src/lbgpu_prime.h:82-84: opposites adjacent, a odd <-> a+1)
 *   - macro vars  [subs][0..D][n] = rho, ux, uy[, uz]  (src/lattice.c:2748)
 *   - solids      one byte per node; solid iff the byte == 1, the device
 *                 rule of src/lattice.c:2291/:2314 (255 counts as fluid)
 *   - real        double (precision 8) or float (precision 4)
 *   - times       the reference's: the step at an odd time is
 *                 stream-collide-stream, at an even time collide; a run
 *                 starts from the natural-order state at an even time.
 *
 * Every call returns LBX_OK (0) or an error code; lbx_last_error() gives a
 * message for the calling thread.  A domain handle is not thread-safe: use
 * one per host thread.  The library owns all device memory and a CUDA stream
 * per domain; host buffers are the caller's and are copied during the call.
 */
#ifndef LBX_H
#define LBX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int lbx_status;
enum {
  LBX_OK = 0,
  LBX_ERR_INVALID = 1,   /* bad argument or unsupported combination   */
  LBX_ERR_CUDA = 2,      /* a CUDA runtime call failed                 */
  LBX_ERR_NOMEM = 3,     /* device allocation failed                   */
  LBX_ERR_STATE = 4,     /* call out of order (AA parity, closed handle) */
  LBX_ERR_NUMERIC = 5    /* non-finite or negative density detected    */
};

/* Step flags. */
enum {
  LBX_WRITE_MV = 1u      /* store rho and u this step: is_end_of_frame_mem_c */
};

/* Parameters.  Field names and meanings are those of the reference's
 * params.in (src/params.h:40-660) and of the __constant__ block its kernels
 * read (src/lattice.c:2224-2268). */
typedef struct lbx_params {
  int dims;                 /* 2 (D2Q9) or 3 (D3Q19)                       */
  int LX, LY, LZ;           /* LZ must be 1 when dims == 2                 */
  int nsubs;                /* 1: flow; 2: flow + solute (sigma) lattice   */
  int precision;            /* 8 = double, 4 = float                       */
  int accurate;             /* ACCURATE: 1 = shifted populations f - w rho_A */
  int compressible;         /* COMPRESSIBLE: 0 = He-Luo incompressible     */
  double tau[2];            /* tau[0] flow, tau[1] solute                  */
  double rho_A[2];          /* reference density per substance             */
  double gaccel[6];         /* body acceleration gforce_{x,y,z}[subs]      */
  double sink;              /* solute sink coefficient                     */
  int sigma_t_on, sigma_t_off; /* solute active for sigma_t_on<=t<=sigma_t_off */
  /* 2D faces: north = row j=LY-1, south = row j=0 (src/bcs.c GPU code) */
  int pressure_n_in[2], pressure_s_in[2];    /* 1 = rho_in, 2 = table      */
  int pressure_n_out[2], pressure_s_out[2];  /* 1 = rho_out                */
  int zeroconcgrad_n, zeroconcgrad_s;        /* solute zero gradient       */
  double rho_in, rho_out;
  double pfadd, pfmul;      /* table density = pfadd + pfmul * table[t%len] */
  int bc_ramp_start, bc_ramp_stop;           /* < 0: no ramp               */
  const double* pressure_n_table; int pressure_n_len;
  const double* pressure_s_table; int pressure_s_len;
  int device;               /* CUDA device ordinal                         */
  int layout;               /* LBX_LAYOUT_*: device storage of populations */
  /* 3D faces: top = plane k=LZ-1, bottom = plane k=0.  The reference reads
   * these flags (src/params.h:191-198, :282-307) but has no device code for
   * them; here they are the 2D rules carried to the z faces: Zou-He density
   * with zero tangential velocity (the D3Q19 reconstruction of the
   * reference's CPU top/bottom code, src/bcs.c:596-870), the solute's
   * zero-gradient rule, and a constant solute concentration that sets the
   * face's unknown populations to w_a X with sum_a g_a = rho_sigma_in.
   * Applied before each step in the order t_in, t_out, b_in, b_out (per
   * substance), then constcon t/b, zeroconcgrad t/b; need LZ >= 3. */
  int pressure_t_in[2], pressure_b_in[2];    /* 1 = rho_in                 */
  int pressure_t_out[2], pressure_b_out[2];  /* 1 = rho_out                */
  int constcon_t_in, constcon_b_in;          /* solute C = rho_sigma_in    */
  int zeroconcgrad_t, zeroconcgrad_b;        /* solute zero gradient       */
  double rho_sigma_in;
  int kahan;                /* KAHAN_SUMMATION (src/flags.h:46-49): the flow's
                               density sums are compensated (fk_add,
                               src/lattice.c:3099-3114)                    */
  int walsh;                /* WALSH_NS_ON with COMPUTE_ON_SOLIDS
                               (src/flags.h:56-63): partial bounce-back by a
                               per-node fraction ns (lbx_set_ns, default 0);
                               every node is updated and streaming ignores
                               the solids.  Dense layout; no face
                               boundaries, batches or adjoint runs.        */
  /* Zou-He velocity on the z faces (3D; the reference's CPU rule,
   * src/bcs.c:764-862): the unknowns of the top (k = LZ-1) or bottom (k = 0)
   * plane from rho = (known sums) / (1 +- u_z) and J = rho u_z with zero
   * tangential velocity; u_z = uz_in on the *_in faces, uz_out on the *_out
   * faces (|u_z| < 1).  Ordered after the pressure faces of the same face
   * and substance (the last configured operation on a face decides). */
  int velocity_t_in[2], velocity_t_out[2], velocity_b_in[2], velocity_b_out[2];
  double uz_in, uz_out;
} lbx_params;

/* Device storage of the populations.  DENSE keeps the reference's
 * [subs][a][N] array; COMPACT stores fluid nodes only ([subs][a][F], dense
 * node order) and moves only the bytes of fluid nodes each step.  Both
 * compute the same results; uploads and downloads always use the dense
 * exchange format.  AUTO picks COMPACT when solids are at least 5% of the
 * nodes, DENSE otherwise. */
enum { LBX_LAYOUT_AUTO = 0, LBX_LAYOUT_DENSE = 1, LBX_LAYOUT_COMPACT = 2 };

typedef struct lbx_domain lbx_domain;

/* FP64 reductions over the current macro variables (see lbx_reduce). */
typedef struct lbx_reductions {
  double mass;              /* sum over fluid nodes of rho (subs 0)        */
  double solute_mass;       /* sum over fluid nodes of C (subs 1), else 0  */
  double momentum[3];       /* sum over fluid nodes of rho*u (subs 0)      */
  double u_sum[3];          /* sum over fluid nodes of u (subs 0)          */
  double rho_min, rho_max;  /* over fluid nodes (subs 0)                   */
  long long fluid_nodes;
  int nonfinite;            /* count of non-finite rho/u values seen       */
} lbx_reductions;

/* Fill `p` with the reference defaults: tau 1, rho_A 1, no force, no faces,
 * ramp off, double precision, shifted incompressible model. */
void lbx_params_default(lbx_params* p);

/* Allocate the device lattice and classify nodes from `solids`
 * (LX*LY*LZ bytes, host).  Replaces construct_lattice's device part:
 * the constant upload of src/latman.c:147-376, the cudaMalloc of
 * src/latman.c:461-493 and the solid upload of src/lbgpu_prime.cu:170-257. */
lbx_status lbx_create(const lbx_params* p, const uint8_t* solids,
                      lbx_domain** out);

/* Release everything.  Replaces src/latman.c:2144-2172 (device part). */
lbx_status lbx_destroy(lbx_domain* d);

/* Populations of one substance, [Q][N] reals in the reference's order.
 * Replaces the per-direction cudaMemcpy of src/lbgpu_prime.cu:316-343
 * (upload) and :874-900 (download).  Uploaded populations are the
 * natural-order state of an even time, so the next step must be at an odd
 * time (as after init_problem in the reference's main). */
lbx_status lbx_upload_f(lbx_domain* d, int subs, const void* f_host);
lbx_status lbx_download_f(lbx_domain* d, int subs, void* f_host);

/* Macro variables of one substance, [1+D][N] reals.  Replaces
 * src/lbgpu_prime.cu:345-350 (upload) and :544-583 / :765-804 (download:
 * rho, ux, uy[, uz]; uz may be NULL in 2D). */
lbx_status lbx_upload_mv(lbx_domain* d, int subs, const void* mv_host);
lbx_status lbx_download_mv(lbx_domain* d, int subs, void* rho, void* ux,
                           void* uy, void* uz);

/* Equilibrium initial state on the device from host rho/u ([N] reals each
 * for substance `subs`; uz is not read in 2D): the f = feq loop of
 * src/latman.c:1786-1840 (shifted deviations for the flow lattice of an
 * ACCURATE run, full feq otherwise).  Solid nodes are initialised too.
 * rho is required; a velocity component passed as NULL is zero (the
 * reference's init_problem always starts at rest), so the reference's
 * start moves one plane across the host link instead of Q.  The
 * substance's macro variables then hold rho and u, as init_problem leaves
 * them (src/latman.c:1302-1780). */
lbx_status lbx_init_equilibrium(lbx_domain* d, int subs, const void* rho,
                                const void* ux, const void* uy,
                                const void* uz);

/* One lattice step at `time`: the system boundaries of bcs_1 / bcs_2 and
 * then k_stream_collide_stream (odd time) or k_collide (even time).
 * Replaces src/lbgpu_prime.cu:490-530 (odd) and :722-752 (even).  Steps
 * must alternate odd/even starting from an odd time (LBX_ERR_STATE
 * otherwise).  Asynchronous: returns once the work is queued. */
lbx_status lbx_step(lbx_domain* d, int time, unsigned flags);

/* The pair of steps time, time+1 (time odd). */
lbx_status lbx_step_pair(lbx_domain* d, int time, unsigned flags);

/* Steps t0+1 .. t0+nsteps (t0 even), writing macro variables at every time
 * that is a multiple of frame_rate (frame_rate <= 0: never) -- the
 * is_end_of_frame rule of src/lattice.c:2094-2097.  Stretches of
 * frame-free steps with unchanged launch arguments are replayed from CUDA
 * graphs (one AA pair, or eight pairs per graph launch; captured on first
 * use and kept while the arguments and the stream stay the same).
 * Asynchronous. */
lbx_status lbx_run(lbx_domain* d, int t0, int nsteps, int frame_rate);

/* Run the domain's work on the caller's CUDA stream (a cudaStream_t passed
 * as void*; NULL is the CUDA default stream).  The domain uses a stream of
 * its own until the first call.  Lets a caller order lbx launches with its
 * own work and time them with its own events.  A compact-layout domain
 * with z faces also queues each step's face-plane launch on a second,
 * internal stream, forked from this stream by an event and joined back
 * into it before the step's later work: everything a step does is ordered
 * after the caller's earlier work on this stream and before its later
 * work, and a stream capture of lbx calls captures both streams. */
lbx_status lbx_set_stream(lbx_domain* d, void* stream);

/* How lbx_run advances a stretch of frame-free AA pairs whose launch
 * arguments do not change (no extension of the reference's interface: the
 * reference launches every step, src/lbgpu_prime.cu:517-527, :741-750).
 *   LBX_RUN_AUTO   (default) the tiled path where it applies and the lattice
 *                  is small enough for it to pay, else STEPS;
 *   LBX_RUN_STEPS  one launch per step, replayed from captured CUDA graphs;
 *   LBX_RUN_TILED  the tiled path wherever it applies: 2D, one substance, no
 *                  Walsh run, no plane record, faces absent or fused.  One
 *                  cooperative launch runs rounds of K steps (K = 6 in FP64,
 *                  10 in FP32) on tiles held in shared memory with halos K
 *                  deep; FP64 results are bit-identical to STEPS.
 * LBX_ERR_INVALID for another mode. */
enum { LBX_RUN_AUTO = 0, LBX_RUN_STEPS = 1, LBX_RUN_TILED = 2 };
lbx_status lbx_set_run_mode(lbx_domain* d, int mode);

/* Wait for all queued work of the domain; reports asynchronous errors. */
lbx_status lbx_sync(lbx_domain* d);

/* FP64 on-device conservation diagnostics over the macro variables last
 * written (a step with LBX_WRITE_MV): mass, momentum, solute mass, density
 * range and a non-finite count over device-rule fluid nodes (mask byte not
 * 1).  LBX_ERR_NUMERIC (with `out` filled) when a value is non-finite.
 * Synchronous. */
lbx_status lbx_reduce(lbx_domain* d, lbx_reductions* out);

/* The reductions of lbx_reduce for callers that cannot allocate device
 * memory -- a host program whose device memory is handed in full to its own
 * pool allocator, or one that must not add an allocation (which can
 * synchronize the device, or fail) to a time-critical loop.  No counterpart
 * in the reference.  mv ([nsubs][1+dims][N] reals) and solids (N bytes) are
 * device pointers the caller owns; the work is queued on `stream` (NULL: the
 * default stream) and the call waits for it.  Scratch lives in a fixed array
 * inside the library (384 KiB, held on every GPU that loads the library
 * until exit), so N is limited to 67,108,864 nodes (LBX_ERR_INVALID beyond).
 * The first call in a CUDA context (the device's primary context, or a
 * driver-API context the caller made current) looks up that array's device
 * address and keeps it for the context; make it before any stream capture.
 * A cudaDeviceReset between calls is not supported: the kept address would
 * outlive the context it belongs to.  Calls share the array: calls that
 * overlap on the GPU race.  Allocates nothing: no cudaMalloc, cudaFree or allocating
 * library call. */
lbx_status lbx_reduce_mv_static(const void* mv, const uint8_t* solids,
                                long long N, int dims, int nsubs, int precision,
                                void* stream, lbx_reductions* out);

/* ---- frame output ---------------------------------------------------------
 * The statistics the reference's output_frame reports per substance
 * (compute_{max,min,ave}_{u,rho}, src/compute.c:1159-1416, written by
 * dump_frame_summary, src/lbio.c:140-290): over the nodes whose mask byte
 * is 0 (the host rule, is_not_solid, src/lattice.c:163-194), the max and
 * min of |rho| and |u_c| and the means of rho and u_c; u_z is 0 in 2D.  A
 * NaN never replaces a running max or min (as in the reference); sums are
 * FP64 on the device, in a fixed order (reproducible). */
typedef struct lbx_frame_stats {
  long long nodes;
  double max_rho, min_rho, ave_rho;
  double max_u[3], min_u[3], ave_u[3];
} lbx_frame_stats;

/* Statistics of substance `subs` from the macro variables last written.
 * Synchronous. */
lbx_status lbx_frame_stats_compute(lbx_domain* d, int subs, lbx_frame_stats* out);

/* Asynchronous frame output.  lbx_frame_enqueue, called after a step with
 * LBX_WRITE_MV, queues on the domain's stream the statistics of every
 * substance and a device-side snapshot of the macro variables, then copies
 * both to page-locked host memory on a second stream, and returns at once:
 * the copies overlap the steps queued after it, and no later step waits
 * for them (replaces the synchronous per-frame cudaMemcpy and
 * cudaThreadSynchronize of src/lbgpu_prime.cu:544-583, :765-804).
 * lbx_frame_wait blocks until the oldest queued frame has landed and
 * returns it; its mv pointers ([1+D][N] reals per substance, page-locked)
 * stay valid until the second lbx_frame_enqueue after the wait.  At most
 * two frames are outstanding (LBX_ERR_STATE beyond); lbx_frame_wait with
 * none outstanding is LBX_ERR_STATE.  The first enqueue allocates two
 * device and three host buffers of the macro variables' size (the third
 * keeps a returned frame's view alive through the next enqueue when two
 * frames were outstanding at its wait). */
typedef struct lbx_frame {
  int time;
  int nsubs;
  const void* mv[2];
  lbx_frame_stats stats[2];
} lbx_frame;

lbx_status lbx_frame_enqueue(lbx_domain* d, int time);
lbx_status lbx_frame_wait(lbx_domain* d, lbx_frame* out);

/* PEST point sampling (PEST_OUTPUT_ON, src/latman.c:899-1232): `count`
 * samples in time order (time[k] non-decreasing, node[k] = y*LX + x as the
 * reference indexes them).  A step whose time is the next untaken sample's
 * writes the macro variables and stores, for every sample due then, the
 * solute's C and the flow's u_x and u_y at its node on the device.  As in
 * the reference a sample whose time never comes (earlier than the run, or
 * already passed) leaves it and every later sample untaken.  Needs
 * nsubs = 2 (the reference reads the solute).  count = 0 clears. */
lbx_status lbx_pest_set(lbx_domain* d, int count, const int* time, const int* node);
/* The samples so far (arrays of `count`; NaN where not taken) and the
 * number taken.  Synchronous. */
lbx_status lbx_pest_read(lbx_domain* d, double* conc, double* ux, double* uy, int* taken);

/* Device pointers to the populations ([nsubs][Q][N], the dense exchange
 * format; with the compact layout this first writes the current state into
 * it, and the pointer is valid until the next step) and macro variables
 * ([nsubs][1+D][N]) for callers that keep data on the device. */
lbx_status lbx_device_f(lbx_domain* d, void** ptr);
lbx_status lbx_device_mv(lbx_domain* d, void** ptr);

/* Counts from classification: fluid nodes, whether the 2D face boundaries
 * run fused into the step kernels (1) or as separate kernels (0), and the
 * layout in use (LBX_LAYOUT_DENSE or LBX_LAYOUT_COMPACT). */
lbx_status lbx_info(lbx_domain* d, long long* fluid_nodes, int* faces_fused,
                    int* layout);

/* Number of this library's kernels launched on the domain so far. */
long long lbx_launch_count(lbx_domain* d);

/* Plane record: from the next step on, every step appends the means over
 * the fluid nodes of `plane` -- the plane k = plane in 3D, the row j = plane
 * in 2D -- of the solute concentration C (NaN for a step with no active
 * solute) and of the flow velocity u_x, summed in FP64 on the device.  The
 * C channel is the breakthrough curve at that plane.  Holds up to
 * `capacity` steps; restarting clears it.  No counterpart in the reference,
 * whose observables are the per-frame dumps of src/lbio.c:2507-2562. */
lbx_status lbx_btc_start(lbx_domain* d, int plane, int capacity);

/* Copy up to `max` recorded steps (oldest first) into `c_out` (C means) and
 * `ux_out` (u_x means), either may be NULL, and the number of steps recorded
 * since lbx_btc_start into `*count` (which may exceed capacity; later steps
 * are then not stored).  Synchronizes the stream. */
lbx_status lbx_btc_read(lbx_domain* d, double* c_out, double* ux_out, int max,
                        long long* count);

/* Constant-concentration face with a per-node concentration: `conc` holds
 * LX*LY values (i fastest) for the top (top != 0) or bottom face, used
 * instead of rho_sigma_in; NULL returns to rho_sigma_in.  Copied. */
lbx_status lbx_set_face_profile(lbx_domain* d, int top, const double* conc);

/* Walsh runs (params.walsh = 1): the per-node solid fraction ns, N values in
 * dense node order, each in [0, 1], stored in the run's precision (the
 * reference's ns_mem_d, src/lbgpu_prime.cu:259-264, filled from ns_memblock:
 * src/latman.c:48-80 sets ns where the mask is solid and 0 elsewhere,
 * src/lbio.c:694-743 reads byte/255 from a .raw file).  LBX_ERR_STATE for a
 * domain created without walsh, LBX_ERR_INVALID for a value outside [0, 1]. */
lbx_status lbx_set_ns(lbx_domain* d, const double* ns);

/* Stop recording and release the record. */
lbx_status lbx_btc_stop(lbx_domain* d);

/* ---- Discrete adjoint (no counterpart in the reference) -----------------
 * Objective over a plane (k in 3D, j in 2D), averaged over the steps
 * t_first..t_last:
 *   J = w_c  * mean_t (mean over the plane's fluid nodes of the solute C)
 *     + w_ux * mean_t (mean over the plane's fluid nodes of the flow u_x),
 * with C and u the values the steps compute (those lbx_btc_* records).
 * lbx_adjoint_forward runs `nsteps` steps from the current natural-order
 * state at even time t0 (as lbx_run does), storing the state every
 * `checkpoint_every` steps on the device, and returns J.
 * lbx_adjoint_backward then runs the reverse stream-collide sweep,
 * recomputing each checkpoint interval, and returns dJ/d(gaccel[0..2]),
 * dJ/dtau[0], dJ/dtau[1] and, when the arrays are given, dJ/d(profile) of
 * the bottom / top constant-concentration faces (LX*LY values, i fastest;
 * lbx_set_face_profile).  Adjoint populations are in the run's precision;
 * gradient sums are FP64.  Covers the compact layout, the shifted
 * incompressible model, flow + solute with the solute's z faces; other
 * configurations are rejected with LBX_ERR_INVALID. */
typedef struct lbx_objective {
  int plane;
  int t_first, t_last;
  double w_c, w_ux;
} lbx_objective;

typedef struct lbx_gradient {
  double J;
  double d_gaccel[3];       /* flow body force */
  double d_tau;             /* tau[0] */
  double d_tau_s;           /* tau[1] */
} lbx_gradient;

lbx_status lbx_adjoint_forward(lbx_domain* d, int t0, int nsteps, int checkpoint_every,
                               const lbx_objective* obj, double* J);
lbx_status lbx_adjoint_backward(lbx_domain* d, lbx_gradient* out, double* d_profile_b,
                                double* d_profile_t);

/* ---- batches of independent lattices ---------------------------------------
 * Many samples of uneven size (same dims, precision and collision model;
 * each with its own extents, mask, tau, rho_A and body force; one substance;
 * no face boundaries) stepped together: the reference runs one lattice per
 * process, so a study over many samples pays one set of launches per sample
 * and step.  Populations of all samples share one compact fluid-only array;
 * lbx_batch_run then advances every sample with one launch per step
 * (FUSED, graph-replayed), with one cooperative launch per run of steps
 * (PERSISTENT), or with one launch per sample per step (SEQUENTIAL, the
 * per-sample baseline).  AUTO uses the mode lbx_batch_autotune chose
 * (FUSED before any tuning).  Results are per sample identical to running
 * the sample alone. */
typedef struct lbx_batch lbx_batch;
enum { LBX_BATCH_AUTO = 0, LBX_BATCH_FUSED = 1, LBX_BATCH_PERSISTENT = 2,
       LBX_BATCH_SEQUENTIAL = 3 };

lbx_status lbx_batch_create(int nsamples, const lbx_params* params,
                            const uint8_t* const* solids, lbx_batch** out);
lbx_status lbx_batch_destroy(lbx_batch* b);
/* Per sample, dense [Q][N] populations (the natural-order state of an even
 * time) and [1+D][N] macro variables, as for a domain. */
lbx_status lbx_batch_upload_f(lbx_batch* b, int sample, const void* f_host);
lbx_status lbx_batch_download_f(lbx_batch* b, int sample, void* f_host);
lbx_status lbx_batch_download_mv(lbx_batch* b, int sample, void* rho, void* ux,
                                 void* uy, void* uz);
lbx_status lbx_batch_init_equilibrium(lbx_batch* b, int sample, const void* rho,
                                      const void* ux, const void* uy,
                                      const void* uz);
/* Steps t0+1 .. t0+nsteps of every sample, macro variables at multiples of
 * frame_rate, in `mode` (LBX_BATCH_*). */
lbx_status lbx_batch_run(lbx_batch* b, int t0, int nsteps, int frame_rate, int mode);
/* Times FUSED at block sizes 128/256 and PERSISTENT at the full and half
 * resident grid, each in every sample order below, on `steps` trial steps;
 * restores the populations and keeps the fastest mode, block size and
 * order (AUTO then uses that mode). */
lbx_status lbx_batch_autotune(lbx_batch* b, int steps, int* mode, int* block);
/* Order of the samples in the batch's compact population array (the order
 * of its thread blocks): largest first (the default; the last blocks of a
 * step are small ones), interleaved (largest, smallest, second largest,
 * ...) or as given.  Setting another order rebuilds the batch's tables and
 * moves the populations; results are the same in every order.  No
 * counterpart in the reference, which runs one lattice. */
enum { LBX_BATCH_LAYOUT_LARGEST_FIRST = 0, LBX_BATCH_LAYOUT_INTERLEAVED = 1,
       LBX_BATCH_LAYOUT_GIVEN = 2 };
lbx_status lbx_batch_set_layout(lbx_batch* b, int layout);
lbx_status lbx_batch_get_layout(lbx_batch* b, int* layout);
lbx_status lbx_batch_set_stream(lbx_batch* b, void* stream);
lbx_status lbx_batch_sync(lbx_batch* b);
/* FP64 reductions over one sample's macro variables (as lbx_reduce). */
lbx_status lbx_batch_reduce(lbx_batch* b, int sample, lbx_reductions* out);
long long lbx_batch_launch_count(lbx_batch* b);

/* Message for the last failed call on this thread ("" if none). */
const char* lbx_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* LBX_H */
