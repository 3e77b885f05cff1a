/*
 * kmm.h - C ABI of libkmm, a B200 (sm_100a) implementation of one RK3 time step of the
 * PoongBack Kim-Moin-Moser channel solver with a passive scalar (yaojieuh/CHANNEL_PASSIVE).
 *
 * The ABI is plain C: pointers, sizes and int status codes, no C++ or torch types.  It is
 * what the reference's Fortran driver (main.f90) would bind through ISO_C_BINDING in place of
 * its own routines; every entry point names the reference routine it replaces.
 *
 * Array conventions (shared with the reference):
 *   complex arrays are interleaved (re, im) doubles, Fortran column-major:
 *     state   U(ny, nxh, nz, nf)        -> element (y, kx, kz, f) at 2*(y + ny*(kx + nxh*(kz + nz*f)))
 *     stores  RK_STORE(ny, nxh, nz, 3)
 *     X-pencil Up(nxh, nz32, ny)        (dft_x_realspace.f90:31)
 *   band matrices are real (2*bw+1, ny) in the reference's near-boundary packed form
 *   (module_labs.f90:301-328).
 * Wavenumber order: kx = 0..nx/2-1; kz = 0..nz/2, -nz/2+1..-1 (module_ppdfftw.f90:347-384).
 *
 * Status codes: 0 = success; nonzero = failure with a message from kmm_last_error().  The
 * reference aborts through mpi_abort on the same conditions (read_input_file.f90:230-238,
 * dft_x_realspace.f90:494-497); a Fortran shim converts a nonzero status into mpi_abort.
 */
#ifndef KMM_H
#define KMM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KMM_OK 0
#define KMM_ERR_CONFIG 1      /* invalid configuration (read_input_file.f90:146-228 checks) */
#define KMM_ERR_CUDA 2        /* CUDA runtime error or no device */
#define KMM_ERR_DT 3          /* dt <= 1e-14 or dt > 1e5 (dft_x_realspace.f90:494-497) */
#define KMM_ERR_NONFINITE 4   /* NaN / Inf in the velocity maximum or in uploaded state */
#define KMM_ERR_ARG 5         /* null pointer, bad substep, size mismatch */
#define KMM_ERR_TIMEOUT 6     /* a bounded device wait gave up (a TMA tile copy of the z transforms) */
#define KMM_ERR_IO 7          /* checkpoint file: unreadable, missing dataset, unexpected shape or
                                 type (the checks of module_hdf5_io.f90:212-345, same messages) */

#define KMM_PREC_FP64 0       /* every kernel in FP64 */
#define KMM_PREC_MIXED 1      /* FP32 transforms/products, FP64 state, v-influence and mean modes */

#define KMM_GRID_SINE 0       /* the reference's breakpoint map (labs_fill_full.cpp:92) */
#define KMM_GRID_TANH 1       /* the commented tanh map (labs_fill_full.cpp:89) */

/* Mirrors the positional `input` file read by read_input_file.f90:38-89, plus the
 * switches this implementation adds (fixed dt, precision, opposition control). */
typedef struct kmm_config {
  int32_t nx, ny, nz;         /* modes in x, collocation points in y, modes in z */
  int32_t no_of_field;        /* must be 10 (fields 1..10 are used, wavespace.f90:29) */
  int32_t rk_scheme;          /* must be 3 (read_input_file.f90:190-195) */
  int32_t labs_k;             /* B-spline order minus one (GSL order = labs_k+1) */
  double lmfx, lmfy, lmfz;    /* Lx = 2 pi lmfx, Ly = 2 lmfy, Lz = 2 pi lmfz */
  double stretch;             /* breakpoint stretching factor */
  int32_t grid;               /* KMM_GRID_SINE or KMM_GRID_TANH */
  double nu, pr;              /* viscosity, Prandtl number */
  double bulk_vel_u, bulk_vel_w, bulk_t; /* target bulk U, W and theta */
  double u_gal;               /* Galilean shift of the mean flow */
  double cfl, dt_factor, dy_factor;      /* CFL number, dt relaxation, dy safety factor */
  int32_t fixed_dt;           /* 0: dt from the CFL rule each step (reference); 1: dt held */
  int32_t precision;          /* KMM_PREC_FP64 or KMM_PREC_MIXED */
  double control_amp;         /* opposition control amplitude A; 0 = no control (reference) */
  double control_yd;          /* detection plane y_d (-1 < y_d < 0); mirrored at the top wall */
  int32_t device;             /* CUDA device ordinal */
  int32_t n_scalar;           /* passive scalars: 1 (the reference; 0 reads as 1) or 2 */
  double pr2;                 /* Prandtl number of the second scalar */
  double bulk_t2;             /* target bulk value of the second scalar */
  int32_t autotune;           /* 1: kmm_create runs kmm_autotune before it returns */
  int32_t reserved;
} kmm_config;

/* Per-step diagnostics printed by main.f90:147-151. */
typedef struct kmm_scalars {
  double dt;                  /* time step used by the last substep */
  double velmax;              /* max(|u| dxr + |v| dyr + |w| dzr) of the last substep 1 */
  double phi_dpdx[4];         /* mean forcing per substep; [3] = sum/dt after a full step */
  double phi_dtdx[4];         /* scalar forcing per substep; [3] = sum/dt after a full step */
  double wall_shear_stress;   /* 0.5 nu (dU/dy|bottom - dU/dy|top), substep 3 */
  double wall_theta_stress;   /* 0.5 nu/pr (dT/dy|bottom - dT/dy|top), substep 3 */
  double phi_dtdx2[4];        /* the second scalar's forcing (n_scalar = 2), as phi_dtdx */
  double wall_theta_stress2;  /* the second scalar's wall flux, 0.5 nu/pr2 (dT2/dy|bottom - top) */
} kmm_scalars;

typedef struct kmm_info {
  int32_t bw;                 /* LABS band half-width detected by LABS_eval_bw */
  int32_t nxh, nx32, nz32;
  int64_t nmodes;             /* nxh * nz */
  int64_t device_bytes;       /* HBM held by the handle */
  int32_t fft_radix_x[8];     /* radix passes of the x transform (0-terminated) */
  int32_t fft_radix_z[8];
} kmm_info;

/* Launch shapes chosen by kmm_autotune (the hand-tuned defaults before it runs), and the
 * measured device time (ms) of every candidate it tried. */
typedef struct kmm_tuning {
  int32_t z_lines_per_block;  /* z transforms (y_to_x, x_to_y): kx lines a block transforms */
  int32_t x_rows_per_block;   /* x pass (dft_x_realspace): z rows a block takes */
  int32_t x_threads;          /*   and its threads */
  int32_t modes_per_block;    /* (kx, kz) systems a block of the hvhg solver takes (32, 64) */
  int32_t u_layout;           /* U factor storage: 0 = [offset][y][mode], 1 = [y][offset][mode] */
  int32_t assemble_threads;   /* threads per block of the C1/C2 assembly */
  int32_t tuned;              /* 1 once kmm_autotune has run */
  int32_t tables_shared;      /* 1: the hvhg solver copies the B-spline operator tables it reads
                                 into shared memory first */
  int32_t helm_modes_per_block;  /* systems a block of the Helmholtz solver takes (32, 64, 128;
                                    32, 64, 96 with two scalars) */
  int32_t helm_tables_shared;    /* 1: the Helmholtz solver reads the tables from shared memory */
  int32_t helm_stage_ahead;      /* rows its sweeps stage ahead through shared memory (1, 2) */
  int32_t z_tma;              /* 1: the z transforms stage each block's input tile through TMA
                                 (cp.async.bulk.tensor into shared memory) */
  int32_t hvhg_stage_ahead;   /* rows the hvhg sweeps stage ahead through shared memory (0: they
                                 prefetch into L1 instead; 1, 2) */
  int32_t factor_cache;       /* 1 (fixed time step, one scalar; the default there): the Helmholtz
                                 sweeps read each substep's operator factors and influence
                                 solutions, computed once for the current dt (again after dt
                                 changes) instead of every substep; same numbers.  0 elsewhere */
  double ms_z[3];             /* zinv + zfwd per z variant */
  double ms_x[3];             /* x pass per x variant */
  double ms_modes[2];         /* hvhg at 32 and 64 modes per block (best tables choice) */
  double ms_layout[2];        /* Helmholtz per U layout */
  double ms_assemble[3];      /* assembly at 128, 256, 512 threads */
  double ms_tables[2];        /* hvhg with the tables read through L1 / from shared memory */
  double ms_helm[12];         /* Helmholtz at [32, 64, 128 modes][tables via L1, shared]
                                 [look-ahead 1, 2] (row-major; 0 where a shape does not fit) */
  double ms_z_tma[3];         /* zinv + zfwd per z variant with TMA-staged input tiles (0 where
                                 the grid does not allow them) */
  double ms_hvhg[12];         /* hvhg at [32, 64 modes][tables via L1, shared][staging 0, 1, 2
                                 rows] (row-major; 0 where a shape was not timed) */
  double ms_step[2];          /* one step through the step graph with the shapes kept, and with
                                 the shapes the handle had before tuning: each knob group keeps
                                 its per-kernel pick only where the step gets 1% faster with it (0
                                 where a step could not run: the CFL rule on a zero state; the
                                 entry shapes then stay) */
} kmm_tuning;

typedef struct kmm_handle kmm_handle;

/* Thread-local text of the last failure. */
const char *kmm_last_error(void);

/* Fills the reference defaults (single rank, Re_tau 180 style channel). */
int kmm_config_default(kmm_config *cfg);

/* Parses the positional `input` text file (read_input_file.f90:38-89) into cfg. */
int kmm_read_input_file(const char *path, kmm_config *cfg);

/* LABS_initialize + RK3_initialize + ppdfftw_initialize (module_labs.f90:77-238,
 * module_runge_kutta.f90:28-54, module_ppdfftw.f90:499-588): builds the B-spline
 * operators, allocates the HBM-resident state and plans the transforms. */
int kmm_create(const kmm_config *cfg, kmm_handle **out);
int kmm_destroy(kmm_handle *h);
int kmm_get_info(const kmm_handle *h, kmm_info *info);

/* Host copies of the operators: y(ny), integration weights(ny), bands (2bw+1, ny) each. */
int kmm_get_operators(const kmm_handle *h, double *y, double *integ, double *d0, double *d1,
                      double *d2, double *d0_lu);

/* Drop-in for the GSL builder LABS_fill_full (labs_fill_full.cpp:35-195; Fortran interface
 * module_labs.f90:46-65).  Same arguments, all by reference; K is the GSL order. */
void kmm_labs_fill_full(double *M0, double *M1, double *M2, double *M3, double *M4, double *yc,
                        double *yknot, double *int_coeff, double *center_coeff, int *K, int *N,
                        double *STRETCH, double *Ly);

/* State exchange in the reference layout (module_ppdfftw.f90:298-335 allocations).
 * U holds nf >= 7 fields; fields 1,2,3,7 (u, v, w, theta) are used.  rk holds the 3 stores.
 * With a second passive scalar (n_scalar = 2, no counterpart in the reference, which carries one
 * scalar) U needs nf >= 11 and holds it in field 11, and rk holds a fourth store (its RK term,
 * which between steps is the scalar itself, as RK_STORE 3 is theta).
 * Host pointers; pinned memory makes the copies asynchronous-capable. */
int kmm_upload_state(kmm_handle *h, const double *U, int nf, const double *rk, double dt);
int kmm_download_state(kmm_handle *h, double *U, int nf, double *rk);

/* set_initial_data_uvw (initial_step.f90:139-179): uploads u, v, w, theta and builds the
 * RK stores on the device. */
int kmm_set_initial_data_uvw(kmm_handle *h, const double *U, int nf, double dt);

/* time_march (time_march.f90:36-128): one RK3 substep (1..3) on the resident state.
 * out may be NULL. */
int kmm_time_march(kmm_handle *h, int rk_substep, kmm_scalars *out);

/* nsteps full RK3 steps (the main.f90:134-193 loop body without I/O), replayed from a
 * CUDA graph; out receives the diagnostics of the last step. */
int kmm_step(kmm_handle *h, int nsteps, kmm_scalars *out);

/* An ensemble of independent channels (one handle each; any sizes, precisions and control
 * settings) stepped together: every handle's nsteps graph launches are enqueued on its own
 * stream before any handle is waited on, so the channels run concurrently and small grids share
 * the GPU.  outs (may be NULL) receives each handle's diagnostics of its last step.  Returns the
 * status of the first handle that fails (all handles are still waited on).  No counterpart in
 * the reference, which runs one channel per job.  Each handle must appear once. */
int kmm_ensemble_step(kmm_handle *const *hs, int n, int nsteps, kmm_scalars *outs);

/* Same as kmm_step but only enqueues the work on the handle's stream (no host sync,
 * no error check); kmm_sync then waits and reports. */
int kmm_step_async(kmm_handle *h, int nsteps);
int kmm_sync(kmm_handle *h, kmm_scalars *out);

/* End-to-end drop-in with host-resident state: upload U/RK from host memory, run nsteps
 * RK3 steps, download U/RK back.  This is time_march with the reference's ownership of
 * U and RK_STORE (the caller keeps them in host memory).  rk may be NULL: between RK3 steps
 * RK_STORE is a function of u, v, w, theta, so the stores are then rebuilt from U on the
 * device as the reference's restart option 1 does (initial_step.f90:31-33, set_initial_data_uvw)
 * and only U (fields 1, 2, 3, 7) crosses the bus, each way. */
int kmm_step_host(kmm_handle *h, double *U, int nf, double *rk, int nsteps, kmm_scalars *out);

/* The pressure of the current state, as a statistics step computes it (get_pressure /
 * cal_pressure / solve_ppe, get_pressure.f90:1-137, called from get_statistics.f90:458):
 * the substep-1 products with f6 = v v, the pressure Poisson equation per (kx, kz) with
 * D1 (Neumann) rows at the walls whose values are stat_PPE_boundary = nu d2v/dy2 of the
 * state's v at the walls (get_y_dir_deriv_of_field_with_PPE_BC, get_statistics.f90:689-719),
 * and -<vv> for the (0,0) mode.  P receives U(:,:,:,6) of the reference, (ny, nxh, nz)
 * complex128 in host memory.  The state is not changed.  The products are formed in FP64 on
 * a mixed-precision handle too; there the first call allocates an FP64 slab and product
 * planes (96 bytes per point of the 3/2 grid's kx-half plus 96 per spectral point). */
int kmm_get_pressure(kmm_handle *h, double *P);

/* Statistics of the current state, as a statistics step computes them at the start of RK
 * substep 1 (time_march.f90:47-110): get_statistics_1 (get_statistics.f90:9-368), write_spectra
 * (write_energy_spectra.f90:9-399), the physical-space moments of dft_x_realspace
 * (dft_x_realspace.f90:128-155, 238-484) and get_statistics_2 (get_statistics.f90:376-539).
 * Host outputs, each may be NULL:
 *   lines    [KMM_STAT_NLINES][ny]           the stat file's lines, in the order of the
 *                                            KMM_STAT_* indices (kmm_stat_line_name)
 *   spec_kx  [KMM_STAT_NSPEC][nxh][ny]       Exx_kx datasets, STAT(ny, nxh) each
 *   spec_kz  [KMM_STAT_NSPEC][nz][ny]        Exx_kz datasets, STAT(ny, nz) each; as in the
 *                                            reference, "Eozoz_kz" holds the ox-oz cospectrum
 *                                            (write_energy_spectra.f90:218-219)
 *   centre   [2]                             U_c and T_c
 *   P        (ny, nxh, nz) complex128        the pressure (kmm_get_pressure)
 * The state is not changed.  The first call allocates the statistics buffers on the device
 * (and on a mixed-precision handle the FP64 buffers of kmm_get_pressure: every statistic is
 * computed in FP64 in both precisions). */
#define KMM_STAT_NLINES 58
#define KMM_STAT_NSPEC 18
int kmm_get_statistics(kmm_handle *h, double *lines, double *spec_kx, double *spec_kz,
                       double *centre, double *P);
/* Dataset names of line i (without the stat file's path) and of spectrum i (without the
 * "E" prefix and the "_kx"/"_kz" suffix); NULL out of range. */
const char *kmm_stat_line_name(int i);
const char *kmm_stat_spec_name(int i);

/* The cudaStream_t (as void*) every launch of the handle goes to, for event timing. */
int kmm_get_stream(const kmm_handle *h, void **stream);

/* Autotuner (no counterpart in the reference): times the candidate launch shapes of the z
 * transforms, the x pass, the per-mode solvers (systems per block, U factor layout) and the
 * assembly on the handle's own grid and buffers, keeps the fastest of each, and reports them
 * (out may be NULL).  The state is left unchanged; the next kmm_step captures its graph with
 * the chosen shapes.  kmm_get_tuning reports the shapes in use and the timings of the last
 * kmm_autotune (zero before one ran; a handle created with cfg.autotune = 1 has them). */
int kmm_autotune(kmm_handle *h, kmm_tuning *out);
int kmm_get_tuning(const kmm_handle *h, kmm_tuning *out);
/* Pins the launch shapes of t (its shape fields; the timings are ignored), for instance a tuning
 * recorded from an earlier kmm_autotune on the same grid.  Every shape must be one of the grid's
 * candidates (KMM_ERR_ARG otherwise).  Results do not depend on the shapes: every candidate runs
 * the same arithmetic per line and per mode. */
int kmm_set_tuning(kmm_handle *h, const kmm_tuning *t);

/* Kernel ids reported by kmm_profile_step. */
#define KMM_NKERNEL 8
#define KMM_K_BEGIN 0       /* per-substep scalar reset */
#define KMM_K_ZINV 1        /* y_to_x: z inverse transform of u, v, w, theta */
#define KMM_K_XPHYS 2       /* dft_x_realspace: x transforms + products + CFL */
#define KMM_K_DT 3          /* CFL dt update (substep 1) */
#define KMM_K_ZFWD 4        /* x_to_y: z forward transform of the 8 products (+ rescale) */
#define KMM_K_HVHG 5        /* wavespace part 1: control probe, mean-mode fork, hvhg D0 solves */
#define KMM_K_HELMHOLTZ 6   /* wavespace part 2: theta, g, phi and v Helmholtz solves */
#define KMM_K_ASSEMBLE 7    /* wavespace part 3: C1/C2 assembly, u and w (the join of the mean-mode
                               lines, which run beside the solver kernels, is outside every id) */

/* Runs nsteps RK3 steps launching kernel by kernel with a CUDA event pair around every
 * launch on the handle's stream; ms[k] = mean device time per launch of kernel k,
 * launches[k] = number of launches.  Same numerics as kmm_step. */
int kmm_profile_step(kmm_handle *h, int nsteps, double *ms, int *launches);

int kmm_get_dt(const kmm_handle *h, double *dt);
int kmm_set_dt(kmm_handle *h, double dt);

/* Opposition-control gains per mode, (nxh, nz) Fortran order, float; NULL resets to 1. */
int kmm_set_control_gains(kmm_handle *h, const float *gains);

/* Opposition control at the wall rows of the v solve (the hook of solve_v_f.f90:251-257, whose
 * commented lines read v at a fixed collocation row): v_wall(kx, kz) = amp * gains(kx, kz) *
 * v(kx, kz, y_d) at the bottom wall and with v at -y_d at the top wall.  amp = 0 turns the
 * control off (the reference's behaviour); otherwise y_d must lie in (-1, 0).  gains as in
 * kmm_set_control_gains (NULL = 1).  Waits for the handle's queued steps; the next kmm_step
 * captures its graph again when amp changes. */
int kmm_set_control(kmm_handle *h, double amp, const float *gains, double y_d);

/* ---- Device-level building blocks (caller device pointers, reference layouts, cudaStream_t
 * passed as void*).  Complex buffers are interleaved doubles. ---- */

/* y_to_x (y_to_x.f90:21-50) for one field: Y-pencil (ny,nxh,nz) -> X-pencil (nxh,nz32,ny).
 * xp is double or float complex according to the handle's precision. */
int kmm_dev_y_to_x(kmm_handle *h, const double *u_ypencil, void *xp, void *stream);

/* x_to_y (x_to_y.f90:21-46) for one field, including rescale_data's 1/(nx32*nz32)
 * (rescale_data.f90:31-33) when rescale != 0. */
int kmm_dev_x_to_y(kmm_handle *h, const void *xp, double *u_ypencil, int rescale, void *stream);

/* dft_x_realspace (dft_x_realspace.f90:68-213) on an X-pencil with 10 field slots
 * (slot stride nxh*nz32*ny complex); reads slots 1,2,3,7 and writes 1-5, 7-9 (slot 10,
 * the copy of v, is not produced: the v state is used directly).  velmax (substep 1)
 * is written to *velmax_dev (device double) when not NULL. */
int kmm_dev_dft_x_realspace(kmm_handle *h, void *xp, int rk_substep, double *velmax_dev,
                            void *stream);

/* wavespace (wavespace.f90:22-113) on U (ny,nxh,nz,10) and RK_STORE (ny,nxh,nz,3) in the
 * reference layout, with dt given; slot 10 holds v for the control.  Products in slots
 * 1-5, 7-9 on entry; u, v, w, theta in slots 1,2,3,7 on exit. */
int kmm_dev_wavespace(kmm_handle *h, double *U, double *rk, int rk_substep, double dt,
                      kmm_scalars *out, void *stream);

/* Batched LABS kernels (module_labs.f90) on mode-fastest device arrays, for testing:
 * a_modes (2bw+1, ny, nmodes) [band element fastest over modes: index ((j*(2bw+1))+r)*nm+m],
 * b (ny, nmodes) complex. */
int kmm_dev_labs_lu(kmm_handle *h, double *a_modes, int nmodes, void *stream);
int kmm_dev_labs_bs(kmm_handle *h, const double *a_modes, double *b, int nmodes, void *stream);
int kmm_dev_labs_mat_mul(kmm_handle *h, int which, const double *x, double *b, int nmodes,
                         void *stream); /* which: 0 = D0, 1 = D1, 2 = D2 */

/* ---- The reference's per-mode routines with their argument lists, batched over modes ----
 * Each call applies one routine to nmodes independent (kx, kz) modes on the handle's device, one
 * GPU thread per mode, in the routine's own statement order through the packed-band LU,
 * substitution and mat-vec of module_labs.f90.  The caller's buffers are the routine's scratch,
 * as in the Fortran; nothing is allocated.
 *   line arguments   device, complex doubles, ny values per mode, mode fastest: value y (1..ny)
 *                    of mode m at complex index (y-1)*nmodes + m; 16-byte aligned
 *   D0_lu, D0..D2    device, (2*bw+1, ny) Fortran bands shared by all modes (kmm_get_operators)
 *   D_buf            device, one (2*bw+1, ny) band per mode: entry (r, j) of mode m at
 *                    ((j-1)*(2bw+1) + r-1)*nmodes + m
 *   kx, kz           device, nmodes physical wavenumbers (kx_int / LMFx, kz_int / LMFz)
 *   rk_substep, dt   the module globals RK_SUBSTEP and dt (module_runge_kutta.f90:14-21)
 * ny must equal the handle's; bw is the handle's. */

/* hvhg (hvhg.f90:28-163): on exit u1 = h_g, u5 = h_v, u7 = h_theta; u2, u3, u4, u8, u9 are
 * overwritten as in the reference.  nx32 and nz32 are accepted as hvhg.f90:28 declares them
 * (its body does not read them). */
int kmm_dev_hvhg(kmm_handle *h, double *u1, double *u2, double *u3, double *u4, double *u5, double *u7,
                 double *u8, double *u9, const double *D0_lu, const double *D1, const double *D2,
                 const double *kx, const double *kz, int64_t nx32, int64_t nz32, int nmodes, void *stream);

/* solve_g (solve_g.f90:28-201): u1 = h_g on entry, g on exit; store_g = RK_STORE 1 of the
 * substep in and out; buf1, buf2 scratch; D_buf receives the factored (1 + beta k^2) D0 - beta D2
 * with Dirichlet rows, which solve_v_f reads next. */
int kmm_dev_solve_g(kmm_handle *h, double *u1, double *store_g, double *buf1, double *buf2,
                    const double *D0_lu, const double *D0, const double *D2, double *D_buf,
                    const double *kx, const double *kz, double nu, int ny, int rk_substep, double dt,
                    int nmodes, void *stream);

/* solve_t (solve_t.f90:28-201): solve_g with the diffusivity nu / pr, for the passive scalar. */
int kmm_dev_solve_t(kmm_handle *h, double *u7, double *store_t, double *buf1, double *buf2,
                    const double *D0_lu, const double *D0, const double *D2, double *D_buf,
                    const double *kx, const double *kz, double nu, double pr, int ny, int rk_substep,
                    double dt, int nmodes, void *stream);

/* solve_v_f (solve_v_f.f90:38-375): hv = h_v on entry; v, dv = dv/dy and store_phi on exit;
 * buf1..buf3 scratch; D_buf holds solve_g's factors on entry and the v operator's on exit.
 * vwall (device, complex [2][nmodes], may be NULL) gives v at the bottom and top wall rows of
 * the v solve (the opposition-control hook at solve_v_f.f90:251-257); NULL gives the reference's
 * zero walls.  vold is accepted as the reference declares it; only its commented control lines
 * read it. */
int kmm_dev_solve_v_f(kmm_handle *h, double *v, double *dv, double *hv, double *store_phi,
                      double *buf1, double *buf2, double *buf3, const double *vold,
                      const double *D0_lu, const double *D0, const double *D1, const double *D2,
                      double *D_buf, const double *kx, const double *kz, double nu, int ny,
                      int rk_substep, double dt, const double *vwall, int nmodes, void *stream);

/* solve_u_w (solve_u_w.f90:18-42): g -> u and f (= dv/dy) -> w, in place. */
int kmm_dev_solve_u_w(kmm_handle *h, double *g, double *f, const double *kx, const double *kz,
                      int nmodes, void *stream);

/* ---- Discrete adjoint of the RK3 step: gradients of the opposition control ----
 * No counterpart in the reference (its control is commented out).  The control of
 * kmm_set_control sets v at the wall rows of the v solve to v_wall(m) = A g(m) P(w . v_m): A the
 * amplitude, g the per-mode gains, w . v the value of v at the detection plane, P the projection
 * the physical round trip applies (kz Nyquist row zeroed, Hermitian part on kx = 0).  Objective
 * over N steps at a fixed time step:
 *   J = (w_tau / N) sum_n tau_w(n) + (w_q / N) sum_n q_w(n),
 * tau_w and q_w the wall shear stress and wall scalar flux of each step (kmm_scalars).
 * kmm_adjoint_forward runs nsteps RK3 steps from the current state (as kmm_step does) keeping one
 * checkpoint per step in HBM (u, v, w, theta and the three stores: 7 ny nxh nz complex doubles
 * each) and returns J.  kmm_adjoint_backward applies the transpose of the recorded steps,
 * recomputing each step's substeps from its checkpoint, and returns dJ/dA and dJ/dg
 * (dJ_dgains: (nxh, nz) Fortran order like kmm_set_control_gains, may be NULL); the state is left
 * where kmm_adjoint_forward left it.  kmm_adjoint_release frees the checkpoints and buffers
 * (kmm_destroy does too).  The adjoint is FP64: a mixed-precision handle, or one with the CFL
 * time step, gets KMM_ERR_CONFIG. */
int kmm_adjoint_forward(kmm_handle *h, int nsteps, double w_tau, double w_q, double *J);
int kmm_adjoint_backward(kmm_handle *h, double *dJ_dA, double *dJ_dgains);
int kmm_adjoint_release(kmm_handle *h);

/* ---- Checkpoint files (channel_hdf5_io, module_hdf5_io.f90:6-456) --------------------------
 * HDF5 files with the reference's datasets and layout, read and written by the library itself
 * (no HDF5 library): root-group datasets, lines (1-D float64 / int32), planes (Fortran (a, b)),
 * fields (Fortran (ny, nx/2, nz) of (re, im) pairs: ESIO layout 0, and on reading the legacy
 * ESIO layouts 1 and 2 that an int32[8] esio_field_metadata attribute announces).  One process
 * holds the whole file: the reference's MPI decomposition becomes the (start, count) arguments of
 * the reads.  A file is written when it is closed; a file opened with readwrite = 1 is read whole
 * and written again on close. */
typedef struct kmm_io kmm_io;
/* io_file_create (module_hdf5_io.f90:63-78): overwrite = 0 refuses an existing path.  Like the
 * reference it sets the root attribute Native_IO. */
int kmm_io_create(const char *path, int32_t overwrite, kmm_io **out);
/* io_file_open (:80-95) */
int kmm_io_open(const char *path, int32_t readwrite, kmm_io **out);
/* io_file_close (:107-114): writes the file if it was created or changed; frees io either way. */
int kmm_io_close(kmm_io *io);
/* io_string_set on "/" (:169-210): replaces the root attribute `name`. */
int kmm_io_string_set(kmm_io *io, const char *name, const char *value);
int kmm_io_string_get(kmm_io *io, const char *name, char *buf, int64_t len);
/* 1 if the root group holds dataset `name`, 0 if not (negative on a bad argument). */
int kmm_io_exists(kmm_io *io, const char *name);
/* io_line_write_double / _integer (:347-376): a 1-D dataset of n values, optional comment. */
int kmm_io_line_write_double(kmm_io *io, const char *name, int64_t n, const double *v, const char *comment);
int kmm_io_line_write_integer(kmm_io *io, const char *name, int64_t n, const int32_t *v, const char *comment);
/* io_line_read_double / _integer (:357-386): values [start, start + count) of a line of n. */
int kmm_io_line_read_double(kmm_io *io, const char *name, int64_t n, int64_t start, int64_t count, double *v);
int kmm_io_line_read_integer(kmm_io *io, const char *name, int64_t n, int64_t start, int64_t count, int32_t *v);
/* io_plane_write_double (:388-403): v is Fortran (na, nb). */
int kmm_io_plane_write_double(kmm_io *io, const char *name, int64_t na, int64_t nb, const double *v,
                              const char *comment);
int kmm_io_plane_read_double(kmm_io *io, const char *name, int64_t na, int64_t nb, double *v);
/* io_field_writev_double / io_field_readv_double (:405-419): v is Fortran (ncomp, ny, nxh, nz);
 * a read takes kx [x0, x0 + xn) and kz [z0, z0 + zn) (all of y) into (ncomp, ny, xn, zn). */
int kmm_io_field_writev_double(kmm_io *io, const char *name, int64_t ny, int64_t nxh, int64_t nz, int32_t ncomp,
                               const double *v);
int kmm_io_field_readv_double(kmm_io *io, const char *name, int64_t ny, int64_t nxh, int64_t nz, int32_t ncomp,
                              int64_t x0, int64_t xn, int64_t z0, int64_t zn, double *v);
/* A dataset of any C-order shape (rank 0 = scalar) of float64 (kind 0; ncomp > 1 makes each element
 * an array of ncomp float64) or int32 (kind 1), and an int32 attribute on a dataset: for files
 * the readers above must refuse, and for tools.  kmm_io_delete removes a dataset. */
int kmm_io_dataset_write_raw(kmm_io *io, const char *name, int32_t rank, const int64_t *cdims, int32_t kind,
                             int32_t ncomp, const void *data);
int kmm_io_attr_write_integer(kmm_io *io, const char *dataset, const char *name, int64_t n, const int32_t *v);
int kmm_io_delete(kmm_io *io, const char *name);

/* data_store / data_store_f (data_store.f90:11-173, 176-420): writes the handle's state as a
 * restart file: the root attributes, the scalar lines (timestep, time, nu, Pr, U_gal, U_avg,
 * W_avg, T_avg, Re, LMFx/y/z, Lx/y/z, Stretch, dt, nx, ny, nz, LABS_K, LABS_BW), the mean
 * profiles U_mean (with U_gal added back), W_mean, T_mean, the operator lines and planes
 * (LABS_COL, LABS_CENTER_LINE, LABS_INTEGRATE, LABS_KNOT, LABS_D0/D1/D2_FULL, LABS_D0/D1/D2_BAND)
 * and the fields selected by `fields` (the input file's write_u ... write_t switches):
 * u, v, w and theta from the state, g and phi from RK_STORE 1 and 2.  timestep and time are
 * the caller's (the driver counts them); dt is the handle's. */
#define KMM_STORE_U 1
#define KMM_STORE_V 2
#define KMM_STORE_W 4
#define KMM_STORE_G 8
#define KMM_STORE_PHI 16
#define KMM_STORE_THETA 32
#define KMM_STORE_ALL 63
int kmm_data_store(kmm_handle *h, const char *path, int32_t timestep, double time, int32_t fields);
/* initial_step with a restart file (initial_step.f90:15-56, 184-513): restart_option 1 reads
 * u, v, w, theta (data_read_uvw) and runs set_initial_data_uvw; 2 reads g, phi, theta and the
 * mean profiles (data_read_gphi) and rebuilds u, v, w (set_initial_data_gphi); 3 reads v, g,
 * theta and the mean profiles (data_read_vg) and rebuilds u, w and phi (set_initial_data_vg).
 * U_gal is taken off the mean streamwise velocity as the reference does.  The handle's dt
 * becomes the file's; timestep, time and dt are returned. */
typedef struct kmm_restart_info {
  int32_t timestep;
  int32_t reserved;
  double time;
  double dt;
} kmm_restart_info;
int kmm_restart(kmm_handle *h, const char *path, int32_t restart_option, kmm_restart_info *out);

/* Allocation-free batched Helmholtz solve.  No counterpart in the reference: it exists for
 * callers that may not allocate device memory (code running while a stream is captured into a
 * CUDA graph, hosts whose device memory is reserved up front by another allocator, loops that
 * cannot afford cudaMalloc's device-wide synchronisation).  It needs no handle.
 * For every mode m it builds A_m = a[m] D0 - b[m] D2 with Dirichlet first and last rows,
 * factors it and solves A_m x = rhs_m in place.
 *   d0_band, d2_band  device, real (2*bw+1, ny) column-major bands: entry r (1..2bw+1) of
 *                     column j (1..ny) at band[(j-1)*(2bw+1) + r-1]; column j holds row j of the
 *                     operator, the near-boundary rows packed as kmm_get_operators returns them
 *   a, b              device, nmodes doubles
 *   rhs               device, complex (ny, nmodes), mode fastest, 16-byte aligned; overwritten
 *                     by x
 * The per-mode scratch band is a fixed array inside the library of KMM_NOALLOC_MAX_DOUBLES
 * doubles (16 MiB), held by every GPU that loads the library until exit; calls with
 * (2*bw+1)*ny*nmodes above it, or a misaligned rhs, are rejected with KMM_ERR_ARG.  The first
 * call on each device looks the array up (cudaGetSymbolAddress); make that call before any
 * stream capture.  A cudaDeviceReset invalidates that lookup: do not call this entry point on a
 * device after resetting it.  All calls share the array: calls that overlap on the GPU race. */
#define KMM_NOALLOC_MAX_DOUBLES 2097152
int kmm_helmholtz_solve_noalloc(int ny, int bw, int nmodes, const double *d0_band,
                                const double *d2_band, const double *a, const double *b,
                                double *rhs, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* KMM_H */
