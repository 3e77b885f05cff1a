// kmm_internal.h - handle layout, HBM layout and helpers shared by the libkmm sources.
//
// HBM layout (all complex, one plane per wall-normal index y, kx fastest):
//   S   [4][ny][nz][nxh]    double2   state u, v, w, theta           (fields 1,2,3,7 of U)
//   RK  [3][ny][nz][nxh]    double2   low-storage RK terms           (RK_STORE 1..3)
//   P   [8][ny][nz][nxh]    R2        spectral products f1..f5, f7..f9 (fields 1-5, 7-9)
//   MID [8][ny][nz32][nxh]  R2        x-spectral / z-physical slab = the reference X-pencil
// With a second passive scalar theta2 (Handle::nsc = 2): S field 4 = theta2, RK store 3 = its
// RK term, P and MID fields 8..10 = u theta2, v theta2, w theta2 (MID field 4 = theta2 in).
//                                     Up(nxh, nz32, ny) (dft_x_realspace.f90:31)
// A (kx, kz) mode m = kz_index * nxh + kx owns the strided line S[f][.][m]: a warp of 32
// consecutive modes reads one 32-element contiguous run per y, so the per-mode solver is
// coalesced without any staging.  R2 is double2 (FP64 path) or float2 (mixed path).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/kmm.h"

namespace kmm {

constexpr int kMaxPass = 8;
// Physical-space moment sums of a statistics substep (stats.cuh moment_terms).
constexpr int kNumMoments = 18;
// Spectra per direction of a statistics step (stats.cu k_spectra).
constexpr int kNumSpec = KMM_STAT_NSPEC;
constexpr int kMinBw = 2;
constexpr int kMaxBw = 7;

// One radix-{2,3,4,5} plan of a length-n complex transform.  pos[i] is where natural index
// i sits in the decimation-in-time input (and where frequency i sits in the
// decimation-in-frequency output); tw[t] = exp(-2 pi i t / n).
struct FftPlan {
  int n = 0;
  int npass = 0;
  int radix[kMaxPass] = {0};
  const int *pos = nullptr;
  const double2 *tw64 = nullptr;
  const float2 *tw32 = nullptr;
};

// Device-side scalars written by the kernels and read back by the host.
struct DevScalars {
  double dt;                    // time step in use
  double dt_prev;               // dt before the last CFL update
  unsigned long long velmax_bits;  // max |u|dxr+|v|dyr+|w|dzr as the bits of a non-negative double
  double phi_dpdx[4];
  double phi_dtdx[4];
  double wall_shear_stress;
  double wall_theta_stress;
  double phi_dtdx2[4];          // the second passive scalar's forcing (n_scalar = 2)
  double wall_theta_stress2;
  int err;                      // KMM_ERR_* raised on the device, 0 if none
  int nonfinite;                // set when a non-finite velocity was seen
};

// Host-side copy of the wall-normal operators.
struct HostOps {
  int ny = 0, k = 0, bw = 0;
  std::vector<double> y, knots, brk, integ, center;
  std::vector<double> full[5];   // [point * ny + basis]
  std::vector<double> band[3];   // (2bw+1, ny) Fortran order
  std::vector<double> d0_lu;
  std::vector<double> off[3];    // offset rows of D0, D1, D2: [(r-1)*(4bw+1) + e + 2bw]
  std::vector<double> l0, u0;    // profile LU of D0 (see build_offset_tables)
  std::vector<double> wlo, whi;  // control weights: v(y_d) = w . v
};

// Builds the operators (LABS_fill_full + LABS_eval_bw + LABS_full_to_band + LABS_lu(D0)).
int build_host_ops(int k_order, int ny, double stretch, double ly, int grid, HostOps &ops,
                   std::string &err);
// Control weights for the detection planes y_d and -y_d.
int build_control_weights(HostOps &ops, double yd, std::string &err);
void host_band_lu(std::vector<double> &a, int bw, int n);

// The discrete adjoint's buffers (adjoint.cu), made by the first kmm_adjoint_forward.
struct Adjoint;

// Launch shapes the autotuner (kmm_autotune, tune.cu) chooses; the defaults are the hand-tuned ones.
struct Tuning {
  int z = 0;              // z-transform variant (lines per block, transforms2.cu ZVar)
  int ztma = 0;           // 1: the z transforms stage each block's input tile through TMA
  int x = 0;              // x-pass variant (rows per block and threads, XVar)
  int groups = 1;         // 32-mode groups per block of the hvhg kernel (1 or 2)
  int hgroups = 1;        // 32-mode groups per block of the Helmholtz kernel (1, 2 or 4)
  int hstab = 0;          // 1: the Helmholtz kernel reads the operator tables from shared memory
  int stage = 1;          // steps of staging look-ahead of the Helmholtz sweeps (1 or 2)
  int ulayout = 0;        // U factor storage: 0 = [offset][y][mode], 1 = [y][offset][mode]
  int asm_threads = 256;  // threads per block of the assembly kernel
  int stab = 0;           // 1: the hvhg kernel reads the operator tables from shared memory
  int hvstage = 0;        // rows the hvhg sweeps stage ahead through shared memory (0: L1 prefetch)
  int fcache = 0;         // 1: the Helmholtz sweeps read the per-substep operator factors and
                          // influence solutions cached for the current dt (fixed time step only)
  bool tuned = false;
  // device ms of every candidate of the last autotune (kmm_tuning's ms_* fields)
  double ms_z[3] = {}, ms_x[3] = {}, ms_modes[2] = {}, ms_layout[2] = {}, ms_assemble[3] = {}, ms_tables[2] = {};
  double ms_helm[3][2][2] = {};  // [32/64/128 modes][tables via L1 / shared][look-ahead 1 / 2]
  double ms_z_tma[3] = {};       // the z variants with TMA-staged input tiles
  double ms_hvhg[2][2][3] = {};  // [32/64 modes][tables via L1 / shared][staging 0 / 1 / 2 rows]
  double ms_step[2] = {};        // graph step with the kept shapes / with the shapes before tuning
};

struct Handle {
  kmm_config cfg{};
  int nx = 0, ny = 0, nz = 0, nxh = 0, nx32 = 0, nz32 = 0, bw = 0;
  int64_t nmodes = 0;           // nxh * nz
  int64_t ns = 0;               // ny * nmodes            (spectral plane stack per field)
  int64_t nm = 0;               // ny * nz32 * nxh        (mid slab per field)
  bool mixed = false;
  int nsc = 1;                  // passive scalars (1 or 2): S holds 3 + nsc fields, RK 2 + nsc stores,
                                // P and MID 8 + 3 (nsc - 1) product fields
  double dxr = 0, dzr = 0, cflx = 0, rescale = 0, lmfxr = 0, lmfzr = 0;
  HostOps ops;
  std::vector<int> radix_x, radix_z;

  cudaStream_t stream = nullptr;
  double2 *S = nullptr, *RK = nullptr;
  void *P = nullptr, *MID = nullptr;       // R2 arrays
  double *dops = nullptr;                  // D0, D1, D2, D0_LU bands, integ, dyr, wlo, whi
  float *gains = nullptr;                  // control gains per mode
  double2 *vwall = nullptr;                // [2][nmodes] control wall velocities
  double2 *zc = nullptr;                   // per-mode solver: forward lines  [8][ny][nmodes]
  double2 *ec = nullptr;                   //                  hvhg outputs   [9][ny][nmodes]
  double *xr = nullptr;                    //                  real lines     [6][ny][nmodes]
  double *ub = nullptr;                    //                  U factors, 3 roles (split_ub_role each)
  double *vf = nullptr;                    //                  v operator LU per mode (vop_factor_doubles)
  double2 *dvw = nullptr;                  //                  wall derivatives [3][nmodes]
  double *w00 = nullptr;                   // mean-mode lines (3 threads)
  // With a fixed time step the Helmholtz operators of each substep (theta's and the one g and
  // phi share) do not change between steps: their profile LU per mode, the influence solutions
  // phi_h, D2 phi_h, v_h, dv_h / dy and v_h's wall derivatives, cached for the dt in fcdt
  // (factor_cache_possible; made at kmm_create).
  double *hf = nullptr;                    // [substep][theta, g/phi] LBand then UBand (vop_factor_doubles)
  double *hinf = nullptr;                  // [substep][4][ny][nmodes] influence lines
  double2 *hdvh = nullptr;                 // [substep][nmodes] (dv_h(1), dv_h(n))
  double *fcdt = nullptr;                  // [substep] the dt the cache holds (NaN: none)
  double *stat = nullptr;                  // statistics buffers (stat_layout), made on first use
  double2 *mid64 = nullptr, *p64 = nullptr;  // mixed handles: FP64 slab [6][nm] and products [6][ns]
                                             // of the pressure / statistics pass, made on first use
  cudaStream_t side = nullptr;             // mean-mode lines run here, forked from / joined to stream
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  cudaStream_t copy = nullptr;             // host <-> device copies of kmm_step_host, beside stream
  cudaEvent_t ev_io[9] = {};               // its per-field hand-offs between copy and stream
  double2 *staging = nullptr;              // [7][nz][nxh][ny] reference-layout staging
  int *fftpos = nullptr;
  double2 *tw64 = nullptr;
  float2 *tw32 = nullptr;
  DevScalars *dsc = nullptr;
  FftPlan px, pz;
  int64_t device_bytes = 0;

  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  Adjoint *adj = nullptr;                  // discrete adjoint state (adjoint.cu), or null
  Tuning tune;                             // launch shapes (kmm_autotune)
};

// Offsets of the operator arrays inside dops (doubles).
struct OpsOffsets {
  int64_t d0, d1, d2, d0lu, integ, dyr, wlo, whi;
  int64_t t0;  // offset tables T0, T1, T2 [ny][4bw+1], then the D0 profile LU L0 [ny][2bw+1], U0 [ny][2bw]
  int64_t total;
};
OpsOffsets ops_offsets(int bw, int ny);

// Kernel launchers (transforms.cu, labs_kernels.cu).
// fp64: compute in FP64 on a mixed handle too (mid then holds double2 lines; zfwd writes double2).
cudaError_t launch_zinv(Handle &h, const double2 *src_planes, void *mid, int nfield,
                        cudaStream_t st, bool fp64 = false);
cudaError_t launch_xphys(Handle &h, void *mid, int substep, cudaStream_t st);
cudaError_t launch_zfwd(Handle &h, const void *mid, void *dst_planes, int nfield, double scale,
                        bool dst_fp64, cudaStream_t st, bool fp64 = false);
cudaError_t launch_update_dt(Handle &h, int substep, cudaStream_t st);
cudaError_t launch_begin_substep(Handle &h, int substep, cudaStream_t st);
cudaError_t launch_init_stores(Handle &h, cudaStream_t st);
// set_initial_data_uvw in two parts: RK_STORE 2 of the modes other than (0,0), which needs only
// v (launch_init_phi), and the element-wise rest (launch_init_elem, needs u, w, theta).
cudaError_t launch_init_phi(Handle &h, cudaStream_t st);
cudaError_t launch_init_elem(Handle &h, cudaStream_t st);
cudaError_t launch_ref_to_planes(const double2 *src, double2 *dst, int nfield, int64_t nmodes,
                                 int ny, cudaStream_t st);
cudaError_t launch_planes_to_ref(const double2 *src, double2 *dst, int nfield, int64_t nmodes,
                                 int ny, cudaStream_t st);
cudaError_t launch_labs_lu(Handle &h, double *a, int nmodes, cudaStream_t st);
cudaError_t launch_labs_bs(Handle &h, const double *a, double2 *b, int nmodes, cudaStream_t st);
cudaError_t launch_labs_mat_mul(Handle &h, int which, const double2 *x, double2 *b, int nmodes,
                                cudaStream_t st);

void set_error(const std::string &msg);
// Frees a checkpoint file handle without writing it (an error part-way through a data store).
void io_discard(kmm_io *io);

// Makes a handle's device current for the lifetime of the guard and gives the caller's current
// device back on destruction.  Every handle entry point holds one, so handles on several GPUs,
// or a caller that changes the current device between calls, always launch on the handle's own
// device (its streams, graph and buffers belong to it).
struct DeviceGuard {
  int prev = -1;
  bool ok = true;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) ok = cudaSetDevice(dev) == cudaSuccess;
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
  DeviceGuard(const DeviceGuard &) = delete;
  DeviceGuard &operator=(const DeviceGuard &) = delete;
};

// Sets the dynamic shared-memory limits of every kernel instantiation the handle uses.
void prepare_kernels(Handle &h);
void convert_planes_d2f(const double2 *src, float2 *dst, int64_t n, cudaStream_t st);
cudaError_t prepare_transforms2();
// Whether a padded line length has a compile-time four-step shape (transforms2.cu).
bool fft4_supported(int N);
// The z lines per block and x rows / threads per block of tile variants zvar, xvar on h's grid
// (0 where the length has no four-step shape).
void tile_shapes(const Handle &h, int zvar, int xvar, int *z_lines, int *x_rows, int *x_threads);
// Runs the autotuner (tune.cu) on h's grid and buffers; the state is left unchanged.
int autotune(Handle &h, kmm_tuning *out);
// Four-step transforms (transforms2.cu); return cudaErrorNotSupported for other lengths.
cudaError_t launch_zinv2(Handle &h, const double2 *src_planes, void *mid, int nfield, cudaStream_t st,
                         bool fp64 = false);
// stat: the statistics-step variant (f6 = v v, no CFL), in FP64 on every handle (mid holds
// double2 lines); mom (stat only, may be null) receives per-block moment sums
// [ny][xphys2_row_blocks(h)][kNumMoments].
cudaError_t launch_xphys2(Handle &h, void *mid, int substep, cudaStream_t st, bool stat = false,
                          double *mom = nullptr);
int xphys2_row_blocks(const Handle &h);
// The transpose of the x pass at a base state (FP64 handles, four-step lengths): base_mid slots
// 0..3 hold u, v, w, theta; lmid slots 0..7 hold the lambda of the products (times scale) on entry
// and slots 0..3 the lambda of u, v, w, theta on exit.
cudaError_t launch_xadj2(Handle &h, const double2 *base_mid, double2 *lmid, double scale, cudaStream_t st);
cudaError_t launch_zfwd2(Handle &h, const void *mid, void *dst_planes, int nfield, double scale,
                         bool dst_fp64, cudaStream_t st, bool fp64 = false);
// Per-mode solves of one substep (wavespace_split.cu): hvhg, Helmholtz and assembly kernels on
// st, the mean lines on h.side (joined back to st before return).
cudaError_t launch_wavespace_split(Handle &h, int substep, const double *dt_override, cudaStream_t st);
// The three parts of launch_wavespace_split (control probe + mean fork + hvhg; Helmholtz;
// assembly + mean join), for per-kernel timing.
cudaError_t launch_ws_hvhg(Handle &h, int substep, const double *dt_override, cudaStream_t st);
cudaError_t launch_ws_helmholtz(Handle &h, int substep, const double *dt_override, cudaStream_t st);
cudaError_t launch_ws_assemble(Handle &h, int substep, const double *dt_override, cudaStream_t st);
// The assembly kernel alone, and the join of the mean lines (the side stream) onto st; the
// kernel-by-kernel profile records the assembly without the join.
cudaError_t launch_ws_assemble_only(Handle &h, int substep, const double *dt_ptr, cudaStream_t st);
cudaError_t launch_ws_join(Handle &h, cudaStream_t st);
// The pressure of the state (pressure.cu): p planes [y][mode] into out, with the wall values
// bc [2][nmodes] (launch_ydiff); mom as in launch_xphys2.  The products are formed in FP64 on
// every handle (a mixed handle's in mid64 / p64, which diag_buffers makes).  Uses MID and P (or
// mid64 and p64), the solver lines zc and U region 0 as scratch; cudaErrorNotSupported for x
// lengths without a four-step shape.
cudaError_t launch_pressure(Handle &h, double2 *out, const double2 *bc, double *mom, cudaStream_t st);
// Makes a mixed handle's mid64 and p64 (nothing on an FP64 handle); a KMM_ERR_* code.
int diag_buffers(Handle &h);
// y derivatives of the state (stats.cu): for each field f in {u, v, w} with bit f of mask set,
// ec line f = D1 D0^{-1} f per mode (zc lines 0..2 scratch); with the v bit set, dvw lines 0
// and 1 = the pressure wall values nu (D2 D0^{-1} v) on rows 1 and ny.
cudaError_t launch_ydiff(Handle &h, int mask, cudaStream_t st);
// Offsets (doubles) inside Handle::stat: x-pass moment sums [ny][row blocks][kNumMoments],
// transport inputs [4][ny], lines [KMM_STAT_NLINES][ny], spectra [kNumSpec][nxh][ny] and
// [kNumSpec][nz][ny], centre-line values [2], the centre-line vector [ny], line scratch.
struct StatLayout {
  int64_t part, tr, lines, skx, skz, scal, center, scr, total;
};
StatLayout stat_layout(const Handle &h);
// The statistics of the state (stats.cu) into Handle::stat; uses the buffers of
// launch_pressure plus ec and dvw as scratch and leaves the pressure planes in staging[0].
cudaError_t launch_statistics(Handle &h, cudaStream_t st);
// The v operator's profile LU per mode (wavespace_split.cu): doubles of its L part and of the
// whole (L then U), and the kernel that fills it once per handle.
int64_t vop_lband_doubles(const Handle &h);
int64_t vop_factor_doubles(const Handle &h);
// Whether the handle can cache the Helmholtz factors: a fixed time step and one scalar.
bool factor_cache_possible(const Handle &h);
cudaError_t launch_vop_factor(Handle &h, cudaStream_t st);
// Doubles of U factor storage per solver role.
int64_t split_ub_role(const Handle &h);
// Operator tables in shared memory for the hvhg and Helmholtz kernels (their bytes per block,
// whether hvhg's block holds them) and the Helmholtz shapes a block can hold (groups, tables,
// look-ahead); default_solver_shapes sets a new handle's solver shapes.
size_t solver_tables_bytes(const Handle &h);
// Whether the z transforms of variant zvar can stage their input tiles through TMA on this grid
// (four-step length, tile within the shared-memory limit, tile map accepted by the encoder).
bool z_tma_possible(const Handle &h, int zvar);
bool hvhg_tables_fit(const Handle &h);
bool hvhg_shape_fits(const Handle &h, int groups, int stab, int stage);
bool helm_shape_fits(const Handle &h, int hgroups, int hstab, int stage);
void default_solver_shapes(Handle &h);

// One time_march substep enqueued kernel by kernel on st (api.cu), the device scalars read back,
// and the step graph captured if it is not yet.
int run_substep(Handle &h, int substep, cudaStream_t st);
int read_device_scalars(Handle &h, kmm_scalars *out, int *dev_err);
int capture_step_graph(Handle &h);

// Frees the discrete adjoint's buffers (adjoint.cu).
void adjoint_free(Handle &h);

}  // namespace kmm
