// tune.cu - the autotuner: launch shapes picked by timing on the handle's own grid.
//
// No counterpart in the reference (FFTW's planner, FFTW_MEASURE at module_ppdfftw.f90:422-477, is
// its nearest relative: it times candidate plans at set-up and keeps the fastest).  The
// candidates are
//   z transforms   kx lines per block (transforms2.cu ZVar; zinv + zfwd timed together),
//   x pass         z rows per block and threads (XVar),
//   per-mode solve 32 or 64 (kx, kz) systems per block of k_hvhg and k_helmholtz (one scalar),
//                  each with the operator tables read through L1 or copied to shared memory
//                  (where a block can hold them), then the U factor storage layout of the
//                  Helmholtz roles,
//   assembly       threads per block.
// Each candidate runs once to warm up, then kReps times between CUDA events on the handle's
// stream; the minimum of the means wins.  The solver runs mutate the state, so the state, the
// stores and the device scalars are saved first and put back after every run and at the end.
#include <cuda_runtime.h>

#include <cstddef>
#include <cstring>
#include <string>
#include <vector>

#include "kmm_internal.h"

namespace kmm {
namespace {

constexpr int kReps = 5;

#define TUNE_CUDA(call)                                                                  \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess) {                                                             \
      set_error(std::string("autotune: ") + cudaGetErrorString(e_) + " at " #call);      \
      return KMM_ERR_CUDA;                                                               \
    }                                                                                    \
  } while (0)

struct Timer {
  cudaEvent_t a = nullptr, b = nullptr;
  ~Timer() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
};

}  // namespace

int autotune(Handle &h, kmm_tuning *out) {
  cudaStream_t st = h.stream;
  Timer t;
  TUNE_CUDA(cudaEventCreate(&t.a));
  TUNE_CUDA(cudaEventCreate(&t.b));
  const int nfld = 3 + h.nsc, nst = 2 + h.nsc;
  const size_t fb = sizeof(double2) * (size_t)h.ns;
  // save the state, the stores and the device scalars (staging holds 10 fields >= nfld + nst)
  TUNE_CUDA(cudaStreamSynchronize(st));
  TUNE_CUDA(cudaMemcpyAsync(h.staging, h.S, nfld * fb, cudaMemcpyDeviceToDevice, st));
  TUNE_CUDA(cudaMemcpyAsync(h.staging + nfld * h.ns, h.RK, nst * fb, cudaMemcpyDeviceToDevice, st));
  DevScalars dsc;
  TUNE_CUDA(cudaMemcpy(&dsc, h.dsc, sizeof(dsc), cudaMemcpyDeviceToHost));
  auto restore = [&]() -> int {
    TUNE_CUDA(cudaMemcpyAsync(h.S, h.staging, nfld * fb, cudaMemcpyDeviceToDevice, st));
    TUNE_CUDA(cudaMemcpyAsync(h.RK, h.staging + nfld * h.ns, nst * fb, cudaMemcpyDeviceToDevice, st));
    TUNE_CUDA(cudaMemcpyAsync(h.dsc, &dsc, sizeof(dsc), cudaMemcpyHostToDevice, st));
    return KMM_OK;
  };
  // mean device ms of kReps runs of `body` after one warm-up run; `prep` runs before each, untimed
  auto measure = [&](auto &&prep, auto &&body, double *ms) -> int {
    int rc;
    if ((rc = prep())) return rc;
    TUNE_CUDA(body());
    double total = 0.0;
    for (int i = 0; i < kReps; ++i) {
      if ((rc = prep())) return rc;
      TUNE_CUDA(cudaEventRecord(t.a, st));
      TUNE_CUDA(body());
      TUNE_CUDA(cudaEventRecord(t.b, st));
      TUNE_CUDA(cudaEventSynchronize(t.b));
      float f = 0.f;
      TUNE_CUDA(cudaEventElapsedTime(&f, t.a, t.b));
      total += f;
    }
    *ms = total / kReps;
    return KMM_OK;
  };
  auto none = []() -> int { return KMM_OK; };
  auto best = [](const double *ms, int n) {
    int b = 0;
    for (int i = 1; i < n; ++i)
      if (ms[i] < ms[b]) b = i;
    return b;
  };
  kmm_tuning rep;
  std::memset(&rep, 0, sizeof(rep));
  int rc;
  const int nprod = 5 + 3 * h.nsc;
  // z transforms
  for (int v = 0; v < 3; ++v) {
    h.tune.z = v;
    auto body = [&]() {
      cudaError_t e = launch_zinv(h, h.S, h.MID, nfld, st);
      if (e == cudaSuccess) e = launch_zfwd(h, h.MID, h.P, nprod, h.rescale, !h.mixed, st);
      return e;
    };
    if ((rc = measure(none, body, &rep.ms_z[v]))) return rc;
  }
  h.tune.z = best(rep.ms_z, 3);
  // x pass, each run on fresh z-inverse slabs
  for (int v = 0; v < 3; ++v) {
    h.tune.x = v;
    auto prep = [&]() -> int {
      TUNE_CUDA(launch_zinv(h, h.S, h.MID, nfld, st));
      return KMM_OK;
    };
    auto body = [&]() { return launch_xphys(h, h.MID, 2, st); };
    if ((rc = measure(prep, body, &rep.ms_x[v]))) return rc;
  }
  h.tune.x = best(rep.ms_x, 3);
  // the per-mode solves of substep 2 on products of the saved state
  {
    TUNE_CUDA(launch_zinv(h, h.S, h.MID, nfld, st));
    TUNE_CUDA(launch_xphys(h, h.MID, 2, st));
    TUNE_CUDA(launch_zfwd(h, h.MID, h.P, nprod, h.rescale, !h.mixed, st));
  }
  // hvhg forks the mean lines to the side stream; join them so no run overlaps the next restore
  auto solve = [&]() {
    cudaError_t e = launch_ws_hvhg(h, 2, nullptr, st);
    if (e == cudaSuccess) e = launch_ws_helmholtz(h, 2, nullptr, st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, h.ev_join, 0);
    return e;
  };
  const int ng = h.nsc == 1 ? 2 : 1;
  double ms_gs[2][2];  // [groups - 1][tables in shared memory]
  int bg = 1, bs = 0;
  for (int g = 0; g < ng; ++g)
    for (int sh = 0; sh < 2; ++sh) {
      ms_gs[g][sh] = 0.0;
      if (sh && !solver_tables_fit(h, g + 1)) continue;
      h.tune.groups = g + 1;
      h.tune.stab = sh;
      h.tune.ulayout = 0;
      if ((rc = measure(restore, solve, &ms_gs[g][sh]))) return rc;
      if (ms_gs[g][sh] < ms_gs[bg - 1][bs] || (g == 0 && sh == 0)) {
        bg = g + 1;
        bs = sh;
      }
    }
  // report the fastest measured time of each knob value (0: not measured)
  auto keep_min = [](double &acc, double v) {
    if (v > 0.0 && (acc == 0.0 || v < acc)) acc = v;
  };
  for (int g = 0; g < ng; ++g)
    for (int sh = 0; sh < 2; ++sh) {
      keep_min(rep.ms_modes[g], ms_gs[g][sh]);
      keep_min(rep.ms_tables[sh], ms_gs[g][sh]);
    }
  h.tune.groups = bg;
  h.tune.stab = bs;
  rep.ms_layout[0] = ms_gs[bg - 1][bs];
  h.tune.ulayout = 1;
  if ((rc = measure(restore, solve, &rep.ms_layout[1]))) return rc;
  h.tune.ulayout = best(rep.ms_layout, 2);
  const int athreads[3] = {128, 256, 512};
  for (int i = 0; i < 3; ++i) {
    h.tune.asm_threads = athreads[i];
    auto prep = [&]() -> int {
      int r = restore();
      if (r) return r;
      TUNE_CUDA(solve());
      return KMM_OK;
    };
    auto body = [&]() { return launch_ws_assemble(h, 2, nullptr, st); };
    if ((rc = measure(prep, body, &rep.ms_assemble[i]))) return rc;
  }
  h.tune.asm_threads = athreads[best(rep.ms_assemble, 3)];
  if ((rc = restore())) return rc;
  TUNE_CUDA(cudaStreamSynchronize(st));
  TUNE_CUDA(cudaStreamSynchronize(h.side));
  h.tune.tuned = true;
  std::memcpy(h.tune.ms_z, rep.ms_z, sizeof(rep.ms_z));
  std::memcpy(h.tune.ms_x, rep.ms_x, sizeof(rep.ms_x));
  std::memcpy(h.tune.ms_modes, rep.ms_modes, sizeof(rep.ms_modes));
  std::memcpy(h.tune.ms_layout, rep.ms_layout, sizeof(rep.ms_layout));
  std::memcpy(h.tune.ms_assemble, rep.ms_assemble, sizeof(rep.ms_assemble));
  std::memcpy(h.tune.ms_tables, rep.ms_tables, sizeof(rep.ms_tables));
  // the step graph holds the old launch shapes: capture it again at the next step
  if (h.gexec) cudaGraphExecDestroy(h.gexec);
  if (h.graph) cudaGraphDestroy(h.graph);
  h.gexec = nullptr;
  h.graph = nullptr;
  if (out) kmm_get_tuning(reinterpret_cast<const kmm_handle *>(&h), out);
  return KMM_OK;
}

}  // namespace kmm

using namespace kmm;

extern "C" {

int kmm_get_tuning(const kmm_handle *hh, kmm_tuning *out) {
  if (!hh || !out) return KMM_ERR_ARG;
  const Handle &h = *reinterpret_cast<const Handle *>(hh);
  std::memset(out, 0, sizeof(*out));
  tile_shapes(h, h.tune.z, h.tune.x, &out->z_lines_per_block, &out->x_rows_per_block, &out->x_threads);
  out->modes_per_block = 32 * (h.nsc == 1 ? h.tune.groups : 1);
  out->u_layout = h.tune.ulayout;
  out->assemble_threads = h.tune.asm_threads;
  out->tuned = h.tune.tuned ? 1 : 0;
  out->tables_shared = h.tune.stab;
  std::memcpy(out->ms_z, h.tune.ms_z, sizeof(out->ms_z));
  std::memcpy(out->ms_x, h.tune.ms_x, sizeof(out->ms_x));
  std::memcpy(out->ms_modes, h.tune.ms_modes, sizeof(out->ms_modes));
  std::memcpy(out->ms_layout, h.tune.ms_layout, sizeof(out->ms_layout));
  std::memcpy(out->ms_assemble, h.tune.ms_assemble, sizeof(out->ms_assemble));
  std::memcpy(out->ms_tables, h.tune.ms_tables, sizeof(out->ms_tables));
  return KMM_OK;
}

int kmm_set_tuning(kmm_handle *hh, const kmm_tuning *t) {
  if (!hh || !t) return KMM_ERR_ARG;
  Handle &h = *reinterpret_cast<Handle *>(hh);
  Tuning next = h.tune;
  // map each requested shape to the candidate that has it on this grid
  int zv = -1, xv = -1;
  for (int v = 2; v >= 0; --v) {
    int zl = 0, xr = 0, xt = 0;
    tile_shapes(h, v, v, &zl, &xr, &xt);
    if (zl == t->z_lines_per_block) zv = v;
    if (xr == t->x_rows_per_block && xt == t->x_threads) xv = v;
  }
  const int g = t->modes_per_block == 32 ? 1 : t->modes_per_block == 64 ? 2 : 0;
  const bool asm_ok = t->assemble_threads == 128 || t->assemble_threads == 256 || t->assemble_threads == 512;
  const bool tab_ok = t->tables_shared == 0 || (t->tables_shared == 1 && g != 0 && solver_tables_fit(h, g));
  if (zv < 0 || xv < 0 || g == 0 || (g == 2 && h.nsc != 1) || (t->u_layout != 0 && t->u_layout != 1) || !asm_ok ||
      !tab_ok) {
    set_error("kmm_set_tuning: a requested shape is not among this grid's candidates (see kmm_autotune)");
    return KMM_ERR_ARG;
  }
  next.z = zv;
  next.x = xv;
  next.groups = g;
  next.ulayout = t->u_layout;
  next.asm_threads = t->assemble_threads;
  next.stab = t->tables_shared;
  DeviceGuard dg(h.cfg.device);
  cudaStreamSynchronize(h.stream);
  h.tune = next;
  if (h.gexec) cudaGraphExecDestroy(h.gexec);
  if (h.graph) cudaGraphDestroy(h.graph);
  h.gexec = nullptr;
  h.graph = nullptr;
  return KMM_OK;
}

int kmm_autotune(kmm_handle *hh, kmm_tuning *out) {
  if (!hh) return KMM_ERR_ARG;
  Handle &h = *reinterpret_cast<Handle *>(hh);
  DeviceGuard dg(h.cfg.device);
  return autotune(h, out);
}

}  // extern "C"
