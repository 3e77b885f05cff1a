// tune.cu - the autotuner: launch shapes picked by timing on the handle's own grid.
//
// No counterpart in the reference (FFTW's planner, FFTW_MEASURE at module_ppdfftw.f90:422-477, is
// its nearest relative: it times candidate plans at set-up and keeps the fastest).  The
// candidates are
//   z transforms   kx lines per block (transforms2.cu ZVar; zinv + zfwd timed together), each
//                  with per-thread input loads or TMA-staged input tiles,
//   x pass         z rows per block and threads (XVar),
//   hvhg           32 or 64 (kx, kz) systems per block (one scalar) x the operator tables read
//                  through L1 or copied to shared memory x rows prefetched into L1 or staged
//                  through a shared-memory ring 1 or 2 rows ahead,
//   Helmholtz      32, 64 or 128 systems per block x tables through L1 / in shared memory x one
//                  or two rows of staging look-ahead, where a block's shared memory holds the
//                  shape; then the U factor storage layout,
//   assembly       threads per block.
// Each candidate runs once to warm up, then kReps times between CUDA events on the handle's
// stream; the minimum of the means wins.  Last, whole steps through the step graph decide which
// of those picks stay, one knob group at a time from the shapes the handle had before: in the
// step the solver kernels share the GPU with the mean lines on the side stream, which the
// per-kernel timings do not see.  The solver runs mutate the state, so the state, the stores and the device
// scalars are saved first and put back after every run and at the end.
#include <cuda_runtime.h>

#include <cstddef>
#include <cstring>
#include <string>
#include <vector>

#include "kmm_internal.h"

namespace kmm {
namespace {

constexpr int kReps = 5;
constexpr int kSteps = 3;  // graph steps per timed run of the final comparison
// A knob group's pick replaces the entry shapes only for a step at least 1% faster: step times of
// two shape sets within a few tenths of a percent reorder from one run (or box) to the next.
constexpr double kMinGain = 0.99;

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
  const Tuning entry = h.tune;  // the shapes the handle had before
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
  // z transforms: lines per block, each with per-thread input loads or TMA-staged input tiles
  // (where the grid allows the tile map)
  double best_z = 0.0;
  int bz = 0, bt = 0;
  for (int t = 0; t < 2; ++t)
    for (int v = 0; v < 3; ++v) {
      if (t && !z_tma_possible(h, v)) continue;
      h.tune.z = v;
      h.tune.ztma = t;
      auto body = [&]() {
        cudaError_t e = launch_zinv(h, h.S, h.MID, nfld, st);
        if (e == cudaSuccess) e = launch_zfwd(h, h.MID, h.P, nprod, h.rescale, !h.mixed, st);
        return e;
      };
      double *slot = t ? &rep.ms_z_tma[v] : &rep.ms_z[v];
      if ((rc = measure(none, body, slot))) return rc;
      if (best_z == 0.0 || *slot < best_z) {
        best_z = *slot;
        bz = v;
        bt = t;
      }
    }
  h.tune.z = bz;
  h.tune.ztma = bt;
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
  // hvhg forks the mean lines to the side stream: every restore first waits for them.  The join
  // event's last record may sit in the captured step graph, which a wait outside the graph
  // refuses: record it on the side stream first.
  TUNE_CUDA(cudaEventRecord(h.ev_join, h.side));
  auto restore_joined = [&]() -> int {
    TUNE_CUDA(cudaStreamWaitEvent(st, h.ev_join, 0));
    return restore();
  };
  auto keep_min = [](double &acc, double v) {
    if (v > 0.0 && (acc == 0.0 || v < acc)) acc = v;
  };
  // k_hvhg: modes per block x tables through L1 / in shared memory x staging (L1 prefetch, or a
  // shared-memory ring 1 or 2 rows ahead)
  const int ng = h.nsc == 1 ? 2 : 1;
  {
    double best_ms = 0.0;
    int bg = 1, bs = 0, ba = 0;
    for (int g = 1; g <= ng; ++g)
      for (int sh = 0; sh < 2; ++sh)
        for (int sa = 0; sa <= 2; ++sa) {
          if (!hvhg_shape_fits(h, g, sh, sa)) continue;
          h.tune.groups = g;
          h.tune.stab = sh;
          h.tune.hvstage = sa;
          double ms = 0.0;
          auto body = [&]() { return launch_ws_hvhg(h, 2, nullptr, st); };
          if ((rc = measure(restore_joined, body, &ms))) return rc;
          rep.ms_hvhg[((g - 1) * 2 + sh) * 3 + sa] = ms;
          keep_min(rep.ms_modes[g - 1], ms);
          keep_min(rep.ms_tables[sh], ms);
          if (best_ms == 0.0 || ms < best_ms) {
            best_ms = ms;
            bg = g;
            bs = sh;
            ba = sa;
          }
        }
    h.tune.groups = bg;
    h.tune.stab = bs;
    h.tune.hvstage = ba;
  }
  // k_helmholtz after the chosen hvhg: modes per block x tables x staging look-ahead, then the
  // U factor layout
  auto after_hvhg = [&]() -> int {
    int r = restore_joined();
    if (r) return r;
    TUNE_CUDA(launch_ws_hvhg(h, 2, nullptr, st));
    return KMM_OK;
  };
  auto helm = [&]() { return launch_ws_helmholtz(h, 2, nullptr, st); };
  {
    h.tune.ulayout = 0;
    double best_ms = 0.0;
    int bg = 1, bs = 0, ba = 1;
    const int hg_n[3] = {1, 2, 4};
    for (int gi = 0; gi < 3; ++gi)
      for (int sh = 0; sh < 2; ++sh)
        for (int sa = 1; sa <= 2; ++sa) {
          const int g = hg_n[gi];
          if (!helm_shape_fits(h, g, sh, sa)) continue;
          h.tune.hgroups = g;
          h.tune.hstab = sh;
          h.tune.stage = sa;
          double ms = 0.0;
          if ((rc = measure(after_hvhg, helm, &ms))) return rc;
          rep.ms_helm[(gi * 2 + sh) * 2 + sa - 1] = ms;
          if (best_ms == 0.0 || ms < best_ms) {
            best_ms = ms;
            bg = g;
            bs = sh;
            ba = sa;
          }
        }
    h.tune.hgroups = bg;
    h.tune.hstab = bs;
    h.tune.stage = ba;
    rep.ms_layout[0] = best_ms;
  }
  h.tune.ulayout = 1;
  if ((rc = measure(after_hvhg, helm, &rep.ms_layout[1]))) return rc;
  h.tune.ulayout = rep.ms_layout[1] < rep.ms_layout[0] ? 1 : 0;
  auto solve = [&]() {
    cudaError_t e = launch_ws_hvhg(h, 2, nullptr, st);
    if (e == cudaSuccess) e = launch_ws_helmholtz(h, 2, nullptr, st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, h.ev_join, 0);
    return e;
  };
  const int athreads[3] = {128, 256, 512};
  for (int i = 0; i < 3; ++i) {
    h.tune.asm_threads = athreads[i];
    auto prep = [&]() -> int {
      int r = restore_joined();
      if (r) return r;
      TUNE_CUDA(solve());
      return KMM_OK;
    };
    auto body = [&]() { return launch_ws_assemble(h, 2, nullptr, st); };
    if ((rc = measure(prep, body, &rep.ms_assemble[i]))) return rc;
  }
  h.tune.asm_threads = athreads[best(rep.ms_assemble, 3)];
  // Whole steps through the step graph (the solver kernels beside the mean lines on the side
  // stream, as the step runs them) decide which picks stay: starting from the shapes the handle
  // had, each knob group takes its per-kernel pick only where the step gets 1% faster with it.  With
  // a fixed time step and no dt set yet (a handle tuned at creation) the timed steps use
  // dt = 1e-3; where a step cannot run (the CFL rule on a zero state) the entry shapes stay.
  const Tuning picked = h.tune;
  DevScalars dsc_step = dsc;
  dsc_step.err = 0;
  if (h.cfg.fixed_dt && !(dsc_step.dt > 1e-14)) dsc_step.dt = 1e-3;
  auto restore_step = [&]() -> int {
    TUNE_CUDA(cudaMemcpyAsync(h.S, h.staging, nfld * fb, cudaMemcpyDeviceToDevice, st));
    TUNE_CUDA(cudaMemcpyAsync(h.RK, h.staging + nfld * h.ns, nst * fb, cudaMemcpyDeviceToDevice, st));
    TUNE_CUDA(cudaMemcpyAsync(h.dsc, &dsc_step, sizeof(dsc_step), cudaMemcpyHostToDevice, st));
    return KMM_OK;
  };
  auto drop_graph = [&]() {
    if (h.gexec) cudaGraphExecDestroy(h.gexec);
    if (h.graph) cudaGraphDestroy(h.graph);
    h.gexec = nullptr;
    h.graph = nullptr;
  };
  // device ms of one step with `shapes`; 0 where the step raised a device error
  auto time_steps = [&](const Tuning &shapes, double *ms) -> int {
    h.tune = shapes;
    drop_graph();
    int r = capture_step_graph(h);
    if (r) return r;
    auto body = [&]() {
      cudaError_t e = cudaSuccess;
      for (int i = 0; i < kSteps && e == cudaSuccess; ++i) e = cudaGraphLaunch(h.gexec, st);
      return e;
    };
    if ((r = measure(restore_step, body, ms))) return r;
    *ms /= kSteps;
    int err = 0;
    TUNE_CUDA(cudaMemcpy(&err, &h.dsc->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) *ms = 0.0;
    return KMM_OK;
  };
  auto take_group = [&](Tuning t, int g) {
    switch (g) {
      case 0: t.z = picked.z; t.ztma = picked.ztma; break;
      case 1: t.x = picked.x; break;
      case 2: t.groups = picked.groups; t.stab = picked.stab; t.hvstage = picked.hvstage; break;
      case 3: t.hgroups = picked.hgroups; t.hstab = picked.hstab; t.stage = picked.stage; t.ulayout = picked.ulayout; break;
      default: t.asm_threads = picked.asm_threads; break;
    }
    return t;
  };
  auto same_shapes = [](const Tuning &a, const Tuning &b) {
    return a.z == b.z && a.ztma == b.ztma && a.x == b.x && a.groups == b.groups && a.stab == b.stab &&
           a.hvstage == b.hvstage && a.hgroups == b.hgroups && a.hstab == b.hstab && a.stage == b.stage &&
           a.ulayout == b.ulayout && a.asm_threads == b.asm_threads;
  };
  if ((rc = restore_joined())) return rc;  // the side stream's last mean lines are done
  Tuning kept = entry;
  if ((rc = time_steps(kept, &rep.ms_step[1]))) return rc;
  double kept_ms = rep.ms_step[1];
  for (int g = 0; g < 5 && kept_ms > 0.0; ++g) {
    const Tuning cand = take_group(kept, g);
    if (same_shapes(cand, kept)) continue;
    double ms = 0.0;
    if ((rc = time_steps(cand, &ms))) return rc;
    if (ms > 0.0 && ms < kMinGain * kept_ms) {
      kept = cand;
      kept_ms = ms;
    }
  }
  rep.ms_step[0] = kept_ms;
  h.tune = kept;
  drop_graph();
  // the captures left the join event's last record inside a graph: record it outside again
  TUNE_CUDA(cudaEventRecord(h.ev_join, h.side));
  if ((rc = restore_joined())) return rc;
  TUNE_CUDA(cudaStreamSynchronize(st));
  TUNE_CUDA(cudaStreamSynchronize(h.side));
  h.tune.tuned = true;
  std::memcpy(h.tune.ms_z, rep.ms_z, sizeof(rep.ms_z));
  std::memcpy(h.tune.ms_x, rep.ms_x, sizeof(rep.ms_x));
  std::memcpy(h.tune.ms_modes, rep.ms_modes, sizeof(rep.ms_modes));
  std::memcpy(h.tune.ms_layout, rep.ms_layout, sizeof(rep.ms_layout));
  std::memcpy(h.tune.ms_assemble, rep.ms_assemble, sizeof(rep.ms_assemble));
  std::memcpy(h.tune.ms_tables, rep.ms_tables, sizeof(rep.ms_tables));
  std::memcpy(h.tune.ms_helm, rep.ms_helm, sizeof(rep.ms_helm));
  std::memcpy(h.tune.ms_z_tma, rep.ms_z_tma, sizeof(rep.ms_z_tma));
  std::memcpy(h.tune.ms_hvhg, rep.ms_hvhg, sizeof(rep.ms_hvhg));
  std::memcpy(h.tune.ms_step, rep.ms_step, sizeof(rep.ms_step));
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
  out->helm_modes_per_block = 32 * h.tune.hgroups;
  out->helm_tables_shared = h.tune.hstab;
  out->helm_stage_ahead = h.nsc == 1 ? h.tune.stage : 1;
  out->z_tma = h.tune.ztma;
  out->hvhg_stage_ahead = h.tune.hvstage;
  out->u_layout = h.tune.ulayout;
  out->assemble_threads = h.tune.asm_threads;
  out->tuned = h.tune.tuned ? 1 : 0;
  out->tables_shared = h.tune.stab;
  out->factor_cache = h.tune.fcache;
  std::memcpy(out->ms_z, h.tune.ms_z, sizeof(out->ms_z));
  std::memcpy(out->ms_x, h.tune.ms_x, sizeof(out->ms_x));
  std::memcpy(out->ms_modes, h.tune.ms_modes, sizeof(out->ms_modes));
  std::memcpy(out->ms_layout, h.tune.ms_layout, sizeof(out->ms_layout));
  std::memcpy(out->ms_assemble, h.tune.ms_assemble, sizeof(out->ms_assemble));
  std::memcpy(out->ms_tables, h.tune.ms_tables, sizeof(out->ms_tables));
  std::memcpy(out->ms_helm, h.tune.ms_helm, sizeof(out->ms_helm));
  std::memcpy(out->ms_z_tma, h.tune.ms_z_tma, sizeof(out->ms_z_tma));
  std::memcpy(out->ms_hvhg, h.tune.ms_hvhg, sizeof(out->ms_hvhg));
  std::memcpy(out->ms_step, h.tune.ms_step, sizeof(out->ms_step));
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
  const bool tab_ok = (t->tables_shared == 0 || t->tables_shared == 1) &&
                      (t->hvhg_stage_ahead >= 0 && t->hvhg_stage_ahead <= 2) && g != 0 &&
                      hvhg_shape_fits(h, g, t->tables_shared, t->hvhg_stage_ahead);
  const int hg = t->helm_modes_per_block == 32 ? 1 : t->helm_modes_per_block == 64 ? 2
                 : t->helm_modes_per_block == 96 ? 3 : t->helm_modes_per_block == 128 ? 4 : 0;
  const bool helm_ok = hg != 0 && (t->helm_tables_shared == 0 || t->helm_tables_shared == 1) &&
                       (t->helm_stage_ahead == 1 || t->helm_stage_ahead == 2) &&
                       helm_shape_fits(h, hg, t->helm_tables_shared, t->helm_stage_ahead);
  const bool tma_ok = t->z_tma == 0 || (t->z_tma == 1 && zv >= 0 && z_tma_possible(h, zv));
  const bool fc_ok = t->factor_cache == 0 || (t->factor_cache == 1 && h.hf);
  if (zv < 0 || xv < 0 || g == 0 || (g == 2 && h.nsc != 1) || (t->u_layout != 0 && t->u_layout != 1) || !asm_ok ||
      !tab_ok || !helm_ok || !tma_ok || !fc_ok) {
    set_error("kmm_set_tuning: a requested shape is not among this grid's candidates (see kmm_autotune)");
    return KMM_ERR_ARG;
  }
  next.z = zv;
  next.x = xv;
  next.groups = g;
  next.ulayout = t->u_layout;
  next.asm_threads = t->assemble_threads;
  next.stab = t->tables_shared;
  next.hgroups = hg;
  next.hstab = t->helm_tables_shared;
  next.stage = t->helm_stage_ahead;
  next.ztma = t->z_tma;
  next.hvstage = t->hvhg_stage_ahead;
  next.fcache = t->factor_cache;
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
