// api.cu - the C ABI of libkmm (include/kmm.h).
//
// kmm_create         LABS_initialize + RK3_initialize + ppdfftw_initialize
//                    (module_labs.f90:77-238, module_runge_kutta.f90:28-54,
//                    module_ppdfftw.f90:499-588)
// kmm_time_march     time_march (time_march.f90:36-128), one substep
// kmm_step           the main.f90:134-193 loop body (three substeps) from a CUDA graph
// kmm_upload_state / kmm_download_state   the Y-pencil U / RK_STORE arrays
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "kmm_internal.h"

namespace kmm {

static thread_local std::string g_err;
void set_error(const std::string &msg) { g_err = msg; }

OpsOffsets ops_offsets(int bw, int ny) {
  OpsOffsets o;
  const int64_t band = (int64_t)(2 * bw + 1) * ny;
  o.d0 = 0;
  o.d1 = band;
  o.d2 = 2 * band;
  o.d0lu = 3 * band;
  o.integ = 4 * band;
  o.dyr = o.integ + ny;
  o.wlo = o.dyr + ny;
  o.whi = o.wlo + ny;
  o.t0 = o.whi + ny;
  o.total = o.t0 + (int64_t)ny * (3 * (4 * bw + 1) + (2 * bw + 1) + 2 * bw);
  return o;
}

namespace {

constexpr double kPiF = 3.14159265358979323;  // module_global_variable.f90:28

#define KMM_CUDA(call)                                                                   \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess) {                                                             \
      set_error(std::string("CUDA error: ") + cudaGetErrorString(e_) + " at " #call);    \
      return KMM_ERR_CUDA;                                                               \
    }                                                                                    \
  } while (0)

bool factor_radices(int n, std::vector<int> &rs) {
  rs.clear();
  int m = n;
  while (m % 4 == 0) { rs.push_back(4); m /= 4; }
  while (m % 2 == 0) { rs.push_back(2); m /= 2; }
  while (m % 3 == 0) { rs.push_back(3); m /= 3; }
  while (m % 5 == 0) { rs.push_back(5); m /= 5; }
  return m == 1 && (int)rs.size() <= kMaxPass && !rs.empty();
}

// pos(i) = (i mod r_m) * (n / r_m) + pos_{r_1..r_{m-1}}(i div r_m)
void digit_positions(int n, const std::vector<int> &rs, std::vector<int> &pos) {
  pos.assign(n, 0);
  for (int i = 0; i < n; ++i) {
    int idx = i, len = n, p = 0;
    for (int q = (int)rs.size() - 1; q >= 0; --q) {
      const int r = rs[q];
      len /= r;
      p += (idx % r) * len;
      idx /= r;
    }
    pos[i] = p;
  }
}

template <typename T> int dalloc(Handle &h, T **p, size_t count) {
  const size_t bytes = sizeof(T) * (count ? count : 1);
  cudaError_t e = cudaMalloc((void **)p, bytes);
  if (e != cudaSuccess) {
    set_error(std::string("cudaMalloc of ") + std::to_string(bytes) + " bytes failed: " + cudaGetErrorString(e));
    return KMM_ERR_CUDA;
  }
  h.device_bytes += (int64_t)bytes;
  return KMM_OK;
}

}  // namespace

int diag_buffers(Handle &h) {
  int rc = KMM_OK;
  if (!h.mixed) return rc;
  if (!h.mid64 && (rc = dalloc(h, &h.mid64, 6 * (size_t)h.nm))) return rc;
  if (!h.p64 && (rc = dalloc(h, &h.p64, 6 * (size_t)h.ns))) return rc;
  return rc;
}

namespace {

int validate(const kmm_config &c) {
  auto bad = [](const std::string &m) { set_error(m); return KMM_ERR_CONFIG; };
  if (c.no_of_field < 10) return bad("no_of_field must be >= 10: fields 1..10 are used (wavespace.f90:29)");
  if (c.rk_scheme != 3) return bad("Currently only 3rd order Runge-Kutta method is supported (rk_scheme = 3)");
  if (c.nx < 4 || c.nz < 4 || (c.nx % 2) || (c.nz % 2)) return bad("nx and nz must be even and >= 4");
  if (c.ny <= 2 * c.labs_k) return bad("K, order of B-spline, is too large (need ny > 2*labs_k)");
  if (c.labs_k < 1) return bad("labs_k must be >= 1");
  if (!(c.nu > 0.0) || !(c.pr > 0.0)) return bad("nu and pr must be positive");
  if (!(c.lmfx > 0.0) || !(c.lmfz > 0.0) || !(c.lmfy > 0.0)) return bad("LMFx, LMFy, LMFz must be positive");
  if (c.precision != KMM_PREC_FP64 && c.precision != KMM_PREC_MIXED) return bad("unknown precision");
  if (c.grid != KMM_GRID_SINE && c.grid != KMM_GRID_TANH) return bad("unknown grid map");
  if (c.control_amp != 0.0 && !(c.control_yd > -1.0 && c.control_yd < 0.0))
    return bad("control detection plane y_d must lie in (-1, 0)");
  if (c.n_scalar < 0 || c.n_scalar > 2) return bad("n_scalar must be 1 or 2");
  if (c.n_scalar == 2 && !(c.pr2 > 0.0)) return bad("pr2 (the second scalar's Prandtl number) must be positive");
  std::vector<int> rs;
  if (!factor_radices(c.nx * 3 / 2, rs) || !factor_radices(c.nz * 3 / 2, rs))
    return bad("3/2-padded lengths must factor into 2, 3, 5 with at most 8 passes");
  return KMM_OK;
}

int upload_ops(Handle &h) {
  OpsOffsets off = ops_offsets(h.bw, h.ny);
  std::vector<double> buf((size_t)off.total, 0.0);
  const size_t band = (size_t)(2 * h.bw + 1) * h.ny;
  std::memcpy(buf.data() + off.d0, h.ops.band[0].data(), band * sizeof(double));
  std::memcpy(buf.data() + off.d1, h.ops.band[1].data(), band * sizeof(double));
  std::memcpy(buf.data() + off.d2, h.ops.band[2].data(), band * sizeof(double));
  std::memcpy(buf.data() + off.d0lu, h.ops.d0_lu.data(), band * sizeof(double));
  std::memcpy(buf.data() + off.integ, h.ops.integ.data(), h.ny * sizeof(double));
  // dyr, module_ppdfftw.f90:573-583
  const std::vector<double> &y = h.ops.y;
  const double dyf = h.cfg.dy_factor;
  for (int i = 1; i <= h.ny; ++i) {
    double d;
    if (i == 1) d = 1.0 / (dyf * std::fabs(y[1] - y[0]));
    else if (i == h.ny) d = 1.0 / (dyf * std::fabs(y[h.ny - 1] - y[h.ny - 2]));
    else d = 1.0 / (dyf * std::fmin(std::fabs(y[i - 1] - y[i - 2]), std::fabs(y[i - 1] - y[i])));
    buf[off.dyr + i - 1] = d;
  }
  if (!h.ops.wlo.empty()) {
    std::memcpy(buf.data() + off.wlo, h.ops.wlo.data(), h.ny * sizeof(double));
    std::memcpy(buf.data() + off.whi, h.ops.whi.data(), h.ny * sizeof(double));
  }
  {
    double *t = buf.data() + off.t0;
    for (int d = 0; d < 3; ++d) {
      std::memcpy(t, h.ops.off[d].data(), h.ops.off[d].size() * sizeof(double));
      t += h.ops.off[d].size();
    }
    std::memcpy(t, h.ops.l0.data(), h.ops.l0.size() * sizeof(double));
    t += h.ops.l0.size();
    std::memcpy(t, h.ops.u0.data(), h.ops.u0.size() * sizeof(double));
  }
  KMM_CUDA(cudaMemcpy(h.dops, buf.data(), buf.size() * sizeof(double), cudaMemcpyHostToDevice));
  return KMM_OK;
}

int make_plans(Handle &h) {
  // one table region per length: pos (int) and twiddles (double2, float2)
  std::vector<int> rsx, rsz, posx, posz;
  factor_radices(h.nx32, rsx);
  factor_radices(h.nz32, rsz);
  digit_positions(h.nx32, rsx, posx);
  digit_positions(h.nz32, rsz, posz);
  h.radix_x = rsx;
  h.radix_z = rsz;
  const int nt = h.nx32 + h.nz32;
  int rc;
  if ((rc = dalloc(h, &h.fftpos, nt))) return rc;
  if ((rc = dalloc(h, &h.tw64, nt))) return rc;
  if ((rc = dalloc(h, &h.tw32, nt))) return rc;
  std::vector<int> pos(nt);
  std::vector<double2> t64(nt);
  std::vector<float2> t32(nt);
  auto fill = [&](int base, int n, const std::vector<int> &p) {
    for (int i = 0; i < n; ++i) {
      pos[base + i] = p[i];
      const long double ang = -2.0L * 3.141592653589793238462643383279502884L * (long double)i / (long double)n;
      const double c = (double)cosl(ang), s = (double)sinl(ang);
      t64[base + i] = make_double2(c, s);
      t32[base + i] = make_float2((float)cosl(ang), (float)sinl(ang));
    }
  };
  fill(0, h.nx32, posx);
  fill(h.nx32, h.nz32, posz);
  KMM_CUDA(cudaMemcpy(h.fftpos, pos.data(), nt * sizeof(int), cudaMemcpyHostToDevice));
  KMM_CUDA(cudaMemcpy(h.tw64, t64.data(), nt * sizeof(double2), cudaMemcpyHostToDevice));
  KMM_CUDA(cudaMemcpy(h.tw32, t32.data(), nt * sizeof(float2), cudaMemcpyHostToDevice));
  auto setp = [&](FftPlan &pl, int n, const std::vector<int> &rs, int base) {
    pl.n = n;
    pl.npass = (int)rs.size();
    for (int q = 0; q < kMaxPass; ++q) pl.radix[q] = q < pl.npass ? rs[q] : 0;
    pl.pos = h.fftpos + base;
    pl.tw64 = h.tw64 + base;
    pl.tw32 = h.tw32 + base;
  };
  setp(h.px, h.nx32, rsx, 0);
  setp(h.pz, h.nz32, rsz, h.nx32);
  return KMM_OK;
}

// One substep = the kernel sequence of time_march.  When ev is given, an event pair is
// recorded around every launch (ev[2*i], ev[2*i+1]) and ids[i] receives the kernel id.
int enqueue_substep(Handle &h, int s, cudaStream_t st, cudaEvent_t *ev = nullptr, int *ids = nullptr,
                    int *nrec = nullptr) {
  auto rec = [&](int id, auto &&launch) -> int {
    if (ev) KMM_CUDA(cudaEventRecord(ev[2 * (*nrec)], st));
    KMM_CUDA(launch());
    if (ev) {
      KMM_CUDA(cudaEventRecord(ev[2 * (*nrec) + 1], st));
      ids[(*nrec)++] = id;
    }
    return KMM_OK;
  };
  int rc;
  if ((rc = rec(KMM_K_BEGIN, [&] { return launch_begin_substep(h, s, st); }))) return rc;
  if ((rc = rec(KMM_K_ZINV, [&] { return launch_zinv(h, h.S, h.MID, 3 + h.nsc, st); }))) return rc;
  if ((rc = rec(KMM_K_XPHYS, [&] { return launch_xphys(h, h.MID, s, st); }))) return rc;
  if (s == 1)
    if ((rc = rec(KMM_K_DT, [&] { return launch_update_dt(h, s, st); }))) return rc;
  if ((rc = rec(KMM_K_ZFWD, [&] { return launch_zfwd(h, h.MID, h.P, 5 + 3 * h.nsc, h.rescale, !h.mixed, st); })))
    return rc;
  if ((rc = rec(KMM_K_HVHG, [&] { return launch_ws_hvhg(h, s, nullptr, st); }))) return rc;
  if ((rc = rec(KMM_K_HELMHOLTZ, [&] { return launch_ws_helmholtz(h, s, nullptr, st); }))) return rc;
  if ((rc = rec(KMM_K_ASSEMBLE, [&] { return launch_ws_assemble_only(h, s, nullptr, st); }))) return rc;
  // the mean lines (side stream) join here, outside the assembly's event pair
  KMM_CUDA(launch_ws_join(h, st));
  return KMM_OK;
}

int read_scalars(Handle &h, kmm_scalars *out, int *dev_err) {
  DevScalars d;
  KMM_CUDA(cudaMemcpy(&d, h.dsc, sizeof(d), cudaMemcpyDeviceToHost));
  *dev_err = d.err;
  if (out) {
    out->dt = d.dt;
    double vm;
    std::memcpy(&vm, &d.velmax_bits, sizeof(vm));
    out->velmax = vm;
    for (int i = 0; i < 4; ++i) {
      out->phi_dpdx[i] = d.phi_dpdx[i];
      out->phi_dtdx[i] = d.phi_dtdx[i];
    }
    out->wall_shear_stress = d.wall_shear_stress;
    out->wall_theta_stress = d.wall_theta_stress;
    for (int i = 0; i < 4; ++i) out->phi_dtdx2[i] = d.phi_dtdx2[i];
    out->wall_theta_stress2 = d.wall_theta_stress2;
  }
  return KMM_OK;
}

int check_device_error(Handle &h, int err) {
  if (!err) return KMM_OK;
  // clear the flag so the caller can retry with another dt
  int zero = 0;
  KMM_CUDA(cudaMemcpy(&h.dsc->err, &zero, sizeof(int), cudaMemcpyHostToDevice));
  if (err == KMM_ERR_DT) set_error("ABORT due to timestep dt (dt <= 1e-14 or dt > 1e5)");
  else if (err == KMM_ERR_NONFINITE) set_error("non-finite velocity in the physical-space step");
  else if (err == KMM_ERR_TIMEOUT) set_error("a bounded device wait gave up: a TMA tile copy of the z transforms did not complete");
  else set_error("device error " + std::to_string(err));
  return err;
}

// U slots of the state fields S 0..4: u, v, w, theta (fields 1, 2, 3, 7) and theta2 (field 11).
constexpr int kStateSlots[5] = {0, 1, 2, 6, 10};

int upload_fields(Handle &h, const double *U, int nf, const double *rk, cudaStream_t st) {
  const size_t fb = sizeof(double2) * (size_t)h.ns;
  const int nfld = 3 + h.nsc, nst = 2 + h.nsc;
  for (int i = 0; i < nfld; ++i)
    KMM_CUDA(cudaMemcpyAsync(h.staging + i * h.ns, U + 2 * (size_t)kStateSlots[i] * h.ns, fb, cudaMemcpyHostToDevice, st));
  KMM_CUDA(launch_ref_to_planes(h.staging, h.S, nfld, h.nmodes, h.ny, st));
  if (rk) {
    KMM_CUDA(cudaMemcpyAsync(h.staging + nfld * h.ns, rk, nst * fb, cudaMemcpyHostToDevice, st));
    KMM_CUDA(launch_ref_to_planes(h.staging + nfld * h.ns, h.RK, nst, h.nmodes, h.ny, st));
  }
  (void)nf;
  return KMM_OK;
}

int download_fields(Handle &h, double *U, int nf, double *rk, cudaStream_t st) {
  const size_t fb = sizeof(double2) * (size_t)h.ns;
  const int nfld = 3 + h.nsc, nst = 2 + h.nsc;
  KMM_CUDA(launch_planes_to_ref(h.S, h.staging, nfld, h.nmodes, h.ny, st));
  if (rk) KMM_CUDA(launch_planes_to_ref(h.RK, h.staging + nfld * h.ns, nst, h.nmodes, h.ny, st));
  if (U)
    for (int i = 0; i < nfld; ++i)
      KMM_CUDA(cudaMemcpyAsync(U + 2 * (size_t)kStateSlots[i] * h.ns, h.staging + i * h.ns, fb, cudaMemcpyDeviceToHost, st));
  if (rk) KMM_CUDA(cudaMemcpyAsync(rk, h.staging + nfld * h.ns, nst * fb, cudaMemcpyDeviceToHost, st));
  (void)nf;
  return KMM_OK;
}

// Fields a caller's U must hold: 7 (theta is field 7), 11 with a second scalar (field 11).
int min_fields(const Handle &h) { return h.nsc == 2 ? 11 : 7; }

int set_dt_device(Handle &h, double dt) {
  DevScalars d;
  KMM_CUDA(cudaMemcpy(&d, h.dsc, sizeof(d), cudaMemcpyDeviceToHost));
  d.dt = dt;
  d.err = 0;
  KMM_CUDA(cudaMemcpy(h.dsc, &d, sizeof(d), cudaMemcpyHostToDevice));
  return KMM_OK;
}

int ensure_graph(Handle &h) {
  if (h.gexec) return KMM_OK;
  KMM_CUDA(cudaStreamBeginCapture(h.stream, cudaStreamCaptureModeThreadLocal));
  int rc = KMM_OK;
  for (int s = 1; s <= 3 && rc == KMM_OK; ++s) rc = enqueue_substep(h, s, h.stream);
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(h.stream, &g);
  if (rc != KMM_OK) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) {
    set_error(std::string("graph capture failed: ") + cudaGetErrorString(e));
    return KMM_ERR_CUDA;
  }
  h.graph = g;
  KMM_CUDA(cudaGraphInstantiate(&h.gexec, g, 0));
  return KMM_OK;
}

void finish_step_scalars(kmm_scalars *out) {
  if (!out) return;
  out->phi_dpdx[3] = (out->phi_dpdx[0] + out->phi_dpdx[1] + out->phi_dpdx[2]) / out->dt;  // main.f90:147
  out->phi_dtdx[3] = (out->phi_dtdx[0] + out->phi_dtdx[1] + out->phi_dtdx[2]) / out->dt;  // main.f90:148
  out->phi_dtdx2[3] = (out->phi_dtdx2[0] + out->phi_dtdx2[1] + out->phi_dtdx2[2]) / out->dt;
}

}  // namespace

int run_substep(Handle &h, int substep, cudaStream_t st) { return enqueue_substep(h, substep, st); }

int read_device_scalars(Handle &h, kmm_scalars *out, int *dev_err) { return read_scalars(h, out, dev_err); }

int capture_step_graph(Handle &h) { return ensure_graph(h); }

}  // namespace kmm

using namespace kmm;

extern "C" {

const char *kmm_last_error(void) { return g_err.c_str(); }

int kmm_config_default(kmm_config *c) {
  if (!c) return KMM_ERR_ARG;
  std::memset(c, 0, sizeof(*c));
  c->nx = 64;
  c->ny = 65;
  c->nz = 64;
  c->no_of_field = 10;
  c->rk_scheme = 3;
  c->labs_k = 6;
  c->lmfx = 1.0;
  c->lmfy = 1.0;
  c->lmfz = 0.5;
  c->stretch = 0.9;
  c->grid = KMM_GRID_SINE;
  c->nu = 1.0 / 2800.0;
  c->pr = 0.71;
  c->bulk_vel_u = 1.0;
  c->bulk_vel_w = 0.0;
  c->bulk_t = 1.0;
  c->u_gal = 0.0;
  c->cfl = 1.0;
  c->dt_factor = 0.0;
  c->dy_factor = 1.0;
  c->fixed_dt = 0;
  c->precision = KMM_PREC_FP64;
  c->control_amp = 0.0;
  c->control_yd = -1.0 + 15.0 / 180.0;
  c->device = 0;
  c->n_scalar = 1;
  c->pr2 = 0.2;
  c->bulk_t2 = 1.0;
  return KMM_OK;
}

int kmm_read_input_file(const char *path, kmm_config *cfg) {
  if (!path || !cfg) return KMM_ERR_ARG;
  std::ifstream f(path);
  if (!f) {
    set_error(std::string("cannot open input file ") + path);
    return KMM_ERR_CONFIG;
  }
  kmm_config_default(cfg);
  std::vector<std::string> lines;
  std::string ln;
  while (std::getline(f, ln)) lines.push_back(ln);
  // value line k (0-based) is file line 2k+1, after a skipped header line
  auto vals = [&](int k) -> std::vector<std::string> {
    std::vector<std::string> out;
    if (2 * k + 1 >= (int)lines.size()) return out;
    std::string s = lines[2 * k + 1];
    for (char &ch : s) if (ch == ',') ch = ' ';
    std::istringstream is(s);
    std::string tok;
    while (is >> tok) out.push_back(tok);
    return out;
  };
  auto num = [](const std::string &t) {  // Fortran list-directed reals accept d exponents
    std::string s = t;
    for (char &ch : s) if (ch == 'd' || ch == 'D') ch = 'e';
    return std::stod(s);
  };
  try {
    auto v = vals(0);
    if (v.size() < 4) throw std::runtime_error("nx ny nz no_of_field");
    cfg->nx = (int)num(v[0]); cfg->ny = (int)num(v[1]); cfg->nz = (int)num(v[2]); cfg->no_of_field = (int)num(v[3]);
    v = vals(3); if (v.empty()) throw std::runtime_error("rk_scheme"); cfg->rk_scheme = (int)num(v[0]);
    v = vals(4); if (v.empty()) throw std::runtime_error("labs_k"); cfg->labs_k = (int)num(v[0]);
    v = vals(5); if (v.size() < 3) throw std::runtime_error("LMFx LMFy LMFz");
    cfg->lmfx = num(v[0]); cfg->lmfy = num(v[1]); cfg->lmfz = num(v[2]);
    v = vals(6); if (v.empty()) throw std::runtime_error("stretch"); cfg->stretch = num(v[0]);
    v = vals(8); if (v.size() < 2) throw std::runtime_error("nu pr"); cfg->nu = num(v[0]); cfg->pr = num(v[1]);
    v = vals(9); if (v.size() < 3) throw std::runtime_error("bulk velocities");
    cfg->bulk_vel_u = num(v[0]); cfg->bulk_vel_w = num(v[1]); cfg->bulk_t = num(v[2]);
    v = vals(10); if (v.empty()) throw std::runtime_error("u_gal"); cfg->u_gal = num(v[0]);
    v = vals(13); if (v.empty()) throw std::runtime_error("CFL"); cfg->cfl = num(v[0]);
    v = vals(14); if (v.empty()) throw std::runtime_error("dt_factor"); cfg->dt_factor = num(v[0]);
    v = vals(15); if (v.empty()) throw std::runtime_error("dy_factor"); cfg->dy_factor = num(v[0]);
  } catch (const std::exception &e) {
    set_error(std::string("malformed input file (") + e.what() + ")");
    return KMM_ERR_CONFIG;
  }
  return validate(*cfg);
}

int kmm_create(const kmm_config *cfg, kmm_handle **out) {
  if (!cfg || !out) {
    set_error("null argument");
    return KMM_ERR_ARG;
  }
  *out = nullptr;
  int rc = validate(*cfg);
  if (rc) return rc;
  Handle *h = new Handle();
  h->cfg = *cfg;
  h->nx = cfg->nx;
  h->ny = cfg->ny;
  h->nz = cfg->nz;
  h->nxh = cfg->nx / 2;
  h->nx32 = cfg->nx * 3 / 2;
  h->nz32 = cfg->nz * 3 / 2;
  h->nmodes = (int64_t)h->nxh * h->nz;
  h->ns = (int64_t)h->ny * h->nmodes;
  h->nm = (int64_t)h->ny * h->nz32 * h->nxh;
  h->mixed = cfg->precision == KMM_PREC_MIXED;
  h->nsc = cfg->n_scalar == 2 ? 2 : 1;
  // read_input_file.f90:94-116
  const double lx = cfg->lmfx * 2 * kPiF, lz = cfg->lmfz * 2 * kPiF;
  h->dxr = (double)cfg->nx / lx;
  h->dzr = (double)cfg->nz / lz;
  h->cflx = cfg->cfl / kPiF;
  h->rescale = 1.0 / ((double)h->nx32 * h->nz32);
  h->lmfxr = 1.0 / cfg->lmfx;
  h->lmfzr = 1.0 / cfg->lmfz;
  std::string err;
  rc = build_host_ops(cfg->labs_k + 1, cfg->ny, cfg->stretch, cfg->lmfy * 2, cfg->grid, h->ops, err);
  if (!rc && cfg->control_amp != 0.0) rc = build_control_weights(h->ops, cfg->control_yd, err);
  if (rc) {
    set_error(err);
    delete h;
    return rc;
  }
  h->bw = h->ops.bw;
  if (h->nsc == 2 && !fft4_supported(h->nx32)) {
    set_error("a second scalar needs nx*3/2 among the four-step lengths (12 ... 576)");
    delete h;
    return KMM_ERR_CONFIG;
  }
  if (h->bw < kMinBw || h->bw > kMaxBw) {
    set_error("detected band width " + std::to_string(h->bw) + " outside the compiled range 2..7");
    delete h;
    return KMM_ERR_CONFIG;
  }
  // The per-mode kernels index within a line, or within a U region of BW lines, in 32 bits.
  if ((int64_t)(2 * h->bw) * h->ns >= (int64_t)INT32_MAX) {
    set_error("grid too large: 2*bw*ny*nz*nx/2 must stay below 2^31");
    delete h;
    return KMM_ERR_CONFIG;
  }
  auto fail = [&](int code) {
    kmm_destroy(reinterpret_cast<kmm_handle *>(h));
    return code;
  };
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= cfg->device || cfg->device < 0) {
    set_error("no CUDA device available for the requested ordinal");
    delete h;
    return KMM_ERR_CUDA;
  }
  // the handle's resources live on cfg->device; the caller's current device is restored on return
  DeviceGuard dg(cfg->device);
  if (!dg.ok) {
    set_error("cudaSetDevice failed");
    delete h;
    return KMM_ERR_CUDA;
  }
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming) != cudaSuccess ||
      cudaStreamCreateWithFlags(&h->copy, cudaStreamNonBlocking) != cudaSuccess) {
    set_error("cudaStreamCreate failed");
    return fail(KMM_ERR_CUDA);
  }
  for (auto &ev : h->ev_io)
    if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
      set_error("cudaEventCreate failed");
      return fail(KMM_ERR_CUDA);
    }
  const size_t r2 = h->mixed ? sizeof(float2) : sizeof(double2);
  OpsOffsets off = ops_offsets(h->bw, h->ny);
  const int nfld = 3 + h->nsc, nst = 2 + h->nsc, nprod = 5 + 3 * h->nsc, x2 = h->nsc - 1;
  if ((rc = dalloc(*h, &h->S, nfld * h->ns))) return fail(rc);
  if ((rc = dalloc(*h, &h->RK, nst * h->ns))) return fail(rc);
  if ((rc = dalloc(*h, reinterpret_cast<char **>(&h->P), nprod * h->ns * r2))) return fail(rc);
  if ((rc = dalloc(*h, reinterpret_cast<char **>(&h->MID), nprod * h->nm * r2))) return fail(rc);
  if ((rc = dalloc(*h, &h->dops, (size_t)off.total))) return fail(rc);
  if ((rc = dalloc(*h, &h->gains, (size_t)h->nmodes))) return fail(rc);
  if ((rc = dalloc(*h, &h->vwall, 2 * (size_t)h->nmodes))) return fail(rc);
  if ((rc = dalloc(*h, &h->zc, (8 + 2 * x2) * (size_t)h->ns))) return fail(rc);
  if ((rc = dalloc(*h, &h->ec, (9 + 2 * x2) * (size_t)h->ns))) return fail(rc);
  if ((rc = dalloc(*h, &h->xr, 6 * (size_t)h->ns))) return fail(rc);
  if ((rc = dalloc(*h, &h->ub, (3 + x2) * (size_t)split_ub_role(*h)))) return fail(rc);
  if ((rc = dalloc(*h, &h->vf, (size_t)vop_factor_doubles(*h)))) return fail(rc);
  if ((rc = dalloc(*h, &h->dvw, 3 * (size_t)h->nmodes))) return fail(rc);
  if (factor_cache_possible(*h)) {
    // per substep: the two Helmholtz operators' factors, the four influence lines, v_h's walls
    if ((rc = dalloc(*h, &h->hf, 6 * (size_t)vop_factor_doubles(*h)))) return fail(rc);
    if ((rc = dalloc(*h, &h->hinf, 12 * (size_t)h->ns))) return fail(rc);
    if ((rc = dalloc(*h, &h->hdvh, 3 * (size_t)h->nmodes))) return fail(rc);
    if ((rc = dalloc(*h, &h->fcdt, 3))) return fail(rc);
    const double none[3] = {NAN, NAN, NAN};  // no dt cached yet
    if (cudaMemcpy(h->fcdt, none, sizeof(none), cudaMemcpyHostToDevice) != cudaSuccess) {
      set_error("factor cache set-up failed");
      return fail(KMM_ERR_CUDA);
    }
  }
  if ((rc = dalloc(*h, &h->w00, (3 + x2) * (size_t)h->ny * (8 + 2 * h->bw)))) return fail(rc);
  if ((rc = dalloc(*h, &h->staging, 10 * h->ns))) return fail(rc);
  if ((rc = dalloc(*h, &h->dsc, 1))) return fail(rc);
  if (cudaMemset(h->S, 0, sizeof(double2) * nfld * h->ns) != cudaSuccess ||
      cudaMemset(h->RK, 0, sizeof(double2) * nst * h->ns) != cudaSuccess ||
      cudaMemset(h->dsc, 0, sizeof(DevScalars)) != cudaSuccess) {
    set_error("cudaMemset failed");
    return fail(KMM_ERR_CUDA);
  }
  {
    std::vector<float> ones((size_t)h->nmodes, 1.0f);
    if (cudaMemcpy(h->gains, ones.data(), ones.size() * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) {
      set_error("gain upload failed");
      return fail(KMM_ERR_CUDA);
    }
  }
  if ((rc = upload_ops(*h))) return fail(rc);
  if ((rc = make_plans(*h))) return fail(rc);
  prepare_kernels(*h);
  {
    const cudaError_t e = prepare_transforms2();
    if (e != cudaSuccess) {
      set_error(std::string("transform set-up failed: ") + cudaGetErrorString(e));
      return fail(KMM_ERR_CUDA);
    }
  }
  if (cudaGetLastError() != cudaSuccess) {
    set_error("kernel attribute set-up failed");
    return fail(KMM_ERR_CUDA);
  }
  {
    // the v operator depends on k^2 alone: factor it once for the run
    cudaError_t e = launch_vop_factor(*h, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) {
      set_error(std::string("v operator factorisation failed: ") + cudaGetErrorString(e));
      return fail(KMM_ERR_CUDA);
    }
  }
  default_solver_shapes(*h);  // the untuned solver launch shapes
  // FP64 with two scalars at x lengths of 576 and more: 128 threads a row (x variant 1) instead
  // of 64, which the six packed output lines' shared memory had held to two warps a block
  // (384x257x384: x pass 8.54 -> 6.15 ms, 17.0 -> 19.4 steps/s, the tuner's pick there)
  if (!h->mixed && h->nsc == 2 && h->nx32 >= 576) h->tune.x = 1;
  // with a fixed time step the Helmholtz sweeps read their operators' cached factors
  h->tune.fcache = h->hf ? 1 : 0;
  // the z transforms stage their input tiles through TMA where the grid allows the tile map
  // (0.062 -> 0.054 ms y_to_x, 312 -> 315 steps/s at 192x129x192 mixed, same-box A/B)
  h->tune.ztma = z_tma_possible(*h, h->tune.z) ? 1 : 0;
  if (cfg->autotune && (rc = autotune(*h, nullptr))) return fail(rc);
  *out = reinterpret_cast<kmm_handle *>(h);
  return KMM_OK;
}

int kmm_destroy(kmm_handle *hh) {
  if (!hh) return KMM_OK;
  Handle *h = reinterpret_cast<Handle *>(hh);
  DeviceGuard dg(h->cfg.device);
  if (h->gexec) cudaGraphExecDestroy(h->gexec);
  if (h->graph) cudaGraphDestroy(h->graph);
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->side) cudaStreamSynchronize(h->side);
  adjoint_free(*h);
  void *ptrs[] = {h->S, h->RK, h->P, h->MID, h->dops, h->gains, h->vwall, h->zc,
                  h->ec, h->xr, h->ub, h->vf, h->dvw, h->w00, h->staging, h->stat,
                  h->mid64, h->p64, h->hf, h->hinf, h->hdvh, h->fcdt, h->fftpos, h->tw64, h->tw32, h->dsc};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  if (h->copy) cudaStreamSynchronize(h->copy);
  if (h->ev_fork) cudaEventDestroy(h->ev_fork);
  if (h->ev_join) cudaEventDestroy(h->ev_join);
  for (auto ev : h->ev_io)
    if (ev) cudaEventDestroy(ev);
  if (h->copy) cudaStreamDestroy(h->copy);
  if (h->side) cudaStreamDestroy(h->side);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return KMM_OK;
}

int kmm_get_info(const kmm_handle *hh, kmm_info *info) {
  if (!hh || !info) return KMM_ERR_ARG;
  const Handle *h = reinterpret_cast<const Handle *>(hh);
  std::memset(info, 0, sizeof(*info));
  info->bw = h->bw;
  info->nxh = h->nxh;
  info->nx32 = h->nx32;
  info->nz32 = h->nz32;
  info->nmodes = h->nmodes;
  info->device_bytes = h->device_bytes;
  for (size_t i = 0; i < h->radix_x.size() && i < 8; ++i) info->fft_radix_x[i] = h->radix_x[i];
  for (size_t i = 0; i < h->radix_z.size() && i < 8; ++i) info->fft_radix_z[i] = h->radix_z[i];
  return KMM_OK;
}

int kmm_get_operators(const kmm_handle *hh, double *y, double *integ, double *d0, double *d1,
                      double *d2, double *d0_lu) {
  if (!hh) return KMM_ERR_ARG;
  const Handle *h = reinterpret_cast<const Handle *>(hh);
  const size_t band = (size_t)(2 * h->bw + 1) * h->ny;
  if (y) std::memcpy(y, h->ops.y.data(), h->ny * sizeof(double));
  if (integ) std::memcpy(integ, h->ops.integ.data(), h->ny * sizeof(double));
  if (d0) std::memcpy(d0, h->ops.band[0].data(), band * sizeof(double));
  if (d1) std::memcpy(d1, h->ops.band[1].data(), band * sizeof(double));
  if (d2) std::memcpy(d2, h->ops.band[2].data(), band * sizeof(double));
  if (d0_lu) std::memcpy(d0_lu, h->ops.d0_lu.data(), band * sizeof(double));
  return KMM_OK;
}

int kmm_upload_state(kmm_handle *hh, const double *U, int nf, const double *rk, double dt) {
  if (!hh || !U || nf < 7) {
    set_error("kmm_upload_state: null pointer or nf < 7");
    return KMM_ERR_ARG;
  }
  Handle &h = *reinterpret_cast<Handle *>(hh);
  if (nf < min_fields(h)) {
    set_error("kmm_upload_state: a second scalar needs nf >= 11 (it is field 11)");
    return KMM_ERR_ARG;
  }
  DeviceGuard dg(h.cfg.device);
  int rc = upload_fields(h, U, nf, rk, h.stream);
  if (rc) return rc;
  KMM_CUDA(cudaStreamSynchronize(h.stream));
  return set_dt_device(h, dt);
}

int kmm_download_state(kmm_handle *hh, double *U, int nf, double *rk) {
  if (!hh || (!U && !rk) || (U && nf < 7)) {
    set_error("kmm_download_state: null pointer or nf < 7");
    return KMM_ERR_ARG;
  }
  Handle &h = *reinterpret_cast<Handle *>(hh);
  if (U && nf < min_fields(h)) {
    set_error("kmm_download_state: a second scalar needs nf >= 11 (it is field 11)");
    return KMM_ERR_ARG;
  }
  DeviceGuard dg(h.cfg.device);
  int rc = download_fields(h, U, nf, rk, h.stream);
  if (rc) return rc;
  KMM_CUDA(cudaStreamSynchronize(h.stream));
  return KMM_OK;
}

int kmm_set_initial_data_uvw(kmm_handle *hh, const double *U, int nf, double dt) {
  if (!hh || !U || nf < 7) {
    set_error("kmm_set_initial_data_uvw: null pointer or nf < 7");
    return KMM_ERR_ARG;
  }
  Handle &h = *reinterpret_cast<Handle *>(hh);
  if (nf < min_fields(h)) {
    set_error("kmm_set_initial_data_uvw: a second scalar needs nf >= 11 (it is field 11)");
    return KMM_ERR_ARG;
  }
  DeviceGuard dg(h.cfg.device);
  int rc = upload_fields(h, U, nf, nullptr, h.stream);
  if (rc) return rc;
  KMM_CUDA(launch_init_stores(h, h.stream));
  KMM_CUDA(cudaStreamSynchronize(h.stream));
  return set_dt_device(h, dt);
}

int kmm_time_march(kmm_handle *hh, int s, kmm_scalars *out) {
  if (!hh || s < 1 || s > 3) {
    set_error("kmm_time_march: bad handle or rk_substep");
    return KMM_ERR_ARG;
  }
  Handle &h = *reinterpret_cast<Handle *>(hh);
  DeviceGuard dg(h.cfg.device);
  int rc = enqueue_substep(h, s, h.stream);
  if (rc) return rc;
  KMM_CUDA(cudaStreamSynchronize(h.stream));
  int err = 0;
  if ((rc = read_scalars(h, out, &err))) return rc;
  return check_device_error(h, err);
}

int kmm_step_async(kmm_handle *hh, int nsteps) {
  if (!hh || nsteps < 0) return KMM_ERR_ARG;
  Handle &h = *reinterpret_cast<Handle *>(hh);
  DeviceGuard dg(h.cfg.device);
  int rc = ensure_graph(h);
  if (rc) return rc;
  for (int i = 0; i < nsteps; ++i) KMM_CUDA(cudaGraphLaunch(h.gexec, h.stream));
  return KMM_OK;
}

int kmm_sync(kmm_handle *hh, kmm_scalars *out) {
  if (!hh) return KMM_ERR_ARG;
  Handle &h = *reinterpret_cast<Handle *>(hh);
  DeviceGuard dg(h.cfg.device);
  KMM_CUDA(cudaStreamSynchronize(h.stream));
  int err = 0, rc;
  if ((rc = read_scalars(h, out, &err))) return rc;
  finish_step_scalars(out);
  return check_device_error(h, err);
}

int kmm_step(kmm_handle *hh, int nsteps, kmm_scalars *out) {
  int rc = kmm_step_async(hh, nsteps);
  if (rc) return rc;
  return kmm_sync(hh, out);
}

int kmm_ensemble_step(kmm_handle *const *hs, int n, int nsteps, kmm_scalars *outs) {
  if (!hs || n < 0 || nsteps < 0) {
    set_error("kmm_ensemble_step: null handle array or negative count");
    return KMM_ERR_ARG;
  }
  for (int i = 0; i < n; ++i)
    if (!hs[i]) {
      set_error("kmm_ensemble_step: null handle " + std::to_string(i));
      return KMM_ERR_ARG;
    }
  int first = KMM_OK;
  std::string msg;
  std::vector<char> queued((size_t)n, 0);
  for (int i = 0; i < n; ++i) {  // enqueue every channel before waiting on any
    const int rc = kmm_step_async(hs[i], nsteps);
    if (rc == KMM_OK) queued[(size_t)i] = 1;
    else if (first == KMM_OK) {
      first = rc;
      msg = kmm_last_error();
    }
  }
  for (int i = 0; i < n; ++i) {
    if (!queued[(size_t)i]) continue;
    const int rc = kmm_sync(hs[i], outs ? &outs[i] : nullptr);
    if (rc != KMM_OK && first == KMM_OK) {
      first = rc;
      msg = kmm_last_error();
    }
  }
  if (first != KMM_OK) set_error("kmm_ensemble_step: " + msg);
  return first;
}

// kmm_step_host without RK_STORE: the four fields cross the bus one at a time on h.copy while
// h.stream lays out the ones already there, and the D0 solve that rebuilds RK_STORE 2 from v
// (v goes first) runs under the copies of u, w, theta; on the way back each field's layout
// permutation overlaps the previous field's copy.  Same kernels and arithmetic as the serial
// path, in another order.
static int step_host_pipelined(Handle &h, double *U, int nsteps, kmm_scalars *out) {
  const size_t fb = sizeof(double2) * (size_t)h.ns;
  const int slots[4] = {0, 1, 2, 6};  // U slots of u, v, w, theta = S fields 0..3
  const int order[4] = {1, 0, 2, 3};
  cudaEvent_t *ev = h.ev_io;
  // the copies may overwrite staging only after earlier work on stream is done with it
  KMM_CUDA(cudaEventRecord(ev[8], h.stream));
  KMM_CUDA(cudaStreamWaitEvent(h.copy, ev[8], 0));
  for (int i = 0; i < 4; ++i) {
    const int f = order[i];
    KMM_CUDA(cudaMemcpyAsync(h.staging + f * h.ns, U + 2 * (size_t)slots[f] * h.ns, fb, cudaMemcpyHostToDevice,
                             h.copy));
    KMM_CUDA(cudaEventRecord(ev[f], h.copy));
  }
  for (int i = 0; i < 4; ++i) {
    const int f = order[i];
    KMM_CUDA(cudaStreamWaitEvent(h.stream, ev[f], 0));
    KMM_CUDA(launch_ref_to_planes(h.staging + f * h.ns, h.S + f * h.ns, 1, h.nmodes, h.ny, h.stream));
    if (f == 1) KMM_CUDA(launch_init_phi(h, h.stream));
  }
  KMM_CUDA(launch_init_elem(h, h.stream));
  int rc;
  if ((rc = kmm_step_async(reinterpret_cast<kmm_handle *>(&h), nsteps))) return rc;
  for (int f = 0; f < 4; ++f) {
    KMM_CUDA(launch_planes_to_ref(h.S + f * h.ns, h.staging + f * h.ns, 1, h.nmodes, h.ny, h.stream));
    KMM_CUDA(cudaEventRecord(ev[4 + f], h.stream));
    KMM_CUDA(cudaStreamWaitEvent(h.copy, ev[4 + f], 0));
    KMM_CUDA(cudaMemcpyAsync(U + 2 * (size_t)slots[f] * h.ns, h.staging + f * h.ns, fb, cudaMemcpyDeviceToHost,
                             h.copy));
  }
  KMM_CUDA(cudaEventRecord(ev[8], h.copy));
  KMM_CUDA(cudaStreamWaitEvent(h.stream, ev[8], 0));
  return kmm_sync(reinterpret_cast<kmm_handle *>(&h), out);
}

int kmm_step_host(kmm_handle *hh, double *U, int nf, double *rk, int nsteps, kmm_scalars *out) {
  if (!hh || !U || nf < 7) {
    set_error("kmm_step_host: null pointer or nf < 7");
    return KMM_ERR_ARG;
  }
  Handle &h = *reinterpret_cast<Handle *>(hh);
  DeviceGuard dg(h.cfg.device);
  if (nf < min_fields(h)) {
    set_error("kmm_step_host: a second scalar needs nf >= 11 (it is field 11)");
    return KMM_ERR_ARG;
  }
  if (!rk && h.nsc == 1) return step_host_pipelined(h, U, nsteps, out);
  int rc = upload_fields(h, U, nf, rk, h.stream);
  if (rc) return rc;
  // Without rk the stores are rebuilt from U, as the reference's restart option 1 does
  // (initial_step.f90:31-33).
  if (!rk) KMM_CUDA(launch_init_stores(h, h.stream));
  if ((rc = kmm_step_async(hh, nsteps))) return rc;
  if ((rc = download_fields(h, U, nf, rk, h.stream))) return rc;
  return kmm_sync(hh, out);
}

int kmm_get_pressure(kmm_handle *hh, double *P) {
  if (!hh || !P) {
    set_error("kmm_get_pressure: null pointer");
    return KMM_ERR_ARG;
  }
  Handle &h = *reinterpret_cast<Handle *>(hh);
  DeviceGuard dg(h.cfg.device);
  double2 *planes = h.staging, *ref = h.staging + h.ns;
  int rc;
  if ((rc = diag_buffers(h))) return rc;
  // the wall values nu d2v/dy2 of the state's v into dvw (get_statistics_1's dv/dy call)
  KMM_CUDA(launch_ydiff(h, 2, h.stream));
  const cudaError_t e = launch_pressure(h, planes, h.dvw, nullptr, h.stream);
  if (e == cudaErrorNotSupported) {
    set_error("kmm_get_pressure: nx*3/2 has no four-step FFT shape");
    return KMM_ERR_CONFIG;
  }
  KMM_CUDA(e);
  KMM_CUDA(launch_planes_to_ref(planes, ref, 1, h.nmodes, h.ny, h.stream));
  KMM_CUDA(cudaMemcpyAsync(P, ref, sizeof(double2) * (size_t)h.ns, cudaMemcpyDeviceToHost, h.stream));
  KMM_CUDA(cudaStreamSynchronize(h.stream));
  return KMM_OK;
}

int kmm_get_statistics(kmm_handle *hh, double *lines, double *spec_kx, double *spec_kz, double *centre,
                       double *P) {
  if (!hh) {
    set_error("kmm_get_statistics: null handle");
    return KMM_ERR_ARG;
  }
  Handle &h = *reinterpret_cast<Handle *>(hh);
  DeviceGuard dg(h.cfg.device);
  const StatLayout L = stat_layout(h);
  int rc;
  if ((rc = diag_buffers(h))) return rc;
  if (!h.stat) {
    if ((rc = dalloc(h, &h.stat, L.total))) return rc;
    KMM_CUDA(cudaMemcpy(h.stat + L.center, h.ops.center.data(), sizeof(double) * (size_t)h.ny,
                        cudaMemcpyHostToDevice));
  }
  const cudaError_t e = launch_statistics(h, h.stream);
  if (e == cudaErrorNotSupported) {
    set_error("kmm_get_statistics: nx*3/2 has no four-step FFT shape, or nx/2 is too large for the spectra");
    return KMM_ERR_CONFIG;
  }
  KMM_CUDA(e);
  const size_t ny = (size_t)h.ny;
  if (lines)
    KMM_CUDA(cudaMemcpyAsync(lines, h.stat + L.lines, sizeof(double) * KMM_STAT_NLINES * ny,
                             cudaMemcpyDeviceToHost, h.stream));
  if (spec_kx)
    KMM_CUDA(cudaMemcpyAsync(spec_kx, h.stat + L.skx, sizeof(double) * KMM_STAT_NSPEC * (size_t)h.nxh * ny,
                             cudaMemcpyDeviceToHost, h.stream));
  if (spec_kz)
    KMM_CUDA(cudaMemcpyAsync(spec_kz, h.stat + L.skz, sizeof(double) * KMM_STAT_NSPEC * (size_t)h.nz * ny,
                             cudaMemcpyDeviceToHost, h.stream));
  if (centre)
    KMM_CUDA(cudaMemcpyAsync(centre, h.stat + L.scal, 2 * sizeof(double), cudaMemcpyDeviceToHost, h.stream));
  if (P) {
    double2 *ref = h.staging + h.ns;
    KMM_CUDA(launch_planes_to_ref(h.staging, ref, 1, h.nmodes, h.ny, h.stream));
    KMM_CUDA(cudaMemcpyAsync(P, ref, sizeof(double2) * (size_t)h.ns, cudaMemcpyDeviceToHost, h.stream));
  }
  KMM_CUDA(cudaStreamSynchronize(h.stream));
  return KMM_OK;
}

namespace {
// Dataset names of the reference's stat file (get_statistics.f90:60-284, 376-530) and of its
// spectra file (write_energy_spectra.f90:76-226).
const char *const kLineNames[KMM_STAT_NLINES] = {
    "U", "W", "Theta", "dUdy", "dWdy", "dTdy",
    "uu", "vv", "P", "ww", "tt", "uv", "uw", "vw", "ut", "wt", "vt",
    "2nududxidudxi", "2nudvdxidvdxi", "2nudwdxidwdxi", "2nududxidvdxi",
    "omega_x_omega_x", "omega_y_omega_y", "omega_z_omega_z", "omega_x_omega_y",
    "omega_y_omega_z", "omega_x_omega_z", "v_omega_z", "w_omega_y",
    "uuu", "vvv", "www", "uuuu", "vvvv", "wwww",
    "u6", "v6", "w6", "u8", "v8", "w8", "u10", "v10", "w10",
    "-duuvdy", "-dvvvdy", "-dvwwdy", "-duvvdy",
    "up", "-dpudy", "vp", "-2dpvdy", "wp", "pp",
    "2pdudx", "2pdvdy", "2pdwdz", "pdudy+pdvdx"};
const char *const kSpecNames[KMM_STAT_NSPEC] = {"uu", "vv", "ww", "tt", "uv", "vw", "uw", "ut", "vt",
                                                "wt", "oxox", "oyoy", "ozoz", "oxoy", "oxoz", "oyoz",
                                                "voz", "woy"};
}  // namespace

const char *kmm_stat_line_name(int i) { return (i >= 0 && i < KMM_STAT_NLINES) ? kLineNames[i] : nullptr; }
const char *kmm_stat_spec_name(int i) { return (i >= 0 && i < KMM_STAT_NSPEC) ? kSpecNames[i] : nullptr; }

int kmm_get_stream(const kmm_handle *hh, void **stream) {
  if (!hh || !stream) return KMM_ERR_ARG;
  *stream = reinterpret_cast<void *>(reinterpret_cast<const Handle *>(hh)->stream);
  return KMM_OK;
}

int kmm_profile_step(kmm_handle *hh, int nsteps, double *ms, int *launches) {
  if (!hh || nsteps <= 0 || !ms || !launches) return KMM_ERR_ARG;
  Handle &h = *reinterpret_cast<Handle *>(hh);
  DeviceGuard dg(h.cfg.device);
  const int per_step = 3 * KMM_NKERNEL;
  const int nmax = per_step * nsteps;
  std::vector<cudaEvent_t> ev(2 * nmax, nullptr);
  std::vector<int> ids(nmax, -1);
  for (auto &e : ev) KMM_CUDA(cudaEventCreate(&e));
  int nrec = 0, rc = KMM_OK;
  for (int n = 0; n < nsteps && rc == KMM_OK; ++n)
    for (int s = 1; s <= 3 && rc == KMM_OK; ++s) rc = enqueue_substep(h, s, h.stream, ev.data(), ids.data(), &nrec);
  cudaError_t se = cudaStreamSynchronize(h.stream);
  for (int k = 0; k < KMM_NKERNEL; ++k) {
    ms[k] = 0.0;
    launches[k] = 0;
  }
  for (int i = 0; i < nrec && se == cudaSuccess; ++i) {
    float t = 0.f;
    cudaEventElapsedTime(&t, ev[2 * i], ev[2 * i + 1]);
    ms[ids[i]] += t;
    launches[ids[i]] += 1;
  }
  for (int k = 0; k < KMM_NKERNEL; ++k)
    if (launches[k]) ms[k] /= launches[k];
  for (auto &e : ev) cudaEventDestroy(e);
  if (rc) return rc;
  if (se != cudaSuccess) {
    set_error(std::string("profile step failed: ") + cudaGetErrorString(se));
    return KMM_ERR_CUDA;
  }
  int err = 0;
  if ((rc = read_scalars(h, nullptr, &err))) return rc;
  return check_device_error(h, err);
}

int kmm_get_dt(const kmm_handle *hh, double *dt) {
  if (!hh || !dt) return KMM_ERR_ARG;
  const Handle &h = *reinterpret_cast<const Handle *>(hh);
  DeviceGuard dg(h.cfg.device);
  KMM_CUDA(cudaMemcpy(dt, &h.dsc->dt, sizeof(double), cudaMemcpyDeviceToHost));
  return KMM_OK;
}

int kmm_set_dt(kmm_handle *hh, double dt) {
  if (!hh) return KMM_ERR_ARG;
  return set_dt_device(*reinterpret_cast<Handle *>(hh), dt);
}

int kmm_set_control_gains(kmm_handle *hh, const float *gains) {
  if (!hh) return KMM_ERR_ARG;
  Handle &h = *reinterpret_cast<Handle *>(hh);
  DeviceGuard dg(h.cfg.device);
  std::vector<float> g((size_t)h.nmodes, 1.0f);
  if (gains) {
    // input (nxh, nz) Fortran order = mode index kz * nxh + kx, the device order
    std::memcpy(g.data(), gains, g.size() * sizeof(float));
  }
  // steps already queued on the handle's stream read the gains: let them finish first
  KMM_CUDA(cudaStreamSynchronize(h.stream));
  KMM_CUDA(cudaMemcpy(h.gains, g.data(), g.size() * sizeof(float), cudaMemcpyHostToDevice));
  return KMM_OK;
}

int kmm_set_control(kmm_handle *hh, double amp, const float *gains, double yd) {
  if (!hh) return KMM_ERR_ARG;
  if (!std::isfinite(amp)) {
    set_error("kmm_set_control: non-finite amplitude");
    return KMM_ERR_ARG;
  }
  Handle &h = *reinterpret_cast<Handle *>(hh);
  DeviceGuard dg(h.cfg.device);
  if (amp != 0.0) {
    std::string err;
    HostOps ops = h.ops;  // the handle keeps its weights if the new plane is refused
    const int rc = build_control_weights(ops, yd, err);
    if (rc) {
      set_error("kmm_set_control: " + err);
      return rc;
    }
    const OpsOffsets off = ops_offsets(h.bw, h.ny);
    KMM_CUDA(cudaStreamSynchronize(h.stream));
    KMM_CUDA(cudaMemcpy(h.dops + off.wlo, ops.wlo.data(), sizeof(double) * (size_t)h.ny, cudaMemcpyHostToDevice));
    KMM_CUDA(cudaMemcpy(h.dops + off.whi, ops.whi.data(), sizeof(double) * (size_t)h.ny, cudaMemcpyHostToDevice));
    h.ops.wlo = ops.wlo;
    h.ops.whi = ops.whi;
    h.cfg.control_yd = yd;
  }
  const int rc = kmm_set_control_gains(hh, gains);
  if (rc) return rc;
  if (amp != h.cfg.control_amp) {
    // the amplitude is a kernel argument captured in the step graph: capture it again
    KMM_CUDA(cudaStreamSynchronize(h.stream));
    if (h.gexec) cudaGraphExecDestroy(h.gexec);
    if (h.graph) cudaGraphDestroy(h.graph);
    h.gexec = nullptr;
    h.graph = nullptr;
    h.cfg.control_amp = amp;
  }
  return KMM_OK;
}

int kmm_dev_y_to_x(kmm_handle *hh, const double *u, void *xp, void *stream) {
  if (!hh || !u || !xp) return KMM_ERR_ARG;
  Handle &h = *reinterpret_cast<Handle *>(hh);
  DeviceGuard dg(h.cfg.device);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  KMM_CUDA(launch_ref_to_planes(reinterpret_cast<const double2 *>(u), h.staging, 1, h.nmodes, h.ny, st));
  KMM_CUDA(launch_zinv(h, h.staging, xp, 1, st));
  return KMM_OK;
}

int kmm_dev_x_to_y(kmm_handle *hh, const void *xp, double *u, int rescale, void *stream) {
  if (!hh || !u || !xp) return KMM_ERR_ARG;
  Handle &h = *reinterpret_cast<Handle *>(hh);
  DeviceGuard dg(h.cfg.device);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  KMM_CUDA(launch_zfwd(h, xp, h.staging, 1, rescale ? h.rescale : 1.0, true, st));
  KMM_CUDA(launch_planes_to_ref(h.staging, reinterpret_cast<double2 *>(u), 1, h.nmodes, h.ny, st));
  return KMM_OK;
}

int kmm_dev_dft_x_realspace(kmm_handle *hh, void *xp, int s, double *velmax_dev, void *stream) {
  if (!hh || !xp || s < 1 || s > 3) return KMM_ERR_ARG;
  Handle &h = *reinterpret_cast<Handle *>(hh);
  if (h.nsc != 1) {
    set_error("kmm_dev_dft_x_realspace: the reference's 10-slot X-pencil carries one scalar");
    return KMM_ERR_CONFIG;
  }
  DeviceGuard dg(h.cfg.device);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const size_t r2 = h.mixed ? sizeof(float2) : sizeof(double2);
  const size_t fb = r2 * (size_t)h.nm;
  char *x = reinterpret_cast<char *>(xp);
  char *mid = reinterpret_cast<char *>(h.MID);
  const int in_slots[4] = {0, 1, 2, 6};
  const int out_slots[8] = {0, 1, 2, 3, 4, 6, 7, 8};
  for (int i = 0; i < 4; ++i)
    KMM_CUDA(cudaMemcpyAsync(mid + i * fb, x + in_slots[i] * fb, fb, cudaMemcpyDeviceToDevice, st));
  KMM_CUDA(launch_begin_substep(h, 1, st));
  KMM_CUDA(launch_xphys(h, h.MID, s, st));
  for (int i = 0; i < 8; ++i)
    KMM_CUDA(cudaMemcpyAsync(x + out_slots[i] * fb, mid + i * fb, fb, cudaMemcpyDeviceToDevice, st));
  if (velmax_dev)
    KMM_CUDA(cudaMemcpyAsync(velmax_dev, &h.dsc->velmax_bits, sizeof(double), cudaMemcpyDeviceToDevice, st));
  return KMM_OK;
}

int kmm_dev_wavespace(kmm_handle *hh, double *U, double *rk, int s, double dt, kmm_scalars *out,
                      void *stream) {
  if (!hh || !U || !rk || s < 1 || s > 3) return KMM_ERR_ARG;
  Handle &h = *reinterpret_cast<Handle *>(hh);
  if (h.nsc != 1) {
    set_error("kmm_dev_wavespace: the reference's 10-slot U carries one scalar");
    return KMM_ERR_CONFIG;
  }
  DeviceGuard dg(h.cfg.device);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const double2 *Uc = reinterpret_cast<const double2 *>(U);
  const int pslots[8] = {0, 1, 2, 3, 4, 6, 7, 8};
  for (int i = 0; i < 8; ++i)
    KMM_CUDA(launch_ref_to_planes(Uc + pslots[i] * h.ns, h.staging + i * h.ns, 1, h.nmodes, h.ny, st));
  if (h.mixed) convert_planes_d2f(h.staging, reinterpret_cast<float2 *>(h.P), 8 * h.ns, st);
  else KMM_CUDA(cudaMemcpyAsync(h.P, h.staging, sizeof(double2) * 8 * h.ns, cudaMemcpyDeviceToDevice, st));
  KMM_CUDA(launch_ref_to_planes(Uc + 9 * h.ns, h.S + h.ns, 1, h.nmodes, h.ny, st));  // v for control
  KMM_CUDA(launch_ref_to_planes(reinterpret_cast<const double2 *>(rk), h.RK, 3, h.nmodes, h.ny, st));
  KMM_CUDA(cudaStreamSynchronize(st));
  int rc = set_dt_device(h, dt);
  if (rc) return rc;
  KMM_CUDA(launch_wavespace_split(h, s, nullptr, st));
  const int sslots[4] = {0, 1, 2, 6};
  for (int i = 0; i < 4; ++i)
    KMM_CUDA(launch_planes_to_ref(h.S + i * h.ns, reinterpret_cast<double2 *>(U) + sslots[i] * h.ns, 1, h.nmodes, h.ny, st));
  KMM_CUDA(launch_planes_to_ref(h.RK, reinterpret_cast<double2 *>(rk), 3, h.nmodes, h.ny, st));
  KMM_CUDA(cudaStreamSynchronize(st));
  int err = 0;
  if ((rc = read_scalars(h, out, &err))) return rc;
  return check_device_error(h, err);
}

int kmm_dev_labs_lu(kmm_handle *hh, double *a, int nm, void *stream) {
  if (!hh || !a || nm <= 0) return KMM_ERR_ARG;
  Handle &h = *reinterpret_cast<Handle *>(hh);
  DeviceGuard dg(h.cfg.device);
  KMM_CUDA(launch_labs_lu(h, a, nm, reinterpret_cast<cudaStream_t>(stream)));
  return KMM_OK;
}

int kmm_dev_labs_bs(kmm_handle *hh, const double *a, double *b, int nm, void *stream) {
  if (!hh || !a || !b || nm <= 0) return KMM_ERR_ARG;
  Handle &h = *reinterpret_cast<Handle *>(hh);
  DeviceGuard dg(h.cfg.device);
  KMM_CUDA(launch_labs_bs(h, a, reinterpret_cast<double2 *>(b), nm, reinterpret_cast<cudaStream_t>(stream)));
  return KMM_OK;
}

int kmm_dev_labs_mat_mul(kmm_handle *hh, int which, const double *x, double *b, int nm, void *stream) {
  if (!hh || !x || !b || nm <= 0 || which < 0 || which > 2) return KMM_ERR_ARG;
  Handle &h = *reinterpret_cast<Handle *>(hh);
  DeviceGuard dg(h.cfg.device);
  KMM_CUDA(launch_labs_mat_mul(h, which, reinterpret_cast<const double2 *>(x), reinterpret_cast<double2 *>(b), nm,
                               reinterpret_cast<cudaStream_t>(stream)));
  return KMM_OK;
}

}  // extern "C"
