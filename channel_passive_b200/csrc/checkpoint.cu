// checkpoint.cu - restart files of a handle: data_store (data_store.f90:11-173) and the restart
// branch of initial_step (initial_step.f90:15-56, 184-513), through the HDF5 codec of h5io.cpp.
//
// The state crosses to the host in the reference layout (kmm_download_state / kmm_upload_state),
// so a file written here is the file the reference writes for the same state, and a reference
// file restarts a handle.  Restart options 2 and 3 rebuild u, v, w (and phi) from the fields the
// file holds, per mode, with the reference's packed-band LU, substitution and mat-vec (labs.cuh,
// compiled for the host here) in the statement order of set_initial_data_gphi / _vg; this runs
// once per restart on the host cores, one thread per block of kz rows.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <ctime>
#include <string>
#include <thread>
#include <vector>

#include "kmm_internal.h"
#include "labs.cuh"

namespace kmm {
namespace {

// A checkpoint file that is dropped unwritten unless it is closed explicitly.
struct Io {
  kmm_io *io = nullptr;
  ~Io() {
    if (io) io_discard(io);
  }
};

// wavenumber of kz index j (0..nz/2, -nz/2+1..-1, module_ppdfftw.f90:347-384)
int kz_of(int j, int nz) { return j <= nz / 2 ? j : j - nz; }

template <typename F>
void over_kz(int nz, F &&fn) {
  const unsigned nt = std::max(1u, std::min(std::thread::hardware_concurrency(), 32u));
  std::vector<std::thread> pool;
  for (unsigned t = 0; t < nt; ++t)
    pool.emplace_back([&, t] {
      for (int j = (int)t; j < nz; j += (int)nt) fn(j);
    });
  for (std::thread &th : pool) th.join();
}

// set_initial_data_gphi (initial_step.f90:430-513): u, v, w from g, phi (RK stores 1, 2), theta
// from RK store 3; the mean mode takes U, W, theta from the stores.
template <int BW>
void rebuild_gphi(const Handle &h, double2 *U, const double2 *RK) {
  const int ny = h.ny, nxh = h.nxh, nz = h.nz, ld = 2 * BW + 1;
  const int64_t ns = (int64_t)ny * nxh * nz;
  const double *D0 = h.ops.band[0].data(), *D1 = h.ops.band[1].data(), *D2 = h.ops.band[2].data();
  over_kz(nz, [&](int j) {
    std::vector<double> Dbuf((size_t)ld * ny);
    std::vector<double2> c(ny);
    for (int k = 0; k < nxh; ++k) {
      const int64_t o = (int64_t)ny * (k + (int64_t)nxh * j);
      double2 *u1 = U + o, *u2 = U + ns + o, *u3 = U + 2 * ns + o, *u7 = U + 6 * ns + o;
      const double2 *g = RK + o, *phi = RK + ns + o, *th = RK + 2 * ns + o;
      if (k == 0 && j == 0) {
        for (int i = 0; i < ny; ++i) {
          u1[i] = g[i];
          u3[i] = phi[i];
          u7[i] = th[i];
          u2[i] = z2(0.0, 0.0);
        }
        continue;
      }
      const double kx = (double)k, kz = (double)kz_of(j, nz);
      const double k2 = (kz * h.lmfzr) * (kz * h.lmfzr) + (kx * h.lmfxr) * (kx * h.lmfxr);
      const double2 kxx = z2(0.0, kx * h.lmfxr / k2), kzz = z2(0.0, kz * h.lmfzr / k2);
      auto B = [&](int r, int m) -> double & { return Dbuf[(size_t)(m - 1) * ld + r - 1]; };
      auto A = [&](const double *a, int r, int m) { return a[(size_t)(m - 1) * ld + r - 1]; };
      for (int m : {1, ny}) {
        for (int i = 1; i <= 2 * BW + 1; ++i) B(i, m) = 0.0;
        B(BW + 1, m) = -k2 * A(D0, BW + 1, m) + A(D2, BW + 1, m);
      }
      for (int m = 2; m <= ny - 1; ++m)
        for (int i = 1; i <= 2 * BW + 1; ++i) B(i, m) = -k2 * A(D0, i, m) + A(D2, i, m);
      labs_lu<BW>(BandM<BW>{Dbuf.data(), 1}, ny);
      for (int i = 0; i < ny; ++i) c[i] = phi[i];
      c[0] = z2(0.0, 0.0);
      c[ny - 1] = z2(0.0, 0.0);
      labs_bs<BW>(BandM<BW>{Dbuf.data(), 1}, DLine{c.data(), 1}, ny);
      labs_mat_mul<BW>(BandM<BW>{const_cast<double *>(D0), 1}, DLine{c.data(), 1}, DLine{u2, 1}, ny);
      labs_mat_mul<BW>(BandM<BW>{const_cast<double *>(D1), 1}, DLine{c.data(), 1}, DLine{u3, 1}, ny);
      for (int i = 0; i < ny; ++i) {
        const double2 dxg = zmul(kxx, g[i]), dzg = zmul(kzz, g[i]);
        const double2 dxf = zmul(kxx, u3[i]), dzf = zmul(kzz, u3[i]);
        u1[i] = zsub(dxf, dzg);
        u3[i] = zadd(dxg, dzf);
      }
      for (int i = 0; i < ny; ++i) u7[i] = th[i];
    }
  });
}

// set_initial_data_vg (initial_step.f90:301-353): u, w and phi (RK store 2) from v and g (RK
// store 1), theta from RK store 3; the mean mode takes U, W, theta from the stores.
template <int BW>
void rebuild_vg(const Handle &h, double2 *U, double2 *RK) {
  const int ny = h.ny, nxh = h.nxh, nz = h.nz;
  const int64_t ns = (int64_t)ny * nxh * nz;
  double *D0lu = const_cast<double *>(h.ops.d0_lu.data());
  double *D1 = const_cast<double *>(h.ops.band[1].data()), *D2 = const_cast<double *>(h.ops.band[2].data());
  over_kz(nz, [&](int j) {
    std::vector<double2> c(ny), dv(ny);
    for (int k = 0; k < nxh; ++k) {
      const int64_t o = (int64_t)ny * (k + (int64_t)nxh * j);
      double2 *u1 = U + o, *u2 = U + ns + o, *u3 = U + 2 * ns + o, *u7 = U + 6 * ns + o;
      double2 *g = RK + o, *phi = RK + ns + o, *th = RK + 2 * ns + o;
      if (k == 0 && j == 0) {
        for (int i = 0; i < ny; ++i) {
          u1[i] = g[i];
          u2[i] = z2(0.0, 0.0);
          u3[i] = phi[i];
          u7[i] = th[i];
        }
        continue;
      }
      const double kx = (double)k, kz = (double)kz_of(j, nz);
      for (int i = 0; i < ny; ++i) c[i] = u2[i];
      labs_bs<BW>(BandM<BW>{D0lu, 1}, DLine{c.data(), 1}, ny);
      labs_mat_mul<BW>(BandM<BW>{D1, 1}, DLine{c.data(), 1}, DLine{dv.data(), 1}, ny);
      labs_mat_mul<BW>(BandM<BW>{D2, 1}, DLine{c.data(), 1}, DLine{phi, 1}, ny);
      const double k2 = (kx * h.lmfxr) * (kx * h.lmfxr) + (kz * h.lmfzr) * (kz * h.lmfzr);
      for (int i = 0; i < ny; ++i) phi[i] = zsub(phi[i], zscale(k2, u2[i]));
      const double2 kxx = z2(0.0, kx * h.lmfxr / k2), kzz = z2(0.0, kz * h.lmfzr / k2);
      for (int i = 0; i < ny; ++i) {
        const double2 dxg = zmul(kxx, g[i]), dzg = zmul(kzz, g[i]);
        const double2 dxf = zmul(kxx, dv[i]), dzf = zmul(kzz, dv[i]);
        u1[i] = zsub(dxf, dzg);
        u3[i] = zadd(dxg, dzf);
      }
      for (int i = 0; i < ny; ++i) u7[i] = th[i];
    }
  });
}

template <typename F>
void by_bw(int bw, F &&fn) {
  switch (bw) {
    case 2: fn.template operator()<2>(); break;
    case 3: fn.template operator()<3>(); break;
    case 4: fn.template operator()<4>(); break;
    case 5: fn.template operator()<5>(); break;
    case 6: fn.template operator()<6>(); break;
    case 7: fn.template operator()<7>(); break;
    default: break;
  }
}

#define IO(call)                 \
  do {                           \
    const int rc_ = (call);      \
    if (rc_ != KMM_OK) return rc_; \
  } while (0)

}  // namespace
}  // namespace kmm

using namespace kmm;

extern "C" {

int kmm_data_store(kmm_handle *hh, const char *path, int32_t timestep, double time, int32_t fields) {
  if (!hh || !path || fields < 0 || fields > KMM_STORE_ALL) return KMM_ERR_ARG;
  Handle &h = *reinterpret_cast<Handle *>(hh);
  const kmm_config &c = h.cfg;
  const int ny = h.ny, nxh = h.nxh, nz = h.nz, nf = h.nsc == 2 ? 11 : 7, nst = 2 + h.nsc;
  const int64_t ns = (int64_t)ny * nxh * nz;
  std::vector<double2> U((size_t)(ns * nf)), RK((size_t)(ns * nst));
  IO(kmm_download_state(hh, reinterpret_cast<double *>(U.data()), nf, reinterpret_cast<double *>(RK.data())));
  double dt = 0.0;
  IO(kmm_get_dt(hh, &dt));
  // data_store adds U_gal to the mean streamwise velocity before it writes U_mean and u
  for (int i = 0; i < ny; ++i) U[i].x += c.u_gal;

  Io f;
  IO(kmm_io_create(path, 1, &f.io));
  kmm_io *io = f.io;
  IO(kmm_io_string_set(io, "Readme",
                       "This file contains the information necessary to restart inhomogeneous channel flow. "
                       "It features the instantaneous 3D velocity field and the problem definition."));
  {
    const std::time_t now = std::time(nullptr);
    std::tm t{};
    localtime_r(&now, &t);
    char d[32], s[32];
    std::snprintf(d, sizeof d, "%4d/%2d/%2d", t.tm_year + 1900, t.tm_mon + 1, t.tm_mday);
    std::snprintf(s, sizeof s, "%2d:%2d:%2d", t.tm_hour, t.tm_min, t.tm_sec);
    IO(kmm_io_string_set(io, "Date of Saving (Year/Month/Day) : ", d));
    IO(kmm_io_string_set(io, "Time of Saving (Hour:Minute:Second) : ", s));
  }
  auto wi = [&](const char *n, int32_t v, const char *cm) { return kmm_io_line_write_integer(io, n, 1, &v, cm); };
  auto wd = [&](const char *n, double v, const char *cm) { return kmm_io_line_write_double(io, n, 1, &v, cm); };
  const double pi2 = 2.0 * M_PI;
  IO(wi("timestep", timestep, "Current step in time"));
  IO(wd("time", time, "Simulation Time"));
  IO(wd("nu", c.nu, "Viscosity or 1/Re"));
  IO(wd("Pr", c.pr, "Prantal number"));
  IO(wd("U_gal", c.u_gal, "Galilean transformation velocity"));
  IO(wd("U_avg", c.bulk_vel_u, "Bulk(average) velocity U - used for forcing"));
  IO(wd("W_avg", c.bulk_vel_w, "Bulk(average) velocity W - used for forcing"));
  IO(wd("T_avg", c.bulk_t, "Bulk(average) passive scalar - used for forcing"));
  IO(wd("Re", 1.0 / c.nu, "Reynold Number (not Re_tau)"));
  IO(wd("LMFx", c.lmfx, "Length Multiplication Factor(streamwise direction) : Lx=LMFx*2pi"));
  IO(wd("LMFy", c.lmfy, "Length Multiplication Factor(wall normal direction) : Ly=LMFy*2"));
  IO(wd("LMFz", c.lmfz, "Length Multiplication Factor(spanwise direction) : Lz=LMFz*2pi"));
  IO(wd("Lx", c.lmfx * pi2, "Length in streamwise direction : Lx"));
  IO(wd("Ly", c.lmfy * 2.0, "Length in wall normal direction : Ly"));
  IO(wd("Lz", c.lmfz * pi2, "Length in spanwise direction : Lz"));
  IO(wd("Stretch", c.stretch, "Stretch Factor for non-uniform grid"));
  IO(wd("dt", dt, "Time advance interval"));
  IO(wi("nx", c.nx, "Number of x modes"));
  IO(wi("ny", c.ny, "Number of y points"));
  IO(wi("nz", c.nz, "Number of z modes"));
  IO(wi("LABS_K", c.labs_k, "B-Spline Order"));
  IO(wi("LABS_BW", h.bw, "Bandwidth of Matrix"));
  // the mean profiles: the real parts of the (0, 0) mode of u, w and theta
  std::vector<double> prof(ny);
  auto mean_line = [&](int field, const char *n, const char *cm) {
    for (int i = 0; i < ny; ++i) prof[i] = U[(size_t)(field * ns + i)].x;
    return kmm_io_line_write_double(io, n, ny, prof.data(), cm);
  };
  IO(mean_line(0, "U_mean", "U average"));
  IO(mean_line(2, "W_mean", "W average"));
  IO(mean_line(6, "T_mean", "T average"));
  if (h.nsc == 2) IO(mean_line(10, "T2_mean", "T2 average (second passive scalar)"));
  IO(kmm_io_line_write_double(io, "LABS_COL", ny, h.ops.y.data(), "Collocation points in y"));
  IO(kmm_io_line_write_double(
      io, "LABS_CENTER_LINE", ny, h.ops.center.data(),
      "Center Line Coeff: LABS_CENTER_LINE / e.g. U_c = LABS_CENTER_LINE * TRANSPOSE(D-^-1 * u)"));
  IO(kmm_io_line_write_double(
      io, "LABS_INTEGRATE", ny, h.ops.integ.data(),
      "Integration Coefficient: LABS_INT / e.g. Int u dy = LABS_INT * TRANSPOSE(D0^-1 * u) = LABS_INT * TRANSPOSE(cu)"));
  auto field = [&](const double2 *src, const char *n) {
    return kmm_io_field_writev_double(io, n, ny, nxh, nz, 2, reinterpret_cast<const double *>(src));
  };
  if (fields & KMM_STORE_U) IO(field(U.data(), "u"));
  if (fields & KMM_STORE_V) IO(field(U.data() + ns, "v"));
  if (fields & KMM_STORE_W) IO(field(U.data() + 2 * ns, "w"));
  if (fields & KMM_STORE_G) IO(field(RK.data(), "g"));
  if (fields & KMM_STORE_PHI) IO(field(RK.data() + ns, "phi"));
  if (fields & KMM_STORE_THETA) {
    IO(field(U.data() + 6 * ns, "theta"));
    if (h.nsc == 2) IO(field(U.data() + 10 * ns, "theta2"));
  }
  IO(kmm_io_line_write_double(io, "LABS_KNOT", (int64_t)h.ops.brk.size(), h.ops.brk.data(), "KNOT points in y"));
  const char *full_cm[3] = {"Zeroth order operator(FULL): D0 / e.g. u = D0*cu ",
                            "First order operator(FULL): D1 / e.g. dudy = D1*cu = D1*(D0^-1)*u",
                            "Second order operator(FULL): D2 / e.g. d2udy2 = D2*cu = D2*(D0^-1)*u"};
  const char *band_cm[3] = {"Zeroth order operator(BAND): D0 / e.g. u = D0*cu ",
                            "First order operator(BAND): D1 / e.g. dudy = D1*cu = D1*(D0^-1)*u",
                            "Second order operator(BAND): D2 / e.g. d2udy2 = D2*cu = D2*(D0^-1)*u"};
  const char *full_n[3] = {"LABS_D0_FULL", "LABS_D1_FULL", "LABS_D2_FULL"};
  const char *band_n[3] = {"LABS_D0_BAND", "LABS_D1_BAND", "LABS_D2_BAND"};
  for (int d = 0; d < 3; ++d) IO(kmm_io_plane_write_double(io, full_n[d], ny, ny, h.ops.full[d].data(), full_cm[d]));
  for (int d = 0; d < 3; ++d)
    IO(kmm_io_plane_write_double(io, band_n[d], 2 * h.bw + 1, ny, h.ops.band[d].data(), band_cm[d]));
  kmm_io *done = f.io;
  f.io = nullptr;
  return kmm_io_close(done);
}

int kmm_restart(kmm_handle *hh, const char *path, int32_t restart_option, kmm_restart_info *out) {
  if (!hh || !path || restart_option < 1 || restart_option > 3) return KMM_ERR_ARG;
  Handle &h = *reinterpret_cast<Handle *>(hh);
  if (h.nsc == 2 && restart_option != 1) {
    set_error("kmm_restart: options 2 and 3 rebuild the reference's one scalar; a second scalar restarts with option 1");
    return KMM_ERR_CONFIG;
  }
  const int ny = h.ny, nxh = h.nxh, nz = h.nz, nf = h.nsc == 2 ? 11 : 7;
  const int64_t ns = (int64_t)ny * nxh * nz;
  Io f;
  IO(kmm_io_open(path, 0, &f.io));
  kmm_io *io = f.io;
  kmm_restart_info info{};
  IO(kmm_io_line_read_integer(io, "timestep", 1, 0, 1, &info.timestep));
  IO(kmm_io_line_read_double(io, "time", 1, 0, 1, &info.time));
  IO(kmm_io_line_read_double(io, "dt", 1, 0, 1, &info.dt));
  std::vector<double2> U((size_t)(ns * nf)), RK((size_t)(ns * 3));
  auto field = [&](const char *n, double2 *dst) {
    return kmm_io_field_readv_double(io, n, ny, nxh, nz, 2, 0, nxh, 0, nz, reinterpret_cast<double *>(dst));
  };
  auto means_into_stores = [&]() -> int {
    // data_read_gphi / data_read_vg: the (0, 0) mode of the stores holds U_mean - U_gal, W_mean, T_mean
    std::vector<double> m(ny);
    const char *names[3] = {"U_mean", "W_mean", "T_mean"};
    for (int s = 0; s < 3; ++s) {
      IO(kmm_io_line_read_double(io, names[s], ny, 0, ny, m.data()));
      for (int i = 0; i < ny; ++i) RK[(size_t)(s * ns + i)] = z2(s == 0 ? m[i] - h.cfg.u_gal : m[i], 0.0);
    }
    return KMM_OK;
  };
  if (restart_option == 1) {
    IO(field("u", U.data()));
    IO(field("v", U.data() + ns));
    IO(field("w", U.data() + 2 * ns));
    IO(field("theta", U.data() + 6 * ns));
    if (h.nsc == 2) IO(field("theta2", U.data() + 10 * ns));
    for (int i = 0; i < ny; ++i) U[i].x -= h.cfg.u_gal;  // data_read_uvw
  } else if (restart_option == 2) {
    IO(field("g", RK.data()));
    IO(field("phi", RK.data() + ns));
    IO(field("theta", RK.data() + 2 * ns));
    IO(means_into_stores());
  } else {
    IO(field("v", U.data() + ns));
    IO(field("g", RK.data()));
    IO(field("theta", RK.data() + 2 * ns));
    IO(means_into_stores());
  }
  kmm_io *done = f.io;
  f.io = nullptr;
  IO(kmm_io_close(done));
  if (restart_option == 1) {
    IO(kmm_set_initial_data_uvw(hh, reinterpret_cast<double *>(U.data()), nf, info.dt));
  } else {
    if (restart_option == 2)
      by_bw(h.bw, [&]<int BW>() { rebuild_gphi<BW>(h, U.data(), RK.data()); });
    else
      by_bw(h.bw, [&]<int BW>() { rebuild_vg<BW>(h, U.data(), RK.data()); });
    IO(kmm_upload_state(hh, reinterpret_cast<double *>(U.data()), nf, reinterpret_cast<double *>(RK.data()),
                        info.dt));
  }
  if (out) *out = info;
  return KMM_OK;
}

}  // extern "C"
