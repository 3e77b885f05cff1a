// noalloc.cu - an allocation-free batched Helmholtz solve.
//
// Some callers of this library cannot allocate device memory:
//  * code that runs while a CUDA stream is being captured into a graph, where cudaMalloc is
//    not a stream operation and must not be called;
//  * host programs whose device memory is reserved up front by another allocator or by a fixed
//    memory plan, so that a library call has no right to take more;
//  * time-critical loops that cannot afford the device-wide synchronisation of cudaMalloc and
//    cudaFree.
// The handle-based entry points of this library allocate their scratch in kmm_create.  This
// entry point needs no handle: the caller passes the operators, the coefficients and the
// right-hand sides, and the per-mode scratch band lives in g_noalloc_band, a file-scope
// __device__ array that every GPU loading the library holds until the process exits.
//
// For every mode m it builds A_m = a_m D0 - b_m D2 with Dirichlet first and last rows (the
// left-hand side that solve_g and solve_t build), factors it with the packed-band LU and solves
// A_m x = rhs_m in place (the kernels of labs.cuh).
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "kmm_internal.h"
#include "labs.cuh"

namespace kmm {
namespace {

// The scratch: one (2bw+1) x ny band per mode, mode fastest.  Every entry a call reads is
// written earlier in the same call, so nothing needs clearing; the array keeps the last call's
// contents, and calls that overlap on the GPU race on it.
__device__ __align__(256) double g_noalloc_band[KMM_NOALLOC_MAX_DOUBLES];

// The array's device address per device ordinal, looked up once.  A cudaDeviceReset unloads the
// module and invalidates these addresses; a process that resets a device must not call this
// entry point on that device again.
constexpr int kMaxDevices = 64;
std::mutex g_mutex;
double *g_band_ptr[kMaxDevices] = {};

template <int BW>
__global__ void k_helmholtz_noalloc(int ny, int nm, const double *d0, const double *d2,
                                    const double *acoef, const double *bcoef, double2 *rhs,
                                    double *band) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= nm) return;
  constexpr int ld = 2 * BW + 1;
  BandS<BW> D0{d0}, D2{d2};
  BandM<BW> A{band + m, nm};
  const double a = acoef[m], b = bcoef[m];
  for (int i = 1; i <= ld; ++i) A.set(i, 1, 0.0);
  A.set(BW + 1, 1, a * D0.g(BW + 1, 1) - b * D2.g(BW + 1, 1));
  for (int j = 2; j <= ny - 1; ++j)
    for (int i = 1; i <= ld; ++i) A.set(i, j, a * D0.g(i, j) - b * D2.g(i, j));
  for (int i = 1; i <= ld; ++i) A.set(i, ny, 0.0);
  A.set(BW + 1, ny, a * D0.g(BW + 1, ny) - b * D2.g(BW + 1, ny));
  labs_lu<BW>(A, ny);
  labs_bs<BW>(A, DLine{rhs + m, nm}, ny);
}

template <int BW>
cudaError_t launch(int ny, int nm, const double *d0, const double *d2, const double *a,
                   const double *b, double2 *rhs, double *band, cudaStream_t st) {
  k_helmholtz_noalloc<BW><<<(nm + 127) / 128, 128, 0, st>>>(ny, nm, d0, d2, a, b, rhs, band);
  return cudaGetLastError();
}

}  // namespace
}  // namespace kmm

using namespace kmm;

extern "C" int kmm_helmholtz_solve_noalloc(int ny, int bw, int nmodes, const double *d0_band,
                                           const double *d2_band, const double *a,
                                           const double *b, double *rhs, void *stream) {
  if (!d0_band || !d2_band || !a || !b || !rhs) {
    set_error("kmm_helmholtz_solve_noalloc: null pointer");
    return KMM_ERR_ARG;
  }
  if (bw < kMinBw || bw > kMaxBw || ny < 4 * bw + 2 || nmodes <= 0) {
    set_error("kmm_helmholtz_solve_noalloc: need 2 <= bw <= 7, ny >= 4*bw+2 and nmodes > 0");
    return KMM_ERR_ARG;
  }
  if ((reinterpret_cast<uintptr_t>(rhs) & 15u) != 0) {
    set_error("kmm_helmholtz_solve_noalloc: rhs must be 16-byte aligned (it is read as complex doubles)");
    return KMM_ERR_ARG;
  }
  const long long need = (long long)(2 * bw + 1) * ny * nmodes;
  if (need > (long long)KMM_NOALLOC_MAX_DOUBLES) {
    set_error("kmm_helmholtz_solve_noalloc: (2*bw+1)*ny*nmodes = " + std::to_string(need) +
              " doubles exceeds the fixed scratch of KMM_NOALLOC_MAX_DOUBLES = " +
              std::to_string((long long)KMM_NOALLOC_MAX_DOUBLES));
    return KMM_ERR_ARG;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    set_error("kmm_helmholtz_solve_noalloc: no current CUDA device");
    return KMM_ERR_CUDA;
  }
  double *band = nullptr;
  {
    // once per device, with that device current: the device address of the scratch array
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_band_ptr[dev]) {
      double *p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void **>(&p), g_noalloc_band);
      if (e != cudaSuccess || !p) {
        set_error(std::string("kmm_helmholtz_solve_noalloc: cudaGetSymbolAddress failed: ") +
                  cudaGetErrorString(e));
        return KMM_ERR_CUDA;
      }
      g_band_ptr[dev] = p;
    }
    band = g_band_ptr[dev];
  }
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  double2 *r = reinterpret_cast<double2 *>(rhs);
  cudaError_t e;
  switch (bw) {
    case 2: e = launch<2>(ny, nmodes, d0_band, d2_band, a, b, r, band, st); break;
    case 3: e = launch<3>(ny, nmodes, d0_band, d2_band, a, b, r, band, st); break;
    case 4: e = launch<4>(ny, nmodes, d0_band, d2_band, a, b, r, band, st); break;
    case 5: e = launch<5>(ny, nmodes, d0_band, d2_band, a, b, r, band, st); break;
    case 6: e = launch<6>(ny, nmodes, d0_band, d2_band, a, b, r, band, st); break;
    default: e = launch<7>(ny, nmodes, d0_band, d2_band, a, b, r, band, st); break;
  }
  if (e != cudaSuccess) {
    set_error(std::string("kmm_helmholtz_solve_noalloc: launch failed: ") + cudaGetErrorString(e));
    return KMM_ERR_CUDA;
  }
  return KMM_OK;
}
