// Kernels shared by both methods: the running DFT capture, the non-finite
// check and the device step counter.
//
// Running DFT (the reference's DataCapture is an empty stub,
// include/DataCapture.hpp:61-191; this capture is defined here):
//   X_f += x[n] * exp(-2 pi i f n), n = t+1 for E, t+1.5 for H,
// accumulated in FP64 whatever the field precision.
#include "internal.h"

namespace fdtdb {

template <typename R>
__global__ void __launch_bounds__(256) dft_kernel(int phase, const DftRegionDev* __restrict__ regions, int nreg,
                                                  long long total, const R* const* __restrict__ fields, int nx, int ny,
                                                  int pitch, const Control* __restrict__ ctrl) {
  const long long p = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (p >= total) return;
  int r = 0;
  while (r + 1 < nreg && regions[r + 1].pt_off <= p) r++;
  const DftRegionDev& g = regions[r];
  const long long q = p - g.pt_off;
  const int i = g.lo[0] + static_cast<int>(q % g.ext[0]);
  const int j = g.lo[1] + static_cast<int>((q / g.ext[0]) % g.ext[1]);
  const int k = g.lo[2] + static_cast<int>(q / (static_cast<long long>(g.ext[0]) * g.ext[1]));
  const R* f = fields[g.comp];
  const double x = static_cast<double>(f[(static_cast<long long>(k) * ny + j) * pitch + i]);
  const double n = static_cast<double>(ctrl->t) + (phase == 0 ? 1.0 : 1.5);
  for (int fi = 0; fi < g.nf; fi++) {
    double s, c;
    sincospi(2.0 * g.freqs[fi] * n, &s, &c);
    double* acc = g.acc + (static_cast<long long>(fi) * g.npts + q) * 2;
    acc[0] += x * c;
    acc[1] -= x * s;
  }
  (void)nx;
}

int launch_dft(int phase, int precision, const DftRegionDev* regions, int nreg, long long total_pts,
               const void* const* fields, int nx, int ny, int pitch, const Control* ctrl, cudaStream_t s) {
  if (nreg == 0 || total_pts == 0) return 0;
  const unsigned blocks = static_cast<unsigned>((total_pts + 255) / 256);
  if (precision == 0)
    dft_kernel<double><<<blocks, 256, 0, s>>>(phase, regions, nreg, total_pts,
                                              reinterpret_cast<const double* const*>(fields), nx, ny, pitch, ctrl);
  else
    dft_kernel<float><<<blocks, 256, 0, s>>>(phase, regions, nreg, total_pts,
                                             reinterpret_cast<const float* const*>(fields), nx, ny, pitch, ctrl);
  return 1;
}

template <typename R>
__global__ void finite_kernel(const R* __restrict__ p, long long n, int* flag) {
  for (long long x = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; x < n;
       x += static_cast<long long>(gridDim.x) * blockDim.x) {
    if (!isfinite(p[x])) {
      *flag = 1;
      return;
    }
  }
}

int launch_finite_check(const void* p, long long n, int is_f32, int* flag, cudaStream_t s) {
  if (n == 0) return 0;
  if (is_f32) finite_kernel<float><<<148 * 4, 256, 0, s>>>(static_cast<const float*>(p), n, flag);
  else finite_kernel<double><<<148 * 4, 256, 0, s>>>(static_cast<const double*>(p), n, flag);
  return 1;
}

__global__ void step_advance_kernel(Control* ctrl) { ctrl->t += 1; }

int launch_step_advance(Control* ctrl, cudaStream_t s) {
  step_advance_kernel<<<1, 1, 0, s>>>(ctrl);
  return 1;
}

}  // namespace fdtdb
