// Kernels shared by both methods: the running DFT capture, the non-finite
// check and the device step counter.
//
// Running DFT (the reference's DataCapture is an empty stub,
// include/DataCapture.hpp:61-191; this capture is defined here):
//   X_f += x[n] * exp(-2 pi i f n), n = t+1 for E, t+1.5 for H,
// accumulated in FP64 whatever the field precision.
#include <algorithm>

#include "internal.h"

namespace fdtdb {

// The capture is chunked: every half step a gather copies the region values
// into slot `slot` (the samples taken since the last flush, counted on the
// host) of a ring of kDftChunk samples per point; a flush
// folds the pending samples into the FP64 accumulators in one pass, with the
// twiddles of the chunk computed once per block in shared memory. This reads
// and writes each 16-byte accumulator once per chunk instead of once per step.
// One grid row (blockIdx.y) per region: the region is uniform over the
// block, and point indices within a region fit 32 bits.
// One quantity of cell c. f holds the phase's three field arrays (E for
// kinds 0, 2, 3 of the E phase; H for kinds 0, 1 of the H phase). The
// surface current Je (UpdateSurfaceCurrentE, SurfaceQuantities.hpp:256-296)
// reads H at the cell and its lower neighbours, Jh (UpdateSurfaceCurrentH,
// :315-356) E at the cell and its upper neighbours, rho
// (UpdateSurfaceChargeDensity, :203-242) E at the cell and its lower
// neighbours; each sum is formed in the reference's order and multiplied by
// scale (1/dx, -1/dx, eps0/dx; with 1/eta folded in for the stored eta*H of
// the FP32 method). The host keeps the boxes of derived kinds in the interior.
template <typename R>
__device__ __forceinline__ R quantity_sample(const DftRegionDev& g, const R* const* f, long long c, long long sy,
                                             long long sz) {
  const R s = static_cast<R>(g.scale);
  switch (g.kind) {
    case 0:
      return f[g.comp][c];
    case 1:
      if (g.mode == kTE) {
        if (g.comp == 0) return s * (f[2][c] - f[2][c - sy]);
        return s * (-f[2][c] + f[2][c - 1]);
      }
      if (g.comp == 0) return s * (f[2][c] - f[2][c - sy] - f[1][c] + f[1][c - sz]);
      if (g.comp == 1) return s * (f[0][c] - f[0][c - sz] - f[2][c] + f[2][c - 1]);
      return s * (f[1][c] - f[1][c - 1] - f[0][c] + f[0][c - sy]);
    case 2:
      if (g.mode == kTM) {
        if (g.comp == 0) return s * (f[2][c + sy] - f[2][c]);
        return s * (-f[2][c + 1] + f[2][c]);
      }
      if (g.comp == 0) return s * (f[2][c + sy] - f[2][c] - f[1][c + sz] + f[1][c]);
      if (g.comp == 1) return s * (f[0][c + sz] - f[0][c] - f[2][c + 1] + f[2][c]);
      return s * (f[1][c + 1] - f[1][c] - f[0][c + sy] + f[0][c]);
    default:
      if (g.mode == kTE) return s * (f[0][c] + f[1][c] - f[0][c - 1] - f[1][c - sy]);
      return s * (f[0][c] + f[1][c] + f[2][c] - f[0][c - 1] - f[1][c - sy] - f[2][c - sz]);
  }
}

template <typename R>
__device__ __forceinline__ R quantity_at_point(const DftRegionDev& g, const R* const* f, int ny, int pitch, int q) {
  const int ex = g.ext[0], ey = g.ext[1];
  const int r = q / ex;
  const int i = g.lo[0] + (q - r * ex);
  const int j = g.lo[1] + r % ey;
  const int k = g.lo[2] + r / ey;
  const long long sz = static_cast<long long>(ny) * pitch;
  return quantity_sample(g, f, k * sz + static_cast<long long>(j) * pitch + i, pitch, sz);
}

// points per thread of the gather: all their loads are issued before any
// store, so that more of the (often one-per-sector) field reads are in flight
constexpr int kGatherPts = 4;

template <typename R>
__global__ void __launch_bounds__(256) dft_gather_kernel(const DftRegionDev* __restrict__ regions, long long total,
                                                         const R* const* __restrict__ fields, int ny, int pitch,
                                                         long long slot, R* buf) {
  const DftRegionDev& g = regions[blockIdx.y];
  const int q0 = blockIdx.x * (256 * kGatherPts) + threadIdx.x;
  if (q0 >= g.npts) return;
  R v[kGatherPts];
#pragma unroll
  for (int u = 0; u < kGatherPts; u++) {
    const int q = q0 + u * 256;
    if (q < g.npts) v[u] = quantity_at_point(g, fields, ny, pitch, q);
  }
  R* out = buf + slot * total + g.pt_off;
#pragma unroll
  for (int u = 0; u < kGatherPts; u++) {
    const int q = q0 + u * 256;
    if (q < g.npts) out[q] = v[u];
  }
}

template <typename R>
__global__ void __launch_bounds__(256) quantity_read_kernel(const DftRegionDev g, const R* const* __restrict__ fields,
                                                            int ny, int pitch, R* out) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= g.npts) return;
  out[q] = quantity_at_point(g, fields, ny, pitch, q);
}

int launch_quantity_read(int precision, const DftRegionDev& r, const void* const* fields, int ny, int pitch,
                         void* out, cudaStream_t s) {
  if (r.npts == 0) return 0;
  const unsigned grid = static_cast<unsigned>((r.npts + 255) / 256);
  if (precision == 0)
    quantity_read_kernel<double><<<grid, 256, 0, s>>>(r, reinterpret_cast<const double* const*>(fields), ny, pitch,
                                                      static_cast<double*>(out));
  else
    quantity_read_kernel<float><<<grid, 256, 0, s>>>(r, reinterpret_cast<const float* const*>(fields), ny, pitch,
                                                     static_cast<float*>(out));
  return 1;
}

template <typename R>
__global__ void __launch_bounds__(256) dft_flush_kernel(int phase, const DftRegionDev* __restrict__ regions,
                                                        long long total, const R* __restrict__ buf,
                                                        const Control* __restrict__ ctrl, int nsamp) {
  __shared__ double2 tw[kDftChunk * 8];
  const DftRegionDev& g = regions[blockIdx.y];
  const long long q = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (static_cast<long long>(blockIdx.x) * blockDim.x >= g.npts) return;  // block-uniform
  if (nsamp <= 0) return;
  const double nbase = static_cast<double>(ctrl->dft_base) + (phase == 0 ? 1.0 : 1.5);
  for (int f0 = 0; f0 < g.nf; f0 += 8) {
    const int nfb = min(8, g.nf - f0);
    __syncthreads();
    for (int e = threadIdx.x; e < nsamp * nfb; e += blockDim.x) {
      const int m = e / nfb, f = e % nfb;
      double sn, cs;
      sincospi(2.0 * g.freqs[f0 + f] * (nbase + m), &sn, &cs);
      tw[m * 8 + f] = make_double2(cs, -sn);
    }
    __syncthreads();
    if (q >= g.npts) continue;
    double re[8] = {0, 0, 0, 0, 0, 0, 0, 0}, im[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int m = 0; m < nsamp; m++) {
      const double x = static_cast<double>(buf[static_cast<long long>(m) * total + g.pt_off + q]) * g.acc_scale;
#pragma unroll
      for (int f = 0; f < 8; f++) {
        if (f < nfb) {
          const double2 w = tw[m * 8 + f];
          re[f] += x * w.x;
          im[f] += x * w.y;
        }
      }
    }
#pragma unroll
    for (int f = 0; f < 8; f++) {
      if (f < nfb) {
        double* acc = g.acc + (static_cast<long long>(f0 + f) * g.npts + q) * 2;
        acc[0] += re[f];
        acc[1] += im[f];
      }
    }
  }
}

// after a flush of nsamp samples the next sample is nsamp steps later
__global__ void dft_rebase_kernel(Control* ctrl, int nsamp) { ctrl->dft_base += nsamp; }

__global__ void dft_set_base_kernel(Control* ctrl, long long base) { ctrl->dft_base = base; }

int launch_dft_gather(int precision, const DftRegionDev* regions, int nreg, long long total_pts, long long max_pts,
                      const void* const* fields, int ny, int pitch, int slot, void* buf, cudaStream_t s) {
  if (nreg == 0 || total_pts == 0) return 0;
  const dim3 grid(static_cast<unsigned>((max_pts + 256 * kGatherPts - 1) / (256 * kGatherPts)), nreg);
  if (precision == 0)
    dft_gather_kernel<double><<<grid, 256, 0, s>>>(regions, total_pts, reinterpret_cast<const double* const*>(fields),
                                                   ny, pitch, slot, static_cast<double*>(buf));
  else
    dft_gather_kernel<float><<<grid, 256, 0, s>>>(regions, total_pts, reinterpret_cast<const float* const*>(fields),
                                                  ny, pitch, slot, static_cast<float*>(buf));
  return 1;
}

int launch_dft_flush(int phase, int precision, const DftRegionDev* regions, int nreg, long long max_pts,
                     long long total_pts, const void* buf, const Control* ctrl, int nsamp, cudaStream_t s) {
  if (nreg == 0 || total_pts == 0 || nsamp <= 0) return 0;
  dim3 grid(static_cast<unsigned>((max_pts + 255) / 256), nreg);
  if (precision == 0)
    dft_flush_kernel<double><<<grid, 256, 0, s>>>(phase, regions, total_pts, static_cast<const double*>(buf), ctrl, nsamp);
  else
    dft_flush_kernel<float><<<grid, 256, 0, s>>>(phase, regions, total_pts, static_cast<const float*>(buf), ctrl, nsamp);
  return 1;
}

int launch_dft_rebase(Control* ctrl, int nsamp, cudaStream_t s) {
  dft_rebase_kernel<<<1, 1, 0, s>>>(ctrl, nsamp);
  return 1;
}

int launch_dft_set_base(Control* ctrl, long long base, cudaStream_t s) {
  dft_set_base_kernel<<<1, 1, 0, s>>>(ctrl, base);
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

// Squared difference of two stored fields of equal extent, each scaled to SI
// units, and the squared reference: out[0] += sum (a sa - b sb)^2,
// out[1] += sum (b sb)^2 over the nx cells of every row (j, k); the rows of a
// and b are rla and rlb values long (FP32 rows are padded). FP64 sums.
template <typename RA, typename RB>
__global__ void __launch_bounds__(256) field_diff_kernel(const RA* __restrict__ a, long long rla, double sa,
                                                         const RB* __restrict__ b, long long rlb, double sb, int nx,
                                                         long long nrows, double* out) {
  double d2 = 0.0, r2 = 0.0;
  for (long long row = blockIdx.x; row < nrows; row += gridDim.x) {
    const RA* pa = a + row * rla;
    const RB* pb = b + row * rlb;
    for (int i = threadIdx.x; i < nx; i += blockDim.x) {
      const double va = static_cast<double>(pa[i]) * sa, vb = static_cast<double>(pb[i]) * sb;
      d2 += (va - vb) * (va - vb);
      r2 += vb * vb;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    d2 += __shfl_down_sync(0xffffffffu, d2, o);
    r2 += __shfl_down_sync(0xffffffffu, r2, o);
  }
  __shared__ double part[2][8];
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    part[0][w] = d2;
    part[1][w] = r2;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = 1; q < (blockDim.x >> 5); q++) {
      d2 += part[0][q];
      r2 += part[1][q];
    }
    atomicAdd(out, d2);
    atomicAdd(out + 1, r2);
  }
}

int launch_field_diff(const void* a, int a_f32, long long rla, double sa, const void* b, int b_f32, long long rlb,
                      double sb, int nx, long long nrows, double* out, cudaStream_t s) {
  const unsigned blocks = static_cast<unsigned>(std::min<long long>(nrows, 148LL * 8));
  if (blocks == 0) return 0;
  if (a_f32 && b_f32)
    field_diff_kernel<float, float><<<blocks, 256, 0, s>>>(static_cast<const float*>(a), rla, sa,
                                                            static_cast<const float*>(b), rlb, sb, nx, nrows, out);
  else if (a_f32)
    field_diff_kernel<float, double><<<blocks, 256, 0, s>>>(static_cast<const float*>(a), rla, sa,
                                                             static_cast<const double*>(b), rlb, sb, nx, nrows, out);
  else if (b_f32)
    field_diff_kernel<double, float><<<blocks, 256, 0, s>>>(static_cast<const double*>(a), rla, sa,
                                                             static_cast<const float*>(b), rlb, sb, nx, nrows, out);
  else
    field_diff_kernel<double, double><<<blocks, 256, 0, s>>>(static_cast<const double*>(a), rla, sa,
                                                              static_cast<const double*>(b), rlb, sb, nx, nrows, out);
  return 1;
}

__global__ void step_advance_kernel(Control* ctrl, unsigned* epoch) {
  ctrl->t += 1;
  if (epoch) *epoch += 1u;
}

__global__ void chunk_start_kernel(Control* ctrl) { ctrl->t0 = ctrl->t; }
__global__ void set_step_kernel(Control* ctrl, long long t) {
  ctrl->t = t;
  ctrl->t0 = t;
}

// Boundary conditions (include/BoundaryUpdates.hpp:230-760): on each face
// with one, the outer cell takes the image of the interior cell next to the
// face (periodic: of the interior cell at the far end of the axis), every
// component of the half step's field times the sign of the condition.
// Launch: blockIdx.z = face; the 2D thread grid spans the face's two
// transverse axes (u, v) = (y, z) for x faces, (x, z) for y faces and (x, y)
// for z faces, so y and z faces are read and written along x, coalesced.
__host__ __device__ float bc_sign(int kind, int ft, int c, int axis) {
  const bool normal = c == axis;
  switch (kind) {
    case 1: return ft == 0 ? (normal ? 1.f : -1.f) : (normal ? -1.f : 1.f);  // PEC
    case 2: return ft == 0 ? (normal ? -1.f : 1.f) : (normal ? 1.f : -1.f);  // PMC
    case 3: return normal ? -1.f : 1.f;                                      // symmetric
    case 4: return normal ? 1.f : -1.f;                                      // antisymmetric
    default: return 1.f;                                                     // periodic
  }
}

template <typename T>
__global__ void __launch_bounds__(256) boundary_kernel(BcFaces f, int ft, T* f0, T* f1, T* f2, int nx, int ny,
                                                       int nz, int rowlen) {
  const BcFace& b = f.face[blockIdx.z];
  const int ua = b.axis == 0 ? 1 : 0, va = b.axis == 2 ? 1 : 2;  // transverse axes
  const int n[3] = {nx, ny, nz};
  const int three = nz > 1;
  const int u = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int v = (va < 2 || three) ? 1 + static_cast<int>(blockIdx.y * blockDim.y + threadIdx.y)
                                  : static_cast<int>(blockIdx.y * blockDim.y + threadIdx.y);
  if (u > n[ua] - 2) return;
  if (va == 2 && !three ? v != 0 : v > n[va] - 2) return;
  int dst[3], src[3];
  dst[ua] = src[ua] = u;
  dst[va] = src[va] = v;
  const int na = n[b.axis];
  dst[b.axis] = b.side == 0 ? 0 : na - 1;
  src[b.axis] = b.kind == 5 ? (b.side == 0 ? na - 2 : 1) : (b.side == 0 ? 1 : na - 2);
  const long long cs = (static_cast<long long>(src[2]) * ny + src[1]) * rowlen + src[0];
  const long long cd = (static_cast<long long>(dst[2]) * ny + dst[1]) * rowlen + dst[0];
  const T s0 = static_cast<T>(b.sgn[ft][0]), s1 = static_cast<T>(b.sgn[ft][1]), s2 = static_cast<T>(b.sgn[ft][2]);
  const T v0 = f0 ? f0[cs] : T(0), v1 = f1 ? f1[cs] : T(0), v2 = f2 ? f2[cs] : T(0);
  if (f0) f0[cd] = s0 * v0;
  if (f1) f1[cd] = s1 * v1;
  if (f2) f2[cd] = s2 * v2;
}

int launch_boundaries(const BcFaces& f, int ft, int is_f32, void* const* fields, int nx, int ny, int nz, int rowlen,
                      cudaStream_t s) {
  if (f.n == 0) return 0;
  // the largest transverse extents over the faces
  int mu = 1, mv = 1;
  const int n[3] = {nx, ny, nz};
  for (int q = 0; q < f.n; q++) {
    const int ax = f.face[q].axis;
    const int ua = ax == 0 ? 1 : 0, va = ax == 2 ? 1 : 2;
    mu = std::max(mu, n[ua] - 2);
    mv = std::max(mv, va == 2 && nz == 1 ? 1 : n[va] - 2);
  }
  const dim3 block(32, 8, 1);
  const dim3 grid(static_cast<unsigned>((mu + 31) / 32), static_cast<unsigned>((mv + 7) / 8), f.n);
  if (is_f32)
    boundary_kernel<float><<<grid, block, 0, s>>>(f, ft, static_cast<float*>(fields[0]), static_cast<float*>(fields[1]),
                                                  static_cast<float*>(fields[2]), nx, ny, nz, rowlen);
  else
    boundary_kernel<double><<<grid, block, 0, s>>>(f, ft, static_cast<double*>(fields[0]),
                                                   static_cast<double*>(fields[1]), static_cast<double*>(fields[2]),
                                                   nx, ny, nz, rowlen);
  return 1;
}

int launch_chunk_start(Control* ctrl, cudaStream_t s) {
  chunk_start_kernel<<<1, 1, 0, s>>>(ctrl);
  return 1;
}

int launch_set_step(Control* ctrl, long long t, cudaStream_t s) {
  set_step_kernel<<<1, 1, 0, s>>>(ctrl, t);
  return 1;
}

// A soft source on every cell of an inclusive box (a line source is a box one
// cell wide): field += scale * vals[t + shift] on each cell, t the current
// step; shift = -1 with a negative scale takes back the previous step's value
// (the fused method stores E and H with their transient source included).
template <typename T>
__global__ void box_source_kernel(T* f, int lox, int loy, int loz, int ex, int ey, long long n, int pitch, int ny,
                                  const double* vals, int nvals, double scale, int shift, const Control* ctrl) {
  const long long q = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  const long long t = ctrl->t + shift;
  if (q >= n || t < 0 || t >= nvals) return;
  const int i = lox + static_cast<int>(q % ex);
  const long long r = q / ex;
  const int j = loy + static_cast<int>(r % ey);
  const int k = loz + static_cast<int>(r / ey);
  const long long c = (static_cast<long long>(k) * ny + j) * pitch + i;
  f[c] = f[c] + static_cast<T>(scale * vals[t]);
}

int launch_box_source(int is_f32, void* field, const int* lo, const int* hi, int pitch, int ny, const double* vals,
                      int nvals, double scale, int shift, const Control* ctrl, cudaStream_t s) {
  const int ex = hi[0] - lo[0] + 1, ey = hi[1] - lo[1] + 1, ez = hi[2] - lo[2] + 1;
  const long long n = static_cast<long long>(ex) * ey * ez;
  const unsigned blocks = static_cast<unsigned>((n + 255) / 256);
  if (is_f32)
    box_source_kernel<float><<<blocks, 256, 0, s>>>(static_cast<float*>(field), lo[0], lo[1], lo[2], ex, ey, n, pitch,
                                                    ny, vals, nvals, scale, shift, ctrl);
  else
    box_source_kernel<double><<<blocks, 256, 0, s>>>(static_cast<double*>(field), lo[0], lo[1], lo[2], ex, ey, n,
                                                     pitch, ny, vals, nvals, scale, shift, ctrl);
  return 1;
}

__global__ void batch_advance_kernel(Control* const* ctrls, int n, int nsteps) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    ctrls[i]->t += nsteps;
    ctrls[i]->dft_base = ctrls[i]->t;
  }
}

int launch_batch_advance(Control* const* ctrls, int n, int nsteps, cudaStream_t s) {
  batch_advance_kernel<<<(n + 127) / 128, 128, 0, s>>>(ctrls, n, nsteps);
  return 1;
}

int launch_step_advance(Control* ctrl, cudaStream_t s) { return launch_step_advance(ctrl, nullptr, s); }

int launch_step_advance(Control* ctrl, unsigned* epoch, cudaStream_t s) {
  step_advance_kernel<<<1, 1, 0, s>>>(ctrl, epoch);
  return 1;
}

}  // namespace fdtdb
