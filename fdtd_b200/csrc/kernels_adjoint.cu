// Discrete adjoint of the FP32 fused 2D TM step, for d(objective)/d(eps_r).
//
// Forward step t (kernels_fused.cu, TM, non-dispersive, design cells outside
// the CPML):
//   E:  Ez' = Ez + ie (Fx r_zx + Fy r_zy + Gx psi_zx + Gy psi_zy)
//       psi_zx' = Bx psi_zx + Cx r_zx,  r_zx = Hy - Hy[i-1]
//       psi_zy' = By psi_zy + Cy r_zy,  r_zy = -(Hx - Hx[j-1])
//   H:  Hx' = Hx - (Fy r_xy + Gy psi_xy),  psi_xy' = By psi_xy + Cy r_xy,  r_xy = Ez'[j+1] - Ez'
//       Hy' = Hy - (Fx r_yx + Gx psi_yx),  psi_yx' = Bx psi_yx + Cx r_yx,  r_yx = -(Ez'[i+1] - Ez')
// (E coefficients for the E half, H coefficients for the H half; sources are
// affine in the state and drop out). Reversing step t, given the adjoints
// (a*) of the state after it, is four per-cell gathers:
//   A1  H cell: rb_xy = -Fy aHx + Cy apsi_xy,  apsi_xy <- By apsi_xy - Gy aHx   (Hy likewise)
//   A2  E cell: aEz += rb_xy[j-1] - rb_xy - rb_yx[i-1] + rb_yx  (+ objective)
//   A3  E cell: db = ie aEz;  rb_zx = Fx db + Cx apsi_zx,  apsi_zx <- Bx apsi_zx + Gx db  (zy likewise);
//               grad += -aEz ie^2 d_t,  d_t = Fx r_zx + Fy r_zy of the forward step
//   A4  H cell: aHy += rb_zx - rb_zx[i+1];  aHx += -rb_zy + rb_zy[j+1]
// A1 and A4 read only the cell's own adjoints besides the rb arrays of the
// other half, so the reverse of step t runs as two launches: the H kernel
// (A4 of step t+1, then A1 of step t) and the E kernel (A2, A3 of step t).
// The objective J = sum_p |X_p|^2, X_p the DFT of Ez at the probe cells
// (sample n = t+1 after the E half of step t), adds
// dJ/dEz_p(n) = 2 Re(X_p e^{2 pi i f n}) to aEz at the probes.
// The gradient accumulates in FP64.
#include "internal.h"

namespace fdtdb {

namespace {

__device__ __forceinline__ bool interior(const AdjArgs& a, int i, int j) {
  return i >= 1 && i <= a.nx - 2 && j >= 1 && j <= a.ny - 2;
}

// 1/eps per cell as the E sweep takes it (material row, or the eps map)
__global__ void adj_inv_eps_kernel(const __grid_constant__ FusedArgs a, float* ie) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= a.nx || j >= a.ny) return;
  const long long c = static_cast<long long>(j) * a.pitch + i;
  int mid = 0;
  if (a.ids) mid = a.ids[c];
  else if (a.bids) mid = a.bids[(j >> a.bshift) * a.nbx + (i >> a.bshift)];
  const MatF32& m = a.mats[mid];
  float v = m.inv_eps;
  if (a.inv_eps_map && m.npoles == 0) {
    const float u = a.inv_eps_map[c];
    if (u > 0.f) v = u;
  }
  ie[c] = v;
}

// d_t of every design cell from the state at the start of step t
__global__ void adj_capture_kernel(const AdjArgs a, const float* __restrict__ hx, const float* __restrict__ hy,
                                   float* __restrict__ slot) {
  const int dw = a.dhi[0] - a.dlo[0] + 1;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= a.ndesign) return;
  const int i = a.dlo[0] + q % dw, j = a.dlo[1] + q / dw;
  const long long c = static_cast<long long>(j) * a.pitch + i;
  const float r_zx = hy[c] - hy[c - 1];
  const float r_zy = -(hx[c] - hx[c - a.pitch]);
  slot[q] = a.prof[0][0].F[i] * r_zx + a.prof[0][1].F[j] * r_zy;
}

__global__ void __launch_bounds__(256) adj_h_kernel(const AdjArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (!interior(a, i, j)) return;
  const long long c = static_cast<long long>(j) * a.pitch + i;
  // A4 of step t+1 (the rb_z arrays are zero before the first reversed step)
  const float ahx = a.ahx[c] + (-a.rzy[c] + a.rzy[c + a.pitch]);
  const float ahy = a.ahy[c] + (a.rzx[c] - a.rzx[c + 1]);
  a.ahx[c] = ahx;
  a.ahy[c] = ahy;
  // A1 of step t: Hx (curl along y), Hy (curl along x)
  float rxy = -a.prof[1][1].F[j] * ahx;
  const int sy = a.pml_axis[1] ? slab_index(a.slab[1], j) : -1;
  if (sy >= 0) {
    const long long p = static_cast<long long>(sy) * a.pitch + i;
    const float ps = a.apxy[p];
    rxy += a.prof[1][1].C[j] * ps;
    a.apxy[p] = a.prof[1][1].B[j] * ps - a.prof[1][1].G[j] * ahx;
  }
  float ryx = -a.prof[1][0].F[i] * ahy;
  const int sx = a.pml_axis[0] ? slab_index(a.slab[0], i) : -1;
  if (sx >= 0) {
    const long long p = static_cast<long long>(j) * a.slab[0].W + sx;
    const float ps = a.apyx[p];
    ryx += a.prof[1][0].C[i] * ps;
    a.apyx[p] = a.prof[1][0].B[i] * ps - a.prof[1][0].G[i] * ahy;
  }
  a.rxy[c] = rxy;
  a.ryx[c] = ryx;
}

// `back` counts the steps between this one and the last of the recomputed
// segment, whose end the step counter holds: n = t + 1 = ctrl->t - back
__global__ void __launch_bounds__(256) adj_e_kernel(const AdjArgs a, int back, const float* __restrict__ dslot) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (!interior(a, i, j)) return;
  const long long c = static_cast<long long>(j) * a.pitch + i;
  const long long n = a.ctrl->t - back;
  // A2
  float v = a.rxy[c - a.pitch] - a.rxy[c] - a.ryx[c - 1] + a.ryx[c];
  if (i >= a.plo[0] && i <= a.phi[0] && j >= a.plo[1] && j <= a.phi[1]) {
    const long long q = static_cast<long long>(j - a.plo[1]) * (a.phi[0] - a.plo[0] + 1) + (i - a.plo[0]);
    double sn, cs;
    sincospi(2.0 * a.freq * static_cast<double>(n), &sn, &cs);
    v += static_cast<float>(2.0 * (a.X[2 * q] * cs - a.X[2 * q + 1] * sn));
  }
  const float ae = a.aez[c] + v;
  a.aez[c] = ae;
  // A3
  const float ie = a.ie[c];
  const float db = ie * ae;
  if (i >= a.dlo[0] && i <= a.dhi[0] && j >= a.dlo[1] && j <= a.dhi[1]) {
    const int q = (j - a.dlo[1]) * (a.dhi[0] - a.dlo[0] + 1) + (i - a.dlo[0]);
    const double die = ie;
    a.grad[q] += -static_cast<double>(ae) * die * die * static_cast<double>(dslot[q]);
  }
  float rx = a.prof[0][0].F[i] * db, ry = a.prof[0][1].F[j] * db;
  const int sx = a.pml_axis[0] ? slab_index(a.slab[0], i) : -1;
  if (sx >= 0) {
    const long long p = static_cast<long long>(j) * a.slab[0].W + sx;
    const float ps = a.apzx[p];
    rx += a.prof[0][0].C[i] * ps;
    a.apzx[p] = a.prof[0][0].B[i] * ps + a.prof[0][0].G[i] * db;
  }
  const int sy = a.pml_axis[1] ? slab_index(a.slab[1], j) : -1;
  if (sy >= 0) {
    const long long p = static_cast<long long>(sy) * a.pitch + i;
    const float ps = a.apzy[p];
    ry += a.prof[0][1].C[j] * ps;
    a.apzy[p] = a.prof[0][1].B[j] * ps + a.prof[0][1].G[j] * db;
  }
  a.rzx[c] = rx;
  a.rzy[c] = ry;
}

}  // namespace

int launch_adjoint_inv_eps(const FusedArgs& fa, float* ie, cudaStream_t s) {
  dim3 block(32, 8), grid((fa.nx + 31) / 32, (fa.ny + 7) / 8);
  adj_inv_eps_kernel<<<grid, block, 0, s>>>(fa, ie);
  return 1;
}

int launch_adjoint_capture(const AdjArgs& a, const float* hx, const float* hy, float* slot, cudaStream_t s) {
  adj_capture_kernel<<<(a.ndesign + 255) / 256, 256, 0, s>>>(a, hx, hy, slot);
  return 1;
}

// the reverse of the step `back` steps before the one that ends at the
// device step counter
int launch_adjoint_step(const AdjArgs& a, int back, const float* dslot, cudaStream_t s) {
  dim3 block(32, 8), grid((a.nx + 31) / 32, (a.ny + 7) / 8);
  adj_h_kernel<<<grid, block, 0, s>>>(a);
  adj_e_kernel<<<grid, block, 0, s>>>(a, back, dslot);
  return 2;
}

}  // namespace fdtdb
