// TFSF corrections for the FP32 fused method, as one small kernel per half
// step over the cells of the TFSF planes (TFSFPlane::updateD / updateB,
// include/Source.hpp:595-619).
//
// The sweeps leave E (resp. H) updated without the plane corrections; since
// the fused update is linear in the flux increment, adding the correction
// afterwards is exact in exact arithmetic: E += dE with dE = (1/eps_inf) *
// (dt/eps0) * corr, and for a dispersive cell every pole current gains
// b_q * dE (Jt' = a Jt + b E' depends on E' linearly; P' does not depend on E').
// For H: Ht -= (eta dt/mu0) * corr.
//
// A cell on several planes (box edges) is handled by the thread of the first
// plane that contains it, which applies every plane's correction in plane
// order; the result is deterministic.
#include <algorithm>

#include "fused3d_common.cuh"

namespace fdtdb {

namespace {

__device__ __forceinline__ bool in_plane(const PlaneDev& p, int i, int j, int k) {
  return i >= p.lo[0] && i <= p.hi[0] && j >= p.lo[1] && j <= p.hi[1] && k >= p.lo[2] && k <= p.hi[2];
}

// correction of flux I of type ft for cell (i,j,k), generic in the mode
template <int MODE>
__device__ double plane_corr(const FusedArgs& a, const PlaneDev& p, long long row, int ft, int I, int i, int j, int k) {
  constexpr int dim = MODE == kThreeD ? 3 : 2;
  const AuxTab& aux = a.aux[p.aux];
  const int idx[3] = {i, j, k};
  const int d1 = dir1(I);
  const int ds[2] = {d1, third(I, d1)};
  double sum = 0.0;
  for (int q = 0; q < 2; q++) {
    const int J = ds[q], K = third(I, J);
    const bool present = ft == 0 ? hasH(MODE, K) : hasE(MODE, K);
    if (!present || J >= dim || p.normal[J] == 0.0) continue;
    double proj = 0;
    for (int d = 0; d < dim; d++) {
      const double off = ft == 0 ? (d == K ? -0.5 : 0.0) : (d == K ? 0.0 : -0.5);
      proj += p.k[d] * ((static_cast<double>(idx[d]) - p.origin[d]) * a.dx + off * a.dx);
    }
    const double sv = ft == 0 ? f3d::interp_row(aux.Htab + row * aux.L, aux.L, proj, a.dx, 0.5)
                              : f3d::interp_row(aux.Etab + row * aux.L, aux.L, proj, a.dx, 0.0);
    const float* Fr = a.prof[ft][J].F + a.flen[J];  // raw F follows the scaled F
    const double* pol = ft == 0 ? p.pol_h : p.pol_e;
    sum += levi(I, J, K) * (static_cast<double>(Fr[idx[J]]) / a.dx) * p.normal[J] * sv * pol[K];
  }
  return sum;
}

}  // namespace

// One grid row (blockIdx.y) per plane; cell indices within a plane fit 32 bits.
template <int MODE>
__global__ void __launch_bounds__(256) tfsf_fused_kernel(const __grid_constant__ FusedArgs a, int ft) {
  const int q = blockIdx.y;
  const PlaneDev& p = a.planes[q];
  const int ex = p.hi[0] - p.lo[0] + 1, ey = p.hi[1] - p.lo[1] + 1, ez = p.hi[2] - p.lo[2] + 1;
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= ex * ey * ez) return;
  const int rr = r / ex;
  const int i = p.lo[0] + (r - rr * ex);
  const int j = p.lo[1] + rr % ey;
  const int k = p.lo[2] + rr / ey;
  for (int q0 = 0; q0 < q; q0++)
    if (in_plane(a.planes[q0], i, j, k)) return;  // an earlier plane's thread owns this cell
  const long long t = a.ctrl->t;
  const long long row = t - a.ctrl->t0 + (ft == 0 ? 0 : 1);
  const long long c = (static_cast<long long>(k) * a.ny + j) * a.pitch + i;
  // the cell's fields (and material id) are read before the corrections are
  // formed, so that their latency overlaps the aux-table lookups
  float f0[3] = {0.f, 0.f, 0.f};
  for (int I = 0; I < 3; I++) {
    const bool has = ft == 0 ? hasE(MODE, I) : hasH(MODE, I);
    if (has) f0[I] = ft == 0 ? a.E[I][c] : a.H[I][c];
  }
  int mid = 0;
  if (ft == 0 || a.has_mu) {
    if (a.ids) mid = a.ids[c];
    else if (a.bids) mid = a.bids[((k >> a.bshift) * a.nby + (j >> a.bshift)) * a.nbx + (i >> a.bshift)];
  }
  const float iemap = (ft == 0 && a.inv_eps_map) ? a.inv_eps_map[c] : 0.f;
  double corr[3] = {0.0, 0.0, 0.0};
  for (int q1 = q; q1 < a.nplanes; q1++) {
    const PlaneDev& pp = a.planes[q1];
    if (!in_plane(pp, i, j, k)) continue;
    for (int I = 0; I < 3; I++) {
      const bool has = ft == 0 ? hasE(MODE, I) : hasH(MODE, I);
      if (has) corr[I] += plane_corr<MODE>(a, pp, row, ft, I, i, j, k);
    }
  }
  if (ft == 0) {
    const MatF32& m = a.mats[mid];
    float ie = m.inv_eps;
    if (m.npoles == 0 && iemap > 0.f) ie = iemap;
    const double sc = a.dt / kEps0 * ie;
    for (int I = 0; I < 3; I++) {
      if (!hasE(MODE, I)) continue;
      const float dE = static_cast<float>(sc * corr[I]);
      a.E[I][c] = f0[I] + dE;
      const int np = m.npoles < 0 ? 1 : m.npoles;
      for (int pq = 0; pq < np && pq < 2; pq++) a.J[pq][I][c] += m.b[pq] * dE;
    }
  } else {
    // the correction goes to B; H = B/(mu_r mu0)
    const double sc = a.eta * a.dt / kMu0 * (a.has_mu ? static_cast<double>(a.mats[mid].inv_mu) : 1.0);
    for (int I = 0; I < 3; I++)
      if (hasH(MODE, I)) a.H[I][c] = f0[I] - static_cast<float>(sc * corr[I]);
  }
}

int launch_tfsf_fused(int mode, const FusedArgs& a, int ft, cudaStream_t s) {
  if (a.nplanes == 0) return 0;
  long long most = 0;
  for (int q = 0; q < a.nplanes; q++) {
    const PlaneDev& p = a.planes[q];
    most = std::max(most, static_cast<long long>(p.hi[0] - p.lo[0] + 1) * (p.hi[1] - p.lo[1] + 1) *
                              (p.hi[2] - p.lo[2] + 1));
  }
  const dim3 grid(static_cast<unsigned>((most + 255) / 256), a.nplanes);
  switch (mode) {
    case kTE: tfsf_fused_kernel<kTE><<<grid, 256, 0, s>>>(a, ft); break;
    case kTM: tfsf_fused_kernel<kTM><<<grid, 256, 0, s>>>(a, ft); break;
    default: tfsf_fused_kernel<kThreeD><<<grid, 256, 0, s>>>(a, ft); break;
  }
  return 1;
}

}  // namespace fdtdb
