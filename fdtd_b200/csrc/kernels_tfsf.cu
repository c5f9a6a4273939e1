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

// the two axes of a plane other than its normal axis, the lower first
__host__ __device__ __forceinline__ void plane_axes(int normal, int& u, int& v) {
  u = normal == 0 ? 1 : 0;
  v = normal == 2 ? 1 : 2;
}

// Correction of flux I of type ft at cell idx from plane p, whose normal is
// axis A: TFSFPlane's dir_update term along J = A (the other curl direction
// of I has no normal component), with K = third(I, A). The aux row is
// interpolated at the projection of the cell's field point on k, as
// Aux1D::interpolateE/H do (Source.hpp:442-458); the projection is formed in
// units of dx, the index is clamped to the row.
template <int MODE>
__device__ __forceinline__ double plane_corr(const FusedArgs& a, const PlaneDev& p, long long row, int ft, int I,
                                            const int (&idx)[3], double inv_dx) {
  constexpr int dim = MODE == kThreeD ? 3 : 2;
  const int A = p.axis, K = third(I, A);
  const AuxTab& aux = a.aux[p.aux];
  double nd = static_cast<double>(aux.L) / 2.0 - (ft == 0 ? 0.5 : 0.0);
#pragma unroll
  for (int d = 0; d < dim; d++) {
    const double off = ft == 0 ? (d == K ? -0.5 : 0.0) : (d == K ? 0.0 : -0.5);
    nd += p.k[d] * ((static_cast<double>(idx[d]) - p.origin[d]) + off);
  }
  nd = fmin(fmax(nd, 0.0), static_cast<double>(aux.L - 1));
  long long n = static_cast<long long>(nd);
  if (n > aux.L - 2) n = aux.L - 2;
  const double frac = nd - static_cast<double>(n);
  const double* tab = (ft == 0 ? aux.Htab : aux.Etab) + row * aux.L;
  const double sv = (1.0 - frac) * tab[n] + frac * tab[n + 1];
  const float* Fr = a.prof[ft][A].F + a.flen[A];  // raw F follows the scaled F
  const double* pol = ft == 0 ? p.pol_h : p.pol_e;
  return levi(I, A, K) * (static_cast<double>(Fr[idx[A]]) * inv_dx) * p.normal[A] * sv * pol[K];
}

}  // namespace

// One cell's corrections: the components that a plane containing it
// corrects (those tangential to the plane whose curl partner is in the
// mode), from every such plane in plane order. Grid of the kernel below: x
// over the cells of a plane's lower in-plane axis (128 per CTA), y over its
// other in-plane axis, z over the planes.
template <int MODE>
__device__ __forceinline__ void tfsf_cell(const FusedArgs& a, int ft, int q, const int (&idx)[3]) {
  const int i = idx[0], j = idx[1], k = idx[2];
  for (int q0 = 0; q0 < q; q0++)
    if (in_plane(a.planes[q0], i, j, k)) return;  // an earlier plane's thread owns this cell
  // the components any plane at this cell corrects
  unsigned comps = 0, planes = 0;
  for (int q1 = q; q1 < a.nplanes; q1++) {
    const PlaneDev& pp = a.planes[q1];
    if (!in_plane(pp, i, j, k)) continue;
    planes |= 1u << q1;
#pragma unroll
    for (int I = 0; I < 3; I++) {
      const int K = third(I, pp.axis);
      const bool has = ft == 0 ? hasE(MODE, I) && hasH(MODE, K) : hasH(MODE, I) && hasE(MODE, K);
      if (I != pp.axis && has) comps |= 1u << I;
    }
  }
  const long long c = (static_cast<long long>(k) * a.ny + j) * a.pitch + i;
  // the cell's fields (and material id) are read before the corrections are
  // formed, so that their latency overlaps the aux-table lookups
  float f0[3] = {0.f, 0.f, 0.f};
#pragma unroll
  for (int I = 0; I < 3; I++)
    if (comps >> I & 1) f0[I] = ft == 0 ? a.E[I][c] : a.H[I][c];
  int mid = 0;
  if (ft == 0 || a.has_mu) {
    if (a.ids) mid = a.ids[c];
    else if (a.bids) mid = a.bids[((k >> a.bshift) * a.nby + (j >> a.bshift)) * a.nbx + (i >> a.bshift)];
  }
  const float iemap = (ft == 0 && a.inv_eps_map) ? a.inv_eps_map[c] : 0.f;
  const long long t = a.ctrl->t;
  const long long row = t - a.ctrl->t0 + (ft == 0 ? 0 : 1);
  const double inv_dx = 1.0 / a.dx;
  double corr[3] = {0.0, 0.0, 0.0};
  for (unsigned m = planes; m; m &= m - 1) {
    const PlaneDev& pp = a.planes[__ffs(m) - 1];
#pragma unroll
    for (int I = 0; I < 3; I++) {
      const int K = third(I, pp.axis);
      const bool has = ft == 0 ? hasE(MODE, I) && hasH(MODE, K) : hasH(MODE, I) && hasE(MODE, K);
      if (I != pp.axis && has) corr[I] += plane_corr<MODE>(a, pp, row, ft, I, idx, inv_dx);
    }
  }
  if (ft == 0) {
    const MatF32& m = a.mats[mid];
    float ie = m.inv_eps;
    if (m.npoles == 0 && iemap > 0.f) ie = iemap;
    const double sc = a.dt / kEps0 * ie;
    const int np = m.npoles < 0 ? 1 : m.npoles;
#pragma unroll
    for (int I = 0; I < 3; I++) {
      if (!(comps >> I & 1)) continue;
      const float dE = static_cast<float>(sc * corr[I]);
      a.E[I][c] = f0[I] + dE;
      for (int pq = 0; pq < np && pq < 2; pq++) a.J[pq][I][c] += m.b[pq] * dE;
    }
  } else {
    // the correction goes to B; H = B/(mu_r mu0)
    const double sc = a.eta * a.dt / kMu0 * (a.has_mu ? static_cast<double>(a.mats[mid].inv_mu) : 1.0);
#pragma unroll
    for (int I = 0; I < 3; I++)
      if (comps >> I & 1) a.H[I][c] = f0[I] - static_cast<float>(sc * corr[I]);
  }
}

template <int MODE>
__global__ void __launch_bounds__(128) tfsf_fused_kernel(const __grid_constant__ FusedArgs a, int ft) {
  const int q = blockIdx.z;
  const PlaneDev& p = a.planes[q];
  int u, v;
  plane_axes(p.axis, u, v);
  const int uu = blockIdx.x * blockDim.x + threadIdx.x, vv = blockIdx.y;
  if (p.lo[u] + uu > p.hi[u] || p.lo[v] + vv > p.hi[v]) return;
  int idx[3];
  idx[u] = p.lo[u] + uu;
  idx[v] = p.lo[v] + vv;
  // a plane is one cell thick along its normal as a rule; a thicker one is
  // walked cell by cell
  for (int w = p.lo[p.axis]; w <= p.hi[p.axis]; w++) {
    idx[p.axis] = w;
    tfsf_cell<MODE>(a, ft, q, idx);
  }
}

int launch_tfsf_fused(int mode, const FusedArgs& a, int ft, cudaStream_t s) {
  if (a.nplanes == 0) return 0;
  int most_u = 1, most_v = 1;
  for (int q = 0; q < a.nplanes; q++) {
    const PlaneDev& p = a.planes[q];
    int u, v;
    plane_axes(p.axis, u, v);
    most_u = std::max(most_u, p.hi[u] - p.lo[u] + 1);
    most_v = std::max(most_v, p.hi[v] - p.lo[v] + 1);
  }
  const dim3 grid(static_cast<unsigned>((most_u + 127) / 128), static_cast<unsigned>(most_v), a.nplanes);
  switch (mode) {
    case kTE: tfsf_fused_kernel<kTE><<<grid, 128, 0, s>>>(a, ft); break;
    case kTM: tfsf_fused_kernel<kTM><<<grid, 128, 0, s>>>(a, ft); break;
    default: tfsf_fused_kernel<kThreeD><<<grid, 128, 0, s>>>(a, ft); break;
  }
  return 1;
}

}  // namespace fdtdb
