// FP64 "plain" method: one fused kernel per half step that performs, for each
// interior cell, exactly the per-cell operations of the reference's passes in
// the reference's floating-point order:
//   E half: YeeUpdate on every E flux (YeeUpdates.hpp:396-405), TFSFPlane::
//           updateD (Source.hpp:595-609), D-target SoftSource, UpdatePML<..,
//           Electric, X|Y|Z> (PML.hpp:306-354), the material update
//           (DispersiveMaterials.hpp:354-359, :710-735, :979-998) and
//           E-target SoftSource::apply (Source.hpp:209-211).
//   H half: the same for B/H with updateB and VacuumUpdate/ConstantUpdate.
// Every reference pass reads only fields that the current half step does not
// write (H in the E half, E in the H half), or the cell's own state, so fusing
// the passes per cell leaves every result unchanged.
//
// This file is compiled with -fmad=false: no multiply-add contraction, so each
// product and sum rounds as in the reference compiled with -ffp-contract=off.
#include "internal.h"

namespace fdtdb {

__device__ __forceinline__ double interp_aux(const double* row, int L, double loc, double dx, double shift) {
  // Aux1D::interpolateE / interpolateH (include/Source.hpp:442-458); the host
  // checked that every plane cell lands in 0 <= n <= L-2.
  double nd = static_cast<double>(L) / 2.0 + loc / dx - shift;
  unsigned long long n = static_cast<unsigned long long>(nd);
  double frac = nd - static_cast<double>(n);
  return (1.0 - frac) * row[n] + frac * row[n + 1];
}

// TFSFPlane::field_update::dir_update (Source.hpp:506-531) for flux I of type
// ft at cell idx, summed over d1, d2 as in field_update::get (:542-553).
template <int MODE>
__device__ double tfsf_term(const PlaneDev& p, const AuxTab& aux, long long row, int ft, int I, const int idx[3],
                            const Prof<double> (&prof)[2][3], double dx) {
  constexpr int dim = MODE == kThreeD ? 3 : 2;
  const int d1 = dir1(I);
  const int ds[2] = {d1, third(I, d1)};
  double terms[2];
#pragma unroll
  for (int q = 0; q < 2; q++) {
    const int J = ds[q], K = third(I, J);
    const bool present = ft == 0 ? hasH(MODE, K) : hasE(MODE, K);
    if (!present) {
      terms[q] = 0.0;
      continue;
    }
    // CurlField offsets (FDTDConstants.hpp:680-744): H_K sits at -0.5 along K
    // only, E_K at -0.5 along the two axes other than K.
    double src[3];
#pragma unroll
    for (int d = 0; d < dim; d++) {
      const double off = ft == 0 ? (d == K ? -0.5 : 0.0) : (d == K ? 0.0 : -0.5);
      const double center = (static_cast<double>(idx[d]) - p.origin[d]) * dx;
      src[d] = center + off * dx;
    }
    double proj = 0;
#pragma unroll
    for (int d = 0; d < dim; d++) proj += p.k[d] * src[d];
    const double sv = ft == 0 ? interp_aux(aux.Htab + row * aux.L, aux.L, proj, dx, 0.5)
                              : interp_aux(aux.Etab + row * aux.L, aux.L, proj, dx, 0.0);
    const double Fdx = prof[ft][J].F[idx[J]];
    const double* pol = ft == 0 ? p.pol_h : p.pol_e;
    terms[q] = (levi(I, J, K) == 1 ? Fdx : -Fdx) * p.normal[J] * sv * pol[K];
  }
  return terms[0] + terms[1];
}

// YeeUpdate::update_all (YeeUpdates.hpp:396-405) of flux F at cell c with the
// summed curl terms: F = TimePolicy::get(F) + (Coeff*curl_coeff*dt) * curl,
// then TimePolicy::increment moves the old flux into the history (BD3:
// :209-213, :231-236; BD4: :258-263, :282-288). sdt = Coeff*curl_coeff*dt.
__device__ __forceinline__ void time_policy_update(const PlainArgs& a, int ft, int I, long long c, double* F,
                                                   double sdt, double curl) {
  const double old = F[c];
  if (a.bd == 0) {
    F[c] = old + sdt * curl;
    return;
  }
  double* h0 = a.hist[ft][0][I] + c;
  double* h1 = a.hist[ft][1][I] + c;
  if (a.bd == 2) {
    const double get = a.bdk[0] * old + a.bdk[1] * *h0 - a.bdk[2] * *h1;
    F[c] = get + sdt * curl;
  } else {
    double* h2 = a.hist[ft][2][I] + c;
    const double get = a.bdk[0] * old + a.bdk[1] * *h0 - a.bdk[2] * *h1 + a.bdk[3] * *h2;
    F[c] = get + sdt * curl;
    *h2 = *h1;
  }
  *h1 = *h0;
  *h0 = old;
}

template <int MODE>
__global__ void __launch_bounds__(256) plain_e_kernel(const __grid_constant__ PlainArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int k = MODE == kThreeD ? blockIdx.z + 1 : 0;
  if (i > a.nx - 2 || j > a.ny - 2) return;
  const long long sy = a.nx, sz = static_cast<long long>(a.nx) * a.ny;
  const long long c = k * sz + j * sy + i;
  const long long str[3] = {1, sy, sz};
  const int idx[3] = {i, j, k};
  const double dt = a.dt;
  const long long t = a.ctrl->t;

  // YeeUpdate<Mode, D_I, TimePolicy>: a = LC*F/dx*(H_K - H_K[-J])
#pragma unroll
  for (int I = 0; I < 3; I++) {
    if (!hasE(MODE, I)) continue;
    const int d1 = dir1(I);
    const int ds[2] = {d1, third(I, d1)};
    double at[2];
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const int J = ds[q], K = third(I, J);
      if (!hasH(MODE, K)) {
        at[q] = 0.0;
        continue;
      }
      const double diff = a.H.f[K][c] - a.H.f[K][c - str[J]];
      const double fdx = a.prof[0][J].F[idx[J]];
      at[q] = (levi(I, J, K) == 1 ? fdx : -fdx) * diff;
    }
    time_policy_update(a, 0, I, c, a.D.f[I], a.cc * dt, at[0] + at[1]);
  }
  // TFSFPlane::updateD
  for (int q = 0; q < a.nplanes; q++) {
    const PlaneDev& p = a.planes[q];
    if (i < p.lo[0] || i > p.hi[0] || j < p.lo[1] || j > p.hi[1] || k < p.lo[2] || k > p.hi[2]) continue;
    const AuxTab& ax = a.aux[p.aux];
    const long long row = t - a.ctrl->t0;
#pragma unroll
    for (int I = 2; I >= 0; I--) {
      if (!hasE(MODE, I)) continue;
      a.D.f[I][c] += a.cc * dt * tfsf_term<MODE>(p, ax, row, 0, I, idx, a.prof, a.dx);
    }
  }
  // SoftSource on D
  for (int s = 0; s < a.nsrc; s++) {
    const SourceDev& sr = a.src[s];
    if (sr.target != 1 || sr.cell != c) continue;
    a.D.f[sr.comp][c] += t < sr.nvals ? sr.vals[t] : 0.0;
  }
  // UpdatePML<Mode, Electric, J>, J = X, Y, Z in that order
#pragma unroll
  for (int J = 0; J < 3; J++) {
    if (!a.pml_axis[J]) continue;
    const int s = slab_index(a.slab[J], idx[J]);
    if (s < 0) continue;
    long long pidx;
    if (J == 0) pidx = (static_cast<long long>(k) * a.ny + j) * a.slab[0].W + s;
    else if (J == 1) pidx = (static_cast<long long>(k) * a.slab[1].W + s) * a.nx + i;
    else pidx = (static_cast<long long>(s) * a.ny + j) * a.nx + i;
    const double B = a.prof[0][J].B[idx[J]];
    const double Cdx = a.prof[0][J].C[idx[J]];
    const double G = a.prof[0][J].G[idx[J]];
#pragma unroll
    for (int I = 2; I >= 0; I--) {
      if (!hasE(MODE, I) || I == J) continue;
      const int K = third(I, J);
      double* ps = a.psi[0][I][J] + pidx;
      const double psi = *ps;
      a.D.f[I][c] += dt * psi * G;
      const double diff = a.H.f[K][c] - a.H.f[K][c - str[J]];
      *ps = B * psi + (levi(I, J, K) == 1 ? Cdx : -Cdx) * diff;
    }
  }
  // material update
  int mid = 0;
  if (a.ids) mid = a.ids[c];
  else if (a.bids) mid = a.bids[((k >> a.bshift) * a.nby + (j >> a.bshift)) * a.nbx + (i >> a.bshift)];
  const MatF64 m = a.mats[mid];
#pragma unroll
  for (int I = 2; I >= 0; I--) {
    if (!hasE(MODE, I)) continue;
    const double D = a.D.f[I][c];
    if (m.kind <= 1) {
      // a per-cell permittivity replaces the ConstantUpdate K of the cell
      const double den = (a.eps_map && a.eps_map[c] > 0.0) ? a.eps_map[c] * kEps0 : m.den_e;
      a.E.f[I][c] = D / den;
    } else if (m.kind == 2) {
      // drude::DrudeUpdate::implicit_update (DispersiveMaterials.hpp:979-998)
      double P = a.P[0].f[I][c], Jc = a.J[0].f[I][c];
      P += dt * Jc;
      const double E = (D - P) / m.den_e;
      Jc = Jc * m.c1[0] / m.c2[0] + m.c3[0] * E;
      a.P[0].f[I][c] = P;
      a.J[0].f[I][c] = Jc;
      a.E.f[I][c] = E;
    } else {
      // lorentz::LorentzUpdate::implicit_update (DispersiveMaterials.hpp:710-735),
      // one term per pole
      double num = D;
      double P[kMaxPoles];
      for (int q = 0; q < m.npoles; q++) {
        P[q] = a.P[q].f[I][c] + dt * a.J[q].f[I][c];
        a.P[q].f[I][c] = P[q];
        num = num - P[q];
      }
      const double E = num / m.den_e;
      for (int q = 0; q < m.npoles; q++) {
        const double Jc = a.J[q].f[I][c];
        a.J[q].f[I][c] = m.c1[q] * Jc + m.c2[q] * E - m.c3[q] * P[q];
      }
      a.E.f[I][c] = E;
    }
  }
  // SoftSource on E
  for (int s = 0; s < a.nsrc; s++) {
    const SourceDev& sr = a.src[s];
    if (sr.target != 0 || sr.cell != c) continue;
    a.E.f[sr.comp][c] += t < sr.nvals ? sr.vals[t] : 0.0;
  }
}

template <int MODE>
__global__ void __launch_bounds__(256) plain_h_kernel(const __grid_constant__ PlainArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int k = MODE == kThreeD ? blockIdx.z + 1 : 0;
  if (i > a.nx - 2 || j > a.ny - 2) return;
  const long long sy = a.nx, sz = static_cast<long long>(a.nx) * a.ny;
  const long long c = k * sz + j * sy + i;
  const long long str[3] = {1, sy, sz};
  const int idx[3] = {i, j, k};
  const double dt = a.dt;
  const long long t = a.ctrl->t;

  // YeeUpdate<Mode, B_I, TimePolicy>: a = LC*F/dx*(E_K[+J] - E_K)
#pragma unroll
  for (int I = 0; I < 3; I++) {
    if (!hasH(MODE, I)) continue;
    const int d1 = dir1(I);
    const int ds[2] = {d1, third(I, d1)};
    double at[2];
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const int J = ds[q], K = third(I, J);
      if (!hasE(MODE, K)) {
        at[q] = 0.0;
        continue;
      }
      const double diff = a.E.f[K][c + str[J]] - a.E.f[K][c];
      const double fdx = a.prof[1][J].F[idx[J]];
      at[q] = (levi(I, J, K) == 1 ? fdx : -fdx) * diff;
    }
    time_policy_update(a, 1, I, c, a.B.f[I], -a.cc * dt, at[0] + at[1]);
  }
  // TFSFPlane::updateB (the aux grid was advanced by updateD: row + 1)
  for (int q = 0; q < a.nplanes; q++) {
    const PlaneDev& p = a.planes[q];
    if (i < p.lo[0] || i > p.hi[0] || j < p.lo[1] || j > p.hi[1] || k < p.lo[2] || k > p.hi[2]) continue;
    const AuxTab& ax = a.aux[p.aux];
    const long long row = t - a.ctrl->t0 + 1;
#pragma unroll
    for (int I = 2; I >= 0; I--) {
      if (!hasH(MODE, I)) continue;
      a.B.f[I][c] += -a.cc * dt * tfsf_term<MODE>(p, ax, row, 1, I, idx, a.prof, a.dx);
    }
  }
  // SoftSource on B
  for (int s = 0; s < a.nsrc; s++) {
    const SourceDev& sr = a.src[s];
    if (sr.target != 3 || sr.cell != c) continue;
    a.B.f[sr.comp][c] += t < sr.nvals ? sr.vals[t] : 0.0;
  }
  // UpdatePML<Mode, Magnetic, J>
#pragma unroll
  for (int J = 0; J < 3; J++) {
    if (!a.pml_axis[J]) continue;
    const int s = slab_index(a.slab[J], idx[J]);
    if (s < 0) continue;
    long long pidx;
    if (J == 0) pidx = (static_cast<long long>(k) * a.ny + j) * a.slab[0].W + s;
    else if (J == 1) pidx = (static_cast<long long>(k) * a.slab[1].W + s) * a.nx + i;
    else pidx = (static_cast<long long>(s) * a.ny + j) * a.nx + i;
    const double B = a.prof[1][J].B[idx[J]];
    const double Cdx = a.prof[1][J].C[idx[J]];
    const double G = a.prof[1][J].G[idx[J]];
#pragma unroll
    for (int I = 2; I >= 0; I--) {
      if (!hasH(MODE, I) || I == J) continue;
      const int K = third(I, J);
      double* ps = a.psi[1][I][J] + pidx;
      const double psi = *ps;
      a.B.f[I][c] += -dt * psi * G;
      const double diff = a.E.f[K][c + str[J]] - a.E.f[K][c];
      *ps = B * psi + (levi(I, J, K) == 1 ? Cdx : -Cdx) * diff;
    }
  }
  // VacuumUpdate / ConstantUpdate<Mode, Magnetic>: H = B/(mu_r*mu0)
  int mid = 0;
  if (a.ids) mid = a.ids[c];
  else if (a.bids) mid = a.bids[((k >> a.bshift) * a.nby + (j >> a.bshift)) * a.nbx + (i >> a.bshift)];
  const double den = a.mats[mid].den_h;
#pragma unroll
  for (int I = 2; I >= 0; I--) {
    if (!hasH(MODE, I)) continue;
    a.H.f[I][c] = a.B.f[I][c] / den;
  }
  // SoftSource on H
  for (int s = 0; s < a.nsrc; s++) {
    const SourceDev& sr = a.src[s];
    if (sr.target != 2 || sr.cell != c) continue;
    a.H.f[sr.comp][c] += t < sr.nvals ? sr.vals[t] : 0.0;
  }
}

template <int MODE>
static int launch_plain(const PlainArgs& a, cudaStream_t s, bool e) {
  dim3 block(32, 8, 1);
  dim3 grid((a.nx - 2 + 31) / 32, (a.ny - 2 + 7) / 8, MODE == kThreeD ? a.nz - 2 : 1);
  if (e) plain_e_kernel<MODE><<<grid, block, 0, s>>>(a);
  else plain_h_kernel<MODE><<<grid, block, 0, s>>>(a);
  return 1;
}

int launch_plain_e(int mode, const PlainArgs& a, cudaStream_t s) {
  switch (mode) {
    case kTE: return launch_plain<kTE>(a, s, true);
    case kTM: return launch_plain<kTM>(a, s, true);
    default: return launch_plain<kThreeD>(a, s, true);
  }
}
int launch_plain_h(int mode, const PlainArgs& a, cudaStream_t s) {
  switch (mode) {
    case kTE: return launch_plain<kTE>(a, s, false);
    case kTM: return launch_plain<kTM>(a, s, false);
    default: return launch_plain<kThreeD>(a, s, false);
  }
}

// ----------------------------------------------------------------------------
// Aux1D::time_step (include/Source.hpp:413-435) advanced nsteps times by one
// CTA, writing Ez and Hy after every step into the tables (row 0 = the state
// on entry). coef holds the aux CPML profile: [ft][B,Cdx,Fdx,G][L].
// Cells 0 and L-1 see the zero ghost cells of Aux1D::Stencil1D.
__global__ void aux_kernel(int L, double dt, double dx, double* Dz, double* Ez, double* By, double* Hy,
                           double* psiE, double* psiH, const double* coef, const double* vals, int nvals,
                           long long s0, int nsteps, double* Etab, double* Htab) {
  const double* eB = coef;
  const double* eC = coef + L;
  const double* eF = coef + 2 * L;
  const double* eG = coef + 3 * L;
  const double* hB = coef + 4 * L;
  const double* hC = coef + 5 * L;
  const double* hF = coef + 6 * L;
  const double* hG = coef + 7 * L;
  for (int x = threadIdx.x; x < L; x += blockDim.x) {
    Etab[x] = Ez[x];
    Htab[x] = Hy[x];
  }
  for (int s = 1; s <= nsteps; s++) {
    const long long sa = s0 + s;  // aux step number
    __syncthreads();
    // YeeUpdate<TEM,Dz> then UpdatePML<TEM,Electric,X> then VacuumUpdate E
    for (int x = threadIdx.x; x < L; x += blockDim.x) {
      const double hm = x > 0 ? Hy[x - 1] : 0.0;
      const double diff = Hy[x] - hm;
      double D = Dz[x] + dt * (eF[x] * diff + 0.0);
      const double psi = psiE[x];
      D += dt * psi * eG[x];
      psiE[x] = eB[x] * psi + eC[x] * diff;
      Dz[x] = D;
      Ez[x] = D / kEps0;
    }
    __syncthreads();
    if (threadIdx.x == 0) Ez[kAuxNpml + 5] += (sa >= 1 && sa <= nvals) ? vals[sa - 1] : 0.0;
    __syncthreads();
    // YeeUpdate<TEM,By>, UpdatePML<TEM,Magnetic,X>, VacuumUpdate H
    for (int x = threadIdx.x; x < L; x += blockDim.x) {
      const double ep = x < L - 1 ? Ez[x + 1] : 0.0;
      const double diff = ep - Ez[x];
      double B = By[x] + -dt * (0.0 + -hF[x] * diff);
      const double psi = psiH[x];
      B += -dt * psi * hG[x];
      psiH[x] = hB[x] * psi + -hC[x] * diff;
      By[x] = B;
    }
    __syncthreads();
    for (int x = threadIdx.x; x < L; x += blockDim.x) {
      Hy[x] = By[x] / kMu0;
      Etab[static_cast<long long>(s) * L + x] = Ez[x];
    }
    __syncthreads();
    for (int x = threadIdx.x; x < L; x += blockDim.x) Htab[static_cast<long long>(s) * L + x] = Hy[x];
  }
}

int launch_aux_precompute(int L, double dt, double dx, double* Dz, double* Ez, double* By, double* Hy,
                          double* psiE, double* psiH, const double* coef, const double* vals, int nvals,
                          long long s0, int nsteps, double* Etab, double* Htab, cudaStream_t s) {
  (void)dx;
  aux_kernel<<<1, 1024, 0, s>>>(L, dt, dx, Dz, Ez, By, Hy, psiE, psiH, coef, vals, nvals, s0, nsteps, Etab, Htab);
  return 1;
}

}  // namespace fdtdb
