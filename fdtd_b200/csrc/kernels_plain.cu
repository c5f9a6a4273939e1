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

constexpr int kPlainThreads = 256;  // 32 x 8 cells per CTA

__device__ __forceinline__ void cp_async8(double* dst, const double* src) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(src) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// shared-memory slots (one double per thread each) of the plain kernels:
// E half: H at the cell and its curl neighbours, D, the CPML integrators,
// and P, J of NP poles; H half: E and its neighbours, B, the integrators
__host__ __device__ constexpr int plain_e_slots(int mode, int np) {
  int n = 0;
  for (int K = 0; K < 3; K++) n += hasH(mode, K) ? 1 : 0;
  for (int I = 0; I < 3; I++)
    for (int J = 0; J < 3; J++)
      if (I != J && hasE(mode, I) && hasH(mode, third(I, J))) n++;
  for (int I = 0; I < 3; I++) n += hasE(mode, I) ? 1 : 0;
  for (int J = 0; J < 3; J++)
    for (int I = 0; I < 3; I++)
      if (hasE(mode, I) && I != J && !(mode != kThreeD && J == 2)) n++;
  for (int I = 0; I < 3; I++) n += hasE(mode, I) ? 2 * np : 0;
  return n;
}

__host__ __device__ constexpr int plain_h_slots(int mode) {
  int n = 0;
  for (int K = 0; K < 3; K++) n += hasE(mode, K) ? 1 : 0;
  for (int I = 0; I < 3; I++)
    for (int J = 0; J < 3; J++)
      if (I != J && hasH(mode, I) && hasE(mode, third(I, J))) n++;
  for (int I = 0; I < 3; I++) n += hasH(mode, I) ? 1 : 0;
  for (int J = 0; J < 3; J++)
    for (int I = 0; I < 3; I++)
      if (hasH(mode, I) && I != J && !(mode != kThreeD && J == 2)) n++;
  return n;
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

// Both kernels first request every operand of their cell -- the H (E)
// values of the curl, the flux, the CPML integrators and, with every
// material dispersive, P and J -- with cp.async into the thread's own
// shared-memory slots (copies in flight hold no registers), read them back,
// apply the passes above to registers in the reference's order, and store
// the results at the end. The arrays may alias as far as the compiler knows,
// so reading each pass's operands after the previous pass's stores would
// make a cell wait for one memory round trip per pass; here all the reads
// are in flight together. The arithmetic, and so every result, is the same.
//
// NP: poles of P and J read with the fields (0: read after the material id,
// for the cells whose material has poles). HIST: the BD3/BD4 time policy's
// flux history is read and moved (a separate instantiation, so that the
// leapfrog's kernels keep their registers).
template <int MODE, int NP, bool HIST>
__global__ void __launch_bounds__(kPlainThreads, 2) plain_e_kernel(const __grid_constant__ PlainArgs a) {
  extern __shared__ double smd[];
  constexpr int NPS = NP > 0 ? NP : 1;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
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

  // ---- every read of the cell, copied into the thread's shared-memory slots
  // (cp.async: in flight together without holding registers), then read
  // back; the CPML integrators only where the cell lies in a slab
  double* slot = smd + tid;
  int ns = 0;
  int s_hc[3] = {}, s_hn[3][3] = {}, s_d[3] = {}, s_ps[3][3] = {}, s_p[NPS][3] = {}, s_j[NPS][3] = {};
#pragma unroll
  for (int K = 0; K < 3; K++)
    if (hasH(MODE, K)) {
      s_hc[K] = ns++;
      cp_async8(slot + s_hc[K] * kPlainThreads, a.H.f[K] + c);
    }
#pragma unroll
  for (int I = 0; I < 3; I++) {
    if (!hasE(MODE, I)) continue;
#pragma unroll
    for (int J = 0; J < 3; J++) {
      if (J == I) continue;
      const int K = third(I, J);
      if (!hasH(MODE, K)) continue;
      s_hn[K][J] = ns++;
      cp_async8(slot + s_hn[K][J] * kPlainThreads, a.H.f[K] + c - str[J]);
    }
  }
#pragma unroll
  for (int I = 0; I < 3; I++)
    if (hasE(MODE, I)) {
      s_d[I] = ns++;
      cp_async8(slot + s_d[I] * kPlainThreads, a.D.f[I] + c);
    }
  long long pidx[3] = {-1, -1, -1};
#pragma unroll
  for (int J = 0; J < 3; J++) {
    const int s = a.pml_axis[J] ? slab_index(a.slab[J], idx[J]) : -1;
    if (s >= 0) {
      if (J == 0) pidx[J] = (static_cast<long long>(k) * a.ny + j) * a.slab[0].W + s;
      else if (J == 1) pidx[J] = (static_cast<long long>(k) * a.slab[1].W + s) * a.nx + i;
      else pidx[J] = (static_cast<long long>(s) * a.ny + j) * a.nx + i;
    }
#pragma unroll
    for (int I = 0; I < 3; I++) {
      if (!hasE(MODE, I) || I == J || (MODE != kThreeD && J == 2)) continue;
      s_ps[I][J] = ns++;
      if (pidx[J] >= 0) cp_async8(slot + s_ps[I][J] * kPlainThreads, a.psi[0][I][J] + pidx[J]);
    }
  }
#pragma unroll
  for (int q = 0; q < NP; q++)
#pragma unroll
    for (int I = 0; I < 3; I++)
      if (hasE(MODE, I)) {
        s_p[q][I] = ns++;
        s_j[q][I] = ns++;
        if (q < a.dispersive) {
          cp_async8(slot + s_p[q][I] * kPlainThreads, a.P[q].f[I] + c);
          cp_async8(slot + s_j[q][I] * kPlainThreads, a.J[q].f[I] + c);
        }
      }
  double h0[3] = {}, h1[3] = {}, h2[3] = {};
#pragma unroll
  for (int I = 0; I < 3; I++) {
    if (!hasE(MODE, I)) continue;
    if (HIST) {
      h0[I] = a.hist[0][0][I][c];
      h1[I] = a.hist[0][1][I][c];
      if (a.bd == 3) h2[I] = a.hist[0][2][I][c];
    }
  }
  int mid = 0;
  if (a.ids) mid = a.ids[c];
  else if (a.bids) mid = a.bids[((k >> a.bshift) * a.nby + (j >> a.bshift)) * a.nbx + (i >> a.bshift)];
  cp_async_wait_all();
  double hc[3] = {0.0, 0.0, 0.0}, hn[3][3] = {}, d[3] = {0.0, 0.0, 0.0}, ps[3][3] = {};
  double pp[NPS][3] = {}, jj[NPS][3] = {};
#pragma unroll
  for (int K = 0; K < 3; K++)
    if (hasH(MODE, K)) hc[K] = slot[s_hc[K] * kPlainThreads];
#pragma unroll
  for (int K = 0; K < 3; K++)
#pragma unroll
    for (int J = 0; J < 3; J++)
      if (J != K && hasH(MODE, K)) {
        const int I = third(J, K);
        if (hasE(MODE, I)) hn[K][J] = slot[s_hn[K][J] * kPlainThreads];
      }
#pragma unroll
  for (int I = 0; I < 3; I++)
    if (hasE(MODE, I)) d[I] = slot[s_d[I] * kPlainThreads];
#pragma unroll
  for (int J = 0; J < 3; J++)
#pragma unroll
    for (int I = 0; I < 3; I++)
      if (hasE(MODE, I) && I != J && !(MODE != kThreeD && J == 2) && pidx[J] >= 0)
        ps[I][J] = slot[s_ps[I][J] * kPlainThreads];
#pragma unroll
  for (int q = 0; q < NP; q++)
#pragma unroll
    for (int I = 0; I < 3; I++)
      if (hasE(MODE, I) && q < a.dispersive) {
        pp[q][I] = slot[s_p[q][I] * kPlainThreads];
        jj[q][I] = slot[s_j[q][I] * kPlainThreads];
      }
  const double eps_cell = a.eps_map ? a.eps_map[c] : 0.0;

  // ---- YeeUpdate<Mode, D_I, TimePolicy>: a = LC*F/dx*(H_K - H_K[-J])
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
      const double diff = hc[K] - hn[K][J];
      const double fdx = a.prof[0][J].F[idx[J]];
      at[q] = (levi(I, J, K) == 1 ? fdx : -fdx) * diff;
    }
    // TimePolicy::get + increment (YeeUpdates.hpp:182-294), as time_policy_update
    const double old = d[I], sdt = a.cc * dt, curl = at[0] + at[1];
    if (!HIST) {
      d[I] = old + sdt * curl;
    } else if (a.bd == 2) {
      const double get = a.bdk[0] * old + a.bdk[1] * h0[I] - a.bdk[2] * h1[I];
      d[I] = get + sdt * curl;
      h1[I] = h0[I];
      h0[I] = old;
    } else {
      const double get = a.bdk[0] * old + a.bdk[1] * h0[I] - a.bdk[2] * h1[I] + a.bdk[3] * h2[I];
      d[I] = get + sdt * curl;
      h2[I] = h1[I];
      h1[I] = h0[I];
      h0[I] = old;
    }
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
      d[I] += a.cc * dt * tfsf_term<MODE>(p, ax, row, 0, I, idx, a.prof, a.dx);
    }
  }
  // SoftSource on D
  for (int s = 0; s < a.nsrc; s++) {
    const SourceDev& sr = a.src[s];
    if (sr.target != 1 || sr.cell != c) continue;
    const double v = t < sr.nvals ? sr.vals[t] : 0.0;
#pragma unroll
    for (int I = 0; I < 3; I++)
      if (sr.comp == I) d[I] += v;
  }
  // UpdatePML<Mode, Electric, J>, J = X, Y, Z in that order
#pragma unroll
  for (int J = 0; J < 3; J++) {
    if (pidx[J] < 0) continue;
    const double B = a.prof[0][J].B[idx[J]];
    const double Cdx = a.prof[0][J].C[idx[J]];
    const double G = a.prof[0][J].G[idx[J]];
#pragma unroll
    for (int I = 2; I >= 0; I--) {
      if (!hasE(MODE, I) || I == J) continue;
      const int K = third(I, J);
      const double psi = ps[I][J];
      d[I] += dt * psi * G;
      const double diff = hc[K] - hn[K][J];
      ps[I][J] = B * psi + (levi(I, J, K) == 1 ? Cdx : -Cdx) * diff;
    }
  }
  // material update
  const MatF64& m = a.mats[mid];
  if (NP == 0 && m.kind >= 2) {
    for (int q = 0; q < NPS; q++)  // NP == 0: NPS == 1, pole 0 here, further poles below
#pragma unroll
      for (int I = 0; I < 3; I++)
        if (hasE(MODE, I)) {
          pp[q][I] = a.P[q].f[I][c];
          jj[q][I] = a.J[q].f[I][c];
        }
  }
  double e[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int I = 2; I >= 0; I--) {
    if (!hasE(MODE, I)) continue;
    const double D = d[I];
    if (m.kind <= 1) {
      // a per-cell permittivity replaces the ConstantUpdate K of the cell
      const double den = (a.eps_map && eps_cell > 0.0) ? eps_cell * kEps0 : m.den_e;
      e[I] = D / den;
    } else if (m.kind == 2) {
      // drude::DrudeUpdate::implicit_update (DispersiveMaterials.hpp:979-998)
      double P = pp[0][I], Jc = jj[0][I];
      P += dt * Jc;
      const double E = (D - P) / m.den_e;
      Jc = Jc * m.c1[0] / m.c2[0] + m.c3[0] * E;
      pp[0][I] = P;
      jj[0][I] = Jc;
      e[I] = E;
    } else if (NP > 0 && m.npoles <= NP) {
      // lorentz::LorentzUpdate::implicit_update (DispersiveMaterials.hpp:710-735),
      // one term per pole, on the staged poles
      double num = D;
      double P[NPS];
#pragma unroll
      for (int q = 0; q < NPS; q++) {
        if (q >= m.npoles) continue;
        P[q] = pp[q][I] + dt * jj[q][I];
        pp[q][I] = P[q];
        num = num - P[q];
      }
      const double E = num / m.den_e;
#pragma unroll
      for (int q = 0; q < NPS; q++) {
        if (q >= m.npoles) continue;
        jj[q][I] = m.c1[q] * jj[q][I] + m.c2[q] * E - m.c3[q] * P[q];
      }
      e[I] = E;
    } else {
      // the same with the poles read and written here
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
      e[I] = E;
    }
  }
  // SoftSource on E
  for (int s = 0; s < a.nsrc; s++) {
    const SourceDev& sr = a.src[s];
    if (sr.target != 0 || sr.cell != c) continue;
    const double v = t < sr.nvals ? sr.vals[t] : 0.0;
#pragma unroll
    for (int I = 0; I < 3; I++)
      if (sr.comp == I) e[I] += v;
  }

  // ---- every write of the cell
#pragma unroll
  for (int I = 0; I < 3; I++) {
    if (!hasE(MODE, I)) continue;
    a.D.f[I][c] = d[I];
    a.E.f[I][c] = e[I];
    if (HIST) {
      a.hist[0][0][I][c] = h0[I];
      a.hist[0][1][I][c] = h1[I];
      if (a.bd == 3) a.hist[0][2][I][c] = h2[I];
    }
  }
#pragma unroll
  for (int J = 0; J < 3; J++) {
    if (pidx[J] < 0) continue;
#pragma unroll
    for (int I = 0; I < 3; I++)
      if (hasE(MODE, I) && I != J) a.psi[0][I][J][pidx[J]] = ps[I][J];
  }
  const bool staged = NP > 0 ? (m.kind == 2 || m.npoles <= NP) : m.kind == 2;
  if (m.kind >= 2 && staged) {
    const int np = m.kind == 2 ? 1 : m.npoles;
#pragma unroll
    for (int q = 0; q < NPS; q++) {
      if (q >= np) continue;
#pragma unroll
      for (int I = 0; I < 3; I++)
        if (hasE(MODE, I)) {
          a.P[q].f[I][c] = pp[q][I];
          a.J[q].f[I][c] = jj[q][I];
        }
    }
  }
}

template <int MODE, bool HIST>
__global__ void __launch_bounds__(kPlainThreads, 2) plain_h_kernel(const __grid_constant__ PlainArgs a) {
  extern __shared__ double smd[];
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
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

  // ---- every read of the cell, through the thread's shared-memory slots
  double* slot = smd + tid;
  int ns = 0;
  int s_ec[3] = {}, s_en[3][3] = {}, s_b[3] = {}, s_ps[3][3] = {};
#pragma unroll
  for (int K = 0; K < 3; K++)
    if (hasE(MODE, K)) {
      s_ec[K] = ns++;
      cp_async8(slot + s_ec[K] * kPlainThreads, a.E.f[K] + c);
    }
#pragma unroll
  for (int I = 0; I < 3; I++) {
    if (!hasH(MODE, I)) continue;
#pragma unroll
    for (int J = 0; J < 3; J++) {
      if (J == I) continue;
      const int K = third(I, J);
      if (!hasE(MODE, K)) continue;
      s_en[K][J] = ns++;
      cp_async8(slot + s_en[K][J] * kPlainThreads, a.E.f[K] + c + str[J]);
    }
  }
#pragma unroll
  for (int I = 0; I < 3; I++)
    if (hasH(MODE, I)) {
      s_b[I] = ns++;
      cp_async8(slot + s_b[I] * kPlainThreads, a.B.f[I] + c);
    }
  long long pidx[3] = {-1, -1, -1};
#pragma unroll
  for (int J = 0; J < 3; J++) {
    const int s = a.pml_axis[J] ? slab_index(a.slab[J], idx[J]) : -1;
    if (s >= 0) {
      if (J == 0) pidx[J] = (static_cast<long long>(k) * a.ny + j) * a.slab[0].W + s;
      else if (J == 1) pidx[J] = (static_cast<long long>(k) * a.slab[1].W + s) * a.nx + i;
      else pidx[J] = (static_cast<long long>(s) * a.ny + j) * a.nx + i;
    }
#pragma unroll
    for (int I = 0; I < 3; I++) {
      if (!hasH(MODE, I) || I == J || (MODE != kThreeD && J == 2)) continue;
      s_ps[I][J] = ns++;
      if (pidx[J] >= 0) cp_async8(slot + s_ps[I][J] * kPlainThreads, a.psi[1][I][J] + pidx[J]);
    }
  }
  double h0[3] = {}, h1[3] = {}, h2[3] = {};
#pragma unroll
  for (int I = 0; I < 3; I++) {
    if (!hasH(MODE, I)) continue;
    if (HIST) {
      h0[I] = a.hist[1][0][I][c];
      h1[I] = a.hist[1][1][I][c];
      if (a.bd == 3) h2[I] = a.hist[1][2][I][c];
    }
  }
  int mid = 0;
  if (a.ids) mid = a.ids[c];
  else if (a.bids) mid = a.bids[((k >> a.bshift) * a.nby + (j >> a.bshift)) * a.nbx + (i >> a.bshift)];
  cp_async_wait_all();
  double ec[3] = {0.0, 0.0, 0.0}, en[3][3] = {}, b[3] = {0.0, 0.0, 0.0}, ps[3][3] = {};
#pragma unroll
  for (int K = 0; K < 3; K++)
    if (hasE(MODE, K)) ec[K] = slot[s_ec[K] * kPlainThreads];
#pragma unroll
  for (int K = 0; K < 3; K++)
#pragma unroll
    for (int J = 0; J < 3; J++)
      if (J != K && hasE(MODE, K)) {
        const int I = third(J, K);
        if (hasH(MODE, I)) en[K][J] = slot[s_en[K][J] * kPlainThreads];
      }
#pragma unroll
  for (int I = 0; I < 3; I++)
    if (hasH(MODE, I)) b[I] = slot[s_b[I] * kPlainThreads];
#pragma unroll
  for (int J = 0; J < 3; J++)
#pragma unroll
    for (int I = 0; I < 3; I++)
      if (hasH(MODE, I) && I != J && !(MODE != kThreeD && J == 2) && pidx[J] >= 0)
        ps[I][J] = slot[s_ps[I][J] * kPlainThreads];

  // ---- YeeUpdate<Mode, B_I, TimePolicy>: a = LC*F/dx*(E_K[+J] - E_K)
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
      const double diff = en[K][J] - ec[K];
      const double fdx = a.prof[1][J].F[idx[J]];
      at[q] = (levi(I, J, K) == 1 ? fdx : -fdx) * diff;
    }
    const double old = b[I], sdt = -a.cc * dt, curl = at[0] + at[1];
    if (!HIST) {
      b[I] = old + sdt * curl;
    } else if (a.bd == 2) {
      const double get = a.bdk[0] * old + a.bdk[1] * h0[I] - a.bdk[2] * h1[I];
      b[I] = get + sdt * curl;
      h1[I] = h0[I];
      h0[I] = old;
    } else {
      const double get = a.bdk[0] * old + a.bdk[1] * h0[I] - a.bdk[2] * h1[I] + a.bdk[3] * h2[I];
      b[I] = get + sdt * curl;
      h2[I] = h1[I];
      h1[I] = h0[I];
      h0[I] = old;
    }
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
      b[I] += -a.cc * dt * tfsf_term<MODE>(p, ax, row, 1, I, idx, a.prof, a.dx);
    }
  }
  // SoftSource on B
  for (int s = 0; s < a.nsrc; s++) {
    const SourceDev& sr = a.src[s];
    if (sr.target != 3 || sr.cell != c) continue;
    const double v = t < sr.nvals ? sr.vals[t] : 0.0;
#pragma unroll
    for (int I = 0; I < 3; I++)
      if (sr.comp == I) b[I] += v;
  }
  // UpdatePML<Mode, Magnetic, J>
#pragma unroll
  for (int J = 0; J < 3; J++) {
    if (pidx[J] < 0) continue;
    const double B = a.prof[1][J].B[idx[J]];
    const double Cdx = a.prof[1][J].C[idx[J]];
    const double G = a.prof[1][J].G[idx[J]];
#pragma unroll
    for (int I = 2; I >= 0; I--) {
      if (!hasH(MODE, I) || I == J) continue;
      const int K = third(I, J);
      const double psi = ps[I][J];
      b[I] += -dt * psi * G;
      const double diff = en[K][J] - ec[K];
      ps[I][J] = B * psi + (levi(I, J, K) == 1 ? Cdx : -Cdx) * diff;
    }
  }
  // VacuumUpdate / ConstantUpdate<Mode, Magnetic>: H = B/(mu_r*mu0)
  const double den = a.mats[mid].den_h;
  double h[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int I = 2; I >= 0; I--) {
    if (!hasH(MODE, I)) continue;
    h[I] = b[I] / den;
  }
  // SoftSource on H
  for (int s = 0; s < a.nsrc; s++) {
    const SourceDev& sr = a.src[s];
    if (sr.target != 2 || sr.cell != c) continue;
    const double v = t < sr.nvals ? sr.vals[t] : 0.0;
#pragma unroll
    for (int I = 0; I < 3; I++)
      if (sr.comp == I) h[I] += v;
  }

  // ---- every write of the cell
#pragma unroll
  for (int I = 0; I < 3; I++) {
    if (!hasH(MODE, I)) continue;
    a.B.f[I][c] = b[I];
    a.H.f[I][c] = h[I];
    if (HIST) {
      a.hist[1][0][I][c] = h0[I];
      a.hist[1][1][I][c] = h1[I];
      if (a.bd == 3) a.hist[1][2][I][c] = h2[I];
    }
  }
#pragma unroll
  for (int J = 0; J < 3; J++) {
    if (pidx[J] < 0) continue;
#pragma unroll
    for (int I = 0; I < 3; I++)
      if (hasH(MODE, I) && I != J) a.psi[1][I][J][pidx[J]] = ps[I][J];
  }
}

// the shared-memory carveout that holds the two CTAs per SM that the
// kernels' registers allow (plus the 1 KB the runtime reserves per CTA); the
// rest of the SM's memory stays L1, which serves the neighbour reads
static int plain_carveout(size_t smem) {
  int dev = 0, max_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&max_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
  if (max_sm <= 0) return cudaSharedmemCarveoutMaxShared;
  const size_t need = 2 * (smem + 1024);
  return static_cast<int>(need * 100 / max_sm + 1 > 100 ? 100 : need * 100 / max_sm + 1);
}

template <class F>
static void plain_launch(F fn, size_t smem, const dim3& grid, const dim3& block, const PlainArgs& a,
                         cudaStream_t s) {
  once_per_device(reinterpret_cast<const void*>(fn), [&] {
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, plain_carveout(smem));
  });
  fn<<<grid, block, smem, s>>>(a);
}

template <int MODE>
static int launch_plain(const PlainArgs& a, cudaStream_t s, bool e) {
  dim3 block(32, kPlainThreads / 32, 1);
  dim3 grid((a.nx - 2 + 31) / 32, (a.ny - 2 + block.y - 1) / block.y, MODE == kThreeD ? a.nz - 2 : 1);
  constexpr size_t sh = plain_h_slots(MODE) * kPlainThreads * sizeof(double);
  constexpr size_t s0 = plain_e_slots(MODE, 0) * kPlainThreads * sizeof(double);
  constexpr size_t s1 = plain_e_slots(MODE, 1) * kPlainThreads * sizeof(double);
  constexpr size_t s2 = plain_e_slots(MODE, 2) * kPlainThreads * sizeof(double);
  if (!e) {
    if (a.bd) plain_launch(plain_h_kernel<MODE, true>, sh, grid, block, a, s);
    else plain_launch(plain_h_kernel<MODE, false>, sh, grid, block, a, s);
  } else if (a.bd) {
    plain_launch(plain_e_kernel<MODE, 0, true>, s0, grid, block, a, s);
  } else if (a.all_dispersive && a.dispersive == 1) {
    plain_launch(plain_e_kernel<MODE, 1, false>, s1, grid, block, a, s);
  } else if (a.all_dispersive && a.dispersive == 2) {
    plain_launch(plain_e_kernel<MODE, 2, false>, s2, grid, block, a, s);
  } else {
    plain_launch(plain_e_kernel<MODE, 0, false>, s0, grid, block, a, s);
  }
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
