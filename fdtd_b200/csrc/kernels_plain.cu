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
__device__ __forceinline__ double tfsf_term(const PlaneDev& p, const AuxTab& aux, long long row, int ft, int I,
                                            const int (&idx)[3],
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

// a cell's index within a TFSF plane's box, x fastest
__device__ __forceinline__ long long plane_cell(const PlaneDev& p, int i, int j, int k) {
  const long long ex = p.hi[0] - p.lo[0] + 1, ey = p.hi[1] - p.lo[1] + 1;
  return (static_cast<long long>(k - p.lo[2]) * ey + (j - p.lo[1])) * ex + (i - p.lo[0]);
}

// The TFSF corrections of half step ft for every cell of every plane:
// ft 0 (cc*dt) * TFSFPlane::updateD's term, ft 1 (-cc*dt) * updateB's term,
// the expressions the sweeps used to form per cell, in the same operation
// order (this file is compiled without FMA contraction). Formed here in one
// coalesced launch instead of by the one lane of each warp that holds an
// x-normal face cell while the rest of the warp waits. Grid: x over a
// plane's lower in-plane axis (128 cells per CTA), y over its other
// in-plane axis, z over the planes.
template <int MODE>
__global__ void __launch_bounds__(128) tfsf_pre_kernel(const __grid_constant__ PlainArgs a, int ft) {
  const PlaneDev& p = a.planes[blockIdx.z];
  const int u = p.axis == 0 ? 1 : 0, v = p.axis == 2 ? 1 : 2;
  const int uu = blockIdx.x * blockDim.x + threadIdx.x, vv = blockIdx.y;
  if (p.lo[u] + uu > p.hi[u] || p.lo[v] + vv > p.hi[v]) return;
  int idx[3];
  idx[u] = p.lo[u] + uu;
  idx[v] = p.lo[v] + vv;
  const AuxTab& ax = a.aux[p.aux];
  const long long row = a.ctrl->t - a.ctrl->t0 + ft;
  const double dt = a.dt;
  for (int w = p.lo[p.axis]; w <= p.hi[p.axis]; w++) {
    idx[p.axis] = w;
    double* out = a.tfsf_pre + 3 * (p.off + plane_cell(p, idx[0], idx[1], idx[2]));
#pragma unroll
    for (int I = 2; I >= 0; I--) {
      if (ft == 0 ? !hasE(MODE, I) : !hasH(MODE, I)) continue;
      out[I] = ft == 0 ? a.cc * dt * tfsf_term<MODE>(p, ax, row, 0, I, idx, a.prof, a.dx)
                       : -a.cc * dt * tfsf_term<MODE>(p, ax, row, 1, I, idx, a.prof, a.dx);
    }
  }
}

int launch_tfsf_pre(int mode, const PlainArgs& a, int ft, cudaStream_t s) {
  if (a.nplanes == 0) return 0;
  int most_u = 1, most_v = 1;
  for (int q = 0; q < a.nplanes; q++) {
    const PlaneDev& p = a.planes[q];
    const int u = p.axis == 0 ? 1 : 0, v = p.axis == 2 ? 1 : 2;
    most_u = most_u > p.hi[u] - p.lo[u] + 1 ? most_u : p.hi[u] - p.lo[u] + 1;
    most_v = most_v > p.hi[v] - p.lo[v] + 1 ? most_v : p.hi[v] - p.lo[v] + 1;
  }
  const dim3 grid(static_cast<unsigned>((most_u + 127) / 128), static_cast<unsigned>(most_v), a.nplanes);
  switch (mode) {
    case kTE: tfsf_pre_kernel<kTE><<<grid, 128, 0, s>>>(a, ft); break;
    case kTM: tfsf_pre_kernel<kTM><<<grid, 128, 0, s>>>(a, ft); break;
    default: tfsf_pre_kernel<kThreeD><<<grid, 128, 0, s>>>(a, ft); break;
  }
  return 1;
}

constexpr int kPlainThreads = 256;  // 32 x 8 cells per CTA (two-pole E sweep: 32 x 4)

// f[comp] += v with comp known only at run time, as selects: indexing the
// array with comp would put it (a cell's whole D, E, B or H) in local memory
__device__ __forceinline__ void add_to_component(double (&f)[3], int comp, double v) {
#pragma unroll
  for (int I = 0; I < 3; I++) {
    const double sum = f[I] + v;
    f[I] = comp == I ? sum : f[I];
  }
}

__device__ __forceinline__ void cp_async8(double* dst, const double* src) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(src) : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }

template <int N>
__device__ __forceinline__ void cp_async_wait_group() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Shared-memory slots (one double per thread each) of the plain kernels,
// numbered once for the copies and the reads: E half: H at the cell and at
// its curl neighbours, D, the CPML integrators and P, J of NP poles; H half:
// E at the cell and its neighbours, B and the integrators.
struct PlainSlots {
  int own[3];     // H (E half) or E (H half) at the cell
  int nb[3][3];   // [K][J]: component K at the neighbour along J
  int flux[3];    // D or B
  int psi[3][3];  // [I][J]
  int p[2][3], j[2][3];
  int n;
};

__host__ __device__ constexpr PlainSlots plain_slots(int mode, int ft, int np) {
  PlainSlots s{};
  int n = 0;
  // ft 0: the E half (fluxes of E, curl of H); 1: the H half
  for (int K = 0; K < 3; K++)
    if (ft == 0 ? hasH(mode, K) : hasE(mode, K)) s.own[K] = n++;
  for (int I = 0; I < 3; I++)
    for (int J = 0; J < 3; J++) {
      if (I == J || !(ft == 0 ? hasE(mode, I) : hasH(mode, I))) continue;
      const int K = third(I, J);
      if (ft == 0 ? hasH(mode, K) : hasE(mode, K)) s.nb[K][J] = n++;
    }
  for (int I = 0; I < 3; I++)
    if (ft == 0 ? hasE(mode, I) : hasH(mode, I)) s.flux[I] = n++;
  for (int J = 0; J < 3; J++)
    for (int I = 0; I < 3; I++)
      if ((ft == 0 ? hasE(mode, I) : hasH(mode, I)) && I != J && !(mode != kThreeD && J == 2)) s.psi[I][J] = n++;
  for (int q = 0; q < np; q++)
    for (int I = 0; I < 3; I++)
      if (hasE(mode, I)) {
        s.p[q][I] = n++;
        s.j[q][I] = n++;
      }
  s.n = n;
  return s;
}

// Each thread takes ZC cells along z (planes k0 .. k0 + ZC - 1 of its (i, j)):
// it requests every operand of all of them -- the H (E) values of the curl,
// the flux, the CPML integrators and, with every material dispersive, P and
// J -- with cp.async into its own shared-memory slots (copies in flight hold
// no registers), then, cell by cell, reads them back, applies the passes
// above to registers in the reference's order and stores the results. The
// arrays may alias as far as the compiler knows, so reading each pass's
// operands after the previous pass's stores would make a cell wait for one
// memory round trip per pass; here all the reads of ZC cells are in flight
// together. The arithmetic, and so every result, is the same.
//
// NP: poles of P and J read with the fields (0: read after the material id,
// for the cells whose material has poles). HIST: the BD3/BD4 time policy's
// flux history is read and moved (a separate instantiation, so that the
// leapfrog's kernels keep their registers).

// What a cell reads besides its staged operands, loaded before the wait for
// the copies so that these loads are in flight with them: the step count,
// the cell's material id and eps-map value, and the curl's F profile values.
struct PlainPre {
  long long t;
  int mid;
  double eps_cell;
  double fdx[3];
  unsigned planes, srcs;  // the TFSF planes and sources whose boxes meet the CTA's cells
};

// The TFSF planes and soft sources that can touch the cells of this CTA
// (columns i0..i0+31, rows j0..j1, planes k0..k1): the same for every
// thread of the CTA, so the per-cell loops over them are uniform and skip
// the planes and sources elsewhere in the grid.
__device__ __forceinline__ void plain_masks(const PlainArgs& a, int i0, int j0, int j1, int k0, int k1,
                                            PlainPre& r) {
  const int i1 = i0 + 31;
  r.planes = 0;
  for (int q = 0; q < a.nplanes; q++) {
    const PlaneDev& p = a.planes[q];
    if (p.lo[0] <= i1 && p.hi[0] >= i0 && p.lo[1] <= j1 && p.hi[1] >= j0 && p.lo[2] <= k1 && p.hi[2] >= k0)
      r.planes |= 1u << q;
  }
  r.srcs = 0;
  for (int q = 0; q < a.nsrc; q++) {
    const SourceDev& sr = a.src[q];
    if (sr.i >= i0 && sr.i <= i1 && sr.j >= j0 && sr.j <= j1 && sr.k >= k0 && sr.k <= k1) r.srcs |= 1u << q;
  }
}

// the per-cell part of it for plane k; t and the x and y profile values
// come from `base` (the same for every plane of the thread's column)
template <int MODE>
__device__ __forceinline__ PlainPre plain_pre_at(const PlainArgs& a, int ft, int i, int j, int k, long long c,
                                                 const PlainPre& base) {
  PlainPre r;
  r.t = base.t;
  r.mid = 0;
  // the H half reads a cell's material only for its mu_r; a table of one
  // material needs no id at all
  const bool any = ft == 0 ? !a.single_mat : !a.uniform_mu;
  if (any && a.ids) r.mid = a.ids[c];
  else if (any && a.bids) r.mid = a.bids[((k >> a.bshift) * a.nby + (j >> a.bshift)) * a.nbx + (i >> a.bshift)];
  r.eps_cell = (ft == 0 && a.eps_map) ? a.eps_map[c] : 0.0;
  r.fdx[0] = base.fdx[0];
  r.fdx[1] = base.fdx[1];
  r.fdx[2] = MODE != kThreeD ? 1.0 : a.prof[ft][2].F[k];
  r.planes = base.planes;
  r.srcs = base.srcs;
  return r;
}

template <int MODE>
__device__ __forceinline__ PlainPre plain_pre(const PlainArgs& a, int ft, int i, int j, int k, long long c, int nz) {
  PlainPre base;
  base.t = a.ctrl->t;
  base.fdx[0] = a.prof[ft][0].F[i];
  base.fdx[1] = a.prof[ft][1].F[j];
  const int j0 = blockIdx.y * blockDim.y + 1;
  plain_masks(a, blockIdx.x * 32 + 1, j0, j0 + blockDim.y - 1, k, k + nz - 1, base);
  return plain_pre_at<MODE>(a, ft, i, j, k, c, base);
}

// the copies of one cell of the E half; sets the CPML integrator indices
template <int MODE, int NP, int T>
__device__ __forceinline__ void plain_e_stage(const PlainArgs& a, int i, int j, int k, double* slot,
                                              long long (&pidx)[3]) {
  constexpr PlainSlots S = plain_slots(MODE, 0, NP);
  const long long sy = a.nx, sz = static_cast<long long>(a.nx) * a.ny;
  const long long c = k * sz + j * sy + i;
  const long long str[3] = {1, sy, sz};
  const int idx[3] = {i, j, k};
#pragma unroll
  for (int K = 0; K < 3; K++)
    if (hasH(MODE, K)) cp_async8(slot + S.own[K] * T, a.H.f[K] + c);
#pragma unroll
  for (int I = 0; I < 3; I++) {
    if (!hasE(MODE, I)) continue;
#pragma unroll
    for (int J = 0; J < 3; J++) {
      if (J == I) continue;
      const int K = third(I, J);
      if (hasH(MODE, K)) cp_async8(slot + S.nb[K][J] * T, a.H.f[K] + c - str[J]);
    }
  }
#pragma unroll
  for (int I = 0; I < 3; I++)
    if (hasE(MODE, I)) cp_async8(slot + S.flux[I] * T, a.D.f[I] + c);
#pragma unroll
  for (int J = 0; J < 3; J++) {
    pidx[J] = -1;
    const int s = a.pml_axis[J] ? slab_index(a.slab[J], idx[J]) : -1;
    if (s < 0) continue;
    if (J == 0) pidx[J] = (static_cast<long long>(k) * a.ny + j) * a.slab[0].W + s;
    else if (J == 1) pidx[J] = (static_cast<long long>(k) * a.slab[1].W + s) * a.nx + i;
    else pidx[J] = (static_cast<long long>(s) * a.ny + j) * a.nx + i;
#pragma unroll
    for (int I = 0; I < 3; I++)
      if (hasE(MODE, I) && I != J && !(MODE != kThreeD && J == 2))
        cp_async8(slot + S.psi[I][J] * T, a.psi[0][I][J] + pidx[J]);
  }
#pragma unroll
  for (int q = 0; q < NP; q++)
#pragma unroll
    for (int I = 0; I < 3; I++)
      if (hasE(MODE, I) && q < a.dispersive) {
        cp_async8(slot + S.p[q][I] * T, a.P[q].f[I] + c);
        cp_async8(slot + S.j[q][I] * T, a.J[q].f[I] + c);
      }
}

// the reference's E half of one cell from its slots
template <int MODE, int NP, bool HIST, int T>
__device__ __forceinline__ void plain_e_cell(const PlainArgs& a, int i, int j, int k, const double* slot,
                                             const long long (&pidx)[3], const PlainPre& pre) {
  constexpr PlainSlots S = plain_slots(MODE, 0, NP);
  constexpr int NPS = NP > 0 ? NP : 1;
  const long long sy = a.nx, sz = static_cast<long long>(a.nx) * a.ny;
  const long long c = k * sz + j * sy + i;
  const int idx[3] = {i, j, k};
  const double dt = a.dt;
  const long long t = pre.t;
  double h0[3] = {}, h1[3] = {}, h2[3] = {};
#pragma unroll
  for (int I = 0; I < 3; I++) {
    if (!hasE(MODE, I) || !HIST) continue;
    h0[I] = a.hist[0][0][I][c];
    h1[I] = a.hist[0][1][I][c];
    if (a.bd == 3) h2[I] = a.hist[0][2][I][c];
  }
  const int mid = pre.mid;
  const double eps_cell = pre.eps_cell;
  double hc[3] = {0.0, 0.0, 0.0}, hn[3][3] = {}, d[3] = {0.0, 0.0, 0.0}, ps[3][3] = {};
  double pp[NPS][3] = {}, jj[NPS][3] = {};
#pragma unroll
  for (int K = 0; K < 3; K++)
    if (hasH(MODE, K)) hc[K] = slot[S.own[K] * T];
#pragma unroll
  for (int K = 0; K < 3; K++)
#pragma unroll
    for (int J = 0; J < 3; J++)
      if (J != K && hasH(MODE, K) && hasE(MODE, third(J, K))) hn[K][J] = slot[S.nb[K][J] * T];
#pragma unroll
  for (int I = 0; I < 3; I++)
    if (hasE(MODE, I)) d[I] = slot[S.flux[I] * T];
#pragma unroll
  for (int J = 0; J < 3; J++)
#pragma unroll
    for (int I = 0; I < 3; I++)
      if (hasE(MODE, I) && I != J && !(MODE != kThreeD && J == 2) && pidx[J] >= 0)
        ps[I][J] = slot[S.psi[I][J] * T];
#pragma unroll
  for (int q = 0; q < NP; q++)
#pragma unroll
    for (int I = 0; I < 3; I++)
      if (hasE(MODE, I) && q < a.dispersive) {
        pp[q][I] = slot[S.p[q][I] * T];
        jj[q][I] = slot[S.j[q][I] * T];
      }

  // YeeUpdate<Mode, D_I, TimePolicy>: a = LC*F/dx*(H_K - H_K[-J]), then
  // F = TimePolicy::get(F) + (Coeff*curl_coeff*dt) * curl and the history
  // moves on (YeeUpdates.hpp:182-294, :396-405)
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
      const double fdx = pre.fdx[J];
      at[q] = (levi(I, J, K) == 1 ? fdx : -fdx) * diff;
    }
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
  // TFSFPlane::updateD: the corrections formed for this half step by
  // tfsf_pre_kernel, added in plane order
  for (unsigned mq = pre.planes; mq; mq &= mq - 1) {
    const int q = __ffs(mq) - 1;
    const PlaneDev& p = a.planes[q];
    if (i < p.lo[0] || i > p.hi[0] || j < p.lo[1] || j > p.hi[1] || k < p.lo[2] || k > p.hi[2]) continue;
    const double* v = a.tfsf_pre + 3 * (p.off + plane_cell(p, i, j, k));
#pragma unroll
    for (int I = 2; I >= 0; I--) {
      if (!hasE(MODE, I)) continue;
      d[I] += v[I];
    }
  }
  // SoftSource on D
  for (unsigned ms = pre.srcs; ms; ms &= ms - 1) {
    const SourceDev& sr = a.src[__ffs(ms) - 1];
    if (sr.target != 1 || sr.cell != c) continue;
    const double v = t < sr.nvals ? sr.vals[t] : 0.0;
    add_to_component(d, sr.comp, v);
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
  // material update; the row's scalars are read once, into registers (the
  // table may alias the stored arrays as far as the compiler knows, so a
  // member read after a store would be read again)
  const MatF64& m = a.mats[mid];
  const int mkind = m.kind, mnp = m.npoles;
  const double mden = m.den_e;
  double mc1[NPS], mc2[NPS], mc3[NPS];
#pragma unroll
  for (int q = 0; q < NPS; q++) {
    const bool used = q == 0 ? mkind >= 2 : (NP > 0 && mkind == 3);
    mc1[q] = used ? m.c1[q] : 0.0;
    mc2[q] = used ? m.c2[q] : 0.0;
    mc3[q] = used ? m.c3[q] : 0.0;
  }
  if (NP == 0 && mkind >= 2) {
#pragma unroll
    for (int I = 0; I < 3; I++)
      if (hasE(MODE, I)) {
        pp[0][I] = a.P[0].f[I][c];
        jj[0][I] = a.J[0].f[I][c];
      }
  }
  double e[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int I = 2; I >= 0; I--) {
    if (!hasE(MODE, I)) continue;
    const double D = d[I];
    if (mkind <= 1) {
      // a per-cell permittivity replaces the ConstantUpdate K of the cell
      const double den = (a.eps_map && eps_cell > 0.0) ? eps_cell * kEps0 : mden;
      e[I] = D / den;
    } else if (mkind == 2) {
      // drude::DrudeUpdate::implicit_update (DispersiveMaterials.hpp:979-998)
      double P = pp[0][I], Jc = jj[0][I];
      P += dt * Jc;
      const double E = (D - P) / mden;
      Jc = Jc * mc1[0] / mc2[0] + mc3[0] * E;
      pp[0][I] = P;
      jj[0][I] = Jc;
      e[I] = E;
    } else if (NP > 0 && mnp <= NP) {
      // lorentz::LorentzUpdate::implicit_update (DispersiveMaterials.hpp:710-735),
      // one term per pole, on the staged poles
      double num = D;
      double P[NPS];
#pragma unroll
      for (int q = 0; q < NPS; q++) {
        if (q >= mnp) continue;
        P[q] = pp[q][I] + dt * jj[q][I];
        pp[q][I] = P[q];
        num = num - P[q];
      }
      const double E = num / mden;
#pragma unroll
      for (int q = 0; q < NPS; q++) {
        if (q >= mnp) continue;
        jj[q][I] = mc1[q] * jj[q][I] + mc2[q] * E - mc3[q] * P[q];
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
  for (unsigned ms = pre.srcs; ms; ms &= ms - 1) {
    const SourceDev& sr = a.src[__ffs(ms) - 1];
    if (sr.target != 0 || sr.cell != c) continue;
    const double v = t < sr.nvals ? sr.vals[t] : 0.0;
    add_to_component(e, sr.comp, v);
  }
  // every write of the cell
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
  const bool staged = NP > 0 ? (mkind == 2 || mnp <= NP) : mkind == 2;
  if (mkind >= 2 && staged) {
    const int np = mkind == 2 ? 1 : mnp;
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

template <int MODE, int NP, bool HIST, int ZC, int T>
__global__ void __launch_bounds__(T, T == 256 ? 2 : 3) plain_e_kernel(const __grid_constant__ PlainArgs a) {
  extern __shared__ double smd[];
  constexpr int NS = plain_slots(MODE, 0, NP).n;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int k0 = MODE == kThreeD ? a.kbeg + blockIdx.z * ZC : 0;
  if (i > a.nx - 2 || j > a.ny - 2) return;
  const long long sz = static_cast<long long>(a.nx) * a.ny, cij = static_cast<long long>(j) * a.nx + i;
  const int nz = MODE == kThreeD ? min(ZC, a.kend - k0) : 1;
  long long pc[3], pn[3];
  plain_e_stage<MODE, NP, T>(a, i, j, k0, smd + tid, pc);
  PlainPre rc = plain_pre<MODE>(a, 0, i, j, k0, k0 * sz + cij, nz), rn = rc;
  cp_async_commit();
#pragma unroll 1
  for (int z = 0; z < nz; z++) {
    double* cur = smd + tid + (z & 1) * NS * T;
    if (z + 1 < nz) {
      plain_e_stage<MODE, NP, T>(a, i, j, k0 + z + 1, smd + tid + ((z & 1) ^ 1) * NS * T, pn);
      rn = plain_pre_at<MODE>(a, 0, i, j, k0 + z + 1, (k0 + z + 1) * sz + cij, rc);
      cp_async_commit();
      cp_async_wait_group<1>();
    } else {
      cp_async_wait_group<0>();
    }
    plain_e_cell<MODE, NP, HIST, T>(a, i, j, k0 + z, cur, pc, rc);
#pragma unroll
    for (int J = 0; J < 3; J++) pc[J] = pn[J];
    rc = rn;
  }
}

// the copies of one cell of the H half
template <int MODE, int T>
__device__ __forceinline__ void plain_h_stage(const PlainArgs& a, int i, int j, int k, double* slot,
                                              long long (&pidx)[3]) {
  constexpr PlainSlots S = plain_slots(MODE, 1, 0);
  const long long sy = a.nx, sz = static_cast<long long>(a.nx) * a.ny;
  const long long c = k * sz + j * sy + i;
  const long long str[3] = {1, sy, sz};
  const int idx[3] = {i, j, k};
#pragma unroll
  for (int K = 0; K < 3; K++)
    if (hasE(MODE, K)) cp_async8(slot + S.own[K] * T, a.E.f[K] + c);
#pragma unroll
  for (int I = 0; I < 3; I++) {
    if (!hasH(MODE, I)) continue;
#pragma unroll
    for (int J = 0; J < 3; J++) {
      if (J == I) continue;
      const int K = third(I, J);
      if (hasE(MODE, K)) cp_async8(slot + S.nb[K][J] * T, a.E.f[K] + c + str[J]);
    }
  }
#pragma unroll
  for (int I = 0; I < 3; I++)
    if (hasH(MODE, I)) cp_async8(slot + S.flux[I] * T, a.B.f[I] + c);
#pragma unroll
  for (int J = 0; J < 3; J++) {
    pidx[J] = -1;
    const int s = a.pml_axis[J] ? slab_index(a.slab[J], idx[J]) : -1;
    if (s < 0) continue;
    if (J == 0) pidx[J] = (static_cast<long long>(k) * a.ny + j) * a.slab[0].W + s;
    else if (J == 1) pidx[J] = (static_cast<long long>(k) * a.slab[1].W + s) * a.nx + i;
    else pidx[J] = (static_cast<long long>(s) * a.ny + j) * a.nx + i;
#pragma unroll
    for (int I = 0; I < 3; I++)
      if (hasH(MODE, I) && I != J && !(MODE != kThreeD && J == 2))
        cp_async8(slot + S.psi[I][J] * T, a.psi[1][I][J] + pidx[J]);
  }
}

// the reference's H half of one cell from its slots
template <int MODE, bool HIST, int T>
__device__ __forceinline__ void plain_h_cell(const PlainArgs& a, int i, int j, int k, const double* slot,
                                             const long long (&pidx)[3], const PlainPre& pre) {
  constexpr PlainSlots S = plain_slots(MODE, 1, 0);
  const long long sy = a.nx, sz = static_cast<long long>(a.nx) * a.ny;
  const long long c = k * sz + j * sy + i;
  const int idx[3] = {i, j, k};
  const double dt = a.dt;
  const long long t = pre.t;
  double h0[3] = {}, h1[3] = {}, h2[3] = {};
#pragma unroll
  for (int I = 0; I < 3; I++) {
    if (!hasH(MODE, I) || !HIST) continue;
    h0[I] = a.hist[1][0][I][c];
    h1[I] = a.hist[1][1][I][c];
    if (a.bd == 3) h2[I] = a.hist[1][2][I][c];
  }
  const int mid = pre.mid;
  double ec[3] = {0.0, 0.0, 0.0}, en[3][3] = {}, b[3] = {0.0, 0.0, 0.0}, ps[3][3] = {};
#pragma unroll
  for (int K = 0; K < 3; K++)
    if (hasE(MODE, K)) ec[K] = slot[S.own[K] * T];
#pragma unroll
  for (int K = 0; K < 3; K++)
#pragma unroll
    for (int J = 0; J < 3; J++)
      if (J != K && hasE(MODE, K) && hasH(MODE, third(J, K))) en[K][J] = slot[S.nb[K][J] * T];
#pragma unroll
  for (int I = 0; I < 3; I++)
    if (hasH(MODE, I)) b[I] = slot[S.flux[I] * T];
#pragma unroll
  for (int J = 0; J < 3; J++)
#pragma unroll
    for (int I = 0; I < 3; I++)
      if (hasH(MODE, I) && I != J && !(MODE != kThreeD && J == 2) && pidx[J] >= 0)
        ps[I][J] = slot[S.psi[I][J] * T];

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
      const double diff = en[K][J] - ec[K];
      const double fdx = pre.fdx[J];
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
  // TFSFPlane::updateB (the aux grid was advanced by updateD: row + 1), as
  // formed by tfsf_pre_kernel
  for (unsigned mq = pre.planes; mq; mq &= mq - 1) {
    const int q = __ffs(mq) - 1;
    const PlaneDev& p = a.planes[q];
    if (i < p.lo[0] || i > p.hi[0] || j < p.lo[1] || j > p.hi[1] || k < p.lo[2] || k > p.hi[2]) continue;
    const double* v = a.tfsf_pre + 3 * (p.off + plane_cell(p, i, j, k));
#pragma unroll
    for (int I = 2; I >= 0; I--) {
      if (!hasH(MODE, I)) continue;
      b[I] += v[I];
    }
  }
  // SoftSource on B
  for (unsigned ms = pre.srcs; ms; ms &= ms - 1) {
    const SourceDev& sr = a.src[__ffs(ms) - 1];
    if (sr.target != 3 || sr.cell != c) continue;
    const double v = t < sr.nvals ? sr.vals[t] : 0.0;
    add_to_component(b, sr.comp, v);
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
  for (unsigned ms = pre.srcs; ms; ms &= ms - 1) {
    const SourceDev& sr = a.src[__ffs(ms) - 1];
    if (sr.target != 2 || sr.cell != c) continue;
    const double v = t < sr.nvals ? sr.vals[t] : 0.0;
    add_to_component(h, sr.comp, v);
  }
  // every write of the cell
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

template <int MODE, bool HIST, int ZC, int T>
__global__ void __launch_bounds__(T, T == 256 ? 2 : 3) plain_h_kernel(const __grid_constant__ PlainArgs a) {
  extern __shared__ double smd[];
  constexpr int NS = plain_slots(MODE, 1, 0).n;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int k0 = MODE == kThreeD ? a.kbeg + blockIdx.z * ZC : 0;
  if (i > a.nx - 2 || j > a.ny - 2) return;
  const long long sz = static_cast<long long>(a.nx) * a.ny, cij = static_cast<long long>(j) * a.nx + i;
  const int nz = MODE == kThreeD ? min(ZC, a.kend - k0) : 1;
  long long pc[3], pn[3];
  plain_h_stage<MODE, T>(a, i, j, k0, smd + tid, pc);
  PlainPre rc = plain_pre<MODE>(a, 1, i, j, k0, k0 * sz + cij, nz), rn = rc;
  cp_async_commit();
#pragma unroll 1
  for (int z = 0; z < nz; z++) {
    double* cur = smd + tid + (z & 1) * NS * T;
    if (z + 1 < nz) {
      plain_h_stage<MODE, T>(a, i, j, k0 + z + 1, smd + tid + ((z & 1) ^ 1) * NS * T, pn);
      rn = plain_pre_at<MODE>(a, 1, i, j, k0 + z + 1, (k0 + z + 1) * sz + cij, rc);
      cp_async_commit();
      cp_async_wait_group<1>();
    } else {
      cp_async_wait_group<0>();
    }
    plain_h_cell<MODE, HIST, T>(a, i, j, k0 + z, cur, pc, rc);
#pragma unroll
    for (int J = 0; J < 3; J++) pc[J] = pn[J];
    rc = rn;
  }
}

// the shared-memory carveout that holds the two CTAs per SM that the
// kernels' registers allow (plus the 1 KB the runtime reserves per CTA); the
// rest of the SM's memory stays L1, which serves the neighbour reads (a
// larger carveout slowed the sweeps measurably)
static int plain_carveout(size_t smem, int ctas) {
  int dev = 0, max_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&max_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
  if (max_sm <= 0) return cudaSharedmemCarveoutMaxShared;
  const size_t need = ctas * (smem + 1024);
  return static_cast<int>(need * 100 / max_sm + 1 > 100 ? 100 : need * 100 / max_sm + 1);
}

template <class F>
static void plain_launch(F fn, size_t smem, const dim3& grid, const dim3& block, const PlainArgs& a,
                         cudaStream_t s) {
  const int ctas = block.x * block.y == 256 ? 2 : 3;
  once_per_device(reinterpret_cast<const void*>(fn), [&] {
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, plain_carveout(smem, ctas));
  });
  fn<<<grid, block, smem, s>>>(a);
}

// ZC planes per thread along z (3D): the copies of plane z + 1 go into the
// second set of slots while plane z is computed from the first, so the
// copies of the next cell overlap the FP64 arithmetic of this one (with one
// plane per thread the copies and the arithmetic of a thread alternate, and
// two CTAs per SM cannot fill the gaps). Two-pole grids, whose 30 slots per
// cell doubled would leave one 256-thread CTA per SM, take CTAs of 32 x 4
// threads, three per SM. BD3/BD4 kernels take one plane per thread.
template <int MODE>
static int launch_plain(const PlainArgs& a, cudaStream_t s, bool e) {
  constexpr int ZP = MODE == kThreeD ? 8 : 1;
  constexpr int T2 = MODE == kThreeD ? 128 : kPlainThreads;
  auto grid = [&](int zc, int t) {
    return dim3((a.nx - 2 + 31) / 32, (a.ny - 2 + t / 32 - 1) / (t / 32),
                MODE == kThreeD ? (a.kend - a.kbeg + zc - 1) / zc : 1);
  };
  auto bytes = [](int ft, int np, int zc, int t) {
    return static_cast<size_t>(plain_slots(MODE, ft, np).n) * (zc > 1 ? 2 : 1) * t * sizeof(double);
  };
  constexpr int T = kPlainThreads;
  const dim3 block(32, T / 32, 1), block2(32, T2 / 32, 1);
  if (!e) {
    if (a.bd) plain_launch(plain_h_kernel<MODE, true, 1, T>, bytes(1, 0, 1, T), grid(1, T), block, a, s);
    else plain_launch(plain_h_kernel<MODE, false, ZP, T>, bytes(1, 0, ZP, T), grid(ZP, T), block, a, s);
  } else if (a.bd) {
    plain_launch(plain_e_kernel<MODE, 0, true, 1, T>, bytes(0, 0, 1, T), grid(1, T), block, a, s);
  } else if (a.all_dispersive && a.dispersive == 1) {
    plain_launch(plain_e_kernel<MODE, 1, false, ZP, T>, bytes(0, 1, ZP, T), grid(ZP, T), block, a, s);
  } else if (a.all_dispersive && a.dispersive == 2) {
    plain_launch(plain_e_kernel<MODE, 2, false, ZP, T2>, bytes(0, 2, ZP, T2), grid(ZP, T2), block2, a, s);
  } else {
    plain_launch(plain_e_kernel<MODE, 0, false, ZP, T>, bytes(0, 0, ZP, T), grid(ZP, T), block, a, s);
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
// The forward (explicit) material updates, XUpdate<Mode, ft, forward = true>:
// the flux from the field on every interior cell. Electric: ConstantUpdate
// and VacuumUpdate D = (K*eps0)*E (DispersiveMaterials.hpp:345-349), Drude
// P = (-dt*J + (1+b)*P)/(1+b), J = (J - c*E)/(1+b), D = (K*eps0)*E + P with
// b = gamma*dt and c = ((dt*w)*w)*eps0 (:922-934). Magnetic: B = (mu_r*mu0)*H.
// Components in the order nested_for_each_tuple_type visits them (z, y, x).
template <int MODE>
__global__ void material_explicit_kernel(const __grid_constant__ PlainArgs a, int ft) {
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  const int k = MODE == kThreeD ? 1 + static_cast<int>(blockIdx.z) : 0;
  if (i > a.nx - 2 || j > a.ny - 2) return;
  const long long c = (static_cast<long long>(k) * a.ny + j) * a.nx + i;
  int mid = 0;
  if (a.ids) mid = a.ids[c];
  else if (a.bids) mid = a.bids[((k >> a.bshift) * a.nby + (j >> a.bshift)) * a.nbx + (i >> a.bshift)];
  const MatF64& m = a.mats[mid];
  if (ft == 1) {
#pragma unroll
    for (int I = 2; I >= 0; I--)
      if (hasH(MODE, I)) a.B.f[I][c] = m.den_h * a.H.f[I][c];
    return;
  }
  const double eps_cell = a.eps_map ? a.eps_map[c] : 0.0;
  const double dt = a.dt;
#pragma unroll
  for (int I = 2; I >= 0; I--) {
    if (!hasE(MODE, I)) continue;
    const double E = a.E.f[I][c];
    if (m.kind <= 1) {
      const double den = (a.eps_map && eps_cell > 0.0) ? eps_cell * kEps0 : m.den_e;
      a.D.f[I][c] = den * E;
    } else {
      const double b = m.gamma[0] * dt;
      const double cc = dt * m.freq[0] * m.freq[0] * kEps0;
      const double P = a.P[0].f[I][c], Jc = a.J[0].f[I][c];
      const double Pn = (-dt * Jc + (1.0 + b) * P) / (1.0 + b);
      a.P[0].f[I][c] = Pn;
      a.J[0].f[I][c] = (Jc - cc * E) / (1.0 + b);
      a.D.f[I][c] = m.den_e * E + Pn;
    }
  }
}

int launch_material_explicit(int mode, const PlainArgs& a, int ft, cudaStream_t s) {
  const dim3 block(32, 8, 1);
  const dim3 grid((a.nx - 2 + 31) / 32, (a.ny - 2 + 7) / 8, mode == kThreeD ? a.nz - 2 : 1);
  switch (mode) {
    case kTE: material_explicit_kernel<kTE><<<grid, block, 0, s>>>(a, ft); break;
    case kTM: material_explicit_kernel<kTM><<<grid, block, 0, s>>>(a, ft); break;
    default: material_explicit_kernel<kThreeD><<<grid, block, 0, s>>>(a, ft); break;
  }
  return 1;
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
