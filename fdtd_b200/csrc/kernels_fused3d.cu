// FP32 fused 3D sweeps, vectorised: the update of kernels_fused.cu (same
// equations, same scaled variables) with each thread owning four consecutive
// x cells, so every field access is a 128-bit load or store.
//
// Tile: a warp covers 128 cells along x (array index x4 = 4*lane + 128*bx,
// the outer ring included so rows stay 16-byte aligned), kRows warps cover
// kRows rows along y, and the CTA marches along z over a chunk of planes.
// The next plane's loads are issued before the current plane is computed
// (register double buffering) so each thread keeps ~9 independent 128-bit
// loads in flight. The E sweep marches +z and carries H(k-1); the H sweep
// marches -z and carries E(k+1). x neighbours come from warp shuffles, y
// neighbours from a second 128-bit load of the adjacent row (an L1/L2 hit).
// Ring and padding cells are computed but keep their old value on store.
#include "internal.h"

namespace fdtdb {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kRows = 4;

__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ void st4(float* p, float4 v) { *reinterpret_cast<float4*>(p) = v; }
__device__ __forceinline__ float el(const float4& v, int e) { return e == 0 ? v.x : (e == 1 ? v.y : (e == 2 ? v.z : v.w)); }
__device__ __forceinline__ void set_el(float4& v, int e, float x) {
  if (e == 0) v.x = x;
  else if (e == 1) v.y = x;
  else if (e == 2) v.z = x;
  else v.w = x;
}

__device__ __forceinline__ double interp_row(const double* row, int L, double loc, double dx, double shift) {
  double nd = static_cast<double>(L) / 2.0 + loc / dx - shift;
  unsigned long long n = static_cast<unsigned long long>(nd);
  double frac = nd - static_cast<double>(n);
  return (1.0 - frac) * row[n] + frac * row[n + 1];
}

// TFSF correction of flux I (ft 0 = D, 1 = B): sum_J LeviCivita * F_J/dx *
// n_J * inc_K * pol_K (include/Source.hpp:506-553), in SI flux units per dt.
__device__ double tfsf3(const FusedArgs& a, const PlaneDev& p, long long row, int ft, int I, int i, int j, int k) {
  const AuxTab& aux = a.aux[p.aux];
  const int idx[3] = {i, j, k};
  const int d1 = dir1(I);
  const int ds[2] = {d1, third(I, d1)};
  double sum = 0.0;
  for (int q = 0; q < 2; q++) {
    const int J = ds[q], K = third(I, J);
    if (p.normal[J] == 0.0) continue;
    double proj = 0;
    for (int d = 0; d < 3; d++) {
      const double off = ft == 0 ? (d == K ? -0.5 : 0.0) : (d == K ? 0.0 : -0.5);
      proj += p.k[d] * ((static_cast<double>(idx[d]) - p.origin[d]) * a.dx + off * a.dx);
    }
    const double sv = ft == 0 ? interp_row(aux.Htab + row * aux.L, aux.L, proj, a.dx, 0.5)
                              : interp_row(aux.Etab + row * aux.L, aux.L, proj, a.dx, 0.0);
    const float* Fr = a.prof[ft][J].F + a.flen[J];  // raw F follows the scaled F
    const double* pol = ft == 0 ? p.pol_h : p.pol_e;
    sum += levi(I, J, K) * (static_cast<double>(Fr[idx[J]]) / a.dx) * p.normal[J] * sv * pol[K];
  }
  return sum;
}

__device__ __forceinline__ bool hits_slab(const Slab& s, int lo, int hi) {
  return (s.wlo > 0 && lo <= s.wlo) || (s.W - s.wlo > 0 && hi >= s.hi0);
}

struct EPlane {
  float4 hx, hy, hz, hx_ym, hz_ym, ex, ey, ez;
  unsigned ids;
};
struct HPlane {
  float4 ex, ey, ez, ex_yp, ez_yp, hx, hy, hz;
};

__device__ __forceinline__ float4 sub4(float4 a, float4 b) {
  return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w);
}

// Material update of one E component for the 4 cells of a group: returns the
// new E (plus this step's E-target source values), updating P/J in place.
template <int MAXP>
__device__ __forceinline__ float4 e_comp(const FusedArgs& a, int I, long long c, float4 eo, float4 d, float4 ie,
                                         const bool ok[4], bool disp, bool uniform, const MatF32& m0,
                                         const int mids[4], float4 add) {
  float4 en;
  if (MAXP != 0 && disp) {
    constexpr int NP = MAXP <= 0 ? 1 : MAXP;
    float4 jt[NP], pt[NP];
#pragma unroll
    for (int q = 0; q < NP; q++) {
      jt[q] = ld4(a.J[q][I] + c);
      if (MAXP > 0) pt[q] = ld4(a.P[q][I] + c);
    }
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const MatF32& m = uniform ? m0 : a.mats[mids[e]];
      const int np = m.npoles < 0 ? 1 : m.npoles;
      float js = 0.f;
#pragma unroll
      for (int q = 0; q < NP; q++)
        if (q < np) js += el(jt[q], e);
      const float x = ok[e] ? el(eo, e) + el(ie, e) * (el(d, e) - js) : el(eo, e);
      set_el(en, e, x);
      if (!ok[e]) continue;
#pragma unroll
      for (int q = 0; q < NP; q++) {
        if (q >= np) continue;
        if (MAXP < 0 || m.npoles < 0) {
          set_el(jt[q], e, m.a[q] * el(jt[q], e) + m.b[q] * x);
        } else {
          const float pn = el(pt[q], e) + el(jt[q], e);
          set_el(pt[q], e, pn);
          set_el(jt[q], e, m.a[q] * el(jt[q], e) + m.b[q] * x - m.c[q] * pn);
        }
      }
    }
#pragma unroll
    for (int q = 0; q < NP; q++) {
      st4(a.J[q][I] + c, jt[q]);
      if (MAXP > 0) st4(a.P[q][I] + c, pt[q]);
    }
  } else {
#pragma unroll
    for (int e = 0; e < 4; e++) set_el(en, e, ok[e] ? el(eo, e) + el(ie, e) * el(d, e) : el(eo, e));
  }
  return make_float4(en.x + add.x, en.y + add.y, en.z + add.z, en.w + add.w);
}

}  // namespace

template <int MAXP>
__global__ void __launch_bounds__(32 * kRows) fused3d_e_kernel(const FusedArgs a, int kchunk) {
  const int lane = threadIdx.x;
  const int x4 = blockIdx.x * 128 + lane * 4;
  const int j = 1 + blockIdx.y * kRows + threadIdx.y;
  const int jl = min(j, a.ny - 2);
  const bool row_ok = j <= a.ny - 2;
  const int kbeg = 1 + blockIdx.z * kchunk;
  const int kend = min(kbeg + kchunk, a.nz - 1);
  const long long sy = a.pitch, sz = static_cast<long long>(a.pitch) * a.ny;
  const long long t = a.ctrl->t;
  const int xlo = blockIdx.x * 128, xhi = xlo + 127;
  const int j0 = 1 + blockIdx.y * kRows, j1 = min(j0 + kRows - 1, a.ny - 2);
  const bool pml_x = a.pml_axis[0] && hits_slab(a.slab[0], xlo, xhi);
  const bool pml_y = a.pml_axis[1] && hits_slab(a.slab[1], j0, j1);
  unsigned plane_mask = 0;
  for (int q = 0; q < a.nplanes; q++) {
    const PlaneDev& p = a.planes[q];
    if (p.lo[0] <= xhi && p.hi[0] >= xlo && p.lo[1] <= j1 && p.hi[1] >= j0 && p.lo[2] <= kend - 1 && p.hi[2] >= kbeg)
      plane_mask |= 1u << q;
  }
  bool src_here = false;
  for (int s = 0; s < a.nsrc; s++)
    if (a.src[s].j == j && a.src[s].i >= x4 && a.src[s].i < x4 + 4 && a.src[s].k >= kbeg && a.src[s].k < kend)
      src_here = true;
  const bool uniform_mat = !a.ids && !a.bids;
  const MatF32 m0 = a.mats[0];
  // valid (updated) cells of this thread's group
  bool ok[4];
#pragma unroll
  for (int e = 0; e < 4; e++) ok[e] = row_ok && x4 + e >= 1 && x4 + e <= a.nx - 2;
  const float4 fsx = ld4(a.prof[0][0].F + x4);  // scaled F along x, padded to the pitch
  const float fsy = a.prof[0][1].F[jl];

  auto load = [&](int k, EPlane& P) {
    const long long c = k * sz + jl * sy + x4;
    P.hx = ld4(a.H[0] + c);
    P.hy = ld4(a.H[1] + c);
    P.hz = ld4(a.H[2] + c);
    P.hx_ym = ld4(a.H[0] + c - sy);
    P.hz_ym = ld4(a.H[2] + c - sy);
    P.ex = ld4(a.E[0] + c);
    P.ey = ld4(a.E[1] + c);
    P.ez = ld4(a.E[2] + c);
    if (a.ids) P.ids = *reinterpret_cast<const unsigned*>(a.ids + c);
  };

  float4 hx_km, hy_km;  // H at k-1
  {
    const long long c = (kbeg - 1) * sz + jl * sy + x4;
    hx_km = ld4(a.H[0] + c);
    hy_km = ld4(a.H[1] + c);
  }
  EPlane cur, nxt;
  load(kbeg, cur);
  for (int k = kbeg; k < kend; k++) {
    if (k + 1 < kend) load(k + 1, nxt);
    const long long c = k * sz + jl * sy + x4;
    // x-1 neighbours of Hy, Hz
    float hy_xm0 = __shfl_up_sync(kFull, cur.hy.w, 1);
    float hz_xm0 = __shfl_up_sync(kFull, cur.hz.w, 1);
    if (lane == 0) {
      hy_xm0 = a.H[1][c - 1];
      hz_xm0 = a.H[2][c - 1];
    }
    const float fsz = a.prof[0][2].F[k];
    float4 dX, dY, dZ;  // flux increments (E units)
    float4 rxy, rxz, ryz, ryx, rzx, rzy;
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const float hy_xm = e == 0 ? hy_xm0 : el(cur.hy, e - 1);
      const float hz_xm = e == 0 ? hz_xm0 : el(cur.hz, e - 1);
      set_el(rxy, e, el(cur.hz, e) - el(cur.hz_ym, e));
      set_el(rxz, e, -(el(cur.hy, e) - el(hy_km, e)));
      set_el(ryz, e, el(cur.hx, e) - el(hx_km, e));
      set_el(ryx, e, -(el(cur.hz, e) - hz_xm));
      set_el(rzx, e, el(cur.hy, e) - hy_xm);
      set_el(rzy, e, -(el(cur.hx, e) - el(cur.hx_ym, e)));
      set_el(dX, e, fsy * el(rxy, e) + fsz * el(rxz, e));
      set_el(dY, e, fsz * el(ryz, e) + el(fsx, e) * el(ryx, e));
      set_el(dZ, e, el(fsx, e) * el(rzx, e) + fsy * el(rzy, e));
    }
    hx_km = cur.hx;
    hy_km = cur.hy;
    if (row_ok) {
      // CPML, y and z slabs: psi rows share the field layout (128-bit access)
      const int sjy = pml_y ? slab_index(a.slab[1], j) : -1;
      const int skz = a.pml_axis[2] ? slab_index(a.slab[2], k) : -1;
      if (sjy >= 0) {
        const long long pi = (static_cast<long long>(k) * a.slab[1].W + sjy) * a.pitch + x4;
        const float B = a.prof[0][1].B[j], Cs = a.prof[0][1].C[j], G = a.prof[0][1].G[j];
        float4 px = ld4(a.psi[0][0][1] + pi), pz = ld4(a.psi[0][2][1] + pi);
#pragma unroll
        for (int e = 0; e < 4; e++) {
          set_el(dX, e, el(dX, e) + el(px, e) * G);
          if (!ok[e]) continue;
          set_el(px, e, B * el(px, e) + Cs * el(rxy, e));
          set_el(dZ, e, el(dZ, e) + el(pz, e) * G);
          set_el(pz, e, B * el(pz, e) + Cs * el(rzy, e));
        }
        st4(a.psi[0][0][1] + pi, px);
        st4(a.psi[0][2][1] + pi, pz);
      }
      if (skz >= 0) {
        const long long pi = (static_cast<long long>(skz) * a.ny + j) * a.pitch + x4;
        const float B = a.prof[0][2].B[k], Cs = a.prof[0][2].C[k], G = a.prof[0][2].G[k];
        float4 px = ld4(a.psi[0][0][2] + pi), py = ld4(a.psi[0][1][2] + pi);
#pragma unroll
        for (int e = 0; e < 4; e++) {
          set_el(dX, e, el(dX, e) + el(px, e) * G);
          if (!ok[e]) continue;
          set_el(px, e, B * el(px, e) + Cs * el(rxz, e));
          set_el(dY, e, el(dY, e) + el(py, e) * G);
          set_el(py, e, B * el(py, e) + Cs * el(ryz, e));
        }
        st4(a.psi[0][0][2] + pi, px);
        st4(a.psi[0][1][2] + pi, py);
      }
      if (pml_x) {
#pragma unroll
        for (int e = 0; e < 4; e++) {
          const int i = x4 + e;
          if (!ok[e]) continue;
          const int s = slab_index(a.slab[0], i);
          if (s < 0) continue;
          const long long pi = (static_cast<long long>(k) * a.ny + j) * a.slab[0].W + s;
          const float B = a.prof[0][0].B[i], Cs = a.prof[0][0].C[i], G = a.prof[0][0].G[i];
          float py = a.psi[0][1][0][pi], pz = a.psi[0][2][0][pi];
          set_el(dY, e, el(dY, e) + py * G);
          set_el(dZ, e, el(dZ, e) + pz * G);
          a.psi[0][1][0][pi] = B * py + Cs * el(ryx, e);
          a.psi[0][2][0][pi] = B * pz + Cs * el(rzx, e);
        }
      }
      // TFSF updateD
      if (plane_mask) {
        const long long row = t - a.ctrl->t0;
        const double sc = a.dt / kEps0;
        for (int q = 0; q < a.nplanes; q++) {
          if (!(plane_mask >> q & 1u)) continue;
          const PlaneDev& p = a.planes[q];
          if (j < p.lo[1] || j > p.hi[1] || k < p.lo[2] || k > p.hi[2]) continue;
          for (int e = 0; e < 4; e++) {
            const int i = x4 + e;
            if (!ok[e] || i < p.lo[0] || i > p.hi[0]) continue;
            set_el(dX, e, el(dX, e) + static_cast<float>(sc * tfsf3(a, p, row, 0, 0, i, j, k)));
            set_el(dY, e, el(dY, e) + static_cast<float>(sc * tfsf3(a, p, row, 0, 1, i, j, k)));
            set_el(dZ, e, el(dZ, e) + static_cast<float>(sc * tfsf3(a, p, row, 0, 2, i, j, k)));
          }
        }
      }
      // sources: D-target adds to the flux; E-target undoes last step's value
      // (kept in E by the previous step) and adds this step's after the update
      float4 uX = make_float4(0.f, 0.f, 0.f, 0.f), uY = uX, uZ = uX, aX = uX, aY = uX, aZ = uX;
      if (src_here) {
        for (int s = 0; s < a.nsrc; s++) {
          const SourceDev& sr = a.src[s];
          if (sr.j != j || sr.k != k || sr.i < x4 || sr.i >= x4 + 4) continue;
          const int e = sr.i - x4;
          const double v = t < sr.nvals ? sr.vals[t] : 0.0;
          if (sr.target == 1) {
            const float dv = static_cast<float>(v * a.src_scale_d);
            if (sr.comp == 0) set_el(dX, e, el(dX, e) + dv);
            else if (sr.comp == 1) set_el(dY, e, el(dY, e) + dv);
            else set_el(dZ, e, el(dZ, e) + dv);
          } else {
            const float u = static_cast<float>(a.src_last[s]), ad = static_cast<float>(v);
            if (sr.comp == 0) { set_el(uX, e, el(uX, e) + u); set_el(aX, e, el(aX, e) + ad); }
            else if (sr.comp == 1) { set_el(uY, e, el(uY, e) + u); set_el(aY, e, el(aY, e) + ad); }
            else { set_el(uZ, e, el(uZ, e) + u); set_el(aZ, e, el(aZ, e) + ad); }
            a.src_last[s] = v;
          }
        }
      }
      // material update
      float4 ie;
      int mids[4] = {0, 0, 0, 0};
      bool disp = false;
      if (uniform_mat) {
        ie = make_float4(m0.inv_eps, m0.inv_eps, m0.inv_eps, m0.inv_eps);
        disp = MAXP != 0 && m0.npoles != 0;
      } else {
#pragma unroll
        for (int e = 0; e < 4; e++) {
          int mid;
          if (a.ids) mid = (cur.ids >> (8 * e)) & 0xff;
          else mid = a.bids[((k >> a.bshift) * a.nby + (j >> a.bshift)) * a.nbx + (min(x4 + e, a.nx - 1) >> a.bshift)];
          mids[e] = mid;
          set_el(ie, e, a.mats[mid].inv_eps);
          if (MAXP != 0 && a.mats[mid].npoles != 0) disp = true;
        }
      }
      st4(a.E[0] + c, e_comp<MAXP>(a, 0, c, sub4(cur.ex, uX), dX, ie, ok, disp, uniform_mat, m0, mids, aX));
      st4(a.E[1] + c, e_comp<MAXP>(a, 1, c, sub4(cur.ey, uY), dY, ie, ok, disp, uniform_mat, m0, mids, aY));
      st4(a.E[2] + c, e_comp<MAXP>(a, 2, c, sub4(cur.ez, uZ), dZ, ie, ok, disp, uniform_mat, m0, mids, aZ));
    }
    cur = nxt;
  }
}

__global__ void __launch_bounds__(32 * kRows) fused3d_h_kernel(const FusedArgs a, int kchunk) {
  const int lane = threadIdx.x;
  const int x4 = blockIdx.x * 128 + lane * 4;
  const int j = 1 + blockIdx.y * kRows + threadIdx.y;
  const int jl = min(j, a.ny - 2);
  const bool row_ok = j <= a.ny - 2;
  const int kbeg = 1 + blockIdx.z * kchunk;
  const int kend = min(kbeg + kchunk, a.nz - 1);
  const long long sy = a.pitch, sz = static_cast<long long>(a.pitch) * a.ny;
  const long long t = a.ctrl->t;
  const int xlo = blockIdx.x * 128, xhi = xlo + 127;
  const int j0 = 1 + blockIdx.y * kRows, j1 = min(j0 + kRows - 1, a.ny - 2);
  const bool pml_x = a.pml_axis[0] && hits_slab(a.slab[0], xlo, xhi);
  const bool pml_y = a.pml_axis[1] && hits_slab(a.slab[1], j0, j1);
  unsigned plane_mask = 0;
  for (int q = 0; q < a.nplanes; q++) {
    const PlaneDev& p = a.planes[q];
    if (p.lo[0] <= xhi && p.hi[0] >= xlo && p.lo[1] <= j1 && p.hi[1] >= j0 && p.lo[2] <= kend - 1 && p.hi[2] >= kbeg)
      plane_mask |= 1u << q;
  }
  bool ok[4];
#pragma unroll
  for (int e = 0; e < 4; e++) ok[e] = row_ok && x4 + e >= 1 && x4 + e <= a.nx - 2;
  const float4 fsx = ld4(a.prof[1][0].F + x4);
  const float fsy = a.prof[1][1].F[jl];

  auto load = [&](int k, HPlane& P) {
    const long long c = k * sz + jl * sy + x4;
    P.ex = ld4(a.E[0] + c);
    P.ey = ld4(a.E[1] + c);
    P.ez = ld4(a.E[2] + c);
    P.ex_yp = ld4(a.E[0] + c + sy);
    P.ez_yp = ld4(a.E[2] + c + sy);
    P.hx = ld4(a.H[0] + c);
    P.hy = ld4(a.H[1] + c);
    P.hz = ld4(a.H[2] + c);
  };

  float4 ex_kp, ey_kp;  // E at k+1
  {
    const long long c = kend * sz + jl * sy + x4;
    ex_kp = ld4(a.E[0] + c);
    ey_kp = ld4(a.E[1] + c);
  }
  HPlane cur, nxt;
  load(kend - 1, cur);
  for (int k = kend - 1; k >= kbeg; k--) {
    if (k - 1 >= kbeg) load(k - 1, nxt);
    const long long c = k * sz + jl * sy + x4;
    float ey_xp3 = __shfl_down_sync(kFull, cur.ey.x, 1);
    float ez_xp3 = __shfl_down_sync(kFull, cur.ez.x, 1);
    if (lane == 31) {
      ey_xp3 = a.E[1][c + 4];
      ez_xp3 = a.E[2][c + 4];
    }
    const float fsz = a.prof[1][2].F[k];
    float4 dX, dY, dZ;
    float4 rxy, rxz, ryz, ryx, rzx, rzy;
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const float ey_xp = e == 3 ? ey_xp3 : el(cur.ey, e + 1);
      const float ez_xp = e == 3 ? ez_xp3 : el(cur.ez, e + 1);
      set_el(rxy, e, el(cur.ez_yp, e) - el(cur.ez, e));
      set_el(rxz, e, -(el(ey_kp, e) - el(cur.ey, e)));
      set_el(ryz, e, el(ex_kp, e) - el(cur.ex, e));
      set_el(ryx, e, -(ez_xp - el(cur.ez, e)));
      set_el(rzx, e, ey_xp - el(cur.ey, e));
      set_el(rzy, e, -(el(cur.ex_yp, e) - el(cur.ex, e)));
      set_el(dX, e, fsy * el(rxy, e) + fsz * el(rxz, e));
      set_el(dY, e, fsz * el(ryz, e) + el(fsx, e) * el(ryx, e));
      set_el(dZ, e, el(fsx, e) * el(rzx, e) + fsy * el(rzy, e));
    }
    ex_kp = cur.ex;
    ey_kp = cur.ey;
    if (row_ok) {
      const int sjy = pml_y ? slab_index(a.slab[1], j) : -1;
      const int skz = a.pml_axis[2] ? slab_index(a.slab[2], k) : -1;
      if (sjy >= 0) {
        const long long pi = (static_cast<long long>(k) * a.slab[1].W + sjy) * a.pitch + x4;
        const float B = a.prof[1][1].B[j], Cs = a.prof[1][1].C[j], G = a.prof[1][1].G[j];
        float4 px = ld4(a.psi[1][0][1] + pi), pz = ld4(a.psi[1][2][1] + pi);
#pragma unroll
        for (int e = 0; e < 4; e++) {
          set_el(dX, e, el(dX, e) + el(px, e) * G);
          if (!ok[e]) continue;
          set_el(px, e, B * el(px, e) + Cs * el(rxy, e));
          set_el(dZ, e, el(dZ, e) + el(pz, e) * G);
          set_el(pz, e, B * el(pz, e) + Cs * el(rzy, e));
        }
        st4(a.psi[1][0][1] + pi, px);
        st4(a.psi[1][2][1] + pi, pz);
      }
      if (skz >= 0) {
        const long long pi = (static_cast<long long>(skz) * a.ny + j) * a.pitch + x4;
        const float B = a.prof[1][2].B[k], Cs = a.prof[1][2].C[k], G = a.prof[1][2].G[k];
        float4 px = ld4(a.psi[1][0][2] + pi), py = ld4(a.psi[1][1][2] + pi);
#pragma unroll
        for (int e = 0; e < 4; e++) {
          set_el(dX, e, el(dX, e) + el(px, e) * G);
          if (!ok[e]) continue;
          set_el(px, e, B * el(px, e) + Cs * el(rxz, e));
          set_el(dY, e, el(dY, e) + el(py, e) * G);
          set_el(py, e, B * el(py, e) + Cs * el(ryz, e));
        }
        st4(a.psi[1][0][2] + pi, px);
        st4(a.psi[1][1][2] + pi, py);
      }
      if (pml_x) {
#pragma unroll
        for (int e = 0; e < 4; e++) {
          const int i = x4 + e;
          if (!ok[e]) continue;
          const int s = slab_index(a.slab[0], i);
          if (s < 0) continue;
          const long long pi = (static_cast<long long>(k) * a.ny + j) * a.slab[0].W + s;
          const float B = a.prof[1][0].B[i], Cs = a.prof[1][0].C[i], G = a.prof[1][0].G[i];
          float py = a.psi[1][1][0][pi], pz = a.psi[1][2][0][pi];
          set_el(dY, e, el(dY, e) + py * G);
          set_el(dZ, e, el(dZ, e) + pz * G);
          a.psi[1][1][0][pi] = B * py + Cs * el(ryx, e);
          a.psi[1][2][0][pi] = B * pz + Cs * el(rzx, e);
        }
      }
      if (plane_mask) {
        const long long row = t - a.ctrl->t0 + 1;
        const double sc = a.eta * a.dt / kMu0;
        for (int q = 0; q < a.nplanes; q++) {
          if (!(plane_mask >> q & 1u)) continue;
          const PlaneDev& p = a.planes[q];
          if (j < p.lo[1] || j > p.hi[1] || k < p.lo[2] || k > p.hi[2]) continue;
          for (int e = 0; e < 4; e++) {
            const int i = x4 + e;
            if (!ok[e] || i < p.lo[0] || i > p.hi[0]) continue;
            set_el(dX, e, el(dX, e) + static_cast<float>(sc * tfsf3(a, p, row, 1, 0, i, j, k)));
            set_el(dY, e, el(dY, e) + static_cast<float>(sc * tfsf3(a, p, row, 1, 1, i, j, k)));
            set_el(dZ, e, el(dZ, e) + static_cast<float>(sc * tfsf3(a, p, row, 1, 2, i, j, k)));
          }
        }
      }
      float4 hx = cur.hx, hy = cur.hy, hz = cur.hz;
#pragma unroll
      for (int e = 0; e < 4; e++) {
        if (!ok[e]) continue;
        set_el(hx, e, el(hx, e) - el(dX, e));
        set_el(hy, e, el(hy, e) - el(dY, e));
        set_el(hz, e, el(hz, e) - el(dZ, e));
      }
      st4(a.H[0] + c, hx);
      st4(a.H[1] + c, hy);
      st4(a.H[2] + c, hz);
    }
    cur = nxt;
  }
}

static int kchunk3d(int nz, int blocks_xy) {
  // several waves of 148 SMs x 4 CTAs; chunks of at least 32 planes
  const int interior = nz - 2;
  int chunks = (148 * 4 * 3 + blocks_xy - 1) / blocks_xy;
  chunks = max(1, min(chunks, interior / 32));
  return (interior + chunks - 1) / chunks;
}

bool fused3d_supported(const FusedArgs& a) { return a.pitch % 4 == 0 && (a.bids == nullptr || a.bshift >= 2); }

int launch_fused3d_e(const FusedArgs& a, cudaStream_t s) {
  const int bx = (a.pitch + 127) / 128, by = (a.ny - 2 + kRows - 1) / kRows;
  const int kchunk = kchunk3d(a.nz, bx * by);
  const int bz = (a.nz - 2 + kchunk - 1) / kchunk;
  dim3 grid(bx, by, bz), block(32, kRows, 1);
  switch (a.max_poles) {
    case 0: fused3d_e_kernel<0><<<grid, block, 0, s>>>(a, kchunk); break;
    case -1: fused3d_e_kernel<-1><<<grid, block, 0, s>>>(a, kchunk); break;
    case 1: fused3d_e_kernel<1><<<grid, block, 0, s>>>(a, kchunk); break;
    default: fused3d_e_kernel<2><<<grid, block, 0, s>>>(a, kchunk); break;
  }
  return 1;
}

int launch_fused3d_h(const FusedArgs& a, cudaStream_t s) {
  const int bx = (a.pitch + 127) / 128, by = (a.ny - 2 + kRows - 1) / kRows;
  const int kchunk = kchunk3d(a.nz, bx * by);
  const int bz = (a.nz - 2 + kchunk - 1) / kchunk;
  fused3d_h_kernel<<<dim3(bx, by, bz), dim3(32, kRows, 1), 0, s>>>(a, kchunk);
  return 1;
}

}  // namespace fdtdb
