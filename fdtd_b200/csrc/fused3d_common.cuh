// Device helpers shared by the FP32 fused 3D sweeps (kernels_fused3d.cu and
// kernels_fused3d_tma.cu): 128-bit group access, the aux-grid interpolation
// used by the TFSF kernel, and the per-group material update.
#pragma once
#include "internal.h"

namespace fdtdb {
namespace f3d {

__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ void st4(float* p, float4 v) { *reinterpret_cast<float4*>(p) = v; }
__device__ __forceinline__ float el(const float4& v, int e) { return e == 0 ? v.x : (e == 1 ? v.y : (e == 2 ? v.z : v.w)); }
__device__ __forceinline__ void set_el(float4& v, int e, float x) {
  if (e == 0) v.x = x;
  else if (e == 1) v.y = x;
  else if (e == 2) v.z = x;
  else v.w = x;
}

__device__ __forceinline__ float4 sub4(float4 a, float4 b) {
  return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w);
}

// Material update of one E component for the 4 cells of a group: returns the
// new E (plus this step's E-target source values), updating P/J in place.
// spj: the group's J (then P) values already staged in shared memory, slot
// (q*3 + I) for J and (NP*3 + q*3 + I) for P, `stride` float4 apart; null
// reads them from global memory.
template <int MAXP>
__device__ __forceinline__ float4 e_comp(const FusedArgs& a, int I, long long c, float4 eo, float4 d, float4 ie,
                                         const bool ok[4], bool disp, bool uniform, const MatF32& m0,
                                         const int mids[4], float4 add, const float4* spj = nullptr,
                                         int stride = 0) {
  float4 en;
  if (MAXP != 0 && disp) {
    constexpr int NP = MAXP <= 0 ? 1 : MAXP;
    float4 jt[NP], pt[NP];
#pragma unroll
    for (int q = 0; q < NP; q++) {
      jt[q] = spj ? spj[(q * 3 + I) * stride] : ld4(a.J[q][I] + c);
      if (MAXP > 0) pt[q] = spj ? spj[(NP * 3 + q * 3 + I) * stride] : ld4(a.P[q][I] + c);
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


// Context of one thread's 4-cell group, fixed over a sweep.
struct GroupCtx {
  int x4, j, lane;
  bool ok[4];
  bool row_ok, pml_y, src_here, uniform_mat;
  int sx4;  // the group's first position in the aligned x-slab rows, or -1 (no x-slab cell)
  float4 fsx;
  float fsy;
  long long t;
};

__device__ __forceinline__ GroupCtx make_ctx(const FusedArgs& a, int ft, int x4, int j, int lane, int kbeg, int kend) {
  GroupCtx g;
  g.x4 = x4;
  g.j = j;
  g.lane = lane;
  g.row_ok = j <= a.ny - 2;
#pragma unroll
  for (int e = 0; e < 4; e++) g.ok[e] = g.row_ok && x4 + e >= 1 && x4 + e <= a.nx - 2;
  g.sx4 = a.pml_axis[0] ? slab_group4(a.slab[0], x4) : -1;
  g.pml_y = a.pml_axis[1] && slab_index(a.slab[1], min(j, a.ny - 2)) >= 0;
  g.src_here = false;
  for (int s = 0; s < a.nsrc; s++)
    if ((a.src[s].target < 2) == (ft == 0) && a.src[s].j == j && a.src[s].i >= x4 && a.src[s].i < x4 + 4 &&
        a.src[s].k >= kbeg && a.src[s].k < kend)
      g.src_here = true;
  g.uniform_mat = !a.ids && !a.bids;
  g.fsx = ld4(a.prof[ft][0].F + x4);
  g.fsy = a.prof[ft][1].F[min(j, a.ny - 2)];
  g.t = a.ctrl->t;
  return g;
}

// The E update of one group at plane k from the H values around it (own,
// y-1, z-1 and the x-1 neighbour of the group's first cell), the old E and
// the material ids; writes E (and psi, P, J) to global memory.
template <int MAXP>
__device__ __forceinline__ void e_group_update(const FusedArgs& a, const GroupCtx& g, int k, float4 hx, float4 hy,
                                               float4 hz, float4 hx_ym, float4 hz_ym, float4 hx_km, float4 hy_km,
                                               float hy_xm0, float hz_xm0, float4 exo, float4 eyo, float4 ezo,
                                               unsigned ids4, const float* staged_px = nullptr,
                                               const float4* spj = nullptr, int pj_stride = 0) {
  if (!g.row_ok) return;
  const int j = g.j, x4 = g.x4;
  const long long c = (static_cast<long long>(k) * a.ny + j) * a.pitch + x4;
  const float fsz = a.prof[0][2].F[k];
  float4 dX, dY, dZ, rxy, rxz, ryz, ryx, rzx, rzy;
#pragma unroll
  for (int e = 0; e < 4; e++) {
    const float hy_xm = e == 0 ? hy_xm0 : el(hy, e - 1);
    const float hz_xm = e == 0 ? hz_xm0 : el(hz, e - 1);
    set_el(rxy, e, el(hz, e) - el(hz_ym, e));
    set_el(rxz, e, -(el(hy, e) - el(hy_km, e)));
    set_el(ryz, e, el(hx, e) - el(hx_km, e));
    set_el(ryx, e, -(el(hz, e) - hz_xm));
    set_el(rzx, e, el(hy, e) - hy_xm);
    set_el(rzy, e, -(el(hx, e) - el(hx_ym, e)));
    set_el(dX, e, g.fsy * el(rxy, e) + fsz * el(rxz, e));
    set_el(dY, e, fsz * el(ryz, e) + el(g.fsx, e) * el(ryx, e));
    set_el(dZ, e, el(g.fsx, e) * el(rzx, e) + g.fsy * el(rzy, e));
  }
  // CPML: y and z slabs share the field row layout (128-bit access)
  const int sjy = g.pml_y ? slab_index(a.slab[1], j) : -1;
  const int skz = a.pml_axis[2] ? slab_index(a.slab[2], k) : -1;
  if (sjy >= 0) {
    const long long pi = (static_cast<long long>(k) * a.slab[1].W + sjy) * a.pitch + x4;
    const float B = a.prof[0][1].B[j], Cs = a.prof[0][1].C[j], G = a.prof[0][1].G[j];
    float4 px = ld4(a.psi[0][0][1] + pi), pz = ld4(a.psi[0][2][1] + pi);
#pragma unroll
    for (int e = 0; e < 4; e++) {
      if (!g.ok[e]) continue;
      set_el(dX, e, el(dX, e) + el(px, e) * G);
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
      if (!g.ok[e]) continue;
      set_el(dX, e, el(dX, e) + el(px, e) * G);
      set_el(px, e, B * el(px, e) + Cs * el(rxz, e));
      set_el(dY, e, el(dY, e) + el(py, e) * G);
      set_el(py, e, B * el(py, e) + Cs * el(ryz, e));
    }
    st4(a.psi[0][0][2] + pi, px);
    st4(a.psi[0][1][2] + pi, py);
  }
  if (g.sx4 >= 0) {
    // the group's x-slab integrators as one aligned float4 per component;
    // cells outside the slab have zero coefficients and keep zero, cells
    // not updated keep theirs
    const long long pi = (static_cast<long long>(k) * a.ny + j) * a.slab[0].W4 + g.sx4;
    const float4 B = ld4(a.prof[0][0].B + x4), Cs = ld4(a.prof[0][0].C + x4), G = ld4(a.prof[0][0].G + x4);
    float4 py = staged_px ? reinterpret_cast<const float4*>(staged_px)[0] : ld4(a.psi[0][1][0] + pi);
    float4 pz = staged_px ? reinterpret_cast<const float4*>(staged_px)[1] : ld4(a.psi[0][2][0] + pi);
#pragma unroll
    for (int e = 0; e < 4; e++) {
      if (!g.ok[e]) continue;
      const float y = el(py, e), z = el(pz, e);
      set_el(dY, e, el(dY, e) + y * el(G, e));
      set_el(dZ, e, el(dZ, e) + z * el(G, e));
      set_el(py, e, el(B, e) * y + el(Cs, e) * el(ryx, e));
      set_el(pz, e, el(B, e) * z + el(Cs, e) * el(rzx, e));
    }
    st4(a.psi[0][1][0] + pi, py);
    st4(a.psi[0][2][0] + pi, pz);
  }
  // sources: D-target adds to the flux; E-target undoes last step's value
  // (kept in E by the previous step) and adds this step's after the update
  float4 uX = make_float4(0.f, 0.f, 0.f, 0.f), uY = uX, uZ = uX, aX = uX, aY = uX, aZ = uX;
  if (g.src_here) {
    for (int q = 0; q < a.nsrc; q++) {
      const SourceDev& sr = a.src[q];
      if (sr.target > 1 || sr.j != j || sr.k != k || sr.i < x4 || sr.i >= x4 + 4) continue;
      const int e = sr.i - x4;
      const double v = g.t < sr.nvals ? sr.vals[g.t] : 0.0;
      if (sr.target == 1) {
        const float dv = static_cast<float>(v * a.src_scale_d);
        if (sr.comp == 0) set_el(dX, e, el(dX, e) + dv);
        else if (sr.comp == 1) set_el(dY, e, el(dY, e) + dv);
        else set_el(dZ, e, el(dZ, e) + dv);
      } else {
        const float u = static_cast<float>(a.src_last[q]), ad = static_cast<float>(v);
        if (sr.comp == 0) {
          set_el(uX, e, el(uX, e) + u);
          set_el(aX, e, el(aX, e) + ad);
        } else if (sr.comp == 1) {
          set_el(uY, e, el(uY, e) + u);
          set_el(aY, e, el(aY, e) + ad);
        } else {
          set_el(uZ, e, el(uZ, e) + u);
          set_el(aZ, e, el(aZ, e) + ad);
        }
        a.src_last[q] = v;
      }
    }
  }
  // material update
  const MatF32& m0 = a.mats[0];
  float4 ie;
  int mids[4] = {0, 0, 0, 0};
  bool disp = false;
  if (g.uniform_mat) {
    ie = make_float4(m0.inv_eps, m0.inv_eps, m0.inv_eps, m0.inv_eps);
    disp = MAXP != 0 && m0.npoles != 0;
  } else {
    // with every material dispersive the P/J loads need not wait for the
    // material lookups
    if (MAXP != 0 && a.all_dispersive) disp = true;
    if (!a.ids && a.bshift >= 2) {
      const int mid = a.bids[((k >> a.bshift) * a.nby + (j >> a.bshift)) * a.nbx + (x4 >> a.bshift)];
      const MatF32& m = a.mats[mid];
      ie = make_float4(m.inv_eps, m.inv_eps, m.inv_eps, m.inv_eps);
#pragma unroll
      for (int e = 0; e < 4; e++) mids[e] = mid;
      if (MAXP != 0 && m.npoles != 0) disp = true;
    } else {
#pragma unroll
      for (int e = 0; e < 4; e++) {
        int mid;
        if (a.ids) mid = (ids4 >> (8 * e)) & 0xff;
        else mid = a.bids[((k >> a.bshift) * a.nby + (j >> a.bshift)) * a.nbx + (min(x4 + e, a.nx - 1) >> a.bshift)];
        mids[e] = mid;
        set_el(ie, e, a.mats[mid].inv_eps);
        if (MAXP != 0 && a.mats[mid].npoles != 0) disp = true;
      }
    }
  }
  if (a.inv_eps_map) {
    // per-cell permittivity of non-dispersive cells
    const float4 v = ld4(a.inv_eps_map + c);
#pragma unroll
    for (int e = 0; e < 4; e++)
      if (el(v, e) > 0.f && a.mats[mids[e]].npoles == 0) set_el(ie, e, el(v, e));
  }
  st4(a.E[0] + c,
      e_comp<MAXP>(a, 0, c, sub4(exo, uX), dX, ie, g.ok, disp, g.uniform_mat, m0, mids, aX, spj, pj_stride));
  st4(a.E[1] + c,
      e_comp<MAXP>(a, 1, c, sub4(eyo, uY), dY, ie, g.ok, disp, g.uniform_mat, m0, mids, aY, spj, pj_stride));
  st4(a.E[2] + c,
      e_comp<MAXP>(a, 2, c, sub4(ezo, uZ), dZ, ie, g.ok, disp, g.uniform_mat, m0, mids, aZ, spj, pj_stride));
}

// 1/mu_r of the group's 4 cells: H = B/(mu_r mu0) (the magnetic
// ConstantUpdate, DispersiveMaterials.hpp:354-359), so the flux change of the
// step is scaled per cell before it is added to the stored eta*H.
__device__ __forceinline__ float4 group_inv_mu(const FusedArgs& a, const GroupCtx& g, int k, long long c) {
  float4 r;
  if (g.uniform_mat) {
    const float m = a.mats[0].inv_mu;
    return make_float4(m, m, m, m);
  }
  if (a.ids) {
    const unsigned w = *reinterpret_cast<const unsigned*>(a.ids + c);
#pragma unroll
    for (int e = 0; e < 4; e++) set_el(r, e, a.mats[(w >> (8 * e)) & 0xff].inv_mu);
  } else {
#pragma unroll
    for (int e = 0; e < 4; e++)
      set_el(r, e,
             a.mats[a.bids[((k >> a.bshift) * a.nby + (g.j >> a.bshift)) * a.nbx + (min(g.x4 + e, a.nx - 1) >> a.bshift)]]
                 .inv_mu);
  }
  return r;
}

// The H update of one group at plane k from the E values around it (own,
// y+1, z+1 and the x+1 neighbour of the group's last cell) and the old H.
// MU: some material has mu_r != 1 (a separate instantiation, so that the
// common case keeps its registers).
template <bool MU>
__device__ __forceinline__ void h_group_update(const FusedArgs& a, const GroupCtx& g, int k, float4 ex, float4 ey,
                                               float4 ez, float4 ex_yp, float4 ez_yp, float4 ex_kp, float4 ey_kp,
                                               float ey_xp3, float ez_xp3, float4 hx, float4 hy, float4 hz,
                                               const float* staged_px = nullptr) {
  if (!g.row_ok) return;
  const int j = g.j, x4 = g.x4;
  const long long c = (static_cast<long long>(k) * a.ny + j) * a.pitch + x4;
  const float fsz = a.prof[1][2].F[k];
  float4 dX, dY, dZ, rxy, rxz, ryz, ryx, rzx, rzy;
#pragma unroll
  for (int e = 0; e < 4; e++) {
    const float ey_xp = e == 3 ? ey_xp3 : el(ey, e + 1);
    const float ez_xp = e == 3 ? ez_xp3 : el(ez, e + 1);
    set_el(rxy, e, el(ez_yp, e) - el(ez, e));
    set_el(rxz, e, -(el(ey_kp, e) - el(ey, e)));
    set_el(ryz, e, el(ex_kp, e) - el(ex, e));
    set_el(ryx, e, -(ez_xp - el(ez, e)));
    set_el(rzx, e, ey_xp - el(ey, e));
    set_el(rzy, e, -(el(ex_yp, e) - el(ex, e)));
    set_el(dX, e, g.fsy * el(rxy, e) + fsz * el(rxz, e));
    set_el(dY, e, fsz * el(ryz, e) + el(g.fsx, e) * el(ryx, e));
    set_el(dZ, e, el(g.fsx, e) * el(rzx, e) + g.fsy * el(rzy, e));
  }
  const int sjy = g.pml_y ? slab_index(a.slab[1], j) : -1;
  const int skz = a.pml_axis[2] ? slab_index(a.slab[2], k) : -1;
  if (sjy >= 0) {
    const long long pi = (static_cast<long long>(k) * a.slab[1].W + sjy) * a.pitch + x4;
    const float B = a.prof[1][1].B[j], Cs = a.prof[1][1].C[j], G = a.prof[1][1].G[j];
    float4 px = ld4(a.psi[1][0][1] + pi), pz = ld4(a.psi[1][2][1] + pi);
#pragma unroll
    for (int e = 0; e < 4; e++) {
      if (!g.ok[e]) continue;
      set_el(dX, e, el(dX, e) + el(px, e) * G);
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
      if (!g.ok[e]) continue;
      set_el(dX, e, el(dX, e) + el(px, e) * G);
      set_el(px, e, B * el(px, e) + Cs * el(rxz, e));
      set_el(dY, e, el(dY, e) + el(py, e) * G);
      set_el(py, e, B * el(py, e) + Cs * el(ryz, e));
    }
    st4(a.psi[1][0][2] + pi, px);
    st4(a.psi[1][1][2] + pi, py);
  }
  if (g.sx4 >= 0) {
    // the group's x-slab integrators as one aligned float4 per component;
    // cells outside the slab have zero coefficients and keep zero, cells
    // not updated keep theirs
    const long long pi = (static_cast<long long>(k) * a.ny + j) * a.slab[0].W4 + g.sx4;
    const float4 B = ld4(a.prof[1][0].B + x4), Cs = ld4(a.prof[1][0].C + x4), G = ld4(a.prof[1][0].G + x4);
    float4 py = staged_px ? reinterpret_cast<const float4*>(staged_px)[0] : ld4(a.psi[1][1][0] + pi);
    float4 pz = staged_px ? reinterpret_cast<const float4*>(staged_px)[1] : ld4(a.psi[1][2][0] + pi);
#pragma unroll
    for (int e = 0; e < 4; e++) {
      if (!g.ok[e]) continue;
      const float y = el(py, e), z = el(pz, e);
      set_el(dY, e, el(dY, e) + y * el(G, e));
      set_el(dZ, e, el(dZ, e) + z * el(G, e));
      set_el(py, e, el(B, e) * y + el(Cs, e) * el(ryx, e));
      set_el(pz, e, el(B, e) * z + el(Cs, e) * el(rzx, e));
    }
    st4(a.psi[1][1][0] + pi, py);
    st4(a.psi[1][2][0] + pi, pz);
  }
  // sources: B-target adds to the flux; H-target undoes last step's value
  // and adds this step's after the update (H is stored as eta*H)
  float4 aX = make_float4(0.f, 0.f, 0.f, 0.f), aY = aX, aZ = aX;
  if (g.src_here) {
    for (int q = 0; q < a.nsrc; q++) {
      const SourceDev& sr = a.src[q];
      if (sr.target < 2 || sr.j != j || sr.k != k || sr.i < x4 || sr.i >= x4 + 4) continue;
      const int e = sr.i - x4;
      const double v = g.t < sr.nvals ? sr.vals[g.t] : 0.0;
      if (sr.target == 3) {
        const float dv = static_cast<float>(v * a.src_scale_b);
        if (sr.comp == 0) set_el(dX, e, el(dX, e) - dv);
        else if (sr.comp == 1) set_el(dY, e, el(dY, e) - dv);
        else set_el(dZ, e, el(dZ, e) - dv);
      } else {
        const float u = static_cast<float>(a.src_last[q] * a.src_scale_h), ad = static_cast<float>(v * a.src_scale_h);
        if (sr.comp == 0) {
          set_el(hx, e, el(hx, e) - u);
          set_el(aX, e, el(aX, e) + ad);
        } else if (sr.comp == 1) {
          set_el(hy, e, el(hy, e) - u);
          set_el(aY, e, el(aY, e) + ad);
        } else {
          set_el(hz, e, el(hz, e) - u);
          set_el(aZ, e, el(aZ, e) + ad);
        }
        a.src_last[q] = v;
      }
    }
  }
  if (MU) {
    const float4 im = group_inv_mu(a, g, k, c);
#pragma unroll
    for (int e = 0; e < 4; e++) {
      set_el(dX, e, el(dX, e) * el(im, e));
      set_el(dY, e, el(dY, e) * el(im, e));
      set_el(dZ, e, el(dZ, e) * el(im, e));
    }
  }
#pragma unroll
  for (int e = 0; e < 4; e++) {
    if (!g.ok[e]) continue;
    set_el(hx, e, el(hx, e) - el(dX, e) + el(aX, e));
    set_el(hy, e, el(hy, e) - el(dY, e) + el(aY, e));
    set_el(hz, e, el(hz, e) - el(dZ, e) + el(aZ, e));
  }
  st4(a.H[0] + c, hx);
  st4(a.H[1] + c, hy);
  st4(a.H[2] + c, hz);
}

}  // namespace f3d
}  // namespace fdtdb
