// FP32 fused method: one sweep per half step over E/H state only.
//
// The reference advances D/B and derives E/H from them (D/B-flux form,
// include/DispersiveMaterials.hpp:342-360). With the constitutive relations
// being linear, the same update can be written on E and H directly, which
// halves the state that has to stream through HBM:
//   E' = E + (1/eps_inf) * ( sum_J Fs_J * raw_IJ + sum_J psi_IJ G_J - sum_p Jt_p )
//   psi_IJ' = B_J psi_IJ + Cs_J raw_IJ        (raw_IJ = LeviCivita(I,J,K) * dH_K along J)
//   Lorentz pole: Pt' = Pt + Jt; Jt' = a Jt + b E' - c Pt'
//   Drude pole:   Jt' = a Jt + b E'            (P is not needed)
//   Ht' = Ht - ( sum_J Fs_J * raw_IJ + sum_J psi_IJ G_J ),  Ht = eta*H
// with Fs = (dt/(eps0 eta dx)) F for E and (eta dt/(mu0 dx)) F for H, Pt = P/eps0,
// Jt = dt J/eps0, and psi scaled to E units. All of this is the reference's
// arithmetic (YeeUpdates.hpp:396-405, PML.hpp:315-323, DispersiveMaterials.hpp:
// 710-735, :979-998) regrouped; coefficients are computed in FP64 on the host.
//
// Thread mapping: a CTA of 32 x BY threads covers a 32 x BY tile of (x, y)
// and marches along z over a chunk of planes; the k-1 plane of the z
// neighbours stays in registers, x neighbours come from warp shuffles.
// These scalar sweeps carry the 2D modes; 3D grids use kernels_fused3d*.cu.
// TFSF corrections are applied after each sweep by kernels_tfsf.cu.
#include "internal.h"

namespace fdtdb {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kBY = 8;

// the x slab of the FP32 method is in the aligned layout (Slab::lo4)
__device__ __forceinline__ long long psi_index(const FusedArgs& a, int J, int s, int i, int j, int k) {
  if (J == 0) return (static_cast<long long>(k) * a.ny + j) * a.slab[0].W4 + slab_index4(a.slab[0], i);
  if (J == 1) return (static_cast<long long>(k) * a.slab[1].W + s) * a.pitch + i;
  return (static_cast<long long>(s) * a.ny + j) * a.pitch + i;
}

__device__ __forceinline__ bool range_hits_slab(const Slab& s, int lo, int hi) {
  return (s.wlo > 0 && lo <= s.wlo) || (s.W - s.wlo > 0 && hi >= s.hi0);
}

template <int MODE, int MAXP>
__global__ void __launch_bounds__(256) fused_e_kernel(const __grid_constant__ FusedArgs a, int kchunk) {
  const int lane = threadIdx.x;
  const int i0 = blockIdx.x * 32 + 1, j0 = blockIdx.y * kBY + 1;
  const int i = i0 + lane, j = j0 + threadIdx.y;
  const bool active = i <= a.nx - 2 && j <= a.ny - 2;
  const int il = min(i, a.nx - 2), jl = min(j, a.ny - 2);
  int kbeg = 0, kend = 1;
  if (MODE == kThreeD) {
    kbeg = 1 + blockIdx.z * kchunk;
    kend = min(kbeg + kchunk, a.nz - 1);
  }
  const long long sy = a.pitch, sz = static_cast<long long>(a.pitch) * a.ny;
  const long long t = a.ctrl->t;
  // CTA-level feature tests
  const int i1 = min(i0 + 31, a.nx - 2), j1 = min(j0 + kBY - 1, a.ny - 2);
  bool pml_x = a.pml_axis[0] && range_hits_slab(a.slab[0], i0, i1);
  bool pml_y = a.pml_axis[1] && range_hits_slab(a.slab[1], j0, j1);
  bool pml_zr = MODE == kThreeD && a.pml_axis[2];

  float hx_m = 0.f, hy_m = 0.f;
  if (MODE == kThreeD) {
    const long long cp = (kbeg - 1) * sz + jl * sy + il;
    hx_m = a.H[0][cp];
    hy_m = a.H[1][cp];
  }
  const float fsx = a.prof[0][0].F[il], fsy = a.prof[0][1].F[jl];
  for (int k = kbeg; k < kend; k++) {
    const long long c = k * sz + jl * sy + il;
    const float hx = hasH(MODE, 0) ? a.H[0][c] : 0.f;
    const float hy = hasH(MODE, 1) ? a.H[1][c] : 0.f;
    const float hz = hasH(MODE, 2) ? a.H[2][c] : 0.f;
    float hy_xm = __shfl_up_sync(kFull, hy, 1);
    float hz_xm = __shfl_up_sync(kFull, hz, 1);
    if (lane == 0) {
      if (hasH(MODE, 1)) hy_xm = a.H[1][c - 1];
      if (hasH(MODE, 2)) hz_xm = a.H[2][c - 1];
    }
    const float hx_ym = hasH(MODE, 0) ? a.H[0][c - sy] : 0.f;
    const float hz_ym = hasH(MODE, 2) ? a.H[2][c - sy] : 0.f;
    // raw_IJ = LeviCivita(I,J,K) * (H_K - H_K[-J])
    const float r_xy = hz - hz_ym, r_xz = -(hy - hy_m);
    const float r_yz = hx - hx_m, r_yx = -(hz - hz_xm);
    const float r_zx = hy - hy_xm, r_zy = -(hx - hx_ym);
    if (MODE == kThreeD) {
      hx_m = hx;
      hy_m = hy;
    }
    if (!active) continue;
    const float fsz = MODE == kThreeD ? a.prof[0][2].F[k] : 1.f;
    float dx_ = fsy * r_xy + fsz * r_xz;
    float dy_ = fsz * r_yz + fsx * r_yx;
    float dz_ = fsx * r_zx + fsy * r_zy;
    // CPML: E += psi_old * G, psi = B psi + Cs raw
    const bool pml_z = pml_zr && slab_index(a.slab[2], k) >= 0;
    if (pml_x | pml_y | pml_z) {
      const int idx[3] = {i, j, k};
      const float raw[3][3] = {{0.f, r_xy, r_xz}, {r_yx, 0.f, r_yz}, {r_zx, r_zy, 0.f}};
      float* dsum[3] = {&dx_, &dy_, &dz_};
      const bool on[3] = {pml_x, pml_y, pml_z};
#pragma unroll
      for (int J = 0; J < 3; J++) {
        if (!on[J]) continue;
        const int s = slab_index(a.slab[J], idx[J]);
        if (s < 0) continue;
        const long long pidx = psi_index(a, J, s, i, j, k);
        const float B = a.prof[0][J].B[idx[J]], Cs = a.prof[0][J].C[idx[J]], G = a.prof[0][J].G[idx[J]];
#pragma unroll
        for (int I = 0; I < 3; I++) {
          if (!hasE(MODE, I) || I == J || !hasH(MODE, third(I, J))) continue;
          float* ps = a.psi[0][I][J] + pidx;
          const float psi = *ps;
          *dsum[I] += psi * G;
          *ps = B * psi + Cs * raw[I][J];
        }
      }
    }
    // D-target sources add to the flux before the material update
    float undo0 = 0.f, undo1 = 0.f, undo2 = 0.f, add0 = 0.f, add1 = 0.f, add2 = 0.f;
    for (int s = 0; s < a.nsrc; s++) {
      const SourceDev& sr = a.src[s];
      if (sr.target > 1 || sr.cell != c) continue;
      const double v = t < sr.nvals ? sr.vals[t] : 0.0;
      if (sr.target == 1) {
        const float dv = static_cast<float>(v * a.src_scale_d);
        if (sr.comp == 0) dx_ += dv;
        else if (sr.comp == 1) dy_ += dv;
        else dz_ += dv;
      } else {
        const float u = static_cast<float>(a.src_last[s]), ad = static_cast<float>(v);
        if (sr.comp == 0) { undo0 += u; add0 += ad; }
        else if (sr.comp == 1) { undo1 += u; add1 += ad; }
        else { undo2 += u; add2 += ad; }
        a.src_last[s] = v;
      }
    }
    // material update
    int mid = 0;
    if (a.ids) mid = a.ids[c];
    else if (a.bids) mid = a.bids[((k >> a.bshift) * a.nby + (j >> a.bshift)) * a.nbx + (i >> a.bshift)];
    const MatF32& m = a.mats[mid];
    float ie = m.inv_eps;
    if (a.inv_eps_map && m.npoles == 0) {
      const float v = a.inv_eps_map[c];
      if (v > 0.f) ie = v;
    }
    float d[3] = {dx_, dy_, dz_};
#pragma unroll
    for (int I = 0; I < 3; I++) {
      if (!hasE(MODE, I)) continue;
      float e = a.E[I][c] - (I == 0 ? undo0 : (I == 1 ? undo1 : undo2));
      if (MAXP != 0 && m.npoles != 0) {
        float jsum = 0.f;
        float jt[2] = {0.f, 0.f};
        const int np = m.npoles < 0 ? 1 : m.npoles;
#pragma unroll
        for (int q = 0; q < (MAXP < 0 ? 1 : MAXP); q++) {
          if (q < np) {
            jt[q] = a.J[q][I][c];
            jsum += jt[q];
          }
        }
        e = e + ie * (d[I] - jsum);
#pragma unroll
        for (int q = 0; q < (MAXP < 0 ? 1 : MAXP); q++) {
          if (q >= np) continue;
          if (m.npoles < 0) {
            a.J[q][I][c] = m.a[q] * jt[q] + m.b[q] * e;
          } else {
            const float pn = a.P[q][I][c] + jt[q];
            a.P[q][I][c] = pn;
            a.J[q][I][c] = m.a[q] * jt[q] + m.b[q] * e - m.c[q] * pn;
          }
        }
      } else {
        e = e + ie * d[I];
      }
      a.E[I][c] = e + (I == 0 ? add0 : (I == 1 ? add1 : add2));
    }
  }
}

template <int MODE>
__global__ void __launch_bounds__(256) fused_h_kernel(const __grid_constant__ FusedArgs a, int kchunk) {
  const int lane = threadIdx.x;
  const int i0 = blockIdx.x * 32 + 1, j0 = blockIdx.y * kBY + 1;
  const int i = i0 + lane, j = j0 + threadIdx.y;
  const bool active = i <= a.nx - 2 && j <= a.ny - 2;
  const int il = min(i, a.nx - 2), jl = min(j, a.ny - 2);
  int kbeg = 0, kend = 1;
  if (MODE == kThreeD) {
    kbeg = 1 + blockIdx.z * kchunk;
    kend = min(kbeg + kchunk, a.nz - 1);
  }
  const long long sy = a.pitch, sz = static_cast<long long>(a.pitch) * a.ny;
  const int i1 = min(i0 + 31, a.nx - 2), j1 = min(j0 + kBY - 1, a.ny - 2);
  bool pml_x = a.pml_axis[0] && range_hits_slab(a.slab[0], i0, i1);
  bool pml_y = a.pml_axis[1] && range_hits_slab(a.slab[1], j0, j1);
  bool pml_zr = MODE == kThreeD && a.pml_axis[2];
  float ex_c = 0.f, ey_c = 0.f;
  if (MODE == kThreeD) {
    const long long c0 = kbeg * sz + jl * sy + il;
    ex_c = a.E[0][c0];
    ey_c = a.E[1][c0];
  }
  const float fsx = a.prof[1][0].F[il], fsy = a.prof[1][1].F[jl];
  for (int k = kbeg; k < kend; k++) {
    const long long c = k * sz + jl * sy + il;
    float ex = 0.f, ey = 0.f, ex_zp = 0.f, ey_zp = 0.f;
    if (MODE == kThreeD) {
      ex = ex_c;
      ey = ey_c;
      ex_zp = a.E[0][c + sz];
      ey_zp = a.E[1][c + sz];
      ex_c = ex_zp;
      ey_c = ey_zp;
    } else {
      ex = hasE(MODE, 0) ? a.E[0][c] : 0.f;
      ey = hasE(MODE, 1) ? a.E[1][c] : 0.f;
    }
    const float ez = hasE(MODE, 2) ? a.E[2][c] : 0.f;
    float ey_xp = __shfl_down_sync(kFull, ey, 1);
    float ez_xp = __shfl_down_sync(kFull, ez, 1);
    if (lane == 31 || i == a.nx - 2) {
      if (hasE(MODE, 1)) ey_xp = a.E[1][c + 1];
      if (hasE(MODE, 2)) ez_xp = a.E[2][c + 1];
    }
    const float ex_yp = hasE(MODE, 0) ? a.E[0][c + sy] : 0.f;
    const float ez_yp = hasE(MODE, 2) ? a.E[2][c + sy] : 0.f;
    // raw_IJ = LeviCivita(I,J,K) * (E_K[+J] - E_K)
    const float r_xy = ez_yp - ez, r_xz = -(ey_zp - ey);
    const float r_yz = ex_zp - ex, r_yx = -(ez_xp - ez);
    const float r_zx = ey_xp - ey, r_zy = -(ex_yp - ex);
    if (!active) continue;
    const float fsz = MODE == kThreeD ? a.prof[1][2].F[k] : 1.f;
    float dx_ = fsy * r_xy + fsz * r_xz;
    float dy_ = fsz * r_yz + fsx * r_yx;
    float dz_ = fsx * r_zx + fsy * r_zy;
    const bool pml_z = pml_zr && slab_index(a.slab[2], k) >= 0;
    if (pml_x | pml_y | pml_z) {
      const int idx[3] = {i, j, k};
      const float raw[3][3] = {{0.f, r_xy, r_xz}, {r_yx, 0.f, r_yz}, {r_zx, r_zy, 0.f}};
      float* dsum[3] = {&dx_, &dy_, &dz_};
      const bool on[3] = {pml_x, pml_y, pml_z};
#pragma unroll
      for (int J = 0; J < 3; J++) {
        if (!on[J]) continue;
        const int s = slab_index(a.slab[J], idx[J]);
        if (s < 0) continue;
        const long long pidx = psi_index(a, J, s, i, j, k);
        const float B = a.prof[1][J].B[idx[J]], Cs = a.prof[1][J].C[idx[J]], G = a.prof[1][J].G[idx[J]];
#pragma unroll
        for (int I = 0; I < 3; I++) {
          if (!hasH(MODE, I) || I == J || !hasE(MODE, third(I, J))) continue;
          float* ps = a.psi[1][I][J] + pidx;
          const float psi = *ps;
          *dsum[I] += psi * G;
          *ps = B * psi + Cs * raw[I][J];
        }
      }
    }
    float add0 = 0.f, add1 = 0.f, add2 = 0.f, undo0 = 0.f, undo1 = 0.f, undo2 = 0.f;
    for (int s = 0; s < a.nsrc; s++) {
      const SourceDev& sr = a.src[s];
      if (sr.target < 2 || sr.cell != c) continue;
      const long long t = a.ctrl->t;
      const double v = t < sr.nvals ? sr.vals[t] : 0.0;
      if (sr.target == 3) {
        const float dv = static_cast<float>(v * a.src_scale_b);
        if (sr.comp == 0) dx_ -= dv;
        else if (sr.comp == 1) dy_ -= dv;
        else dz_ -= dv;
      } else {
        const float u = static_cast<float>(a.src_last[s] * a.src_scale_h), ad = static_cast<float>(v * a.src_scale_h);
        if (sr.comp == 0) { undo0 += u; add0 += ad; }
        else if (sr.comp == 1) { undo1 += u; add1 += ad; }
        else { undo2 += u; add2 += ad; }
        a.src_last[s] = v;
      }
    }
    if (a.has_mu) {
      // H = B/(mu_r mu0): the step's flux change scales by 1/mu_r
      int mid = 0;
      if (a.ids) mid = a.ids[c];
      else if (a.bids) mid = a.bids[((k >> a.bshift) * a.nby + (j >> a.bshift)) * a.nbx + (i >> a.bshift)];
      const float im = a.mats[mid].inv_mu;
      dx_ *= im;
      dy_ *= im;
      dz_ *= im;
    }
    if (hasH(MODE, 0)) a.H[0][c] = a.H[0][c] - undo0 - dx_ + add0;
    if (hasH(MODE, 1)) a.H[1][c] = a.H[1][c] - undo1 - dy_ + add1;
    if (hasH(MODE, 2)) a.H[2][c] = a.H[2][c] - undo2 - dz_ + add2;
  }
}

static int kchunk_for(int nz, int blocks_xy) {
  // enough CTAs for ~4 waves of 148 SMs x 4 CTAs, chunks of >= 32 planes
  const int interior = nz - 2;
  int chunks = (148 * 4 * 4 + blocks_xy - 1) / blocks_xy;
  chunks = max(1, min(chunks, interior / 32));
  return (interior + chunks - 1) / chunks;
}

template <int MODE, int MAXP>
static int launch_e_t(const FusedArgs& a, cudaStream_t s) {
  dim3 block(32, kBY, 1);
  const int bx = (a.nx - 2 + 31) / 32, by = (a.ny - 2 + kBY - 1) / kBY;
  int kchunk = 1, bz = 1;
  if (MODE == kThreeD) {
    kchunk = kchunk_for(a.nz, bx * by);
    bz = (a.nz - 2 + kchunk - 1) / kchunk;
  }
  fused_e_kernel<MODE, MAXP><<<dim3(bx, by, bz), block, 0, s>>>(a, kchunk);
  return 1;
}

template <int MODE>
static int launch_e_m(const FusedArgs& a, cudaStream_t s) {
  switch (a.max_poles) {
    case 0: return launch_e_t<MODE, 0>(a, s);
    case -1: return launch_e_t<MODE, -1>(a, s);
    case 1: return launch_e_t<MODE, 1>(a, s);
    default: return launch_e_t<MODE, 2>(a, s);
  }
}

int launch_fused_e(int mode, const FusedArgs& a, cudaStream_t s) {
  switch (mode) {
    case kTE: return launch_e_m<kTE>(a, s);
    case kTM: return launch_e_m<kTM>(a, s);
    default: return launch_e_m<kThreeD>(a, s);
  }
}

template <int MODE>
static int launch_h_t(const FusedArgs& a, cudaStream_t s) {
  dim3 block(32, kBY, 1);
  const int bx = (a.nx - 2 + 31) / 32, by = (a.ny - 2 + kBY - 1) / kBY;
  int kchunk = 1, bz = 1;
  if (MODE == kThreeD) {
    kchunk = kchunk_for(a.nz, bx * by);
    bz = (a.nz - 2 + kchunk - 1) / kchunk;
  }
  fused_h_kernel<MODE><<<dim3(bx, by, bz), block, 0, s>>>(a, kchunk);
  return 1;
}

int launch_fused_h(int mode, const FusedArgs& a, cudaStream_t s) {
  switch (mode) {
    case kTE: return launch_h_t<kTE>(a, s);
    case kTM: return launch_h_t<kTM>(a, s);
    default: return launch_h_t<kThreeD>(a, s);
  }
}

}  // namespace fdtdb
