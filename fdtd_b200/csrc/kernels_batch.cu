// Batched 2D FP32 grids in one persistent launch.
//
// Many independent TE/TM grids of uneven sizes (each an fdtd_grid set up with
// the ordinary calls) are advanced together by ONE cooperative kernel that
// runs every requested step: the work list holds (grid, tile) items, a tile
// being 128 cells x the grid's item rows (a multiple of the CTA's ROWS, set
// per grid by the tuner from the grid's size); each CTA takes items
// round-robin; the E phase of all grids, a grid
// barrier, the H phase, a barrier, next step. The update per 4-cell group is
// the fused E/H form of kernels_fused.cu restated for 2D with 128-bit access.
//
// The grid barrier spins with a bound: after kBarrierLimit polls a CTA sets
// the batch error flag and returns, and a CTA that sees the flag set returns
// too, so a lost CTA cannot hang the GPU. Loads of cells another CTA may have
// written in the previous phase go through L2 (__ldcg): L1 is not coherent
// across CTAs.
#include "fused3d_common.cuh"

namespace fdtdb {

namespace {

using namespace f3d;
constexpr long long kBarrierLimit = 1LL << 26;

// Loads of the group updates: through L2 only (CG, the persistent kernel,
// whose phases follow one another inside one launch), or cached in L1 as
// well (the per-half-step launches: a launch reads nothing that another CTA
// of the same launch writes, and L1 holds the neighbour rows of a CTA)
template <bool CG>
__device__ __forceinline__ float4 ldg4(const float* p) {
  return CG ? __ldcg(reinterpret_cast<const float4*>(p)) : *reinterpret_cast<const float4*>(p);
}
template <bool CG, typename T>
__device__ __forceinline__ T ldg1(const T* p) {
  return CG ? __ldcg(p) : *p;
}

__device__ bool grid_barrier(BatchCtl* ctl, unsigned nblocks) {
  __syncthreads();
  int ok = 1;
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    volatile unsigned* gen = &ctl->gen;
    volatile int* err = &ctl->error;
    const unsigned g = *gen;
    __threadfence();
    if (atomicAdd(&ctl->count, 1u) == nblocks - 1) {
      ctl->count = 0;
      __threadfence();
      atomicAdd(&ctl->gen, 1u);
    } else {
      long long n = 0;
      while (*gen == g) {
        if (*err) {
          ok = 0;
          break;
        }
        if (++n > kBarrierLimit) {
          atomicOr(&ctl->error, 1);
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
  }
  return __syncthreads_and(ok) != 0;
}

// E update of one 4-cell group of a 2D grid
template <int MODE, int MAXP, bool CG>
__device__ void e_group_2d(const FusedArgs& a, int x4, int j, int lane, long long t) {
  const bool row_ok = j <= a.ny - 2;
  const int jl = min(j, a.ny - 2);
  bool ok[4];
#pragma unroll
  for (int e = 0; e < 4; e++) ok[e] = row_ok && x4 + e >= 1 && x4 + e <= a.nx - 2;
  const long long c = static_cast<long long>(jl) * a.pitch + x4;
  // every operand of the group is requested before any is used: one memory
  // round trip per group (the lane-0 x neighbour and the old E included)
  const int Ie0 = MODE == kTE ? 0 : 2;
  const float4 eo0 = ldg4<CG>(a.E[Ie0] + c);
  const float4 eo1 = MODE == kTE ? ldg4<CG>(a.E[1] + c) : eo0;
  const unsigned ids4 = a.ids ? ldg1<CG>(reinterpret_cast<const unsigned*>(a.ids + c)) : 0u;
  const int Ih = MODE == kTE ? 2 : 1;
  const float hxm_l0 = lane == 0 ? ldg1<CG>(a.H[Ih] + c - 1) : 0.f;
  const float4 fsx = ld4(a.prof[0][0].F + x4);
  const float fsy = a.prof[0][1].F[jl];
  // CPML integrators of the group, requested with the fields
  const int Ipy = MODE == kTE ? 0 : 2, Ipx = MODE == kTE ? 1 : 2;
  const int sj = (row_ok && a.pml_axis[1]) ? slab_index(a.slab[1], j) : -1;
  const long long piy = static_cast<long long>(max(sj, 0)) * a.pitch + x4;
  float4 psy = make_float4(0.f, 0.f, 0.f, 0.f);
  if (sj >= 0) psy = ldg4<CG>(a.psi[0][Ipy][1] + piy);
  // the x-slab integrators of the group: one aligned float4 (Slab::lo4)
  const int sx4 = (row_ok && a.pml_axis[0]) ? slab_group4(a.slab[0], x4) : -1;
  const long long pix = static_cast<long long>(j) * a.slab[0].W4 + max(sx4, 0);
  float4 psx = make_float4(0.f, 0.f, 0.f, 0.f);
  if (sx4 >= 0) psx = ldg4<CG>(a.psi[0][Ipx][0] + pix);
  float4 dX = make_float4(0.f, 0.f, 0.f, 0.f), dY = dX, dZ = dX, rxy = dX, ryx = dX, rzx = dX, rzy = dX;
  if (MODE == kTE) {
    const float4 hz = ldg4<CG>(a.H[2] + c), hz_ym = ldg4<CG>(a.H[2] + c - a.pitch);
    float hz_xm0 = __shfl_up_sync(0xffffffffu, hz.w, 1);
    if (lane == 0) hz_xm0 = hxm_l0;
#pragma unroll
    for (int e = 0; e < 4; e++) {
      set_el(rxy, e, el(hz, e) - el(hz_ym, e));
      set_el(ryx, e, -(el(hz, e) - (e == 0 ? hz_xm0 : el(hz, e - 1))));
      set_el(dX, e, fsy * el(rxy, e));
      set_el(dY, e, el(fsx, e) * el(ryx, e));
    }
  } else {
    const float4 hx = ldg4<CG>(a.H[0] + c), hy = ldg4<CG>(a.H[1] + c), hx_ym = ldg4<CG>(a.H[0] + c - a.pitch);
    float hy_xm0 = __shfl_up_sync(0xffffffffu, hy.w, 1);
    if (lane == 0) hy_xm0 = hxm_l0;
#pragma unroll
    for (int e = 0; e < 4; e++) {
      set_el(rzx, e, el(hy, e) - (e == 0 ? hy_xm0 : el(hy, e - 1)));
      set_el(rzy, e, -(el(hx, e) - el(hx_ym, e)));
      set_el(dZ, e, el(fsx, e) * el(rzx, e) + fsy * el(rzy, e));
    }
  }
  if (!row_ok) return;
  // CPML: y slab rows share the field layout; x slab cells are compact
  if (sj >= 0) {
    const float B = a.prof[0][1].B[j], Cs = a.prof[0][1].C[j], G = a.prof[0][1].G[j];
    float4 ps = psy;
#pragma unroll
    for (int e = 0; e < 4; e++) {
      if (!ok[e]) continue;
      const float raw = MODE == kTE ? el(rxy, e) : el(rzy, e);
      if (MODE == kTE) set_el(dX, e, el(dX, e) + el(ps, e) * G);
      else set_el(dZ, e, el(dZ, e) + el(ps, e) * G);
      set_el(ps, e, B * el(ps, e) + Cs * raw);
    }
    st4(a.psi[0][Ipy][1] + piy, ps);
  }
  if (sx4 >= 0) {
    // cells outside the slab have zero coefficients and keep zero
    const float4 B = ld4(a.prof[0][0].B + x4), Cs = ld4(a.prof[0][0].C + x4), G = ld4(a.prof[0][0].G + x4);
    float4 ps = psx;
#pragma unroll
    for (int e = 0; e < 4; e++) {
      if (!ok[e]) continue;
      const float p = el(psx, e);
      const float raw = MODE == kTE ? el(ryx, e) : el(rzx, e);
      if (MODE == kTE) set_el(dY, e, el(dY, e) + p * el(G, e));
      else set_el(dZ, e, el(dZ, e) + p * el(G, e));
      set_el(ps, e, el(B, e) * p + el(Cs, e) * raw);
    }
    st4(a.psi[0][Ipx][0] + pix, ps);
  }
  // sources and material update (shared with the 3D sweeps)
  float4 uX = make_float4(0.f, 0.f, 0.f, 0.f), uY = uX, uZ = uX, aX = uX, aY = uX, aZ = uX;
  for (int q = 0; q < a.nsrc; q++) {
    const SourceDev& sr = a.src[q];
    if (sr.target > 1 || sr.j != j || sr.i < x4 || sr.i >= x4 + 4) continue;
    const int e = sr.i - x4;
    const double v = t < sr.nvals ? sr.vals[t] : 0.0;
    if (sr.target == 1) {
      const float dv = static_cast<float>(v * a.src_scale_d);
      if (sr.comp == 0) set_el(dX, e, el(dX, e) + dv);
      else if (sr.comp == 1) set_el(dY, e, el(dY, e) + dv);
      else set_el(dZ, e, el(dZ, e) + dv);
    } else {
      const float u = static_cast<float>(a.src_last[q]), ad = static_cast<float>(v);
      if (sr.comp == 0) { set_el(uX, e, el(uX, e) + u); set_el(aX, e, el(aX, e) + ad); }
      else if (sr.comp == 1) { set_el(uY, e, el(uY, e) + u); set_el(aY, e, el(aY, e) + ad); }
      else { set_el(uZ, e, el(uZ, e) + u); set_el(aZ, e, el(aZ, e) + ad); }
      a.src_last[q] = v;
    }
  }
  const bool uniform = !a.ids;
  const MatF32& m0 = a.mats[0];
  float4 ie;
  int mids[4] = {0, 0, 0, 0};
  bool disp = false;
#pragma unroll
  for (int e = 0; e < 4; e++) {
    const int mid = uniform ? 0 : static_cast<int>((ids4 >> (8 * e)) & 0xff);
    mids[e] = mid;
    set_el(ie, e, a.mats[mid].inv_eps);
    if (MAXP != 0 && a.mats[mid].npoles != 0) disp = true;
  }
  if (a.inv_eps_map) {
    const float4 v = ld4(a.inv_eps_map + c);
#pragma unroll
    for (int e = 0; e < 4; e++)
      if (el(v, e) > 0.f && a.mats[mids[e]].npoles == 0) set_el(ie, e, el(v, e));
  }
  if (MODE == kTE) {
    st4(a.E[0] + c, e_comp<MAXP>(a, 0, c, sub4(eo0, uX), dX, ie, ok, disp, uniform, m0, mids, aX));
    st4(a.E[1] + c, e_comp<MAXP>(a, 1, c, sub4(eo1, uY), dY, ie, ok, disp, uniform, m0, mids, aY));
  } else {
    st4(a.E[2] + c, e_comp<MAXP>(a, 2, c, sub4(eo0, uZ), dZ, ie, ok, disp, uniform, m0, mids, aZ));
  }
}

// H update of one 4-cell group of a 2D grid
template <int MODE, bool CG>
__device__ void h_group_2d(const FusedArgs& a, int x4, int j, int lane, long long t) {
  const bool row_ok = j <= a.ny - 2;
  const int jl = min(j, a.ny - 2);
  bool ok[4];
#pragma unroll
  for (int e = 0; e < 4; e++) ok[e] = row_ok && x4 + e >= 1 && x4 + e <= a.nx - 2;
  const long long c = static_cast<long long>(jl) * a.pitch + x4;
  // operands first, as in e_group_2d: the old H and the lane-31 x neighbour too
  const int Ih0 = MODE == kTE ? 2 : 0;
  const float4 ho0 = ldg4<CG>(a.H[Ih0] + c);
  const float4 ho1 = MODE == kTE ? ho0 : ldg4<CG>(a.H[1] + c);
  const int Ie = MODE == kTE ? 1 : 2;
  const float exp_l31 = lane == 31 ? ldg1<CG>(a.E[Ie] + c + 4) : 0.f;
  const float4 fsx = ld4(a.prof[1][0].F + x4);
  const float fsy = a.prof[1][1].F[jl];
  const int Ipy = MODE == kTE ? 2 : 0, Ipx = MODE == kTE ? 2 : 1;
  const int sj = (row_ok && a.pml_axis[1]) ? slab_index(a.slab[1], j) : -1;
  const long long piy = static_cast<long long>(max(sj, 0)) * a.pitch + x4;
  float4 psy = make_float4(0.f, 0.f, 0.f, 0.f);
  if (sj >= 0) psy = ldg4<CG>(a.psi[1][Ipy][1] + piy);
  // the x-slab integrators of the group: one aligned float4 (Slab::lo4)
  const int sx4 = (row_ok && a.pml_axis[0]) ? slab_group4(a.slab[0], x4) : -1;
  const long long pix = static_cast<long long>(j) * a.slab[0].W4 + max(sx4, 0);
  float4 psx = make_float4(0.f, 0.f, 0.f, 0.f);
  if (sx4 >= 0) psx = ldg4<CG>(a.psi[1][Ipx][0] + pix);
  float4 dX = make_float4(0.f, 0.f, 0.f, 0.f), dY = dX, dZ = dX, rxy = dX, ryx = dX, rzx = dX, rzy = dX;
  if (MODE == kTE) {
    const float4 ex = ldg4<CG>(a.E[0] + c), ey = ldg4<CG>(a.E[1] + c), ex_yp = ldg4<CG>(a.E[0] + c + a.pitch);
    float ey_xp3 = __shfl_down_sync(0xffffffffu, ey.x, 1);
    if (lane == 31) ey_xp3 = exp_l31;
#pragma unroll
    for (int e = 0; e < 4; e++) {
      set_el(rzx, e, (e == 3 ? ey_xp3 : el(ey, e + 1)) - el(ey, e));
      set_el(rzy, e, -(el(ex_yp, e) - el(ex, e)));
      set_el(dZ, e, el(fsx, e) * el(rzx, e) + fsy * el(rzy, e));
    }
  } else {
    const float4 ez = ldg4<CG>(a.E[2] + c), ez_yp = ldg4<CG>(a.E[2] + c + a.pitch);
    float ez_xp3 = __shfl_down_sync(0xffffffffu, ez.x, 1);
    if (lane == 31) ez_xp3 = exp_l31;
#pragma unroll
    for (int e = 0; e < 4; e++) {
      set_el(rxy, e, el(ez_yp, e) - el(ez, e));
      set_el(ryx, e, -((e == 3 ? ez_xp3 : el(ez, e + 1)) - el(ez, e)));
      set_el(dX, e, fsy * el(rxy, e));
      set_el(dY, e, el(fsx, e) * el(ryx, e));
    }
  }
  if (!row_ok) return;
  if (sj >= 0) {
    const float B = a.prof[1][1].B[j], Cs = a.prof[1][1].C[j], G = a.prof[1][1].G[j];
    float4 ps = psy;
#pragma unroll
    for (int e = 0; e < 4; e++) {
      if (!ok[e]) continue;
      const float raw = MODE == kTE ? el(rzy, e) : el(rxy, e);
      if (MODE == kTE) set_el(dZ, e, el(dZ, e) + el(ps, e) * G);
      else set_el(dX, e, el(dX, e) + el(ps, e) * G);
      set_el(ps, e, B * el(ps, e) + Cs * raw);
    }
    st4(a.psi[1][Ipy][1] + piy, ps);
  }
  if (sx4 >= 0) {
    const float4 B = ld4(a.prof[1][0].B + x4), Cs = ld4(a.prof[1][0].C + x4), G = ld4(a.prof[1][0].G + x4);
    float4 ps = psx;
#pragma unroll
    for (int e = 0; e < 4; e++) {
      if (!ok[e]) continue;
      const float p = el(psx, e);
      const float raw = MODE == kTE ? el(rzx, e) : el(ryx, e);
      if (MODE == kTE) set_el(dZ, e, el(dZ, e) + p * el(G, e));
      else set_el(dY, e, el(dY, e) + p * el(G, e));
      set_el(ps, e, el(B, e) * p + el(Cs, e) * raw);
    }
    st4(a.psi[1][Ipx][0] + pix, ps);
  }
  float4 uX = make_float4(0.f, 0.f, 0.f, 0.f), uY = uX, uZ = uX, aX = uX, aY = uX, aZ = uX;
  for (int q = 0; q < a.nsrc; q++) {
    const SourceDev& sr = a.src[q];
    if (sr.target < 2 || sr.j != j || sr.i < x4 || sr.i >= x4 + 4) continue;
    const int e = sr.i - x4;
    const double v = t < sr.nvals ? sr.vals[t] : 0.0;
    if (sr.target == 3) {
      const float dv = static_cast<float>(v * a.src_scale_b);
      if (sr.comp == 0) set_el(dX, e, el(dX, e) - dv);
      else if (sr.comp == 1) set_el(dY, e, el(dY, e) - dv);
      else set_el(dZ, e, el(dZ, e) - dv);
    } else {
      const float u = static_cast<float>(a.src_last[q] * a.src_scale_h), ad = static_cast<float>(v * a.src_scale_h);
      if (sr.comp == 0) { set_el(uX, e, el(uX, e) + u); set_el(aX, e, el(aX, e) + ad); }
      else if (sr.comp == 1) { set_el(uY, e, el(uY, e) + u); set_el(aY, e, el(aY, e) + ad); }
      else { set_el(uZ, e, el(uZ, e) + u); set_el(aZ, e, el(aZ, e) + ad); }
      a.src_last[q] = v;
    }
  }
  auto upd = [&](int I, float4 h, float4 d, float4 u, float4 ad) {
#pragma unroll
    for (int e = 0; e < 4; e++)
      if (ok[e]) set_el(h, e, el(h, e) - el(u, e) - el(d, e) + el(ad, e));
    st4(a.H[I] + c, h);
  };
  if (MODE == kTE) {
    upd(2, ho0, dZ, uZ, aZ);
  } else {
    upd(0, ho0, dX, uX, aX);
    upd(1, ho1, dY, uY, aY);
  }
}

}  // namespace

// item = (grid index << 24) | tile; tile = ty * (pitch/128) + tx
template <int MODE, int MAXP, int ROWS>
__global__ void __launch_bounds__(32 * ROWS) batch_kernel(const FusedArgs* __restrict__ grids,
                                                          const unsigned* __restrict__ items, int nitems,
                                                          BatchCtl* ctl, int nsteps) {
  const int lane = threadIdx.x, ty = threadIdx.y;
  // every grid of a batch has taken the same number of steps; the counters
  // are advanced by a separate kernel after this one
  const long long t0 = grids[0].ctrl->t;
  for (int s = 0; s < nsteps; s++) {
    const long long t = t0 + s;
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
      const unsigned w = items[it];
      const FusedArgs& a = grids[w >> 24];
      const int tiles_x = a.pitch / 128, tile = static_cast<int>(w & 0xffffffu);
      const int R = a.item_rows > 0 ? a.item_rows : ROWS;
      const int x4 = (tile % tiles_x) * 128 + 4 * lane, j = 1 + (tile / tiles_x) * R + ty;
      for (int r = 0; r < R; r += ROWS) e_group_2d<MODE, MAXP, true>(a, x4, j + r, lane, t);
    }
    if (!grid_barrier(ctl, gridDim.x)) return;
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
      const unsigned w = items[it];
      const FusedArgs& a = grids[w >> 24];
      const int tiles_x = a.pitch / 128, tile = static_cast<int>(w & 0xffffffu);
      const int R = a.item_rows > 0 ? a.item_rows : ROWS;
      const int x4 = (tile % tiles_x) * 128 + 4 * lane, j = 1 + (tile / tiles_x) * R + ty;
      for (int r = 0; r < R; r += ROWS) h_group_2d<MODE, true>(a, x4, j + r, lane, t);
    }
    if (!grid_barrier(ctl, gridDim.x)) return;
  }
}

// The same update, one CTA per item and one launch per half step (the batch's
// "phase" launch mode): the hardware block scheduler keeps many items in
// flight per SM where the persistent kernel walks its items one after
// another. `s` is the step offset from the counters, which a separate kernel
// advances after the last step of a launch sequence.
template <int MODE, int MAXP, int ROWS, int PHASE>
__global__ void __launch_bounds__(32 * ROWS) batch_phase_kernel(const FusedArgs* __restrict__ grids,
                                                                const unsigned* __restrict__ items, int s) {
  const int lane = threadIdx.x, ty = threadIdx.y;
  const unsigned w = items[blockIdx.x];
  const FusedArgs& a = grids[w >> 24];
  const long long t = grids[0].ctrl->t + s;
  const int tiles_x = a.pitch / 128, tile = static_cast<int>(w & 0xffffffu);
  const int R = a.item_rows > 0 ? a.item_rows : ROWS;
  const int x4 = (tile % tiles_x) * 128 + 4 * lane, j = 1 + (tile / tiles_x) * R + ty;
  for (int r = 0; r < R; r += ROWS) {
    if (PHASE == 0) e_group_2d<MODE, MAXP, false>(a, x4, j + r, lane, t);
    else h_group_2d<MODE, false>(a, x4, j + r, lane, t);
  }
}

// ---------------------------------------------------------------------------
// Temporal blocking: T whole steps per launch from shared memory.
//
// A CTA loads a window of kTbW x kTbH cells of one grid (every field
// component of the mode, the cells' 1/eps, the four CPML integrators) into
// shared memory, advances the window T steps there, and writes back the
// inner tile that T steps leave exact: a step's dependence reaches one cell
// in every direction (E from H at i-1, j-1; H from E at i+1, j+1), so the
// values within T cells of the window's edges (those inside the grid) go
// stale while the tile (kTbW - 2T) x (kTbH - 2T) stays exact. The tiles
// cover every cell of every grid once; the windows overlap, so a launch
// reads one copy of the state and writes the other (the batch keeps a second
// copy), and launches come in pairs that end on the grids' own arrays.
// Non-dispersive grids with sources inside their interiors only; the per-cell
// arithmetic is e_group_2d's and h_group_2d's, in the same order.
constexpr int kTbW = 64, kTbH = 32, kTbTy = 4;  // window; CTA of 64 x 4 threads, 8 rows each
constexpr int kTbRows = kTbH / kTbTy;

struct TbSrc {
  int lx, ly, q;
};

__device__ __forceinline__ double src_value(const SourceDev& sr, long long t) {
  return t >= 0 && t < sr.nvals ? sr.vals[t] : 0.0;
}

template <int MODE, int T>
__global__ void __launch_bounds__(kTbW * kTbTy, 3) batch_tb_kernel(const FusedArgs* __restrict__ rd,
                                                                  const FusedArgs* __restrict__ wr,
                                                                  const unsigned* __restrict__ items, int s) {
  constexpr int OW = kTbW - 2 * T, OH = kTbH - 2 * T;
  constexpr int N = kTbW * kTbH;
  // F[0..2]: TE Ex, Ey, Hz; TM Ez, Hx, Hy. PS[0..3]: the E integrators of
  // the y and x slabs, then H's. YP[ft][0..3][row]: F, B, C, G of the y axis.
  extern __shared__ float tb_sm[];
  float* F = tb_sm;
  float* IE = tb_sm + 3 * N;
  float* PS = tb_sm + 4 * N;
  __shared__ float YP[2][4][kTbH];
  __shared__ int YS[kTbH];  // the row is in the y slab
  __shared__ TbSrc srcs[kMaxSources];
  __shared__ int nsl;

  const unsigned w = items[blockIdx.x];
  const FusedArgs& a = rd[w >> 24];
  const FusedArgs& b = wr[w >> 24];
  const int nx = a.nx, ny = a.ny;
  const long long pitch = a.pitch;
  const int tiles_x = (nx + OW - 1) / OW, tile = static_cast<int>(w & 0xffffffu);
  const int x0 = (tile % tiles_x) * OW - T, y0 = (tile / tiles_x) * OH - T;
  const long long t0 = rd[0].ctrl->t + s;
  constexpr bool TE = MODE == kTE;
  const float* src0 = TE ? a.E[0] : a.E[2];
  const float* src1 = TE ? a.E[1] : a.H[0];
  const float* src2 = TE ? a.H[2] : a.H[1];
  const float* psrc[4] = {a.psi[0][TE ? 0 : 2][1], a.psi[0][TE ? 1 : 2][0], a.psi[1][TE ? 2 : 0][1],
                          a.psi[1][TE ? 2 : 1][0]};

  const int tid = threadIdx.y * kTbW + threadIdx.x;
  if (tid == 0) {
    int n = 0;
    for (int q = 0; q < a.nsrc; q++) {
      const int lx = a.src[q].i - x0, ly = a.src[q].j - y0;
      if (lx >= 0 && lx < kTbW && ly >= 0 && ly < kTbH) srcs[n++] = {lx, ly, q};
    }
    nsl = n;
  }
  if (tid < 2 * kTbH) {
    const int ft = tid / kTbH, ly = tid % kTbH, gy = y0 + ly;
    const bool rowok = gy >= 1 && gy <= ny - 2;
    const int sj = (rowok && a.pml_axis[1]) ? slab_index(a.slab[1], gy) : -1;
    YP[ft][0][ly] = rowok ? a.prof[ft][1].F[gy] : 0.f;
    YP[ft][1][ly] = sj >= 0 ? a.prof[ft][1].B[gy] : 0.f;
    YP[ft][2][ly] = sj >= 0 ? a.prof[ft][1].C[gy] : 0.f;
    YP[ft][3][ly] = sj >= 0 ? a.prof[ft][1].G[gy] : 0.f;
    if (ft == 0) YS[ly] = sj >= 0;
  }
  // this thread's column and its x profiles
  const int lx = threadIdx.x, gx = x0 + lx;
  const bool col_in = gx >= 0 && gx < nx;
  const bool col_ok = gx >= 1 && gx <= nx - 2;
  const int sx4 = (col_in && a.pml_axis[0]) ? slab_group4(a.slab[0], gx & ~3) : -1;
  float fx[2] = {0.f, 0.f}, bx[2] = {0.f, 0.f}, cx[2] = {0.f, 0.f}, gxp[2] = {0.f, 0.f};
#pragma unroll
  for (int ft = 0; ft < 2; ft++) {
    if (col_ok) fx[ft] = a.prof[ft][0].F[gx];
    if (sx4 >= 0) {
      bx[ft] = a.prof[ft][0].B[gx];
      cx[ft] = a.prof[ft][0].C[gx];
      gxp[ft] = a.prof[ft][0].G[gx];
    }
  }
  const MatF32* mats = a.mats;
#pragma unroll
  for (int r = 0; r < kTbRows; r++) {
    const int ly = threadIdx.y + kTbTy * r, gy = y0 + ly, l = ly * kTbW + lx;
    const bool in = col_in && gy >= 0 && gy < ny;
    const long long c = gy * pitch + gx;
    float f0 = 0.f, f1 = 0.f, f2 = 0.f, ie = 0.f, p0 = 0.f, p1 = 0.f, p2 = 0.f, p3 = 0.f;
    if (in) {
      f0 = src0[c];
      f1 = src1[c];
      f2 = src2[c];
      const int mid = a.ids ? a.ids[c] : 0;
      ie = mats[mid].inv_eps;
      if (a.inv_eps_map) {
        const float v = a.inv_eps_map[c];
        if (v > 0.f && mats[mid].npoles == 0) ie = v;
      }
      if (gy >= 1 && gy <= ny - 2) {
        const int sj = a.pml_axis[1] ? slab_index(a.slab[1], gy) : -1;
        if (sj >= 0) {
          p0 = psrc[0][sj * pitch + gx];
          p2 = psrc[2][sj * pitch + gx];
        }
        if (sx4 >= 0) {
          const long long pi = gy * static_cast<long long>(a.slab[0].W4) + sx4 + (gx & 3);
          p1 = psrc[1][pi];
          p3 = psrc[3][pi];
        }
      }
    }
    F[l] = f0;
    F[N + l] = f1;
    F[2 * N + l] = f2;
    IE[l] = ie;
    PS[l] = p0;
    PS[N + l] = p1;
    PS[2 * N + l] = p2;
    PS[3 * N + l] = p3;
  }
  __syncthreads();

  for (int st = 0; st < T; st++) {
    const long long t = t0 + st;
    // E half
#pragma unroll
    for (int r = 0; r < kTbRows; r++) {
      const int ly = threadIdx.y + kTbTy * r, gy = y0 + ly, l = ly * kTbW + lx;
      if (!(col_ok && lx >= 1 && ly >= 1 && gy >= 1 && gy <= ny - 2)) continue;
      const float fsy = YP[0][0][ly];
      const bool sy = YS[ly];
      float dX = 0.f, dY = 0.f, dZ = 0.f, rxy = 0.f, ryx = 0.f, rzx = 0.f, rzy = 0.f;
      if (TE) {
        const float hz = F[2 * N + l], hz_ym = F[2 * N + l - kTbW], hz_xm = F[2 * N + l - 1];
        rxy = hz - hz_ym;
        ryx = -(hz - hz_xm);
        dX = fsy * rxy;
        dY = fx[0] * ryx;
      } else {
        const float hx = F[N + l], hy = F[2 * N + l], hx_ym = F[N + l - kTbW], hy_xm = F[2 * N + l - 1];
        rzx = hy - hy_xm;
        rzy = -(hx - hx_ym);
        dZ = fx[0] * rzx + fsy * rzy;
      }
      if (sy) {
        const float B = YP[0][1][ly], Cs = YP[0][2][ly], G = YP[0][3][ly];
        const float ps = PS[l];
        const float raw = TE ? rxy : rzy;
        if (TE) dX = dX + ps * G;
        else dZ = dZ + ps * G;
        PS[l] = B * ps + Cs * raw;
      }
      if (sx4 >= 0) {
        const float p = PS[N + l];
        const float raw = TE ? ryx : rzx;
        if (TE) dY = dY + p * gxp[0];
        else dZ = dZ + p * gxp[0];
        PS[N + l] = bx[0] * p + cx[0] * raw;
      }
      float uX = 0.f, uY = 0.f, uZ = 0.f, aX = 0.f, aY = 0.f, aZ = 0.f;
      for (int k = 0; k < nsl; k++) {
        if (srcs[k].lx != lx || srcs[k].ly != ly) continue;
        const int q = srcs[k].q;
        const SourceDev& sr = a.src[q];
        if (sr.target > 1) continue;
        const double v = src_value(sr, t);
        if (sr.target == 1) {
          const float dv = static_cast<float>(v * a.src_scale_d);
          if (sr.comp == 0) dX = dX + dv;
          else if (sr.comp == 1) dY = dY + dv;
          else dZ = dZ + dv;
        } else {
          const float u = static_cast<float>(st == 0 ? a.src_last[q] : src_value(sr, t - 1)),
                      ad = static_cast<float>(v);
          if (sr.comp == 0) { uX = uX + u; aX = aX + ad; }
          else if (sr.comp == 1) { uY = uY + u; aY = aY + ad; }
          else { uZ = uZ + u; aZ = aZ + ad; }
        }
      }
      const float ie = IE[l];
      if (TE) {
        const float ex = F[l] - uX, ey = F[N + l] - uY;
        const float exn = ex + ie * dX, eyn = ey + ie * dY;
        F[l] = exn + aX;
        F[N + l] = eyn + aY;
      } else {
        const float ez = F[l] - uZ;
        const float ezn = ez + ie * dZ;
        F[l] = ezn + aZ;
      }
    }
    __syncthreads();
    // H half
#pragma unroll
    for (int r = 0; r < kTbRows; r++) {
      const int ly = threadIdx.y + kTbTy * r, gy = y0 + ly, l = ly * kTbW + lx;
      if (!(col_ok && lx <= kTbW - 2 && ly <= kTbH - 2 && gy >= 1 && gy <= ny - 2)) continue;
      const float fsy = YP[1][0][ly];
      const bool sy = YS[ly];
      float dX = 0.f, dY = 0.f, dZ = 0.f, rxy = 0.f, ryx = 0.f, rzx = 0.f, rzy = 0.f;
      if (TE) {
        const float ex = F[l], ey = F[N + l], ex_yp = F[l + kTbW], ey_xp = F[N + l + 1];
        rzx = ey_xp - ey;
        rzy = -(ex_yp - ex);
        dZ = fx[1] * rzx + fsy * rzy;
      } else {
        const float ez = F[l], ez_yp = F[l + kTbW], ez_xp = F[l + 1];
        rxy = ez_yp - ez;
        ryx = -(ez_xp - ez);
        dX = fsy * rxy;
        dY = fx[1] * ryx;
      }
      if (sy) {
        const float B = YP[1][1][ly], Cs = YP[1][2][ly], G = YP[1][3][ly];
        const float ps = PS[2 * N + l];
        const float raw = TE ? rzy : rxy;
        if (TE) dZ = dZ + ps * G;
        else dX = dX + ps * G;
        PS[2 * N + l] = B * ps + Cs * raw;
      }
      if (sx4 >= 0) {
        const float p = PS[3 * N + l];
        const float raw = TE ? rzx : ryx;
        if (TE) dZ = dZ + p * gxp[1];
        else dY = dY + p * gxp[1];
        PS[3 * N + l] = bx[1] * p + cx[1] * raw;
      }
      float uX = 0.f, uY = 0.f, uZ = 0.f, aX = 0.f, aY = 0.f, aZ = 0.f;
      for (int k = 0; k < nsl; k++) {
        if (srcs[k].lx != lx || srcs[k].ly != ly) continue;
        const int q = srcs[k].q;
        const SourceDev& sr = a.src[q];
        if (sr.target < 2) continue;
        const double v = src_value(sr, t);
        if (sr.target == 3) {
          const float dv = static_cast<float>(v * a.src_scale_b);
          if (sr.comp == 0) dX = dX - dv;
          else if (sr.comp == 1) dY = dY - dv;
          else dZ = dZ - dv;
        } else {
          const double last = st == 0 ? a.src_last[q] : src_value(sr, t - 1);
          const float u = static_cast<float>(last * a.src_scale_h), ad = static_cast<float>(v * a.src_scale_h);
          if (sr.comp == 0) { uX = uX + u; aX = aX + ad; }
          else if (sr.comp == 1) { uY = uY + u; aY = aY + ad; }
          else { uZ = uZ + u; aZ = aZ + ad; }
        }
      }
      if (TE) {
        F[2 * N + l] = F[2 * N + l] - uZ - dZ + aZ;
      } else {
        F[N + l] = F[N + l] - uX - dX + aX;
        F[2 * N + l] = F[2 * N + l] - uY - dY + aY;
      }
    }
    __syncthreads();
  }

  // the exact tile back, into the other copy of the state
  float* dst0 = TE ? b.E[0] : b.E[2];
  float* dst1 = TE ? b.E[1] : b.H[0];
  float* dst2 = TE ? b.H[2] : b.H[1];
  float* pdst[4] = {b.psi[0][TE ? 0 : 2][1], b.psi[0][TE ? 1 : 2][0], b.psi[1][TE ? 2 : 0][1],
                    b.psi[1][TE ? 2 : 1][0]};
  const bool col_own = col_in && lx >= T && lx < T + OW;
#pragma unroll
  for (int r = 0; r < kTbRows; r++) {
    const int ly = threadIdx.y + kTbTy * r, gy = y0 + ly, l = ly * kTbW + lx;
    if (!(col_own && ly >= T && ly < T + OH && gy >= 0 && gy < ny)) continue;
    const long long c = gy * pitch + gx;
    dst0[c] = F[l];
    dst1[c] = F[N + l];
    dst2[c] = F[2 * N + l];
    if (gy >= 1 && gy <= ny - 2) {
      const int sj = a.pml_axis[1] ? slab_index(a.slab[1], gy) : -1;
      if (sj >= 0) {
        pdst[0][sj * pitch + gx] = PS[l];
        pdst[2][sj * pitch + gx] = PS[2 * N + l];
      }
      if (sx4 >= 0) {
        const long long pi = gy * static_cast<long long>(a.slab[0].W4) + sx4 + (gx & 3);
        pdst[1][pi] = PS[N + l];
        pdst[3][pi] = PS[3 * N + l];
      }
    }
  }
  // the soft sources' last values, by the tile that holds the source cell
  if (tid == 0) {
    for (int k = 0; k < nsl; k++) {
      const int sl = srcs[k].lx, sly = srcs[k].ly;
      if (sl < T || sl >= T + OW || sly < T || sly >= T + OH) continue;
      const SourceDev& sr = a.src[srcs[k].q];
      if (sr.target == 0 || sr.target == 2) b.src_last[srcs[k].q] = src_value(sr, t0 + T - 1);
    }
  }
}

template <int MODE, int T>
static int tb_launch(const FusedArgs* rd, const FusedArgs* wr, const unsigned* items, int nitems, int s,
                     cudaStream_t st) {
  constexpr size_t smem = 8 * kTbW * kTbH * sizeof(float);
  auto fn = batch_tb_kernel<MODE, T>;
  // the largest shared-memory split: three 65 KB windows per SM
  once_per_device(reinterpret_cast<const void*>(fn), [&] {
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
  });
  fn<<<nitems, dim3(kTbW, kTbTy), smem, st>>>(rd, wr, items, s);
  return 1;
}

template <int MODE, int MAXP, int ROWS>
static void* batch_fn() {
  return reinterpret_cast<void*>(batch_kernel<MODE, MAXP, ROWS>);
}

template <int MODE, int MAXP, int ROWS>
static void* phase_fn(int phase) {
  return phase == 0 ? reinterpret_cast<void*>(batch_phase_kernel<MODE, MAXP, ROWS, 0>)
                    : reinterpret_cast<void*>(batch_phase_kernel<MODE, MAXP, ROWS, 1>);
}

void* batch_phase_ptr(int mode, int maxp, int rows, int phase) {
#define FDTD_PHASE_ROWS(M, P)                    \
  switch (rows) {                                \
    case 1: return phase_fn<M, P, 1>(phase);     \
    case 2: return phase_fn<M, P, 2>(phase);     \
    case 4: return phase_fn<M, P, 4>(phase);     \
    default: return phase_fn<M, P, 8>(phase);    \
  }
#define FDTD_PHASE_POLES(M)                      \
  switch (maxp) {                                \
    case 0: FDTD_PHASE_ROWS(M, 0)                \
    case -1: FDTD_PHASE_ROWS(M, -1)              \
    case 1: FDTD_PHASE_ROWS(M, 1)                \
    default: FDTD_PHASE_ROWS(M, 2)               \
  }
  if (mode == kTE) FDTD_PHASE_POLES(kTE)
  FDTD_PHASE_POLES(kTM)
#undef FDTD_PHASE_POLES
#undef FDTD_PHASE_ROWS
}

int batch_tb_tile(int depth, int* tw, int* th) {
  if (depth < 1 || 2 * depth >= kTbH) return 0;
  *tw = kTbW - 2 * depth;
  *th = kTbH - 2 * depth;
  return 1;
}

int launch_batch_tb(int mode, int depth, const FusedArgs* rd, const FusedArgs* wr, const unsigned* items,
                    int nitems, int s, cudaStream_t st) {
  if (nitems <= 0) return 0;
  const bool te = mode == kTE;
  switch (depth) {
    case 2: return te ? tb_launch<kTE, 2>(rd, wr, items, nitems, s, st) : tb_launch<kTM, 2>(rd, wr, items, nitems, s, st);
    case 3: return te ? tb_launch<kTE, 3>(rd, wr, items, nitems, s, st) : tb_launch<kTM, 3>(rd, wr, items, nitems, s, st);
    case 4: return te ? tb_launch<kTE, 4>(rd, wr, items, nitems, s, st) : tb_launch<kTM, 4>(rd, wr, items, nitems, s, st);
    default: return 0;
  }
}

void* batch_kernel_ptr(int mode, int maxp, int rows) {
#define FDTD_BATCH_ROWS(M, P)                 \
  switch (rows) {                             \
    case 1: return batch_fn<M, P, 1>();       \
    case 2: return batch_fn<M, P, 2>();       \
    case 4: return batch_fn<M, P, 4>();       \
    default: return batch_fn<M, P, 8>();      \
  }
#define FDTD_BATCH_POLES(M)                   \
  switch (maxp) {                             \
    case 0: FDTD_BATCH_ROWS(M, 0)             \
    case -1: FDTD_BATCH_ROWS(M, -1)           \
    case 1: FDTD_BATCH_ROWS(M, 1)             \
    default: FDTD_BATCH_ROWS(M, 2)            \
  }
  if (mode == kTE) {
    FDTD_BATCH_POLES(kTE)
  }
  FDTD_BATCH_POLES(kTM)
#undef FDTD_BATCH_POLES
#undef FDTD_BATCH_ROWS
}

}  // namespace fdtdb
