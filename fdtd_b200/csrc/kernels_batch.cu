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
