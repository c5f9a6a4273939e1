// FP32 fused 3D sweeps, "staged" feeding: one thread per 4-cell group and
// plane, as the flat sweeps, but every global operand of the group is
// requested at thread start with cp.async into the thread's own slots of
// shared memory. The copies need no registers while in flight, so all of a
// thread's loads are outstanding at once however tight the register budget;
// after cp.async.wait_all the thread reads its slots back (each thread reads
// only what it copied itself, so no CTA barrier is needed) and runs the same
// update as the other sweeps (fused3d_common.cuh).
#include <algorithm>

#include "fused3d_common.cuh"

namespace fdtdb {

namespace {

using namespace f3d;
constexpr unsigned kFull = 0xffffffffu;
constexpr int kRowsA = 4;
constexpr int kThreads = 32 * kRowsA;
constexpr int kSlotsE = 12;  // hx_km, hy_km, hx, hy, hz, hx_ym, hz_ym, ex, ey, ez, x-slab psi (2)
// with every material dispersive, the ADE state follows: J (then P) of each
// pole and component
template <int MAXP>
constexpr int pj_slots() {
  return MAXP == 0 ? 0 : (MAXP < 0 ? 3 : 6 * MAXP);
}
constexpr int kSlotsH = 12;  // ex_kp, ey_kp, ex, ey, ez, ex_yp, ez_yp, hx, hy, hz, x-slab psi (2)

__device__ __forceinline__ void cp_async16(float4* dst, const float* src) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(src) : "memory");
}

__device__ __forceinline__ void cp_async4(unsigned* dst, const void* src) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(src) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// the x-slab CPML integrators of a group (two components) into slots
// px[0..3], px[4..7]; only cells inside the slab are copied
__device__ __forceinline__ void stage_x_slab(const FusedArgs& a, const GroupCtx& g, int ft, int k, float* px) {
  if (!g.pml_x) return;
#pragma unroll
  for (int e = 0; e < 4; e++) {
    const int sx = g.ok[e] ? slab_index(a.slab[0], g.x4 + e) : -1;
    if (sx < 0) continue;
    const long long pi = (static_cast<long long>(k) * a.ny + g.j) * a.slab[0].W + sx;
    cp_async4(reinterpret_cast<unsigned*>(px + e), a.psi[ft][1][0] + pi);
    cp_async4(reinterpret_cast<unsigned*>(px + 4 + e), a.psi[ft][2][0] + pi);
  }
}

}  // namespace

// PJ: every material of the grid is dispersive, so the group's J (and P)
// are staged with the fields and all of the thread's loads are in flight at
// once (they are otherwise read per component, after the fields arrive)
template <int MAXP, int MINB, bool PJ>
__global__ void __launch_bounds__(kThreads, MINB) staged_e_kernel(const __grid_constant__ FusedArgs a) {
  extern __shared__ float4 sm[];
  constexpr int kPJ = PJ ? pj_slots<MAXP>() : 0;
  const int lane = threadIdx.x, tid = threadIdx.y * 32 + lane;
  const int x4 = blockIdx.x * 128 + lane * 4;
  const int j = 1 + blockIdx.y * kRowsA + threadIdx.y;
  const int jl = min(j, a.ny - 2);
  const int k = 1 + blockIdx.z;
  const long long sy = a.pitch, sz = static_cast<long long>(a.pitch) * a.ny;
  const long long c = k * sz + jl * sy + x4;
  float4* s = sm + tid;
  unsigned* sid = reinterpret_cast<unsigned*>(sm + (kSlotsE + kPJ) * kThreads) + tid;
  cp_async16(s + 0 * kThreads, a.H[0] + c - sz);
  cp_async16(s + 1 * kThreads, a.H[1] + c - sz);
  cp_async16(s + 2 * kThreads, a.H[0] + c);
  cp_async16(s + 3 * kThreads, a.H[1] + c);
  cp_async16(s + 4 * kThreads, a.H[2] + c);
  cp_async16(s + 5 * kThreads, a.H[0] + c - sy);
  cp_async16(s + 6 * kThreads, a.H[2] + c - sy);
  cp_async16(s + 7 * kThreads, a.E[0] + c);
  cp_async16(s + 8 * kThreads, a.E[1] + c);
  cp_async16(s + 9 * kThreads, a.E[2] + c);
  if (a.ids) cp_async4(sid, a.ids + c);
  if (PJ) {
    constexpr int NP = MAXP < 0 ? 1 : MAXP;
#pragma unroll
    for (int q = 0; q < NP; q++)
#pragma unroll
      for (int I = 0; I < 3; I++) {
        cp_async16(s + (kSlotsE + q * 3 + I) * kThreads, a.J[q][I] + c);
        if (MAXP > 0) cp_async16(s + (kSlotsE + NP * 3 + q * 3 + I) * kThreads, a.P[q][I] + c);
      }
  }
  float hy_xm0 = 0.f, hz_xm0 = 0.f;
  if (lane == 0) {
    hy_xm0 = a.H[1][c - 1];
    hz_xm0 = a.H[2][c - 1];
  }
  const GroupCtx g = make_ctx(a, 0, x4, j, lane, k, k + 1);
  // slots 10 and 11 hold this thread's 8 x-slab floats
  float* px = reinterpret_cast<float*>(sm + 10 * kThreads) + 8 * tid;
  if (g.row_ok) stage_x_slab(a, g, 0, k, px);
  cp_async_wait_all();
  const float4 hy = s[3 * kThreads], hz = s[4 * kThreads];
  const float hy_sh = __shfl_up_sync(kFull, hy.w, 1);
  const float hz_sh = __shfl_up_sync(kFull, hz.w, 1);
  if (lane != 0) {
    hy_xm0 = hy_sh;
    hz_xm0 = hz_sh;
  }
  e_group_update<MAXP>(a, g, k, s[2 * kThreads], hy, hz, s[5 * kThreads], s[6 * kThreads], s[0], s[1 * kThreads],
                       hy_xm0, hz_xm0, s[7 * kThreads], s[8 * kThreads], s[9 * kThreads], a.ids ? *sid : 0u, px,
                       PJ ? s + kSlotsE * kThreads : nullptr, kThreads);
}

template <int MINB, bool MU>
__global__ void __launch_bounds__(kThreads, MINB) staged_h_kernel(const __grid_constant__ FusedArgs a) {
  extern __shared__ float4 sm[];
  const int lane = threadIdx.x, tid = threadIdx.y * 32 + lane;
  const int x4 = blockIdx.x * 128 + lane * 4;
  const int j = 1 + blockIdx.y * kRowsA + threadIdx.y;
  const int jl = min(j, a.ny - 2);
  // planes from the top down, as the flat H sweep
  const int k = a.nz - 2 - blockIdx.z;
  const long long sy = a.pitch, sz = static_cast<long long>(a.pitch) * a.ny;
  const long long c = k * sz + jl * sy + x4;
  float4* s = sm + tid;
  cp_async16(s + 0 * kThreads, a.E[0] + c + sz);
  cp_async16(s + 1 * kThreads, a.E[1] + c + sz);
  cp_async16(s + 2 * kThreads, a.E[0] + c);
  cp_async16(s + 3 * kThreads, a.E[1] + c);
  cp_async16(s + 4 * kThreads, a.E[2] + c);
  cp_async16(s + 5 * kThreads, a.E[0] + c + sy);
  cp_async16(s + 6 * kThreads, a.E[2] + c + sy);
  cp_async16(s + 7 * kThreads, a.H[0] + c);
  cp_async16(s + 8 * kThreads, a.H[1] + c);
  cp_async16(s + 9 * kThreads, a.H[2] + c);
  float ey_xp3 = 0.f, ez_xp3 = 0.f;
  if (lane == 31) {
    ey_xp3 = a.E[1][c + 4];
    ez_xp3 = a.E[2][c + 4];
  }
  const GroupCtx g = make_ctx(a, 1, x4, j, lane, k, k + 1);
  float* px = reinterpret_cast<float*>(sm + 10 * kThreads) + 8 * tid;
  if (g.row_ok) stage_x_slab(a, g, 1, k, px);
  cp_async_wait_all();
  const float4 ey = s[3 * kThreads], ez = s[4 * kThreads];
  const float ey_sh = __shfl_down_sync(kFull, ey.x, 1);
  const float ez_sh = __shfl_down_sync(kFull, ez.x, 1);
  if (lane != 31) {
    ey_xp3 = ey_sh;
    ez_xp3 = ez_sh;
  }
  h_group_update<MU>(a, g, k, s[2 * kThreads], ey, ez, s[5 * kThreads], s[6 * kThreads], s[0], s[1 * kThreads], ey_xp3,
                 ez_xp3, s[7 * kThreads], s[8 * kThreads], s[9 * kThreads], px);
}

// The shared-memory carveout (percent of the largest) that holds `ctas` CTAs
// of `smem` bytes each (plus the 1 KB the runtime reserves per CTA): asking
// for no more leaves the rest of the SM's 256 KB to L1, which holds the
// sweeps' register spills.
static int carveout_for(int ctas, size_t smem) {
  int dev = 0, max_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&max_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
  if (max_sm <= 0) return cudaSharedmemCarveoutMaxShared;
  const size_t need = static_cast<size_t>(ctas) * (smem + 1024);
  return static_cast<int>(std::min<size_t>(100, (need * 100 + max_sm - 1) / max_sm));
}

// CTAs per SM: 7 (6 for two poles) with the ADE state read per component;
// with it staged, as many as the shared memory holds (two poles: 4 x 49.7 KB)
template <int MAXP, bool PJ>
static void staged_e_launch(const FusedArgs& a, cudaStream_t s) {
  dim3 grid(a.pitch / 128, (a.ny - 2 + kRowsA - 1) / kRowsA, a.nz - 2), block(32, kRowsA, 1);
  constexpr int slots = kSlotsE + (PJ ? pj_slots<MAXP>() : 0);
  constexpr int minb = !PJ ? (MAXP >= 2 ? 6 : 7) : (MAXP >= 2 ? 4 : (MAXP == 1 ? 6 : 7));
  const size_t smem = slots * kThreads * sizeof(float4) + kThreads * sizeof(unsigned);
  auto fn = staged_e_kernel<MAXP, minb, PJ>;
  static bool attrs = false;  // once: the shared-memory split that holds minb CTAs, the rest as L1
  if (!attrs) {
    cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, carveout_for(minb, smem));
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    attrs = true;
  }
  fn<<<grid, block, smem, s>>>(a);
}

template <int MAXP>
static void staged_e_dispatch(const FusedArgs& a, cudaStream_t s) {
  if constexpr (MAXP != 0) {
    if (a.all_dispersive) {
      staged_e_launch<MAXP, true>(a, s);
      return;
    }
  }
  staged_e_launch<MAXP, false>(a, s);
}

int launch_staged_e(const FusedArgs& a, cudaStream_t s) {
  switch (a.max_poles) {
    case 0: staged_e_dispatch<0>(a, s); break;
    case -1: staged_e_dispatch<-1>(a, s); break;
    case 1: staged_e_dispatch<1>(a, s); break;
    default: staged_e_dispatch<2>(a, s); break;
  }
  return 1;
}

template <bool MU>
static void staged_h_dispatch(const FusedArgs& a, cudaStream_t s) {
  dim3 grid(a.pitch / 128, (a.ny - 2 + kRowsA - 1) / kRowsA, a.nz - 2), block(32, kRowsA, 1);
  const size_t smem = kSlotsH * kThreads * sizeof(float4);
  static bool carveout = false;
  if (!carveout) {
    cudaFuncSetAttribute(staged_h_kernel<8, MU>, cudaFuncAttributePreferredSharedMemoryCarveout,
                         carveout_for(8, smem));
    carveout = true;
  }
  staged_h_kernel<8, MU><<<grid, block, smem, s>>>(a);
}

int launch_staged_h(const FusedArgs& a, cudaStream_t s) {
  if (a.has_mu) staged_h_dispatch<true>(a, s);
  else staged_h_dispatch<false>(a, s);
  return 1;
}

}  // namespace fdtdb
