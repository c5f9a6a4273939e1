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

// the x-slab CPML integrators of a group (two components, one aligned
// float4 each) into the slots px[0..3], px[4..7]
__device__ __forceinline__ void stage_x_slab(const FusedArgs& a, const GroupCtx& g, int ft, int k, float* px) {
  if (g.sx4 < 0) return;
  const long long pi = (static_cast<long long>(k) * a.ny + g.j) * a.slab[0].W4 + g.sx4;
  cp_async16(reinterpret_cast<float4*>(px), a.psi[ft][1][0] + pi);
  cp_async16(reinterpret_cast<float4*>(px + 4), a.psi[ft][2][0] + pi);
}

}  // namespace

// The E update of one tile: the 4-cell groups of x block bx (128 cells),
// rows 1 + 4 by .. 4 + 4 by, plane k; one group per thread of the CTA's 128.
// PJ: every material of the grid is dispersive, so the group's J (and P)
// are staged with the fields and all of the thread's loads are in flight at
// once (they are otherwise read per component, after the fields arrive)
struct NoHook {
  __device__ void operator()() const {}
};

// hook() runs after every copy of the tile has been requested, before the
// wait for them (the one-launch kernel does its bookkeeping there).
template <int MAXP, bool PJ, class Hook = NoHook>
__device__ __forceinline__ void e_tile(const FusedArgs& a, int bx, int by, int k, float4* sm, Hook hook = Hook()) {
  constexpr int kPJ = PJ ? pj_slots<MAXP>() : 0;
  const int lane = threadIdx.x, tid = threadIdx.y * 32 + lane;
  const int x4 = bx * 128 + lane * 4;
  const int j = 1 + by * kRowsA + threadIdx.y;
  const int jl = min(j, a.ny - 2);
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
  hook();
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

template <int MAXP, int MINB, bool PJ>
__global__ void __launch_bounds__(kThreads, MINB) staged_e_kernel(const __grid_constant__ FusedArgs a) {
  extern __shared__ float4 sm[];
  e_tile<MAXP, PJ>(a, blockIdx.x, blockIdx.y, a.kbeg + blockIdx.z, sm);
}

// The H update of one tile (as e_tile).
template <bool MU>
__device__ __forceinline__ void h_tile(const FusedArgs& a, int bx, int by, int k, float4* sm) {
  const int lane = threadIdx.x, tid = threadIdx.y * 32 + lane;
  const int x4 = bx * 128 + lane * 4;
  const int j = 1 + by * kRowsA + threadIdx.y;
  const int jl = min(j, a.ny - 2);
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

template <int MINB, bool MU>
__global__ void __launch_bounds__(kThreads, MINB) staged_h_kernel(const __grid_constant__ FusedArgs a) {
  extern __shared__ float4 sm[];
  // planes from the top down, as the flat H sweep
  h_tile<MU>(a, blockIdx.x, blockIdx.y, a.kend - 1 - blockIdx.z, sm);
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
  dim3 grid(a.pitch / 128, (a.ny - 2 + kRowsA - 1) / kRowsA, a.kend - a.kbeg), block(32, kRowsA, 1);
  constexpr int slots = kSlotsE + (PJ ? pj_slots<MAXP>() : 0);
  constexpr int minb = !PJ ? (MAXP >= 2 ? 6 : 7) : (MAXP >= 2 ? 4 : (MAXP == 1 ? 6 : 7));
  const size_t smem = slots * kThreads * sizeof(float4) + kThreads * sizeof(unsigned);
  auto fn = staged_e_kernel<MAXP, minb, PJ>;
  // once per device: the shared-memory split that holds minb CTAs, the rest as L1
  once_per_device(reinterpret_cast<const void*>(fn), [&] {
    cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, carveout_for(minb, smem));
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  });
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
  dim3 grid(a.pitch / 128, (a.ny - 2 + kRowsA - 1) / kRowsA, a.kend - a.kbeg), block(32, kRowsA, 1);
  const size_t smem = kSlotsH * kThreads * sizeof(float4);
  once_per_device(reinterpret_cast<const void*>(staged_h_kernel<8, MU>), [&] {
    cudaFuncSetAttribute(staged_h_kernel<8, MU>, cudaFuncAttributePreferredSharedMemoryCarveout, carveout_for(8, smem));
  });
  staged_h_kernel<8, MU><<<grid, block, smem, s>>>(a);
}

int launch_staged_h(const FusedArgs& a, cudaStream_t s) {
  if (a.has_mu) staged_h_dispatch<true>(a, s);
  else staged_h_dispatch<false>(a, s);
  return 1;
}

// ---------------------------------------------------------------------------
// The whole step in one launch (staged_eh_kernel).
//
// The two sweeps read each E and H word twice per step: the E sweep reads H
// and E, the H sweep E and H again. Here one persistent launch runs both, in
// an order that keeps what the H items read in L2: work items are tiles of
// one plane (128 cells x 8 rows) of one sweep, taken round-robin by the
// resident CTAs in the order
//   E(1) .. E(lag),  E(lag+1) H(1),  E(lag+2) H(2),  ..,  E(np) H(np-lag),
//   H(np-lag+1) .. H(np)
// (each a batch of every tile of the plane), so H of plane k runs about lag
// planes after E of plane k has stored the E it reads, and the E and H of
// the planes in between are still in L2. An E item updates its two 4-row
// halves one after the other (the E update stages 24 operands per group,
// which is what the shared memory holds); an H item stages both halves at
// once (12 operands per group each), so the H updates keep as many copies in
// flight per SM as the standalone H sweep does with twice the CTAs.
//
// Dependences. E of tile t at plane k reads H at planes k and k-1 of t, and
// at plane k of t's x-1 and y-1 neighbours; H of tile t at plane k reads E at
// planes k and k+1 of t and at plane k of the x+1 and y+1 neighbours, and
// overwrites the H that the E tiles at (k, t), (k, t+x), (k, t+y) and
// (k+1, t) read. So H(k, t) runs once those four E tiles are done: each E
// tile publishes the launch's epoch in flags[k][t], and an H tile starts
// reading E only once its four flags hold it. Every dependence points to an
// earlier item, and every CTA is resident (cooperative launch), so the
// earliest unfinished item can always run: no cycle of waits. Each wait is
// bounded; on expiry the kernel sets bit 1 of the grid's error flags and
// stops waiting for the rest of the launch (the step's result is then
// wrong, but the launch ends). E values that another CTA wrote in this
// launch are read through L2 only (cp.async.cg, ld.global.cg).
//
// The bookkeeping is the CTA's first thread's, off the copies' path:
// * an E tile's flag is stored (release: fence, then a relaxed store) during
//   the CTA's next item, once that item's copies are in flight, so the
//   fence's wait for the E tile's stores overlaps the next loads; it is
//   always published before the CTA waits for anything, and at the end, so
//   no CTA waits while holding an unpublished flag;
// * when the CTA's next item is an H tile, its four flags are read (relaxed
//   loads, then the fence: an acquire) during the current item; if all hold
//   the epoch, that H tile starts its E copies without a wait (flags only
//   move forward). The outcome reaches the CTA through shared memory and
//   the barrier that ends every item.
//
// The epoch is read from device memory at launch and advanced by the step
// counter's kernel after it, never reset, so flags of an earlier launch
// never satisfy a later one.
namespace {

constexpr int kRowsEH = 2 * kRowsA;  // rows of an item's tile: two 4-row halves
constexpr int kDepPolls = 1 << 18;   // a few tenths of a second with the back-off below

__device__ __forceinline__ unsigned ld_relaxed_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_relaxed_u32(unsigned* p, unsigned v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

__device__ __forceinline__ bool reached(unsigned v, unsigned target) { return static_cast<int>(v - target) >= 0; }

// Waits (bounded) until the flags f[0], f[o1], f[o2], f[o3] have all
// reached `target` (an offset of 0 stands for a dependence the tile does not
// have), reading the four together with relaxed loads; the fence after the
// last poll makes the wait an acquire. false if it gave up, or if another
// wait of the launch gave up before (bit 1 of *err).
__device__ __forceinline__ bool wait_epochs(const unsigned* f, long long o1, long long o2, long long o3,
                                            unsigned target, const int* err) {
  bool ok = false;
  for (int it = 0; it < kDepPolls; it++) {
    const unsigned v0 = ld_relaxed_u32(f), v1 = ld_relaxed_u32(f + o1), v2 = ld_relaxed_u32(f + o2),
                   v3 = ld_relaxed_u32(f + o3);
    ok = reached(v0, target) && reached(v1, target) && reached(v2, target) && reached(v3, target);
    if (ok) break;
    if ((it & 63) == 63 && (*reinterpret_cast<const volatile int*>(err) & 2)) break;
    __nanosleep(it < 32 ? 32 : 256);
  }
  fence_acq_rel_gpu();
  return ok;
}

// item -> (E or H, plane k, tile) in the schedule's order
struct EhItem {
  bool e;
  int k, tile;
};

__device__ __forceinline__ EhItem eh_decode(const EhSched& s, int T, long long it) {
  const int L = s.lag, NP = s.np;
  const int b = static_cast<int>(it / T);
  EhItem r;
  r.tile = static_cast<int>(it - static_cast<long long>(b) * T);
  if (b < L) {
    r.e = true;
    r.k = 1 + b;
  } else if (b < 2 * NP - L) {
    const int m = b - L;
    r.e = (m & 1) == 0;
    r.k = r.e ? L + 1 + (m >> 1) : 1 + (m >> 1);
  } else {
    r.e = false;
    r.k = NP - L + 1 + (b - (2 * NP - L));
  }
  return r;
}

// offsets (from an H tile's own flag) of the E tiles it reads: x+1, y+1 and
// the plane above; 0 where the tile has no such neighbour
__device__ __forceinline__ void eh_deps(const EhSched& s, int T, const EhItem& q, long long& ox, long long& oy,
                                        long long& oz) {
  const int bx = q.tile % s.nbx, by = q.tile / s.nbx;
  ox = bx + 1 < s.nbx ? 1 : 0;
  oy = by + 1 < s.nby ? s.nbx : 0;
  oz = q.k < s.np ? T : 0;
}

}  // namespace

// The H update of both 4-row halves of an 8-row tile at once: half h stages
// its 12 operands per group in slots 12 h .. 12 h + 11. The tile's own H and
// CPML integrators are requested first, then dep() (the wait for the E tiles
// it reads, when one is needed), then E; hook() runs once every copy is in
// flight.
template <class Dep, class Hook>
__device__ __forceinline__ void h_pair(const FusedArgs& a, int bx, int by8, int k, float4* sm, Dep dep, Hook hook) {
  const int lane = threadIdx.x, tid = threadIdx.y * 32 + lane;
  const int x4 = bx * 128 + lane * 4;
  const long long sy = a.pitch, sz = static_cast<long long>(a.pitch) * a.ny;
  long long c[2];
#pragma unroll
  for (int h = 0; h < 2; h++) {
    const int j = 1 + (2 * by8 + h) * kRowsA + threadIdx.y;
    c[h] = k * sz + min(j, a.ny - 2) * sy + x4;
    float4* s = sm + tid + h * 12 * kThreads;
    cp_async16(s + 7 * kThreads, a.H[0] + c[h]);
    cp_async16(s + 8 * kThreads, a.H[1] + c[h]);
    cp_async16(s + 9 * kThreads, a.H[2] + c[h]);
    const GroupCtx g = make_ctx(a, 1, x4, j, lane, k, k + 1);
    if (g.row_ok) stage_x_slab(a, g, 1, k, reinterpret_cast<float*>(sm + (h * 12 + 10) * kThreads) + 8 * tid);
  }
  dep();
  float ey_xp3[2] = {0.f, 0.f}, ez_xp3[2] = {0.f, 0.f};
#pragma unroll
  for (int h = 0; h < 2; h++) {
    float4* s = sm + tid + h * 12 * kThreads;
    cp_async16(s + 0 * kThreads, a.E[0] + c[h] + sz);
    cp_async16(s + 1 * kThreads, a.E[1] + c[h] + sz);
    cp_async16(s + 2 * kThreads, a.E[0] + c[h]);
    cp_async16(s + 3 * kThreads, a.E[1] + c[h]);
    cp_async16(s + 4 * kThreads, a.E[2] + c[h]);
    cp_async16(s + 5 * kThreads, a.E[0] + c[h] + sy);
    cp_async16(s + 6 * kThreads, a.E[2] + c[h] + sy);
    if (lane == 31) {
      ey_xp3[h] = __ldcg(a.E[1] + c[h] + 4);
      ez_xp3[h] = __ldcg(a.E[2] + c[h] + 4);
    }
  }
  hook();
  cp_async_wait_all();
  // one copy of the update's code for both halves (the kernel's code is
  // large enough that instruction fetch stalls it)
#pragma unroll 1
  for (int h = 0; h < 2; h++) {
    const int j = 1 + (2 * by8 + h) * kRowsA + threadIdx.y;
    const float4* s = sm + tid + h * 12 * kThreads;
    const GroupCtx g = make_ctx(a, 1, x4, j, lane, k, k + 1);
    const float4 ey = s[3 * kThreads], ez = s[4 * kThreads];
    const float ey_sh = __shfl_down_sync(kFull, ey.x, 1);
    const float ez_sh = __shfl_down_sync(kFull, ez.x, 1);
    h_group_update<false>(a, g, k, s[2 * kThreads], ey, ez, s[5 * kThreads], s[6 * kThreads], s[0], s[1 * kThreads],
                          lane != 31 ? ey_sh : ey_xp3[h], lane != 31 ? ez_sh : ez_xp3[h], s[7 * kThreads],
                          s[8 * kThreads], s[9 * kThreads],
                          reinterpret_cast<const float*>(sm + (h * 12 + 10) * kThreads) + 8 * tid);
  }
}

template <int MAXP, int MINB, bool PJ>
__global__ void __launch_bounds__(kThreads, MINB)
    staged_eh_kernel(const __grid_constant__ FusedArgs a, const __grid_constant__ EhSched s) {
  extern __shared__ float4 sm[];
  __shared__ int s_ready[2];  // by item parity: the item's E dependences were seen reached
  const bool lead = threadIdx.x == 0 && threadIdx.y == 0;
  const unsigned target = *s.epoch + 1u;
  const int T = s.nbx * s.nby;
  const int halves4 = (a.ny - 2 + kRowsA - 1) / kRowsA;  // 4-row halves with rows to update
  if (lead) s_ready[0] = 0;
  __syncthreads();
  unsigned* pending = nullptr;  // lead: the E flag still to be published
  int par = 0;
  for (long long it = blockIdx.x; it < s.nitems; it += gridDim.x, par ^= 1) {
    const EhItem q = eh_decode(s, T, it);
    const int bx = q.tile % s.nbx, by8 = q.tile / s.nbx;
    unsigned* f = s.flags + static_cast<long long>(q.k - 1) * T + q.tile;
    const bool ready = s_ready[par] != 0;
    auto publish = [&] {
      if (pending) {
        fence_acq_rel_gpu();
        st_relaxed_u32(pending, target);
        pending = nullptr;
      }
    };
    // once every copy of the item is in flight: publish, and look at the
    // next item's dependences
    auto hook = [&] {
      if (!lead) return;
      bool next = false;
      const long long nx = it + gridDim.x;
      if (nx < s.nitems) {
        const EhItem n = eh_decode(s, T, nx);
        if (!n.e) {
          long long ox, oy, oz;
          eh_deps(s, T, n, ox, oy, oz);
          const unsigned* g = s.flags + static_cast<long long>(n.k - 1) * T + n.tile;
          const unsigned v0 = ld_relaxed_u32(g), v1 = ld_relaxed_u32(g + ox), v2 = ld_relaxed_u32(g + oy),
                         v3 = ld_relaxed_u32(g + oz);
          next = reached(v0, target) && reached(v1, target) && reached(v2, target) && reached(v3, target);
        }
      }
      // one fence: the acquire of those loads and the release of the flag
      fence_acq_rel_gpu();
      if (pending) {
        st_relaxed_u32(pending, target);
        pending = nullptr;
      }
      s_ready[par ^ 1] = next ? 1 : 0;
    };
    if (q.e) {
      // the two halves in turn, through one copy of the E update's code; the
      // bookkeeping runs with the first half's copies in flight
      const int nh = 2 * by8 + 1 < halves4 ? 2 : 1;
#pragma unroll 1
      for (int h = 0; h < nh; h++) {
        auto hook_h = [&] {
          if (h == 0) hook();
        };
        e_tile<MAXP, PJ>(a, bx, 2 * by8 + h, q.k, sm, hook_h);
      }
      __syncthreads();  // every thread's stores are issued before the flag is published
      if (lead) pending = f;
    } else {
      auto dep = [&] {
        if (ready) return;
        if (lead) {
          publish();
          long long ox, oy, oz;
          eh_deps(s, T, q, ox, oy, oz);
          if (!wait_epochs(f, ox, oy, oz, target, &a.ctrl->error)) atomicOr(&a.ctrl->error, 2);
        }
        __syncthreads();
      };
      h_pair(a, bx, by8, q.k, sm, dep, hook);
      __syncthreads();
    }
  }
  if (lead && pending) {
    fence_acq_rel_gpu();
    st_relaxed_u32(pending, target);
  }
}

namespace {

// the kernel and its dynamic shared memory for a grid's materials
struct EhKernel {
  const void* fn;
  size_t smem;
  int minb;
};

// shared memory: the larger of an E item's slots (with its material ids) and
// an H item's two halves of 12 slots; 4 CTAs per SM at 49-50 KB each
template <int MAXP, bool PJ>
EhKernel eh_kernel() {
  constexpr int slots = kSlotsE + (PJ ? pj_slots<MAXP>() : 0);
  constexpr size_t e_bytes = slots * kThreads * sizeof(float4) + kThreads * sizeof(unsigned);
  constexpr size_t h_bytes = 2 * kSlotsH * kThreads * sizeof(float4);
  constexpr int minb = 4;
  return {reinterpret_cast<const void*>(staged_eh_kernel<MAXP, minb, PJ>), e_bytes > h_bytes ? e_bytes : h_bytes,
          minb};
}

EhKernel eh_select(const FusedArgs& a) {
  const bool pj = a.all_dispersive != 0;
  switch (a.max_poles) {
    case 0: return eh_kernel<0, false>();
    case -1: return pj ? eh_kernel<-1, true>() : eh_kernel<-1, false>();
    case 1: return pj ? eh_kernel<1, true>() : eh_kernel<1, false>();
    default: return pj ? eh_kernel<2, true>() : eh_kernel<2, false>();
  }
}

}  // namespace

bool staged_eh_plan(const FusedArgs& a, EhSched* s, int* blocks) {
  if (a.pitch % 128 != 0 || a.has_mu || a.nplanes > 0 || a.nz < 3) return false;
  const EhKernel k = eh_select(a);
  once_per_device(k.fn, [&] {
    cudaFuncSetAttribute(k.fn, cudaFuncAttributePreferredSharedMemoryCarveout, carveout_for(k.minb, k.smem));
    cudaFuncSetAttribute(k.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(k.smem));
  });
  int dev = 0, sms = 0, per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k.fn, kThreads, k.smem) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (per_sm <= 0 || sms <= 0) return false;
  s->nbx = a.pitch / 128;
  s->nby = (a.ny - 2 + kRowsEH - 1) / kRowsEH;
  s->np = a.nz - 2;
  const long long T = static_cast<long long>(s->nbx) * s->nby;
  if (T * s->np >= (1LL << 31)) return false;
  *blocks = per_sm * sms;
  // H of plane k waits for E of plane k+1, (2 lag - 1) batches earlier: with
  // lag >= blocks / T + 1 that is at least two rounds of the resident CTAs
  s->lag = static_cast<int>(std::min<long long>(s->np, (*blocks + T - 1) / T + 1));
  s->nitems = 2 * T * s->np;
  return true;
}

int launch_staged_eh(const FusedArgs& a, const EhSched& s, int blocks, cudaStream_t st) {
  const EhKernel k = eh_select(a);
  FusedArgs args = a;
  EhSched sched = s;
  void* params[] = {&args, &sched};
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(32, kRowsA, 1);
  cfg.dynamicSmemBytes = k.smem;
  cfg.stream = st;
  cudaLaunchAttribute attr;
  attr.id = cudaLaunchAttributeCooperative;
  attr.val.cooperative = 1;
  cfg.attrs = &attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelExC(&cfg, k.fn, params);
  return 1;
}

}  // namespace fdtdb
