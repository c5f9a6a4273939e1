// FP32 fused 3D sweeps with a TMA pipeline (sm_100a).
//
// Same update as kernels_fused3d.cu. A CTA of kTY warps owns a 128 x kTY
// tile of (x, y) and marches along z over a chunk of planes. Thread 0 issues
// cp.async.bulk.tensor loads of the planes ahead into a kStages-deep ring of
// shared-memory stages, each guarded by an mbarrier (complete_tx); the
// warps wait on the stage's barrier, compute the plane out of shared memory
// and write their 128-bit groups straight to global memory. Neighbour cells
// along y and x are part of the loaded box (the halo rows/columns), so the
// only register carry is the previous plane along z.
//
//   E sweep (+z): box of H {132 x (kTY+1)} at (x0-4, j0-1) -- x-1 and y-1
//                 halos -- plus E {128 x kTY} and the uint8 material ids.
//   H sweep (-z): box of E {132 x (kTY+1)} at (x0, j0) -- x+1 and y+1
//                 halos -- plus H {128 x kTY}.
// Every mbarrier wait is bounded; on expiry the CTA records an error in the
// control block, waits (bounded) for its outstanding copies and returns.
// Each CTA loads its own tiles (none is shared across a cluster); the tensor
// maps cover this GPU's memory only.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "fused3d_common.cuh"

namespace fdtdb {

namespace {

using namespace f3d;

constexpr int kTY = 8;
constexpr int kStages = 4;
constexpr int kHW = 132;                                        // halo row width (floats)
constexpr int kHaloBytes = ((kHW * (kTY + 1) * 4 + 127) / 128) * 128;  // one halo tile, padded
constexpr int kHaloTx = kHW * (kTY + 1) * 4;                    // bytes a halo box delivers
constexpr int kTileBytes = 128 * kTY * 4;
constexpr int kIdsBytes = 128 * kTY;
constexpr int kStageE = 3 * kHaloBytes + 3 * kTileBytes + kIdsBytes;
constexpr int kStageH = 3 * kHaloBytes + 3 * kTileBytes;
constexpr unsigned kFull = 0xffffffffu;
constexpr long long kWaitLimit = 1LL << 24;  // polls of one mbarrier before giving up

__device__ __forceinline__ uint32_t saddr(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(saddr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  for (long long n = 0; n < kWaitLimit; n++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void tma_load(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(saddr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(saddr(bar))
      : "memory");
}
__device__ __forceinline__ float4 lds4(const float* p) { return *reinterpret_cast<const float4*>(p); }

}  // namespace

struct TmaMapsE {
  CUtensorMap H[3];  // box {132, kTY+1, 1}
  CUtensorMap E[3];  // box {128, kTY, 1}
  CUtensorMap ids;   // box {128, kTY, 1}, uint8
};
struct TmaMapsH {
  CUtensorMap E[3];  // box {132, kTY+1, 1}
  CUtensorMap H[3];  // box {128, kTY, 1}
};

// on a timed-out wait: wait (bounded) for the copies still in flight, so no
// TMA write lands in shared memory after the CTA has gone
__device__ void drain(uint64_t* full, int it, int kcount) {
  for (int q = it; q < it + kStages && q < kcount; q++) mbar_wait_bounded(&full[q % kStages], (q / kStages) & 1);
}

template <int MAXP>
__global__ void __launch_bounds__(32 * kTY, 2) tma_e_kernel(const __grid_constant__ FusedArgs a,
                                                            const __grid_constant__ TmaMapsE m, int kchunk) {
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem);
  unsigned char* stages = smem + 128;
  const int lane = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + lane;
  const int x0 = blockIdx.x * 128, x4 = x0 + lane * 4;
  const int j0 = 1 + blockIdx.y * kTY, j = j0 + ty;
  const int jl = min(j, a.ny - 2);
  const int kbeg = 1 + blockIdx.z * kchunk;
  const int kend = min(kbeg + kchunk, a.nz - 1);
  const int kcount = kend - kbeg;
  const long long sy = a.pitch, sz = static_cast<long long>(a.pitch) * a.ny;
  const bool have_ids = a.ids != nullptr;
  const uint32_t tx = 3 * kHaloTx + 3 * kTileBytes + (have_ids ? kIdsBytes : 0);

  if (tid == 0) {
    for (int s = 0; s < kStages; s++) mbar_init(&full[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  auto issue = [&](int k, int s) {
    unsigned char* st = stages + s * kStageE;
    mbar_expect_tx(&full[s], tx);
    for (int c = 0; c < 3; c++) tma_load(st + c * kHaloBytes, &m.H[c], &full[s], x0 - 4, j0 - 1, k);
    for (int c = 0; c < 3; c++) tma_load(st + 3 * kHaloBytes + c * kTileBytes, &m.E[c], &full[s], x0, j0, k);
    if (have_ids) tma_load(st + 3 * kHaloBytes + 3 * kTileBytes, &m.ids, &full[s], x0, j0, k);
  };
  if (tid == 0)
    for (int s = 0; s < kStages && s < kcount; s++) issue(kbeg + s, s);

  const GroupCtx g = make_ctx(a, 0, x4, j, lane, kbeg, kend);
  float4 hx_km, hy_km;
  {
    const long long c = (kbeg - 1) * sz + jl * sy + x4;
    hx_km = ld4(a.H[0] + c);
    hy_km = ld4(a.H[1] + c);
  }
  for (int it = 0; it < kcount; it++) {
    const int k = kbeg + it, s = it % kStages;
    const bool timeout = !mbar_wait_bounded(&full[s], (it / kStages) & 1);
    if (!timeout) {
      const unsigned char* st = stages + s * kStageE;
      const float* sHx = reinterpret_cast<const float*>(st);
      const float* sHy = reinterpret_cast<const float*>(st + kHaloBytes);
      const float* sHz = reinterpret_cast<const float*>(st + 2 * kHaloBytes);
      const float* sE = reinterpret_cast<const float*>(st + 3 * kHaloBytes);
      const int own = (ty + 1) * kHW + 4 + 4 * lane, ym = ty * kHW + 4 + 4 * lane;
      const float4 hx = lds4(sHx + own), hy = lds4(sHy + own), hz = lds4(sHz + own);
      const float4 hx_ym = lds4(sHx + ym), hz_ym = lds4(sHz + ym);
      float hy_xm0 = __shfl_up_sync(kFull, hy.w, 1);
      float hz_xm0 = __shfl_up_sync(kFull, hz.w, 1);
      if (lane == 0) {
        hy_xm0 = sHy[(ty + 1) * kHW + 3];
        hz_xm0 = sHz[(ty + 1) * kHW + 3];
      }
      const int eo = ty * 128 + 4 * lane;
      const float4 exo = lds4(sE + eo), eyo = lds4(sE + kTY * 128 + eo), ezo = lds4(sE + 2 * kTY * 128 + eo);
      const unsigned ids4 =
          have_ids ? reinterpret_cast<const unsigned*>(st + 3 * kHaloBytes + 3 * kTileBytes)[ty * 32 + lane] : 0u;
      e_group_update<MAXP>(a, g, k, hx, hy, hz, hx_ym, hz_ym, hx_km, hy_km, hy_xm0, hz_xm0, exo, eyo, ezo, ids4);
      hx_km = hx;
      hy_km = hy;
    }
    if (__syncthreads_or(timeout)) {
      if (tid == 0) {
        atomicOr(&a.ctrl->error, 1);
        drain(full, it, kcount);
      }
      return;
    }
    if (tid == 0 && it + kStages < kcount) issue(k + kStages, s);
  }
}

template <bool MU>
__global__ void __launch_bounds__(32 * kTY, 2) tma_h_kernel(const __grid_constant__ FusedArgs a,
                                                          const __grid_constant__ TmaMapsH m, int kchunk) {
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem);
  unsigned char* stages = smem + 128;
  const int lane = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + lane;
  const int x0 = blockIdx.x * 128, x4 = x0 + lane * 4;
  const int j0 = 1 + blockIdx.y * kTY, j = j0 + ty;
  const int jl = min(j, a.ny - 2);
  const int kbeg = 1 + blockIdx.z * kchunk;
  const int kend = min(kbeg + kchunk, a.nz - 1);
  const int kcount = kend - kbeg;
  const long long sy = a.pitch, sz = static_cast<long long>(a.pitch) * a.ny;
  const uint32_t tx = 3 * kHaloTx + 3 * kTileBytes;

  if (tid == 0) {
    for (int s = 0; s < kStages; s++) mbar_init(&full[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  auto issue = [&](int k, int s) {
    unsigned char* st = stages + s * kStageH;
    mbar_expect_tx(&full[s], tx);
    for (int c = 0; c < 3; c++) tma_load(st + c * kHaloBytes, &m.E[c], &full[s], x0, j0, k);
    for (int c = 0; c < 3; c++) tma_load(st + 3 * kHaloBytes + c * kTileBytes, &m.H[c], &full[s], x0, j0, k);
  };
  // planes are visited from kend-1 down to kbeg
  if (tid == 0)
    for (int s = 0; s < kStages && s < kcount; s++) issue(kend - 1 - s, s);

  const GroupCtx g = make_ctx(a, 1, x4, j, lane, kbeg, kend);
  float4 ex_kp, ey_kp;
  {
    const long long c = kend * sz + jl * sy + x4;
    ex_kp = ld4(a.E[0] + c);
    ey_kp = ld4(a.E[1] + c);
  }
  for (int it = 0; it < kcount; it++) {
    const int k = kend - 1 - it, s = it % kStages;
    const bool timeout = !mbar_wait_bounded(&full[s], (it / kStages) & 1);
    if (!timeout) {
      const unsigned char* st = stages + s * kStageH;
      const float* sEx = reinterpret_cast<const float*>(st);
      const float* sEy = reinterpret_cast<const float*>(st + kHaloBytes);
      const float* sEz = reinterpret_cast<const float*>(st + 2 * kHaloBytes);
      const float* sH = reinterpret_cast<const float*>(st + 3 * kHaloBytes);
      const int own = ty * kHW + 4 * lane, yp = (ty + 1) * kHW + 4 * lane;
      const float4 ex = lds4(sEx + own), ey = lds4(sEy + own), ez = lds4(sEz + own);
      const float4 ex_yp = lds4(sEx + yp), ez_yp = lds4(sEz + yp);
      float ey_xp3 = __shfl_down_sync(kFull, ey.x, 1);
      float ez_xp3 = __shfl_down_sync(kFull, ez.x, 1);
      if (lane == 31) {
        ey_xp3 = sEy[ty * kHW + 128];
        ez_xp3 = sEz[ty * kHW + 128];
      }
      const int ho = ty * 128 + 4 * lane;
      const float4 hx = lds4(sH + ho), hy = lds4(sH + kTY * 128 + ho), hz = lds4(sH + 2 * kTY * 128 + ho);
      h_group_update<MU>(a, g, k, ex, ey, ez, ex_yp, ez_yp, ex_kp, ey_kp, ey_xp3, ez_xp3, hx, hy, hz);
      ex_kp = ex;
      ey_kp = ey;
    }
    if (__syncthreads_or(timeout)) {
      if (tid == 0) {
        atomicOr(&a.ctrl->error, 1);
        drain(full, it, kcount);
      }
      return;
    }
    if (tid == 0 && it + kStages < kcount) issue(k - kStages, s);
  }
}

// ---------------------------------------------------------------- host side

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

bool make_map(CUtensorMap* m, void* base, CUtensorMapDataType type, int esize, int pitch, int ny, int nz, int bx,
              int by) {
  auto fn = encode_fn();
  if (!fn) return false;
  const cuuint64_t dims[3] = {static_cast<cuuint64_t>(pitch), static_cast<cuuint64_t>(ny), static_cast<cuuint64_t>(nz)};
  const cuuint64_t strides[2] = {static_cast<cuuint64_t>(pitch) * esize,
                                 static_cast<cuuint64_t>(pitch) * ny * esize};
  const cuuint32_t box[3] = {static_cast<cuuint32_t>(bx), static_cast<cuuint32_t>(by), 1};
  const cuuint32_t es[3] = {1, 1, 1};
  return fn(m, type, 3, base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

struct TmaState {
  TmaMapsE e;
  TmaMapsH h;
  bool ok = false;
};

// Builds the tensor maps for the current arrays; false if TMA cannot be used
// (then the caller keeps the register-prefetch sweeps).
bool tma_prepare(const FusedArgs& a, TmaState** state) {
  if (!*state) *state = new TmaState();
  TmaState& st = **state;
  st.ok = false;
  if (a.pitch % 128 != 0 || a.nz < 3) return false;
  if (a.bids && a.bshift < 2) return false;
  bool ok = true;
  for (int c = 0; c < 3; c++) {
    ok = ok && make_map(&st.e.H[c], a.H[c], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, a.pitch, a.ny, a.nz, kHW, kTY + 1);
    ok = ok && make_map(&st.e.E[c], a.E[c], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, a.pitch, a.ny, a.nz, 128, kTY);
    ok = ok && make_map(&st.h.E[c], a.E[c], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, a.pitch, a.ny, a.nz, kHW, kTY + 1);
    ok = ok && make_map(&st.h.H[c], a.H[c], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, a.pitch, a.ny, a.nz, 128, kTY);
  }
  if (a.ids)
    ok = ok && make_map(&st.e.ids, const_cast<uint8_t*>(a.ids), CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, a.pitch, a.ny, a.nz,
                        128, kTY);
  else
    st.e.ids = st.e.E[0];
  if (!ok) return false;
  {
    // the attributes belong to the current device's context: set on every
    // preparation (a host call), so each device has them before its launches
    const int se = 128 + kStages * kStageE, sh = 128 + kStages * kStageH;
    ok = cudaFuncSetAttribute(tma_e_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, se) == cudaSuccess &&
         cudaFuncSetAttribute(tma_e_kernel<-1>, cudaFuncAttributeMaxDynamicSharedMemorySize, se) == cudaSuccess &&
         cudaFuncSetAttribute(tma_e_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, se) == cudaSuccess &&
         cudaFuncSetAttribute(tma_e_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, se) == cudaSuccess &&
         cudaFuncSetAttribute(tma_h_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sh) == cudaSuccess &&
         cudaFuncSetAttribute(tma_h_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sh) == cudaSuccess;
    if (!ok) return false;
  }
  st.ok = true;
  return true;
}

void tma_release(TmaState* state) { delete state; }

static int tma_kchunk(const FusedArgs& a, int* bz) {
  const int bx = a.pitch / 128, by = (a.ny - 2 + kTY - 1) / kTY;
  const int resident = 148 * 2;
  int chunks = (resident + (bx * by) / 2) / (bx * by);
  chunks = max(1, min(chunks, (a.nz - 2) / 16));
  const int kchunk = (a.nz - 2 + chunks - 1) / chunks;
  *bz = (a.nz - 2 + kchunk - 1) / kchunk;
  return kchunk;
}

int launch_tma_e(const FusedArgs& a, const TmaState* st, cudaStream_t s) {
  int bz;
  const int kchunk = tma_kchunk(a, &bz);
  dim3 grid(a.pitch / 128, (a.ny - 2 + kTY - 1) / kTY, bz), block(32, kTY, 1);
  const int smem = 128 + kStages * kStageE;
  switch (a.max_poles) {
    case 0: tma_e_kernel<0><<<grid, block, smem, s>>>(a, st->e, kchunk); break;
    case -1: tma_e_kernel<-1><<<grid, block, smem, s>>>(a, st->e, kchunk); break;
    case 1: tma_e_kernel<1><<<grid, block, smem, s>>>(a, st->e, kchunk); break;
    default: tma_e_kernel<2><<<grid, block, smem, s>>>(a, st->e, kchunk); break;
  }
  return 1;
}

int launch_tma_h(const FusedArgs& a, const TmaState* st, cudaStream_t s) {
  int bz;
  const int kchunk = tma_kchunk(a, &bz);
  dim3 grid(a.pitch / 128, (a.ny - 2 + kTY - 1) / kTY, bz), block(32, kTY, 1);
  if (a.has_mu) tma_h_kernel<true><<<grid, block, 128 + kStages * kStageH, s>>>(a, st->h, kchunk);
  else tma_h_kernel<false><<<grid, block, 128 + kStages * kStageH, s>>>(a, st->h, kchunk);
  return 1;
}

}  // namespace fdtdb
