// FP32 fused 3D sweeps without TMA: the update of fused3d_common.cuh (each
// thread owns four consecutive x cells; every field access is 128-bit) with
// two ways of feeding it:
//   * "regs": the CTA (a 128 x kRows tile of (x, y)) marches along z over a
//     chunk of planes; the next plane's loads are issued before the current
//     one is computed and the k-1 (E sweep) or k+1 (H sweep) plane is carried
//     in registers;
//   * "flat": one thread per group and plane, no march: the neighbour planes
//     come through L2 (planes are launched in order, so plane k-1 was read just
//     before), and many resident warps keep the loads in flight.
// x neighbours come from warp shuffles; ring and padding cells keep their
// value.
#include "fused3d_common.cuh"

namespace fdtdb {

namespace {

using namespace f3d;
constexpr unsigned kFull = 0xffffffffu;
constexpr int kRows = 4;

}  // namespace

template <int MAXP>
__global__ void __launch_bounds__(32 * kRows) fused3d_e_kernel(const __grid_constant__ FusedArgs a, int kchunk) {
  const int lane = threadIdx.x;
  const int x4 = blockIdx.x * 128 + lane * 4;
  const int j = 1 + blockIdx.y * kRows + threadIdx.y;
  const int jl = min(j, a.ny - 2);
  const int kbeg = 1 + blockIdx.z * kchunk;
  const int kend = min(kbeg + kchunk, a.nz - 1);
  const long long sy = a.pitch, sz = static_cast<long long>(a.pitch) * a.ny;
  const GroupCtx g = make_ctx(a, 0, x4, j, lane, kbeg, kend);
  float4 hx_km, hy_km;
  {
    const long long c = (kbeg - 1) * sz + jl * sy + x4;
    hx_km = ld4(a.H[0] + c);
    hy_km = ld4(a.H[1] + c);
  }
  float4 hx, hy, hz, hx_ym, hz_ym, ex, ey, ez;
  unsigned ids = 0;
  auto load = [&](int k) {
    const long long c = k * sz + jl * sy + x4;
    hx = ld4(a.H[0] + c);
    hy = ld4(a.H[1] + c);
    hz = ld4(a.H[2] + c);
    hx_ym = ld4(a.H[0] + c - sy);
    hz_ym = ld4(a.H[2] + c - sy);
    ex = ld4(a.E[0] + c);
    ey = ld4(a.E[1] + c);
    ez = ld4(a.E[2] + c);
    if (a.ids) ids = *reinterpret_cast<const unsigned*>(a.ids + c);
  };
  load(kbeg);
  for (int k = kbeg; k < kend; k++) {
    const float4 chx = hx, chy = hy, chz = hz, chx_ym = hx_ym, chz_ym = hz_ym, cex = ex, cey = ey, cez = ez;
    const unsigned cids = ids;
    if (k + 1 < kend) load(k + 1);
    float hy_xm0 = __shfl_up_sync(kFull, chy.w, 1);
    float hz_xm0 = __shfl_up_sync(kFull, chz.w, 1);
    if (lane == 0) {
      const long long c = k * sz + jl * sy + x4;
      hy_xm0 = a.H[1][c - 1];
      hz_xm0 = a.H[2][c - 1];
    }
    e_group_update<MAXP>(a, g, k, chx, chy, chz, chx_ym, chz_ym, hx_km, hy_km, hy_xm0, hz_xm0, cex, cey, cez, cids);
    hx_km = chx;
    hy_km = chy;
  }
}

__global__ void __launch_bounds__(32 * kRows) fused3d_h_kernel(const __grid_constant__ FusedArgs a, int kchunk) {
  const int lane = threadIdx.x;
  const int x4 = blockIdx.x * 128 + lane * 4;
  const int j = 1 + blockIdx.y * kRows + threadIdx.y;
  const int jl = min(j, a.ny - 2);
  const int kbeg = 1 + blockIdx.z * kchunk;
  const int kend = min(kbeg + kchunk, a.nz - 1);
  const long long sy = a.pitch, sz = static_cast<long long>(a.pitch) * a.ny;
  const GroupCtx g = make_ctx(a, 1, x4, j, lane, kbeg, kend);
  float4 ex_kp, ey_kp;
  {
    const long long c = kend * sz + jl * sy + x4;
    ex_kp = ld4(a.E[0] + c);
    ey_kp = ld4(a.E[1] + c);
  }
  float4 ex, ey, ez, ex_yp, ez_yp, hx, hy, hz;
  auto load = [&](int k) {
    const long long c = k * sz + jl * sy + x4;
    ex = ld4(a.E[0] + c);
    ey = ld4(a.E[1] + c);
    ez = ld4(a.E[2] + c);
    ex_yp = ld4(a.E[0] + c + sy);
    ez_yp = ld4(a.E[2] + c + sy);
    hx = ld4(a.H[0] + c);
    hy = ld4(a.H[1] + c);
    hz = ld4(a.H[2] + c);
  };
  load(kend - 1);
  for (int k = kend - 1; k >= kbeg; k--) {
    const float4 cex = ex, cey = ey, cez = ez, cex_yp = ex_yp, cez_yp = ez_yp, chx = hx, chy = hy, chz = hz;
    if (k - 1 >= kbeg) load(k - 1);
    float ey_xp3 = __shfl_down_sync(kFull, cey.x, 1);
    float ez_xp3 = __shfl_down_sync(kFull, cez.x, 1);
    if (lane == 31) {
      const long long c = k * sz + jl * sy + x4;
      ey_xp3 = a.E[1][c + 4];
      ez_xp3 = a.E[2][c + 4];
    }
    h_group_update(a, g, k, cex, cey, cez, cex_yp, cez_yp, ex_kp, ey_kp, ey_xp3, ez_xp3, chx, chy, chz);
    ex_kp = cex;
    ey_kp = cey;
  }
}

template <int MAXP>
__global__ void __launch_bounds__(32 * kRows) flat_e_kernel(const __grid_constant__ FusedArgs a) {
  const int lane = threadIdx.x;
  const int x4 = blockIdx.x * 128 + lane * 4;
  const int j = 1 + blockIdx.y * kRows + threadIdx.y;
  const int jl = min(j, a.ny - 2);
  const int k = 1 + blockIdx.z;
  const long long sy = a.pitch, sz = static_cast<long long>(a.pitch) * a.ny;
  const GroupCtx g = make_ctx(a, 0, x4, j, lane, k, k + 1);
  const long long c = k * sz + jl * sy + x4;
  const float4 hx = ld4(a.H[0] + c), hy = ld4(a.H[1] + c), hz = ld4(a.H[2] + c);
  const float4 hx_ym = ld4(a.H[0] + c - sy), hz_ym = ld4(a.H[2] + c - sy);
  const float4 hx_km = ld4(a.H[0] + c - sz), hy_km = ld4(a.H[1] + c - sz);
  const float4 ex = ld4(a.E[0] + c), ey = ld4(a.E[1] + c), ez = ld4(a.E[2] + c);
  const unsigned ids = a.ids ? *reinterpret_cast<const unsigned*>(a.ids + c) : 0u;
  float hy_xm0 = __shfl_up_sync(kFull, hy.w, 1);
  float hz_xm0 = __shfl_up_sync(kFull, hz.w, 1);
  if (lane == 0) {
    hy_xm0 = a.H[1][c - 1];
    hz_xm0 = a.H[2][c - 1];
  }
  e_group_update<MAXP>(a, g, k, hx, hy, hz, hx_ym, hz_ym, hx_km, hy_km, hy_xm0, hz_xm0, ex, ey, ez, ids);
}

__global__ void __launch_bounds__(32 * kRows) flat_h_kernel(const __grid_constant__ FusedArgs a) {
  const int lane = threadIdx.x;
  const int x4 = blockIdx.x * 128 + lane * 4;
  const int j = 1 + blockIdx.y * kRows + threadIdx.y;
  const int jl = min(j, a.ny - 2);
  // planes from the top down, so plane k+1 was read just before plane k
  const int k = a.nz - 2 - blockIdx.z;
  const long long sy = a.pitch, sz = static_cast<long long>(a.pitch) * a.ny;
  const GroupCtx g = make_ctx(a, 1, x4, j, lane, k, k + 1);
  const long long c = k * sz + jl * sy + x4;
  const float4 ex = ld4(a.E[0] + c), ey = ld4(a.E[1] + c), ez = ld4(a.E[2] + c);
  const float4 ex_yp = ld4(a.E[0] + c + sy), ez_yp = ld4(a.E[2] + c + sy);
  const float4 ex_kp = ld4(a.E[0] + c + sz), ey_kp = ld4(a.E[1] + c + sz);
  const float4 hx = ld4(a.H[0] + c), hy = ld4(a.H[1] + c), hz = ld4(a.H[2] + c);
  float ey_xp3 = __shfl_down_sync(kFull, ey.x, 1);
  float ez_xp3 = __shfl_down_sync(kFull, ez.x, 1);
  if (lane == 31) {
    ey_xp3 = a.E[1][c + 4];
    ez_xp3 = a.E[2][c + 4];
  }
  h_group_update(a, g, k, ex, ey, ez, ex_yp, ez_yp, ex_kp, ey_kp, ey_xp3, ez_xp3, hx, hy, hz);
}

static int kchunk3d(int nz, int blocks_xy) {
  // several waves of 148 SMs x 3 CTAs; chunks of at least 32 planes
  const int interior = nz - 2;
  int chunks = (148 * 3 * 3 + blocks_xy - 1) / blocks_xy;
  chunks = max(1, min(chunks, interior / 32));
  return (interior + chunks - 1) / chunks;
}

bool fused3d_supported(const FusedArgs& a) { return a.pitch % 128 == 0; }

int launch_fused3d_e(const FusedArgs& a, cudaStream_t s) {
  const int bx = a.pitch / 128, by = (a.ny - 2 + kRows - 1) / kRows;
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
  const int bx = a.pitch / 128, by = (a.ny - 2 + kRows - 1) / kRows;
  const int kchunk = kchunk3d(a.nz, bx * by);
  const int bz = (a.nz - 2 + kchunk - 1) / kchunk;
  fused3d_h_kernel<<<dim3(bx, by, bz), dim3(32, kRows, 1), 0, s>>>(a, kchunk);
  return 1;
}

int launch_flat_e(const FusedArgs& a, cudaStream_t s) {
  dim3 grid(a.pitch / 128, (a.ny - 2 + kRows - 1) / kRows, a.nz - 2), block(32, kRows, 1);
  switch (a.max_poles) {
    case 0: flat_e_kernel<0><<<grid, block, 0, s>>>(a); break;
    case -1: flat_e_kernel<-1><<<grid, block, 0, s>>>(a); break;
    case 1: flat_e_kernel<1><<<grid, block, 0, s>>>(a); break;
    default: flat_e_kernel<2><<<grid, block, 0, s>>>(a); break;
  }
  return 1;
}

int launch_flat_h(const FusedArgs& a, cudaStream_t s) {
  dim3 grid(a.pitch / 128, (a.ny - 2 + kRows - 1) / kRows, a.nz - 2), block(32, kRows, 1);
  flat_h_kernel<<<grid, block, 0, s>>>(a);
  return 1;
}

}  // namespace fdtdb
