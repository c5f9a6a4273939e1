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

template <bool MU>
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
    h_group_update<MU>(a, g, k, cex, cey, cez, cex_yp, cez_yp, ex_kp, ey_kp, ey_xp3, ez_xp3, chx, chy, chz);
    ex_kp = cex;
    ey_kp = cey;
  }
}

// NZ consecutive planes per thread: every load of the NZ planes is issued
// before the first plane is computed; plane k's H (E) doubles as plane k+1's
// z neighbour in the E (H) sweep. MINB is the CTA count per SM the register
// allocation targets.
template <int MAXP, int NZ, int MINB>
__global__ void __launch_bounds__(32 * kRows, MINB) flat_e_kernel(const __grid_constant__ FusedArgs a) {
  const int lane = threadIdx.x;
  const int x4 = blockIdx.x * 128 + lane * 4;
  const int j = 1 + blockIdx.y * kRows + threadIdx.y;
  const int jl = min(j, a.ny - 2);
  const int k0 = 1 + blockIdx.z * NZ;
  const long long sy = a.pitch, sz = static_cast<long long>(a.pitch) * a.ny;
  const GroupCtx g = make_ctx(a, 0, x4, j, lane, k0, k0 + NZ);
  const long long c0 = k0 * sz + jl * sy + x4;
  float4 hx[NZ + 1], hy[NZ + 1], hz[NZ], hx_ym[NZ], hz_ym[NZ], ex[NZ], ey[NZ], ez[NZ];
  unsigned ids[NZ];
  // lane 0 takes its x-1 neighbours from the previous group's last cell: load
  // them with the rest, so the warp waits for one round trip, not two
  float hy_xm_l0[NZ], hz_xm_l0[NZ];
  hx[0] = ld4(a.H[0] + c0 - sz);
  hy[0] = ld4(a.H[1] + c0 - sz);
#pragma unroll
  for (int q = 0; q < NZ; q++) {
    const int k = k0 + q;
    const long long c = c0 + q * sz;
    const bool in = k <= a.nz - 2;
    const long long cc = in ? c : c0;  // planes past the grid read a valid plane and are not computed
    hy_xm_l0[q] = 0.f;
    hz_xm_l0[q] = 0.f;
    if (lane == 0) {
      hy_xm_l0[q] = a.H[1][cc - 1];
      hz_xm_l0[q] = a.H[2][cc - 1];
    }
    hx[q + 1] = ld4(a.H[0] + cc);
    hy[q + 1] = ld4(a.H[1] + cc);
    hz[q] = ld4(a.H[2] + cc);
    hx_ym[q] = ld4(a.H[0] + cc - sy);
    hz_ym[q] = ld4(a.H[2] + cc - sy);
    ex[q] = ld4(a.E[0] + cc);
    ey[q] = ld4(a.E[1] + cc);
    ez[q] = ld4(a.E[2] + cc);
    ids[q] = a.ids ? *reinterpret_cast<const unsigned*>(a.ids + cc) : 0u;
  }
#pragma unroll
  for (int q = 0; q < NZ; q++) {
    const int k = k0 + q;
    float hy_xm0 = __shfl_up_sync(kFull, hy[q + 1].w, 1);
    float hz_xm0 = __shfl_up_sync(kFull, hz[q].w, 1);
    if (k > a.nz - 2) break;
    if (lane == 0) {
      hy_xm0 = hy_xm_l0[q];
      hz_xm0 = hz_xm_l0[q];
    }
    e_group_update<MAXP>(a, g, k, hx[q + 1], hy[q + 1], hz[q], hx_ym[q], hz_ym[q], hx[q], hy[q], hy_xm0, hz_xm0, ex[q],
                         ey[q], ez[q], ids[q]);
  }
}

template <int NZ, int MINB, bool MU>
__global__ void __launch_bounds__(32 * kRows, MINB) flat_h_kernel(const __grid_constant__ FusedArgs a) {
  const int lane = threadIdx.x;
  const int x4 = blockIdx.x * 128 + lane * 4;
  const int j = 1 + blockIdx.y * kRows + threadIdx.y;
  const int jl = min(j, a.ny - 2);
  // groups of planes from the top down, so the planes above were read just before
  const int ktop = a.nz - 2 - blockIdx.z * NZ;
  const long long sy = a.pitch, sz = static_cast<long long>(a.pitch) * a.ny;
  const GroupCtx g = make_ctx(a, 1, x4, j, lane, max(1, ktop - NZ + 1), ktop + 1);
  const long long ctop = ktop * sz + jl * sy + x4;
  // index q = 0 is plane ktop, q = 1 plane ktop-1, ...; ex/ey[q] hold plane ktop+1-q
  float4 ex[NZ + 1], ey[NZ + 1], ez[NZ], ex_yp[NZ], ez_yp[NZ], hx[NZ], hy[NZ], hz[NZ];
  // lane 31 takes its x+1 neighbours from the next group's first cell: load
  // them with the rest (one round trip per warp)
  float ey_xp_l31[NZ], ez_xp_l31[NZ];
  ex[0] = ld4(a.E[0] + ctop + sz);
  ey[0] = ld4(a.E[1] + ctop + sz);
#pragma unroll
  for (int q = 0; q < NZ; q++) {
    const int k = ktop - q;
    const long long cc = k >= 1 ? ctop - q * sz : ctop;
    ey_xp_l31[q] = 0.f;
    ez_xp_l31[q] = 0.f;
    if (lane == 31) {
      ey_xp_l31[q] = a.E[1][cc + 4];
      ez_xp_l31[q] = a.E[2][cc + 4];
    }
    ex[q + 1] = ld4(a.E[0] + cc);
    ey[q + 1] = ld4(a.E[1] + cc);
    ez[q] = ld4(a.E[2] + cc);
    ex_yp[q] = ld4(a.E[0] + cc + sy);
    ez_yp[q] = ld4(a.E[2] + cc + sy);
    hx[q] = ld4(a.H[0] + cc);
    hy[q] = ld4(a.H[1] + cc);
    hz[q] = ld4(a.H[2] + cc);
  }
#pragma unroll
  for (int q = 0; q < NZ; q++) {
    const int k = ktop - q;
    float ey_xp3 = __shfl_down_sync(kFull, ey[q + 1].x, 1);
    float ez_xp3 = __shfl_down_sync(kFull, ez[q].x, 1);
    if (k < 1) break;
    if (lane == 31) {
      ey_xp3 = ey_xp_l31[q];
      ez_xp3 = ez_xp_l31[q];
    }
    h_group_update<MU>(a, g, k, ex[q + 1], ey[q + 1], ez[q], ex_yp[q], ez_yp[q], ex[q], ey[q], ey_xp3, ez_xp3, hx[q],
                   hy[q], hz[q]);
  }
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
  if (a.has_mu) fused3d_h_kernel<true><<<dim3(bx, by, bz), dim3(32, kRows, 1), 0, s>>>(a, kchunk);
  else fused3d_h_kernel<false><<<dim3(bx, by, bz), dim3(32, kRows, 1), 0, s>>>(a, kchunk);
  return 1;
}

// Register targets chosen on B200 (Gcell/s of the 384^3 Drude and 768^3
// two-pole Lorentz workloads): 8 CTAs of 128 threads per SM (<= 64 registers)
// except the two-pole E sweep, which spills there and takes 6.
template <int MAXP>
static void flat_e_dispatch(const FusedArgs& a, cudaStream_t s) {
  dim3 grid(a.pitch / 128, (a.ny - 2 + kRows - 1) / kRows, a.nz - 2), block(32, kRows, 1);
  flat_e_kernel<MAXP, 1, (MAXP >= 2 ? 6 : 7)><<<grid, block, 0, s>>>(a);
}

int launch_flat_e(const FusedArgs& a, cudaStream_t s) {
  switch (a.max_poles) {
    case 0: flat_e_dispatch<0>(a, s); break;
    case -1: flat_e_dispatch<-1>(a, s); break;
    case 1: flat_e_dispatch<1>(a, s); break;
    default: flat_e_dispatch<2>(a, s); break;
  }
  return 1;
}

int launch_flat_h(const FusedArgs& a, cudaStream_t s) {
  dim3 grid(a.pitch / 128, (a.ny - 2 + kRows - 1) / kRows, a.nz - 2), block(32, kRows, 1);
  if (a.has_mu) flat_h_kernel<1, 8, true><<<grid, block, 0, s>>>(a);
  else flat_h_kernel<1, 8, false><<<grid, block, 0, s>>>(a);
  return 1;
}

}  // namespace fdtdb
