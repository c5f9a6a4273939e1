// Internal declarations shared by the fdtd_b200 CUDA sources.
#pragma once
#include <cstdint>
#include <mutex>
#include <set>
#include <utility>

#include <cuda_runtime.h>

namespace fdtdb {

constexpr int kTEM = 0, kTE = 1, kTM = 2, kThreeD = 3;
constexpr int kMaxPoles = 4;
constexpr int kMaxPlanes = 12;
constexpr int kMaxSources = 16;
constexpr int kAuxNpml = 15;  // Aux1D::mNPML (include/Source.hpp:362)
constexpr int kDftChunk = 64;  // samples buffered per DFT point before a flush
constexpr int kGraphSteps = kDftChunk;  // steps per captured CUDA graph

// Runs set(), once per (current device, key) in the process, under a lock:
// for kernel attributes (dynamic shared memory limit, carveout), which belong
// to a device's context, so that grids on several devices and several host
// threads each see them set before their first launch.
template <typename F>
inline void once_per_device(const void* key, F set) {
  static std::mutex mu;
  static std::set<std::pair<int, const void*>> done;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  if (done.insert({dev, key}).second) set();
}

// include/FDTDConstants.hpp:394-398
constexpr double kPi = 3.14159265358979323846264338327950288;
constexpr double kEps0 = 8.854e-12;
constexpr double kMu0 = kPi * 4.0e-7;

// Which E / H components a mode carries (FieldComponents, FDTDConstants.hpp:844-874)
__host__ __device__ constexpr bool hasE(int mode, int c) {
  return mode == kThreeD || (mode == kTE && c < 2) || (mode == kTM && c == 2);
}
__host__ __device__ constexpr bool hasH(int mode, int c) {
  return mode == kThreeD || (mode == kTE && c == 2) || (mode == kTM && c < 2);
}
// LeviCivita<I,J,K>::value (FDTDConstants.hpp:602-637)
__host__ __device__ constexpr int levi(int I, int J, int K) {
  return ((I == 0 && J == 1 && K == 2) || (I == 1 && J == 2 && K == 0) || (I == 2 && J == 0 && K == 1)) ? 1
         : ((I == 2 && J == 1 && K == 0) || (I == 0 && J == 2 && K == 1) || (I == 1 && J == 0 && K == 2)) ? -1
                                                                                                            : 0;
}
__host__ __device__ constexpr int third(int I, int J) { return 3 - I - J; }
// d1 of YeeUpdate::update_all (YeeUpdates.hpp:397)
__host__ __device__ constexpr int dir1(int I) { return I == 0 ? 1 : (I == 1 ? 2 : 0); }

// CPML slab of one axis: lo slab = cells 1..wlo, hi slab = hi0..hi0+whi-1
struct Slab {
  int wlo, hi0, W;
  // The x slab of the 3D FP32 method in rows of W4 floats: cell i < lo4 at
  // i, cell i >= hb at lo4 + i - hb (lo4, hb, W4 multiples of 4), so that
  // each 4-cell group that touches the slab is one aligned float4; the
  // padding cells have zero CPML coefficients and keep zero integrators.
  int lo4, hb, W4;
};
__host__ __device__ inline int slab_index(const Slab& s, int i) {
  if (i <= s.wlo) return i - 1;
  if (i >= s.hi0) return s.wlo + (i - s.hi0);
  return -1;
}
// position of slab cell i (slab_index(s, i) >= 0) in the aligned x layout
__host__ __device__ inline int slab_index4(const Slab& s, int i) { return i < s.lo4 ? i : s.lo4 + (i - s.hb); }
// first position of the 4-cell group at x4 in the aligned x layout, or -1
__host__ __device__ inline int slab_group4(const Slab& s, int x4) {
  if (x4 < s.lo4) return x4;
  if (x4 >= s.hb && x4 < s.hb + (s.W4 - s.lo4)) return s.lo4 + (x4 - s.hb);
  return -1;
}
// The slabs of an axis of n cells with CPML of plo and phi cells at its two
// ends (0: none): cells 1 .. plo + 1 and n - 2 - phi .. n - 2 carry integrators
inline Slab make_slab(int n, int plo, int phi) {
  Slab s;
  const int wlo = plo > 0 ? plo + 1 : 0, whi = phi > 0 ? phi + 1 : 0;
  s.wlo = wlo;
  s.hi0 = n - 1 - whi;
  s.W = wlo + whi;
  s.lo4 = wlo > 0 ? (wlo + 1 + 3) / 4 * 4 : 0;
  const int hb4 = s.hi0 / 4 * 4;
  s.hb = whi > 0 ? (hb4 > s.lo4 ? hb4 : s.lo4) : n + 4;
  s.W4 = s.lo4 + (whi > 0 ? (n + 3) / 4 * 4 - s.hb : 0);
  return s;
}

// 1D CPML coefficients of one (field type, axis)
template <typename R>
struct Prof {
  const R* B;    // exp(-nu dt)
  const R* C;    // plain: C/dx; fused: scaled C
  const R* F;    // plain: F/dx; fused: scaled F
  const R* G;
};

// Material coefficients for the FP64 plain method (reference operation order)
struct MatF64 {
  int kind, npoles;
  double den_e;  // eps_inf * eps0
  double den_h;  // mu_r * mu0
  // Drude: c1 = 1-b, c2 = 1+b, c3 = ((w*w)/dt)*eps0
  // Lorentz: c1 = bm/b, c2 = ((q*delta)*eps0), c3 = q = (freq*w)/b
  double c1[kMaxPoles], c2[kMaxPoles], c3[kMaxPoles];
  // the storage's own values, for the forward (explicit) updates
  double freq[kMaxPoles], gamma[kMaxPoles];
};

// Material coefficients for the FP32 fused method (scaled variables)
struct MatF32 {
  float inv_eps;  // 1/eps_inf
  int npoles;     // 0: non-dispersive; Drude: -1 (one J only)
  float a[2], b[2], c[2];
  float inv_mu;   // 1/mu_r (magnetic ConstantUpdate K; 1 for VacuumUpdate)
  // Drude: Jt' = a*Jt + b*E
  // Lorentz pole: Pt' = Pt + Jt; Jt' = a*Jt + b*E - c*Pt'
};

struct SourceDev {
  long long cell;  // linear index into the field arrays
  int comp, target, nvals;
  const double* vals;
  int i, j, k;
};

struct PlaneDev {
  int axis, aux;
  int lo[3], hi[3];
  double normal[3], k[3], pol_e[3], pol_h[3], origin[3];
  long long off;  // FP64 method: the plane's first cell in the table of precomputed corrections
};

struct AuxTab {
  int L;
  const double* Etab;  // [rows][L]: Ez after (t0 + row) aux steps
  const double* Htab;  // [rows][L]: Hy after (t0 + row) aux steps
};

struct Control {
  long long t;   // steps taken
  long long t0;  // first step of the current aux table chunk
  long long dft_base;  // step of the first sample in the DFT buffers
  unsigned int done_blocks;
  int error;
};

template <typename R>
struct FieldSet {
  R* f[3];
};

struct PlainArgs {
  int nx, ny, nz;
  double dt, dx;
  FieldSet<double> D, E, B, H;
  FieldSet<double> P[kMaxPoles], J[kMaxPoles];
  double* psi[2][3][3];
  Prof<double> prof[2][3];
  Slab slab[3];
  int pml_axis[3];
  const uint8_t* ids;
  const uint16_t* bids;
  int bshift, nbx, nby;
  const MatF64* mats;
  const double* eps_map;  // per-cell relative permittivity of non-dispersive cells (> 0), or null
  int dispersive;      // most poles of any material (Drude: 1)
  int all_dispersive;  // every material has poles: P and J are read with the fields
  int single_mat;      // the table holds one material: no cell's id is read
  int uniform_mu;      // every material has the same mu_r: the H half reads no id
  int nsrc;
  SourceDev src[kMaxSources];
  int nplanes;
  PlaneDev planes[kMaxPlanes];
  AuxTab aux[kMaxPlanes];
  Control* ctrl;
  // time policy of the curl updates (include/YeeUpdates.hpp:182-294): bd
  // history levels (0 BD1, 2 BD3, 3 BD4), bdk the coefficients of
  // TimePolicy::get, cc its curl_coeff; hist[D|B][level][comp]
  int bd;
  double bdk[4];
  double cc;
  double* hist[2][3][3];
  int kbeg, kend;  // 3D: the sweeps update planes kbeg .. kend-1 (all interior planes: 1 .. nz-2)
  // the half step's TFSF corrections of every plane cell ([off + cell][3]),
  // formed before each sweep by launch_tfsf_pre
  double* tfsf_pre;
};

struct FusedArgs {
  int nx, ny, nz, pitch;
  int flen[3];   // length of each axis' scaled profile; the raw F follows it
  float ce, ch;  // dt/(eps0 eta dx), eta dt/(mu0 dx)
  float* E[3];
  float* H[3];   // eta * H
  float* P[2][3];
  float* J[2][3];
  float* psi[2][3][3];
  Prof<float> prof[2][3];
  Slab slab[3];
  int pml_axis[3];
  const uint8_t* ids;
  const uint16_t* bids;
  int bshift, nbx, nby;
  const MatF32* mats;
  const float* inv_eps_map;  // per-cell 1/eps of non-dispersive cells (> 0), or null
  int max_poles;  // 0 none, -1 Drude only, 1..2 Lorentz
  int all_dispersive;  // every material of the table has poles
  int has_mu;          // some material has mu_r != 1: the H updates scale by 1/mu_r
  int nsrc;
  SourceDev src[kMaxSources];
  float src_scale_d;  // 1/eps0 for D-target sources
  float src_scale_b;  // eta/mu0 for B-target sources
  float src_scale_h;  // eta for H-target sources (H is stored as eta*H)
  double* src_last;   // per source: value added to E at the previous step
  int nplanes;
  PlaneDev planes[kMaxPlanes];
  AuxTab aux[kMaxPlanes];
  double dx, dt;
  double eta;
  Control* ctrl;
  int item_rows;  // batches: rows of one work item of this grid (a multiple of the kernel's rows; 0: the kernel's)
  int kbeg, kend;  // the staged 3D sweeps update planes kbeg .. kend-1 (all interior planes: 1 .. nz-2)
};

struct DftRegionDev {
  int comp, nf;
  // quantity: kind 0 a field component (comp of the phase's E or H), 1 the
  // surface current Je, 2 Jh, 3 the surface charge density rho (comp 0);
  // mode the grid's EM mode; scale the factor of the derived quantities
  int kind, mode;
  double scale;
  double acc_scale;  // factor of every sample as the flush folds it (1/eta for stored eta*H)
  int lo[3], ext[3];
  long long npts, pt_off;
  const double* freqs;
  double* acc;  // [nf][npts][2]
};

// adjoint of the FP32 fused 2D TM step (kernels_adjoint.cu); all arrays in
// the grid's pitch layout unless noted
struct AdjArgs {
  int nx, ny, pitch;
  Prof<float> prof[2][3];
  Slab slab[3];
  int pml_axis[3];
  const float* ie;                  // 1/eps per cell
  float *aez, *ahx, *ahy;           // adjoint fields
  float *apzx, *apzy, *apxy, *apyx; // adjoint CPML integrators (compact slabs)
  float *rxy, *ryx, *rzx, *rzy;     // adjoints of the curl differences
  int plo[2], phi[2];               // probe box (inclusive)
  const double* X;                  // probe DFT (re, im), probe box order
  double freq;                      // cycles per step
  int dlo[2], dhi[2];               // design box (inclusive)
  int ndesign;
  double* grad;                     // dJ/deps_r, design box order
  const Control* ctrl;              // the grid's step counter
};

// kernel launchers (stream-ordered); each returns the number of launches
int launch_plain_e(int mode, const PlainArgs& a, cudaStream_t s);
int launch_plain_h(int mode, const PlainArgs& a, cudaStream_t s);
// the forward material updates of field type ft on every interior cell
int launch_material_explicit(int mode, const PlainArgs& a, int ft, cudaStream_t s);
// the TFSF corrections of half step ft for every cell of every plane into a.tfsf_pre
int launch_tfsf_pre(int mode, const PlainArgs& a, int ft, cudaStream_t s);
int launch_fused_e(int mode, const FusedArgs& a, cudaStream_t s);
int launch_fused_h(int mode, const FusedArgs& a, cudaStream_t s);
bool fused3d_supported(const FusedArgs& a);
struct TmaState;
bool tma_prepare(const FusedArgs& a, TmaState** state);
void tma_release(TmaState* state);
int launch_tma_e(const FusedArgs& a, const TmaState* st, cudaStream_t s);
int launch_tma_h(const FusedArgs& a, const TmaState* st, cudaStream_t s);
int launch_flat_e(const FusedArgs& a, cudaStream_t s);
int launch_flat_h(const FusedArgs& a, cudaStream_t s);
int launch_staged_e(const FusedArgs& a, cudaStream_t s);
int launch_staged_h(const FusedArgs& a, cudaStream_t s);
// The whole 3D FP32 step (E and H sweeps) in one persistent launch: work
// items are tiles of one plane (128 cells x 4 rows) of the E or the H sweep,
// ordered E(1..lag), then E(k), H(k - lag) for k = lag+1..np, then the last
// H planes; the CTAs take items round-robin, and an H tile first waits for
// the E tiles it reads (flags holding the launch's epoch).
struct EhSched {
  int nbx, nby;           // tiles per plane: x blocks of 128 cells, y blocks of 4 rows
  int np;                 // interior planes (nz - 2)
  int lag;                // H of plane k - lag follows E of plane k
  long long nitems;       // 2 * np * nbx * nby
  unsigned* flags;        // [np][nbx * nby]: epoch at which E of (plane, tile) was stored
  const unsigned* epoch;  // steps launched so far; this launch's epoch is *epoch + 1
};
// Plans the one-launch step of grid `a` on the current device: the tiles,
// the resident CTAs (`blocks`) and the lag. false if the grid needs the two
// sweeps (or the kernel cannot be resident).
bool staged_eh_plan(const FusedArgs& a, EhSched* s, int* blocks);
int launch_staged_eh(const FusedArgs& a, const EhSched& s, int blocks, cudaStream_t st);
int launch_tfsf_fused(int mode, const FusedArgs& a, int ft, cudaStream_t s);
int launch_fused3d_e(const FusedArgs& a, cudaStream_t s);
int launch_fused3d_h(const FusedArgs& a, cudaStream_t s);
int launch_aux_precompute(int L, double dt, double dx, double* Dz, double* Ez, double* By, double* Hy,
                          double* psiE, double* psiH, const double* coef, const double* vals, int nvals,
                          long long s0, int nsteps, double* Etab, double* Htab, cudaStream_t s);
int launch_dft_gather(int precision, const DftRegionDev* regions, int nreg, long long total_pts, long long max_pts,
                      const void* const* fields, int ny, int pitch, int slot, void* buf, cudaStream_t s);
// one quantity over a box into out (npts values of the field precision)
int launch_quantity_read(int precision, const DftRegionDev& r, const void* const* fields, int ny, int pitch,
                         void* out, cudaStream_t s);
int launch_dft_flush(int phase, int precision, const DftRegionDev* regions, int nreg, long long max_pts,
                     long long total_pts, const void* buf, const Control* ctrl, int nsamp, cudaStream_t s);
int launch_dft_rebase(Control* ctrl, int nsamp, cudaStream_t s);
int launch_dft_set_base(Control* ctrl, long long base, cudaStream_t s);
int launch_finite_check(const void* p, long long n, int is_f32, int* flag, cudaStream_t s);
int launch_step_advance(Control* ctrl, cudaStream_t s);
// advances the step counter and, if non-null, the one-launch step's epoch
int launch_step_advance(Control* ctrl, unsigned* epoch, cudaStream_t s);
// out[0] += sum over rows of (a*sa - b*sb)^2, out[1] += sum (b*sb)^2 (FP64)
int launch_field_diff(const void* a, int a_f32, long long rla, double sa, const void* b, int b_f32, long long rlb,
                      double sb, int nx, long long nrows, double* out, cudaStream_t s);
int launch_chunk_start(Control* ctrl, cudaStream_t s);
// ctrl->t = ctrl->t0 = t, on the stream
int launch_set_step(Control* ctrl, long long t, cudaStream_t s);
// faces with a boundary condition (kind 1 PEC, 2 PMC, 3 symmetric,
// 4 antisymmetric, 5 periodic)
struct BcFace {
  int axis, side, kind;
  float sgn[2][3];  // the condition's sign per component, E (0) and H (1) half
};
// the sign of component c of field type ft for a face of `kind` normal to axis
__host__ __device__ float bc_sign(int kind, int ft, int c, int axis);
struct BcFaces {
  int n;
  BcFace face[6];
};
int launch_boundaries(const BcFaces& f, int ft, int is_f32, void* const* fields, int nx, int ny, int nz, int rowlen,
                      cudaStream_t s);
int launch_adjoint_inv_eps(const FusedArgs& fa, float* ie, cudaStream_t s);
int launch_adjoint_capture(const AdjArgs& a, const float* hx, const float* hy, float* slot, cudaStream_t s);
int launch_adjoint_step(const AdjArgs& a, int back, const float* dslot, cudaStream_t s);
int launch_box_source(int is_f32, void* field, const int* lo, const int* hi, int pitch, int ny, const double* vals,
                      int nvals, double scale, int shift, const Control* ctrl, cudaStream_t s);
// control block of a batch's persistent kernel (grid barrier + error flag)
struct BatchCtl {
  unsigned count;  // CTAs arrived at the current barrier
  unsigned gen;    // barrier generation
  int error;       // bit 0: a barrier wait expired
  int pad;
};
void* batch_kernel_ptr(int mode, int maxp, int rows);
void* batch_phase_ptr(int mode, int maxp, int rows, int phase);
int launch_batch_advance(Control* const* ctrls, int n, int nsteps, cudaStream_t s);
// temporal blocking of a batch (depth 2, 3 or 4 steps per launch): the exact
// tile of a window (*tw x *th cells; 0 for an unsupported depth), and one
// launch over the tiles `items` that reads the state through `rd` and writes
// it through `wr` (one FusedArgs per grid each), steps s .. s + depth - 1
// past the counters
int batch_tb_tile(int depth, int* tw, int* th);
int launch_batch_tb(int mode, int depth, const FusedArgs* rd, const FusedArgs* wr, const unsigned* items,
                    int nitems, int s, cudaStream_t st);

}  // namespace fdtdb
