// Host implementation of the C ABI declared in include/fdtd_b200.h.
//
// Set-up work (CPML grading, material coefficients, TFSF plane checks) is
// done here on the host in FP64, in the reference's operation order; this file
// is compiled with -Xcompiler -ffp-contract=off so that, e.g., the coefficients
// of NewPML::setPMLParameters (include/PML.hpp:84-102) round exactly as in the
// reference. The time loop itself is a fixed sequence of stream-ordered
// launches per step: E sweep, E-phase DFT, H sweep, H-phase DFT, step counter.
#include <cmath>
#include <cstdio>
#include <algorithm>
#include <cstring>
#include <exception>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "../../include/fdtd_b200.h"
#include "internal.h"

using namespace fdtdb;

static thread_local std::string g_err;

static int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

#define CK(call)                                                                         \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess) return fail(FDTD_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

extern "C" const char* fdtd_last_error_string(void) { return g_err.c_str(); }

// No C++ exception may leave the C ABI: each entry point is a function-try-
// block whose handler turns a host allocation failure (std::bad_alloc from a
// container, say) or any other exception into an error code.
static int host_failure() {
  try {
    throw;
  } catch (const std::bad_alloc&) {
    g_err = "host memory allocation failed";
    return FDTD_ERR_NOMEM;
  } catch (const std::exception& e) {
    try {
      g_err = std::string("host error: ") + e.what();
    } catch (...) {
    }
    return FDTD_ERR_INVALID;
  } catch (...) {
    return FDTD_ERR_INVALID;
  }
}

namespace {

// the reference's constexpr Newton sqrt (include/FDTDConstants.hpp:136-156)
double ref_sqrt(double x) {
  double curr = x, prev = 0.0;
  while (curr != prev) {
    double next = 0.5 * (curr + x / curr);
    prev = curr;
    curr = next;
  }
  return curr;
}
double imp0() { return ref_sqrt(kMu0 / kEps0); }

// PMLParameterModel(dx) and PMLParameterModel(m, ma, sMax, kMax, aMax)
// (include/PML.hpp:368-393)
struct PmlModel {
  double m, ma, smax, kmax, amax;
  explicit PmlModel(double dx) : m(3), ma(1), smax(0.8 * (m + 1) / (imp0() * dx)), kmax(5), amax(0.05) {}
  PmlModel(double m_, double ma_, double smax_, double kmax_, double amax_)
      : m(m_), ma(ma_), smax(smax_), kmax(kmax_), amax(amax_) {}
  double K(double x) const { if (x < 0.0) return 1.0; return x > 1.0 ? 1.0 : 1.0 + pow(x, m) * (kmax - 1.0); }
  double S(double x) const { if (x < 0.0) return 0.0; return x > 1.0 ? 0.0 : pow(x, m) * smax; }
  double A(double x) const { if (x < 0.0) return 0.0; return x > 1.0 ? 0.0 : pow(1.0 - x, ma) * amax; }
};

// NewPML::setPMLParameters (include/PML.hpp:84-102)
void set_params(double K, double S, double A, double dt, double& B, double& C, double& F, double& G) {
  double nu = 1.0 / kEps0 * (S / K + A);
  B = exp(-dt * nu);
  C = (nu == 0) ? 0.0 : S / K * 1.0 / (S + K * A) * (B - 1.0);
  double u = -S / (kEps0 * K * K);
  F = (nu == 0) ? 1.0 / K : 1.0 / K - 1.0 / dt * (1.0 - B - nu * dt) * u / (nu * nu);
  G = (nu == 0) ? 0.0 : 1.0 / dt * (1.0 - B) / nu;
}

struct Profile {  // one (field type, axis)
  std::vector<double> B, C, F, G;
  void reset(int n) {
    B.assign(n, 0.0);
    C.assign(n, 0.0);
    F.assign(n, 1.0);  // NewPML defaults (PML.hpp:40-55)
    G.assign(n, 0.0);
  }
};

// grading loop of tests/testTM.cpp:44-71 for one side of one axis
void grade(const PmlModel& p, double dt, int n, int np, int side, Profile& e, Profile& h) {
  for (int i = 1; i < np + 2; i++) {
    double x = static_cast<double>(np - i + 1) / static_cast<double>(np);
    double xm = x - 0.5 / static_cast<double>(np);
    int ce = side == 0 ? i : n - i;
    int cm = side == 0 ? i : n - 1 - i;
    if (ce >= 0 && ce < n) set_params(p.K(x), p.S(x), p.A(x), dt, e.B[ce], e.C[ce], e.F[ce], e.G[ce]);
    if (cm >= 0 && cm < n) set_params(p.K(xm), p.S(xm), p.A(xm), dt, h.B[cm], h.C[cm], h.F[cm], h.G[cm]);
  }
}

struct SourceH {
  int comp, target, i, j, k;
  std::vector<double> vals;
  double* d_vals = nullptr;
};

struct BoxSourceH {
  int comp, target, lo[3], hi[3];
  double* d_vals = nullptr;
  int nvals = 0;
};

struct AuxH {
  int ncells, L;
  std::vector<double> vals;
  double *d_state = nullptr;  // Dz, Ez, By, Hy, psiE, psiH (6L)
  double *d_coef = nullptr;   // 8L
  double *d_vals = nullptr;
  double *d_tab = nullptr;    // 2 * cap * L
  long long cap = 0;
};

struct PlaneH {
  PlaneDev dev;
};

struct DftH {
  int comp, nf;
  int lo[3], hi[3];
  long long npts;
  std::vector<double> freqs;
  double* d_freqs = nullptr;
  double* d_acc = nullptr;
};

}  // namespace

struct fdtd_grid {
  fdtd_grid_desc d{};
  int n[3]{1, 1, 1};
  int pitch = 0;
  bool f32 = false;
  cudaStream_t stream = nullptr;
  std::vector<void*> allocs;
  std::map<void*, size_t> sizes;
  long long bytes = 0;
  long long launches = 0;
  long long t = 0;
  int pml[3][2]{};
  // the grading of each CPML side: PMLParameterModel(dx) unless
  // fdtd_set_pml_model gave the model's five parameters
  bool pml_custom[3][2]{};
  double pml_model[3][2][5]{};
  Profile prof[2][3];
  std::vector<fdtd_material> mats;
  // device state
  void* E[3]{};
  void* H[3]{};
  void* D[3]{};
  void* B[3]{};
  void* P[kMaxPoles][3]{};
  void* J[kMaxPoles][3]{};
  void* psi[2][3][3]{};
  void* d_prof[2][3][4]{};  // F32 F array holds scaled F then raw F
  int npoles_alloc = 0;
  Slab slab[3]{};
  uint8_t* d_ids = nullptr;
  uint16_t* d_bids = nullptr;
  void* d_eps_map = nullptr;  // plain: double eps; fused: float 1/eps (pitch layout)
  double* d_tfsf_pre = nullptr;  // plain: the half step's TFSF corrections, 3 per plane cell
  long long tfsf_cells = 0;      // cells of all TFSF planes
  int bshift = 0, nbx = 0, nby = 0, nbz = 0;
  void* d_mats = nullptr;
  int max_poles = 0;
  std::vector<SourceH> srcs;
  std::vector<BoxSourceH> boxes;
  double* d_src_last = nullptr;
  std::vector<PlaneH> planes;
  std::vector<AuxH> auxes;
  std::vector<DftH> dfts;
  DftRegionDev* d_dft[2]{};
  int ndft[2]{};
  long long dft_pts[2]{};
  long long dft_maxpts[2]{};
  void* d_dft_buf[2]{};   // [kDftChunk][points] samples per phase
  int dft_pending = 0;    // samples in the buffers: the slot of the next one
  void** d_fieldptrs = nullptr;  // [E0,E1,E2,H0,H1,H2]
  Control* ctrl = nullptr;
  int* d_flag = nullptr;
  char* h_stage = nullptr;  // two pinned chunks of kStageChunk bytes for large reads
  cudaEvent_t stage_ev[2]{};
  bool dirty_dft = true;
  bool dirty_pml = false;  // host CPML profiles changed: device profiles and slabs follow before use
  int next_half = 0;  // fdtd_step_half: the phase expected next
  bool half_split = false;  // fdtd_step_half_part: part 0 of the half step ran, part 1 is due
  BcFaces bcs{};      // faces with a boundary condition
  int scheme = 1;     // time policy of the curl updates: 1 BD1, 3 BD3, 4 BD4
  void* hist[2][3][3]{};  // FP64 flux history [D|B][level][comp] of BD3/BD4
  int sweep_kind = FDTD_SWEEP_AUTO;
  TmaState* tma = nullptr;
  unsigned* d_eh = nullptr;  // one-launch step: [0] epoch, then the E tile flags
  long long eh_words = 0;
  long long version = 0;        // bumped by every change a captured graph would bake in
  long long graph_version = -1;
  cudaGraphExec_t graph = nullptr;
  long long graph_launches = 0;
  bool use_graphs = true;
};

namespace {

size_t elem(const fdtd_grid* g) { return g->f32 ? 4 : 8; }

// Copies `bytes` from pinned `src` into a host buffer with several threads.
// A fresh pageable buffer's first touch costs a page fault per 4 KB, which one
// thread takes one after another; the kernel serves faults of different
// threads in parallel. Each thread takes at least 1 MB.
void parallel_host_copy(char* dst, const char* src, size_t bytes) {
  constexpr size_t kPerThread = size_t(1) << 20;
  const size_t most = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  const size_t nt = std::max<size_t>(1, std::min(most, bytes / kPerThread));
  if (nt == 1) {
    std::memcpy(dst, src, bytes);
    return;
  }
  const size_t per = (bytes + nt - 1) / nt;
  std::vector<std::thread> th;
  for (size_t q = 0; q < nt; q++) {
    const size_t lo = q * per, hi = std::min(bytes, lo + per);
    if (lo >= hi) break;
    try {
      th.emplace_back([=] { std::memcpy(dst + lo, src + lo, hi - lo); });
    } catch (...) {
      // no thread to be had (resource limits): this thread copies the slice;
      // nothing may throw across the C ABI
      std::memcpy(dst + lo, src + lo, hi - lo);
    }
  }
  for (auto& t : th) t.join();
}

long long rowlen(const fdtd_grid* g) { return g->f32 ? g->pitch : g->n[0]; }
long long field_elems(const fdtd_grid* g) { return rowlen(g) * g->n[1] * g->n[2]; }

int dalloc(fdtd_grid* g, void** p, size_t bytes) {
  g->version++;
  *p = nullptr;
  if (bytes == 0) bytes = 16;
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    return fail(e == cudaErrorMemoryAllocation ? FDTD_ERR_NOMEM : FDTD_ERR_CUDA,
                std::string("cudaMalloc failed: ") + cudaGetErrorString(e));
  }
  e = cudaMemsetAsync(*p, 0, bytes, g->stream);
  if (e != cudaSuccess) return fail(FDTD_ERR_CUDA, cudaGetErrorString(e));
  g->allocs.push_back(*p);
  g->sizes[*p] = bytes;
  g->bytes += static_cast<long long>(bytes);
  return FDTD_OK;
}

void dfree(fdtd_grid* g, void* p) {
  g->version++;
  if (!p) return;
  for (size_t q = 0; q < g->allocs.size(); q++)
    if (g->allocs[q] == p) {
      g->allocs.erase(g->allocs.begin() + q);
      break;
    }
  auto it = g->sizes.find(p);
  if (it != g->sizes.end()) {
    g->bytes -= static_cast<long long>(it->second);
    g->sizes.erase(it);
  }
  cudaFree(p);
}

int upload_vec(fdtd_grid* g, void** p, const void* src, size_t bytes) {
  if (*p) dfree(g, *p);
  int rc = dalloc(g, p, bytes);
  if (rc) return rc;
  CK(cudaMemcpyAsync(*p, src, bytes, cudaMemcpyHostToDevice, g->stream));
  return FDTD_OK;
}

int dim_of(const fdtd_grid* g) { return g->d.mode == kThreeD ? 3 : 2; }

double eta() { return imp0(); }
double ce_of(const fdtd_grid* g) { return g->d.dt / (kEps0 * eta() * g->d.dx); }
double ch_of(const fdtd_grid* g) { return eta() * g->d.dt / (kMu0 * g->d.dx); }

int upload_profiles(fdtd_grid* g) {
  CK(cudaStreamSynchronize(g->stream));
  for (int ft = 0; ft < 2; ft++)
    for (int a = 0; a < 3; a++) {
      const Profile& p = g->prof[ft][a];
      const int n = g->n[a];
      for (int q = 0; q < 4; q++) {
        if (g->f32) {
          const double c = ft == 0 ? ce_of(g) : ch_of(g);
          const int len = a == 0 ? g->pitch : n;  // x profiles padded to the row pitch
          std::vector<float> v(q == 2 ? 2 * len : len, 0.0f);
          for (int i = 0; i < n; i++) {
            if (q == 0) v[i] = static_cast<float>(p.B[i]);
            if (q == 1) v[i] = static_cast<float>(c * p.C[i]);
            if (q == 2) {
              v[i] = static_cast<float>(c * p.F[i]);
              v[len + i] = static_cast<float>(p.F[i]);
            }
            if (q == 3) v[i] = static_cast<float>(p.G[i]);
          }
          int rc = upload_vec(g, &g->d_prof[ft][a][q], v.data(), v.size() * sizeof(float));
          if (rc) return rc;
        } else {
          std::vector<double> v(n);
          for (int i = 0; i < n; i++) {
            if (q == 0) v[i] = p.B[i];
            if (q == 1) v[i] = p.C[i] / g->d.dx;  // (C*LC)/dx = LC*(C/dx)
            if (q == 2) v[i] = p.F[i] / g->d.dx;  // (LC*F)/dx = LC*(F/dx)
            if (q == 3) v[i] = p.G[i];
          }
          int rc = upload_vec(g, &g->d_prof[ft][a][q], v.data(), v.size() * sizeof(double));
          if (rc) return rc;
        }
      }
    }
  return FDTD_OK;
}

int alloc_psi(fdtd_grid* g);

// fdtd_set_pml regrades the host profiles only; the device profiles and the
// CPML integrator slabs (zeroed) follow here, once, before anything reads them
int ensure_pml(fdtd_grid* g) {
  if (!g->dirty_pml) return FDTD_OK;
  int rc = upload_profiles(g);
  if (rc) return rc;
  rc = alloc_psi(g);
  if (rc) return rc;
  g->dirty_pml = false;
  return FDTD_OK;
}

// The one-launch 3D FP32 step keeps an epoch and one flag per E tile of
// every plane (zeroed); laid out once, before any step that may use it.
bool eh_wanted(const fdtd_grid* g) {
  return g->f32 && g->d.mode == kThreeD && (g->sweep_kind == FDTD_SWEEP_EH || g->sweep_kind == FDTD_SWEEP_AUTO);
}

int ensure_eh(fdtd_grid* g) {
  if (!eh_wanted(g) || g->d_eh) return FDTD_OK;
  const long long nbx = g->pitch / 128, nby = (g->n[1] - 2 + 7) / 8, np = g->n[2] - 2;  // tiles of 128 x 8
  if (nbx <= 0 || nby <= 0 || np <= 0) return FDTD_OK;
  g->eh_words = 1 + nbx * nby * np;
  return dalloc(g, reinterpret_cast<void**>(&g->d_eh), static_cast<size_t>(g->eh_words) * sizeof(unsigned));
}

// the FP32 method keeps its x slabs in the aligned layout (Slab::lo4)
static bool xslab_aligned(const fdtd_grid* g) { return g->f32; }
static long long xslab_row(const fdtd_grid* g) { return xslab_aligned(g) ? g->slab[0].W4 : g->slab[0].W; }

int alloc_psi(fdtd_grid* g) {
  for (int ft = 0; ft < 2; ft++)
    for (int I = 0; I < 3; I++)
      for (int J = 0; J < 3; J++) {
        if (g->psi[ft][I][J]) {
          dfree(g, g->psi[ft][I][J]);
          g->psi[ft][I][J] = nullptr;
        }
      }
  for (int a = 0; a < 3; a++) g->slab[a] = make_slab(g->n[a], g->pml[a][0], g->pml[a][1]);
  for (int ft = 0; ft < 2; ft++)
    for (int I = 0; I < 3; I++) {
      const bool has = ft == 0 ? hasE(g->d.mode, I) : hasH(g->d.mode, I);
      if (!has) continue;
      for (int J = 0; J < 3; J++) {
        if (J == I || g->slab[J].W == 0) continue;
        long long cnt;
        if (J == 0) cnt = static_cast<long long>(g->n[2]) * g->n[1] * xslab_row(g);
        else if (J == 1) cnt = static_cast<long long>(g->n[2]) * g->slab[1].W * rowlen(g);
        else cnt = static_cast<long long>(g->slab[2].W) * g->n[1] * rowlen(g);
        int rc = dalloc(g, &g->psi[ft][I][J], cnt * elem(g));
        if (rc) return rc;
      }
    }
  return FDTD_OK;
}

long long cell_index(const fdtd_grid* g, int i, int j, int k) {
  return (static_cast<long long>(k) * g->n[1] + j) * rowlen(g) + i;
}

bool interior(const fdtd_grid* g, int i, int j, int k) {
  if (i < 1 || i > g->n[0] - 2 || j < 1 || j > g->n[1] - 2) return false;
  if (g->d.mode == kThreeD) return k >= 1 && k <= g->n[2] - 2;
  return k == 0;
}

int build_materials(fdtd_grid* g) {
  const double dt = g->d.dt;
  int maxp = 0;
  bool drude = false;
  if (g->f32) {
    std::vector<MatF32> v(g->mats.size());
    for (size_t q = 0; q < g->mats.size(); q++) {
      const fdtd_material& m = g->mats[q];
      MatF32& o = v[q];
      memset(&o, 0, sizeof(o));
      o.inv_eps = static_cast<float>(m.kind == FDTD_VACUUM ? 1.0 : 1.0 / m.eps_inf);
      o.inv_mu = static_cast<float>(1.0 / m.mu_r);
      if (m.kind == FDTD_DRUDE) {
        const double bb = m.gamma[0] * dt * 0.5, w = dt * m.freq[0];
        o.npoles = -1;
        o.a[0] = static_cast<float>((1.0 - bb) / (1.0 + bb));
        o.b[0] = static_cast<float>(w * w);
        drude = true;
      } else if (m.kind == FDTD_LORENTZ) {
        if (m.npoles > 2) return fail(FDTD_ERR_UNSUPPORTED, "the FP32 fused method takes at most 2 Lorentz poles");
        o.npoles = m.npoles;
        for (int p = 0; p < m.npoles; p++) {
          const double bb = 1.0 + m.gamma[p] * dt, bm = 1.0 - m.gamma[p] * dt, w = m.freq[p] * dt;
          o.a[p] = static_cast<float>(bm / bb);
          o.b[p] = static_cast<float>(w * w * m.delta_eps[p] / bb);
          o.c[p] = static_cast<float>(w * w / bb);
        }
        maxp = std::max(maxp, m.npoles);
      }
    }
    g->max_poles = maxp > 0 ? maxp : (drude ? -1 : 0);
    if (drude && maxp == 0) maxp = 1;
    int rc = upload_vec(g, &g->d_mats, v.data(), v.size() * sizeof(MatF32));
    if (rc) return rc;
  } else {
    std::vector<MatF64> v(g->mats.size());
    for (size_t q = 0; q < g->mats.size(); q++) {
      const fdtd_material& m = g->mats[q];
      MatF64& o = v[q];
      memset(&o, 0, sizeof(o));
      o.kind = m.kind;
      o.npoles = m.kind == FDTD_DRUDE ? 1 : (m.kind == FDTD_LORENTZ ? m.npoles : 0);
      // VacuumStorage K = 1 (DispersiveMaterials.hpp:446-457)
      o.den_e = (m.kind == FDTD_VACUUM ? 1.0 : m.eps_inf) * kEps0;
      o.den_h = m.mu_r * kMu0;
      for (int p = 0; p < o.npoles; p++) {
        o.freq[p] = m.freq[p];
        o.gamma[p] = m.gamma[p];
      }
      if (m.kind == FDTD_DRUDE) {
        // drude::DrudeUpdate::implicit_update (DispersiveMaterials.hpp:986-996)
        const double b = m.gamma[0] * dt * 0.5;
        const double w = dt * m.freq[0];
        o.c1[0] = 1.0 - b;
        o.c2[0] = 1.0 + b;
        o.c3[0] = w * w / dt * kEps0;
      } else if (m.kind == FDTD_LORENTZ) {
        // lorentz::LorentzUpdate::implicit_update (DispersiveMaterials.hpp:719-732)
        for (int p = 0; p < m.npoles; p++) {
          const double b = 1.0 + m.gamma[p] * dt;
          const double bm = 1.0 - m.gamma[p] * dt;
          const double w = m.freq[p] * dt;
          const double qq = m.freq[p] * w / b;
          o.c1[p] = bm / b;
          o.c2[p] = qq * m.delta_eps[p] * kEps0;
          o.c3[p] = qq;
        }
      }
      maxp = std::max(maxp, o.npoles);
    }
    g->max_poles = maxp;
    int rc = upload_vec(g, &g->d_mats, v.data(), v.size() * sizeof(MatF64));
    if (rc) return rc;
  }
  // polarisation state for the poles in use
  const int need = g->f32 ? (g->max_poles < 0 ? 1 : g->max_poles) : maxp;
  for (int p = g->npoles_alloc; p < need; p++)
    for (int c = 0; c < 3; c++) {
      if (!hasE(g->d.mode, c)) continue;
      int rc = dalloc(g, &g->P[p][c], field_elems(g) * elem(g));
      if (rc) return rc;
      rc = dalloc(g, &g->J[p][c], field_elems(g) * elem(g));
      if (rc) return rc;
    }
  g->npoles_alloc = std::max(g->npoles_alloc, need);
  return FDTD_OK;
}

// Aux1D set-up (include/Source.hpp:368-390): a TEM grid of ncells+50 cells
// with a 15-cell CPML graded like the main grid, both sides in one loop.
int build_aux(fdtd_grid* g, AuxH& a) {
  const int L = a.L;
  Profile e, h;
  e.reset(L);
  h.reset(L);
  PmlModel pm(g->d.dx);
  for (int i = 1; i < kAuxNpml + 2; i++) {
    double x = static_cast<double>(kAuxNpml - i + 1) / static_cast<double>(kAuxNpml);
    double xm = x - 0.5 / static_cast<double>(kAuxNpml);
    set_params(pm.K(x), pm.S(x), pm.A(x), g->d.dt, e.B[i], e.C[i], e.F[i], e.G[i]);
    set_params(pm.K(xm), pm.S(xm), pm.A(xm), g->d.dt, h.B[i], h.C[i], h.F[i], h.G[i]);
    set_params(pm.K(x), pm.S(x), pm.A(x), g->d.dt, e.B[L - i], e.C[L - i], e.F[L - i], e.G[L - i]);
    set_params(pm.K(xm), pm.S(xm), pm.A(xm), g->d.dt, h.B[L - 1 - i], h.C[L - 1 - i], h.F[L - 1 - i],
               h.G[L - 1 - i]);
  }
  std::vector<double> coef(8 * static_cast<size_t>(L));
  for (int i = 0; i < L; i++) {
    coef[i] = e.B[i];
    coef[L + i] = e.C[i] / g->d.dx;
    coef[2 * L + i] = e.F[i] / g->d.dx;
    coef[3 * L + i] = e.G[i];
    coef[4 * L + i] = h.B[i];
    coef[5 * L + i] = h.C[i] / g->d.dx;
    coef[6 * L + i] = h.F[i] / g->d.dx;
    coef[7 * L + i] = h.G[i];
  }
  int rc = upload_vec(g, reinterpret_cast<void**>(&a.d_coef), coef.data(), coef.size() * sizeof(double));
  if (rc) return rc;
  rc = dalloc(g, reinterpret_cast<void**>(&a.d_state), 6 * static_cast<size_t>(L) * sizeof(double));
  if (rc) return rc;
  return upload_vec(g, reinterpret_cast<void**>(&a.d_vals), a.vals.data(),
                    std::max<size_t>(1, a.vals.size()) * sizeof(double));
}

// Quantities by code (fdtd_add_dft, fdtd_read_quantity): 0..2 E, 3..5 H,
// 6..8 Je, 9..11 Jh, 12 rho. Phase 0 samples after the E half (E, Jh, rho),
// phase 1 after the H half (H, Je).
int quantity_phase(int q) { return (q >= 3 && q < 9) ? 1 : 0; }

bool quantity_in_mode(const fdtd_grid* g, int q) {
  const int m = g->d.mode;
  if (q < 0 || q > 12) return false;
  if (q < 3) return hasE(m, q);
  if (q < 6) return hasH(m, q - 3);
  if (q < 9) return hasE(m, q - 6);
  if (q < 12) return hasH(m, q - 9);
  return m != FDTD_TM;
}

int quantity_check(const fdtd_grid* g, int q, const int* lo, const int* hi) {
  if (q < 0 || q > 12) return fail(FDTD_ERR_INVALID, "quantity must be 0..12");
  if (!quantity_in_mode(g, q)) return fail(FDTD_ERR_INVALID, "quantity not in this mode");
  const int dim = dim_of(g);
  for (int d = 0; d < 3; d++) {
    if (lo[d] < 0 || hi[d] >= g->n[d] || lo[d] > hi[d]) return fail(FDTD_ERR_INVALID, "box outside the grid");
    if (q >= 6 && d < dim && (lo[d] < 1 || hi[d] > g->n[d] - 2))
      return fail(FDTD_ERR_INVALID, "surface quantities are defined on interior cells only");
  }
  return FDTD_OK;
}

// the device description of quantity q over lo..hi
DftRegionDev quantity_region(const fdtd_grid* g, int q, const int* lo, const int* hi) {
  DftRegionDev o{};
  o.mode = g->d.mode;
  o.kind = q < 6 ? 0 : q < 9 ? 1 : q < 12 ? 2 : 3;
  o.comp = q < 12 ? q % 3 : 0;
  const double dx = g->d.dx;
  // SurfaceQuantities.hpp:211, :265, :324: 1.0/dx, -1.0/dx, eps0/dx; the
  // FP32 method stores eta*H, so Je takes a further 1/eta
  if (o.kind == 1) o.scale = g->f32 ? 1.0 / dx / eta() : 1.0 / dx;
  else if (o.kind == 2) o.scale = -1.0 / dx;
  else if (o.kind == 3) o.scale = kEps0 / dx;
  o.npts = 1;
  for (int d = 0; d < 3; d++) {
    o.lo[d] = lo[d];
    o.ext[d] = hi[d] - lo[d] + 1;
    o.npts *= o.ext[d];
  }
  return o;
}

// fold the buffered DFT samples of both phases into the accumulators
int flush_dft(fdtd_grid* g, cudaStream_t s) {
  int n = 0;
  for (int ph = 0; ph < 2; ph++)
    n += launch_dft_flush(ph, g->f32 ? 1 : 0, g->d_dft[ph], g->ndft[ph], g->dft_maxpts[ph], g->dft_pts[ph],
                          g->d_dft_buf[ph], g->ctrl, g->dft_pending, s);
  if (g->dft_pending > 0) n += launch_dft_rebase(g->ctrl, g->dft_pending, s);
  g->dft_pending = 0;
  return n;
}

int rebuild_dft(fdtd_grid* g) {
  if (g->dft_pending > 0) {
    // samples that fdtd_step_half left in the old layout's buffers
    CK(cudaDeviceSynchronize());
    g->launches += flush_dft(g, g->stream);
    CK(cudaStreamSynchronize(g->stream));
  }
  for (int ph = 0; ph < 2; ph++) {
    std::vector<DftRegionDev> v;
    long long off = 0;
    for (auto& r : g->dfts) {
      if (quantity_phase(r.comp) != ph) continue;
      DftRegionDev o = quantity_region(g, r.comp, r.lo, r.hi);
      o.nf = r.nf;
      o.npts = r.npts;
      o.pt_off = off;
      // spectra of H in SI units: the FP32 method stores eta*H
      o.acc_scale = g->f32 && r.comp >= 3 && r.comp < 6 ? 1.0 / eta() : 1.0;
      o.freqs = r.d_freqs;
      o.acc = r.d_acc;
      off += r.npts;
      v.push_back(o);
    }
    g->ndft[ph] = static_cast<int>(v.size());
    g->dft_pts[ph] = off;
    g->dft_maxpts[ph] = 0;
    for (auto& o : v) g->dft_maxpts[ph] = std::max(g->dft_maxpts[ph], o.npts);
    if (!v.empty()) {
      int rc = upload_vec(g, reinterpret_cast<void**>(&g->d_dft[ph]), v.data(), v.size() * sizeof(DftRegionDev));
      if (rc) return rc;
      if (g->d_dft_buf[ph]) dfree(g, g->d_dft_buf[ph]);
      rc = dalloc(g, &g->d_dft_buf[ph], static_cast<size_t>(kDftChunk) * off * elem(g));
      if (rc) return rc;
    }
  }
  if (!g->dfts.empty()) {
    // the first sample of the new layout is that of the next step
    g->launches += launch_dft_set_base(g->ctrl, g->t, g->stream);
  }
  g->dirty_dft = false;
  return FDTD_OK;
}

template <typename Args>
void fill_common(fdtd_grid* g, Args& a) {
  a.nx = g->n[0];
  a.ny = g->n[1];
  a.nz = g->n[2];
  for (int x = 0; x < 3; x++) {
    a.slab[x] = g->slab[x];
    a.pml_axis[x] = (g->pml[x][0] > 0 || g->pml[x][1] > 0) ? 1 : 0;
  }
  a.ids = g->d_ids;
  a.bids = g->d_bids;
  a.bshift = g->bshift;
  a.nbx = g->nbx;
  a.nby = g->nby;
  a.nsrc = static_cast<int>(g->srcs.size());
  for (size_t s = 0; s < g->srcs.size(); s++) {
    const SourceH& sh = g->srcs[s];
    SourceDev& o = a.src[s];
    o.cell = cell_index(g, sh.i, sh.j, sh.k);
    o.comp = sh.comp;
    o.target = sh.target;
    o.nvals = static_cast<int>(sh.vals.size());
    o.vals = sh.d_vals;
    o.i = sh.i;
    o.j = sh.j;
    o.k = sh.k;
  }
  a.nplanes = static_cast<int>(g->planes.size());
  for (size_t q = 0; q < g->planes.size(); q++) a.planes[q] = g->planes[q].dev;
  for (size_t q = 0; q < g->auxes.size(); q++) {
    const AuxH& ax = g->auxes[q];
    a.aux[q].L = ax.L;
    a.aux[q].Etab = ax.d_tab;
    a.aux[q].Htab = ax.d_tab + ax.cap * ax.L;
  }
  a.ctrl = g->ctrl;
}

PlainArgs plain_args(fdtd_grid* g) {
  PlainArgs a;
  memset(&a, 0, sizeof(a));
  fill_common(g, a);
  a.dt = g->d.dt;
  a.dx = g->d.dx;
  for (int c = 0; c < 3; c++) {
    a.D.f[c] = static_cast<double*>(g->D[c]);
    a.E.f[c] = static_cast<double*>(g->E[c]);
    a.B.f[c] = static_cast<double*>(g->B[c]);
    a.H.f[c] = static_cast<double*>(g->H[c]);
    for (int p = 0; p < kMaxPoles; p++) {
      a.P[p].f[c] = static_cast<double*>(g->P[p][c]);
      a.J[p].f[c] = static_cast<double*>(g->J[p][c]);
    }
  }
  for (int ft = 0; ft < 2; ft++)
    for (int I = 0; I < 3; I++)
      for (int J = 0; J < 3; J++) a.psi[ft][I][J] = static_cast<double*>(g->psi[ft][I][J]);
  for (int ft = 0; ft < 2; ft++)
    for (int x = 0; x < 3; x++) {
      a.prof[ft][x].B = static_cast<const double*>(g->d_prof[ft][x][0]);
      a.prof[ft][x].C = static_cast<const double*>(g->d_prof[ft][x][1]);
      a.prof[ft][x].F = static_cast<const double*>(g->d_prof[ft][x][2]);
      a.prof[ft][x].G = static_cast<const double*>(g->d_prof[ft][x][3]);
    }
  a.mats = static_cast<const MatF64*>(g->d_mats);
  a.eps_map = static_cast<const double*>(g->d_eps_map);
  a.tfsf_pre = g->d_tfsf_pre;
  a.dispersive = g->max_poles;
  a.all_dispersive = g->mats.empty() ? 0 : 1;
  for (auto& m : g->mats)
    if (m.kind != FDTD_DRUDE && m.kind != FDTD_LORENTZ) a.all_dispersive = 0;
  a.single_mat = g->mats.size() <= 1 ? 1 : 0;
  a.uniform_mu = 1;
  for (auto& m : g->mats)
    if (m.mu_r != g->mats[0].mu_r) a.uniform_mu = 0;
  // TimePolicy constants (include/YeeUpdates.hpp:184-186, :205-215, :254-265),
  // folded by the host compiler as the reference's constexpr divisions are
  a.cc = 1.0;
  if (g->scheme == 3) {
    a.bd = 2;
    a.cc = 24.0 / 23.0;
    a.bdk[0] = 21.0 / 23.0;
    a.bdk[1] = 3.0 / 23.0;
    a.bdk[2] = 1.0 / 23.0;
  } else if (g->scheme == 4) {
    a.bd = 3;
    a.cc = 24.0 / 22.0;
    a.bdk[0] = 17.0 / 22.0;
    a.bdk[1] = 9.0 / 22.0;
    a.bdk[2] = 5.0 / 22.0;
    a.bdk[3] = 1.0 / 22.0;
  }
  for (int ft = 0; ft < 2; ft++)
    for (int l = 0; l < 3; l++)
      for (int c = 0; c < 3; c++) a.hist[ft][l][c] = static_cast<double*>(g->hist[ft][l][c]);
  a.kbeg = 1;
  a.kend = g->n[2] - 1;
  return a;
}

FusedArgs fused_args(fdtd_grid* g) {
  FusedArgs a;
  memset(&a, 0, sizeof(a));
  fill_common(g, a);
  a.pitch = g->pitch;
  a.flen[0] = g->pitch;
  a.flen[1] = g->n[1];
  a.flen[2] = g->n[2];
  a.ce = static_cast<float>(ce_of(g));
  a.ch = static_cast<float>(ch_of(g));
  for (int c = 0; c < 3; c++) {
    a.E[c] = static_cast<float*>(g->E[c]);
    a.H[c] = static_cast<float*>(g->H[c]);
    for (int p = 0; p < 2; p++) {
      a.P[p][c] = static_cast<float*>(g->P[p][c]);
      a.J[p][c] = static_cast<float*>(g->J[p][c]);
    }
  }
  for (int ft = 0; ft < 2; ft++)
    for (int I = 0; I < 3; I++)
      for (int J = 0; J < 3; J++) a.psi[ft][I][J] = static_cast<float*>(g->psi[ft][I][J]);
  for (int ft = 0; ft < 2; ft++)
    for (int x = 0; x < 3; x++) {
      a.prof[ft][x].B = static_cast<const float*>(g->d_prof[ft][x][0]);
      a.prof[ft][x].C = static_cast<const float*>(g->d_prof[ft][x][1]);
      a.prof[ft][x].F = static_cast<const float*>(g->d_prof[ft][x][2]);
      a.prof[ft][x].G = static_cast<const float*>(g->d_prof[ft][x][3]);
    }
  a.mats = static_cast<const MatF32*>(g->d_mats);
  a.inv_eps_map = static_cast<const float*>(g->d_eps_map);
  a.max_poles = g->max_poles;
  a.all_dispersive = 1;
  a.has_mu = 0;
  for (auto& m : g->mats) {
    if (m.kind != FDTD_DRUDE && m.kind != FDTD_LORENTZ) a.all_dispersive = 0;
    if (m.mu_r != 1.0) a.has_mu = 1;
  }
  a.src_scale_d = static_cast<float>(1.0 / kEps0);
  a.src_scale_b = static_cast<float>(eta() / kMu0);
  a.src_scale_h = static_cast<float>(eta());
  a.src_last = g->d_src_last;
  a.dx = g->d.dx;
  a.dt = g->d.dt;
  a.eta = eta();
  a.kbeg = 1;
  a.kend = g->n[2] - 1;
  return a;
}

}  // namespace

extern "C" {

int fdtd_grid_create(const fdtd_grid_desc* desc, fdtd_grid** out) try {
  if (!desc || !out) return fail(FDTD_ERR_INVALID, "null argument");
  *out = nullptr;
  const fdtd_grid_desc& d = *desc;
  if (d.mode != FDTD_TE && d.mode != FDTD_TM && d.mode != FDTD_THREED)
    return fail(FDTD_ERR_UNSUPPORTED, "mode must be FDTD_TE, FDTD_TM or FDTD_THREED");
  if (d.precision != FDTD_PLAIN_F64 && d.precision != FDTD_FUSED_F32)
    return fail(FDTD_ERR_INVALID, "precision must be FDTD_PLAIN_F64 or FDTD_FUSED_F32");
  if (d.nx < 3 || d.ny < 3 || (d.mode == FDTD_THREED ? d.nz < 3 : d.nz != 1))
    return fail(FDTD_ERR_INVALID, "need nx, ny >= 3, and nz >= 3 in 3D or nz == 1 in 2D");
  if (!(d.dx > 0) || !(d.dt > 0)) return fail(FDTD_ERR_INVALID, "dx and dt must be positive");
  if (static_cast<long long>(d.nx) * d.ny * d.nz > (1LL << 40)) return fail(FDTD_ERR_INVALID, "grid too large");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(FDTD_ERR_CUDA, "no CUDA device available");
  }
  if (d.device < 0 || d.device >= ndev) return fail(FDTD_ERR_INVALID, "bad device ordinal");
  CK(cudaSetDevice(d.device));
  fdtd_grid* g = new fdtd_grid();
  g->d = d;
  g->n[0] = d.nx;
  g->n[1] = d.ny;
  g->n[2] = d.nz;
  g->f32 = d.precision == FDTD_FUSED_F32;
  // FP32 rows are padded to a multiple of 128 cells: the vectorised sweeps
  // read whole 128-cell groups of a row
  g->pitch = g->f32 ? ((d.nx + 127) / 128) * 128 : d.nx;
  if (cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete g;
    return fail(FDTD_ERR_CUDA, "cudaStreamCreate failed");
  }
  int rc = FDTD_OK;
  const size_t fb = field_elems(g) * elem(g);
  for (int c = 0; c < 3 && !rc; c++) {
    if (hasE(d.mode, c)) {
      rc = dalloc(g, &g->E[c], fb);
      if (!rc && !g->f32) rc = dalloc(g, &g->D[c], fb);
    }
    if (!rc && hasH(d.mode, c)) {
      rc = dalloc(g, &g->H[c], fb);
      if (!rc && !g->f32) rc = dalloc(g, &g->B[c], fb);
    }
  }
  if (!rc) rc = dalloc(g, reinterpret_cast<void**>(&g->ctrl), sizeof(Control));
  if (!rc) rc = dalloc(g, reinterpret_cast<void**>(&g->d_flag), sizeof(int));
  if (!rc) {
    void* ptrs[6] = {g->E[0], g->E[1], g->E[2], g->H[0], g->H[1], g->H[2]};
    rc = upload_vec(g, reinterpret_cast<void**>(&g->d_fieldptrs), ptrs, sizeof(ptrs));
  }
  for (int ft = 0; ft < 2; ft++)
    for (int a = 0; a < 3; a++) g->prof[ft][a].reset(g->n[a]);
  if (!rc) rc = upload_profiles(g);
  if (!rc) rc = alloc_psi(g);
  if (!rc) {
    fdtd_material vac;
    memset(&vac, 0, sizeof(vac));
    vac.kind = FDTD_VACUUM;
    vac.eps_inf = 1.0;
    vac.mu_r = 1.0;
    g->mats.assign(1, vac);
    rc = build_materials(g);
  }
  if (!rc) {
    cudaError_t e = cudaStreamSynchronize(g->stream);
    if (e != cudaSuccess) rc = fail(FDTD_ERR_CUDA, cudaGetErrorString(e));
  }
  if (rc) {
    fdtd_grid_destroy(g);
    return rc;
  }
  *out = g;
  return FDTD_OK;
} catch (...) {
  return host_failure();
}

int fdtd_grid_destroy(fdtd_grid* g) try {
  if (!g) return FDTD_OK;
  cudaSetDevice(g->d.device);
  if (g->stream) cudaStreamSynchronize(g->stream);
  for (void* p : g->allocs) cudaFree(p);
  if (g->h_stage) cudaFreeHost(g->h_stage);
  for (auto& e : g->stage_ev)
    if (e) cudaEventDestroy(e);
  if (g->stream) cudaStreamDestroy(g->stream);
  tma_release(g->tma);
  if (g->graph) cudaGraphExecDestroy(g->graph);
  delete g;
  return FDTD_OK;
} catch (...) {
  return host_failure();
}

static int set_pml_side(fdtd_grid* g, int axis, int side, int ncells, const double* model) {
  if (!g) return fail(FDTD_ERR_INVALID, "null grid");
  if (axis < 0 || axis >= dim_of(g) || side < 0 || side > 1) return fail(FDTD_ERR_INVALID, "bad axis or side");
  if (ncells < 1) return fail(FDTD_ERR_INVALID, "ncells must be >= 1");
  if (model) {
    for (int q = 0; q < 5; q++)
      if (!std::isfinite(model[q])) return fail(FDTD_ERR_INVALID, "CPML model parameters must be finite");
    if (model[3] < 1.0) return fail(FDTD_ERR_INVALID, "kappa_max must be >= 1 (kappa grows from 1 in the layer)");
    if (model[2] < 0.0 || model[4] < 0.0) return fail(FDTD_ERR_INVALID, "sigma_max and alpha_max must be >= 0");
  }
  const int other = g->pml[axis][1 - side];
  const int w = (ncells + 1) + (other > 0 ? other + 1 : 0);
  if (w > g->n[axis] - 2) return fail(FDTD_ERR_INVALID, "CPML slabs overlap: grid too small for the widths");
  CK(cudaSetDevice(g->d.device));
  g->pml[axis][side] = ncells;
  g->pml_custom[axis][side] = model != nullptr;
  for (int q = 0; q < 5; q++) g->pml_model[axis][side][q] = model ? model[q] : 0.0;
  // regrade the whole axis in side order (min first), as the user loop would
  for (int ft = 0; ft < 2; ft++) g->prof[ft][axis].reset(g->n[axis]);
  for (int s = 0; s < 2; s++) {
    if (g->pml[axis][s] <= 0) continue;
    const double* pm = g->pml_model[axis][s];
    const PmlModel p = g->pml_custom[axis][s] ? PmlModel(pm[0], pm[1], pm[2], pm[3], pm[4]) : PmlModel(g->d.dx);
    grade(p, g->d.dt, g->n[axis], g->pml[axis][s], s, g->prof[0][axis], g->prof[1][axis]);
  }
  g->dirty_pml = true;
  g->version++;
  return FDTD_OK;
}

int fdtd_set_pml(fdtd_grid* g, int axis, int side, int ncells) try {
  return set_pml_side(g, axis, side, ncells, nullptr);
} catch (...) {
  return host_failure();
}

int fdtd_set_pml_model(fdtd_grid* g, int axis, int side, int ncells, double m, double ma, double sigma_max,
                       double kappa_max, double alpha_max) try {
  const double model[5] = {m, ma, sigma_max, kappa_max, alpha_max};
  return set_pml_side(g, axis, side, ncells, model);
} catch (...) {
  return host_failure();
}

int fdtd_set_materials(fdtd_grid* g, const fdtd_material* mats, int n) try {
  if (!g || !mats) return fail(FDTD_ERR_INVALID, "null argument");
  if (n < 1 || n > 65536) return fail(FDTD_ERR_INVALID, "material count must be 1..65536");
  for (int q = 0; q < n; q++) {
    const fdtd_material& m = mats[q];
    if (m.kind < FDTD_VACUUM || m.kind > FDTD_LORENTZ) return fail(FDTD_ERR_INVALID, "bad material kind");
    if (m.kind == FDTD_DRUDE && m.npoles != 1) return fail(FDTD_ERR_INVALID, "Drude takes npoles = 1");
    if (m.kind == FDTD_LORENTZ && (m.npoles < 1 || m.npoles > FDTD_MAX_POLES))
      return fail(FDTD_ERR_INVALID, "Lorentz takes 1..4 poles");
    if (m.kind != FDTD_VACUUM && !(m.eps_inf > 0)) return fail(FDTD_ERR_INVALID, "eps_inf must be positive");
    if (!(m.mu_r > 0)) return fail(FDTD_ERR_INVALID, "mu_r must be positive");
  }
  CK(cudaSetDevice(g->d.device));
  g->mats.assign(mats, mats + n);
  return build_materials(g);
} catch (...) {
  return host_failure();
}

int fdtd_set_material_ids(fdtd_grid* g, const uint8_t* ids) try {
  if (!g || !ids) return fail(FDTD_ERR_INVALID, "null argument");
  const long long n = static_cast<long long>(g->n[0]) * g->n[1] * g->n[2];
  // range check in one pass, then the rows copied straight into the padded
  // device layout (the padding stays zero)
  uint8_t top = 0;
  for (long long c = 0; c < n; c++) top = ids[c] > top ? ids[c] : top;
  if (top >= g->mats.size()) return fail(FDTD_ERR_INVALID, "material id out of range of the material table");
  const size_t rows = static_cast<size_t>(g->n[1]) * g->n[2], rl = static_cast<size_t>(rowlen(g));
  CK(cudaSetDevice(g->d.device));
  if (g->d_bids) {
    dfree(g, g->d_bids);
    g->d_bids = nullptr;
  }
  if (g->d_ids) dfree(g, g->d_ids);
  g->d_ids = nullptr;
  const int rc = dalloc(g, reinterpret_cast<void**>(&g->d_ids), static_cast<size_t>(field_elems(g)));
  if (rc) return rc;
  CK(cudaMemcpy2DAsync(g->d_ids, rl, ids, static_cast<size_t>(g->n[0]), static_cast<size_t>(g->n[0]), rows,
                       cudaMemcpyHostToDevice, g->stream));
  CK(cudaStreamSynchronize(g->stream));  // the caller's array may go once the call returns
  return FDTD_OK;
} catch (...) {
  return host_failure();
}

int fdtd_set_material_blocks(fdtd_grid* g, int block_shift, const uint16_t* ids, int nbx, int nby, int nbz) try {
  if (!g || !ids) return fail(FDTD_ERR_INVALID, "null argument");
  if (block_shift < 0 || block_shift > 16) return fail(FDTD_ERR_INVALID, "bad block_shift");
  for (int a = 0; a < 3; a++) {
    const int nb = a == 0 ? nbx : (a == 1 ? nby : nbz);
    if (nb < 1 || ((g->n[a] - 1) >> block_shift) >= nb) return fail(FDTD_ERR_INVALID, "block map does not cover the grid");
  }
  const size_t nb = static_cast<size_t>(nbx) * nby * nbz;
  for (size_t q = 0; q < nb; q++)
    if (ids[q] >= g->mats.size()) return fail(FDTD_ERR_INVALID, "material id out of range of the material table");
  CK(cudaSetDevice(g->d.device));
  if (g->d_ids) {
    dfree(g, g->d_ids);
    g->d_ids = nullptr;
  }
  g->bshift = block_shift;
  g->nbx = nbx;
  g->nby = nby;
  g->nbz = nbz;
  return upload_vec(g, reinterpret_cast<void**>(&g->d_bids), ids, nb * sizeof(uint16_t));
} catch (...) {
  return host_failure();
}

int fdtd_set_eps_map(fdtd_grid* g, const double* eps) try {
  if (!g) return fail(FDTD_ERR_INVALID, "null grid");
  CK(cudaSetDevice(g->d.device));
  if (!eps) {
    if (g->d_eps_map) dfree(g, g->d_eps_map);
    g->d_eps_map = nullptr;
    return FDTD_OK;
  }
  const long long nx = g->n[0], ny = g->n[1], nz = g->n[2], rl = rowlen(g);
  std::vector<char> buf(field_elems(g) * elem(g), 0);
  for (long long k = 0; k < nz; k++)
    for (long long j = 0; j < ny; j++)
      for (long long i = 0; i < nx; i++) {
        const double e = eps[(k * ny + j) * nx + i];
        if (!(e == e) || std::isinf(e)) return fail(FDTD_ERR_INVALID, "non-finite permittivity");
        const long long q = (k * ny + j) * rl + i;
        if (g->f32) reinterpret_cast<float*>(buf.data())[q] = e > 0 ? static_cast<float>(1.0 / e) : 0.0f;
        else reinterpret_cast<double*>(buf.data())[q] = e > 0 ? e : 0.0;
      }
  return upload_vec(g, &g->d_eps_map, buf.data(), buf.size());
} catch (...) {
  return host_failure();
}

int fdtd_add_source(fdtd_grid* g, int comp, int target, int i, int j, int k, const double* vals, int nvals) try {
  if (!g || (!vals && nvals > 0)) return fail(FDTD_ERR_INVALID, "null argument");
  if (target < 0 || target > 3) return fail(FDTD_ERR_INVALID, "target must be 0 (E), 1 (D), 2 (H) or 3 (B)");
  if (comp < 0 || comp > 2 || !(target < 2 ? hasE(g->d.mode, comp) : hasH(g->d.mode, comp)))
    return fail(FDTD_ERR_INVALID, "component not in this mode");
  if (!interior(g, i, j, k)) return fail(FDTD_ERR_INVALID, "source cell must be an interior cell");
  if (g->srcs.size() >= static_cast<size_t>(kMaxSources)) return fail(FDTD_ERR_UNSUPPORTED, "too many sources");
  if (nvals < 0) return fail(FDTD_ERR_INVALID, "nvals < 0");
  CK(cudaSetDevice(g->d.device));
  SourceH s;
  s.comp = comp;
  s.target = target;
  s.i = i;
  s.j = j;
  s.k = k;
  s.vals.assign(vals, vals + nvals);
  int rc = upload_vec(g, reinterpret_cast<void**>(&s.d_vals), s.vals.data(),
                      std::max<size_t>(1, s.vals.size()) * sizeof(double));
  if (rc) return rc;
  g->srcs.push_back(s);
  if (g->d_src_last) dfree(g, g->d_src_last);
  return dalloc(g, reinterpret_cast<void**>(&g->d_src_last), kMaxSources * sizeof(double));
} catch (...) {
  return host_failure();
}

int fdtd_add_source_box(fdtd_grid* g, int comp, int target, const int* lo, const int* hi, const double* vals,
                        int nvals) try {
  if (!g || !lo || !hi || (!vals && nvals > 0)) return fail(FDTD_ERR_INVALID, "null argument");
  if (target == 1 || target == 3)
    return fail(FDTD_ERR_UNSUPPORTED, "box sources add to E (target 0) or H (target 2); use point sources for D or B");
  if (target != 0 && target != 2) return fail(FDTD_ERR_INVALID, "target must be 0 (E) or 2 (H)");
  if (comp < 0 || comp > 2 || !(target == 0 ? hasE(g->d.mode, comp) : hasH(g->d.mode, comp)))
    return fail(FDTD_ERR_INVALID, "component not in this mode");
  if (nvals < 0) return fail(FDTD_ERR_INVALID, "nvals < 0");
  for (int d = 0; d < 3; d++)
    if (hi[d] < lo[d]) return fail(FDTD_ERR_INVALID, "empty source box");
  if (!interior(g, lo[0], lo[1], lo[2]) || !interior(g, hi[0], hi[1], hi[2]))
    return fail(FDTD_ERR_INVALID, "source box must lie in the interior cells");
  CK(cudaSetDevice(g->d.device));
  BoxSourceH b;
  b.comp = comp;
  b.target = target;
  for (int d = 0; d < 3; d++) {
    b.lo[d] = lo[d];
    b.hi[d] = hi[d];
  }
  std::vector<double> v(vals, vals + nvals);
  int rc = upload_vec(g, reinterpret_cast<void**>(&b.d_vals), v.data(), std::max<size_t>(1, v.size()) * sizeof(double));
  if (rc) return rc;
  b.nvals = nvals;
  g->boxes.push_back(b);
  g->version++;
  return FDTD_OK;
} catch (...) {
  return host_failure();
}

// the box sources of one phase (0 = E, 1 = H): shift 0 adds this step's
// value, shift -1 takes back the previous step's (fused method only)
static int launch_boxes(fdtd_grid* g, int phase, int shift, cudaStream_t s) {
  int n = 0;
  for (const auto& b : g->boxes) {
    if ((b.target == 0) != (phase == 0)) continue;
    void* f = phase == 0 ? g->E[b.comp] : g->H[b.comp];
    const double scale = (phase == 1 && g->f32 ? eta() : 1.0) * (shift < 0 ? -1.0 : 1.0);
    n += launch_box_source(g->f32 ? 1 : 0, f, b.lo, b.hi, static_cast<int>(rowlen(g)), g->n[1], b.d_vals, b.nvals,
                           scale, shift, g->ctrl, s);
  }
  return n;
}

// the boundary images of one half step (0: E, 1: H)
static int launch_bc(fdtd_grid* g, int phase, cudaStream_t s) {
  if (g->bcs.n == 0) return 0;
  void* f[3];
  for (int q = 0; q < 3; q++) f[q] = phase == 0 ? g->E[q] : g->H[q];
  return launch_boundaries(g->bcs, phase, g->f32 ? 1 : 0, f, g->n[0], g->n[1], g->n[2], static_cast<int>(rowlen(g)),
                           s);
}

int fdtd_set_boundary(fdtd_grid* g, int axis, int side, int kind) try {
  if (!g) return fail(FDTD_ERR_INVALID, "null grid");
  if (axis < 0 || axis >= dim_of(g) || side < 0 || side > 1) return fail(FDTD_ERR_INVALID, "bad axis or side");
  if (kind < FDTD_BC_NONE || kind > FDTD_BC_PERIODIC) return fail(FDTD_ERR_INVALID, "bad boundary kind");
  BcFaces nb{};
  for (int q = 0; q < g->bcs.n; q++)
    if (g->bcs.face[q].axis != axis || g->bcs.face[q].side != side) nb.face[nb.n++] = g->bcs.face[q];
  if (kind != FDTD_BC_NONE) {
    BcFace fc{axis, side, kind, {}};
    for (int ft = 0; ft < 2; ft++)
      for (int c = 0; c < 3; c++) fc.sgn[ft][c] = bc_sign(kind, ft, c, axis);
    nb.face[nb.n++] = fc;
  }
  g->bcs = nb;
  g->version++;
  return FDTD_OK;
} catch (...) {
  return host_failure();
}

int fdtd_set_time_scheme(fdtd_grid* g, int scheme) try {
  if (!g) return fail(FDTD_ERR_INVALID, "null grid");
  if (scheme != FDTD_BD1 && scheme != FDTD_BD3 && scheme != FDTD_BD4)
    return fail(FDTD_ERR_INVALID, "time scheme must be FDTD_BD1, FDTD_BD3 or FDTD_BD4");
  if (g->f32 && scheme != FDTD_BD1)
    return fail(FDTD_ERR_UNSUPPORTED, "the FP32 fused method steps with the leapfrog (BD1) scheme only");
  if (g->next_half != 0) return fail(FDTD_ERR_INVALID, "a half step is pending");
  CK(cudaSetDevice(g->d.device));
  for (int ft = 0; ft < 2; ft++)
    for (int l = 0; l < 3; l++)
      for (int c = 0; c < 3; c++)
        if (g->hist[ft][l][c]) {
          dfree(g, g->hist[ft][l][c]);
          g->hist[ft][l][c] = nullptr;
        }
  const int levels = scheme == FDTD_BD1 ? 0 : scheme - 1;
  for (int ft = 0; ft < 2; ft++)
    for (int l = 0; l < levels; l++)
      for (int c = 0; c < 3; c++) {
        if (!(ft == 0 ? hasE(g->d.mode, c) : hasH(g->d.mode, c))) continue;
        const int rc = dalloc(g, &g->hist[ft][l][c], static_cast<size_t>(field_elems(g)) * elem(g));
        if (rc != FDTD_OK) return rc;
      }
  g->scheme = scheme;
  g->version++;
  return FDTD_OK;
} catch (...) {
  return host_failure();
}

int fdtd_add_tfsf_plane(fdtd_grid* g, int axis, int orient, const int* lo, const int* hi, const double* origin,
                        const double* k, const double* pol_e, const double* pol_h, int aux_ncells,
                        const double* aux_vals, int naux) try {
  if (!g || !lo || !hi || !origin || !k || !pol_e || !pol_h || (!aux_vals && naux > 0))
    return fail(FDTD_ERR_INVALID, "null argument");
  const int dim = dim_of(g);
  if (axis < 0 || axis >= dim || orient < 0 || orient > 1) return fail(FDTD_ERR_INVALID, "bad axis or orientation");
  if (aux_ncells < 1 || naux < 0) return fail(FDTD_ERR_INVALID, "bad aux grid size");
  if (g->planes.size() >= static_cast<size_t>(kMaxPlanes)) return fail(FDTD_ERR_UNSUPPORTED, "too many TFSF planes");
  for (int d = 0; d < 3; d++) {
    if (lo[d] > hi[d]) return fail(FDTD_ERR_INVALID, "empty TFSF plane");
    if (d < dim && (lo[d] < 1 || hi[d] > g->n[d] - 2)) return fail(FDTD_ERR_INVALID, "TFSF plane outside the interior");
    if (d >= dim && (lo[d] != 0 || hi[d] != 0)) return fail(FDTD_ERR_INVALID, "2D TFSF plane needs k range 0..0");
  }
  PlaneDev p;
  memset(&p, 0, sizeof(p));
  p.axis = axis;
  for (int d = 0; d < 3; d++) {
    p.lo[d] = lo[d];
    p.hi[d] = hi[d];
    p.origin[d] = origin[d];
    p.pol_e[d] = pol_e[d];
    p.pol_h[d] = pol_h[d];
  }
  // TFSFPlane constructor (Source.hpp:556-570): unit normal and wave vector
  p.normal[axis] = orient == 1 ? 1 : -1;
  double N = 0;
  for (int d = 0; d < dim; d++) N += p.normal[d] * p.normal[d];
  N = std::sqrt(N);
  for (int d = 0; d < dim; d++) p.normal[d] /= N;
  double K = 0;
  for (int d = 0; d < dim; d++) K += k[d] * k[d];
  K = std::sqrt(K);
  if (!(K > 0)) return fail(FDTD_ERR_INVALID, "zero wave vector");
  for (int d = 0; d < dim; d++) p.k[d] = k[d] / K;
  const int L = aux_ncells + 2 * kAuxNpml + 20;
  // every interpolation the corrections make must land inside the aux grid
  // (Aux1D::interpolateE/H have no bounds check)
  for (int corner = 0; corner < 8; corner++) {
    int idx[3];
    for (int d = 0; d < 3; d++) idx[d] = (corner >> d & 1) ? hi[d] : lo[d];
    for (int ft = 0; ft < 2; ft++)
      for (int Kc = 0; Kc < 3; Kc++) {
        double proj = 0;
        for (int d = 0; d < dim; d++) {
          const double off = ft == 0 ? (d == Kc ? -0.5 : 0.0) : (d == Kc ? 0.0 : -0.5);
          proj += p.k[d] * ((static_cast<double>(idx[d]) - origin[d]) * g->d.dx + off * g->d.dx);
        }
        const double nd = static_cast<double>(L) / 2.0 + proj / g->d.dx - (ft == 0 ? 0.5 : 0.0);
        if (!(nd >= 0.0) || std::floor(nd) + 1 > L - 1)
          return fail(FDTD_ERR_INVALID, "TFSF plane projects outside its aux grid: raise aux_ncells");
      }
  }
  CK(cudaSetDevice(g->d.device));
  // planes with the same aux grid share one
  int aux = -1;
  std::vector<double> vals(aux_vals, aux_vals + naux);
  for (size_t q = 0; q < g->auxes.size(); q++)
    if (g->auxes[q].ncells == aux_ncells && g->auxes[q].vals == vals) aux = static_cast<int>(q);
  if (aux < 0) {
    if (g->t != 0) return fail(FDTD_ERR_UNSUPPORTED, "a new aux grid must be added before the first step");
    AuxH a;
    a.ncells = aux_ncells;
    a.L = L;
    a.vals = vals;
    int rc = build_aux(g, a);
    if (rc) return rc;
    g->auxes.push_back(a);
    aux = static_cast<int>(g->auxes.size()) - 1;
  }
  p.aux = aux;
  // the FP64 method forms each half step's corrections of all plane cells in
  // one launch before its sweep (a table of 3 values per cell)
  p.off = g->tfsf_cells;
  const long long cells = static_cast<long long>(p.hi[0] - p.lo[0] + 1) * (p.hi[1] - p.lo[1] + 1) *
                          (p.hi[2] - p.lo[2] + 1);
  if (!g->f32) {
    if (g->d_tfsf_pre) dfree(g, g->d_tfsf_pre);
    g->d_tfsf_pre = nullptr;
    const int rc = dalloc(g, reinterpret_cast<void**>(&g->d_tfsf_pre),
                          static_cast<size_t>(g->tfsf_cells + cells) * 3 * sizeof(double));
    if (rc) return rc;
  }
  g->tfsf_cells += cells;
  PlaneH ph;
  ph.dev = p;
  g->planes.push_back(ph);
  g->version++;
  return FDTD_OK;
} catch (...) {
  return host_failure();
}

int fdtd_add_dft(fdtd_grid* g, int comp, const int* lo, const int* hi, const double* freqs, int nf, int* handle) try {
  if (!g || !lo || !hi || !freqs || !handle) return fail(FDTD_ERR_INVALID, "null argument");
  const int qc = quantity_check(g, comp, lo, hi);
  if (qc != FDTD_OK) return qc;
  if (nf < 1) return fail(FDTD_ERR_INVALID, "nf must be >= 1");
  if (g->next_half != 0) return fail(FDTD_ERR_INVALID, "DFT regions are added between whole steps");
  DftH r;
  r.comp = comp;
  r.nf = nf;
  r.npts = 1;
  for (int d = 0; d < 3; d++) {
    if (lo[d] < 0 || hi[d] >= g->n[d] || lo[d] > hi[d]) return fail(FDTD_ERR_INVALID, "DFT box outside the grid");
    r.lo[d] = lo[d];
    r.hi[d] = hi[d];
    r.npts *= hi[d] - lo[d] + 1;
  }
  if (r.npts >= (1LL << 31)) return fail(FDTD_ERR_UNSUPPORTED, "a DFT region holds at most 2^31 - 1 points");
  CK(cudaSetDevice(g->d.device));
  r.freqs.assign(freqs, freqs + nf);
  int rc = upload_vec(g, reinterpret_cast<void**>(&r.d_freqs), freqs, nf * sizeof(double));
  if (rc) return rc;
  rc = dalloc(g, reinterpret_cast<void**>(&r.d_acc), static_cast<size_t>(nf) * r.npts * 2 * sizeof(double));
  if (rc) return rc;
  g->dfts.push_back(r);
  *handle = static_cast<int>(g->dfts.size()) - 1;
  g->dirty_dft = true;
  return FDTD_OK;
} catch (...) {
  return host_failure();
}

int fdtd_dft_npoints(fdtd_grid* g, int handle, long long* npoints) try {
  if (!g || !npoints || handle < 0 || handle >= static_cast<int>(g->dfts.size()))
    return fail(FDTD_ERR_INVALID, "bad DFT handle");
  *npoints = g->dfts[handle].npts;
  return FDTD_OK;
} catch (...) {
  return host_failure();
}

}  // extern "C"

// Reads `bytes` of device memory into a pageable host buffer. Large reads go
// through the grid's two pinned chunks: the copy engine fills one at full
// link speed while host threads move the other into `out`, instead of the
// driver's own staging with a single-threaded copy and page faults.
static int read_to_host(fdtd_grid* g, void* out, const void* src, size_t bytes) {
  constexpr size_t kStageChunk = size_t(8) << 20;
  if (bytes < kStageChunk) {
    CK(cudaStreamSynchronize(g->stream));
    CK(cudaMemcpy(out, src, bytes, cudaMemcpyDeviceToHost));
    return FDTD_OK;
  }
  if (!g->h_stage) {
    CK(cudaHostAlloc(reinterpret_cast<void**>(&g->h_stage), 2 * kStageChunk, cudaHostAllocDefault));
    for (auto& e : g->stage_ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  const char* d = static_cast<const char*>(src);
  char* h = static_cast<char*>(out);
  const size_t nch = (bytes + kStageChunk - 1) / kStageChunk;
  auto issue = [&](size_t c) -> cudaError_t {
    const size_t off = c * kStageChunk, len = std::min(kStageChunk, bytes - off);
    cudaError_t e = cudaMemcpyAsync(g->h_stage + (c % 2) * kStageChunk, d + off, len, cudaMemcpyDeviceToHost,
                                    g->stream);
    if (e == cudaSuccess) e = cudaEventRecord(g->stage_ev[c % 2], g->stream);
    return e;
  };
  CK(issue(0));
  for (size_t c = 0; c < nch; c++) {
    // the other chunk's previous contents were copied out in the last pass
    if (c + 1 < nch) CK(issue(c + 1));
    CK(cudaEventSynchronize(g->stage_ev[c % 2]));
    const size_t off = c * kStageChunk;
    parallel_host_copy(h + off, g->h_stage + (c % 2) * kStageChunk, std::min(kStageChunk, bytes - off));
  }
  return FDTD_OK;
}

extern "C" {

int fdtd_dft_read(fdtd_grid* g, int handle, double* out) try {
  if (!g || !out || handle < 0 || handle >= static_cast<int>(g->dfts.size()))
    return fail(FDTD_ERR_INVALID, "bad DFT handle");
  CK(cudaSetDevice(g->d.device));
  if (g->dft_pending > 0) g->launches += flush_dft(g, g->stream);  // samples left by fdtd_step_half
  const DftH& r = g->dfts[handle];
  const size_t n = static_cast<size_t>(r.nf) * r.npts * 2;
  CK(cudaStreamSynchronize(g->stream));
  return read_to_host(g, out, r.d_acc, n * sizeof(double));
} catch (...) {
  return host_failure();
}

static int step_impl(fdtd_grid* g, int nsteps, void* stream, double* prof);
static int enqueue_steps(fdtd_grid* g, int nsteps, cudaStream_t s, double* prof);

// The TFSF aux tables for a call of nsteps steps: at least 257 rows, so that
// calls of up to 256 steps keep them (and the step graph, whose launches hold
// their addresses; dalloc and dfree make the graph stale).
static int ensure_aux_tables(fdtd_grid* g, int nsteps) {
  for (auto& a : g->auxes) {
    if (a.cap >= nsteps + 1) continue;
    if (a.d_tab) dfree(g, a.d_tab);
    a.d_tab = nullptr;
    const long long cap = std::max<long long>(nsteps + 1, 257);
    int rc = dalloc(g, reinterpret_cast<void**>(&a.d_tab), 2 * static_cast<size_t>(cap) * a.L * sizeof(double));
    if (rc) return rc;
    a.cap = cap;
    CK(cudaStreamSynchronize(g->stream));
  }
  return FDTD_OK;
}

// The captured graph of kGraphSteps steps, captured again when anything it
// holds changed (g->version). Pending DFT samples must have been folded.
static int ensure_step_graph(fdtd_grid* g, cudaStream_t s) {
  if (g->graph && g->graph_version == g->version) return FDTD_OK;
  if (g->graph) {
    cudaGraphExecDestroy(g->graph);
    g->graph = nullptr;
  }
  const long long before = g->launches;
  CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  int rc = enqueue_steps(g, kGraphSteps, s, nullptr);
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamEndCapture(s, &graph);
  if (rc) return rc;
  if (e != cudaSuccess) return fail(FDTD_ERR_CUDA, std::string("stream capture: ") + cudaGetErrorString(e));
  e = cudaGraphInstantiate(&g->graph, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return fail(FDTD_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
  g->graph_launches = g->launches - before;
  g->launches = before;
  g->graph_version = g->version;
  return FDTD_OK;
}

int fdtd_step(fdtd_grid* g, int nsteps, void* stream) try {
  return step_impl(g, nsteps, stream, nullptr);
} catch (...) {
  return host_failure();
}

int fdtd_prepare(fdtd_grid* g) try {
  if (!g) return fail(FDTD_ERR_INVALID, "null grid");
  CK(cudaSetDevice(g->d.device));
  int rc = ensure_pml(g);
  if (rc) return rc;
  rc = ensure_eh(g);
  if (rc) return rc;
  if (g->dirty_dft) {
    rc = rebuild_dft(g);
    if (rc) return rc;
  }
  // the step graph too (its capture launches nothing), so that the first
  // call of kGraphSteps or more steps replays it at once
  if (g->use_graphs && g->next_half == 0 && !g->half_split) {
    rc = ensure_aux_tables(g, kGraphSteps);
    if (rc) return rc;
    if (g->dft_pending > 0) g->launches += flush_dft(g, g->stream);
    rc = ensure_step_graph(g, g->stream);
    if (rc) return rc;
  }
  CK(cudaStreamSynchronize(g->stream));
  return FDTD_OK;
} catch (...) {
  return host_failure();
}

int fdtd_profile_step(fdtd_grid* g, int nsteps, void* stream, double* ms) try {
  if (!ms) return fail(FDTD_ERR_INVALID, "null argument");
  return step_impl(g, nsteps, stream, ms);
} catch (...) {
  return host_failure();
}

// Enqueues nsteps steps on s (kernels only, so it can run under stream
// capture). With `prof`, CUDA events bracket each part of every step.
static int enqueue_steps(fdtd_grid* g, int nsteps, cudaStream_t s, double* prof) {
  const int mode = g->d.mode;
  const void* const* fE = reinterpret_cast<const void* const*>(g->d_fieldptrs);
  const void* const* fH = fE + 3;
  // kernel sequence of one step; with `prof`, CUDA events bracket each kernel
  // on the launching stream and the elapsed times are summed per kernel kind
  cudaEvent_t ev[6] = {};
  if (prof) {
    for (auto& e : ev) CK(cudaEventCreate(&e));
    for (int q = 0; q < 5; q++) prof[q] = 0.0;
  }
  FusedArgs fa;
  PlainArgs pa;
  if (g->f32) fa = fused_args(g);
  else pa = plain_args(g);
  const bool use3d = g->f32 && mode == kThreeD && fused3d_supported(fa);
  const bool use_tma = use3d && g->sweep_kind == FDTD_SWEEP_TMA && tma_prepare(fa, &g->tma);
  if (g->sweep_kind == FDTD_SWEEP_TMA && !use_tma)
    return fail(FDTD_ERR_UNSUPPORTED, "the TMA sweep is not available for this grid");
  // AUTO takes the staged sweeps, the fastest measured on B200
  const bool use_staged =
      use3d && (g->sweep_kind == FDTD_SWEEP_STAGED || g->sweep_kind == FDTD_SWEEP_AUTO);
  const bool use_flat = use3d && !use_tma && !use_staged && g->sweep_kind == FDTD_SWEEP_FLAT;
  const bool boxes = !g->boxes.empty();
  // the whole step in one launch: 3D FP32 grids without TFSF planes, box
  // sources, boundary conditions or mu_r != 1 (whose extra kernels run
  // between the two sweeps)
  EhSched eh{};
  int eh_blocks = 0;
  const bool use_eh = use3d && !use_tma && eh_wanted(g) && g->d_eh && !boxes && g->bcs.n == 0 &&
                      g->sweep_kind == FDTD_SWEEP_EH && staged_eh_plan(fa, &eh, &eh_blocks);
  if (g->sweep_kind == FDTD_SWEEP_EH && !use_eh)
    return fail(FDTD_ERR_UNSUPPORTED,
                "the one-launch step needs a 3D FP32 grid without TFSF planes, box sources, boundary conditions "
                "or mu_r != 1");
  if (use_eh) {
    eh.epoch = g->d_eh;
    eh.flags = g->d_eh + 1;
  }
  for (int q = 0; q < nsteps; q++) {
    if (prof) CK(cudaEventRecord(ev[0], s));
    if (use_eh) {
      g->launches += launch_staged_eh(fa, eh, eh_blocks, s);
      if (prof) CK(cudaEventRecord(ev[1], s));
      g->launches += launch_dft_gather(1, g->d_dft[0], g->ndft[0], g->dft_pts[0], g->dft_maxpts[0], fE, g->n[1],
                                       static_cast<int>(rowlen(g)), g->dft_pending, g->d_dft_buf[0], s);
      if (prof) {
        CK(cudaEventRecord(ev[2], s));
        CK(cudaEventRecord(ev[3], s));
      }
      g->launches += launch_dft_gather(1, g->d_dft[1], g->ndft[1], g->dft_pts[1], g->dft_maxpts[1], fH, g->n[1],
                                       static_cast<int>(rowlen(g)), g->dft_pending, g->d_dft_buf[1], s);
      if (prof) CK(cudaEventRecord(ev[4], s));
      g->launches += launch_step_advance(g->ctrl, g->d_eh, s);
      if (!g->dfts.empty() && ++g->dft_pending == kDftChunk) g->launches += flush_dft(g, s);
      if (prof) {
        CK(cudaEventRecord(ev[5], s));
        CK(cudaEventSynchronize(ev[5]));
        for (int k = 0; k < 5; k++) {
          float ms = 0.f;
          CK(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
          prof[k] += ms / nsteps;
        }
      }
      continue;
    }
    if (boxes && g->f32) g->launches += launch_boxes(g, 0, -1, s);
    if (g->f32) {
      g->launches += use_tma      ? launch_tma_e(fa, g->tma, s)
                     : use_staged ? launch_staged_e(fa, s)
                     : use_flat   ? launch_flat_e(fa, s)
                     : use3d    ? launch_fused3d_e(fa, s)
                                : launch_fused_e(mode, fa, s);
    }
    else {
      if (!g->planes.empty()) g->launches += launch_tfsf_pre(mode, pa, 0, s);
      g->launches += launch_plain_e(mode, pa, s);
    }
    if (prof) CK(cudaEventRecord(ev[1], s));
    if (g->f32) g->launches += launch_tfsf_fused(mode, fa, 0, s);
    if (boxes) g->launches += launch_boxes(g, 0, 0, s);
    g->launches += launch_bc(g, 0, s);
    g->launches += launch_dft_gather(g->f32 ? 1 : 0, g->d_dft[0], g->ndft[0], g->dft_pts[0], g->dft_maxpts[0], fE, g->n[1],
                                     static_cast<int>(rowlen(g)), g->dft_pending, g->d_dft_buf[0], s);
    if (prof) CK(cudaEventRecord(ev[2], s));
    if (boxes && g->f32) g->launches += launch_boxes(g, 1, -1, s);
    if (g->f32) {
      g->launches += use_tma      ? launch_tma_h(fa, g->tma, s)
                     : use_staged ? launch_staged_h(fa, s)
                     : use_flat   ? launch_flat_h(fa, s)
                     : use3d    ? launch_fused3d_h(fa, s)
                                : launch_fused_h(mode, fa, s);
    }
    else {
      if (!g->planes.empty()) g->launches += launch_tfsf_pre(mode, pa, 1, s);
      g->launches += launch_plain_h(mode, pa, s);
    }
    if (prof) CK(cudaEventRecord(ev[3], s));
    if (g->f32) g->launches += launch_tfsf_fused(mode, fa, 1, s);
    if (boxes) g->launches += launch_boxes(g, 1, 0, s);
    g->launches += launch_bc(g, 1, s);
    g->launches += launch_dft_gather(g->f32 ? 1 : 0, g->d_dft[1], g->ndft[1], g->dft_pts[1], g->dft_maxpts[1], fH, g->n[1],
                                     static_cast<int>(rowlen(g)), g->dft_pending, g->d_dft_buf[1], s);
    if (prof) CK(cudaEventRecord(ev[4], s));
    g->launches += launch_step_advance(g->ctrl, s);
    if (!g->dfts.empty() && ++g->dft_pending == kDftChunk) g->launches += flush_dft(g, s);
    if (prof) {
      CK(cudaEventRecord(ev[5], s));
      CK(cudaEventSynchronize(ev[5]));
      for (int k = 0; k < 5; k++) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
        prof[k] += ms / nsteps;
      }
    }
  }
  if (prof)
    for (auto& e : ev) cudaEventDestroy(e);
  if (g->dft_pending > 0) g->launches += flush_dft(g, s);
  return FDTD_OK;
}

static int step_impl(fdtd_grid* g, int nsteps, void* stream, double* prof) {
  if (!g) return fail(FDTD_ERR_INVALID, "null grid");
  if (g->next_half != 0 || g->half_split) return fail(FDTD_ERR_INVALID, "an E half step was taken without its H half");
  if (nsteps < 0) return fail(FDTD_ERR_INVALID, "nsteps < 0");
  if (nsteps == 0) return FDTD_OK;
  CK(cudaSetDevice(g->d.device));
  {
    // before any graph capture: the CPML set-up synchronises its stream
    int prc = ensure_pml(g);
    if (prc) return prc;
    prc = ensure_eh(g);
    if (prc) return prc;
  }
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : g->stream;
  if (s != g->stream) {
    // order the caller's stream after any set-up work on ours
    cudaEvent_t ev;
    CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    CK(cudaEventRecord(ev, g->stream));
    CK(cudaStreamWaitEvent(s, ev, 0));
    CK(cudaEventDestroy(ev));
  }
  if (g->dirty_dft) {
    int rc = rebuild_dft(g);
    if (rc) return rc;
    CK(cudaStreamSynchronize(g->stream));
  }
  // TFSF: precompute the aux grids' Ez/Hy for this chunk of steps
  {
    const int rc = ensure_aux_tables(g, nsteps);
    if (rc) return rc;
  }
  for (auto& a : g->auxes) {
    double* st = a.d_state;
    const int L = a.L;
    g->launches += launch_aux_precompute(L, g->d.dt, g->d.dx, st, st + L, st + 2 * L, st + 3 * L, st + 4 * L,
                                         st + 5 * L, a.d_coef, a.d_vals, static_cast<int>(a.vals.size()), g->t,
                                         nsteps, a.d_tab, a.d_tab + a.cap * L, s);
  }
  // the tables' first row is this step (set on the stream: no host wait)
  if (!g->auxes.empty()) g->launches += launch_set_step(g->ctrl, g->t, s);
  // a captured graph takes its samples from slot 0 on
  if (g->dft_pending > 0) g->launches += flush_dft(g, s);
  // one graph replay = kGraphSteps steps (and, with DFT regions, one flush)
  const bool graphs = !prof && g->use_graphs && nsteps >= kGraphSteps;
  int done = 0;
  if (graphs) {
    const int rc = ensure_step_graph(g, s);
    if (rc) return rc;
    for (; done + kGraphSteps <= nsteps; done += kGraphSteps) {
      CK(cudaGraphLaunch(g->graph, s));
      g->launches += g->graph_launches;
    }
  }
  if (done < nsteps) {
    int rc = enqueue_steps(g, nsteps - done, s, prof);
    if (rc) return rc;
  }
  CK(cudaGetLastError());
  g->t += nsteps;
  return FDTD_OK;
}

int fdtd_set_sweep_kernel(fdtd_grid* g, int kind) try {
  if (!g) return fail(FDTD_ERR_INVALID, "null grid");
  if (kind < FDTD_SWEEP_AUTO || kind > FDTD_SWEEP_EH) return fail(FDTD_ERR_INVALID, "bad sweep kernel kind");
  g->sweep_kind = kind;
  g->version++;
  return FDTD_OK;
} catch (...) {
  return host_failure();
}

// One half step, for callers that exchange data between the halves (the
// ghost planes of a z-slab decomposition): the launches of one step of
// enqueue_steps, split after the E-phase DFT gather; phase 0 also advances
// the TFSF aux grids by one step. Launched eagerly, never from a graph.
//
// part -1 runs the whole half step. Parts 0 and 1 split it so that a ghost
// plane's transfer can overlap the sweep: part 0 runs what comes before the
// sweep and sweeps every plane whose update reads no ghost plane (E half:
// planes 2 .. nz-2; plane 1 differences H along z with plane 0. H half:
// planes 1 .. nz-3; plane nz-2 reads E of plane nz-1); part 1 sweeps the
// remaining plane and runs everything after the sweep. Per cell the updates
// are those of the whole sweep, so the results are identical.
static int half_step_impl(fdtd_grid* g, int phase, int part, void* stream) {
  if (!g) return fail(FDTD_ERR_INVALID, "null grid");
  if (phase != 0 && phase != 1) return fail(FDTD_ERR_INVALID, "phase must be 0 (E) or 1 (H)");
  if (part < -1 || part > 1) return fail(FDTD_ERR_INVALID, "part must be -1 (whole), 0 or 1");
  if (phase != g->next_half) return fail(FDTD_ERR_INVALID, "half steps alternate, the E half first");
  if (part == 1 && !g->half_split) return fail(FDTD_ERR_INVALID, "part 1 of a half step comes after its part 0");
  if (part != 1 && g->half_split) return fail(FDTD_ERR_INVALID, "part 0 of this half step is waiting for its part 1");
  const int mode = g->d.mode;
  if (part >= 0 && (mode != kThreeD || g->n[2] < 4))
    return fail(FDTD_ERR_UNSUPPORTED, "a half step splits along z on 3D grids of 2 or more interior planes");
  CK(cudaSetDevice(g->d.device));
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : g->stream;
  if (s != g->stream && part != 1) CK(cudaStreamSynchronize(g->stream));
  if (part != 1 && g->dirty_dft) {
    int rc = rebuild_dft(g);
    if (rc) return rc;
    CK(cudaStreamSynchronize(g->stream));
  }
  const bool boxes = !g->boxes.empty();
  if (part != 1 && phase == 0) {
    for (auto& a : g->auxes) {
      if (a.cap < 2) {
        if (a.d_tab) dfree(g, a.d_tab);
        a.d_tab = nullptr;
        int rc = dalloc(g, reinterpret_cast<void**>(&a.d_tab), 2 * static_cast<size_t>(2) * a.L * sizeof(double));
        if (rc) return rc;
        a.cap = 2;
        CK(cudaStreamSynchronize(g->stream));
      }
      double* st = a.d_state;
      const int L = a.L;
      g->launches += launch_aux_precompute(L, g->d.dt, g->d.dx, st, st + L, st + 2 * L, st + 3 * L, st + 4 * L,
                                           st + 5 * L, a.d_coef, a.d_vals, static_cast<int>(a.vals.size()), g->t, 1,
                                           a.d_tab, a.d_tab + a.cap * L, s);
    }
    if (!g->auxes.empty()) g->launches += launch_chunk_start(g->ctrl, s);
  }
  {
    const int prc = ensure_pml(g);
    if (prc) return prc;
  }
  FusedArgs fa;
  PlainArgs pa;
  if (g->f32) fa = fused_args(g);
  else pa = plain_args(g);
  const bool use3d = g->f32 && mode == kThreeD && fused3d_supported(fa);
  if (part >= 0 && g->f32 && !use3d)
    return fail(FDTD_ERR_UNSUPPORTED, "the split half step needs the staged 3D sweeps (row pitch a multiple of 128)");
  // the planes of this part: E half part 0 = 2 .. nz-2, part 1 = 1; H half
  // part 0 = 1 .. nz-3, part 1 = nz-2
  if (part >= 0) {
    const int nz = g->n[2];
    const int kb = phase == 0 ? (part == 0 ? 2 : 1) : (part == 0 ? 1 : nz - 2);
    const int ke = phase == 0 ? (part == 0 ? nz - 1 : 2) : (part == 0 ? nz - 2 : nz - 1);
    fa.kbeg = pa.kbeg = kb;
    fa.kend = pa.kend = ke;
  }
  const void* const* fields = reinterpret_cast<const void* const*>(g->d_fieldptrs) + (phase == 0 ? 0 : 3);
  if (part != 1 && boxes && g->f32) g->launches += launch_boxes(g, phase, -1, s);
  if (g->f32) {
    if (phase == 0) g->launches += use3d ? launch_staged_e(fa, s) : launch_fused_e(mode, fa, s);
    else g->launches += use3d ? launch_staged_h(fa, s) : launch_fused_h(mode, fa, s);
  } else {
    if (part != 1 && !g->planes.empty()) g->launches += launch_tfsf_pre(mode, pa, phase, s);
    g->launches += phase == 0 ? launch_plain_e(mode, pa, s) : launch_plain_h(mode, pa, s);
  }
  if (part == 0) {
    CK(cudaGetLastError());
    g->half_split = true;
    return FDTD_OK;
  }
  g->half_split = false;
  if (g->f32) g->launches += launch_tfsf_fused(mode, fa, phase, s);
  if (boxes) g->launches += launch_boxes(g, phase, 0, s);
  g->launches += launch_bc(g, phase, s);
  g->launches += launch_dft_gather(g->f32 ? 1 : 0, g->d_dft[phase], g->ndft[phase], g->dft_pts[phase],
                                   g->dft_maxpts[phase], fields, g->n[1], static_cast<int>(rowlen(g)),
                                   g->dft_pending, g->d_dft_buf[phase], s);
  if (phase == 1) {
    g->launches += launch_step_advance(g->ctrl, s);
    if (!g->dfts.empty() && ++g->dft_pending == kDftChunk) g->launches += flush_dft(g, s);
    g->t += 1;
  }
  CK(cudaGetLastError());
  g->next_half = 1 - phase;
  return FDTD_OK;
}

int fdtd_step_half(fdtd_grid* g, int phase, void* stream) try {
  if (g && g->half_split) return fail(FDTD_ERR_INVALID, "part 0 of this half step is waiting for its part 1");
  return half_step_impl(g, phase, -1, stream);
} catch (...) {
  return host_failure();
}

int fdtd_step_half_part(fdtd_grid* g, int phase, int part, void* stream) try {
  if (part != 0 && part != 1) return fail(FDTD_ERR_INVALID, "part must be 0 or 1");
  return half_step_impl(g, phase, part, stream);
} catch (...) {
  return host_failure();
}

// The reference's forward (explicit) material updates, XUpdate<Mode, ft,
// forward = true> (DispersiveMaterials.hpp:345-349, :922-934): the flux (and
// the Drude P and J) from the field, on every interior cell. Only the FP64
// plain method stores D and B; the reference's explicit Lorentz update is a
// static_assert (:697-706), so grids with a Lorentz material refuse ft 0.
int fdtd_material_explicit(fdtd_grid* g, int ft, void* stream) try {
  if (!g) return fail(FDTD_ERR_INVALID, "null grid");
  if (ft != 0 && ft != 1) return fail(FDTD_ERR_INVALID, "ft must be 0 (electric) or 1 (magnetic)");
  if (g->f32) return fail(FDTD_ERR_UNSUPPORTED, "the FP32 fused method stores no D or B");
  if (g->half_split) return fail(FDTD_ERR_INVALID, "part 0 of this half step is waiting for its part 1");
  if (ft == 0)
    for (const fdtd_material& m : g->mats)
      if (m.kind == FDTD_LORENTZ) return fail(FDTD_ERR_UNSUPPORTED, "the reference has no explicit Lorentz update");
  CK(cudaSetDevice(g->d.device));
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : g->stream;
  if (s != g->stream) CK(cudaStreamSynchronize(g->stream));
  const PlainArgs pa = plain_args(g);
  g->launches += launch_material_explicit(g->d.mode, pa, ft, s);
  CK(cudaGetLastError());
  return FDTD_OK;
} catch (...) {
  return host_failure();
}

// one z plane of a stored E or H component to or from a compact device
// buffer (nx * ny values of the grid's precision, x fastest; H of the FP32
// method is the stored eta * H)
int fdtd_copy_plane(fdtd_grid* g, int which, int k, void* dev_buf, int to_grid, void* stream) try {
  if (!g || !dev_buf) return fail(FDTD_ERR_INVALID, "null argument");
  if (k < 0 || k >= g->n[2]) return fail(FDTD_ERR_INVALID, "plane index out of range");
  void* f = nullptr;
  if (which >= FDTD_EX && which <= FDTD_EZ) f = g->E[which - FDTD_EX];
  else if (which >= FDTD_HX && which <= FDTD_HZ) f = g->H[which - FDTD_HX];
  if (!f) return fail(FDTD_ERR_INVALID, "only the stored E and H components of the mode are copied");
  CK(cudaSetDevice(g->d.device));
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : g->stream;
  const size_t es = elem(g), row = static_cast<size_t>(rowlen(g)) * es, w = static_cast<size_t>(g->n[0]) * es;
  char* plane = static_cast<char*>(f) + static_cast<size_t>(k) * g->n[1] * row;
  if (to_grid) CK(cudaMemcpy2DAsync(plane, row, dev_buf, w, w, g->n[1], cudaMemcpyDeviceToDevice, s));
  else CK(cudaMemcpy2DAsync(dev_buf, w, plane, row, w, g->n[1], cudaMemcpyDeviceToDevice, s));
  return FDTD_OK;
} catch (...) {
  return host_failure();
}

int fdtd_copy_plane_between(fdtd_grid* src, int which, int k_src, fdtd_grid* dst, int k_dst, void* stream) try {
  if (!src || !dst) return fail(FDTD_ERR_INVALID, "null grid");
  if (src->f32 != dst->f32 || src->d.mode != dst->d.mode || src->n[0] != dst->n[0] || src->n[1] != dst->n[1])
    return fail(FDTD_ERR_INVALID, "the two grids differ in precision, mode or plane extent");
  if (k_src < 0 || k_src >= src->n[2] || k_dst < 0 || k_dst >= dst->n[2])
    return fail(FDTD_ERR_INVALID, "plane index out of range");
  auto field = [&](fdtd_grid* g) -> void* {
    if (which >= FDTD_EX && which <= FDTD_EZ) return g->E[which - FDTD_EX];
    if (which >= FDTD_HX && which <= FDTD_HZ) return g->H[which - FDTD_HX];
    return nullptr;
  };
  void* fs = field(src);
  void* fd = field(dst);
  if (!fs || !fd) return fail(FDTD_ERR_INVALID, "only the stored E and H components of the mode are copied");
  CK(cudaSetDevice(dst->d.device));
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : dst->stream;
  const size_t es = elem(src), row = static_cast<size_t>(rowlen(src)) * es, w = static_cast<size_t>(src->n[0]) * es;
  const char* ps = static_cast<const char*>(fs) + static_cast<size_t>(k_src) * src->n[1] * row;
  char* pd = static_cast<char*>(fd) + static_cast<size_t>(k_dst) * dst->n[1] * row;
  // one strided copy; between devices the runtime routes it over the peer
  // link (unified addressing), within one device it is a device copy
  CK(cudaMemcpy2DAsync(pd, row, ps, row, w, src->n[1], cudaMemcpyDefault, s));
  return FDTD_OK;
} catch (...) {
  return host_failure();
}

int fdtd_use_graphs(fdtd_grid* g, int enable) try {
  if (!g) return fail(FDTD_ERR_INVALID, "null grid");
  g->use_graphs = enable != 0;
  return FDTD_OK;
} catch (...) {
  return host_failure();
}

int fdtd_error_flags(fdtd_grid* g, int* flags) try {
  if (!g || !flags) return fail(FDTD_ERR_INVALID, "null argument");
  CK(cudaSetDevice(g->d.device));
  Control c;
  CK(cudaStreamSynchronize(g->stream));
  CK(cudaMemcpy(&c, g->ctrl, sizeof(c), cudaMemcpyDeviceToHost));
  *flags = c.error;
  return FDTD_OK;
} catch (...) {
  return host_failure();
}

int fdtd_synchronize(fdtd_grid* g) try {
  if (!g) return fail(FDTD_ERR_INVALID, "null grid");
  CK(cudaSetDevice(g->d.device));
  CK(cudaStreamSynchronize(g->stream));
  CK(cudaDeviceSynchronize());
  return FDTD_OK;
} catch (...) {
  return host_failure();
}

// which -> (device pointer, scale to SI, element layout)
static int locate(fdtd_grid* g, int which, void** p, double* scale, int* psi_axis) {
  *p = nullptr;
  if (which >= 18 && which < 36) {
    const int prc = ensure_pml(g);
    if (prc) return prc;
  }
  *scale = 1.0;
  *psi_axis = -1;
  const double eps0 = kEps0, dt = g->d.dt;
  if (which < 0) return fail(FDTD_ERR_INVALID, "bad field selector");
  if (which < 3) {
    if (g->f32) return fail(FDTD_ERR_UNSUPPORTED, "the fused method does not store D");
    *p = g->D[which];
  } else if (which < 6) {
    *p = g->E[which - 3];
  } else if (which < 9) {
    if (g->f32) return fail(FDTD_ERR_UNSUPPORTED, "the fused method does not store B");
    *p = g->B[which - 6];
  } else if (which < 12) {
    *p = g->H[which - 9];
    if (g->f32) *scale = 1.0 / eta();
  } else if (which < 18 || which >= 36) {
    int pole = 0, r = 0;
    if (which < 18) r = which - 12;
    else {
      pole = 1 + (which - 36) / 6;
      r = (which - 36) % 6;
    }
    if (pole >= kMaxPoles) return fail(FDTD_ERR_INVALID, "bad field selector");
    *p = r < 3 ? g->P[pole][r] : g->J[pole][r - 3];
    if (g->f32) *scale = r < 3 ? eps0 : eps0 / dt;
  } else {
    const int q = which - 18, ft = q / 9, I = (q / 3) % 3, J = q % 3;
    *p = g->psi[ft][I][J];
    *psi_axis = J;
    if (g->f32) *scale = ft == 0 ? eps0 / dt : kMu0 / (eta() * dt);
  }
  return FDTD_OK;
}

int fdtd_read_quantity(fdtd_grid* g, int q, const int* lo, const int* hi, double* host) try {
  if (!g || !lo || !hi || !host) return fail(FDTD_ERR_INVALID, "null argument");
  const int qc = quantity_check(g, q, lo, hi);
  if (qc != FDTD_OK) return qc;
  CK(cudaSetDevice(g->d.device));
  const DftRegionDev r = quantity_region(g, q, lo, hi);
  if (r.npts >= (1LL << 31)) return fail(FDTD_ERR_UNSUPPORTED, "a box holds at most 2^31 - 1 cells");
  if (!g->d_fieldptrs) return fail(FDTD_ERR_INVALID, "grid has no fields");
  // a scratch of its own: the grid's tracked allocations would invalidate
  // its captured step graphs
  void* buf = nullptr;
  cudaError_t ae = cudaMalloc(&buf, static_cast<size_t>(r.npts) * elem(g));
  if (ae != cudaSuccess) {
    cudaGetLastError();
    return fail(ae == cudaErrorMemoryAllocation ? FDTD_ERR_NOMEM : FDTD_ERR_CUDA, cudaGetErrorString(ae));
  }
  const void* const* fields = reinterpret_cast<const void* const*>(g->d_fieldptrs) + (quantity_phase(q) == 0 ? 0 : 3);
  g->launches += launch_quantity_read(g->f32 ? 1 : 0, r, fields, g->n[1], static_cast<int>(rowlen(g)), buf, g->stream);
  std::vector<char> h(static_cast<size_t>(r.npts) * elem(g));
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  if (e == cudaSuccess) e = cudaMemcpy(h.data(), buf, h.size(), cudaMemcpyDeviceToHost);
  cudaFree(buf);
  if (e != cudaSuccess) return fail(FDTD_ERR_CUDA, cudaGetErrorString(e));
  const double hs = (g->f32 && q >= 3 && q < 6) ? 1.0 / eta() : 1.0;  // stored H is eta*H
  for (long long p = 0; p < r.npts; p++)
    host[p] = g->f32 ? static_cast<double>(reinterpret_cast<float*>(h.data())[p]) * hs
                     : reinterpret_cast<double*>(h.data())[p];
  return FDTD_OK;
} catch (...) {
  return host_failure();
}

int fdtd_download(fdtd_grid* g, int which, double* host) try {
  if (!g || !host) return fail(FDTD_ERR_INVALID, "null argument");
  void* p;
  double scale;
  int J;
  int rc = locate(g, which, &p, &scale, &J);
  if (rc) return rc;
  CK(cudaSetDevice(g->d.device));
  CK(cudaStreamSynchronize(g->stream));
  const long long nx = g->n[0], ny = g->n[1], nz = g->n[2];
  const long long ncell = nx * ny * nz;
  if (!p) {
    memset(host, 0, ncell * sizeof(double));
    return FDTD_OK;
  }
  long long cnt = field_elems(g);
  if (J >= 0) {
    if (J == 0) cnt = nz * ny * xslab_row(g);
    else if (J == 1) cnt = nz * g->slab[1].W * rowlen(g);
    else cnt = static_cast<long long>(g->slab[2].W) * ny * rowlen(g);
  }
  std::vector<char> buf(cnt * elem(g));
  CK(cudaMemcpy(buf.data(), p, buf.size(), cudaMemcpyDeviceToHost));
  auto val = [&](long long q) -> double {
    return g->f32 ? static_cast<double>(reinterpret_cast<float*>(buf.data())[q])
                  : reinterpret_cast<double*>(buf.data())[q];
  };
  const long long rl = rowlen(g);
  for (long long k = 0; k < nz; k++)
    for (long long j = 0; j < ny; j++)
      for (long long i = 0; i < nx; i++) {
        const long long o = (k * ny + j) * nx + i;
        if (J < 0) {
          host[o] = val((k * ny + j) * rl + i) * scale;
        } else {
          const int idx[3] = {static_cast<int>(i), static_cast<int>(j), static_cast<int>(k)};
          const bool in = interior(g, idx[0], idx[1], idx[2]);
          const int s = in ? slab_index(g->slab[J], idx[J]) : -1;
          if (s < 0) {
            host[o] = 0.0;
            continue;
          }
          long long q;
          if (J == 0) q = (k * ny + j) * xslab_row(g) + (xslab_aligned(g) ? slab_index4(g->slab[0], idx[0]) : s);
          else if (J == 1) q = (k * g->slab[1].W + s) * rl + i;
          else q = (static_cast<long long>(s) * ny + j) * rl + i;
          host[o] = val(q) * scale;
        }
      }
  return FDTD_OK;
} catch (...) {
  return host_failure();
}

int fdtd_upload(fdtd_grid* g, int which, const double* host) try {
  if (!g || !host) return fail(FDTD_ERR_INVALID, "null argument");
  void* p;
  double scale;
  int J;
  int rc = locate(g, which, &p, &scale, &J);
  if (rc) return rc;
  if (!p) return fail(FDTD_ERR_UNSUPPORTED, "field not stored for this grid");
  if (J >= 0) return fail(FDTD_ERR_UNSUPPORTED, "CPML integrators cannot be uploaded");
  CK(cudaSetDevice(g->d.device));
  CK(cudaStreamSynchronize(g->stream));
  const long long nx = g->n[0], ny = g->n[1], nz = g->n[2], rl = rowlen(g);
  std::vector<char> buf(field_elems(g) * elem(g), 0);
  for (long long k = 0; k < nz; k++)
    for (long long j = 0; j < ny; j++)
      for (long long i = 0; i < nx; i++) {
        const double v = host[(k * ny + j) * nx + i] / scale;
        const long long q = (k * ny + j) * rl + i;
        if (g->f32) reinterpret_cast<float*>(buf.data())[q] = static_cast<float>(v);
        else reinterpret_cast<double*>(buf.data())[q] = v;
      }
  CK(cudaMemcpy(p, buf.data(), buf.size(), cudaMemcpyHostToDevice));
  return FDTD_OK;
} catch (...) {
  return host_failure();
}

int fdtd_check_finite(fdtd_grid* g) try {
  if (!g) return fail(FDTD_ERR_INVALID, "null grid");
  CK(cudaSetDevice(g->d.device));
  CK(cudaMemsetAsync(g->d_flag, 0, sizeof(int), g->stream));
  std::vector<void*> arrs;
  for (int c = 0; c < 3; c++) {
    arrs.push_back(g->E[c]);
    arrs.push_back(g->H[c]);
    arrs.push_back(g->D[c]);
    arrs.push_back(g->B[c]);
  }
  for (void* p : arrs)
    if (p) g->launches += launch_finite_check(p, field_elems(g), g->f32 ? 1 : 0, g->d_flag, g->stream);
  int flag = 0;
  CK(cudaMemcpyAsync(&flag, g->d_flag, sizeof(int), cudaMemcpyDeviceToHost, g->stream));
  CK(cudaStreamSynchronize(g->stream));
  if (flag) return fail(FDTD_ERR_NONFINITE, "a field holds NaN or Inf");
  return FDTD_OK;
} catch (...) {
  return host_failure();
}

int fdtd_field_error(fdtd_grid* g, fdtd_grid* ref, int which, double* err_sq, double* ref_sq) try {
  if (!g || !ref || !err_sq || !ref_sq) return fail(FDTD_ERR_INVALID, "null argument");
  if (g->d.device != ref->d.device) return fail(FDTD_ERR_INVALID, "the two grids live on different devices");
  for (int d = 0; d < 3; d++)
    if (g->n[d] != ref->n[d]) return fail(FDTD_ERR_INVALID, "the two grids differ in shape");
  if (which >= 18 && which < 36) return fail(FDTD_ERR_UNSUPPORTED, "CPML integrators are not compared");
  void *pa, *pb;
  double sa, sb;
  int ja, jb;
  int rc = locate(g, which, &pa, &sa, &ja);
  if (rc) return rc;
  rc = locate(ref, which, &pb, &sb, &jb);
  if (rc) return rc;
  if (!pa || !pb) return fail(FDTD_ERR_UNSUPPORTED, "field not stored by one of the grids");
  CK(cudaSetDevice(g->d.device));
  CK(cudaStreamSynchronize(ref->stream));
  double* out = nullptr;
  cudaError_t e = cudaMalloc(&out, 2 * sizeof(double));
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(e == cudaErrorMemoryAllocation ? FDTD_ERR_NOMEM : FDTD_ERR_CUDA, cudaGetErrorString(e));
  }
  double h[2] = {0.0, 0.0};
  e = cudaMemsetAsync(out, 0, 2 * sizeof(double), g->stream);
  if (e == cudaSuccess) {
    g->launches += launch_field_diff(pa, g->f32 ? 1 : 0, rowlen(g), sa, pb, ref->f32 ? 1 : 0, rowlen(ref), sb,
                                     g->n[0], static_cast<long long>(g->n[1]) * g->n[2], out, g->stream);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, g->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  cudaFree(out);
  if (e != cudaSuccess) return fail(FDTD_ERR_CUDA, cudaGetErrorString(e));
  *err_sq = h[0];
  *ref_sq = h[1];
  return FDTD_OK;
} catch (...) {
  return host_failure();
}

int fdtd_get_step(fdtd_grid* g, long long* step) try {
  if (!g || !step) return fail(FDTD_ERR_INVALID, "null argument");
  *step = g->t;
  return FDTD_OK;
} catch (...) {
  return host_failure();
}

int fdtd_launch_count(fdtd_grid* g, long long* count) try {
  if (!g || !count) return fail(FDTD_ERR_INVALID, "null argument");
  *count = g->launches;
  return FDTD_OK;
} catch (...) {
  return host_failure();
}

int fdtd_memory_bytes(fdtd_grid* g, long long* bytes) try {
  if (!g || !bytes) return fail(FDTD_ERR_INVALID, "null argument");
  *bytes = g->bytes;
  return FDTD_OK;
} catch (...) {
  return host_failure();
}

}  // extern "C"

// ---------------------------------------------------------------- batches

struct fdtd_batch {
  std::vector<fdtd_grid*> grids;
  int mode = 0, maxp = 0, device = 0;
  FusedArgs* d_args = nullptr;
  Control** d_ctrls = nullptr;
  BatchCtl* d_ctl = nullptr;
  unsigned* d_items = nullptr;
  int nitems = 0, rows = 0, blocks = 0;
  int persistent = 1;  // 1: one cooperative kernel for all steps; 0: one kernel per half step
  std::vector<FusedArgs> h_args;  // host copy of d_args
  std::vector<int> mult;          // per grid: work-item rows = rows * mult
  std::vector<int> cls;           // per grid: its size class (quartile of cell counts), for the tuner
  cudaStream_t stream = nullptr;
  std::map<int, cudaGraphExec_t> graphs;  // keyed by steps per launch
  // measured ms per step: persistent with rows 1, 2, 4, 8, then per-phase with rows 1, 2, 4, 8
  std::vector<float> tune_ms;
  float tune_best_ms = 0.f;  // with the per-class item heights
  // temporal blocking (fdtd_batch_set_temporal): steps per launch (0: off),
  // the grids' arguments on the second copy of their state, the tiles
  int tb = 0;
  FusedArgs* d_args_b = nullptr;
  unsigned* d_tb_items = nullptr;
  int n_tb_items = 0;
  std::vector<void*> tb_bufs;  // the second copy
  std::vector<float> tb_ms;    // tuner: ms per step with 2, 3 and 4 steps per launch (0: not timed)
};

namespace {

// the mutable state of a grid (what a step changes): fields, poles, CPML
// integrators, source bookkeeping and the step counter
std::vector<std::pair<void*, size_t>> grid_state(fdtd_grid* g) {
  std::vector<void*> ptrs;
  for (int c = 0; c < 3; c++) {
    ptrs.push_back(g->E[c]);
    ptrs.push_back(g->H[c]);
    for (int q = 0; q < kMaxPoles; q++) {
      ptrs.push_back(g->P[q][c]);
      ptrs.push_back(g->J[q][c]);
    }
  }
  for (int ft = 0; ft < 2; ft++)
    for (int I = 0; I < 3; I++)
      for (int J = 0; J < 3; J++) ptrs.push_back(g->psi[ft][I][J]);
  ptrs.push_back(g->d_src_last);
  ptrs.push_back(g->ctrl);
  std::vector<std::pair<void*, size_t>> out;
  for (void* p : ptrs)
    if (p && g->sizes.count(p)) out.emplace_back(p, g->sizes[p]);
  return out;
}

// the work list of kernel tile height `rows`, each grid's items `rows *
// b->mult[grid]` rows high (the grids' arguments are re-uploaded with it)
int batch_items(fdtd_batch* b, int rows) {
  std::vector<unsigned> items;
  for (size_t q = 0; q < b->grids.size(); q++) {
    const fdtd_grid* g = b->grids[q];
    const int R = rows * b->mult[q];
    b->h_args[q].item_rows = R;
    const int tx = g->pitch / 128, ty = (g->n[1] - 2 + R - 1) / R;
    for (int t = 0; t < tx * ty; t++) items.push_back(static_cast<unsigned>(q) << 24 | static_cast<unsigned>(t));
  }
  CK(cudaMemcpy(b->d_args, b->h_args.data(), b->h_args.size() * sizeof(FusedArgs), cudaMemcpyHostToDevice));
  // consecutive items (tiles of one grid) go to consecutive CTAs
  b->nitems = static_cast<int>(items.size());
  if (b->d_items) cudaFree(b->d_items);
  b->d_items = nullptr;
  CK(cudaMalloc(&b->d_items, items.size() * sizeof(unsigned)));
  CK(cudaMemcpy(b->d_items, items.data(), items.size() * sizeof(unsigned), cudaMemcpyHostToDevice));
  void* fn = batch_kernel_ptr(b->mode, b->maxp, rows);
  int per_sm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 32 * rows, 0));
  int sms = 0;
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device));
  if (per_sm < 1) return fail(FDTD_ERR_CUDA, "batch kernel does not fit on an SM");
  b->blocks = std::min(b->nitems, per_sm * sms);
  b->rows = rows;
  return FDTD_OK;
}

// Temporal blocking needs grids without poles whose sources lie inside their
// interiors (a window applies a source only where it updates the cell).
const char* tb_unsupported(const fdtd_batch* b) {
  if (b->maxp != 0) return "temporal blocking takes grids without dispersive materials";
  for (const FusedArgs& a : b->h_args)
    for (int q = 0; q < a.nsrc; q++)
      if (a.src[q].i < 1 || a.src[q].i > a.nx - 2 || a.src[q].j < 1 || a.src[q].j > a.ny - 2)
        return "temporal blocking takes sources inside the grid's interior only";
  return nullptr;
}

// frees the second copy of the state and the tiles (temporal blocking off)
void tb_release(fdtd_batch* b) {
  cudaFree(b->d_args_b);
  cudaFree(b->d_tb_items);
  for (void* p : b->tb_bufs) cudaFree(p);
  b->d_args_b = nullptr;
  b->d_tb_items = nullptr;
  b->n_tb_items = 0;
  b->tb_bufs.clear();
  b->tb = 0;
}

// The second copy of every array a step changes (fields, CPML integrators,
// the soft sources' last values) and the grids' arguments pointing at it;
// laid out once, a copy of the current state. On failure nothing is kept.
int tb_prepare(fdtd_batch* b) {
  if (b->d_args_b) return FDTD_OK;
  CK(cudaDeviceSynchronize());
  std::vector<FusedArgs> args = b->h_args;
  bool ok = true;
  for (size_t q = 0; q < b->grids.size() && ok; q++) {
    fdtd_grid* g = b->grids[q];
    FusedArgs& a = args[q];
    // a same-sized copy of the state array p (null if p is not one)
    auto twin = [&](void* p) -> void* {
      if (!g->sizes.count(p)) return nullptr;
      void* d = nullptr;
      if (cudaMalloc(&d, g->sizes[p]) != cudaSuccess) return nullptr;
      b->tb_bufs.push_back(d);
      if (cudaMemcpy(d, p, g->sizes[p], cudaMemcpyDeviceToDevice) != cudaSuccess) return nullptr;
      return d;
    };
    for (int c = 0; c < 3 && ok; c++) {
      if (g->E[c]) ok = ok && (a.E[c] = static_cast<float*>(twin(g->E[c])));
      if (g->H[c]) ok = ok && (a.H[c] = static_cast<float*>(twin(g->H[c])));
    }
    for (int ft = 0; ft < 2; ft++)
      for (int I = 0; I < 3; I++)
        for (int J = 0; J < 3; J++)
          if (g->psi[ft][I][J]) ok = ok && (a.psi[ft][I][J] = static_cast<float*>(twin(g->psi[ft][I][J])));
    if (g->d_src_last) ok = ok && (a.src_last = static_cast<double*>(twin(g->d_src_last)));
  }
  if (ok) ok = cudaMalloc(&b->d_args_b, args.size() * sizeof(FusedArgs)) == cudaSuccess;
  if (ok)
    ok = cudaMemcpy(b->d_args_b, args.data(), args.size() * sizeof(FusedArgs), cudaMemcpyHostToDevice) == cudaSuccess;
  if (!ok) {
    const cudaError_t e = cudaGetLastError();
    tb_release(b);
    return fail(FDTD_ERR_CUDA, std::string("temporal blocking: the second copy of the state: ") + cudaGetErrorString(e));
  }
  return FDTD_OK;
}

// the tiles of the temporally blocked launches of depth `depth`
int tb_items(fdtd_batch* b, int depth) {
  int tw = 0, th = 0;
  if (!batch_tb_tile(depth, &tw, &th)) return fail(FDTD_ERR_INVALID, "temporal blocking depth must be 2, 3 or 4");
  std::vector<unsigned> items;
  for (size_t q = 0; q < b->grids.size(); q++) {
    const fdtd_grid* g = b->grids[q];
    const long long nt = static_cast<long long>((g->n[0] + tw - 1) / tw) * ((g->n[1] + th - 1) / th);
    if (nt >= (1 << 24)) return fail(FDTD_ERR_UNSUPPORTED, "grid too large to batch");
    for (long long t = 0; t < nt; t++) items.push_back(static_cast<unsigned>(q) << 24 | static_cast<unsigned>(t));
  }
  if (b->d_tb_items) cudaFree(b->d_tb_items);
  b->d_tb_items = nullptr;
  b->n_tb_items = static_cast<int>(items.size());
  CK(cudaMalloc(&b->d_tb_items, items.size() * sizeof(unsigned)));
  CK(cudaMemcpy(b->d_tb_items, items.data(), items.size() * sizeof(unsigned), cudaMemcpyHostToDevice));
  return FDTD_OK;
}

int batch_launch(fdtd_batch* b, int nsteps, cudaStream_t s) {
  const FusedArgs* args = b->d_args;
  const unsigned* items = b->d_items;
  int s0 = 0;
  if (b->tb > 0) {
    // pairs of launches of tb steps each, there and back, so that the state
    // ends in the grids' own arrays; the rest one kernel per half step
    const int T = b->tb, pairs = nsteps / (2 * T);
    for (int p = 0; p < pairs; p++) {
      launch_batch_tb(b->mode, T, b->d_args, b->d_args_b, b->d_tb_items, b->n_tb_items, s0, s);
      launch_batch_tb(b->mode, T, b->d_args_b, b->d_args, b->d_tb_items, b->n_tb_items, s0 + T, s);
      s0 += 2 * T;
    }
    CK(cudaGetLastError());
  }
  if (!b->persistent || b->tb > 0) {
    void* fe = batch_phase_ptr(b->mode, b->maxp, b->rows, 0);
    void* fh = batch_phase_ptr(b->mode, b->maxp, b->rows, 1);
    for (int q = s0; q < nsteps; q++) {
      void* params[] = {&args, &items, &q};
      CK(cudaLaunchKernel(fe, dim3(b->nitems), dim3(32, b->rows), params, 0, s));
      CK(cudaLaunchKernel(fh, dim3(b->nitems), dim3(32, b->rows), params, 0, s));
    }
    return FDTD_OK;
  }
  void* fn = batch_kernel_ptr(b->mode, b->maxp, b->rows);
  int nitems = b->nitems;
  BatchCtl* ctl = b->d_ctl;
  void* params[] = {&args, &items, &nitems, &ctl, &nsteps};
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(b->blocks);
  cfg.blockDim = dim3(32, b->rows);
  cfg.stream = s;
  cudaLaunchAttribute attr;
  attr.id = cudaLaunchAttributeCooperative;
  attr.val.cooperative = 1;
  cfg.attrs = &attr;
  cfg.numAttrs = 1;
  CK(cudaLaunchKernelExC(&cfg, fn, params));
  return FDTD_OK;
}

}  // namespace

extern "C" {

int fdtd_batch_create(int n, fdtd_grid* const* grids, fdtd_batch** out) try {
  if (!grids || !out || n < 1) return fail(FDTD_ERR_INVALID, "need at least one grid");
  if (n > 255) return fail(FDTD_ERR_UNSUPPORTED, "at most 255 grids per batch");
  *out = nullptr;
  fdtd_batch* b = new fdtd_batch();
  b->grids.assign(grids, grids + n);
  const fdtd_grid* g0 = grids[0];
  b->mode = g0->d.mode;
  b->device = g0->d.device;
  for (auto* g : b->grids) {
    const char* why = nullptr;
    if (!g) why = "null grid";
    else if (!g->f32) why = "batched grids use the FP32 fused method";
    else if (g->d.mode != FDTD_TE && g->d.mode != FDTD_TM) why = "batched grids are 2D (TE or TM)";
    else if (g->d.mode != b->mode) why = "batched grids share one mode";
    else if (g->d.device != b->device) why = "batched grids share one device";
    else if (!g->planes.empty() || !g->dfts.empty()) why = "batched grids carry no TFSF planes or DFT regions";
    else if (!g->boxes.empty()) why = "batched grids carry no box sources";
    else if (g->bcs.n > 0) why = "batched grids carry no boundary conditions";
    else if (std::any_of(g->mats.begin(), g->mats.end(), [](const fdtd_material& m) { return m.mu_r != 1.0; }))
      why = "batched grids take mu_r = 1";
    else if (g->t != g0->t) why = "batched grids must have taken the same number of steps";
    else if (static_cast<long long>(g->pitch / 128) * g->n[1] >= (1 << 24)) why = "grid too large to batch";
    if (why) {
      delete b;
      return fail(FDTD_ERR_UNSUPPORTED, why);
    }
    b->maxp = std::max(b->maxp, g->max_poles == -1 ? 1 : g->max_poles);
  }
  if (b->maxp == 1) {
    // Drude-only batches keep the Drude kernel (no P arrays)
    bool lorentz = false;
    for (auto* g : b->grids) lorentz = lorentz || g->max_poles > 0;
    if (!lorentz) b->maxp = -1;
  }
  CK(cudaSetDevice(b->device));
  CK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
  std::vector<FusedArgs> args;
  std::vector<Control*> ctrls;
  for (auto* g : b->grids) {
    const int prc = ensure_pml(g);
    if (prc) return prc;
    CK(cudaStreamSynchronize(g->stream));
    args.push_back(fused_args(g));
    ctrls.push_back(g->ctrl);
  }
  CK(cudaMalloc(&b->d_args, args.size() * sizeof(FusedArgs)));
  CK(cudaMemcpy(b->d_args, args.data(), args.size() * sizeof(FusedArgs), cudaMemcpyHostToDevice));
  b->h_args = args;
  b->mult.assign(b->grids.size(), 1);
  {
    // size classes: quartiles of the grids' cell counts
    std::vector<int> order(b->grids.size());
    for (size_t q = 0; q < order.size(); q++) order[q] = static_cast<int>(q);
    auto cells = [&](int q) { return static_cast<long long>(b->grids[q]->n[0]) * b->grids[q]->n[1]; };
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cells(x) < cells(y); });
    b->cls.assign(b->grids.size(), 0);
    const int nc = std::min<int>(4, static_cast<int>(order.size()));
    for (size_t r = 0; r < order.size(); r++) b->cls[order[r]] = static_cast<int>(r * nc / order.size());
  }
  CK(cudaMalloc(&b->d_ctrls, ctrls.size() * sizeof(Control*)));
  CK(cudaMemcpy(b->d_ctrls, ctrls.data(), ctrls.size() * sizeof(Control*), cudaMemcpyHostToDevice));
  CK(cudaMalloc(&b->d_ctl, sizeof(BatchCtl)));
  CK(cudaMemset(b->d_ctl, 0, sizeof(BatchCtl)));
  int rc = batch_items(b, 4);
  if (rc) {
    fdtd_batch_destroy(b);
    return rc;
  }
  *out = b;
  return FDTD_OK;
} catch (...) {
  return host_failure();
}

int fdtd_batch_destroy(fdtd_batch* b) try {
  if (!b) return FDTD_OK;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
  cudaFree(b->d_args);
  cudaFree(b->d_ctrls);
  cudaFree(b->d_ctl);
  cudaFree(b->d_items);
  tb_release(b);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return FDTD_OK;
} catch (...) {
  return host_failure();
}

// Times every tile height on a copy of the state (restored afterwards) and
// keeps the fastest.
int fdtd_batch_tune(fdtd_batch* b, int steps) try {
  if (!b || steps < 1) return fail(FDTD_ERR_INVALID, "bad argument");
  CK(cudaSetDevice(b->device));
  CK(cudaDeviceSynchronize());
  std::vector<std::pair<void*, size_t>> state;
  for (auto* g : b->grids)
    for (auto& st : grid_state(g)) state.push_back(st);
  size_t total = 0;
  for (auto& st : state) total += (st.second + 255) / 256 * 256;
  void* scratch = nullptr;
  CK(cudaMalloc(&scratch, total));
  auto copy = [&](bool save) -> int {
    size_t off = 0;
    for (auto& st : state) {
      char* sp = static_cast<char*>(scratch) + off;
      CK(cudaMemcpyAsync(save ? sp : st.first, save ? st.first : sp, st.second, cudaMemcpyDeviceToDevice, b->stream));
      off += (st.second + 255) / 256 * 256;
    }
    return FDTD_OK;
  };
  int rc = copy(true);
  b->tb = 0;
  // candidates: the persistent kernel and the per-phase launches, each with
  // tiles of 1, 2, 4 or 8 rows
  const int cand[4] = {1, 2, 4, 8};
  b->mult.assign(b->grids.size(), 1);
  float best = 1e30f;
  int best_rows = 4, best_persistent = 1;
  b->tune_ms.assign(8, 0.f);
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  for (int q = 0; q < 8 && !rc; q++) {
    b->persistent = q < 4 ? 1 : 0;
    rc = batch_items(b, cand[q % 4]);
    if (!rc) rc = batch_launch(b, 1, b->stream);  // warm-up
    if (!rc) rc = copy(false);
    CK(cudaEventRecord(e0, b->stream));
    if (!rc) rc = batch_launch(b, steps, b->stream);
    CK(cudaEventRecord(e1, b->stream));
    CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    b->tune_ms[q] = ms / steps;
    if (ms < best) {
      best = ms;
      best_rows = cand[q % 4];
      best_persistent = b->persistent;
    }
    if (!rc) rc = copy(false);
  }
  // per size class: the work-item height, in multiples 1, 2, 4, 8 of the
  // chosen kernel tile height, one class after the other (largest grids
  // first), the others held at their best so far
  b->persistent = best_persistent;
  const int ncls = b->cls.empty() ? 0 : 1 + *std::max_element(b->cls.begin(), b->cls.end());
  for (int c = ncls - 1; c >= 0 && !rc; c--) {
    int keep = 1;
    for (int m : {2, 4, 8}) {
      std::vector<int> old = b->mult;
      for (size_t q = 0; q < b->grids.size(); q++)
        if (b->cls[q] == c) b->mult[q] = m;
      rc = batch_items(b, best_rows);
      if (!rc) rc = batch_launch(b, 1, b->stream);
      if (!rc) rc = copy(false);
      CK(cudaEventRecord(e0, b->stream));
      if (!rc) rc = batch_launch(b, steps, b->stream);
      CK(cudaEventRecord(e1, b->stream));
      CK(cudaEventSynchronize(e1));
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, e0, e1));
      if (!rc) rc = copy(false);
      if (ms < best) {
        best = ms;
        keep = m;
      } else {
        b->mult = old;
      }
    }
    for (size_t q = 0; q < b->grids.size(); q++)
      if (b->cls[q] == c) b->mult[q] = keep;
  }
  // temporal blocking with 2, 3 and 4 steps per launch, timed over whole
  // pairs of launches
  float best_step = best / steps;
  int best_tb = 0;
  b->tb_ms.assign(3, 0.f);
  if (!rc && !tb_unsupported(b)) {
    rc = tb_prepare(b);
    if (!rc) rc = batch_items(b, best_rows);
    for (int depth = 2; depth <= 4 && !rc; depth++) {
      const int n = (steps + 2 * depth - 1) / (2 * depth) * (2 * depth);
      rc = tb_items(b, depth);
      b->tb = depth;
      if (!rc) rc = batch_launch(b, 2 * depth, b->stream);  // warm-up
      if (!rc) rc = copy(false);
      CK(cudaEventRecord(e0, b->stream));
      if (!rc) rc = batch_launch(b, n, b->stream);
      CK(cudaEventRecord(e1, b->stream));
      CK(cudaEventSynchronize(e1));
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, e0, e1));
      if (!rc) rc = copy(false);
      b->tb_ms[depth - 2] = ms / n;
      if (ms / n < best_step) {
        best_step = ms / n;
        best_tb = depth;
      }
    }
    b->tb = 0;
    if (!rc && best_tb) rc = tb_items(b, best_tb);
  }
  CK(cudaStreamSynchronize(b->stream));
  if (!best_tb) tb_release(b);  // the second copy is kept only while in use
  if (!rc) b->tb = best_tb;
  b->tune_best_ms = best_step;
  CK(cudaStreamSynchronize(b->stream));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(scratch);
  if (rc) return rc;
  int err = 0;
  CK(cudaMemcpy(&err, &b->d_ctl->error, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) return fail(FDTD_ERR_TIMEOUT, "a batch grid barrier expired while tuning");
  for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
  b->graphs.clear();
  b->persistent = best_persistent;
  return batch_items(b, best_rows);
} catch (...) {
  return host_failure();
}

int fdtd_batch_set_temporal(fdtd_batch* b, int depth) try {
  if (!b) return fail(FDTD_ERR_INVALID, "null batch");
  if (depth != 0 && depth != 2 && depth != 3 && depth != 4)
    return fail(FDTD_ERR_INVALID, "temporal blocking depth must be 0, 2, 3 or 4");
  CK(cudaSetDevice(b->device));
  CK(cudaStreamSynchronize(b->stream));
  if (depth > 0) {
    if (const char* why = tb_unsupported(b)) return fail(FDTD_ERR_UNSUPPORTED, why);
    int rc = tb_prepare(b);
    if (!rc) rc = tb_items(b, depth);
    if (rc) return rc;
  }
  for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
  b->graphs.clear();
  if (depth == 0) tb_release(b);
  b->tb = depth;
  return FDTD_OK;
} catch (...) {
  return host_failure();
}

int fdtd_batch_temporal(fdtd_batch* b, int* depth, float* tuned_ms) try {
  if (!b) return fail(FDTD_ERR_INVALID, "null batch");
  if (depth) *depth = b->tb;
  if (tuned_ms)
    for (int q = 0; q < 3; q++) tuned_ms[q] = q < static_cast<int>(b->tb_ms.size()) ? b->tb_ms[q] : 0.f;
  return FDTD_OK;
} catch (...) {
  return host_failure();
}

int fdtd_batch_configure(fdtd_batch* b, int persistent, int rows) try {
  if (!b) return fail(FDTD_ERR_INVALID, "null batch");
  if (rows != 1 && rows != 2 && rows != 4 && rows != 8) return fail(FDTD_ERR_INVALID, "rows must be 1, 2, 4 or 8");
  CK(cudaSetDevice(b->device));
  CK(cudaStreamSynchronize(b->stream));
  for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
  b->graphs.clear();
  tb_release(b);
  b->persistent = persistent ? 1 : 0;
  b->mult.assign(b->grids.size(), 1);
  return batch_items(b, rows);
} catch (...) {
  return host_failure();
}

int fdtd_batch_set_item_rows(fdtd_batch* b, const int* rows_per_grid) try {
  if (!b || !rows_per_grid) return fail(FDTD_ERR_INVALID, "null argument");
  std::vector<int> m(b->grids.size());
  for (size_t q = 0; q < b->grids.size(); q++) {
    const int r = rows_per_grid[q];
    if (r < b->rows || r % b->rows != 0 || (r / b->rows & (r / b->rows - 1)) != 0 || r / b->rows > 8)
      return fail(FDTD_ERR_INVALID, "item rows must be the tile height times 1, 2, 4 or 8");
    m[q] = r / b->rows;
  }
  CK(cudaSetDevice(b->device));
  CK(cudaStreamSynchronize(b->stream));
  for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
  b->graphs.clear();
  b->mult = m;
  return batch_items(b, b->rows);
} catch (...) {
  return host_failure();
}

int fdtd_batch_item_rows(fdtd_batch* b, int* rows_per_grid, int* size_class, float* tuned_ms) try {
  if (!b) return fail(FDTD_ERR_INVALID, "null batch");
  for (size_t q = 0; q < b->grids.size(); q++) {
    if (rows_per_grid) rows_per_grid[q] = b->rows * b->mult[q];
    if (size_class) size_class[q] = b->cls[q];
  }
  if (tuned_ms) *tuned_ms = b->tune_best_ms;
  return FDTD_OK;
} catch (...) {
  return host_failure();
}

int fdtd_batch_step(fdtd_batch* b, int nsteps, void* stream) try {
  if (!b || nsteps < 0) return fail(FDTD_ERR_INVALID, "bad argument");
  if (nsteps == 0) return FDTD_OK;
  CK(cudaSetDevice(b->device));
  for (auto* g : b->grids)
    if (g->t != b->grids[0]->t) return fail(FDTD_ERR_INVALID, "a batched grid was stepped on its own");
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : b->stream;
  for (auto* g : b->grids) {
    cudaEvent_t ev;
    CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    CK(cudaEventRecord(ev, g->stream));
    CK(cudaStreamWaitEvent(s, ev, 0));
    CK(cudaEventDestroy(ev));
  }
  // one persistent kernel for all the steps and the step counters, replayed
  // from a CUDA graph
  auto it = b->graphs.find(nsteps);
  if (it == b->graphs.end()) {
    CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    int rc = batch_launch(b, nsteps, s);
    if (!rc) launch_batch_advance(b->d_ctrls, static_cast<int>(b->grids.size()), nsteps, s);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(s, &graph);
    if (rc) return rc;
    if (e != cudaSuccess) return fail(FDTD_ERR_CUDA, std::string("batch capture: ") + cudaGetErrorString(e));
    cudaGraphExec_t exec = nullptr;
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(FDTD_ERR_CUDA, std::string("batch instantiate: ") + cudaGetErrorString(e));
    it = b->graphs.emplace(nsteps, exec).first;
  }
  CK(cudaGraphLaunch(it->second, s));
  const long long tb_steps = b->tb > 0 ? nsteps / (2 * b->tb) * 2LL * b->tb : 0;
  for (auto* g : b->grids) {
    g->t += nsteps;
    if (b->tb > 0) g->launches += tb_steps / b->tb + 2LL * (nsteps - tb_steps) + 1;
    else g->launches += b->persistent ? 2 : 2LL * nsteps + 1;
  }
  // later work on any member grid's own stream follows the batch
  cudaEvent_t ev;
  CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  CK(cudaEventRecord(ev, s));
  for (auto* g : b->grids) CK(cudaStreamWaitEvent(g->stream, ev, 0));
  CK(cudaEventDestroy(ev));
  return FDTD_OK;
} catch (...) {
  return host_failure();
}

int fdtd_batch_info(fdtd_batch* b, int* rows, int* blocks, int* items, int* persistent, float* tune_ms) try {
  if (!b) return fail(FDTD_ERR_INVALID, "null batch");
  if (rows) *rows = b->rows;
  if (blocks) *blocks = b->persistent ? b->blocks : b->nitems;
  if (items) *items = b->nitems;
  if (persistent) *persistent = b->persistent;
  if (tune_ms)
    for (int q = 0; q < 8; q++) tune_ms[q] = q < static_cast<int>(b->tune_ms.size()) ? b->tune_ms[q] : 0.f;
  return FDTD_OK;
} catch (...) {
  return host_failure();
}

int fdtd_batch_error_flags(fdtd_batch* b, int* flags) try {
  if (!b || !flags) return fail(FDTD_ERR_INVALID, "null argument");
  CK(cudaSetDevice(b->device));
  CK(cudaStreamSynchronize(b->stream));
  CK(cudaDeviceSynchronize());
  CK(cudaMemcpy(flags, &b->d_ctl->error, sizeof(int), cudaMemcpyDeviceToHost));
  return FDTD_OK;
} catch (...) {
  return host_failure();
}

}  // extern "C"

// ----------------------------------------------------------------------------
// fdtd_step_static_scratch: the time step for callers that must not allocate
// device memory once their grid is set up.
//
// The only scratch a step needs is the TFSF incident-field table: for every
// plane, the aux grid's Ez and Hy after each step of the call, 2 (nsteps + 1) L
// doubles. fdtd_step keeps it in a per-grid buffer that it grows with
// cudaMalloc when a call asks for more steps than any call before. Here the
// table lives in the fixed array below instead, so stepping allocates nothing:
// no cudaMalloc, no cudaFree, no allocating library call, no graph. Steps run
// as eagerly launched kernels, the same kernels and order as fdtd_step.
//
// * Size limit: kStaticAuxBytes (4 MiB) for the tables of all planes of one
//   call, i.e. at most 4 MiB / (16 bytes x sum of the planes' L) - 1 steps per
//   call; a larger call is refused with FDTD_ERR_INVALID and the limit in the
//   message (split it into several calls).
// * The device address of the array is looked up with cudaGetSymbolAddress
//   once per device, on the first call there, and cached. That first lookup
//   may make the runtime load this library's device code, so make the first
//   call before any stream capture starts.
// * Nothing in the array has to start at zero: the aux precompute kernel
//   writes every row of every table before the sweeps of the call read it.
// * The array is one per device, shared by every grid on it. Calls whose GPU
//   work overlaps (different streams, different host threads) race on it;
//   order them on one stream or synchronise between them.
namespace {

constexpr size_t kStaticAuxBytes = size_t(4) << 20;
static __device__ __align__(256) double g_static_aux[kStaticAuxBytes / sizeof(double)];

std::mutex g_static_aux_mu;
double* g_static_aux_addr[64] = {};

int static_aux_address(int device, double** out) {
  if (device < 0 || device >= 64) return fail(FDTD_ERR_INVALID, "device index out of range");
  std::lock_guard<std::mutex> lock(g_static_aux_mu);
  if (!g_static_aux_addr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_static_aux);
    if (e != cudaSuccess || !p)
      return fail(FDTD_ERR_CUDA, std::string("cudaGetSymbolAddress(static TFSF table): ") + cudaGetErrorString(e));
    g_static_aux_addr[device] = static_cast<double*>(p);
  }
  *out = g_static_aux_addr[device];
  return FDTD_OK;
}

}  // namespace

extern "C" int fdtd_step_static_scratch(fdtd_grid* g, int nsteps, void* stream) try {
  if (!g) return fail(FDTD_ERR_INVALID, "null grid");
  if (g->next_half != 0 || g->half_split) return fail(FDTD_ERR_INVALID, "an E half step was taken without its H half");
  if (nsteps < 0) return fail(FDTD_ERR_INVALID, "nsteps < 0");
  if (nsteps == 0) return FDTD_OK;
  CK(cudaSetDevice(g->d.device));
  double* base = nullptr;
  int rc = static_aux_address(g->d.device, &base);
  if (rc) return rc;
  size_t row = 0;  // doubles per step over all planes' tables
  for (auto& a : g->auxes) row += 2 * static_cast<size_t>(a.L);
  const size_t cap = kStaticAuxBytes / sizeof(double);
  if (row > 0 && row * (static_cast<size_t>(nsteps) + 1) > cap) {
    const long long most = static_cast<long long>(cap / row) - 1;
    return fail(FDTD_ERR_INVALID, "fdtd_step_static_scratch: " + std::to_string(nsteps) +
                                      " steps need " + std::to_string(row * (nsteps + 1) * sizeof(double)) +
                                      " bytes of TFSF table, more than the fixed " +
                                      std::to_string(kStaticAuxBytes) + "; this grid takes at most " +
                                      std::to_string(most < 0 ? 0 : most) + " steps per call");
  }
  if (g->dirty_pml)
    return fail(FDTD_ERR_INVALID,
                "fdtd_step_static_scratch: the CPML changed since the last fdtd_step; fdtd_prepare (or one "
                "fdtd_step) lays out its integrator slabs first");
  if (g->dirty_dft) {
    // laying out DFT regions allocates their sample buffers
    if (!g->dfts.empty())
      return fail(FDTD_ERR_INVALID,
                  "fdtd_step_static_scratch: DFT regions were added since the last fdtd_step; fdtd_prepare (or "
                  "one fdtd_step) lays out their buffers first");
    rc = rebuild_dft(g);
    if (rc) return rc;
  }
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : g->stream;
  if (!g->auxes.empty()) {
    // the TFSF step counter goes up from a host value, and the call waits
    // for that copy: neither is possible while the stream is being captured
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(s, &cs));
    if (cs != cudaStreamCaptureStatusNone)
      return fail(FDTD_ERR_UNSUPPORTED,
                  "fdtd_step_static_scratch: a grid with TFSF planes uploads its step counter and synchronises "
                  "the stream, which a stream under capture cannot do");
  }
  if (s != g->stream) CK(cudaStreamSynchronize(g->stream));  // set-up work on the grid's stream first
  // point each plane's table at its slice of the fixed array for this call
  double* saved_tab[kMaxPlanes];
  long long saved_cap[kMaxPlanes];
  const int naux = static_cast<int>(g->auxes.size());
  double* p = base;
  for (int q = 0; q < naux; q++) {
    AuxH& a = g->auxes[q];
    saved_tab[q] = a.d_tab;
    saved_cap[q] = a.cap;
    a.d_tab = p;
    a.cap = nsteps + 1;
    p += 2 * static_cast<size_t>(a.cap) * a.L;
    double* st = a.d_state;
    const int L = a.L;
    g->launches += launch_aux_precompute(L, g->d.dt, g->d.dx, st, st + L, st + 2 * L, st + 3 * L, st + 4 * L,
                                         st + 5 * L, a.d_coef, a.d_vals, static_cast<int>(a.vals.size()), g->t,
                                         nsteps, a.d_tab, a.d_tab + a.cap * L, s);
  }
  if (naux > 0) {
    Control c{};
    c.t = g->t;
    c.t0 = g->t;
    cudaError_t e = cudaMemcpyAsync(g->ctrl, &c, sizeof(long long) * 2, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // the host value must outlive the copy
    if (e != cudaSuccess) rc = fail(FDTD_ERR_CUDA, std::string("step control upload: ") + cudaGetErrorString(e));
  }
  // as in fdtd_step: pending DFT samples are folded first, so the call's
  // samples fill the ring from slot 0 on
  if (!rc && g->dft_pending > 0) g->launches += flush_dft(g, s);
  if (!rc) rc = enqueue_steps(g, nsteps, s, nullptr);
  for (int q = 0; q < naux; q++) {
    g->auxes[q].d_tab = saved_tab[q];
    g->auxes[q].cap = saved_cap[q];
  }
  if (rc) return rc;
  CK(cudaGetLastError());
  g->t += nsteps;
  return FDTD_OK;
} catch (...) {
  return host_failure();
}

// ----------------------------------------------------------------------------
// Adjoint gradient d(objective)/d(eps_r) of a 2D TM FP32 fused grid.
//
// Objective: J = sum over a probe box of |X|^2, X the running DFT of Ez at
// one frequency. Forward: the grid's own steps (graph-replayed), with a copy
// of the whole time-stepped state (E, H, CPML integrators, source history,
// step counter) every `ckpt_every` steps. Backward, per checkpoint segment
// from the last: restore the checkpoint, recompute the segment's steps with
// the same kernels (no DFT), keeping d_t of each design cell, then reverse
// the segment's steps with the adjoint kernels of kernels_adjoint.cu. At the
// end the grid is put back to its state after the forward.
namespace {

struct AdjBuf {
  std::vector<void*> allocs;
  ~AdjBuf() {
    for (void* p : allocs) cudaFree(p);
  }
};

}  // namespace

struct fdtd_adjoint {
  fdtd_grid* g = nullptr;
  int device = 0;
  int plo[2], phi[2], dlo[2], dhi[2];
  double freq = 0.0;
  int ckpt_every = 64;
  int dft = -1;
  long long nsteps = 0;
  bool forwarded = false;
  std::vector<std::pair<void*, size_t>> state;
  size_t state_bytes = 0;
  int nckpt = 0;
  AdjBuf buf;
  char* d_ckpt = nullptr;
  char* d_final = nullptr;
  float* d_ie = nullptr;
  float* adj[7] = {};   // aez, ahx, ahy, rxy, ryx, rzx, rzy
  float* apsi[4] = {};  // apzx, apzy, apxy, apyx
  size_t psi_elems[4] = {};
  float* d_store = nullptr;
  double* d_X = nullptr;
  double* d_grad = nullptr;
  double J = 0.0;
  std::map<int, cudaGraphExec_t> graphs;  // one replayable segment per length
  std::map<int, long long> graph_launches;
  ~fdtd_adjoint() {
    for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
  }
};

static int adj_alloc(fdtd_adjoint* a, void** p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, std::max<size_t>(bytes, 16));
  if (e != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    return fail(FDTD_ERR_NOMEM, std::string("adjoint buffers: ") + cudaGetErrorString(e));
  }
  a->buf.allocs.push_back(*p);
  return FDTD_OK;
}

static int adj_copy_state(fdtd_adjoint* a, char* base, bool save, cudaStream_t s) {
  size_t off = 0;
  for (auto& st : a->state) {
    char* sp = base + off;
    CK(cudaMemcpyAsync(save ? sp : st.first, save ? st.first : sp, st.second, cudaMemcpyDeviceToDevice, s));
    off += (st.second + 255) / 256 * 256;
  }
  return FDTD_OK;
}

// one time step of the forward without DFT capture: the E/H sweeps and the
// box sources of enqueue_steps, in its order (adjoint grids carry no TFSF)
static int adj_recompute_step(fdtd_grid* g, const FusedArgs& fa, cudaStream_t s) {
  const bool boxes = !g->boxes.empty();
  if (boxes) g->launches += launch_boxes(g, 0, -1, s);
  g->launches += launch_fused_e(g->d.mode, fa, s);
  if (boxes) g->launches += launch_boxes(g, 0, 0, s);
  if (boxes) g->launches += launch_boxes(g, 1, -1, s);
  g->launches += launch_fused_h(g->d.mode, fa, s);
  if (boxes) g->launches += launch_boxes(g, 1, 0, s);
  g->launches += launch_step_advance(g->ctrl, s);
  return FDTD_OK;
}

// recompute `len` steps from the restored checkpoint, keeping d_t of the
// design cells, then reverse them
static int adj_enqueue_segment(fdtd_adjoint* a, const FusedArgs& fa, const AdjArgs& aa, int len, cudaStream_t s) {
  fdtd_grid* g = a->g;
  const int nd = aa.ndesign;
  const float* hx = static_cast<const float*>(g->H[0]);
  const float* hy = static_cast<const float*>(g->H[1]);
  for (int k = 0; k < len; k++) {
    g->launches += launch_adjoint_capture(aa, hx, hy, a->d_store + static_cast<size_t>(k) * nd, s);
    int rc = adj_recompute_step(g, fa, s);
    if (rc) return rc;
  }
  for (int k = len - 1; k >= 0; k--)
    g->launches += launch_adjoint_step(aa, len - 1 - k, a->d_store + static_cast<size_t>(k) * nd, s);
  return FDTD_OK;
}

extern "C" {

int fdtd_adjoint_create(fdtd_grid* g, const int* probe_lo, const int* probe_hi, double freq, const int* design_lo,
                        const int* design_hi, int ckpt_every, fdtd_adjoint** out) try {
  if (!g || !probe_lo || !probe_hi || !design_lo || !design_hi || !out) return fail(FDTD_ERR_INVALID, "null argument");
  if (!g->f32 || g->d.mode != FDTD_TM)
    return fail(FDTD_ERR_UNSUPPORTED, "the adjoint takes 2D TM grids of the FP32 fused method");
  if (g->t != 0) return fail(FDTD_ERR_INVALID, "the adjoint starts from a grid that has not been stepped");
  if (!g->planes.empty()) return fail(FDTD_ERR_UNSUPPORTED, "the adjoint takes grids without TFSF planes");
  if (g->max_poles != 0) return fail(FDTD_ERR_UNSUPPORTED, "the adjoint takes non-dispersive materials");
  if (g->bcs.n > 0) return fail(FDTD_ERR_UNSUPPORTED, "the adjoint takes grids without boundary conditions");
  for (auto& m : g->mats)
    if (m.mu_r != 1.0) return fail(FDTD_ERR_UNSUPPORTED, "the adjoint takes mu_r = 1");
  if (ckpt_every < 1 || ckpt_every > 4096) return fail(FDTD_ERR_INVALID, "ckpt_every must be 1..4096");
  {
    const int prc = ensure_pml(g);
    if (prc) return prc;
  }
  if (!interior(g, probe_lo[0], probe_lo[1], 0) || !interior(g, probe_hi[0], probe_hi[1], 0) ||
      probe_lo[0] > probe_hi[0] || probe_lo[1] > probe_hi[1])
    return fail(FDTD_ERR_INVALID, "probe box must be a non-empty box of interior cells");
  for (int d = 0; d < 2; d++) {
    if (design_lo[d] > design_hi[d] || design_lo[d] < 1 || design_hi[d] > g->n[d] - 2)
      return fail(FDTD_ERR_INVALID, "design box must be a non-empty box of interior cells");
    for (int x = design_lo[d]; x <= design_hi[d]; x++)
      if (slab_index(g->slab[d], x) >= 0) return fail(FDTD_ERR_UNSUPPORTED, "design box must lie outside the CPML");
  }
  for (const auto& sh : g->srcs)
    if (sh.target == 1 && sh.i >= design_lo[0] && sh.i <= design_hi[0] && sh.j >= design_lo[1] &&
        sh.j <= design_hi[1])
      return fail(FDTD_ERR_UNSUPPORTED, "D-target sources inside the design box are not supported");
  CK(cudaSetDevice(g->d.device));
  const int lo3[3] = {probe_lo[0], probe_lo[1], 0}, hi3[3] = {probe_hi[0], probe_hi[1], 0};
  int handle = -1;
  int rc = fdtd_add_dft(g, 2, lo3, hi3, &freq, 1, &handle);
  if (rc) return rc;
  fdtd_adjoint* a = new fdtd_adjoint();
  a->g = g;
  a->device = g->d.device;
  for (int d = 0; d < 2; d++) {
    a->plo[d] = probe_lo[d];
    a->phi[d] = probe_hi[d];
    a->dlo[d] = design_lo[d];
    a->dhi[d] = design_hi[d];
  }
  a->freq = freq;
  a->ckpt_every = ckpt_every;
  a->dft = handle;
  *out = a;
  return FDTD_OK;
} catch (...) {
  return host_failure();
}

int fdtd_adjoint_destroy(fdtd_adjoint* a) try {
  if (!a) return FDTD_OK;
  cudaSetDevice(a->device);
  cudaDeviceSynchronize();
  delete a;
  return FDTD_OK;
} catch (...) {
  return host_failure();
}

int fdtd_adjoint_forward(fdtd_adjoint* a, int nsteps, double* J) try {
  if (!a || !J) return fail(FDTD_ERR_INVALID, "null argument");
  if (a->forwarded) return fail(FDTD_ERR_INVALID, "one forward per adjoint handle");
  if (nsteps < 1) return fail(FDTD_ERR_INVALID, "nsteps < 1");
  fdtd_grid* g = a->g;
  if (g->t != 0) return fail(FDTD_ERR_INVALID, "the grid was stepped after the adjoint was created");
  CK(cudaSetDevice(g->d.device));
  if (g->dirty_dft) {
    int rc = rebuild_dft(g);
    if (rc) return rc;
  }
  cudaStream_t s = g->stream;
  a->state = grid_state(g);
  a->state_bytes = 0;
  for (auto& st : a->state) a->state_bytes += (st.second + 255) / 256 * 256;
  a->nckpt = (nsteps + a->ckpt_every - 1) / a->ckpt_every;
  int rc = adj_alloc(a, reinterpret_cast<void**>(&a->d_ckpt), a->state_bytes * a->nckpt);
  if (!rc) rc = adj_alloc(a, reinterpret_cast<void**>(&a->d_final), a->state_bytes);
  if (rc) return rc;
  for (int q = 0; q < a->nckpt; q++) {
    rc = adj_copy_state(a, a->d_ckpt + a->state_bytes * q, true, s);
    if (!rc) rc = step_impl(g, std::min(a->ckpt_every, nsteps - q * a->ckpt_every), nullptr, nullptr);
    if (rc) return rc;
  }
  rc = adj_copy_state(a, a->d_final, true, s);
  if (rc) return rc;
  const DftH& r = g->dfts[a->dft];
  rc = adj_alloc(a, reinterpret_cast<void**>(&a->d_X), static_cast<size_t>(r.npts) * 2 * sizeof(double));
  if (rc) return rc;
  CK(cudaMemcpyAsync(a->d_X, r.d_acc, r.npts * 2 * sizeof(double), cudaMemcpyDeviceToDevice, s));
  std::vector<double> X(static_cast<size_t>(r.npts) * 2);
  CK(cudaMemcpyAsync(X.data(), r.d_acc, X.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  double sum = 0.0;
  for (long long p = 0; p < r.npts; p++) sum += X[2 * p] * X[2 * p] + X[2 * p + 1] * X[2 * p + 1];
  a->J = sum;
  a->nsteps = nsteps;
  a->forwarded = true;
  *J = sum;
  return FDTD_OK;
} catch (...) {
  return host_failure();
}

int fdtd_adjoint_backward(fdtd_adjoint* a, double* grad) try {
  if (!a || !grad) return fail(FDTD_ERR_INVALID, "null argument");
  if (!a->forwarded) return fail(FDTD_ERR_INVALID, "run fdtd_adjoint_forward first");
  fdtd_grid* g = a->g;
  if (g->t != a->nsteps) return fail(FDTD_ERR_INVALID, "the grid was stepped after the adjoint forward");
  CK(cudaSetDevice(g->d.device));
  cudaStream_t s = g->stream;
  const size_t fe = static_cast<size_t>(field_elems(g));
  const int dw = a->dhi[0] - a->dlo[0] + 1, nd = dw * (a->dhi[1] - a->dlo[1] + 1);
  int rc = FDTD_OK;
  if (!a->d_ie) {
    rc = adj_alloc(a, reinterpret_cast<void**>(&a->d_ie), fe * sizeof(float));
    for (int q = 0; q < 7 && !rc; q++) rc = adj_alloc(a, reinterpret_cast<void**>(&a->adj[q]), fe * sizeof(float));
    // adjoint CPML integrators: the compact slabs of psi_zx, psi_zy (E) and psi_yx, psi_xy (H)
    const size_t sx = static_cast<size_t>(g->n[1]) * g->slab[0].W, sy = static_cast<size_t>(g->slab[1].W) * rowlen(g);
    const size_t sizes[4] = {sx, sy, sy, sx};
    for (int q = 0; q < 4 && !rc; q++) {
      a->psi_elems[q] = sizes[q];
      rc = adj_alloc(a, reinterpret_cast<void**>(&a->apsi[q]), sizes[q] * sizeof(float));
    }
    if (!rc) rc = adj_alloc(a, reinterpret_cast<void**>(&a->d_store), static_cast<size_t>(a->ckpt_every) * nd * sizeof(float));
    if (!rc) rc = adj_alloc(a, reinterpret_cast<void**>(&a->d_grad), nd * sizeof(double));
    if (rc) return rc;
  }
  FusedArgs fa = fused_args(g);
  g->launches += launch_adjoint_inv_eps(fa, a->d_ie, s);
  for (int q = 0; q < 7; q++) CK(cudaMemsetAsync(a->adj[q], 0, fe * sizeof(float), s));
  for (int q = 0; q < 4; q++) CK(cudaMemsetAsync(a->apsi[q], 0, std::max<size_t>(a->psi_elems[q], 4) * sizeof(float), s));
  CK(cudaMemsetAsync(a->d_grad, 0, nd * sizeof(double), s));
  AdjArgs aa;
  memset(&aa, 0, sizeof(aa));
  aa.nx = g->n[0];
  aa.ny = g->n[1];
  aa.pitch = g->pitch;
  for (int ft = 0; ft < 2; ft++)
    for (int x = 0; x < 3; x++) aa.prof[ft][x] = fa.prof[ft][x];
  for (int x = 0; x < 3; x++) {
    aa.slab[x] = fa.slab[x];
    aa.pml_axis[x] = fa.pml_axis[x];
  }
  aa.ie = a->d_ie;
  aa.aez = a->adj[0];
  aa.ahx = a->adj[1];
  aa.ahy = a->adj[2];
  aa.rxy = a->adj[3];
  aa.ryx = a->adj[4];
  aa.rzx = a->adj[5];
  aa.rzy = a->adj[6];
  aa.apzx = a->apsi[0];
  aa.apzy = a->apsi[1];
  aa.apxy = a->apsi[2];
  aa.apyx = a->apsi[3];
  for (int d = 0; d < 2; d++) {
    aa.plo[d] = a->plo[d];
    aa.phi[d] = a->phi[d];
    aa.dlo[d] = a->dlo[d];
    aa.dhi[d] = a->dhi[d];
  }
  aa.X = a->d_X;
  aa.freq = a->freq;
  aa.ndesign = nd;
  aa.grad = a->d_grad;
  aa.ctrl = g->ctrl;
  // every segment of one length is the same launch sequence (the kernels read
  // the step from the device counter the checkpoint restores): one captured
  // graph per length, replayed; without graphs the launches go out one by one
  for (int q = a->nckpt - 1; q >= 0 && !rc; q--) {
    const long long t0 = static_cast<long long>(q) * a->ckpt_every;
    const int len = static_cast<int>(std::min<long long>(a->ckpt_every, a->nsteps - t0));
    rc = adj_copy_state(a, a->d_ckpt + a->state_bytes * q, false, s);
    if (rc) break;
    if (!g->use_graphs) {
      rc = adj_enqueue_segment(a, fa, aa, len, s);
      continue;
    }
    auto it = a->graphs.find(len);
    if (it == a->graphs.end()) {
      const long long before = g->launches;
      CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      rc = adj_enqueue_segment(a, fa, aa, len, s);
      cudaGraph_t graph = nullptr;
      cudaError_t e = cudaStreamEndCapture(s, &graph);
      a->graph_launches[len] = g->launches - before;
      g->launches = before;
      if (rc) return rc;
      if (e != cudaSuccess) return fail(FDTD_ERR_CUDA, std::string("adjoint capture: ") + cudaGetErrorString(e));
      cudaGraphExec_t exec = nullptr;
      e = cudaGraphInstantiate(&exec, graph, 0);
      cudaGraphDestroy(graph);
      if (e != cudaSuccess) return fail(FDTD_ERR_CUDA, std::string("adjoint instantiate: ") + cudaGetErrorString(e));
      it = a->graphs.emplace(len, exec).first;
    }
    CK(cudaGraphLaunch(it->second, s));
    g->launches += a->graph_launches[len];
  }
  // the grid goes back to its state after the forward
  if (!rc) rc = adj_copy_state(a, a->d_final, false, s);
  if (rc) return rc;
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(grad, a->d_grad, nd * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return FDTD_OK;
} catch (...) {
  return host_failure();
}

}  // extern "C"
