// fdtd_b200.hpp: pederson/fdtd's functor names over the fdtd_b200 C ABI.
//
// In the reference a user applies update functors to a container of cells,
// once per pass of a time loop (tests/testTM.cpp:102-113). Here the same
// functor types are handed to a gpu::Grid once, as the plan of one step; the
// grid checks the plan against the fused schedule and then runs any number of
// steps on the GPU:
//
//   gpu::Grid<TM, double> grid(256, 256, 1, dx, dt, 2000);
//   grid.set_pml(Dir::X, 16); grid.set_pml(Dir::Y, 16);
//   auto src = grid.add(make_soft_source<Ez>(signal, grid.cell(128, 128)));
//   grid.plan({YeeUpdate<TM, Dz>(dt, dx),
//              UpdatePML<TM, FieldType::Electric, Dir::X>(dt, dx), ...,
//              VacuumUpdate<TM, FieldType::Electric>(), src, ...});
//   grid.step(2000);
//
// Header-only; link with libfdtd_b200.so. Errors throw fdtd::gpu::Error
// carrying the C status and message.
#pragma once

#include <array>
#include <cctype>
#include <map>
#include <cmath>
#include <complex>
#include <cstdint>
#include <algorithm>
#include <functional>
#include <initializer_list>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "fdtd_b200.h"

namespace fdtd {

// ------------------------------------------------------------ vocabulary
// Modes, field types, directions and field tags as in
// include/FDTDConstants.hpp:410-445, :457-486, :648-744.
struct EMMode {};
struct TEM : EMMode { static constexpr int value = FDTD_TEM, dim = 1; };
struct TE : EMMode { static constexpr int value = FDTD_TE, dim = 2; };
struct TM : EMMode { static constexpr int value = FDTD_TM, dim = 2; };
struct ThreeD : EMMode { static constexpr int value = FDTD_THREED, dim = 3; };

enum class FieldType : char { Electric = 0, Magnetic, NONE };
enum class Dir : char { X = 0, Y, Z, NONE };
enum class Orientation : char { MIN = 0, MAX, NONE };

namespace detail {
template <int Which, FieldType FT, int Comp, bool Flux>
struct FieldTag {
  static constexpr int which = Which;      // fdtd_download selector
  static constexpr FieldType field_type = FT;
  static constexpr int comp = Comp;        // 0..2 = x, y, z
  static constexpr bool flux = Flux;       // D/B (true) or E/H
};
}  // namespace detail
struct Ex : detail::FieldTag<FDTD_EX, FieldType::Electric, 0, false> {};
struct Ey : detail::FieldTag<FDTD_EY, FieldType::Electric, 1, false> {};
struct Ez : detail::FieldTag<FDTD_EZ, FieldType::Electric, 2, false> {};
struct Dx : detail::FieldTag<FDTD_DX, FieldType::Electric, 0, true> {};
struct Dy : detail::FieldTag<FDTD_DY, FieldType::Electric, 1, true> {};
struct Dz : detail::FieldTag<FDTD_DZ, FieldType::Electric, 2, true> {};
struct Hx : detail::FieldTag<FDTD_HX, FieldType::Magnetic, 0, false> {};
struct Hy : detail::FieldTag<FDTD_HY, FieldType::Magnetic, 1, false> {};
struct Hz : detail::FieldTag<FDTD_HZ, FieldType::Magnetic, 2, false> {};
struct Bx : detail::FieldTag<FDTD_BX, FieldType::Magnetic, 0, true> {};
struct By : detail::FieldTag<FDTD_BY, FieldType::Magnetic, 1, true> {};
struct Bz : detail::FieldTag<FDTD_BZ, FieldType::Magnetic, 2, true> {};

// include/FDTDConstants.hpp:394-398 (imp0 with the reference's Newton sqrt)
constexpr double pi = 3.14159265358979323846264338327950288;
constexpr double eps0 = 8.854e-12;
constexpr double mu0 = pi * 4.0e-7;
constexpr double c0 = 2.99792458e+8;
namespace detail {
constexpr double newton_sqrt(double x, double curr, double prev) {
  return curr == prev ? curr : newton_sqrt(x, 0.5 * (curr + x / curr), curr);
}
}  // namespace detail
constexpr double imp0 = detail::newton_sqrt(mu0 / eps0, mu0 / eps0, 0);

template <class Mode>
constexpr bool has_component(FieldType ft, int c) {
  return Mode::value == FDTD_THREED ||
         (ft == FieldType::Electric ? ((Mode::value == FDTD_TE && c < 2) || (Mode::value == FDTD_TM && c == 2))
                                    : ((Mode::value == FDTD_TE && c == 2) || (Mode::value == FDTD_TM && c < 2)));
}

// ------------------------------------------------------------ signals
// SinData / RickerData (include/Source.hpp:100-167)
struct Sinusoid {
  double freq, phase, delay;
  explicit Sinusoid(double f, double ph = 0) : freq(f), phase(ph), delay(10.0 / f * pi / 2.0) {}
  double operator()(double t) const { return std::tanh(t / delay) * std::sin(freq * t + phase); }
};
struct Ricker {
  double freq, delay;
  explicit Ricker(double f) : freq(f), delay(2.0 / f) {}
  double operator()(double t) const {
    const double p = pi * freq * (t - delay);
    return (1.0 - 2.0 * p * p) * std::exp(-p * p);
  }
};

// ------------------------------------------------------------ plan ops
namespace detail {
enum class OpKind { Yee, Pml, Material, Source, TfsfD, TfsfB, BoundaryE, BoundaryH };
struct Op {
  OpKind kind;
  FieldType ft = FieldType::NONE;
  int comp = -1, axis = -1;
  fdtd_material mat{};
  int source = -1, plane = -1;
  int scheme = FDTD_BD1;
};
inline fdtd_material blank_material(int kind) {
  fdtd_material m{};
  m.kind = kind;
  m.eps_inf = 1.0;
  m.mu_r = 1.0;
  return m;
}
}  // namespace detail

// Time policies of the curl update (include/YeeUpdates.hpp:182-294). The
// TFSF corrections of a grid follow the policy of its YeeUpdates, as a
// TFSFPlane<..., TimePolicy> built with the same policy does.
struct TemporalScheme {};
struct BD1 : TemporalScheme { static constexpr int value = FDTD_BD1; };
struct BD3 : TemporalScheme { static constexpr int value = FDTD_BD3; };
struct BD4 : TemporalScheme { static constexpr int value = FDTD_BD4; };

// YeeUpdate<Mode, Flux, TimePolicy> (include/YeeUpdates.hpp:343-405); BD3
// and BD4 on FP64 grids only
template <class Mode, class Flux, class TimePolicy = BD1>
struct YeeUpdate {
  static_assert(Flux::flux, "YeeUpdate acts on a flux component (D or B)");
  static_assert(std::is_base_of<TemporalScheme, TimePolicy>::value, "YeeUpdate needs a valid TemporalScheme");
  double dt, dx;
  YeeUpdate(double deltat, double deltax) : dt(deltat), dx(deltax) {}
  operator detail::Op() const {
    detail::Op o{detail::OpKind::Yee};
    o.ft = Flux::field_type;
    o.comp = Flux::comp;
    o.scheme = TimePolicy::value;
    return o;
  }
};

// UpdatePML<Mode, FieldType, Dir> (include/PML.hpp:296-355)
template <class Mode, FieldType ft, Dir d>
struct UpdatePML {
  double dt, dx;
  UpdatePML(double deltat, double deltax) : dt(deltat), dx(deltax) {}
  operator detail::Op() const {
    detail::Op o{detail::OpKind::Pml};
    o.ft = ft;
    o.axis = static_cast<int>(d);
    return o;
  }
};

// Material updates (include/DispersiveMaterials.hpp:489-497, :881-884, :1208-1211)
template <class Mode, FieldType ft, bool forward = false>
struct VacuumUpdate {
  static_assert(!forward, "a plan takes the implicit updates; Grid::apply_forward_materials runs the forward ones");
  operator detail::Op() const {
    detail::Op o{detail::OpKind::Material};
    o.ft = ft;
    o.mat = detail::blank_material(FDTD_VACUUM);
    return o;
  }
};
template <class Mode, FieldType ft, bool forward = false>
struct ConstantUpdate {
  static_assert(!forward, "a plan takes the implicit updates; Grid::apply_forward_materials runs the forward ones");
  double K;
  explicit ConstantUpdate(double k) : K(k) {}
  operator detail::Op() const {
    detail::Op o{detail::OpKind::Material};
    o.ft = ft;
    o.mat = detail::blank_material(FDTD_CONSTANT);
    if (ft == FieldType::Electric) o.mat.eps_inf = K;
    else o.mat.mu_r = K;
    return o;
  }
};
template <class Mode, FieldType ft, bool forward = false>
struct DrudeUpdate {
  static_assert(ft == FieldType::Electric && !forward,
                "Drude acts on the electric field, implicitly in a plan (Grid::apply_forward_materials runs the forward one)");
  double K, Freq, Gamma;
  DrudeUpdate(double k, double freq, double gamma, double /*dt*/ = 0) : K(k), Freq(freq), Gamma(gamma) {}
  operator detail::Op() const {
    detail::Op o{detail::OpKind::Material};
    o.ft = ft;
    o.mat = detail::blank_material(FDTD_DRUDE);
    o.mat.eps_inf = K;
    o.mat.npoles = 1;
    o.mat.delta_eps[0] = 1.0;
    o.mat.freq[0] = Freq;
    o.mat.gamma[0] = Gamma;
    return o;
  }
};
// The reference ignores Delta (include/DispersiveMaterials.hpp:710-735); so does
// this functor. LorentzPoles below takes per-pole strengths.
template <class Mode, FieldType ft, bool forward = false>
struct LorentzUpdate {
  static_assert(ft == FieldType::Electric && !forward, "Lorentz acts on the electric field, implicitly");
  double K, Delta, Freq, Gamma;
  LorentzUpdate(double k, double delta, double freq, double gamma, double /*dt*/ = 0)
      : K(k), Delta(delta), Freq(freq), Gamma(gamma) {}
  operator detail::Op() const {
    detail::Op o{detail::OpKind::Material};
    o.ft = ft;
    o.mat = detail::blank_material(FDTD_LORENTZ);
    o.mat.eps_inf = K;
    o.mat.npoles = 1;
    o.mat.delta_eps[0] = 1.0;
    o.mat.freq[0] = Freq;
    o.mat.gamma[0] = Gamma;
    return o;
  }
};
// Multi-pole Lorentz (an extension): E = (D - sum P_q)/(eps_inf eps0),
// J_q' = a_q J_q + b_q (delta_q eps0 E - P_q).
struct LorentzPoles {
  double eps_inf;
  std::vector<std::array<double, 3>> poles;  // (delta_eps, freq, gamma)
  operator detail::Op() const {
    detail::Op o{detail::OpKind::Material};
    o.ft = FieldType::Electric;
    o.mat = detail::blank_material(FDTD_LORENTZ);
    o.mat.eps_inf = eps_inf;
    o.mat.npoles = static_cast<int>(poles.size());
    for (size_t q = 0; q < poles.size() && q < FDTD_MAX_POLES; q++) {
      o.mat.delta_eps[q] = poles[q][0];
      o.mat.freq[q] = poles[q][1];
      o.mat.gamma[q] = poles[q][2];
    }
    return o;
  }
};

// PMLParameterModel (include/PML.hpp:368-393): the grading the GPU applies.
struct PMLParameterModel {
  double mM, mMa, msMax, mkMax, maMax;
  explicit PMLParameterModel(double dx) : mM(3), mMa(1), msMax(0.8 * (3 + 1) / (imp0 * dx)), mkMax(5), maMax(0.05) {}
  PMLParameterModel(double m, double ma, double sMax, double kMax, double aMax)
      : mM(m), mMa(ma), msMax(sMax), mkMax(kMax), maMax(aMax) {}
  double K(double x) const { return x < 0.0 ? 1.0 : (x > 1.0 ? 1.0 : 1.0 + std::pow(x, mM) * (mkMax - 1.0)); }
  double S(double x) const { return x < 0.0 ? 0.0 : (x > 1.0 ? 0.0 : std::pow(x, mM) * msMax); }
  double A(double x) const { return x < 0.0 ? 0.0 : (x > 1.0 ? 0.0 : std::pow(1.0 - x, mMa) * maMax); }
};

namespace gpu {

class Error : public std::runtime_error {
 public:
  Error(int code, const std::string& msg) : std::runtime_error(msg), code(code) {}
  int code;
};
inline void check(int rc) {
  if (rc != FDTD_OK) throw Error(rc, fdtd_last_error_string());
}

struct CellRef {
  int i, j, k;
};

}  // namespace gpu

// SoftSource<Signal, Cell, GetField<F>> (include/Source.hpp:183-261):
// the signal is evaluated at t = n*dt for step n.
struct SoftSourceSpec {
  int comp, target;
  gpu::CellRef cell;
  std::function<double(double)> signal;
  int index = -1;
  operator detail::Op() const {
    detail::Op o{detail::OpKind::Source};
    o.ft = FieldType::Electric;
    o.comp = comp;
    o.source = index;
    o.axis = target;
    return o;
  }
};
template <class F, class Signal>
SoftSourceSpec make_soft_source(Signal sig, gpu::CellRef c) {
  static_assert(F::field_type == FieldType::Electric, "soft sources act on E or D");
  return SoftSourceSpec{F::comp, F::flux ? 1 : 0, c, std::function<double(double)>(sig)};
}

// Aux1D (include/Source.hpp:280-462): the source is evaluated at the
// accumulated aux time t_s = t_{s-1} + dt, as Aux1D::time_step does.
template <typename scalar = double>
struct Aux1D {
  int ncells;
  double dx, dt;
  std::function<double(double)> signal;
  template <class Signal>
  Aux1D(int n, double deltax, double deltat, Signal sig) : ncells(n), dx(deltax), dt(deltat), signal(sig) {}
  std::vector<double> table(int nsteps) const {
    std::vector<double> v(nsteps);
    double t = 0;
    for (int s = 0; s < nsteps; s++) {
      t += dt;
      v[s] = signal(t);
    }
    return v;
  }
};

// TFSFPlane (include/Source.hpp:472-634): cells lo..hi, normal along dd with
// orientation o, location functor ((i,j,k) - origin) * dx. The polarisation
// defaults to the reference's for TE/TM; pass it for ThreeD (where the
// reference leaves it unset) or to override.
struct TFSFPlaneSpec {
  int axis, orient;
  std::array<int, 3> lo, hi;
  std::array<double, 3> origin, k, pol_e, pol_h;
  std::shared_ptr<Aux1D<double>> aux;
  int index = -1;
  struct D {
    int index;
    operator detail::Op() const {
      detail::Op o{detail::OpKind::TfsfD};
      o.plane = index;
      return o;
    }
  };
  struct B {
    int index;
    operator detail::Op() const {
      detail::Op o{detail::OpKind::TfsfB};
      o.plane = index;
      return o;
    }
  };
};
template <class Mode, Dir dd, Orientation o>
TFSFPlaneSpec make_tfsf_plane(std::array<int, 3> lo, std::array<int, 3> hi, std::array<double, 3> origin,
                              std::array<double, 3> k, std::shared_ptr<Aux1D<double>> aux,
                              const std::array<double, 3>* pol_e = nullptr, const std::array<double, 3>* pol_h = nullptr) {
  TFSFPlaneSpec p;
  p.axis = static_cast<int>(dd);
  p.orient = o == Orientation::MAX ? 1 : 0;
  p.lo = lo;
  p.hi = hi;
  p.origin = origin;
  p.k = k;
  p.aux = aux;
  double K = 0;
  for (int d = 0; d < Mode::dim; d++) K += k[d] * k[d];
  K = std::sqrt(K);
  std::array<double, 3> kn{0, 0, 0};
  for (int d = 0; d < Mode::dim; d++) kn[d] = k[d] / K;
  if (Mode::value == FDTD_TE) {  // Source.hpp:573-576
    p.pol_h = {0, 0, 1};
    p.pol_e = {kn[1], -kn[0], 0};
  } else {  // TM and TEM (Source.hpp:577-584); ThreeD: E along z, H along the aux Hy
    p.pol_e = {0, 0, 1};
    p.pol_h = Mode::value == FDTD_TM ? std::array<double, 3>{kn[1], -kn[0], 0} : std::array<double, 3>{0, 1, 0};
  }
  if (pol_e) p.pol_e = *pol_e;
  if (pol_h) p.pol_h = *pol_h;
  return p;
}

// make_pec_boundary / make_pmc_boundary / make_symmetric_boundary /
// make_antisymmetric_boundary / make_periodic_boundary<Mode, d, o>
// (include/BoundaryUpdates.hpp:529-830) over the interior cells next to the
// face (d, o); the periodic partner is the interior cell at the far end of
// the axis. Added to a grid, the spec gives the plan ops of updateE() (after
// the E sources) and updateH() (after the magnetic material update).
struct BoundarySpec {
  int axis, side, kind;
  int index = -1;
  struct E {
    int index;
    operator detail::Op() const {
      detail::Op o{detail::OpKind::BoundaryE};
      o.plane = index;
      return o;
    }
  };
  struct H {
    int index;
    operator detail::Op() const {
      detail::Op o{detail::OpKind::BoundaryH};
      o.plane = index;
      return o;
    }
  };
  E updateE() const { return E{index}; }
  H updateH() const { return H{index}; }
};
template <class Mode, Dir d, Orientation o>
BoundarySpec make_pec_boundary() { return {static_cast<int>(d), o == Orientation::MAX ? 1 : 0, FDTD_BC_PEC}; }
template <class Mode, Dir d, Orientation o>
BoundarySpec make_pmc_boundary() { return {static_cast<int>(d), o == Orientation::MAX ? 1 : 0, FDTD_BC_PMC}; }
template <class Mode, Dir d, Orientation o>
BoundarySpec make_symmetric_boundary() {
  return {static_cast<int>(d), o == Orientation::MAX ? 1 : 0, FDTD_BC_SYMMETRIC};
}
template <class Mode, Dir d, Orientation o>
BoundarySpec make_antisymmetric_boundary() {
  return {static_cast<int>(d), o == Orientation::MAX ? 1 : 0, FDTD_BC_ANTISYMMETRIC};
}
template <class Mode, Dir d, Orientation o>
BoundarySpec make_periodic_boundary() {
  return {static_cast<int>(d), o == Orientation::MAX ? 1 : 0, FDTD_BC_PERIODIC};
}

namespace gpu {

// A grid of Mode on one GPU; Real = double for the FP64 plain method, float
// for the FP32 fused method. max_steps bounds the steps for which source
// signals are tabulated.
template <class Mode, class Real>
class Grid {
  static_assert(Mode::value != FDTD_TEM, "the GPU grid holds TE, TM or ThreeD");

 public:
  Grid(int nx, int ny, int nz, double dx, double dt, int max_steps, int device = 0)
      : dx_(dx), dt_(dt), max_steps_(max_steps) {
    fdtd_grid_desc d{Mode::value, std::is_same<Real, double>::value ? FDTD_PLAIN_F64 : FDTD_FUSED_F32,
                     nx, ny, nz, dx, dt, device};
    fdtd_grid* g = nullptr;
    check(fdtd_grid_create(&d, &g));
    g_.reset(g);
    n_ = {nx, ny, nz};
  }

  CellRef cell(int i, int j, int k = 0) const { return CellRef{i, j, k}; }
  fdtd_grid* handle() const { return g_.get(); }

  // CPML of n cells on one side, or on both sides, of an axis
  void set_pml(Dir d, Orientation o, int n) {
    check(fdtd_set_pml(g_.get(), static_cast<int>(d), o == Orientation::MAX ? 1 : 0, n));
    pml_axes_[static_cast<int>(d)] = true;
  }
  void set_pml(Dir d, int n) {
    set_pml(d, Orientation::MIN, n);
    set_pml(d, Orientation::MAX, n);
  }
  // the same, graded with a PMLParameterModel of the caller's parameters
  // (the loop of tests/testTM.cpp:44-71 with another model)
  void set_pml(Dir d, Orientation o, int n, const PMLParameterModel& m) {
    check(fdtd_set_pml_model(g_.get(), static_cast<int>(d), o == Orientation::MAX ? 1 : 0, n, m.mM, m.mMa, m.msMax,
                             m.mkMax, m.maMax));
    pml_axes_[static_cast<int>(d)] = true;
  }

  // A per-cell material map: ids index `mats` (the role of MaterialMap,
  // include/MaterialMap.hpp:204-284). The plan's material op must then be
  // MaterialMapUpdate.
  // the same from C-ABI material rows (e.g. xml::read_material_map's values)
  void set_material_map(const std::vector<fdtd_material>& mats, const std::vector<uint8_t>& ids) {
    check(fdtd_set_materials(g_.get(), mats.data(), static_cast<int>(mats.size())));
    check(fdtd_set_material_ids(g_.get(), ids.data()));
    has_map_ = true;
  }
  void set_material_map(const std::vector<detail::Op>& mats, const std::vector<uint8_t>& ids) {
    std::vector<fdtd_material> m;
    for (auto& o : mats) m.push_back(o.mat);
    check(fdtd_set_materials(g_.get(), m.data(), static_cast<int>(m.size())));
    check(fdtd_set_material_ids(g_.get(), ids.data()));
    has_map_ = true;
  }

  SoftSourceSpec add(SoftSourceSpec s) {
    std::vector<double> v(max_steps_);
    for (int n = 0; n < max_steps_; n++) v[n] = s.signal(n * dt_);
    check(fdtd_add_source(g_.get(), s.comp, s.target, s.cell.i, s.cell.j, s.cell.k, v.data(), max_steps_));
    s.index = nsrc_++;
    return s;
  }
  BoundarySpec add(BoundarySpec b) {
    check(fdtd_set_boundary(g_.get(), b.axis, b.side, b.kind));
    b.index = nbc_++;
    return b;
  }
  TFSFPlaneSpec add(TFSFPlaneSpec p) {
    const std::vector<double> v = p.aux->table(max_steps_ + 1);
    check(fdtd_add_tfsf_plane(g_.get(), p.axis, p.orient, p.lo.data(), p.hi.data(), p.origin.data(), p.k.data(),
                              p.pol_e.data(), p.pol_h.data(), p.aux->ncells, v.data(), static_cast<int>(v.size())));
    p.index = nplanes_++;
    return p;
  }

  // The plan of one step, checked against the fused schedule.
  void plan(std::initializer_list<detail::Op> ops) {
    plan_.assign(ops.begin(), ops.end());
    validate();
  }

  void step(int n) {
    if (!validated_) throw Error(FDTD_ERR_INVALID, "no plan: call plan() first");
    if (steps_ + n > max_steps_) throw Error(FDTD_ERR_INVALID, "more steps than the grid was created for");
    check(fdtd_step(g_.get(), n, nullptr));
    steps_ += n;
  }

  // The forward (explicit) material updates, XUpdate<Mode, ft, forward = true>
  // (include/DispersiveMaterials.hpp:345-349, :922-934), of the grid's
  // material table on every interior cell: D (and the Drude P, J) from E, or
  // B from H. FP64 grids; no Lorentz material for FieldType::Electric.
  void apply_forward_materials(FieldType ft) {
    check(fdtd_material_explicit(g_.get(), static_cast<int>(ft), nullptr));
  }

  template <class F>
  std::vector<double> get() const {
    std::vector<double> v(static_cast<size_t>(n_[0]) * n_[1] * n_[2]);
    check(fdtd_download(g_.get(), F::which, v.data()));
    return v;
  }

  // A quantity (FDTD_Q_*) on the cells lo..hi, x fastest: a field, or what
  // UpdateSurfaceCurrentE / UpdateSurfaceCurrentH / UpdateSurfaceChargeDensity
  // (include/SurfaceQuantities.hpp:203-356) would leave in those cells now.
  std::vector<double> read(int quantity, std::array<int, 3> lo, std::array<int, 3> hi) const {
    size_t n = 1;
    for (int d = 0; d < 3; d++) n *= static_cast<size_t>(std::max(0, hi[d] - lo[d] + 1));
    std::vector<double> v(n);
    check(fdtd_read_quantity(g_.get(), quantity, lo.data(), hi.data(), v.data()));
    return v;
  }

  // Running DFT of a quantity (FDTD_Q_*) over lo..hi at freqs (cycles per
  // step), from the next step on; the reference's DataCapture has no Fourier
  // capture. dft(handle) returns [nf][points].
  int add_dft(int quantity, std::array<int, 3> lo, std::array<int, 3> hi, const std::vector<double>& freqs) {
    int h = -1;
    check(fdtd_add_dft(g_.get(), quantity, lo.data(), hi.data(), freqs.data(), static_cast<int>(freqs.size()), &h));
    dft_nf_.push_back(static_cast<int>(freqs.size()));
    return h;
  }
  std::vector<std::complex<double>> dft(int handle) const {
    long long np = 0;
    check(fdtd_dft_npoints(g_.get(), handle, &np));
    std::vector<double> raw(static_cast<size_t>(dft_nf_.at(handle)) * np * 2);
    check(fdtd_dft_read(g_.get(), handle, raw.data()));
    std::vector<std::complex<double>> out(raw.size() / 2);
    for (size_t q = 0; q < out.size(); q++) out[q] = {raw[2 * q], raw[2 * q + 1]};
    return out;
  }

 private:
  struct Deleter {
    void operator()(fdtd_grid* g) const { fdtd_grid_destroy(g); }
  };

  // E half: Yee on every E flux, TFSF D, D-target sources, CPML E per axis
  // in X, Y, Z order, material E, E-target sources, boundary updateE; H half:
  // Yee on every B flux, TFSF B, CPML H, material H, boundary updateH
  // (tests/testTM.cpp:102-113). Every YeeUpdate takes one time policy.
  void validate() {
    size_t q = 0;
    auto fail = [](const std::string& m) { throw Error(FDTD_ERR_UNSUPPORTED, "plan: " + m); };
    int scheme = -1;
    for (int half = 0; half < 2; half++) {
      const FieldType ft = half == 0 ? FieldType::Electric : FieldType::Magnetic;
      bool seen[3] = {false, false, false};
      while (q < plan_.size() && plan_[q].kind == detail::OpKind::Yee && plan_[q].ft == ft) {
        if (seen[plan_[q].comp]) fail("a YeeUpdate appears twice");
        if (scheme >= 0 && plan_[q].scheme != scheme) fail("every YeeUpdate must take the same time policy");
        scheme = plan_[q].scheme;
        seen[plan_[q].comp] = true;
        q++;
      }
      for (int c = 0; c < 3; c++)
        if (has_component<Mode>(ft, c) != seen[c]) fail("YeeUpdate must cover exactly the mode's flux components");
      const detail::OpKind tf = half == 0 ? detail::OpKind::TfsfD : detail::OpKind::TfsfB;
      int planes = 0;
      while (q < plan_.size() && plan_[q].kind == tf) {
        planes++;
        q++;
      }
      if (planes != 0 && planes != nplanes_) fail("every TFSF plane must be updated");
      if (half == 0)
        while (q < plan_.size() && plan_[q].kind == detail::OpKind::Source && plan_[q].axis == 1) q++;
      int last_axis = -1;
      bool axes[3] = {false, false, false};
      while (q < plan_.size() && plan_[q].kind == detail::OpKind::Pml && plan_[q].ft == ft) {
        if (plan_[q].axis <= last_axis) fail("UpdatePML axes must come in X, Y, Z order");
        last_axis = plan_[q].axis;
        axes[last_axis] = true;
        q++;
      }
      for (int a = 0; a < 3; a++)
        if (axes[a] != pml_axes_[a]) fail("UpdatePML must cover exactly the axes with CPML");
      if (q >= plan_.size() || plan_[q].kind != detail::OpKind::Material || plan_[q].ft != ft)
        fail("a material update of the half step is missing");
      if (half == 0) mat_e_ = plan_[q].mat;
      else mat_h_ = plan_[q].mat;
      q++;
      if (half == 0)
        while (q < plan_.size() && plan_[q].kind == detail::OpKind::Source && plan_[q].axis == 0) q++;
      const detail::OpKind bk = half == 0 ? detail::OpKind::BoundaryE : detail::OpKind::BoundaryH;
      int nb = 0;
      while (q < plan_.size() && plan_[q].kind == bk) {
        nb++;
        q++;
      }
      if (nb != nbc_) fail("every boundary must be updated once in each half step");
    }
    if (q != plan_.size()) fail("operations after the magnetic boundary updates");
    if (scheme != scheme_) {
      check(fdtd_set_time_scheme(g_.get(), scheme));
      scheme_ = scheme;
    }
    if (!has_map_) {
      fdtd_material m = mat_e_;
      m.mu_r = mat_h_.mu_r;
      check(fdtd_set_materials(g_.get(), &m, 1));
    }
    validated_ = true;
  }

  std::unique_ptr<fdtd_grid, Deleter> g_;
  std::array<int, 3> n_{};
  double dx_, dt_;
  int max_steps_, steps_ = 0, nsrc_ = 0, nplanes_ = 0, nbc_ = 0, scheme_ = FDTD_BD1;
  bool pml_axes_[3] = {false, false, false};
  bool has_map_ = false, validated_ = false;
  std::vector<detail::Op> plan_;
  std::vector<int> dft_nf_;
  fdtd_material mat_e_{}, mat_h_{};
};

// The material op of a plan whose grid carries a per-cell material map.
struct MaterialMapUpdate {
  FieldType ft;
  operator detail::Op() const {
    detail::Op o{detail::OpKind::Material};
    o.ft = ft;
    o.mat = detail::blank_material(FDTD_VACUUM);
    return o;
  }
};

}  // namespace gpu

// ------------------------------------------------------------ configuration files
// Readers of the reference's XML configuration: MaterialMap::readXML
// (include/MaterialMap.hpp:236-282) with MaterialPair::readXML (:134-181) and
// the storages' readXML (DispersiveMaterials.hpp:411-427, :466-471,
// :822-865, :1117-1147); PMLOptions::readXML (PML.hpp:215-281);
// BoundaryOptions::readXML (BoundaryUpdates.hpp:163-223). The reference reads
// them with tinyxml2; this is a small element-tree parser of its own (tags
// and text; declarations, comments and attributes are skipped). Unknown
// names throw, as MapNameTo does (FDTDConstants.hpp:107-124); dispersions and
// boundaries the GPU path does not implement throw Error(FDTD_ERR_UNSUPPORTED).
namespace xml {

struct Node {
  std::string tag, text;
  std::vector<Node> kids;
  const Node* child(const std::string& t) const {
    for (auto& k : kids)
      if (k.tag == t) return &k;
    return nullptr;
  }
};

namespace detail {
inline void skip_ws(const std::string& s, size_t& p) {
  while (p < s.size() && std::isspace(static_cast<unsigned char>(s[p]))) p++;
}
inline std::string trim(const std::string& t) {
  size_t a = 0, b = t.size();
  while (a < b && std::isspace(static_cast<unsigned char>(t[a]))) a++;
  while (b > a && std::isspace(static_cast<unsigned char>(t[b - 1]))) b--;
  return t.substr(a, b - a);
}
inline void skip_misc(const std::string& s, size_t& p) {
  for (;;) {
    skip_ws(s, p);
    if (s.compare(p, 4, "<!--") == 0) {
      const size_t e = s.find("-->", p);
      p = e == std::string::npos ? s.size() : e + 3;
    } else if (s.compare(p, 2, "<?") == 0) {
      const size_t e = s.find("?>", p);
      p = e == std::string::npos ? s.size() : e + 2;
    } else {
      return;
    }
  }
}
inline Node parse_element(const std::string& s, size_t& p) {
  if (p >= s.size() || s[p] != '<') throw std::runtime_error("xml: element expected");
  const size_t e = s.find('>', p);
  if (e == std::string::npos) throw std::runtime_error("xml: unterminated tag");
  std::string head = s.substr(p + 1, e - p - 1);
  p = e + 1;
  const bool empty = !head.empty() && head.back() == '/';
  if (empty) head.pop_back();
  Node n;
  n.tag = head.substr(0, head.find_first_of(" \t\r\n"));
  if (empty) return n;
  for (;;) {
    const size_t lt = s.find('<', p);
    if (lt == std::string::npos) throw std::runtime_error("xml: unterminated element " + n.tag);
    n.text += s.substr(p, lt - p);
    p = lt;
    if (s.compare(p, 4, "<!--") == 0 || s.compare(p, 2, "<?") == 0) {
      skip_misc(s, p);
      continue;
    }
    if (s.compare(p, 2, "</") == 0) {
      const size_t ce = s.find('>', p);
      if (ce == std::string::npos || trim(s.substr(p + 2, ce - p - 2)) != n.tag)
        throw std::runtime_error("xml: mismatched closing tag for " + n.tag);
      p = ce + 1;
      n.text = trim(n.text);
      return n;
    }
    n.kids.push_back(parse_element(s, p));
  }
}
inline double number(const Node* n) {
  if (!n) throw std::runtime_error("xml: value missing");
  return std::stod(n->text);
}
}  // namespace detail

// the document element of an XML text
inline Node parse(const std::string& text) {
  size_t p = 0;
  detail::skip_misc(text, p);
  return detail::parse_element(text, p);
}

// One material of a map: the C-ABI row (kind, eps_inf, mu_r, poles). Electric
// Vacuum/Constant/Drude/Lorentz and magnetic Vacuum/Constant are supported;
// a Lorentz <Delta> is read but, as in the reference's update, not used.
inline fdtd_material material_pair(const Node& pair) {
  const Node* el = pair.child("Electric");
  const Node* mg = pair.child("Magnetic");
  if (!el || !mg || el->kids.empty() || mg->kids.empty())
    throw std::runtime_error("xml: a MaterialPair needs <Electric> and <Magnetic>");
  static const char* known[] = {"Vacuum", "Constant", "Conductive", "Drude", "FluidDrude", "Lorentz",
                                "MagnetizedDrude", "SelfMagnetizedDrude", "MagnetizedFluidDrude",
                                "SelfMagnetizedFluidDrude", "MultiCoefficient", "Anisotropic"};
  auto check_name = [&](const std::string& t) {
    for (auto* k : known)
      if (t == k) return;
    throw std::runtime_error("xml: unknown dispersion " + t);
  };
  const Node& e = el->kids[0];
  const Node& m = mg->kids[0];
  check_name(e.tag);
  check_name(m.tag);
  fdtd_material r = ::fdtd::detail::blank_material(FDTD_VACUUM);
  if (m.tag == "Constant") r.mu_r = detail::number(m.child("Constant"));
  else if (m.tag != "Vacuum")
    throw gpu::Error(FDTD_ERR_UNSUPPORTED, "magnetic dispersion " + m.tag + " is not implemented on the GPU path");
  if (e.tag == "Vacuum") return r;
  r.eps_inf = detail::number(e.child("Constant"));
  if (e.tag == "Constant") {
    r.kind = FDTD_CONSTANT;
  } else if (e.tag == "Drude" || e.tag == "Lorentz") {
    r.kind = e.tag == "Drude" ? FDTD_DRUDE : FDTD_LORENTZ;
    r.npoles = 1;
    r.delta_eps[0] = 1.0;
    r.freq[0] = detail::number(e.child("Freq"));
    r.gamma[0] = detail::number(e.child("Gamma"));
  } else {
    throw gpu::Error(FDTD_ERR_UNSUPPORTED, "electric dispersion " + e.tag + " is not implemented on the GPU path");
  }
  return r;
}

// identifier -> material; the first of repeated identifiers is kept, as
// std::map::insert does
inline std::map<std::string, fdtd_material> read_material_map(const std::string& text) {
  const Node root = parse(text);
  std::map<std::string, fdtd_material> out;
  for (auto& item : root.kids) {
    if (item.tag != "Item") continue;
    const Node* id = item.child("Identifier");
    const Node* pair = item.child("MaterialPair");
    if (!id || !pair) throw std::runtime_error("xml: an <Item> needs <Identifier> and <MaterialPair>");
    out.emplace(id->text, material_pair(*pair));
  }
  return out;
}

// PMLOptions: N (default 10) and a 0/1 flag per face (default off)
struct PMLOptions {
  int N = 10;
  bool face[3][2] = {{false, false}, {false, false}, {false, false}};
};
inline PMLOptions read_pml_options(const std::string& text) {
  const Node root = parse(text);
  PMLOptions o;
  static const char* axes[3] = {"X", "Y", "Z"};
  for (auto& c : root.kids) {
    if (c.tag == "N") o.N = static_cast<int>(detail::number(&c));
    for (int a = 0; a < 3; a++) {
      if (c.tag != axes[a]) continue;
      for (auto& m : c.kids) {
        const int side = m.tag == "MIN" ? 0 : m.tag == "MAX" ? 1 : -1;
        if (side < 0) continue;
        if (m.text != "0" && m.text != "1") throw std::runtime_error("xml: a 0/1 flag is expected in <" + m.tag + ">");
        o.face[a][side] = m.text == "1";
      }
    }
  }
  return o;
}

// BoundaryOptions: a boundary name per face (default PEC)
struct BoundaryOptions {
  std::string face[3][2] = {{"PEC", "PEC"}, {"PEC", "PEC"}, {"PEC", "PEC"}};
  // the specs of the faces of a dim-dimensional grid that carry a condition
  // (NONE and Parallel faces get none; BlochPeriodic is not implemented)
  std::vector<BoundarySpec> specs(int dim) const {
    std::vector<BoundarySpec> v;
    for (int a = 0; a < dim; a++)
      for (int s = 0; s < 2; s++) {
        const std::string& f = face[a][s];
        int kind = -1;
        if (f == "PEC") kind = FDTD_BC_PEC;
        else if (f == "PMC") kind = FDTD_BC_PMC;
        else if (f == "Symmetric") kind = FDTD_BC_SYMMETRIC;
        else if (f == "Antisymmetric") kind = FDTD_BC_ANTISYMMETRIC;
        else if (f == "Periodic") kind = FDTD_BC_PERIODIC;
        else if (f == "BlochPeriodic")
          throw gpu::Error(FDTD_ERR_UNSUPPORTED, "BlochPeriodic boundaries are not implemented on the GPU path");
        if (kind >= 0) v.push_back(BoundarySpec{a, s, kind});
      }
    return v;
  }
};
// the CPML of the flagged faces on a grid's axes
template <class Grid>
void apply(Grid& grid, const PMLOptions& o, int dim) {
  for (int a = 0; a < dim; a++)
    for (int s = 0; s < 2; s++)
      if (o.face[a][s]) grid.set_pml(static_cast<Dir>(a), s == 0 ? Orientation::MIN : Orientation::MAX, o.N);
}

inline BoundaryOptions read_boundary_options(const std::string& text) {
  const Node root = parse(text);
  BoundaryOptions o;
  static const char* axes[3] = {"X", "Y", "Z"};
  static const char* names[] = {"Periodic", "BlochPeriodic", "PEC", "PMC", "Symmetric", "Antisymmetric",
                                "Parallel", "NONE"};
  for (auto& c : root.kids)
    for (int a = 0; a < 3; a++) {
      if (c.tag != axes[a]) continue;
      for (auto& m : c.kids) {
        const int side = m.tag == "MIN" ? 0 : m.tag == "MAX" ? 1 : -1;
        if (side < 0) continue;
        const std::string name = m.kids.empty() ? m.text : m.kids[0].tag;
        bool ok = false;
        for (auto* n : names) ok = ok || name == n;
        if (!ok) throw std::runtime_error("xml: unknown boundary " + name);
        o.face[a][side] = name;
      }
    }
  return o;
}

}  // namespace xml
}  // namespace fdtd
