// Reference runner: drives pederson/fdtd's own update functors (compiled from
// the reference headers, unmodified) through a user time loop, the way the
// reference's tests do (tests/testTM.cpp:31-113, include/Source.hpp:413-435).
//
// TEST INFRASTRUCTURE ONLY. This program is the checker that pins the C
// restatement in oracle/fdtd_oracle.c and generates tests/golden fixtures.
// It is never linked into, or called by, the product library.
//
// Build: see oracle/Makefile (g++ -std=c++17 -ffp-contract=off, reference
// headers on the include path). Two compile fixes are applied here without
// touching the reference:
//  * DispersiveAtomicUpdate (include/DispersiveMaterials.hpp:260-282) puts
//    enable_if on a class template parameter, which g++13 rejects when any
//    material functor is instantiated; ref_compile_fixes.hpp holds partial
//    specialisations that forward to UpdateStruct::implicit_update /
//    explicit_update with the same argument order as :272-280.
//  * `static constexpr double val` (:370, :745, :1047) is ODR-used; C++17
//    makes it implicitly inline.
//  * BD3::get and BD3::get_reverse (include/YeeUpdates.hpp:209-221) take the
//    cell by const reference and call BD(i) on it, but BDFields
//    (include/YeeFields.hpp:188-200) only has a non-const BD(i); the history
//    mixin below is BDFields with a const BD(i) added.
//
// Scenario file (whitespace separated tokens, see oracle/pyoracle.py writer):
//   mode <0 TEM|1 TE|2 TM|3 ThreeD>
//   dims nx ny nz
//   dxdt dx dt
//   pml nlo_x nhi_x nlo_y nhi_y nlo_z nhi_z
//   explicit 1                    (optional: after the steps, the forward material
//                                 updates XUpdate<Mode, ft, true>, E then H)
//   pmlmodel axis side m ma sMax kMax aMax   (optional, per side: grade it with
//                                 PMLParameterModel(m, ma, sMax, kMax, aMax))
//   nmat M  then M lines: kind K delta freq gamma mu_r
//        kind 0 vacuum, 1 constant, 2 drude, 3 lorentz
//   matids <path|none>            uint8 per cell, index (k*ny+j)*nx+i
//   nsrc S then S lines: comp target i j k path  (comp 0..2, target 0=E 1=D
//        2=H 3=B,
//        path: float64 per step, value added at step t)
//   ntfsf T (T planes) then: aux_ncells aux_path origin_x origin_y origin_z
//        kx ky kz set_pol pe_x pe_y pe_z ph_x ph_y ph_z, and T lines:
//        axis orient i0 i1 j0 j1 k0 k1 (inclusive). set_pol 0 keeps the
//        plane's own polarisation (TE/TM defaults), 1 sets pe/ph.
//        aux_path: float64 per aux step (value for aux step s at index s-1)
//   scheme S (optional; 1 BD1 (default), 3 BD3, 4 BD4: the TimePolicy of
//        every YeeUpdate and TFSFPlane, include/YeeUpdates.hpp:182-294)
//   nbc B then B lines: axis side kind (optional; kind 1 PEC, 2 PMC,
//        3 symmetric, 4 antisymmetric, 5 periodic), applied with the
//        reference's make_*_boundary (include/BoundaryUpdates.hpp) to the
//        interior cells next to the face, after the E sources (updateE) and
//        after the H sources (updateH)
//   steps N
//   out path
// Output: float64 arrays in order D(3) E(3) B(3) H(3) P(3) J(3), the CPML
// integrators psi[ft][I][J] (18), and the surface quantities rho, Je(3),
// Jh(3) that UpdateSurfaceChargeDensity, UpdateSurfaceCurrentE and
// UpdateSurfaceCurrentH (include/SurfaceQuantities.hpp:203-356) give on every
// interior cell after the last step (zero where the mode has none), each
// nx*ny*nz long. The wall time of the time loop alone is printed as
// "loop_seconds <s>".
#include <fdtd.h>
#include "ref_compile_fixes.hpp"
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <string>
#include <vector>
#include <memory>
#include <fstream>
#include <chrono>
#include <cstddef>
#include <iterator>


using namespace fdtd;

static std::vector<double> read_f64(const std::string& path) {
  std::vector<double> v;
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) { fprintf(stderr, "cannot open %s\n", path.c_str()); exit(2); }
  fseek(f, 0, SEEK_END); long n = ftell(f); fseek(f, 0, SEEK_SET);
  v.resize(n / 8);
  if (fread(v.data(), 8, v.size(), f) != v.size()) { fprintf(stderr, "short read\n"); exit(2); }
  fclose(f);
  return v;
}

struct Mat { int kind; double K, delta, freq, gamma, mu; };
struct Src { int comp, target, i, j, k; std::vector<double> vals; };
struct PlaneSpec { int axis, orient, lo[3], hi[3]; };
struct BcSpec { int axis, side, kind; };

struct Scenario {
  int mode = 2, nx = 1, ny = 1, nz = 1;
  int scheme = 1;
  double dx = 1, dt = 1;
  int pml[3][2] = {{0, 0}, {0, 0}, {0, 0}};
  // per side: 0 = PMLParameterModel(dx), 1 = PMLParameterModel(m, ma, sMax, kMax, aMax)
  int explicit_after = 0;  // after the steps, the forward material updates (flux from field)
  int pml_custom[3][2] = {{0, 0}, {0, 0}, {0, 0}};
  double pml_model[3][2][5] = {};
  std::vector<Mat> mats;
  std::vector<uint8_t> ids;
  std::vector<Src> srcs;
  int aux_ncells = 0; std::vector<double> aux_vals; double origin[3] = {0, 0, 0}, kvec[3] = {1, 0, 0};
  int set_pol = 0; double pol_e[3] = {0, 0, 0}, pol_h[3] = {0, 0, 0};
  std::vector<PlaneSpec> planes;
  std::vector<BcSpec> bcs;
  int steps = 0;
  std::string out;
};

// History of the multi-step time policies: the reference's BDFields with a
// const accessor (see the compile fixes above).
template <int n, class Mode>
struct History : public BDFields<n, Mode, double> {
  typedef BDFields<n, Mode, double> Base;
  using Base::BD;
  const typename Base::Fields& BD(int i) const { return const_cast<History*>(this)->Base::BD(i); }
};
struct NoHistory {};
template <class TP> struct Levels { static constexpr int n = 0; };
template <> struct Levels<BD3> { static constexpr int n = 2; };
template <> struct Levels<BD4> { static constexpr int n = 3; };
template <class Mode, class TP>
using HistoryOf = std::conditional_t<Levels<TP>::n == 0, NoHistory, History<(Levels<TP>::n > 0 ? Levels<TP>::n : 1), Mode>>;

// The user-side cell: the reference's YeeCell mixins plus neighbour pointers
// (the neighbour contract of include/DefaultInterfaces.hpp:66-79), and the
// field history when the time policy needs one.
template <class Mode, class TP = BD1>
struct Cell : public YeeCell<YeeFields<Mode, double, std::array>, DoublePolarization<double>,
                             VacuumMagnetization<double>, NewPML<Mode, double>>,
              public HistoryOf<Mode, TP>, public SurfaceQuantities<Mode> {
  Cell* nmin[3] = {nullptr, nullptr, nullptr};
  Cell* nmax[3] = {nullptr, nullptr, nullptr};
  int ci = 0, cj = 0, ck = 0;
  Cell& getNeighborMin(int d) { return *nmin[d]; }
  Cell& getNeighborMax(int d) { return *nmax[d]; }
};

// Iterator over a list of cell pointers that dereferences to the cell, as
// TFSFPlane (include/Source.hpp:595-619) expects.
template <class C>
struct PtrIt {
  typename std::vector<C*>::iterator it;
  C& operator*() const { return **it; }
  PtrIt& operator++() { ++it; return *this; }
  PtrIt operator++(int) { PtrIt t = *this; ++it; return t; }
  bool operator!=(const PtrIt& o) const { return it != o.it; }
  bool operator==(const PtrIt& o) const { return it == o.it; }
};

// Iterator over cell pointers with the iterator traits DerivedIterator
// (include/BoundaryUpdates.hpp:415-478) reads.
template <class C>
struct BcIt {
  typedef std::ptrdiff_t difference_type;
  typedef C value_type;
  typedef C& reference;
  typedef C* pointer;
  typedef std::forward_iterator_tag iterator_category;
  typename std::vector<C*>::iterator it;
  C& operator*() const { return **it; }
  BcIt& operator++() { ++it; return *this; }
  BcIt operator++(int) { BcIt t = *this; ++it; return t; }
  bool operator!=(const BcIt& o) const { return it != o.it; }
  bool operator==(const BcIt& o) const { return it == o.it; }
};

// the periodic partner of a boundary cell: the interior cell at the other
// end of the axis (the Functor of make_periodic_boundary)
template <class C>
struct PartnerF {
  std::vector<C*>* cells;
  std::vector<C*>* partners;
  C& operator()(BcIt<C> it) const { return *(*partners)[it.it - cells->begin()]; }
};

struct TableSignal {
  const std::vector<double>* tab; double dt;
  double operator()(double t) const {
    long s = std::lround(t / dt);
    if (s < 1 || s > (long)tab->size()) return 0.0;
    return (*tab)[s - 1];
  }
};

// per-step table signal for SoftSource::apply(t) with t the step index
struct StepSignal {
  const std::vector<double>* tab;
  double operator()(double t) const {
    long s = static_cast<long>(t);
    return (s >= 0 && s < (long)tab->size()) ? (*tab)[s] : 0.0;
  }
};

// Location functor of a TFSF plane: ((i,j,k) - origin) * dx.
template <class Mode, class TP>
struct LocF {
  const double* origin;
  double dx;
  std::array<double, Mode::dim> operator()(PtrIt<Cell<Mode, TP>> it) const {
    Cell<Mode, TP>& c = *it;
    std::array<double, Mode::dim> pt;
    int idx[3] = {c.ci, c.cj, c.ck};
    for (int d = 0; d < Mode::dim; d++) pt[d] = (static_cast<double>(idx[d]) - origin[d]) * dx;
    return pt;
  }
};
template <class Mode, class TP>
using PlaneOf = TFSFPlane<Mode, LocF<Mode, TP>, PtrIt<Cell<Mode, TP>>, Aux1D<double>, TP>;

// TFSFPlane keeps its polarisation vectors private and, for ThreeD, leaves
// them uninitialised (include/Source.hpp:572-584). The runner sets them
// through member pointers obtained by explicit template instantiation, which
// the language exempts from access checking; the reference is not modified.
template <typename Tag, typename Tag::type M>
struct Rob {
  friend typename Tag::type get(Tag) { return M; }
};
template <class Mode, class TP>
struct PolE {
  typedef std::array<double, 3> PlaneOf<Mode, TP>::*type;
  friend type get(PolE);
};
template <class Mode, class TP>
struct PolH {
  typedef std::array<double, 3> PlaneOf<Mode, TP>::*type;
  friend type get(PolH);
};
#define FDTD_ROB(M, TP)                                                       \
  template struct Rob<PolE<M, TP>, &PlaneOf<M, TP>::mPolarization>;           \
  template struct Rob<PolH<M, TP>, &PlaneOf<M, TP>::mPolarizationH>;
FDTD_ROB(TE, BD1) FDTD_ROB(TM, BD1) FDTD_ROB(ThreeD, BD1)
FDTD_ROB(TE, BD3) FDTD_ROB(TM, BD3) FDTD_ROB(ThreeD, BD3)
FDTD_ROB(TE, BD4) FDTD_ROB(TM, BD4) FDTD_ROB(ThreeD, BD4)
#undef FDTD_ROB

template <class Mode, class F>
constexpr bool has_field() {
  return Detail::tuple_contains_type<F, typename FieldComponents<Mode>::electric>::value ||
         Detail::tuple_contains_type<F, typename FieldComponents<Mode>::magnetic>::value;
}

// a surface quantity of the cell, or 0 where SurfaceQuantities<Mode> has none
#define FDTD_SQ(name)                                                  \
  template <class C> auto sq_##name(C& c, int) -> decltype(c.name()) { \
    return c.name();                                                   \
  }                                                                    \
  template <class C> double sq_##name(C&, long) { return 0.0; }
FDTD_SQ(rho) FDTD_SQ(Jex) FDTD_SQ(Jey) FDTD_SQ(Jez) FDTD_SQ(Jhx) FDTD_SQ(Jhy) FDTD_SQ(Jhz)
#undef FDTD_SQ

template <class Mode, class F, class C>
double field_or_zero(C& c) {
  if constexpr (Detail::tuple_contains_type<F, typename FieldComponents<Mode>::electric>::value ||
                Detail::tuple_contains_type<F, typename FieldComponents<Mode>::magnetic>::value)
    return GetField<F>::get(c);
  else return 0.0;
}
template <class Mode, class F, class Flux, class C>
double flux_or_zero(C& c) {
  if constexpr (Detail::tuple_contains_type<F, typename FieldComponents<Mode>::electric>::value ||
                Detail::tuple_contains_type<F, typename FieldComponents<Mode>::magnetic>::value)
    return GetField<Flux>::get(c);
  else return 0.0;
}

template <class Mode, class Flux, class TP, class C> void yee(C& c, double dt, double dx) {
  if constexpr (Detail::tuple_contains_type<Flux, typename FieldComponents<Mode>::electric_flux>::value ||
                Detail::tuple_contains_type<Flux, typename FieldComponents<Mode>::magnetic_flux>::value)
    YeeUpdate<Mode, Flux, TP>(dt, dx)(c);
}

template <class Mode, class TP>
static int run(Scenario& s) {
  typedef Cell<Mode, TP> C;
  const int nx = s.nx, ny = s.ny, nz = s.nz;
  const int dim = Mode::dim;
  std::vector<C> cells((size_t)nx * ny * nz);
  auto at = [&](int i, int j, int k) -> C& { return cells[((size_t)k * ny + j) * nx + i]; };
  int n[3] = {nx, ny, nz};
  // wire neighbours of interior cells only; the outer ring is never updated
  std::vector<C*> interior;
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        C& c = at(i, j, k); c.ci = i; c.cj = j; c.ck = k;
        int idx[3] = {i, j, k};
        bool in = true;
        for (int d = 0; d < dim; d++) if (idx[d] < 1 || idx[d] > n[d] - 2) in = false;
        if (!in) continue;
        for (int d = 0; d < dim; d++) {
          int lo[3] = {i, j, k}, hi[3] = {i, j, k};
          lo[d]--; hi[d]++;
          c.nmin[d] = &at(lo[0], lo[1], lo[2]);
          c.nmax[d] = &at(hi[0], hi[1], hi[2]);
        }
        interior.push_back(&c);
      }
  // CPML profile, following tests/testTM.cpp:44-71 per axis and side, with
  // the reference's own PMLParameterModel constructors (include/PML.hpp:372-377)
  for (int a = 0; a < dim; a++) {
    for (int side = 0; side < 2; side++) {
      int np = s.pml[a][side];
      if (np <= 0) continue;
      const double* pm = s.pml_model[a][side];
      const PMLParameterModel p = s.pml_custom[a][side] ? PMLParameterModel(pm[0], pm[1], pm[2], pm[3], pm[4])
                                                        : PMLParameterModel(s.dx);
      for (int i = 1; i < np + 2; i++) {
        double x = static_cast<double>(np - i + 1) / static_cast<double>(np);
        double xm = x - 0.5 / static_cast<double>(np);
        int ce = side == 0 ? i : n[a] - i;
        int cm = side == 0 ? i : n[a] - 1 - i;
        for (auto& c : cells) {
          int idx[3] = {c.ci, c.cj, c.ck};
          if (idx[a] == ce) {
            if (a == 0) c.template setPMLParameters<FieldType::Electric, Dir::X>(p.K(x), p.S(x), p.A(x), s.dt);
            if (a == 1) c.template setPMLParameters<FieldType::Electric, Dir::Y>(p.K(x), p.S(x), p.A(x), s.dt);
            if (a == 2) c.template setPMLParameters<FieldType::Electric, Dir::Z>(p.K(x), p.S(x), p.A(x), s.dt);
          }
          if (idx[a] == cm) {
            if (a == 0) c.template setPMLParameters<FieldType::Magnetic, Dir::X>(p.K(xm), p.S(xm), p.A(xm), s.dt);
            if (a == 1) c.template setPMLParameters<FieldType::Magnetic, Dir::Y>(p.K(xm), p.S(xm), p.A(xm), s.dt);
            if (a == 2) c.template setPMLParameters<FieldType::Magnetic, Dir::Z>(p.K(xm), p.S(xm), p.A(xm), s.dt);
          }
        }
      }
    }
  }
  bool pmlax[3];
  for (int a = 0; a < 3; a++) pmlax[a] = (a < dim) && (s.pml[a][0] > 0 || s.pml[a][1] > 0);

  // material functors (include/DispersiveMaterials.hpp:489-497, :881-884, :1208-1211)
  const double dt = s.dt, dx = s.dx;
  std::vector<std::function<void(C&)>> eupd, hupd;
  for (auto& m : s.mats) {
    switch (m.kind) {
      case 0: { VacuumUpdate<Mode, FieldType::Electric> u; eupd.push_back([u](C& c) mutable { u(c); }); break; }
      case 1: { ConstantUpdate<Mode, FieldType::Electric> u(m.K); eupd.push_back([u](C& c) mutable { u(c); }); break; }
      case 2: { DrudeUpdate<Mode, FieldType::Electric> u(m.K, m.freq, m.gamma, dt); eupd.push_back([u](C& c) mutable { u(c); }); break; }
      case 3: { LorentzUpdate<Mode, FieldType::Electric> u(m.K, m.delta, m.freq, m.gamma, dt); eupd.push_back([u](C& c) mutable { u(c); }); break; }
      default: fprintf(stderr, "bad material kind\n"); return 3;
    }
    if (m.mu == 1.0) { VacuumUpdate<Mode, FieldType::Magnetic> u; hupd.push_back([u](C& c) mutable { u(c); }); }
    else { ConstantUpdate<Mode, FieldType::Magnetic> u(m.mu); hupd.push_back([u](C& c) mutable { u(c); }); }
  }
  auto matid = [&](C& c) -> int { return s.ids.empty() ? 0 : s.ids[((size_t)c.ck * ny + c.cj) * nx + c.ci]; };

  // TFSF planes over one shared 1D auxiliary grid (include/Source.hpp:280-634)
  typedef std::array<double, Mode::dim> PT;
  std::vector<std::vector<C*>> plane_cells(s.planes.size());
  LocF<Mode, TP> loc{s.origin, dx};
  typedef PlaneOf<Mode, TP> PlaneT;
  std::vector<std::unique_ptr<PlaneT>> planes;
  if (!s.planes.empty()) {
    PT kv; for (int d = 0; d < Mode::dim; d++) kv[d] = s.kvec[d];
    for (size_t q = 0; q < s.planes.size(); q++) {
      auto& ps = s.planes[q];
      for (int k = ps.lo[2]; k <= ps.hi[2]; k++)
        for (int j = ps.lo[1]; j <= ps.hi[1]; j++)
          for (int i = ps.lo[0]; i <= ps.hi[0]; i++) plane_cells[q].push_back(&at(i, j, k));
      PT normal; for (int d = 0; d < Mode::dim; d++) normal[d] = 0;
      normal[ps.axis] = ps.orient == 1 ? 1 : -1;
      PtrIt<C> b{plane_cells[q].begin()}, e{plane_cells[q].end()};
      // one aux grid per plane: every updateD advances its plane's aux grid
      auto aux = std::make_shared<Aux1D<double>>(s.aux_ncells, dx, dt, TableSignal{&s.aux_vals, dt});
      planes.emplace_back(new PlaneT(kv, normal, loc, b, e, aux));
      if (s.set_pol) {
        (*planes.back()).*get(PolE<Mode, TP>()) = {s.pol_e[0], s.pol_e[1], s.pol_e[2]};
        (*planes.back()).*get(PolH<Mode, TP>()) = {s.pol_h[0], s.pol_h[1], s.pol_h[2]};
      }
    }
  }

  std::vector<std::function<void(double)>> appliers, dappliers, happliers, bappliers;
  for (auto& sr : s.srcs) {
    C& c = at(sr.i, sr.j, sr.k);
    StepSignal sig{&sr.vals};
    auto& lst = sr.target == 0 ? appliers : sr.target == 1 ? dappliers : sr.target == 2 ? happliers : bappliers;
    auto add = [&](auto src) { lst.push_back([src](double t) mutable { src.apply(t); }); };
    if (sr.target == 0) {
      if (sr.comp == 0) { if constexpr (has_field<Mode, Ex>()) add(make_soft_source<Ex>(sig, c)); }
      if (sr.comp == 1) { if constexpr (has_field<Mode, Ey>()) add(make_soft_source<Ey>(sig, c)); }
      if (sr.comp == 2) { if constexpr (has_field<Mode, Ez>()) add(make_soft_source<Ez>(sig, c)); }
    } else if (sr.target == 2) {
      if (sr.comp == 0) { if constexpr (has_field<Mode, Hx>()) add(make_soft_source<Hx>(sig, c)); }
      if (sr.comp == 1) { if constexpr (has_field<Mode, Hy>()) add(make_soft_source<Hy>(sig, c)); }
      if (sr.comp == 2) { if constexpr (has_field<Mode, Hz>()) add(make_soft_source<Hz>(sig, c)); }
    } else if (sr.target == 3) {
      if (sr.comp == 0) { if constexpr (has_field<Mode, Hx>()) add(make_soft_source<Bx>(sig, c)); }
      if (sr.comp == 1) { if constexpr (has_field<Mode, Hy>()) add(make_soft_source<By>(sig, c)); }
      if (sr.comp == 2) { if constexpr (has_field<Mode, Hz>()) add(make_soft_source<Bz>(sig, c)); }
    } else {
      if (sr.comp == 0) { if constexpr (has_field<Mode, Ex>()) add(make_soft_source<Dx>(sig, c)); }
      if (sr.comp == 1) { if constexpr (has_field<Mode, Ey>()) add(make_soft_source<Dy>(sig, c)); }
      if (sr.comp == 2) { if constexpr (has_field<Mode, Ez>()) add(make_soft_source<Dz>(sig, c)); }
    }
  }

  // boundary conditions on the faces (the boundary cells are the interior
  // cells next to the face; their outer neighbours take the image)
  std::vector<std::vector<C*>> bc_cells(s.bcs.size()), bc_partners(s.bcs.size());
  std::vector<BoundaryData> bcs;
  for (size_t q = 0; q < s.bcs.size(); q++) {
    const BcSpec& b = s.bcs[q];
    int lo[3] = {1, 1, dim == 3 ? 1 : 0}, hi[3] = {nx - 2, ny - 2, dim == 3 ? nz - 2 : 0};
    lo[b.axis] = hi[b.axis] = b.side == 0 ? 1 : n[b.axis] - 2;
    for (int k = lo[2]; k <= hi[2]; k++)
      for (int j = lo[1]; j <= hi[1]; j++)
        for (int i = lo[0]; i <= hi[0]; i++) {
          bc_cells[q].push_back(&at(i, j, k));
          int p[3] = {i, j, k};
          p[b.axis] = b.side == 0 ? n[b.axis] - 2 : 1;
          bc_partners[q].push_back(&at(p[0], p[1], p[2]));
        }
    BcIt<C> bb{bc_cells[q].begin()}, be{bc_cells[q].end()};
    PartnerF<C> pf{&bc_cells[q], &bc_partners[q]};
#define FDTD_BC(D, O)                                                                                      \
  if (b.kind == 1) bcs.push_back(make_pec_boundary<Mode, D, O>(bb, be));                                 \
  else if (b.kind == 2) bcs.push_back(make_pmc_boundary<Mode, D, O>(bb, be));                            \
  else if (b.kind == 3) bcs.push_back(make_symmetric_boundary<Mode, D, O>(bb, be));                      \
  else if (b.kind == 4) bcs.push_back(make_antisymmetric_boundary<Mode, D, O>(bb, be));                  \
  else bcs.push_back(make_periodic_boundary<Mode, D, O>(bb, be, pf));
    if (b.axis == 0) { if (b.side == 0) { FDTD_BC(Dir::X, Orientation::MIN) } else { FDTD_BC(Dir::X, Orientation::MAX) } }
    else if (b.axis == 1) { if (b.side == 0) { FDTD_BC(Dir::Y, Orientation::MIN) } else { FDTD_BC(Dir::Y, Orientation::MAX) } }
    else { if (b.side == 0) { FDTD_BC(Dir::Z, Orientation::MIN) } else { FDTD_BC(Dir::Z, Orientation::MAX) } }
#undef FDTD_BC
  }

  const auto clock0 = std::chrono::steady_clock::now();
  for (int t = 0; t < s.steps; t++) {
    // ---- E half step: curl, TFSF, CPML per axis, material, sources
    for (C* c : interior) yee<Mode, Dx, TP>(*c, dt, dx);
    for (C* c : interior) yee<Mode, Dy, TP>(*c, dt, dx);
    for (C* c : interior) yee<Mode, Dz, TP>(*c, dt, dx);
    for (auto& pl : planes) pl->updateD(dt, dx);
    for (auto& ap : dappliers) ap(static_cast<double>(t));
    if (pmlax[0]) for (C* c : interior) UpdatePML<Mode, FieldType::Electric, Dir::X>(dt, dx)(*c);
    if (pmlax[1]) for (C* c : interior) UpdatePML<Mode, FieldType::Electric, Dir::Y>(dt, dx)(*c);
    if constexpr (Mode::dim == 3) { if (pmlax[2]) for (C* c : interior) UpdatePML<Mode, FieldType::Electric, Dir::Z>(dt, dx)(*c); }
    for (C* c : interior) eupd[matid(*c)](*c);
    for (auto& ap : appliers) ap(static_cast<double>(t));
    for (auto& b : bcs) b.updateE();
    // ---- H half step
    for (C* c : interior) yee<Mode, Bx, TP>(*c, dt, dx);
    for (C* c : interior) yee<Mode, By, TP>(*c, dt, dx);
    for (C* c : interior) yee<Mode, Bz, TP>(*c, dt, dx);
    for (auto& pl : planes) pl->updateB(dt, dx);
    for (auto& ap : bappliers) ap(static_cast<double>(t));
    if (pmlax[0]) for (C* c : interior) UpdatePML<Mode, FieldType::Magnetic, Dir::X>(dt, dx)(*c);
    if (pmlax[1]) for (C* c : interior) UpdatePML<Mode, FieldType::Magnetic, Dir::Y>(dt, dx)(*c);
    if constexpr (Mode::dim == 3) { if (pmlax[2]) for (C* c : interior) UpdatePML<Mode, FieldType::Magnetic, Dir::Z>(dt, dx)(*c); }
    for (C* c : interior) hupd[matid(*c)](*c);
    for (auto& ap : happliers) ap(static_cast<double>(t));
    for (auto& b : bcs) b.updateH();
  }

  const double loop_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - clock0).count();
  printf("loop_seconds %.9f\n", loop_s);
  if (s.explicit_after) {
    // the reference's forward material functors, XUpdate<Mode, ft, true>
    // (DispersiveMaterials.hpp:489-497, :1208-1211): flux from field
    std::vector<std::function<void(C&)>> eexp, hexp;
    for (auto& m : s.mats) {
      switch (m.kind) {
        case 0: { VacuumUpdate<Mode, FieldType::Electric, true> u; eexp.push_back([u](C& c) mutable { u(c); }); break; }
        case 1: { ConstantUpdate<Mode, FieldType::Electric, true> u(m.K); eexp.push_back([u](C& c) mutable { u(c); }); break; }
        case 2: { DrudeUpdate<Mode, FieldType::Electric, true> u(m.K, m.freq, m.gamma, dt); eexp.push_back([u](C& c) mutable { u(c); }); break; }
        default: fprintf(stderr, "no forward update for this material kind\n"); return 5;
      }
      if (m.mu == 1.0) { VacuumUpdate<Mode, FieldType::Magnetic, true> u; hexp.push_back([u](C& c) mutable { u(c); }); }
      else { ConstantUpdate<Mode, FieldType::Magnetic, true> u(m.mu); hexp.push_back([u](C& c) mutable { u(c); }); }
    }
    for (C* c : interior) eexp[matid(*c)](*c);
    for (C* c : interior) hexp[matid(*c)](*c);
  }
  {
    UpdateSurfaceChargeDensity<Mode> rho(dx);
    UpdateSurfaceCurrentE<Mode> je(dx);
    UpdateSurfaceCurrentH<Mode> jh(dx);
    for (C* c : interior) {
      rho(*c);
      je(*c);
      jh(*c);
    }
  }
  FILE* f = fopen(s.out.c_str(), "wb");
  if (!f) return 4;
  std::vector<double> buf(cells.size());
  auto dump = [&](auto getter) {
    for (size_t q = 0; q < cells.size(); q++) buf[q] = getter(cells[q]);
    fwrite(buf.data(), 8, buf.size(), f);
  };
  dump([](C& c) { return flux_or_zero<Mode, Ex, Dx>(c); });
  dump([](C& c) { return flux_or_zero<Mode, Ey, Dy>(c); });
  dump([](C& c) { return flux_or_zero<Mode, Ez, Dz>(c); });
  dump([](C& c) { return field_or_zero<Mode, Ex>(c); });
  dump([](C& c) { return field_or_zero<Mode, Ey>(c); });
  dump([](C& c) { return field_or_zero<Mode, Ez>(c); });
  dump([](C& c) { return flux_or_zero<Mode, Hx, Bx>(c); });
  dump([](C& c) { return flux_or_zero<Mode, Hy, By>(c); });
  dump([](C& c) { return flux_or_zero<Mode, Hz, Bz>(c); });
  dump([](C& c) { return field_or_zero<Mode, Hx>(c); });
  dump([](C& c) { return field_or_zero<Mode, Hy>(c); });
  dump([](C& c) { return field_or_zero<Mode, Hz>(c); });
  dump([](C& c) { return c.Px(); });
  dump([](C& c) { return c.Py(); });
  dump([](C& c) { return c.Pz(); });
  dump([](C& c) { return c.Jx(); });
  dump([](C& c) { return c.Jy(); });
  dump([](C& c) { return c.Jz(); });
#define PSI(ft, I, J) dump([](C& c) { return c.template pmlI<FieldType::ft, Dir::I, Dir::J>(); });
  PSI(Electric, X, X) PSI(Electric, X, Y) PSI(Electric, X, Z)
  PSI(Electric, Y, X) PSI(Electric, Y, Y) PSI(Electric, Y, Z)
  PSI(Electric, Z, X) PSI(Electric, Z, Y) PSI(Electric, Z, Z)
  PSI(Magnetic, X, X) PSI(Magnetic, X, Y) PSI(Magnetic, X, Z)
  PSI(Magnetic, Y, X) PSI(Magnetic, Y, Y) PSI(Magnetic, Y, Z)
  PSI(Magnetic, Z, X) PSI(Magnetic, Z, Y) PSI(Magnetic, Z, Z)
  dump([](C& c) { return static_cast<double>(sq_rho(c, 0)); });
  dump([](C& c) { return static_cast<double>(sq_Jex(c, 0)); });
  dump([](C& c) { return static_cast<double>(sq_Jey(c, 0)); });
  dump([](C& c) { return static_cast<double>(sq_Jez(c, 0)); });
  dump([](C& c) { return static_cast<double>(sq_Jhx(c, 0)); });
  dump([](C& c) { return static_cast<double>(sq_Jhy(c, 0)); });
  dump([](C& c) { return static_cast<double>(sq_Jhz(c, 0)); });
  fclose(f);
  return 0;
}

int main(int argc, char** argv) {
  if (argc < 2) { fprintf(stderr, "usage: ref_runner scenario.txt\n"); return 1; }
  std::ifstream in(argv[1]);
  Scenario s;
  std::string key;
  while (in >> key) {
    if (key == "mode") in >> s.mode;
    else if (key == "dims") in >> s.nx >> s.ny >> s.nz;
    else if (key == "dxdt") in >> s.dx >> s.dt;
    else if (key == "pml") for (int a = 0; a < 3; a++) in >> s.pml[a][0] >> s.pml[a][1];
    else if (key == "explicit") in >> s.explicit_after;
    else if (key == "pmlmodel") {
      int a, sd;
      in >> a >> sd;
      s.pml_custom[a][sd] = 1;
      for (int q = 0; q < 5; q++) in >> s.pml_model[a][sd][q];
    }
    else if (key == "nmat") {
      int m; in >> m; s.mats.resize(m);
      for (auto& x : s.mats) in >> x.kind >> x.K >> x.delta >> x.freq >> x.gamma >> x.mu;
    } else if (key == "matids") {
      std::string p; in >> p;
      if (p != "none") {
        FILE* f = fopen(p.c_str(), "rb");
        s.ids.resize((size_t)s.nx * s.ny * s.nz);
        if (!f || fread(s.ids.data(), 1, s.ids.size(), f) != s.ids.size()) { fprintf(stderr, "bad ids\n"); return 2; }
        fclose(f);
      }
    } else if (key == "nsrc") {
      int m; in >> m; s.srcs.resize(m);
      for (auto& x : s.srcs) { std::string p; in >> x.comp >> x.target >> x.i >> x.j >> x.k >> p; x.vals = read_f64(p); }
    } else if (key == "ntfsf") {
      int m; in >> m; std::string p;
      in >> s.aux_ncells >> p >> s.origin[0] >> s.origin[1] >> s.origin[2] >> s.kvec[0] >> s.kvec[1] >> s.kvec[2];
      in >> s.set_pol >> s.pol_e[0] >> s.pol_e[1] >> s.pol_e[2] >> s.pol_h[0] >> s.pol_h[1] >> s.pol_h[2];
      if (m > 0) s.aux_vals = read_f64(p);
      s.planes.resize(m);
      for (auto& x : s.planes) in >> x.axis >> x.orient >> x.lo[0] >> x.hi[0] >> x.lo[1] >> x.hi[1] >> x.lo[2] >> x.hi[2];
    } else if (key == "nbc") {
      int m; in >> m;
      s.bcs.resize(m);
      for (auto& b : s.bcs) in >> b.axis >> b.side >> b.kind;
    } else if (key == "scheme") in >> s.scheme;
    else if (key == "steps") in >> s.steps;
    else if (key == "out") in >> s.out;
    else { fprintf(stderr, "unknown key %s\n", key.c_str()); return 1; }
  }
  if (s.scheme != 1 && s.scheme != 3 && s.scheme != 4) { fprintf(stderr, "bad scheme\n"); return 1; }
  switch (s.mode * 10 + s.scheme) {
    case 11: return run<TE, BD1>(s);
    case 13: return run<TE, BD3>(s);
    case 14: return run<TE, BD4>(s);
    case 21: return run<TM, BD1>(s);
    case 23: return run<TM, BD3>(s);
    case 24: return run<TM, BD4>(s);
    case 31: return run<ThreeD, BD1>(s);
    case 33: return run<ThreeD, BD3>(s);
    case 34: return run<ThreeD, BD4>(s);
    default: fprintf(stderr, "mode %d not supported\n", s.mode); return 1;
  }
}
