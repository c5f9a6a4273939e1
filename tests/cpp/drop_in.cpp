// The reference's time loop written against fdtd_b200.hpp (the drop-in
// layer), run on the GPU. Usage: drop_in <tm|bd|td> <out.bin>
//   tm: 2D TM, FP64 plain, 40 x 36, 6-cell CPML, Gaussian soft source on Ez
//       (the user loop of tests/testTM.cpp with the reference's names);
//   bd: 2D TM, FP64 plain, 36 x 30, BD3 time policy, PEC face at x min,
//       CPML at x max, periodic faces in y; also writes the surface current
//       Jh_x on the interior and the running DFT of Je_z on a box;
//   td: 3D, FP32 fused, 24^3, 4-cell CPML, Drude cube in a material map,
//       x-propagating TFSF box (6 planes) with an Aux1D Gaussian;
//   pm: the tm loop with the x-min and y-max CPML graded by
//       PMLParameterModel(m, ma, sMax, kMax, aMax) of the caller's values;
//   fw: the tm loop, then Grid::apply_forward_materials of E and of H
//       (the reference's XUpdate<Mode, ft, true>); writes Dz, Bx, By.
// Writes the listed fields (float64, x fastest) to out.bin.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <vector>

#include "fdtd_b200.hpp"

using namespace fdtd;

template <class V>
static void dump(std::ofstream& f, const V& v) {
  f.write(reinterpret_cast<const char*>(v.data()), v.size() * sizeof(double));
}

int main(int argc, char** argv) {
  if (argc < 3) return 1;
  const double dx = 1e-6;
  std::ofstream out(argv[2], std::ios::binary);
  try {
    if (!strcmp(argv[1], "tm")) {
      const double dt = 0.99 / std::sqrt(2.0) * dx / c0;
      const int steps = 80;
      gpu::Grid<TM, double> grid(40, 36, 1, dx, dt, steps);
      grid.set_pml(Dir::X, 6);
      grid.set_pml(Dir::Y, 6);
      auto gauss = [dt](double t) { const double n = t / dt; return std::exp(-((n - 20.0) / 6.0) * ((n - 20.0) / 6.0)); };
      auto src = grid.add(make_soft_source<Ez>(gauss, grid.cell(20, 18)));
      grid.plan({YeeUpdate<TM, Dz>(dt, dx),
                 UpdatePML<TM, FieldType::Electric, Dir::X>(dt, dx),
                 UpdatePML<TM, FieldType::Electric, Dir::Y>(dt, dx),
                 VacuumUpdate<TM, FieldType::Electric>(),
                 src,
                 YeeUpdate<TM, Bx>(dt, dx), YeeUpdate<TM, By>(dt, dx),
                 UpdatePML<TM, FieldType::Magnetic, Dir::X>(dt, dx),
                 UpdatePML<TM, FieldType::Magnetic, Dir::Y>(dt, dx),
                 VacuumUpdate<TM, FieldType::Magnetic>()});
      grid.step(30);
      grid.step(steps - 30);
      dump(out, grid.get<Ez>());
      dump(out, grid.get<Hx>());
      dump(out, grid.get<Hy>());
      // a plan out of the fused order is refused
      try {
        grid.plan({VacuumUpdate<TM, FieldType::Electric>(), YeeUpdate<TM, Dz>(dt, dx)});
        return 3;
      } catch (const gpu::Error& e) {
        if (e.code != FDTD_ERR_UNSUPPORTED) return 4;
      }
    } else if (!strcmp(argv[1], "fw")) {
      // the tm loop, then the forward (explicit) material updates of E and H
      const double dt = 0.99 / std::sqrt(2.0) * dx / c0;
      const int steps = 80;
      gpu::Grid<TM, double> grid(40, 36, 1, dx, dt, steps);
      grid.set_pml(Dir::X, 6);
      grid.set_pml(Dir::Y, 6);
      auto gauss = [dt](double t) { const double n = t / dt; return std::exp(-((n - 20.0) / 6.0) * ((n - 20.0) / 6.0)); };
      auto src = grid.add(make_soft_source<Ez>(gauss, grid.cell(20, 18)));
      grid.plan({YeeUpdate<TM, Dz>(dt, dx),
                 UpdatePML<TM, FieldType::Electric, Dir::X>(dt, dx),
                 UpdatePML<TM, FieldType::Electric, Dir::Y>(dt, dx),
                 VacuumUpdate<TM, FieldType::Electric>(),
                 src,
                 YeeUpdate<TM, Bx>(dt, dx), YeeUpdate<TM, By>(dt, dx),
                 UpdatePML<TM, FieldType::Magnetic, Dir::X>(dt, dx),
                 UpdatePML<TM, FieldType::Magnetic, Dir::Y>(dt, dx),
                 VacuumUpdate<TM, FieldType::Magnetic>()});
      grid.step(steps);
      grid.apply_forward_materials(FieldType::Electric);
      grid.apply_forward_materials(FieldType::Magnetic);
      dump(out, grid.get<Dz>());
      dump(out, grid.get<Bx>());
      dump(out, grid.get<By>());
    } else if (!strcmp(argv[1], "pm")) {
      const double dt = 0.99 / std::sqrt(2.0) * dx / c0;
      const int steps = 80;
      const double s0 = 0.8 * 4 / (imp0 * dx);
      gpu::Grid<TM, double> grid(40, 36, 1, dx, dt, steps);
      grid.set_pml(Dir::X, Orientation::MIN, 6, PMLParameterModel(4.0, 2.0, 1.3 * s0, 8.0, 0.1));
      grid.set_pml(Dir::X, Orientation::MAX, 6);
      grid.set_pml(Dir::Y, Orientation::MIN, 6);
      grid.set_pml(Dir::Y, Orientation::MAX, 6, PMLParameterModel(3.5, 1.5, 2.0 * s0, 3.0, 0.2));
      auto gauss = [dt](double t) { const double n = t / dt; return std::exp(-((n - 20.0) / 6.0) * ((n - 20.0) / 6.0)); };
      auto src = grid.add(make_soft_source<Ez>(gauss, grid.cell(20, 18)));
      grid.plan({YeeUpdate<TM, Dz>(dt, dx),
                 UpdatePML<TM, FieldType::Electric, Dir::X>(dt, dx),
                 UpdatePML<TM, FieldType::Electric, Dir::Y>(dt, dx),
                 VacuumUpdate<TM, FieldType::Electric>(),
                 src,
                 YeeUpdate<TM, Bx>(dt, dx), YeeUpdate<TM, By>(dt, dx),
                 UpdatePML<TM, FieldType::Magnetic, Dir::X>(dt, dx),
                 UpdatePML<TM, FieldType::Magnetic, Dir::Y>(dt, dx),
                 VacuumUpdate<TM, FieldType::Magnetic>()});
      grid.step(steps);
      dump(out, grid.get<Ez>());
      dump(out, grid.get<Hx>());
      dump(out, grid.get<Hy>());
    } else if (!strcmp(argv[1], "bd")) {
      const double dt = 0.5 / std::sqrt(2.0) * dx / c0;
      const int steps = 90;
      gpu::Grid<TM, double> grid(36, 30, 1, dx, dt, steps);
      grid.set_pml(Dir::X, Orientation::MAX, 6);
      auto pec = grid.add(make_pec_boundary<TM, Dir::X, Orientation::MIN>());
      auto ylo = grid.add(make_periodic_boundary<TM, Dir::Y, Orientation::MIN>());
      auto yhi = grid.add(make_periodic_boundary<TM, Dir::Y, Orientation::MAX>());
      auto gauss = [dt](double t) { const double n = std::round(t / dt); return std::exp(-((n - 20.0) / 6.0) * ((n - 20.0) / 6.0)); };
      auto src = grid.add(make_soft_source<Ez>(gauss, grid.cell(10, 8)));
      grid.plan({YeeUpdate<TM, Dz, BD3>(dt, dx),
                 UpdatePML<TM, FieldType::Electric, Dir::X>(dt, dx),
                 VacuumUpdate<TM, FieldType::Electric>(),
                 src,
                 pec.updateE(), ylo.updateE(), yhi.updateE(),
                 YeeUpdate<TM, Bx, BD3>(dt, dx), YeeUpdate<TM, By, BD3>(dt, dx),
                 UpdatePML<TM, FieldType::Magnetic, Dir::X>(dt, dx),
                 VacuumUpdate<TM, FieldType::Magnetic>(),
                 pec.updateH(), ylo.updateH(), yhi.updateH()});
      const int hd = grid.add_dft(FDTD_Q_JEZ, {2, 2, 0}, {33, 27, 0}, {0.03, 0.05});
      grid.step(steps);
      dump(out, grid.get<Ez>());
      dump(out, grid.get<Hx>());
      dump(out, grid.get<Hy>());
      // surface current Jh_x on the interior, and the Je_z spectrum
      dump(out, grid.read(FDTD_Q_JHX, {1, 1, 0}, {34, 28, 0}));
      std::vector<double> spec;
      for (auto& z : grid.dft(hd)) {
        spec.push_back(z.real());
        spec.push_back(z.imag());
      }
      dump(out, spec);
      // mixed time policies are refused
      try {
        grid.plan({YeeUpdate<TM, Dz, BD3>(dt, dx), UpdatePML<TM, FieldType::Electric, Dir::X>(dt, dx),
                   VacuumUpdate<TM, FieldType::Electric>(), pec.updateE(), ylo.updateE(), yhi.updateE(),
                   YeeUpdate<TM, Bx, BD4>(dt, dx), YeeUpdate<TM, By, BD4>(dt, dx),
                   UpdatePML<TM, FieldType::Magnetic, Dir::X>(dt, dx), VacuumUpdate<TM, FieldType::Magnetic>(),
                   pec.updateH(), ylo.updateH(), yhi.updateH()});
        return 3;
      } catch (const gpu::Error& e) {
        if (e.code != FDTD_ERR_UNSUPPORTED) return 4;
      }
    } else {
      const double dt = 0.99 / std::sqrt(3.0) * dx / c0;
      const int n = 24, steps = 50, c = n / 2;
      gpu::Grid<ThreeD, float> grid(n, n, n, dx, dt, steps);
      grid.set_pml(Dir::X, 4);
      grid.set_pml(Dir::Y, 4);
      grid.set_pml(Dir::Z, 4);
      std::vector<uint8_t> ids(n * n * n, 0);
      for (int k = 10; k < 14; k++)
        for (int j = 10; j < 14; j++)
          for (int i = 10; i < 14; i++) ids[(k * n + j) * n + i] = 1;
      grid.set_material_map({VacuumUpdate<ThreeD, FieldType::Electric>(),
                             DrudeUpdate<ThreeD, FieldType::Electric>(1.0, 0.3 / dt, 0.01 / dt, dt)},
                            ids);
      auto pulse = [dt](double t) { const double s = std::round(t / dt); return std::exp(-((s - 20.0) / 6.0) * ((s - 20.0) / 6.0)); };
      auto aux = std::make_shared<Aux1D<double>>(n, dx, dt, pulse);
      const std::array<double, 3> origin{double(c), double(c), double(c)}, k{1, 0, 0}, pe{0, 0, 1}, ph{0, 1, 0};
      std::vector<detail::Op> plan_d, plan_b;
      const int lo = 7, hi = 16;
      std::vector<TFSFPlaneSpec> planes;
      planes.push_back(grid.add(make_tfsf_plane<ThreeD, Dir::X, Orientation::MIN>({lo - 1, lo, lo}, {lo - 1, hi, hi}, origin, k, aux, &pe, &ph)));
      planes.push_back(grid.add(make_tfsf_plane<ThreeD, Dir::X, Orientation::MAX>({hi, lo, lo}, {hi, hi, hi}, origin, k, aux, &pe, &ph)));
      planes.push_back(grid.add(make_tfsf_plane<ThreeD, Dir::Y, Orientation::MIN>({lo, lo - 1, lo}, {hi, lo - 1, hi}, origin, k, aux, &pe, &ph)));
      planes.push_back(grid.add(make_tfsf_plane<ThreeD, Dir::Y, Orientation::MAX>({lo, hi, lo}, {hi, hi, hi}, origin, k, aux, &pe, &ph)));
      planes.push_back(grid.add(make_tfsf_plane<ThreeD, Dir::Z, Orientation::MIN>({lo, lo, lo - 1}, {hi, hi, lo - 1}, origin, k, aux, &pe, &ph)));
      planes.push_back(grid.add(make_tfsf_plane<ThreeD, Dir::Z, Orientation::MAX>({lo, lo, hi}, {hi, hi, hi}, origin, k, aux, &pe, &ph)));
      grid.plan({YeeUpdate<ThreeD, Dx>(dt, dx), YeeUpdate<ThreeD, Dy>(dt, dx), YeeUpdate<ThreeD, Dz>(dt, dx),
                 TFSFPlaneSpec::D{0}, TFSFPlaneSpec::D{1}, TFSFPlaneSpec::D{2}, TFSFPlaneSpec::D{3},
                 TFSFPlaneSpec::D{4}, TFSFPlaneSpec::D{5},
                 UpdatePML<ThreeD, FieldType::Electric, Dir::X>(dt, dx),
                 UpdatePML<ThreeD, FieldType::Electric, Dir::Y>(dt, dx),
                 UpdatePML<ThreeD, FieldType::Electric, Dir::Z>(dt, dx),
                 gpu::MaterialMapUpdate{FieldType::Electric},
                 YeeUpdate<ThreeD, Bx>(dt, dx), YeeUpdate<ThreeD, By>(dt, dx), YeeUpdate<ThreeD, Bz>(dt, dx),
                 TFSFPlaneSpec::B{0}, TFSFPlaneSpec::B{1}, TFSFPlaneSpec::B{2}, TFSFPlaneSpec::B{3},
                 TFSFPlaneSpec::B{4}, TFSFPlaneSpec::B{5},
                 UpdatePML<ThreeD, FieldType::Magnetic, Dir::X>(dt, dx),
                 UpdatePML<ThreeD, FieldType::Magnetic, Dir::Y>(dt, dx),
                 UpdatePML<ThreeD, FieldType::Magnetic, Dir::Z>(dt, dx),
                 VacuumUpdate<ThreeD, FieldType::Magnetic>()});
      grid.step(steps);
      dump(out, grid.get<Ex>());
      dump(out, grid.get<Ey>());
      dump(out, grid.get<Ez>());
      dump(out, grid.get<Hx>());
      dump(out, grid.get<Hy>());
      dump(out, grid.get<Hz>());
    }
  } catch (const gpu::Error& e) {
    fprintf(stderr, "fdtd error %d: %s\n", e.code, e.what());
    return 2;
  }
  return 0;
}
