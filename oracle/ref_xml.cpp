// Reference config writer: builds the reference's own MaterialMap,
// PMLOptions and BoundaryOptions (compiled from the reference headers,
// unmodified) from a spec file and prints their print_summary XML
// (include/MaterialMap.hpp:46-98, :229-248; include/PML.hpp:146-212;
// include/BoundaryUpdates.hpp:43-113).
//
// TEST INFRASTRUCTURE ONLY. The reference's XML readers need tinyxml2, which
// is not available here; the text its writers produce is what the loaders in
// fdtd_b200/config_xml.py are checked against. Never linked into the product.
//
// Spec file (whitespace separated):
//   nmat M, then M lines: name ekind K delta freq gamma mkind mK
//        ekind 0 Vacuum, 1 Constant, 2 Drude, 3 Lorentz, 4 Conductive (K, freq)
//        mkind 0 Vacuum, 1 Constant
//   pml N xmin xmax ymin ymax zmin zmax       (flags 0/1)
//   bc  xmin xmax ymin ymax zmin zmax          (Boundary enum values,
//        include/BoundaryUpdates.hpp:17-26; BlochPeriodic excluded)
// Output: "=== materials", "=== pml", "=== boundaries" sections.
#include <fdtd.h>
#include "ref_compile_fixes.hpp"
#include <cstdio>
#include <fstream>
#include <iostream>
#include <string>
#include <utility>

using namespace fdtd;

typedef YeeCell<YeeFields<ThreeD, double, std::array>, DoublePolarization<double>, VacuumMagnetization<double>,
                NewPML<ThreeD, double>>
    Cell;

// make_material_pair (include/MaterialMap.hpp:185-193) keeps a printer of
// its argument's type: an lvalue argument would leave it holding a reference
// to this function's parameter, so the functors are passed as rvalues.
template <class E>
static MaterialPair<Cell> with_magnetic(E e, int mkind, double mK) {
  if (mkind == 0) return make_material_pair<Cell>(std::move(e), VacuumUpdate<ThreeD, FieldType::Magnetic>());
  return make_material_pair<Cell>(std::move(e), ConstantUpdate<ThreeD, FieldType::Magnetic>(mK));
}

int main(int argc, char** argv) {
  if (argc < 2) {
    fprintf(stderr, "usage: ref_xml spec.txt\n");
    return 1;
  }
  std::ifstream in(argv[1]);
  std::string key;
  MaterialMap<std::string, Cell> mm;
  PMLOptions po;
  BoundaryOptions bo;
  const double dt = 1e-17;
  while (in >> key) {
    if (key == "nmat") {
      int m;
      in >> m;
      for (int q = 0; q < m; q++) {
        std::string name;
        int ek, mk;
        double K, delta, freq, gamma, mK;
        in >> name >> ek >> K >> delta >> freq >> gamma >> mk >> mK;
        switch (ek) {
          case 0: mm.emplace(name, with_magnetic(VacuumUpdate<ThreeD, FieldType::Electric>(), mk, mK)); break;
          case 1: mm.emplace(name, with_magnetic(ConstantUpdate<ThreeD, FieldType::Electric>(K), mk, mK)); break;
          case 2:
            mm.emplace(name, with_magnetic(DrudeUpdate<ThreeD, FieldType::Electric>(K, freq, gamma, dt), mk, mK));
            break;
          case 3:
            mm.emplace(name,
                       with_magnetic(LorentzUpdate<ThreeD, FieldType::Electric>(K, delta, freq, gamma, dt), mk, mK));
            break;
          default:
            mm.emplace(name, with_magnetic(ConductiveUpdate<ThreeD, FieldType::Electric>(K, freq, dt), mk, mK));
        }
      }
    } else if (key == "pml") {
      int b[6];
      in >> po.N() >> b[0] >> b[1] >> b[2] >> b[3] >> b[4] >> b[5];
      for (int a = 0; a < 3; a++)
        for (int s = 0; s < 2; s++)
          po.get(static_cast<Dir>(a), s == 0 ? Orientation::MIN : Orientation::MAX) = b[2 * a + s] != 0;
    } else if (key == "bc") {
      for (int a = 0; a < 3; a++)
        for (int s = 0; s < 2; s++) {
          int k;
          in >> k;
          bo.get(static_cast<Dir>(a), s == 0 ? Orientation::MIN : Orientation::MAX) = static_cast<Boundary>(k);
        }
    } else {
      fprintf(stderr, "unknown key %s\n", key.c_str());
      return 1;
    }
  }
  std::cout << "=== materials" << std::endl;
  mm.print_summary(std::cout);
  std::cout << "=== pml" << std::endl;
  po.print_summary(std::cout);
  std::cout << "=== boundaries" << std::endl;
  bo.print_summary(std::cout);
  return 0;
}
