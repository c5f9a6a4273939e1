// The C++ configuration readers (fdtd::xml in fdtd_b200.hpp) on XML text:
// usage: config_xml <materials.xml> <pml.xml> <boundaries.xml>. Prints what
// they read, one record per line, and checks their errors; needs no GPU.
#include <cstdio>
#include <fstream>
#include <sstream>

#include "fdtd_b200.hpp"

using namespace fdtd;

static std::string slurp(const char* path) {
  std::ifstream f(path);
  std::stringstream ss;
  ss << f.rdbuf();
  return ss.str();
}

int main(int argc, char** argv) {
  if (argc < 4) return 1;
  const auto mats = xml::read_material_map(slurp(argv[1]));
  for (auto& kv : mats) {
    const fdtd_material& m = kv.second;
    printf("mat %s %d %.17g %.17g %d %.17g %.17g\n", kv.first.c_str(), m.kind, m.eps_inf, m.mu_r, m.npoles,
           m.npoles ? m.freq[0] : 0.0, m.npoles ? m.gamma[0] : 0.0);
  }
  const auto po = xml::read_pml_options(slurp(argv[2]));
  printf("pml %d", po.N);
  for (int a = 0; a < 3; a++)
    for (int s = 0; s < 2; s++) printf(" %d", po.face[a][s] ? 1 : 0);
  printf("\n");
  const auto bo = xml::read_boundary_options(slurp(argv[3]));
  printf("bc");
  for (int a = 0; a < 3; a++)
    for (int s = 0; s < 2; s++) printf(" %s", bo.face[a][s].c_str());
  printf("\n");
  for (auto& b : bo.specs(3)) printf("spec %d %d %d\n", b.axis, b.side, b.kind);
  // errors: an unknown dispersion, a dispersion the GPU path lacks, a
  // malformed document, an unknown boundary
  int fails = 0;
  try {
    xml::read_material_map("<M><Item><Identifier>a</Identifier><MaterialPair><Electric><Glass/></Electric>"
                           "<Magnetic><Vacuum/></Magnetic></MaterialPair></Item></M>");
  } catch (const gpu::Error&) {
  } catch (const std::runtime_error&) {
    fails |= 1;
  }
  try {
    xml::read_material_map("<M><Item><Identifier>c</Identifier><MaterialPair><Electric><Conductive><Constant>1"
                           "</Constant><Freq>5e12</Freq></Conductive></Electric><Magnetic><Vacuum></Vacuum>"
                           "</Magnetic></MaterialPair></Item></M>");
  } catch (const gpu::Error& e) {
    if (e.code == FDTD_ERR_UNSUPPORTED) fails |= 2;
  }
  try {
    xml::parse("<A><B>1</A>");
  } catch (const std::runtime_error&) {
    fails |= 4;
  }
  try {
    xml::read_boundary_options("<B><X><MIN>Mirror</MIN></X></B>");
  } catch (const std::runtime_error&) {
    fails |= 8;
  }
  // a declaration and a comment are skipped
  const auto po2 = xml::read_pml_options("<?xml version=\"1.0\"?><!-- c --><PML><N>7</N><Y><MAX>1</MAX></Y></PML>");
  if (po2.N == 7 && po2.face[1][1] && !po2.face[0][0]) fails |= 16;
  printf("errors %d\n", fails);
  return 0;
}
