// The aligned x-slab layout of the FP32 method (Slab::lo4, make_slab in
// fdtd_b200/csrc/internal.h), checked on the host for every axis length
// 6..300 and CPML widths 0..20 at each end:
// * every slab cell (slab_index >= 0) has a position in [0, W4), and no two
//   slab cells share one;
// * the 4-cell group of each slab cell starts at slab_group4(x4), 16-byte
//   aligned, and the cell sits at its offset within the group;
// * a group that holds no slab cell has no position, and a position that no
//   slab cell holds belongs to a cell outside the slabs (zero coefficients).
// Exit status 1 on the first violation.
#include <cstdio>
#include <vector>

#include "../../fdtd_b200/csrc/internal.h"

using fdtdb::Slab;

int main() {
  long checked = 0;
  for (int n = 6; n <= 300; n++)
    for (int plo = 0; plo <= 20; plo++)
      for (int phi = 0; phi <= 20; phi++) {
        if (plo + phi + 3 > n) continue;
        const Slab s = fdtdb::make_slab(n, plo, phi);
        if (s.lo4 % 4 || s.W4 % 4 || (phi > 0 && s.hb % 4)) {
          printf("n %d plo %d phi %d: lo4 %d hb %d W4 %d not multiples of 4\n", n, plo, phi, s.lo4, s.hb, s.W4);
          return 1;
        }
        std::vector<int> owner(s.W4 > 0 ? s.W4 : 1, -1);
        for (int i = 1; i <= n - 2; i++) {
          if (fdtdb::slab_index(s, i) < 0) continue;
          const int q = fdtdb::slab_index4(s, i);
          const int g = fdtdb::slab_group4(s, i / 4 * 4);
          if (q < 0 || q >= s.W4 || owner[q] >= 0 || g < 0 || g % 4 || g + i % 4 != q) {
            printf("n %d plo %d phi %d: cell %d at %d (group %d, W4 %d)\n", n, plo, phi, i, q, g, s.W4);
            return 1;
          }
          owner[q] = i;
        }
        // groups without slab cells have no position
        for (int x4 = 0; x4 < n; x4 += 4) {
          bool any = false;
          for (int e = 0; e < 4; e++)
            if (x4 + e >= 1 && x4 + e <= n - 2 && fdtdb::slab_index(s, x4 + e) >= 0) any = true;
          const int g = fdtdb::slab_group4(s, x4);
          if (g >= 0) {
            if (g + 4 > s.W4) {
              printf("n %d plo %d phi %d: group %d at %d past W4 %d\n", n, plo, phi, x4, g, s.W4);
              return 1;
            }
            for (int e = 0; e < 4; e++) {
              const int c = x4 + e;
              const bool slab = c >= 1 && c <= n - 2 && fdtdb::slab_index(s, c) >= 0;
              if (!slab && owner[g + e] >= 0) {
                printf("n %d plo %d phi %d: padding position %d held by cell %d\n", n, plo, phi, g + e, owner[g + e]);
                return 1;
              }
            }
          } else if (any) {
            printf("n %d plo %d phi %d: group %d holds slab cells but no position\n", n, plo, phi, x4);
            return 1;
          }
        }
        checked++;
      }
  printf("%ld layouts checked\n", checked);
  return 0;
}
