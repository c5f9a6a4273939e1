/* CPU oracle for the FDTD time-step hot path: a plain-C restatement of
 * pederson/fdtd's per-cell update functors, written in the reference's
 * arithmetic order and compiled without FMA contraction.
 *
 * TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py as the checker. The product library never
 * links, loads or calls it.
 *
 * The API mirrors the GPU C-ABI in include/fdtd_b200.h so one Python driver
 * can set up both the same way. All units are SI, as in the reference. */
#ifndef FDTD_ORACLE_H
#define FDTD_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_grid oracle_grid;

/* material kinds (include/DispersiveMaterials.hpp:2076-2105) */
enum { OR_VACUUM = 0, OR_CONSTANT = 1, OR_DRUDE = 2, OR_LORENTZ = 3 };
#define OR_MAX_POLES 4

typedef struct {
  int kind;
  int npoles;           /* Drude: 1. Lorentz: 1..OR_MAX_POLES */
  double eps_inf;       /* the reference's K (relative permittivity) */
  double mu_r;          /* magnetic ConstantUpdate K; 1 = VacuumUpdate */
  double delta_eps[OR_MAX_POLES]; /* Lorentz pole strength (reference ignores it: 1) */
  double freq[OR_MAX_POLES];      /* Drude plasma / Lorentz resonance, rad/s */
  double gamma[OR_MAX_POLES];     /* damping, 1/s */
} oracle_material;

oracle_grid* oracle_create(int mode, int nx, int ny, int nz, double dx, double dt);
void oracle_destroy(oracle_grid* g);
/* CPML of `ncells` on one side (0 = min, 1 = max) of `axis`, graded with
 * PMLParameterModel(dx) (include/PML.hpp:368-393). */
int oracle_set_pml(oracle_grid* g, int axis, int side, int ncells);
/* the forward (explicit) material updates of field type ft (0 electric, 1
   magnetic) on every interior cell; -2 with a Lorentz material */
int oracle_material_explicit(oracle_grid* g, int ft);
/* the same side graded with PMLParameterModel(m, ma, sMax, kMax, aMax) */
int oracle_set_pml_model(oracle_grid* g, int axis, int side, int ncells, double m, double ma, double smax,
                         double kmax, double amax);
int oracle_set_materials(oracle_grid* g, const oracle_material* m, int n);
int oracle_set_material_ids(oracle_grid* g, const uint8_t* ids);
/* comp 0..2 = x,y,z; target 0 = E (after the constitutive update),
 * 1 = D (before the CPML pass), 2 = H (after the magnetic constitutive
 * update), 3 = B (before the magnetic CPML pass). vals[t] is added at step t. */
int oracle_add_source(oracle_grid* g, int comp, int target, int i, int j, int k,
                      const double* vals, int nvals);
/* the same source on every cell of the inclusive box lo..hi; target 0 (E) or
 * 2 (H); applied after the point sources of the same field */
int oracle_add_source_box(oracle_grid* g, int comp, int target, const int* lo, const int* hi, const double* vals,
                          int nvals);
/* per-cell relative permittivity (ncell doubles, x fastest): vacuum and
 * constant cells with a value > 0 take it in place of eps_inf; NULL removes */
int oracle_set_eps_map(oracle_grid* g, const double* eps);
/* boundary condition of face (axis, side): 0 none (the outer cells stay
 * zero), 1 PEC, 2 PMC, 3 symmetric, 4 antisymmetric, 5 periodic; applied
 * after the sources of each half step */
int oracle_set_boundary(oracle_grid* g, int axis, int side, int kind);
/* time policy of every curl update and TFSF correction
 * (include/YeeUpdates.hpp:182-294): 1 BD1 (leapfrog, the default), 3 BD3,
 * 4 BD4; the flux history starts at zero */
int oracle_set_time_scheme(oracle_grid* g, int scheme);
/* One TFSF plane (include/Source.hpp:472-634) with its own Aux1D grid.
 * axis/orient give the normal; lo/hi are inclusive cell ranges; origin (in
 * cells) and k define the location functor and wave vector; pol_e / pol_h are
 * the E and H polarisation vectors; aux_vals[s-1] is the aux source value at
 * aux step s. */
int oracle_add_tfsf_plane(oracle_grid* g, int axis, int orient, const int* lo, const int* hi,
                          const double* origin, const double* kvec, const double* pol_e,
                          const double* pol_h, int aux_ncells, const double* aux_vals, int naux);
/* Running DFT of one quantity over an inclusive box: 0..2 E, 3..5 H, 6..8
 * the surface current Je (from H, sampled after the H half), 9..11 Jh (from
 * E), 12 the surface charge density rho (from E; not in TM). */
int oracle_add_dft(oracle_grid* g, int comp, const int* lo, const int* hi,
                   const double* freqs, int nf);
/* the quantity (codes as for oracle_add_dft) on every cell of the inclusive
 * box lo..hi, x fastest, from the current fields; boxes of quantities 6..12
 * lie in the interior */
int oracle_read_quantity(const oracle_grid* g, int q, const int* lo, const int* hi, double* out);
int oracle_step(oracle_grid* g, int nsteps);
/* one half step: 0 = the E half, 1 = the H half (ends the step); the two
 * must alternate, E first */
int oracle_step_half(oracle_grid* g, int phase);
/* which: 0..2 D, 3..5 E, 6..8 B, 9..11 H, 12..14 P(pole 0), 15..17 J(pole 0),
 * 18..35 psi[ft][I][J]; 36.. P/J of further poles (6 per pole). */
int oracle_get(const oracle_grid* g, int which, double* out);
int oracle_set(oracle_grid* g, int which, const double* in);
/* out: [nf][npoints][2] (re, im) */
int oracle_dft_get(const oracle_grid* g, int handle, double* out);
int oracle_dft_npoints(const oracle_grid* g, int handle);
/* the 1D CPML coefficient profile of one axis: out[4][n] = B, C, F, G */
int oracle_pml_profile(const oracle_grid* g, int ft, int axis, double* out);
double oracle_imp0(void);
/* FP64 adjoint of a TM run from a fresh grid: runs nsteps, returns
 * J = sum_probes |DFT_freq(Ez)|^2 and dJ/deps_r over the design box (x
 * fastest). Non-dispersive materials with mu_r = 1, no TFSF planes. */
int oracle_adjoint_tm(oracle_grid* g, int nsteps, const int* plo, const int* phi, double freq, const int* dlo,
                      const int* dhi, double* J, double* grad);

#ifdef __cplusplus
}
#endif
#endif
