/* CPU oracle: plain-C restatement of pederson/fdtd's time-step hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker for tests/, smoke() and bench.py's
 * CPU baseline); never part of the product.
 *
 * Every update below follows the reference functor it names, in the same
 * floating-point operation order, so that with -ffp-contract=off it matches
 * the reference compiled the same way bit for bit (pinned by
 * tests/test_oracle_cpu.py against oracle/_ref/ref_runner and the fixtures in
 * tests/golden/).
 *
 * Schedule of one step (the user loop of tests/testTM.cpp:102-113 and
 * include/Source.hpp:413-435; the reference fixes no place for TFSF planes and
 * soft sources in a user loop, so they sit where this schedule puts them, and
 * the GPU library follows the same schedule):
 *   E half: YeeUpdate on every E flux, TFSF updateD, D-target sources,
 *           UpdatePML<Electric, X|Y|Z>, material update, E-target sources,
 *           DFT of E.
 *   H half: YeeUpdate on every B flux, TFSF updateB, B-target sources,
 *           UpdatePML<Magnetic, X|Y|Z>, material update, H-target sources,
 *           DFT of H.
 * Only interior cells (1..n-2 along each active axis) are updated; the outer
 * ring keeps its initial zeros, as in tests/testTM.cpp:33-40,103. */
#include "fdtd_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* include/FDTDConstants.hpp:394-398 */
static const double k_pi = 3.14159265358979323846264338327950288;
static const double k_eps0 = 8.854e-12;
#define K_MU0 (k_pi * 4.0e-7)

/* include/FDTDConstants.hpp:136-156: the reference's constexpr Newton sqrt,
 * reproduced because imp0 = sqrt(mu0/eps0) is evaluated with it. */
static double ref_sqrt(double x) {
  double curr = x, prev = 0.0;
  while (curr != prev) {
    double next = 0.5 * (curr + x / curr);
    prev = curr;
    curr = next;
  }
  return curr;
}
double oracle_imp0(void) { return ref_sqrt(K_MU0 / k_eps0); }

enum { TEM = 0, TE = 1, TM = 2, THREED = 3 };

typedef struct {
  int axis, orient, lo[3], hi[3];
  double origin[3], k[3], pol_e[3], pol_h[3], normal[3];
  /* Aux1D state: TEM grid with Dz, Ez, By, Hy and CPML */
  int L;
  double *Dz, *Ez, *By, *Hy, *psiE, *psiH;
  double *pB[2], *pC[2], *pF[2], *pG[2];
  double t;
  double* vals;
  int nvals;
} plane_t;

typedef struct {
  int comp, lo[3], hi[3], nf, npts;
  double* freqs;
  double* acc; /* [nf][npts][2] */
} dft_t;

typedef struct {
  int comp, target, i, j, k, nvals;
  int i1, j1, k1; /* box sources: the inclusive upper corner */
  double* vals;
} src_t;

struct oracle_grid {
  int mode, n[3];
  size_t ncell;
  double dx, dt;
  int hasE[3], hasH[3];
  double *D[3], *E[3], *B[3], *H[3];
  double *P[OR_MAX_POLES][3], *J[OR_MAX_POLES][3];
  double* psi[2][3][3];
  /* 1D CPML coefficients per (field type, axis): B, C, F, G */
  double* cB[2][3];
  double* cC[2][3];
  double* cF[2][3];
  double* cG[2][3];
  int pml[3][2];
  oracle_material mats[256];
  int nmat;
  uint8_t* ids;
  src_t* srcs;
  int nsrc;
  src_t* boxes;
  int nbox;
  double* eps_map; /* per-cell relative permittivity of vacuum/constant cells, or NULL */
  int bc[3][2];    /* boundary condition of each face: 0 none, 1..5 (oracle_set_boundary) */
  int scheme;      /* time policy of the curl updates: 1 BD1, 3 BD3, 4 BD4 */
  double* hist[2][3][3]; /* [D|B][level][comp]: the flux history BD(level) of BD3/BD4 */
  plane_t* planes;
  int nplanes;
  dft_t* dfts;
  int ndft;
  long t; /* steps taken */
};

static int lc(int I, int J, int K) {
  if ((I == 0 && J == 1 && K == 2) || (I == 1 && J == 2 && K == 0) || (I == 2 && J == 0 && K == 1)) return 1;
  if ((I == 2 && J == 1 && K == 0) || (I == 0 && J == 2 && K == 1) || (I == 1 && J == 0 && K == 2)) return -1;
  return 0;
}
static int third(int I, int J) { return 3 - I - J; }

/* PMLParameterModel(dx) (include/PML.hpp:368-393) */
typedef struct { double m, ma, smax, kmax, amax; } pml_model;
static pml_model model_for(double dx) {
  pml_model p;
  p.m = 3; p.ma = 1;
  p.smax = 0.8 * (p.m + 1) / (oracle_imp0() * dx);
  p.kmax = 5; p.amax = 0.05;
  return p;
}
static double mK(const pml_model* p, double x) { if (x < 0.0) return 1.0; return x > 1.0 ? 1.0 : 1.0 + pow(x, p->m) * (p->kmax - 1.0); }
static double mS(const pml_model* p, double x) { if (x < 0.0) return 0.0; return x > 1.0 ? 0.0 : pow(x, p->m) * p->smax; }
static double mA(const pml_model* p, double x) { if (x < 0.0) return 0.0; return x > 1.0 ? 0.0 : pow(1.0 - x, p->ma) * p->amax; }

/* NewPML::setPMLParameters (include/PML.hpp:84-102) */
static void set_params(double K, double S, double A, double dt, double* B, double* C, double* F, double* G) {
  double nu = 1.0 / k_eps0 * (S / K + A);
  *B = exp(-dt * nu);
  *C = (nu == 0) ? 0.0 : S / K * 1.0 / (S + K * A) * (*B - 1.0);
  double u = -S / (k_eps0 * K * K);
  *F = (nu == 0) ? 1.0 / K : 1.0 / K - 1.0 / dt * (1.0 - *B - nu * dt) * u / (nu * nu);
  *G = (nu == 0) ? 0.0 : 1.0 / dt * (1.0 - *B) / nu;
}

/* grading loop of tests/testTM.cpp:44-71 for one side of one axis, with
   the model of PMLParameterModel(dx) or PMLParameterModel(m, ma, sMax,
   kMax, aMax) (include/PML.hpp:370-377) */
static void grade(pml_model p, double dt, int n, int np, int side, double* B[2], double* C[2], double* F[2], double* G[2]) {
  for (int i = 1; i < np + 2; i++) {
    double x = (double)(np - i + 1) / (double)np;
    double xm = x - 0.5 / (double)np;
    int ce = side == 0 ? i : n - i;
    int cm = side == 0 ? i : n - 1 - i;
    if (ce >= 0 && ce < n) set_params(mK(&p, x), mS(&p, x), mA(&p, x), dt, &B[0][ce], &C[0][ce], &F[0][ce], &G[0][ce]);
    if (cm >= 0 && cm < n) set_params(mK(&p, xm), mS(&p, xm), mA(&p, xm), dt, &B[1][cm], &C[1][cm], &F[1][cm], &G[1][cm]);
  }
}

static double* zalloc(size_t n) { return (double*)calloc(n ? n : 1, sizeof(double)); }

oracle_grid* oracle_create(int mode, int nx, int ny, int nz, double dx, double dt) {
  if (mode != TE && mode != TM && mode != THREED) return NULL;
  if (nx < 3 || ny < 3 || nz < 1 || (mode == THREED && nz < 3) || (mode != THREED && nz != 1)) return NULL;
  oracle_grid* g = (oracle_grid*)calloc(1, sizeof(oracle_grid));
  g->mode = mode; g->n[0] = nx; g->n[1] = ny; g->n[2] = nz;
  g->ncell = (size_t)nx * ny * nz;
  g->dx = dx; g->dt = dt;
  for (int c = 0; c < 3; c++) {
    g->hasE[c] = mode == THREED || (mode == TE && c < 2) || (mode == TM && c == 2);
    g->hasH[c] = mode == THREED || (mode == TE && c == 2) || (mode == TM && c < 2);
    g->D[c] = zalloc(g->ncell); g->E[c] = zalloc(g->ncell);
    g->B[c] = zalloc(g->ncell); g->H[c] = zalloc(g->ncell);
    for (int q = 0; q < OR_MAX_POLES; q++) { g->P[q][c] = zalloc(g->ncell); g->J[q][c] = zalloc(g->ncell); }
  }
  for (int f = 0; f < 2; f++)
    for (int I = 0; I < 3; I++)
      for (int J = 0; J < 3; J++) g->psi[f][I][J] = zalloc(g->ncell);
  for (int f = 0; f < 2; f++)
    for (int a = 0; a < 3; a++) {
      int n = g->n[a];
      g->cB[f][a] = zalloc(n); g->cC[f][a] = zalloc(n); g->cF[f][a] = zalloc(n); g->cG[f][a] = zalloc(n);
      for (int i = 0; i < n; i++) g->cF[f][a][i] = 1.0; /* NewPML defaults (PML.hpp:40-55) */
    }
  g->scheme = 1;
  g->nmat = 1;
  memset(&g->mats[0], 0, sizeof(oracle_material));
  g->mats[0].kind = OR_VACUUM; g->mats[0].eps_inf = 1.0; g->mats[0].mu_r = 1.0;
  return g;
}

void oracle_destroy(oracle_grid* g) {
  if (!g) return;
  for (int c = 0; c < 3; c++) {
    free(g->D[c]); free(g->E[c]); free(g->B[c]); free(g->H[c]);
    for (int q = 0; q < OR_MAX_POLES; q++) { free(g->P[q][c]); free(g->J[q][c]); }
  }
  for (int f = 0; f < 2; f++) {
    for (int I = 0; I < 3; I++) for (int J = 0; J < 3; J++) free(g->psi[f][I][J]);
    for (int a = 0; a < 3; a++) { free(g->cB[f][a]); free(g->cC[f][a]); free(g->cF[f][a]); free(g->cG[f][a]); }
  }
  free(g->ids);
  for (int s = 0; s < g->nsrc; s++) free(g->srcs[s].vals);
  free(g->srcs);
  for (int s = 0; s < g->nbox; s++) free(g->boxes[s].vals);
  free(g->boxes);
  free(g->eps_map);
  for (int f = 0; f < 2; f++)
    for (int l = 0; l < 3; l++)
      for (int c = 0; c < 3; c++) free(g->hist[f][l][c]);
  for (int p = 0; p < g->nplanes; p++) {
    plane_t* pl = &g->planes[p];
    free(pl->Dz); free(pl->Ez); free(pl->By); free(pl->Hy); free(pl->psiE); free(pl->psiH); free(pl->vals);
    for (int f = 0; f < 2; f++) { free(pl->pB[f]); free(pl->pC[f]); free(pl->pF[f]); free(pl->pG[f]); }
  }
  free(g->planes);
  for (int d = 0; d < g->ndft; d++) { free(g->dfts[d].freqs); free(g->dfts[d].acc); }
  free(g->dfts);
  free(g);
}

static int set_pml_side(oracle_grid* g, int axis, int side, int ncells, pml_model p) {
  int dim = g->mode == THREED ? 3 : 2;
  if (axis < 0 || axis >= dim || side < 0 || side > 1 || ncells < 1) return -1;
  g->pml[axis][side] = ncells;
  double* B[2] = {g->cB[0][axis], g->cB[1][axis]};
  double* C[2] = {g->cC[0][axis], g->cC[1][axis]};
  double* F[2] = {g->cF[0][axis], g->cF[1][axis]};
  double* G[2] = {g->cG[0][axis], g->cG[1][axis]};
  grade(p, g->dt, g->n[axis], ncells, side, B, C, F, G);
  return 0;
}

int oracle_set_pml(oracle_grid* g, int axis, int side, int ncells) {
  return set_pml_side(g, axis, side, ncells, model_for(g->dx));
}

int oracle_set_pml_model(oracle_grid* g, int axis, int side, int ncells, double m, double ma, double smax,
                         double kmax, double amax) {
  pml_model p;
  p.m = m; p.ma = ma; p.smax = smax; p.kmax = kmax; p.amax = amax;
  return set_pml_side(g, axis, side, ncells, p);
}

int oracle_pml_profile(const oracle_grid* g, int ft, int axis, double* out) {
  if (ft < 0 || ft > 1 || axis < 0 || axis > 2) return -1;
  int n = g->n[axis];
  memcpy(out, g->cB[ft][axis], n * sizeof(double));
  memcpy(out + n, g->cC[ft][axis], n * sizeof(double));
  memcpy(out + 2 * n, g->cF[ft][axis], n * sizeof(double));
  memcpy(out + 3 * n, g->cG[ft][axis], n * sizeof(double));
  return 0;
}

int oracle_set_materials(oracle_grid* g, const oracle_material* m, int n) {
  if (n < 1 || n > 256) return -1;
  for (int q = 0; q < n; q++)
    if (m[q].npoles < 0 || m[q].npoles > OR_MAX_POLES) return -1;
  memcpy(g->mats, m, n * sizeof(oracle_material));
  g->nmat = n;
  return 0;
}

int oracle_set_material_ids(oracle_grid* g, const uint8_t* ids) {
  if (!g->ids) g->ids = (uint8_t*)malloc(g->ncell);
  memcpy(g->ids, ids, g->ncell);
  return 0;
}

int oracle_add_source(oracle_grid* g, int comp, int target, int i, int j, int k, const double* vals, int nvals) {
  if (comp < 0 || comp > 2 || target < 0 || target > 3) return -1;
  if (i < 0 || i >= g->n[0] || j < 0 || j >= g->n[1] || k < 0 || k >= g->n[2]) return -1;
  g->srcs = (src_t*)realloc(g->srcs, (g->nsrc + 1) * sizeof(src_t));
  src_t* s = &g->srcs[g->nsrc++];
  s->comp = comp; s->target = target; s->i = i; s->j = j; s->k = k; s->nvals = nvals;
  s->vals = zalloc(nvals);
  memcpy(s->vals, vals, nvals * sizeof(double));
  return 0;
}

int oracle_add_source_box(oracle_grid* g, int comp, int target, const int* lo, const int* hi, const double* vals,
                          int nvals) {
  if (comp < 0 || comp > 2 || (target != 0 && target != 2)) return -1;
  for (int d = 0; d < 3; d++)
    if (lo[d] < 0 || hi[d] >= g->n[d] || lo[d] > hi[d]) return -1;
  g->boxes = (src_t*)realloc(g->boxes, (g->nbox + 1) * sizeof(src_t));
  src_t* s = &g->boxes[g->nbox++];
  s->comp = comp; s->target = target; s->nvals = nvals;
  s->i = lo[0]; s->j = lo[1]; s->k = lo[2]; s->i1 = hi[0]; s->j1 = hi[1]; s->k1 = hi[2];
  s->vals = zalloc(nvals);
  memcpy(s->vals, vals, nvals * sizeof(double));
  return 0;
}

/* every cell of each box source of `target` (0 = E, 2 = H) gets the value of
 * step t, after the point sources of the same field */
static void apply_boxes(oracle_grid* g, int target) {
  const size_t sy = (size_t)g->n[0], sz = (size_t)g->n[0] * g->n[1];
  for (int s = 0; s < g->nbox; s++) {
    const src_t* b = &g->boxes[s];
    if (b->target != target) continue;
    const double v = g->t < b->nvals ? b->vals[g->t] : 0.0;
    double* f = target == 0 ? g->E[b->comp] : g->H[b->comp];
    for (int k = b->k; k <= b->k1; k++)
      for (int j = b->j; j <= b->j1; j++)
        for (int i = b->i; i <= b->i1; i++) f[k * sz + j * sy + i] += v;
  }
}

int oracle_set_boundary(oracle_grid* g, int axis, int side, int kind) {
  int dim = g->mode == THREED ? 3 : 2;
  if (axis < 0 || axis >= dim || side < 0 || side > 1 || kind < 0 || kind > 5) return -1;
  g->bc[axis][side] = kind;
  return 0;
}

/* sign of the image of component c of field type ft (0 E, 1 H) across a face
 * normal to `axis` (include/BoundaryUpdates.hpp:528-536, 612-618, 663-670,
 * 716-723); periodic keeps the sign */
static double bc_mask(int kind, int ft, int c, int axis) {
  const int normal = c == axis;
  switch (kind) {
    case 1: return ft == 0 ? (normal ? 1.0 : -1.0) : (normal ? -1.0 : 1.0);  /* PEC */
    case 2: return ft == 0 ? (normal ? -1.0 : 1.0) : (normal ? 1.0 : -1.0);  /* PMC */
    case 3: return normal ? -1.0 : 1.0;                                       /* symmetric */
    case 4: return normal ? 1.0 : -1.0;                                       /* antisymmetric */
    default: return 1.0;                                                      /* periodic */
  }
}

/* every face with a boundary condition: its outer cells take the masked
 * image of the interior cells next to the face (periodic: of the interior
 * cells at the far end of the axis), for E (ft 0) or H (ft 1) */
static void apply_boundaries(oracle_grid* g, int ft) {
  const int dim = g->mode == THREED ? 3 : 2;
  const size_t sy = (size_t)g->n[0], sz = (size_t)g->n[0] * g->n[1];
  for (int a = 0; a < dim; a++)
    for (int side = 0; side < 2; side++) {
      const int kind = g->bc[a][side];
      if (!kind) continue;
      int lo[3] = {1, 1, dim == 3 ? 1 : 0}, hi[3] = {g->n[0] - 2, g->n[1] - 2, dim == 3 ? g->n[2] - 2 : 0};
      lo[a] = hi[a] = side == 0 ? 1 : g->n[a] - 2;
      for (int k = lo[2]; k <= hi[2]; k++)
        for (int j = lo[1]; j <= hi[1]; j++)
          for (int i = lo[0]; i <= hi[0]; i++) {
            int src[3] = {i, j, k}, dst[3] = {i, j, k};
            dst[a] = side == 0 ? 0 : g->n[a] - 1;
            if (kind == 5) src[a] = side == 0 ? g->n[a] - 2 : 1;
            const size_t cs = src[2] * sz + src[1] * sy + src[0], cd = dst[2] * sz + dst[1] * sy + dst[0];
            for (int c = 0; c < 3; c++) {
              if (ft == 0 && g->hasE[c]) g->E[c][cd] = bc_mask(kind, 0, c, a) * g->E[c][cs];
              if (ft == 1 && g->hasH[c]) g->H[c][cd] = bc_mask(kind, 1, c, a) * g->H[c][cs];
            }
          }
    }
}

int oracle_set_time_scheme(oracle_grid* g, int scheme) {
  if (scheme != 1 && scheme != 3 && scheme != 4) return -1;
  int levels = scheme == 1 ? 0 : scheme - 1;
  for (int f = 0; f < 2; f++)
    for (int l = 0; l < 3; l++)
      for (int c = 0; c < 3; c++) {
        free(g->hist[f][l][c]);
        g->hist[f][l][c] = l < levels ? zalloc(g->ncell) : NULL;
      }
  g->scheme = scheme;
  return 0;
}

/* curl_coeff of the time policy (YeeUpdates.hpp:185, :206, :255) */
static double curl_coeff(int scheme) { return scheme == 3 ? 24.0 / 23.0 : scheme == 4 ? 24.0 / 22.0 : 1.0; }

/* YeeUpdate::update_all (YeeUpdates.hpp:396-405) for flux F[c] of field type
 * ft with the summed curl terms `curl`: F = TimePolicy::get(F) + Coeff *
 * curl_coeff * dt * curl, then TimePolicy::increment shifts the history
 * (BD3: :209-213, :231-236; BD4: :258-263, :282-288). */
static void yee_flux(oracle_grid* g, int ft, int I, size_t c, double curl) {
  double* F = ft == 0 ? g->D[I] : g->B[I];
  double coeff = ft == 0 ? 1.0 : -1.0;
  double hold = F[c];
  if (g->scheme == 1) {
    F[c] = F[c] + coeff * 1.0 * g->dt * curl;
    return;
  }
  double* h0 = g->hist[ft][0][I];
  double* h1 = g->hist[ft][1][I];
  if (g->scheme == 3) {
    double get = 21.0 / 23.0 * F[c] + 3.0 / 23.0 * h0[c] - 1.0 / 23.0 * h1[c];
    F[c] = get + coeff * (24.0 / 23.0) * g->dt * curl;
    h1[c] = h0[c];
    h0[c] = hold;
  } else {
    double* h2 = g->hist[ft][2][I];
    double get = 17.0 / 22.0 * F[c] + 9.0 / 22.0 * h0[c] - 5.0 / 22.0 * h1[c] + 1.0 / 22.0 * h2[c];
    F[c] = get + coeff * (24.0 / 22.0) * g->dt * curl;
    h2[c] = h1[c];
    h1[c] = h0[c];
    h0[c] = hold;
  }
}

int oracle_set_eps_map(oracle_grid* g, const double* eps) {
  if (!eps) {
    free(g->eps_map);
    g->eps_map = NULL;
    return 0;
  }
  if (!g->eps_map) g->eps_map = zalloc(g->ncell);
  memcpy(g->eps_map, eps, g->ncell * sizeof(double));
  return 0;
}

/* Aux1D (include/Source.hpp:280-462): TEM grid of ncells + 2*15 + 20 cells,
 * fixed 15-cell CPML graded like the main grid, source at cell 20. */
#define AUX_NPML 15
int oracle_add_tfsf_plane(oracle_grid* g, int axis, int orient, const int* lo, const int* hi,
                          const double* origin, const double* kvec, const double* pol_e,
                          const double* pol_h, int aux_ncells, const double* aux_vals, int naux) {
  int dim = g->mode == THREED ? 3 : 2;
  if (axis < 0 || axis >= dim || aux_ncells < 1) return -1;
  g->planes = (plane_t*)realloc(g->planes, (g->nplanes + 1) * sizeof(plane_t));
  plane_t* p = &g->planes[g->nplanes++];
  memset(p, 0, sizeof(*p));
  p->axis = axis; p->orient = orient;
  for (int d = 0; d < 3; d++) {
    p->lo[d] = lo[d]; p->hi[d] = hi[d]; p->origin[d] = origin[d];
    p->pol_e[d] = pol_e[d]; p->pol_h[d] = pol_h[d];
    p->normal[d] = 0;
  }
  p->normal[axis] = orient == 1 ? 1 : -1;
  /* TFSFPlane constructor: normalise normal and k over the mode's dims
   * (include/Source.hpp:560-570) */
  double N = 0;
  for (int d = 0; d < dim; d++) N += p->normal[d] * p->normal[d];
  N = sqrt(N);
  for (int d = 0; d < dim; d++) p->normal[d] /= N;
  double K = 0;
  for (int d = 0; d < dim; d++) K += kvec[d] * kvec[d];
  K = sqrt(K);
  for (int d = 0; d < 3; d++) p->k[d] = d < dim ? kvec[d] / K : 0.0;
  int L = aux_ncells + 2 * AUX_NPML + 20;
  p->L = L;
  p->Dz = zalloc(L); p->Ez = zalloc(L); p->By = zalloc(L); p->Hy = zalloc(L);
  p->psiE = zalloc(L); p->psiH = zalloc(L);
  for (int f = 0; f < 2; f++) {
    p->pB[f] = zalloc(L); p->pC[f] = zalloc(L); p->pF[f] = zalloc(L); p->pG[f] = zalloc(L);
    for (int i = 0; i < L; i++) p->pF[f][i] = 1.0;
  }
  /* Aux1D::setup_tasks (Source.hpp:380-389): both sides in one loop */
  pml_model pm = model_for(g->dx);
  for (int i = 1; i < AUX_NPML + 2; i++) {
    double x = (double)(AUX_NPML - i + 1) / (double)AUX_NPML;
    double xm = x - 0.5 / (double)AUX_NPML;
    set_params(mK(&pm, x), mS(&pm, x), mA(&pm, x), g->dt, &p->pB[0][i], &p->pC[0][i], &p->pF[0][i], &p->pG[0][i]);
    set_params(mK(&pm, xm), mS(&pm, xm), mA(&pm, xm), g->dt, &p->pB[1][i], &p->pC[1][i], &p->pF[1][i], &p->pG[1][i]);
    set_params(mK(&pm, x), mS(&pm, x), mA(&pm, x), g->dt, &p->pB[0][L - i], &p->pC[0][L - i], &p->pF[0][L - i], &p->pG[0][L - i]);
    set_params(mK(&pm, xm), mS(&pm, xm), mA(&pm, xm), g->dt, &p->pB[1][L - 1 - i], &p->pC[1][L - 1 - i], &p->pF[1][L - 1 - i], &p->pG[1][L - 1 - i]);
  }
  p->vals = zalloc(naux);
  memcpy(p->vals, aux_vals, naux * sizeof(double));
  p->nvals = naux;
  p->t = 0;
  return 0;
}

/* Aux1D::time_step (Source.hpp:413-435). Cells 0 and L-1 see zero ghosts. */
static void aux_step(plane_t* p, double dt, double dx) {
  int L = p->L;
  p->t += dt;
  /* the source value is looked up by aux step number, s = round(t/dt) */
  long s = lround(p->t / dt);
  /* YeeUpdate<TEM,Dz>: Dz + dt*(a<X> + 0.0) */
  for (int i = 0; i < L; i++) {
    double hm = i > 0 ? p->Hy[i - 1] : 0.0;
    double a = 1 * p->pF[0][i] / dx * (p->Hy[i] - hm);
    p->Dz[i] = p->Dz[i] + 1.0 * 1.0 * dt * (a + 0.0);
  }
  /* UpdatePML<TEM, Electric, X> */
  for (int i = 0; i < L; i++) {
    double hm = i > 0 ? p->Hy[i - 1] : 0.0;
    p->Dz[i] += 1.0 * dt * p->psiE[i] * p->pG[0][i];
    p->psiE[i] = p->pB[0][i] * p->psiE[i] + p->pC[0][i] * 1 / dx * (p->Hy[i] - hm);
  }
  for (int i = 0; i < L; i++) p->Ez[i] = p->Dz[i] / (1.0 * k_eps0);
  p->Ez[AUX_NPML + 5] += (s >= 1 && s <= p->nvals) ? p->vals[s - 1] : 0.0;
  /* YeeUpdate<TEM,By>: By + (-dt)*(0.0 + a<X>), a<X> = -F/dx*(Ez[+1]-Ez) */
  for (int i = 0; i < L; i++) {
    double ep = i < L - 1 ? p->Ez[i + 1] : 0.0;
    double a = -1 * p->pF[1][i] / dx * (ep - p->Ez[i]);
    p->By[i] = p->By[i] + -1.0 * 1.0 * dt * (0.0 + a);
  }
  /* UpdatePML<TEM, Magnetic, X> */
  for (int i = 0; i < L; i++) {
    double ep = i < L - 1 ? p->Ez[i + 1] : 0.0;
    p->By[i] += -1.0 * dt * p->psiH[i] * p->pG[1][i];
    p->psiH[i] = p->pB[1][i] * p->psiH[i] + p->pC[1][i] * -1 / dx * (ep - p->Ez[i]);
  }
  for (int i = 0; i < L; i++) p->Hy[i] = p->By[i] / (1.0 * K_MU0);
}

/* Aux1D::interpolateE / interpolateH (Source.hpp:442-458) */
static double interp(const double* f, int L, double loc, double dx, double shift) {
  double nd = (double)L / 2.0 + loc / dx - shift;
  size_t n = (size_t)nd;
  double frac = (nd - n);
  (void)L;
  return (1.0 - frac) * f[n] + frac * f[n + 1];
}

/* Yee staggering offsets, include/FDTDConstants.hpp:680-744 */
static const double offE[3][3] = {{0.0, -0.5, -0.5}, {-0.5, 0.0, -0.5}, {-0.5, -0.5, 0.0}};
static const double offH[3][3] = {{-0.5, 0.0, 0.0}, {0.0, -0.5, 0.0}, {0.0, 0.0, -0.5}};

/* TFSFPlane::field_update (Source.hpp:489-554), applied to one flux component
 * I of type ft (0 = D, 1 = B) at cell (i,j,k). */
static void tfsf_cell(oracle_grid* g, plane_t* p, int ft, int I, int i, int j, int k) {
  int dim = g->mode == THREED ? 3 : 2;
  int idx3[3] = {i, j, k};
  size_t c = ((size_t)k * g->n[1] + j) * g->n[0] + i;
  int d1 = I == 0 ? 1 : (I == 1 ? 2 : 0);
  int d2 = third(I, d1);
  int ds[2] = {d1, d2};
  double terms[2];
  for (int q = 0; q < 2; q++) {
    int J = ds[q], K = third(I, J);
    int present = ft == 0 ? g->hasH[K] : g->hasE[K];
    if (!present) { terms[q] = 0.0; continue; }
    const double* off = ft == 0 ? offH[K] : offE[K];
    double center[3], src[3];
    for (int d = 0; d < dim; d++) center[d] = ((double)idx3[d] - p->origin[d]) * g->dx;
    for (int d = 0; d < dim; d++) src[d] = center[d] + off[d] * g->dx;
    double proj = 0;
    for (int d = 0; d < dim; d++) proj += p->k[d] * src[d];
    double sv = ft == 0 ? interp(p->Hy, p->L, proj, g->dx, 0.5) : interp(p->Ez, p->L, proj, g->dx, 0.0);
    double Fj = g->cF[ft][J][idx3[J]];
    const double* pol = ft == 0 ? p->pol_h : p->pol_e;
    terms[q] = lc(I, J, K) * Fj / (g->dx) * p->normal[J] * sv * pol[K];
  }
  double coeff = ft == 0 ? 1.0 : -1.0;
  double* F = ft == 0 ? g->D[I] : g->B[I];
  F[c] += coeff * curl_coeff(g->scheme) * g->dt * (terms[0] + terms[1]);
}

static void tfsf_apply(oracle_grid* g, int ft) {
  for (int q = 0; q < g->nplanes; q++) {
    plane_t* p = &g->planes[q];
    for (int k = p->lo[2]; k <= p->hi[2]; k++)
      for (int j = p->lo[1]; j <= p->hi[1]; j++)
        for (int i = p->lo[0]; i <= p->hi[0]; i++)
          for (int I = 2; I >= 0; I--) {
            int present = ft == 0 ? g->hasE[I] : g->hasH[I];
            if (present) tfsf_cell(g, p, ft, I, i, j, k);
          }
    if (ft == 0) aux_step(p, g->dt, g->dx); /* updateD advances the aux grid */
  }
}

/* Quantities of a cell, by code: 0..2 E, 3..5 H, 6..8 the surface current
 * Je (UpdateSurfaceCurrentE, SurfaceQuantities.hpp:256-296), 9..11 Jh
 * (UpdateSurfaceCurrentH, :315-356), 12 the surface charge density rho
 * (UpdateSurfaceChargeDensity, :203-242), each in the reference's operation
 * order. Je reads H at the cell and its lower neighbours, Jh reads E at the
 * cell and its upper neighbours, rho reads E at the cell and its lower
 * neighbours. */
static int quantity_present(const oracle_grid* g, int q) {
  if (q < 0 || q > 12) return 0;
  if (q < 3) return g->hasE[q];
  if (q < 6) return g->hasH[q - 3];
  if (q < 9) return g->hasE[q - 6];
  if (q < 12) return g->hasH[q - 9];
  return g->mode != TM;
}

static double quantity_at(const oracle_grid* g, int q, size_t c) {
  const size_t sy = (size_t)g->n[0], sz = (size_t)g->n[0] * g->n[1];
  const double dx = g->dx;
  double* const* E = g->E;
  double* const* H = g->H;
  if (q < 3) return E[q][c];
  if (q < 6) return H[q - 3][c];
  if (q < 9) {
    if (g->mode == TE) {
      if (q == 6) return 1.0 / dx * (H[2][c] - H[2][c - sy]);
      return 1.0 / dx * (-H[2][c] + H[2][c - 1]);
    }
    if (q == 6) return 1.0 / dx * (H[2][c] - H[2][c - sy] - H[1][c] + H[1][c - sz]);
    if (q == 7) return 1.0 / dx * (H[0][c] - H[0][c - sz] - H[2][c] + H[2][c - 1]);
    return 1.0 / dx * (H[1][c] - H[1][c - 1] - H[0][c] + H[0][c - sy]);
  }
  if (q < 12) {
    if (g->mode == TM) {
      if (q == 9) return -1.0 / dx * (E[2][c + sy] - E[2][c]);
      return -1.0 / dx * (-E[2][c + 1] + E[2][c]);
    }
    if (q == 9) return -1.0 / dx * (E[2][c + sy] - E[2][c] - E[1][c + sz] + E[1][c]);
    if (q == 10) return -1.0 / dx * (E[0][c + sz] - E[0][c] - E[2][c + 1] + E[2][c]);
    return -1.0 / dx * (E[1][c + 1] - E[1][c] - E[0][c + sy] + E[0][c]);
  }
  if (g->mode == TE) return k_eps0 / dx * (E[0][c] + E[1][c] - E[0][c - 1] - E[1][c - sy]);
  return k_eps0 / dx * (E[0][c] + E[1][c] + E[2][c] - E[0][c - 1] - E[1][c - sy] - E[2][c - sz]);
}

/* the box must lie in the interior (the quantities read +-1 neighbours) */
static int quantity_box_ok(const oracle_grid* g, int q, const int* lo, const int* hi) {
  int dim = g->mode == THREED ? 3 : 2;
  for (int d = 0; d < 3; d++) {
    if (lo[d] > hi[d]) return 0;
    if (q < 6) {
      if (lo[d] < 0 || hi[d] >= g->n[d]) return 0;
    } else if (d < dim) {
      if (lo[d] < 1 || hi[d] > g->n[d] - 2) return 0;
    } else if (lo[d] != 0 || hi[d] != 0) return 0;
  }
  return quantity_present(g, q);
}

int oracle_read_quantity(const oracle_grid* g, int q, const int* lo, const int* hi, double* out) {
  if (!quantity_box_ok(g, q, lo, hi)) return -1;
  size_t p = 0;
  for (int k = lo[2]; k <= hi[2]; k++)
    for (int j = lo[1]; j <= hi[1]; j++)
      for (int i = lo[0]; i <= hi[0]; i++) out[p++] = quantity_at(g, q, ((size_t)k * g->n[1] + j) * g->n[0] + i);
  return 0;
}

/* phase of a quantity's samples: 0 (after the E half: E, Jh, rho) or 1 (after
 * the H half: H, Je) */
static int quantity_phase(int q) { return (q >= 3 && q < 9) ? 1 : 0; }

static void dft_apply(oracle_grid* g, int ft, double n) {
  for (int d = 0; d < g->ndft; d++) {
    dft_t* r = &g->dfts[d];
    if (quantity_phase(r->comp) != ft) continue;
    for (int f = 0; f < r->nf; f++) {
      double ph = 2.0 * k_pi * r->freqs[f] * n;
      double wr = cos(ph), wi = -sin(ph);
      int p = 0;
      for (int k = r->lo[2]; k <= r->hi[2]; k++)
        for (int j = r->lo[1]; j <= r->hi[1]; j++)
          for (int i = r->lo[0]; i <= r->hi[0]; i++, p++) {
            double v = quantity_at(g, r->comp, ((size_t)k * g->n[1] + j) * g->n[0] + i);
            r->acc[((size_t)f * r->npts + p) * 2] += v * wr;
            r->acc[((size_t)f * r->npts + p) * 2 + 1] += v * wi;
          }
    }
  }
}

int oracle_add_dft(oracle_grid* g, int comp, const int* lo, const int* hi, const double* freqs, int nf) {
  if (comp < 0 || comp > 12 || nf < 1) return -1;
  if (comp < 6) {
    for (int d = 0; d < 3; d++)
      if (lo[d] < 0 || hi[d] >= g->n[d] || lo[d] > hi[d]) return -1;
  } else if (!quantity_box_ok(g, comp, lo, hi)) return -1;
  g->dfts = (dft_t*)realloc(g->dfts, (g->ndft + 1) * sizeof(dft_t));
  dft_t* r = &g->dfts[g->ndft];
  r->comp = comp; r->nf = nf;
  r->npts = 1;
  for (int d = 0; d < 3; d++) { r->lo[d] = lo[d]; r->hi[d] = hi[d]; r->npts *= hi[d] - lo[d] + 1; }
  r->freqs = zalloc(nf);
  memcpy(r->freqs, freqs, nf * sizeof(double));
  r->acc = zalloc((size_t)nf * r->npts * 2);
  return g->ndft++;
}

int oracle_dft_npoints(const oracle_grid* g, int handle) {
  if (handle < 0 || handle >= g->ndft) return -1;
  return g->dfts[handle].npts;
}

int oracle_dft_get(const oracle_grid* g, int handle, double* out) {
  if (handle < 0 || handle >= g->ndft) return -1;
  const dft_t* r = &g->dfts[handle];
  memcpy(out, r->acc, (size_t)r->nf * r->npts * 2 * sizeof(double));
  return 0;
}

/* one half step: phase 0 = the E half, 1 = the H half (which ends the step) */
static void step_half(oracle_grid* g, int phase) {
  const int nx = g->n[0], ny = g->n[1], nz = g->n[2];
  const int three = g->mode == THREED;
  const double dt = g->dt, dx = g->dx;
  const size_t sx = 1, sy = (size_t)nx, sz = (size_t)nx * ny;
  const size_t str[3] = {sx, sy, sz};
  const int k0 = three ? 1 : 0, k1 = three ? nz - 2 : 0;
  int pmlax[3];
  for (int a = 0; a < 3; a++) pmlax[a] = g->pml[a][0] > 0 || g->pml[a][1] > 0;

  if (phase == 1) goto h_half;
  /* ---------------- E half step ---------------- */
  for (int k = k0; k <= k1; k++)
    for (int j = 1; j <= ny - 2; j++)
      for (int i = 1; i <= nx - 2; i++) {
        size_t c = k * sz + j * sy + i;
        int idx[3] = {i, j, k};
        /* YeeUpdate::update_all (YeeUpdates.hpp:396-405) on each E flux */
        for (int I = 0; I < 3; I++) {
          if (!g->hasE[I]) continue;
          int d1 = I == 0 ? 1 : (I == 1 ? 2 : 0);
          int d2 = third(I, d1);
          int ds[2] = {d1, d2};
          double a[2];
          for (int q = 0; q < 2; q++) {
            int J = ds[q], K = third(I, J);
            if (!g->hasH[K]) { a[q] = 0.0; continue; }
            /* atomic_update::get (:373-377); H difference (:107-113) */
            double diff = g->H[K][c] - g->H[K][c - str[J]];
            a[q] = lc(I, J, K) * g->cF[0][J][idx[J]] / (dx) * diff;
          }
          yee_flux(g, 0, I, c, a[0] + a[1]);
        }
      }
  tfsf_apply(g, 0);
  for (int s = 0; s < g->nsrc; s++) {
    src_t* sr = &g->srcs[s];
    if (sr->target != 1 || !g->hasE[sr->comp]) continue;
    size_t c = sr->k * sz + sr->j * sy + sr->i;
    g->D[sr->comp][c] += g->t < sr->nvals ? sr->vals[g->t] : 0.0;
  }
  /* UpdatePML<Mode, Electric, J> (PML.hpp:306-329) per axis, in X, Y, Z order */
  for (int J = 0; J < 3; J++) {
    if (!pmlax[J]) continue;
    for (int k = k0; k <= k1; k++)
      for (int j = 1; j <= ny - 2; j++)
        for (int i = 1; i <= nx - 2; i++) {
          size_t c = k * sz + j * sy + i;
          int idx[3] = {i, j, k};
          for (int I = 2; I >= 0; I--) {
            if (!g->hasE[I] || I == J) continue;
            int K = third(I, J);
            double* ps = &g->psi[0][I][J][c];
            g->D[I][c] += 1.0 * dt * *ps * g->cG[0][J][idx[J]];
            double diff = g->H[K][c] - g->H[K][c - str[J]];
            *ps = g->cB[0][J][idx[J]] * *ps + g->cC[0][J][idx[J]] * lc(I, J, K) / dx * diff;
          }
        }
  }
  /* material update (DispersiveMaterials.hpp:354-359, :710-735, :979-998) */
  for (int k = k0; k <= k1; k++)
    for (int j = 1; j <= ny - 2; j++)
      for (int i = 1; i <= nx - 2; i++) {
        size_t c = k * sz + j * sy + i;
        const oracle_material* m = &g->mats[g->ids ? g->ids[c] : 0];
        for (int I = 2; I >= 0; I--) {
          if (!g->hasE[I]) continue;
          double* D = &g->D[I][c];
          double* E = &g->E[I][c];
          if (m->kind <= OR_CONSTANT && g->eps_map && g->eps_map[c] > 0.0) {
            /* a per-cell ConstantUpdate<Mode, Electric>(K) */
            *E = *D / (g->eps_map[c] * k_eps0);
          } else if (m->kind == OR_VACUUM) {
            *E = *D / (1.0 * k_eps0);
          } else if (m->kind == OR_CONSTANT) {
            *E = *D / (m->eps_inf * k_eps0);
          } else if (m->kind == OR_DRUDE) {
            double* P = &g->P[0][I][c];
            double* Jc = &g->J[0][I][c];
            double b = m->gamma[0] * dt * 0.5;
            double w = dt * m->freq[0];
            *P += dt * *Jc;
            *E = (*D - *P) / (m->eps_inf * k_eps0);
            *Jc = *Jc * (1.0 - b) / (1.0 + b) + w * w / dt * k_eps0 * *E;
          } else { /* Lorentz, generalised to npoles with strength delta_eps */
            double num = *D;
            for (int q = 0; q < m->npoles; q++) {
              g->P[q][I][c] += dt * g->J[q][I][c];
              num = num - g->P[q][I][c];
            }
            *E = num / (m->eps_inf * k_eps0);
            for (int q = 0; q < m->npoles; q++) {
              double b = 1.0 + m->gamma[q] * dt;
              double bm = 1.0 - m->gamma[q] * dt;
              double w = m->freq[q] * dt;
              double qq = m->freq[q] * w / b;
              double* Jc = &g->J[q][I][c];
              *Jc = bm / b * *Jc + qq * m->delta_eps[q] * k_eps0 * *E - qq * g->P[q][I][c];
            }
          }
        }
      }
  for (int s = 0; s < g->nsrc; s++) {
    src_t* sr = &g->srcs[s];
    if (sr->target != 0 || !g->hasE[sr->comp]) continue;
    size_t c = sr->k * sz + sr->j * sy + sr->i;
    g->E[sr->comp][c] += g->t < sr->nvals ? sr->vals[g->t] : 0.0;
  }
  apply_boxes(g, 0);
  apply_boundaries(g, 0);
  dft_apply(g, 0, (double)(g->t + 1));
  return;

h_half:
  /* ---------------- H half step ---------------- */
  for (int k = k0; k <= k1; k++)
    for (int j = 1; j <= ny - 2; j++)
      for (int i = 1; i <= nx - 2; i++) {
        size_t c = k * sz + j * sy + i;
        int idx[3] = {i, j, k};
        for (int I = 0; I < 3; I++) {
          if (!g->hasH[I]) continue;
          int d1 = I == 0 ? 1 : (I == 1 ? 2 : 0);
          int d2 = third(I, d1);
          int ds[2] = {d1, d2};
          double a[2];
          for (int q = 0; q < 2; q++) {
            int J = ds[q], K = third(I, J);
            if (!g->hasE[K]) { a[q] = 0.0; continue; }
            /* E difference (YeeUpdates.hpp:98-103) */
            double diff = g->E[K][c + str[J]] - g->E[K][c];
            a[q] = lc(I, J, K) * g->cF[1][J][idx[J]] / (dx) * diff;
          }
          yee_flux(g, 1, I, c, a[0] + a[1]);
        }
      }
  tfsf_apply(g, 1);
  for (int s = 0; s < g->nsrc; s++) {
    src_t* sr = &g->srcs[s];
    if (sr->target != 3 || !g->hasH[sr->comp]) continue;
    size_t c = sr->k * sz + sr->j * sy + sr->i;
    g->B[sr->comp][c] += g->t < sr->nvals ? sr->vals[g->t] : 0.0;
  }
  for (int J = 0; J < 3; J++) {
    if (!pmlax[J]) continue;
    for (int k = k0; k <= k1; k++)
      for (int j = 1; j <= ny - 2; j++)
        for (int i = 1; i <= nx - 2; i++) {
          size_t c = k * sz + j * sy + i;
          int idx[3] = {i, j, k};
          for (int I = 2; I >= 0; I--) {
            if (!g->hasH[I] || I == J) continue;
            int K = third(I, J);
            double* ps = &g->psi[1][I][J][c];
            g->B[I][c] += -1.0 * dt * *ps * g->cG[1][J][idx[J]];
            double diff = g->E[K][c + str[J]] - g->E[K][c];
            *ps = g->cB[1][J][idx[J]] * *ps + g->cC[1][J][idx[J]] * lc(I, J, K) / dx * diff;
          }
        }
  }
  for (int k = k0; k <= k1; k++)
    for (int j = 1; j <= ny - 2; j++)
      for (int i = 1; i <= nx - 2; i++) {
        size_t c = k * sz + j * sy + i;
        const oracle_material* m = &g->mats[g->ids ? g->ids[c] : 0];
        for (int I = 2; I >= 0; I--) {
          if (!g->hasH[I]) continue;
          g->H[I][c] = g->B[I][c] / (m->mu_r * K_MU0);
        }
      }
  for (int s = 0; s < g->nsrc; s++) {
    src_t* sr = &g->srcs[s];
    if (sr->target != 2 || !g->hasH[sr->comp]) continue;
    size_t c = sr->k * sz + sr->j * sy + sr->i;
    g->H[sr->comp][c] += g->t < sr->nvals ? sr->vals[g->t] : 0.0;
  }
  apply_boxes(g, 2);
  apply_boundaries(g, 1);
  dft_apply(g, 1, (double)g->t + 1.5);
  g->t++;
}

static void step_one(oracle_grid* g) {
  step_half(g, 0);
  step_half(g, 1);
}

int oracle_step(oracle_grid* g, int nsteps) {
  for (int s = 0; s < nsteps; s++) step_one(g);
  return 0;
}

/* The forward (explicit) material updates, XUpdate<Mode, ft, forward = true>
   (DispersiveMaterials.hpp:345-349 constant and vacuum, :922-934 Drude): the
   flux -- and the Drude P and J -- from the field, on every interior cell.
   The reference's Lorentz explicit update is a static_assert (:697-706):
   grids with a Lorentz material are refused (-2). */
int oracle_material_explicit(oracle_grid* g, int ft) {
  if (ft != 0 && ft != 1) return -1;
  for (int q = 0; q < g->nmat; q++)
    if (ft == 0 && g->mats[q].kind == OR_LORENTZ) return -2;
  const int nx = g->n[0], ny = g->n[1], nz = g->n[2];
  const size_t sy = nx, sz = (size_t)nx * ny;
  const int k0 = g->mode == THREED ? 1 : 0, k1 = g->mode == THREED ? nz - 2 : 0;
  const double dt = g->dt;
  for (int k = k0; k <= k1; k++)
    for (int j = 1; j <= ny - 2; j++)
      for (int i = 1; i <= nx - 2; i++) {
        size_t c = k * sz + j * sy + i;
        const oracle_material* m = &g->mats[g->ids ? g->ids[c] : 0];
        for (int I = 2; I >= 0; I--) {
          if (ft == 1) {
            if (g->hasH[I]) g->B[I][c] = m->mu_r * K_MU0 * g->H[I][c];
            continue;
          }
          if (!g->hasE[I]) continue;
          const double E = g->E[I][c];
          if (m->kind <= OR_CONSTANT) {
            const double K = (g->eps_map && g->eps_map[c] > 0.0) ? g->eps_map[c]
                             : (m->kind == OR_VACUUM ? 1.0 : m->eps_inf);
            g->D[I][c] = K * k_eps0 * E;
          } else { /* Drude */
            double* P = &g->P[0][I][c];
            double* Jc = &g->J[0][I][c];
            double b = m->gamma[0] * dt;
            double cc = dt * m->freq[0] * m->freq[0] * k_eps0;
            *P = (-dt * *Jc + (1.0 + b) * *P) / (1.0 + b);
            *Jc = (*Jc - cc * E) / (1.0 + b);
            g->D[I][c] = m->eps_inf * k_eps0 * E + *P;
          }
        }
      }
  return 0;
}

int oracle_step_half(oracle_grid* g, int phase) {
  if (phase != 0 && phase != 1) return -1;
  step_half(g, phase);
  return 0;
}

static double* which_ptr(const oracle_grid* g, int which) {
  if (which < 0) return NULL;
  if (which < 3) return g->D[which];
  if (which < 6) return g->E[which - 3];
  if (which < 9) return g->B[which - 6];
  if (which < 12) return g->H[which - 9];
  if (which < 15) return g->P[0][which - 12];
  if (which < 18) return g->J[0][which - 15];
  if (which < 36) { int q = which - 18; return g->psi[q / 9][(q / 3) % 3][q % 3]; }
  int q = which - 36, pole = 1 + q / 6, r = q % 6;
  if (pole >= OR_MAX_POLES) return NULL;
  return r < 3 ? g->P[pole][r] : g->J[pole][r - 3];
}

int oracle_get(const oracle_grid* g, int which, double* out) {
  double* p = which_ptr(g, which);
  if (!p) return -1;
  memcpy(out, p, g->ncell * sizeof(double));
  return 0;
}

int oracle_set(oracle_grid* g, int which, const double* in) {
  double* p = which_ptr(g, which);
  if (!p) return -1;
  memcpy(p, in, g->ncell * sizeof(double));
  return 0;
}

/* ------------------------------------------------------------------------
 * FP64 discrete adjoint of the TM step above (oracle_step), for
 *   J = sum over the probe box of |X|^2,  X = the DFT of Ez at `freq`
 *       (cycles per step; E samples at n = t + 1, as dft_apply),
 * and its gradient with respect to the relative permittivity of every cell
 * of the design box. It runs the forward itself from a fresh grid (t = 0),
 * keeping D_z of the design cells after every step, then walks the steps
 * backwards through the transpose of each update in reverse order:
 *   H half:  B_x' = B_x - dt (F/dx diff_xy + G psi_xy),  psi_xy' = B psi_xy + C/dx diff_xy
 *            (diff_xy = E_z[+y] - E_z), and likewise B_y with diff_yx = E_z[+x] - E_z
 *            entering with the Levi-Civita sign -1; H = B / mu0.
 *   E half:  D_z' = D_z + dt (F_x/dx diff_zx - F_y/dx diff_zy) + dt (G_x psi_zx + G_y psi_zy)
 *            (old psi), psi_zx' = B_x psi_zx + C_x/dx diff_zx, psi_zy' = B_y psi_zy - C_y/dx diff_zy,
 *            E_z = D_z' / (eps_r eps0)  =>  dJ/deps_r += lambda_E * (-D_z' / (eps_r^2 eps0)).
 * Sources are affine in the state and drop out. Supported: TM, non-dispersive
 * materials with mu_r = 1, no TFSF planes. Test infrastructure only. */
int oracle_adjoint_tm(oracle_grid* g, int nsteps, const int* plo, const int* phi, double freq, const int* dlo,
                      const int* dhi, double* J_out, double* grad) {
  if (g->mode != TM || g->t != 0 || g->nplanes > 0 || nsteps < 1 || g->scheme != 1) return -1;
  for (int m = 0; m < g->nmat; m++)
    if (g->mats[m].kind > OR_CONSTANT || g->mats[m].mu_r != 1.0) return -1;
  for (int d = 0; d < 2; d++)
    if (dlo[d] < 1 || dhi[d] > g->n[d] - 2 || dlo[d] > dhi[d]) return -1;
  const int nx = g->n[0], ny = g->n[1];
  const size_t sy = (size_t)nx, nc = g->ncell;
  const double dt = g->dt, dx = g->dx;
  int lo3[3] = {plo[0], plo[1], 0}, hi3[3] = {phi[0], phi[1], 0};
  const int h = oracle_add_dft(g, 2, lo3, hi3, &freq, 1);
  if (h < 0) return -1;
  const int dw = dhi[0] - dlo[0] + 1, nd = dw * (dhi[1] - dlo[1] + 1);
  double* Dst = zalloc((size_t)nsteps * nd);
  double* eps = zalloc(nd);
  for (int q = 0; q < nd; q++) {
    size_t c = (size_t)(dlo[1] + q / dw) * sy + dlo[0] + q % dw;
    const oracle_material* m = &g->mats[g->ids ? g->ids[c] : 0];
    eps[q] = (g->eps_map && g->eps_map[c] > 0.0) ? g->eps_map[c] : (m->kind == OR_VACUUM ? 1.0 : m->eps_inf);
  }
  for (int t = 0; t < nsteps; t++) {
    step_one(g);
    for (int q = 0; q < nd; q++) Dst[(size_t)t * nd + q] = g->D[2][(size_t)(dlo[1] + q / dw) * sy + dlo[0] + q % dw];
  }
  const dft_t* r = &g->dfts[h];
  double J = 0.0;
  for (int p = 0; p < r->npts; p++) J += r->acc[2 * p] * r->acc[2 * p] + r->acc[2 * p + 1] * r->acc[2 * p + 1];
  *J_out = J;

  double *lD = zalloc(nc), *lBx = zalloc(nc), *lBy = zalloc(nc), *lE = zalloc(nc);
  double *lpzx = zalloc(nc), *lpzy = zalloc(nc), *lpxy = zalloc(nc), *lpyx = zalloc(nc);
  double *qxy = zalloc(nc), *qyx = zalloc(nc), *qzx = zalloc(nc), *qzy = zalloc(nc);
  const double *eF[2] = {g->cF[0][0], g->cF[0][1]}, *eG[2] = {g->cG[0][0], g->cG[0][1]};
  const double *eB[2] = {g->cB[0][0], g->cB[0][1]}, *eC[2] = {g->cC[0][0], g->cC[0][1]};
  const double *hF[2] = {g->cF[1][0], g->cF[1][1]}, *hG[2] = {g->cG[1][0], g->cG[1][1]};
  const double *hB[2] = {g->cB[1][0], g->cB[1][1]}, *hC[2] = {g->cC[1][0], g->cC[1][1]};
  for (int q = 0; q < nd; q++) grad[q] = 0.0;
  for (int t = nsteps - 1; t >= 0; t--) {
    /* H half, reversed: adjoints of diff_xy (qxy) and diff_yx (qyx) */
    for (int j = 1; j <= ny - 2; j++)
      for (int i = 1; i <= nx - 2; i++) {
        size_t c = j * sy + i;
        qxy[c] = -dt * hF[1][j] / dx * lBx[c] + hC[1][j] / dx * lpxy[c];
        lpxy[c] = -dt * hG[1][j] * lBx[c] + hB[1][j] * lpxy[c];
        qyx[c] = dt * hF[0][i] / dx * lBy[c] - hC[0][i] / dx * lpyx[c];
        lpyx[c] = -dt * hG[0][i] * lBy[c] + hB[0][i] * lpyx[c];
      }
    const double ph = 2.0 * k_pi * freq * (double)(t + 1);
    const double cs = cos(ph), sn = sin(ph);
    for (int j = 1; j <= ny - 2; j++)
      for (int i = 1; i <= nx - 2; i++) {
        size_t c = j * sy + i;
        double v = qxy[c - sy] - qxy[c] + qyx[c - 1] - qyx[c];
        if (i >= plo[0] && i <= phi[0] && j >= plo[1] && j <= phi[1]) {
          int p = (j - plo[1]) * (phi[0] - plo[0] + 1) + (i - plo[0]);
          v += 2.0 * (r->acc[2 * p] * cs - r->acc[2 * p + 1] * sn);
        }
        lE[c] = v;
      }
    /* E half, reversed */
    for (int j = 1; j <= ny - 2; j++)
      for (int i = 1; i <= nx - 2; i++) {
        size_t c = j * sy + i;
        const oracle_material* m = &g->mats[g->ids ? g->ids[c] : 0];
        double e = (g->eps_map && g->eps_map[c] > 0.0) ? g->eps_map[c] : (m->kind == OR_VACUUM ? 1.0 : m->eps_inf);
        if (i >= dlo[0] && i <= dhi[0] && j >= dlo[1] && j <= dhi[1]) {
          int q = (j - dlo[1]) * dw + (i - dlo[0]);
          grad[q] += lE[c] * (-Dst[(size_t)t * nd + q] / (e * e * k_eps0));
        }
        lD[c] += lE[c] / (e * k_eps0);
        qzx[c] = eC[0][i] / dx * lpzx[c] + dt * eF[0][i] / dx * lD[c];
        lpzx[c] = dt * eG[0][i] * lD[c] + eB[0][i] * lpzx[c];
        qzy[c] = -eC[1][j] / dx * lpzy[c] - dt * eF[1][j] / dx * lD[c];
        lpzy[c] = dt * eG[1][j] * lD[c] + eB[1][j] * lpzy[c];
      }
    for (int j = 1; j <= ny - 2; j++)
      for (int i = 1; i <= nx - 2; i++) {
        size_t c = j * sy + i;
        lBy[c] += (qzx[c] - qzx[c + 1]) / K_MU0;
        lBx[c] += (qzy[c] - qzy[c + sy]) / K_MU0;
      }
  }
  free(lD); free(lBx); free(lBy); free(lE); free(lpzx); free(lpzy); free(lpxy); free(lpyx);
  free(qxy); free(qyx); free(qzx); free(qzy); free(Dst); free(eps);
  return 0;
}
