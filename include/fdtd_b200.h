/* fdtd_b200: C ABI of the B200 (sm_100a) implementation of pederson/fdtd's
 * time-step hot path.
 *
 * The reference has no ABI: a user owns an AoS container of YeeCell objects
 * and applies compile-time update functors to it in a time loop
 * (tests/testTM.cpp:102-113). Each entry point below replaces one piece of
 * that loop, for a whole grid held as SoA arrays in device memory:
 *
 *   reference                                              here
 *   ---------------------------------------------------    ----------------------------
 *   container of YeeCell<YeeFields<Mode,..>, ..>            fdtd_grid_create
 *     (include/YeeCell.hpp:74-97, YeeFields.hpp:37-174)
 *   PMLParameterModel(dx) + NewPML::setPMLParameters per     fdtd_set_pml
 *     cell (PML.hpp:84-102, :368-393; testTM.cpp:44-71)
 *   Vacuum/Constant/Drude/LorentzUpdate functor per cell     fdtd_set_materials,
 *     (DispersiveMaterials.hpp:489-497, :881-884,            fdtd_set_material_ids,
 *     :1208-1211; MaterialMap.hpp:45-70)                     fdtd_set_material_blocks
 *   SoftSource<Signal,Cell,GetField<F>>::apply(t)            fdtd_add_source
 *     (Source.hpp:183-261)
 *   make_tfsf_plane + Aux1D (Source.hpp:280-634)             fdtd_add_tfsf_plane
 *   DataCapture / VolumeData (DataCapture.hpp:23-191; a      fdtd_add_dft, fdtd_dft_read
 *     stub in the reference: no Fourier capture exists)
 *   one pass of the user loop: YeeUpdate<Mode,D*>,           fdtd_step
 *     UpdatePML<Mode,Electric,d>, material E, sources,
 *     YeeUpdate<Mode,B*>, UpdatePML<Mode,Magnetic,d>,
 *     material H (YeeUpdates.hpp:343-405, PML.hpp:296-355)
 *   reading cell.Ez() etc.                                   fdtd_download / fdtd_upload
 *   UpdateSurfaceCurrentE/H, UpdateSurfaceChargeDensity      fdtd_read_quantity, and
 *     on cells, then cell.Jez() etc.                         fdtd_add_dft of FDTD_Q_J*,
 *     (SurfaceQuantities.hpp:169-356)                        FDTD_Q_RHO
 *
 * Ownership: the grid handle owns all device memory; host pointers passed in
 * are read during the call only. Errors: every call returns FDTD_OK (0) or a
 * negative fdtd_status; fdtd_last_error_string() describes the last error of
 * the calling thread. Threading: one handle per host thread; work is ordered
 * on the stream given to fdtd_step (NULL = the handle's own stream). */
#ifndef FDTD_B200_H
#define FDTD_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fdtd_grid fdtd_grid;

/* modes: the reference's Detail::EMMode order (FDTDConstants.hpp:410-415) */
enum { FDTD_TEM = 0, FDTD_TE = 1, FDTD_TM = 2, FDTD_THREED = 3 };

/* precision / method */
enum {
  FDTD_PLAIN_F64 = 0, /* FP64, D/B/E/H stored, the reference's operation order */
  FDTD_FUSED_F32 = 1  /* FP32, E/H form, fused sweeps */
};

enum {
  FDTD_OK = 0,
  FDTD_ERR_INVALID = -1,     /* bad argument or state */
  FDTD_ERR_CUDA = -2,        /* a CUDA call failed */
  FDTD_ERR_UNSUPPORTED = -3, /* valid, but not supported by this method */
  FDTD_ERR_NOMEM = -4,       /* a device or host allocation failed */
  FDTD_ERR_NONFINITE = -5,   /* a field went non-finite (fdtd_check_finite) */
  FDTD_ERR_TIMEOUT = -6      /* a bounded device wait gave up */
};

/* material kinds (DispersiveMaterials.hpp:2076-2105) */
enum { FDTD_VACUUM = 0, FDTD_CONSTANT = 1, FDTD_DRUDE = 2, FDTD_LORENTZ = 3 };
#define FDTD_MAX_POLES 4

/* field selectors for fdtd_download / fdtd_upload */
enum {
  FDTD_DX = 0, FDTD_DY, FDTD_DZ, FDTD_EX, FDTD_EY, FDTD_EZ,
  FDTD_BX, FDTD_BY, FDTD_BZ, FDTD_HX, FDTD_HY, FDTD_HZ,
  FDTD_PX, FDTD_PY, FDTD_PZ, FDTD_JX, FDTD_JY, FDTD_JZ, /* pole 0 */
  FDTD_PSI0 = 18 /* 18 + 9*ft + 3*I + J: CPML integrator psi[ft][I][J] */
  /* 36 + 6*(pole-1) + {0..5}: P/J of poles 1.. */
};

typedef struct {
  int mode;      /* FDTD_TE, FDTD_TM or FDTD_THREED */
  int precision; /* FDTD_PLAIN_F64 or FDTD_FUSED_F32 */
  int nx, ny, nz;/* cells per axis, including the fixed outer ring; nz = 1 in 2D */
  double dx;     /* cell size, m */
  double dt;     /* time step, s */
  int device;    /* CUDA device ordinal */
} fdtd_grid_desc;

typedef struct {
  int kind;   /* FDTD_VACUUM, FDTD_CONSTANT, FDTD_DRUDE, FDTD_LORENTZ */
  int npoles; /* Drude: 1; Lorentz: 1..FDTD_MAX_POLES */
  double eps_inf; /* relative permittivity: the reference storages' K */
  double mu_r;    /* relative permeability: 1 = VacuumUpdate<Mode,Magnetic> */
  double delta_eps[FDTD_MAX_POLES]; /* Lorentz pole strength; the reference ignores
                                       its Delta (DispersiveMaterials.hpp:710-735), i.e. 1 */
  double freq[FDTD_MAX_POLES];  /* Drude plasma / Lorentz resonance frequency, rad/s */
  double gamma[FDTD_MAX_POLES]; /* damping rate, 1/s */
} fdtd_material;

/* Create a grid. All fields start at zero; every cell is material 0
 * (vacuum unless fdtd_set_materials says otherwise). */
int fdtd_grid_create(const fdtd_grid_desc* desc, fdtd_grid** out);
int fdtd_grid_destroy(fdtd_grid* g);

/* CPML of `ncells` on side 0 (min) or 1 (max) of `axis`, graded with
 * PMLParameterModel(dx) (m=3, m_a=1, sigma_max=0.8(m+1)/(imp0 dx), kappa_max=5,
 * alpha_max=0.05) and placed as in tests/testTM.cpp:44-71. */
int fdtd_set_pml(fdtd_grid* g, int axis, int side, int ncells);
/* The same CPML graded with the five-parameter PMLParameterModel(m, ma,
 * sMax, kMax, aMax) (include/PML.hpp:376-377): kappa = 1 + x^m (kappa_max -
 * 1), sigma = x^m sigma_max, alpha = (1 - x)^ma alpha_max at depth x into the
 * layer, and the coefficients of NewPML::setPMLParameters (PML.hpp:84-102)
 * from them, in FP64 on the host. fdtd_set_pml returns a side to the
 * default model. kappa_max >= 1; sigma_max, alpha_max >= 0. */
int fdtd_set_pml_model(fdtd_grid* g, int axis, int side, int ncells, double m, double ma, double sigma_max,
                       double kappa_max, double alpha_max);

/* Material table (n <= 65536 entries; per-cell ids address the first 256). */
int fdtd_set_materials(fdtd_grid* g, const fdtd_material* mats, int n);
/* Per-cell material ids, uint8, x fastest: index (k*ny + j)*nx + i. */
int fdtd_set_material_ids(fdtd_grid* g, const uint8_t* ids);
/* Per-block ids: cell (i,j,k) takes ids[((k>>s)*nby + (j>>s))*nbx + (i>>s)]. */
int fdtd_set_material_blocks(fdtd_grid* g, int block_shift, const uint16_t* ids, int nbx, int nby, int nbz);

/* Per-cell relative permittivity (nx*ny*nz doubles, x fastest): a cell whose
 * value is > 0 and whose material is vacuum or constant takes it in place of
 * the material's eps_inf (a ConstantUpdate<Mode, Electric>(K) per cell);
 * values <= 0 keep the material. NULL removes the map. */
int fdtd_set_eps_map(fdtd_grid* g, const double* eps);

/* Boundary condition of face (axis, side 0 = min, 1 = max), the
 * make_pec/pmc/symmetric/antisymmetric/periodic_boundary of the reference
 * (BoundaryUpdates.hpp:528-845) applied to the interior cells next to the
 * face: after the sources of each half step, the outer cell beyond the face
 * takes that cell's E (then H) times the condition's sign per component
 * (PEC: E normal +, tangential -; H the opposite; PMC the reverse of PEC;
 * symmetric: normal -, tangential +; antisymmetric the reverse), or, for
 * periodic, the value of the interior cell at the far end of the axis.
 * FDTD_BC_NONE (the default) leaves the outer cells at zero. Bloch-periodic
 * is not offered: its complex factor has no meaning for the real fields. */
enum { FDTD_BC_NONE = 0, FDTD_BC_PEC = 1, FDTD_BC_PMC = 2, FDTD_BC_SYMMETRIC = 3, FDTD_BC_ANTISYMMETRIC = 4,
       FDTD_BC_PERIODIC = 5 };
int fdtd_set_boundary(fdtd_grid* g, int axis, int side, int kind);

/* Time policy of every curl update and TFSF correction, the TimePolicy
 * template argument of YeeUpdate and TFSFPlane (BD1, BD3, BD4 of
 * include/YeeUpdates.hpp:182-294): the flux update becomes
 * F = TimePolicy::get(F) + Coeff*curl_coeff*dt*curl with the flux history
 * (F of the previous two or three steps, zero at first) moved on each step.
 * BD3 and BD4 need a smaller time step than the leapfrog BD1 (they diverge at
 * 0.99 of the Courant limit; 0.5 is stable). FP64 plain grids only: an FP32
 * grid answers FDTD_ERR_UNSUPPORTED for BD3/BD4. Setting a scheme clears the
 * history. */
enum { FDTD_BD1 = 1, FDTD_BD3 = 3, FDTD_BD4 = 4 };
int fdtd_set_time_scheme(fdtd_grid* g, int scheme);

/* Soft source (SoftSource<Signal, Cell, GetField<F>>::apply): vals[t] is
 * added at step t (counted from grid creation) to component comp (0..2) of
 * E after the constitutive update (target 0), D before the CPML pass (1),
 * H after the magnetic constitutive update (2) or B before the magnetic CPML
 * pass (3). */
int fdtd_add_source(fdtd_grid* g, int comp, int target, int i, int j, int k, const double* vals, int nvals);
/* The same soft source on every interior cell of the inclusive box lo..hi
 * (a line source is a box one cell wide): one SoftSource per cell in the
 * reference, all driven by one signal. Targets E (0) or H (2) only; it is
 * applied after the point sources of the same field. */
int fdtd_add_source_box(fdtd_grid* g, int comp, int target, const int* lo, const int* hi, const double* vals,
                        int nvals);

/* One TFSF plane (TFSFPlane, Source.hpp:472-634): corrections on the cells
 * lo..hi (inclusive) with normal orient (0 = -axis, 1 = +axis), wave vector
 * k, polarisations pol_e/pol_h, location functor ((i,j,k) - origin) * dx, and
 * an Aux1D grid of aux_ncells + 50 cells whose source value at aux step s is
 * aux_vals[s-1]. Planes with equal aux grids share one on the device. */
int fdtd_add_tfsf_plane(fdtd_grid* g, int axis, int orient, const int* lo, const int* hi,
                        const double* origin, const double* k, const double* pol_e, const double* pol_h,
                        int aux_ncells, const double* aux_vals, int naux);

/* Quantities of a cell: the fields and the surface quantities of
 * SurfaceQuantities<Mode> (include/SurfaceQuantities.hpp:169-356). */
enum {
  FDTD_Q_EX = 0, FDTD_Q_EY, FDTD_Q_EZ, FDTD_Q_HX, FDTD_Q_HY, FDTD_Q_HZ,
  /* UpdateSurfaceCurrentE: Je = curl H / dx on the cell and its lower
   * neighbours (components of E present in the mode) */
  FDTD_Q_JEX = 6, FDTD_Q_JEY, FDTD_Q_JEZ,
  /* UpdateSurfaceCurrentH: Jh = -curl E / dx on the cell and its upper
   * neighbours (components of H present in the mode) */
  FDTD_Q_JHX = 9, FDTD_Q_JHY, FDTD_Q_JHZ,
  /* UpdateSurfaceChargeDensity: rho = eps0 div E / dx (TE and ThreeD; the
   * reference's TM functor does nothing) */
  FDTD_Q_RHO = 12
};

/* Running DFT of quantity comp (FDTD_Q_*) over the inclusive box lo..hi at
 * nf frequencies (cycles per step). X_f = sum_n x[n] exp(-2 pi i f n), with
 * n = t+1 for the quantities of E (E, Jh, rho) sampled at the end of step
 * t's E half and t+1.5 for those of H (H, Je). Boxes of surface quantities
 * lie in the interior. */
int fdtd_add_dft(fdtd_grid* g, int comp, const int* lo, const int* hi, const double* freqs, int nf, int* handle);

/* Quantity q (FDTD_Q_*) on every cell of the inclusive box lo..hi from the
 * current fields, x fastest, into host (FP64): the snapshot of applying the
 * reference's UpdateSurfaceCurrentE / UpdateSurfaceCurrentH /
 * UpdateSurfaceChargeDensity functors to those cells and reading them back.
 * Synchronises the grid's stream. */
int fdtd_read_quantity(fdtd_grid* g, int q, const int* lo, const int* hi, double* host);
int fdtd_dft_npoints(fdtd_grid* g, int handle, long long* npoints);
/* host out: [nf][npoints][2] doubles (re, im), points x fastest. Blocks
 * until the spectrum is in `out`. Spectra of 8 MB and more pass through two
 * pinned 8 MB chunks that the grid allocates at its first such read and
 * keeps until fdtd_grid_destroy; several host threads copy them into `out`. */
int fdtd_dft_read(fdtd_grid* g, int handle, double* out);

/* Advance nsteps full time steps on `stream` (a cudaStream_t, or NULL for the
 * handle's stream). Returns once the work is enqueued. */
int fdtd_step(fdtd_grid* g, int nsteps, void* stream);
/* Half a time step: phase 0 = the E half (curl of H, CPML, materials,
 * sources, TFSF, E-phase DFT sample; it also advances the TFSF aux grids one
 * step), phase 1 = the H half, which completes the step. The halves must
 * alternate, E first; fdtd_step refuses to run between them. For callers
 * that exchange data between the halves, such as the ghost planes of a
 * z-slab decomposition (the reference does the same between its E and H
 * functors across MPI ranks, BoundaryUpdates.hpp:919-1051). Launched eagerly. */
int fdtd_step_half(fdtd_grid* g, int phase, void* stream);
/* The half step `phase` in two parts (3D grids), so that a ghost plane can
 * travel while the sweep runs: part 0 sweeps every plane whose update reads
 * no ghost plane -- for the E half planes 2 .. nz-2 (plane 1 reads H of plane
 * 0), for the H half planes 1 .. nz-3 (plane nz-2 reads E of plane nz-1) --
 * and part 1, called once plane 0 (E half) or plane nz-1 (H half) holds the
 * neighbour's values, sweeps the remaining plane and runs the rest of the
 * half step. Parts 0 then 1 give exactly fdtd_step_half's results; other
 * calls on the grid between them are refused. FP32 grids need the staged
 * sweeps (FDTD_SWEEP_AUTO or FDTD_SWEEP_STAGED). Launched eagerly. */
int fdtd_step_half_part(fdtd_grid* g, int phase, int part, void* stream);
/* Copy z plane k of a stored component (FDTD_EX..FDTD_EZ, FDTD_HX..FDTD_HZ)
 * between the grid and a compact device buffer of nx*ny values of the grid's
 * precision, x fastest (to_grid = 1: buffer to grid). The FP32 method stores
 * eta*H, and that is what is copied. Stream-ordered on `stream`. */
int fdtd_copy_plane(fdtd_grid* g, int which, int k, void* dev_buf, int to_grid, void* stream);
/* Copy z plane k_src of a stored component of grid src straight into z plane
 * k_dst of the same component of grid dst (same precision, mode and x-y
 * extent; the same or another device, a peer copy then), on `stream` (NULL =
 * dst's stream) -- a ghost-plane exchange between two slabs held by one
 * process, with no staging buffer (the reference's MPI boundary exchange,
 * BoundaryUpdates.hpp:919-1051, between two ranks). The caller orders it after
 * the half step that wrote the source plane. */
int fdtd_copy_plane_between(fdtd_grid* src, int which, int k_src, fdtd_grid* dst, int k_dst, void* stream);
/* The reference's forward (explicit) material updates of field type ft
 * (0 electric, 1 magnetic) on every interior cell, XUpdate<Mode, ft,
 * forward = true> (DispersiveMaterials.hpp:345-349, :922-934): D = eps*E
 * (VacuumUpdate, ConstantUpdate, the eps map), for Drude cells P and J
 * advanced explicitly and D = eps_inf*eps0*E + P; B = mu_r*mu0*H. FP64 grids
 * only (FDTD_ERR_UNSUPPORTED on FP32, which stores no D or B); grids with a
 * Lorentz material refuse ft 0, as the reference's explicit Lorentz update is
 * a static_assert (:697-706). Stream-ordered on `stream` (NULL = the grid's). */
int fdtd_material_explicit(fdtd_grid* g, int ft, void* stream);
/* Lays out the device state that the set-up calls defer: the CPML
 * coefficient profiles and integrator slabs (fdtd_set_pml regrades on the
 * host only), the DFT sample buffers and the TFSF tables, and (with graphs
 * on, between whole steps) captures the CUDA graph of 64 steps that
 * fdtd_step replays, so that the first long call starts at once. fdtd_step
 * and fdtd_step_half do all of it themselves; call it before the first
 * fdtd_step_static_scratch of a grid that has not stepped, which allocates
 * nothing. No counterpart in the reference (its cells carry their CPML state
 * from construction). */
int fdtd_prepare(fdtd_grid* g);
/* fdtd_step for callers that cannot allocate device memory while stepping
 * (no counterpart in the reference, whose steps run on the host). Same
 * kernels, order and results as fdtd_step, launched eagerly; the per-call
 * TFSF incident-field table goes into one fixed 4 MiB device array instead of
 * a buffer that grows with cudaMalloc, so a call allocates nothing.
 * - At most 4 MiB / (16 bytes x the sum of the planes' aux lengths L) - 1
 *   steps per call (L = the plane's aux_ncells + 50); a larger call
 *   returns FDTD_ERR_INVALID naming the limit. Without TFSF planes, no limit.
 * - The array's address is looked up once per device on the first call, which
 *   may load the library's device code: make that call before any stream
 *   capture.
 * - DFT regions added (or a CPML set) since the last step need fdtd_prepare
 *   (or one fdtd_step) to lay out their buffers; until then this returns
 *   FDTD_ERR_INVALID. So does a call between the halves of fdtd_step_half.
 * - With TFSF planes the call uploads the step counter from the host and
 *   waits for that copy; on a stream under capture it returns
 *   FDTD_ERR_UNSUPPORTED.
 * - The array is shared by all grids of a device: calls whose GPU work
 *   overlaps (other streams or host threads) race on it. */
int fdtd_step_static_scratch(fdtd_grid* g, int nsteps, void* stream);
/* fdtd_step with CUDA events on the launching stream around each part of a
 * step: ms[0..4] receive the mean per-step time (milliseconds) of the E sweep,
 * the E-phase extras (TFSF kernel of the FP32 method, DFT gather), the H sweep,
 * the H-phase extras, and the step counter plus the amortised DFT flush.
 * Synchronises after every step; for measurement, not production. */
int fdtd_profile_step(fdtd_grid* g, int nsteps, void* stream, double* ms);
/* Which kernels carry the 3D FP32 fused sweeps: FDTD_SWEEP_AUTO (the
 * default: currently the staged sweeps, the fastest measured on B200), FDTD_SWEEP_REGS (z-marching, register prefetch),
 * FDTD_SWEEP_TMA (z-marching, TMA pipeline into shared memory; or
 * FDTD_ERR_UNSUPPORTED), FDTD_SWEEP_FLAT (one thread per 4-cell group and
 * plane), FDTD_SWEEP_STAGED (flat, with every operand of a thread copied
 * into shared memory by cp.async at thread start) or FDTD_SWEEP_EH (the
 * staged E and H updates of a whole step in one persistent launch, H tiles
 * following the E tiles they read by a few planes so that E and H are read
 * from HBM about once per step; grids without TFSF planes, box sources,
 * boundary conditions or mu_r != 1, else FDTD_ERR_UNSUPPORTED at the step).
 * All compute the same update, cell for cell. */
enum { FDTD_SWEEP_AUTO = 0, FDTD_SWEEP_REGS = 1, FDTD_SWEEP_TMA = 2, FDTD_SWEEP_FLAT = 3, FDTD_SWEEP_STAGED = 4,
       FDTD_SWEEP_EH = 5 };
int fdtd_set_sweep_kernel(fdtd_grid* g, int kind);
/* Replay a captured CUDA graph per 64 steps inside fdtd_step (default 1), or
 * launch every kernel from the host (0). Results are identical. */
int fdtd_use_graphs(fdtd_grid* g, int enable);
/* Device-side error flags accumulated by the kernels (0 = none; bit 0: a
 * bounded wait on a TMA stage expired and the sweep was abandoned; bit 1: in
 * the one-launch step an H tile's bounded wait for the E tiles it reads
 * expired, so that step's result is not valid). */
int fdtd_error_flags(fdtd_grid* g, int* flags);
/* Wait for all work on the handle's streams. */
int fdtd_synchronize(fdtd_grid* g);

/* Copy one field to/from a host array of nx*ny*nz doubles (x fastest), in SI
 * units whatever the precision. Fields the method does not store return
 * FDTD_ERR_UNSUPPORTED. */
int fdtd_download(fdtd_grid* g, int which, double* host);
int fdtd_upload(fdtd_grid* g, int which, const double* host);

/* Checks every stored field for NaN/Inf; FDTD_ERR_NONFINITE if any. */
int fdtd_check_finite(fdtd_grid* g);

/* Relative-L2 error of one field of grid g against the same field of grid
 * ref (same shape and device, either precision), computed on the device in
 * FP64 and in SI units over every cell: err_sq = sum (g - ref)^2, ref_sq =
 * sum ref^2, so the relative L2 error is sqrt(err_sq / ref_sq). `which` is a
 * field selector of fdtd_download (E, H, and D, B, P, J where both grids
 * store them; not the CPML integrators). Waits for both grids' streams. The
 * reference keeps no second copy of its fields to compare against; this
 * states the FP32 method's error against an FP64 plain grid at sizes where
 * downloading both would not fit host memory. */
int fdtd_field_error(fdtd_grid* g, fdtd_grid* ref, int which, double* err_sq, double* ref_sq);

/* Steps taken so far, and kernels this handle launched so far. */
int fdtd_get_step(fdtd_grid* g, long long* step);
int fdtd_launch_count(fdtd_grid* g, long long* count);
/* Device bytes held by the grid. */
int fdtd_memory_bytes(fdtd_grid* g, long long* bytes);

/* ------------------------------------------------------------ batches
 * Many independent FP32 2D grids (TE or TM, same mode and device, no TFSF,
 * DFT or box sources, equal step counts), each set up with the calls above,
 * advanced together by fdtd_batch_step as one replayed CUDA graph: either one
 * persistent cooperative kernel for all the steps (grid barriers between the
 * half steps), or one kernel per half step over the tiles of every grid; the
 * tuner picks. The grids stay usable on their own (download etc.). */
typedef struct fdtd_batch fdtd_batch;
int fdtd_batch_create(int n, fdtd_grid* const* grids, fdtd_batch** out);
int fdtd_batch_destroy(fdtd_batch* b);
/* Autotuner: times both launch modes with each tile height (1, 2, 4, 8 rows
 * of 128 cells) for `steps` steps on a snapshot of the grids' state; then,
 * for the fastest, each size class of grids (quartiles of the cell counts,
 * largest first) in turn with work items 1, 2, 4 or 8 times that height;
 * then temporal blocking with 2, 3 and 4 steps per launch where the grids
 * allow it (which lays out the second copy of the state that mode needs);
 * restores the state and keeps the fastest. */
int fdtd_batch_tune(fdtd_batch* b, int steps);
/* Choose the launch mode (1: persistent, 0: one kernel per half step) and
 * the tile height (1, 2, 4 or 8) without tuning; every grid's work items are
 * one tile high; temporal blocking off. */
int fdtd_batch_configure(fdtd_batch* b, int persistent, int rows);
/* Per grid of the batch (in creation order): the rows of its work items and
 * its size class (0 = the quarter of the grids with the fewest cells .. 3);
 * the tuner's ms per step with those heights (0 if not tuned). Any output
 * pointer may be NULL. */
int fdtd_batch_item_rows(fdtd_batch* b, int* rows_per_grid, int* size_class, float* tuned_ms);
/* Set the work-item rows of every grid (in creation order): the tile height
 * in use times 1, 2, 4 or 8. The tuner's choice, by hand. */
int fdtd_batch_set_item_rows(fdtd_batch* b, const int* rows_per_grid);
/* Temporal blocking: each launch advances every grid `depth` steps (2, 3 or
 * 4) from shared memory, reading one copy of the state and writing a second
 * one that the batch allocates (the grids' fields, CPML integrators and
 * source values, once more); launches come in pairs, so the state ends in the
 * grids' own arrays, and the steps of a call beyond whole pairs run one kernel
 * per half step. Results equal the other launch modes bit for bit. Grids
 * without dispersive materials whose sources lie inside their interiors
 * (FDTD_ERR_UNSUPPORTED otherwise); 0 turns it off. fdtd_batch_configure turns
 * it off too; fdtd_batch_tune also times depths 2, 3 and 4 and keeps one if
 * it is faster. */
int fdtd_batch_set_temporal(fdtd_batch* b, int depth);
/* The depth in use (0: off) and the tuner's ms per step with depths 2, 3, 4
 * (tuned_ms[3]; 0 if not timed). Either pointer may be NULL. */
int fdtd_batch_temporal(fdtd_batch* b, int* depth, float* tuned_ms);
int fdtd_batch_step(fdtd_batch* b, int nsteps, void* stream);
/* Tile height in use, CTAs per launch, work items, the launch mode (1:
 * persistent, 0: per half step), and the tuner's ms per step (tune_ms[8]:
 * persistent with tile heights 1, 2, 4, 8, then per half step with 1, 2, 4,
 * 8; 0 if not tuned). Any output pointer may be NULL. */
int fdtd_batch_info(fdtd_batch* b, int* rows, int* blocks, int* items, int* persistent, float* tune_ms);
/* Bit 0: a bounded grid-barrier wait expired and the kernel gave up. */
int fdtd_batch_error_flags(fdtd_batch* b, int* flags);

/* Last error of the calling thread ("" if none). */
/* ---- adjoint gradient (2D TM, FP32 fused method) ----
 * d(objective)/d(eps_r) over a design box by the discrete adjoint of the
 * time step. Objective J = sum over the probe box (inclusive, z = 0) of
 * |X|^2, X the running DFT of Ez at `freq` (cycles per step, samples as
 * fdtd_add_dft). The grid must be unstepped, without TFSF planes or
 * dispersive materials; the design box must lie outside the CPML and hold no
 * D-target source. create adds the probe DFT region to the grid. forward
 * steps the grid nsteps times, checkpointing the state every ckpt_every
 * steps, and returns J; backward recomputes each segment from its checkpoint,
 * reverses it, leaves the grid in its post-forward state and writes
 * dJ/deps_r of every design cell (x fastest) to the host array grad. One
 * forward and one backward per handle; destroy it before its grid.
 * The reference has no adjoint; its per-cell permittivity is the K of
 * ConstantUpdate (DispersiveMaterials.hpp:354-359). */
typedef struct fdtd_adjoint fdtd_adjoint;
int fdtd_adjoint_create(fdtd_grid* g, const int* probe_lo, const int* probe_hi, double freq, const int* design_lo,
                        const int* design_hi, int ckpt_every, fdtd_adjoint** out);
int fdtd_adjoint_forward(fdtd_adjoint* a, int nsteps, double* J);
int fdtd_adjoint_backward(fdtd_adjoint* a, double* grad);
int fdtd_adjoint_destroy(fdtd_adjoint* a);

const char* fdtd_last_error_string(void);

#ifdef __cplusplus
}
#endif
#endif
