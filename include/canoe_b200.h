/*
 * canoe_b200.h -- C ABI of the B200-native dynamical-core hot path of canoe.
 *
 * Every entry point is `extern "C"`, takes plain pointers and sizes, and
 * returns an int status (0 = success, see canoe_status). Arrays follow the
 * reference layout AthenaArray<Real>(NV, nc3, nc2, nc1) with i (x1, the
 * vertical) fastest and NGHOST = 3 ghost cells on each side of every active
 * dimension (canoe src/interface/hydro.hpp:54-67).  Variable slots are
 * IDN = 0 (dry density in the conserved state, total density in the
 * primitive state), 1..ny mass fractions (primitive) or species densities
 * (conserved), IVX = 1+ny, IVY, IVZ, IPR = IEN = 4+ny
 * (canoe src/tasklist/implicit_hydro_tasks.cpp:300-311).
 *
 * Pointers named d_* are device pointers (cudaMalloc'd by the caller),
 * h_* are host pointers.  `stream` is a cudaStream_t passed as void*.
 *
 * Each declaration names the reference interface it replaces (file:line,
 * relative to the canoe source tree; Athena++ functions are those hooked by
 * canoe's patches).
 */
#ifndef CANOE_B200_H_
#define CANOE_B200_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CANOE_NGHOST 3
#define CANOE_MAX_NY 8    /* max mass-fraction slots (vapors + clouds) */
#define CANOE_MAX_VAPOR 4 /* max condensable vapors                    */
#define CANOE_MAX_NV (5 + CANOE_MAX_NY)

/* status codes */
enum canoe_status {
  CANOE_OK = 0,
  CANOE_ERR_ARG = 1,      /* invalid argument (size, null pointer, flag)   */
  CANOE_ERR_CUDA = 2,     /* a CUDA runtime call failed                    */
  CANOE_ERR_NUMERIC = 3,  /* device error word set (NaN / negative p, rho) */
  CANOE_ERR_NOCONV = 4,   /* Newton iteration did not converge             */
  CANOE_ERR_UNSUPPORTED = 5
};

/* device error-word bits (canoe src/checks.cpp:53-149 glog checks) */
enum canoe_errbit {
  CANOE_EBIT_NEG_DENSITY = 1,
  CANOE_EBIT_NEG_PRESSURE = 2,
  CANOE_EBIT_NAN = 4,
  CANOE_EBIT_SATADJ_NOCONV = 8,
  CANOE_EBIT_SATADJ_FALLBACK = 16,
  CANOE_EBIT_TIMEOUT = 32        /* a bounded wait for an async copy gave up */
};

/* boundary flags (Athena BoundaryFlag subset used on this path) */
enum canoe_bc {
  CANOE_BC_REFLECT = 0,
  CANOE_BC_PERIODIC = 1,
  CANOE_BC_OUTFLOW = 2,
  CANOE_BC_EXO3 = 3, /* cubed-sphere panel edge: ghosts filled by the exo3 exchange */
  CANOE_BC_BLOCK = 4 /* x2 / x3 side shared with a neighbouring MeshBlock: ghosts
                      * filled from the neighbour's interior (Athena's block
                      * boundary, BoundaryFlag::block) */
};

/* reconstruction order (Athena `xorder`): 2 = PLM, 3 = PPM */
enum canoe_recon { CANOE_RECON_PLM = 2, CANOE_RECON_PPM = 3 };

/* Riemann solver (canoe RSOLVER, src/snap/CMakeLists.txt:28) */
enum canoe_rsolver { CANOE_RSOLVER_LMARS = 0, CANOE_RSOLVER_HLLC = 1 };

/* precision of reconstruction + Riemann fluxes */
enum canoe_precision { CANOE_FP64 = 0, CANOE_FP32_PERTURBATION = 1 };

/*
 * Ideal-moist thermodynamics (snapy IdealMoist + kintera ThermoY parameters).
 * Slot n = 1..ny is stored at index n-1 of the per-slot arrays, matching
 * `cv_ratio_m1[n - 1]` / `inv_mu_ratio_m1[n - 1]` in
 * canoe src/interface/eos.hpp:48-67.  Vapors occupy slots 1..nvapor, clouds
 * nvapor+1..ny.
 */
typedef struct canoe_thermo {
  int32_t ny;      /* vapors + clouds                                   */
  int32_t nvapor;  /* vapors (slots 1..nvapor)                          */
  double rd;       /* dry specific gas constant [J/kg/K]   eos.hpp:14   */
  double gammad;   /* dry adiabatic index                  eos.hpp:18   */
  double grav;     /* signed x1 gravity (hsrc.GetG1()), <0 points to -x1 */
  double cv_ratio_m1[CANOE_MAX_NY];     /* cv_n / cv_d - 1                 */
  double inv_mu_ratio_m1[CANOE_MAX_NY]; /* mu_d / mu_n - 1 (vapors)        */
  double u0[CANOE_MAX_NY];              /* latent energy offset [J/kg]     */
  /* phase change, per vapor v = 0..nvapor-1 (kintera "ideal" nucleation) */
  int32_t liq_slot[CANOE_MAX_VAPOR];    /* slot of the liquid, -1 if none  */
  int32_t ice_slot[CANOE_MAX_VAPOR];    /* slot of the ice, -1 if none     */
  double t3[CANOE_MAX_VAPOR];           /* triple-point temperature [K]    */
  double p3[CANOE_MAX_VAPOR];           /* triple-point pressure [Pa]      */
  double beta_l[CANOE_MAX_VAPOR], delta_l[CANOE_MAX_VAPOR];
  double beta_s[CANOE_MAX_VAPOR], delta_s[CANOE_MAX_VAPOR];
} canoe_thermo_t;

/* Newton saturation-adjustment controls */
typedef struct canoe_satadj_opts {
  double tol;      /* |dT| stopping tolerance [K]                       */
  int32_t max_iter;/* Newton iterations before the bracketing fallback  */
  int32_t warm;    /* start: 0 the unadjusted temperature (cold),
                      1 t_guess[], 2 gated: t_guess[] when it exceeds the
                      cold start by 0.05 K (latent heating), else cold   */
} canoe_satadj_opts_t;

/* One MeshBlock: a Cartesian (or cubed-sphere panel) block. */
typedef struct canoe_block_config {
  int32_t nx1, nx2, nx3;  /* interior cells; nx3 == 1 => 2-D (no x3 ghosts) */
  int32_t bc[6];          /* ix1, ox1, ix2, ox2, ix3, ox3 (canoe_bc)          */
  double x2min, x3min;    /* lower edges                                      */
  double dx2, dx3;        /* uniform widths                                   */
  const double *h_x1f;    /* nx1+1 interior x1 face positions (nonuniform ok) */
  int32_t recon;          /* canoe_recon                                      */
  int32_t rsolver;        /* canoe_rsolver                                    */
  int32_t implicit_flag;  /* bit0 X1, bit1 X2, bit2 X3, bit3 full 5x5
                           * (implicit_solver.cpp:47, solve_implicit_3d.cpp:
                           * 25-142); X2 / X3 on dry blocks only          */
  int32_t precision;      /* canoe_precision                                  */
  int32_t satadj;         /* 1: saturation adjustment at the last RK stage    */
  double cfl;             /* CFL number for canoe_block_new_dt                */
  canoe_thermo_t thermo;
} canoe_block_config_t;

typedef struct canoe_block *canoe_block_t;
typedef struct canoe_mlp *canoe_mlp_t;

/* The six panels of an equiangular gnomonic cubed-sphere shell, one
 * MeshBlock per panel (canoe src/exo3: CUBED_SPHERE build with NBLOCKS = 6,
 * so cs_find_block_id.cpp:83-91 gives bound_lim = 0).  Panel p holds the
 * reference's blockID p + 1; x2 and x3 are the panel's equiangular
 * coordinates in [-pi/4, pi/4] with nside cells each, x1 the radius. */
typedef struct canoe_shell_config {
  int32_t nx1;          /* radial cells                                  */
  int32_t nside;        /* cells along each panel edge (even)            */
  int32_t bc_x1[2];     /* inner / outer radial boundary (canoe_bc)      */
  const double *h_x1f;  /* nx1+1 radial faces [m] from the planet centre */
  int32_t recon;        /* canoe_recon                                   */
  int32_t rsolver;      /* CANOE_RSOLVER_HLLC (hllc_transform)           */
  int32_t implicit_flag;/* bit0 X1, bit3 full 5x5                        */
  int32_t precision;    /* canoe_precision                               */
  double cfl;
  canoe_thermo_t thermo;
} canoe_shell_config_t;

typedef struct canoe_shell *canoe_shell_t;
typedef struct canoe_batch *canoe_batch_t;
typedef struct canoe_mesh *canoe_mesh_t;

/* ---------------- version / diagnostics ---------------- */
const char *canoe_version(void);
const char *canoe_last_error(void);
int canoe_device_sm_count(int *out);

/* Self-test of the bounded waits that guard the kernels' bulk copies: one
 * thread waits at most `spins` polls for an mbarrier phase that is complete
 * (complete != 0) or cannot complete before the wait (complete == 0), and
 * *h_bits receives CANOE_EBIT_TIMEOUT if the wait gave up.  The kernel then
 * completes the phase itself, so nothing stays pending.  No reference
 * counterpart (the reference has no device waits). */
int canoe_selftest_bounded_wait(int spins, int complete, uint32_t *h_bits);

/* Self-test of the bounded wait for the tensor cores' completion in the
 * warm-start inference: one warpgroup allocates tensor memory, issues the
 * layer-2 MMAs on zero operands and commits them (issue != 0) or issues
 * nothing (issue == 0), and waits at most `spins` polls; *h_bits receives
 * CANOE_EBIT_TIMEOUT if the wait gave up and CANOE_EBIT_NAN if a completed
 * accumulator did not read back as zeros.  The tensor memory is freed in
 * both cases.  No reference counterpart. */
int canoe_selftest_umma_wait(int spins, int issue, uint32_t *h_bits);

/* Measured non-tensor FMA throughput of the current GPU in TFLOP/s (2 flops
 * per FMA): FP64 (fp32 == 0) or FP32, eight independent chains per thread on
 * every SM, timed with CUDA events after a warm-up launch.  The denominator
 * the bench uses for FP64 / FP32 arithmetic.  No reference counterpart. */
int canoe_measure_fma_peak(int fp32, double *h_tflops);

/* ---------------- operator-level entry points (device pointers) --------- */

/* Hydro::RiemannSolver, LMARS: canoe src/snap/riemann/lmars.cpp:19-85.
 * d_wl, d_wr: (NV, n) face states; d_flx: (NV, n) fluxes.  ivx is the
 * variable slot of the normal velocity (IVX, IVY or IVZ). */
int canoe_riemann_lmars(const canoe_thermo_t *th, int ivx, const double *d_wl,
                        const double *d_wr, double *d_flx, int64_t n,
                        void *stream);

/* Hydro::RiemannSolver, HLLC: canoe src/snap/riemann/hllc_transform.cpp:25-233
 * (Cartesian branch). Same layout as canoe_riemann_lmars. */
int canoe_riemann_hllc(const canoe_thermo_t *th, int ivx, const double *d_wl,
                       const double *d_wr, double *d_flx, int64_t n,
                       void *stream);

/* Saturation adjustment, kintera ThermoY::forward(rho, intEng, yfrac) as
 * called from ImplicitHydroTasks::UpdateAllConserved,
 * canoe src/tasklist/implicit_hydro_tasks.cpp:290-313.  Operates in place on
 * conserved cells d_u laid out (NV, ncells); d_t_guess (ncells, may be NULL
 * unless opts->warm) is the initial temperature; d_t_out (may be NULL)
 * receives the converged temperature; d_iters (may be NULL) the Newton
 * iteration count per cell.  d_stats[0..3] (may be NULL) accumulates
 * {cells, total iterations, fallbacks, non-converged}. */
int canoe_saturation_adjust(const canoe_thermo_t *th,
                            const canoe_satadj_opts_t *opts, double *d_u,
                            int64_t ncells, const double *d_t_guess,
                            double *d_t_out, int32_t *d_iters,
                            unsigned long long *d_stats, void *stream);

/* ---------------- learned warm start (no reference counterpart) ---------
 * A 4 -> 64 -> 64 -> 1 tanh network maps (density, specific internal
 * energy, total H2O, total NH3) to the converged temperature of the
 * saturation adjustment, as a correction to the temperature the cell would
 * have with all water as vapour.  It only supplies the Newton starting point: the
 * tolerance, the fallback and therefore the answer are those of the plain
 * solve.  Parameters are FP32 (layout w1[64*4] b1[64] w2[64*64] b2[64]
 * w3[64] b3[1], row-major [out][in]); inference uses a BF16 copy of w2 on
 * the tensor cores with FP32 accumulation. */
int canoe_mlp_create(uint64_t seed, canoe_mlp_t *out);
int canoe_mlp_destroy(canoe_mlp_t m);
int canoe_mlp_nparams(void);
int canoe_mlp_set_params(canoe_mlp_t m, const float *h_params);
int canoe_mlp_get_params(canoe_mlp_t m, float *h_params);
/* inputs are normalised as (x - mean) / std; the output as
 * T = T_vapour + y std + mean, T_vapour the all-vapour temperature */
int canoe_mlp_set_normalization(canoe_mlp_t m, const float *in_mean, const float *in_std,
                                float out_mean, float out_std);
int canoe_mlp_get_normalization(canoe_mlp_t m, float *in_mean, float *in_std,
                                float *out_mean, float *out_std);
/* mean-squared error of normalised outputs d_y over n normalised inputs
 * d_x (n x 4) and its gradient (into d_grad, or the network's own buffer
 * when NULL); *loss_out (may be NULL) receives the loss (blocking). */
int canoe_mlp_loss_grad(canoe_mlp_t m, const float *d_x, const float *d_y, int64_t n,
                        float *d_grad, float *loss_out, void *stream);
/* one Adam step with the network's own gradient buffer */
int canoe_mlp_adam_step(canoe_mlp_t m, float lr, float beta1, float beta2, float eps,
                        void *stream);
/* normalised forward pass: FP32 CUDA cores (tensor_core = 0) or the BF16
 * tensor-core path of the warm start (tensor_core = 1: tcgen05 MMAs with the
 * layer-2 accumulator in tensor memory; an output is NaN if its CTA's bounded
 * wait for the MMAs gave up) */
int canoe_mlp_forward(canoe_mlp_t m, const float *d_x, float *d_y, int64_t n, int tensor_core,
                      void *stream);
/* canoe_saturation_adjust with the network's guess as the starting point
 * (opts->warm 1 or 2); d_guess_out (may be NULL) receives the guesses. */
int canoe_saturation_adjust_learned(const canoe_thermo_t *th,
                                    const canoe_satadj_opts_t *opts, canoe_mlp_t m,
                                    double *d_u, int64_t ncells, double *d_t_out,
                                    int32_t *d_iters, unsigned long long *d_stats,
                                    double *d_guess_out, void *stream);

/* ---------------- MeshBlock-level entry points ---------------- */

/* MeshBlock + MeshBlock::Impl construction (canoe src/mesh_setup.cpp:98-101,
 * src/impl.cpp:38-112): allocates every device array of the block. */
int canoe_block_create(const canoe_block_config_t *cfg, canoe_block_t *out);
int canoe_block_destroy(canoe_block_t b);
/* sizes: nv, nc1, nc2, nc3 (with ghosts) */
int canoe_block_dims(canoe_block_t b, int32_t *nv, int32_t *nc1, int32_t *nc2,
                     int32_t *nc3);

/* upload / download the conserved state u and primitive state w
 * (NV, nc3, nc2, nc1) host arrays; set_conserved recomputes w (cons->prim +
 * boundary ghosts).  Blocking. */
int canoe_block_set_conserved(canoe_block_t b, const double *h_u);
int canoe_block_get_conserved(canoe_block_t b, double *h_u);
int canoe_block_get_primitive(canoe_block_t b, double *h_w);
/* device views of the live state (for zero-copy callers) */
int canoe_block_device_ptrs(canoe_block_t b, double **d_u, double **d_w);
int canoe_block_set_stream(canoe_block_t b, void *stream);

/* Hydro::CalculateFluxes(w, b, bcc, order): Athena calculate_fluxes.cpp with
 * canoe patches/19.calculate_fluxes.patch:19-185 (ChangeToTemperature at
 * :24, RestoreFromTemperature at :42, RiemannSolver per direction).  Writes
 * the three face-flux arrays: d_flx1 (NV, nc3, nc2, nc1+1), d_flx2
 * (NV, nc3, nc2+1, nc1), d_flx3 (NV, nc3+1, nc2, nc1); interior faces only. */
int canoe_block_calculate_fluxes(canoe_block_t b, double *d_flx1,
                                 double *d_flx2, double *d_flx3);

/* ImplicitSolver::SolveImplicit3D(du, w, dt): canoe src/snap/implicit/
 * solve_implicit_3d.cpp:19-142, the directions of implicit_flag in the
 * reference's order X3, X2, X1, each with PartialCorrection
 * (partial_correction.cpp:26-170) or FullCorrection (full_correction.cpp:
 * 32-161) and ForwardSweep / BackwardSubstitution (forward_backward.hpp:
 * 15-137), or the periodic sweep (periodic_forward_backward.hpp:15-234) when
 * both ends of the direction are periodic.  X2 / X3 write back IDN, the
 * normal momentum and IEN, as the reference's transposition does.  d_du
 * (NV, nc3, nc2, nc1) is corrected in place; the block's current primitive
 * state is used as w. */
int canoe_block_solve_implicit(canoe_block_t b, double *d_du, double dt);

/* One full time step of the block (all RK3 stages): the Athena task list as
 * rewritten by ImplicitHydroTasks (src/tasklist/implicit_hydro_tasks.cpp:
 * 45-313): CalculateFluxes -> IntegrateHydro -> AddSourceTerms ->
 * ImplicitCorrection -> UpdateAllConserved -> boundaries -> cons2prim.
 * dt < 0 uses the block's own CFL time step (Hydro::NewBlockTimeStep with
 * patches/21.new_blockdt.patch) computed on the device. */
int canoe_block_step(canoe_block_t b, double dt);

/* One time step like canoe_block_step(b, dt) that allocates nothing, for
 * callers that cannot let a library allocate device memory while they run
 * (a host model whose memory pool holds the GPU's memory, where a cudaMalloc
 * would fail or synchronize the device inside its own time step).  No
 * counterpart in the reference.
 *   cfg   block configuration as for canoe_block_create
 *   d_u   device conserved state (NV, nc3, nc2, nc1), ghosts included:
 *         read, advanced by dt in place
 *   d_w   device buffer of the same shape: receives the primitive state
 *         (with ghosts) of the advanced u
 *   d_err optional device word, cleared, then set to canoe_errbit bits;
 *         NULL keeps the bits in the library's scratch
 *   dt    time step (> 0); the pressure profile of the FP32 flux path is
 *         the level mean of the state on entry
 * The step's other arrays (du, u1, geometry, dt) live in one fixed device
 * array of 16 MiB (2 Mi doubles) per device, which must hold
 * 2 NV nc3 nc2 nc1 + 4 nc1 + 8 doubles: larger blocks return CANOE_ERR_ARG.
 * The configuration is checked exactly as canoe_block_create checks it.
 * The first call on a device looks up that array's address.  With CUDA's
 * lazy module loading that first call is also when the library's module is
 * loaded onto the device and the 16 MiB array takes its device memory, so a
 * caller makes one call (a warm-up step on a scratch state is enough) at
 * set-up, before it hands the GPU's free memory to its own pool; later
 * calls allocate nothing.  h_x1f is copied to the device on every call
 * from the caller's host memory.  All calls on a device share the array, so
 * calls that overlap in time (other streams or threads) race and corrupt
 * each other's results: order them on one stream.  The saturation
 * adjustment (cfg->satadj) uses the cold start.  X2 / X3 implicit solves
 * (implicit_flag bits 1, 2) need line scratch: such a cfg returns
 * CANOE_ERR_UNSUPPORTED. */
int canoe_block_step_noalloc(const canoe_block_config_t *cfg, double *d_u, double *d_w,
                             uint32_t *d_err, double dt, void *stream);

/* Capture one step (all RK stages, device dt) as a CUDA graph on first use and
 * replay it for every canoe_block_step(b, dt <= 0) call.  No reference
 * counterpart: the reference drives the task list from the host per stage
 * (main.cpp:119-121). */
int canoe_block_use_graph(canoe_block_t b, int on);

/* One step like canoe_block_step, timing each kernel class with CUDA events
 * on the block's stream; adds milliseconds to ms[0..6] = {x1 flux, x2 flux,
 * x3 flux, RK update + implicit solve, saturation adjustment, cons->prim +
 * ghosts, dt}.  No reference counterpart (the reference times whole runs,
 * src/mesh_destroy.cpp:43-53). */
int canoe_block_step_profile(canoe_block_t b, double dt, float *ms, int nclass);

/* Pin the time step: dt > 0 makes every following step (graph replays
 * included) use dt; dt <= 0 returns to the CFL step of
 * canoe_block_new_dt.  The reference fixes dt only through its input file
 * (Athena <time> dt); no direct counterpart. */
int canoe_block_set_fixed_dt(canoe_block_t b, double dt);

/* User explicit source of the stage: the viscous and thermal dissipation
 * of the dense sinking bubble example with diffusivity K [m^2/s] and
 * reference pressure p0 of its potential temperature, added into du with
 * the stage weight before the implicit solve (the Diffusion function that
 * examples/2019-Li-snap/straka.cpp:125-190 enrolls with
 * EnrollUserExplicitSourceFunction, applied by
 * ImplicitHydroTasks::AddSourceTerms, src/tasklist/implicit_hydro_tasks.cpp:
 * 192-216).  2-D blocks (nx3 = 1) only; K = 0 turns it off. */
int canoe_block_set_diffusion(canoe_block_t b, double K, double p0);

/* wait for the block's stream (steps are asynchronous) */
int canoe_block_synchronize(canoe_block_t b);

/* Hydro::NewBlockTimeStep with canoe patches/21.new_blockdt.patch:20-40;
 * reads back the CFL time step of the current state. */
int canoe_block_new_dt(canoe_block_t b, double *dt_out);

/* Use the network m (NULL: none) for the saturation adjustment of every
 * following step, in the gated start mode.  The network must outlive its
 * use by the block.  No reference counterpart. */
int canoe_block_set_mlp(canoe_block_t b, canoe_mlp_t m);

/* read and clear the block's saturation-adjustment counters {cells,
 * evaluations of f, fallbacks, not converged} accumulated by its steps */
int canoe_block_satadj_stats(canoe_block_t b, unsigned long long *h_stats);

/* read and clear the block's device error word (canoe_errbit bits) */
int canoe_block_error_word(canoe_block_t b, uint32_t *bits);

/* Threads per x1 pencil (CTA of the column kernel): a multiple of 32 in
 * 64..256, 0 for the default (with the 3x3 implicit solve the column height
 * rounded up to a multiple of 32, within 64..128; 224 with the 5x5 solve;
 * 160 otherwise).  Kernels without the 3x3 solve use at most 160
 * and the 5x5 solve always 224.  Results do not depend on it.  No reference
 * counterpart (the reference sweeps columns serially). */
int canoe_block_set_column_threads(canoe_block_t b, int threads);

/* Cells per thread of the x2 / x3 register-window flux runs (4..256; 0 = 16
 * with the FP32 flux path, 32 in FP64).  The results do not depend on it.
 * No reference counterpart: the reference's CalculateFluxes loops over
 * whole pencils (patches/19.calculate_fluxes.patch). */
int canoe_block_set_flux_run(canoe_block_t b, int cells);

/* The block's launch shapes: threads per x1 pencil and cells per x2 / x3
 * flux run (0 = the defaults), as set or as canoe_batch_autotune chose them.
 * No reference counterpart. */
int canoe_block_get_shapes(canoe_block_t b, int32_t *col_threads, int32_t *flux_run);

/* ---------------- batches of uneven blocks ----------------
 * Steps many blocks as one CUDA graph whose branches (one per block, on the
 * block's own stream) run concurrently; each block uses its own device dt
 * (canoe_block_set_fixed_dt or its CFL step).  The reference steps its
 * MeshBlocks one after another in the task list (TaskList::
 * DoTaskListOneStage, called at main.cpp:119-121); no direct counterpart. */
/* ---------------- meshes of MeshBlocks (block boundaries) ----------------
 * Athena refreshes every block's ghost zones from its neighbours between RK
 * stages with the boundary tasks SEND_HYD -> RECV_HYD -> SETB_HYD
 * (patches/24.time_integrator.patch:17-19), run per stage by
 * TaskList::DoTaskListOneStage over all blocks (main.cpp:119-121).  Here the
 * blocks of a mesh stay resident on one GPU and a device copy fills the
 * ghosts.  Blocks split the domain in x2 / x3 only (x1, the vertical, stays
 * whole so that the hydrostatic scan and the implicit column solve stay in
 * one block); neighbours share nx1, the x1 faces, the thermodynamics and the
 * extent of the shared face. */

/* Declare nb the neighbour of b across side (2 ix2, 3 ox2, 4 ix3, 5 ox3);
 * b's bc[side] must be CANOE_BC_BLOCK.  A periodic domain is the mesh whose
 * edge blocks name each other (Athena's periodic neighbour).
 * BoundaryValues' neighbour list (bvals.hpp, NeighborBlock). */
int canoe_block_set_neighbor(canoe_block_t b, int side, canoe_block_t nb);

/* One RK stage (0, 1, 2) of one block on its stream: the per-stage task
 * list of ImplicitHydroTasks (src/tasklist/implicit_hydro_tasks.cpp:45-313)
 * up to cons2prim with the physical boundaries: CalculateFluxes ->
 * IntegrateHydro -> AddSourceTerms -> ImplicitCorrection -> (stage 2)
 * UpdateAllConserved -> ConservedToPrimitive.  dt > 0 at stage 0 sets the
 * step's dt (the host's Mesh::dt); dt <= 0 keeps the device dt of the last
 * completed step.  Stage 2 ends with the block's own CFL dt
 * (canoe_block_new_dt), from which the host takes the mesh minimum
 * (Mesh::NewTimeStep). */
int canoe_block_stage(canoe_block_t b, int stage, double dt);

/* SEND_HYD / RECV_HYD / SETB_HYD of block b as one device copy on b's
 * stream: the NGHOST ghost layers of the primitive state on every
 * CANOE_BC_BLOCK side are copied from the neighbour's interior.  The
 * neighbours' stage must be complete (same stream, or ordered by the host). */
int canoe_block_exchange_ghosts(canoe_block_t b);

/* The ghost exchange across GPUs, for blocks whose neighbour lives on
 * another device (each rank a process, one GPU each, the transfer by NCCL
 * or peer copies): pack copies the NGHOST interior layers of b next to
 * `side` -- what the neighbour across `side` needs -- into the contiguous
 * device buffer d_buf; unpack writes a buffer received from the neighbour
 * across `side` into b's ghost layers on that side.  Both run on b's
 * stream.  Buffers hold NV x nx3 x NGHOST x nc1 doubles for an x2 side and
 * NV x NGHOST x nx2 x nc1 for an x3 side (canoe_block_side_doubles).
 * The MPI send / receive of Athena's BoundaryVariable (bvals_cc.cpp, with
 * the cubed-sphere hook of patches/33.bvals_cc_cpp.patch:21). */
int canoe_block_side_doubles(canoe_block_t b, int side, int64_t *n);
int canoe_block_pack_side(canoe_block_t b, int side, double *d_buf);
int canoe_block_unpack_side(canoe_block_t b, int side, const double *d_buf);

/* A mesh of blocks whose block sides name each other: canoe_mesh_step runs
 * every RK stage of every block on the mesh's stream with the ghost
 * exchange between stages and the mesh-wide CFL minimum (dt <= 0), as
 * main.cpp:119-121 drives the task list.  Blocks must outlive the mesh.
 * The FP32 flux path's reference pressure becomes the mesh-wide level mean
 * of the blocks' states at creation. */
int canoe_mesh_create(canoe_block_t *blocks, int n, canoe_mesh_t *out);
int canoe_mesh_destroy(canoe_mesh_t m);
int canoe_mesh_use_graph(canoe_mesh_t m, int on);
int canoe_mesh_step(canoe_mesh_t m, double dt);
int canoe_mesh_new_dt(canoe_mesh_t m, double *dt_out);
int canoe_mesh_synchronize(canoe_mesh_t m);

int canoe_batch_create(canoe_block_t *blocks, int n, canoe_batch_t *out);
int canoe_batch_destroy(canoe_batch_t q);
int canoe_batch_use_graph(canoe_batch_t q, int on);
int canoe_batch_step(canoe_batch_t q);
int canoe_batch_synchronize(canoe_batch_t q);
/* pick, by timing, the fastest threads per x1 pencil of every block (each
 * block timed alone) and then the fastest cells per x2 / x3 flux run for the
 * batch (the whole batch timed); the blocks' states are restored;
 * h_threads[n] (may be NULL) gets the thread choices, canoe_block_get_shapes
 * both */
int canoe_batch_autotune(canoe_batch_t q, int32_t *h_threads);

/* ---------------- cubed-sphere shell (exo3) ----------------
 * All six panels resident on one GPU in one array (6, NV, nc3, nc2, nc1),
 * panel p = blockID - 1; conserved momenta covariant, primitive velocities
 * contravariant (patches/26.adiabatic_hydro.patch).  The path is dry
 * (ny = 0), HLLC and FP64, like the reference's exo3 build
 * (cmake/examples/exo3.cmake: RSOLVER hllc_transform). */

/* the six MeshBlocks of CubedSphere (src/exo3/cubed_sphere.cpp:25-33) with
 * the GnomonicEquiangle tables (gnomonic_equiangle.cpp:24-222) */
int canoe_shell_create(const canoe_shell_config_t *cfg, canoe_shell_t *out);
int canoe_shell_destroy(canoe_shell_t s);
int canoe_shell_dims(canoe_shell_t s, int32_t *nv, int32_t *nc1, int32_t *nc2,
                     int32_t *nc3);
int canoe_shell_set_stream(canoe_shell_t s, void *stream);

/* load the host conserved state of all panels; fill != 0 then runs the panel
 * ghost exchange and cons -> prim (the boundary step of the task list) */
int canoe_shell_set_conserved(canoe_shell_t s, const double *h_u, int fill);
int canoe_shell_get_conserved(canoe_shell_t s, double *h_u);
int canoe_shell_get_primitive(canoe_shell_t s, double *h_w);

/* Panel ghost exchange of the conserved state on device: what
 * cs::PackData (src/exo3/cubed_sphere_utility.cpp:379-623, hooked at
 * patches/33.bvals_cc_cpp.patch:21) with InteprolateX2/X3 (:100-376) and
 * CubedSphere::TransformOX (cs_transform_ox.cpp:11-230) send over MPI, as one
 * gather with interpolation and velocity rotation per ghost cell. */
int canoe_shell_fill_ghosts(canoe_shell_t s);

/* Hydro::CalculateFluxes of every panel with the CUBED_SPHERE branches of
 * patches/19.calculate_fluxes.patch, including the L/R face-state swap of
 * CubedSphere::SynchronizeFluxes{Send,Recv,Wait} (cubed_sphere.cpp:250-681).
 * Device outputs (6, NV, nc3, nc2, nc1+1), (6, NV, nc3, nc2+1, nc1),
 * (6, NV, nc3+1, nc2, nc1); d_f1 may be NULL. */
int canoe_shell_calculate_fluxes(canoe_shell_t s, double *d_f1, double *d_f2, double *d_f3);

/* One RK3 step of all panels with time step dt (> 0). */
int canoe_shell_step(canoe_shell_t s, double dt);
int canoe_shell_synchronize(canoe_shell_t s);
int canoe_shell_error_word(canoe_shell_t s, uint32_t *bits);

#ifdef __cplusplus
}
#endif

#endif /* CANOE_B200_H_ */
