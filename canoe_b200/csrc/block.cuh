// block.cuh -- MeshBlock geometry as seen by the kernels, kernel launchers
// shared between translation units, and the block object behind the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "physics.cuh"

namespace cb {

// Geometry of one MeshBlock in the reference layout (NV, nc3, nc2, nc1),
// i fastest (canoe src/interface/hydro.hpp:54-67).
struct Geom {
  int ny, nv;
  int nx1, nx2, nx3, nc1, nc2, nc3;
  int is, ie, js, je, ks, ke;
  int f2, f3;
  int bc[6];
  int64_t sk;  // stride between k planes  (nc2 * nc1)
  int64_t sv;  // stride between variables (nc3 * nc2 * nc1)
  double dx2, dx3;
  const double *x1f, *x1v, *dx1f;  // device arrays, nc1+1 / nc1 / nc1
  // horizontally uniform reference pressure per x1 level (nc1): the FP32
  // flux path works on p' = p - pref so that p ~ 1e5 never enters FP32
  const double *pref;
  // device error word (canoe_errbit) for kernels that report on their own
  uint32_t *err;
  // set per launch: 1 when the pencil rows may be moved by bulk copies
  // (16-byte aligned arrays, nc1 even)
  int bulk;
  // cubed-sphere panel: device geometry tables (kShellTabs arrays of
  // nc3 * nc2 doubles, row-major [k][j]); null for a Cartesian block
  const double *shell;
  // threads per x1 pencil (a multiple of 32 in 64..160; 0 = 160), chosen
  // per block by canoe_batch_autotune
  int col_threads;
  // cells per thread of the x2 / x3 register-window flux runs (4..256; 0 =
  // 16 in FP32, 32 in FP64), chosen per block by canoe_batch_autotune; the
  // results do not depend on it
  int flux_run = 0;
  // x1 pencil launches over npanel equal blocks stored pstride doubles apart
  // (the six panels of a cubed-sphere shell share one geometry)
  int npanel = 1;
  int64_t pstride = 0;
};

// geometry tables of a cubed-sphere panel (gnomonic_equiangle.cpp:140-222)
enum ShellTab {
  kTabCosC, kTabSinC,     // cell cosine / sine of the coordinate angle
  kTabCosF2, kTabSinF2,   // at x2 faces
  kTabCosF3, kTabSinF3,   // at x3 faces
  kTabDx2A, kTabDx3A,     // angular widths of the cell
  kTabDx2AF3, kTabDx3AF2, // angular widths along x3 / x2 faces
  kTabCth1, kTabCth2, kTabCth3,  // flux-projection cosines (cell, x2 face, x3 face)
  kShellTabs
};

// RK3 (SSPRK(3,3), Shu & Osher 1988) register weights per stage:
// u = g1 u + g2 u1, du weight beta (ImplicitHydroTasks::IntegrateHydro).
struct Stage {
  double g1, g2, beta;
};
extern const Stage kRK3[3];

// error reporting ----------------------------------------------------------
void set_error(const std::string &msg);
int cuda_status(cudaError_t e, const char *what);
#define CB_CUDA(call)                                   \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) return cb::cuda_status(e_, #call); \
  } while (0)

// kernels launched from the step driver (defined in flux.cu, update.cu,
// eos.cu).  `dtp` points at the device copy of the step's dt; every kernel
// multiplies it by the stage's beta so that a step can be captured in a CUDA
// graph without baking dt in.
// x1 pencil kernel (column.cuh) modes.  kColFluxOnly: x1 fluxes out
// (flx_out and the x1 part of du); kColStep: the fused stage (x1 divergence,
// x1 solve, register update of u); kColSolveOnly: the x1 solve of a given du;
// kColDivOnly: du += x1 divergence and sources, written back (the x2 / x3
// solves run next); kColSolveStep: the x1 solve of the stored du and the
// register update
enum ColMode { kColFluxOnly = 0, kColStep = 1, kColSolveOnly = 2, kColDivOnly = 3,
               kColSolveStep = 4 };
int launch_x1col(const Geom &g, const canoe_thermo_t &th, int recon, int rs,
                 int implicit_flag, int precision, int mode, const double *w, double *du, double *u,
                 double *u1, const double *dtp, const Stage &s, int stage,
                 double *flx_out, cudaStream_t st);
// implicit solves along x2 (dir 1) and x3 (dir 2) of a dry block (lines.cu):
// whether the flag asks for one in a direction the block has, the doubles
// of each of the two line-major scratch arrays, and the solve of du in place
// (wt, dut: scratch; dxl: nx_dir + 2 NGHOST line spacings)
bool line_solve_on(const Geom &g, int implicit_flag, int dir);
size_t line_scratch_doubles(const Geom &g, int implicit_flag);
int launch_line_solve(int dir, const Geom &g, const canoe_thermo_t &th, int implicit_flag,
                      const double *w, double *du, double *wt, double *dut,
                      const double *dxl, const double *dtp, const Stage &s,
                      cudaStream_t st);
int launch_flux_x23(int dir, const Geom &g, const canoe_thermo_t &th, int recon,
                    int rs, int precision, const double *w, double *du,
                    const double *dtp, double beta, double *flx_out,
                    cudaStream_t st);
int launch_cons_to_prim(const Geom &g, const canoe_thermo_t &th, const double *u,
                        double *w, uint32_t *err, unsigned long long *dt_acc,
                        double cfl, int implicit_flag, cudaStream_t st);
int launch_level_mean_pressure(const Geom &g, int ny, const double *w, double *pref,
                               cudaStream_t st);
int launch_dt_finalize(double *d_dt, unsigned long long *dt_acc, double cfl,
                       double fixed_dt, cudaStream_t st);
struct MlpView;
int launch_satadj(const canoe_thermo_t &th, const canoe_satadj_opts_t &o,
                  double *u, int64_t ncells, int64_t stride, const Geom *g,
                  const double *t_guess, double *t_out, int32_t *iters,
                  unsigned long long *stats, cudaStream_t st,
                  const MlpView *mlp = nullptr, double *guess_out = nullptr,
                  uint32_t *err = nullptr);
MlpView mlp_view(const struct canoe_mlp *m);

// ghost slabs copied between neighbouring blocks (exchange.cu): NV x nk x
// nj rows of nc1 doubles; dst / src point at the first row's first cell,
// variable and k strides in doubles for each side (j rows are nc1 apart)
struct Slab {
  double *dst;
  const double *src;
  int64_t dsv, dsk, ssv, ssk;
  int nk, nj;
};
struct SlabSet {
  Slab s[4];
  int n, nv, nc1;
};
int launch_exchange(const SlabSet &ss, cudaStream_t st);

// the dissipation source of the dense sinking bubble (source.cu): du +=
// beta dt K rho / (dx dy) (lap v1, lap v2, cp T / theta lap theta), 2-D
int launch_diffusion(const Geom &g, const canoe_thermo_t &th, const double *w, double *du,
                     const double *dtp, double beta, double K, double p0, cudaStream_t st);

// all checks a block configuration passes before a step runs on it (capi.cu);
// 0 or a canoe_status with the message set
int validate_block_config(const canoe_block_config_t &c);

// raise a kernel's dynamic shared-memory limit once per (kernel, size)
int ensure_smem(const void *kernel, size_t bytes);


}  // namespace cb
