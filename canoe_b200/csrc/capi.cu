// capi.cu -- the extern "C" boundary (include/canoe_b200.h): MeshBlock
// objects that own their device arrays, the RK3 step driver, and the
// operator-level entry points.  There is no CPU fallback: every entry point
// runs CUDA kernels or returns an error.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "column.cuh"
#include "mlp.cuh"

namespace cb {

const Stage kRK3[3] = {{0., 1., 1.}, {0.25, 0.75, 0.25}, {2. / 3., 1. / 3., 2. / 3.}};

static thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }

int cuda_status(cudaError_t e, const char *what) {
  g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
  return CANOE_ERR_CUDA;
}

int ensure_smem(const void *kernel, size_t bytes) {
  static std::mutex mu;
  static std::map<const void *, size_t> done;
  std::lock_guard<std::mutex> lk(mu);
  auto it = done.find(kernel);
  if (it != done.end() && it->second >= bytes) return 0;
  if (bytes > 48 * 1024)
    CB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)bytes));
  done[kernel] = bytes;
  return 0;
}

namespace {

// operator-level Riemann kernel over (NV, n) face arrays
template <int NY, int RS, int DIR>
__global__ void k_riemann_faces(canoe_thermo_t th, const double *__restrict__ wl,
                                const double *__restrict__ wr,
                                double *__restrict__ flx, int64_t n) {
  constexpr int NV = 5 + NY;
  int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= n) return;
  double a[NV], b[NV], o[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    a[v] = wl[v * n + f];
    b[v] = wr[v * n + f];
  }
  riemann<double, NY, RS, DIR>(th, a, b, o);
#pragma unroll
  for (int v = 0; v < NV; ++v) flx[v * n + f] = o[v];
}

template <int NY, int RS>
int riemann_faces(const canoe_thermo_t &th, int dir, const double *wl,
                  const double *wr, double *flx, int64_t n, cudaStream_t st) {
  unsigned nb = (unsigned)((n + 127) / 128);
  if (dir == 0) k_riemann_faces<NY, RS, 0><<<nb, 128, 0, st>>>(th, wl, wr, flx, n);
  else if (dir == 1) k_riemann_faces<NY, RS, 1><<<nb, 128, 0, st>>>(th, wl, wr, flx, n);
  else k_riemann_faces<NY, RS, 2><<<nb, 128, 0, st>>>(th, wl, wr, flx, n);
  CB_CUDA(cudaGetLastError());
  return 0;
}

int riemann_entry(int rs, const canoe_thermo_t *th, int ivx, const double *wl,
                  const double *wr, double *flx, int64_t n, void *stream) {
  if (!th || !wl || !wr || !flx || n < 0) {
    set_error("null pointer or negative size");
    return CANOE_ERR_ARG;
  }
  const int dir = ivx - (1 + th->ny);
  if (dir < 0 || dir > 2) {
    set_error("ivx must be IVX, IVY or IVZ");
    return CANOE_ERR_ARG;
  }
  if (n == 0) return 0;
  cudaStream_t st = (cudaStream_t)stream;
#define CB_R(NY) \
  return rs == CANOE_RSOLVER_LMARS ? riemann_faces<NY, 0>(*th, dir, wl, wr, flx, n, st) \
                                   : riemann_faces<NY, 1>(*th, dir, wl, wr, flx, n, st)
  switch (th->ny) {
    case 0: CB_R(0);
    case 1: CB_R(1);
    case 2: CB_R(2);
    case 3: CB_R(3);
    case 6: CB_R(6);
    default:
      set_error("unsupported number of mass-fraction slots");
      return CANOE_ERR_UNSUPPORTED;
  }
#undef CB_R
}

int check_thermo(const canoe_thermo_t &th) {
  if (th.ny < 0 || th.ny > CANOE_MAX_NY || th.nvapor < 0 || th.nvapor > th.ny ||
      th.nvapor > CANOE_MAX_VAPOR) {
    set_error("invalid species counts in canoe_thermo_t");
    return CANOE_ERR_ARG;
  }
  if (!(th.gammad > 1.) || !(th.rd > 0.)) {
    set_error("invalid gammad / rd");
    return CANOE_ERR_ARG;
  }
  for (int v = 0; v < th.nvapor; ++v) {
    for (int s : {th.liq_slot[v], th.ice_slot[v]})
      if (s != -1 && (s <= th.nvapor || s > th.ny)) {
        set_error("condensate slot outside the cloud range");
        return CANOE_ERR_ARG;
      }
  }
  return 0;
}

}  // namespace
}  // namespace cb

using namespace cb;

struct canoe_block {
  canoe_block_config_t cfg;
  Geom g;
  canoe_thermo_t th;
  double *d_u = nullptr, *d_w = nullptr, *d_u1 = nullptr, *d_du = nullptr;
  double *d_x1f = nullptr, *d_x1v = nullptr, *d_dx1f = nullptr;
  double *d_scr = nullptr, *d_dt = nullptr, *d_pref = nullptr;
  unsigned long long *d_dtacc = nullptr;
  unsigned long long *d_sat = nullptr;  // saturation-adjustment statistics
  uint32_t *d_err = nullptr;
  // x2 / x3 implicit solves: line-major scratch of w and du, line spacings
  // (nx2 + 2 NG entries of dx2, then nx3 + 2 NG of dx3)
  double *d_wt = nullptr, *d_dut = nullptr, *d_dxl = nullptr;
  bool lines = false;
  cudaStream_t st = nullptr;
  bool own_stream = false;
  cudaGraphExec_t gexec = nullptr;
  bool graph = false;
  double fixed_dt = 0.;  // > 0: every step uses this dt instead of the CFL one
  canoe_mlp_t mlp = nullptr;  // learned warm start of the saturation adjustment
  size_t nvals = 0;
  // block boundaries: the neighbour across each side and the ghost slabs of
  // w that canoe_block_exchange_ghosts copies from the neighbours
  canoe_block *nb[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  SlabSet slabs{};
  // user source: the sinking bubble's dissipation (diffusivity, p0; 0 = off)
  double diff_K = 0., diff_p0 = 1.e5;
};

// Every check a block configuration must pass before a step may run on it
// (shared by canoe_block_create and canoe_block_step_noalloc, so that the two
// entry points accept exactly the same configurations).
namespace cb {
int validate_block_config(const canoe_block_config_t &c) {
  if (int rc = check_thermo(c.thermo)) return rc;
  if (c.nx1 < 4 || c.nx2 < 1 || c.nx3 < 1 || !c.h_x1f) {
    set_error("block needs nx1 >= 4, nx2, nx3 >= 1 and x1 faces");
    return CANOE_ERR_ARG;
  }
  if (c.nx3 > 1 && c.nx2 == 1) {
    set_error("a 3-D block needs nx2 > 1");
    return CANOE_ERR_ARG;
  }
  if (c.recon != CANOE_RECON_PLM && c.recon != CANOE_RECON_PPM) {
    set_error("recon must be 2 (PLM) or 3 (PPM)");
    return CANOE_ERR_ARG;
  }
  if (c.rsolver != CANOE_RSOLVER_LMARS && c.rsolver != CANOE_RSOLVER_HLLC) {
    set_error("unknown Riemann solver");
    return CANOE_ERR_ARG;
  }
  if (c.precision != CANOE_FP64 && c.precision != CANOE_FP32_PERTURBATION) {
    set_error("precision must be CANOE_FP64 or CANOE_FP32_PERTURBATION");
    return CANOE_ERR_ARG;
  }
  for (int q = 0; q < 6; ++q) {
    const int f = c.bc[q];
    const bool phys = f == CANOE_BC_REFLECT || f == CANOE_BC_PERIODIC || f == CANOE_BC_OUTFLOW;
    // x1 (the vertical) is never split between blocks: the hydrostatic scan
    // and the implicit column solve stay in one block
    if (!(phys || (q >= 2 && f == CANOE_BC_BLOCK))) {
      set_error(q < 2 ? "x1 boundaries must be reflect, periodic or outflow"
                      : "x2 / x3 boundaries must be reflect, periodic, outflow or block");
      return CANOE_ERR_ARG;
    }
  }
  if ((c.bc[2] == CANOE_BC_BLOCK || c.bc[3] == CANOE_BC_BLOCK) && c.nx2 > 1 &&
      (c.implicit_flag & 2)) {
    set_error("an implicit x2 solve across a block boundary is not provided");
    return CANOE_ERR_UNSUPPORTED;
  }
  if ((c.bc[4] == CANOE_BC_BLOCK || c.bc[5] == CANOE_BC_BLOCK) && c.nx3 > 1 &&
      (c.implicit_flag & 4)) {
    set_error("an implicit x3 solve across a block boundary is not provided");
    return CANOE_ERR_UNSUPPORTED;
  }
  if ((((c.implicit_flag & 2) && c.nx2 > 1) || ((c.implicit_flag & 4) && c.nx3 > 1)) &&
      c.thermo.ny > 0) {
    // the reference's moist x2 / x3 update reads w at the transposed
    // indices (forward_backward.hpp:107-110 under solve_implicit_3d.cpp:
    // 35-89), i.e. at unrelated cells
    set_error("x2 / x3 implicit solves are provided for a dry block");
    return CANOE_ERR_UNSUPPORTED;
  }
  for (int i = 0; i < c.nx1; ++i)
    if (!(c.h_x1f[i + 1] > c.h_x1f[i])) {
      set_error("x1 faces must increase");
      return CANOE_ERR_ARG;
    }
  if (c.recon == CANOE_RECON_PPM) {
    double d0 = c.h_x1f[1] - c.h_x1f[0];
    for (int i = 1; i < c.nx1; ++i)
      if (std::fabs((c.h_x1f[i + 1] - c.h_x1f[i]) - d0) > 1e-9 * d0) {
        set_error("PPM needs a uniform x1 grid");
        return CANOE_ERR_UNSUPPORTED;
      }
  }
  return 0;
}
}  // namespace cb

static int block_free(canoe_block *b) {
  if (!b) return 0;
  if (b->gexec) cudaGraphExecDestroy(b->gexec);
  for (void *p : {(void *)b->d_u, (void *)b->d_w, (void *)b->d_u1, (void *)b->d_du,
                  (void *)b->d_x1f, (void *)b->d_x1v, (void *)b->d_dx1f,
                  (void *)b->d_scr, (void *)b->d_dt, (void *)b->d_pref, (void *)b->d_dtacc,
                  (void *)b->d_err, (void *)b->d_sat, (void *)b->d_wt, (void *)b->d_dut,
                  (void *)b->d_dxl})
    if (p) cudaFree(p);
  if (b->own_stream && b->st) cudaStreamDestroy(b->st);
  delete b;
  return 0;
}

// optional per-kernel-class timing of a step (CUDA events on b->st)
struct StepTimer {
  cudaEvent_t ev[64];
  int cls[64];
  int n = 0;
  int mark(cudaStream_t st, int c) {
    if (n >= 64) return 0;
    cls[n] = c;
    CB_CUDA(cudaEventRecord(ev[n++], st));
    return 0;
  }
};

// the x3 then x2 implicit solves of du, in place (solve_implicit_3d.cpp:25-89)
static int line_solves(canoe_block *b, double *du, const double *dtp, const Stage &sg) {
  const Geom &g = b->g;
  for (int dir = 2; dir >= 1; --dir) {
    if (!line_solve_on(g, b->cfg.implicit_flag, dir)) continue;
    const double *dxl = b->d_dxl + (dir == 2 ? g.nx2 + 2 * NG : 0);
    if (int rc = launch_line_solve(dir, g, b->th, b->cfg.implicit_flag, b->d_w, du, b->d_wt,
                                   b->d_dut, dxl, dtp, sg, b->st))
      return rc;
  }
  return 0;
}

// one RK stage of block b on stream st (the per-stage task list up to
// cons2prim with the physical boundaries); dtp: the step's device dt, acc:
// the CFL accumulator fed at the last stage
static int stage_launches(canoe_block *b, int s, double *dtp, unsigned long long *acc,
                          cudaStream_t st, StepTimer *tm = nullptr) {
  const Geom &g = b->g;
  const Stage &sg = kRK3[s];
  int rc;
#define CB_MARK(c) \
  if (tm && (rc = tm->mark(st, c))) return rc;
  CB_MARK(-1);
  if (g.f2 && (rc = launch_flux_x23(1, g, b->th, b->cfg.recon, b->cfg.rsolver, b->cfg.precision,
                                    b->d_w, b->d_du, dtp, sg.beta, nullptr, st)))
    return rc;
  CB_MARK(1);
  if (g.f3 && (rc = launch_flux_x23(2, g, b->th, b->cfg.recon, b->cfg.rsolver, b->cfg.precision,
                                    b->d_w, b->d_du, dtp, sg.beta, nullptr, st)))
    return rc;
  CB_MARK(2);
  // user sources into du (AddSourceTerms), before the x1 pencil solves it
  if (b->diff_K > 0. &&
      (rc = launch_diffusion(g, b->th, b->d_w, b->d_du, dtp, sg.beta, b->diff_K, b->diff_p0, st)))
    return rc;
  if (!b->lines) {
    if ((rc = launch_x1col(g, b->th, b->cfg.recon, b->cfg.rsolver, b->cfg.implicit_flag,
                           b->cfg.precision, kColStep, b->d_w, b->d_du, b->d_u, b->d_u1, dtp,
                           sg, s, nullptr, st)))
      return rc;
  } else {
    // du complete before the x3, x2, x1 solves (solve_implicit_3d.cpp:25-142)
    if ((rc = launch_x1col(g, b->th, b->cfg.recon, b->cfg.rsolver, b->cfg.implicit_flag,
                           b->cfg.precision, kColDivOnly, b->d_w, b->d_du, b->d_u, b->d_u1,
                           dtp, sg, s, nullptr, st)))
      return rc;
    for (int dir = 2; dir >= 1; --dir) {
      if (!line_solve_on(g, b->cfg.implicit_flag, dir)) continue;
      const double *dxl = b->d_dxl + (dir == 2 ? g.nx2 + 2 * NG : 0);
      if ((rc = launch_line_solve(dir, g, b->th, b->cfg.implicit_flag, b->d_w, b->d_du,
                                  b->d_wt, b->d_dut, dxl, dtp, sg, st)))
        return rc;
    }
    if ((rc = launch_x1col(g, b->th, b->cfg.recon, b->cfg.rsolver, b->cfg.implicit_flag,
                           b->cfg.precision, kColSolveStep, b->d_w, b->d_du, b->d_u, b->d_u1,
                           dtp, sg, s, nullptr, st)))
      return rc;
  }
  CB_MARK(0);
  if (s == 2 && b->cfg.satadj && b->th.ny > 0) {
    canoe_satadj_opts_t o{1e-8, 30, b->mlp ? 2 : 0};
    const int64_t nin = (int64_t)g.nx1 * g.nx2 * g.nx3;
    MlpView mv;
    if (b->mlp) mv = mlp_view(b->mlp);
    if ((rc = launch_satadj(b->th, o, b->d_u, nin, g.sv, &g, nullptr, nullptr, nullptr,
                            b->d_sat, st, b->mlp ? &mv : nullptr, nullptr, b->d_err)))
      return rc;
    CB_MARK(4);
  }
  if ((rc = launch_cons_to_prim(g, b->th, b->d_u, b->d_w, b->d_err, s == 2 ? acc : nullptr,
                                b->cfg.cfl, b->cfg.implicit_flag, st)))
    return rc;
  CB_MARK(5);
#undef CB_MARK
  return 0;
}

// one RK3 step, all launches on b->st; fixed_dt <= 0 uses the device dt
static int step_launches(canoe_block *b, double fixed_dt, StepTimer *tm = nullptr) {
  int rc;
  if (tm && (rc = tm->mark(b->st, -1))) return rc;
  if (fixed_dt > 0.) {
    // write the fixed dt; the accumulator reset is harmless here
    if ((rc = launch_dt_finalize(b->d_dt, b->d_dtacc, b->cfg.cfl, fixed_dt, b->st))) return rc;
  }
  for (int s = 0; s < 3; ++s)
    if ((rc = stage_launches(b, s, b->d_dt, b->d_dtacc, b->st, tm))) return rc;
  if ((rc = launch_dt_finalize(b->d_dt, b->d_dtacc, b->cfg.cfl, b->fixed_dt, b->st))) return rc;
  if (tm && (rc = tm->mark(b->st, 6))) return rc;
  return 0;
}

extern "C" {

const char *canoe_version(void) { return "canoe_b200 0.1 (sm_100a)"; }

const char *canoe_last_error(void) { return g_last_error.c_str(); }

int canoe_device_sm_count(int *out) {
  int dev = 0;
  CB_CUDA(cudaGetDevice(&dev));
  CB_CUDA(cudaDeviceGetAttribute(out, cudaDevAttrMultiProcessorCount, dev));
  return 0;
}

int canoe_riemann_lmars(const canoe_thermo_t *th, int ivx, const double *wl,
                        const double *wr, double *flx, int64_t n, void *stream) {
  return riemann_entry(CANOE_RSOLVER_LMARS, th, ivx, wl, wr, flx, n, stream);
}

int canoe_riemann_hllc(const canoe_thermo_t *th, int ivx, const double *wl,
                       const double *wr, double *flx, int64_t n, void *stream) {
  return riemann_entry(CANOE_RSOLVER_HLLC, th, ivx, wl, wr, flx, n, stream);
}

int canoe_saturation_adjust(const canoe_thermo_t *th, const canoe_satadj_opts_t *opts,
                            double *d_u, int64_t ncells, const double *d_t_guess,
                            double *d_t_out, int32_t *d_iters,
                            unsigned long long *d_stats, void *stream) {
  if (!th || !opts || !d_u || ncells < 0) {
    set_error("null pointer or negative size");
    return CANOE_ERR_ARG;
  }
  if (int rc = check_thermo(*th)) return rc;
  if (opts->warm && !d_t_guess) {
    set_error("warm start requested without t_guess");
    return CANOE_ERR_ARG;
  }
  if (!(opts->tol > 0.) || opts->max_iter < 1) {
    set_error("tol must be > 0 and max_iter >= 1");
    return CANOE_ERR_ARG;
  }
  return launch_satadj(*th, *opts, d_u, ncells, ncells, nullptr, d_t_guess, d_t_out,
                       d_iters, d_stats, (cudaStream_t)stream);
}

int canoe_block_create(const canoe_block_config_t *cfg, canoe_block_t *out) {
  if (!cfg || !out) {
    set_error("null pointer");
    return CANOE_ERR_ARG;
  }
  *out = nullptr;
  if (int rc = validate_block_config(*cfg)) return rc;
  canoe_block *b = new canoe_block();
  b->cfg = *cfg;
  b->cfg.h_x1f = nullptr;
  b->th = cfg->thermo;
  Geom &g = b->g;
  g.ny = b->th.ny;
  g.nv = 5 + g.ny;
  g.nx1 = cfg->nx1;
  g.nx2 = cfg->nx2;
  g.nx3 = cfg->nx3;
  g.f2 = cfg->nx2 > 1;
  g.f3 = cfg->nx3 > 1;
  g.nc1 = g.nx1 + 2 * NG;
  g.nc2 = g.f2 ? g.nx2 + 2 * NG : 1;
  g.nc3 = g.f3 ? g.nx3 + 2 * NG : 1;
  g.is = NG;
  g.ie = NG + g.nx1 - 1;
  g.js = g.f2 ? NG : 0;
  g.je = g.js + g.nx2 - 1;
  g.ks = g.f3 ? NG : 0;
  g.ke = g.ks + g.nx3 - 1;
  for (int q = 0; q < 6; ++q) g.bc[q] = cfg->bc[q];
  g.sk = (int64_t)g.nc2 * g.nc1;
  g.sv = (int64_t)g.nc3 * g.sk;
  g.dx2 = cfg->dx2;
  g.dx3 = cfg->dx3;
  // x1 geometry with mirrored ghost faces
  std::vector<double> xf(g.nc1 + 1), xv(g.nc1), dx(g.nc1);
  for (int i = 0; i <= g.nx1; ++i) xf[g.is + i] = cfg->h_x1f[i];
  for (int q = 1; q <= NG; ++q) {
    xf[g.is - q] = 2. * xf[g.is] - xf[g.is + q];
    xf[g.ie + 1 + q] = 2. * xf[g.ie + 1] - xf[g.ie + 1 - q];
  }
  for (int i = 0; i < g.nc1; ++i) {
    xv[i] = 0.5 * (xf[i] + xf[i + 1]);
    dx[i] = xf[i + 1] - xf[i];
  }
  b->nvals = (size_t)g.nv * g.sv;
  const size_t bytes = b->nvals * sizeof(double);
  int rc = 0;
  auto fail = [&](cudaError_t e, const char *w) {
    rc = cuda_status(e, w);
    block_free(b);
    return rc;
  };
  cudaError_t e;
  if ((e = cudaMalloc(&b->d_u, bytes))) return fail(e, "cudaMalloc u");
  if ((e = cudaMalloc(&b->d_w, bytes))) return fail(e, "cudaMalloc w");
  if ((e = cudaMalloc(&b->d_u1, bytes))) return fail(e, "cudaMalloc u1");
  if ((e = cudaMalloc(&b->d_du, bytes))) return fail(e, "cudaMalloc du");
  if ((e = cudaMalloc(&b->d_x1f, (g.nc1 + 1) * sizeof(double)))) return fail(e, "cudaMalloc x1f");
  if ((e = cudaMalloc(&b->d_x1v, g.nc1 * sizeof(double)))) return fail(e, "cudaMalloc x1v");
  if ((e = cudaMalloc(&b->d_dx1f, g.nc1 * sizeof(double)))) return fail(e, "cudaMalloc dx1f");
  if ((e = cudaMalloc(&b->d_dt, 2 * sizeof(double)))) return fail(e, "cudaMalloc dt");
  if ((e = cudaMalloc(&b->d_pref, g.nc1 * sizeof(double)))) return fail(e, "cudaMalloc pref");
  if ((e = cudaMemset(b->d_pref, 0, g.nc1 * sizeof(double)))) return fail(e, "cudaMemset pref");
  if ((e = cudaMalloc(&b->d_dtacc, sizeof(unsigned long long)))) return fail(e, "cudaMalloc dtacc");
  if ((e = cudaMalloc(&b->d_err, sizeof(uint32_t)))) return fail(e, "cudaMalloc err");
  if ((e = cudaMalloc(&b->d_sat, 4 * sizeof(unsigned long long)))) return fail(e, "cudaMalloc sat");
  if ((e = cudaMemset(b->d_sat, 0, 4 * sizeof(unsigned long long)))) return fail(e, "cudaMemset sat");
  if ((e = cudaMemset(b->d_u, 0, bytes))) return fail(e, "cudaMemset u");
  if ((e = cudaMemset(b->d_w, 0, bytes))) return fail(e, "cudaMemset w");
  if ((e = cudaMemset(b->d_u1, 0, bytes))) return fail(e, "cudaMemset u1");
  if ((e = cudaMemset(b->d_du, 0, bytes))) return fail(e, "cudaMemset du");
  if ((e = cudaMemset(b->d_err, 0, sizeof(uint32_t)))) return fail(e, "cudaMemset err");
  unsigned long long inf = 0x7ff0000000000000ULL;
  double zero2[2] = {0., 0.};
  if ((e = cudaMemcpy(b->d_dtacc, &inf, sizeof(inf), cudaMemcpyHostToDevice))) return fail(e, "copy");
  if ((e = cudaMemcpy(b->d_dt, zero2, sizeof(zero2), cudaMemcpyHostToDevice))) return fail(e, "copy");
  if ((e = cudaMemcpy(b->d_x1f, xf.data(), xf.size() * sizeof(double), cudaMemcpyHostToDevice))) return fail(e, "copy");
  if ((e = cudaMemcpy(b->d_x1v, xv.data(), xv.size() * sizeof(double), cudaMemcpyHostToDevice))) return fail(e, "copy");
  if ((e = cudaMemcpy(b->d_dx1f, dx.data(), dx.size() * sizeof(double), cudaMemcpyHostToDevice))) return fail(e, "copy");
  b->lines = line_solve_on(g, cfg->implicit_flag, 1) || line_solve_on(g, cfg->implicit_flag, 2);
  if (b->lines) {
    const size_t nl = line_scratch_doubles(g, cfg->implicit_flag) * sizeof(double);
    if ((e = cudaMalloc(&b->d_wt, nl))) return fail(e, "cudaMalloc line scratch");
    if ((e = cudaMalloc(&b->d_dut, nl))) return fail(e, "cudaMalloc line scratch");
    const int n2 = g.nx2 + 2 * NG, n3 = g.nx3 + 2 * NG;
    std::vector<double> dl(n2 + n3);
    for (int q = 0; q < n2; ++q) dl[q] = g.dx2;
    for (int q = 0; q < n3; ++q) dl[n2 + q] = g.dx3;
    if ((e = cudaMalloc(&b->d_dxl, dl.size() * sizeof(double)))) return fail(e, "cudaMalloc dxl");
    if ((e = cudaMemcpy(b->d_dxl, dl.data(), dl.size() * sizeof(double), cudaMemcpyHostToDevice)))
      return fail(e, "copy");
  }
  if ((e = cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking))) return fail(e, "stream");
  b->own_stream = true;
  g.x1f = b->d_x1f;
  g.x1v = b->d_x1v;
  g.dx1f = b->d_dx1f;
  g.pref = b->d_pref;
  g.err = b->d_err;
  *out = b;
  return 0;
}

int canoe_block_destroy(canoe_block_t b) {
  if (b && b->st) cudaStreamSynchronize(b->st);
  return block_free(b);
}

int canoe_block_dims(canoe_block_t b, int32_t *nv, int32_t *nc1, int32_t *nc2,
                     int32_t *nc3) {
  if (!b) return CANOE_ERR_ARG;
  if (nv) *nv = b->g.nv;
  if (nc1) *nc1 = b->g.nc1;
  if (nc2) *nc2 = b->g.nc2;
  if (nc3) *nc3 = b->g.nc3;
  return 0;
}

int canoe_block_set_stream(canoe_block_t b, void *stream) {
  if (!b) return CANOE_ERR_ARG;
  CB_CUDA(cudaStreamSynchronize(b->st));
  if (b->own_stream) cudaStreamDestroy(b->st);
  b->st = (cudaStream_t)stream;
  b->own_stream = false;
  if (b->gexec) {
    cudaGraphExecDestroy(b->gexec);
    b->gexec = nullptr;
  }
  return 0;
}

int canoe_block_set_conserved(canoe_block_t b, const double *h_u) {
  if (!b || !h_u) return CANOE_ERR_ARG;
  CB_CUDA(cudaMemcpyAsync(b->d_u, h_u, b->nvals * sizeof(double), cudaMemcpyHostToDevice, b->st));
  if (int rc = launch_cons_to_prim(b->g, b->th, b->d_u, b->d_w, b->d_err, b->d_dtacc,
                                   b->cfg.cfl, b->cfg.implicit_flag, b->st))
    return rc;
  if (int rc = launch_dt_finalize(b->d_dt, b->d_dtacc, b->cfg.cfl, 0., b->st)) return rc;
  // reference pressure profile of the FP32 flux path (fixed for the run)
  if (int rc = launch_level_mean_pressure(b->g, b->th.ny, b->d_w, b->d_pref, b->st)) return rc;
  CB_CUDA(cudaStreamSynchronize(b->st));
  return 0;
}

int canoe_block_get_conserved(canoe_block_t b, double *h_u) {
  if (!b || !h_u) return CANOE_ERR_ARG;
  CB_CUDA(cudaMemcpyAsync(h_u, b->d_u, b->nvals * sizeof(double), cudaMemcpyDeviceToHost, b->st));
  CB_CUDA(cudaStreamSynchronize(b->st));
  return 0;
}

int canoe_block_get_primitive(canoe_block_t b, double *h_w) {
  if (!b || !h_w) return CANOE_ERR_ARG;
  CB_CUDA(cudaMemcpyAsync(h_w, b->d_w, b->nvals * sizeof(double), cudaMemcpyDeviceToHost, b->st));
  CB_CUDA(cudaStreamSynchronize(b->st));
  return 0;
}

int canoe_block_device_ptrs(canoe_block_t b, double **d_u, double **d_w) {
  if (!b) return CANOE_ERR_ARG;
  if (d_u) *d_u = b->d_u;
  if (d_w) *d_w = b->d_w;
  return 0;
}

int canoe_block_calculate_fluxes(canoe_block_t b, double *f1, double *f2, double *f3) {
  if (!b || !f1 || (b->g.f2 && !f2) || (b->g.f3 && !f3)) {
    set_error("null flux array");
    return CANOE_ERR_ARG;
  }
  const Geom &g = b->g;
  const Stage one{0., 1., 1.};
  int rc;
  if (g.f2 && (rc = launch_flux_x23(1, g, b->th, b->cfg.recon, b->cfg.rsolver,
                                    b->cfg.precision, b->d_w, b->d_du, b->d_dt, 1., f2, b->st)))
    return rc;
  if (g.f3 && (rc = launch_flux_x23(2, g, b->th, b->cfg.recon, b->cfg.rsolver,
                                    b->cfg.precision, b->d_w, b->d_du, b->d_dt, 1., f3, b->st)))
    return rc;
  if ((rc = launch_x1col(g, b->th, b->cfg.recon, b->cfg.rsolver, b->cfg.implicit_flag,
                         b->cfg.precision, kColFluxOnly, b->d_w, b->d_du, b->d_u, b->d_u1, b->d_dt, one, 1, f1,
                         b->st)))
    return rc;
  CB_CUDA(cudaStreamSynchronize(b->st));
  return 0;
}

int canoe_block_solve_implicit(canoe_block_t b, double *d_du, double dt) {
  if (!b || !d_du || !(dt > 0.)) {
    set_error("null du or non-positive dt");
    return CANOE_ERR_ARG;
  }
  if (!(b->cfg.implicit_flag & 1) && !b->lines) return 0;
  // the solve reads dt through the device dt slot: use slot 1 as a scratch
  CB_CUDA(cudaMemcpyAsync(b->d_dt + 1, &dt, sizeof(double), cudaMemcpyHostToDevice, b->st));
  const Stage one{0., 1., 1.};
  if (b->lines)
    if (int rc = line_solves(b, d_du, b->d_dt + 1, one)) return rc;
  int rc = launch_x1col(b->g, b->th, b->cfg.recon, b->cfg.rsolver, b->cfg.implicit_flag,
                        b->cfg.precision, kColSolveOnly, b->d_w, d_du, b->d_u, b->d_u1, b->d_dt + 1, one, 1,
                        nullptr, b->st);
  if (rc) return rc;
  CB_CUDA(cudaStreamSynchronize(b->st));
  return 0;
}

int canoe_block_use_graph(canoe_block_t b, int on) {
  if (!b) return CANOE_ERR_ARG;
  b->graph = on != 0;
  return 0;
}

int canoe_block_set_diffusion(canoe_block_t b, double K, double p0) {
  if (!b || !(K >= 0.) || !(p0 > 0.)) {
    set_error("diffusivity must be >= 0 and p0 > 0");
    return CANOE_ERR_ARG;
  }
  if (K > 0. && (b->g.nx3 != 1 || b->g.nx2 < 2 || b->lines)) {
    set_error("the dissipation source is defined on 2-D blocks without x2 implicit solves");
    return CANOE_ERR_UNSUPPORTED;
  }
  b->diff_K = K;
  b->diff_p0 = p0;
  if (b->gexec) {  // the captured step changes
    cudaGraphExecDestroy(b->gexec);
    b->gexec = nullptr;
  }
  return 0;
}

int canoe_block_set_fixed_dt(canoe_block_t b, double dt) {
  if (!b) return CANOE_ERR_ARG;
  b->fixed_dt = dt > 0. ? dt : 0.;
  if (b->gexec) {
    cudaGraphExecDestroy(b->gexec);
    b->gexec = nullptr;
  }
  if (int rc = launch_dt_finalize(b->d_dt, b->d_dtacc, b->cfg.cfl, b->fixed_dt, b->st)) return rc;
  CB_CUDA(cudaStreamSynchronize(b->st));
  return 0;
}

// a block with block boundaries needs its ghosts exchanged between stages
static int needs_mesh(const canoe_block *b) {
  for (int q = 2; q < 6; ++q)
    if (b->cfg.bc[q] == CANOE_BC_BLOCK) {
      set_error("a block with block boundaries steps through canoe_mesh_step, or per stage "
                "with canoe_block_stage and canoe_block_exchange_ghosts");
      return CANOE_ERR_UNSUPPORTED;
    }
  return 0;
}

int canoe_block_step(canoe_block_t b, double dt) {
  if (!b) return CANOE_ERR_ARG;
  if (int rc = needs_mesh(b)) return rc;
  if (b->graph && !(dt > 0.)) {
    if (!b->gexec) {
      cudaGraph_t graph;
      CB_CUDA(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
      int rc = step_launches(b, 0.);
      cudaError_t e = cudaStreamEndCapture(b->st, &graph);
      if (rc) return rc;
      if (e != cudaSuccess) return cuda_status(e, "cudaStreamEndCapture");
      e = cudaGraphInstantiate(&b->gexec, graph, 0);
      cudaGraphDestroy(graph);
      if (e != cudaSuccess) return cuda_status(e, "cudaGraphInstantiate");
    }
    CB_CUDA(cudaGraphLaunch(b->gexec, b->st));
    return 0;
  }
  return step_launches(b, dt);
}

int canoe_block_step_profile(canoe_block_t b, double dt, float *ms, int nclass) {
  if (!b || !ms || nclass < 7) {
    set_error("canoe_block_step_profile needs ms[7]");
    return CANOE_ERR_ARG;
  }
  if (int rc = needs_mesh(b)) return rc;
  StepTimer tm;
  for (int q = 0; q < 64; ++q) CB_CUDA(cudaEventCreate(&tm.ev[q]));
  int rc = step_launches(b, dt, &tm);
  if (!rc) {
    CB_CUDA(cudaEventSynchronize(tm.ev[tm.n - 1]));
    for (int q = 1; q < tm.n; ++q) {
      float t = 0.f;
      CB_CUDA(cudaEventElapsedTime(&t, tm.ev[q - 1], tm.ev[q]));
      if (tm.cls[q] >= 0 && tm.cls[q] < nclass) ms[tm.cls[q]] += t;
    }
  }
  for (int q = 0; q < 64; ++q) cudaEventDestroy(tm.ev[q]);
  return rc;
}

int canoe_block_synchronize(canoe_block_t b) {
  if (!b) return CANOE_ERR_ARG;
  CB_CUDA(cudaStreamSynchronize(b->st));
  return 0;
}

int canoe_block_new_dt(canoe_block_t b, double *dt_out) {
  if (!b || !dt_out) return CANOE_ERR_ARG;
  CB_CUDA(cudaMemcpyAsync(dt_out, b->d_dt, sizeof(double), cudaMemcpyDeviceToHost, b->st));
  CB_CUDA(cudaStreamSynchronize(b->st));
  return 0;
}

int canoe_block_set_mlp(canoe_block_t b, canoe_mlp_t m) {
  if (!b) return CANOE_ERR_ARG;
  b->mlp = m;
  if (b->gexec) {
    cudaGraphExecDestroy(b->gexec);
    b->gexec = nullptr;
  }
  return 0;
}

int canoe_block_satadj_stats(canoe_block_t b, unsigned long long *h_stats) {
  if (!b || !h_stats) return CANOE_ERR_ARG;
  CB_CUDA(cudaMemcpyAsync(h_stats, b->d_sat, 4 * sizeof(unsigned long long),
                          cudaMemcpyDeviceToHost, b->st));
  CB_CUDA(cudaMemsetAsync(b->d_sat, 0, 4 * sizeof(unsigned long long), b->st));
  CB_CUDA(cudaStreamSynchronize(b->st));
  return 0;
}

int canoe_saturation_adjust_learned(const canoe_thermo_t *th, const canoe_satadj_opts_t *opts,
                                    canoe_mlp_t m, double *d_u, int64_t ncells,
                                    double *d_t_out, int32_t *d_iters,
                                    unsigned long long *d_stats, double *d_guess_out,
                                    void *stream) {
  if (!th || !opts || !m || !d_u || ncells < 0) {
    set_error("null pointer or negative size");
    return CANOE_ERR_ARG;
  }
  if (int rc = check_thermo(*th)) return rc;
  if (opts->warm != 1 && opts->warm != 2) {
    set_error("the learned saturation adjustment needs opts->warm 1 or 2");
    return CANOE_ERR_ARG;
  }
  MlpView mv = mlp_view(m);
  return launch_satadj(*th, *opts, d_u, ncells, ncells, nullptr, nullptr, d_t_out, d_iters,
                       d_stats, (cudaStream_t)stream, &mv, d_guess_out);
}

int canoe_block_error_word(canoe_block_t b, uint32_t *bits) {
  if (!b || !bits) return CANOE_ERR_ARG;
  CB_CUDA(cudaMemcpyAsync(bits, b->d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, b->st));
  CB_CUDA(cudaMemsetAsync(b->d_err, 0, sizeof(uint32_t), b->st));
  CB_CUDA(cudaStreamSynchronize(b->st));
  return 0;
}


int canoe_block_set_column_threads(canoe_block_t b, int threads) {
  if (!b) return CANOE_ERR_ARG;
  if (threads != 0 && (threads < 64 || threads > 256 || threads % 32)) {
    set_error("threads per x1 pencil must be a multiple of 32 in 64..256 (0: default)");
    return CANOE_ERR_ARG;
  }
  b->g.col_threads = threads;
  if (b->gexec) {
    cudaGraphExecDestroy(b->gexec);
    b->gexec = nullptr;
  }
  return 0;
}

int canoe_block_set_flux_run(canoe_block_t b, int cells) {
  if (!b) return CANOE_ERR_ARG;
  if (cells != 0 && (cells < 4 || cells > 256)) {
    set_error("cells per x2 / x3 flux run must be in 4..256 (0: default)");
    return CANOE_ERR_ARG;
  }
  b->g.flux_run = cells;
  if (b->gexec) {
    cudaGraphExecDestroy(b->gexec);
    b->gexec = nullptr;
  }
  return 0;
}

int canoe_block_get_shapes(canoe_block_t b, int32_t *col_threads, int32_t *flux_run) {
  if (!b) return CANOE_ERR_ARG;
  if (col_threads) *col_threads = b->g.col_threads;
  if (flux_run) *flux_run = b->g.flux_run;
  return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// meshes of blocks on one GPU: ghost slabs copied between neighbours between
// RK stages (Athena's SEND_HYD / RECV_HYD / SETB_HYD), the mesh-wide CFL dt

namespace {

// the ghost slab of b across side q (2 ix2, 3 ox2, 4 ix3, 5 ox3) and the
// slab of nb's interior it is filled from; interior k (x2 sides) or j (x3
// sides) only: the x2 flux pass reads j-ghosts at interior k and the x3 pass
// k-ghosts at interior j, so the corner ghosts are never read
Slab side_slab(const canoe_block *b, int q, const canoe_block *nb) {
  const Geom &g = b->g, &h = nb->g;
  Slab sl;
  sl.dsv = g.sv;
  sl.dsk = g.sk;
  sl.ssv = h.sv;
  sl.ssk = h.sk;
  if (q == 2 || q == 3) {
    sl.nk = g.nx3;
    sl.nj = NG;
    const int jd = q == 3 ? g.je + 1 : g.js - NG;  // first ghost row of b
    const int js = q == 3 ? h.js : h.je - NG + 1;  // first interior row of nb
    sl.dst = b->d_w + (int64_t)g.ks * g.sk + (int64_t)jd * g.nc1;
    sl.src = nb->d_w + (int64_t)h.ks * h.sk + (int64_t)js * h.nc1;
  } else {
    sl.nk = NG;
    sl.nj = g.nx2;
    const int kd = q == 5 ? g.ke + 1 : g.ks - NG;
    const int ks = q == 5 ? h.ks : h.ke - NG + 1;
    sl.dst = b->d_w + (int64_t)kd * g.sk + (int64_t)g.js * g.nc1;
    sl.src = nb->d_w + (int64_t)ks * h.sk + (int64_t)h.js * h.nc1;
  }
  return sl;
}

void rebuild_slabs(canoe_block *b) {
  b->slabs.n = 0;
  b->slabs.nv = b->g.nv;
  b->slabs.nc1 = b->g.nc1;
  for (int q = 2; q < 6; ++q)
    if (b->nb[q]) b->slabs.s[b->slabs.n++] = side_slab(b, q, b->nb[q]);
}

}  // namespace

struct canoe_mesh {
  std::vector<canoe_block *> blocks;
  cudaStream_t st = nullptr;
  double *d_dt = nullptr;  // the mesh's step dt (2 doubles)
  unsigned long long *d_acc = nullptr;  // mesh-wide CFL minimum
  double fixed_dt = 0.;
  bool graph = false;
  cudaGraphExec_t gexec = nullptr;
};

static int mesh_free(canoe_mesh *m) {
  if (!m) return 0;
  if (m->st) cudaStreamSynchronize(m->st);
  if (m->gexec) cudaGraphExecDestroy(m->gexec);
  if (m->d_dt) cudaFree(m->d_dt);
  if (m->d_acc) cudaFree(m->d_acc);
  if (m->st) cudaStreamDestroy(m->st);
  delete m;
  return 0;
}

// one step of every block: per stage, every block's stage, then every
// block's ghost exchange (main.cpp:119-121 over the task list of
// ImplicitHydroTasks); fixed_dt <= 0 uses the mesh's device dt
static int mesh_launches(canoe_mesh *m, double fixed_dt) {
  int rc;
  const canoe_block *b0 = m->blocks[0];
  if (fixed_dt > 0. &&
      (rc = launch_dt_finalize(m->d_dt, m->d_acc, b0->cfg.cfl, fixed_dt, m->st)))
    return rc;
  for (int s = 0; s < 3; ++s) {
    for (canoe_block *b : m->blocks)
      if ((rc = stage_launches(b, s, m->d_dt, m->d_acc, m->st))) return rc;
    for (canoe_block *b : m->blocks)
      if ((rc = launch_exchange(b->slabs, m->st))) return rc;
  }
  return launch_dt_finalize(m->d_dt, m->d_acc, b0->cfg.cfl, m->fixed_dt, m->st);
}

extern "C" {

int canoe_block_set_neighbor(canoe_block_t b, int side, canoe_block_t nb) {
  if (!b || !nb || side < 2 || side > 5) {
    set_error("canoe_block_set_neighbor: null block or side outside 2..5");
    return CANOE_ERR_ARG;
  }
  if (b->cfg.bc[side] != CANOE_BC_BLOCK) {
    set_error("canoe_block_set_neighbor: the side's boundary flag is not CANOE_BC_BLOCK");
    return CANOE_ERR_ARG;
  }
  const Geom &g = b->g, &h = nb->g;
  const bool x2 = side < 4;
  if ((x2 && !g.f2) || (!x2 && !g.f3)) {
    set_error("canoe_block_set_neighbor: the block has no cells along that direction");
    return CANOE_ERR_ARG;
  }
  if (g.nv != h.nv || g.nx1 != h.nx1 || g.nc1 != h.nc1 || b->cfg.precision != nb->cfg.precision ||
      std::memcmp(&b->th, &nb->th, sizeof(canoe_thermo_t)) != 0) {
    set_error("canoe_block_set_neighbor: neighbours share nx1, the thermodynamics and the "
              "precision");
    return CANOE_ERR_ARG;
  }
  std::vector<double> xa(g.nc1 + 1), xb(h.nc1 + 1);
  CB_CUDA(cudaMemcpy(xa.data(), b->d_x1f, xa.size() * sizeof(double), cudaMemcpyDeviceToHost));
  CB_CUDA(cudaMemcpy(xb.data(), nb->d_x1f, xb.size() * sizeof(double), cudaMemcpyDeviceToHost));
  if (xa != xb) {
    set_error("canoe_block_set_neighbor: neighbours share the x1 faces");
    return CANOE_ERR_ARG;
  }
  // the shared face: x2 neighbours have the same nx3 (and f3), x3 ones the
  // same nx2; the neighbour holds at least NGHOST cells across it
  if (x2 ? (g.nx3 != h.nx3 || g.f3 != h.f3 || h.nx2 < NG || !h.f2)
         : (g.nx2 != h.nx2 || h.nx3 < NG || !h.f3)) {
    set_error("canoe_block_set_neighbor: the shared face differs or the neighbour is "
              "thinner than NGHOST cells");
    return CANOE_ERR_ARG;
  }
  b->nb[side] = nb;
  rebuild_slabs(b);
  if (b->gexec) {
    cudaGraphExecDestroy(b->gexec);
    b->gexec = nullptr;
  }
  return 0;
}

int canoe_block_stage(canoe_block_t b, int stage, double dt) {
  if (!b || stage < 0 || stage > 2) {
    set_error("canoe_block_stage: null block or stage outside 0..2");
    return CANOE_ERR_ARG;
  }
  int rc;
  if (stage == 0 && dt > 0. &&
      (rc = launch_dt_finalize(b->d_dt, b->d_dtacc, b->cfg.cfl, dt, b->st)))
    return rc;
  if ((rc = stage_launches(b, stage, b->d_dt, b->d_dtacc, b->st))) return rc;
  if (stage == 2)
    return launch_dt_finalize(b->d_dt, b->d_dtacc, b->cfg.cfl, b->fixed_dt, b->st);
  return 0;
}

int canoe_block_exchange_ghosts(canoe_block_t b) {
  if (!b) return CANOE_ERR_ARG;
  for (int q = 2; q < 6; ++q)
    if (b->cfg.bc[q] == CANOE_BC_BLOCK && !b->nb[q]) {
      set_error("canoe_block_exchange_ghosts: a block side has no neighbour");
      return CANOE_ERR_ARG;
    }
  return launch_exchange(b->slabs, b->st);
}

static int side_ok(const canoe_block *b, int side) {
  if (!b || side < 2 || side > 5 || (side < 4 && !b->g.f2) || (side >= 4 && !b->g.f3)) {
    set_error("side must be 2..5 and the block must have cells along its direction");
    return CANOE_ERR_ARG;
  }
  return 0;
}

int canoe_block_side_doubles(canoe_block_t b, int side, int64_t *n) {
  if (int rc = side_ok(b, side)) return rc;
  if (!n) return CANOE_ERR_ARG;
  const Geom &g = b->g;
  *n = (int64_t)g.nv * (side < 4 ? g.nx3 : g.nx2) * NG * g.nc1;
  return 0;
}

// the layers of b next to `side` as a slab whose other end is a contiguous
// buffer (rows in the order variable, k, j)
static Slab buffer_slab(const canoe_block *b, int side, bool ghosts) {
  const Geom &g = b->g;
  Slab sl;
  const bool x2 = side < 4, lo = (side & 1) == 0;
  sl.nk = x2 ? g.nx3 : NG;
  sl.nj = x2 ? NG : g.nx2;
  int k0 = g.ks, j0 = g.js;
  if (x2)
    j0 = ghosts ? (lo ? g.js - NG : g.je + 1) : (lo ? g.js : g.je - NG + 1);
  else
    k0 = ghosts ? (lo ? g.ks - NG : g.ke + 1) : (lo ? g.ks : g.ke - NG + 1);
  double *p = b->d_w + (int64_t)k0 * g.sk + (int64_t)j0 * g.nc1;
  sl.dst = p;
  sl.src = p;
  sl.dsv = sl.ssv = g.sv;
  sl.dsk = sl.ssk = g.sk;
  return sl;
}

int canoe_block_pack_side(canoe_block_t b, int side, double *d_buf) {
  if (int rc = side_ok(b, side)) return rc;
  if (!d_buf) return CANOE_ERR_ARG;
  Slab sl = buffer_slab(b, side, false);
  sl.dst = d_buf;  // contiguous: k rows of nj x nc1, variables of nk rows
  sl.dsk = (int64_t)sl.nj * b->g.nc1;
  sl.dsv = (int64_t)sl.nk * sl.dsk;
  SlabSet ss{};
  ss.s[0] = sl;
  ss.n = 1;
  ss.nv = b->g.nv;
  ss.nc1 = b->g.nc1;
  return launch_exchange(ss, b->st);
}

int canoe_block_unpack_side(canoe_block_t b, int side, const double *d_buf) {
  if (int rc = side_ok(b, side)) return rc;
  if (!d_buf) return CANOE_ERR_ARG;
  Slab sl = buffer_slab(b, side, true);
  sl.src = d_buf;
  sl.ssk = (int64_t)sl.nj * b->g.nc1;
  sl.ssv = (int64_t)sl.nk * sl.ssk;
  SlabSet ss{};
  ss.s[0] = sl;
  ss.n = 1;
  ss.nv = b->g.nv;
  ss.nc1 = b->g.nc1;
  return launch_exchange(ss, b->st);
}

int canoe_mesh_create(canoe_block_t *blocks, int n, canoe_mesh_t *out) {
  if (!blocks || n < 1 || !out) {
    set_error("canoe_mesh_create: null pointer or no blocks");
    return CANOE_ERR_ARG;
  }
  *out = nullptr;
  for (int q = 0; q < n; ++q) {
    canoe_block *b = blocks[q];
    if (!b) return CANOE_ERR_ARG;
    for (int side = 2; side < 6; ++side) {
      if (b->cfg.bc[side] != CANOE_BC_BLOCK) continue;
      const canoe_block *nb = b->nb[side];
      if (!nb || std::find(blocks, blocks + n, nb) == blocks + n) {
        set_error("canoe_mesh_create: a block side names no neighbour of the mesh");
        return CANOE_ERR_ARG;
      }
    }
    if (b->cfg.cfl != blocks[0]->cfg.cfl || b->g.nc1 != blocks[0]->g.nc1) {
      set_error("canoe_mesh_create: the blocks share the CFL number and nx1");
      return CANOE_ERR_ARG;
    }
  }
  canoe_mesh *m = new canoe_mesh();
  m->blocks.assign(blocks, blocks + n);
  cudaError_t e;
  auto fail = [&](cudaError_t err, const char *what) {
    int rc = cuda_status(err, what);
    mesh_free(m);
    return rc;
  };
  if ((e = cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking))) return fail(e, "stream");
  if ((e = cudaMalloc(&m->d_dt, 2 * sizeof(double)))) return fail(e, "cudaMalloc dt");
  if ((e = cudaMalloc(&m->d_acc, sizeof(unsigned long long)))) return fail(e, "cudaMalloc acc");
  // the blocks' own work is done before the mesh takes over
  for (canoe_block *b : m->blocks)
    if ((e = cudaStreamSynchronize(b->st))) return fail(e, "block stream");
  // the mesh-wide CFL dt of the current states and the FP32 path's
  // reference pressure as the level mean over every block's columns
  const int nc1 = blocks[0]->g.nc1;
  std::vector<double> pref(nc1, 0.), pb(nc1);
  double dtmin = 0., ncols = 0.;
  for (canoe_block *b : m->blocks) {
    double dtb = 0.;
    if ((e = cudaMemcpy(&dtb, b->d_dt, sizeof(double), cudaMemcpyDeviceToHost)))
      return fail(e, "copy dt");
    dtmin = (dtmin == 0. || dtb < dtmin) ? dtb : dtmin;
    if ((e = cudaMemcpy(pb.data(), b->d_pref, nc1 * sizeof(double), cudaMemcpyDeviceToHost)))
      return fail(e, "copy pref");
    const double c = (double)b->g.nx2 * b->g.nx3;
    for (int i = 0; i < nc1; ++i) pref[i] += c * pb[i];
    ncols += c;
  }
  for (int i = 0; i < nc1; ++i) pref[i] /= ncols;
  for (canoe_block *b : m->blocks)
    if ((e = cudaMemcpy(b->d_pref, pref.data(), nc1 * sizeof(double), cudaMemcpyHostToDevice)))
      return fail(e, "copy pref");
  const double dt2[2] = {dtmin, 0.};
  const unsigned long long inf = 0x7ff0000000000000ULL;
  if ((e = cudaMemcpy(m->d_dt, dt2, sizeof(dt2), cudaMemcpyHostToDevice))) return fail(e, "copy");
  if ((e = cudaMemcpy(m->d_acc, &inf, sizeof(inf), cudaMemcpyHostToDevice))) return fail(e, "copy");
  // the ghosts of block sides, from the states as they are
  for (canoe_block *b : m->blocks)
    if (int rc = launch_exchange(b->slabs, m->st)) {
      mesh_free(m);
      return rc;
    }
  if ((e = cudaStreamSynchronize(m->st))) return fail(e, "exchange");
  *out = m;
  return 0;
}

int canoe_mesh_destroy(canoe_mesh_t m) { return mesh_free(m); }

int canoe_mesh_use_graph(canoe_mesh_t m, int on) {
  if (!m) return CANOE_ERR_ARG;
  m->graph = on != 0;
  return 0;
}

int canoe_mesh_step(canoe_mesh_t m, double dt) {
  if (!m) return CANOE_ERR_ARG;
  if (m->graph && !(dt > 0.)) {
    if (!m->gexec) {
      cudaGraph_t graph;
      CB_CUDA(cudaStreamBeginCapture(m->st, cudaStreamCaptureModeThreadLocal));
      int rc = mesh_launches(m, 0.);
      cudaError_t e = cudaStreamEndCapture(m->st, &graph);
      if (rc) return rc;
      if (e != cudaSuccess) return cuda_status(e, "cudaStreamEndCapture");
      e = cudaGraphInstantiate(&m->gexec, graph, 0);
      cudaGraphDestroy(graph);
      if (e != cudaSuccess) return cuda_status(e, "cudaGraphInstantiate");
    }
    CB_CUDA(cudaGraphLaunch(m->gexec, m->st));
    return 0;
  }
  return mesh_launches(m, dt);
}

int canoe_mesh_new_dt(canoe_mesh_t m, double *dt_out) {
  if (!m || !dt_out) return CANOE_ERR_ARG;
  CB_CUDA(cudaMemcpyAsync(dt_out, m->d_dt, sizeof(double), cudaMemcpyDeviceToHost, m->st));
  CB_CUDA(cudaStreamSynchronize(m->st));
  return 0;
}

int canoe_mesh_synchronize(canoe_mesh_t m) {
  if (!m) return CANOE_ERR_ARG;
  CB_CUDA(cudaStreamSynchronize(m->st));
  return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// batches of uneven blocks: one step of every block as one graph whose
// branches (one per block, on the block's stream) run concurrently

struct canoe_batch {
  std::vector<canoe_block *> blocks;
  cudaStream_t st = nullptr;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join;
  cudaGraphExec_t gexec = nullptr;
  bool graph = true;
};

static int batch_free(canoe_batch *q) {
  if (!q) return 0;
  if (q->gexec) cudaGraphExecDestroy(q->gexec);
  for (cudaEvent_t e : q->join) cudaEventDestroy(e);
  if (q->fork) cudaEventDestroy(q->fork);
  if (q->st) cudaStreamDestroy(q->st);
  delete q;
  return 0;
}

// fork from the batch stream to every block stream, step, join
static int batch_launches(canoe_batch *q) {
  CB_CUDA(cudaEventRecord(q->fork, q->st));
  for (size_t n = 0; n < q->blocks.size(); ++n) {
    canoe_block *b = q->blocks[n];
    CB_CUDA(cudaStreamWaitEvent(b->st, q->fork, 0));
    if (int rc = step_launches(b, 0.)) return rc;
    CB_CUDA(cudaEventRecord(q->join[n], b->st));
    CB_CUDA(cudaStreamWaitEvent(q->st, q->join[n], 0));
  }
  return 0;
}

extern "C" {

int canoe_batch_create(canoe_block_t *blocks, int n, canoe_batch_t *out) {
  if (!blocks || n <= 0 || !out) {
    set_error("canoe_batch_create: no blocks");
    return CANOE_ERR_ARG;
  }
  canoe_batch *q = new canoe_batch();
  for (int i = 0; i < n; ++i) {
    if (!blocks[i]) {
      batch_free(q);
      set_error("canoe_batch_create: null block");
      return CANOE_ERR_ARG;
    }
    q->blocks.push_back(blocks[i]);
  }
  cudaError_t e;
  if ((e = cudaStreamCreateWithFlags(&q->st, cudaStreamNonBlocking)) ||
      (e = cudaEventCreateWithFlags(&q->fork, cudaEventDisableTiming))) {
    batch_free(q);
    return cuda_status(e, "canoe_batch_create");
  }
  q->join.resize(n, nullptr);
  for (int i = 0; i < n; ++i)
    if ((e = cudaEventCreateWithFlags(&q->join[i], cudaEventDisableTiming))) {
      batch_free(q);
      return cuda_status(e, "canoe_batch_create");
    }
  *out = q;
  return 0;
}

int canoe_batch_destroy(canoe_batch_t q) {
  if (q && q->st) cudaStreamSynchronize(q->st);
  return batch_free(q);
}

int canoe_batch_use_graph(canoe_batch_t q, int on) {
  if (!q) return CANOE_ERR_ARG;
  q->graph = on != 0;
  if (q->gexec) {
    cudaGraphExecDestroy(q->gexec);
    q->gexec = nullptr;
  }
  return 0;
}

int canoe_batch_step(canoe_batch_t q) {
  if (!q) return CANOE_ERR_ARG;
  if (!q->graph) return batch_launches(q);
  if (!q->gexec) {
    cudaGraph_t graph;
    CB_CUDA(cudaStreamBeginCapture(q->st, cudaStreamCaptureModeThreadLocal));
    int rc = batch_launches(q);
    cudaError_t e = cudaStreamEndCapture(q->st, &graph);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_status(e, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(&q->gexec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return cuda_status(e, "cudaGraphInstantiate");
  }
  CB_CUDA(cudaGraphLaunch(q->gexec, q->st));
  return 0;
}

int canoe_batch_synchronize(canoe_batch_t q) {
  if (!q) return CANOE_ERR_ARG;
  CB_CUDA(cudaStreamSynchronize(q->st));
  return 0;
}

// Per block, time steps of the block alone with each candidate number of
// threads per x1 pencil (64 .. 256) and keep the fastest; then time steps of
// the whole batch with each candidate number of cells per x2 / x3 flux run
// (the default, 8 .. 64) and keep the fastest for every block.  The blocks'
// states, dt and counters are restored afterwards.  h_threads (may be NULL)
// receives the thread choices; canoe_block_get_shapes gives both.
int canoe_batch_autotune(canoe_batch_t q, int32_t *h_threads) {
  if (!q) return CANOE_ERR_ARG;
  static const int cand[] = {64, 96, 128, 160, 192, 256};
  static const int run_cand[] = {0, 8, 16, 32, 64};
  const size_t nb = q->blocks.size();
  cudaEvent_t e0, e1;
  CB_CUDA(cudaEventCreate(&e0));
  CB_CUDA(cudaEventCreate(&e1));
  // every block's state, kept until the batch-wide sweep is done
  std::vector<double *> su(nb, nullptr), sw(nb, nullptr);
  std::vector<double> dts(2 * nb, 0.);
  int rc = 0;
  for (size_t n = 0; n < nb && !rc; ++n) {
    canoe_block *b = q->blocks[n];
    const size_t bytes = b->nvals * sizeof(double);
    if (cudaMalloc(&su[n], bytes) || cudaMalloc(&sw[n], bytes)) {
      rc = cuda_status(cudaErrorMemoryAllocation, "canoe_batch_autotune");
      break;
    }
    cudaMemcpyAsync(su[n], b->d_u, bytes, cudaMemcpyDeviceToDevice, b->st);
    cudaMemcpyAsync(sw[n], b->d_w, bytes, cudaMemcpyDeviceToDevice, b->st);
    cudaMemcpyAsync(&dts[2 * n], b->d_dt, 2 * sizeof(double), cudaMemcpyDeviceToHost, b->st);
    cudaStreamSynchronize(b->st);
  }
  auto restore = [&](size_t n) {
    canoe_block *b = q->blocks[n];
    const size_t bytes = b->nvals * sizeof(double);
    cudaMemcpyAsync(b->d_u, su[n], bytes, cudaMemcpyDeviceToDevice, b->st);
    cudaMemcpyAsync(b->d_w, sw[n], bytes, cudaMemcpyDeviceToDevice, b->st);
    cudaMemcpyAsync(b->d_dt, &dts[2 * n], 2 * sizeof(double), cudaMemcpyHostToDevice, b->st);
    cudaStreamSynchronize(b->st);
  };
  // threads per x1 pencil, block by block: one warm-up step, then two timed
  // steps of the block alone, with the default flux runs
  for (size_t n = 0; n < nb && !rc; ++n) {
    canoe_block *b = q->blocks[n];
    float best = 1e30f, ms = 0.f;
    int pick = kColThreads;
    b->g.flux_run = 0;
    for (int c : cand) {
      b->g.col_threads = c;
      rc = step_launches(b, 0.);
      if (!rc) {
        cudaEventRecord(e0, b->st);
        for (int k = 0; k < 2 && !rc; ++k) rc = step_launches(b, 0.);
        cudaEventRecord(e1, b->st);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&ms, e0, e1);
      }
      restore(n);
      if (rc) break;
      if (ms < best) {
        best = ms;
        pick = c;
      }
    }
    b->g.col_threads = pick;
    if (h_threads) h_threads[n] = pick;
  }
  // cells per x2 / x3 flux run, for the batch as a whole: the blocks share
  // the GPU when the batch steps, so a block timed alone favours shorter
  // runs (more CTAs) than pay off in the batch
  if (!rc) {
    float best = 1e30f, ms = 0.f;
    int run_pick = 0;
    for (int c : run_cand) {
      for (canoe_block *b : q->blocks) b->g.flux_run = c;
      rc = batch_launches(q);
      if (!rc) {
        cudaEventRecord(e0, q->st);
        for (int k = 0; k < 2 && !rc; ++k) rc = batch_launches(q);
        cudaEventRecord(e1, q->st);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&ms, e0, e1);
      }
      cudaStreamSynchronize(q->st);
      for (size_t n = 0; n < nb; ++n) restore(n);
      if (rc) break;
      if (ms < best) {
        best = ms;
        run_pick = c;
      }
    }
    for (canoe_block *b : q->blocks) b->g.flux_run = run_pick;
  }
  for (size_t n = 0; n < nb; ++n) {
    canoe_block *b = q->blocks[n];
    if (b->gexec) {
      cudaGraphExecDestroy(b->gexec);
      b->gexec = nullptr;
    }
    cudaMemsetAsync(b->d_sat, 0, 4 * sizeof(unsigned long long), b->st);
    cudaMemsetAsync(b->d_err, 0, sizeof(uint32_t), b->st);
    cudaStreamSynchronize(b->st);
    if (su[n]) cudaFree(su[n]);
    if (sw[n]) cudaFree(sw[n]);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (q->gexec) {
    cudaGraphExecDestroy(q->gexec);
    q->gexec = nullptr;
  }
  if (!rc) CB_CUDA(cudaGetLastError());
  return rc;
}

}  // extern "C"
