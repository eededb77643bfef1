// noalloc.cu -- one time step of a MeshBlock that allocates nothing.
//
// canoe_block_create owns its arrays through cudaMalloc.  Some callers cannot
// allocate device memory once they are running: a host model that has
// reserved the GPU's memory for its own pool up front (a cudaMalloc then
// fails or, where it succeeds, synchronizes the device in the middle of the
// caller's time step), or one that must not let a library take memory it
// cannot account for.  canoe_block_step_noalloc works on the state the caller
// owns -- the conserved state u (in / out) and a buffer for the primitive
// state w (out) -- and keeps everything else the step needs (the divergence
// scratch du, the RK register u1, the x1 geometry, the reference pressure
// profile, dt and the error word) in one file-scope device array of fixed
// size.  It launches the kernels of canoe_block_step in the same order.
//
// What must start at zero: the error word (cleared on every call; the
// caller's word when it passes one, else a word in the scratch array).  du is
// written by the x2 flux kernel before it is read (and not read at all in a
// single column), u1 is written at RK stage 0, and the geometry, pressure
// profile and dt are written at the start of each call, so none of them
// needs clearing.
//
// The scratch array is shared by every call on a device: two calls that
// overlap in time (different streams, or different host threads without an
// ordering between them) race on it and corrupt each other's results.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "column.cuh"

namespace cb {
namespace {

// 16 MiB of scratch: 2 * NV * nc3 * nc2 * nc1 + 4 * nc1 + 8 doubles must fit
constexpr size_t kNoAllocDoubles = (size_t)2 << 20;
__device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

// device address of g_noalloc_scratch, looked up once per device
constexpr int kMaxDevices = 64;
double *g_scratch_addr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mu;

int scratch_address(double **out) {
  int dev = 0;
  CB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("canoe_block_step_noalloc: device ordinal out of range");
    return CANOE_ERR_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    g_scratch_addr[dev] = static_cast<double *>(p);
  }
  *out = g_scratch_addr[dev];
  return 0;
}

// x1 ghost faces mirrored about the boundary faces, cell centres and widths
// (the same arithmetic as canoe_block_create does on the host)
__global__ void k_x1_geometry(double *x1f, double *x1v, double *dx1f, int is, int ie, int nc1) {
  const int t = threadIdx.x;
  if (t < NG) {
    const int q = t + 1;
    x1f[is - q] = 2. * x1f[is] - x1f[is + q];
    x1f[ie + 1 + q] = 2. * x1f[ie + 1] - x1f[ie + 1 - q];
  }
  __syncthreads();
  for (int i = t; i < nc1; i += blockDim.x) {
    x1v[i] = 0.5 * (x1f[i] + x1f[i + 1]);
    dx1f[i] = x1f[i + 1] - x1f[i];
  }
}

}  // namespace
}  // namespace cb

using namespace cb;

extern "C" int canoe_block_step_noalloc(const canoe_block_config_t *cfg, double *d_u,
                                        double *d_w, uint32_t *d_err, double dt, void *stream) {
  if (!cfg || !d_u || !d_w || !cfg->h_x1f || !(dt > 0.)) {
    set_error("canoe_block_step_noalloc: null pointer or non-positive dt");
    return CANOE_ERR_ARG;
  }
  // the same checks as canoe_block_create: a configuration it refuses is
  // refused here too
  if (int rc = validate_block_config(*cfg)) return rc;
  for (int q = 2; q < 6; ++q)
    if (cfg->bc[q] == CANOE_BC_BLOCK) {
      set_error("canoe_block_step_noalloc: block boundaries need a mesh (canoe_mesh_step)");
      return CANOE_ERR_UNSUPPORTED;
    }
  const canoe_thermo_t &th = cfg->thermo;
  const cudaStream_t st = (cudaStream_t)stream;
  Geom g{};
  g.ny = th.ny;
  g.nv = 5 + th.ny;
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
  if (line_solve_on(g, cfg->implicit_flag, 1) || line_solve_on(g, cfg->implicit_flag, 2)) {
    set_error("canoe_block_step_noalloc: x2 / x3 implicit solves need line scratch; use "
              "canoe_block_step");
    return CANOE_ERR_UNSUPPORTED;
  }
  const size_t nvals = (size_t)g.nv * (size_t)g.sv;
  const size_t need = 2 * nvals + 4 * (size_t)g.nc1 + 8;
  if (need > kNoAllocDoubles) {
    set_error("canoe_block_step_noalloc: the block needs " + std::to_string(need) +
              " doubles of scratch, more than the fixed " + std::to_string(kNoAllocDoubles));
    return CANOE_ERR_ARG;
  }
  double *scr = nullptr;
  if (int rc = scratch_address(&scr)) return rc;
  // scratch layout: du | u1 | x1f (nc1+1) | x1v | dx1f | pref | dt[2] | acc | err
  double *du = scr;
  double *u1 = du + nvals;
  double *x1f = u1 + nvals;
  double *x1v = x1f + g.nc1 + 1;
  double *dx1f = x1v + g.nc1;
  double *pref = dx1f + g.nc1;
  double *dtp = pref + g.nc1;
  unsigned long long *acc = reinterpret_cast<unsigned long long *>(dtp + 2);
  uint32_t *err = d_err ? d_err : reinterpret_cast<uint32_t *>(dtp + 3);

  CB_CUDA(cudaMemcpyAsync(x1f + g.is, cfg->h_x1f, (g.nx1 + 1) * sizeof(double),
                          cudaMemcpyHostToDevice, st));
  k_x1_geometry<<<1, 128, 0, st>>>(x1f, x1v, dx1f, g.is, g.ie, g.nc1);
  CB_CUDA(cudaGetLastError());
  CB_CUDA(cudaMemsetAsync(err, 0, sizeof(uint32_t), st));
  g.x1f = x1f;
  g.x1v = x1v;
  g.dx1f = dx1f;
  g.pref = pref;
  g.err = err;
  int rc;
  // w (with ghosts) and the reference pressure profile of the state on entry
  if ((rc = launch_cons_to_prim(g, th, d_u, d_w, err, nullptr, cfg->cfl, cfg->implicit_flag,
                                st)))
    return rc;
  if ((rc = launch_level_mean_pressure(g, th.ny, d_w, pref, st))) return rc;
  if ((rc = launch_dt_finalize(dtp, acc, cfg->cfl, dt, st))) return rc;
  for (int s = 0; s < 3; ++s) {
    const Stage &sg = kRK3[s];
    if (g.f2 && (rc = launch_flux_x23(1, g, th, cfg->recon, cfg->rsolver, cfg->precision, d_w,
                                      du, dtp, sg.beta, nullptr, st)))
      return rc;
    if (g.f3 && (rc = launch_flux_x23(2, g, th, cfg->recon, cfg->rsolver, cfg->precision, d_w,
                                      du, dtp, sg.beta, nullptr, st)))
      return rc;
    if ((rc = launch_x1col(g, th, cfg->recon, cfg->rsolver, cfg->implicit_flag, cfg->precision,
                           kColStep, d_w, du, d_u, u1, dtp, sg, s, nullptr, st)))
      return rc;
    if (s == 2 && cfg->satadj && th.ny > 0) {
      const canoe_satadj_opts_t o{1e-8, 30, 0};
      const int64_t nin = (int64_t)g.nx1 * g.nx2 * g.nx3;
      if ((rc = launch_satadj(th, o, d_u, nin, g.sv, &g, nullptr, nullptr, nullptr, nullptr, st)))
        return rc;
    }
    if ((rc = launch_cons_to_prim(g, th, d_u, d_w, err, nullptr, cfg->cfl, cfg->implicit_flag,
                                  st)))
      return rc;
  }
  return 0;
}
