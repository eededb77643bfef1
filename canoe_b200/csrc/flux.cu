// flux.cu -- the x2 / x3 part of Hydro::CalculateFluxes (Athena
// calculate_fluxes.cpp with canoe patches/19.calculate_fluxes.patch), fused
// with the flux divergence of the RK stage.
//
//  k_flux_x23: x2 / x3 fluxes on (32 i) x (8 cells) tiles staged in shared
//              memory.  The x2 pass writes du = -beta dt div F2 and the x3
//              pass subtracts beta dt div F3; the x1 pencil kernel
//              (column.cuh) adds the x1 part and finishes the stage.
//
// Every kernel reads dt from device memory (*dtp) so a whole step can be
// replayed from a CUDA graph.
#include <cuda_runtime.h>

#include <cstdio>

#include "block.cuh"

namespace cb {

namespace {

constexpr int TI = 32;  // tile width along i
constexpr int TD = 8;   // tile length along the flux direction

// R = double: the FP64 path.  R = float: reconstruction and Riemann fluxes
// in FP32 on p' = p - pref(i); pref is the same on both sides of an x2 / x3
// face, so it cancels from the momentum-flux divergence exactly.
// FP32 tiles: four CTAs per SM (64 registers); FP64: three
template <int NY, int RECON, int RS, int DIR, bool WF, typename R>
__global__ void __launch_bounds__(256, sizeof(R) == 4 ? 4 : 3)
    k_flux_x23(Geom g, canoe_thermo_t th, const double *__restrict__ w,
               double *__restrict__ du, const double *__restrict__ dtp,
               double beta, double *__restrict__ fout) {
  using S = Slots<NY>;
  constexpr int NV = S::NV;
  constexpr int QR = TD + 2 * NG;  // staged rows
  constexpr int RR = TD + 2;       // reconstructed cells
  constexpr bool PERT = sizeof(R) == 4;
  extern __shared__ double sm_[];
  R *sm = reinterpret_cast<R *>(sm_);
  R *q = sm;                       // [NV][QR][TI]
  R *WL = q + NV * QR * TI;        // [NV][RR][TI]
  R *WR = WL + NV * RR * TI;       // [NV][RR][TI]
  R *F = q;                        // [NV][TD+1][TI]

  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i = g.is + blockIdx.x * TI + tx;
  const bool iok = i <= g.ie;
  const int dlo = DIR == 1 ? g.js : g.ks;
  const int dhi = DIR == 1 ? g.je : g.ke;
  const int d0 = dlo + blockIdx.y * TD;
  const int nd = min(TD, dhi - d0 + 1);
  const int o = (DIR == 1 ? g.ks : g.js) + blockIdx.z;
  const int64_t sd = DIR == 1 ? g.nc1 : g.sk;
  const int64_t base = (DIR == 1 ? (int64_t)o * g.sk : (int64_t)o * g.nc1) + i;

  const double pref = PERT ? g.pref[iok ? i : g.is] : 0.;
  // x3 adds to the du of the x2 pass: this thread's du values are loaded at
  // entry so that their latency hides behind the reconstruction
  double dpre[NV];
  if (DIR == 2 && iok && ty < nd && blockDim.y >= TD) {
    const int64_t off = base + (int64_t)(d0 + ty) * sd;
#pragma unroll
    for (int n = 0; n < NV; ++n) dpre[n] = du[n * g.sv + off];
  }
  // P0: stage cells d0-3 .. d0+nd+2
  for (int c = ty; c < nd + 2 * NG; c += blockDim.y) {
    const int64_t off = base + (int64_t)(d0 - NG + c) * sd;
#pragma unroll
    for (int n = 0; n < NV; ++n) {
      double v = iok ? w[n * g.sv + off] : 1.;
      if (PERT && n == S::IPR) v = iok ? v - pref : 0.;
      q[(n * QR + c) * TI + tx] = R(v);
    }
  }
  __syncthreads();
  // P1: reconstruct cells d0-1 .. d0+nd (local c = 0 .. nd+1)
  for (int c = ty; c < nd + 2; c += blockDim.y) {
#pragma unroll
    for (int n = 0; n < NV; ++n) {
      const R *qc = q + (n * QR + c) * TI + tx;
      R wl_, wr_;
      if constexpr (RECON == CANOE_RECON_PPM)
        ppm_cell(qc[0], qc[TI], qc[2 * TI], qc[3 * TI], qc[4 * TI], wl_, wr_);
      else
        plm_cell(qc[TI], qc[2 * TI], qc[3 * TI], wl_, wr_);
      WL[(n * RR + c) * TI + tx] = wl_;
      WR[(n * RR + c) * TI + tx] = wr_;
    }
  }
  __syncthreads();
  // P2: faces d0 .. d0+nd (local f = 0 .. nd): left cell c = f, right c = f+1
  for (int f = ty; f <= nd; f += blockDim.y) {
    R wl[NV], wr[NV], fx[NV];
#pragma unroll
    for (int n = 0; n < NV; ++n) {
      wl[n] = WR[(n * RR + f) * TI + tx];
      wr[n] = WL[(n * RR + f + 1) * TI + tx];
    }
    if constexpr (PERT)
      riemann_pert<R, NY, RS, DIR>(th, wl, wr, R(pref), fx);
    else
      riemann<R, NY, RS, DIR>(th, wl, wr, fx);
#pragma unroll
    for (int n = 0; n < NV; ++n) F[(n * (TD + 1) + f) * TI + tx] = fx[n];
    if constexpr (WF) {
      if (iok) {
        const int fd = d0 + f;
#pragma unroll
        for (int n = 0; n < NV; ++n) {
          int64_t idx = DIR == 1
              ? (((int64_t)n * g.nc3 + o) * (g.nc2 + 1) + fd) * g.nc1 + i
              : (((int64_t)n * (g.nc3 + 1) + fd) * g.nc2 + o) * g.nc1 + i;
          double v = fx[n];
          if (PERT && n == S::IVX + DIR) v += pref;  // report the full flux
          fout[idx] = v;
        }
      }
    }
  }
  __syncthreads();
  // P3: du -= beta dt (F(c+1) - F(c)) / dx
  if (!iok) return;
  const double wght = beta * dtp[0];
  const double idx = 1. / (DIR == 1 ? g.dx2 : g.dx3);
  for (int c = ty; c < nd; c += blockDim.y) {
    const int64_t off = base + (int64_t)(d0 + c) * sd;
#pragma unroll
    for (int n = 0; n < NV; ++n) {
      double d = ((double)F[(n * (TD + 1) + c + 1) * TI + tx] -
                  (double)F[(n * (TD + 1) + c) * TI + tx]) * idx;
      if (DIR == 1)
        du[n * g.sv + off] = -(wght * d);  // x2 runs first: initialise du
      else if (blockDim.y >= TD)
        du[n * g.sv + off] = dpre[n] - wght * d;  // c == ty: the prefetched cell
      else
        du[n * g.sv + off] -= wght * d;
    }
  }
}

template <int NY, typename R>
size_t x23_smem() {
  constexpr int NV = 5 + NY;
  return sizeof(R) * (size_t)NV * TI * ((TD + 2 * NG) + 2 * (TD + 2));
}

template <int NY, int RECON, int RS, int DIR, bool WF, typename R>
int run_x23(const Geom &g, const canoe_thermo_t &th, const double *w, double *du,
            const double *dtp, double beta, double *fo, cudaStream_t st) {
  auto kern = k_flux_x23<NY, RECON, RS, DIR, WF, R>;
  size_t sm = x23_smem<NY, R>();
  if (int rc = ensure_smem((const void *)kern, sm)) return rc;
  const int nd = DIR == 1 ? g.nx2 : g.nx3;
  const int no = DIR == 1 ? g.nx3 : g.nx2;
  dim3 grid((g.nx1 + TI - 1) / TI, (nd + TD - 1) / TD, no);
  kern<<<grid, dim3(TI, 8), sm, st>>>(g, th, w, du, dtp, beta, fo);
  CB_CUDA(cudaGetLastError());
  return 0;
}

}  // namespace

#define CB_DISPATCH_NY(ny, CALL)                      \
  switch (ny) {                                       \
    case 0: { constexpr int NY = 0; return CALL; }    \
    case 1: { constexpr int NY = 1; return CALL; }    \
    case 2: { constexpr int NY = 2; return CALL; }    \
    case 3: { constexpr int NY = 3; return CALL; }    \
    case 6: { constexpr int NY = 6; return CALL; }    \
    default:                                          \
      set_error("unsupported number of mass-fraction slots"); \
      return CANOE_ERR_UNSUPPORTED;                   \
  }

template <int NY, int DIR, typename RT>
static int x23_dispatch(const Geom &g, const canoe_thermo_t &th, int recon, int rs,
                        const double *w, double *du, const double *dtp, double beta,
                        double *fo, cudaStream_t st) {
  const bool wf = fo != nullptr;
#define CB_X23(R, S, W) return run_x23<NY, R, S, DIR, W, RT>(g, th, w, du, dtp, beta, fo, st)
  if (recon == CANOE_RECON_PPM) {
    if (rs == CANOE_RSOLVER_LMARS) { if (wf) CB_X23(3, 0, true); else CB_X23(3, 0, false); }
    else { if (wf) CB_X23(3, 1, true); else CB_X23(3, 1, false); }
  } else {
    if (rs == CANOE_RSOLVER_LMARS) { if (wf) CB_X23(2, 0, true); else CB_X23(2, 0, false); }
    else { if (wf) CB_X23(2, 1, true); else CB_X23(2, 1, false); }
  }
#undef CB_X23
}

int launch_flux_x23(int dir, const Geom &g, const canoe_thermo_t &th, int recon,
                    int rs, int precision, const double *w, double *du,
                    const double *dtp, double beta, double *fo, cudaStream_t st) {
  const bool f32 = precision == CANOE_FP32_PERTURBATION;
  if (dir == 1) {
    if (f32)
      CB_DISPATCH_NY(th.ny, (x23_dispatch<NY, 1, float>(g, th, recon, rs, w, du, dtp, beta, fo, st)));
    CB_DISPATCH_NY(th.ny, (x23_dispatch<NY, 1, double>(g, th, recon, rs, w, du, dtp, beta, fo, st)));
  } else {
    if (f32)
      CB_DISPATCH_NY(th.ny, (x23_dispatch<NY, 2, float>(g, th, recon, rs, w, du, dtp, beta, fo, st)));
    CB_DISPATCH_NY(th.ny, (x23_dispatch<NY, 2, double>(g, th, recon, rs, w, du, dtp, beta, fo, st)));
  }
}

}  // namespace cb
