// flux.cu -- the x2 / x3 part of Hydro::CalculateFluxes (Athena
// calculate_fluxes.cpp with canoe patches/19.calculate_fluxes.patch), fused
// with the flux divergence of the RK stage.
//
//  k_flux_x23_run: x2 / x3 fluxes, one thread per run of RL cells along
//              the flux direction with its stencil in registers (the step's
//              kernel).  The x2 pass writes du = -beta dt div F2 and the x3
//              pass subtracts beta dt div F3; the x1 pencil kernel
//              (column.cuh) adds the x1 part and finishes the stage.
//  k_flux_x23: the same on (32 i) x (8 cells) tiles staged in shared
//              memory (kFluxRun = 0).
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

// k_flux_x23_run: the same fluxes with one thread per (i, o, run of RL
// cells along the flux direction).  The thread marches along its run with a
// window of w in registers: each step reconstructs one cell, solves the
// Riemann problem at that cell's lower face and finishes the divergence of
// the cell below.  No shared memory and no barriers; the next cell's loads
// are issued one step ahead.  Every slope, interface value, flux and
// difference is the tile kernel's expression on the same operands, so both
// give the same bits.
// default cells per run (Geom::flux_run overrides it): 16 in FP32, 32 in
// FP64 (measured on C2 128x256x256: x2
// 0.343 / 0.355 / 0.365 ms per FP32 launch at 16 / 32 / 8 cells, FP64 0.732
// / 0.714 / 0.790 ms)
template <typename R>
constexpr int run_len() { return sizeof(R) == 4 ? 16 : 32; }
constexpr int RBY = 4;  // orthogonal lines per CTA (blockDim.y)

template <int NY, int RECON, int RS, int DIR, bool WF, typename R>
__global__ void __launch_bounds__(32 * RBY)
    k_flux_x23_run(Geom g, canoe_thermo_t th, const double *__restrict__ w,
                   double *__restrict__ du, const double *__restrict__ dtp, double beta,
                   double *__restrict__ fout) {
  using S = Slots<NY>;
  constexpr int NV = S::NV;
  constexpr int H = RECON == CANOE_RECON_PPM ? 2 : 1;
  constexpr bool PERT = sizeof(R) == 4;
  const int i = g.is + blockIdx.x * 32 + threadIdx.x;
  const int o = (DIR == 1 ? g.ks : g.js) + blockIdx.y * RBY + threadIdx.y;
  if (i > g.ie || o > (DIR == 1 ? g.ke : g.je)) return;
  const int dlo = DIR == 1 ? g.js : g.ks;
  const int dhi = DIR == 1 ? g.je : g.ke;
  const int RL = g.flux_run > 0 ? g.flux_run : run_len<R>();
  const int s0 = dlo + blockIdx.z * RL;
  const int s1 = min(s0 + RL, dhi + 1);  // one past the run's last cell
  const int64_t sd = DIR == 1 ? g.nc1 : g.sk;
  const int64_t base = (DIR == 1 ? (int64_t)o * g.sk : (int64_t)o * g.nc1) + i;
  const double pref = PERT ? g.pref[i] : 0.;
  const double wght = beta * dtp[0];
  const double idx = 1. / (DIR == 1 ? g.dx2 : g.dx3);

  // PLM: q[m] is cell c - 1 + m.  PPM streams what the parabola of cell c
  // needs: q[0], q[1] = cells c, c+1 (q[2] receives c+2), sl = the limited
  // slope of cell c and fl = the interface value below cell c, so each
  // slope and each interface value is computed once per cell, not three and
  // two times.
  R q[3][NV];
  R sl[NV], fl[NV];
  double nx[NV];
  auto fetch = [&](int c) {
    const int64_t off = base + (int64_t)c * sd;
#pragma unroll
    for (int n = 0; n < NV; ++n) nx[n] = w[n * g.sv + off];
  };
  auto put = [&](R *qm) {
#pragma unroll
    for (int n = 0; n < NV; ++n) {
      double v = nx[n];
      if (PERT && n == S::IPR) v -= pref;
      qm[n] = R(v);
    }
  };
  // the first reconstructed cell is s0 - 1
  if constexpr (RECON == CANOE_RECON_PPM) {
    R qa[NV], qb[NV];
    fetch(s0 - 3);
    put(qa);
    fetch(s0 - 2);
    put(qb);
    fetch(s0 - 1);
    put(q[0]);
    fetch(s0);
    put(q[1]);
#pragma unroll
    for (int n = 0; n < NV; ++n) {
      const R sb = ppm_slope(qa[n], qb[n], q[0][n]);
      sl[n] = ppm_slope(qb[n], q[0][n], q[1][n]);
      fl[n] = ppm_face(qb[n], q[0][n], sb, sl[n]);
    }
  } else {
    fetch(s0 - 2);
    put(q[0]);
    fetch(s0 - 1);
    put(q[1]);
  }
  fetch(s0 - 1 + H);
  R wrp[NV], fp[NV];
  double dpre[NV];
  for (int c = s0 - 1; c <= s1; ++c) {
    put(q[2]);
    if (c < s1) fetch(c + H + 1);  // one step ahead
    if (DIR == 2 && c > s0) {
      const int64_t off = base + (int64_t)(c - 1) * sd;
#pragma unroll
      for (int n = 0; n < NV; ++n) dpre[n] = du[n * g.sv + off];
    }
    R wl[NV], wr[NV];
#pragma unroll
    for (int n = 0; n < NV; ++n) {
      if constexpr (RECON == CANOE_RECON_PPM) {
        const R sr = ppm_slope(q[0][n], q[1][n], q[2][n]);
        const R fr = ppm_face(q[0][n], q[1][n], sl[n], sr);
        wl[n] = fl[n];
        wr[n] = fr;
        ppm_limit(q[0][n], wl[n], wr[n]);
        sl[n] = sr;
        fl[n] = fr;
      } else {
        plm_cell(q[0][n], q[1][n], q[2][n], wl[n], wr[n]);
      }
    }
    if (c >= s0) {
      // face c: left state = wR of cell c-1, right state = wL of cell c
      R fx[NV];
      if constexpr (PERT)
        riemann_pert<R, NY, RS, DIR>(th, wrp, wl, R(pref), fx);
      else
        riemann<R, NY, RS, DIR>(th, wrp, wl, fx);
      if constexpr (WF) {
#pragma unroll
        for (int n = 0; n < NV; ++n) {
          int64_t fi = DIR == 1
              ? (((int64_t)n * g.nc3 + o) * (g.nc2 + 1) + c) * g.nc1 + i
              : (((int64_t)n * (g.nc3 + 1) + c) * g.nc2 + o) * g.nc1 + i;
          double v = fx[n];
          if (PERT && n == S::IVX + DIR) v += pref;  // report the full flux
          fout[fi] = v;
        }
      }
      if (c > s0) {
        // du of cell c-1 from its faces c-1 and c
        const int64_t off = base + (int64_t)(c - 1) * sd;
#pragma unroll
        for (int n = 0; n < NV; ++n) {
          const double d = ((double)fx[n] - (double)fp[n]) * idx;
          if (DIR == 1)
            du[n * g.sv + off] = -(wght * d);
          else
            du[n * g.sv + off] = dpre[n] - wght * d;
        }
      }
#pragma unroll
      for (int n = 0; n < NV; ++n) fp[n] = fx[n];
    }
#pragma unroll
    for (int n = 0; n < NV; ++n) wrp[n] = wr[n];
#pragma unroll
    for (int n = 0; n < NV; ++n) {
      q[0][n] = q[1][n];
      q[1][n] = q[2][n];
    }
  }
}

// 1: the x2 / x3 fluxes run as k_flux_x23_run, 0: as the tile kernel
constexpr int kFluxRun = 1;

template <int NY, typename R>
size_t x23_smem() {
  constexpr int NV = 5 + NY;
  return sizeof(R) * (size_t)NV * TI * ((TD + 2 * NG) + 2 * (TD + 2));
}

template <int NY, int RECON, int RS, int DIR, bool WF, typename R>
int run_x23(const Geom &g, const canoe_thermo_t &th, const double *w, double *du,
            const double *dtp, double beta, double *fo, cudaStream_t st) {
  const int nd = DIR == 1 ? g.nx2 : g.nx3;
  const int no = DIR == 1 ? g.nx3 : g.nx2;
  const int RL = g.flux_run > 0 ? g.flux_run : run_len<R>();
  // a 2-D block (one line across the flux direction) keeps the tile kernel:
  // its runs would fill one warp in four of each CTA, and the 150 x 100
  // bubble would march 20 warps in all (x2 pass 4 x slower than the tiles);
  // thin 3-D blocks keep the runs, whose launches overlap in a batch
  if (kFluxRun != 0 && no >= RBY) {
    dim3 grid((g.nx1 + 31) / 32, (no + RBY - 1) / RBY, (nd + RL - 1) / RL);
    k_flux_x23_run<NY, RECON, RS, DIR, WF, R><<<grid, dim3(32, RBY), 0, st>>>(g, th, w, du, dtp,
                                                                              beta, fo);
    CB_CUDA(cudaGetLastError());
    return 0;
  }
  auto kern = k_flux_x23<NY, RECON, RS, DIR, WF, R>;
  size_t sm = x23_smem<NY, R>();
  if (int rc = ensure_smem((const void *)kern, sm)) return rc;
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
