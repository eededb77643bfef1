// flux.cu -- Hydro::CalculateFluxes on the device, fused with the flux
// divergence of the RK stage.
//
//  k_flux_x1:  one CTA per x1 pencil (k, j).  The pencil (NV x nc1) is staged
//              in shared memory, Decomposition::ChangeToTemperature runs on
//              it (hydrostatic face pressure psf by a warp suffix-scan, log-mean
//              psv, RovRd, rho -> T, p -> p'), every variable is reconstructed,
//              RestoreFromTemperature is applied at the faces, the Riemann
//              solver produces the x1 fluxes, and the x1 divergence plus the
//              constant-gravity source are written to du.
//              (canoe patches/19.calculate_fluxes.patch:24-45,
//               src/snap/decomposition/change_to_temperature.cpp:40-167)
//  k_flux_x23: x2 / x3 fluxes on (32 i) x (8 cells) tiles staged in shared
//              memory; adds the x2 / x3 divergence to du.
//
// Every kernel reads dt from device memory (*dtp) so a whole step can be
// replayed from a CUDA graph.
#include <cuda_runtime.h>

#include <cstdio>

#include "block.cuh"

namespace cb {

namespace {

template <int NY, int RECON, int RS, bool WF>
__global__ void __launch_bounds__(128)
    k_flux_x1(Geom g, canoe_thermo_t th, const double *__restrict__ w,
              double *__restrict__ du, const double *__restrict__ dtp,
              double beta, double *__restrict__ fout) {
  using S = Slots<NY>;
  constexpr int NV = S::NV;
  extern __shared__ double sm[];
  const int nc1 = g.nc1, is = g.is, ie = g.ie, nx1 = g.nx1;
  double *q = sm;                    // [NV][nc1]   (later F [NV][nx1+1])
  double *WL = q + NV * nc1;         // [NV][nc1]
  double *WR = WL + NV * nc1;        // [NV][nc1]
  double *psf = WR + NV * nc1;       // [nc1+1]
  double *psv = psf + nc1 + 1;       // [nc1]
  double *gam = psv + nc1;           // [nc1]
  double *rho0 = gam + nc1;          // [nc1]
  double *F = q;

  const int j = g.js + (int)(blockIdx.x % (unsigned)g.nx2);
  const int k = g.ks + (int)(blockIdx.x / (unsigned)g.nx2);
  const int64_t base = (int64_t)k * g.sk + (int64_t)j * nc1;
  const int tid = threadIdx.x, nth = blockDim.x;
  const double grav = th.grav;

  // P0: stage the pencil
  for (int n = 0; n < NV; ++n)
    for (int i = tid; i < nc1; i += nth) {
      double v = w[n * g.sv + base + i];
      q[n * nc1 + i] = v;
      if (n == 0) rho0[i] = v;
    }
  __syncthreads();

  // P1: hydrostatic decomposition (change_to_temperature.cpp:45-128)
  if (grav != 0.) {
    double *rho = q, *pre = q + S::IPR * nc1;
    if (tid < 32) {
      const int lane = tid;
      double ptop = 0.;
      if (lane == 0) {
        double RdTv = pre[ie] / rho[ie];
        ptop = pre[ie] * exp(grav * g.dx1f[ie] / (2 * RdTv));
      }
      ptop = __shfl_sync(0xffffffffu, ptop, 0);
      const double gb = g.bc[0] == CANOE_BC_REFLECT ? -grav : grav;
      // suffix sum over m = ie .. is-NG (reverse index r = ie - m)
      const int L = nx1 + NG;
      const int cnt = (L + 31) / 32;
      const int r0 = lane * cnt, r1 = min(r0 + cnt, L);
      double loc = 0.;
      for (int r = r0; r < r1; ++r) {
        int m = ie - r;
        double gm = m >= is ? grav : gb;
        loc += -gm * rho[m] * g.dx1f[m];
      }
      double inc = loc;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        double t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
      }
      double acc = ptop + (inc - loc);
      for (int r = r0; r < r1; ++r) {
        int m = ie - r;
        double gm = m >= is ? grav : gb;
        acc = acc - gm * rho[m] * g.dx1f[m];
        psf[m] = acc;
      }
      if (lane == 0) {
        psf[ie + 1] = ptop;
        const double gt = g.bc[1] == CANOE_BC_REFLECT ? -grav : grav;
        double p = ptop;
        for (int i = ie + 1; i <= ie + NG; ++i) {
          p = p + gt * rho[i] * g.dx1f[i];
          psf[i + 1] = p;
        }
      }
    }
    __syncthreads();
    for (int i = tid; i < nc1; i += nth) {
      double a = psf[i], b = psf[i + 1];
      double pv = fabs(a - b) < 1.E-6 ? 0.5 * (a + b) : (a - b) / log(a / b);
      double feps = 1.;
#pragma unroll
      for (int n = 1; n <= NY; ++n)
        if (n <= th.nvapor) feps += q[n * nc1 + i] * th.inv_mu_ratio_m1[n - 1];
      double gm = th.rd * feps;
      psv[i] = pv;
      gam[i] = gm;
      rho[i] = pre[i] / (rho[i] * gm);
      pre[i] -= pv;
    }
    __syncthreads();
    if (tid == 0) {
      if (g.bc[0] == CANOE_BC_OUTFLOW)
        for (int i = is - NG; i < is; ++i) {
          rho[i] = rho[is];
          pre[i] = pre[is];
        }
      if (g.bc[1] == CANOE_BC_OUTFLOW)
        for (int i = ie + 1; i <= ie + NG; ++i) {
          rho[i] = rho[ie];
          pre[i] = pre[ie];
        }
    }
    __syncthreads();
  }

  // P2: reconstruct cells is-1 .. ie+1, every variable
  const int ncell = nx1 + 2;
  for (int t = tid; t < NV * ncell; t += nth) {
    const int n = t / ncell, c = is - 1 + t % ncell;
    const double *qn = q + n * nc1;
    double wl_, wr_;
    if constexpr (RECON == CANOE_RECON_PPM)
      ppm_cell(qn[c - 2], qn[c - 1], qn[c], qn[c + 1], qn[c + 2], wl_, wr_);
    else
      plm_cell_nu(qn[c - 1], qn[c], qn[c + 1], g.x1v[c - 1], g.x1v[c],
                  g.x1v[c + 1], g.x1f[c], g.x1f[c + 1], wl_, wr_);
    WL[n * nc1 + c] = wl_;
    WR[n * nc1 + c] = wr_;
  }
  __syncthreads();

  // P3: faces is .. ie+1: restore + Riemann (F aliases q)
  for (int f = is + tid; f <= ie + 1; f += nth) {
    double wl[NV], wr[NV], fx[NV];
#pragma unroll
    for (int n = 0; n < NV; ++n) {
      wl[n] = WR[n * nc1 + f - 1];
      wr[n] = WL[n * nc1 + f];
    }
    if (grav != 0.) {  // change_to_temperature.cpp:155-164
      double pf = psf[f];
      double gamma = sqrt(gam[f] * gam[f - 1]);
      double pr = wr[S::IPR] + pf;
      if (pr < 0.) pr = pf;
      wr[S::IPR] = pr;
      wr[0] = pr / (wr[0] * gamma);
      double pl = wl[S::IPR] + pf;
      if (pl < 0.) pl = pf;
      wl[S::IPR] = pl;
      wl[0] = pl / (wl[0] * gamma);
    }
    riemann<double, NY, RS, 0>(th, wl, wr, fx);
    // F may alias q: every thread finished reading q in P2
#pragma unroll
    for (int n = 0; n < NV; ++n) F[n * (nx1 + 1) + (f - is)] = fx[n];
    if constexpr (WF) {
#pragma unroll
      for (int n = 0; n < NV; ++n)
        fout[(((int64_t)n * g.nc3 + k) * g.nc2 + j) * (nc1 + 1) + f] = fx[n];
    }
  }
  __syncthreads();

  // P4: du = -beta dt div F1 + gravity source
  const double wght = beta * dtp[0];
  for (int i = is + tid; i <= ie; i += nth) {
    const int f0 = i - is;
    const double idx = 1. / g.dx1f[i];
    double fm0 = 0., fm1 = 0.;
#pragma unroll
    for (int n = 0; n <= NY; ++n) {
      fm0 += F[n * (nx1 + 1) + f0];
      fm1 += F[n * (nx1 + 1) + f0 + 1];
    }
#pragma unroll
    for (int n = 0; n < NV; ++n) {
      double d = (F[n * (nx1 + 1) + f0 + 1] - F[n * (nx1 + 1) + f0]) / g.dx1f[i];
      double v = -(wght * d);
      if (n == S::IVX) v += wght * grav * rho0[i];
      if (n == S::IPR) v += wght * grav * 0.5 * (fm0 + fm1);
      du[n * g.sv + base + i] = v;
    }
    (void)idx;
  }
}

constexpr int TI = 32;  // tile width along i
constexpr int TD = 8;   // tile length along the flux direction

template <int NY, int RECON, int RS, int DIR, bool WF>
__global__ void __launch_bounds__(256)
    k_flux_x23(Geom g, canoe_thermo_t th, const double *__restrict__ w,
               double *__restrict__ du, const double *__restrict__ dtp,
               double beta, double *__restrict__ fout) {
  using S = Slots<NY>;
  constexpr int NV = S::NV;
  constexpr int QR = TD + 2 * NG;  // staged rows
  constexpr int RR = TD + 2;       // reconstructed cells
  extern __shared__ double sm[];
  double *q = sm;                  // [NV][QR][TI]
  double *WL = q + NV * QR * TI;   // [NV][RR][TI]
  double *WR = WL + NV * RR * TI;  // [NV][RR][TI]
  double *F = q;                   // [NV][TD+1][TI]

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

  // P0: stage cells d0-3 .. d0+nd+2
  for (int c = ty; c < nd + 2 * NG; c += blockDim.y) {
    const int64_t off = base + (int64_t)(d0 - NG + c) * sd;
#pragma unroll
    for (int n = 0; n < NV; ++n)
      q[(n * QR + c) * TI + tx] = iok ? w[n * g.sv + off] : 1.;
  }
  __syncthreads();
  // P1: reconstruct cells d0-1 .. d0+nd (local c = 0 .. nd+1)
  for (int c = ty; c < nd + 2; c += blockDim.y) {
#pragma unroll
    for (int n = 0; n < NV; ++n) {
      const double *qc = q + (n * QR + c) * TI + tx;
      double wl_, wr_;
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
    double wl[NV], wr[NV], fx[NV];
#pragma unroll
    for (int n = 0; n < NV; ++n) {
      wl[n] = WR[(n * RR + f) * TI + tx];
      wr[n] = WL[(n * RR + f + 1) * TI + tx];
    }
    riemann<double, NY, RS, DIR>(th, wl, wr, fx);
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
          fout[idx] = fx[n];
        }
      }
    }
  }
  __syncthreads();
  // P3: du -= beta dt (F(c+1) - F(c)) / dx
  if (!iok) return;
  const double wght = beta * dtp[0];
  const double dx = DIR == 1 ? g.dx2 : g.dx3;
  for (int c = ty; c < nd; c += blockDim.y) {
    const int64_t off = base + (int64_t)(d0 + c) * sd;
#pragma unroll
    for (int n = 0; n < NV; ++n) {
      double d = (F[(n * (TD + 1) + c + 1) * TI + tx] - F[(n * (TD + 1) + c) * TI + tx]) / dx;
      du[n * g.sv + off] -= wght * d;
    }
  }
}

template <int NY>
size_t x1_smem(const Geom &g) {
  constexpr int NV = 5 + NY;
  return sizeof(double) * (3 * (size_t)NV * g.nc1 + 4 * (size_t)g.nc1 + 1);
}

template <int NY>
size_t x23_smem() {
  constexpr int NV = 5 + NY;
  return sizeof(double) * (size_t)NV * TI * ((TD + 2 * NG) + 2 * (TD + 2));
}

template <int NY, int RECON, int RS, bool WF>
int run_x1(const Geom &g, const canoe_thermo_t &th, const double *w, double *du,
           const double *dtp, double beta, double *fo, cudaStream_t st) {
  auto kern = k_flux_x1<NY, RECON, RS, WF>;
  size_t sm = x1_smem<NY>(g);
  static bool attr = false;
  if (!attr) {
    CB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 200 * 1024));
    attr = true;
  }
  unsigned nblk = (unsigned)g.nx2 * (unsigned)g.nx3;
  kern<<<nblk, 128, sm, st>>>(g, th, w, du, dtp, beta, fo);
  CB_CUDA(cudaGetLastError());
  return 0;
}

template <int NY, int RECON, int RS, int DIR, bool WF>
int run_x23(const Geom &g, const canoe_thermo_t &th, const double *w, double *du,
            const double *dtp, double beta, double *fo, cudaStream_t st) {
  auto kern = k_flux_x23<NY, RECON, RS, DIR, WF>;
  size_t sm = x23_smem<NY>();
  static bool attr = false;
  if (!attr) {
    CB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 200 * 1024));
    attr = true;
  }
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

template <int NY>
static int x1_dispatch(const Geom &g, const canoe_thermo_t &th, int recon, int rs,
                       const double *w, double *du, const double *dtp, double beta,
                       double *fo, cudaStream_t st) {
  const bool wf = fo != nullptr;
#define CB_X1(R, S, W) return run_x1<NY, R, S, W>(g, th, w, du, dtp, beta, fo, st)
  if (recon == CANOE_RECON_PPM) {
    if (rs == CANOE_RSOLVER_LMARS) { if (wf) CB_X1(3, 0, true); else CB_X1(3, 0, false); }
    else { if (wf) CB_X1(3, 1, true); else CB_X1(3, 1, false); }
  } else {
    if (rs == CANOE_RSOLVER_LMARS) { if (wf) CB_X1(2, 0, true); else CB_X1(2, 0, false); }
    else { if (wf) CB_X1(2, 1, true); else CB_X1(2, 1, false); }
  }
#undef CB_X1
}

template <int NY, int DIR>
static int x23_dispatch(const Geom &g, const canoe_thermo_t &th, int recon, int rs,
                        const double *w, double *du, const double *dtp, double beta,
                        double *fo, cudaStream_t st) {
  const bool wf = fo != nullptr;
#define CB_X23(R, S, W) return run_x23<NY, R, S, DIR, W>(g, th, w, du, dtp, beta, fo, st)
  if (recon == CANOE_RECON_PPM) {
    if (rs == CANOE_RSOLVER_LMARS) { if (wf) CB_X23(3, 0, true); else CB_X23(3, 0, false); }
    else { if (wf) CB_X23(3, 1, true); else CB_X23(3, 1, false); }
  } else {
    if (rs == CANOE_RSOLVER_LMARS) { if (wf) CB_X23(2, 0, true); else CB_X23(2, 0, false); }
    else { if (wf) CB_X23(2, 1, true); else CB_X23(2, 1, false); }
  }
#undef CB_X23
}

int launch_flux_x1(const Geom &g, const canoe_thermo_t &th, int recon, int rs,
                   int precision, const double *w, double *du, const double *dtp,
                   double beta, double *fo, cudaStream_t st) {
  (void)precision;
  if (g.nx1 + NG > 32 * 64) {
    set_error("x1 pencil too long");
    return CANOE_ERR_ARG;
  }
  CB_DISPATCH_NY(th.ny, (x1_dispatch<NY>(g, th, recon, rs, w, du, dtp, beta, fo, st)));
}

int launch_flux_x23(int dir, const Geom &g, const canoe_thermo_t &th, int recon,
                    int rs, int precision, const double *w, double *du,
                    const double *dtp, double beta, double *fo, cudaStream_t st) {
  (void)precision;
  if (dir == 1) {
    CB_DISPATCH_NY(th.ny, (x23_dispatch<NY, 1>(g, th, recon, rs, w, du, dtp, beta, fo, st)));
  } else {
    CB_DISPATCH_NY(th.ny, (x23_dispatch<NY, 2>(g, th, recon, rs, w, du, dtp, beta, fo, st)));
  }
}

}  // namespace cb
