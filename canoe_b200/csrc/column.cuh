// column.cuh -- one CTA per vertical (x1) pencil: x1 fluxes, the implicit
// vertical solve and the RK register update, fused.
//
// Per pencil (k, j), all in shared memory:
//  P0  stage the primitive pencil w(:, k, j, 0..nc1-1)
//  P1  Decomposition::ChangeToTemperature (canoe src/snap/decomposition/
//      change_to_temperature.cpp:40-136): hydrostatic face pressure psf summed
//      serially from the top in the reference's order, log-mean psv, RovRd,
//      rho -> T, p -> p'
//  P2  PLM / PPM reconstruction of every variable (Athena precon, restated)
//  P3  RestoreFromTemperature at the faces (:138-167) + the Riemann solver
//      (canoe src/snap/riemann/lmars.cpp, hllc_transform.cpp)
//  P4  du = du(x2, x3 divergence from the earlier kernels) - beta dt div F1
//      + constant-gravity source
//  P5  block rows a, b, c of the implicit correction (PartialCorrection,
//      src/snap/implicit/partial_correction.cpp:26-154, N = 3, or
//      FullCorrection, full_correction.cpp:32-145, N = 5): |A| at the faces
//      and flux Jacobians of the cells are built once and shared
//  P6  the block-tridiagonal solve by block cyclic reduction across the CTA
//      (the reference eliminates sequentially, forward_backward.hpp:15-137;
//      both solve the same system)
//  P7  forward_backward.hpp:101-124 species correction and the register
//      update u = g1 u + g2 u1 + du (implicit_hydro_tasks.cpp:152-160, 283)
// Every global access is contiguous along the pencil.
#pragma once

#include "blockmat.cuh"

namespace cb {

enum ColMode { kColFluxOnly = 0, kColStep = 1, kColSolveOnly = 2 };

// threads per pencil: 5 warps cover the nx1 + 1 faces and nx1 + 2 cells of a
// 128-level column in one pass
constexpr int kColThreads = 160;

template <int N>
struct ColRow {
  static constexpr int NN = N * N;
  // a | b | c | rhs (x after the solve), padded to an odd number of doubles
  // so that neighbouring rows fall in different shared-memory banks
  static constexpr int ROW = (3 * NN + N) | 1;
};

// shared-memory plan (doubles) of one pencil
struct ColSmem {
  int wp, dc, uni, total;
};

__host__ __device__ inline ColSmem col_smem(int nv, int nc1, int nx1, int n_impl) {
  ColSmem s;
  s.wp = 0;                  // [NV][nc1] pristine pencil
  s.dc = nv * nc1;           // [NV][nx1] du of the column
  s.uni = s.dc + nv * nx1;   // union region
  const int flux = 3 * nv * nc1 + 3 * nc1 + 1;
  int solve = 0;
  if (n_impl) {
    const int nn = n_impl * n_impl;
    solve = nx1 * ((3 * nn + n_impl) | 1) + (nx1 + 1) * nn + (nx1 + 2) * nn;
  }
  s.total = s.uni + (flux > solve ? flux : solve);
  return s;
}

// R = double: the FP64 path.  R = float: reconstruction and Riemann fluxes in
// FP32 on the perturbation p' from the FP64 hydrostatic face pressure psf;
// the divergence of psf and the gravity source are added in FP64.
template <int NY, int RECON, int RS, int N, int MODE, typename R>
__global__ void __launch_bounds__(kColThreads, N == 5 ? 1 : 3)
    k_x1col(Geom g, canoe_thermo_t th, const double *__restrict__ w,
            double *__restrict__ du, double *__restrict__ u, double *__restrict__ u1,
            const double *__restrict__ dtp, Stage st, int stage,
            double *__restrict__ fout) {
  using S = Slots<NY>;
  constexpr int NV = S::NV;
  extern __shared__ double sm[];
  const int nc1 = g.nc1, is = g.is, ie = g.ie, nx1 = g.nx1;
  const ColSmem L = col_smem(NV, nc1, nx1, N);
  double *wp = sm + L.wp;
  double *dc = sm + L.dc;
  double *un = sm + L.uni;

  const int j = g.js + (int)(blockIdx.x % (unsigned)g.nx2);
  const int k = g.ks + (int)(blockIdx.x / (unsigned)g.nx2);
  const int64_t base = (int64_t)k * g.sk + (int64_t)j * nc1;
  const int tid = threadIdx.x, nth = blockDim.x;
  const double grav = th.grav;
  const double wght = st.beta * dtp[0];

  // P0: stage the pencil
  for (int n = 0; n < NV; ++n)
    for (int i = tid; i < nc1; i += nth) wp[n * nc1 + i] = w[n * g.sv + base + i];

  constexpr bool PERT = sizeof(R) == 4;
  if constexpr (MODE != kColSolveOnly) {
    R *q = reinterpret_cast<R *>(un);          // [NV][nc1] transformed copy, later F
    R *WL = q + NV * nc1;                      // [NV][nc1]
    R *WR = WL + NV * nc1;                     // [NV][nc1]
    double *psf = un + (3 * NV * nc1 * (int)sizeof(R) + 7) / 8;  // [nc1+1]
    double *psv = psf + nc1 + 1;               // [nc1]
    double *gam = psv + nc1;                   // [nc1]
    R *F = q;                                  // [NV][nx1+1]
    // without gravity the FP32 path uses one constant reference pressure
    const double pcst = (PERT && grav == 0.) ? g.pref[is] : 0.;
    for (int n = 0; n < NV; ++n)
      for (int i = tid; i < nc1; i += nth) {
        double v = wp[n * nc1 + i];
        if (n == S::IPR) v -= pcst;
        q[n * nc1 + i] = R(v);
      }
    // P1
    if (grav != 0.) {
      R *rho = q, *pre = q + S::IPR * nc1;
      const double *rho0 = wp, *pre0 = wp + S::IPR * nc1;
      for (int i = tid; i < nc1; i += nth) psv[i] = g.dx1f[i];
      __syncthreads();
      if (tid == 0) {
        const double *dx = psv;
        const double *rho = rho0, *pre = pre0;
        double RdTv = pre[ie] / rho[ie];
        double acc = pre[ie] * exp(grav * dx[ie] / (2 * RdTv));
        psf[ie + 1] = acc;
        for (int i = ie; i >= is; --i) {
          acc = acc - grav * rho[i] * dx[i];
          psf[i] = acc;
        }
        const double gb = g.bc[0] == CANOE_BC_REFLECT ? -grav : grav;
        for (int i = is - 1; i >= is - NG; --i) {
          acc = acc - gb * rho[i] * dx[i];
          psf[i] = acc;
        }
        const double gt = g.bc[1] == CANOE_BC_REFLECT ? -grav : grav;
        double p = psf[ie + 1];
        for (int i = ie + 1; i <= ie + NG; ++i) {
          p = p + gt * rho[i] * dx[i];
          psf[i + 1] = p;
        }
      }
      __syncthreads();
      for (int i = tid; i < nc1; i += nth) {
        double a = psf[i], b = psf[i + 1];
        double pv = fabs(a - b) < 1.E-6 ? 0.5 * (a + b) : (a - b) / log(a / b);
        double feps = 1.;
#pragma unroll
        for (int n = 1; n <= NY; ++n)
          if (n <= th.nvapor) feps += wp[n * nc1 + i] * th.inv_mu_ratio_m1[n - 1];
        double gm = th.rd * feps;
        psv[i] = pv;
        gam[i] = gm;
        rho[i] = R(pre0[i] / (rho0[i] * gm));
        pre[i] = R(pre0[i] - pv);
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
    }
    __syncthreads();
    // P2
    const int ncell = nx1 + 2;
    for (int t = tid; t < NV * ncell; t += nth) {
      const int n = t / ncell, c = is - 1 + t % ncell;
      const R *qn = q + n * nc1;
      R wl_, wr_;
      if constexpr (RECON == CANOE_RECON_PPM)
        ppm_cell(qn[c - 2], qn[c - 1], qn[c], qn[c + 1], qn[c + 2], wl_, wr_);
      else
        plm_cell_nu(qn[c - 1], qn[c], qn[c + 1], R(g.x1v[c - 1]), R(g.x1v[c]),
                    R(g.x1v[c + 1]), R(g.x1f[c]), R(g.x1f[c + 1]), wl_, wr_);
      WL[n * nc1 + c] = wl_;
      WR[n * nc1 + c] = wr_;
    }
    __syncthreads();
    // P3 (F aliases q, which nobody reads after P2)
    for (int f = is + tid; f <= ie + 1; f += nth) {
      R wl[NV], wr[NV], fx[NV];
#pragma unroll
      for (int n = 0; n < NV; ++n) {
        wl[n] = WR[n * nc1 + f - 1];
        wr[n] = WL[n * nc1 + f];
      }
      const double pf = grav != 0. ? psf[f] : pcst;
      if (grav != 0.) {
        const double gamma = sqrt(gam[f] * gam[f - 1]);
        if constexpr (PERT) {
          // keep p' relative to psf(f); floor p = psf(f) as the reference does
          R pr = wr[S::IPR], pl = wl[S::IPR];
          if (R(pf) + pr < R(0)) pr = R(0);
          if (R(pf) + pl < R(0)) pl = R(0);
          wr[S::IPR] = pr;
          wl[S::IPR] = pl;
          wr[0] = (R(pf) + pr) / (wr[0] * R(gamma));
          wl[0] = (R(pf) + pl) / (wl[0] * R(gamma));
        } else {
          double pr = wr[S::IPR] + pf;
          if (pr < 0.) pr = pf;
          wr[S::IPR] = pr;
          wr[0] = pr / (wr[0] * gamma);
          double pl = wl[S::IPR] + pf;
          if (pl < 0.) pl = pf;
          wl[S::IPR] = pl;
          wl[0] = pl / (wl[0] * gamma);
        }
      }
      if constexpr (PERT)
        riemann_pert<R, NY, RS, 0>(th, wl, wr, R(pf), fx);
      else
        riemann<R, NY, RS, 0>(th, wl, wr, fx);
#pragma unroll
      for (int n = 0; n < NV; ++n) F[n * (nx1 + 1) + (f - is)] = fx[n];
      if constexpr (MODE == kColFluxOnly) {
#pragma unroll
        for (int n = 0; n < NV; ++n) {
          double v = fx[n];
          if (PERT && n == S::IVX) v += pf;  // report the full flux
          fout[(((int64_t)n * g.nc3 + k) * g.nc2 + j) * (nc1 + 1) + f] = v;
        }
      }
    }
    __syncthreads();
    // P4
    for (int i = is + tid; i <= ie; i += nth) {
      const int f0 = i - is;
      const double idx = 1. / g.dx1f[i];
      double fm0 = 0., fm1 = 0.;
#pragma unroll
      for (int n = 0; n <= NY; ++n) {
        fm0 += (double)F[n * (nx1 + 1) + f0];
        fm1 += (double)F[n * (nx1 + 1) + f0 + 1];
      }
#pragma unroll
      for (int n = 0; n < NV; ++n) {
        double d = ((double)F[n * (nx1 + 1) + f0 + 1] - (double)F[n * (nx1 + 1) + f0]) * idx;
        // FP32 path: the momentum flux lacks psf, whose divergence is FP64
        if (PERT && n == S::IVX && grav != 0.) d += (psf[i + 1] - psf[i]) * idx;
        double v = -(wght * d);
        if (n == S::IVX) v += wght * grav * wp[i];
        if (n == S::IPR) v += wght * grav * 0.5 * (fm0 + fm1);
        if constexpr (MODE == kColFluxOnly) {
          du[n * g.sv + base + i] = v;
        } else {
          const double prev = g.f2 ? du[n * g.sv + base + i] : 0.;
          dc[n * nx1 + f0] = prev + v;
        }
      }
    }
    if constexpr (MODE == kColFluxOnly) return;
  } else {
    for (int n = 0; n < NV; ++n)
      for (int r = tid; r < nx1; r += nth) dc[n * nx1 + r] = du[n * g.sv + base + is + r];
  }
  __syncthreads();

  if constexpr (N > 0) {
    constexpr int NN = ColRow<N>::NN, ROW = ColRow<N>::ROW;
    double *blk = un;                        // [nx1][ROW]
    double *sA = blk + nx1 * ROW;            // [nx1+1][NN] |A| at faces is-1/2..ie+1/2
    double *sJ = sA + (nx1 + 1) * NN;        // [nx1+2][NN] J of cells is-1..ie+1
    const double gm1 = th.gammad - 1.;
    const double dt = wght;
    const double idt = 1. / dt;
    const double area = g.dx2 * g.dx3;
    // P5a: |A| at face t (between cells is-1+t and is+t) and J of cell is-1+t
    for (int t = tid; t < nx1 + 2; t += nth) {
      const int ic = is - 1 + t;
      double wl[NV], wr[NV];
#pragma unroll
      for (int n = 0; n < NV; ++n) wl[n] = wp[n * nc1 + ic];
      M<N> J;
      jacobian<N, NY>(J, gm1, wl);
#pragma unroll
      for (int e = 0; e < NN; ++e) sJ[t * NN + e] = J.a[e / N][e % N];
      if (t <= nx1) {
#pragma unroll
        for (int n = 0; n < NV; ++n) wr[n] = wp[n * nc1 + ic + 1];
        M<N> A;
        abs_jacobian<N, NY>(A, th, gm1, wl, wr);
#pragma unroll
        for (int e = 0; e < NN; ++e) sA[t * NN + e] = A.a[e / N][e % N];
      }
    }
    __syncthreads();
    // P5b: block rows (partial_correction.cpp:128-154); b of the first and c
    // of the last row couple to ghosts: the reflecting condition folds them
    // into a, and the sweep never uses them, so they are zeroed here
    for (int r = tid; r < nx1; r += nth) {
      const int i = is + r;
      const double i2v = 1. / (2. * (g.dx1f[i] * g.dx2 * g.dx3));
      double *row = blk + r * ROW;
#pragma unroll
      for (int e = 0; e < NN; ++e) {
        const int rr = e / N, qq = e % N;
        const double Am = sA[r * NN + e], Ap = sA[(r + 1) * NN + e];
        const double Jm = sJ[r * NN + e], Jc = sJ[(r + 1) * NN + e], Jn = sJ[(r + 2) * NN + e];
        double phi;
        if (N == 3) phi = ((rr == 1 && qq == 0) || (rr == 2 && qq == 1)) ? grav : 0.;
        else phi = ((rr == 1 && qq == 0) || (rr == 4 && qq == 1)) ? grav : 0.;
        double a = (Am * area + Ap * area + (area - area) * Jc) * i2v + (rr == qq ? idt : 0.) - phi;
        const double b = -(Am + Jm) * area * i2v;
        const double c = -(Ap - Jn) * area * i2v;
        if (i == is) a += (qq == 1 ? -b : b);
        if (i == ie) a += (qq == 1 ? -c : c);
        row[e] = a;
        row[NN + e] = i == is ? 0. : b;
        row[2 * NN + e] = i == ie ? 0. : c;
      }
      // right-hand side (forward_backward.hpp:24-41)
      double r0 = dc[r];
#pragma unroll
      for (int n = 1; n <= NY; ++n) r0 += dc[n * nx1 + r];
      double *rh = row + 3 * NN;
      rh[0] = r0 / dt;
      rh[1] = dc[S::IVX * nx1 + r] / dt;
      if constexpr (N == 3) {
        rh[2] = dc[S::IPR * nx1 + r] / dt;
      } else {
        rh[2] = dc[S::IVY * nx1 + r] / dt;
        rh[3] = dc[S::IVZ * nx1 + r] / dt;
        rh[4] = dc[S::IPR * nx1 + r] / dt;
      }
    }
    __syncthreads();
    // P6: block cyclic reduction.  Rows with (r+1) % 2s == 0 survive level s;
    // rows with (r+1) % 2s == s are eliminated (their a is replaced by a^-1).
    auto ld = [&](const double *p) {
      M<N> m;
#pragma unroll
      for (int e = 0; e < NN; ++e) m.a[e / N][e % N] = p[e];
      return m;
    };
    auto stm = [&](double *p, const M<N> &m) {
#pragma unroll
      for (int e = 0; e < NN; ++e) p[e] = m.a[e / N][e % N];
    };
    auto ldv = [&](const double *p) {
      V<N> v;
#pragma unroll
      for (int e = 0; e < N; ++e) v.a[e] = p[e];
      return v;
    };
    auto stv = [&](double *p, const V<N> &v) {
#pragma unroll
      for (int e = 0; e < N; ++e) p[e] = v.a[e];
    };
    // active rows are compacted onto the lowest threads so that a level
    // with few rows occupies few warps
    int s = 1;
    for (; 2 * s - 1 < nx1; s *= 2) {
      const int ne = (nx1 + s) / (2 * s);  // eliminated rows r = s-1 + 2 s m
      for (int m = tid; m < ne; m += nth) {
        const int r = s - 1 + 2 * s * m;
        stm(blk + r * ROW, inv(ld(blk + r * ROW)));
      }
      __syncthreads();
      const int nu = nx1 / (2 * s);  // surviving rows r = 2 s (m+1) - 1
      for (int m = tid; m < nu; m += nth) {
        const int r = 2 * s * (m + 1) - 1;
        double *row = blk + r * ROW;
        const double *lo = blk + (r - s) * ROW;
        M<N> a = ld(row), b = ld(row + NN), c = ld(row + 2 * NN);
        V<N> rh = ldv(row + 3 * NN);
        // alpha = -b a_lo^-1
        M<N> al = mm(b, ld(lo));
#pragma unroll
        for (int e = 0; e < NN; ++e) al.a[e / N][e % N] = -al.a[e / N][e % N];
        M<N> t = mm(al, ld(lo + 2 * NN));
        V<N> tv = mv(al, ldv(lo + 3 * NN));
#pragma unroll
        for (int e = 0; e < NN; ++e) a.a[e / N][e % N] += t.a[e / N][e % N];
#pragma unroll
        for (int e = 0; e < N; ++e) rh.a[e] += tv.a[e];
        M<N> bn = mm(al, ld(lo + NN));
        M<N> cn;
        if (r + s < nx1) {
          const double *hi = blk + (r + s) * ROW;
          M<N> ga = mm(c, ld(hi));
#pragma unroll
          for (int e = 0; e < NN; ++e) ga.a[e / N][e % N] = -ga.a[e / N][e % N];
          t = mm(ga, ld(hi + NN));
          tv = mv(ga, ldv(hi + 3 * NN));
#pragma unroll
          for (int e = 0; e < NN; ++e) a.a[e / N][e % N] += t.a[e / N][e % N];
#pragma unroll
          for (int e = 0; e < N; ++e) rh.a[e] += tv.a[e];
          cn = mm(ga, ld(hi + 2 * NN));
        } else {
#pragma unroll
          for (int e = 0; e < NN; ++e) cn.a[e / N][e % N] = 0.;
        }
        stm(row, a);
        stm(row + NN, bn);
        stm(row + 2 * NN, cn);
        stv(row + 3 * NN, rh);
      }
      __syncthreads();
    }
    // the last surviving row r = s - 1 is decoupled
    if (tid == 0) {
      double *row = blk + (s - 1) * ROW;
      M<N> ai = inv(ld(row));
      stm(row, ai);
      stv(row + 3 * NN, mv(ai, ldv(row + 3 * NN)));
    }
    __syncthreads();
    for (s /= 2; s >= 1; s /= 2) {
      const int ne = (nx1 + s) / (2 * s);
      for (int m = tid; m < ne; m += nth) {
        const int r = s - 1 + 2 * s * m;
        double *row = blk + r * ROW;
        V<N> rh = ldv(row + 3 * NN);
        if (r - s >= 0) {
          V<N> t = mv(ld(row + NN), ldv(blk + (r - s) * ROW + 3 * NN));
#pragma unroll
          for (int e = 0; e < N; ++e) rh.a[e] -= t.a[e];
        }
        if (r + s < nx1) {
          V<N> t = mv(ld(row + 2 * NN), ldv(blk + (r + s) * ROW + 3 * NN));
#pragma unroll
          for (int e = 0; e < N; ++e) rh.a[e] -= t.a[e];
        }
        stv(row + 3 * NN, mv(ld(row), rh));
      }
      __syncthreads();
    }
    // P7a: species correction (forward_backward.hpp:101-124) into dc
    for (int r = tid; r < nx1; r += nth) {
      const double *x = blk + r * ROW + 3 * NN;
      const int i = is + r;
      double dv[NV];
#pragma unroll
      for (int n = 0; n < NV; ++n) dv[n] = dc[n * nx1 + r];
      double dens = dv[0];
#pragma unroll
      for (int n = 1; n <= NY; ++n) dens += dv[n];
      dens = x[0] - dens;
      dv[0] = x[0];
#pragma unroll
      for (int n = 1; n <= NY; ++n) dv[n] += dens * wp[n * nc1 + i];
      dv[S::IVX] = x[1];
      if constexpr (N == 3) {
        dv[S::IPR] = x[2];
      } else {
        dv[S::IVY] = x[2];
        dv[S::IVZ] = x[3];
        dv[S::IPR] = x[4];
      }
#pragma unroll
      for (int n = 1; n <= NY; ++n) dv[0] -= dv[n];
#pragma unroll
      for (int n = 0; n < NV; ++n) dc[n * nx1 + r] = dv[n];
    }
    __syncthreads();
  }

  // P7b: write back
  if constexpr (MODE == kColSolveOnly) {
    for (int n = 0; n < NV; ++n)
      for (int r = tid; r < nx1; r += nth) du[n * g.sv + base + is + r] = dc[n * nx1 + r];
  } else {
    for (int n = 0; n < NV; ++n)
      for (int r = tid; r < nx1; r += nth) {
        const int64_t x = n * g.sv + base + is + r;
        const double uo = u[x];
        double ur;
        if (stage == 0) {
          u1[x] = uo;
          ur = uo;
        } else {
          ur = u1[x];
        }
        const double t = st.g1 * uo + st.g2 * ur;
        u[x] = t + dc[n * nx1 + r];
      }
  }
}

// launcher for one NY (instantiated in column_ny*.cu)
template <int NY, typename R>
int run_x1col_p(const Geom &g, const canoe_thermo_t &th, int recon, int rs, int flag,
                int mode, const double *w, double *du, double *u, double *u1,
                const double *dtp, const Stage &s, int stage, double *fout,
                cudaStream_t st) {
  const int nimpl = (mode == kColFluxOnly || !(flag & 1)) ? 0 : ((flag & 8) ? 5 : 3);
  if (mode == kColSolveOnly && nimpl == 0) return 0;
  const ColSmem L = col_smem(5 + NY, g.nc1, g.nx1, nimpl);
  const size_t smem = sizeof(double) * (size_t)L.total;
  if (smem > 227 * 1024) {
    set_error("x1 pencil too long for shared memory");
    return CANOE_ERR_UNSUPPORTED;
  }
  const unsigned nblk = (unsigned)g.nx2 * (unsigned)g.nx3;
  auto go = [&](auto kern) -> int {
    if (int rc = ensure_smem((const void *)kern, smem)) return rc;
    kern<<<nblk, kColThreads, smem, st>>>(g, th, w, du, u, u1, dtp, s, stage, fout);
    CB_CUDA(cudaGetLastError());
    return 0;
  };
  const bool ppm = recon == CANOE_RECON_PPM, hllc = rs == CANOE_RSOLVER_HLLC;
#define CB_COL(NIMPL, MODE)                                                        \
  (ppm ? (hllc ? go(k_x1col<NY, 3, 1, NIMPL, MODE, R>) : go(k_x1col<NY, 3, 0, NIMPL, MODE, R>)) \
       : (hllc ? go(k_x1col<NY, 2, 1, NIMPL, MODE, R>) : go(k_x1col<NY, 2, 0, NIMPL, MODE, R>)))
  if (mode == kColFluxOnly) return CB_COL(0, kColFluxOnly);
  if (mode == kColSolveOnly)
    return nimpl == 3 ? go(k_x1col<NY, 3, 1, 3, kColSolveOnly, double>)
                      : go(k_x1col<NY, 3, 1, 5, kColSolveOnly, double>);
  if (nimpl == 0) return CB_COL(0, kColStep);
  if (nimpl == 3) return CB_COL(3, kColStep);
  return CB_COL(5, kColStep);
#undef CB_COL
}

template <int NY>
int run_x1col(const Geom &g, const canoe_thermo_t &th, int recon, int rs, int flag,
              int prec, int mode, const double *w, double *du, double *u, double *u1,
              const double *dtp, const Stage &s, int stage, double *fout,
              cudaStream_t st) {
  if (prec == CANOE_FP32_PERTURBATION && mode != kColSolveOnly)
    return run_x1col_p<NY, float>(g, th, recon, rs, flag, mode, w, du, u, u1, dtp, s, stage,
                                  fout, st);
  return run_x1col_p<NY, double>(g, th, recon, rs, flag, mode, w, du, u, u1, dtp, s, stage,
                                 fout, st);
}

}  // namespace cb
