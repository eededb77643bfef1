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
//      both solve the same system).  Periodic x1 (PER): the cyclic system of
//      periodic_forward_backward.hpp:15-234 is solved by bordering: the
//      reduction runs on rows 0..n-2 with N extra right-hand columns (the
//      couplings of rows 0 and n-2 to row n-1), then row n-1 closes with one
//      N x N Schur-complement solve
//  P7  forward_backward.hpp:101-124 species correction and the register
//      update u = g1 u + g2 u1 + du (implicit_hydro_tasks.cpp:152-160, 283)
// Every global access is contiguous along the pencil.
#pragma once

#include "blockmat.cuh"
#include "bulk.cuh"

namespace cb {


// threads per pencil: 5 warps cover the nx1 + 1 faces and nx1 + 2 cells of a
// 128-level column in one pass
constexpr int kColThreads = 160;
// the full 5x5 solve runs row-parallel (8-lane segments per block row-op),
// 7 warps per pencil and two pencils per SM
constexpr int kCol5Threads = 224;
// the 3x3 solve with the compact plan: 4 warps per pencil by default (four
// pencils per SM at 128 levels), up to 8 when a batch's autotuner picks them
// for tall columns, whose shared memory allows fewer pencils per SM
constexpr bool kCompact3 = true;
constexpr int kCol3Threads = 128;
constexpr int kCol3ThreadsMax = 256;

// the compact shared-memory plan (|A| and J staged in the rows' own slots,
// no u / u1 prefetch): the 5x5 solve, and the 3x3 one when kCompact3
template <int N, bool PER, int GEO>
struct ColPlan {
  static constexpr bool compact = !PER && (N == 5 || (N == 3 && kCompact3));
  static constexpr int threads =
      !compact ? kColThreads : (N == 5 ? kCol5Threads : kCol3ThreadsMax);
  // registers: 65536 / (threads x blocks) = 128 per thread for the 3x3 plans
  static constexpr int blocks = N == 5 ? (PER ? 1 : 2) : (compact ? 2 : 3);
};

// doubles per block row a | b | c | rhs (x after the solve), rounded up to
// 1 mod 16; with one more double after every 16 rows (row r starts at
// r ROW + r / 16) the rows a reduction level touches, 2s apart, fall in
// distinct 8-byte shared-memory banks for s = 1, 2, 4, 8 (the padding of
// Harris, Sengupta and Owens, GPU Gems 3 ch. 39, applied to whole rows)
__host__ __device__ constexpr int col_row(int n) { return ((3 * n * n + n + 14) / 16) * 16 + 1; }
__host__ __device__ constexpr int col_rows(int n, int nx1) {
  return nx1 * col_row(n) + (nx1 >> 4) + 1;
}

template <int N>
struct ColRow {
  static constexpr int NN = N * N;
  static constexpr int ROW = col_row(N);
};

// shared-memory plan (doubles) of one pencil
struct ColSmem {
  int wp, dc, uni, stg, z, mbar, total;
};

__host__ __device__ inline int even_up(int x) { return (x + 1) & ~1; }

__host__ __device__ inline ColSmem col_smem(int nv, int nc1, int nx1, int n_impl, int per = 0,
                                            int compact = 0) {
  ColSmem s;
  s.wp = 0;                  // [NV][nc1] pristine pencil
  s.dc = nv * nc1;           // [NV][nc1] du of the column (interior at is)
  s.uni = even_up(2 * nv * nc1);  // union region
  const int flux = 3 * nv * nc1 + 3 * nc1 + 1;
  int solve = 0;
  s.stg = 0;
  s.z = 0;
  if (n_impl && compact) {
    // compact plan: |A| and J are staged in the rows' own c and b slots
    // (plus three blocks past the last row, at stg), and u / u1 are not
    // prefetched
    const int nn = n_impl * n_impl;
    const int rows = even_up(col_rows(n_impl, nx1));
    s.stg = s.uni + rows;
    solve = rows + 3 * nn;
  } else if (n_impl) {
    const int nn = n_impl * n_impl;
    const int rows = even_up(col_rows(n_impl, nx1));
    // |A| and J, later reused as the staging area of u and u1
    const int aj = (nx1 + 1) * nn + (nx1 + 2) * nn;
    const int st = 2 * nv * nc1;
    s.stg = s.uni + rows;
    solve = rows + (aj > st ? aj : st);
    if (per) {  // [nx1][nn] bordering columns of the periodic solve
      s.z = s.uni + solve;
      solve += nx1 * nn;
    }
  }
  s.mbar = s.uni + even_up(flux > solve ? flux : solve);
  s.total = s.mbar + 4;  // 3 mbarriers, 8 bytes each
  return s;
}

// R = double: the FP64 path.  R = float: reconstruction and Riemann fluxes in
// FP32 on the perturbation p' from the FP64 hydrostatic face pressure psf;
// the divergence of psf and the gravity source are added in FP64.
//
// Latency hiding inside the CTA: the pencil rows of w and du arrive by bulk
// copies issued at entry; u and u1 are fetched into the dead |A| / J area
// while the cyclic reduction runs (plans with a separate |A| / J area), or,
// in the compact plans, moved into L2 by bulk prefetches issued at entry;
// the serial hydrostatic scan (one lane of warp 0) overlaps the
// reconstruction of the variables it does not touch.
//
// GEO = 1: a cubed-sphere panel (dry, HLLC, FP64 or FP32 fluxes; the six
// panels of a shell in one launch through Geom::npanel): covariant kinetic energy
// in the Riemann problem and the covariant flux projection
// (hllc_transform.cpp:92-101, 245-272), radial face areas and cell volumes
// (gnomonic_equiangle.cpp:224-432), the coordinate source terms
// (AddCoordTermsDivergence, :833-878) and the implicit solve on velocities
// projected to the local frame (solve_implicit_3d.cpp:105-137).
//
// PER: periodic x1 (both ends), implicit modes only; the cyclic solve and the
// reference's periodic du update without the species correction
// (periodic_forward_backward.hpp:207-225).
template <int NY, int RECON, int RS, int N, int MODE, typename R, int GEO = 0, bool PER = false>
__global__ void __launch_bounds__(ColPlan<N, PER, GEO>::threads, ColPlan<N, PER, GEO>::blocks)
    k_x1col(Geom g, canoe_thermo_t th, const double *__restrict__ w,
            double *__restrict__ du, double *__restrict__ u, double *__restrict__ u1,
            const double *__restrict__ dtp, Stage st, int stage,
            double *__restrict__ fout) {
  using S = Slots<NY>;
  constexpr int NV = S::NV;
  extern __shared__ double sm[];
  const int nc1 = g.nc1, is = g.is, ie = g.ie, nx1 = g.nx1;
  const ColSmem L = col_smem(NV, nc1, nx1, N, PER, ColPlan<N, PER, GEO>::compact);
  double *wp = sm + L.wp;
  double *dc = sm + L.dc;
  double *un = sm + L.uni;
  uint64_t *mbar = reinterpret_cast<uint64_t *>(sm + L.mbar);

  const unsigned ncol = (unsigned)g.nx2 * (unsigned)g.nx3;
  const unsigned col = blockIdx.x % ncol;
  const int j = g.js + (int)(col % (unsigned)g.nx2);
  const int k = g.ks + (int)(col / (unsigned)g.nx2);
  const int64_t base = (int64_t)k * g.sk + (int64_t)j * nc1;
  if (g.npanel > 1) {  // panel of this column: shift the block arrays
    const int64_t poff = (int64_t)(blockIdx.x / ncol) * g.pstride;
    w += poff;
    du += poff;
    u += poff;
    u1 += poff;
  }
  const int tid = threadIdx.x, nth = blockDim.x;
  const int warp = tid >> 5, lane = tid & 31;
  // panel geometry of the column (GEO)
  const int64_t nkj = (int64_t)g.nc3 * g.nc2;
  auto tab = [&](int t, int kk, int jj) { return g.shell[t * nkj + (int64_t)kk * g.nc2 + jj]; };
  const double grav = th.grav;
  const double wght = st.beta * dtp[0];
  const bool bulk = g.bulk != 0;
  constexpr bool SOLVE_ONLY = MODE == kColSolveOnly || MODE == kColSolveStep;
  constexpr bool UPDATE = MODE == kColStep || MODE == kColSolveStep;
  constexpr bool NEED_DU = MODE != kColFluxOnly;
  const bool load_du = NEED_DU && (SOLVE_ONLY || g.f2);
  const uint32_t row_bytes = (uint32_t)nc1 * 8u;

  // a wait that gave up: report, give the copies still in flight on
  // mbarriers q0 .. q1-1 a second bounded wait, leave
  auto bail = [&](int q0, int q1) {
    if (tid == 0 && g.err) atomicOr(g.err, (uint32_t)CANOE_EBIT_TIMEOUT);
    for (int q = q0; q < q1; ++q) mbar_wait(mbar + q, 0);
  };

  // x1 spacing of this thread's first cell, read while the pencil rows are
  // in flight (the hydrostatic scan's operands take it after the wait)
  const double dx_first = g.dx1f[tid < nc1 ? tid : nc1 - 1];

  // P0: stage the pencil (and du)
  if (bulk) {
    if (tid == 0) {
      for (int q = 0; q < 3; ++q) mbar_init(mbar + q, 1);
      fence_mbar_init();
      mbar_expect_tx(mbar, NV * row_bytes);
      for (int n = 0; n < NV; ++n) bulk_g2s(wp + n * nc1, w + n * g.sv + base, row_bytes, mbar);
      if (load_du) {
        mbar_expect_tx(mbar + 1, NV * row_bytes);
        for (int n = 0; n < NV; ++n)
          bulk_g2s(dc + n * nc1, du + n * g.sv + base, row_bytes, mbar + 1);
      }
      // the compact plans read u and u1 only at the register update: start
      // moving their rows into L2 now
      if constexpr (UPDATE && ColPlan<N, PER, GEO>::compact) {
        for (int n = 0; n < NV; ++n) {
          bulk_prefetch_l2(u + n * g.sv + base, row_bytes);
          if (stage != 0) bulk_prefetch_l2(u1 + n * g.sv + base, row_bytes);
        }
      }
    }
    __syncthreads();
    if (!__syncthreads_and(mbar_wait(mbar, 0))) {
      bail(0, load_du ? 2 : 1);
      return;
    }
  } else {
    for (int n = 0; n < NV; ++n)
      for (int i = tid; i < nc1; i += nth) wp[n * nc1 + i] = w[n * g.sv + base + i];
    if (load_du)
      for (int n = 0; n < NV; ++n)
        for (int i = is + tid; i <= ie; i += nth) dc[n * nc1 + i] = du[n * g.sv + base + i];
  }

  constexpr bool PERT = sizeof(R) == 4;
  if constexpr (!SOLVE_ONLY) {
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
    // operands of the hydrostatic scan, staged where psv / gam go later:
    // gam <- grav rho(i) (rounded as the scan's product), psv <- dx1f(i)
    if (grav != 0.)
      for (int i = tid; i < nc1; i += nth) {
        gam[i] = grav * wp[i];
        psv[i] = i == tid ? dx_first : g.dx1f[i];
      }
    __syncthreads();
    // P2 for variable n over the cells is-1 .. ie+1, items t0, t0+dt, ...
    const int ncell = nx1 + 2;
    auto recon = [&](int n, int c) {
      const R *qn = q + n * nc1;
      R wl_, wr_;
      if constexpr (RECON == CANOE_RECON_PPM)
        ppm_cell(qn[c - 2], qn[c - 1], qn[c], qn[c + 1], qn[c + 2], wl_, wr_);
      else
        plm_cell_nu(qn[c - 1], qn[c], qn[c + 1], R(g.x1v[c - 1]), R(g.x1v[c]),
                    R(g.x1v[c + 1]), R(g.x1f[c]), R(g.x1f[c + 1]), wl_, wr_);
      WL[n * nc1 + c] = wl_;
      WR[n * nc1 + c] = wr_;
    };
    // P1 (the scan) overlapped with P2 of the variables other than rho, p
    if (grav != 0.) {
      R *rho = q, *pre = q + S::IPR * nc1;
      const double *rho0 = wp, *pre0 = wp + S::IPR * nc1;
      if (warp == 0) {
        if (lane == 0) {
          const double *dx = psv, *gr = gam;
          double RdTv = pre0[ie] / rho0[ie];
          double acc = pre0[ie] * exp(grav * dx[ie] / (2 * RdTv));
          psf[ie + 1] = acc;
          // psf(i) = psf(i+1) - grav rho(i) dx(i), from the top, in the
          // reference's order.  Chunks of 8 levels: the operands of the next
          // chunk are loaded before this chunk's results are stored.
          int i = ie;
          if (i - 7 >= is) {
            double x[8], d[8];
#pragma unroll
            for (int t = 0; t < 8; ++t) {
              x[t] = gr[i - t];
              d[t] = dx[i - t];
            }
            for (;;) {
              double pn[8];
#pragma unroll
              for (int t = 0; t < 8; ++t) {
                acc = acc - x[t] * d[t];
                pn[t] = acc;
              }
              const int inext = i - 8;
              const bool more = inext - 7 >= is;
              if (more) {
#pragma unroll
                for (int t = 0; t < 8; ++t) {
                  x[t] = gr[inext - t];
                  d[t] = dx[inext - t];
                }
              }
#pragma unroll
              for (int t = 0; t < 8; ++t) psf[i - t] = pn[t];
              i = inext;
              if (!more) break;
            }
          }
          for (; i >= is; --i) {
            acc = acc - gr[i] * dx[i];
            psf[i] = acc;
          }
          const double gb = g.bc[0] == CANOE_BC_REFLECT ? -grav : grav;
          for (int i = is - 1; i >= is - NG; --i) {
            acc = acc - gb * rho0[i] * dx[i];
            psf[i] = acc;
          }
          const double gt = g.bc[1] == CANOE_BC_REFLECT ? -grav : grav;
          double p = psf[ie + 1];
          for (int i = ie + 1; i <= ie + NG; ++i) {
            p = p + gt * rho0[i] * dx[i];
            psf[i + 1] = p;
          }
        }
      } else {
        for (int t = tid - 32; t < (NV - 2) * ncell; t += nth - 32) {
          recon(t / ncell + 1, is - 1 + t % ncell);  // slots 1 .. NV-2
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
        // outflow ghosts take the transformed values of the first / last
        // interior cell (change_to_temperature.cpp:114-127)
        const bool ob = (i < is && g.bc[0] == CANOE_BC_OUTFLOW);
        const bool ot = (i > ie && g.bc[1] == CANOE_BC_OUTFLOW);
        if (!ob && !ot) {
          rho[i] = R(pre0[i] / (rho0[i] * gm));
          pre[i] = R(pre0[i] - pv);
        }
      }
      __syncthreads();
      if (g.bc[0] == CANOE_BC_OUTFLOW || g.bc[1] == CANOE_BC_OUTFLOW) {
        for (int i = tid; i < nc1; i += nth) {
          const bool ob = (i < is && g.bc[0] == CANOE_BC_OUTFLOW);
          const bool ot = (i > ie && g.bc[1] == CANOE_BC_OUTFLOW);
          if (ob || ot) {
            const int c = ob ? is : ie;
            rho[i] = rho[c];
            pre[i] = pre[c];
          }
        }
        __syncthreads();
      }
      for (int t = tid; t < 2 * ncell; t += nth)
        recon(t < ncell ? 0 : S::IPR, is - 1 + t % ncell);
    } else {
      for (int t = tid; t < NV * ncell; t += nth) recon(t / ncell, is - 1 + t % ncell);
    }
    __syncthreads();
    // P3 (F aliases q, which nobody reads after P2).  prep: the face states
    // restored from the decomposition; solve: the Riemann flux; emit: F
    auto prep = [&](int f, R *wl, R *wr) -> double {
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
      return pf;
    };
    auto solve = [&](R *wl, R *wr, double pf, R *fx) {
      if constexpr (GEO) {
        if constexpr (PERT)
          hllc_pert<R, NY, 0, true>(th, wl, wr, R(pf), fx, R(tab(kTabCosC, k, j)));
        else
          hllc<R, NY, 0, true>(th, wl, wr, fx, R(tab(kTabCosC, k, j)));
        const R cth = R(tab(kTabCth1, k, j));
        const R ty = fx[S::IVY], tz = fx[S::IVZ];
        fx[S::IVY] = ty + tz * cth;
        fx[S::IVZ] = tz + ty * cth;
      } else if constexpr (PERT) {
        riemann_pert<R, NY, RS, 0>(th, wl, wr, R(pf), fx);
      } else {
        riemann<R, NY, RS, 0>(th, wl, wr, fx);
      }
    };
    auto emit = [&](int f, const R *fx, double pf) {
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
    };
    for (int f = is + tid; f <= ie + 1; f += nth) {
      R wl[NV], wr[NV], fx[NV];
      const double pf = prep(f, wl, wr);
      solve(wl, wr, pf, fx);
      emit(f, fx, pf);
    }
    if (bulk && load_du) {
      if (!__syncthreads_and(mbar_wait(mbar + 1, 0))) {
        bail(1, 2);
        return;
      }
    } else {
      __syncthreads();
    }
    // P4
    for (int i = is + tid; i <= ie; i += nth) {
      const int f0 = i - is;
      const double idx = 1. / g.dx1f[i];
      // constant x1 acceleration (HydroSourceTerms::ConstantAcceleration
      // with canoe patches/25.constant_acc.patch:35-52): src = dt rho g on
      // the x1 momentum, src v1 on the energy
      const double gsrc = wght * wp[i] * grav;
      // GEO: radial face areas, cell volume and coordinate sources
      double a1m = 0., a1p = 0., vol = 1., csrc[3] = {0., 0., 0.};
      if constexpr (GEO) {
        const double d2 = tab(kTabDx2A, k, j), d3 = tab(kTabDx3A, k, j);
        const double sc = tab(kTabSinC, k, j), cc = tab(kTabCosC, k, j);
        const double xv = g.x1v[i], df = g.dx1f[i];
        a1m = d2 * d3 * g.x1f[i] * g.x1f[i] * sc;
        a1p = d2 * d3 * g.x1f[i + 1] * g.x1f[i + 1] * sc;
        vol = df * d2 * d3 * xv * xv * sc;
        const double a2m = xv * tab(kTabDx3AF2, k, j) * df;
        const double a2p = xv * tab(kTabDx3AF2, k, j + 1) * df;
        const double a3m = xv * tab(kTabDx2AF3, k, j) * df;
        const double a3p = xv * tab(kTabDx2AF3, k + 1, j) * df;
        const double v1 = wp[S::IVX * nc1 + i], v2 = wp[S::IVY * nc1 + i],
                     v3 = wp[S::IVZ * nc1 + i];
        const double pr = wp[S::IPR * nc1 + i], rho = wp[i];
        const double v_2 = v2 + v3 * cc, v_3 = v3 + v2 * cc, sine2 = sc * sc;
        const double x_ov_rD = (a2m * tab(kTabSinF2, k, j) - a2p * tab(kTabSinF2, k, j + 1)) / vol;
        const double y_ov_rC = (a3m * tab(kTabSinF3, k, j) - a3p * tab(kTabSinF3, k + 1, j)) / vol;
        csrc[0] = wght * ((2.0 * pr + rho * (v2 * v_2 + v3 * v_3)) / xv);
        csrc[1] = wght * (-x_ov_rD * (pr + rho * v3 * v3 * sine2) - rho * v1 * v_2 / xv);
        csrc[2] = wght * (-y_ov_rC * (pr + rho * v2 * v2 * sine2) - rho * v1 * v_3 / xv);
      }
#pragma unroll
      for (int n = 0; n < NV; ++n) {
        double v;
        if constexpr (GEO) {
          double dfl = a1p * (double)F[n * (nx1 + 1) + f0 + 1] -
                       a1m * (double)F[n * (nx1 + 1) + f0];
          // FP32 path: the momentum flux lacks psf, whose divergence is FP64
          if (PERT && n == S::IVX && grav != 0.) dfl += a1p * psf[i + 1] - a1m * psf[i];
          v = -(wght * dfl / vol);
          if (n == S::IVX) v += csrc[0];
          if (n == S::IVY) v += csrc[1];
          if (n == S::IVZ) v += csrc[2];
        } else {
          double d = ((double)F[n * (nx1 + 1) + f0 + 1] - (double)F[n * (nx1 + 1) + f0]) * idx;
          // FP32 path: the momentum flux lacks psf, whose divergence is FP64
          if (PERT && n == S::IVX && grav != 0.) d += (psf[i + 1] - psf[i]) * idx;
          v = -(wght * d);
        }
        if (n == S::IVX) v += gsrc;
        if (n == S::IPR) v += gsrc * wp[S::IVX * nc1 + i];
        if constexpr (MODE == kColFluxOnly) {
          du[n * g.sv + base + i] = v;
        } else {
          const double prev = g.f2 ? dc[n * nc1 + i] : 0.;
          dc[n * nc1 + i] = prev + v;
        }
      }
    }
    if constexpr (MODE == kColFluxOnly) return;
  } else if (bulk) {
    if (!__syncthreads_and(mbar_wait(mbar + 1, 0))) {
      bail(1, 2);
      return;
    }
  }
  __syncthreads();

  if constexpr (N > 0) {
    constexpr int NN = ColRow<N>::NN, ROW = ColRow<N>::ROW;
    double *blk = un;                        // [nx1][ROW] + r / 16 padding
    auto RP = [&](int r) { return blk + r * ROW + (r >> 4); };  // row r
    double *sA = sm + L.stg;                 // [nx1+1][NN] |A| at faces is-1/2..ie+1/2
    double *sJ = sA + (nx1 + 1) * NN;        // [nx1+2][NN] J of cells is-1..ie+1
    // COMPACT (row-parallel 5x5): |A| at face t < nx1 sits in row t's c
    // slot, J of cell is-1+t < nx1 in row t's b slot, the last three blocks
    // at stg
    constexpr bool COMPACT = ColPlan<N, PER, GEO>::compact;
    auto pA = [&](int t) -> double * {
      if constexpr (COMPACT) return t < nx1 ? RP(t) + 2 * NN : sA;
      else return sA + t * NN;
    };
    auto pJ = [&](int t) -> double * {
      if constexpr (COMPACT) return t < nx1 ? RP(t) + NN : sA + (t - nx1 + 1) * NN;
      else return sJ + t * NN;
    };
    const double gm1 = th.gammad - 1.;
    const double dt = wght;
    const double idt = 1. / dt;
    const double area = g.dx2 * g.dx3;
    // GEO: the velocities of the solve are projected to the local frame
    double pcos = 0., psin = 1.;
    if constexpr (GEO) {
      pcos = tab(kTabCosC, k, j);
      psin = tab(kTabSinC, k, j);
    }
    // P5a: |A| at face t (between cells is-1+t and is+t) and J of cell is-1+t
    auto cell_state = [&](int ic, double *v) {
#pragma unroll
      for (int n = 0; n < NV; ++n) v[n] = wp[n * nc1 + ic];
      if constexpr (GEO) {
        v[S::IVY] += v[S::IVZ] * pcos;
        v[S::IVZ] *= psin;
      }
    };
    auto put_m = [&](double *p, const M<N> &m) {
#pragma unroll
      for (int e = 0; e < NN; ++e) p[e] = m.a[e / N][e % N];
    };
    for (int t = tid; t < nx1 + 2; t += nth) {
      double wl[NV], wr[NV];
      cell_state(is - 1 + t, wl);
      M<N> J;
      jacobian<N, NY, R>(J, gm1, wl);
      put_m(pJ(t), J);
      if (t <= nx1) {
        cell_state(is + t, wr);
        M<N> A;
        abs_jacobian<N, NY, R>(A, th, gm1, wl, wr);
        put_m(pA(t), A);
      }
    }
    __syncthreads();
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
    // P5b: block rows (partial_correction.cpp:128-154); b of the first and c
    // of the last row couple to ghosts: the reflecting condition folds them
    // into a, and the sweep never uses them, so they are zeroed here.  Rows
    // that the first reduction level eliminates (r even) keep a^-1.
    // PER: the reduction covers rows 0..nr-1 = n-2; b of row 0 (the upper
    // corner, coupling to row n-1) and c of row n-2 move into the bordering
    // columns Z, and row n-1 keeps a, b and, in place of c, the lower corner:
    // c of the ghost row is-1 (periodic_forward_backward.hpp:67-72).
    const int nr = PER ? nx1 - 1 : nx1;
    double *zb = sm + L.z;  // PER: [nr][NN]
    // 3x3, not periodic: cyclic reduction over levels s = 1 .. pcr/2 by the
    // whole CTA, then parallel cyclic reduction (Hockney and Jesshope) of the
    // at most 32 surviving rows in warp 0, one row per lane; pcr is the
    // smallest power of two that leaves at most 32 rows.  Rows that a
    // cyclic-reduction level eliminates are stored with a^-1, the rows that
    // reach the parallel reduction with a itself.
    int pcr = 1 << 30;
    if constexpr (N == 3 && !PER) {
      pcr = 1;
      while (nr / pcr > 32) pcr *= 2;
    }
    // face areas and the cell volume's reciprocal doubled, of row r
    auto row_geom = [&](int r, double &aL, double &aR, double &i2v) {
      const int i = is + r;
      aL = area;
      aR = area;
      i2v = 1. / (2. * (g.dx1f[i] * g.dx2 * g.dx3));
      if constexpr (GEO) {  // GetFace1Area / GetCellVolume
        const double d2 = tab(kTabDx2A, k, j), d3 = tab(kTabDx3A, k, j), sc = tab(kTabSinC, k, j);
        aL = d2 * d3 * g.x1f[i] * g.x1f[i] * sc;
        aR = d2 * d3 * g.x1f[i + 1] * g.x1f[i + 1] * sc;
        i2v = 1. / (2. * (g.dx1f[i] * d2 * d3 * g.x1v[i] * g.x1v[i] * sc));
      }
    };
    auto put_rhs = [&](int r) {  // forward_backward.hpp:24-41
      const int i = is + r;
      double r0 = dc[i];
#pragma unroll
      for (int n = 1; n <= NY; ++n) r0 += dc[n * nc1 + i];
      double *rh = RP(r) + 3 * NN;
      rh[0] = r0 / dt;
      rh[1] = dc[S::IVX * nc1 + i] / dt;
      if constexpr (N == 3) {
        rh[2] = dc[S::IPR * nc1 + i] / dt;
      } else {
        rh[2] = dc[S::IVY * nc1 + i] / dt;
        rh[3] = dc[S::IVZ * nc1 + i] / dt;
        rh[4] = dc[S::IPR * nc1 + i] / dt;
      }
    };
    if constexpr (COMPACT) {
      // a and the right-hand side first; b and c overwrite the staged J and
      // |A| one matrix row at a time, after every row has read them
      for (int r = tid; r < nx1; r += nth) {
        const int i = is + r;
        double aL, aR, i2v;
        row_geom(r, aL, aR, i2v);
        const double *Am = pA(r), *Ap = pA(r + 1), *Jm = pJ(r), *Jc = pJ(r + 1), *Jn = pJ(r + 2);
        double *row = RP(r);
        M<N> am;
#pragma unroll
        for (int e = 0; e < NN; ++e) {
          const int rr = e / N, qq = e % N;
          const double phi = ((rr == 1 && qq == 0) || (rr == N - 1 && qq == 1)) ? grav : 0.;
          double a = (Am[e] * aL + Ap[e] * aR + (aR - aL) * Jc[e]) * i2v + (rr == qq ? idt : 0.) - phi;
          if (i == is) {
            const double b = -(Am[e] + Jm[e]) * aL * i2v;
            a += (qq == 1 ? -b : b);
          }
          if (i == ie) {
            const double c = -(Ap[e] - Jn[e]) * aR * i2v;
            a += (qq == 1 ? -c : c);
          }
          if constexpr (N == 5)
            row[e] = a;  // the row-parallel reduction inverts its pivots
          else
            am.a[rr][qq] = a;
        }
        // N = 3: rows that the first level eliminates keep a^-1
        if constexpr (N == 3) stm(row, ((r & 1) == 0 && 1 < nr && pcr > 1) ? inv(am) : am);
        put_rhs(r);
      }
      for (int r0 = 0; r0 < nx1; r0 += nth) {
        const int r = r0 + tid, i = is + r;
        const bool on = r < nx1;
        double aL = 0., aR = 0., i2v = 0.;
        if (on) row_geom(r, aL, aR, i2v);
#pragma unroll
        for (int q = 0; q < N; ++q) {
          double bv[N], cv[N];
          if (on) {
            const double *Am = pA(r) + q * N, *Ap = pA(r + 1) + q * N;
            const double *Jm = pJ(r) + q * N, *Jn = pJ(r + 2) + q * N;
#pragma unroll
            for (int kk = 0; kk < N; ++kk) {
              bv[kk] = i == is ? 0. : -(Am[kk] + Jm[kk]) * aL * i2v;
              cv[kk] = i == ie ? 0. : -(Ap[kk] - Jn[kk]) * aR * i2v;
            }
          }
          __syncthreads();
          if (on) {
            double *row = RP(r);
#pragma unroll
            for (int kk = 0; kk < N; ++kk) {
              row[NN + q * N + kk] = bv[kk];
              row[2 * NN + q * N + kk] = cv[kk];
            }
          }
        }
      }
    }
    if constexpr (!COMPACT) for (int r = tid; r < nx1; r += nth) {
      const int i = is + r;
      double aL, aR, i2v;
      row_geom(r, aL, aR, i2v);
      double *row = RP(r);
      M<N> am;
#pragma unroll
      for (int e = 0; e < NN; ++e) {
        const int rr = e / N, qq = e % N;
        const double Am = sA[r * NN + e], Ap = sA[(r + 1) * NN + e];
        const double Jm = sJ[r * NN + e], Jc = sJ[(r + 1) * NN + e], Jn = sJ[(r + 2) * NN + e];
        double phi;
        if (N == 3) phi = ((rr == 1 && qq == 0) || (rr == 2 && qq == 1)) ? grav : 0.;
        else phi = ((rr == 1 && qq == 0) || (rr == 4 && qq == 1)) ? grav : 0.;
        double a = (Am * aL + Ap * aR + (aR - aL) * Jc) * i2v + (rr == qq ? idt : 0.) - phi;
        const double b = -(Am + Jm) * aL * i2v;
        const double c = -(Ap - Jn) * aR * i2v;
        if constexpr (PER) {
          am.a[rr][qq] = a;
          row[NN + e] = r == 0 ? 0. : b;
          if (r == nx1 - 1) {  // lower corner: c of row is-1
            const double i2g = 1. / (2. * (g.dx1f[is - 1] * g.dx2 * g.dx3));
            row[2 * NN + e] = -(sA[e] - sJ[NN + e]) * area * i2g;
          } else {
            row[2 * NN + e] = r == nr - 1 ? 0. : c;
            zb[r * NN + e] = (r == 0 ? b : 0.) + (r == nr - 1 ? c : 0.);
          }
        } else {
          if (i == is) a += (qq == 1 ? -b : b);
          if (i == ie) a += (qq == 1 ? -c : c);
          am.a[rr][qq] = a;
          row[NN + e] = i == is ? 0. : b;
          row[2 * NN + e] = i == ie ? 0. : c;
        }
      }
      stm(row, ((r & 1) == 0 && 1 < nr && r < nr) ? inv(am) : am);
      put_rhs(r);
    }
    if (bulk) fence_proxy_async();
    __syncthreads();
    // u and u1 travel into the |A| / J area while the reduction runs
    double *su = sA, *su1 = sA + NV * nc1;
    const bool pre_u = bulk && UPDATE && !COMPACT;
    if (pre_u && tid == 0) {
      mbar_expect_tx(mbar + 2, (stage == 0 ? 1 : 2) * NV * row_bytes);
      for (int n = 0; n < NV; ++n) bulk_g2s(su + n * nc1, u + n * g.sv + base, row_bytes, mbar + 2);
      if (stage != 0)
        for (int n = 0; n < NV; ++n)
          bulk_g2s(su1 + n * nc1, u1 + n * g.sv + base, row_bytes, mbar + 2);
    }
    // P6: block cyclic reduction.  Level s updates the rows r = 2s(m+1) - 1
    // from their neighbours r -/+ s, whose a was replaced by a^-1 when they
    // were formed; a surviving row that the next level eliminates stores its
    // new a^-1 right away.  Levels with at most 32 surviving rows run in
    // warp 0 alone.
    auto level = [&](int s, int m) {
      const int r = 2 * s * (m + 1) - 1;
      double *row = RP(r);
      const double *lo = RP(r - s);
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
      M<N> zr;
      if constexpr (PER) {
        zr = ld(zb + r * NN);
        t = mm(al, ld(zb + (r - s) * NN));
#pragma unroll
        for (int e = 0; e < NN; ++e) zr.a[e / N][e % N] += t.a[e / N][e % N];
      }
      if (r + s < nr) {
        const double *hi = RP(r + s);
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
        if constexpr (PER) {
          t = mm(ga, ld(zb + (r + s) * NN));
#pragma unroll
          for (int e = 0; e < NN; ++e) zr.a[e / N][e % N] += t.a[e / N][e % N];
        }
      } else {
#pragma unroll
        for (int e = 0; e < NN; ++e) cn.a[e / N][e % N] = 0.;
      }
      const bool next_elim = (m & 1) == 0 && 4 * s - 1 < nr && 2 * s < pcr;
      stm(row, next_elim ? inv(a) : a);
      stm(row + NN, bn);
      stm(row + 2 * NN, cn);
      stv(row + 3 * NN, rh);
      if constexpr (PER) stm(zb + r * NN, zr);
    };
    auto back = [&](int s, int m) {
      const int r = s - 1 + 2 * s * m;
      double *row = RP(r);
      V<N> rh = ldv(row + 3 * NN);
      M<N> zr;
      if constexpr (PER) zr = ld(zb + r * NN);
      if (r - s >= 0) {
        const M<N> bm = ld(row + NN);
        V<N> t = mv(bm, ldv(RP(r - s) + 3 * NN));
#pragma unroll
        for (int e = 0; e < N; ++e) rh.a[e] -= t.a[e];
        if constexpr (PER) {
          const M<N> tz = mm(bm, ld(zb + (r - s) * NN));
#pragma unroll
          for (int e = 0; e < NN; ++e) zr.a[e / N][e % N] -= tz.a[e / N][e % N];
        }
      }
      if (r + s < nr) {
        const M<N> cm = ld(row + 2 * NN);
        V<N> t = mv(cm, ldv(RP(r + s) + 3 * NN));
#pragma unroll
        for (int e = 0; e < N; ++e) rh.a[e] -= t.a[e];
        if constexpr (PER) {
          const M<N> tz = mm(cm, ld(zb + (r + s) * NN));
#pragma unroll
          for (int e = 0; e < NN; ++e) zr.a[e / N][e % N] -= tz.a[e / N][e % N];
        }
      }
      const M<N> ai = ld(row);
      stv(row + 3 * NN, mv(ai, rh));
      if constexpr (PER) stm(zb + r * NN, mm(ai, zr));
    };
    if constexpr (N == 5 && !PER) {
      // row-parallel reduction: an 8-lane segment per block row-op, lane
      // g < 5 owning row g of the 5x5 blocks (blockmat.cuh inv5_rows); the
      // neighbours' blocks are read as shared-memory broadcasts
      const int seg = tid >> 3, nseg = nth >> 3, g = tid & 7, gg = g < 5 ? g : 0;
      const unsigned smask = 0xFFu << (tid & 24);
      // the block of row r: its a replaced by a^-1 in place
      auto invert_row = [&](int r) {
        double *row = RP(r);
        double ar[5], iv[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) ar[q] = row[gg * 5 + q];
        const int c = inv5_rows(ar, iv, g, smask);
        if (g < 5 && c >= 0)
#pragma unroll
          for (int q = 0; q < 5; ++q) row[c * 5 + q] = iv[q];
      };
      auto level5 = [&](int s, int m) {
        const int r = 2 * s * (m + 1) - 1;
        double *row = RP(r);
        const double *lo = RP(r - s);
        double ar[5], br[5], cr[5], al[5], bn[5], cn[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) {
          ar[q] = row[gg * 5 + q];
          br[q] = row[NN + gg * 5 + q];
          cr[q] = row[2 * NN + gg * 5 + q];
        }
        double rh = row[3 * NN + gg];
        // alpha = -b a_lo^-1
#pragma unroll
        for (int q = 0; q < 5; ++q) {
          double t = 0.;
#pragma unroll
          for (int k = 0; k < 5; ++k) t += br[k] * lo[k * 5 + q];
          al[q] = -t;
        }
#pragma unroll
        for (int q = 0; q < 5; ++q) {
          double t = 0., u = 0.;
#pragma unroll
          for (int k = 0; k < 5; ++k) {
            t += al[k] * lo[2 * NN + k * 5 + q];
            u += al[k] * lo[NN + k * 5 + q];
          }
          ar[q] += t;
          bn[q] = u;
        }
        {
          double t = 0.;
#pragma unroll
          for (int k = 0; k < 5; ++k) t += al[k] * lo[3 * NN + k];
          rh += t;
        }
        if (r + s < nr) {
          const double *hi = RP(r + s);
          double ga[5];
#pragma unroll
          for (int q = 0; q < 5; ++q) {
            double t = 0.;
#pragma unroll
            for (int k = 0; k < 5; ++k) t += cr[k] * hi[k * 5 + q];
            ga[q] = -t;
          }
#pragma unroll
          for (int q = 0; q < 5; ++q) {
            double t = 0., u = 0.;
#pragma unroll
            for (int k = 0; k < 5; ++k) {
              t += ga[k] * hi[NN + k * 5 + q];
              u += ga[k] * hi[2 * NN + k * 5 + q];
            }
            ar[q] += t;
            cn[q] = u;
          }
          double t = 0.;
#pragma unroll
          for (int k = 0; k < 5; ++k) t += ga[k] * hi[3 * NN + k];
          rh += t;
        } else {
#pragma unroll
          for (int q = 0; q < 5; ++q) cn[q] = 0.;
        }
        // every lane has read row r before any writes it (the shuffles of
        // the inverse and the data dependence order them)
        const bool next_elim = (m & 1) == 0 && 4 * s - 1 < nr;
        if (next_elim) {
          double iv[5];
          const int c = inv5_rows(ar, iv, g, smask);
          if (g < 5 && c >= 0)
#pragma unroll
            for (int q = 0; q < 5; ++q) row[c * 5 + q] = iv[q];
        } else if (g < 5) {
#pragma unroll
          for (int q = 0; q < 5; ++q) row[g * 5 + q] = ar[q];
        }
        if (g < 5) {
#pragma unroll
          for (int q = 0; q < 5; ++q) {
            row[NN + g * 5 + q] = bn[q];
            row[2 * NN + g * 5 + q] = cn[q];
          }
          row[3 * NN + g] = rh;
        }
      };
      auto back5 = [&](int s, int m) {
        const int r = s - 1 + 2 * s * m;
        double *row = RP(r);
        double t = row[3 * NN + gg];
        if (r - s >= 0) {
          const double *x = RP(r - s) + 3 * NN;
          double u = 0.;
#pragma unroll
          for (int k = 0; k < 5; ++k) u += row[NN + gg * 5 + k] * x[k];
          t -= u;
        }
        if (r + s < nr) {
          const double *x = RP(r + s) + 3 * NN;
          double u = 0.;
#pragma unroll
          for (int k = 0; k < 5; ++k) u += row[2 * NN + gg * 5 + k] * x[k];
          t -= u;
        }
        double xr = 0.;
#pragma unroll
        for (int k = 0; k < 5; ++k) xr += row[gg * 5 + k] * __shfl_sync(smask, t, k, 8);
        if (g < 5) row[3 * NN + g] = xr;
      };
      int stop = 1;  // first s with 2 s - 1 >= nr
      while (2 * stop - 1 < nr) stop *= 2;
      if (1 < nr)
        for (int m = seg; 2 * m < nr; m += nseg) invert_row(2 * m);
      __syncthreads();
      for (int s = 1; s < stop; s *= 2) {
        for (int m = seg; m < nr / (2 * s); m += nseg) level5(s, m);
        __syncthreads();
      }
      // the last surviving row r = stop - 1 is decoupled
      if (seg == 0) {
        double *row = RP(stop - 1);
        double ar[5], iv[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) ar[q] = row[gg * 5 + q];
        const double rr = row[3 * NN + gg];
        const int c = inv5_rows(ar, iv, g, smask);
        double x = 0.;
#pragma unroll
        for (int k = 0; k < 5; ++k) x += iv[k] * __shfl_sync(smask, rr, k, 8);
        if (g < 5 && c >= 0) row[3 * NN + c] = x;
      }
      __syncthreads();
      for (int s = stop / 2; s >= 1; s /= 2) {
        for (int m = seg; m < (nr + s) / (2 * s); m += nseg) back5(s, m);
        __syncthreads();
      }
    } else if constexpr (N == 3 && !PER) {
      for (int s = 1; s < pcr; s *= 2) {
        for (int m = tid; m < nr / (2 * s); m += nth) level(s, m);
        __syncthreads();
      }
      // the surviving rows r = pcr (q + 1) - 1, q < nq, form a block
      // tridiagonal system of their own; each parallel-reduction level with
      // stride d couples row q to q -/+ 2d, and after the last one every row
      // is decoupled
      if (warp == 0) {
        const int nq = nr / pcr;
        const bool act = lane < nq;
        double *row = RP(act ? pcr * (lane + 1) - 1 : 0);
        auto qrow = [&](int q) { return RP(pcr * (q + 1) - 1); };
        for (int d = 1; d < nq; d *= 2) {
          M<N> a;
          if (act) {
            a = ld(row);
            stm(row, inv(a));  // neighbours read a^-1, b, c and rhs
          }
          __syncwarp();
          M<N> an, bn, cn;
          V<N> rn;
          if (act) {
            an = a;
            rn = ldv(row + 3 * NN);
            if (lane - d >= 0) {
              const double *lo = qrow(lane - d);
              M<N> al = mm(ld(row + NN), ld(lo));
#pragma unroll
              for (int e = 0; e < NN; ++e) al.a[e / N][e % N] = -al.a[e / N][e % N];
              const M<N> t = mm(al, ld(lo + 2 * NN));
              const V<N> tv = mv(al, ldv(lo + 3 * NN));
#pragma unroll
              for (int e = 0; e < NN; ++e) an.a[e / N][e % N] += t.a[e / N][e % N];
#pragma unroll
              for (int e = 0; e < N; ++e) rn.a[e] += tv.a[e];
              bn = mm(al, ld(lo + NN));
            } else {
#pragma unroll
              for (int e = 0; e < NN; ++e) bn.a[e / N][e % N] = 0.;
            }
            if (lane + d < nq) {
              const double *hi = qrow(lane + d);
              M<N> ga = mm(ld(row + 2 * NN), ld(hi));
#pragma unroll
              for (int e = 0; e < NN; ++e) ga.a[e / N][e % N] = -ga.a[e / N][e % N];
              const M<N> t = mm(ga, ld(hi + NN));
              const V<N> tv = mv(ga, ldv(hi + 3 * NN));
#pragma unroll
              for (int e = 0; e < NN; ++e) an.a[e / N][e % N] += t.a[e / N][e % N];
#pragma unroll
              for (int e = 0; e < N; ++e) rn.a[e] += tv.a[e];
              cn = mm(ga, ld(hi + 2 * NN));
            } else {
#pragma unroll
              for (int e = 0; e < NN; ++e) cn.a[e / N][e % N] = 0.;
            }
          }
          __syncwarp();  // every lane has read its neighbours' rows
          if (act) {
            stm(row, an);
            stm(row + NN, bn);
            stm(row + 2 * NN, cn);
            stv(row + 3 * NN, rn);
          }
          __syncwarp();
        }
        if (act) stv(row + 3 * NN, mv(inv(ld(row)), ldv(row + 3 * NN)));
      }
      __syncthreads();
      for (int s = pcr / 2; s >= 1; s /= 2) {
        for (int m = tid; m < (nr + s) / (2 * s); m += nth) back(s, m);
        __syncthreads();
      }
    } else {
      int stop = 1;  // first s with 2 s - 1 >= nr
      while (2 * stop - 1 < nr) stop *= 2;
      int s = 1;
      for (; s < stop && nr / (2 * s) > 32; s *= 2) {
        for (int m = tid; m < nr / (2 * s); m += nth) level(s, m);
        __syncthreads();
      }
      const int s_warp = s;  // first level done by warp 0
      // first back level done by all threads: the largest s with > 32 rows
      int sb = 1;
      while (2 * sb < stop && (nr + 2 * sb) / (4 * sb) > 32) sb *= 2;
      if ((nr + sb) / (2 * sb) <= 32) sb = 0;  // every back level fits in warp 0
      if (warp == 0) {
        for (s = s_warp; s < stop; s *= 2) {
          for (int m = lane; m < nr / (2 * s); m += 32) level(s, m);
          __syncwarp();
        }
        // the last surviving row r = stop - 1 is decoupled
        if (lane == 0) {
          double *row = RP(stop - 1);
          M<N> ai = inv(ld(row));
          stm(row, ai);
          stv(row + 3 * NN, mv(ai, ldv(row + 3 * NN)));
          if constexpr (PER) stm(zb + (stop - 1) * NN, mm(ai, ld(zb + (stop - 1) * NN)));
        }
        __syncwarp();
        for (s = stop / 2; s >= 1 && s > sb; s /= 2) {
          for (int m = lane; m < (nr + s) / (2 * s); m += 32) back(s, m);
          __syncwarp();
        }
      }
      __syncthreads();
      for (s = sb; s >= 1; s /= 2) {
        for (int m = tid; m < (nr + s) / (2 * s); m += nth) back(s, m);
        __syncthreads();
      }
    }
    if constexpr (PER) {
      // rows 0..n-2 hold y and Z with x = y - Z x(n-1); row n-1:
      // (a - s Z0 - b Z(n-2)) x(n-1) = rhs - s y0 - b y(n-2)
      if (tid == 0) {
        double *row = RP(nx1 - 1);
        const M<N> bl = ld(row + NN), sc = ld(row + 2 * NN);
        M<N> sch = ld(row);
        V<N> rh = ldv(row + 3 * NN);
        const M<N> t0 = mm(sc, ld(zb)), t1 = mm(bl, ld(zb + (nr - 1) * NN));
        const V<N> v0 = mv(sc, ldv(RP(0) + 3 * NN)), v1 = mv(bl, ldv(RP(nr - 1) + 3 * NN));
#pragma unroll
        for (int e = 0; e < NN; ++e) sch.a[e / N][e % N] -= t0.a[e / N][e % N] + t1.a[e / N][e % N];
#pragma unroll
        for (int e = 0; e < N; ++e) rh.a[e] -= v0.a[e] + v1.a[e];
        stv(row + 3 * NN, mv(inv(sch), rh));
      }
      __syncthreads();
      const V<N> xl = ldv(RP(nx1 - 1) + 3 * NN);
      for (int r = tid; r < nr; r += nth) {
        double *x = RP(r) + 3 * NN;
        const V<N> t = mv(ld(zb + r * NN), xl);
#pragma unroll
        for (int e = 0; e < N; ++e) x[e] -= t.a[e];
      }
      __syncthreads();
    }
    // P7a: species correction (forward_backward.hpp:101-124) into dc
    for (int r = tid; r < nx1; r += nth) {
      const double *x = RP(r) + 3 * NN;
      const int i = is + r;
      double dv[NV];
#pragma unroll
      for (int n = 0; n < NV; ++n) dv[n] = dc[n * nc1 + i];
      double dens = dv[0];
#pragma unroll
      for (int n = 1; n <= NY; ++n) dens += dv[n];
      dens = x[0] - dens;
      dv[0] = x[0];
      if constexpr (!PER) {  // the periodic update leaves du_n as it is
#pragma unroll
        for (int n = 1; n <= NY; ++n) dv[n] += dens * wp[n * nc1 + i];
      }
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
      for (int n = 0; n < NV; ++n) dc[n * nc1 + i] = dv[n];
    }
    if (pre_u) {
      if (!__syncthreads_and(mbar_wait(mbar + 2, 0))) {
        bail(2, 3);
        return;
      }
    } else {
      __syncthreads();
    }
    if constexpr (UPDATE) {
      if (pre_u) {
        for (int n = 0; n < NV; ++n)
          for (int i = is + tid; i <= ie; i += nth) {
            const int64_t x = n * g.sv + base + i;
            const double uo = su[n * nc1 + i];
            double ur;
            if (stage == 0) {
              u1[x] = uo;
              ur = uo;
            } else {
              ur = su1[n * nc1 + i];
            }
            const double t = st.g1 * uo + st.g2 * ur;
            u[x] = t + dc[n * nc1 + i];
          }
        return;
      }
    }
  }

  // P7b: write back.  A cell's NV values of u (and u1) are all loaded before
  // any store, so that the loads are in flight together (stores to u could
  // otherwise alias the next variable's load as far as the compiler knows)
  if constexpr (!UPDATE) {
    for (int n = 0; n < NV; ++n)
      for (int i = is + tid; i <= ie; i += nth) du[n * g.sv + base + i] = dc[n * nc1 + i];
  } else {
    for (int i = is + tid; i <= ie; i += nth) {
      double uo[NV], ur[NV];
#pragma unroll
      for (int n = 0; n < NV; ++n) uo[n] = u[n * g.sv + base + i];
      if (stage != 0) {
#pragma unroll
        for (int n = 0; n < NV; ++n) ur[n] = u1[n * g.sv + base + i];
      } else {
#pragma unroll
        for (int n = 0; n < NV; ++n) {
          ur[n] = uo[n];
          u1[n * g.sv + base + i] = uo[n];
        }
      }
#pragma unroll
      for (int n = 0; n < NV; ++n) {
        const double t = st.g1 * uo[n] + st.g2 * ur[n];
        u[n * g.sv + base + i] = t + dc[n * nc1 + i];
      }
    }
  }
}

// launch shape of one x1 pencil launch: shared memory, grid, threads, and
// whether the rows can travel by bulk copies
struct ColLaunch {
  Geom g;
  size_t smem;
  unsigned nblk;
  int nthr;
};

inline int col_prepare(const Geom &g, int nv, int nimpl, bool per, const double *w,
                       const double *du, const double *u, const double *u1, ColLaunch &cl) {
  const int compact =
      !per && (nimpl == 5 || (nimpl == 3 && kCompact3)) ? 1 : 0;
  const ColSmem L = col_smem(nv, g.nc1, g.nx1, nimpl, per ? 1 : 0, compact);
  cl.smem = sizeof(double) * (size_t)L.total;
  if (cl.smem > 227 * 1024) {
    set_error("x1 pencil too long for shared memory");
    return CANOE_ERR_UNSUPPORTED;
  }
  cl.nblk = (unsigned)g.nx2 * (unsigned)g.nx3 * (unsigned)(g.npanel > 1 ? g.npanel : 1);
  // threads per pencil: the kernel strides every loop by blockDim and needs
  // at least two warps (warp 0 runs the scan while the others reconstruct)
  cl.nthr = (g.col_threads >= 64 && g.col_threads <= kColThreads && g.col_threads % 32 == 0)
                ? g.col_threads
                : kColThreads;
  // compact 3x3 default: one thread per level rounded up to a warp, between
  // 2 and 4 warps.  Short columns need little shared memory, so the register
  // file sets the pencils per SM: at 64 levels eight pencils of 2 warps run
  // where four of 4 warps would
  if (compact)
    cl.nthr = nimpl == 5 ? kCol5Threads
                         : (g.col_threads >= 64 && g.col_threads <= kCol3ThreadsMax &&
                            g.col_threads % 32 == 0)
                               ? g.col_threads
                               : min(max((g.nx1 + 31) / 32 * 32, 64), kCol3Threads);
  // bulk copies move whole pencil rows: 16-byte aligned bases and an even
  // row length keep every row 16-byte aligned
  auto al16 = [](const void *p) { return p == nullptr || ((uintptr_t)p & 15) == 0; };
  cl.g = g;
  cl.g.bulk = (g.nc1 % 2 == 0) && al16(w) && al16(du) && al16(u) && al16(u1) ? 1 : 0;
  return 0;
}

template <class K>
int col_go(K kern, const ColLaunch &cl, const canoe_thermo_t &th, const double *w, double *du,
           double *u, double *u1, const double *dtp, const Stage &s, int stage, double *fout,
           cudaStream_t st) {
  if (int rc = ensure_smem((const void *)kern, cl.smem)) return rc;
  kern<<<cl.nblk, cl.nthr, cl.smem, st>>>(cl.g, th, w, du, u, u1, dtp, s, stage, fout);
  CB_CUDA(cudaGetLastError());
  return 0;
}

// implicit modes with periodic x1 at both ends; instantiated in
// column_per_ny*.cu (column_per.cuh)
template <int NY, typename R>
int run_x1col_per(const Geom &g, const canoe_thermo_t &th, int recon, int rs, int flag,
                  int mode, const double *w, double *du, double *u, double *u1,
                  const double *dtp, const Stage &s, int stage, double *fout,
                  cudaStream_t st);

// launcher for one NY (instantiated in column_ny*.cu)
template <int NY, typename R>
int run_x1col_p(const Geom &g, const canoe_thermo_t &th, int recon, int rs, int flag,
                int mode, const double *w, double *du, double *u, double *u1,
                const double *dtp, const Stage &s, int stage, double *fout,
                cudaStream_t st) {
  const int nimpl =
      (mode == kColFluxOnly || mode == kColDivOnly || !(flag & 1)) ? 0 : ((flag & 8) ? 5 : 3);
  if (mode == kColSolveOnly && nimpl == 0) return 0;
  if (nimpl && g.bc[0] == CANOE_BC_PERIODIC)
    return run_x1col_per<NY, R>(g, th, recon, rs, flag, mode, w, du, u, u1, dtp, s, stage,
                                fout, st);
  ColLaunch cl;
  if (int rc = col_prepare(g, 5 + NY, nimpl, false, w, du, u, u1, cl)) return rc;
  auto go = [&](auto kern) -> int {
    return col_go(kern, cl, th, w, du, u, u1, dtp, s, stage, fout, st);
  };
  const bool ppm = recon == CANOE_RECON_PPM, hllc = rs == CANOE_RSOLVER_HLLC;
  if (g.shell) {  // cubed-sphere panel: dry, FP64, HLLC
    if constexpr (NY == 0) {
      if (!hllc) {
        set_error("the cubed-sphere panel uses the HLLC solver");
        return CANOE_ERR_UNSUPPORTED;
      }
#define CB_GCOL(NIMPL, MODE) \
  (ppm ? go(k_x1col<NY, 3, 1, NIMPL, MODE, R, 1>) : go(k_x1col<NY, 2, 1, NIMPL, MODE, R, 1>))
      if (mode == kColFluxOnly) return CB_GCOL(0, kColFluxOnly);
      if (mode != kColStep) {
        set_error("only the fused stage is provided on a cubed-sphere panel");
        return CANOE_ERR_UNSUPPORTED;
      }
      if (nimpl == 0) return CB_GCOL(0, kColStep);
      if (nimpl == 3) return CB_GCOL(3, kColStep);
      return CB_GCOL(5, kColStep);
#undef CB_GCOL
    } else {
      set_error("the cubed-sphere panel is dry");
      return CANOE_ERR_UNSUPPORTED;
    }
  }
#define CB_COL(NIMPL, MODE)                                                        \
  (ppm ? (hllc ? go(k_x1col<NY, 3, 1, NIMPL, MODE, R>) : go(k_x1col<NY, 3, 0, NIMPL, MODE, R>)) \
       : (hllc ? go(k_x1col<NY, 2, 1, NIMPL, MODE, R>) : go(k_x1col<NY, 2, 0, NIMPL, MODE, R>)))
  if (mode == kColFluxOnly) return CB_COL(0, kColFluxOnly);
  if (mode == kColDivOnly) return CB_COL(0, kColDivOnly);
  if (mode == kColSolveOnly)
    return nimpl == 3 ? go(k_x1col<NY, 3, 1, 3, kColSolveOnly, double>)
                      : go(k_x1col<NY, 3, 1, 5, kColSolveOnly, double>);
  if (mode == kColSolveStep)
    return nimpl == 0   ? go(k_x1col<NY, 3, 1, 0, kColSolveStep, double>)
           : nimpl == 3 ? go(k_x1col<NY, 3, 1, 3, kColSolveStep, double>)
                        : go(k_x1col<NY, 3, 1, 5, kColSolveStep, double>);
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
  if (prec == CANOE_FP32_PERTURBATION && mode != kColSolveOnly && mode != kColSolveStep)
    return run_x1col_p<NY, float>(g, th, recon, rs, flag, mode, w, du, u, u1, dtp, s, stage,
                                  fout, st);
  return run_x1col_p<NY, double>(g, th, recon, rs, flag, mode, w, du, u, u1, dtp, s, stage,
                                 fout, st);
}

}  // namespace cb
