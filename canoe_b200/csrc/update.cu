// update.cu -- the RK register update of ImplicitHydroTasks (IntegrateHydro,
// src/tasklist/implicit_hydro_tasks.cpp:134-190, and ImplicitCorrection,
// :267-288) fused with the implicit vertical solve
// (ImplicitSolver::SolveImplicit3D, src/snap/implicit/solve_implicit_3d.cpp:
// 91-142, X1 direction).
//
// k_update_explicit: u = g1 u + g2 u1 + du per interior cell.
// k_column<N>:       one thread per vertical column.  The block-tridiagonal
//   coefficients (PartialCorrection, partial_correction.cpp:26-170, N = 3;
//   FullCorrection, full_correction.cpp:32-161, N = 5) are built level by
//   level from a rolling register window (Roe-averaged |A| at the lower and
//   upper faces, flux Jacobians of the three cells) and eliminated at once
//   (ForwardSweep, forward_backward.hpp:15-85), so a, b, c are never stored;
//   only the eliminated (a^-1 c, delta) pairs go to a scratch laid out
//   [level][element][column] so that neighbouring threads write neighbouring
//   words.  The backward substitution (forward_backward.hpp:87-137) reads them
//   back top-down and writes either the corrected du or, fused, the new u.
#include <cuda_runtime.h>

#include "block.cuh"

namespace cb {

namespace {

template <int N>
struct M {
  double a[N][N];
};
template <int N>
struct V {
  double a[N];
};

template <int N>
__device__ __forceinline__ M<N> mm(const M<N> &x, const M<N> &y) {
  M<N> r;
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = 0; j < N; ++j) {
      double s = 0.;
#pragma unroll
      for (int k = 0; k < N; ++k) s += x.a[i][k] * y.a[k][j];
      r.a[i][j] = s;
    }
  return r;
}

template <int N>
__device__ __forceinline__ V<N> mv(const M<N> &x, const V<N> &y) {
  V<N> r;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    double s = 0.;
#pragma unroll
    for (int k = 0; k < N; ++k) s += x.a[i][k] * y.a[k];
    r.a[i] = s;
  }
  return r;
}

__device__ __forceinline__ M<3> inv(const M<3> &m) {
  const double(*a)[3] = m.a;
  double c00 = a[1][1] * a[2][2] - a[1][2] * a[2][1];
  double c01 = a[1][2] * a[2][0] - a[1][0] * a[2][2];
  double c02 = a[1][0] * a[2][1] - a[1][1] * a[2][0];
  double det = a[0][0] * c00 + a[0][1] * c01 + a[0][2] * c02;
  double id = 1. / det;
  M<3> r;
  r.a[0][0] = c00 * id;
  r.a[1][0] = c01 * id;
  r.a[2][0] = c02 * id;
  r.a[0][1] = (a[0][2] * a[2][1] - a[0][1] * a[2][2]) * id;
  r.a[1][1] = (a[0][0] * a[2][2] - a[0][2] * a[2][0]) * id;
  r.a[2][1] = (a[0][1] * a[2][0] - a[0][0] * a[2][1]) * id;
  r.a[0][2] = (a[0][1] * a[1][2] - a[0][2] * a[1][1]) * id;
  r.a[1][2] = (a[0][2] * a[1][0] - a[0][0] * a[1][2]) * id;
  r.a[2][2] = (a[0][0] * a[1][1] - a[0][1] * a[1][0]) * id;
  return r;
}

// Gauss-Jordan with partial pivoting
__device__ __forceinline__ M<5> inv(const M<5> &m) {
  double a[5][10];
#pragma unroll
  for (int i = 0; i < 5; ++i)
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      a[i][j] = m.a[i][j];
      a[i][5 + j] = (i == j) ? 1. : 0.;
    }
#pragma unroll
  for (int c = 0; c < 5; ++c) {
    int p = c;
#pragma unroll
    for (int r = c + 1; r < 5; ++r)
      if (fabs(a[r][c]) > fabs(a[p][c])) p = r;
    if (p != c) {
#pragma unroll
      for (int r = c + 1; r < 5; ++r)
        if (r == p)
#pragma unroll
          for (int j = 0; j < 10; ++j) {
            double t = a[c][j];
            a[c][j] = a[r][j];
            a[r][j] = t;
          }
    }
    double ip = 1. / a[c][c];
#pragma unroll
    for (int j = 0; j < 10; ++j) a[c][j] *= ip;
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      if (r == c) continue;
      double f = a[r][c];
      if (f != 0.)
#pragma unroll
        for (int j = 0; j < 10; ++j) a[r][j] -= f * a[c][j];
    }
  }
  M<5> r;
#pragma unroll
  for (int i = 0; i < 5; ++i)
#pragma unroll
    for (int j = 0; j < 5; ++j) r.a[i][j] = a[i][5 + j];
  return r;
}

// row / column selection of the reduced (partial) system: (rho, m1, E)
template <int N>
__device__ __forceinline__ constexpr int sel(int r) {
  return N == 5 ? r : (r == 2 ? 4 : r);
}

// FluxJacobian (flux_decomposition.hpp:102-120), reduced to N x N
template <int N, int NY>
__device__ __forceinline__ void jacobian(M<N> &d, double gm1, const double *w) {
  using S = Slots<NY>;
  double v1 = w[S::IVX], v2 = w[S::IVY], v3 = w[S::IVZ];
  double rho = w[0], pres = w[S::IPR];
  double s2 = v1 * v1 + v2 * v2 + v3 * v3;
  double c1 = ((gm1 - 1) * s2 / 2 - (gm1 + 1) / gm1 * pres / rho) * v1;
  double c2 = (gm1 + 1) / gm1 * pres / rho + s2 / 2 - gm1 * v1 * v1;
  const double f[5][5] = {{0, 1., 0., 0., 0.},
                          {gm1 * s2 / 2 - v1 * v1, (2. - gm1) * v1, -gm1 * v2, -gm1 * v3, gm1},
                          {-v1 * v2, v2, v1, 0., 0.},
                          {-v1 * v3, v3, 0., v1, 0.},
                          {c1, c2, -gm1 * v2 * v1, -gm1 * v3 * v1, (gm1 + 1) * v1}};
#pragma unroll
  for (int r = 0; r < N; ++r)
#pragma unroll
    for (int c = 0; c < N; ++c) d.a[r][c] = f[sel<N>(r)][sel<N>(c)];
}

// |A| = R |Lambda| R^-1 at the face between cells with primitive states wl,
// wr: RoeAverage (:34-67), SoundSpeed, Eigenvalue (:70-75), Eigenvector
// (:78-99); only the N x N reduced block is formed.
template <int N, int NY>
__device__ __forceinline__ void abs_jacobian(M<N> &A, const canoe_thermo_t &th,
                                             double gm1, const double *wl,
                                             const double *wr) {
  using S = Slots<NY>;
  double prim[S::NV];
  double sqrtdl = sqrt(wl[0]);
  double sqrtdr = sqrt(wr[0]);
  double isdlpdr = 1.0 / (sqrtdl + sqrtdr);
  prim[0] = sqrtdl * sqrtdr;
  prim[S::IVX] = (sqrtdl * wl[S::IVX] + sqrtdr * wr[S::IVX]) * isdlpdr;
  prim[S::IVY] = (sqrtdl * wl[S::IVY] + sqrtdr * wr[S::IVY]) * isdlpdr;
  prim[S::IVZ] = (sqrtdl * wl[S::IVZ] + sqrtdr * wr[S::IVZ]) * isdlpdr;
#pragma unroll
  for (int n = 1; n <= NY; ++n) prim[n] = (sqrtdl * wl[n] + sqrtdr * wr[n]) * isdlpdr;
  double el = wl[S::IPR] / gm1 + 0.5 * wl[0] *
              (wl[S::IVX] * wl[S::IVX] + wl[S::IVY] * wl[S::IVY] + wl[S::IVZ] * wl[S::IVZ]);
  double er = wr[S::IPR] / gm1 + 0.5 * wr[0] *
              (wr[S::IVX] * wr[S::IVX] + wr[S::IVY] * wr[S::IVY] + wr[S::IVZ] * wr[S::IVZ]);
  double hbar = ((el + wl[S::IPR]) / sqrtdl + (er + wr[S::IPR]) / sqrtdr) * isdlpdr;
  prim[S::IPR] = (hbar - 0.5 * (prim[S::IVX] * prim[S::IVX] + prim[S::IVY] * prim[S::IVY] +
                                prim[S::IVZ] * prim[S::IVZ])) *
                 gm1 / (gm1 + 1.) * prim[0];
  double cs = sound_speed<double, NY>(th, prim);
  double r = prim[0], u = prim[S::IVX], v = prim[S::IVY], w = prim[S::IVZ],
         p = prim[S::IPR];
  double ke = 0.5 * (u * u + v * v + w * w);
  double hp = (gm1 + 1.) / gm1 * p / r;
  double h = hp + ke;
  const double R[5][5] = {{1., 1., 1., 0., 0.},
                          {u - cs, u, u + cs, 0., 0.},
                          {v, v, v, 1., 0.},
                          {w, w, w, 0., 1.},
                          {h - u * cs, ke, h + u * cs, v, w}};
  const double Ri[5][5] = {
      {(cs * ke + u * hp) / (2. * cs * hp), (-hp - cs * u) / (2. * cs * hp), -v / (2. * hp),
       -w / (2. * hp), 1. / (2. * hp)},
      {(hp - ke) / hp, u / hp, v / hp, w / hp, -1. / hp},
      {(cs * ke - u * hp) / (2. * cs * hp), (hp - cs * u) / (2. * cs * hp), -v / (2. * hp),
       -w / (2. * hp), 1. / (2. * hp)},
      {-v, 0., 1., 0., 0.},
      {-w, 0., 0., 1., 0.}};
  const double lam[5] = {fabs(u - cs), fabs(u), fabs(u + cs), fabs(u), fabs(u)};
#pragma unroll
  for (int a = 0; a < N; ++a)
#pragma unroll
    for (int b = 0; b < N; ++b) {
      double s = 0.;
#pragma unroll
      for (int k = 0; k < 5; ++k) s += (R[sel<N>(a)][k] * lam[k]) * Ri[k][sel<N>(b)];
      A.a[a][b] = s;
    }
}

template <int NY>
__device__ __forceinline__ void load_w(const Geom &g, const double *__restrict__ w,
                                       int64_t base, int i, double *out) {
#pragma unroll
  for (int n = 0; n < Slots<NY>::NV; ++n) out[n] = w[n * g.sv + base + i];
}

template <int N, int NY, int MODE>
__global__ void __launch_bounds__(128)
    k_column(Geom g, canoe_thermo_t th, const double *__restrict__ w,
             double *__restrict__ du, double *__restrict__ u, double *__restrict__ u1,
             const double *__restrict__ dtp, Stage st, int stage,
             double *__restrict__ scr) {
  using S = Slots<NY>;
  constexpr int NV = S::NV;
  constexpr int NE = N * N + N;  // scratch words per level
  const int ncol = g.nx2 * g.nx3;
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= ncol) return;
  const int j = g.js + col % g.nx2, k = g.ks + col / g.nx2;
  const int64_t base = (int64_t)k * g.sk + (int64_t)j * g.nc1;
  const int is = g.is, ie = g.ie;
  const double dt = st.beta * dtp[0];
  const double gm1 = th.gammad - 1.;
  const double grav = th.grav;
  const double area = g.dx2 * g.dx3;
  const double idt = 1. / dt;

  double wc[NV], wn[NV];
  M<N> Jm, Jc, Jn, Am, Ap, aC;
  V<N> dl;
  // cells is-1 and is
  load_w<NY>(g, w, base, is - 1, wc);
  jacobian<N, NY>(Jm, gm1, wc);
  load_w<NY>(g, w, base, is, wn);
  jacobian<N, NY>(Jc, gm1, wn);
  abs_jacobian<N, NY>(Am, th, gm1, wc, wn);  // face is - 1/2
#pragma unroll
  for (int n = 0; n < NV; ++n) wc[n] = wn[n];

  for (int i = is; i <= ie; ++i) {
    // upper neighbour i+1 (a ghost at i = ie)
    load_w<NY>(g, w, base, i + 1, wn);
    jacobian<N, NY>(Jn, gm1, wn);
    abs_jacobian<N, NY>(Ap, th, gm1, wc, wn);  // face i + 1/2
    const double vol = g.dx1f[i] * g.dx2 * g.dx3;
    M<N> a, b, c;
#pragma unroll
    for (int r = 0; r < N; ++r)
#pragma unroll
      for (int q = 0; q < N; ++q) {
        double phi = 0.;
        if (N == 3) phi = ((r == 1 && q == 0) || (r == 2 && q == 1)) ? grav : 0.;
        else phi = ((r == 1 && q == 0) || (r == 4 && q == 1)) ? grav : 0.;
        a.a[r][q] = (Am.a[r][q] * area + Ap.a[r][q] * area + (area - area) * Jc.a[r][q]) /
                        (2. * vol) +
                    (r == q ? idt : 0.) - phi;
        b.a[r][q] = -(Am.a[r][q] + Jm.a[r][q]) * area / (2. * vol);
        c.a[r][q] = -(Ap.a[r][q] - Jn.a[r][q]) * area / (2. * vol);
      }
    // reflecting ends (partial_correction.cpp:153-154): a += b Bnd, c Bnd,
    // Bnd = diag(1, -1, 1, ...)
    if (i == is) {
#pragma unroll
      for (int r = 0; r < N; ++r)
#pragma unroll
        for (int q = 0; q < N; ++q) a.a[r][q] += (q == 1 ? -b.a[r][q] : b.a[r][q]);
    }
    if (i == ie) {
#pragma unroll
      for (int r = 0; r < N; ++r)
#pragma unroll
        for (int q = 0; q < N; ++q) a.a[r][q] += (q == 1 ? -c.a[r][q] : c.a[r][q]);
    }
    // right-hand side (forward_backward.hpp:24-41)
    V<N> rhs;
    {
      double r0 = du[base + i];
#pragma unroll
      for (int n = 1; n <= NY; ++n) r0 += du[n * g.sv + base + i];
      rhs.a[0] = r0 / dt;
      rhs.a[1] = du[S::IVX * g.sv + base + i] / dt;
      if constexpr (N == 3) {
        rhs.a[2] = du[S::IPR * g.sv + base + i] / dt;
      } else {
        rhs.a[2] = du[S::IVY * g.sv + base + i] / dt;
        rhs.a[3] = du[S::IVZ * g.sv + base + i] / dt;
        rhs.a[4] = du[S::IPR * g.sv + base + i] / dt;
      }
    }
    // forward elimination
    M<N> ai;
    V<N> d;
    if (i == is) {
      ai = inv(a);
      d = mv(ai, rhs);
    } else {
      M<N> t = mm(b, aC);
#pragma unroll
      for (int r = 0; r < N; ++r)
#pragma unroll
        for (int q = 0; q < N; ++q) t.a[r][q] = a.a[r][q] - t.a[r][q];
      ai = inv(t);
      V<N> bd = mv(b, dl);
#pragma unroll
      for (int r = 0; r < N; ++r) bd.a[r] = rhs.a[r] - bd.a[r];
      d = mv(ai, bd);
    }
    aC = mm(ai, c);
    dl = d;
    double *sp = scr + (int64_t)(i - is) * NE * ncol + col;
#pragma unroll
    for (int r = 0; r < N; ++r)
#pragma unroll
      for (int q = 0; q < N; ++q) sp[(r * N + q) * ncol] = aC.a[r][q];
#pragma unroll
    for (int r = 0; r < N; ++r) sp[(N * N + r) * ncol] = d.a[r];
    // shift the window
    Am = Ap;
    Jm = Jc;
    Jc = Jn;
#pragma unroll
    for (int n = 0; n < NV; ++n) wc[n] = wn[n];
  }

  // backward substitution and the conserved update, top-down
  V<N> dn = dl;  // delta at i+1 (final)
  for (int i = ie; i >= is; --i) {
    const double *sp = scr + (int64_t)(i - is) * NE * ncol + col;
    V<N> d;
    if (i == ie) {
      d = dn;
    } else {
      M<N> ac;
#pragma unroll
      for (int r = 0; r < N; ++r)
#pragma unroll
        for (int q = 0; q < N; ++q) ac.a[r][q] = sp[(r * N + q) * ncol];
#pragma unroll
      for (int r = 0; r < N; ++r) d.a[r] = sp[(N * N + r) * ncol];
      V<N> t = mv(ac, dn);
#pragma unroll
      for (int r = 0; r < N; ++r) d.a[r] -= t.a[r];
    }
    dn = d;
    // forward_backward.hpp:101-124
    double dv[NV];
#pragma unroll
    for (int n = 0; n < NV; ++n) dv[n] = du[n * g.sv + base + i];
    double dens = dv[0];
#pragma unroll
    for (int n = 1; n <= NY; ++n) dens += dv[n];
    dens = d.a[0] - dens;
    dv[0] = d.a[0];
#pragma unroll
    for (int n = 1; n <= NY; ++n) dv[n] += dens * w[n * g.sv + base + i];
    dv[S::IVX] = d.a[1];
    if constexpr (N == 3) {
      dv[S::IPR] = d.a[2];
    } else {
      dv[S::IVY] = d.a[2];
      dv[S::IVZ] = d.a[3];
      dv[S::IPR] = d.a[4];
    }
#pragma unroll
    for (int n = 1; n <= NY; ++n) dv[0] -= dv[n];
    if constexpr (MODE == kUpdateCorrectOnly) {
#pragma unroll
      for (int n = 0; n < NV; ++n) du[n * g.sv + base + i] = dv[n];
    } else {
#pragma unroll
      for (int n = 0; n < NV; ++n) {
        const int64_t x = n * g.sv + base + i;
        double uo = u[x];
        double ur;
        if (stage == 0) {
          u1[x] = uo;
          ur = uo;
        } else {
          ur = u1[x];
        }
        double t = st.g1 * uo + st.g2 * ur;
        u[x] = t + dv[n];
      }
    }
  }
}

template <int NY>
__global__ void k_update_explicit(Geom g, const double *__restrict__ du,
                                  double *__restrict__ u, double *__restrict__ u1,
                                  Stage st, int stage) {
  const int64_t ncell = (int64_t)g.nx1 * g.nx2 * g.nx3;
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ncell) return;
  const int i = g.is + (int)(t % g.nx1);
  const int64_t r = t / g.nx1;
  const int j = g.js + (int)(r % g.nx2), k = g.ks + (int)(r / g.nx2);
  const int64_t base = (int64_t)k * g.sk + (int64_t)j * g.nc1 + i;
#pragma unroll
  for (int n = 0; n < Slots<NY>::NV; ++n) {
    const int64_t x = n * g.sv + base;
    double uo = u[x];
    double ur;
    if (stage == 0) {
      u1[x] = uo;
      ur = uo;
    } else {
      ur = u1[x];
    }
    double v = st.g1 * uo + st.g2 * ur;
    u[x] = v + du[x];
  }
}

template <int NY>
int run_update(const Geom &g, const canoe_thermo_t &th, int flag, const double *w,
               double *du, double *u, double *u1, const double *dtp, const Stage &s,
               int stage, int mode, double *scr, cudaStream_t st) {
  if (flag & 1) {
    const int ncol = g.nx2 * g.nx3;
    const int nt = 128;
    const int nb = (ncol + nt - 1) / nt;
    if (flag & 8) {
      if (mode == kUpdateRK)
        k_column<5, NY, kUpdateRK><<<nb, nt, 0, st>>>(g, th, w, du, u, u1, dtp, s, stage, scr);
      else
        k_column<5, NY, kUpdateCorrectOnly><<<nb, nt, 0, st>>>(g, th, w, du, u, u1, dtp, s, stage, scr);
    } else {
      if (mode == kUpdateRK)
        k_column<3, NY, kUpdateRK><<<nb, nt, 0, st>>>(g, th, w, du, u, u1, dtp, s, stage, scr);
      else
        k_column<3, NY, kUpdateCorrectOnly><<<nb, nt, 0, st>>>(g, th, w, du, u, u1, dtp, s, stage, scr);
    }
  } else {
    if (mode != kUpdateRK) return 0;
    const int64_t ncell = (int64_t)g.nx1 * g.nx2 * g.nx3;
    const int nt = 256;
    k_update_explicit<NY><<<(unsigned)((ncell + nt - 1) / nt), nt, 0, st>>>(g, du, u, u1, s, stage);
  }
  CB_CUDA(cudaGetLastError());
  return 0;
}

}  // namespace

size_t implicit_scratch_doubles(const Geom &g, int flag) {
  if (!(flag & 1)) return 0;
  const int N = (flag & 8) ? 5 : 3;
  return (size_t)g.nx1 * (N * N + N) * (size_t)g.nx2 * g.nx3;
}

int launch_update(const Geom &g, const canoe_thermo_t &th, int flag, const double *w,
                  double *du, double *u, double *u1, const double *dtp, const Stage &s,
                  int stage, int mode, double *scr, cudaStream_t st) {
  if ((flag & 1) && g.bc[0] == CANOE_BC_PERIODIC) {
    set_error("implicit X1 solve with periodic x1 boundaries is not supported");
    return CANOE_ERR_UNSUPPORTED;
  }
  switch (th.ny) {
    case 0: return run_update<0>(g, th, flag, w, du, u, u1, dtp, s, stage, mode, scr, st);
    case 1: return run_update<1>(g, th, flag, w, du, u, u1, dtp, s, stage, mode, scr, st);
    case 2: return run_update<2>(g, th, flag, w, du, u, u1, dtp, s, stage, mode, scr, st);
    case 3: return run_update<3>(g, th, flag, w, du, u, u1, dtp, s, stage, mode, scr, st);
    case 6: return run_update<6>(g, th, flag, w, du, u, u1, dtp, s, stage, mode, scr, st);
    default:
      set_error("unsupported number of mass-fraction slots");
      return CANOE_ERR_UNSUPPORTED;
  }
}

}  // namespace cb
