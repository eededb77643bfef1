// implicit.cpp -- oracle restatement of canoe's implicit vertical solver,
// X1 direction: ImplicitSolver::SolveImplicit3D (src/snap/implicit/
// solve_implicit_3d.cpp:91-142) -> PartialCorrection (partial_correction.cpp:
// 26-170) / FullCorrection (full_correction.cpp:32-161) -> ForwardSweep /
// BackwardSubstitution (forward_backward.hpp:15-137), or, with periodic x1,
// PeriodicForwardSweep / PeriodicBackwardSubstitution
// (periodic_forward_backward.hpp:15-234), single block per column
// (first_block = last_block = true, no MPI pipeline).
// Small dense matrices are plain arrays instead of Eigen; 3x3 inverses use
// the adjugate, 5x5 inverses Gauss-Jordan with partial pivoting.
// TEST INFRASTRUCTURE ONLY.
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "oracle.hpp"

namespace oracle {

namespace {

template <int N>
struct Mat {
  double a[N][N];
  void zero() { std::memset(a, 0, sizeof(a)); }
};
template <int N>
struct Vec {
  double a[N];
};

template <int N>
Mat<N> mul(const Mat<N> &x, const Mat<N> &y) {
  Mat<N> r;
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j) {
      double s = 0.;
      for (int k = 0; k < N; ++k) s += x.a[i][k] * y.a[k][j];
      r.a[i][j] = s;
    }
  return r;
}
template <int N>
Vec<N> mul(const Mat<N> &x, const Vec<N> &y) {
  Vec<N> r;
  for (int i = 0; i < N; ++i) {
    double s = 0.;
    for (int k = 0; k < N; ++k) s += x.a[i][k] * y.a[k];
    r.a[i] = s;
  }
  return r;
}

Mat<3> inverse(const Mat<3> &m) {
  const double(*a)[3] = m.a;
  double c00 = a[1][1] * a[2][2] - a[1][2] * a[2][1];
  double c01 = a[1][2] * a[2][0] - a[1][0] * a[2][2];
  double c02 = a[1][0] * a[2][1] - a[1][1] * a[2][0];
  double det = a[0][0] * c00 + a[0][1] * c01 + a[0][2] * c02;
  double id = 1. / det;
  Mat<3> r;
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

Mat<5> inverse(const Mat<5> &m) {
  double a[5][10];
  for (int i = 0; i < 5; ++i)
    for (int j = 0; j < 5; ++j) {
      a[i][j] = m.a[i][j];
      a[i][5 + j] = (i == j) ? 1. : 0.;
    }
  for (int c = 0; c < 5; ++c) {
    int p = c;
    for (int r = c + 1; r < 5; ++r)
      if (std::fabs(a[r][c]) > std::fabs(a[p][c])) p = r;
    if (p != c)
      for (int j = 0; j < 10; ++j) std::swap(a[c][j], a[p][j]);
    double ip = 1. / a[c][c];
    for (int j = 0; j < 10; ++j) a[c][j] *= ip;
    for (int r = 0; r < 5; ++r) {
      if (r == c) continue;
      double f = a[r][c];
      if (f != 0.)
        for (int j = 0; j < 10; ++j) a[r][j] -= f * a[c][j];
    }
  }
  Mat<5> r;
  for (int i = 0; i < 5; ++i)
    for (int j = 0; j < 5; ++j) r.a[i][j] = a[i][5 + j];
  return r;
}

// FluxJacobian, flux_decomposition.hpp:102-120 (X1: v1 = w[IVX]).
void flux_jacobian(Mat<5> &d, double gm1, const double *w, int IVX, int IPR) {
  double v1 = w[IVX], v2 = w[IVX + 1], v3 = w[IVX + 2];
  double rho = w[0], pres = w[IPR];
  double s2 = v1 * v1 + v2 * v2 + v3 * v3;
  double c1 = ((gm1 - 1) * s2 / 2 - (gm1 + 1) / gm1 * pres / rho) * v1;
  double c2 = (gm1 + 1) / gm1 * pres / rho + s2 / 2 - gm1 * v1 * v1;
  double r[25] = {0,     1.,           0.,         0.,         0.,
                  gm1 * s2 / 2 - v1 * v1, (2. - gm1) * v1, -gm1 * v2, -gm1 * v3, gm1,
                  -v1 * v2, v2,        v1,         0.,         0.,
                  -v1 * v3, v3,        0.,         v1,         0.,
                  c1,    c2,           -gm1 * v2 * v1, -gm1 * v3 * v1, (gm1 + 1) * v1};
  for (int i = 0; i < 5; ++i)
    for (int j = 0; j < 5; ++j) d.a[i][j] = r[i * 5 + j];
}

// RoeAverage, flux_decomposition.hpp:34-67
void roe_average(double *prim, double gm1, const double *wl, const double *wr,
                 int ny) {
  int IVX = 1 + ny, IVY = 2 + ny, IVZ = 3 + ny, IPR = 4 + ny;
  double sqrtdl = std::sqrt(wl[0]);
  double sqrtdr = std::sqrt(wr[0]);
  double isdlpdr = 1.0 / (sqrtdl + sqrtdr);
  prim[0] = sqrtdl * sqrtdr;
  prim[IVX] = (sqrtdl * wl[IVX] + sqrtdr * wr[IVX]) * isdlpdr;
  prim[IVY] = (sqrtdl * wl[IVY] + sqrtdr * wr[IVY]) * isdlpdr;
  prim[IVZ] = (sqrtdl * wl[IVZ] + sqrtdr * wr[IVZ]) * isdlpdr;
  for (int i = 1; i < IVX; ++i) prim[i] = (sqrtdl * wl[i] + sqrtdr * wr[i]) * isdlpdr;
  double el = wl[IPR] / gm1 +
              0.5 * wl[0] * (wl[IVX] * wl[IVX] + wl[IVY] * wl[IVY] + wl[IVZ] * wl[IVZ]);
  double er = wr[IPR] / gm1 +
              0.5 * wr[0] * (wr[IVX] * wr[IVX] + wr[IVY] * wr[IVY] + wr[IVZ] * wr[IVZ]);
  double hbar = ((el + wl[IPR]) / sqrtdl + (er + wr[IPR]) / sqrtdr) * isdlpdr;
  prim[IPR] = (hbar - 0.5 * (prim[IVX] * prim[IVX] + prim[IVY] * prim[IVY] +
                             prim[IVZ] * prim[IVZ])) *
              gm1 / (gm1 + 1.) * prim[0];
}

// |A| = R |Lambda| R^-1: Eigenvalue (:70-75) and Eigenvector (:78-99)
void abs_jacobian(Mat<5> &A, const double *prim, double cs, double gm1, int ny) {
  int IVX = 1 + ny, IPR = 4 + ny;
  double r = prim[0], u = prim[IVX], v = prim[IVX + 1], w = prim[IVX + 2],
         p = prim[IPR];
  double ke = 0.5 * (u * u + v * v + w * w);
  double hp = (gm1 + 1.) / gm1 * p / r;
  double h = hp + ke;
  double R[25] = {1.,         1., 1.,         0., 0.,  //
                  u - cs,     u,  u + cs,     0., 0.,  //
                  v,          v,  v,          1., 0.,  //
                  w,          w,  w,          0., 1.,  //
                  h - u * cs, ke, h + u * cs, v,  w};
  double Ri[25] = {(cs * ke + u * hp) / (2. * cs * hp), (-hp - cs * u) / (2. * cs * hp),
                   -v / (2. * hp), -w / (2. * hp), 1. / (2. * hp),
                   (hp - ke) / hp, u / hp, v / hp, w / hp, -1. / hp,
                   (cs * ke - u * hp) / (2. * cs * hp), (hp - cs * u) / (2. * cs * hp),
                   -v / (2. * hp), -w / (2. * hp), 1. / (2. * hp),
                   -v, 0., 1., 0., 0.,
                   -w, 0., 0., 1., 0.};
  double lam[5] = {std::fabs(u - cs), std::fabs(u), std::fabs(u + cs), std::fabs(u),
                   std::fabs(u)};
  for (int i = 0; i < 5; ++i)
    for (int j = 0; j < 5; ++j) {
      double s = 0.;
      for (int k = 0; k < 5; ++k) s += (R[i * 5 + k] * lam[k]) * Ri[k * 5 + j];
      A.a[i][j] = s;
    }
}

template <int N>
Mat<N> reduce(const Mat<5> &m) {
  Mat<N> r;
  if constexpr (N == 5) {
    for (int i = 0; i < 5; ++i)
      for (int j = 0; j < 5; ++j) r.a[i][j] = m.a[i][j];
  } else {
    static const int sel[3] = {0, 1, 4};
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) r.a[i][j] = m.a[sel[i]][sel[j]];
  }
  return r;
}

template <int N>
Mat<N> sub(const Mat<N> &x, const Mat<N> &y) {
  Mat<N> r;
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j) r.a[i][j] = x.a[i][j] - y.a[i][j];
  return r;
}
template <int N>
Mat<N> neg(const Mat<N> &x) {
  Mat<N> r;
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j) r.a[i][j] = -x.a[i][j];
  return r;
}
template <int N>
Vec<N> sub(const Vec<N> &x, const Vec<N> &y) {
  Vec<N> r;
  for (int i = 0; i < N; ++i) r.a[i] = x.a[i] - y.a[i];
  return r;
}

// El-Mikkawy (2005) cyclic block-tridiagonal solve of one column,
// periodic_forward_backward.hpp:15-234 with first_block = last_block: the
// row is couples to ie through the upper corner b[is] and the row ie to is
// through the lower corner c[is-1] (the ghost row's upper block).  Leaves the
// solution in delta.
template <int N, class Rhs>
void periodic_sweep(int is, int ie, const std::vector<Mat<N>> &a,
                    const std::vector<Mat<N>> &bb, std::vector<Mat<N>> c, Rhs rhs_of,
                    std::vector<Vec<N>> &delta) {
  const size_t n = a.size();
  std::vector<Mat<N>> ainv(n), gam(n), beta(n);
  std::vector<Vec<N>> zeta(n);
  Mat<N> sbg;
  sbg.zero();
  Vec<N> sbz;
  for (int r = 0; r < N; ++r) sbz.a[r] = 0.;
  // PeriodicForwardSweep (:61-172)
  Vec<N> rhs = rhs_of(is);
  ainv[is] = inverse(a[is]);
  gam[is] = bb[is];
  beta[is] = mul(c[is - 1], ainv[is]);
  zeta[is] = rhs;
  for (int i = is + 1; i <= ie; ++i) {
    rhs = rhs_of(i);
    const Mat<N> bl = mul(bb[i], ainv[i - 1]);
    ainv[i] = inverse(sub(a[i], mul(bl, c[i - 1])));
    gam[i] = mul(neg(bl), gam[i - 1]);
    beta[i] = mul(mul(neg(beta[i - 1]), c[i - 1]), ainv[i]);
    zeta[i] = sub(rhs, mul(bl, zeta[i - 1]));
  }
  gam[ie - 1] = sub(c[ie - 1], mul(mul(bb[ie - 1], ainv[ie - 2]), gam[ie - 2]));
  beta[ie - 1] = mul(sub(bb[ie], mul(beta[ie - 2], c[ie - 2])), ainv[ie - 1]);
  for (int i = is; i < ie; ++i) {
    const Mat<N> t = mul(beta[i], gam[i]);
    const Vec<N> v = mul(beta[i], zeta[i]);
    for (int r = 0; r < N; ++r) {
      sbz.a[r] += v.a[r];
      for (int q = 0; q < N; ++q) sbg.a[r][q] += t.a[r][q];
    }
  }
  ainv[ie] = inverse(sub(a[ie], sbg));
  zeta[ie] = sub(rhs, sbz);
  // PeriodicBackwardSubstitution (:176-204)
  c[ie - 1].zero();
  delta[ie] = mul(ainv[ie], zeta[ie]);
  const Vec<N> last = delta[ie];
  for (int i = ie - 1; i >= is; --i)
    delta[i] = mul(ainv[i], sub(sub(zeta[i], mul(c[i], delta[i + 1])), mul(gam[i], last)));
}

// One implicit line of direction dir (0: x1, 1: x2, 2: x3) through the cell
// (k, j, i) with the line index replaced: PartialCorrection / FullCorrection
// with mydir_ = dir.  The line's primitives are read with the velocity in the
// direction's frame (normal, then the next two cyclically), as CopyPrimitives,
// FluxJacobian and Eigenvector do (flux_decomposition.hpp:14-120); the
// reference transposes du (solve_implicit_3d.cpp:35-56, 68-89) and writes back
// IDN, the normal momentum and IEN only.
template <int N>
void column(Block &b, std::vector<double> &du, double dt, int dir, int k, int j, int i0) {
  const int nc1 = b.nc1, nv = b.nv, ny = b.ny, IVX = b.ivx, IPR = b.ipr;
  const int lo = dir == 0 ? b.is : dir == 1 ? b.js : b.ks;
  const int hi = dir == 0 ? b.ie : dir == 1 ? b.je : b.ke;
  const int is = lo, ie = hi;
  const int nline = (dir == 0 ? b.nc1 : dir == 1 ? b.nc2 : b.nc3);
  const size_t s = b.cells();
  // flat offset of line position t
  auto at = [&](int t) -> size_t {
    if (dir == 0) return b.idx(0, k, j, t);
    if (dir == 1) return b.idx(0, k, t, i0);
    return b.idx(0, t, j, i0);
  };
  const int vn = IVX + dir, vt1 = IVX + (1 + dir) % 3, vt2 = IVX + (2 + dir) % 3;
  // a cubed-sphere panel projects the velocities onto the local frame
  // for the solve (solve_implicit_3d.cpp:105-117)
  double cos_t = 0., sin_t = 1.;
  if (b.geo) {
    cos_t = b.geo->cosc[b.geo->kj(k, j)];
    sin_t = b.geo->sinc[b.geo->kj(k, j)];
  }
  auto W = [&](int t, double *out) {
    const size_t c = at(t);
    for (int n = 0; n < nv; ++n) out[n] = b.w[c + n * s];
    if (dir != 0) {
      const double a = out[vn], bb = out[vt1], cc = out[vt2];
      out[IVX] = a;
      out[IVX + 1] = bb;
      out[IVX + 2] = cc;
    }
    if (b.geo) {
      out[IVX + 1] += out[IVX + 2] * cos_t;
      out[IVX + 2] *= sin_t;
    }
  };
  const double gm1 = b.th.gammad - 1.;
  const double grav = dir == 0 ? b.th.grav : 0.;  // Phi acts in x1 only
  std::vector<Mat<N>> a(nline), bb(nline), c(nline), dfdq(nline);
  std::vector<Vec<N>> delta(nline);
  Mat<5> full;
  double wl[CANOE_MAX_NV], wr[CANOE_MAX_NV], prim[CANOE_MAX_NV];
  // flux Jacobians of cells is-2..ie+1 (partial_correction.cpp:90-101)
  for (int i = is - 2; i <= ie + 1; ++i) {
    W(i, wr);
    flux_jacobian(full, gm1, wr, IVX, IPR);
    dfdq[i] = reduce<N>(full);
  }
  Mat<N> Phi, Dt, Bnd;
  Phi.zero();
  Dt.zero();
  Bnd.zero();
  for (int d = 0; d < N; ++d) {
    Dt.a[d][d] = 1. / dt;
    Bnd.a[d][d] = 1.;
  }
  Bnd.a[1][1] = -1.;
  if constexpr (N == 3) {  // partial_correction.cpp:59-61 (row-major comma fill)
    Phi.a[1][0] = grav;
    Phi.a[2][1] = grav;
  } else {  // full_correction.cpp:57-61
    Phi.a[1][0] = grav;
    Phi.a[4][1] = grav;
  }
  // left edge |A| at face is-1-1/2 (partial_correction.cpp:103-115)
  W(is - 2, wl);
  W(is - 1, wr);
  roe_average(prim, gm1, wl, wr, ny);
  double cs = sound_speed(b.th, prim);
  abs_jacobian(full, prim, cs, gm1, ny);
  Mat<N> Am = reduce<N>(full), Ap;
  const double area = b.dx2 * b.dx3;
  for (int i = is - 1; i <= ie; ++i) {
    // face areas and the cell volume (GetFace{1,2,3}Area, GetCellVolume of
    // the Cartesian block; partial_correction.cpp:116-127)
    W(i, wl);
    W(i + 1, wr);
    roe_average(prim, gm1, wl, wr, ny);
    cs = sound_speed(b.th, prim);
    abs_jacobian(full, prim, cs, gm1, ny);
    Ap = reduce<N>(full);
    double aleft = area, aright = area, vol = b.dx1f[i] * b.dx2 * b.dx3;
    if (dir == 1) {
      aleft = aright = b.dx1f[i0] * b.dx3;
      vol = b.dx1f[i0] * b.dx2 * b.dx3;
    } else if (dir == 2) {
      aleft = aright = b.dx1f[i0] * b.dx2;
      vol = b.dx1f[i0] * b.dx2 * b.dx3;
    }
    if (b.geo) {  // GetFace1Area / GetCellVolume of the panel
      aleft = shell_face1_area(b, k, j, i);
      aright = shell_face1_area(b, k, j, i + 1);
      vol = shell_cell_volume(b, k, j, i);
    }
    for (int r = 0; r < N; ++r)
      for (int q = 0; q < N; ++q) {
        a[i].a[r][q] = (Am.a[r][q] * aleft + Ap.a[r][q] * aright +
                        (aright - aleft) * dfdq[i].a[r][q]) /
                           (2. * vol) +
                       Dt.a[r][q] - Phi.a[r][q];
        bb[i].a[r][q] = -(Am.a[r][q] + dfdq[i - 1].a[r][q]) * aleft / (2. * vol);
        c[i].a[r][q] = -(Ap.a[r][q] - dfdq[i + 1].a[r][q]) * aright / (2. * vol);
      }
    Am = Ap;
  }
  const bool periodic = b.cfg.bc[2 * dir] == CANOE_BC_PERIODIC;
  // reflecting ends (partial_correction.cpp:153-154); none when periodic
  if (!periodic) {
    Mat<N> t = mul(bb[is], Bnd);
    for (int r = 0; r < N; ++r)
      for (int q = 0; q < N; ++q) a[is].a[r][q] += t.a[r][q];
    t = mul(c[ie], Bnd);
    for (int r = 0; r < N; ++r)
      for (int q = 0; q < N; ++q) a[ie].a[r][q] += t.a[r][q];
  }
  // ForwardSweep (forward_backward.hpp:15-85)
  auto D = [&](int n, int t) -> double & { return du[at(t) + n * s]; };
  auto rhs_of = [&](int i) {
    Vec<N> r;
    double r0 = D(0, i);
    for (int n = 1; n < IVX; ++n) r0 += D(n, i);
    r.a[0] = r0 / dt;
    r.a[1] = D(vn, i) / dt;
    if constexpr (N == 3) {
      r.a[2] = D(IPR, i) / dt;
    } else {
      r.a[2] = D(vt1, i) / dt;
      r.a[3] = D(vt2, i) / dt;
      r.a[4] = D(IPR, i) / dt;
    }
    return r;
  };
  // x2 / x3: the reference copies back IDN, the normal momentum and IEN
  // (solve_implicit_3d.cpp:46-55, 79-88); the other slots of du stay
  auto put_line = [&](int i, const Vec<N> &x) {
    D(0, i) = x.a[0];
    D(vn, i) = x.a[1];
    D(IPR, i) = x.a[N - 1];
  };
  if (periodic) {
    periodic_sweep<N>(is, ie, a, bb, c, rhs_of, delta);
    if (dir != 0) {  // dry only (checked by the caller)
      for (int i = is; i <= ie; ++i) put_line(i, delta[i]);
      return;
    }
    // the periodic update carries no species correction: du_n stays, and
    // the dry density takes delta(0) minus the species
    // (periodic_forward_backward.hpp:207-225)
    for (int i = is; i <= ie; ++i) {
      D(0, i) = delta[i].a[0];
      D(IVX, i) = delta[i].a[1];
      if constexpr (N == 3) {
        D(IPR, i) = delta[i].a[2];
      } else {
        D(IVX + 1, i) = delta[i].a[2];
        D(IVX + 2, i) = delta[i].a[3];
        D(IPR, i) = delta[i].a[4];
      }
      for (int n = 1; n < IVX; ++n) D(0, i) -= D(n, i);
    }
    return;
  }
  {
    Vec<N> rhs = rhs_of(is);
    a[is] = inverse(a[is]);
    delta[is] = mul(a[is], rhs);
    a[is] = mul(a[is], c[is]);
  }
  for (int i = is + 1; i <= ie; ++i) {
    Vec<N> rhs = rhs_of(i);
    Mat<N> t = mul(bb[i], a[i - 1]);
    for (int r = 0; r < N; ++r)
      for (int q = 0; q < N; ++q) t.a[r][q] = a[i].a[r][q] - t.a[r][q];
    a[i] = inverse(t);
    Vec<N> bd = mul(bb[i], delta[i - 1]);
    for (int r = 0; r < N; ++r) bd.a[r] = rhs.a[r] - bd.a[r];
    delta[i] = mul(a[i], bd);
    a[i] = mul(a[i], c[i]);
  }
  // BackwardSubstitution (forward_backward.hpp:87-137)
  for (int i = ie - 1; i >= is; --i) {
    Vec<N> t = mul(a[i], delta[i + 1]);
    for (int r = 0; r < N; ++r) delta[i].a[r] -= t.a[r];
  }
  if (dir != 0) {  // dry only (checked by the caller)
    for (int i = is; i <= ie; ++i) put_line(i, delta[i]);
    return;
  }
  for (int i = is; i <= ie; ++i) {
    double dens = D(0, i);
    for (int n = 1; n < IVX; ++n) dens += D(n, i);
    dens = delta[i].a[0] - dens;
    D(0, i) = delta[i].a[0];
    for (int n = 1; n < IVX; ++n) D(n, i) += dens * b.w[b.idx(n, k, j, i)];
    D(IVX, i) = delta[i].a[1];
    if constexpr (N == 3) {
      D(IPR, i) = delta[i].a[2];
    } else {
      D(IVX + 1, i) = delta[i].a[2];
      D(IVX + 2, i) = delta[i].a[3];
      D(IPR, i) = delta[i].a[4];
    }
    for (int n = 1; n < IVX; ++n) D(0, i) -= D(n, i);
  }
}

template <int N>
void periodic_dense(int n, const double *a, const double *b, const double *c,
                    const double *rhs, double *x) {
  std::vector<Mat<N>> A(n + 1), B(n + 1), C(n + 1);
  std::vector<Vec<N>> R(n + 1), D(n + 1);
  for (int i = 0; i <= n; ++i)
    for (int r = 0; r < N; ++r) {
      R[i].a[r] = rhs[i * N + r];
      for (int q = 0; q < N; ++q) {
        A[i].a[r][q] = a[(i * N + r) * N + q];
        B[i].a[r][q] = b[(i * N + r) * N + q];
        C[i].a[r][q] = c[(i * N + r) * N + q];
      }
    }
  periodic_sweep<N>(1, n, A, B, C, [&](int i) { return R[i]; }, D);
  for (int i = 1; i <= n; ++i)
    for (int r = 0; r < N; ++r) x[i * N + r] = D[i].a[r];
}

}  // namespace

int periodic_block_solve(int nb, int n, const double *a, const double *b, const double *c,
                         const double *rhs, double *x) {
  if (n < 3) return 1;
  if (nb == 3) periodic_dense<3>(n, a, b, c, rhs, x);
  else if (nb == 5) periodic_dense<5>(n, a, b, c, rhs, x);
  else return 1;
  return 0;
}

void solve_implicit(Block &b, std::vector<double> &du, double dt) {
  const int flag = b.cfg.implicit_flag;
  const bool full = flag & 8;
  const bool x3 = (flag & 4) && b.cfg.nx3 > 1, x2 = (flag & 2) && b.cfg.nx2 > 1;
  if ((x2 || x3) && (b.ny > 0 || b.geo))
    throw std::runtime_error("x2 / x3 implicit solves are provided for a dry Cartesian block");
  for (int d = 0; d < 3; ++d) {
    const bool p0 = b.cfg.bc[2 * d] == CANOE_BC_PERIODIC, p1 = b.cfg.bc[2 * d + 1] == CANOE_BC_PERIODIC;
    const bool on = d == 0 ? (flag & 1) : d == 1 ? x2 : x3;
    if (!on) continue;
    if (p0 != p1) throw std::runtime_error("a periodic direction needs both boundaries periodic");
    const int n = d == 0 ? b.cfg.nx1 : d == 1 ? b.cfg.nx2 : b.cfg.nx3;
    if (p0 && n < 3) throw std::runtime_error("a periodic implicit solve needs at least 3 cells");
  }
  auto run = [&](int d, int k, int j, int i) {
    if (full)
      column<5>(b, du, dt, d, k, j, i);
    else
      column<3>(b, du, dt, d, k, j, i);
  };
  // solve_implicit_3d.cpp:25-142: X3, then X2, then X1
  if (x3) {
#pragma omp parallel for collapse(2) schedule(dynamic, 16)
    for (int j = b.js; j <= b.je; ++j)
      for (int i = b.is; i <= b.ie; ++i) run(2, 0, j, i);
  }
  if (x2) {
#pragma omp parallel for collapse(2) schedule(dynamic, 16)
    for (int k = b.ks; k <= b.ke; ++k)
      for (int i = b.is; i <= b.ie; ++i) run(1, k, 0, i);
  }
  if (flag & 1) {
#pragma omp parallel for collapse(2) schedule(dynamic, 16)
    for (int k = b.ks; k <= b.ke; ++k)
      for (int j = b.js; j <= b.je; ++j) run(0, k, j, 0);
  }
}

}  // namespace oracle
