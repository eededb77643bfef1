// blockmat.cuh -- small dense block algebra of the implicit vertical solver
// (canoe src/snap/implicit/flux_decomposition.hpp): flux Jacobian, the
// Roe-averaged |A| = R |Lambda| R^-1, 3x3 / 5x5 inverses and products.
// N = 3 is the reduced (rho, m1, E) system of PartialCorrection, N = 5 the
// full system of FullCorrection.
#pragma once

#include "block.cuh"

namespace cb {

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

// entry (i, j) of the inverse of the row-major 3x3 matrix a (adjugate over
// the determinant); inv(M<3>) and the entry-parallel reduction both use it
__device__ __forceinline__ double inv3_entry(const double *a, int i, int j) {
  const double c00 = a[4] * a[8] - a[5] * a[7];
  const double c01 = a[5] * a[6] - a[3] * a[8];
  const double c02 = a[3] * a[7] - a[4] * a[6];
  const double det = a[0] * c00 + a[1] * c01 + a[2] * c02;
  const double id = 1. / det;
  double num;
  switch (3 * i + j) {
    case 0: num = c00; break;
    case 3: num = c01; break;
    case 6: num = c02; break;
    case 1: num = a[2] * a[7] - a[1] * a[8]; break;
    case 4: num = a[0] * a[8] - a[2] * a[6]; break;
    case 7: num = a[1] * a[6] - a[0] * a[7]; break;
    case 2: num = a[1] * a[5] - a[2] * a[4]; break;
    case 5: num = a[2] * a[3] - a[0] * a[5]; break;
    default: num = a[0] * a[4] - a[1] * a[3]; break;
  }
  return num * id;
}

__device__ __forceinline__ M<3> inv(const M<3> &m) {
  const double *a = &m.a[0][0];
  M<3> r;
#pragma unroll
  for (int e = 0; e < 9; ++e) r.a[e / 3][e % 3] = inv3_entry(a, e / 3, e % 3);
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

// Row-parallel 5x5 algebra for the cyclic reduction of the full system.  An
// 8-lane segment of a warp holds one 5x5 block: lane g < 5 owns row g, lanes
// 5..7 follow along (their results are never stored).  Shuffles stay inside
// the segment (width 8, mask smask of the segment's lanes).

// Gauss-Jordan inverse with partial pivoting of the block whose row g is
// ar[], the steps of inv(M<5>) with the pivot rows left in place: at column c
// the largest |ar[c]| among the lanes not yet used as pivots (lowest lane on
// a tie) normalises its row and eliminates column c from every other row.
// On return iv[] is row `pivot_of` of the inverse, where pivot_of is the
// column this lane was the pivot for (rows 0..4 are held by lanes 0..4 in
// some order).
__device__ __forceinline__ int inv5_rows(double ar[5], double iv[5], int g,
                                         unsigned smask) {
#pragma unroll
  for (int q = 0; q < 5; ++q) iv[q] = (q == g) ? 1. : 0.;
  int mine = -1;  // the column this lane pivoted
#pragma unroll
  for (int c = 0; c < 5; ++c) {
    double v = (g < 5 && mine < 0) ? fabs(ar[c]) : -1.;
    int p = g;
#pragma unroll
    for (int off = 4; off >= 1; off >>= 1) {
      const double ov = __shfl_xor_sync(smask, v, off, 8);
      const int op = __shfl_xor_sync(smask, p, off, 8);
      if (ov > v || (ov == v && op < p)) {
        v = ov;
        p = op;
      }
    }
    const double ip = 1. / __shfl_sync(smask, ar[c], p, 8);
    if (g == p) {
      mine = c;
#pragma unroll
      for (int q = c + 1; q < 5; ++q) ar[q] *= ip;
#pragma unroll
      for (int q = 0; q < 5; ++q) iv[q] *= ip;
    }
    double pr[5], pi[5];
#pragma unroll
    for (int q = c + 1; q < 5; ++q) pr[q] = __shfl_sync(smask, ar[q], p, 8);
#pragma unroll
    for (int q = 0; q < 5; ++q) pi[q] = __shfl_sync(smask, iv[q], p, 8);
    if (g != p) {
      const double f = ar[c];
      if (f != 0.) {
#pragma unroll
        for (int q = c + 1; q < 5; ++q) ar[q] -= f * pr[q];
#pragma unroll
        for (int q = 0; q < 5; ++q) iv[q] -= f * pi[q];
      }
    }
  }
  return mine;
}

// row / column selection of the reduced (partial) system: (rho, m1, E)
template <int N>
__device__ __forceinline__ constexpr int sel(int r) {
  return N == 5 ? r : (r == 2 ? 4 : r);
}

// FluxJacobian (flux_decomposition.hpp:102-120), reduced to N x N, evaluated
// in T (double; float for the FP32 flux path, whose implicit blocks are
// formed from FP32 coefficients and eliminated in FP64)
template <int N, int NY, typename T = double>
__device__ __forceinline__ void jacobian(M<N> &d, double gm1_, const double *w) {
  using S = Slots<NY>;
  const T gm1 = T(gm1_);
  T v1 = T(w[S::IVX]), v2 = T(w[S::IVY]), v3 = T(w[S::IVZ]);
  T rho = T(w[0]), pres = T(w[S::IPR]);
  T s2 = v1 * v1 + v2 * v2 + v3 * v3;
  T c1 = ((gm1 - T(1)) * s2 / T(2) - pdiv(pdiv(gm1 + T(1), gm1) * pres, rho)) * v1;
  T c2 = pdiv(pdiv(gm1 + T(1), gm1) * pres, rho) + s2 / T(2) - gm1 * v1 * v1;
  const T f[5][5] = {{T(0), T(1), T(0), T(0), T(0)},
                     {gm1 * s2 / T(2) - v1 * v1, (T(2) - gm1) * v1, -gm1 * v2, -gm1 * v3, gm1},
                     {-v1 * v2, v2, v1, T(0), T(0)},
                     {-v1 * v3, v3, T(0), v1, T(0)},
                     {c1, c2, -gm1 * v2 * v1, -gm1 * v3 * v1, (gm1 + T(1)) * v1}};
#pragma unroll
  for (int r = 0; r < N; ++r)
#pragma unroll
    for (int c = 0; c < N; ++c) d.a[r][c] = double(f[sel<N>(r)][sel<N>(c)]);
}

// |A| = R |Lambda| R^-1 at the face between cells with primitive states wl,
// wr: RoeAverage (:34-67), SoundSpeed, Eigenvalue (:70-75), Eigenvector
// (:78-99); only the N x N reduced block is formed, in T as jacobian.
template <int N, int NY, typename T = double>
__device__ __forceinline__ void abs_jacobian(M<N> &A, const canoe_thermo_t &th,
                                             double gm1_, const double *wl_,
                                             const double *wr_) {
  using S = Slots<NY>;
  const T gm1 = T(gm1_);
  T wl[S::NV], wr[S::NV], prim[S::NV];
#pragma unroll
  for (int n = 0; n < S::NV; ++n) {
    wl[n] = T(wl_[n]);
    wr[n] = T(wr_[n]);
  }
  T sqrtdl = sqrt(wl[0]);
  T sqrtdr = sqrt(wr[0]);
  T isdlpdr = pdiv(T(1), sqrtdl + sqrtdr);
  prim[0] = sqrtdl * sqrtdr;
  prim[S::IVX] = (sqrtdl * wl[S::IVX] + sqrtdr * wr[S::IVX]) * isdlpdr;
  prim[S::IVY] = (sqrtdl * wl[S::IVY] + sqrtdr * wr[S::IVY]) * isdlpdr;
  prim[S::IVZ] = (sqrtdl * wl[S::IVZ] + sqrtdr * wr[S::IVZ]) * isdlpdr;
#pragma unroll
  for (int n = 1; n <= NY; ++n) prim[n] = (sqrtdl * wl[n] + sqrtdr * wr[n]) * isdlpdr;
  T el = pdiv(wl[S::IPR], gm1) + T(0.5) * wl[0] *
         (wl[S::IVX] * wl[S::IVX] + wl[S::IVY] * wl[S::IVY] + wl[S::IVZ] * wl[S::IVZ]);
  T er = pdiv(wr[S::IPR], gm1) + T(0.5) * wr[0] *
         (wr[S::IVX] * wr[S::IVX] + wr[S::IVY] * wr[S::IVY] + wr[S::IVZ] * wr[S::IVZ]);
  T hbar = (pdiv(el + wl[S::IPR], sqrtdl) + pdiv(er + wr[S::IPR], sqrtdr)) * isdlpdr;
  prim[S::IPR] = pdiv((hbar - T(0.5) * (prim[S::IVX] * prim[S::IVX] +
                                        prim[S::IVY] * prim[S::IVY] +
                                        prim[S::IVZ] * prim[S::IVZ])) * gm1,
                      gm1 + T(1)) * prim[0];
  T cs = sound_speed<T, NY>(th, prim);
  T r = prim[0], u = prim[S::IVX], v = prim[S::IVY], w = prim[S::IVZ], p = prim[S::IPR];
  T ke = T(0.5) * (u * u + v * v + w * w);
  T hp = pdiv(pdiv(gm1 + T(1), gm1) * p, r);
  T h = hp + ke;
  const T ihp = pdiv(T(1), hp), i2hp = T(0.5) * ihp, i2chp = pdiv(i2hp, cs);
  const T R[5][5] = {{T(1), T(1), T(1), T(0), T(0)},
                     {u - cs, u, u + cs, T(0), T(0)},
                     {v, v, v, T(1), T(0)},
                     {w, w, w, T(0), T(1)},
                     {h - u * cs, ke, h + u * cs, v, w}};
  // R^-1 of Eigenvector (:94-98) with the divisions by hp, 2 hp and
  // 2 cs hp taken as reciprocals
  const T Ri[5][5] = {
      {(cs * ke + u * hp) * i2chp, (-hp - cs * u) * i2chp, -v * i2hp, -w * i2hp, i2hp},
      {(hp - ke) * ihp, u * ihp, v * ihp, w * ihp, -ihp},
      {(cs * ke - u * hp) * i2chp, (hp - cs * u) * i2chp, -v * i2hp, -w * i2hp, i2hp},
      {-v, T(0), T(1), T(0), T(0)},
      {-w, T(0), T(0), T(1), T(0)}};
  const T lam[5] = {fabs(u - cs), fabs(u), fabs(u + cs), fabs(u), fabs(u)};
#pragma unroll
  for (int a = 0; a < N; ++a)
#pragma unroll
    for (int b = 0; b < N; ++b) {
      T s = T(0);
#pragma unroll
      for (int k = 0; k < 5; ++k) s += (R[sel<N>(a)][k] * lam[k]) * Ri[k][sel<N>(b)];
      A.a[a][b] = double(s);
    }
}

template <int NY>
__device__ __forceinline__ void load_w(const Geom &g, const double *__restrict__ w,
                                       int64_t base, int i, double *out) {
#pragma unroll
  for (int n = 0; n < Slots<NY>::NV; ++n) out[n] = w[n * g.sv + base + i];
}

}  // namespace cb
