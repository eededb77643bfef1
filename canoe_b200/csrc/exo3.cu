// exo3.cu -- the six panels of a cubed-sphere shell, resident on one GPU,
// with the panel ghost exchange on device (canoe src/exo3).
//
// All six panels live in one array (6, NV, nc3, nc2, nc1); panel p holds the
// reference's blockID p + 1 (cs_find_block_id.cpp:11-101 with one block per
// panel).  Per RK stage:
//
//   k_shell_ghosts     u ghosts of every panel edge from the neighbour panel:
//                      the reference packs NGHOST interior layers along the
//                      edge, interpolates them along the edge to the
//                      neighbour's ghost-cell positions, rotates the
//                      velocities through latitude-longitude and reorders
//                      them for the receiver (cubed_sphere_utility.cpp:26-623,
//                      cs_transform_ox.cpp:11-230).  Here the host turns that
//                      bookkeeping into one table row per ghost cell (source
//                      cells, interpolation weights, a 2 x 2 velocity map)
//                      and the kernel gathers.
//   k_shell_c2p        cons -> prim with covariant momenta and contravariant
//                      velocities (patches/26.adiabatic_hydro.patch), x1
//                      ghosts by the radial boundary conditions
//   k_shell_edges      the interior-side reconstructed face state of every
//                      panel edge, rotated into the neighbour's frame: the
//                      L/R swap of cubed_sphere.cpp:312-681
//   k_shell_flux_x23   x2 / x3 fluxes: PrimToLocal2/3, HLLC, FluxToGlobal2/3
//                      and the covariant projection (gnomonic_equiangle.cpp:
//                      604-832, hllc_transform.cpp:46-55, 227-272), with the
//                      swapped states at panel edges, and the divergence
//                      with face areas and cell volumes
//   k_x1col<.., GEO=1> x1 fluxes, coordinate sources, implicit x1 solve and
//                      the RK update (column.cuh)
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "column.cuh"

namespace cb {

namespace {

constexpr double kPi = 3.14159265358979323846;

// ---------------------------------------------------------------------------
// host: panel connectivity for one block per panel.  Directions d: 0 the
// x2 face below js (ox2 = -1), 1 above je (ox2 = +1), 2 below ks (ox3 = -1),
// 3 above ke (ox3 = +1).  Tables of cubed_sphere_utility.cpp:385-398.

const int kDinv[6][4] = {{1, 0, 0, 1}, {0, 0, 0, 0}, {0, 1, 0, 0},
                         {1, 0, 0, 0}, {0, 1, 1, 0}, {1, 1, 0, 0}};
const int kTgside[6][4] = {{-1, -1, -1, -1}, {1, -1, 1, -1}, {-1, -1, 1, -1},
                           {1, 1, 1, -1},    {1, 1, 1, 1},   {-1, 1, 1, -1}};
const int kTgbid[6][4] = {{6, 2, 3, 4}, {1, 5, 3, 4}, {1, 5, 6, 2},
                          {1, 5, 2, 6}, {2, 6, 3, 4}, {1, 5, 4, 3}};
// PackData's buffer order per (block, direction): 0 (n,k,j), 1 (n,j desc,k),
// 2 (n,k desc,j desc), 3 (n,j,k desc)
const int kOrder[6][4] = {{2, 0, 3, 1}, {0, 0, 0, 0}, {1, 3, 0, 0},
                          {3, 1, 0, 0}, {0, 2, 1, 3}, {2, 2, 0, 0}};

// the receiving block's direction for a message sent across face d of
// block b (CubedSphere::TransformOX, cs_transform_ox.cpp:11-230); -1 marks
// a neighbour inside the 2 x 3 block layout, which receives on the face
// opposite to d
int receive_dir(int b, int d) {
  static const int rx[6][4] = {
      // d = 0 (ox2-)  1 (ox2+)  2 (ox3-)  3 (ox3+)
      {0, -1, 0, 0},   // block 1
      {-1, 0, 3, -1},  // block 2
      {2, 2, 3, 2},    // block 3
      {3, 3, -1, -1},  // block 4
      {1, 1, 1, 1},    // block 5
      {0, 1, -1, 2},   // block 6
  };
  const int r = rx[b - 1][d];
  return r >= 0 ? r : (d ^ 1);
}

double interp_location(int loc_n, int nblk, int k, bool ghost) {
  // CalculateInterpLocations (cubed_sphere_utility.cpp:78-98)
  double t0 = std::tan((double)1.0 * (nblk - 1 - 2 * k) / (nblk * 4) * kPi);
  if (ghost) t0 = 1.0 / t0;
  t0 = 1.0 + t0 * t0;
  const double t = std::pow(std::tan((double)1.0 * (2 * loc_n + 1) / (nblk * 4) * kPi), 2.0);
  const double a = std::acos(std::sqrt(t0 / (t0 + t)));
  return loc_n < 0 ? -a : a;
}

// 2 x 2 matrices of the velocity maps
struct Mat2 {
  double a[2][2];
};
Mat2 mat_mul(const Mat2 &x, const Mat2 &y) {
  Mat2 r;
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j) r.a[i][j] = x.a[i][0] * y.a[0][j] + x.a[i][1] * y.a[1][j];
  return r;
}

// (V2, V3) -> (U, V) at gnomonic point (X, Y) of block b
// (VecTransRLLFromABP, cubed_sphere_transform.cpp:37-61)
Mat2 rll_from_abp(double X, double Y, int b) {
  const double C = std::sqrt(1 + X * X), D = std::sqrt(1 + Y * Y);
  const double E = std::sqrt(X * X + Y * Y), del = std::sqrt(1 + X * X + Y * Y);
  Mat2 m{};
  if (b == 1) {
    m.a[0][0] = -del * Y / (D * E);
    m.a[0][1] = del * X / (C * E);
    m.a[1][0] = -X / (D * E);
    m.a[1][1] = -Y / (C * E);
  } else if (b == 5) {
    m.a[0][0] = del * Y / (D * E);
    m.a[0][1] = -del * X / (C * E);
    m.a[1][0] = X / (D * E);
    m.a[1][1] = Y / (C * E);
  } else {
    m.a[0][0] = 0.;
    m.a[0][1] = del / (C * D);
    m.a[1][0] = -1.;
    m.a[1][1] = X * Y / (C * D);
  }
  return m;
}

// (U, V) -> (V2, V3) (VecTransABPFromRLL, cubed_sphere_transform.cpp:11-35)
Mat2 abp_from_rll(double X, double Y, int b) {
  const double C = std::sqrt(1 + X * X), D = std::sqrt(1 + Y * Y);
  const double E = std::sqrt(X * X + Y * Y), del = std::sqrt(1 + X * X + Y * Y);
  Mat2 m{};
  if (b == 1) {
    m.a[0][0] = -D * Y / (del * E);
    m.a[0][1] = -D * X / E;
    m.a[1][0] = C * X / (del * E);
    m.a[1][1] = -C * Y / E;
  } else if (b == 5) {
    m.a[0][0] = D * Y / (del * E);
    m.a[0][1] = D * X / E;
    m.a[1][0] = -C * X / (del * E);
    m.a[1][1] = C * Y / E;
  } else {
    m.a[0][0] = X * Y / del;
    m.a[0][1] = -1.;
    m.a[1][0] = C * D / del;
    m.a[1][1] = 0.;
  }
  return m;
}

// covariant -> contravariant at (X, Y) and back
Mat2 raise_at(double X, double Y) {
  const double s = std::sqrt(1 + X * X + Y * Y) / std::sqrt(1 + X * X) / std::sqrt(1 + Y * Y);
  const double c = -X * Y / std::sqrt(1 + X * X) / std::sqrt(1 + Y * Y);
  return Mat2{{{1. / (s * s), -c / (s * s)}, {-c / (s * s), 1. / (s * s)}}};
}
Mat2 lower_at(double X, double Y) {
  const double c = -X * Y / std::sqrt(1 + X * X) / std::sqrt(1 + Y * Y);
  return Mat2{{{1., c}, {c, 1.}}};
}

// ---------------------------------------------------------------------------
// table rows

struct GhostRow {
  int dst, dk, dj;          // target panel and ghost cell (k, j)
  int src, k1, j1, k2, j2;  // source panel and the two interpolation cells
  double a, b, d;           // value = (a v1 + b v2) / d
  double m[2][2];           // (IVY, IVZ) map, after interpolation
};

struct EdgeRow {
  int src, sdir, spos;  // source panel, its edge and position along it
  int dst, ddir, dpos;  // receiving panel, edge and position
  double m[2][2];       // (IVY, IVZ) map
};

// one ghost-table row per target ghost cell of the four face slabs
std::vector<GhostRow> build_ghost_table(int N) {
  const int NGh = NG, js = NG, je = NG + N - 1, ks = NG, ke = NG + N - 1;
  std::vector<GhostRow> rows;
  std::vector<double> src_x(N), src_coord(N), tgt_x(N);
  for (int m = 0; m < N; ++m) src_coord[m] = kPi / 2.0 / N * (m + 0.5) - kPi / 4.0;
  for (int p = 0; p < 6; ++p) {
    const int b = p + 1;
    for (int d = 0; d < 4; ++d) {
      const int ox2 = d == 0 ? -1 : d == 1 ? 1 : 0, ox3 = d == 2 ? -1 : d == 3 ? 1 : 0;
      const bool along_j = ox3 != 0;  // x3 face: interpolate along j
      // the sender's region: NGHOST layers x N along the edge
      const int sj = ox2 > 0 ? je - NGh + 1 : js, ej = ox2 < 0 ? js + NGh - 1 : je;
      const int sk = ox3 > 0 ? ke - NGh + 1 : ks, ek = ox3 < 0 ? ks + NGh - 1 : ke;
      const int dk = ek - sk + 1, dj = ej - sj + 1;
      const bool lower = (ox2 < 0 || ox3 < 0);
      const int tgt = kTgbid[p][d] - 1, tdir = receive_dir(b, d);
      const int dinv = kDinv[p][d], tside = kTgside[p][d];
      // receiving slab
      const int rox2 = tdir == 0 ? -1 : tdir == 1 ? 1 : 0, rox3 = tdir == 2 ? -1 : tdir == 3 ? 1 : 0;
      const int tsj = rox2 == 0 ? js : (rox2 > 0 ? je + 1 : js - NGh);
      const int tej = rox2 == 0 ? je : (rox2 > 0 ? je + NGh : js - 1);
      const int tsk = rox3 == 0 ? ks : (rox3 > 0 ? ke + 1 : ks - NGh);
      const int tnj = tej - tsj + 1;
      // buffer position of the region element (kk, jj) in the pack order
      const int order = kOrder[p][d];
      auto pos_of = [&](int kk, int jj) {
        switch (order) {
          case 0: return kk * dj + jj;
          case 1: return (dj - 1 - jj) * dk + kk;
          case 2: return (dk - 1 - kk) * dj + (dj - 1 - jj);
          default: return jj * dk + (dk - 1 - kk);
        }
      };
      for (int kk = 0; kk < dk; ++kk)
        for (int jj = 0; jj < dj; ++jj) {
          const int layer = along_j ? (lower ? kk : dk - 1 - kk) : (lower ? jj : dj - 1 - jj);
          const int t = along_j ? jj : kk;  // index along the edge
          for (int m = 0; m < N; ++m) src_x[m] = interp_location(m - N / 2, N, layer, false);
          const double yq = interp_location(-N / 2 + t, N, layer, true);
          int sp = 0;
          while (sp + 2 < N && yq > src_x[sp + 1]) ++sp;
          const double y1 = src_x[sp], y2 = src_x[sp + 1];
          GhostRow r{};
          const int q = pos_of(kk, jj);
          r.dst = tgt;
          r.dk = tsk + q / tnj;
          r.dj = tsj + q % tnj;
          r.src = p;
          if (along_j) {
            r.k1 = r.k2 = sk + kk;
            r.j1 = sj + sp;
            r.j2 = sj + sp + 1;
          } else {
            r.j1 = r.j2 = sj + jj;
            r.k1 = sk + sp;
            r.k2 = sk + sp + 1;
          }
          r.a = y2 - yq;
          r.b = yq - y1;
          r.d = y2 - y1;
          // velocity map: raise at the source point, through lat-lon into
          // the target block, lower at the target point
          const double tc = dinv == 1 ? -src_coord[t] : src_coord[t];
          const double perp_t = std::tan(tside * (kPi / 2.0 / N * (layer + 0.5) + kPi / 4.0));
          const double perp_s =
              std::tan((lower ? -1 : 1) * (-kPi / 2.0 / N * (layer + 0.5) + kPi / 4.0));
          const double along_s =
              std::tan((r.a * src_coord[sp] + r.b * src_coord[sp + 1]) / r.d);
          double scy, scz, tcy, tcz;
          if (along_j) {
            scy = along_s;
            scz = perp_s;
            tcy = std::tan(tc);
            tcz = perp_t;
          } else {
            scz = along_s;
            scy = perp_s;
            tcz = std::tan(tc);
            tcy = perp_t;
            const int tb = tgt + 1;
            if (((tb == 1 || tb == 5) && (b == 3 || b == 4)) ||
                ((tb == 3 || tb == 4) && (b == 1 || b == 5))) {
              const double x = tcy;
              tcy = tcz;
              tcz = x;
            }
          }
          const Mat2 mm = mat_mul(lower_at(tcy, tcz),
                                  mat_mul(abp_from_rll(tcy, tcz, tgt + 1),
                                          mat_mul(rll_from_abp(scy, scz, b), raise_at(scy, scz))));
          std::memcpy(r.m, mm.a, sizeof(r.m));
          rows.push_back(r);
        }
    }
  }
  return rows;
}

// one edge-table row per face along every panel edge
std::vector<EdgeRow> build_edge_table(int N) {
  std::vector<EdgeRow> rows;
  std::vector<double> cv(N);
  for (int m = 0; m < N; ++m) cv[m] = -kPi / 4. + (m + 0.5) * kPi / 2. / N;
  for (int p = 0; p < 6; ++p) {
    const int b = p + 1;
    for (int d = 0; d < 4; ++d) {
      const int tgt = kTgbid[p][d] - 1, tdir = receive_dir(b, d);
      const bool inv = kDinv[p][d] == 1;
      for (int t = 0; t < N; ++t) {
        EdgeRow r{};
        r.src = p;
        r.sdir = d;
        r.spos = inv ? N - 1 - t : t;  // the sender walks its edge backwards
        r.dst = tgt;
        r.ddir = tdir;
        r.dpos = t;
        const double along = cv[r.spos];
        double x2s, x3s;
        if (d == 0) { x2s = -kPi / 4.; x3s = along; }
        else if (d == 1) { x2s = kPi / 4.; x3s = along; }
        else if (d == 2) { x2s = along; x3s = -kPi / 4.; }
        else { x2s = along; x3s = kPi / 4.; }
        const double pa = inv ? -along : along;
        double x2d, x3d;
        if (tdir == 0) { x2d = -kPi / 4.; x3d = pa; }
        else if (tdir == 1) { x2d = kPi / 4.; x3d = pa; }
        else if (tdir == 2) { x2d = pa; x3d = -kPi / 4.; }
        else { x2d = pa; x3d = kPi / 4.; }
        const Mat2 mm = mat_mul(abp_from_rll(std::tan(x2d), std::tan(x3d), tgt + 1),
                                rll_from_abp(std::tan(x2s), std::tan(x3s), b));
        std::memcpy(r.m, mm.a, sizeof(r.m));
        rows.push_back(r);
      }
    }
  }
  return rows;
}

// geometry tables (gnomonic_equiangle.cpp:140-198) and the flux-projection
// cosines of hllc_transform.cpp:249-263
std::vector<double> build_geometry(int N) {
  const int nc = N + 2 * NG;
  std::vector<double> xf(nc + 1), xv(nc);
  for (int j = 0; j <= nc; ++j) xf[j] = -kPi / 4. + (j - NG) * (kPi / 2. / N);
  for (int j = 0; j < nc; ++j) xv[j] = 0.5 * (xf[j + 1] + xf[j]);
  const size_t nkj = (size_t)nc * nc;
  std::vector<double> t(kShellTabs * nkj);
  auto at = [&](int tb, int k, int j) -> double & { return t[tb * nkj + (size_t)k * nc + j]; };
  for (int k = 0; k < nc; ++k)
    for (int j = 0; j < nc; ++j) {
      const double x = std::tan(xv[j]), xfj = std::tan(xf[j]);
      const double y = std::tan(xv[k]), yfk = std::tan(xf[k]);
      const double C = std::sqrt(1.0 + x * x), Cf = std::sqrt(1.0 + xfj * xfj);
      const double D = std::sqrt(1.0 + y * y), Df = std::sqrt(1.0 + yfk * yfk);
      at(kTabCosC, k, j) = -x * y / (C * D);
      at(kTabSinC, k, j) = std::sqrt(1.0 + x * x + y * y) / (C * D);
      at(kTabCosF2, k, j) = -xfj * y / (Cf * D);
      at(kTabSinF2, k, j) = std::sqrt(1.0 + xfj * xfj + y * y) / (Cf * D);
      at(kTabCosF3, k, j) = -x * yfk / (C * Df);
      at(kTabSinF3, k, j) = std::sqrt(1.0 + x * x + yfk * yfk) / (C * Df);
      const double x1 = std::tan(xf[j]), x2 = std::tan(xf[j + 1]);
      double d1 = std::sqrt(1.0 + x1 * x1 + y * y), d2 = std::sqrt(1.0 + x2 * x2 + y * y);
      at(kTabDx2A, k, j) = std::acos((1 + x1 * x2 + y * y) / (d1 * d2));
      d1 = std::sqrt(1.0 + x1 * x1 + yfk * yfk);
      d2 = std::sqrt(1.0 + x2 * x2 + yfk * yfk);
      at(kTabDx2AF3, k, j) = std::acos((1 + x1 * x2 + yfk * yfk) / (d1 * d2));
      const double y1 = std::tan(xf[k]), y2 = std::tan(xf[k + 1]);
      d1 = std::sqrt(1.0 + x * x + y1 * y1);
      d2 = std::sqrt(1.0 + x * x + y2 * y2);
      at(kTabDx3A, k, j) = std::acos((1 + x * x + y1 * y2) / (d1 * d2));
      d1 = std::sqrt(1.0 + xfj * xfj + y1 * y1);
      d2 = std::sqrt(1.0 + xfj * xfj + y2 * y2);
      at(kTabDx3AF2, k, j) = std::acos((1 + xfj * xfj + y1 * y2) / (d1 * d2));
      at(kTabCth1, k, j) = -x * y / std::sqrt(1. + x * x) / std::sqrt(1. + y * y);
      at(kTabCth2, k, j) = -xfj * y / std::sqrt(1. + xfj * xfj) / std::sqrt(1. + y * y);
      at(kTabCth3, k, j) = -x * yfk / std::sqrt(1. + x * x) / std::sqrt(1. + yfk * yfk);
    }
  return t;
}

// ---------------------------------------------------------------------------
// kernels (dry: NV = 5, slots IDN 0, IVX 1, IVY 2, IVZ 3, IPR 4)

constexpr int kNV = 5;

__global__ void k_shell_ghosts(double *__restrict__ u, const GhostRow *__restrict__ rows,
                               int nrows, Geom g, int64_t pvals) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)nrows * g.nx1) return;
  const GhostRow r = rows[t / g.nx1];
  const int i = g.is + (int)(t % g.nx1);
  const double *s = u + r.src * pvals;
  double *o = u + r.dst * pvals;
  const int64_t c1 = (int64_t)r.k1 * g.sk + (int64_t)r.j1 * g.nc1 + i;
  const int64_t c2 = (int64_t)r.k2 * g.sk + (int64_t)r.j2 * g.nc1 + i;
  const int64_t co = (int64_t)r.dk * g.sk + (int64_t)r.dj * g.nc1 + i;
  double v[kNV];
#pragma unroll
  for (int n = 0; n < kNV; ++n) v[n] = (r.a * s[n * g.sv + c1] + r.b * s[n * g.sv + c2]) / r.d;
  const double vy = v[2], vz = v[3];
  v[2] = r.m[0][0] * vy + r.m[0][1] * vz;
  v[3] = r.m[1][0] * vy + r.m[1][1] * vz;
#pragma unroll
  for (int n = 0; n < kNV; ++n) o[n * g.sv + co] = v[n];
}

// cons -> prim of the interior and the four face ghost slabs of every panel
// (corners are not filled), x1 ghosts by the radial boundary condition
__global__ void k_shell_c2p(const double *__restrict__ u, double *__restrict__ w, Geom g,
                            double gm1, int64_t pvals, uint32_t *err) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t ncol = (int64_t)g.nc3 * g.nc2;
  if (t >= 6 * ncol * g.nx1) return;
  const int i = g.is + (int)(t % g.nx1);
  const int64_t col = t / g.nx1;
  const int p = (int)(col / ncol);
  const int kj = (int)(col % ncol);
  const int k = kj / g.nc2, j = kj % g.nc2;
  const bool kin = k >= g.ks && k <= g.ke, jin = j >= g.js && j <= g.je;
  if (!kin && !jin) return;
  const int64_t nkj = ncol;
  const double cth = g.shell[kTabCosC * nkj + kj];
  const int64_t c = p * pvals + (int64_t)k * g.sk + (int64_t)j * g.nc1;
  const double u_d = u[c + i], u_m1 = u[g.sv + c + i], u_m2 = u[2 * g.sv + c + i],
               u_m3 = u[3 * g.sv + c + i], u_e = u[4 * g.sv + c + i];
  const double di = 1.0 / u_d;
  double v1 = u_m1 * di, v2 = u_m2 * di, v3 = u_m3 * di;
  const double sth2 = 1. - cth * cth;
  const double a = v2, b = v3;
  v2 = a / sth2 - b * cth / sth2;
  v3 = -a * cth / sth2 + b / sth2;
  const double e_k = 0.5 * (u_m1 * v1 + u_m2 * v2 + u_m3 * v3);
  const double pr = gm1 * (u_e - e_k);
  const double wv[kNV] = {u_d, v1, v2, v3, pr};
  uint32_t bits = 0;
  if (!(u_d > 0.)) bits |= CANOE_EBIT_NEG_DENSITY;
  if (!(pr > 0.)) bits |= CANOE_EBIT_NEG_PRESSURE;
  if (!isfinite(pr) || !isfinite(v1) || !isfinite(v2) || !isfinite(v3)) bits |= CANOE_EBIT_NAN;
  if (bits && err) atomicOr(err, bits);
#pragma unroll
  for (int n = 0; n < kNV; ++n) w[n * g.sv + c + i] = wv[n];
  // x1 ghosts: the mirror images of this cell
  const int gl = i - g.is + 1, gu = g.ie - i + 1;  // 1-based depth from each wall
  if (gl <= NG) {
    const bool refl = g.bc[0] == CANOE_BC_REFLECT;
    if (refl) {
#pragma unroll
      for (int n = 0; n < kNV; ++n) w[n * g.sv + c + g.is - gl] = (n == 1 ? -wv[n] : wv[n]);
    } else if (gl == 1) {
      for (int q = 1; q <= NG; ++q)
#pragma unroll
        for (int n = 0; n < kNV; ++n) w[n * g.sv + c + g.is - q] = wv[n];
    }
  }
  if (gu <= NG) {
    const bool refl = g.bc[1] == CANOE_BC_REFLECT;
    if (refl) {
#pragma unroll
      for (int n = 0; n < kNV; ++n) w[n * g.sv + c + g.ie + gu] = (n == 1 ? -wv[n] : wv[n]);
    } else if (gu == 1) {
      for (int q = 1; q <= NG; ++q)
#pragma unroll
        for (int n = 0; n < kNV; ++n) w[n * g.sv + c + g.ie + q] = wv[n];
    }
  }
}

// interior-side face states of the panel edges, rotated into the receiving
// panel's frame; lr layout [panel][edge][pos][n][i - is].  R = float: the
// FP32 path, reconstructed on p' = p - pref(i) as its flux kernel does.
template <int RECON, typename R>
__global__ void k_shell_edges(const double *__restrict__ w, const EdgeRow *__restrict__ rows,
                              int nrows, Geom g, int64_t pvals, double *__restrict__ lr) {
  constexpr bool PERT = sizeof(R) == 4;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)nrows * g.nx1) return;
  const EdgeRow r = rows[t / g.nx1];
  const int ii = (int)(t % g.nx1), i = g.is + ii;
  const double *s = w + r.src * pvals;
  // the cell next to the edge and the stride across it
  int64_t c0, sd;
  const bool up = (r.sdir & 1) != 0;
  if (r.sdir < 2) {  // x2 edge at row k = spos
    const int j = up ? g.je : g.js;
    c0 = (int64_t)(g.ks + r.spos) * g.sk + (int64_t)j * g.nc1 + i;
    sd = g.nc1;
  } else {  // x3 edge at column j = spos
    const int k = up ? g.ke : g.ks;
    c0 = (int64_t)k * g.sk + (int64_t)(g.js + r.spos) * g.nc1 + i;
    sd = g.sk;
  }
  const double pref = PERT ? g.pref[i] : 0.;
  R v[kNV];
#pragma unroll
  for (int n = 0; n < kNV; ++n) {
    const double *q = s + n * g.sv + c0;
    const double sh = (PERT && n == 4) ? pref : 0.;
    R wL, wR;
    if constexpr (RECON == CANOE_RECON_PPM)
      ppm_cell(R(q[-2 * sd] - sh), R(q[-sd] - sh), R(q[0] - sh), R(q[sd] - sh),
               R(q[2 * sd] - sh), wL, wR);
    else
      plm_cell(R(q[-sd] - sh), R(q[0] - sh), R(q[sd] - sh), wL, wR);
    v[n] = up ? wR : wL;
  }
  const R vy = v[2], vz = v[3];
  v[2] = R(r.m[0][0]) * vy + R(r.m[0][1]) * vz;
  v[3] = R(r.m[1][0]) * vy + R(r.m[1][1]) * vz;
  const int N = g.nx2;
  double *o = lr + ((((int64_t)r.dst * 4 + r.ddir) * N + r.dpos) * kNV) * g.nx1 + ii;
#pragma unroll
  for (int n = 0; n < kNV; ++n) o[(int64_t)n * g.nx1] = (double)v[n];
}

constexpr int TI = 32, TD = 8;

// the x2 (DIR 1) / x3 (DIR 2) flux at the face of table index kj from its
// left / right states (overwritten): PrimToLocal2/3, HLLC, FluxToGlobal2/3
// and the covariant projection
template <int DIR, typename R>
__device__ __forceinline__ void shell_face_flux(const Geom &g, const canoe_thermo_t &th,
                                                R *wl, R *wr, double pref, int64_t kj,
                                                int64_t nkj, double *fx) {
  constexpr bool PERT = sizeof(R) == 4;
  R fr[kNV];
  if (DIR == 1) {
    // PrimToLocal2 with Face2Metric: T22 = 1/sqrt(gi22), T32 = g23/sqrt(g33)
    const double ct = g.shell[kTabCosF2 * nkj + kj], st = g.shell[kTabSinF2 * nkj + kj];
    const double gi22 = 1.0 / (st * st);
    const double T22 = 1.0 / sqrt(gi22), T32 = ct / sqrt(1.0), T33 = sqrt(1.0);
    auto loc = [&](R *x) {
      const R u2 = x[2], u3 = x[3];
      x[2] = R(T22) * u2;
      x[3] = R(T32) * u2 + R(T33) * u3;
    };
    loc(wl);
    loc(wr);
    if constexpr (PERT)
      hllc_pert<R, 0, 1>(th, wl, wr, R(pref), fr);
    else
      hllc<R, 0, 1>(th, wl, wr, fr);
#pragma unroll
    for (int n = 0; n < kNV; ++n) fx[n] = fr[n];
    if (PERT) fx[2] += pref;
    const double F22 = sqrt(gi22), F32 = -sqrt(gi22) * ct / 1.0, F33 = 1.0 / sqrt(1.0);
    const double txy = fx[2], txz = fx[3];
    fx[2] = F22 * txy;
    fx[3] = F32 * txy + F33 * txz;
    const double cth = g.shell[kTabCth2 * nkj + kj];
    const double ty_ = fx[2], tz_ = fx[3];
    fx[2] = ty_ + tz_ * cth;
    fx[3] = tz_ + ty_ * cth;
  } else {
    // PrimToLocal3 with Face3Metric: T22 = sqrt(g22), T23 = g23/sqrt(g22),
    // T33 = 1/sqrt(gi33)
    const double ct = g.shell[kTabCosF3 * nkj + kj], st = g.shell[kTabSinF3 * nkj + kj];
    const double gi33 = 1.0 / (st * st);
    const double T22 = sqrt(1.0), T23 = ct / sqrt(1.0), T33 = 1.0 / sqrt(gi33);
    auto loc = [&](R *x) {
      const R u2 = x[2], u3 = x[3];
      x[2] = R(T22) * u2 + R(T23) * u3;
      x[3] = R(T33) * u3;
    };
    loc(wl);
    loc(wr);
    if constexpr (PERT)
      hllc_pert<R, 0, 2>(th, wl, wr, R(pref), fr);
    else
      hllc<R, 0, 2>(th, wl, wr, fr);
#pragma unroll
    for (int n = 0; n < kNV; ++n) fx[n] = fr[n];
    if (PERT) fx[3] += pref;
    const double F22 = 1.0 / sqrt(1.0), F23 = -ct / 1.0 * sqrt(gi33), F33 = sqrt(gi33);
    const double txy = fx[2], txz = fx[3];
    fx[2] = F22 * txy + F23 * txz;
    fx[3] = F33 * txz;
    const double cth = g.shell[kTabCth3 * nkj + kj];
    const double ty_ = fx[2], tz_ = fx[3];
    fx[2] = ty_ + tz_ * cth;
    fx[3] = tz_ + ty_ * cth;
  }
}

// x2 (DIR 1) / x3 (DIR 2) fluxes and their divergence on (32 i) x (8 cells)
// tiles; blockIdx.z runs over panel x rows.  R = float: reconstruction and
// the Riemann solver in FP32 on p' = p - pref(i); the metric transforms, the
// projection and the divergence stay FP64, with pref added back to the
// normal momentum flux before them (the transforms mix it into the
// transverse components, and face areas differ across a cell).
// FP32 tiles: four CTAs per SM (64 registers); FP64: two
template <int RECON, int DIR, bool WF, typename R>
__global__ void __launch_bounds__(256, sizeof(R) == 4 ? 4 : 2)
    k_shell_flux_x23(Geom g, canoe_thermo_t th, const double *__restrict__ w,
                     double *__restrict__ du, const double *__restrict__ dtp, double beta,
                     int64_t pvals, const double *__restrict__ lr, double *__restrict__ fout) {
  constexpr int QR = TD + 2 * NG, RR = TD + 2;
  constexpr bool PERT = sizeof(R) == 4;
  extern __shared__ double sm_[];
  R *smr = reinterpret_cast<R *>(sm_);
  R(*q)[QR][TI] = reinterpret_cast<R(*)[QR][TI]>(smr);
  R(*WL)[RR][TI] = reinterpret_cast<R(*)[RR][TI]>(smr + kNV * QR * TI);
  R(*WR)[RR][TI] = reinterpret_cast<R(*)[RR][TI]>(smr + kNV * (QR + RR) * TI);
  // FP64 fluxes: over q (FP64 path, P1 reads q last) or after WR (FP32)
  double(*F)[TD + 1][TI] = reinterpret_cast<double(*)[TD + 1][TI]>(
      PERT ? reinterpret_cast<double *>(smr + kNV * (QR + 2 * RR) * TI) : sm_);
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i = g.is + blockIdx.x * TI + tx;
  const bool iok = i <= g.ie;
  const int N = g.nx2;
  const int no = N;
  const int p = blockIdx.z / no;
  const int o = (DIR == 1 ? g.ks : g.js) + (int)(blockIdx.z % no);
  const int dlo = DIR == 1 ? g.js : g.ks, dhi = DIR == 1 ? g.je : g.ke;
  const int d0 = dlo + blockIdx.y * TD;
  const int nd = min(TD, dhi - d0 + 1);
  const int64_t sd = DIR == 1 ? g.nc1 : g.sk;
  const int64_t pb = p * pvals;
  const int64_t base = (DIR == 1 ? (int64_t)o * g.sk : (int64_t)o * g.nc1) + i;
  const int64_t nkj = (int64_t)g.nc3 * g.nc2;
  const double pref = PERT ? g.pref[iok ? i : g.is] : 0.;
  // x3 adds to the du of the x2 pass: this thread's du values are loaded at
  // entry so that their latency hides behind the reconstruction
  double dpre[kNV];
  if (DIR == 2 && iok && ty < nd && blockDim.y >= TD) {
    const int64_t off = pb + base + (int64_t)(d0 + ty) * sd;
#pragma unroll
    for (int n = 0; n < kNV; ++n) dpre[n] = du[n * g.sv + off];
  }
  for (int c = ty; c < nd + 2 * NG; c += blockDim.y) {
    const int64_t off = pb + base + (int64_t)(d0 - NG + c) * sd;
#pragma unroll
    for (int n = 0; n < kNV; ++n) {
      double v = iok ? w[n * g.sv + off] : 1.;
      if (PERT && n == 4) v = iok ? v - pref : 0.;
      q[n][c][tx] = R(v);
    }
  }
  __syncthreads();
  for (int c = ty; c < nd + 2; c += blockDim.y) {
#pragma unroll
    for (int n = 0; n < kNV; ++n) {
      R wl_, wr_;
      if constexpr (RECON == CANOE_RECON_PPM)
        ppm_cell(q[n][c][tx], q[n][c + 1][tx], q[n][c + 2][tx], q[n][c + 3][tx],
                 q[n][c + 4][tx], wl_, wr_);
      else
        plm_cell(q[n][c + 1][tx], q[n][c + 2][tx], q[n][c + 3][tx], wl_, wr_);
      WL[n][c][tx] = wl_;
      WR[n][c][tx] = wr_;
    }
  }
  __syncthreads();
  for (int f = ty; f <= nd; f += blockDim.y) {
    const int fd = d0 + f;
    R wl[kNV], wr[kNV];
    double fx[kNV];
#pragma unroll
    for (int n = 0; n < kNV; ++n) {
      wl[n] = WR[n][f][tx];
      wr[n] = WL[n][f + 1][tx];
    }
    // panel edges: the ghost side is the neighbour's swapped state
    const int pos = o - (DIR == 1 ? g.ks : g.js);
    if (iok && fd == dlo) {
      const double *s = lr + ((((int64_t)p * 4 + (DIR == 1 ? 0 : 2)) * N + pos) * kNV) * g.nx1 +
                        (i - g.is);
#pragma unroll
      for (int n = 0; n < kNV; ++n) wl[n] = R(s[(int64_t)n * g.nx1]);
    }
    if (iok && fd == dhi + 1) {
      const double *s = lr + ((((int64_t)p * 4 + (DIR == 1 ? 1 : 3)) * N + pos) * kNV) * g.nx1 +
                        (i - g.is);
#pragma unroll
      for (int n = 0; n < kNV; ++n) wr[n] = R(s[(int64_t)n * g.nx1]);
    }
    const int kf = DIR == 1 ? o : fd, jf = DIR == 1 ? fd : o;
    const int64_t kj = (int64_t)kf * g.nc2 + jf;
    shell_face_flux<DIR, R>(g, th, wl, wr, pref, kj, nkj, fx);
#pragma unroll
    for (int n = 0; n < kNV; ++n) F[n][f][tx] = fx[n];
    if constexpr (WF) {
      if (iok) {
#pragma unroll
        for (int n = 0; n < kNV; ++n) {
          const int64_t idx =
              DIR == 1 ? (((int64_t)(p * kNV + n) * g.nc3 + o) * (g.nc2 + 1) + fd) * g.nc1 + i
                       : (((int64_t)(p * kNV + n) * (g.nc3 + 1) + fd) * g.nc2 + o) * g.nc1 + i;
          fout[idx] = fx[n];
        }
      }
    }
  }
  __syncthreads();
  if (!iok) return;
  const double wght = beta * dtp[0];
  const double xv = g.x1v[i], df = g.dx1f[i];
  for (int c = ty; c < nd; c += blockDim.y) {
    const int dc = d0 + c;
    const int kc = DIR == 1 ? o : dc, jc = DIR == 1 ? dc : o;
    const int64_t kj = (int64_t)kc * g.nc2 + jc;
    const double d2 = g.shell[kTabDx2A * nkj + kj], d3 = g.shell[kTabDx3A * nkj + kj];
    const double vol = df * d2 * d3 * xv * xv * g.shell[kTabSinC * nkj + kj];
    double am, ap;
    if (DIR == 1) {
      am = xv * g.shell[kTabDx3AF2 * nkj + kj] * df;
      ap = xv * g.shell[kTabDx3AF2 * nkj + kj + 1] * df;
    } else {
      am = xv * g.shell[kTabDx2AF3 * nkj + kj] * df;
      ap = xv * g.shell[kTabDx2AF3 * nkj + kj + g.nc2] * df;
    }
    const int64_t off = pb + base + (int64_t)dc * sd;
#pragma unroll
    for (int n = 0; n < kNV; ++n) {
      const double dfl = ap * F[n][c + 1][tx] - am * F[n][c][tx];
      if (DIR == 1)
        du[n * g.sv + off] = -(wght * dfl / vol);
      else if (blockDim.y >= TD)
        du[n * g.sv + off] = dpre[n] - wght * dfl / vol;  // c == ty: the prefetched cell
      else
        du[n * g.sv + off] -= wght * dfl / vol;
    }
  }
}

// The same fluxes with one thread per (i, o, run of SRL cells) marching
// along the flux direction with its stencil in registers, as
// k_flux_x23_run in flux.cu: each step reconstructs one cell (PPM slopes
// and interface values streamed once per cell), takes the swapped state at
// a panel edge, computes the flux at the cell's lower face and finishes the
// divergence of the cell below.  blockIdx.z runs over panel x runs.  Same
// expressions on the same operands as the tile kernel: the same bits.
constexpr int SRL = 16;  // cells per run
constexpr int SBY = 4;   // orthogonal lines per CTA

template <int RECON, int DIR, bool WF, typename R>
__global__ void __launch_bounds__(32 * SBY)
    k_shell_flux_x23_run(Geom g, canoe_thermo_t th, const double *__restrict__ w,
                         double *__restrict__ du, const double *__restrict__ dtp, double beta,
                         int64_t pvals, const double *__restrict__ lr,
                         double *__restrict__ fout) {
  constexpr bool PERT = sizeof(R) == 4;
  const int N = g.nx2;
  const int nrun = (N + SRL - 1) / SRL;
  const int p = blockIdx.z / nrun;
  const int i = g.is + blockIdx.x * 32 + threadIdx.x;
  const int o = (DIR == 1 ? g.ks : g.js) + blockIdx.y * SBY + threadIdx.y;
  if (i > g.ie || o > (DIR == 1 ? g.ke : g.je)) return;
  const int dlo = DIR == 1 ? g.js : g.ks, dhi = DIR == 1 ? g.je : g.ke;
  const int s0 = dlo + (int)(blockIdx.z % nrun) * SRL;
  const int s1 = min(s0 + SRL, dhi + 1);  // one past the run's last cell
  const int64_t sd = DIR == 1 ? g.nc1 : g.sk;
  const int64_t pb = p * pvals;
  const int64_t base = pb + (DIR == 1 ? (int64_t)o * g.sk : (int64_t)o * g.nc1) + i;
  const int64_t nkj = (int64_t)g.nc3 * g.nc2;
  const double pref = PERT ? g.pref[i] : 0.;
  const double wght = beta * dtp[0];
  const double xv = g.x1v[i], df = g.dx1f[i];
  const int pos = o - (DIR == 1 ? g.ks : g.js);
  constexpr int H = RECON == CANOE_RECON_PPM ? 2 : 1;

  R q[3][kNV];  // PLM: cells c-1, c, c+1; PPM: c, c+1, c+2
  R sl[kNV], fl[kNV];
  double nx[kNV];
  auto fetch = [&](int c) {
    const int64_t off = base + (int64_t)c * sd;
#pragma unroll
    for (int n = 0; n < kNV; ++n) nx[n] = w[n * g.sv + off];
  };
  auto put = [&](R *qm) {
#pragma unroll
    for (int n = 0; n < kNV; ++n) {
      double v = nx[n];
      if (PERT && n == 4) v -= pref;
      qm[n] = R(v);
    }
  };
  if constexpr (RECON == CANOE_RECON_PPM) {
    R qa[kNV], qb[kNV];
    fetch(s0 - 3);
    put(qa);
    fetch(s0 - 2);
    put(qb);
    fetch(s0 - 1);
    put(q[0]);
    fetch(s0);
    put(q[1]);
#pragma unroll
    for (int n = 0; n < kNV; ++n) {
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
  R wrp[kNV];
  double fp[kNV], dpre[kNV];
  double amp = 0.;  // lower-face area of the cell below the current face
  for (int c = s0 - 1; c <= s1; ++c) {
    put(q[2]);
    if (c < s1) fetch(c + H + 1);  // one step ahead
    if (DIR == 2 && c > s0) {
      const int64_t off = base + (int64_t)(c - 1) * sd;
#pragma unroll
      for (int n = 0; n < kNV; ++n) dpre[n] = du[n * g.sv + off];
    }
    R wlc[kNV], wrc[kNV];
#pragma unroll
    for (int n = 0; n < kNV; ++n) {
      if constexpr (RECON == CANOE_RECON_PPM) {
        const R sr = ppm_slope(q[0][n], q[1][n], q[2][n]);
        const R fr = ppm_face(q[0][n], q[1][n], sl[n], sr);
        wlc[n] = fl[n];
        wrc[n] = fr;
        ppm_limit(q[0][n], wlc[n], wrc[n]);
        sl[n] = sr;
        fl[n] = fr;
      } else {
        plm_cell(q[0][n], q[1][n], q[2][n], wlc[n], wrc[n]);
      }
    }
    if (c >= s0) {
      // face c: left = wR of cell c-1, right = wL of cell c; at a panel edge
      // the ghost side is the neighbour's swapped state
      R wl[kNV], wr[kNV];
#pragma unroll
      for (int n = 0; n < kNV; ++n) {
        wl[n] = wrp[n];
        wr[n] = wlc[n];
      }
      if (c == dlo) {
        const double *s = lr + ((((int64_t)p * 4 + (DIR == 1 ? 0 : 2)) * N + pos) * kNV) * g.nx1 +
                          (i - g.is);
#pragma unroll
        for (int n = 0; n < kNV; ++n) wl[n] = R(s[(int64_t)n * g.nx1]);
      }
      if (c == dhi + 1) {
        const double *s = lr + ((((int64_t)p * 4 + (DIR == 1 ? 1 : 3)) * N + pos) * kNV) * g.nx1 +
                          (i - g.is);
#pragma unroll
        for (int n = 0; n < kNV; ++n) wr[n] = R(s[(int64_t)n * g.nx1]);
      }
      const int kf = DIR == 1 ? o : c, jf = DIR == 1 ? c : o;
      const int64_t kj = (int64_t)kf * g.nc2 + jf;
      double fx[kNV];
      shell_face_flux<DIR, R>(g, th, wl, wr, pref, kj, nkj, fx);
      if constexpr (WF) {
#pragma unroll
        for (int n = 0; n < kNV; ++n) {
          const int64_t idx =
              DIR == 1 ? (((int64_t)(p * kNV + n) * g.nc3 + o) * (g.nc2 + 1) + c) * g.nc1 + i
                       : (((int64_t)(p * kNV + n) * (g.nc3 + 1) + c) * g.nc2 + o) * g.nc1 + i;
          fout[idx] = fx[n];
        }
      }
      // this face's area: the upper face of cell c-1, the lower one of c
      const double ac = DIR == 1 ? xv * g.shell[kTabDx3AF2 * nkj + kj] * df
                                 : xv * g.shell[kTabDx2AF3 * nkj + kj] * df;
      if (c > s0) {
        const int kc = DIR == 1 ? o : c - 1, jc = DIR == 1 ? c - 1 : o;
        const int64_t kjc = (int64_t)kc * g.nc2 + jc;
        const double d2 = g.shell[kTabDx2A * nkj + kjc], d3 = g.shell[kTabDx3A * nkj + kjc];
        const double vol = df * d2 * d3 * xv * xv * g.shell[kTabSinC * nkj + kjc];
        const int64_t off = base + (int64_t)(c - 1) * sd;
#pragma unroll
        for (int n = 0; n < kNV; ++n) {
          const double dfl = ac * fx[n] - amp * fp[n];
          if (DIR == 1)
            du[n * g.sv + off] = -(wght * dfl / vol);
          else
            du[n * g.sv + off] = dpre[n] - wght * dfl / vol;
        }
      }
#pragma unroll
      for (int n = 0; n < kNV; ++n) fp[n] = fx[n];
      amp = ac;
    }
#pragma unroll
    for (int n = 0; n < kNV; ++n) {
      wrp[n] = wrc[n];
      q[0][n] = q[1][n];
      q[1][n] = q[2][n];
    }
  }
}

// 1: the panel x2 / x3 fluxes run as k_shell_flux_x23_run, 0: as tiles
constexpr int kShellFluxRun = 1;

}  // namespace
}  // namespace cb

// ---------------------------------------------------------------------------
// C ABI

using namespace cb;

struct canoe_shell {
  canoe_shell_config_t cfg;
  canoe_thermo_t th;
  Geom g;
  int64_t pvals = 0;  // values per panel
  double *d_u = nullptr, *d_w = nullptr, *d_u1 = nullptr, *d_du = nullptr;
  double *d_x1f = nullptr, *d_x1v = nullptr, *d_dx1f = nullptr, *d_dt = nullptr;
  double *d_tabs = nullptr, *d_lr = nullptr, *d_pref = nullptr;
  unsigned long long *d_dtacc = nullptr;
  uint32_t *d_err = nullptr;
  GhostRow *d_ghost = nullptr;
  EdgeRow *d_edge = nullptr;
  int nghost = 0, nedge = 0;
  cudaStream_t st = nullptr;
  bool own_stream = false;
};

static int shell_free(canoe_shell *s) {
  if (!s) return 0;
  for (void *p : {(void *)s->d_u, (void *)s->d_w, (void *)s->d_u1, (void *)s->d_du,
                  (void *)s->d_x1f, (void *)s->d_x1v, (void *)s->d_dx1f, (void *)s->d_dt,
                  (void *)s->d_tabs, (void *)s->d_lr, (void *)s->d_pref, (void *)s->d_dtacc,
                  (void *)s->d_err,
                  (void *)s->d_ghost, (void *)s->d_edge})
    if (p) cudaFree(p);
  if (s->own_stream && s->st) cudaStreamDestroy(s->st);
  delete s;
  return 0;
}

// launches of the shell's stage pieces
static int shell_ghosts(canoe_shell *s) {
  const int64_t n = (int64_t)s->nghost * s->g.nx1;
  k_shell_ghosts<<<(unsigned)((n + 255) / 256), 256, 0, s->st>>>(s->d_u, s->d_ghost, s->nghost,
                                                                 s->g, s->pvals);
  CB_CUDA(cudaGetLastError());
  return 0;
}

static int shell_c2p(canoe_shell *s) {
  const int64_t n = 6 * (int64_t)s->g.nc3 * s->g.nc2 * s->g.nx1;
  k_shell_c2p<<<(unsigned)((n + 255) / 256), 256, 0, s->st>>>(
      s->d_u, s->d_w, s->g, s->th.gammad - 1., s->pvals, s->d_err);
  CB_CUDA(cudaGetLastError());
  return 0;
}

static int shell_edges(canoe_shell *s) {
  const int64_t n = (int64_t)s->nedge * s->g.nx1;
  const unsigned nb = (unsigned)((n + 255) / 256);
  const bool f32 = s->cfg.precision == CANOE_FP32_PERTURBATION;
#define CB_SE(RC, R) \
  k_shell_edges<RC, R><<<nb, 256, 0, s->st>>>(s->d_w, s->d_edge, s->nedge, s->g, s->pvals, s->d_lr)
  if (s->cfg.recon == CANOE_RECON_PPM) {
    if (f32) CB_SE(CANOE_RECON_PPM, float); else CB_SE(CANOE_RECON_PPM, double);
  } else {
    if (f32) CB_SE(CANOE_RECON_PLM, float); else CB_SE(CANOE_RECON_PLM, double);
  }
#undef CB_SE
  CB_CUDA(cudaGetLastError());
  return 0;
}

template <typename R>
static int shell_x23_t(canoe_shell *s, int dir, double beta, double *fout) {
  const Geom &g = s->g;
  const bool ppm = s->cfg.recon == CANOE_RECON_PPM;
  if constexpr (kShellFluxRun != 0) {
    dim3 rgrid((g.nx1 + 31) / 32, (g.nx2 + SBY - 1) / SBY, 6 * ((g.nx2 + SRL - 1) / SRL));
    dim3 rblk(32, SBY);
#define CB_SR(RC, D, W)                                                              \
  k_shell_flux_x23_run<RC, D, W, R><<<rgrid, rblk, 0, s->st>>>(                      \
      g, s->th, s->d_w, s->d_du, s->d_dt, beta, s->pvals, s->d_lr, fout)
    if (dir == 1) {
      if (ppm) { if (fout) CB_SR(3, 1, true); else CB_SR(3, 1, false); }
      else { if (fout) CB_SR(2, 1, true); else CB_SR(2, 1, false); }
    } else {
      if (ppm) { if (fout) CB_SR(3, 2, true); else CB_SR(3, 2, false); }
      else { if (fout) CB_SR(2, 2, true); else CB_SR(2, 2, false); }
    }
#undef CB_SR
    CB_CUDA(cudaGetLastError());
    return 0;
  }
  dim3 grid((g.nx1 + TI - 1) / TI, (g.nx2 + TD - 1) / TD, 6 * g.nx2);
  dim3 blk(TI, 8);
  const size_t tiles = sizeof(R) * kNV * TI * ((TD + 2 * NG) + 2 * (TD + 2));
  const size_t smem = sizeof(R) == 8 ? tiles : tiles + sizeof(double) * kNV * (TD + 1) * TI;
#define CB_SX(RC, D, W)                                                                   \
  k_shell_flux_x23<RC, D, W, R><<<grid, blk, smem, s->st>>>(g, s->th, s->d_w, s->d_du,    \
                                                            s->d_dt, beta, s->pvals, s->d_lr, fout)
  if (dir == 1) {
    if (ppm) { if (fout) CB_SX(3, 1, true); else CB_SX(3, 1, false); }
    else { if (fout) CB_SX(2, 1, true); else CB_SX(2, 1, false); }
  } else {
    if (ppm) { if (fout) CB_SX(3, 2, true); else CB_SX(3, 2, false); }
    else { if (fout) CB_SX(2, 2, true); else CB_SX(2, 2, false); }
  }
#undef CB_SX
  CB_CUDA(cudaGetLastError());
  return 0;
}

static int shell_x23(canoe_shell *s, int dir, double beta, double *fout) {
  if (s->cfg.precision == CANOE_FP32_PERTURBATION) return shell_x23_t<float>(s, dir, beta, fout);
  return shell_x23_t<double>(s, dir, beta, fout);
}

extern "C" {

int canoe_shell_create(const canoe_shell_config_t *cfg, canoe_shell_t *out) {
  if (!cfg || !out || !cfg->h_x1f) {
    set_error("canoe_shell_create: null argument");
    return CANOE_ERR_ARG;
  }
  if (cfg->nside < 2 || cfg->nside % 2 || cfg->nx1 < 4) {
    set_error("canoe_shell_create: nside must be even, nx1 >= 4");
    return CANOE_ERR_ARG;
  }
  if (cfg->thermo.ny != 0 || cfg->rsolver != CANOE_RSOLVER_HLLC ||
      (cfg->precision != CANOE_FP64 && cfg->precision != CANOE_FP32_PERTURBATION)) {
    set_error("canoe_shell_create: the cubed-sphere path is dry (ny = 0) and HLLC");
    return CANOE_ERR_UNSUPPORTED;
  }
  if (cfg->bc_x1[0] == CANOE_BC_PERIODIC || cfg->bc_x1[1] == CANOE_BC_PERIODIC) {
    set_error("canoe_shell_create: periodic radial boundaries are not supported");
    return CANOE_ERR_UNSUPPORTED;
  }
  if (cfg->implicit_flag & 6) {
    set_error("canoe_shell_create: the shell's implicit solve is radial (implicit_flag 1 or 9)");
    return CANOE_ERR_UNSUPPORTED;
  }
  canoe_shell *s = new canoe_shell();
  s->cfg = *cfg;
  s->cfg.h_x1f = nullptr;
  s->th = cfg->thermo;
  Geom &g = s->g;
  const int N = cfg->nside;
  g.ny = 0;
  g.nv = kNV;
  g.nx1 = cfg->nx1;
  g.nx2 = g.nx3 = N;
  g.f2 = g.f3 = 1;
  g.nc1 = g.nx1 + 2 * NG;
  g.nc2 = g.nc3 = N + 2 * NG;
  g.is = NG;
  g.ie = NG + g.nx1 - 1;
  g.js = g.ks = NG;
  g.je = g.ke = NG + N - 1;
  g.bc[0] = cfg->bc_x1[0];
  g.bc[1] = cfg->bc_x1[1];
  for (int q = 2; q < 6; ++q) g.bc[q] = CANOE_BC_EXO3;
  g.sk = (int64_t)g.nc2 * g.nc1;
  g.sv = (int64_t)g.nc3 * g.sk;
  g.dx2 = g.dx3 = kPi / 2. / N;
  s->pvals = (int64_t)kNV * g.sv;
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
  const std::vector<double> tabs = build_geometry(N);
  const std::vector<GhostRow> gr = build_ghost_table(N);
  const std::vector<EdgeRow> er = build_edge_table(N);
  s->nghost = (int)gr.size();
  s->nedge = (int)er.size();
  const size_t bytes = 6 * (size_t)s->pvals * sizeof(double);
  const size_t lr_bytes = (size_t)6 * 4 * N * kNV * g.nx1 * sizeof(double);
  cudaError_t e;
  auto fail = [&](cudaError_t ee, const char *what) {
    int rc = cuda_status(ee, what);
    shell_free(s);
    return rc;
  };
  if ((e = cudaMalloc(&s->d_u, bytes))) return fail(e, "cudaMalloc u");
  if ((e = cudaMalloc(&s->d_w, bytes))) return fail(e, "cudaMalloc w");
  if ((e = cudaMalloc(&s->d_u1, bytes))) return fail(e, "cudaMalloc u1");
  if ((e = cudaMalloc(&s->d_du, bytes))) return fail(e, "cudaMalloc du");
  if ((e = cudaMalloc(&s->d_lr, lr_bytes))) return fail(e, "cudaMalloc lr");
  if ((e = cudaMalloc(&s->d_x1f, xf.size() * sizeof(double)))) return fail(e, "cudaMalloc x1f");
  if ((e = cudaMalloc(&s->d_x1v, xv.size() * sizeof(double)))) return fail(e, "cudaMalloc x1v");
  if ((e = cudaMalloc(&s->d_dx1f, dx.size() * sizeof(double)))) return fail(e, "cudaMalloc dx1f");
  if ((e = cudaMalloc(&s->d_dt, 2 * sizeof(double)))) return fail(e, "cudaMalloc dt");
  if ((e = cudaMalloc(&s->d_pref, g.nc1 * sizeof(double)))) return fail(e, "cudaMalloc pref");
  if ((e = cudaMemset(s->d_pref, 0, g.nc1 * sizeof(double)))) return fail(e, "cudaMemset pref");
  if ((e = cudaMalloc(&s->d_dtacc, sizeof(unsigned long long)))) return fail(e, "cudaMalloc acc");
  if ((e = cudaMalloc(&s->d_err, sizeof(uint32_t)))) return fail(e, "cudaMalloc err");
  if ((e = cudaMalloc(&s->d_tabs, tabs.size() * sizeof(double)))) return fail(e, "cudaMalloc tabs");
  if ((e = cudaMalloc(&s->d_ghost, gr.size() * sizeof(GhostRow)))) return fail(e, "cudaMalloc ghost");
  if ((e = cudaMalloc(&s->d_edge, er.size() * sizeof(EdgeRow)))) return fail(e, "cudaMalloc edge");
  for (double *p : {s->d_u, s->d_w, s->d_u1, s->d_du})
    if ((e = cudaMemset(p, 0, bytes))) return fail(e, "cudaMemset state");
  if ((e = cudaMemset(s->d_lr, 0, lr_bytes))) return fail(e, "cudaMemset lr");
  if ((e = cudaMemset(s->d_err, 0, sizeof(uint32_t)))) return fail(e, "cudaMemset err");
  if ((e = cudaMemset(s->d_dt, 0, 2 * sizeof(double)))) return fail(e, "cudaMemset dt");
  struct {
    void *d;
    const void *h;
    size_t n;
  } cps[] = {{s->d_x1f, xf.data(), xf.size() * sizeof(double)},
             {s->d_x1v, xv.data(), xv.size() * sizeof(double)},
             {s->d_dx1f, dx.data(), dx.size() * sizeof(double)},
             {s->d_tabs, tabs.data(), tabs.size() * sizeof(double)},
             {s->d_ghost, gr.data(), gr.size() * sizeof(GhostRow)},
             {s->d_edge, er.data(), er.size() * sizeof(EdgeRow)}};
  for (auto &c : cps)
    if ((e = cudaMemcpy(c.d, c.h, c.n, cudaMemcpyHostToDevice))) return fail(e, "copy tables");
  if ((e = cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking))) return fail(e, "stream");
  s->own_stream = true;
  g.x1f = s->d_x1f;
  g.x1v = s->d_x1v;
  g.dx1f = s->d_dx1f;
  g.pref = s->d_pref;
  g.err = s->d_err;
  g.shell = s->d_tabs;
  *out = s;
  return 0;
}

int canoe_shell_destroy(canoe_shell_t s) {
  if (s && s->st) cudaStreamSynchronize(s->st);
  return shell_free(s);
}

int canoe_shell_dims(canoe_shell_t s, int32_t *nv, int32_t *nc1, int32_t *nc2, int32_t *nc3) {
  if (!s) return CANOE_ERR_ARG;
  if (nv) *nv = kNV;
  if (nc1) *nc1 = s->g.nc1;
  if (nc2) *nc2 = s->g.nc2;
  if (nc3) *nc3 = s->g.nc3;
  return 0;
}

int canoe_shell_set_stream(canoe_shell_t s, void *stream) {
  if (!s) return CANOE_ERR_ARG;
  CB_CUDA(cudaStreamSynchronize(s->st));
  if (s->own_stream) cudaStreamDestroy(s->st);
  s->st = (cudaStream_t)stream;
  s->own_stream = false;
  return 0;
}

int canoe_shell_set_conserved(canoe_shell_t s, const double *h_u, int fill) {
  if (!s || !h_u) return CANOE_ERR_ARG;
  CB_CUDA(cudaMemcpyAsync(s->d_u, h_u, 6 * (size_t)s->pvals * sizeof(double),
                          cudaMemcpyHostToDevice, s->st));
  if (fill) {
    if (int rc = shell_ghosts(s)) return rc;
    if (int rc = shell_c2p(s)) return rc;
    // reference pressure of the FP32 flux path: the level mean of panel 0
    // (every panel holds the same radial levels)
    if (int rc = launch_level_mean_pressure(s->g, 0, s->d_w, s->d_pref, s->st)) return rc;
  }
  CB_CUDA(cudaStreamSynchronize(s->st));
  return 0;
}

int canoe_shell_fill_ghosts(canoe_shell_t s) {
  if (!s) return CANOE_ERR_ARG;
  return shell_ghosts(s);
}

static int shell_get(canoe_shell_t s, const double *d, double *h) {
  if (!s || !h) return CANOE_ERR_ARG;
  CB_CUDA(cudaMemcpyAsync(h, d, 6 * (size_t)s->pvals * sizeof(double), cudaMemcpyDeviceToHost,
                          s->st));
  CB_CUDA(cudaStreamSynchronize(s->st));
  return 0;
}

int canoe_shell_get_conserved(canoe_shell_t s, double *h_u) { return shell_get(s, s->d_u, h_u); }

int canoe_shell_get_primitive(canoe_shell_t s, double *h_w) { return shell_get(s, s->d_w, h_w); }

int canoe_shell_calculate_fluxes(canoe_shell_t s, double *d_f1, double *d_f2, double *d_f3) {
  if (!s || !d_f2 || !d_f3) return CANOE_ERR_ARG;
  Geom g = s->g;
  double one_dt[2] = {0., 0.};
  CB_CUDA(cudaMemcpyAsync(s->d_dt, one_dt, sizeof(one_dt), cudaMemcpyHostToDevice, s->st));
  if (int rc = shell_edges(s)) return rc;
  if (int rc = shell_x23(s, 1, 0., d_f2)) return rc;
  if (int rc = shell_x23(s, 2, 0., d_f3)) return rc;
  if (d_f1) {
    const int64_t fvals = (int64_t)kNV * g.nc3 * g.nc2 * (g.nc1 + 1);
    for (int p = 0; p < 6; ++p)
      if (int rc = launch_x1col(g, s->th, s->cfg.recon, s->cfg.rsolver, 0, s->cfg.precision,
                                kColFluxOnly, s->d_w + p * s->pvals, s->d_du + p * s->pvals,
                                s->d_u + p * s->pvals, s->d_u1 + p * s->pvals, s->d_dt,
                                kRK3[0], 0, d_f1 + p * fvals, s->st))
        return rc;
  }
  CB_CUDA(cudaStreamSynchronize(s->st));
  return 0;
}

int canoe_shell_step(canoe_shell_t s, double dt) {
  if (!s || !(dt > 0.)) {
    set_error("canoe_shell_step: dt must be positive");
    return CANOE_ERR_ARG;
  }
  int rc;
  if ((rc = launch_dt_finalize(s->d_dt, s->d_dtacc, s->cfg.cfl, dt, s->st))) return rc;
  for (int stage = 0; stage < 3; ++stage) {
    const Stage &sg = kRK3[stage];
    if ((rc = shell_edges(s))) return rc;
    if ((rc = shell_x23(s, 1, sg.beta, nullptr))) return rc;
    if ((rc = shell_x23(s, 2, sg.beta, nullptr))) return rc;
    {  // the six panels' x1 pencils in one launch
      Geom g6 = s->g;
      g6.npanel = 6;
      g6.pstride = s->pvals;
      if ((rc = launch_x1col(g6, s->th, s->cfg.recon, s->cfg.rsolver, s->cfg.implicit_flag,
                             s->cfg.precision, kColStep, s->d_w, s->d_du, s->d_u, s->d_u1,
                             s->d_dt, sg, stage, nullptr, s->st)))
        return rc;
    }
    if ((rc = shell_ghosts(s))) return rc;
    if ((rc = shell_c2p(s))) return rc;
  }
  return 0;
}

int canoe_shell_synchronize(canoe_shell_t s) {
  if (!s) return CANOE_ERR_ARG;
  CB_CUDA(cudaStreamSynchronize(s->st));
  return 0;
}

int canoe_shell_error_word(canoe_shell_t s, uint32_t *bits) {
  if (!s || !bits) return CANOE_ERR_ARG;
  CB_CUDA(cudaMemcpyAsync(bits, s->d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, s->st));
  CB_CUDA(cudaMemsetAsync(s->d_err, 0, sizeof(uint32_t), s->st));
  CB_CUDA(cudaStreamSynchronize(s->st));
  return 0;
}

}  // extern "C"
