// exo3.cpp -- oracle restatement of canoe's cubed-sphere (exo3) path on a
// shell of six panels, one MeshBlock per panel (NBLOCKS = 6: bound_lim = 0,
// canoe src/exo3/cs_find_block_id.cpp:83-91).  TEST INFRASTRUCTURE ONLY.
//
//  * gnomonic equiangle tables      gnomonic_equiangle.cpp:24-222
//  * ghost exchange of u            cubed_sphere_utility.cpp:26-623 (PackData,
//    InteprolateX2/X3, CalculateInterpLocations, PackDataR0..R3) called from
//    Athena's LoadBoundaryBufferSameLevel (patches/33.bvals_cc_cpp.patch:21)
//    with the neighbour search of patches/30.bvals_base.patch
//    (CubedSphere::TransformOX, cs_transform_ox.cpp:11-230); the receiving
//    block unpacks in Athena's standard (n, k, j, i) order
//  * L/R face-state swap            cubed_sphere.cpp:250-681
//  * vector transforms              cubed_sphere_transform.cpp:11-61
//  * curvilinear step               patches/19 (CUBED_SPHERE branches),
//    hllc_transform.cpp:46-55, 92-101, 227-272, gnomonic_equiangle.cpp:
//    604-878, solve_implicit_3d.cpp:105-137, patches/26.adiabatic_hydro
//
// Corner ghost cells (both j and k outside the panel) are not exchanged: the
// reference bypasses them (cubed_sphere_utility.cpp:401-405) and nothing on
// this path reads them.
#include <cassert>
#include <cmath>
#include <cstring>
#include <stdexcept>

#include "oracle.hpp"

namespace oracle {

namespace {

constexpr double PI = 3.14159265358979323846;

// ---------------------------------------------------------------------------
// panel connectivity (single block per panel)

// dinv[source][dir], tgside[source][dir], tgbid[source][dir] with dir
// 0: ox2 = -1 (up), 1: ox2 = +1 (down), 2: ox3 = -1 (left), 3: ox3 = +1
// (right); cubed_sphere_utility.cpp:385-398
const int kDinv[6][4] = {{1, 0, 0, 1}, {0, 0, 0, 0}, {0, 1, 0, 0},
                         {1, 0, 0, 0}, {0, 1, 1, 0}, {1, 1, 0, 0}};
const int kTgside[6][4] = {{-1, -1, -1, -1}, {1, -1, 1, -1}, {-1, -1, 1, -1},
                           {1, 1, 1, -1},    {1, 1, 1, 1},   {-1, 1, 1, -1}};
const int kTgbid[6][4] = {{6, 2, 3, 4}, {1, 5, 3, 4}, {1, 5, 6, 2},
                          {1, 5, 2, 6}, {2, 6, 3, 4}, {1, 5, 4, 3}};

// TransformOX (cs_transform_ox.cpp:11-230) for bound_lim = 0: the direction
// (tox2, tox3) under which the target block files the message
void transform_ox(int block_id, int ox2, int ox3, int &tox2, int &tox3) {
  int tb = -1;
  switch (block_id) {
    case 1:
      if (ox3 == -1) { tb = 3; tox2 = -1; tox3 = 0; }
      if (ox2 == -1) { tb = 6; tox2 = -1; tox3 = 0; }
      if (ox3 == 1) { tb = 4; tox2 = -1; tox3 = 0; }
      break;
    case 2:
      if (ox3 == -1) { tb = 3; tox2 = 0; tox3 = 1; }
      if (ox2 == 1) { tb = 5; tox2 = -1; tox3 = 0; }
      break;
    case 3:
      if (ox3 == -1) { tb = 6; tox2 = 0; tox3 = 1; }
      if (ox2 == -1) { tb = 1; tox2 = 0; tox3 = -1; }
      if (ox2 == 1) { tb = 5; tox2 = 0; tox3 = -1; }
      if (ox3 == 1) { tb = 2; tox2 = 0; tox3 = -1; }
      break;
    case 4:
      if (ox2 == -1) { tb = 1; tox2 = 0; tox3 = 1; }
      if (ox2 == 1) { tb = 5; tox2 = 0; tox3 = 1; }
      break;
    case 5:
      if (ox3 == -1) { tb = 3; tox2 = 1; tox3 = 0; }
      if (ox3 == 1) { tb = 4; tox2 = 1; tox3 = 0; }
      if (ox2 == 1) { tb = 6; tox2 = 1; tox3 = 0; }
      if (ox2 == -1) { tb = 2; tox2 = 1; tox3 = 0; }
      break;
    case 6:
      if (ox2 == -1) { tb = 1; tox2 = -1; tox3 = 0; }
      if (ox2 == 1) { tb = 5; tox2 = 1; tox3 = 0; }
      if (ox3 == 1) { tb = 3; tox2 = 0; tox3 = -1; }
      break;
  }
  if (tb < 0) {  // a neighbour inside the 2 x 3 block layout
    tox2 = -ox2;
    tox3 = -ox3;
  }
}

// ---------------------------------------------------------------------------
// vector transforms (cubed_sphere_transform.cpp:11-61)

void vec_abp_from_rll(double X, double Y, int block_id, double U, double V, double *V2,
                      double *V3) {
  double C = std::sqrt(1 + X * X);
  double D = std::sqrt(1 + Y * Y);
  double E = std::sqrt(X * X + Y * Y);
  double delta = std::sqrt(1 + X * X + Y * Y);
  switch (block_id) {
    case 2:
    case 3:
    case 4:
    case 6:
      *V2 = X * Y / delta * U - V;
      *V3 = C * D / delta * U;
      break;
    case 1:
      *V2 = -D * Y / (delta * E) * U - D * X / E * V;
      *V3 = C * X / (delta * E) * U - C * Y / E * V;
      break;
    case 5:
      *V2 = D * Y / (delta * E) * U + D * X / E * V;
      *V3 = -C * X / (delta * E) * U + C * Y / E * V;
      break;
  }
}

void vec_rll_from_abp(double X, double Y, int block_id, double V2, double V3, double *U,
                      double *V) {
  double C = std::sqrt(1 + X * X);
  double D = std::sqrt(1 + Y * Y);
  double E = std::sqrt(X * X + Y * Y);
  double delta = std::sqrt(1 + X * X + Y * Y);
  switch (block_id) {
    case 2:
    case 3:
    case 4:
    case 6:
      *U = delta / (C * D) * V3;
      *V = X * Y / (C * D) * V3 - V2;
      break;
    case 1:
      *U = -delta * Y / (D * E) * V2 + delta * X / (C * E) * V3;
      *V = -X / (D * E) * V2 - Y / (C * E) * V3;
      break;
    case 5:
      *U = delta * Y / (D * E) * V2 - delta * X / (C * E) * V3;
      *V = X / (D * E) * V2 + Y / (C * E) * V3;
      break;
  }
}

// CalculateInterpLocations (cubed_sphere_utility.cpp:78-98)
double interp_location(int loc_n, int nblk, int k, bool ghost) {
  double temp0 = std::tan((double)1.0 * (nblk - 1 - 2 * k) / (nblk * 4) * PI);
  if (ghost) {
    temp0 = 1.0 / temp0;
    temp0 = 1.0 + temp0 * temp0;
  } else {
    temp0 = 1.0 + temp0 * temp0;
  }
  const double t = std::pow(std::tan((double)1.0 * (2 * loc_n + 1) / (nblk * 4) * PI), 2.0);
  if (loc_n < 0) return -std::acos(std::sqrt(temp0 / (temp0 + t)));
  return std::acos(std::sqrt(temp0 / (temp0 + t)));
}

// one panel array (nv, nc3, nc2, nc1) with a 4-index accessor
struct Arr4 {
  double *p;
  int d1, d2, d3;  // extents of the three fastest dims (k, j, i)
  double &operator()(int n, int k, int j, int i) const {
    return p[(((size_t)n * d1 + k) * d2 + j) * d3 + i];
  }
};

// raise (covariant -> contravariant) with the cell's sin / cos, the
// lat-lon round trip and the lower, as in cubed_sphere_utility.cpp:185-211
void rotate_velocity(double src_cy, double src_cz, int block_id, double tgt_cy,
                     double tgt_cz, int tgt_id, double &vy, double &vz) {
  double sth = std::sqrt(1 + src_cy * src_cy + src_cz * src_cz) /
               std::sqrt(1 + src_cy * src_cy) / std::sqrt(1 + src_cz * src_cz);
  double cth = -src_cy * src_cz / std::sqrt(1 + src_cy * src_cy) /
               std::sqrt(1 + src_cz * src_cz);
  double vyt = vy, vzt = vz;
  vy = vyt / sth / sth - vzt * cth / sth / sth;
  vz = vzt / sth / sth - vyt * cth / sth / sth;
  double U, V;
  vec_rll_from_abp(src_cy, src_cz, block_id, vy, vz, &U, &V);
  vec_abp_from_rll(tgt_cy, tgt_cz, tgt_id, U, V, &vy, &vz);
  sth = std::sqrt(1 + tgt_cy * tgt_cy + tgt_cz * tgt_cz) / std::sqrt(1 + tgt_cy * tgt_cy) /
        std::sqrt(1 + tgt_cz * tgt_cz);
  cth = -tgt_cy * tgt_cz / std::sqrt(1 + tgt_cy * tgt_cy) / std::sqrt(1 + tgt_cz * tgt_cz);
  vyt = vy;
  vzt = vz;
  vy = vyt + vzt * cth;
  vz = vzt + vyt * cth;
}

// InteprolateX2 (cubed_sphere_utility.cpp:100-225): along j, for the x3
// faces; tgt has the extents of the source region
void interpolate_x2(const Arr4 &src, const Arr4 &tgt, int block_id, int dir_inv, int tgt_side,
                    int tgt_id, int sn, int en, int si, int ei, int sj, int ej, int sk, int ek,
                    int ivy, int ivz) {
  const int nblk = ej - sj + 1;
  const int n_start = -nblk / 2;
  std::vector<double> src_x2(nblk), src_coord(nblk), tgt_coord(nblk), tgt_x2(nblk);
  for (int n = sn; n <= en; ++n)
    for (int k = sk; k <= ek; ++k) {
      int k_now, src_side;
      if (sk < ej - NG) {
        k_now = k - sk;
        src_side = -1;
      } else {
        k_now = ek - k;
        src_side = 1;
      }
      for (int i = si; i <= ei; ++i) {
        for (int j = 0; j < nblk; ++j) {
          src_x2[j] = interp_location(j - nblk / 2, nblk, k_now, false);
          src_coord[j] = PI / 2.0 / nblk * (j + 0.5) - PI / 4.0;
        }
        for (int j = sj; j <= ej; ++j) {
          tgt_x2[j - sj] = interp_location(n_start + j - sj, nblk, k_now, true);
          if (dir_inv == 1)
            tgt_coord[j - sj] = -src_coord[n_start + nblk / 2 + j - sj];
          else
            tgt_coord[j - sj] = src_coord[n_start + nblk / 2 + j - sj];
        }
        int sp = 0;
        for (int j = sj; j <= ej; ++j) {
          while (tgt_x2[j - sj] > src_x2[sp + 1]) ++sp;
          assert(sp + 1 < nblk);
          const double y1 = src_x2[sp], y2 = src_x2[sp + 1], yq = tgt_x2[j - sj];
          const int j1 = sp - n_start - nblk / 2 + sj, j2 = j1 + 1;
          if (n == ivy || n == ivz) {
            const double v1y = src(ivy, k, j1, i), v1z = src(ivz, k, j1, i);
            const double v2y = src(ivy, k, j2, i), v2z = src(ivz, k, j2, i);
            const double tgt_cy = std::tan(tgt_coord[j - sj]);
            const double tgt_cz =
                std::tan(tgt_side * (PI / 2.0 / nblk * (k_now + 0.5) + PI / 4.0));
            const double src_cy1 = src_coord[sp], src_cy2 = src_coord[sp + 1];
            const double src_cz =
                std::tan(src_side * (-PI / 2.0 / nblk * (k_now + 0.5) + PI / 4.0));
            double vy = ((y2 - yq) * v1y + (yq - y1) * v2y) / (y2 - y1);
            double vz = ((y2 - yq) * v1z + (yq - y1) * v2z) / (y2 - y1);
            const double src_cy =
                std::tan(((y2 - yq) * src_cy1 + (yq - y1) * src_cy2) / (y2 - y1));
            rotate_velocity(src_cy, src_cz, block_id, tgt_cy, tgt_cz, tgt_id, vy, vz);
            tgt(n - sn, k - sk, j - sj, i - si) = (n == ivy) ? vy : vz;
          } else {
            const double v1 = src(n, k, j1, i), v2 = src(n, k, j2, i);
            tgt(n - sn, k - sk, j - sj, i - si) = ((y2 - yq) * v1 + (yq - y1) * v2) / (y2 - y1);
          }
        }
      }
    }
}

// InteprolateX3 (cubed_sphere_utility.cpp:227-378): along k, for the x2 faces
void interpolate_x3(const Arr4 &src, const Arr4 &tgt, int block_id, int dir_inv, int tgt_side,
                    int tgt_id, int sn, int en, int si, int ei, int sj, int ej, int sk, int ek,
                    int ivy, int ivz) {
  const int nblk = ek - sk + 1;
  const int n_start = -nblk / 2;
  std::vector<double> src_x3(nblk), src_coord(nblk), tgt_coord(nblk), tgt_x3(nblk);
  for (int n = sn; n <= en; ++n)
    for (int j = sj; j <= ej; ++j) {
      int k_now, src_side;
      if (sj < ek - NG) {
        k_now = j - sj;
        src_side = -1;
      } else {
        k_now = ej - j;
        src_side = 1;
      }
      for (int i = si; i <= ei; ++i) {
        for (int k = 0; k < nblk; ++k) {
          src_x3[k] = interp_location(k - nblk / 2, nblk, k_now, false);
          src_coord[k] = PI / 2.0 / nblk * (k + 0.5) - PI / 4.0;
        }
        for (int k = sk; k <= ek; ++k) {
          tgt_x3[k - sk] = interp_location(n_start + k - sk, nblk, k_now, true);
          if (dir_inv == 1)
            tgt_coord[k - sk] = -src_coord[n_start + nblk / 2 + k - sk];
          else
            tgt_coord[k - sk] = src_coord[n_start + nblk / 2 + k - sk];
        }
        int sp = 0;
        for (int k = sk; k <= ek; ++k) {
          while (tgt_x3[k - sk] > src_x3[sp + 1]) ++sp;
          assert(sp + 1 < nblk);
          const double y1 = src_x3[sp], y2 = src_x3[sp + 1], yq = tgt_x3[k - sk];
          const int k1 = sp - n_start - nblk / 2 + sk, k2 = k1 + 1;
          if (n == ivy || n == ivz) {
            const double v1y = src(ivy, k1, j, i), v1z = src(ivz, k1, j, i);
            const double v2y = src(ivy, k2, j, i), v2z = src(ivz, k2, j, i);
            double tgt_cz = std::tan(tgt_coord[k - sk]);
            double tgt_cy = std::tan(tgt_side * (PI / 2.0 / nblk * (k_now + 0.5) + PI / 4.0));
            const double src_cz1 = src_coord[sp], src_cz2 = src_coord[sp + 1];
            const double src_cy =
                std::tan(src_side * (-PI / 2.0 / nblk * (k_now + 0.5) + PI / 4.0));
            double vy = ((y2 - yq) * v1y + (yq - y1) * v2y) / (y2 - y1);
            double vz = ((y2 - yq) * v1z + (yq - y1) * v2z) / (y2 - y1);
            const double src_cz =
                std::tan(((y2 - yq) * src_cz1 + (yq - y1) * src_cz2) / (y2 - y1));
            // cubed_sphere_utility.cpp:322-333: the target's axes swap for
            // these pairs of panels
            const int b = block_id, t = tgt_id;
            if ((t == 1 && b == 3) || (t == 1 && b == 4) || (t == 5 && b == 3) ||
                (t == 5 && b == 4) || (t == 3 && b == 1) || (t == 4 && b == 1) ||
                (t == 3 && b == 5) || (t == 4 && b == 5)) {
              const double tmp = tgt_cy;
              tgt_cy = tgt_cz;
              tgt_cz = tmp;
            }
            rotate_velocity(src_cy, src_cz, block_id, tgt_cy, tgt_cz, tgt_id, vy, vz);
            tgt(n - sn, k - sk, j - sj, i - si) = (n == ivy) ? vy : vz;
          } else {
            const double v1 = src(n, k1, j, i), v2 = src(n, k2, j, i);
            tgt(n - sn, k - sk, j - sj, i - si) = ((y2 - yq) * v1 + (yq - y1) * v2) / (y2 - y1);
          }
        }
      }
    }
}

// PackDataR0..R3 (cubed_sphere_utility.cpp:26-76) over a region of a
// (dn, dk, dj, di) array
void pack(const Arr4 &a, int order, int nn, int nk, int nj, int ni, std::vector<double> &buf) {
  buf.clear();
  for (int n = 0; n < nn; ++n) {
    if (order == 0) {
      for (int k = 0; k < nk; ++k)
        for (int j = 0; j < nj; ++j)
          for (int i = 0; i < ni; ++i) buf.push_back(a(n, k, j, i));
    } else if (order == 1) {
      for (int j = nj - 1; j >= 0; --j)
        for (int k = 0; k < nk; ++k)
          for (int i = 0; i < ni; ++i) buf.push_back(a(n, k, j, i));
    } else if (order == 2) {
      for (int k = nk - 1; k >= 0; --k)
        for (int j = nj - 1; j >= 0; --j)
          for (int i = 0; i < ni; ++i) buf.push_back(a(n, k, j, i));
    } else {
      for (int j = 0; j < nj; ++j)
        for (int k = nk - 1; k >= 0; --k)
          for (int i = 0; i < ni; ++i) buf.push_back(a(n, k, j, i));
    }
  }
}

// pack order and interpolation axis per (block, dir): the switch of
// PackData (cubed_sphere_utility.cpp:415-615); axis 2 = InteprolateX2 (x3
// faces), 3 = InteprolateX3 (x2 faces)
int pack_order(int block_id, int dir) {
  static const int order[6][4] = {
      // up (ox2-1), down (ox2+1), left (ox3-1), right (ox3+1)
      {2, 0, 3, 1},  // 1
      {0, 0, 0, 0},  // 2
      {1, 3, 0, 0},  // 3
      {3, 1, 0, 0},  // 4
      {0, 2, 1, 3},  // 5
      {2, 2, 0, 0},  // 6
  };
  return order[block_id - 1][dir];
}

}  // namespace

// ---------------------------------------------------------------------------
// construction

void shell_init(Shell &s, const canoe_shell_config_t &cfg) {
  if (cfg.nside < 2 || cfg.nside % 2)
    throw std::runtime_error("nside must be even and >= 2");
  if (cfg.rsolver != CANOE_RSOLVER_HLLC)
    throw std::runtime_error("the cubed-sphere path uses the HLLC solver (hllc_transform)");
  if (cfg.thermo.ny != 0)
    throw std::runtime_error("the cubed-sphere path is dry (ny = 0): its EOS is the "
                             "adiabatic one of patches/26.adiabatic_hydro.patch");
  s.cfg = cfg;
  s.N = cfg.nside;
  s.nv = 5 + cfg.thermo.ny;
  const int N = s.N;
  canoe_block_config_t bc{};
  bc.nx1 = cfg.nx1;
  bc.nx2 = N;
  bc.nx3 = N;
  bc.bc[0] = cfg.bc_x1[0];
  bc.bc[1] = cfg.bc_x1[1];
  for (int q = 2; q < 6; ++q) bc.bc[q] = CANOE_BC_EXO3;
  bc.dx2 = bc.dx3 = PI / 2. / N;
  bc.h_x1f = cfg.h_x1f;
  bc.recon = cfg.recon;
  bc.rsolver = cfg.rsolver;
  bc.implicit_flag = cfg.implicit_flag;
  bc.precision = cfg.precision;
  bc.satadj = 0;
  bc.cfl = cfg.cfl;
  bc.thermo = cfg.thermo;
  ShellGeo &g = s.geo;
  g.N = N;
  g.nc2 = g.nc3 = N + 2 * NG;
  const int nc = g.nc2;
  // equiangular faces of one panel, ghosts continue the spacing
  // (GenerateMeshX2 / X3, cubed_sphere.cpp:35-72)
  g.x2f.assign(nc + 1, 0.);
  g.x2v.assign(nc, 0.);
  const double d = PI / 2. / N;
  for (int j = 0; j <= nc; ++j) g.x2f[j] = -PI / 4. + (j - NG) * d;
  for (int j = 0; j < nc; ++j) g.x2v[j] = 0.5 * (g.x2f[j + 1] + g.x2f[j]);
  g.x3f = g.x2f;
  g.x3v = g.x2v;
  const size_t nkj = (size_t)nc * nc;
  for (auto *v : {&g.cosc, &g.sinc, &g.cosf2, &g.sinf2, &g.cosf3, &g.sinf3, &g.dx2a, &g.dx3a,
                  &g.dx2a_f3, &g.dx3a_f2})
    v->assign(nkj, 0.);
  for (int k = 0; k < nc; ++k)
    for (int j = 0; j < nc; ++j) {
      const size_t q = g.kj(k, j);
      double x = std::tan(g.x2v[j]);
      double xf = std::tan(g.x2f[j]);
      double y = std::tan(g.x3v[k]);
      double yf = std::tan(g.x3f[k]);
      double C = std::sqrt(1.0 + x * x);
      double Cf = std::sqrt(1.0 + xf * xf);
      double D = std::sqrt(1.0 + y * y);
      double Df = std::sqrt(1.0 + yf * yf);
      g.cosc[q] = -x * y / (C * D);
      g.sinc[q] = std::sqrt(1.0 + x * x + y * y) / (C * D);
      g.cosf2[q] = -xf * y / (Cf * D);
      g.sinf2[q] = std::sqrt(1.0 + xf * xf + y * y) / (Cf * D);
      g.cosf3[q] = -x * yf / (C * Df);
      g.sinf3[q] = std::sqrt(1.0 + x * x + yf * yf) / (C * Df);
      double x1 = std::tan(g.x2f[j]);
      double x2 = std::tan(g.x2f[j + 1]);
      double delta1 = std::sqrt(1.0 + x1 * x1 + y * y);
      double delta2 = std::sqrt(1.0 + x2 * x2 + y * y);
      double delta1f = std::sqrt(1.0 + x1 * x1 + yf * yf);
      double delta2f = std::sqrt(1.0 + x2 * x2 + yf * yf);
      g.dx2a[q] = std::acos((1 + x1 * x2 + y * y) / (delta1 * delta2));
      g.dx2a_f3[q] = std::acos((1 + x1 * x2 + yf * yf) / (delta1f * delta2f));
      double y1 = std::tan(g.x3f[k]);
      double y2 = std::tan(g.x3f[k + 1]);
      delta1 = std::sqrt(1.0 + x * x + y1 * y1);
      delta2 = std::sqrt(1.0 + x * x + y2 * y2);
      delta1f = std::sqrt(1.0 + xf * xf + y1 * y1);
      delta2f = std::sqrt(1.0 + xf * xf + y2 * y2);
      g.dx3a[q] = std::acos((1 + x * x + y1 * y2) / (delta1 * delta2));
      g.dx3a_f2[q] = std::acos((1 + xf * xf + y1 * y2) / (delta1f * delta2f));
    }
  for (int p = 0; p < 6; ++p) {
    block_init(s.p[p], bc);
    s.p[p].geo = &s.geo;
    s.p[p].panel = p;
    const Block &b = s.p[p];
    s.L2[p].assign((size_t)s.nv * b.nc3 * (b.nc2 + 1) * b.nc1, 0.);
    s.R2[p].assign(s.L2[p].size(), 0.);
    s.L3[p].assign((size_t)s.nv * (b.nc3 + 1) * b.nc2 * b.nc1, 0.);
    s.R3[p].assign(s.L3[p].size(), 0.);
  }
}

// ---------------------------------------------------------------------------
// ghost exchange of the conserved state

void shell_fill_ghosts(Shell &s) {
  const int nv = s.nv;
  struct Msg {
    int target, tox2, tox3;
    std::vector<double> buf;
  };
  std::vector<Msg> msgs;
  for (int p = 0; p < 6; ++p) {
    Block &b = s.p[p];
    const int block_id = p + 1;
    const Arr4 src{b.u.data(), b.nc3, b.nc2, b.nc1};
    const int ivy = b.ivy, ivz = b.ivz;
    for (int dir = 0; dir < 4; ++dir) {
      const int ox2 = dir == 0 ? -1 : dir == 1 ? 1 : 0;
      const int ox3 = dir == 2 ? -1 : dir == 3 ? 1 : 0;
      // LoadBoundaryBufferSameLevel region of the face (ox1 = 0)
      const int si = b.is, ei = b.ie;
      const int sj = ox2 > 0 ? b.je - NG + 1 : b.js, ej = ox2 < 0 ? b.js + NG - 1 : b.je;
      const int sk = ox3 > 0 ? b.ke - NG + 1 : b.ks, ek = ox3 < 0 ? b.ks + NG - 1 : b.ke;
      const int dn = nv, dk = ek - sk + 1, dj = ej - sj + 1, di = ei - si + 1;
      std::vector<double> tv((size_t)dn * dk * dj * di);
      const Arr4 tgt{tv.data(), dk, dj, di};
      const int tgt_id = kTgbid[p][dir];
      if (ox3 != 0)
        interpolate_x2(src, tgt, block_id, kDinv[p][dir], kTgside[p][dir], tgt_id, 0, nv - 1, si,
                       ei, sj, ej, sk, ek, ivy, ivz);
      else
        interpolate_x3(src, tgt, block_id, kDinv[p][dir], kTgside[p][dir], tgt_id, 0, nv - 1, si,
                       ei, sj, ej, sk, ek, ivy, ivz);
      Msg m;
      transform_ox(block_id, ox2, ox3, m.tox2, m.tox3);
      m.target = tgt_id - 1;
      pack(tgt, pack_order(block_id, dir), dn, dk, dj, di, m.buf);
      msgs.push_back(std::move(m));
    }
  }
  // SetBoundarySameLevel: unpack into the ghost slab facing (tox2, tox3)
  for (const Msg &m : msgs) {
    Block &t = s.p[m.target];
    const int sj = m.tox2 == 0 ? t.js : (m.tox2 > 0 ? t.je + 1 : t.js - NG);
    const int ej = m.tox2 == 0 ? t.je : (m.tox2 > 0 ? t.je + NG : t.js - 1);
    const int sk = m.tox3 == 0 ? t.ks : (m.tox3 > 0 ? t.ke + 1 : t.ks - NG);
    const int ek = m.tox3 == 0 ? t.ke : (m.tox3 > 0 ? t.ke + NG : t.ks - 1);
    size_t q = 0;
    if (m.buf.size() != (size_t)nv * (ek - sk + 1) * (ej - sj + 1) * (t.ie - t.is + 1))
      throw std::runtime_error("exo3 message size mismatch");
    for (int n = 0; n < nv; ++n)
      for (int k = sk; k <= ek; ++k)
        for (int j = sj; j <= ej; ++j)
          for (int i = t.is; i <= t.ie; ++i) t.u[t.idx(n, k, j, i)] = m.buf[q++];
  }
}

// ---------------------------------------------------------------------------
// cons <-> prim with covariant momentum (patches/26.adiabatic_hydro.patch):
// w velocities are contravariant, u momenta covariant

void shell_cons_to_prim(Shell &s) {
  const ShellGeo &g = s.geo;
  for (int p = 0; p < 6; ++p) {
    Block &b = s.p[p];
    const size_t st = b.cells();
    const double gm1 = b.th.gammad - 1.;
    // interior and the four face ghost slabs (corners are not filled)
    for (int k = 0; k < b.nc3; ++k)
      for (int j = 0; j < b.nc2; ++j) {
        const bool kin = k >= b.ks && k <= b.ke, jin = j >= b.js && j <= b.je;
        if (!kin && !jin) continue;
        const double cth = g.cosc[g.kj(k, j)];
        for (int i = b.is; i <= b.ie; ++i) {
          const size_t c = b.idx(0, k, j, i);
          const double *u = &b.u[c];
          double *w = &b.w[c];
          const double u_d = u[0], u_m1 = u[b.ivx * st], u_m2 = u[b.ivy * st],
                       u_m3 = u[b.ivz * st], u_e = u[b.ipr * st];
          const double di = 1.0 / u_d;
          w[0] = u_d;
          double wv[3] = {u_m1 * di, u_m2 * di, u_m3 * di};
          // CovariantToContravariant (cubed_sphere_utility.hpp:20-28)
          const double v = wv[1], ww = wv[2];
          const double sth2 = 1. - cth * cth;
          wv[1] = v / sth2 - ww * cth / sth2;
          wv[2] = -v * cth / sth2 + ww / sth2;
          const double e_k = 0.5 * (u_m1 * wv[0] + u_m2 * wv[1] + u_m3 * wv[2]);
          w[b.ivx * st] = wv[0];
          w[b.ivy * st] = wv[1];
          w[b.ivz * st] = wv[2];
          w[b.ipr * st] = gm1 * (u_e - e_k);
        }
      }
    // x1 ghosts of every filled column
    const int *bc = b.cfg.bc;
    for (int n = 0; n < b.nv; ++n)
      for (int k = 0; k < b.nc3; ++k)
        for (int j = 0; j < b.nc2; ++j) {
          const bool kin = k >= b.ks && k <= b.ke, jin = j >= b.js && j <= b.je;
          if (!kin && !jin) continue;
          for (int gg = 1; gg <= NG; ++gg) {
            const double sgn = (n == b.ivx) ? -1. : 1.;
            const size_t lo = b.idx(n, k, j, b.is - gg), hi = b.idx(n, k, j, b.ie + gg);
            if (bc[0] == CANOE_BC_REFLECT) b.w[lo] = sgn * b.w[b.idx(n, k, j, b.is + gg - 1)];
            else b.w[lo] = b.w[b.idx(n, k, j, b.is)];
            if (bc[1] == CANOE_BC_REFLECT) b.w[hi] = sgn * b.w[b.idx(n, k, j, b.ie - gg + 1)];
            else b.w[hi] = b.w[b.idx(n, k, j, b.ie)];
          }
        }
  }
}

// PrimitiveToConserved with the covariant momenta (patch 26)
void shell_prim_to_cons(Shell &s) {
  const ShellGeo &g = s.geo;
  for (int p = 0; p < 6; ++p) {
    Block &b = s.p[p];
    const size_t st = b.cells();
    const double igm1 = 1.0 / (b.th.gammad - 1.);
    for (int k = b.ks; k <= b.ke; ++k)
      for (int j = b.js; j <= b.je; ++j) {
        const double cth = g.cosc[g.kj(k, j)];
        for (int i = b.is; i <= b.ie; ++i) {
          const size_t c = b.idx(0, k, j, i);
          const double *w = &b.w[c];
          double *u = &b.u[c];
          const double w_d = w[0], w_vx = w[b.ivx * st], w_vy = w[b.ivy * st],
                       w_vz = w[b.ivz * st], w_p = w[b.ipr * st];
          double m1 = w_vx * w_d, m2 = w_vy * w_d, m3 = w_vz * w_d;
          // ContravariantToCovariant (cubed_sphere_utility.hpp:30-36)
          const double v = m2, ww = m3;
          m2 = v + ww * cth;
          m3 = ww + v * cth;
          u[b.ivx * st] = m1;
          u[b.ivy * st] = m2;
          u[b.ivz * st] = m3;
          u[b.ipr * st] = w_p * igm1 + 0.5 * (m1 * w_vx + m2 * w_vy + m3 * w_vz);
          u[0] = w_d;
        }
      }
  }
}

// ---------------------------------------------------------------------------
// fluxes

namespace {

// SaveLR3DValues for every x2 / x3 face of the interior rows
void save_lr(Shell &s, int p) {
  Block &b = s.p[p];
  const int nv = b.nv;
  // x2: faces js..je+1 of rows k = ks..ke, i = is..ie
  {
    const int m = b.nc2;
    std::vector<double> q(m), l(m + 1), r(m + 1);
    for (int n = 0; n < nv; ++n)
      for (int k = b.ks; k <= b.ke; ++k)
        for (int i = b.is; i <= b.ie; ++i) {
          for (int j = 0; j < m; ++j) q[j] = b.w[b.idx(n, k, j, i)];
          if (b.cfg.recon == CANOE_RECON_PPM) ppm_line(q.data(), b.js, b.je + 1, l.data(), r.data());
          else plm_line(q.data(), b.js, b.je + 1, l.data(), r.data());
          for (int j = b.js; j <= b.je + 1; ++j) {
            const size_t f = (((size_t)n * b.nc3 + k) * (b.nc2 + 1) + j) * b.nc1 + i;
            s.L2[p][f] = l[j];
            s.R2[p][f] = r[j];
          }
        }
  }
  {
    const int m = b.nc3;
    std::vector<double> q(m), l(m + 1), r(m + 1);
    for (int n = 0; n < nv; ++n)
      for (int j = b.js; j <= b.je; ++j)
        for (int i = b.is; i <= b.ie; ++i) {
          for (int k = 0; k < m; ++k) q[k] = b.w[b.idx(n, k, j, i)];
          if (b.cfg.recon == CANOE_RECON_PPM) ppm_line(q.data(), b.ks, b.ke + 1, l.data(), r.data());
          else plm_line(q.data(), b.ks, b.ke + 1, l.data(), r.data());
          for (int k = b.ks; k <= b.ke + 1; ++k) {
            const size_t f = (((size_t)n * (b.nc3 + 1) + k) * b.nc2 + j) * b.nc1 + i;
            s.L3[p][f] = l[k];
            s.R3[p][f] = r[k];
          }
        }
  }
}

}  // namespace

// L/R swap across panel edges (sendNeighborBlocks / recvNeighborBlocks,
// cubed_sphere.cpp:312-681), over the interior i range
void shell_swap_lr(Shell &s) {
  const ShellGeo &g = s.geo;
  struct Msg {
    int target, tox2, tox3;
    std::vector<double> data;
  };
  std::vector<Msg> msgs;
  for (int p = 0; p < 6; ++p) {
    Block &b = s.p[p];
    const int block_id = p + 1;
    const int nv = b.nv, ivy = b.ivy, ivz = b.ivz;
    for (int target_dir = 0; target_dir < 4; ++target_dir) {
      const int ox2 = target_dir == 0 ? -1 : target_dir == 1 ? 1 : 0;
      const int ox3 = target_dir == 2 ? -1 : target_dir == 3 ? 1 : 0;
      const bool left = (target_dir == 1 || target_dir == 3);
      int tox2, tox3;
      transform_ox(block_id, ox2, ox3, tox2, tox3);
      int kb1, kb2, jb1, jb2;
      const int ib1 = b.is, ib2 = b.ie;
      const bool x2dir = ox2 != 0;
      if (ox2 == 1) { jb1 = jb2 = b.je + 1; kb1 = b.ks; kb2 = b.ke; }
      else if (ox2 == -1) { jb1 = jb2 = b.js; kb1 = b.ks; kb2 = b.ke; }
      else if (ox3 == 1) { jb1 = b.js; jb2 = b.je; kb1 = kb2 = b.ke + 1; }
      else { jb1 = b.js; jb2 = b.je; kb1 = kb2 = b.ks; }
      auto face = [&](bool l, int n, int k, int j, int i) -> double {
        if (x2dir) {
          const size_t f = (((size_t)n * b.nc3 + k) * (b.nc2 + 1) + j) * b.nc1 + i;
          return l ? s.L2[p][f] : s.R2[p][f];
        }
        const size_t f = (((size_t)n * (b.nc3 + 1) + k) * b.nc2 + j) * b.nc1 + i;
        return l ? s.L3[p][f] : s.R3[p][f];
      };
      const bool inv = kDinv[p][target_dir] == 1;
      Msg m;
      m.target = kTgbid[p][target_dir] - 1;
      m.tox2 = tox2;
      m.tox3 = tox3;
      for (int n = 0; n < nv; ++n)
        for (int kk = 0; kk <= kb2 - kb1; ++kk)
          for (int jj = 0; jj <= jb2 - jb1; ++jj)
            for (int i = ib1; i <= ib2; ++i) {
              const int k = inv ? kb2 - kk : kb1 + kk;
              const int j = inv ? jb2 - jj : jb1 + jj;
              if (n == ivy || n == ivz) {
                double x2s, x3s, x2d, x3d, pos_along;
                if (ox2 == 1) { x2s = PI / 4.0; x3s = g.x3v[k]; pos_along = x3s; }
                else if (ox2 == -1) { x2s = -PI / 4.0; x3s = g.x3v[k]; pos_along = x3s; }
                else if (ox3 == 1) { x2s = g.x2v[j]; x3s = PI / 4.0; pos_along = x2s; }
                else { x2s = g.x2v[j]; x3s = -PI / 4.0; pos_along = x2s; }
                const double pa = inv ? -pos_along : pos_along;
                if (tox2 == 1) { x2d = PI / 4.0; x3d = pa; }
                else if (tox2 == -1) { x2d = -PI / 4.0; x3d = pa; }
                else if (tox3 == 1) { x2d = pa; x3d = PI / 4.0; }
                else { x2d = pa; x3d = -PI / 4.0; }
                x2d = std::tan(x2d);
                x3d = std::tan(x3d);
                x2s = std::tan(x2s);
                x3s = std::tan(x3s);
                double U, V, vx, vy;
                vec_rll_from_abp(x2s, x3s, block_id, face(left, ivy, k, j, i),
                                 face(left, ivz, k, j, i), &U, &V);
                vec_abp_from_rll(x2d, x3d, m.target + 1, U, V, &vx, &vy);
                m.data.push_back(n == ivy ? vx : vy);
              } else {
                m.data.push_back(face(left, n, k, j, i));
              }
            }
      msgs.push_back(std::move(m));
    }
  }
  for (const Msg &m : msgs) {
    Block &t = s.p[m.target];
    const int ox2 = m.tox2, ox3 = m.tox3;
    const bool left = (ox2 == -1 || ox3 == -1);
    int kb1, kb2, jb1, jb2;
    const bool x2dir = ox2 != 0;
    if (ox2 == 1) { jb1 = jb2 = t.je + 1; kb1 = t.ks; kb2 = t.ke; }
    else if (ox2 == -1) { jb1 = jb2 = t.js; kb1 = t.ks; kb2 = t.ke; }
    else if (ox3 == 1) { jb1 = t.js; jb2 = t.je; kb1 = kb2 = t.ke + 1; }
    else { jb1 = t.js; jb2 = t.je; kb1 = kb2 = t.ks; }
    size_t q = 0;
    for (int n = 0; n < t.nv; ++n)
      for (int k = kb1; k <= kb2; ++k)
        for (int j = jb1; j <= jb2; ++j)
          for (int i = t.is; i <= t.ie; ++i) {
            const double v = m.data[q++];
            if (x2dir) {
              const size_t f = (((size_t)n * t.nc3 + k) * (t.nc2 + 1) + j) * t.nc1 + i;
              (left ? s.L2[m.target] : s.R2[m.target])[f] = v;
            } else {
              const size_t f = (((size_t)n * (t.nc3 + 1) + k) * t.nc2 + j) * t.nc1 + i;
              (left ? s.L3[m.target] : s.R3[m.target])[f] = v;
            }
          }
  }
}

namespace {

// x2 / x3 Riemann fluxes of one panel from the stored face states:
// PrimToLocal2/3 (gnomonic_equiangle.cpp:604-719), HLLC, FluxToGlobal2/3
// (:751-832) and the contravariant -> covariant flux projection
// (hllc_transform.cpp:245-272)
void riemann_x23(Shell &s, int p) {
  Block &b = s.p[p];
  const ShellGeo &g = s.geo;
  const int nv = b.nv, ivx = b.ivx, ivy = b.ivy, ivz = b.ivz;
  std::vector<double> wl(nv), wr(nv), fx(nv);
  // x2 faces
  for (int k = b.ks; k <= b.ke; ++k)
    for (int j = b.js; j <= b.je + 1; ++j) {
      const double cos_t = g.cosf2[g.kj(k, j)], sin_t = g.sinf2[g.kj(k, j)];
      const double g23 = cos_t, g33 = 1.0, gi22 = 1.0 / (sin_t * sin_t);
      const double x = std::tan(g.x2f[j]), y = std::tan(g.x3v[k]);
      const double C = std::sqrt(1. + x * x), D = std::sqrt(1. + y * y);
      const double cth = -x * y / C / D;
      for (int i = b.is; i <= b.ie; ++i) {
        for (int n = 0; n < nv; ++n) {
          const size_t f = (((size_t)n * b.nc3 + k) * (b.nc2 + 1) + j) * b.nc1 + i;
          wl[n] = s.L2[p][f];
          wr[n] = s.R2[p][f];
        }
        const double T22 = 1.0 / std::sqrt(gi22), T32 = g23 / std::sqrt(g33),
                     T33 = std::sqrt(g33);
        for (double *w : {wl.data(), wr.data()}) {
          const double u2 = w[ivy], u3 = w[ivz];
          w[ivy] = T22 * u2;
          w[ivz] = T32 * u2 + T33 * u3;
        }
        riemann_hllc(b.th, ivy, wl.data(), wr.data(), fx.data(), 1);
        const double F22 = std::sqrt(gi22), F32 = -std::sqrt(gi22) * g23 / g33,
                     F33 = 1.0 / std::sqrt(g33);
        const double txy = fx[ivy], txz = fx[ivz];
        fx[ivy] = F22 * txy;
        fx[ivz] = F32 * txy + F33 * txz;
        const double ty = fx[ivy], tz = fx[ivz];
        fx[ivy] = ty + tz * cth;
        fx[ivz] = tz + ty * cth;
        for (int n = 0; n < nv; ++n)
          b.flx2[(((size_t)n * b.nc3 + k) * (b.nc2 + 1) + j) * b.nc1 + i] = fx[n];
      }
    }
  // x3 faces
  for (int k = b.ks; k <= b.ke + 1; ++k)
    for (int j = b.js; j <= b.je; ++j) {
      const double cos_t = g.cosf3[g.kj(k, j)], sin_t = g.sinf3[g.kj(k, j)];
      const double g22 = 1.0, g23 = cos_t, gi33 = 1.0 / (sin_t * sin_t);
      const double x = std::tan(g.x2v[j]), y = std::tan(g.x3f[k]);
      const double C = std::sqrt(1. + x * x), D = std::sqrt(1. + y * y);
      const double cth = -x * y / C / D;
      for (int i = b.is; i <= b.ie; ++i) {
        for (int n = 0; n < nv; ++n) {
          const size_t f = (((size_t)n * (b.nc3 + 1) + k) * b.nc2 + j) * b.nc1 + i;
          wl[n] = s.L3[p][f];
          wr[n] = s.R3[p][f];
        }
        const double T22 = std::sqrt(g22), T23 = g23 / std::sqrt(g22),
                     T33 = 1.0 / std::sqrt(gi33);
        for (double *w : {wl.data(), wr.data()}) {
          const double u2 = w[ivy], u3 = w[ivz];
          w[ivy] = T22 * u2 + T23 * u3;
          w[ivz] = T33 * u3;
        }
        riemann_hllc(b.th, ivz, wl.data(), wr.data(), fx.data(), 1);
        const double F22 = 1.0 / std::sqrt(g22), F23 = -g23 / g22 * std::sqrt(gi33),
                     F33 = std::sqrt(gi33);
        const double txy = fx[ivy], txz = fx[ivz];
        fx[ivy] = F22 * txy + F23 * txz;
        fx[ivz] = F33 * txz;
        const double ty = fx[ivy], tz = fx[ivz];
        fx[ivy] = ty + tz * cth;
        fx[ivz] = tz + ty * cth;
        for (int n = 0; n < nv; ++n)
          b.flx3[(((size_t)n * (b.nc3 + 1) + k) * b.nc2 + j) * b.nc1 + i] = fx[n];
      }
    }
  (void)ivx;
}

// radial geometry of a panel cell (gnomonic_equiangle.cpp:224-432)
double face1_area(const Block &b, int k, int j, int i) {
  const ShellGeo &g = *b.geo;
  const size_t q = g.kj(k, j);
  return g.dx2a[q] * g.dx3a[q] * b.x1f[i] * b.x1f[i] * g.sinc[q];
}
double face2_area(const Block &b, int k, int j, int i) {
  return b.x1v[i] * b.geo->dx3a_f2[b.geo->kj(k, j)] * b.dx1f[i];
}
double face3_area(const Block &b, int k, int j, int i) {
  return b.x1v[i] * b.geo->dx2a_f3[b.geo->kj(k, j)] * b.dx1f[i];
}
double cell_volume(const Block &b, int k, int j, int i) {
  const ShellGeo &g = *b.geo;
  const size_t q = g.kj(k, j);
  return b.dx1f[i] * g.dx2a[q] * g.dx3a[q] * b.x1v[i] * b.x1v[i] * g.sinc[q];
}

}  // namespace

double shell_face1_area(const Block &b, int k, int j, int i) { return face1_area(b, k, j, i); }
double shell_cell_volume(const Block &b, int k, int j, int i) { return cell_volume(b, k, j, i); }

void shell_calculate_fluxes(Shell &s) {
  for (int p = 0; p < 6; ++p) calculate_fluxes_x1_only(s.p[p]);
  for (int p = 0; p < 6; ++p) save_lr(s, p);
  shell_swap_lr(s);
  for (int p = 0; p < 6; ++p) riemann_x23(s, p);
}

// Athena AddFluxDivergence (external; restated) with the panel's areas and
// volumes, then AddCoordTermsDivergence (gnomonic_equiangle.cpp:833-878)
void shell_add_divergence(Block &b, double wght, std::vector<double> &du) {
  const ShellGeo &g = *b.geo;
  const int nc1 = b.nc1, nc2 = b.nc2, nc3 = b.nc3;
  for (int k = b.ks; k <= b.ke; ++k)
    for (int j = b.js; j <= b.je; ++j)
      for (int i = b.is; i <= b.ie; ++i) {
        const double a1m = face1_area(b, k, j, i), a1p = face1_area(b, k, j, i + 1);
        const double a2m = face2_area(b, k, j, i), a2p = face2_area(b, k, j + 1, i);
        const double a3m = face3_area(b, k, j, i), a3p = face3_area(b, k + 1, j, i);
        const double vol = cell_volume(b, k, j, i);
        for (int n = 0; n < b.nv; ++n) {
          const size_t f1 = (((size_t)n * nc3 + k) * nc2 + j) * (nc1 + 1) + i;
          const size_t f2 = (((size_t)n * nc3 + k) * (nc2 + 1) + j) * nc1 + i;
          const size_t f3 = (((size_t)n * (nc3 + 1) + k) * nc2 + j) * nc1 + i;
          double dflx = a1p * b.flx1[f1 + 1] - a1m * b.flx1[f1];
          dflx += a2p * b.flx2[f2 + nc1] - a2m * b.flx2[f2];
          dflx += a3p * b.flx3[f3 + (size_t)nc2 * nc1] - a3m * b.flx3[f3];
          du[b.idx(n, k, j, i)] -= wght * dflx / vol;
        }
        // coordinate source terms
        const size_t q = g.kj(k, j);
        const double cosine = g.cosc[q];
        const double sine2 = g.sinc[q] * g.sinc[q];
        const double v1 = b.w[b.idx(b.ivx, k, j, i)], v2 = b.w[b.idx(b.ivy, k, j, i)],
                     v3 = b.w[b.idx(b.ivz, k, j, i)];
        const double radius = b.x1v[i];
        const double v_2 = v2 + v3 * cosine, v_3 = v3 + v2 * cosine;
        const double pr = b.w[b.idx(b.ipr, k, j, i)], rho = b.w[b.idx(0, k, j, i)];
        const double src1 = (2.0 * pr + rho * (v2 * v_2 + v3 * v_3)) / radius;
        du[b.idx(b.ivx, k, j, i)] += wght * src1;
        const double x_ov_rD =
            (a2m * g.sinf2[q] - a2p * g.sinf2[g.kj(k, j + 1)]) / vol;
        const double y_ov_rC =
            (a3m * g.sinf3[q] - a3p * g.sinf3[g.kj(k + 1, j)]) / vol;
        const double src2 = -x_ov_rD * (pr + rho * v3 * v3 * sine2) - rho * v1 * v_2 / radius;
        du[b.idx(b.ivy, k, j, i)] += wght * src2;
        const double src3 = -y_ov_rC * (pr + rho * v2 * v2 * sine2) - rho * v1 * v_3 / radius;
        du[b.idx(b.ivz, k, j, i)] += wght * src3;
      }
}

// One SSPRK(3,3) step of the shell: boundaries on u (exo3 exchange) and
// cons2prim, fluxes with the L/R swap, divergence + coordinate and gravity
// sources, implicit x1 correction on the projected velocities, update
void shell_step(Shell &s, double dt) {
  static const double g1[3] = {0., 0.25, 2. / 3.};
  static const double g2[3] = {1., 0.75, 1. / 3.};
  static const double be[3] = {1., 0.25, 2. / 3.};
  for (int stage = 0; stage < 3; ++stage) {
    shell_calculate_fluxes(s);
    const double wght = be[stage] * dt;
    for (int p = 0; p < 6; ++p) {
      Block &b = s.p[p];
      for (int n = 0; n < b.nv; ++n)
        for (int k = b.ks; k <= b.ke; ++k)
          for (int j = b.js; j <= b.je; ++j)
            for (int i = b.is; i <= b.ie; ++i) {
              const size_t c = b.idx(n, k, j, i);
              if (stage == 0) b.u1[c] = b.u[c];
              b.u[c] = g1[stage] * b.u[c] + g2[stage] * b.u1[c];
              b.du[c] = 0.;
            }
      shell_add_divergence(b, wght, b.du);
      add_gravity_source(b, wght, b.du);
      if (b.cfg.implicit_flag & 1) solve_implicit(b, b.du, wght);
      for (int n = 0; n < b.nv; ++n)
        for (int k = b.ks; k <= b.ke; ++k)
          for (int j = b.js; j <= b.je; ++j)
            for (int i = b.is; i <= b.ie; ++i) b.u[b.idx(n, k, j, i)] += b.du[b.idx(n, k, j, i)];
    }
    shell_fill_ghosts(s);
    shell_cons_to_prim(s);
  }
}

}  // namespace oracle
