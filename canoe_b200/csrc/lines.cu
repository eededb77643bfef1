// lines.cu -- the implicit solves along x2 and x3 (SolveImplicit3D X2DIR /
// X3DIR, canoe src/snap/implicit/solve_implicit_3d.cpp:25-89).
//
// The reference transposes du so that the direction's index runs fastest
// and reuses the column solver with mydir_ selecting the normal velocity.
// Here w and du are gathered into line-major scratch arrays by 32 x 32
// shared-memory tile transposes (coalesced on both sides), with the
// velocity slots rotated into the direction's frame (normal, then the next
// two cyclically: CopyPrimitives / FluxJacobian / Eigenvector,
// flux_decomposition.hpp:14-120).  The x1 pencil kernel in solve-only mode
// then solves every line, periodic ends included, on a geometry whose "x1"
// is the line, and IDN, the normal momentum and IEN are scattered back, the
// slots the reference copies back (:46-55, :79-88).  Gravity acts in x1
// only (partial_correction.cpp:59-63), so the line solves run without it.
// Dry blocks only: the block refuses moist x2 / x3 solves.
#include "block.cuh"

namespace cb {

namespace {

// line (o, c) of direction dir, position t, in the block layout:
//   x2: cell (ks + o, t, is + c); x3: cell (t, js + o, is + c)
struct LineMap {
  int nv, ivx, ipr, dir;
  int nx1, nout, L, nline;
  int64_t sv, tstride, ostride, obase;
};

__device__ __forceinline__ int src_slot(const LineMap &m, int np) {
  if (np >= m.ivx && np < m.ivx + 3) return m.ivx + (np - m.ivx + m.dir) % 3;
  return np;
}

// block array -> line-major T[np][o][c][t], all NV slots, all t
__global__ void k_line_gather(LineMap m, const double *__restrict__ src,
                              double *__restrict__ dst) {
  __shared__ double tile[32][33];
  const int ntc = (m.nx1 + 31) / 32;
  const int c0 = (int)(blockIdx.x % (unsigned)ntc) * 32;
  const int t0 = (int)(blockIdx.x / (unsigned)ntc) * 32;
  const int o = blockIdx.y, np = blockIdx.z;
  const double *s = src + src_slot(m, np) * m.sv + m.obase + (int64_t)o * m.ostride;
  for (int r = threadIdx.y; r < 32; r += 8) {
    const int t = t0 + r, c = c0 + threadIdx.x;
    if (t < m.L && c < m.nx1) tile[r][threadIdx.x] = s[(int64_t)t * m.tstride + c];
  }
  __syncthreads();
  double *d = dst + ((int64_t)np * m.nout + o) * m.nx1 * m.L;
  for (int r = threadIdx.y; r < 32; r += 8) {
    const int c = c0 + r, t = t0 + threadIdx.x;
    if (t < m.L && c < m.nx1) d[(int64_t)c * m.L + t] = tile[threadIdx.x][r];
  }
}

// line-major T -> block du: slots IDN, normal momentum, IEN; interior t
__global__ void k_line_scatter(LineMap m, const double *__restrict__ src,
                               double *__restrict__ dst) {
  __shared__ double tile[32][33];
  const int ntc = (m.nx1 + 31) / 32;
  const int c0 = (int)(blockIdx.x % (unsigned)ntc) * 32;
  const int t0 = (int)(blockIdx.x / (unsigned)ntc) * 32;
  const int o = blockIdx.y;
  const int np = blockIdx.z == 0 ? 0 : blockIdx.z == 1 ? m.ivx : m.ipr;
  const double *s = src + ((int64_t)np * m.nout + o) * m.nx1 * m.L;
  for (int r = threadIdx.y; r < 32; r += 8) {
    const int c = c0 + r, t = t0 + threadIdx.x;
    if (t < m.L && c < m.nx1) tile[r][threadIdx.x] = s[(int64_t)c * m.L + t];
  }
  __syncthreads();
  double *d = dst + src_slot(m, np) * m.sv + m.obase + (int64_t)o * m.ostride;
  for (int r = threadIdx.y; r < 32; r += 8) {
    const int t = t0 + r, c = c0 + threadIdx.x;
    if (t >= NG && t < NG + m.nline && c < m.nx1)
      d[(int64_t)t * m.tstride + c] = tile[threadIdx.x][r];
  }
}

LineMap line_map(const Geom &g, int dir) {
  LineMap m;
  m.nv = g.nv;
  m.ivx = 1 + g.ny;
  m.ipr = 4 + g.ny;
  m.dir = dir;
  m.nx1 = g.nx1;
  m.nline = dir == 1 ? g.nx2 : g.nx3;
  m.L = m.nline + 2 * NG;
  m.nout = dir == 1 ? g.nx3 : g.nx2;
  m.sv = g.sv;
  if (dir == 1) {
    m.tstride = g.nc1;
    m.ostride = g.sk;
    m.obase = (int64_t)g.ks * g.sk + g.is;
  } else {
    m.tstride = g.sk;
    m.ostride = g.nc1;
    m.obase = (int64_t)g.js * g.nc1 + g.is;
  }
  return m;
}

}  // namespace

bool line_solve_on(const Geom &g, int implicit_flag, int dir) {
  return dir == 1 ? ((implicit_flag & 2) && g.f2) : ((implicit_flag & 4) && g.f3);
}

size_t line_scratch_doubles(const Geom &g, int implicit_flag) {
  size_t n = 0;
  for (int dir = 1; dir <= 2; ++dir)
    if (line_solve_on(g, implicit_flag, dir)) {
      const LineMap m = line_map(g, dir);
      const size_t v = (size_t)m.nv * m.nout * m.nx1 * m.L;
      if (v > n) n = v;
    }
  return n;
}

int launch_line_solve(int dir, const Geom &g, const canoe_thermo_t &th, int implicit_flag,
                      const double *w, double *du, double *wt, double *dut,
                      const double *dxl, const double *dtp, const Stage &s,
                      cudaStream_t st) {
  if (g.ny > 0 || g.shell) {
    set_error("x2 / x3 implicit solves are provided for a dry Cartesian block");
    return CANOE_ERR_UNSUPPORTED;
  }
  const LineMap m = line_map(g, dir);
  const dim3 blk(32, 8);
  const unsigned ntiles = (unsigned)((m.nx1 + 31) / 32) * (unsigned)((m.L + 31) / 32);
  k_line_gather<<<dim3(ntiles, m.nout, m.nv), blk, 0, st>>>(m, w, wt);
  CB_CUDA(cudaGetLastError());
  k_line_gather<<<dim3(ntiles, m.nout, m.nv), blk, 0, st>>>(m, du, dut);
  CB_CUDA(cudaGetLastError());
  // the lines as x1 pencils: nx2 <- nx1 (c), nx3 <- nout (o)
  Geom t = g;
  t.nx1 = m.nline;
  t.nc1 = m.L;
  t.is = NG;
  t.ie = NG + m.nline - 1;
  t.nx2 = t.nc2 = g.nx1;
  t.js = 0;
  t.je = g.nx1 - 1;
  t.nx3 = t.nc3 = m.nout;
  t.ks = 0;
  t.ke = m.nout - 1;
  t.f2 = t.f3 = 0;
  t.bc[0] = g.bc[2 * dir];
  t.bc[1] = g.bc[2 * dir + 1];
  t.sk = (int64_t)t.nc2 * t.nc1;
  t.sv = (int64_t)t.nc3 * t.sk;
  // face area over twice the volume is 1 / (2 dx_line): unit transverse widths
  t.dx2 = t.dx3 = 1.;
  t.x1f = t.x1v = t.dx1f = dxl;
  t.pref = nullptr;
  t.shell = nullptr;
  canoe_thermo_t th0 = th;
  th0.grav = 0.;
  int rc = launch_x1col(t, th0, CANOE_RECON_PPM, CANOE_RSOLVER_HLLC, 1 | (implicit_flag & 8),
                        CANOE_FP64, kColSolveOnly, wt, dut, nullptr, nullptr, dtp, s, 0,
                        nullptr, st);
  if (rc) return rc;
  k_line_scatter<<<dim3(ntiles, m.nout, 3), blk, 0, st>>>(m, dut, du);
  CB_CUDA(cudaGetLastError());
  return 0;
}

}  // namespace cb
