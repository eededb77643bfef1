// source.cu -- a user explicit source term of the stage: the viscous and
// thermal dissipation of the dense sinking bubble example
// (examples/2019-Li-snap/straka.cpp:125-190, enrolled with
// EnrollUserExplicitSourceFunction), added into du with the stage weight
// beta dt as ImplicitHydroTasks::AddSourceTerms adds the user sources
// (src/tasklist/implicit_hydro_tasks.cpp:192-216), after the x2 flux pass
// and before the x1 pencil kernel completes and solves du.
//
// On a 2-D block (nx3 = 1), with K the diffusivity, dx = dx1f(is),
// dy = dx2, and the 5-point sums of the neighbours minus four times the
// cell, S = beta dt K rho / (dx dy):
//   du(IM1) += S lap(v1),  du(IM2) += S lap(v2),
//   du(IEN) += S cp T / theta lap(theta),  theta = T (p0 / p)^((g-1)/g),
// with T = p / (rho R_d f_eps) and cp = g / (g - 1) R_d.
#include <cuda_runtime.h>

#include "block.cuh"

namespace cb {

namespace {

template <int NY>
__device__ __forceinline__ void temp_theta(const canoe_thermo_t &th, const double *w,
                                           int64_t sv, int64_t c, double p0, double chi,
                                           double &T, double &theta) {
  using S = Slots<NY>;
  double feps = 1.;
#pragma unroll
  for (int n = 1; n <= NY; ++n) {
    const double q = w[n * sv + c];
    feps += n <= th.nvapor ? q * th.inv_mu_ratio_m1[n - 1] : -q;
  }
  const double p = w[S::IPR * sv + c];
  T = p / (w[c] * th.rd * feps);
  theta = T * pow(p0 / p, chi);
}

template <int NY>
__global__ void __launch_bounds__(256)
    k_diffusion(Geom g, canoe_thermo_t th, const double *__restrict__ w,
                double *__restrict__ du, const double *__restrict__ dtp, double beta,
                double K, double p0) {
  using S = Slots<NY>;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.nx1 * g.nx2) return;
  const int i = g.is + t % g.nx1, j = g.js + t / g.nx1;
  const int64_t c = (int64_t)j * g.nc1 + i;  // k = ks = 0 on a 2-D block
  const int64_t sv = g.sv, sj = g.nc1;
  const double chi = (th.gammad - 1.) / th.gammad;
  const double cp = th.gammad / (th.gammad - 1.) * th.rd;
  const double dx = g.dx1f[g.is], dy = g.dx2;
  const double s = beta * dtp[0] * K * w[c] / (dx * dy);
  auto lap = [&](int n) {
    const double *v = w + n * sv;
    return v[c - 1] + v[c + 1] + v[c - sj] + v[c + sj] - 4. * v[c];
  };
  double T, th0, tm, thm, tp, thp, tjm, thjm, tjp, thjp;
  temp_theta<NY>(th, w, sv, c, p0, chi, T, th0);
  temp_theta<NY>(th, w, sv, c - 1, p0, chi, tm, thm);
  temp_theta<NY>(th, w, sv, c + 1, p0, chi, tp, thp);
  temp_theta<NY>(th, w, sv, c - sj, p0, chi, tjm, thjm);
  temp_theta<NY>(th, w, sv, c + sj, p0, chi, tjp, thjp);
  du[S::IVX * sv + c] += s * lap(S::IVX);
  du[S::IVY * sv + c] += s * lap(S::IVY);
  du[S::IPR * sv + c] += s * cp * T / th0 * (thp + thm + thjp + thjm - 4. * th0);
}

}  // namespace

int launch_diffusion(const Geom &g, const canoe_thermo_t &th, const double *w, double *du,
                     const double *dtp, double beta, double K, double p0, cudaStream_t st) {
  if (g.nx3 != 1 || g.nx2 < 2) {
    set_error("the dissipation source is defined on 2-D blocks (nx3 = 1, nx2 > 1)");
    return CANOE_ERR_UNSUPPORTED;
  }
  const int n = g.nx1 * g.nx2;
  const unsigned nb = (unsigned)((n + 255) / 256);
  switch (th.ny) {
    case 0: k_diffusion<0><<<nb, 256, 0, st>>>(g, th, w, du, dtp, beta, K, p0); break;
    case 1: k_diffusion<1><<<nb, 256, 0, st>>>(g, th, w, du, dtp, beta, K, p0); break;
    case 2: k_diffusion<2><<<nb, 256, 0, st>>>(g, th, w, du, dtp, beta, K, p0); break;
    case 3: k_diffusion<3><<<nb, 256, 0, st>>>(g, th, w, du, dtp, beta, K, p0); break;
    case 6: k_diffusion<6><<<nb, 256, 0, st>>>(g, th, w, du, dtp, beta, K, p0); break;
    default:
      set_error("unsupported number of mass-fraction slots");
      return CANOE_ERR_UNSUPPORTED;
  }
  CB_CUDA(cudaGetLastError());
  return 0;
}

}  // namespace cb
