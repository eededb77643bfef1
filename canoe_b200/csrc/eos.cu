// eos.cu -- cons -> prim over the whole block (ghost cells included), the
// CFL time step, and the saturation adjustment.
//
// k_cons_to_prim: every cell, interior or ghost, converts the conserved state
//   of its source cell (itself, or its reflected / periodic / outflow image
//   in the interior) and flips the normal velocity for reflecting walls.
//   This is EquationOfState::ConservedToPrimitive (snapy "U->W", canoe
//   src/snap/eos/ideal_moist_hydro.cpp:47-58) and the Athena boundary
//   conditions in one pass; interior cells also feed the device error word
//   (canoe src/checks.cpp:53-149) and the CFL minimum of
//   Hydro::NewBlockTimeStep (patches/21.new_blockdt.patch:20-40).
// k_satadj: the isochoric, isoenergetic saturation adjustment of
//   ImplicitHydroTasks::UpdateAllConserved (src/tasklist/implicit_hydro_tasks.
//   cpp:290-313), Newton on T with a bracketed fallback.
#include <cuda_runtime.h>

#include <algorithm>

#include "block.cuh"
#include "mlp.cuh"

namespace cb {

namespace {

__device__ __forceinline__ int map_ghost(int i, int lo, int hi, int n, int bcl,
                                         int bch, bool &flip) {
  if (i < lo) {
    if (bcl == CANOE_BC_REFLECT) {
      flip = !flip;
      return 2 * lo - 1 - i;
    }
    if (bcl == CANOE_BC_PERIODIC) return i + n;
    return lo;
  }
  if (i > hi) {
    if (bch == CANOE_BC_REFLECT) {
      flip = !flip;
      return 2 * hi + 1 - i;
    }
    if (bch == CANOE_BC_PERIODIC) return i - n;
    return hi;
  }
  return i;
}

__device__ __forceinline__ unsigned long long dbits(double x) {
  return (unsigned long long)__double_as_longlong(x);
}

template <int NY>
__global__ void __launch_bounds__(256)
    k_cons_to_prim(Geom g, canoe_thermo_t th, const double *__restrict__ u,
                   double *__restrict__ w, uint32_t *err,
                   unsigned long long *dt_acc, double cfl, int imp) {
  using S = Slots<NY>;
  constexpr int NV = S::NV;
  const int64_t total = (int64_t)g.nc3 * g.sk;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double dtc = __longlong_as_double(0x7ff0000000000000LL);
  uint32_t bits = 0;
  if (t < total) {
    // 32-bit index arithmetic where the block allows (64-bit division is
    // several times the instructions)
    int i, j, k;
    if (total <= 0x7fffffff) {
      const unsigned tt = (unsigned)t, r = tt / (unsigned)g.nc1;
      i = (int)(tt - r * (unsigned)g.nc1);
      j = (int)(r % (unsigned)g.nc2);
      k = (int)(r / (unsigned)g.nc2);
    } else {
      i = (int)(t % g.nc1);
      j = (int)((t / g.nc1) % g.nc2);
      k = (int)(t / g.sk);
    }
    bool f1 = false, f2 = false, f3 = false;
    const int si = map_ghost(i, g.is, g.ie, g.nx1, g.bc[0], g.bc[1], f1);
    const int sj = g.f2 ? map_ghost(j, g.js, g.je, g.nx2, g.bc[2], g.bc[3], f2) : j;
    const int sk = g.f3 ? map_ghost(k, g.ks, g.ke, g.nx3, g.bc[4], g.bc[5], f3) : k;
    const int64_t src = (int64_t)sk * g.sk + (int64_t)sj * g.nc1 + si;
    double uc[NV], wc[NV];
#pragma unroll
    for (int n = 0; n < NV; ++n) uc[n] = u[n * g.sv + src];
    cons_to_prim<NY>(th, uc, wc);
    if (f1) wc[S::IVX] = -wc[S::IVX];
    if (f2) wc[S::IVY] = -wc[S::IVY];
    if (f3) wc[S::IVZ] = -wc[S::IVZ];
#pragma unroll
    for (int n = 0; n < NV; ++n) w[n * g.sv + t] = wc[n];
    const bool interior = si == i && sj == j && sk == k;
    if (interior) {
      double rho = wc[0], p = wc[S::IPR];
      if (!(rho > 0.)) bits |= (rho != rho) ? CANOE_EBIT_NAN : CANOE_EBIT_NEG_DENSITY;
      if (!(p > 0.)) bits |= (p != p) ? CANOE_EBIT_NAN : CANOE_EBIT_NEG_PRESSURE;
      if (dt_acc) {
        double cs = sound_speed<double, NY>(th, wc);
        double d1 = g.dx1f[i];
        if ((imp & 1) && g.nx2 > 1)
          d1 /= cfl * fabs(wc[S::IVX]);
        else
          d1 /= (fabs(wc[S::IVX]) + cs);
        dtc = d1;
        // implicit x2 / x3: |v| only, as in x1
        if (g.f2)
          dtc = fmin(dtc, (imp & 2) ? g.dx2 / (cfl * fabs(wc[S::IVY]))
                                    : g.dx2 / (fabs(wc[S::IVY]) + cs));
        if (g.f3)
          dtc = fmin(dtc, (imp & 4) ? g.dx3 / (cfl * fabs(wc[S::IVZ]))
                                    : g.dx3 / (fabs(wc[S::IVZ]) + cs));
      }
    }
  }
  // warp reductions, then one per CTA (256 threads): one atomic per CTA on
  // the step's single dt accumulator instead of one per warp
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    dtc = fmin(dtc, __shfl_xor_sync(0xffffffffu, dtc, o));
    bits |= __shfl_xor_sync(0xffffffffu, bits, o);
  }
  __shared__ double sdt[8];
  __shared__ uint32_t sbits[8];
  const int wid = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    sdt[wid] = dtc;
    sbits[wid] = bits;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = 1; q < (int)(blockDim.x >> 5); ++q) {
      dtc = fmin(dtc, sdt[q]);
      bits |= sbits[q];
    }
    if (bits) atomicOr(err, bits);
    if (dt_acc && dtc < __longlong_as_double(0x7ff0000000000000LL)) atomicMin(dt_acc, dbits(dtc));
  }
}

// horizontal mean of the pressure at every x1 level (ghosts included): the
// reference profile of the FP32 flux path
template <int NY>
__global__ void k_level_mean_pressure(Geom g, const double *__restrict__ w,
                                      double *__restrict__ pref) {
  const int i = blockIdx.x;
  const int ncol = g.nx2 * g.nx3;
  double s = 0.;
  for (int c = threadIdx.x; c < ncol; c += blockDim.x) {
    const int j = g.js + c % g.nx2, k = g.ks + c / g.nx2;
    s += w[Slots<NY>::IPR * g.sv + (int64_t)k * g.sk + (int64_t)j * g.nc1 + i];
  }
  __shared__ double red[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t += red[q];
    pref[i] = t / ncol;
  }
}

__global__ void k_dt_finalize(double *d_dt, unsigned long long *acc, double cfl,
                              double fixed_dt) {
  if (fixed_dt > 0.)
    d_dt[0] = fixed_dt;
  else
    d_dt[0] = cfl * __longlong_as_double((long long)*acc);
  *acc = 0x7ff0000000000000ULL;
}

// ---------------------------------------------------------------------------
// saturation adjustment (model and algorithm as documented in the header of
// this function's host entry point, canoe_saturation_adjust)

template <int NY>
struct SatCell {
  double rho, ie, qd;
  double qt[NY > 0 ? NY : 1];
  double qinert[NY + 1];
};

template <int NY>
__device__ __forceinline__ void sat_eval(const canoe_thermo_t &th, const SatCell<NY> &c,
                                         double T, int fv, int fphase, double &f,
                                         double &fp, double *q) {
  const double cvd = th.rd / (th.gammad - 1.);
#pragma unroll
  for (int n = 0; n <= NY; ++n) q[n] = c.qinert[n];
  double cvs = c.qd, lat = 0., dlat = 0.;
#pragma unroll
  for (int n = 1; n <= NY; ++n)
    if (c.qinert[n] != 0.) {
      cvs += c.qinert[n] * (1. + th.cv_ratio_m1[n - 1]);
      lat += c.qinert[n] * th.u0[n - 1];
    }
#pragma unroll
  for (int v = 0; v < (NY > 0 ? NY : 1); ++v) {
    if (v >= th.nvapor) break;
    const int vs = 1 + v, ls = th.liq_slot[v], ss = th.ice_slot[v];
    if (ls < 0 && ss < 0) {
#pragma unroll
      for (int n = 1; n <= NY; ++n)
        if (n == vs) q[n] = c.qt[v];
      cvs += c.qt[v] * (1. + th.cv_ratio_m1[vs - 1]);
      continue;
    }
    bool liquid = (ss < 0) || (ls >= 0 && T >= th.t3[v]);
    if (v == fv) liquid = (fphase == 0);
    const int cs = liquid ? ls : ss;
    const double beta = liquid ? th.beta_l[v] : th.beta_s[v];
    const double delta = liquid ? th.delta_l[v] : th.delta_s[v];
    const double rv = th.rd * (1. + th.inv_mu_ratio_m1[vs - 1]);
    const double lnps =
        log(th.p3[v]) + beta * (1. - th.t3[v] / T) - delta * log(T / th.t3[v]);
    const double qs = exp(lnps) / (c.rho * rv * T);
    double qv, qc, dqv;
    if (qs < c.qt[v]) {
      qv = qs;
      qc = c.qt[v] - qs;
      dqv = qs * (beta * th.t3[v] / (T * T) - delta / T - 1. / T);
    } else {
      qv = c.qt[v];
      qc = 0.;
      dqv = 0.;
    }
    const double cvv = 1. + th.cv_ratio_m1[vs - 1];
    const double cvc = 1. + th.cv_ratio_m1[cs - 1];
#pragma unroll
    for (int n = 1; n <= NY; ++n) {
      if (n == vs) q[n] = qv;
      if (n == cs) q[n] += qc;
    }
    cvs += qv * cvv + qc * cvc;
    lat += qc * th.u0[cs - 1];
    dlat += dqv * (cvd * cvv * T - cvd * cvc * T - th.u0[cs - 1]);
  }
  f = c.rho * (cvd * cvs * T + lat) - c.ie;
  fp = c.rho * (cvd * cvs + dlat);
}

// true when no liquid or ice slot of the cell holds water
template <int NY>
__device__ __forceinline__ bool all_vapour(const canoe_thermo_t &th, const double *q) {
  bool dry = true;
#pragma unroll
  for (int v = 0; v < (NY > 0 ? NY : 1); ++v) {
    if (v >= th.nvapor) break;
#pragma unroll
    for (int n = 1; n <= NY; ++n)
      if ((n == th.liq_slot[v] || n == th.ice_slot[v]) && q[n] != 0.) dry = false;
  }
  return dry;
}

// a guess below this much latent heating [K] keeps the cold start, which is
// exact in one step for cells that stay unsaturated
constexpr double kSatGate = 0.05;

// returns the number of f evaluations; flags bit0 fallback, bit1 not
// converged, bit2 the cell is returned unchanged (no write needed).  Start
// (o.warm): 0 the unadjusted temperature (cold); 1 the guess; 2 gated: the
// guess if it exceeds the cold start by kSatGate.
template <int NY>
__device__ int sat_cell(const canoe_thermo_t &th, const canoe_satadj_opts_t &o,
                        double *uc, double t_guess, double &t_out, int &flags) {
  using S = Slots<NY>;
  const double cvd = th.rd / (th.gammad - 1.);
  SatCell<NY> c;
  c.rho = uc[0];
#pragma unroll
  for (int n = 1; n <= NY; ++n) c.rho += uc[n];
  const double m1 = uc[S::IVX], m2 = uc[S::IVY], m3 = uc[S::IVZ];
  const double ke = 0.5 * (m1 * m1 + m2 * m2 + m3 * m3) / c.rho;
  c.ie = uc[S::IPR] - ke;
  double q[NY + 1];
  double qsum = 0.;
  q[0] = 0.;
#pragma unroll
  for (int n = 1; n <= NY; ++n) {
    q[n] = uc[n] / c.rho;
    qsum += q[n];
  }
  c.qd = 1. - qsum;
  bool member[NY + 1];
#pragma unroll
  for (int n = 0; n <= NY; ++n) {
    c.qinert[n] = 0.;
    member[n] = false;
  }
#pragma unroll
  for (int v = 0; v < (NY > 0 ? NY : 1); ++v) {
    if (v >= th.nvapor) break;
    double qt = 0.;
#pragma unroll
    for (int n = 1; n <= NY; ++n)
      if (n == 1 + v) {
        qt = q[n];
        member[n] = true;
      }
    const int ls = th.liq_slot[v], ss = th.ice_slot[v];
#pragma unroll
    for (int n = 1; n <= NY; ++n)
      if (ls > 0 && n == ls) {
        qt += q[n];
        member[n] = true;
      }
#pragma unroll
    for (int n = 1; n <= NY; ++n)
      if (ss > 0 && n == ss) {
        qt += q[n];
        member[n] = true;
      }
    c.qt[v] = qt;
  }
#pragma unroll
  for (int n = 1; n <= NY; ++n)
    if (!member[n]) c.qinert[n] = q[n];
  double cvs = c.qd, lat = 0.;
#pragma unroll
  for (int n = 1; n <= NY; ++n) {
    cvs += q[n] * (1. + th.cv_ratio_m1[n - 1]);
    lat += q[n] * th.u0[n - 1];
  }
  const double t_cold = (c.ie / c.rho - lat) / (cvd * cvs);

  int iters = 0;
  bool fallback = false, converged = false;
  double T = t_cold;
  const bool guess_ok = isfinite(t_guess) && t_guess > 1. && t_guess < 1.e4;
  if (o.warm == 1 && guess_ok) T = t_guess;
  double fprev = __longlong_as_double(0x7ff0000000000000LL);
  double f, fp;
  double qn[NY + 1];
  // gated start: the guess when it predicts latent heating, else cold
  if (o.warm == 2 && guess_ok && t_guess - t_cold > kSatGate) T = t_guess;
  // a cell whose water is all vapour and that stays below saturation at
  // the cold start is already the equilibrium: Newton would end where it
  // starts (to about 1e-13 K) and write the vapour back through a density
  // round trip, so the first evaluation returns it unchanged (flags bit 2)
  const bool dry_in = all_vapour<NY>(th, q);
  const int it0 = 0;
  for (int it = it0; it < o.max_iter && !converged; ++it) {
    sat_eval<NY>(th, c, T, -1, 0, f, fp, qn);
    if (it == 0 && dry_in && T == t_cold) {
      if (all_vapour<NY>(th, qn)) {
        t_out = t_cold;
        flags = 4;
        return 1;
      }
    }
    if (!(fabs(f) < fprev) && it > 0) {
      fallback = true;
      break;
    }
    const double dT = -f / fp;
    T += dT;
    iters++;
    fprev = fabs(f);
    if (fabs(dT) < o.tol) {
      converged = true;
      // one polishing Newton step: the result no longer depends on which
      // iterate first met the tolerance (cold vs warm start agree to roundoff)
      sat_eval<NY>(th, c, T, -1, 0, f, fp, qn);
      T -= f / fp;
      iters++;
      break;
    }
  }
  if (!converged) {
    fallback = true;
    double lo = 1., hi = 1.e4;
    if (!(T > lo && T < hi)) T = t_cold;
    for (int it = 0; it < 200; ++it) {
      sat_eval<NY>(th, c, T, -1, 0, f, fp, qn);
      if (f < 0.) lo = T;
      else hi = T;
      double tn = T - f / fp;
      if (!(tn > lo && tn < hi)) tn = 0.5 * (lo + hi);
      const double dT = tn - T;
      T = tn;
      iters++;
      if (fabs(dT) < o.tol || hi - lo < o.tol) {
        converged = true;
        sat_eval<NY>(th, c, T, -1, 0, f, fp, qn);
        // polish unless the step leaves the bracket (a root on a jump)
        const double tp = T - f / fp;
        if (tp > lo - 2. * o.tol && tp < hi + 2. * o.tol) T = tp;
        break;
      }
    }
  }
  sat_eval<NY>(th, c, T, -1, 0, f, fp, qn);
  // root on a liquid / ice jump at t3: split the condensate
#pragma unroll
  for (int v = 0; v < (NY > 0 ? NY : 1); ++v) {
    if (v >= th.nvapor) break;
    const int ls = th.liq_slot[v], ss = th.ice_slot[v];
    if (ls < 0 || ss < 0) continue;
    // f is increasing in T, so the root sits on the jump iff
    // f_ice(t3) < 0 < f_liquid(t3); only iterates ending near t3 can be there
    if (fabs(T - th.t3[v]) > 1e-3) continue;
    double fl, fs, fpl, fps;
    double ql[NY + 1], qs_[NY + 1];
    sat_eval<NY>(th, c, th.t3[v], v, 0, fl, fpl, ql);
    sat_eval<NY>(th, c, th.t3[v], v, 1, fs, fps, qs_);
    if ((fl > 0.) == (fs > 0.)) continue;
    const double x = -fs / (fl - fs);
    T = th.t3[v];
    double qc = 0.;
#pragma unroll
    for (int n = 1; n <= NY; ++n)
      if (n == ls) qc = ql[n];
#pragma unroll
    for (int n = 0; n <= NY; ++n) {
      qn[n] = ql[n];
      if (n == ls) qn[n] = x * qc;
      if (n == ss) qn[n] = qc - x * qc;
    }
    break;
  }
#pragma unroll
  for (int n = 1; n <= NY; ++n) uc[n] = qn[n] * c.rho;
  t_out = T;
  flags = (fallback ? 1 : 0) | (converged ? 0 : 2);
  return iters;
}

// network inputs of a conserved cell: rho, specific internal energy, total
// of the first and second condensable families
template <int NY>
__device__ __forceinline__ double mlp_features(const canoe_thermo_t &th, const double *uc,
                                               float *x) {
  using S = Slots<NY>;
  double rho = uc[0];
#pragma unroll
  for (int n = 1; n <= NY; ++n) rho += uc[n];
  const double ke = 0.5 * (uc[S::IVX] * uc[S::IVX] + uc[S::IVY] * uc[S::IVY] +
                           uc[S::IVZ] * uc[S::IVZ]) / rho;
  double fam[2] = {0., 0.};
#pragma unroll
  for (int v = 0; v < 2; ++v) {
    if (v >= th.nvapor) break;
#pragma unroll
    for (int n = 1; n <= NY; ++n)
      if (n == 1 + v || n == th.liq_slot[v] || n == th.ice_slot[v]) fam[v] += uc[n];
  }
  const double ev = (uc[S::IPR] - ke) / rho;
  x[0] = (float)rho;
  x[1] = (float)ev;
  x[2] = (float)(fam[0] / rho);
  x[3] = (float)(fam[1] / rho);
  // temperature with all water as vapour: the baseline the network corrects
  double cvs = 1.;
#pragma unroll
  for (int v = 0; v < 2; ++v)
    if (v < th.nvapor) cvs += fam[v] / rho * th.cv_ratio_m1[v];
  return ev / (th.rd / (th.gammad - 1.) * cvs);
}

// true when a condensable family of the cell is at or above saturation at
// the all-vapour temperature tv (the lowest temperature the adjustment can
// reach); otherwise the all-vapour state is the equilibrium, which the cold
// start finds exactly, and a learned guess cannot help
template <int NY>
__device__ __forceinline__ bool may_condense(const canoe_thermo_t &th, const double *uc,
                                             double tv) {
  double rho = uc[0];
#pragma unroll
  for (int n = 1; n <= NY; ++n) rho += uc[n];
  bool any = false;
#pragma unroll
  for (int v = 0; v < (NY > 0 ? NY : 1); ++v) {
    if (v >= th.nvapor) break;
    const int ls = th.liq_slot[v], ss = th.ice_slot[v];
    if (ls < 0 && ss < 0) continue;
    double fam = 0.;
#pragma unroll
    for (int n = 1; n <= NY; ++n)
      if (n == 1 + v || n == ls || n == ss) fam += uc[n];
    const bool liquid = (ss < 0) || (ls >= 0 && tv >= th.t3[v]);
    const float beta = float(liquid ? th.beta_l[v] : th.beta_s[v]);
    const float delta = float(liquid ? th.delta_l[v] : th.delta_s[v]);
    const float rv = float(th.rd * (1. + th.inv_mu_ratio_m1[v]));
    // a heuristic with a 1e-3 margin: FP32 intrinsics (relative error ~1e-6)
    // are ample and cost a fraction of the FP64 exp / log
    const float r = float(th.t3[v] / tv);
    const float ps = float(th.p3[v]) * __expf(beta * (1.f - r) + delta * __logf(r));
    // vapour density of the family against saturation, with a 1e-3 margin
    any = any || !(float(fam) * rv * float(tv) < (1.f - 1e-3f) * ps);
  }
  return any;
}

// the tensor-core state a CTA of the learned kernel carries across chunks
struct UmmaState {
  uint32_t phase;  // mbarrier phase of the next inference
  bool live;       // false once a bounded wait gave up: no further inference
  bool pending;    // the last inference's MMAs were not seen to complete
  // this warp's statistics so far (cells, evaluations, fallbacks, not
  // converged; the same on every lane), added to the global counters once
  // per CTA or warp by the kernel rather than per chunk: every warp adding
  // to the same four addresses serialised in L2
  uint32_t acc[4];
};

// add a warp's (or CTA's) statistics to the global counters
__device__ __forceinline__ void satadj_flush(unsigned long long *stats, const uint32_t *acc) {
  if (!acc[0]) return;
  atomicAdd(&stats[0], (unsigned long long)acc[0]);
  atomicAdd(&stats[1], (unsigned long long)acc[1]);
  if (acc[2]) atomicAdd(&stats[2], (unsigned long long)acc[2]);
  if (acc[3]) atomicAdd(&stats[3], (unsigned long long)acc[3]);
}

// The network's inference as a call rather than inlined code: most warps of
// a step never run it (no cell near saturation), and inlined it would hold
// registers across the Newton iteration of every warp.
constexpr int kSatWg = 6;  // warpgroups per CTA of the learned adjustment (24 warps)

__device__ __forceinline__ float mlp_infer_call(uint8_t *sm, const float *p, const float *x,
                                             bool warp_run, uint32_t phase, bool *ok) {
  return mlp_umma_infer<kSatWg>(sm, p, x, warp_run, phase, ok);
}

// One chunk of the adjustment: this thread takes cell t.  With LEARNED the
// chunk is the work of warpgroup wg, all of whose threads take part (it
// holds the warpgroup's named barriers), and sm / us are the CTA's shared
// memory and the warpgroup's tensor-core state.
template <int NY, bool LEARNED>
__device__ __forceinline__ void satadj_chunk(
    const canoe_thermo_t &th, const canoe_satadj_opts_t &o, double *__restrict__ u,
    int64_t ncells, int64_t stride, const Geom &g, int use_geom,
    const double *__restrict__ t_guess, double *__restrict__ t_out,
    int32_t *__restrict__ iters, unsigned long long *stats, const MlpView &mv,
    double *__restrict__ guess_out, uint32_t *err, int64_t t, uint8_t *sm, UmmaState &us,
    int wg) {
  using S = Slots<NY>;
  int it = 0, fl = 0;
  bool active = t < ncells;
  int64_t off = t;
  double uc[S::NV];
  if (active) {
    if (use_geom) {
      const int i = g.is + (int)(t % g.nx1);
      const int64_t r = t / g.nx1;
      const int j = g.js + (int)(r % g.nx2), k = g.ks + (int)(r / g.nx2);
      off = (int64_t)k * g.sk + (int64_t)j * g.nc1 + i;
    }
#pragma unroll
    for (int n = 0; n < S::NV; ++n) uc[n] = u[n * stride + off];
  }
  double tg = t_guess && active ? t_guess[t] : 0.;
  double tdry = 0.;
  bool need = false;
  if constexpr (LEARNED) {
    // the chunk's cells go through the tensor cores together (tcgen05,
    // mlp_umma_infer); a chunk with no cell near saturation skips the
    // inference, and within one that runs it, so does a warp whose cells all
    // stay unsaturated
    float x[kMlpIn] = {0.f, 0.f, 0.f, 0.f};
    if (active) {
      tdry = mlp_features<NY>(th, uc, x);
      need = may_condense<NY>(th, uc, tdry);
    }
    tg = __longlong_as_double(0x7ff8000000000000LL);  // no guess: cold start
    // every thread of the warpgroup reaches this barrier
    const bool wg_need = bar_red_or(1 + wg, kUmmaM, need);
    if (wg_need && us.live) {
      const bool warp_run = __any_sync(0xffffffffu, need);
#pragma unroll
      for (int q = 0; q < kMlpIn; ++q)
        x[q] = active ? (x[q] - mv.in_mean[q]) * mv.in_istd[q] : 0.f;
      bool ok = false;
      const float yn = mlp_infer_call(sm, mv.p, x, warp_run, us.phase, &ok);
      if (ok) {
        us.phase ^= 1u;
      } else {
        us.live = false;
        us.pending = true;
        if (threadIdx.x % kUmmaM == 0 && err) atomicOr(err, (uint32_t)CANOE_EBIT_TIMEOUT);
      }
      if (need && ok) tg = tdry + (double)(yn * mv.out_std + mv.out_mean);
    }
    if (guess_out && active) guess_out[t] = tg;
  }
  // the learned start's screen (may_condense, with its 1e-3 margin) also
  // decides the cells that stay all vapour: a warp whose cells are all such
  // ends here, as sat_cell's first evaluation would end them
  bool skip = false;
  if constexpr (LEARNED)
    skip = __all_sync(0xffffffffu, !active || (!need && all_vapour<NY>(th, uc)));
  if (skip) {
    if (active && t_out) t_out[t] = tdry;
    if (active && iters) iters[t] = 0;
  } else if (active) {
    double T;
    it = sat_cell<NY>(th, o, uc, tg, T, fl);
    if (!(fl & 4)) {
#pragma unroll
      for (int n = 1; n <= NY; ++n) u[n * stride + off] = uc[n];
    }
    if (t_out) t_out[t] = T;
    if (iters) iters[t] = it;
  }
  if (stats) {
    uint32_t a = active ? 1u : 0u, b = (uint32_t)it, c = (fl & 1) ? 1u : 0u,
             d = (fl & 2) ? 1u : 0u;
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) {
      a += __shfl_xor_sync(0xffffffffu, a, s);
      b += __shfl_xor_sync(0xffffffffu, b, s);
      c += __shfl_xor_sync(0xffffffffu, c, s);
      d += __shfl_xor_sync(0xffffffffu, d, s);
    }
    us.acc[0] += a;
    us.acc[1] += b;
    us.acc[2] += c;
    us.acc[3] += d;
  }
}


// the cold start: one 256-cell chunk per CTA, three CTAs per SM (80
// registers)
template <int NY>
__global__ void __launch_bounds__(256, 3)
    k_satadj(canoe_thermo_t th, canoe_satadj_opts_t o, double *__restrict__ u,
             int64_t ncells, int64_t stride, Geom g, int use_geom,
             const double *__restrict__ t_guess, double *__restrict__ t_out,
             int32_t *__restrict__ iters, unsigned long long *stats) {
  UmmaState us{0u, false, false, {0u, 0u, 0u, 0u}};
  satadj_chunk<NY, false>(th, o, u, ncells, stride, g, use_geom, t_guess, t_out, iters, stats,
                          MlpView{}, nullptr, nullptr,
                          (int64_t)blockIdx.x * blockDim.x + threadIdx.x, nullptr, us, 0);
  // one set of atomics per warp: a CTA-wide sum first (a barrier at the end)
  // made C4's cold start slower (2.95 -> 3.07 ms)
  if (stats && (threadIdx.x & 31) == 0) satadj_flush(stats, us.acc);
}

// the learned start: one persistent CTA of kSatWg warpgroups per SM (a
// kernel holding TMEM instructions is resident at one CTA per SM, mlp.cuh).
// The CTA stages the network and allocates its TMEM once; warpgroup g of CTA
// b then takes the 128-cell chunks b kSatWg + g, b kSatWg + g + gridDim.x
// kSatWg, ..., independently of the CTA's other warpgroups.
template <int NY>
__global__ void __launch_bounds__(kSatWg * kUmmaM, 1)
    k_satadj_learned(canoe_thermo_t th, canoe_satadj_opts_t o, double *__restrict__ u,
                     int64_t ncells, int64_t stride, Geom g, int use_geom,
                     const double *__restrict__ t_guess, double *__restrict__ t_out,
                     int32_t *__restrict__ iters, unsigned long long *stats, MlpView mv,
                     double *__restrict__ guess_out, uint32_t *err) {
  extern __shared__ __align__(1024) uint8_t dsm[];
  mlp_umma_setup<kSatWg>(dsm, mv.p, mv.w2h);
  UmmaState us{0u, true, false, {0u, 0u, 0u, 0u}};
  const int wg = threadIdx.x / kUmmaM;
  const int64_t nchunk = (ncells + kUmmaM - 1) / kUmmaM;
  for (int64_t c = (int64_t)blockIdx.x * kSatWg + wg; c < nchunk;
       c += (int64_t)gridDim.x * kSatWg)
    satadj_chunk<NY, true>(th, o, u, ncells, stride, g, use_geom, t_guess, t_out, iters, stats,
                           mv, guess_out, err, c * kUmmaM + threadIdx.x % kUmmaM, dsm, us, wg);
  if (stats && (threadIdx.x & 31) == 0) satadj_flush(stats, us.acc);
  mlp_umma_teardown<kSatWg>(dsm, us.pending, us.phase);
}

}  // namespace

int launch_cons_to_prim(const Geom &g, const canoe_thermo_t &th, const double *u,
                        double *w, uint32_t *err, unsigned long long *dt_acc,
                        double cfl, int imp, cudaStream_t st) {
  const int64_t total = (int64_t)g.nc3 * g.sk;
  const unsigned nb = (unsigned)((total + 255) / 256);
  switch (th.ny) {
    case 0: k_cons_to_prim<0><<<nb, 256, 0, st>>>(g, th, u, w, err, dt_acc, cfl, imp); break;
    case 1: k_cons_to_prim<1><<<nb, 256, 0, st>>>(g, th, u, w, err, dt_acc, cfl, imp); break;
    case 2: k_cons_to_prim<2><<<nb, 256, 0, st>>>(g, th, u, w, err, dt_acc, cfl, imp); break;
    case 3: k_cons_to_prim<3><<<nb, 256, 0, st>>>(g, th, u, w, err, dt_acc, cfl, imp); break;
    case 6: k_cons_to_prim<6><<<nb, 256, 0, st>>>(g, th, u, w, err, dt_acc, cfl, imp); break;
    default:
      set_error("unsupported number of mass-fraction slots");
      return CANOE_ERR_UNSUPPORTED;
  }
  CB_CUDA(cudaGetLastError());
  return 0;
}

int launch_level_mean_pressure(const Geom &g, int ny, const double *w, double *pref,
                               cudaStream_t st) {
  switch (ny) {
    case 0: k_level_mean_pressure<0><<<g.nc1, 256, 0, st>>>(g, w, pref); break;
    case 1: k_level_mean_pressure<1><<<g.nc1, 256, 0, st>>>(g, w, pref); break;
    case 2: k_level_mean_pressure<2><<<g.nc1, 256, 0, st>>>(g, w, pref); break;
    case 3: k_level_mean_pressure<3><<<g.nc1, 256, 0, st>>>(g, w, pref); break;
    case 6: k_level_mean_pressure<6><<<g.nc1, 256, 0, st>>>(g, w, pref); break;
    default:
      set_error("unsupported number of mass-fraction slots");
      return CANOE_ERR_UNSUPPORTED;
  }
  CB_CUDA(cudaGetLastError());
  return 0;
}

int launch_dt_finalize(double *d_dt, unsigned long long *acc, double cfl,
                       double fixed_dt, cudaStream_t st) {
  k_dt_finalize<<<1, 1, 0, st>>>(d_dt, acc, cfl, fixed_dt);
  CB_CUDA(cudaGetLastError());
  return 0;
}

int launch_satadj(const canoe_thermo_t &th, const canoe_satadj_opts_t &o, double *u,
                  int64_t ncells, int64_t stride, const Geom *g, const double *t_guess,
                  double *t_out, int32_t *iters, unsigned long long *stats,
                  cudaStream_t st, const MlpView *mlp, double *guess_out, uint32_t *err) {
  if (ncells <= 0) return 0;
  Geom gg{};
  if (g) gg = *g;
  MlpView mv{};
  if (mlp) mv = *mlp;
  const int ug = g ? 1 : 0;
  int grid = 0;
#define CB_SAT(NY)                                                                         \
  if (mlp) {                                                                               \
    CB_CUDA(umma_persistent_grid<kSatWg>(k_satadj_learned<NY>, (ncells + kUmmaM - 1) / kUmmaM, \
                                         &grid));                                          \
    k_satadj_learned<NY><<<grid, kSatWg * kUmmaM, UmmaLayout<kSatWg>::kBytes, st>>>(       \
        th, o, u, ncells, stride, gg, ug, t_guess, t_out, iters, stats, mv, guess_out, err); \
  } else {                                                                                 \
    k_satadj<NY><<<(unsigned)((ncells + 255) / 256), 256, 0, st>>>(                        \
        th, o, u, ncells, stride, gg, ug, t_guess, t_out, iters, stats);                   \
  }
  switch (th.ny) {
    case 1: CB_SAT(1); break;
    case 2: CB_SAT(2); break;
    case 3: CB_SAT(3); break;
    case 6: CB_SAT(6); break;
    case 0: return 0;
    default:
      set_error("unsupported number of mass-fraction slots");
      return CANOE_ERR_UNSUPPORTED;
  }
#undef CB_SAT
  CB_CUDA(cudaGetLastError());
  return 0;
}

}  // namespace cb
