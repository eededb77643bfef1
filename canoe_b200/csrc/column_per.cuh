// column_per.cuh -- the x1 pencil launcher for periodic x1 (both ends) in
// the implicit modes: the kernels with the bordered cyclic solve.  Kept out
// of column_ny*.cu so that the two sets of kernels compile in parallel.
#pragma once

#include "column.cuh"

namespace cb {

template <int NY, typename R>
int run_x1col_per(const Geom &g, const canoe_thermo_t &th, int recon, int rs, int flag,
                  int mode, const double *w, double *du, double *u, double *u1,
                  const double *dtp, const Stage &s, int stage, double *fout,
                  cudaStream_t st) {
  if (g.shell) {
    set_error("periodic radial boundaries are not supported on a cubed-sphere panel");
    return CANOE_ERR_UNSUPPORTED;
  }
  const int nimpl = (flag & 8) ? 5 : 3;
  ColLaunch cl;
  if (int rc = col_prepare(g, 5 + NY, nimpl, true, w, du, u, u1, cl)) return rc;
  auto go = [&](auto kern) -> int {
    return col_go(kern, cl, th, w, du, u, u1, dtp, s, stage, fout, st);
  };
  if (mode == kColSolveOnly)
    return nimpl == 3 ? go(k_x1col<NY, 3, 1, 3, kColSolveOnly, double, 0, true>)
                      : go(k_x1col<NY, 3, 1, 5, kColSolveOnly, double, 0, true>);
  if (mode == kColSolveStep)
    return nimpl == 3 ? go(k_x1col<NY, 3, 1, 3, kColSolveStep, double, 0, true>)
                      : go(k_x1col<NY, 3, 1, 5, kColSolveStep, double, 0, true>);
  const bool ppm = recon == CANOE_RECON_PPM, hllc = rs == CANOE_RSOLVER_HLLC;
#define CB_PCOL(NIMPL)                                                                    \
  (ppm ? (hllc ? go(k_x1col<NY, 3, 1, NIMPL, kColStep, R, 0, true>)                        \
               : go(k_x1col<NY, 3, 0, NIMPL, kColStep, R, 0, true>))                       \
       : (hllc ? go(k_x1col<NY, 2, 1, NIMPL, kColStep, R, 0, true>)                        \
               : go(k_x1col<NY, 2, 0, NIMPL, kColStep, R, 0, true>)))
  return nimpl == 3 ? CB_PCOL(3) : CB_PCOL(5);
#undef CB_PCOL
}

}  // namespace cb
