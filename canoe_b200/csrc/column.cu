// column.cu -- dispatch of the x1 pencil kernel over the species count.
#include "column.cuh"

namespace cb {

#define CB_DECL(NY)                                                                \
  extern template int run_x1col<NY>(const Geom &, const canoe_thermo_t &, int, int, \
                                    int, int, int, const double *, double *, double *, \
                                    double *, const double *, const Stage &, int,   \
                                    double *, cudaStream_t);
CB_DECL(0)
CB_DECL(1)
CB_DECL(2)
CB_DECL(3)
CB_DECL(6)
#undef CB_DECL

int launch_x1col(const Geom &g, const canoe_thermo_t &th, int recon, int rs, int flag,
                 int prec, int mode, const double *w, double *du, double *u, double *u1,
                 const double *dtp, const Stage &s, int stage, double *fo,
                 cudaStream_t st) {
  if ((flag & 1) && mode != kColFluxOnly && g.bc[0] == CANOE_BC_PERIODIC) {
    // the cyclic solve couples the two ends (periodic_forward_backward.hpp)
    if (g.bc[1] != CANOE_BC_PERIODIC) {
      set_error("periodic x1 needs both x1 boundaries periodic");
      return CANOE_ERR_ARG;
    }
    if (g.nx1 < 3) {
      set_error("the periodic implicit x1 solve needs at least 3 levels");
      return CANOE_ERR_ARG;
    }
  }
  switch (th.ny) {
    case 0: return run_x1col<0>(g, th, recon, rs, flag, prec, mode, w, du, u, u1, dtp, s, stage, fo, st);
    case 1: return run_x1col<1>(g, th, recon, rs, flag, prec, mode, w, du, u, u1, dtp, s, stage, fo, st);
    case 2: return run_x1col<2>(g, th, recon, rs, flag, prec, mode, w, du, u, u1, dtp, s, stage, fo, st);
    case 3: return run_x1col<3>(g, th, recon, rs, flag, prec, mode, w, du, u, u1, dtp, s, stage, fo, st);
    case 6: return run_x1col<6>(g, th, recon, rs, flag, prec, mode, w, du, u, u1, dtp, s, stage, fo, st);
    default:
      set_error("unsupported number of mass-fraction slots");
      return CANOE_ERR_UNSUPPORTED;
  }
}

}  // namespace cb
