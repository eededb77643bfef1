// column_per_ny2.cu -- periodic-x1 implicit x1 pencil kernels for NY = 2
#include "column_per.cuh"

namespace cb {
#define CB_PER_INST(R)                                                                        \
  template int run_x1col_per<2, R>(const Geom &, const canoe_thermo_t &, int, int, int, int, \
                                    const double *, double *, double *, double *,             \
                                    const double *, const Stage &, int, double *, cudaStream_t);
CB_PER_INST(double)
CB_PER_INST(float)
#undef CB_PER_INST
}  // namespace cb
