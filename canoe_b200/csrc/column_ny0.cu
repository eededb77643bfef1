// column_ny0.cu -- instantiation of the x1 pencil kernel for NY = 0
#include "column.cuh"

namespace cb {
template int run_x1col<0>(const Geom &, const canoe_thermo_t &, int, int, int, int, int,
                             const double *, double *, double *, double *,
                             const double *, const Stage &, int, double *, cudaStream_t);
}  // namespace cb
