// exchange.cu -- ghost zones of a MeshBlock filled from its neighbours'
// interiors on the same GPU: Athena's SEND_HYD -> RECV_HYD -> SETB_HYD
// boundary tasks (patches/24.time_integrator.patch:17-19) as one device
// copy of the primitive state's ghost slabs.
//
// A slab is NV x nk x nj rows of nc1 doubles, each row contiguous in both
// blocks (i fastest); one warp copies one row with consecutive lanes on
// consecutive doubles, so both sides are coalesced.  Algorithmic bytes: one
// read and one write of NV doubles per ghost cell (16 NV B).
#include <cuda_runtime.h>

#include "block.cuh"

namespace cb {

namespace {

constexpr int kExWarps = 8;

__global__ void __launch_bounds__(kExWarps * 32)
    k_exchange(SlabSet ss) {
  const Slab &sl = ss.s[blockIdx.y];
  const int64_t rows = (int64_t)ss.nv * sl.nk * sl.nj;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int64_t r = (int64_t)blockIdx.x * kExWarps + warp; r < rows;
       r += (int64_t)gridDim.x * kExWarps) {
    const int n = (int)(r / ((int64_t)sl.nk * sl.nj));
    const int rem = (int)(r % ((int64_t)sl.nk * sl.nj));
    const int kk = rem / sl.nj, jj = rem % sl.nj;
    double *d = sl.dst + n * sl.dsv + kk * sl.dsk + (int64_t)jj * ss.nc1;
    const double *s = sl.src + n * sl.ssv + kk * sl.ssk + (int64_t)jj * ss.nc1;
    for (int i = lane; i < ss.nc1; i += 32) d[i] = s[i];
  }
}

}  // namespace

int launch_exchange(const SlabSet &ss, cudaStream_t st) {
  if (ss.n <= 0) return 0;
  int64_t most = 0;
  for (int q = 0; q < ss.n; ++q) {
    const int64_t rows = (int64_t)ss.nv * ss.s[q].nk * ss.s[q].nj;
    most = rows > most ? rows : most;
  }
  const unsigned gx = (unsigned)((most + kExWarps - 1) / kExWarps);
  k_exchange<<<dim3(gx < 4096u ? gx : 4096u, (unsigned)ss.n), kExWarps * 32, 0, st>>>(ss);
  CB_CUDA(cudaGetLastError());
  return 0;
}

}  // namespace cb
