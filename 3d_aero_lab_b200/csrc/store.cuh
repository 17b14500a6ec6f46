// store.cuh - the stage kernels' output store: the cell's own buffer and, on a z slab whose
// neighbour keeps this plane as a halo plane, the neighbour's buffer of the same role.  The
// neighbour may live in this GPU's memory or a peer GPU's (peer stores over NVLink); the
// caller orders the next stage after both slabs' stores.
#pragma once
#include "solver.cuh"

namespace a3d {

__device__ __forceinline__ void store_out(const StageArgs& a, float* __restrict__ Out, long qp, int k,
                                          const float o[5]) {
#pragma unroll
  for (int c = 0; c < 5; c++) Out[c * a.Np + qp] = o[c];
#pragma unroll
  for (int sd = 0; sd < 2; sd++) {
    if (a.peer[sd] && k >= a.peer_k0[sd] && k < a.peer_k1[sd]) {
      float* P = a.peer[sd] + qp + (long)a.peer_dk[sd] * a.NY * a.NXp;
#pragma unroll
      for (int c = 0; c < 5; c++) P[c * a.peer_np[sd]] = o[c];
    }
  }
}

}  // namespace a3d
