// lgpu_counters.cuh — per-warp reduction of the kernels' work counters.
#pragma once

#include "lgpu_intersect.cuh"
#include "lgpu_kernels.cuh"

namespace lgpu {

__device__ __forceinline__ void flush_counters(DevCounters* cnt, uint32_t rays, uint32_t paths,
                                               const TravStats& ts, uint32_t nonfinite) {
  unsigned const full = 0xFFFFFFFFu;
  unsigned long long r = rays, p = paths, nd = ts.nodes, tr = ts.tris, in = ts.insts;
  uint32_t flags = ts.flags;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    r += __shfl_down_sync(full, r, o);
    p += __shfl_down_sync(full, p, o);
    nd += __shfl_down_sync(full, nd, o);
    tr += __shfl_down_sync(full, tr, o);
    in += __shfl_down_sync(full, in, o);
    flags |= __shfl_down_sync(full, flags, o);
    nonfinite += __shfl_down_sync(full, nonfinite, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (r) atomicAdd(&cnt->rays, r);
    if (p) atomicAdd(&cnt->paths, p);
    if (nd) atomicAdd(&cnt->nodes, nd);
    if (tr) atomicAdd(&cnt->tris, tr);
    if (in) atomicAdd(&cnt->insts, in);
    if (flags) atomicOr(&cnt->flags, flags);
    if (nonfinite) atomicAdd(&cnt->nonfinite, nonfinite);
  }
}

}  // namespace lgpu
