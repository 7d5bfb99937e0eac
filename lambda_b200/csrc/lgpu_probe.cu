// lgpu_probe.cu — unit probe of the shading functions (lgpu_probe_shading).
//
// Every query runs one of the functions the render kernels use (materials,
// lights, spectra; lgpu_path.cuh) on explicit inputs, so each can be checked
// against the reference's function of the same name at the same arguments.
#include <stdint.h>

#include "lgpu_kernels.cuh"
#include "lgpu_path.cuh"

namespace lgpu {

namespace {

__device__ __forceinline__ f3 load3(const float* v) { return f3{v[0], v[1], v[2]}; }

__global__ void __launch_bounds__(128) probe_kernel(DevScene S, const lgpu_probe* __restrict__ q, uint64_t n,
                                                    lgpu_probe_result* __restrict__ out) {
  uint64_t const t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= n) return;
  lgpu_probe const Q = q[t];
  lgpu_probe_result r;
  for (int k = 0; k < 16; k++) r.value[k] = 0.f;
  r.prob = 0.f;
  r.dir[0] = r.dir[1] = r.dir[2] = 0.f;
  r.tmax = -1.f;
  r.skip = UINT32_MAX;
  r.ok = 0;
  uint32_t const K = S.hero_k < 16u ? S.hero_k : 16u;
  float x[16];
  for (uint32_t k = 0; k < K; k++) x[k] = lam_coord(S, Q.lambda[k]);
  HitInfo H;
  H.z = 0.f;
  H.p = load3(Q.p);
  H.F.x = load3(Q.F);
  H.F.y = load3(Q.F + 3);
  H.F.z = load3(Q.F + 6);
  H.gn = H.F.z;
  H.front = Q.front != 0;
  H.mat = Q.index;
  H.obj = UINT32_MAX;
  H.face = UINT32_MAX;
  f3 const i = load3(Q.i), o = load3(Q.o);
  XiDraws xr{Q.xi, 4u, 0u};
  switch (Q.op) {
    case LGPU_PROBE_BXDF: {
      DevMaterial const m = S.mats[Q.index];
      BsdfScalars const s = bsdf_scalars(S, m, x[0], i, o, load3(Q.n), H.front);
      for (uint32_t k = 0; k < K; k++) r.value[k] = bsdf_k(S, m, s, x[k], Q.lambda[k], H.front);
      break;
    }
    case LGPU_PROBE_PROB_MATERIAL: {
      DevMaterial const m = S.mats[Q.index];
      r.prob = prob_for_material(S, m, x[0], H, i, o, Q.sample_p);
      break;
    }
    case LGPU_PROBE_SAMPLE_MATERIAL: {
      DevMaterial const m = S.mats[Q.index];
      MatSample const ms = sample_material(S, m, x[0], H, o, Q.sample_p, xr);
      r.ok = ms.ok ? 1u : 0u;
      r.prob = ms.prob;
      r.dir[0] = ms.dir.x;
      r.dir[1] = ms.dir.y;
      r.dir[2] = ms.dir.z;
      if (ms.ok)
        for (uint32_t k = 0; k < K; k++) r.value[k] = mat_mult_k(S, m, ms, x[k], Q.lambda[k], H.front);
      break;
    }
    case LGPU_PROBE_SAMPLE_LIGHT: {
      lgpu_light const L = S.lights[Q.index];
      float tmax;
      uint32_t skip;
      LightSample const ls = sample_light_unoccluded(S, L, H, xr, tmax, skip);
      r.prob = ls.prob;
      r.dir[0] = ls.dir.x;
      r.dir[1] = ls.dir.y;
      r.dir[2] = ls.dir.z;
      r.tmax = tmax;
      r.skip = skip;
      for (uint32_t k = 0; k < K; k++) r.value[k] = spec_at(S, L.spectrum, x[k]) * ls.scale;
      break;
    }
    case LGPU_PROBE_PROB_LIGHT:
      r.prob = prob_for_light(S, S.lights[Q.index], H.p, i);
      break;
    case LGPU_PROBE_SPECTRUM:
      for (uint32_t k = 0; k < K; k++) r.value[k] = spec_at(S, int32_t(Q.index), x[k]);
      break;
  }
  r.n_xi = xr.used;
  out[t] = r;
}

}  // namespace

cudaError_t launch_probe(const DevScene& S, const lgpu_probe* d_q, uint64_t n, lgpu_probe_result* d_out,
                         cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  uint64_t const blocks = (n + 127) / 128;
  probe_kernel<<<dim3(uint32_t(blocks)), 128, 0, st>>>(S, d_q, n, d_out);
  return cudaGetLastError();
}

}  // namespace lgpu
