// lgpu_kernels.cu — closest-hit, render and tone-map kernels.
#include <float.h>
#include <stdint.h>

#include "lgpu_kernels.cuh"
#include "lgpu_path.cuh"

namespace lgpu {

namespace {

__device__ __forceinline__ void flush_counters(DevCounters* cnt, uint32_t rays, uint32_t paths,
                                               uint32_t flags, uint32_t nonfinite) {
  unsigned const full = 0xFFFFFFFFu;
  unsigned long long r = rays, p = paths;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    r += __shfl_down_sync(full, r, o);
    p += __shfl_down_sync(full, p, o);
    flags |= __shfl_down_sync(full, flags, o);
    nonfinite += __shfl_down_sync(full, nonfinite, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (r) atomicAdd(&cnt->rays, r);
    if (p) atomicAdd(&cnt->paths, p);
    if (flags) atomicOr(&cnt->flags, flags);
    if (nonfinite) atomicAdd(&cnt->nonfinite, nonfinite);
  }
}

// intersect::scene on a ray set (cg.hpp:1469-1489)
__global__ void __launch_bounds__(128) trace_kernel(DevScene S, const float* __restrict__ rays, uint64_t n,
                                                    uint32_t flags, lgpu_hit* __restrict__ out,
                                                    DevCounters* cnt) {
  uint64_t const i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  uint32_t fl = 0;
  if (i < n) {
    const float* q = rays + 6 * i;
    Ray const r = make_ray(mk(q[0], q[1], q[2]), mk(q[3], q[4], q[5]));
    HitRec h;
    h.z = kFltMax;
    h.obj = UINT32_MAX;
    h.face = UINT32_MAX;
    StackEntry stack[kStackCap];
    StackEntry tstack[kTlasStackCap];
    bool const ref_order = (flags & LGPU_FLAG_REFERENCE_ORDER) != 0;
    lgpu_hit o;
    if (scene_hit<false>(S, r, h, UINT32_MAX, ref_order, stack, tstack, fl)) {
      HitInfo const H = finalize_hit(S, r, h);
      o.t = H.z;
      o.obj = H.obj;
      o.face = H.face;
      o.mat = H.mat;
      o.p[0] = H.p.x; o.p[1] = H.p.y; o.p[2] = H.p.z;
      o.n[0] = H.F.z.x; o.n[1] = H.F.z.y; o.n[2] = H.F.z.z;
      o.gn[0] = H.gn.x; o.gn[1] = H.gn.y; o.gn[2] = H.gn.z;
      o.front = H.front ? 1u : 0u;
    } else {
      o.t = h.z;
      o.obj = UINT32_MAX;
      o.face = UINT32_MAX;
      o.mat = UINT32_MAX;
      for (int k = 0; k < 3; k++) o.p[k] = o.n[k] = o.gn[k] = 0.f;
      o.front = 0;
    }
    out[i] = o;
  }
  flush_counters(cnt, i < n ? 1u : 0u, 0u, fl, 0u);
}

// Renderer::render (src/renderer.cpp:14-61) for a range of pixels: one
// thread per pixel, all of its samples, film accumulated as XYZ.
template <int K>
__global__ void __launch_bounds__(128) render_kernel(DevScene S, RenderArgs a, float* __restrict__ out,
                                                     DevCounters* cnt) {
  uint32_t const t = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t rays = 0, flags = 0, nonfinite = 0, paths = 0;
  if (t < a.pixel_count) {
    uint32_t const pix = a.pixel_begin + t;
    uint32_t const W = uint32_t(S.cam.width), H = uint32_t(S.cam.height);
    uint32_t const i = pix / W, j = pix - i * W;
    float const omega = S.lambda_sup - S.lambda_inf;
    float const step = omega / float(K);
    float const prob_l = 1.f / omega;
    bool const ref_order = (a.flags & LGPU_FLAG_REFERENCE_ORDER) != 0;
    const lgpu_camera& C = S.cam;
    f3 const Fx = f3{C.base_x[0], C.base_x[1], C.base_x[2]};
    f3 const Fy = f3{C.base_y[0], C.base_y[1], C.base_y[2]};
    f3 const Fz = f3{C.base_z[0], C.base_z[1], C.base_z[2]};
    f3 const P = f3{C.pos[0], C.pos[1], C.pos[2]};
    Stacks st;
    float X = 0.f, Y = 0.f, Z = 0.f;
    uint64_t const stream = (uint64_t(a.stream_tag) << 32) | pix;
    for (uint32_t s = 0; s < a.spp; s++) {
      uint64_t rng = lgpu_path_state(a.seed, stream, uint64_t(a.spp_offset) + s);
      float const u = float(j) + lgpu_flt(&rng);
      float const v = float(i) + lgpu_flt(&rng);
      // sample::camera (cg.hpp:1534-1542)
      float const cu = -0.5f * C.w + C.delta * u;
      float const cv = -0.5f * C.h + C.delta * v;
      f3 const wij = f3{P.x + Fx.x * cu + Fy.x * cv - C.D * Fz.x, P.y + Fx.y * cu + Fy.y * cv - C.D * Fz.y,
                        P.z + Fx.z * cu + Fy.z * cv - C.D * Fz.z};
      float const la = lgpu_flt(&rng) - 0.5f;
      float const lb = lgpu_flt(&rng) - 0.5f;
      float const dd = 2.f * C.dof;
      f3 const wkl = f3{P.x + dd * (Fx.x * la + Fy.x * lb), P.y + dd * (Fx.y * la + Fy.y * lb),
                        P.z + dd * (Fx.z * la + Fy.z * lb)};
      f3 const dir = fnorm(f3{wij.x - wkl.x, wij.y - wkl.y, wij.z - wkl.z});
      // sample::spectrum (cg.hpp:1517-1531)
      float const hero = S.lambda_inf + omega * lgpu_flt(&rng);
      float acc[K];
      PathCounters pc{0u, 0u};
      trace_path<K>(S, make_ray(wkl, dir), hero, step, a.max_scatter, a.sample_p, ref_order, rng, acc, st,
                    pc);
      rays += pc.rays;
      flags |= pc.flags;
      paths++;
      // addHeroλ(λ, Li/prob) (src/renderer.cpp:44)
      float sx = 0.f, sy = 0.f, sz = 0.f;
      bool finite = true;
#pragma unroll
      for (int k = 0; k < K; k++) {
        float const val = acc[k] / prob_l;
        finite = finite && isfinite(val);
        splat_xyz(S, hero_lambda(S, hero, step, k), val, sx, sy, sz);
      }
      nonfinite += finite ? 0u : 1u;
      X += sx;
      Y += sy;
      Z += sz;
    }
    // irradiance / (SPP*K), dotted with the CMFs times Δ, then XYZ2linRGB
    // (src/renderer.cpp:52-56, cg.hpp:144-148, 340-341)
    float const norm = float(a.spp * K);
    X = (X / norm) * S.lambda_delta;
    Y = (Y / norm) * S.lambda_delta;
    Z = (Z / norm) * S.lambda_delta;
    size_t const o = (size_t(H - i - 1) * W + j) * 3;
    out[o + 0] = 3.2404542f * X - 1.5371385f * Y - 0.4985314f * Z;
    out[o + 1] = -0.9692660f * X + 1.8760108f * Y + 0.0415560f * Z;
    out[o + 2] = 0.0556434f * X - 0.2040259f * Y + 1.0572252f * Z;
  }
  flush_counters(cnt, rays, paths, flags, nonfinite);
}

// ---- tone map (src/renderer.cpp:149-176) -------------------------------------

constexpr int kTmThreads = 256;
constexpr uint32_t kTmMaxBlocks = 148 * 8;

// log-average luminance: per-block sums of log(max(Y, ε)) in double
__global__ void __launch_bounds__(kTmThreads) tm_logsum_kernel(const float* __restrict__ rgb, uint64_t n,
                                                               double* __restrict__ partials) {
  double s = 0.0;
  for (uint64_t p = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < n;
       p += uint64_t(gridDim.x) * blockDim.x) {
    float const Yl = 0.2126f * rgb[3 * p] + 0.7152f * rgb[3 * p + 1] + 0.0722f * rgb[3 * p + 2];
    float const y = Yl >= kEps ? Yl : kEps;
    s += double(logf(y));
  }
  __shared__ double red[kTmThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xFFFFFFFFu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kTmThreads / 32; w++) t += red[w];
    partials[blockIdx.x] = t;
  }
}

__global__ void tm_exposure_kernel(const double* __restrict__ partials, uint32_t nb, uint64_t n, float y_mid,
                                   float* __restrict__ exposure) {
  __shared__ double red[32];
  double s = 0.0;
  for (uint32_t b = threadIdx.x; b < nb; b += blockDim.x) s += partials[b];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xFFFFFFFFu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (uint32_t w = 0; w < (blockDim.x + 31) / 32; w++) t += red[w];
    float const ybar = expf(float(t / double(n)));
    exposure[0] = y_mid / ybar;
  }
}

// tonemapping::koiFilmic (cg.hpp:181-194)
__device__ __forceinline__ float koi_filmic(float L) {
  float const x = 10.f * L;
  return (x * (0.3f * x + 0.14f)) / (x * (0.3f * x + 2.8f) + 10.f);
}
// linRGB2sRGB (cg.hpp:149-154) and float2byte (numli.hpp:105-106)
__device__ __forceinline__ uint8_t srgb_byte(float c) {
  float const s = c > 0.0031308f ? 1.055f * powf(c, 1.f / 2.4f) - 0.055f : 12.92f * c;
  int v = int(255.f * s + 0.5f);
  v = v < 0 ? 0 : (v > 255 ? 255 : v);
  return uint8_t(v);
}

__global__ void __launch_bounds__(kTmThreads) tm_map_kernel(const float* __restrict__ rgb, uint64_t n,
                                                            const float* __restrict__ exposure,
                                                            float* __restrict__ out_tm,
                                                            uint8_t* __restrict__ out24) {
  float const e = exposure[0];
  for (uint64_t q = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < 3 * n;
       q += uint64_t(gridDim.x) * blockDim.x) {
    float const L = koi_filmic(e * rgb[q]);
    if (out_tm) out_tm[q] = L;
    if (out24) out24[q] = srgb_byte(L);
  }
}

}  // namespace

cudaError_t launch_trace(const DevScene& S, const float* d_rays, uint64_t n, uint32_t flags,
                         lgpu_hit* d_hits, DevCounters* d_cnt, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  uint64_t const blocks = (n + 127) / 128;
  trace_kernel<<<dim3(uint32_t(blocks)), 128, 0, st>>>(S, d_rays, n, flags, d_hits, d_cnt);
  return cudaGetLastError();
}

cudaError_t launch_render(const DevScene& S, const RenderArgs& a, float* d_out, DevCounters* d_cnt,
                          cudaStream_t st) {
  if (a.pixel_count == 0) return cudaSuccess;
  uint32_t const blocks = (a.pixel_count + 127) / 128;
  switch (S.hero_k) {
    case 4: render_kernel<4><<<blocks, 128, 0, st>>>(S, a, d_out, d_cnt); break;
    case 8: render_kernel<8><<<blocks, 128, 0, st>>>(S, a, d_out, d_cnt); break;
    case 16: render_kernel<16><<<blocks, 128, 0, st>>>(S, a, d_out, d_cnt); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

uint32_t tonemap_partials_needed(uint64_t n_pixels) {
  uint64_t const b = (n_pixels + kTmThreads - 1) / kTmThreads;
  return uint32_t(b < kTmMaxBlocks ? (b ? b : 1) : kTmMaxBlocks);
}

cudaError_t launch_tonemap(const float* d_rgb, uint64_t n_pixels, float y_mid, double* d_partials,
                           uint32_t n_partials, float* d_exposure, float* d_out_tm, uint8_t* d_out24,
                           cudaStream_t st) {
  uint32_t const nb = tonemap_partials_needed(n_pixels);
  if (n_partials < nb) return cudaErrorInvalidValue;
  tm_logsum_kernel<<<nb, kTmThreads, 0, st>>>(d_rgb, n_pixels, d_partials);
  tm_exposure_kernel<<<1, 1024, 0, st>>>(d_partials, nb, n_pixels, y_mid, d_exposure);
  uint64_t const mb = (3 * n_pixels + kTmThreads - 1) / kTmThreads;
  uint32_t const map_blocks = uint32_t(mb < kTmMaxBlocks ? (mb ? mb : 1) : kTmMaxBlocks);
  tm_map_kernel<<<map_blocks, kTmThreads, 0, st>>>(d_rgb, n_pixels, d_exposure, d_out_tm, d_out24);
  return cudaGetLastError();
}

}  // namespace lgpu
