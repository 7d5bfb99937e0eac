// lgpu_rng.h — counter-based path RNG.
//
// The reference draws from one std::mt19937 per pixel, consumed sample after
// sample (stoch.hpp:30-47, src/renderer.cpp:29).  The device instead derives
// an independent PCG32 stream for every (stream, sample) pair, so any path
// can be regenerated from its indices alone (path replay for the adjoint,
// any thread-to-path mapping for the kernels).  flt() returns the top 24
// bits scaled to [0, 1); uint64() joins two draws, high word first, as
// std::uniform_int_distribution<uint64_t> over a 32-bit engine does.
#pragma once

#include <stdint.h>

#if defined(__CUDACC__)
#define LGPU_RNG_FN __host__ __device__ __forceinline__
#else
#define LGPU_RNG_FN static inline
#endif

LGPU_RNG_FN uint64_t lgpu_mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Initial state of the path for sample `sample` of stream `stream` (a pixel
// index, optionally tagged with a job id in the high bits).
LGPU_RNG_FN uint64_t lgpu_path_state(uint64_t seed, uint64_t stream, uint64_t sample) {
  return lgpu_mix64(lgpu_mix64(seed + 0x9E3779B97F4A7C15ull) ^
                    lgpu_mix64(stream * 0x9E3779B97F4A7C15ull + sample + 1ull));
}

LGPU_RNG_FN uint32_t lgpu_pcg_next(uint64_t* s) {
  uint64_t const old = *s;
  *s = old * 6364136223846793005ull + 1442695040888963407ull;
  uint32_t const xs = (uint32_t)(((old >> 18) ^ old) >> 27);
  uint32_t const rot = (uint32_t)(old >> 59);
  return (xs >> rot) | (xs << ((32u - rot) & 31u));
}

LGPU_RNG_FN float lgpu_flt(uint64_t* s) {
  return (float)(lgpu_pcg_next(s) >> 8) * 0x1p-24f;
}

LGPU_RNG_FN uint64_t lgpu_u64(uint64_t* s) {
  uint64_t const hi = lgpu_pcg_next(s);
  uint64_t const lo = lgpu_pcg_next(s);
  return (hi << 32) | lo;
}
