/*
 * lambda_oracle.h — TEST INFRASTRUCTURE ONLY.
 *
 * A CPU restatement in C of the reference's spectral path-tracing hot path
 * (src/renderer.cpp:14-146, lib/numli/cg.hpp), reading the same lgpu_scene
 * the device library takes.  Used by the tests as the checker and by the
 * benchmark's CPU-baseline leg; never by the product.
 *
 * Two random streams:
 *   ORACLE_RNG_MT19937  the reference's: std::mt19937 seeded with the pixel
 *                       index, consumed sample after sample (stoch.hpp:30-47,
 *                       src/renderer.cpp:29), flt() = float(u32)/2^32 as
 *                       generate_canonical<float,24> computes it, uint64()
 *                       = two draws, high word first.
 *   ORACLE_RNG_PCG      the device's counter-based stream (lgpu_rng.h).
 */
#ifndef LAMBDA_ORACLE_H
#define LAMBDA_ORACLE_H

#include <stdint.h>

#include "lambda_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

#define ORACLE_RNG_MT19937 0
#define ORACLE_RNG_PCG 1

/* intersect::scene (cg.hpp:1469-1489) in the reference's object order, with
   the winning trimesh face reported. */
void oracle_intersect(const lgpu_scene* sc, const float* rays, uint64_t n, lgpu_hit* out);

/* Pixel rows [row0, row1) of Renderer::render (src/renderer.cpp:27-56), not
   flipped: out holds (row1-row0)*width*3 floats, band row k = scene row
   row0+k.  Film in float 80-bin spectra like the reference unless fp64. */
void oracle_render_rows(const lgpu_scene* sc, uint32_t spp, uint32_t max_scatter, float sample_p,
                        int rng_mode, uint64_t seed, uint32_t spp_offset, uint64_t row0,
                        uint64_t row1, int fp64, float* out32, double* out64);

/* Random streams, for pinning: n floats / uint64s from a fresh stream. */
void oracle_mt_flt(uint64_t seed, uint64_t n, float* out);
void oracle_mt_u64(uint64_t seed, uint64_t n, uint64_t* out);

/* The reference evaluates f(rng.flt(), rng.flt()) with unspecified argument
   order; g++ evaluates right to left.  1 (default) draws the second
   argument first in the mt19937 mode. */
void oracle_set_mt_arg_order(int right_to_left);

int oracle_max_threads(void);

#ifdef __cplusplus
}
#endif

#endif
