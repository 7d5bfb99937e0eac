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

/* Single functions of the restatement, for pinning them one by one against
   the reference's own (K = the scene's hero_k wavelengths; random draws
   from std::mt19937 seeded with `seed`, as nl::RNG(seed) draws them).  The
   hit is hitinfo's fields (cg.hpp:1138-1149): z, p, F = (x, y, z), gn,
   front, mat, obj. */
typedef struct oracle_hit {
  float z;
  float p[3];
  float Fx[3], Fy[3], Fz[3];
  float gn[3];
  uint32_t front, mat, obj;
} oracle_hit;
/* coefficientλ::operator()(heroλ) of spectrum s (cg.hpp:298-303) */
void oracle_unit_spectrum(const lgpu_scene* sc, uint32_t s, const float* lam, float* out);
/* coefficientλ::addHeroλ into a zero spectrum (cg.hpp:306-320) */
void oracle_unit_add_hero(const lgpu_scene* sc, const float* lam, const float* v, float* out_bins);
/* BxDFcosθ (cg.hpp:1088-1102) */
void oracle_unit_bxdf(const lgpu_scene* sc, uint32_t mat, const float* lam, const float* i,
                      const float* o, const float* n, int front, float* out);
/* probForMateriali as src/renderer.cpp:136-137 calls it */
float oracle_unit_prob_for_material(const lgpu_scene* sc, float l0, const oracle_hit* h,
                                    const float* i, const float* o, float p);
/* sample::materiali (cg.hpp:1953-1968); returns whether a sample was made */
int oracle_unit_sample_material(const lgpu_scene* sc, const float* lam, const oracle_hit* h,
                                const float* o, uint64_t seed, float p, float* prob, float* dir,
                                float* mult);
/* sample::light (cg.hpp:1717-1732) for light `light`, shadow ray included */
void oracle_unit_sample_light(const lgpu_scene* sc, uint32_t light, const float* lam,
                              const oracle_hit* h, uint64_t seed, float* prob, float* dir,
                              float* mult);
/* sample::probForLight (cg.hpp:1735-1747) for the ray (p, d) */
float oracle_unit_prob_for_light(const lgpu_scene* sc, uint32_t light, const float* ray6);

#ifdef __cplusplus
}
#endif

#endif
