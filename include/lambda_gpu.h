/*
 * lambda_gpu.h — C ABI of the B200 (sm_100a) spectral path-tracing library.
 *
 * This is the drop-in boundary for lambda's render call.  The reference
 * renders with the C++ member call
 *
 *     void Renderer::render(nl::cg::scene const&, rendering&);
 *         declared  include/renderer.hpp:39, defined src/renderer.cpp:14,
 *         called    src/main.cpp:41
 *
 * and has no plugin or FFI layer.  A host that keeps the reference's .nls
 * loader, scene structures and CLI flattens its nl::cg::scene into the plain
 * structs below (pointers into the host's own vectors; nothing is copied on
 * the host), calls lgpu_upload_scene + lgpu_render, and receives the linear
 * BT.709 image in the reference's layout (row 0 at the top, W*H*3 floats,
 * normalised by 1/(SPP*HERO_SAMPLES), src/renderer.cpp:52-56).
 *
 * Conventions for every entry point:
 *   - returns LGPU_OK (0) or a negative lgpu_status; the message of the last
 *     failure is available from lgpu_last_error(ctx);
 *   - no C++ exception crosses the boundary;
 *   - calls are synchronous unless the name ends in _async;
 *   - one context per host thread; device memory is owned by the context;
 *   - no torch types: plain pointers and sizes only.
 */
#ifndef LAMBDA_GPU_H
#define LAMBDA_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* 2: lgpu_stats gained order_rays; lgpu_probe_shading and
   lgpu_build_bvh_device were added.
   3: lgpu_stats gained local_stack; lgpu_trace_any,
   LGPU_FLAG_FP64_FILM and lgpu_scene.flags (LGPU_SCENE_HOST_LAYOUT) were
   added; lgpu_trace_closest runs the render's traversal kernels; uploads
   lay the meshes out on the device
   4: a surface-area-heuristic traversal tree per mesh for the instance-BVH
   traversal: lgpu_mesh gained its optional arrays (trav_*),
   lgpu_build_traversal_bvh builds it, lgpu_upload_scene builds the missing
   ones; LGPU_SCENE_REFERENCE_BVH keeps the reference's trees */
#define LGPU_ABI_VERSION 4

typedef struct lgpu_ctx lgpu_ctx;

typedef enum lgpu_status {
  LGPU_OK = 0,
  LGPU_ERR_INVALID_ARGUMENT = -1,
  LGPU_ERR_CUDA = -2,
  LGPU_ERR_OUT_OF_MEMORY = -3,
  LGPU_ERR_NO_SCENE = -4,
  LGPU_ERR_UNSUPPORTED = -5,
  /* a device-side check fired (traversal stack overflow, index out of
     range); the kernel skipped the offending access and reported it */
  LGPU_ERR_DEVICE_CHECK = -6,
  /* a bounded device-side wait ran out before its condition held */
  LGPU_ERR_TIMEOUT = -7,
  LGPU_ERR_NO_DEVICE = -8,
  /* a size is beyond an entry point's stated maximum */
  LGPU_ERR_TOO_LARGE = -9
} lgpu_status;

/* ---- scene description ------------------------------------------------ */

/* Variant order of nl::cg::Object (cg.hpp:857). */
typedef enum lgpu_object_type {
  LGPU_OBJ_SPHERE = 0,
  LGPU_OBJ_PLANE = 1,
  LGPU_OBJ_TRIMESH = 2
} lgpu_object_type;

/* Variant order of nl::cg::Material (cg.hpp:1084-1085). */
typedef enum lgpu_material_type {
  LGPU_MAT_LAMBERTIAN = 0,
  LGPU_MAT_BLINN = 1,
  LGPU_MAT_THINFILM = 2,
  LGPU_MAT_MICROFACET = 3, /* loaded by the reference but never shaded */
  LGPU_MAT_EMITTER = 4,
  LGPU_MAT_DIREMITTER = 5
} lgpu_material_type;

/* Variant order of nl::cg::Light (cg.hpp:904-905). */
typedef enum lgpu_light_type {
  LGPU_LIGHT_AMBIENT = 0,
  LGPU_LIGHT_POINT = 1,
  LGPU_LIGHT_DIR = 2,
  LGPU_LIGHT_SPHERE = 3,
  LGPU_LIGHT_QUADDIR = 4
} lgpu_light_type;

/* nl::cg::transform (cg.hpp:422-425): row-major 4x4 M and its inverse. */
typedef struct lgpu_transform {
  float M[16];
  float M_inv[16];
} lgpu_transform;

/* nl::cg::camera (cg.hpp:1151-1165) after camera::init. */
typedef struct lgpu_camera {
  float base_x[3], base_y[3], base_z[3]; /* camera::base */
  float pos[3];
  float fov, dof, D, delta, h, w; /* delta = camera::Δ */
  uint64_t width, height;
} lgpu_camera;

/* Spectral discretisation.  The reference compiles it in: Nλ = 80 bins on
   [400, 720] nm and HERO_SAMPLES = 16 (cg.hpp:40-41, 244-245).  The CMF
   tables are the host's coefficientλ<Nλ> CMF_X/Y/Z (cg.hpp:329-331). */
typedef struct lgpu_spectral {
  uint32_t n_bins;
  uint32_t hero_k; /* 4, 8 or 16 */
  float lambda_inf, lambda_sup;
  const float* cmf_x; /* n_bins each */
  const float* cmf_y;
  const float* cmf_z;
} lgpu_spectral;

/* One entry of nl::cg::list<Material>.  Spectra are indices into
   lgpu_scene::spectra (-1 when unused):
     lambertian : s[0] = albedo                         (cg.hpp:921-926)
     blinn      : s[0..4] = Kd, Ks, Kt, Le, ior          (cg.hpp:927-993)
     thinfilm   : s[0] = film_ior, s[1] = base_ior       (cg.hpp:995-1052)
     emitter    : s[0] = radiance                        (cg.hpp:1069-1074)
     diremitter : s[0] = radiance, specular              (cg.hpp:1075-1081)
   Blinn's p_d, p_spec, w_r, w_t are the values blinn::init computed. */
typedef struct lgpu_material {
  int32_t type;
  int32_t spectrum[5];
  float alpha;
  float p_d, p_spec, w_r, w_t;
  float d;
  float specular;
} lgpu_material;

/* One entry of nl::cg::list<Object> (cg.hpp:835-857); the object index is
   its position in the array (the reference's objectidx). */
typedef struct lgpu_object {
  int32_t type;
  uint32_t mat;
  uint32_t mesh; /* trimesh only */
  uint32_t reserved;
  lgpu_transform T;
} lgpu_object;

/* One entry of nl::cg::list<Light> (cg.hpp:875-905). */
typedef struct lgpu_light {
  int32_t type;
  int32_t spectrum; /* radiance or radiant_intensity */
  uint32_t obj;     /* sphere / quaddir: the light's own object index */
  float size;       /* spherelight::size */
  float inv_area;   /* quaddirlight::inv_area */
  float spec;       /* quaddirlight::spec */
  float pos[3];     /* pointlight::pos */
  float dir[3];     /* dirlight::dir */
  lgpu_transform T; /* _sphere.T / _plane.T */
} lgpu_light;

/* nl::cg::trimeshdata (cg.hpp:766-820) with its wide BVH in the reference's
   own layout (cg.hpp:596-631): nodes are {childrenbb_idx, data} pairs with
   data = idx<<4 | (count-1)<<1 | leaf; bbs are aabb_avx2 records of 48
   floats (inf[3][8] then sup[3][8]); prim_idxs index faces.  Position and
   normal arrays include fast_obj's dummy element at index 0.
   A host without the reference's trees passes nodes, bbs and prim_idxs as
   NULL (counts 0): lgpu_upload_scene then builds the tree as bvh::build
   does, on the device (lgpu_build_bvh_device; vertex positions must be
   finite). */
typedef struct lgpu_mesh {
  uint32_t n_positions, n_normals, n_faces;
  uint32_t f_stride; /* uint32 words per face in F (9 for nl::cg::triangle) */
  const float* V;    /* n_positions * 3 */
  const float* N;    /* n_normals * 3 */
  const uint32_t* F; /* face f: V idx at F[f*f_stride+0..2], N idx at +3..5 */
  const float* GN;   /* n_faces * 3 geometric normals */
  float bounds[6];   /* trimeshdata::bounds: inf xyz, sup xyz */
  uint32_t n_nodes, n_bbs, n_prim_idxs, reserved;
  const uint32_t* nodes;
  const float* bbs;
  const uint32_t* prim_idxs;
  /* Optional: the mesh's traversal tree, in the same layout, as
     lgpu_build_traversal_bvh builds it over this mesh's faces (a loader
     builds it with the reference's tree, at scene load).  NULL (counts 0):
     lgpu_upload_scene builds it, unless LGPU_SCENE_REFERENCE_BVH. */
  uint32_t n_trav_nodes, n_trav_bbs, n_trav_prim_idxs, reserved2;
  const uint32_t* trav_nodes;
  const float* trav_bbs;
  const uint32_t* trav_prim_idxs;
} lgpu_mesh;

/* lgpu_scene.flags: lay the meshes out on the host (the relayout pass of
   lgpu_upload_scene run on the CPU) instead of on the device.  The device
   reads the meshes' own arrays (V, N, GN, F and the BVH) and builds their
   nodes, leaf triangles and shading records itself; both give identical
   device data. */
#define LGPU_SCENE_HOST_LAYOUT 0x1u
/* lgpu_scene.flags: keep the reference's mesh BVHs for every traversal.  By
   default lgpu_upload_scene also builds, for each mesh, an 8-wide BVH with
   the surface-area heuristic on the host, which the instance-BVH traversal
   (the renders' default) enters instead: the same closest hits in fewer node
   and triangle tests (at exactly equal distances another face can be
   reported).  The reference-order traversal (LGPU_FLAG_REFERENCE_ORDER)
   always uses the reference's trees.  With this flag the meshes' trav_*
   arrays are ignored and none is built. */
#define LGPU_SCENE_REFERENCE_BVH 0x2u

typedef struct lgpu_scene {
  lgpu_camera cam;
  lgpu_spectral spec;
  uint32_t n_objects, n_materials, n_lights, n_meshes, n_spectra;
  uint32_t flags; /* LGPU_SCENE_* upload options (0: defaults) */
  const lgpu_object* objects;
  const lgpu_material* materials;
  const lgpu_light* lights;
  const lgpu_mesh* meshes;
  const float* spectra; /* n_spectra * spec.n_bins */
} lgpu_scene;

/* ---- rendering -------------------------------------------------------- */

/* Traverse objects in the reference's order (linear object loop, children
   sorted far-to-near, cg.hpp:1436-1437, 1477-1487) so that equal-t ties
   resolve exactly as the reference does.  Without it the device uses its
   instance-level BVH. */
#define LGPU_FLAG_REFERENCE_ORDER 0x1u

/* Render with one thread per pixel looping over its samples and bounces
   (the megakernel) instead of the default wavefront kernels.  Both draw
   the same random numbers per path. */
#define LGPU_FLAG_MEGAKERNEL 0x2u

/* Time the wavefront's closest-hit, shadow and shading launches separately
   (CUDA events around each launch) and count their traversal work apart;
   results in lgpu_stats.kernel_*.  For profiling; it adds event records. */
#define LGPU_FLAG_KERNEL_TIMING 0x4u

/* Accumulate the film in double precision, as the reference's FP64 oracle
   film does, and write the image as W*H*3 doubles (the output buffer holds
   doubles, twice the bytes).  Each sample's splat is still computed in
   float; the sums over samples and the colour conversion are double.  For
   oracle images and finite differences, where the float film's rounding
   would hide small differences.  lgpu_render and lgpu_render_device with
   the wavefront kernels only (LGPU_ERR_UNSUPPORTED with the megakernel, in
   batches and for the adjoint). */
#define LGPU_FLAG_FP64_FILM 0x8u

/* Renderer settings (include/renderer.hpp:35-37) plus the device RNG seed. */
typedef struct lgpu_render_params {
  uint32_t spp;             /* Renderer::SPP */
  uint32_t max_scatterings; /* Renderer::MAX_SCATTERINGS */
  float sample_p;           /* Renderer::SAMPLE_P */
  uint32_t flags;
  uint64_t seed;
  uint32_t spp_offset; /* index of the first sample (progressive renders) */
  uint32_t reserved;
} lgpu_render_params;

/* Result of one closest-hit query (nl::cg::hitinfo, cg.hpp:1138-1149). */
typedef struct lgpu_hit {
  float t;       /* hitinfo::z; FLT_MAX on a miss */
  uint32_t obj;  /* UINT32_MAX on a miss */
  uint32_t face; /* trimesh face; UINT32_MAX for spheres and planes */
  uint32_t mat;
  float p[3];  /* world-space hit point */
  float n[3];  /* shading frame z (hitinfo::F.z) */
  float gn[3]; /* geometric normal */
  uint32_t front;
} lgpu_hit;

typedef struct lgpu_stats {
  double last_kernel_ms;  /* device time of the last render/trace kernel */
  uint64_t rays;          /* extension + shadow rays of the last render */
  uint64_t paths;
  uint32_t device_checks;   /* device-side checks that fired */
  uint32_t max_stack;       /* traversal stack bound in use */
  uint32_t nonfinite_paths; /* paths whose radiance was NaN or infinite */
  uint32_t launches;        /* kernel launches of the last render or trace */
  uint64_t node_tests; /* 8-wide node box tests of the last kernel */
  uint64_t tri_tests;  /* triangle tests */
  uint64_t inst_tests; /* object (instance) tests */
  uint64_t upload_bytes; /* host-to-device bytes of the last scene upload */
  /* with LGPU_FLAG_KERNEL_TIMING: [0] closest-hit traversal, [1] shadow
     traversal, [2] shading — summed device time, launches, rays, node,
     triangle and instance tests of each kind */
  double kernel_ms[3];
  uint64_t kernel_launches[3];
  uint64_t kernel_rays[3];
  uint64_t kernel_node_tests[3];
  uint64_t kernel_tri_tests[3];
  uint64_t kernel_inst_tests[3];
  /* extension rays of the last render whose closest hit depends on the
     reference's object order (more than one mesh whose bounds contain the
     ray origin), re-traced with its linear object loop */
  uint64_t order_rays;
  /* 1 if a traversal stack of the last render or trace grew past the 16
     entries per ray kept in shared memory into local memory */
  uint32_t local_stack;
  uint32_t reserved;
} lgpu_stats;

/* Context.  `device` is a CUDA ordinal. */
int lgpu_create(int device, lgpu_ctx** out);
void lgpu_destroy(lgpu_ctx* ctx);
const char* lgpu_last_error(const lgpu_ctx* ctx);
int lgpu_abi_version(void);

/* Copies the scene to the device and lays it out for traversal (replaces
   the implicit scene access of Renderer::render, src/renderer.cpp:14). The
   host keeps ownership of every array it passed. */
int lgpu_upload_scene(lgpu_ctx* ctx, const lgpu_scene* scene);

/* Replaces the materials and the spectrum table of the uploaded scene (slot
   0) without laying out its geometry again; the counts must match the
   uploaded scene.  For parameter updates in inverse rendering (no
   counterpart in the reference). */
int lgpu_update_materials(lgpu_ctx* ctx, const lgpu_scene* scene);

/* Renderer::render (src/renderer.cpp:14-61): renders the uploaded scene into
   the host buffer out_linrgb (cam.width*cam.height*3 floats, row 0 at the
   top). */
int lgpu_render(lgpu_ctx* ctx, const lgpu_render_params* params, float* out_linrgb);

/* Same as lgpu_render with the output in device memory, on `stream`
   (a cudaStream_t, or NULL for the context's stream). */
int lgpu_render_device(lgpu_ctx* ctx, const lgpu_render_params* params,
                       float* d_out_linrgb, void* stream);

/* Scene table for batched renders: uploads n scenes, scene k into slot k,
   replacing whatever was uploaded before (lgpu_upload_scene(ctx, s) is
   lgpu_upload_scenes(ctx, &s, 1); lgpu_render and lgpu_trace_closest use
   slot 0).  All scenes must have the same spectral hero_k. */
int lgpu_upload_scenes(lgpu_ctx* ctx, const lgpu_scene* const* scenes, uint32_t n);

/* One job of a batched render: a slot of the scene table, the settings of
   Renderer::render for it, and its output (that scene's
   cam.width*cam.height*3 floats of linear RGB, row 0 at the top).  A job
   may cover a rectangle of the frame (x0, y0 from the top-left corner of the
   output, width x height pixels; width 0 = the whole frame): it then writes
   only those pixels of `out`, with the values a render of the whole frame
   gives them, so tile jobs of one frame can share one output. */
typedef struct lgpu_job {
  uint32_t scene;
  uint32_t reserved;
  lgpu_render_params params;
  float* out;
  uint32_t x0, y0, width, height;
} lgpu_job;

/* Renders n jobs in one streaming wavefront: paths of all jobs share the
   queues, so small jobs and the tails of large ones keep the GPU busy
   (the batched form of Renderer::render, src/renderer.cpp:14-61; the
   reference renders one scene per call).  Every job's image is identical to
   lgpu_render of its scene with the same params.  A single job takes the
   plain path.  lgpu_render_batch: outputs in host memory;
   lgpu_render_batch_device: outputs in device memory, on `stream` (NULL:
   the context's stream).  The kernel counters of lgpu_get_stats cover the
   whole batch.  LGPU_ERR_TOO_LARGE if the jobs hold 2^31 pixels or more. */
int lgpu_render_batch(lgpu_ctx* ctx, const lgpu_job* jobs, uint32_t n);
int lgpu_render_batch_device(lgpu_ctx* ctx, const lgpu_job* jobs, uint32_t n, void* stream);

/* Gradients of an image loss with respect to material parameters by path
   replay (no counterpart in the reference, which renders only; this is the
   adjoint of Renderer::tracePath, src/renderer.cpp:64-146).  Given
   dloss_dimage = dLoss/d(linear RGB) (cam.width*cam.height*3 floats, the
   lgpu_render layout), renders slot 0 with `params` and writes
     grad_spectra   n_spectra*n_bins floats: dLoss/d(bin) of every
                    spectrum of the uploaded table (lgpu_scene.spectra) used
                    as a Lambertian albedo or a thin-film IOR (0 elsewhere);
     grad_materials n_materials*4 floats per material: [0] dLoss/d thin-film
                    thickness (nm), [1] dLoss/d lobe exponent α (Blinn and
                    thin film), [2..3] 0;
     out_linrgb     the primal image of the same paths (may be NULL).
   Sampling decisions and MIS weights are held fixed (detached), so the
   estimate is unbiased for the gradient of the expected loss.  Paths are
   recomputed from their random streams; nothing per vertex is stored.
   max_scatterings <= 62.  lgpu_adjoint: host buffers; lgpu_adjoint_device:
   device buffers, on `stream` (NULL: the context's stream). */
int lgpu_adjoint(lgpu_ctx* ctx, const lgpu_render_params* params, const float* dloss_dimage,
                 float* grad_spectra, float* grad_materials, float* out_linrgb);
int lgpu_adjoint_device(lgpu_ctx* ctx, const lgpu_render_params* params, const float* d_dloss_dimage,
                        float* d_grad_spectra, float* d_grad_materials, float* d_out_linrgb,
                        void* stream);

/* Launch shape of the wavefront renderer (no counterpart in the reference,
   which renders on CPU threads).  Defaults: queue_cap 2^24, shade_block
   256, trace_per_sm 0, graphs 1, mega_items 0. */
typedef struct lgpu_wave_config {
  uint32_t queue_cap;    /* paths in flight */
  uint32_t shade_block;  /* threads per block of the shading kernel: a multiple of 32 up to 256 */
  uint32_t trace_per_sm; /* resident blocks per SM of the persistent trace kernels (0: occupancy limit) */
  uint32_t graphs;       /* 1: the bounce stages are captured once per chunk as a CUDA graph and replayed */
  uint64_t mega_items;   /* batched renders: jobs with fewer work items (pixels x spp) are rendered by
                            the one-thread-per-pixel kernel on a second stream, beside the wavefront */
} lgpu_wave_config;
int lgpu_get_wave_config(const lgpu_ctx* ctx, lgpu_wave_config* out);
int lgpu_set_wave_config(lgpu_ctx* ctx, const lgpu_wave_config* cfg);

/* Autotuner: renders the jobs with spp divided by spp_divisor (at least 1)
   under candidate launch shapes (queue depth, shading block size, trace
   occupancy, graphs on/off, megakernel split), one dimension at a time,
   keeps the fastest (device time) and makes it the context's configuration;
   writes it to *out when out is not NULL.  Outputs of the jobs are not
   written. */
int lgpu_autotune_batch(lgpu_ctx* ctx, const lgpu_job* jobs, uint32_t n, uint32_t spp_divisor,
                        lgpu_wave_config* out);

/* intersect::scene (cg.hpp:1469-1489) on n rays given as 6 floats each
   (origin xyz, direction xyz) in host memory; writes n lgpu_hit.  The
   rays run through the render's own closest-hit kernels (the persistent
   instance-BVH traversal with its object-order fallback, or with
   LGPU_FLAG_REFERENCE_ORDER the linear object loop), so this is the parity
   probe of the traversal every render uses. */
int lgpu_trace_closest(lgpu_ctx* ctx, const float* rays, uint64_t n,
                       uint32_t flags, lgpu_hit* out);

/* Shadow-ray queries: intersect::scene(sc, ray, hinfo, skip) with hinfo.z
   preset to tmax[i] and an object skip[i] to ignore (UINT32_MAX: none), as
   sample::quaddirlight and sample::spherelight call it (cg.hpp:1652-1656,
   1697-1701).  out_hit[i] = 1 if the reference's call returns true (the
   light is occluded), else 0.  Runs the render's shadow-ray kernel (the
   persistent any-hit traversal, or with LGPU_FLAG_REFERENCE_ORDER the
   linear object loop).  Host buffers: rays 6*n floats, tmax n floats, skip n
   words, out_hit n bytes. */
int lgpu_trace_any(lgpu_ctx* ctx, const float* rays, const float* tmax,
                   const uint32_t* skip, uint64_t n, uint32_t flags,
                   uint8_t* out_hit);

/* Unit probe of the device's shading functions (the parity probe for
   materials and lights, as lgpu_trace_closest is for hits).  Each query
   evaluates one function of the uploaded scene (slot 0) with the render
   kernels' own device code:
     LGPU_PROBE_BXDF             BxDFcosθ(λ, materials[index], i, o, n, front)
                                 (cg.hpp:1088-1102) -> value[k]
     LGPU_PROBE_PROB_MATERIAL    probForMateriali(λ0, materials[index], hit, i, o, p)
                                 with the reference's call-site argument order
                                 (src/renderer.cpp:136-137, cg.hpp:1971-1985) -> prob
     LGPU_PROBE_SAMPLE_MATERIAL  sample::materiali(λ, materials[index], hit, o, p)
                                 (cg.hpp:1953-1968) with the uniform draws xi
                                 -> ok, dir, prob, value[k] = mult
     LGPU_PROBE_SAMPLE_LIGHT     sample::light(λ, lights[index], hit) (cg.hpp:
                                 1560-1732) without its shadow ray -> dir,
                                 prob, value[k] = mult if the light is visible,
                                 tmax / skip of the shadow ray (tmax < 0: none)
     LGPU_PROBE_PROB_LIGHT       probForLight(lights[index], ray(p, i))
                                 (cg.hpp:1735-1747) -> prob
     LGPU_PROBE_SPECTRUM         spectrum `index` of the scene at λ
                                 (coefficientλ::operator(), cg.hpp:298-303) -> value[k]
   The hit is (p, frame F = x, y, z with z the shading normal, front).  xi
   holds the uniform draws in the order the device consumes them (the draws
   of f(a(), b()) are a's then b's).  value has hero_k entries. */
enum {
  LGPU_PROBE_BXDF = 0,
  LGPU_PROBE_PROB_MATERIAL = 1,
  LGPU_PROBE_SAMPLE_MATERIAL = 2,
  LGPU_PROBE_SAMPLE_LIGHT = 3,
  LGPU_PROBE_PROB_LIGHT = 4,
  LGPU_PROBE_SPECTRUM = 5
};

typedef struct lgpu_probe {
  uint32_t op;
  uint32_t index;    /* material, light or spectrum index */
  float lambda[16];  /* hero wavelengths in nm (the first hero_k are used) */
  float p[3];        /* hit point */
  float F[9];        /* shading frame: x, y, z axes */
  float i[3];        /* incident (light) direction; the ray direction of PROB_LIGHT */
  float o[3];        /* outgoing (view) direction */
  float n[3];        /* the normal argument of BXDF */
  uint32_t front;
  float sample_p;    /* SAMPLE_P */
  float xi[4];
} lgpu_probe;

typedef struct lgpu_probe_result {
  float value[16];
  float prob;
  float dir[3];
  float tmax;
  uint32_t skip;
  uint32_t ok;
  uint32_t n_xi; /* draws consumed */
} lgpu_probe_result;

int lgpu_probe_shading(lgpu_ctx* ctx, const lgpu_probe* queries, uint64_t n,
                       lgpu_probe_result* out);

/* Renderer::toneMap (src/renderer.cpp:149-176) followed by the 8-bit sRGB
   encode of rendering::rgb24 (include/renderer.hpp:20-29).  Either output
   may be NULL.  Host buffers of w*h*3 elements; LGPU_ERR_TOO_LARGE if w*h
   is beyond 2^40. */
int lgpu_tonemap(lgpu_ctx* ctx, const float* linrgb, uint64_t w, uint64_t h,
                 float y_mid, float* out_tonemapped, uint8_t* out_rgb24);

int lgpu_get_stats(const lgpu_ctx* ctx, lgpu_stats* out);

/* Tone map without any device allocation (no counterpart in the reference;
   it is lgpu_tonemap for callers that cannot allocate device memory at call
   time, e.g. an engine that owns all device memory in pre-sized pools and
   must not let a cudaMalloc/cudaFree synchronise the device in its frame
   loop).  No context is needed.  The caller passes device (or device-
   accessible) buffers: d_linrgb w*h*3 floats in, d_out_tonemapped w*h*3
   floats and/or d_out_rgb24 w*h*3 bytes out (either may be NULL), and a
   stream (NULL: the legacy default stream); the call returns when the
   results are written.
   Scratch: the reduction's per-block partial sums and the exposure live in
   one file-scope __device__ array of LGPU_NOALLOC_SCRATCH_BYTES bytes that
   every GPU loading the library holds until exit.  Calls share it: two calls
   that overlap on the same GPU race and must be serialised by the caller.
   Every slot a call reads is written by that call first, so nothing needs
   clearing between calls.  The first call on each device looks up the
   array's device address (cudaGetSymbolAddress) with that device current;
   make that first call before any stream capture.  The address is kept for
   the life of the process: it belongs to the CUDA runtime's primary context
   of the device, so the caller must not cudaDeviceReset that device while
   the library is loaded.
   Limit: w*h <= LGPU_NOALLOC_MAX_PIXELS, else LGPU_ERR_TOO_LARGE. */
#define LGPU_NOALLOC_MAX_PIXELS (1ull << 31)
#define LGPU_NOALLOC_SCRATCH_BYTES 9728
int lgpu_tonemap_noalloc(const float* d_linrgb, uint64_t w, uint64_t h, float y_mid,
                         float* d_out_tonemapped, uint8_t* d_out_rgb24, void* stream);

/* Host utility for hosts without the reference's builder: builds the wide
   BVH of one mesh exactly as bvh::build does (cg.hpp:632-749), in the
   reference's layout (see lgpu_mesh).  Every interior node has at least two
   children, so nodes <= 2*n_faces and bbs records <= 2*n_faces: output
   arrays of 4*n_faces words (nodes), 96*n_faces floats (bbs) and n_faces
   words (prim_idxs) always suffice; NULL outputs only return the counts
   (n_nodes counts nodes, n_bbs counts 48-float records). */
int lgpu_build_bvh(const float* V, uint32_t n_positions, const uint32_t* F,
                   uint32_t f_stride, uint32_t n_faces, uint32_t* nodes,
                   uint32_t* n_nodes, float* bbs, uint32_t* n_bbs,
                   uint32_t* prim_idxs, uint32_t* n_prim_idxs);

/* The traversal tree of one mesh (no counterpart in the reference, whose
   traversal uses bvh::build's tree): an 8-wide BVH built with the
   surface-area heuristic on the host threads (a binary tree collapsed to
   8-wide nodes and leaves of at most 2 faces by a cost-optimal dynamic
   program), in the layout and with the array bounds of lgpu_build_bvh.  The instance-BVH
   traversal of the renders enters it instead of the reference's tree: the
   same closest hits in fewer node and triangle tests.  Vertex positions of
   the faces must be finite (else LGPU_ERR_INVALID_ARGUMENT). */
int lgpu_build_traversal_bvh(const float* V, uint32_t n_positions, const uint32_t* F,
                             uint32_t f_stride, uint32_t n_faces, uint32_t* nodes,
                             uint32_t* n_nodes, float* bbs, uint32_t* n_bbs,
                             uint32_t* prim_idxs, uint32_t* n_prim_idxs);

/* lgpu_build_bvh on the context's GPU (bvh::build, cg.hpp:632-749, one
   tree level per step): the same arguments, host arrays in and out, and a
   bit-identical result.  Vertex positions must be finite.  For hosts that load large meshes without the
   reference's trimeshdata, so that building their trees does not cost a
   serial host pass per mesh. */
int lgpu_build_bvh_device(lgpu_ctx* ctx, const float* V, uint32_t n_positions,
                          const uint32_t* F, uint32_t f_stride, uint32_t n_faces,
                          uint32_t* nodes, uint32_t* n_nodes, float* bbs,
                          uint32_t* n_bbs, uint32_t* prim_idxs,
                          uint32_t* n_prim_idxs);

#ifdef __cplusplus
}
#endif

#endif /* LAMBDA_GPU_H */
