// lgpu_scene.h — device-side scene layout shared by the CUDA kernels and the
// host code that builds it.
//
// Layout in HBM (one context, one uploaded scene):
//   objects   DevObject[n_objects]      transforms as 3x4 row blocks
//   meshes    DevMesh[n_meshes]         offsets into the global arrays below
//   nodes     WideNode[...]             8-wide BVH nodes of every mesh, then
//                                       the instance-level BVH (TLAS)
//   tris      TriSlot[...]              leaf triangles in leaf order
//                                       (3 x float4, face id in v0.w)
//   shade     FaceShade[...]            per-face vertex normals + geometric
//                                       normal, indexed by mesh face_base+face
//   spectra   float[n_spectra*n_bins]   coefficient spectra
//   mats      DevMaterial[n_materials]
//   lights    lgpu_light[n_lights]
//
// A WideNode holds the boxes of its (up to) 8 children as six 8-float SoA
// rows, each 32 B, so one child-box test is 12 aligned 16-byte loads; the
// child references follow.  A child reference is either the index of another
// WideNode or, with kLeafBit set, a leaf: (count-1) in bits 28-30 and the
// first triangle slot in bits 0-27.
#pragma once

#include <stdint.h>

#include "lambda_gpu.h"

#ifdef __CUDACC__
#define LGPU_HD __host__ __device__
#else
#define LGPU_HD
#endif

namespace lgpu {

constexpr uint32_t kLeafBit = 0x80000000u;
constexpr uint32_t kEmptyChild = 0xFFFFFFFFu;
constexpr uint32_t kSlotMask = 0x0FFFFFFFu;
constexpr uint32_t kMaxSlots = 0x10000000u;
// traversal stack entries per ray: mesh level (cg.hpp:1407) and instance level
constexpr int kStackCap = 64;
constexpr int kTlasStackCap = 32;
// traversal flags reported by the kernels: a stack bound was hit (the
// traversal stopped; an error), and a traversal stack grew past its
// shared-memory entries into local memory (information)
constexpr uint32_t kTravOverflow = 1u;
constexpr uint32_t kTravLocalStack = 2u;

struct alignas(16) WideNode {
  float lox[8], loy[8], loz[8];
  float hix[8], hiy[8], hiz[8];
  uint32_t child[8];
};
static_assert(sizeof(WideNode) == 224, "WideNode is 7 sectors of 32 B");

struct alignas(16) TriSlot {
  float v0[4];  // xyz + face id bits in [3]
  float v1[4];
  float v2[4];
};

struct FaceShade {
  float n0[3], n1[3], n2[3];
  float gn[3];
};

struct alignas(16) DevObject {
  int32_t type;
  uint32_t mat;
  uint32_t mesh;
  uint32_t reserved;
  float M[12];      // rows 0-2 of transform::M
  float M_inv[12];  // rows 0-2 of transform::M_inv
};

struct DevMesh {
  uint32_t node_base;   // first WideNode of this mesh
  uint32_t slot_base;   // first TriSlot
  uint32_t face_base;   // first FaceShade
  uint32_t root;        // child reference of the root (node or leaf)
  // the root of the traversal tree the instance-BVH traversal enters: a
  // surface-area-heuristic tree in the same node and slot arrays, or `root`
  // (the reference's tree, which the reference-order traversal enters)
  uint32_t trav_root;
  float bounds[6];      // trimeshdata::bounds (inf, sup)
  uint32_t n_faces;
  uint32_t max_stack;   // traversal stack entries this mesh can need
};

struct DevMaterial {
  int32_t type;
  int32_t spectrum[5];
  float alpha, p_d, p_spec, w_r, w_t, d, specular;
};

// Everything a kernel needs, passed by value.
struct DevScene {
  const DevObject* objects;
  const DevMesh* meshes;
  const WideNode* nodes;
  const TriSlot* tris;
  const FaceShade* shade;
  const float* spectra;
  const DevMaterial* mats;
  const lgpu_light* lights;
  const uint32_t* tlas_objects;  // object ids in TLAS leaf order
  uint32_t n_objects, n_meshes, n_materials, n_lights;
  uint32_t tlas_root;  // child reference (node or leaf) of the TLAS root
  uint32_t max_stack;  // max over meshes of DevMesh::max_stack
  uint32_t tlas_max_stack;
  uint32_t n_bins, hero_k;
  float lambda_inf, lambda_sup, lambda_delta;
  const float* cmf;  // 3 * n_bins: X, Y, Z
  lgpu_camera cam;
  float tlas_bounds[6];
};

}  // namespace lgpu
