// lgpu_layout.h — host-side construction of the device scene layout.
#pragma once

#include <memory>
#include <string>
#include <utility>
#include <vector>

#include "lambda_gpu.h"
#include "lgpu_scene.h"

namespace lgpu {

// Wide BVH in the reference's own format (cg.hpp:596-631), built with the
// reference's algorithm (bvh::build, cg.hpp:632-749).
struct RefBvh {
  std::vector<uint32_t> nodes;  // pairs {childrenbb_idx, data}
  std::vector<float> bbs;       // 48 floats per record
  std::vector<uint32_t> prim_idxs;
  uint32_t n_nodes = 0, n_interior = 0;
};

// A wide BVH in the reference's format, by reference (a mesh's traversal
// tree: the caller's arrays or one built at upload).  n_nodes 0: none.
struct TravTree {
  uint32_t n_nodes = 0, n_bbs = 0, n_prims = 0;
  const uint32_t* nodes = nullptr;
  const float* bbs = nullptr;
  const uint32_t* prims = nullptr;
};

struct PrimBox {
  float inf[3], sup[3];
};

// Builds over n primitives given their boxes and centroids
// (centroid[3*i + axis]); leaves hold at most max_leaf primitives (the
// reference's PRIM_PER_LEAF = 4 for meshes).
void build_ref_bvh(uint32_t n, const PrimBox* boxes, const float* centroids, RefBvh& out,
                   size_t max_leaf = 4);

// The traversal tree of a mesh (lgpu_sah.cpp): an 8-wide BVH over the same
// primitive boxes, a binary surface-area-heuristic tree collapsed by a
// cost-optimal dynamic program, in the same format; leaves hold at most
// max_leaf primitives.  Boxes and centroids must
// be finite.
void build_sah_bvh(uint32_t n, const PrimBox* boxes, const float* centroids, RefBvh& out,
                   size_t max_leaf = 2);

// Boxes and centroids of triangle faces as trimeshdata::aabboftri and
// centroidoftri compute them (cg.hpp:776-790).
void triangle_prims(const float* V, const uint32_t* F, uint32_t f_stride, uint32_t n_faces,
                    std::vector<PrimBox>& boxes, std::vector<float>& centroids);

}  // namespace lgpu

#include <cuda_runtime_api.h>

namespace lgpu {

// build_ref_bvh for a triangle mesh, on the device (lgpu_bvh_build.cu):
// host arrays in, the same tree out.  Face indices must be valid.
cudaError_t build_bvh_device(const float* V, uint32_t n_positions, const uint32_t* F, uint32_t f_stride,
                             uint32_t n_faces, RefBvh& out, cudaStream_t st);

// An allocator whose value-initialisation leaves trivial elements
// uninitialised: the layout writes every field of its large arrays itself,
// so growing them need not clear tens of MB first.
template <class T>
struct NoInitAllocator : std::allocator<T> {
  template <class U>
  struct rebind {
    using other = NoInitAllocator<U>;
  };
  NoInitAllocator() = default;
  template <class U>
  NoInitAllocator(const NoInitAllocator<U>&) noexcept {}
  template <class U>
  void construct(U* p) noexcept {
    ::new (static_cast<void*>(p)) U;
  }
  template <class U, class... A>
  void construct(U* p, A&&... a) {
    ::new (static_cast<void*>(p)) U(std::forward<A>(a)...);
  }
};
template <class T>
using BigVector = std::vector<T, NoInitAllocator<T>>;

// The device layout of a scene.  A context keeps one and lays every upload
// out into it, so the arrays keep their capacity (and their pages) from one
// upload to the next.
struct HostLayout {
  std::vector<DevObject> objects;
  std::vector<DevMesh> meshes;
  BigVector<WideNode> nodes;
  BigVector<TriSlot> tris;
  BigVector<FaceShade> shade;
  std::vector<float> spectra;
  std::vector<DevMaterial> mats;
  std::vector<lgpu_light> lights;
  std::vector<uint32_t> tlas_objects;
  std::vector<float> cmf;
  uint32_t tlas_root = 0, max_stack = 0, tlas_max_stack = 0;
  float tlas_bounds[6] = {0, 0, 0, 0, 0, 0};
};

// A mesh whose WideNodes, leaf triangles and shading normals are built on
// the device (build_mesh_layout) from its raw arrays.
struct DeviceMeshJob {
  uint32_t mesh;                  // index in the scene
  uint32_t node_base, n_int;      // its first WideNode and their number
  uint32_t slot_base, face_base;  // its first TriSlot and FaceShade
  size_t childref_off;            // its child references in DeviceLayoutWork::childref
  // the mesh's traversal tree instead of its own BVH (no shading records:
  // the job of the mesh's own BVH, just before this one, writes them)
  const TravTree* tree = nullptr;
};
struct DeviceLayoutWork {
  std::vector<DeviceMeshJob> jobs;
  // per reference node of each mesh: its child reference (WideNode index,
  // or leaf: kLeafBit | (count-1) << 28 | first slot)
  std::vector<uint32_t> childref;
  uint32_t mesh_nodes = 0, mesh_slots = 0, mesh_faces = 0;  // totals over the meshes
};

// Validates the scene and lays it out for the device.  Returns LGPU_OK or
// an lgpu_status with a message in err.  With dev, the meshes are left to
// the device: L.nodes then holds only the instance BVH (its node indices
// follow the meshes' dev->mesh_nodes nodes), L.tris and L.shade stay
// empty, and dev lists what build_mesh_layout has to build; the face and
// primitive indices are checked there.
// trav, if given, holds per mesh its traversal tree (n_nodes 0: none), laid
// out after the mesh's own tree; DevMesh::trav_root is its root,
// or the mesh's own root without one.
int make_layout(const lgpu_scene& sc, HostLayout& L, std::string& err, DeviceLayoutWork* dev = nullptr,
                const std::vector<TravTree>* trav = nullptr);

// The validated material table alone (for lgpu_update_materials).
int make_materials(const lgpu_scene& sc, std::vector<DevMaterial>& mats, std::string& err);

}  // namespace lgpu
