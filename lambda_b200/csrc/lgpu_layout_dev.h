// lgpu_layout_dev.h — the meshes' layout built on the device at upload
// (lgpu_layout_dev.cu).
#pragma once

#include <cuda_runtime.h>

#include "lgpu_scene.h"

namespace lgpu {

// The raw arrays of one mesh in device memory (lgpu_mesh, include/
// lambda_gpu.h) and its child references from relayout_meta.
struct MeshRaw {
  const float* V;
  const float* N;
  const float* GN;
  const uint32_t* F;
  const uint32_t* nodes;
  const float* bbs;
  const uint32_t* prims;
  const uint32_t* childref;
  uint32_t n_positions, n_normals, n_faces, f_stride, n_nodes, n_prims;
};

// Writes the mesh's interior WideNodes into nodes (the scene's node array:
// childref holds global indices), its leaf triangles into tris (its first
// slot) and its shading records into shade (its first face).  *err is
// lowered to mesh * 4 + 1 (a face index out of range) or + 2 (a BVH
// primitive index out of range).  With shade NULL the shading records are
// not written (a second tree of a mesh whose records exist).
cudaError_t build_mesh_layout(const MeshRaw& m, uint32_t mesh, WideNode* nodes, TriSlot* tris, FaceShade* shade,
                              uint32_t* err, cudaStream_t st);

}  // namespace lgpu
