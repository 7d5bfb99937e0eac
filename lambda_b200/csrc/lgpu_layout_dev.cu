// lgpu_layout_dev.cu — the meshes' part of the scene layout built on the
// device at upload: from the raw arrays of nl::cg::trimeshdata and its BVH
// (cg.hpp:766-820, 596-631) to the WideNodes, TriSlots and FaceShades the
// traversal and shading read (lgpu_scene.h).  The host keeps the pass that
// validates the BVH and numbers its nodes (lgpu_layout.cpp, relayout_meta);
// these kernels only move values, so the result is bit-identical to the
// host layout.  Face and primitive indices are checked here: an index out
// of range is skipped and reported through *err (the lowest mesh * 4 +
// kind, kind 1 = a face's vertex or normal index, 2 = a BVH primitive
// index), and the upload fails.
#include "lgpu_layout.h"
#include "lgpu_layout_dev.h"

namespace lgpu {

namespace {

constexpr uint32_t kErrFace = 1, kErrPrim = 2;

// one thread per reference node: the WideNode of an interior node
__global__ void __launch_bounds__(256) k_mesh_nodes(MeshRaw m, WideNode* __restrict__ nodes) {
  uint32_t const q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= m.n_nodes) return;
  uint32_t const d = m.nodes[2 * size_t(q) + 1];
  if (d & 1u) return;  // leaf
  // bbs index and child range were validated by relayout_meta
  const float* bb = m.bbs + 48 * size_t(m.nodes[2 * size_t(q)]);
  uint32_t const first = (d & 0xFFFFFFF0u) >> 4, cnt = ((d & 0xEu) >> 1) + 1;
  WideNode& wn = nodes[m.childref[q]];
#pragma unroll
  for (int c = 0; c < 8; c++) {
    if (uint32_t(c) < cnt) {
      wn.lox[c] = bb[0 * 8 + c];
      wn.loy[c] = bb[1 * 8 + c];
      wn.loz[c] = bb[2 * 8 + c];
      wn.hix[c] = bb[3 * 8 + c];
      wn.hiy[c] = bb[4 * 8 + c];
      wn.hiz[c] = bb[5 * 8 + c];
      wn.child[c] = m.childref[first + c];
    } else {
      wn.lox[c] = wn.loy[c] = wn.loz[c] = 1e30f;
      wn.hix[c] = wn.hiy[c] = wn.hiz[c] = -1e30f;
      wn.child[c] = kEmptyChild;
    }
  }
}

// one thread per leaf slot: the slot's triangle (vertices in leaf order,
// face id in v0.w)
__global__ void __launch_bounds__(256) k_mesh_tris(MeshRaw m, uint32_t mesh, TriSlot* __restrict__ tris,
                                                   uint32_t* err) {
  uint32_t const s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= m.n_prims) return;
  uint32_t const f = m.prims[s];
  if (f >= m.n_faces) {
    atomicMin(err, mesh * 4u + kErrPrim);
    return;
  }
  const uint32_t* t = m.F + size_t(f) * m.f_stride;
  uint32_t const i0 = t[0], i1 = t[1], i2 = t[2];
  if (i0 >= m.n_positions || i1 >= m.n_positions || i2 >= m.n_positions) return;  // k_mesh_shade reports it
  TriSlot ts;
#pragma unroll
  for (int i = 0; i < 3; i++) {
    ts.v0[i] = m.V[3 * size_t(i0) + i];
    ts.v1[i] = m.V[3 * size_t(i1) + i];
    ts.v2[i] = m.V[3 * size_t(i2) + i];
  }
  ts.v0[3] = __uint_as_float(f);
  ts.v1[3] = 0.f;
  ts.v2[3] = 0.f;
  tris[s] = ts;
}

// one thread per face: its three vertex normals and its geometric normal
__global__ void __launch_bounds__(256) k_mesh_shade(MeshRaw m, uint32_t mesh, FaceShade* __restrict__ shade,
                                                    uint32_t* err) {
  uint32_t const f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= m.n_faces) return;
  const uint32_t* t = m.F + size_t(f) * m.f_stride;
  bool bad = false;
#pragma unroll
  for (int k = 0; k < 3; k++) bad = bad || t[k] >= m.n_positions || t[3 + k] >= m.n_normals;
  if (bad) {
    atomicMin(err, mesh * 4u + kErrFace);
    return;
  }
  FaceShade fs;
#pragma unroll
  for (int i = 0; i < 3; i++) {
    fs.n0[i] = m.N[3 * size_t(t[3]) + i];
    fs.n1[i] = m.N[3 * size_t(t[4]) + i];
    fs.n2[i] = m.N[3 * size_t(t[5]) + i];
    fs.gn[i] = m.GN[3 * size_t(f) + i];
  }
  shade[f] = fs;
}

}  // namespace

cudaError_t build_mesh_layout(const MeshRaw& m, uint32_t mesh, WideNode* nodes, TriSlot* tris, FaceShade* shade,
                              uint32_t* err, cudaStream_t st) {
  if (m.n_nodes) k_mesh_nodes<<<(m.n_nodes + 255) / 256, 256, 0, st>>>(m, nodes);
  if (m.n_prims) k_mesh_tris<<<(m.n_prims + 255) / 256, 256, 0, st>>>(m, mesh, tris, err);
  if (m.n_faces && shade) k_mesh_shade<<<(m.n_faces + 255) / 256, 256, 0, st>>>(m, mesh, shade, err);
  return cudaGetLastError();
}

}  // namespace lgpu
