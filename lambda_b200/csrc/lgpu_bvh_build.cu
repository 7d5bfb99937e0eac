// lgpu_bvh_build.cu — the reference's wide BVH builder (bvh::build,
// cg.hpp:632-749) on the device, for lgpu_build_bvh_device.
//
// The reference builds top-down and recursively: a node with more than
// PRIM_PER_LEAF = 4 triangles is split into 8 bins along the longest axis of
// its box by triangle centroid (a bin that would take every triangle is
// replaced by 8 equal chunks of the node's list), each child keeps its
// triangles in the parent's order, and the tree is flattened breadth first.
// Breadth-first order is level order, so the device builds one level per
// step: one block per interior node bins its triangles, scatters them stably
// into its children's ranges, and reduces the children's boxes; the host
// numbers the nodes level by level exactly as the reference's queue does.
//
// Every float operation is the reference's, in its order (the centroid
// (v0 + v1 + v2) / 3, the bin 8 * (c - inf) / len, nl::min / nl::max
// folds), so the output is bit-identical to lgpu_build_bvh's.  A box is a
// fold of nl::min(a, b) = a <= b ? a : b over the triangles in order, whose
// result is the smallest value and, among values that compare equal (+0 and
// -0), the first one: the device reduces (value, position) keys to the same.
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstring>
#include <vector>

#include "lgpu_layout.h"

namespace lgpu {

namespace {

constexpr uint32_t kBuildThreads = 256;
constexpr uint32_t kLeafPrims = 4;  // PRIM_PER_LEAF, cg.hpp:568

__device__ __forceinline__ float nl_min_d(float a, float b) { return a <= b ? a : b; }
__device__ __forceinline__ float nl_max_d(float a, float b) { return a >= b ? a : b; }

// Monotone map of floats to unsigned keys in which +0 and -0 are equal.
__device__ __forceinline__ uint32_t order_key(float v) {
  uint32_t const b = __float_as_uint(v == 0.f ? 0.f : v);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
// Keys for "smallest value, first position" (k < 3: a box minimum) and
// "largest value, first position" (k >= 3: a maximum), both reduced by min.
__device__ __forceinline__ unsigned long long extreme_key(float v, int k, uint32_t pos) {
  uint32_t const o = order_key(v);
  return (static_cast<unsigned long long>(k < 3 ? o : ~o) << 32) | pos;
}

// aabboftri and centroidoftri (cg.hpp:776-790) of every face
__global__ void __launch_bounds__(kBuildThreads) bvh_prims(const float* __restrict__ V,
                                                           const uint32_t* __restrict__ F, uint32_t stride,
                                                           uint32_t nf, float* __restrict__ box,
                                                           float* __restrict__ cent) {
  for (uint32_t f = blockIdx.x * blockDim.x + threadIdx.x; f < nf; f += gridDim.x * blockDim.x) {
    const uint32_t* t = F + size_t(f) * stride;
    float lo[3] = {1e30f, 1e30f, 1e30f}, hi[3] = {-1e30f, -1e30f, -1e30f};
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const float* v = V + 3 * size_t(t[k]);
#pragma unroll
      for (int i = 0; i < 3; i++) {
        lo[i] = nl_min_d(lo[i], v[i]);
        hi[i] = nl_max_d(hi[i], v[i]);
      }
    }
#pragma unroll
    for (int i = 0; i < 3; i++) {
      box[6 * size_t(f) + i] = lo[i];
      box[6 * size_t(f) + 3 + i] = hi[i];
      float const s = __fadd_rn(__fadd_rn(V[3 * size_t(t[0]) + i], V[3 * size_t(t[1]) + i]),
                                V[3 * size_t(t[2]) + i]);
      cent[3 * size_t(f) + i] = __fdiv_rn(s, 3.f);
    }
  }
}

// The fold's result from the reduced key of its extreme: the initial value
// of aabb::init (1e30 / -1e30) stays unless the extreme passes it.
__device__ __forceinline__ float resolve_extreme(unsigned long long key, int k, const float* box,
                                                 const uint32_t* prim_at) {
  float const init = k < 3 ? 1e30f : -1e30f;
  if (key == ~0ull) return init;
  float const v = box[6 * size_t(prim_at[uint32_t(key)]) + k];
  return k < 3 ? nl_min_d(init, v) : nl_max_d(init, v);
}

// Box of the root: the fold over every face in index order (one block).
__global__ void __launch_bounds__(1024) bvh_root_box(const float* __restrict__ box, const uint32_t* __restrict__ idx,
                                                     uint32_t n, float* __restrict__ out) {
  __shared__ unsigned long long key[6];
  if (threadIdx.x < 6) key[threadIdx.x] = ~0ull;
  __syncthreads();
  for (uint32_t j = threadIdx.x; j < n; j += blockDim.x)
#pragma unroll
    for (int k = 0; k < 6; k++) atomicMin(&key[k], extreme_key(box[6 * size_t(idx[j]) + k], k, j));
  __syncthreads();
  if (threadIdx.x < 6) out[threadIdx.x] = resolve_extreme(key[threadIdx.x], threadIdx.x, box, idx);
}

}  // namespace

// One interior node of a level: its range of the triangle order and split.
struct BuildSplit {
  uint32_t start, count, axis;
  float inf, len;
};

namespace {

// bvh::splitbuildnode (cg.hpp:632-683) for every interior node of a level,
// one block per node: bin sizes, the full-bin redistribution, a stable
// scatter of the node's triangles into its children's ranges (bin order,
// each child in the parent's order) and the children's boxes.
__global__ void __launch_bounds__(kBuildThreads) bvh_split(const BuildSplit* __restrict__ splits,
                                                           const uint32_t* __restrict__ idx_in,
                                                           uint32_t* __restrict__ idx_out,
                                                           const float* __restrict__ box,
                                                           const float* __restrict__ cent,
                                                           uint32_t* __restrict__ child_count,
                                                           float* __restrict__ child_box) {
  constexpr int kWarps = kBuildThreads / 32;
  BuildSplit const nd = splits[blockIdx.x];
  const uint32_t* const in = idx_in + nd.start;
  __shared__ uint32_t cnt[8], off[8], run[8], wcnt[8][kWarps];
  __shared__ unsigned long long key[8][6];
  __shared__ uint32_t chunk;  // 0, or the chunk size of the redistribution
  uint32_t const t = threadIdx.x, lane = t & 31u, wid = t >> 5;
  if (t < 8) {
    cnt[t] = 0;
    run[t] = 0;
  }
  if (t < 48) key[t / 6][t % 6] = ~0ull;
  __syncthreads();
  // the bin of position j: int(8 * (c - inf) / len), kept in [0, 7] as
  // the host restatement keeps it (the reference's int() of an
  // out-of-range value is undefined)
  auto bin_of = [&](uint32_t j) -> uint32_t {
    float const c = cent[3 * size_t(in[j]) + nd.axis];
    float const x = __fdiv_rn(__fmul_rn(8.f, __fsub_rn(c, nd.inf)), nd.len);
    int b = (x >= -1.f && x < 8.f) ? int(x) : (x >= 8.f ? 7 : 0);
    return uint32_t(b < 0 ? 0 : (b > 7 ? 7 : b));
  };
  for (uint32_t j = t; j < nd.count; j += blockDim.x) atomicAdd(&cnt[bin_of(j)], 1u);
  __syncthreads();
  if (t == 0) {
    chunk = 0;
    for (int b = 0; b < 8; b++)
      if (cnt[b] == nd.count) chunk = (nd.count + 7) / 8;  // cg.hpp:658-672
    if (chunk)
      for (uint32_t b = 0; b < 8; b++) {
        uint32_t const s = b * chunk, e = min(s + chunk, nd.count);
        cnt[b] = s < e ? e - s : 0;
      }
    uint32_t s = 0;
    for (int b = 0; b < 8; b++) {
      off[b] = s;
      s += cnt[b];
    }
  }
  __syncthreads();
  for (uint32_t base = 0; base < nd.count; base += blockDim.x) {
    uint32_t const j = base + t;
    bool const here = j < nd.count;
    uint32_t b = 8;
    if (here) b = chunk ? j / chunk : bin_of(j);
    uint32_t rank = 0;
#pragma unroll
    for (uint32_t q = 0; q < 8; q++) {
      unsigned const m = __ballot_sync(0xFFFFFFFFu, b == q);
      if (lane == 0) wcnt[q][wid] = __popc(m);
      if (b == q) rank = __popc(m & ((1u << lane) - 1u));
    }
    __syncthreads();
    if (here) {
      uint32_t pos = off[b] + run[b] + rank;
      for (uint32_t v = 0; v < wid; v++) pos += wcnt[b][v];
      uint32_t const prim = in[j];
      idx_out[nd.start + pos] = prim;
#pragma unroll
      for (int k = 0; k < 6; k++) atomicMin(&key[b][k], extreme_key(box[6 * size_t(prim) + k], k, j));
    }
    __syncthreads();
    if (t < 8) {
      uint32_t s = 0;
      for (int v = 0; v < kWarps; v++) s += wcnt[t][v];
      run[t] += s;
    }
    __syncthreads();
  }
  if (t < 8) child_count[8 * size_t(blockIdx.x) + t] = cnt[t];
  if (t < 48) child_box[48 * size_t(blockIdx.x) + t] = resolve_extreme(key[t / 6][t % 6], t % 6, box, in);
}

// Leaves of a level: their triangles to the output, in breadth-first order.
__global__ void __launch_bounds__(kBuildThreads) bvh_leaves(const uint32_t* __restrict__ spans /*src, dst, n*/,
                                                            uint32_t n_leaves, const uint32_t* __restrict__ idx,
                                                            uint32_t* __restrict__ prim_idxs) {
  for (uint32_t l = blockIdx.x * blockDim.x + threadIdx.x; l < n_leaves; l += gridDim.x * blockDim.x)
    for (uint32_t k = 0; k < spans[3 * l + 2]; k++) prim_idxs[spans[3 * l + 1] + k] = idx[spans[3 * l] + k];
}

__global__ void bvh_iota(uint32_t* idx, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) idx[i] = i;
}

struct DevBuf {
  void* p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
  cudaError_t alloc(size_t bytes) { return cudaMalloc(&p, bytes ? bytes : 1); }
};

struct LevelNode {
  uint32_t start, count, bfs;
  float bb[6];  // inf xyz, sup xyz
};

}  // namespace

// bvh::build (cg.hpp:737-749) of a triangle mesh on the device, into the
// reference's layout (as build_ref_bvh).  Inputs are host arrays; indices
// must already be validated.
cudaError_t build_bvh_device(const float* V, uint32_t n_positions, const uint32_t* F, uint32_t stride,
                             uint32_t nf, RefBvh& out, cudaStream_t st) {
  out = RefBvh{};
  if (nf == 0) return cudaSuccess;
  DevBuf dV, dF, dbox, dcent, didx0, didx1, dprims, dsplit, dcc, dcb, dspan;
  cudaError_t e = dV.alloc(3 * size_t(n_positions) * sizeof(float));
  if (e == cudaSuccess) e = dF.alloc(size_t(nf) * stride * sizeof(uint32_t));
  if (e == cudaSuccess) e = dbox.alloc(6 * size_t(nf) * sizeof(float));
  if (e == cudaSuccess) e = dcent.alloc(3 * size_t(nf) * sizeof(float));
  if (e == cudaSuccess) e = didx0.alloc(size_t(nf) * sizeof(uint32_t));
  if (e == cudaSuccess) e = didx1.alloc(size_t(nf) * sizeof(uint32_t));
  if (e == cudaSuccess) e = dprims.alloc(size_t(nf) * sizeof(uint32_t));
  if (e != cudaSuccess) return e;
  e = cudaMemcpyAsync(dV.p, V, 3 * size_t(n_positions) * sizeof(float), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dF.p, F, size_t(nf) * stride * sizeof(uint32_t), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return e;
  uint32_t const grid = (nf + kBuildThreads - 1) / kBuildThreads < 4096 ? (nf + kBuildThreads - 1) / kBuildThreads
                                                                         : 4096;
  bvh_prims<<<grid, kBuildThreads, 0, st>>>(dV.as<float>(), dF.as<uint32_t>(), stride, nf, dbox.as<float>(),
                                            dcent.as<float>());
  bvh_iota<<<grid, kBuildThreads, 0, st>>>(didx0.as<uint32_t>(), nf);
  DevBuf droot;
  e = droot.alloc(6 * sizeof(float));
  if (e != cudaSuccess) return e;
  bvh_root_box<<<1, 1024, 0, st>>>(dbox.as<float>(), didx0.as<uint32_t>(), nf, droot.as<float>());
  LevelNode root{0, nf, 0, {}};
  e = cudaMemcpyAsync(root.bb, droot.p, sizeof(root.bb), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return e;

  std::vector<LevelNode> cur{root}, next;
  std::vector<uint32_t> node_data;     // 2 per node: {childrenbb_idx or interior rank, data}
  std::vector<float> interior_boxes;   // 48 per interior node, breadth-first
  node_data.reserve(4 * size_t(nf));
  node_data.resize(2);
  uint32_t next_free = 1, prim_off = 0, n_interior = 0;
  size_t split_cap = 0, span_cap = 0;
  std::vector<BuildSplit> splits;
  std::vector<uint32_t> spans, counts;
  std::vector<float> cboxes;
  uint32_t* idx_in = didx0.as<uint32_t>();
  uint32_t* idx_out = didx1.as<uint32_t>();
  while (!cur.empty()) {
    splits.clear();
    spans.clear();
    std::vector<uint32_t> interior_of;  // level position of each interior node
    for (uint32_t k = 0; k < cur.size(); k++) {
      const LevelNode& nd = cur[k];
      if (nd.count <= kLeafPrims) {
        node_data[2 * size_t(nd.bfs)] = 0xFFFFFFFFu;
        node_data[2 * size_t(nd.bfs) + 1] = (prim_off << 4) | ((nd.count - 1) << 1) | 1u;
        spans.insert(spans.end(), {nd.start, prim_off, nd.count});
        prim_off += nd.count;
        continue;
      }
      // the splitting axis (cg.hpp:645-649)
      float l[3];
      for (int i = 0; i < 3; i++) l[i] = nd.bb[3 + i] - nd.bb[i];
      uint32_t ax = 0;
      if (l[1] > l[0]) ax = 1;
      if (l[2] > l[1] && l[2] > l[0]) ax = 2;
      splits.push_back(BuildSplit{nd.start, nd.count, ax, nd.bb[ax], l[ax]});
      interior_of.push_back(k);
    }
    uint32_t const n_leaves = uint32_t(spans.size() / 3), n_split = uint32_t(splits.size());
    if (n_leaves) {
      if (spans.size() > span_cap) {
        span_cap = 2 * spans.size();
        if (dspan.p) cudaFree(dspan.p);
        dspan.p = nullptr;
        if ((e = dspan.alloc(span_cap * sizeof(uint32_t))) != cudaSuccess) return e;
      }
      e = cudaMemcpyAsync(dspan.p, spans.data(), spans.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st);
      if (e != cudaSuccess) return e;
      uint32_t const lg = (n_leaves + kBuildThreads - 1) / kBuildThreads;
      bvh_leaves<<<lg < 4096 ? lg : 4096, kBuildThreads, 0, st>>>(dspan.as<uint32_t>(), n_leaves, idx_in,
                                                                  dprims.as<uint32_t>());
    }
    if (!n_split) {
      e = cudaStreamSynchronize(st);
      if (e != cudaSuccess) return e;
      break;
    }
    if (n_split > split_cap) {
      split_cap = 2 * size_t(n_split);
      for (DevBuf* b : {&dsplit, &dcc, &dcb}) {
        if (b->p) cudaFree(b->p);
        b->p = nullptr;
      }
      if ((e = dsplit.alloc(split_cap * sizeof(BuildSplit))) != cudaSuccess) return e;
      if ((e = dcc.alloc(split_cap * 8 * sizeof(uint32_t))) != cudaSuccess) return e;
      if ((e = dcb.alloc(split_cap * 48 * sizeof(float))) != cudaSuccess) return e;
    }
    e = cudaMemcpyAsync(dsplit.p, splits.data(), n_split * sizeof(BuildSplit), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    bvh_split<<<n_split, kBuildThreads, 0, st>>>(dsplit.as<BuildSplit>(), idx_in, idx_out, dbox.as<float>(),
                                                 dcent.as<float>(), dcc.as<uint32_t>(), dcb.as<float>());
    counts.resize(8 * size_t(n_split));
    cboxes.resize(48 * size_t(n_split));
    e = cudaMemcpyAsync(counts.data(), dcc.p, counts.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(cboxes.data(), dcb.p, cboxes.size() * sizeof(float), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    // bvh::convertbuildnodes (cg.hpp:687-728): children numbered in the
    // order the queue pops their parents, in bin order
    next.clear();
    for (uint32_t s = 0; s < n_split; s++) {
      const LevelNode& nd = cur[interior_of[s]];
      uint32_t const first = next_free;
      uint32_t nc = 0, start = nd.start;
      float rec[48];
      for (int a = 0; a < 3; a++)
        for (int c = 0; c < 8; c++) {
          rec[8 * a + c] = 1e30f;
          rec[24 + 8 * a + c] = -1e30f;
        }
      for (int b = 0; b < 8; b++) {
        uint32_t const n = counts[8 * size_t(s) + b];
        if (!n) continue;
        LevelNode ch{start, n, next_free + nc, {}};
        std::memcpy(ch.bb, &cboxes[48 * size_t(s) + 6 * b], sizeof(ch.bb));
        for (int a = 0; a < 3; a++) {
          rec[8 * a + nc] = ch.bb[a];
          rec[24 + 8 * a + nc] = ch.bb[3 + a];
        }
        next.push_back(ch);
        start += n;
        nc++;
      }
      next_free += nc;
      node_data[2 * size_t(nd.bfs)] = n_interior++;  // rank; the record index is set below
      node_data[2 * size_t(nd.bfs) + 1] = (first << 4) | ((nc - 1) << 1);
      interior_boxes.insert(interior_boxes.end(), rec, rec + 48);
    }
    node_data.resize(2 * size_t(next_free));
    std::swap(idx_in, idx_out);
    cur.swap(next);
  }
  out.n_nodes = next_free;
  out.n_interior = n_interior;
  // the reference resizes bbs to n_interior records before appending them
  // (cg.hpp:689-690, 718-722): records start at n_interior
  for (uint32_t k = 0; k < next_free; k++)
    if (!(node_data[2 * size_t(k) + 1] & 1u)) node_data[2 * size_t(k)] += n_interior;
  out.nodes = std::move(node_data);
  out.bbs.assign(48 * size_t(n_interior), 0.f);
  out.bbs.insert(out.bbs.end(), interior_boxes.begin(), interior_boxes.end());
  out.prim_idxs.resize(prim_off);
  e = cudaMemcpyAsync(out.prim_idxs.data(), dprims.p, prim_off * sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  return e;
}

}  // namespace lgpu
