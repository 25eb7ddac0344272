// Host-side interface of the LBVH builder (bvh.cu).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "tt_device.cuh"

namespace tt {

// Grow-only device buffer.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaError_t reserve(size_t n);
  void release();
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

// Replaces OptiX's GAS build/update (tritracer/pipeline.cpp:206-265): a
// Morton-ordered linear BVH (Karras 2012) collapsed to 8-wide nodes. All
// steps are kernels on the caller's stream; nothing synchronises.
class Bvh {
 public:
  // Full build from vertices (float[num_vertices][3]) through cumsum[P].
  cudaError_t build(const float* verts, const int* cumsum, int P, cudaStream_t s);
  // Same topology, boxes and triangle records recomputed from moved vertices.
  cudaError_t refit(const float* verts, const int* cumsum, int P, cudaStream_t s);
  void release();

  BvhView view() const;
  bool built() const { return built_; }
  int P() const { return P_; }
  // device scalars: [0] number of wide nodes, [1] error flag of the collapse
  const int* counters() const { return counters_.as<int>(); }
  // kernels enqueued by build/refit so far
  unsigned long long launches() const { return launches_; }
  // Serialised topology: a host blob of the Morton order, the binary and
  // 8-wide hierarchies (not the triangle records or boxes, which load()
  // rebuilds from the vertices with a refit). save() synchronises `s`; with
  // dst == nullptr it only reports the size.
  cudaError_t save(void* dst, size_t capacity, size_t* bytes, cudaStream_t s);
  // 1: bad blob (magic, version, size or triangle count), else a CUDA error
  int load(const void* src, size_t bytes, const float* verts, const int* cumsum, int P, cudaStream_t s,
           cudaError_t* err);

 private:
  cudaError_t reserve(int P);
  cudaError_t prep(const float* verts, const int* cumsum, int P, bool sorted_only, cudaStream_t s);
  cudaError_t boxes(cudaStream_t s);

  unsigned long long launches_ = 0;
  int P_ = 0;
  int cap_ = 0;
  bool built_ = false;
  DevBuf tri_prim_, tri_sorted_;       // 3 float4 per triangle
  DevBuf centroid_, bounds_;           // float4 per prim; 6 ints (ordered-float bounds)
  DevBuf keys_, vals_, keys2_, vals2_; // radix sort ping-pong
  DevBuf hist_;                        // 256 x tiles
  DevBuf bnode_;                       // binary internal nodes (BinNode)
  DevBuf bparent_, lparent_, flags_;   // parents of internal nodes / leaves, arrival flags
  DevBuf wnodes_, wsrc_, wbin_;        // wide nodes, per-slot binary source, per-node binary source
  DevBuf levels_;                      // per-level wide node counts
  DevBuf counters_;
};

// Device buffers of one BVH carved out of caller-provided memory: the same
// build kernels as Bvh::build, for callers that may not allocate.
struct BvhStorage {
  float4* tri_prim;
  float4* tri_sorted;
  float4* centroid;
  int* bounds;
  uint32_t *keys, *vals, *keys2, *vals2, *hist;
  void* bnode;
  int *bparent, *lparent, *flags;
  float4* wnodes;
  int *wsrc, *wbin, *levels, *counters;
};

// Bytes needed for P triangles (every array 256-byte aligned).
size_t bvh_storage_bytes(int P);
BvhStorage bvh_storage_carve(void* base, int P);
cudaError_t bvh_build_into(const BvhStorage& st, const float* verts, const int* cumsum, int P, cudaStream_t s);
BvhView bvh_storage_view(const BvhStorage& st, int P);

// Stable LSD radix sort of n (key, value) pairs by the low `bits` bits of the
// keys, 8 bits a pass, with the builder's kernels (a histogram, a scan of 1
// or 3 launches and a scatter a pass, sort_pairs_launches in all); nothing
// synchronises. The sorted pairs end in (keys, vals) after an even number of
// passes and in (keys2, vals2) after an odd one (*in_second). hist holds
// sort_pairs_hist_words(n) words.
size_t sort_pairs_hist_words(int n);
// Kernel launches of one sort_pairs call.
int sort_pairs_launches(int n, int bits);
cudaError_t sort_pairs(uint32_t* keys, uint32_t* vals, uint32_t* keys2, uint32_t* vals2, uint32_t* hist, int n,
                       int bits, bool* in_second, cudaStream_t s);

}  // namespace tt
