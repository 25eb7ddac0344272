// Test infrastructure (oracle): argument block shared by the restatement
// (oracle.cpp) and the host build of the reference's sources (refshim/).
#pragma once

extern "C" {
struct or_args {
  int H, W;
  const float* ray_o;
  const float* ray_d;
  const float* verts;
  const int* num_points;
  const int* cumsum;
  int P;
  const float* shs;
  int sh_degree;
  int M;
  const float* opacities;
  const float* sigma;
  const float* bg;
  const float* extra;
  int extra_len;
  int variant;         // 0 plain, 1 reflect, 2 refract, 3 envlight
  int tmin_inclusive;  // 1: optixTrace's closed interval
  int canonical_ties;  // 1: equal-t hits ordered by primitive id
  int exact_geometry;  // 1: FP64 hit point (FP64 precision only)
  int nthreads;
  int row_begin, row_end;  // rows of the image to trace (row_end <= 0: all)
  // backward inputs (precision of the call)
  const void* colors;
  const void* others;
  const float* dL_dpixels;
  const float* dL_dothers;
  // optional per-ray record
  int max_rec;
  int* rec_ids;     // [H*W, max_rec]
  int* rec_count;   // [H*W]
  float* margin;    // [H*W]
  // optional proposed interval per ray, [2][H*W] (t_near plane, t_far plane)
  const float* interval;
  // secondary rays (or_*_secondary only)
  const int* material;
  const float* ior;
  const float* env;
  int env_h, env_w, max_depth;
  int exact_adjoint;  // 1: full chain rule + forward depth (FP64 with exact geometry)
  const float* precomp;  // [P][3] precomputed colours in place of SH, or NULL
  void* dprecomp;        // their gradient (precision of the call), backward only
  // optional log of every k-closest query a ray's forward made (host build of
  // the reference only): per ray up to max_chunks queries, each its lower
  // bound tmin and the 16 primitive ids the any-hit program left in the
  // payload (0xFFFFFFFF for empty slots)
  int max_chunks;
  unsigned* chunk_ids;  // [H*W][max_chunks][16]
  float* chunk_tmin;    // [H*W][max_chunks]
  int* chunk_count;     // [H*W] queries made (may exceed max_chunks)
  // secondary-ray adjoint, optional (precision of the call): gradients of the
  // environment map [env_h][env_w][3] and of the IOR [P]; and the test hook
  // SecInputs::ior_fresnel
  void* denv;
  void* dior;
  const float* ior_fresnel;
};
}
