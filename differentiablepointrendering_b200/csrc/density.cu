// density.cu -- density control of the surfel cloud on the device.
//
// python/density_control.py decides which surfels to remove or split on
// the host (numpy) and pale_bindings.cpp:1081-1395 (remove_points,
// add_new_points) edits the asset before rebuild_bvh.  Here the decisions
// and the edits run on the device asset:
//
// * compute_prune_indices_by_opacity (density_control.py:199-263): a stable
//   radix sort of the opacities gives the quantile threshold and, when more
//   surfels fall at or below it than may be pruned, the lowest ones;
//   remove_points is a stable compaction of the asset.
// * densify_points_long_axis_split (:6-196): candidates by long-axis scale
//   and importance, a stable sort by descending score when the budget binds,
//   the parents in increasing index order, two children per parent split
//   along the long axis; remove_points(parents) + add_points(children)
//   keep the survivors in order and append the children parent by parent.
#include "kernels.h"

namespace pale {

namespace {

inline uint32_t blocks_for(uint64_t n) { return (uint32_t)((n + kBlock - 1) / kBlock); }

// Order-preserving map of a float to an unsigned key (ascending).
__device__ __forceinline__ uint32_t float_key(float f) {
  const uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

__global__ void k_opacity_keys(const float* __restrict__ op, uint32_t n, uint32_t* __restrict__ keys,
                               uint32_t* __restrict__ vals) {
  const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
  if (i >= n) return;
  keys[i] = float_key(op[i]);
  vals[i] = i;
}

__global__ void k_count_le(const float* __restrict__ v, uint32_t n, float thr, uint32_t* __restrict__ count) {
  const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
  const uint32_t c = __syncthreads_count(i < n && v[i] <= thr);
  if (threadIdx.x == 0 && c) atomicAdd(count, c);
}

__global__ void k_fill(uint32_t* __restrict__ a, uint32_t n, uint32_t value) {
  const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
  if (i < n) a[i] = value;
}

// keep[idx[j]] = 0 for j < k (idx: distinct indices below n)
__global__ void k_mark(const uint32_t* __restrict__ idx, uint32_t k, uint32_t n, uint32_t* __restrict__ keep,
                       uint32_t value) {
  const uint32_t j = blockIdx.x * kBlock + threadIdx.x;
  if (j < k && idx[j] < n) keep[idx[j]] = value;
}

__device__ __forceinline__ void copy_point(const PointsDev& s, uint32_t i, const PointsDev& d, uint32_t o) {
  for (int c = 0; c < 3; ++c) {
    d.position[3 * (size_t)o + c] = s.position[3 * (size_t)i + c];
    d.tangent_u[3 * (size_t)o + c] = s.tangent_u[3 * (size_t)i + c];
    d.tangent_v[3 * (size_t)o + c] = s.tangent_v[3 * (size_t)i + c];
    d.albedo[3 * (size_t)o + c] = s.albedo[3 * (size_t)i + c];
  }
  d.scale[2 * (size_t)o] = s.scale[2 * (size_t)i];
  d.scale[2 * (size_t)o + 1] = s.scale[2 * (size_t)i + 1];
  d.opacity[o] = s.opacity[i];
  d.beta[o] = s.beta[i];
  d.shape[o] = s.shape[i];
}

__global__ void k_compact(PointsDev src, const uint32_t* __restrict__ keep, const uint32_t* __restrict__ dst,
                          uint32_t n, PointsDev out) {
  const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
  if (i < n && keep[i]) copy_point(src, i, out, dst[i]);
}

// list[dst[i]] = i where flag[i] (indices in increasing order)
__global__ void k_list(const uint32_t* __restrict__ flag, const uint32_t* __restrict__ dst, uint32_t n,
                       uint32_t* __restrict__ list) {
  const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
  if (i < n && flag[i]) list[dst[i]] = i;
}

// Candidates of the split: long axis max(s_u, s_v) >= min_long, then (with
// importance and grad_threshold > 0) score >= grad_threshold.  Sort key:
// descending score (importance, else the long-axis scale); non-candidates
// sort last.
__global__ void k_split_candidates(PointsDev a, uint32_t n, const float* __restrict__ importance, float min_long,
                                   float grad_threshold, int use_threshold, uint32_t* __restrict__ cand,
                                   uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
  if (i >= n) return;
  const float lng = fmaxf(a.scale[2 * (size_t)i], a.scale[2 * (size_t)i + 1]);
  bool c = lng >= min_long;
  float score = lng;
  if (importance) {
    score = importance[i];
    if (use_threshold) c = c && score >= grad_threshold;
  }
  cand[i] = c ? 1u : 0u;
  keys[i] = c ? ~float_key(score) : 0xFFFFFFFFu;
  vals[i] = i;
}

// Two children per parent (density_control.py:126-176), with the
// reference's arithmetic: the offset magnitude split * 3 * long in double,
// rounded to float before it scales the float32 axis; child scales and
// opacity in double, rounded to float; tangents, albedo and beta copied.
__global__ void k_split_children(PointsDev a, const uint32_t* __restrict__ parents, uint32_t np, uint32_t base,
                                 PointsDev out, double split, double shrink, double reduction) {
  const uint32_t j = blockIdx.x * kBlock + threadIdx.x;
  if (j >= np) return;
  const uint32_t p = parents[j];
  const float su = a.scale[2 * (size_t)p], sv = a.scale[2 * (size_t)p + 1];
  const bool long_u = su >= sv;
  const double lng = long_u ? su : sv, sht = long_u ? sv : su;
  const float* axis = long_u ? a.tangent_u : a.tangent_v;
  const float mag = (float)(split * (3.0 * lng));
  const float cl = (float)(lng * (1.0 - split)), cs = (float)(sht * shrink);
  double op = (double)a.opacity[p] * reduction;
  op = op < 0.0 ? 0.0 : (op > 1.0 ? 1.0 : op);
  for (int s = 0; s < 2; ++s) {
    const uint32_t o = base + 2 * j + s;
    copy_point(a, p, out, o);
    for (int c = 0; c < 3; ++c) {
      const float off = mag * axis[3 * (size_t)p + c];
      const float pc = a.position[3 * (size_t)p + c];
      out.position[3 * (size_t)o + c] = s == 0 ? pc + off : pc - off;
    }
    out.scale[2 * (size_t)o] = long_u ? cl : cs;
    out.scale[2 * (size_t)o + 1] = long_u ? cs : cl;
    out.opacity[o] = (float)op;
    out.shape[o] = 0.0f;
  }
}

}  // namespace

void opacity_sort_keys(const float* op, uint32_t n, uint32_t* keys, uint32_t* vals, cudaStream_t s) {
  if (!n) return;
  k_opacity_keys<<<blocks_for(n), kBlock, 0, s>>>(op, n, keys, vals); note_launch();
}

void count_le(const float* v, uint32_t n, float thr, uint32_t* count, cudaStream_t s) {
  cudaMemsetAsync(count, 0, sizeof(uint32_t), s);
  if (!n) return;
  k_count_le<<<blocks_for(n), kBlock, 0, s>>>(v, n, thr, count); note_launch();
}

void fill_u32(uint32_t* a, uint32_t n, uint32_t value, cudaStream_t s) {
  if (!n) return;
  k_fill<<<blocks_for(n), kBlock, 0, s>>>(a, n, value); note_launch();
}

void mark_indices(const uint32_t* idx, uint32_t k, uint32_t n, uint32_t* flags, uint32_t value, cudaStream_t s) {
  if (!k) return;
  k_mark<<<blocks_for(k), kBlock, 0, s>>>(idx, k, n, flags, value); note_launch();
}

void compact_points(const PointsDev& src, const uint32_t* keep, const uint32_t* dst, uint32_t n, const PointsDev& out,
                    cudaStream_t s) {
  if (!n) return;
  k_compact<<<blocks_for(n), kBlock, 0, s>>>(src, keep, dst, n, out); note_launch();
}

void flagged_list(const uint32_t* flag, const uint32_t* dst, uint32_t n, uint32_t* list, cudaStream_t s) {
  if (!n) return;
  k_list<<<blocks_for(n), kBlock, 0, s>>>(flag, dst, n, list); note_launch();
}

void split_candidates(const PointsDev& a, uint32_t n, const float* importance, float min_long, float grad_threshold,
                      int use_threshold, uint32_t* cand, uint32_t* keys, uint32_t* vals, cudaStream_t s) {
  if (!n) return;
  k_split_candidates<<<blocks_for(n), kBlock, 0, s>>>(a, n, importance, min_long, grad_threshold, use_threshold,
                                                      cand, keys, vals); note_launch();
}

void split_children(const PointsDev& a, const uint32_t* parents, uint32_t np, uint32_t base, const PointsDev& out,
                    double split, double shrink, double reduction, cudaStream_t s) {
  if (!np) return;
  k_split_children<<<blocks_for(np), kBlock, 0, s>>>(a, parents, np, base, out, split, shrink, reduction);
  note_launch();
}

}  // namespace pale
