// build.cu -- device-wide scan, stable radix sort and the surfel LBVH.
//
// The surfel BVH of the reference is a CPU median split rebuilt on every
// rebuild_bvh() (Pale/Renderer/BVH.ixx:49-133, SceneBuild.cpp:476-512).
// Here it is a Morton-code LBVH built on the device:
//   collect surfels (SceneBuild.cpp:203-215) and their beta AABBs
//   (SceneBuild.cpp:395-444) -> 30-bit Morton codes of the centres ->
//   stable LSD radix sort (ties keep index order) -> Karras topology ->
//   bottom-up box refit -> subtrees of <= leaf_size surfels become leaves ->
//   the first `top` nodes in breadth-first order are duplicated at the front
//   of the node array so the traversal can stage them in shared memory.
// Surfels are then permuted into leaf order, the order in which parameters
// and gradients are exchanged (SceneBuild.cpp:723-731).
#include <mutex>
#include <string>

#include "../../include/pale_b200.h"
#include "kernels.h"

namespace pale {

// ------------------------------------------------------------------ scan
constexpr int kScanThreads = 256;
constexpr int kScanItems = 32;
constexpr int kScanTile = kScanThreads * kScanItems;  // 8192 elements per block

__device__ __forceinline__ uint32_t block_exclusive_sum(uint32_t v, uint32_t* s_warp, uint32_t& total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_warp[wid] = x;
  __syncthreads();
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
    uint32_t w = lane < nw ? s_warp[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < nw) s_warp[lane] = w;
  }
  __syncthreads();
  uint32_t warp_prefix = wid > 0 ? s_warp[wid - 1] : 0u;
  total = s_warp[(blockDim.x >> 5) - 1];
  __syncthreads();
  return warp_prefix + x - v;
}

__global__ void k_scan_reduce(const uint32_t* __restrict__ in, uint32_t n, uint32_t* __restrict__ partial) {
  __shared__ uint32_t s_warp[32];
  const size_t base = (size_t)blockIdx.x * kScanTile;
  uint32_t sum = 0;
#pragma unroll 4
  for (int k = 0; k < kScanItems; ++k) {
    size_t i = base + (size_t)k * kScanThreads + threadIdx.x;
    if (i < n) sum += in[i];
  }
  uint32_t total;
  block_exclusive_sum(sum, s_warp, total);
  if (threadIdx.x == 0) partial[blockIdx.x] = total;
}

// Single block: exclusive scan of up to 1024*32 partial sums.
__global__ void __launch_bounds__(1024) k_scan_partials(uint32_t* __restrict__ partial, uint32_t nb,
                                                        uint32_t* __restrict__ total_out) {
  __shared__ uint32_t s_warp[32];
  const int items = 32;
  uint32_t sum = 0;
  const uint32_t base = threadIdx.x * items;
  for (int k = 0; k < items; ++k) {
    uint32_t i = base + k;
    sum += i < nb ? partial[i] : 0u;
  }
  uint32_t total;
  uint32_t run = block_exclusive_sum(sum, s_warp, total);
  // each thread rewrites only its own consecutive range
  for (int k = 0; k < items; ++k) {
    uint32_t i = base + k;
    if (i < nb) {
      uint32_t v = partial[i];
      partial[i] = run;
      run += v;
    }
  }
  if (threadIdx.x == 0 && total_out) *total_out = total;
}

__global__ void k_scan_apply(const uint32_t* __restrict__ in, uint32_t n, const uint32_t* __restrict__ partial,
                             uint32_t* __restrict__ out) {
  __shared__ uint32_t s_warp[32];
  const size_t base = (size_t)blockIdx.x * kScanTile;
  uint32_t carry = partial[blockIdx.x];
  for (int k = 0; k < kScanItems; ++k) {
    size_t i = base + (size_t)k * kScanThreads + threadIdx.x;
    uint32_t v = i < n ? in[i] : 0u;
    uint32_t total;
    uint32_t ex = block_exclusive_sum(v, s_warp, total);
    if (i < n) out[i] = carry + ex;
    carry += total;
  }
}

size_t scan_temp_words(uint32_t n) { return (size_t)(n + kScanTile - 1) / kScanTile + 1; }

void exclusive_scan(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* temp, uint32_t* total,
                    cudaStream_t s) {
  if (n == 0) return;
  uint32_t nb = (n + kScanTile - 1) / kScanTile;
  k_scan_reduce<<<nb, kScanThreads, 0, s>>>(in, n, temp); note_launch();
  k_scan_partials<<<1, 1024, 0, s>>>(temp, nb, total); note_launch();
  k_scan_apply<<<nb, kScanThreads, 0, s>>>(in, n, temp, out); note_launch();
}

// ------------------------------------------------------------ radix sort
// Stable LSD sort of (key, value) pairs, 8-bit digits.  Each block owns a
// tile of kSortTile keys; keys in a tile keep their order (rank = keys of
// the same digit in earlier rounds, earlier warps, lower lanes).
constexpr int kSortThreads = 256;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;

__global__ void k_radix_hist(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ d_n, uint32_t shift,
                             uint32_t tiles, uint32_t* __restrict__ hist) {
  __shared__ uint32_t s_cnt[256];
  s_cnt[threadIdx.x] = 0;
  __syncthreads();
  const uint32_t n = *d_n;
  const size_t base = (size_t)blockIdx.x * kSortTile;
#pragma unroll
  for (int k = 0; k < kSortItems; ++k) {
    size_t i = base + (size_t)k * kSortThreads + threadIdx.x;
    if (i < n) atomicAdd(&s_cnt[(keys[i] >> shift) & 255u], 1u);
  }
  __syncthreads();
  hist[(size_t)threadIdx.x * tiles + blockIdx.x] = s_cnt[threadIdx.x];
}

__global__ void k_radix_scatter(const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
                                const uint32_t* __restrict__ d_n, uint32_t shift, uint32_t tiles,
                                const uint32_t* __restrict__ offsets, uint32_t* __restrict__ keys_out,
                                uint32_t* __restrict__ vals_out) {
  constexpr int kWarps = kSortThreads / 32;
  __shared__ uint32_t s_run[256];
  __shared__ uint32_t s_wcnt[kWarps][256];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const uint32_t n = *d_n;
  s_run[threadIdx.x] = offsets[(size_t)threadIdx.x * tiles + blockIdx.x];
  const size_t base = (size_t)blockIdx.x * kSortTile;
  for (int k = 0; k < kSortItems; ++k) {
    for (int w = 0; w < kWarps; ++w) s_wcnt[w][threadIdx.x] = 0;
    __syncthreads();
    size_t i = base + (size_t)k * kSortThreads + threadIdx.x;
    bool valid = i < n;
    uint32_t key = valid ? keys_in[i] : 0u;
    uint32_t val = valid ? vals_in[i] : 0u;
    uint32_t digit = valid ? ((key >> shift) & 255u) : 256u + (uint32_t)lane;  // unique sentinel per lane
    unsigned peers = __match_any_sync(0xffffffffu, digit);
    unsigned lt = (1u << lane) - 1u;
    uint32_t rank_in_warp = __popc(peers & lt);
    if (valid && rank_in_warp == 0) s_wcnt[wid][digit] = __popc(peers);
    __syncthreads();
    if (valid) {
      uint32_t before = 0;
      for (int w = 0; w < wid; ++w) before += s_wcnt[w][digit];
      uint32_t dst = s_run[digit] + before + rank_in_warp;
      keys_out[dst] = key;
      vals_out[dst] = val;
    }
    __syncthreads();
    uint32_t add = 0;
    for (int w = 0; w < kWarps; ++w) add += s_wcnt[w][threadIdx.x];
    s_run[threadIdx.x] += add;
    __syncthreads();
  }
}

size_t radix_temp_words(uint32_t n_max) {
  uint32_t tiles = (n_max + kSortTile - 1) / kSortTile;
  size_t h = (size_t)tiles * 256 + 1;
  return 2 * h + scan_temp_words((uint32_t)h) + 8;
}

// Sorts (keys, vals) in place; key bits >= `bits` must be zero.
// keys_tmp / vals_tmp are ping-pong buffers of n_max entries.
void radix_sort_pairs(uint32_t* keys, uint32_t* vals, uint32_t* keys_tmp, uint32_t* vals_tmp,
                      const uint32_t* d_n, uint32_t n_max, int bits, uint32_t* temp, cudaStream_t s) {
  if (n_max == 0) return;
  const uint32_t tiles = (n_max + kSortTile - 1) / kSortTile;
  const size_t h = (size_t)tiles * 256;
  uint32_t* hist = temp;
  uint32_t* offs = temp + h + 1;
  uint32_t* stemp = offs + h + 1;
  int passes = (bits + 7) / 8;
  uint32_t *ka = keys, *va = vals, *kb = keys_tmp, *vb = vals_tmp;
  for (int p = 0; p < passes; ++p) {
    uint32_t shift = 8u * p;
    k_radix_hist<<<tiles, kSortThreads, 0, s>>>(ka, d_n, shift, tiles, hist); note_launch();
    exclusive_scan(hist, offs, (uint32_t)h, stemp, nullptr, s);
    k_radix_scatter<<<tiles, kSortThreads, 0, s>>>(ka, va, d_n, shift, tiles, offs, kb, vb); note_launch();
    uint32_t* t = ka; ka = kb; kb = t;
    t = va; va = vb; vb = t;
  }
  if (passes & 1) {
    cudaMemcpyAsync(keys, ka, (size_t)n_max * 4, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(vals, va, (size_t)n_max * 4, cudaMemcpyDeviceToDevice, s);
  }
}

// --------------------------------------------------------- surfel prepare
__device__ __forceinline__ V3 ld3(const float* p, uint32_t i) { return v3(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }
__device__ __forceinline__ void st3(float* p, uint32_t i, V3 a) {
  p[3 * i] = a.x;
  p[3 * i + 1] = a.y;
  p[3 * i + 2] = a.z;
}

// collectPointCloudGeometry (SceneBuild.cpp:203-215) + surfelObjectAabbBeta
// (SceneBuild.cpp:395-444), asset order.
__global__ void k_collect(PointsDev asset, uint32_t n, PointsDev col, float* __restrict__ lo,
                          float* __restrict__ hi) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  V3 p = ld3(asset.position, i);
  V3 tu = normalize(ld3(asset.tangent_u, i));
  V3 tv = normalize(ld3(asset.tangent_v, i));
  V3 al = ld3(asset.albedo, i);
  float su = asset.scale[2 * i], sv = asset.scale[2 * i + 1];
  st3(col.position, i, p);
  st3(col.tangent_u, i, tu);
  st3(col.tangent_v, i, tv);
  col.scale[2 * i] = su;
  col.scale[2 * i + 1] = sv;
  st3(col.albedo, i, v3(clampf(al.x, 0.f, 1.f), clampf(al.y, 0.f, 1.f), clampf(al.z, 0.f, 1.f)));
  col.opacity[i] = clampf(asset.opacity[i], 0.f, 1.f);
  col.beta[i] = asset.beta[i];
  col.shape[i] = asset.shape ? clampf(asset.shape[i], -5.f, 5.f) : 0.f;
  // beta-kernel AABB
  V3 tU = normalize(tu), tV = normalize(tv);
  V3 nn = normalize(cross(tU, tV));
  float rU = 1.0001f * su, rV = 1.0001f * sv;
  float e[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    float cu = rU * comp(tU, a), cv = rV * comp(tV, a);
    float proj = sqrtf(cu * cu + cv * cv);
    e[a] = proj + 0.001f * fabsf(comp(nn, a));
  }
  V3 ext = v3(e[0], e[1], e[2]);
  st3(lo, i, p - ext);
  st3(hi, i, p + ext);
}

// Min/max of positions and of boxes: per-block partials, then one block.
__global__ void k_bounds_partial(const float* __restrict__ pos, const float* __restrict__ lo,
                                 const float* __restrict__ hi, uint32_t n, float* __restrict__ part) {
  __shared__ float s[12][kBlock];
  float acc[12];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    acc[k] = __int_as_float(0x7f800000);
    acc[3 + k] = -__int_as_float(0x7f800000);
    acc[6 + k] = __int_as_float(0x7f800000);
    acc[9 + k] = -__int_as_float(0x7f800000);
  }
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      acc[k] = fminf(acc[k], pos[3 * i + k]);
      acc[3 + k] = fmaxf(acc[3 + k], pos[3 * i + k]);
      acc[6 + k] = fminf(acc[6 + k], lo[3 * i + k]);
      acc[9 + k] = fmaxf(acc[9 + k], hi[3 * i + k]);
    }
  }
#pragma unroll
  for (int k = 0; k < 12; ++k) s[k][threadIdx.x] = acc[k];
  __syncthreads();
  if (threadIdx.x < 12) {
    int k = threadIdx.x;
    bool is_min = (k < 3) || (k >= 6 && k < 9);
    float r = s[k][0];
    for (int t = 1; t < kBlock; ++t) r = is_min ? fminf(r, s[k][t]) : fmaxf(r, s[k][t]);
    part[12 * blockIdx.x + k] = r;
  }
}
__global__ void k_bounds_final(const float* __restrict__ part, uint32_t nb, float* __restrict__ out) {
  int k = threadIdx.x;
  if (k >= 12) return;
  bool is_min = (k < 3) || (k >= 6 && k < 9);
  float r = part[k];
  for (uint32_t b = 1; b < nb; ++b) r = is_min ? fminf(r, part[12 * b + k]) : fmaxf(r, part[12 * b + k]);
  out[k] = r;
}

// Morton expandBits (Karras 2012).
__device__ __forceinline__ uint32_t expand_bits(uint32_t v) {
  v = (v * 0x00010001u) & 0xFF0000FFu;
  v = (v * 0x00000101u) & 0x0F00F00Fu;
  v = (v * 0x00000011u) & 0xC30C30C3u;
  v = (v * 0x00000005u) & 0x49249249u;
  return v;
}
__device__ __forceinline__ uint32_t quantize(float c, float lo, float ext) {
  float f = (ext > 0.f) ? __fdiv_rn(__fsub_rn(c, lo), ext) : 0.f;
  float q = __fmul_rn(f, 1024.0f);
  if (!(q > 0.f)) return 0u;
  if (q >= 1023.f) return 1023u;
  return (uint32_t)q;
}
__global__ void k_morton(const float* __restrict__ pos, uint32_t n, const float* __restrict__ bounds,
                         uint32_t* __restrict__ codes, uint32_t* __restrict__ idx) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float lx = bounds[0], ly = bounds[1], lz = bounds[2];
  float ex = __fsub_rn(bounds[3], lx), ey = __fsub_rn(bounds[4], ly), ez = __fsub_rn(bounds[5], lz);
  codes[i] = (expand_bits(quantize(pos[3 * i], lx, ex)) << 2) | (expand_bits(quantize(pos[3 * i + 1], ly, ey)) << 1) |
             expand_bits(quantize(pos[3 * i + 2], lz, ez));
  idx[i] = i;
}

// --------------------------------------------------------- Karras topology
__device__ __forceinline__ int delta_key(const uint32_t* __restrict__ codes, uint32_t n, int64_t i, int64_t j) {
  if (j < 0 || j >= (int64_t)n) return -1;
  uint64_t ki = ((uint64_t)codes[i] << 32) | (uint64_t)i;
  uint64_t kj = ((uint64_t)codes[j] << 32) | (uint64_t)j;
  return __clzll((long long)(ki ^ kj));
}

// Internal node i of Karras, "Maximizing parallelism in the construction of
// BVHs, octrees and k-d trees" (HPG 2012), over sorted codes with the
// sorted position appended as tie breaker.  Children: >= 0 internal,
// < 0 leaf -(k+1).
__global__ void k_karras(const uint32_t* __restrict__ codes, uint32_t n, int32_t* __restrict__ lc,
                         int32_t* __restrict__ rc, uint32_t* __restrict__ rfirst, uint32_t* __restrict__ rlast,
                         uint32_t* __restrict__ parent, uint32_t* __restrict__ leaf_parent, uint32_t* err) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)n - 1) return;
  int d = (delta_key(codes, n, i, i + 1) - delta_key(codes, n, i, i - 1)) >= 0 ? 1 : -1;
  int dmin = delta_key(codes, n, i, i - d);
  int64_t lmax = 2;
  for (int it = 0; it < 40 && delta_key(codes, n, i, i + lmax * d) > dmin; ++it) lmax *= 2;
  int64_t l = 0;
  for (int64_t t = lmax / 2; t >= 1; t /= 2)
    if (delta_key(codes, n, i, i + (l + t) * d) > dmin) l += t;
  // sorted, distinct keys give l >= 1; anything else is a sort failure
  if (l < 1 || i + l * d < 0 || i + l * d >= (int64_t)n) {
    atomicOr(err, kErrBounds);
    l = 1;
    d = (i + 1 < (int64_t)n) ? 1 : -1;
  }
  int64_t j = i + l * d;
  int dnode = delta_key(codes, n, i, j);
  int64_t s = 0, div = 2, t = (l + div - 1) / div;
  for (int it = 0; it < 64; ++it) {
    if (delta_key(codes, n, i, i + (s + t) * d) > dnode) s += t;
    if (t <= 1) break;
    div *= 2;
    t = (l + div - 1) / div;
  }
  int64_t gamma = i + s * d + (d < 0 ? d : 0);
  int64_t mn = i < j ? i : j, mx = i < j ? j : i;
  if (gamma < mn || gamma >= mx) {
    atomicOr(err, kErrBounds);
    gamma = mn;
  }
  int32_t L = (mn == gamma) ? -(int32_t)(gamma + 1) : (int32_t)gamma;
  int32_t R = (mx == gamma + 1) ? -(int32_t)(gamma + 2) : (int32_t)(gamma + 1);
  lc[i] = L;
  rc[i] = R;
  rfirst[i] = (uint32_t)mn;
  rlast[i] = (uint32_t)mx;
  if (L >= 0) parent[L] = (uint32_t)i; else leaf_parent[-L - 1] = (uint32_t)i;
  if (R >= 0) parent[R] = (uint32_t)i; else leaf_parent[-R - 1] = (uint32_t)i;
}

// Bottom-up refit: the second thread to reach a node computes its box.
// Box unions are exact, so the result does not depend on arrival order.
__global__ void k_refit(const uint32_t* __restrict__ order, uint32_t n, const float* __restrict__ lo,
                        const float* __restrict__ hi, const int32_t* __restrict__ lc, const int32_t* __restrict__ rc,
                        const uint32_t* __restrict__ parent, const uint32_t* __restrict__ leaf_parent,
                        uint32_t* __restrict__ visits, float* box) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t p = leaf_parent[i];
  for (uint32_t guard = 0; guard < 128u; ++guard) {
    __threadfence();
    if (atomicAdd(&visits[p], 1u) == 0u) return;
    __threadfence();
    float b[2][6];
    int32_t ch[2] = {lc[p], rc[p]};
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      if (ch[c] < 0) {
        uint32_t k = order[-ch[c] - 1];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          b[c][a] = lo[3 * k + a];
          b[c][3 + a] = hi[3 * k + a];
        }
      } else {
        const volatile float* src = box + 6 * (size_t)ch[c];
#pragma unroll
        for (int a = 0; a < 6; ++a) b[c][a] = src[a];
      }
    }
    volatile float* dst = box + 6 * (size_t)p;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      dst[a] = fminf(b[0][a], b[1][a]);
      dst[3 + a] = fmaxf(b[0][3 + a], b[1][3 + a]);
    }
    if (p == 0) return;
    p = parent[p];
  }
}

__device__ __forceinline__ uint32_t leaf_word(uint32_t first, uint32_t count) {
  return kLeafFlag | ((count - 1u) << 28) | first;
}

__device__ __forceinline__ void put_child(float* w, int c, const float* b) {
#pragma unroll
  for (int a = 0; a < 6; ++a) w[6 * c + a] = b[a];
}

// Traversal node of Karras node x, stored at slot top + x.
__global__ void k_emit_nodes(const uint32_t* __restrict__ order, uint32_t n, const float* __restrict__ lo,
                             const float* __restrict__ hi, const int32_t* __restrict__ lc,
                             const int32_t* __restrict__ rc, const uint32_t* __restrict__ rfirst,
                             const uint32_t* __restrict__ rlast, const float* __restrict__ box, uint32_t leaf_size,
                             uint32_t top, BvhNode* __restrict__ nodes) {
  uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= n - 1) return;
  float w[16];
  uint32_t words[2];
  int32_t ch[2] = {lc[x], rc[x]};
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    float b[6];
    if (ch[c] < 0) {
      uint32_t sp = (uint32_t)(-ch[c] - 1);
      uint32_t k = order[sp];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        b[a] = lo[3 * k + a];
        b[3 + a] = hi[3 * k + a];
      }
      words[c] = leaf_word(sp, 1);
    } else {
      uint32_t y = (uint32_t)ch[c];
#pragma unroll
      for (int a = 0; a < 6; ++a) b[a] = box[6 * (size_t)y + a];
      uint32_t cnt = rlast[y] - rfirst[y] + 1u;
      words[c] = cnt <= leaf_size ? leaf_word(rfirst[y], cnt) : top + y;
    }
    put_child(w, c, b);
  }
  BvhNode nd;
  nd.a = make_float4(w[0], w[1], w[2], w[3]);
  nd.b = make_float4(w[4], w[5], w[6], w[7]);
  nd.c = make_float4(w[8], w[9], w[10], w[11]);
  nd.d = make_uint4(words[0], words[1], 0u, 0u);
  nodes[top + x] = nd;
}

// Breadth-first copy of the first `top` kept nodes into slots [0, top).
__global__ void k_top_nodes(const uint32_t* __restrict__ rfirst, const uint32_t* __restrict__ rlast, uint32_t n,
                            uint32_t leaf_size, uint32_t top, BvhNode* __restrict__ nodes) {
  extern __shared__ uint32_t s_top[];   // [top] source Karras index, [top] map
  uint32_t* src = s_top;
  __shared__ uint32_t s_count;
  if (threadIdx.x == 0) {
    uint32_t cnt = 0, head = 0;
    if (top > 0) src[cnt++] = 0;
    while (head < cnt) {
      uint32_t x = src[head++];
      BvhNode nd = nodes[top + x];
      uint32_t ws[2] = {nd.d.x, nd.d.y};
      for (int c = 0; c < 2; ++c) {
        uint32_t wd = ws[c];
        if (wd == kEmptyChild || (wd & kLeafFlag)) continue;
        uint32_t y = wd - top;
        if (rlast[y] - rfirst[y] + 1u <= leaf_size) continue;
        if (cnt >= top) continue;
        src[cnt++] = y;
      }
    }
    s_count = cnt;
  }
  __syncthreads();
  const uint32_t cnt = s_count;
  for (uint32_t k = threadIdx.x; k < top; k += blockDim.x) {
    if (k >= cnt) {
      BvhNode z;
      z.a = z.b = z.c = make_float4(0.f, 0.f, 0.f, 0.f);
      z.d = make_uint4(kEmptyChild, kEmptyChild, 0u, 0u);
      nodes[k] = z;
      continue;
    }
    BvhNode nd = nodes[top + src[k]];
    uint32_t ws[2] = {nd.d.x, nd.d.y};
    for (int c = 0; c < 2; ++c) {
      uint32_t wd = ws[c];
      if (wd == kEmptyChild || (wd & kLeafFlag)) continue;
      uint32_t y = wd - top;
      for (uint32_t m = 0; m < cnt; ++m)
        if (src[m] == y) { ws[c] = m; break; }
    }
    nd.d.x = ws[0];
    nd.d.y = ws[1];
    nodes[k] = nd;
  }
}

// One root node holding a single leaf of all n <= leaf_size surfels.
__global__ void k_small_root(const uint32_t* __restrict__ order, uint32_t n, const float* __restrict__ lo,
                             const float* __restrict__ hi, BvhNode* __restrict__ nodes) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  float b[6] = {__int_as_float(0x7f800000), __int_as_float(0x7f800000), __int_as_float(0x7f800000),
                -__int_as_float(0x7f800000), -__int_as_float(0x7f800000), -__int_as_float(0x7f800000)};
  for (uint32_t i = 0; i < n; ++i) {
    uint32_t k = order[i];
    for (int a = 0; a < 3; ++a) {
      b[a] = fminf(b[a], lo[3 * k + a]);
      b[3 + a] = fmaxf(b[3 + a], hi[3 * k + a]);
    }
  }
  BvhNode nd;
  const float inf = __int_as_float(0x7f800000);
  nd.a = make_float4(b[0], b[1], b[2], b[3]);
  nd.b = make_float4(b[4], b[5], inf, inf);
  nd.c = make_float4(inf, -inf, -inf, -inf);
  nd.d = make_uint4(leaf_word(0, n), kEmptyChild, 0u, 0u);
  nodes[0] = nd;
}

// Derived per-surfel arrays (BVH order) from the stored parameters: the
// intersection frame of intersectSurfel (KernelHelpers.h:637-669) and the
// canonical normal of buildIntersectionNormal (:497-502).
__global__ void k_derive(PointsDev p, uint32_t n, float4* __restrict__ pe, float4* __restrict__ nn,
                         float4* __restrict__ uu, float4* __restrict__ vv, float4* __restrict__ cn,
                         float4* __restrict__ alb) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  V3 pos = ld3(p.position, i), tu = ld3(p.tangent_u, i), tv = ld3(p.tangent_v, i);
  V3 uT = normalize(tu);
  V3 vT = normalize(tv - scale(uT, dot(uT, tv)));
  V3 nrm = normalize(cross(uT, vT));
  float beta = p.beta[i];
  pe[i] = f4(pos, 4.0f * expf(beta));
  nn[i] = f4(nrm, p.opacity[i]);
  uu[i] = f4(tu, p.scale[2 * i]);
  vv[i] = f4(tv, p.scale[2 * i + 1]);
  cn[i] = f4(normalize(cross(tu, tv)), beta);
  alb[i] = f4(ld3(p.albedo, i), 1.0f);
}

// Gathers asset-order collected parameters into BVH order.
__global__ void k_permute(PointsDev col, const uint32_t* __restrict__ order, uint32_t n, PointsDev out) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t k = order[i];
  st3(out.position, i, ld3(col.position, k));
  st3(out.tangent_u, i, ld3(col.tangent_u, k));
  st3(out.tangent_v, i, ld3(col.tangent_v, k));
  out.scale[2 * i] = col.scale[2 * k];
  out.scale[2 * i + 1] = col.scale[2 * k + 1];
  st3(out.albedo, i, ld3(col.albedo, k));
  out.opacity[i] = col.opacity[k];
  out.beta[i] = col.beta[k];
  out.shape[i] = col.shape[k];
}

static inline uint32_t blocks_for(uint64_t n, int b = kBlock) { return (uint32_t)((n + b - 1) / b); }

void lbvh_build(const LbvhArgs& A, cudaStream_t s) {
  const uint32_t n = A.n;
  if (n == 0) return;
  k_collect<<<blocks_for(n), kBlock, 0, s>>>(A.asset, n, A.collected, A.lo, A.hi); note_launch();
  uint32_t nb = blocks_for(n) < 148u * 4u ? blocks_for(n) : 148u * 4u;
  k_bounds_partial<<<nb, kBlock, 0, s>>>(A.collected.position, A.lo, A.hi, n, A.bounds_part); note_launch();
  k_bounds_final<<<1, 32, 0, s>>>(A.bounds_part, nb, A.bounds); note_launch();
  k_morton<<<blocks_for(n), kBlock, 0, s>>>(A.collected.position, n, A.bounds, A.codes, A.order); note_launch();
  radix_sort_pairs(A.codes, A.order, A.codes_tmp, A.order_tmp, A.d_n, n, 30, A.sort_temp, s);
  if (n <= A.leaf_size) {
    k_small_root<<<1, 32, 0, s>>>(A.order, n, A.lo, A.hi, A.nodes); note_launch();
  } else {
    k_karras<<<blocks_for(n - 1), kBlock, 0, s>>>(A.codes, n, A.lc, A.rc, A.rfirst, A.rlast, A.parent,
                                                  A.leaf_parent, A.err); note_launch();
    cudaMemsetAsync(A.visits, 0, (size_t)(n - 1) * 4, s);
    k_refit<<<blocks_for(n), kBlock, 0, s>>>(A.order, n, A.lo, A.hi, A.lc, A.rc, A.parent, A.leaf_parent, A.visits,
                                             A.box); note_launch();
    k_emit_nodes<<<blocks_for(n - 1), kBlock, 0, s>>>(A.order, n, A.lo, A.hi, A.lc, A.rc, A.rfirst, A.rlast, A.box,
                                                      A.leaf_size, A.top, A.nodes); note_launch();
    if (A.top > 0)
      k_top_nodes<<<1, kBlock, A.top * sizeof(uint32_t), s>>>(A.rfirst, A.rlast, n, A.leaf_size, A.top, A.nodes); note_launch();
  }
  k_permute<<<blocks_for(n), kBlock, 0, s>>>(A.collected, A.order, n, A.params); note_launch();
  derive_surfels(A.params, n, A.derived, s);
}

namespace {
__device__ __forceinline__ uint32_t pack_down(float a, float b) {
  const __half2 h = __halves2half2(__float2half_rd(a), __float2half_rd(b));
  return *reinterpret_cast<const uint32_t*>(&h);
}
__device__ __forceinline__ uint32_t pack_up(float a, float b) {
  const __half2 h = __halves2half2(__float2half_ru(a), __float2half_ru(b));
  return *reinterpret_cast<const uint32_t*>(&h);
}
// mixed pair: first value a lower bound (down), second an upper bound (up)
__device__ __forceinline__ uint32_t pack_down_up(float a, float b) {
  const __half2 h = __halves2half2(__float2half_rd(a), __float2half_ru(b));
  return *reinterpret_cast<const uint32_t*>(&h);
}

__global__ void k_half_nodes(const BvhNode* __restrict__ in, uint32_t n, BvhNodeH* __restrict__ out) {
  const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
  if (i >= n) return;
  const BvhNode nd = in[i];
  // a = c0.lo.xyz c0.hi.x, b = c0.hi.yz c1.lo.xy, c = c1.lo.z c1.hi.xyz
  BvhNodeH h;
  h.q0 = make_uint4(pack_down(nd.a.x, nd.a.y), pack_down_up(nd.a.z, nd.a.w), pack_up(nd.b.x, nd.b.y),
                    pack_down(nd.b.z, nd.b.w));
  h.q1 = make_uint4(pack_down_up(nd.c.x, nd.c.y), pack_up(nd.c.z, nd.c.w), nd.d.x, nd.d.y);
  out[i] = h;
}
}  // namespace

void half_nodes(const BvhNode* in, uint32_t n, BvhNodeH* out, cudaStream_t s) {
  if (n == 0) return;
  k_half_nodes<<<blocks_for(n), kBlock, 0, s>>>(in, n, out); note_launch();
}

void derive_surfels(const PointsDev& p, uint32_t n, const SurfelArrays& d, cudaStream_t s) {
  if (n == 0) return;
  k_derive<<<blocks_for(n), kBlock, 0, s>>>(p, n, d.pe, d.n, d.u, d.v, d.cn, d.alb); note_launch();
}

// ------------------------------------------- LBVH build without allocation
// Some callers cannot allocate device memory around a call: code that runs
// while a CUDA graph is being captured (cudaMalloc is not capturable), host
// applications that own all device memory through their own allocator and
// forbid the runtime allocator, and latency-critical loops that cannot
// afford cudaMalloc's implicit device synchronisation.  For them the LBVH
// build is also offered with all of its temporaries in this file-scope
// device array.  Every GPU that loads the library holds the array until the
// process exits; every call shares it, so calls that overlap on the GPU race.
constexpr uint32_t kNoAllocMax = PALE_NOALLOC_MAX_SURFELS;
constexpr uint32_t kNoAllocTiles = (kNoAllocMax + kSortTile - 1) / kSortTile;
constexpr size_t kNoAllocSortWords = 2 * ((size_t)kNoAllocTiles * 256 + 1) +
                                     ((size_t)kNoAllocTiles * 256 + 1 + kScanTile - 1) / kScanTile + 1 + 8;
constexpr size_t kNoAllocWords = 17 * (size_t)kNoAllocMax   // collected parameters
                                 + 3 * (size_t)kNoAllocMax  // dummy albedo / opacity / beta inputs
                                 + 6 * (size_t)kNoAllocMax  // boxes lo, hi
                                 + 2 * (size_t)kNoAllocMax  // sort ping-pong
                                 + 7 * (size_t)kNoAllocMax  // topology
                                 + 6 * (size_t)kNoAllocMax  // node boxes
                                 + kNoAllocSortWords + 12 * 592 + 12 + 8;
static __device__ __align__(256) uint32_t g_lbvh_scratch[kNoAllocWords];

__global__ void k_set_words(uint32_t* p, uint32_t n, uint32_t a, uint32_t b) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    p[0] = n;
    p[1] = a;
    (void)b;
  }
}

namespace {
std::mutex g_scratch_mu;
void* g_scratch_addr[128] = {};

// Device address of g_lbvh_scratch on the current device, looked up once
// per device (the host-side symbol is not a device address).  The cached
// address belongs to the device's primary context: after cudaDeviceReset
// the module is loaded again and the address must not be reused, so a
// process that resets a device must not call this entry point afterwards.
cudaError_t scratch_address(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 128) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_lbvh_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return cudaSuccess;
}
}  // namespace

}  // namespace pale

extern "C" uint32_t pale_lbvh_node_count(uint32_t n, uint32_t leaf_size) {
  const uint32_t leaf = leaf_size < 1 ? 1u : (leaf_size > 8 ? 8u : leaf_size);
  if (n == 0) return 0;
  return n <= leaf ? 1u : pale::kTopNodes + n - 1;
}

extern "C" int pale_build_lbvh_noalloc(const float* d_position, const float* d_tangent_u, const float* d_tangent_v,
                                       const float* d_scale, uint32_t n, uint32_t leaf_size, uint32_t* d_codes,
                                       uint32_t* d_order, float* d_nodes, uint32_t* d_status, void* stream) {
  using namespace pale;
  if (n > kNoAllocMax) {
    set_thread_error("pale_build_lbvh_noalloc: " + std::to_string(n) + " surfels exceed the fixed maximum of " +
                     std::to_string(kNoAllocMax));
    return PALE_ERR_ARGUMENT;
  }
  if (n == 0) {
    // nothing to build; a caller-supplied status word still reads 0
    if (d_status && cudaMemsetAsync(d_status, 0, 4, (cudaStream_t)stream) != cudaSuccess) {
      set_thread_error("pale_build_lbvh_noalloc: clearing the status word failed");
      return PALE_ERR_CUDA;
    }
    return PALE_OK;
  }
  if (!d_position || !d_tangent_u || !d_tangent_v || !d_scale || !d_codes || !d_order || !d_nodes) {
    set_thread_error("pale_build_lbvh_noalloc: null device pointer");
    return PALE_ERR_ARGUMENT;
  }
  void* base = nullptr;
  cudaError_t e = scratch_address(&base);
  if (e != cudaSuccess) {
    set_thread_error(std::string("pale_build_lbvh_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
    return PALE_ERR_CUDA;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const uint32_t N = kNoAllocMax;
  uint32_t* w = static_cast<uint32_t*>(base);
  auto take = [&](size_t words) {
    uint32_t* p = w;
    w += words;
    return p;
  };
  float* f_col = reinterpret_cast<float*>(take(17ull * N));
  float* f_dummy = reinterpret_cast<float*>(take(3ull * N));
  float* lo = reinterpret_cast<float*>(take(3ull * N));
  float* hi = reinterpret_cast<float*>(take(3ull * N));
  uint32_t* codes_tmp = take(N);
  uint32_t* order_tmp = take(N);
  int32_t* lc = reinterpret_cast<int32_t*>(take(N));
  int32_t* rc = reinterpret_cast<int32_t*>(take(N));
  uint32_t* rfirst = take(N);
  uint32_t* rlast = take(N);
  uint32_t* parent = take(N);
  uint32_t* leaf_parent = take(N);
  uint32_t* visits = take(N);
  float* box = reinterpret_cast<float*>(take(6ull * N));
  uint32_t* sort_temp = take(kNoAllocSortWords);
  float* bounds_part = reinterpret_cast<float*>(take(12 * 592));
  float* bounds = reinterpret_cast<float*>(take(12));
  uint32_t* words = take(8);   // [0] n for the radix sort, [1] error flags
  uint32_t* err = d_status ? d_status : words + 1;

  PointsDev asset{const_cast<float*>(d_position), const_cast<float*>(d_tangent_u), const_cast<float*>(d_tangent_v),
                  const_cast<float*>(d_scale), f_dummy, f_dummy + N, f_dummy + 2 * N, nullptr};
  PointsDev col{f_col, f_col + 3 * N, f_col + 6 * N, f_col + 9 * N, f_col + 11 * N, f_col + 14 * N, f_col + 15 * N,
                f_col + 16 * N};
  const uint32_t leaf = leaf_size < 1 ? 1u : (leaf_size > 8 ? 8u : leaf_size);
  const uint32_t top = kTopNodes;   // the same staged top as pale_create's build
  // zero what must start at zero: the error word and the refit counters
  cudaMemsetAsync(err, 0, 4, s);
  cudaMemsetAsync(f_dummy, 0, 12ull * N, s);
  k_set_words<<<1, 32, 0, s>>>(words, n, 0u, 0u);
  k_collect<<<blocks_for(n), kBlock, 0, s>>>(asset, n, col, lo, hi);
  uint32_t nb = blocks_for(n) < 148u * 4u ? blocks_for(n) : 148u * 4u;
  k_bounds_partial<<<nb, kBlock, 0, s>>>(col.position, lo, hi, n, bounds_part);
  k_bounds_final<<<1, 32, 0, s>>>(bounds_part, nb, bounds);
  k_morton<<<blocks_for(n), kBlock, 0, s>>>(col.position, n, bounds, d_codes, d_order);
  radix_sort_pairs(d_codes, d_order, codes_tmp, order_tmp, words, n, 30, sort_temp, s);
  if (n <= leaf) {
    k_small_root<<<1, 32, 0, s>>>(d_order, n, lo, hi, reinterpret_cast<BvhNode*>(d_nodes));
  } else {
    BvhNode* nodes = reinterpret_cast<BvhNode*>(d_nodes);
    k_karras<<<blocks_for(n - 1), kBlock, 0, s>>>(d_codes, n, lc, rc, rfirst, rlast, parent, leaf_parent, err);
    cudaMemsetAsync(visits, 0, (size_t)(n - 1) * 4, s);
    k_refit<<<blocks_for(n), kBlock, 0, s>>>(d_order, n, lo, hi, lc, rc, parent, leaf_parent, visits, box);
    k_emit_nodes<<<blocks_for(n - 1), kBlock, 0, s>>>(d_order, n, lo, hi, lc, rc, rfirst, rlast, box, leaf, top, nodes);
    k_top_nodes<<<1, kBlock, top * sizeof(uint32_t), s>>>(rfirst, rlast, n, leaf, top, nodes);
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_thread_error(std::string("pale_build_lbvh_noalloc: launch failed: ") + cudaGetErrorString(e));
    return PALE_ERR_CUDA;
  }
  return PALE_OK;
}
