// common.cuh -- device math, RNG and data layouts of the B200 surfel renderer.
//
// Vector arithmetic keeps the evaluation order of Pale's float3 helpers
// (Pale/Renderer/GPUDataTypes.h:230-330): vector / scalar multiplies by the
// reciprocal, normalize() multiplies by 1/sqrt(sum of squares), dot products
// accumulate x, y, z in order.  The library is compiled with -fmad=false so
// that these expressions round exactly like the host restatement; the
// transcendental functions (expf, powf, sinf, cosf) are CUDA's.
#pragma once

#include <cstdint>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

namespace pale {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kInvPi = 0.318309886183790671538f;
constexpr uint32_t kInvalid = 0xFFFFFFFFu;
constexpr uint32_t kLeafFlag = 0x80000000u;
constexpr uint32_t kEmptyChild = 0xFFFFFFFFu;
constexpr int kBlock = 256;          // threads per block of the per-slot kernels
constexpr int kStackDepth = 64;      // BVH traversal stack entries
constexpr int kMaxLayers = 4096;     // camera-gather layer cap per ray

// Error bits reported through RunState::error.
enum : uint32_t {
  kErrStackOverflow = 1u << 0,
  kErrLayerCap = 1u << 1,
  kErrPhotonCapacity = 1u << 2,
  kErrBounds = 1u << 3,
  kErrQueueCapacity = 1u << 4,
};

// ------------------------------------------------------------------ math
struct V3 {
  float x, y, z;
};
__host__ __device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__host__ __device__ __forceinline__ V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__host__ __device__ __forceinline__ V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__host__ __device__ __forceinline__ V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }
__host__ __device__ __forceinline__ V3 mul(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
__host__ __device__ __forceinline__ V3 scale(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
__host__ __device__ __forceinline__ V3 divs(V3 a, float s) {
  float inv = 1.f / s;
  return v3(a.x * inv, a.y * inv, a.z * inv);
}
__host__ __device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ __forceinline__ V3 cross(V3 a, V3 b) {
  return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__host__ __device__ __forceinline__ float length(V3 a) { return sqrtf(dot(a, a)); }
__host__ __device__ __forceinline__ V3 normalize(V3 a) {
  float s = a.x * a.x + a.y * a.y + a.z * a.z;
  float inv = 1.0f / sqrtf(s);
  return scale(a, inv);
}
__host__ __device__ __forceinline__ V3 vmin(V3 a, V3 b) { return v3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
__host__ __device__ __forceinline__ V3 vmax(V3 a, V3 b) { return v3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }
__host__ __device__ __forceinline__ float vsum(V3 a) { return a.x + a.y + a.z; }
__host__ __device__ __forceinline__ float comp(V3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
__host__ __device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
__device__ __forceinline__ V3 xyz(float4 f) { return v3(f.x, f.y, f.z); }
__device__ __forceinline__ float4 f4(V3 a, float w) { return make_float4(a.x, a.y, a.z, w); }

// Row-major 4x4 matrix times (x, y, z, w): each output row is a 4-term dot
// product summed left to right (GPUDataTypes.h:50-60).
__host__ __device__ __forceinline__ void m4mul(const float* M, float x, float y, float z, float w, float* o) {
#pragma unroll
  for (int r = 0; r < 4; ++r) o[r] = M[4 * r + 0] * x + M[4 * r + 1] * y + M[4 * r + 2] * z + M[4 * r + 3] * w;
}
// toWorldPoint / toObjectSpace origin (KernelHelpers.h:217-246).
__host__ __device__ __forceinline__ V3 xform_point(const float* M, V3 p) {
  float h[4];
  m4mul(M, p.x, p.y, p.z, 1.f, h);
  return divs(v3(h[0], h[1], h[2]), h[3]);
}
// transformDirection (KernelHelpers.h:237-241).
__host__ __device__ __forceinline__ V3 xform_dir(const float* M, V3 d) {
  float h[4];
  m4mul(M, d.x, d.y, d.z, 0.f, h);
  return normalize(v3(h[0], h[1], h[2]));
}

// ------------------------------------------------------------------- RNG
// SplitMix64 seeding, makePerItemSeed1D and Xorshift128
// (KernelHelpers.h:12-115).
__host__ __device__ __forceinline__ uint64_t splitmix_next(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__host__ __device__ __forceinline__ uint64_t per_item_seed(uint64_t base, uint64_t id) {
  uint64_t mixed = base ^ (0x9E3779B97F4A7C15ull + id);
  return splitmix_next(mixed);
}
struct Rng {
  uint32_t x, y, z, w;
  __device__ __forceinline__ explicit Rng(uint64_t seed) {
    uint64_t s = seed;
    x = (uint32_t)splitmix_next(s);
    y = (uint32_t)splitmix_next(s);
    z = (uint32_t)splitmix_next(s);
    w = (uint32_t)splitmix_next(s);
    if (!(x | y | z | w)) w = 0xA511E9B3u;
  }
  __device__ __forceinline__ uint32_t next_u32() {
    uint32_t t = x ^ (x << 11);
    x = y;
    y = z;
    z = w;
    w = (w ^ (w >> 19)) ^ (t ^ (t >> 8));
    return w;
  }
  __device__ __forceinline__ float next_float() { return (float)(next_u32() >> 8) * 0x1.0p-24f; }
};

// ---------------------------------------------------------- device layout
// Traversal node of the surfel LBVH: 16 words holding both children's
// boxes and child words.  Child word: < 0x80000000 internal node index;
// bit 31 set: leaf, bits 28-30 = count-1, bits 0-27 = first surfel;
// 0xFFFFFFFF: no child.
struct BvhNode {
  float4 a;  // c0.lo.x c0.lo.y c0.lo.z c0.hi.x
  float4 b;  // c0.hi.y c0.hi.z c1.lo.x c1.lo.y
  float4 c;  // c1.lo.z c1.hi.x c1.hi.y c1.hi.z
  uint4 d;   // word0 word1 0 0
};
static_assert(sizeof(BvhNode) == 64, "node layout");

// Traversal copy of a node: the two child boxes in half precision rounded
// outwards (lower corners down, upper corners up, so a box only grows and
// no hit is lost) and the two child words, 32 B against BvhNode's 64 B.
//   q0 = halves (c0.lo.x c0.lo.y) (c0.lo.z c0.hi.x) (c0.hi.y c0.hi.z) (c1.lo.x c1.lo.y)
//   q1 = halves (c1.lo.z c1.hi.x) (c1.hi.y c1.hi.z), word0, word1
struct BvhNodeH {
  uint4 q0;
  uint4 q1;
};
static_assert(sizeof(BvhNodeH) == 32, "node layout");
// Traversal stack entries per thread kept in shared memory (the rest local).
#ifndef PALE_SMEM_STACK
#define PALE_SMEM_STACK 8
#endif

#ifndef PALE_HALF_NODES
#define PALE_HALF_NODES 1
#endif
#if PALE_HALF_NODES
using TravNode = BvhNodeH;
#else
using TravNode = BvhNode;
#endif

// Surfel arrays in BVH (leaf) order.
struct SurfelView {
  const float4* pe;    // position, 4*exp(beta)
  const float4* n;     // Gram-Schmidt normal (intersection), opacity
  const float4* u;     // stored unit tangent u, scale u
  const float4* v;     // stored unit tangent v, scale v
  const float4* cn;    // canonical normal normalize(tu x tv), beta
  const float4* alb;   // albedo, alpha_r
  uint32_t count;
};

struct MeshView {
  const float* o2w;        // per mesh instance 16 floats
  const float* w2o;        // per mesh instance 16 floats
  const float4* box;       // per mesh instance: lo (xyz), hi (xyz) as 2 float4
  const uint2* tri_range;  // per mesh instance: first triangle, count
  const float4* tri;       // per triangle 3 float4 object-space vertices
  const float4* wtri;      // per instance triangle 3 float4 world-space vertices,
                           // xform_point(o2w, v) of the object-space ones
  const uint2* wtri_range; // per mesh instance: first world triangle, count
  const uint32_t* material;  // per mesh instance
  const float4* materials;   // base colour rgb, power
  uint32_t instances;
};

struct LightView {
  uint32_t count;
  const uint4* rec;        // mesh instance, tri offset, tri count, 0
  const float4* col;       // colour rgb, power
  const float* area;       // total world area per light
  const float* cdf;        // per emissive triangle inclusive CDF
  const uint32_t* tri;     // per emissive triangle global triangle id
};

struct GridView {
  float radius;
  V3 origin;
  V3 cell;
  int res[3];
  uint32_t cells;
  const uint32_t* cell_off;   // cells+1 exclusive offsets into the sorted photons
  const float4* pa;           // sorted: position, power.r
  const float4* pb;           // sorted: incoming direction, power.g
  const float* pc;            // sorted: power.b
  const uint32_t* attempts;   // deposits attempted (device)
  uint64_t capacity;
};

struct SceneView {
  MeshView mesh;
  SurfelView sf;
  const TravNode* nodes;   // traversal copy of the LBVH nodes
  uint32_t node_count;
  uint32_t top_nodes;      // nodes [0, top_nodes) are the shared-memory copy
  V3 pc_lo, pc_hi;         // box of the whole surfel cloud
  int has_pc;
  LightView lights;
  GridView grid;
};

// Ray record of the work queues (RayState, GPUDataStructures.h:242-250):
// (origin, path id) (direction, bounce) (throughput, pixel).
struct RayRec {
  float4 o;
  float4 d;
  float4 t;
};

// Device-side run state shared by the kernels of one render call.
struct RunState {
  uint32_t active[2];       // queue lengths by bounce parity
  uint32_t seed_cursor;     // index into the seed table
  uint32_t photon_attempts; // deposits attempted so far
  uint32_t photon_base;     // attempts before the current bounce
  uint32_t event_count;     // events of the current bounce
  uint32_t error;
  uint32_t walk_next;       // next ray of a persistent walk (sorted position)
  unsigned long long photon_segments;
  unsigned long long gather_segments;
  unsigned long long adjoint_segments;
  unsigned long long gradient_events;
  unsigned long long gather_queries;
  unsigned long long node_visits;
  unsigned long long surfel_tests;
  unsigned long long photons_scanned;
  unsigned long long gather_node_visits;   // camera-gather kernel only
  unsigned long long gather_surfel_tests;
  unsigned long long gather_photons_scanned;
};

// Per-camera constants of makePrimaryRayFromPixelJitteredFov
// (KernelHelpers.h:764-796); f_x, f_y are computed on the host.
struct CameraRec {
  float inv_view[16];
  float width, height, half_w, half_h, fx, fy;
  uint32_t w, h;
  uint32_t pixel_offset;   // first pixel of this camera in the packed images
  uint32_t seed_slot;      // seed index relative to the cursor
  uint32_t passes;         // gather / adjoint passes of this view
  uint32_t scene;          // index of the view's scene in the call's scene table
  uint32_t depth;          // adjoint bounces of this view
  uint32_t pass_begin;     // the passes [pass_begin, pass_end) of `passes` this call renders
  uint32_t pass_end;       //   (a forward in slices keeps its running sums between calls)
  uint32_t pad[1];
};

__device__ __forceinline__ void flag_error(RunState* st, uint32_t bit) { atomicOr(&st->error, bit); }

// Warp-aggregated 64-bit counter increment.
__device__ __forceinline__ void warp_count(unsigned long long* ctr, uint32_t v) {
  unsigned mask = __activemask();
  uint32_t s = __reduce_add_sync(mask, v);
  int lane = threadIdx.x & 31;
  int leader = __ffs(mask) - 1;
  if (lane == leader && s) atomicAdd(ctr, (unsigned long long)s);
}

// Adds per-thread counts to three global counters with one atomic each per
// block instead of per warp: same-address atomics serialise, and a kernel
// with a block per 256 rays would issue millions.  Every thread of the
// block must call it.
__device__ __forceinline__ void block_count3(unsigned long long* ca, uint32_t va, unsigned long long* cb, uint32_t vb,
                                             unsigned long long* cc, uint32_t vc) {
  __shared__ unsigned long long s_cnt[3];
  if (threadIdx.x < 3) s_cnt[threadIdx.x] = 0ull;
  __syncthreads();
  const uint32_t a = __reduce_add_sync(0xffffffffu, va);
  const uint32_t b = __reduce_add_sync(0xffffffffu, vb);
  const uint32_t c = __reduce_add_sync(0xffffffffu, vc);
  if ((threadIdx.x & 31) == 0) {
    if (a) atomicAdd(&s_cnt[0], (unsigned long long)a);
    if (b) atomicAdd(&s_cnt[1], (unsigned long long)b);
    if (c) atomicAdd(&s_cnt[2], (unsigned long long)c);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (s_cnt[0] && ca) atomicAdd(ca, s_cnt[0]);
    if (s_cnt[1] && cb) atomicAdd(cb, s_cnt[1]);
    if (s_cnt[2] && cc) atomicAdd(cc, s_cnt[2]);
  }
}

}  // namespace pale
