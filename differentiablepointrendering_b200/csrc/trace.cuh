// trace.cuh -- closest-hit scene queries, sampling and photon lookups.
//
// intersect_scene() returns the closest hit over the mesh instances and the
// surfel cloud, the FirstHit mode of intersectScene
// (Pale/Renderer/Kernels/IntersectionKernels.h:954-1097).  The surfel part
// walks the LBVH with a short stack of (node, entry distance) pairs; the
// first `top_nodes` nodes are read from a shared-memory copy staged by the
// calling kernel.
#pragma once

#include "common.cuh"

namespace pale {

struct Hit {
  int inst;        // -1 miss; mesh instance index; == mesh.instances for a surfel
  uint32_t prim;   // triangle id or surfel index (BVH order)
  float t;         // world-space distance along the ray
  float alpha;     // alpha_geom of a surfel hit (0 for meshes)
  V3 pos;          // world hit position
};

struct TraceCounters {
  uint32_t nodes;
  uint32_t tests;
};

// safeInvDir (KernelHelpers.h:140-148).
__device__ __forceinline__ V3 safe_inv(V3 d) {
  return v3(fabsf(d.x) < 1e-6f ? 1e30f : 1.f / d.x, fabsf(d.y) < 1e-6f ? 1e30f : 1.f / d.y,
            fabsf(d.z) < 1e-6f ? 1e30f : 1.f / d.z);
}

// slabIntersectAABB (KernelHelpers.h:150-214): returns the entry distance
// or +inf on a miss.
__device__ __forceinline__ float slab_entry(V3 o, V3 inv, float lx, float ly, float lz, float hx, float hy,
                                            float hz, float limit) {
  float t0x = (lx - o.x) * inv.x, t1x = (hx - o.x) * inv.x;
  float t0y = (ly - o.y) * inv.y, t1y = (hy - o.y) * inv.y;
  float t0z = (lz - o.z) * inv.z, t1z = (hz - o.z) * inv.z;
  float tmin = fmaxf(fmaxf(fminf(t0x, t1x), fminf(t0y, t1y)), fminf(t0z, t1z));
  float tmax = fminf(fminf(fmaxf(t0x, t1x), fmaxf(t0y, t1y)), fmaxf(t0z, t1z));
  if (tmin > tmax || tmax < 0.0f || tmin > limit) return __int_as_float(0x7f800000);
  return tmin;
}

// A box is entered when the slab test hit it (finite entry) no farther
// than the current closest hit.  The finiteness check matters while `best`
// is still +inf: a miss (+inf) must not compare as "<= best".
__device__ __forceinline__ bool entered(float e, float best) { return e < 3.402823466e+38f && e <= best; }

// intersectTriangle (KernelHelpers.h:248-277).
__device__ __forceinline__ bool tri_hit(V3 o, V3 d, V3 v0, V3 v1, V3 v2, float tmin, float& t_out) {
  V3 e1 = v1 - v0, e2 = v2 - v0;
  V3 h = cross(d, e2);
  float a = dot(e1, h);
  if (fabsf(a) < 1.0e-4f) return false;
  float f = 1.0f / a;
  V3 s = o - v0;
  float u = f * dot(s, h);
  if (u < 0.0f || u > 1.0f) return false;
  V3 q = cross(s, e1);
  float v = f * dot(d, q);
  if (v < 0.0f || u + v > 1.0f) return false;
  float t = f * dot(e2, q);
  if (t <= tmin) return false;
  t_out = t;
  return true;
}

// intersectSurfel + opacityBeta (KernelHelpers.h:506-669) on the
// precomputed surfel arrays.
__device__ __forceinline__ bool surfel_hit(const SurfelView& sf, uint32_t i, V3 o, V3 d, float tmin, float tmax,
                                           float& t_out, V3& x_out, float& a_out) {
  const float4 n4 = __ldg(&sf.n[i]);
  const float4 pe = __ldg(&sf.pe[i]);
  V3 n = xyz(n4);
  float nd = dot(n, d);
  if (fabsf(nd) < 1e-6f) return false;
  V3 p = xyz(pe);
  float th = dot(n, p - o) / nd;
  if (th <= tmin || th >= tmax) return false;
  const float4 u4 = __ldg(&sf.u[i]);
  const float4 v4 = __ldg(&sf.v[i]);
  V3 x = o + scale(d, th);
  V3 r = x - p;
  float u = dot(xyz(u4), r) / u4.w;
  float v = dot(xyz(v4), r) / v4.w;
  float r2 = u * u + v * v;
  if (r2 >= 1.0f) return false;
  a_out = powf(1.0f - r2, pe.w);
  t_out = th;
  x_out = x;
  return true;
}

// The hit point and alpha_geom of surfel i at distance th along (o, d):
// the operations of surfel_hit after its distance test, so the values are
// the ones it computed for that hit.
__device__ __forceinline__ void surfel_eval(const SurfelView& sf, uint32_t i, V3 o, V3 d, float th, V3& x_out,
                                            float& a_out) {
  const float4 pe = __ldg(&sf.pe[i]);
  const float4 u4 = __ldg(&sf.u[i]);
  const float4 v4 = __ldg(&sf.v[i]);
  V3 x = o + scale(d, th);
  V3 r = x - xyz(pe);
  float u = dot(xyz(u4), r) / u4.w;
  float v = dot(xyz(v4), r) / v4.w;
  float r2 = u * u + v * v;
  a_out = powf(1.0f - r2, pe.w);
  x_out = x;
}

#if PALE_HALF_NODES
__device__ __forceinline__ float2 half_pair(uint32_t v) {
  return __half22float2(*reinterpret_cast<const __half2*>(&v));
}

__device__ __forceinline__ void load_node(const SceneView& S, const TravNode* __restrict__ smem_top, uint32_t idx,
                                          float4& a, float4& b, float4& c, uint4& w) {
  uint4 q0, q1;
  if (idx < S.top_nodes) {
    q0 = smem_top[idx].q0;
    q1 = smem_top[idx].q1;
  } else {
    const BvhNodeH* nd = S.nodes + idx;
    q0 = __ldg(&nd->q0);
    q1 = __ldg(&nd->q1);
  }
  const float2 p0 = half_pair(q0.x), p1 = half_pair(q0.y), p2 = half_pair(q0.z), p3 = half_pair(q0.w);
  const float2 p4 = half_pair(q1.x), p5 = half_pair(q1.y);
  a = make_float4(p0.x, p0.y, p1.x, p1.y);
  b = make_float4(p2.x, p2.y, p3.x, p3.y);
  c = make_float4(p4.x, p4.y, p5.x, p5.y);
  w = make_uint4(q1.z, q1.w, 0u, 0u);
}
#else
__device__ __forceinline__ void load_node(const SceneView& S, const TravNode* __restrict__ smem_top, uint32_t idx,
                                          float4& a, float4& b, float4& c, uint4& w) {
  if (idx < S.top_nodes) {
    const BvhNode& nd = smem_top[idx];
    a = nd.a; b = nd.b; c = nd.c; w = nd.d;
  } else {
    const BvhNode* nd = S.nodes + idx;
    a = __ldg(&nd->a); b = __ldg(&nd->b); c = __ldg(&nd->c); w = __ldg(&nd->d);
  }
}
#endif

// The traversal stack of one thread: its first PALE_SMEM_STACK entries in
// shared memory after the staged top nodes (entry k of thread t at
// [k * blockDim.x + t], so a warp's accesses hit distinct banks), the rest
// in a local array.  Traversal kernels size their dynamic shared memory for
// it (top_smem).  The local part alone would be 512 B per thread, more than
// L1 holds for four resident blocks, so pops would wait on L2.
struct TravStack {
#if PALE_SMEM_STACK > 0
  uint2* sm;
#endif
  uint32_t node[kStackDepth - PALE_SMEM_STACK];
  float t[kStackDepth - PALE_SMEM_STACK];
  __device__ __forceinline__ TravStack(const TravNode* smem_top, uint32_t top_nodes) {
#if PALE_SMEM_STACK > 0
    sm = reinterpret_cast<uint2*>(const_cast<TravNode*>(smem_top) + top_nodes) + threadIdx.x;
#else
    (void)smem_top;
    (void)top_nodes;
#endif
  }
  __device__ __forceinline__ void push(int sp, uint32_t n, float tt) {
#if PALE_SMEM_STACK > 0
    if (sp < PALE_SMEM_STACK) {
      sm[(size_t)sp * blockDim.x] = make_uint2(n, __float_as_uint(tt));
      return;
    }
#endif
    node[sp - PALE_SMEM_STACK] = n;
    t[sp - PALE_SMEM_STACK] = tt;
  }
  __device__ __forceinline__ void get(int sp, uint32_t& n, float& tt) const {
#if PALE_SMEM_STACK > 0
    if (sp < PALE_SMEM_STACK) {
      const uint2 e = sm[(size_t)sp * blockDim.x];
      n = e.x;
      tt = __uint_as_float(e.y);
      return;
    }
#endif
    n = node[sp - PALE_SMEM_STACK];
    tt = t[sp - PALE_SMEM_STACK];
  }
};

// One walk over the surfel LBVH, one step() at a time, so that a persistent
// kernel can hand a lane a new ray between steps.  A walk's position is a
// child word with its entry distance: an inner node (a step loads it, tests
// its two child boxes, continues with the nearer child hit and pushes the
// farther) or a leaf (a step tests its surfels).  Leaves go through the same
// near-to-far order and stack as inner nodes, so that a warp can run the
// steps of its lanes that stand at leaves together, apart from the inner
// visits (at_leaf()): the surfel test and the node visit are long and
// different code, and a lane that tested its leaf inside the node visit
// kept the other lanes of its warp waiting.  `Leaf` is the walk's leaf
// test (a closest hit, or the K closest hits).
template <class Leaf>
struct WalkBase {
  V3 o, d, inv;
  float tmin;
  uint32_t node, visit;
  float node_t;
  int sp;
  __device__ __forceinline__ void start(V3 o_, V3 d_, float tmin_) {
    o = o_;
    d = d_;
    inv = safe_inv(d_);
    tmin = tmin_;
    node = 0;        // the root, an inner node
    node_t = 0.0f;
    visit = 0;
    sp = 0;
  }
  __device__ __forceinline__ bool at_leaf() const { return (node & kLeafFlag) != 0u; }
  // the next position from the stack whose box the ray can still enter
  __device__ __forceinline__ bool pop(const TravStack& stk, float best) {
    while (sp > 0) {
      --sp;
      uint32_t sn;
      float st_t;
      stk.get(sp, sn, st_t);
      if (st_t <= best) {
        node = sn;
        node_t = st_t;
        return true;
      }
    }
    return false;
  }
  __device__ __forceinline__ bool step(const SceneView& S, const TravNode* __restrict__ smem_top, TravStack& stk,
                                       TraceCounters& ctr, RunState* st) {
    Leaf& self = *static_cast<Leaf*>(this);
    if (at_leaf()) {
      if (node_t <= self.best) {
        const uint32_t f0 = node & 0x0FFFFFFFu, cnt = ((node >> 28) & 7u) + 1u;
        if (f0 + cnt > S.sf.count) {
          flag_error(st, kErrBounds);
        } else {
          for (uint32_t j = 0; j < cnt; ++j) {
            ctr.tests++;
            self.test(S.sf, f0 + j);
          }
        }
      }
      return pop(stk, self.best);
    }
    // an acyclic tree visits each node at most once
    const uint32_t visit_cap = 2u * S.node_count + 64u;
    if (node >= S.node_count || visit > visit_cap) {
      flag_error(st, kErrBounds);
      return false;
    }
    ++visit;
    float4 a, b, c;
    uint4 w;
    load_node(S, smem_top, node, a, b, c, w);
    ctr.nodes++;
    const float best = self.best;
    const float e0 =
        w.x == kEmptyChild ? __int_as_float(0x7f800000) : slab_entry(o, inv, a.x, a.y, a.z, a.w, b.x, b.y, best);
    const float e1 =
        w.y == kEmptyChild ? __int_as_float(0x7f800000) : slab_entry(o, inv, b.z, b.w, c.x, c.y, c.z, c.w, best);
    const bool h0 = entered(e0, best), h1 = entered(e1, best);
    if (h0 && h1) {
      const bool first0 = e0 <= e1;
      if (sp < kStackDepth) {
        stk.push(sp, first0 ? w.y : w.x, first0 ? e1 : e0);
        ++sp;
      } else {
        flag_error(st, kErrStackOverflow);
      }
      node = first0 ? w.x : w.y;
      node_t = first0 ? e0 : e1;
      return true;
    }
    if (h0) {
      node = w.x;
      node_t = e0;
      return true;
    }
    if (h1) {
      node = w.y;
      node_t = e1;
      return true;
    }
    return pop(stk, best);
  }
};

// Closest surfel with t in (tmin, limit): after start(), step() returns
// true while the walk goes on; `hit`, `prim` and `best` then hold the
// closest surfel.
struct ClosestWalk : WalkBase<ClosestWalk> {
  float best;
  uint32_t prim;
  bool hit;
  __device__ __forceinline__ void init(V3 o_, V3 d_, float tmin_, float limit) {
    start(o_, d_, tmin_);
    best = limit;
    prim = 0;
    hit = false;
  }
  __device__ __forceinline__ void test(const SurfelView& sf, uint32_t i) {
    float th, aa;
    V3 xx;
    // only the distance and the surfel stay live in the walk; the hit point
    // and alpha of the closest are evaluated after it
    if (surfel_hit(sf, i, o, d, tmin, best, th, xx, aa)) {
      best = th;
      hit = true;
      prim = i;
    }
  }
};

// Closest surfel with t in (tmin, limit) along (o, d) (the surfel cloud's
// transform is the identity, so this is intersectBLASPointCloudFirstHit,
// IntersectionKernels.h:585-675, where tmin is rayEpsilon = 1e-5).  Returns
// false on a miss.
__device__ __forceinline__ bool surfel_closest(const SceneView& S, const TravNode* __restrict__ smem_top, V3 o, V3 d,
                                               float tmin, float limit, uint32_t& prim, float& t, V3& x,
                                               float& alpha, TraceCounters& ctr, RunState* st) {
  if (S.node_count == 0) return false;
  TravStack stk(smem_top, S.top_nodes);
  ClosestWalk w;
  w.init(o, d, tmin, limit);
  while (w.step(S, smem_top, stk, ctr, st)) {
  }
  if (w.hit) {
    prim = w.prim;
    t = w.best;
    surfel_eval(S.sf, w.prim, o, d, w.best, x, alpha);
  }
  return w.hit;
}

// The K closest surfels with t in (tmin, limit) along (o, d), in increasing
// t (ties keep the surfel found first), with the culling distance of the
// K-th hit found so far.  After init(), step() returns true while the walk
// goes on; `count` (<= K) and t_out/prim_out then hold the hits in order.
template <int K>
struct KHitWalk : WalkBase<KHitWalk<K>> {
  float best;   // t_out[K - 1] once K hits are held
  uint32_t count;
  float t_out[K];
  uint32_t prim_out[K];
  __device__ __forceinline__ void init(V3 o_, V3 d_, float tmin_, float limit) {
    this->start(o_, d_, tmin_);
    best = limit;
    count = 0;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      t_out[k] = limit;
      prim_out[k] = 0;
    }
  }
  __device__ __forceinline__ void test(const SurfelView& sf, uint32_t i) {
    float th, aa;
    V3 xx;
    if (surfel_hit(sf, i, this->o, this->d, this->tmin, best, th, xx, aa)) {
      // insert into the sorted list (static indices: stays in registers)
      uint32_t pj = i;
#pragma unroll
      for (int q = 0; q < K; ++q) {
        if (th < t_out[q]) {
          const float tt = t_out[q];
          const uint32_t pp = prim_out[q];
          t_out[q] = th;
          prim_out[q] = pj;
          th = tt;
          pj = pp;
        }
      }
      count = count < (uint32_t)K ? count + 1 : count;
      if (count == (uint32_t)K) best = t_out[K - 1];
    }
  }
};

// The same walk with its sorted hit list in shared memory instead of
// registers (entry q of a thread at hits[q * blockDim.x], (t, surfel)
// pairs), which frees the registers of the list for one more resident
// block; the list is read only when a surfel is hit.
template <int K>
struct KHitWalkS : WalkBase<KHitWalkS<K>> {
  float best;   // the K-th distance once K hits are held
  uint32_t count;
  uint2* hits;  // this thread's first entry
  __device__ __forceinline__ void bind(uint2* h) { hits = h; }
  __device__ __forceinline__ void init(V3 o_, V3 d_, float tmin_, float limit) {
    this->start(o_, d_, tmin_);
    best = limit;
    count = 0;
#pragma unroll
    for (int k = 0; k < K; ++k) hits[(size_t)k * blockDim.x] = make_uint2(__float_as_uint(limit), 0u);
  }
  __device__ __forceinline__ void test(const SurfelView& sf, uint32_t i) {
    float th, aa;
    V3 xx;
    if (surfel_hit(sf, i, this->o, this->d, this->tmin, best, th, xx, aa)) {
      uint32_t pj = i;
#pragma unroll
      for (int q = 0; q < K; ++q) {
        const uint2 e = hits[(size_t)q * blockDim.x];
        const float tq = __uint_as_float(e.x);
        if (th < tq) {
          hits[(size_t)q * blockDim.x] = make_uint2(__float_as_uint(th), pj);
          th = tq;
          pj = e.y;
        }
      }
      count = count < (uint32_t)K ? count + 1 : count;
      if (count == (uint32_t)K) best = __uint_as_float(hits[(size_t)(K - 1) * blockDim.x].x);
    }
  }
  __device__ __forceinline__ uint32_t prim(int k) const { return hits[(size_t)k * blockDim.x].y; }
};

// One step of a persistent walk loop for the lanes of a warp: the lanes
// whose walk stands at a leaf step together once at least kLeafBatch of
// them (or all of the walking lanes) do, the other times the lanes at inner
// nodes step.  Returns for this lane whether its walk goes on (a lane that
// sat out the step keeps walking).  Every lane of the warp calls it.
template <class W>
__device__ __forceinline__ bool warp_step(W& w, bool walking, const SceneView& S,
                                          const TravNode* __restrict__ smem_top, TravStack& stk, TraceCounters& ctr,
                                          RunState* st) {
  const bool lf = walking && w.at_leaf();
  const unsigned ml = __ballot_sync(0xffffffffu, lf);
  const unsigned ma = __ballot_sync(0xffffffffu, walking);
  const bool leaf_phase = ml != 0u && (ml == ma || __popc(ml) >= kLeafBatch);
  if (walking && lf == leaf_phase) return w.step(S, smem_top, stk, ctr, st);
  return walking;
}

// A 4x4 instance matrix (16 floats, 64 B aligned) in four 16-byte loads.
__device__ __forceinline__ void load_matrix(const float* M, float (&m)[16]) {
  const float4* m4 = reinterpret_cast<const float4*>(M);
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const float4 v = __ldg(&m4[r]);
    m[4 * r] = v.x;
    m[4 * r + 1] = v.y;
    m[4 * r + 2] = v.z;
    m[4 * r + 3] = v.w;
  }
}

// The closest mesh hit, in object space per instance (intersectBLASMesh,
// IntersectionKernels.h:37-105); `best` is the world distance of the hit
// (+inf on a miss).
__device__ __forceinline__ Hit intersect_meshes(const SceneView& S, V3 o, V3 d, V3 invw, float& best) {
  Hit h;
  h.inst = -1;
  h.prim = 0;
  h.t = 3.402823466e+38f;
  h.alpha = 0.f;
  h.pos = v3(0.f, 0.f, 0.f);
  best = __int_as_float(0x7f800000);
  const MeshView& M = S.mesh;
  for (uint32_t i = 0; i < M.instances; ++i) {
    const float4 lo = __ldg(&M.box[2 * i]), hi = __ldg(&M.box[2 * i + 1]);
    if (!entered(slab_entry(o, invw, lo.x, lo.y, lo.z, hi.x, hi.y, hi.z, best), best)) continue;
    float w2o[16];
    load_matrix(M.w2o + 16 * i, w2o);
    V3 oo = xform_point(w2o, o);
    V3 dd = xform_dir(w2o, d);
    uint2 rg = __ldg(&M.tri_range[i]);
    float bt = __int_as_float(0x7f800000);
    bool any = false;
    uint32_t bprim = 0;
    for (uint32_t k = 0; k < rg.y; ++k) {
      const float4* tv = M.tri + 3 * (rg.x + k);
      float t;
      if (tri_hit(oo, dd, xyz(__ldg(&tv[0])), xyz(__ldg(&tv[1])), xyz(__ldg(&tv[2])), 1e-4f, t) && t < bt &&
          t > 0.0f) {
        bt = t;
        any = true;
        bprim = rg.x + k;
      }
    }
    if (!any) continue;
    float o2w[16];
    load_matrix(M.o2w + 16 * i, o2w);
    V3 hw = xform_point(o2w, oo + scale(dd, bt));
    float tw = dot(hw - o, d);
    if (tw > 0.0f && tw < best) {
      best = tw;
      h.inst = (int)i;
      h.t = tw;
      h.pos = hw;
      h.prim = bprim;
      h.alpha = 0.0f;
    }
  }
  return h;
}

// intersectScene, FirstHit mode: mesh instances, then the surfel cloud;
// the closest world-space distance wins (:1060-1081).
__device__ __forceinline__ Hit intersect_scene(const SceneView& S, const TravNode* __restrict__ smem_top, V3 o, V3 d,
                                               TraceCounters& ctr, RunState* st) {
  float best;
  const V3 invw = safe_inv(d);
  Hit h = intersect_meshes(S, o, d, invw, best);
  if (S.has_pc &&
      entered(slab_entry(o, invw, S.pc_lo.x, S.pc_lo.y, S.pc_lo.z, S.pc_hi.x, S.pc_hi.y, S.pc_hi.z, best), best)) {
    V3 dd = normalize(d);
    // prune with the mesh hit plus a relative margin: a surfel beyond the
    // margin cannot have a smaller world distance than the mesh hit
    float limit = best < 3.0e38f ? best * 1.00001f + 1e-6f : __int_as_float(0x7f800000);
    uint32_t prim;
    float t, a;
    V3 x;
    if (surfel_closest(S, smem_top, o, dd, 1e-5f, limit, prim, t, x, a, ctr, st)) {
      float tw = dot(x - o, d);
      if (tw > 0.0f && tw < best) {
        best = tw;
        h.inst = (int)S.mesh.instances;
        h.t = tw;
        h.pos = x;
        h.prim = prim;
        h.alpha = a;
      }
    }
  }
  return h;
}

// intersectScene, Transmit mode (:1066-1090): the closest mesh hit, and the
// surfel cloud's transmissivity T over the whole ray
// (intersectBLASPointCloudTransmit, :837-948): the successive closest
// surfels from the same origin, t in (tMin, inf) with tMin = t_hit + 1e-4
// after each hit (the reference rejects t <= tMin after intersectSurfel's
// t > 1e-5, and tMin >= 1e-5), T *= 1 - opacity * alpha_geom, stopping once
// T <= 0.001.  The cloud is skipped (T = 1) when its box starts beyond the
// mesh hit, as the instance loop culls it.  `max_hits` bounds the walk (the
// kernel flags kErrLayerCap when it is reached).
__device__ __forceinline__ Hit intersect_scene_transmit(const SceneView& S, const TravNode* __restrict__ smem_top,
                                                        V3 o, V3 d, float& T, uint32_t max_hits,
                                                        TraceCounters& ctr, RunState* st) {
  float best;
  const V3 invw = safe_inv(d);
  Hit h = intersect_meshes(S, o, d, invw, best);
  T = 1.0f;
  if (S.has_pc &&
      entered(slab_entry(o, invw, S.pc_lo.x, S.pc_lo.y, S.pc_lo.z, S.pc_hi.x, S.pc_hi.y, S.pc_hi.z, best), best)) {
    const V3 dd = normalize(d);
    float tmin = 1e-5f;
    uint32_t k = 0;
    for (; k < max_hits; ++k) {
      uint32_t prim;
      float t, a;
      V3 x;
      if (!surfel_closest(S, smem_top, o, dd, tmin, __int_as_float(0x7f800000), prim, t, x, a, ctr, st)) break;
      const float alpha_eff = __ldg(&S.sf.n[prim]).w * a;
      T *= 1.0f - alpha_eff;
      tmin = t + 1e-4f;
      if (T <= 0.001f) break;
    }
    if (k == max_hits) flag_error(st, kErrLayerCap);
  }
  return h;
}

// buildIntersectionNormal (KernelHelpers.h:480-503).
__device__ __forceinline__ V3 hit_normal(const SceneView& S, const Hit& h) {
  if (h.inst < (int)S.mesh.instances) {
    // the world-space copy holds xform_point(o2w, v) of the triangle's vertices
    const uint32_t k = h.prim - __ldg(&S.mesh.tri_range[h.inst]).x;
    const float4* tv = S.mesh.wtri + 3 * (__ldg(&S.mesh.wtri_range[h.inst]).x + k);
    const V3 p0 = xyz(__ldg(&tv[0])), p1 = xyz(__ldg(&tv[1])), p2 = xyz(__ldg(&tv[2]));
    return normalize(cross(p1 - p0, p2 - p0));
  }
  return xyz(__ldg(&S.sf.cn[h.prim]));
}

// ------------------------------------------------------------- sampling
// sampleCosineHemisphere, rng-first overload (KernelHelpers.h:317-337).
__device__ __forceinline__ void sample_cosine(Rng& r, V3 n, V3& out, float& pdf) {
  float u1 = r.next_float(), u2 = r.next_float();
  float z = sqrtf(1.f - u1);
  float rr = sqrtf(1 - (z * z));
  float phi = 2.f * kPi * u2;
  float x = rr * cosf(phi), y = rr * sinf(phi);
  V3 up = fabsf(n.z) < .999f ? v3(0, 0, 1) : v3(1, 0, 0);
  V3 tang = normalize(cross(up, n));
  V3 bit = cross(n, tang);
  out = normalize(scale(tang, x) + scale(bit, y) + scale(n, z));
  pdf = fmaxf(0.f, dot(out, n)) / kPi;
}

// sampleUniformHemisphereAroundNormal with the Frisvad basis
// (KernelHelpers.h:541-611).
__device__ __forceinline__ void sample_uniform_hemi(Rng& r, V3 normal, V3& out, float& pdf) {
  V3 n = normalize(normal);
  float u1 = r.next_float(), u2 = r.next_float();
  float z = u1;
  float phi = 2.0f * kPi * u2;
  float rr = sqrtf(fmaxf(0.0f, 1.0f - z * z));
  float x = rr * cosf(phi), y = rr * sinf(phi);
  float sign = copysignf(1.0f, n.z);
  float a = -1.0f / (sign + n.z);
  float b = n.x * n.y * a;
  V3 T = v3(1.0f + sign * n.x * n.x * a, sign * b, -sign * n.x);
  V3 B = v3(b, sign + n.y * n.y * a, -n.y);
  out = normalize(scale(T, x) + scale(B, y) + scale(n, z));
  pdf = 1.0f / (2.0f * kPi);
}

// applyRussianRoulette (KernelHelpers.h:1612-1657).
__device__ __forceinline__ bool russian_roulette(Rng& r, uint32_t bounce, V3& thr, uint32_t start) {
  if (bounce < start) return true;
  if (!isfinite(thr.x) || !isfinite(thr.y) || !isfinite(thr.z)) return false;
  float lum = 0.2126f * thr.x + 0.7152f * thr.y + 0.0722f * thr.z;
  float p = clampf(lum, 0.0f, 0.99f);
  if (r.next_float() > p) return false;
  float c = 1.0f / p;
  c = fminf(c, 10.0f);
  thr = scale(thr, c);
  return true;
}

// sampleMeshAreaLight (KernelHelpers.h:340-449).
__device__ __forceinline__ bool sample_light(const SceneView& S, Rng& r, V3& pos, V3& nrm, V3& dir, V3& power) {
  const LightView& L = S.lights;
  if (L.count == 0) return false;
  float ul = r.next_float();
  uint32_t li = (uint32_t)(ul * (float)L.count);
  if (li > L.count - 1u) li = L.count - 1u;
  uint4 rec = __ldg(&L.rec[li]);
  float area = __ldg(&L.area[li]);
  if (rec.z == 0u || area <= 0.0f) return false;
  float ut = r.next_float();
  uint32_t lo = 0, hi = rec.z - 1u;
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1u;
    if (ut <= __ldg(&L.cdf[rec.y + mid])) hi = mid;
    else lo = mid + 1u;
  }
  uint32_t tri = __ldg(&L.tri[rec.y + lo]);
  const float4* tv = S.mesh.tri + 3 * tri;
  V3 p0 = xyz(__ldg(&tv[0])), p1 = xyz(__ldg(&tv[1])), p2 = xyz(__ldg(&tv[2]));
  float u1 = r.next_float(), u2 = r.next_float();
  float su1 = sqrtf(u1);
  float b0 = 1.0f - su1, b1 = su1 * (1.0f - u2), b2 = su1 * u2;
  V3 xo = scale(p0, b0) + scale(p1, b1) + scale(p2, b2);
  float o2w[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) o2w[k] = __ldg(&S.mesh.o2w[16 * rec.x + k]);
  V3 w0 = xform_point(o2w, p0), w1 = xform_point(o2w, p1), w2 = xform_point(o2w, p2);
  V3 e0 = w1 - w0, e1 = w2 - w0;
  V3 nw = v3(e0.y * e1.z - e0.z * e1.y, e0.z * e1.x - e0.x * e1.z, e0.x * e1.y - e0.y * e1.x);
  float nl = sqrtf(dot(nw, nw));
  if (nl <= 0.0f) return false;
  nw = divs(nw, nl);
  float pdf;
  sample_cosine(r, nw, dir, pdf);
  pos = xform_point(o2w, xo);
  nrm = nw;
  float4 col = __ldg(&L.col[li]);
  power = scale(xyz(col), col.w);
  return true;
}

// --------------------------------------------------------------- photons
// worldToCellClamped / linearCellIndex (KernelHelpers.h:900-987).
__device__ __forceinline__ void world_to_cell(const GridView& G, V3 p, int c[3]) {
  V3 l = p - G.origin;
  float f[3] = {l.x / G.cell.x, l.y / G.cell.y, l.z / G.cell.z};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    int v = (int)floorf(f[a]);
    v = v < 0 ? 0 : v;
    v = v > G.res[a] - 1 ? G.res[a] - 1 : v;
    c[a] = v;
  }
}

// gatherDiffuseIrradianceAtPoint (KernelHelpers.h:990-1037), done by a
// whole warp for one query (x, n), which every lane passes.  Photons are
// stored sorted by cell with ascending deposit index inside a cell, and the
// cells of one grid row (fixed y, z) are contiguous, so each row of the
// query window is one contiguous photon range and walking the rows in
// (z, y) order visits the photons in the reference's cell-by-cell order.
// The rows of the window are concatenated (a warp scan of their lengths),
// and each round the 32 lanes test 32 consecutive photons of that sequence
// with coalesced loads.  Every lane adds the power of the photons it
// accepts (radius and cosine tests) into its own running sum, and the 32
// sums are added by a butterfly of shuffles at the end: the same terms as
// the reference's one-photon-at-a-time loop, summed in another order (the
// result differs from it by float rounding, about 1e-7 relative; a photon
// within a rounding error of the radius can fall on either side).  `terms`
// is this warp's 32 float4 of shared memory (the row compaction).
// Returns the irradiance in every lane and the photons scanned in `count`.
// Per-launch constants of the lookups: 1 / (pi r^2), 1 / cell, and the
// T / D factor of the photon store (0 when nothing was deposited, so an
// empty map gives zero irradiance).
struct GatherConst {
  float inv_area;
  float inv_cx;
  float scale;
  uint32_t total_ph;   // photons in the sorted grid
};

__device__ __forceinline__ GatherConst gather_const(const GridView& G) {
  GatherConst c;
  const float r = G.radius, r2 = r * r;
  c.inv_area = 1.0f / (kPi * r2);
  c.inv_cx = 1.0f / G.cell.x;
  const uint32_t T = *G.attempts;
  const uint32_t D = (uint64_t)T < G.capacity ? T : (uint32_t)G.capacity;
  c.scale = D == 0u ? 0.0f : (float)T / (float)D;
  c.total_ph = __ldg(&G.cell_off[G.cells]);
  return c;
}

// kPipelined: each round's photon records are loaded one round ahead (the
// adjoint's lookups, which wait on L2 more than they issue); camera
// lookups, most of which end after one or two rounds, load them in place.
template <bool kPipelined>
__device__ __forceinline__ V3 gather_irradiance_warp(const GridView& G, const GatherConst& GC, V3 x, V3 n,
                                                     float4* terms, uint32_t& count) {
  const int lane = threadIdx.x & 31;
  const float r = G.radius, r2 = r * r;
  const float invArea = GC.inv_area;
  // window corners: lanes 0-5 each do one coordinate of world_to_cell(x -
  // (r, r, r)) and world_to_cell(x + (r, r, r)), the same operations
  int wc = 0;
  if (lane < 6) {
    const int a = lane % 3;
    const float xa = a == 0 ? x.x : (a == 1 ? x.y : x.z);
    const float oa = a == 0 ? G.origin.x : (a == 1 ? G.origin.y : G.origin.z);
    const float ca = a == 0 ? G.cell.x : (a == 1 ? G.cell.y : G.cell.z);
    const float p = lane < 3 ? xa - r : xa + r;
    int v = (int)floorf((p - oa) / ca);
    v = v < 0 ? 0 : v;
    v = v > G.res[a] - 1 ? G.res[a] - 1 : v;
    wc = v;
  }
  int c0[3], c1[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    c0[a] = __shfl_sync(0xffffffffu, wc, a);
    c1[a] = __shfl_sync(0xffffffffu, wc, 3 + a);
  }
  const int ny = c1[1] - c0[1] + 1;
  const int rows = (c1[2] - c0[2] + 1) * ny;
  // row k of the window is (z, y) = (k / ny, k % ny); (k + 1/2) / ny is at
  // least 1/(2 ny) from an integer, far beyond float rounding
  const float inv_ny = __fdividef(1.0f, (float)ny);
  const float inv_cx = GC.inv_cx;
  const uint32_t total_ph = GC.total_ph;
  float ax = 0.f, ay = 0.f, az = 0.f;   // this lane's sums of the accepted terms
  uint32_t scanned = 0;
  for (int rb = 0; rb < rows; rb += 32) {
    // this lane's row: offsets and length
    const int k = rb + lane;
    uint32_t j0 = 0, len = 0;
    if (k < rows) {
      const int kz = (int)(((float)k + 0.5f) * inv_ny);
      const int cz = c0[2] + kz, cy = c0[1] + (k - kz * ny);
      const uint32_t row = (uint32_t)((cz * G.res[1] + cy) * G.res[0]);
      // Clip the row to the sphere of radius r around x.  A photon binned
      // to cell c lies in [c, c + 1] cells from the origin up to rounding
      // (1% of a cell covers it), except in the edge cells, which also hold
      // the clamped photons from beyond the grid.  Every photon left out
      // lies farther than r * 1.001 from x, so the reference's loop rejects
      // it; the photons kept are summed in the same order.
      const float reach2 = r2 * 1.002f;
      float dy = 0.f, dz = 0.f;
      if (cy > 0) dy = fmaxf(dy, (G.origin.y + (float)cy * G.cell.y - 0.01f * G.cell.y) - x.y);
      if (cy < G.res[1] - 1) dy = fmaxf(dy, x.y - (G.origin.y + (float)(cy + 1) * G.cell.y + 0.01f * G.cell.y));
      if (cz > 0) dz = fmaxf(dz, (G.origin.z + (float)cz * G.cell.z - 0.01f * G.cell.z) - x.z);
      if (cz < G.res[2] - 1) dz = fmaxf(dz, x.z - (G.origin.z + (float)(cz + 1) * G.cell.z + 0.01f * G.cell.z));
      const float rho2 = dy * dy + dz * dz;
      if (rho2 <= reach2) {
        // (an approximate square root is enough: the 1.001 factor covers it)
        const float q = fmaxf(reach2 - rho2, 1e-30f);
        const float w = q * rsqrtf(q) * 1.001f + 0.01f * G.cell.x;
        // (a reciprocal is enough here: the 1% margin covers its rounding)
        int lo = (int)floorf(((x.x - w) - G.origin.x) * inv_cx);
        int hi = (int)floorf(((x.x + w) - G.origin.x) * inv_cx);
        lo = lo > c0[0] ? lo : c0[0];
        hi = hi < c1[0] ? hi : c1[0];
        if (lo <= hi) {
          uint32_t a = __ldg(&G.cell_off[row + lo]);
          uint32_t b = __ldg(&G.cell_off[row + hi + 1]);
          b = b < total_ph ? b : total_ph;
          a = a < b ? a : b;
          j0 = a;
          len = b - a;
        }
      }
    }
    uint32_t incl = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    const uint32_t excl = incl - len;
    const uint32_t seq = __shfl_sync(0xffffffffu, incl, 31);
    scanned += seq;
    // the non-empty rows, compacted into lanes 0..nne-1 in row order (their
    // starts are then strictly increasing); staged through the terms buffer
    const unsigned nm = __ballot_sync(0xffffffffu, len > 0);
    const int nne = __popc(nm);
    uint32_t* cw = reinterpret_cast<uint32_t*>(terms);
    if (len > 0) {
      const int o = __popc(nm & ((1u << lane) - 1u));
      cw[o] = j0;
      cw[32 + o] = excl;
    }
    __syncwarp();
    const uint32_t cj0 = lane < nne ? cw[lane] : 0u;
    const uint32_t cex = lane < nne ? cw[32 + lane] : 0xFFFFFFFFu;
    __syncwarp();
    // The photon of sequence index base + lane: its three records at once
    // (one memory round trip per round).
    auto fetch = [&](uint32_t base, float4& pa, float4& pb, float& pc) {
      const uint32_t v = base + lane;
      // row holding sequence index v: the non-empty rows starting at or
      // before v are those starting before this round plus those starting
      // in the round at lanes <= this one (one bit per row start)
      const bool starts_here = lane < nne && cex >= base && cex - base < 32u;
      const uint32_t smask = __reduce_or_sync(0xffffffffu, starts_here ? (1u << (cex - base)) : 0u);
      const uint32_t before = __popc(__ballot_sync(0xffffffffu, lane < nne && cex < base));
      const int ord = (int)before + __popc(smask & (0xFFFFFFFFu >> (31 - lane))) - 1;
      const uint32_t rj0 = __shfl_sync(0xffffffffu, cj0, ord & 31);
      const uint32_t rex = __shfl_sync(0xffffffffu, cex, ord & 31);
      if (v < seq) {
        const uint32_t j = rj0 + (v - rex);
        pa = __ldg(&G.pa[j]);
        pb = __ldg(&G.pb[j]);
        pc = __ldg(&G.pc[j]);
      }
    };
    float4 pa = make_float4(0.f, 0.f, 0.f, 0.f), pb = pa;
    float pc = 0.f;
    if (kPipelined && seq > 0) fetch(0, pa, pb, pc);
    for (uint32_t base = 0; base < seq; base += 32) {
      float4 na = make_float4(0.f, 0.f, 0.f, 0.f), nb = na;
      float nc = 0.f;
      if (kPipelined) {
        if (base + 32 < seq) fetch(base + 32, na, nb, nc);
      } else {
        fetch(base, pa, pb, pc);
      }
      const uint32_t v = base + lane;
      if (v < seq) {
        const float dx = pa.x - x.x, dy = pa.y - x.y, dz = pa.z - x.z;
        const float d2 = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, dx * dx));
        const float cosine = -__fmaf_rn(n.z, pb.z, __fmaf_rn(n.y, pb.y, n.x * pb.x));
        if (d2 <= r2 && !(cosine < 0.0f)) {
          ax = __fmaf_rn(pa.w, invArea, ax);
          ay = __fmaf_rn(pb.w, invArea, ay);
          az = __fmaf_rn(pc, invArea, az);
        }
      }
      pa = na;
      pb = nb;
      pc = nc;
    }
  }
  count += scanned;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    ax += __shfl_xor_sync(0xffffffffu, ax, o);
    ay += __shfl_xor_sync(0xffffffffu, ay, o);
    az += __shfl_xor_sync(0xffffffffu, az, o);
  }
  const float s = GC.scale;
  return v3(ax * s, ay * s, az * s);
}

}  // namespace pale
