// render.cu -- photon wavefront, photon grid, camera gather and adjoint pass.
//
// Work queues.  The reference appends survivors of a bounce with an atomic
// counter and seeds each item's RNG with its queue slot
// (PrimalKernels.cpp:80-82, AdjointKernels.cpp:99-101).  Here every bounce
// kernel writes its result to a staging record at the input slot and counts
// survivors per 256-slot tile; a one-block scan turns the tile counts into
// offsets and a scatter kernel compacts the staging records in slot order.
// A survivor's new slot is therefore its rank among the survivors -- the
// slot a sequential run of the reference assigns -- so the RNG stream, the
// photon deposit order and the images are deterministic.
//
// Seeds.  The host expands the reference's std::mt19937_64 seed stream
// (SyclBridge.cpp:83-146, 170-227) into a table; RunState::seed_cursor
// walks it on the device, advancing only for bounces that had work, as
// the host loop `for (bounce...; activeCount > 0; ...)` does.
#include "kernels.h"
#include "trace.cuh"

namespace pale {

static inline uint32_t blocks_for(uint64_t n, int b = kBlock) { return (uint32_t)((n + b - 1) / b); }

__device__ __forceinline__ void stage_top_nodes(const SceneView& S, TravNode* smem) {
  for (uint32_t i = threadIdx.x; i < S.top_nodes; i += blockDim.x) smem[i] = S.nodes[i];
  __syncthreads();
}

// The staged top nodes of every scene of a call: scene k's first
// T.s[k].top_nodes nodes at smem[k * T.staged].
__device__ __forceinline__ void stage_top_nodes(const SceneTable& T, TravNode* smem) {
  const uint32_t total = T.n * T.staged;
  for (uint32_t i = threadIdx.x; i < total; i += blockDim.x) {
    const uint32_t k = i / T.staged, j = i - k * T.staged;
    if (j < T.s[k].top_nodes) smem[i] = T.s[k].nodes[j];
  }
  __syncthreads();
}

// The view (index into the call's cameras) that holds packed pixel gp:
// the last camera whose pixel_offset is <= gp.
__device__ __forceinline__ uint32_t view_of_pixel(const CameraRec* __restrict__ cams, uint32_t ncams, uint32_t gp) {
  uint32_t lo = 0, hi = ncams - 1;
  while (lo < hi) {
    const uint32_t mid = (lo + hi + 1) >> 1;
    if (cams[mid].pixel_offset <= gp) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ RayRec make_ray(V3 o, V3 d, V3 thr, uint32_t path, uint32_t bounce, uint32_t pixel) {
  RayRec r;
  r.o = make_float4(o.x, o.y, o.z, __uint_as_float(path));
  r.d = make_float4(d.x, d.y, d.z, __uint_as_float(bounce));
  r.t = make_float4(thr.x, thr.y, thr.z, __uint_as_float(pixel));
  return r;
}

// ---------------------------------------------------------- compaction
// One block: exclusive scan of the per-tile (alive, deposit/event) counts
// of `n_in` slots; updates queue length, deposit/event bases and seeds.
__global__ void __launch_bounds__(1024) k_queue_scan(RunState* st, const uint2* __restrict__ counts, uint2* __restrict__ offsets,
                             uint32_t parity, int emission, uint32_t emission_n, int events, uint64_t photon_cap) {
  __shared__ uint32_t s_wx[32], s_wy[32];
  __shared__ uint32_t s_carry[2];
  const uint32_t n_in = emission ? emission_n : st->active[parity];
  const uint32_t tiles = (n_in + kBlock - 1) / kBlock;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (threadIdx.x == 0) { s_carry[0] = 0; s_carry[1] = 0; }
  __syncthreads();
  for (uint32_t base = 0; base < tiles; base += blockDim.x) {
    uint32_t t = base + threadIdx.x;
    uint2 c = t < tiles ? counts[t] : make_uint2(0u, 0u);
    uint32_t x = c.x, y = c.y;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t ax = __shfl_up_sync(0xffffffffu, x, o), ay = __shfl_up_sync(0xffffffffu, y, o);
      if (lane >= o) { x += ax; y += ay; }
    }
    if (lane == 31) { s_wx[wid] = x; s_wy[wid] = y; }
    __syncthreads();
    if (wid == 0) {
      const int nw = blockDim.x >> 5;
      uint32_t wx = lane < nw ? s_wx[lane] : 0u, wy = lane < nw ? s_wy[lane] : 0u;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t ax = __shfl_up_sync(0xffffffffu, wx, o), ay = __shfl_up_sync(0xffffffffu, wy, o);
        if (lane >= o) { wx += ax; wy += ay; }
      }
      if (lane < nw) { s_wx[lane] = wx; s_wy[lane] = wy; }
    }
    __syncthreads();
    uint32_t px = (wid > 0 ? s_wx[wid - 1] : 0u) + x - c.x;
    uint32_t py = (wid > 0 ? s_wy[wid - 1] : 0u) + y - c.y;
    if (t < tiles) offsets[t] = make_uint2(s_carry[0] + px, s_carry[1] + py);
    __syncthreads();
    if (threadIdx.x == 0) {
      s_carry[0] += s_wx[(blockDim.x >> 5) - 1];
      s_carry[1] += s_wy[(blockDim.x >> 5) - 1];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    st->active[emission ? 0u : (parity ^ 1u)] = s_carry[0];
    if (events) {
      st->event_count = s_carry[1];
    } else {
      st->photon_base = st->photon_attempts;
      st->photon_attempts += s_carry[1];
      if ((uint64_t)st->photon_base + s_carry[1] > photon_cap) atomicOr(&st->error, kErrPhotonCapacity);
    }
    st->seed_cursor += (emission || n_in > 0) ? 1u : 0u;
  }
}

// Compacts staged rays (and deposits or events) of the `n_in` input slots.
template <int kMode>  // 0 photons, 1 adjoint events
__global__ void k_queue_scatter(RunState* st, QueueBufs qb, uint32_t parity, int emission, uint32_t emission_n,
                                PhotonStore ps, EventBufs ev) {
  __shared__ uint32_t s_wx[kBlock / 32], s_wy[kBlock / 32];
  const uint32_t n_in = emission ? emission_n : st->active[parity];
  const uint32_t tile = blockIdx.x;
  if ((uint64_t)tile * kBlock >= n_in) return;
  const uint32_t slot = tile * kBlock + threadIdx.x;
  const bool in = slot < n_in;
  const uint8_t f = in ? qb.flags[slot] : 0;
  const bool alive = f & 1, side = f & 2;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  unsigned ba = __ballot_sync(0xffffffffu, alive), bs = __ballot_sync(0xffffffffu, side);
  unsigned lt = (1u << lane) - 1u;
  if (lane == 0) { s_wx[wid] = __popc(ba); s_wy[wid] = __popc(bs); }
  __syncthreads();
  uint32_t ra = __popc(ba & lt), rs = __popc(bs & lt);
  for (int w = 0; w < wid; ++w) { ra += s_wx[w]; rs += s_wy[w]; }
  const uint2 off = qb.tile_offsets[tile];
  RayRec* out = qb.q[emission ? 0u : (parity ^ 1u)];
  if (alive) {
    uint32_t dst = off.x + ra;
    if (dst < qb.capacity) out[dst] = qb.stage[slot];
    else flag_error(st, kErrQueueCapacity);
  }
  if (side) {
    if (kMode == 0) {
      uint64_t dst = (uint64_t)st->photon_base + off.y + rs;
      if (dst < ps.capacity) {
        ps.a[dst] = ps.sa[slot];
        ps.b[dst] = ps.sb[slot];
        ps.c[dst] = ps.sc[slot];
      }
    } else {
      ev.list[off.y + rs] = ev.stage[slot];
    }
  }
}

__global__ void k_advance(RunState* st, uint32_t by) {
  if (threadIdx.x == 0 && blockIdx.x == 0) st->seed_cursor += by;
}

// --------------------------------------------------------------- photons
// launchRayGenEmitterKernel (PrimalKernels.cpp:13-62).
__global__ void k_photon_emit(PhotonArgs A) {
  const uint32_t g = blockIdx.x * kBlock + threadIdx.x;
  bool alive = false;
  if (g < A.photons_per_launch) {
    const uint64_t base = A.seeds[A.st->seed_cursor];
    Rng r(per_item_seed(base, g));
    V3 pos, nrm, dir, pw;
    if (A.scene.lights.count > 0 && sample_light(A.scene, r, pos, nrm, dir, pw)) {
      V3 thr = scale(scale(pw, (float)A.scene.lights.count), A.inv_emitted);
      A.qb.stage[g] = make_ray(pos, dir, thr, g, 0u, 0u);
      alive = true;
    }
    A.qb.flags[g] = alive ? 1 : 0;
  }
  uint32_t c = __syncthreads_count(alive);
  if (threadIdx.x == 0) A.qb.tile_counts[blockIdx.x] = make_uint2(c, 0u);
}

// launchIntersectKernel for the photon pass (PrimalKernels.cpp:65-321).
__global__ void __launch_bounds__(kBlock) k_photon_bounce(PhotonArgs A, uint32_t parity) {
  extern __shared__ TravNode s_top[];
  const uint32_t n_in = A.st->active[parity];
  if ((uint64_t)blockIdx.x * kBlock >= n_in) return;
  stage_top_nodes(A.scene, s_top);
  const uint32_t slot = blockIdx.x * kBlock + threadIdx.x;
  bool alive = false, dep = false;
  TraceCounters ctr{0, 0};
  if (slot < n_in) {
    const SceneView& S = A.scene;
    const uint64_t base = A.seeds[A.st->seed_cursor];
    Rng r(per_item_seed(base, slot));
    const RayRec ry = A.qb.q[parity][slot];
    const V3 o = xyz(ry.o), d = xyz(ry.d), thr = xyz(ry.t);
    const uint32_t path = __float_as_uint(ry.o.w), bounce = __float_as_uint(ry.d.w) + 1u;
    Hit h = intersect_scene(S, s_top, o, d, ctr, A.st);
    if (h.inst >= 0) {
      V3 no, nd, nt;
      if (h.inst < (int)S.mesh.instances) {
        V3 nrm = hit_normal(S, h);
        // depositPhotonSurface (KernelHelpers.h:1688-1727)
        dep = true;
        A.ps.sa[slot] = f4(h.pos, thr.x);
        A.ps.sb[slot] = f4(d, thr.y);
        A.ps.sc[slot] = thr.z;
        const float4 mat = __ldg(&S.mesh.materials[__ldg(&S.mesh.material[h.inst])]);
        float pdf;
        sample_cosine(r, nrm, nd, pdf);
        no = h.pos + scale(nrm, 1e-6f);
        nt = mul(thr, xyz(mat));
        alive = russian_roulette(r, bounce, nt, A.rr_start);
      } else {
        const float4 cn4 = __ldg(&S.sf.cn[h.prim]);
        const float4 n4 = __ldg(&S.sf.n[h.prim]);
        const float opacity = n4.w;
        float u = r.next_float();
        if (u < A.q_null) {
          float att = 1.0f - h.alpha * opacity;
          float w = att / A.q_null;
          no = h.pos + scale(d, 1e-5f);
          nd = d;
          nt = scale(thr, w);
          alive = russian_roulette(r, bounce, nt, A.rr_start);
        } else if (u < A.q_null + A.q_reflect) {
          V3 cn = xyz(cn4);
          float sc = dot(cn, -d);
          V3 on = scale(cn, (float)(sc >= 0.0f ? 1 : -1));
          dep = true;
          V3 pw = divs(thr, A.q_reflect);
          A.ps.sa[slot] = f4(h.pos, pw.x);
          A.ps.sb[slot] = f4(d, pw.y);
          A.ps.sc[slot] = pw.z;
          float pdf;
          sample_uniform_hemi(r, on, nd, pdf);
          float ct = fmaxf(0.0f, dot(nd, on));
          const float4 al = __ldg(&S.sf.alb[h.prim]);
          V3 fs = scale(scale(xyz(al), al.w), kInvPi);
          float alpha = h.alpha * opacity;
          V3 w = divs(scale(scale(fs, alpha / A.q_reflect), ct), pdf);
          no = h.pos + scale(on, 1e-5f);
          nt = mul(thr, w);
          alive = russian_roulette(r, bounce, nt, A.rr_start);
        } else if (u < A.q_null + A.q_reflect + A.q_transmit) {
          V3 cn = xyz(cn4);
          float sc = dot(cn, -d);
          V3 on = scale(cn, (float)(sc >= 0.0f ? 1 : -1));
          float pdf;
          sample_uniform_hemi(r, on, nd, pdf);
          float ct = fmaxf(0.0f, dot(nd, on));
          const float4 al = __ldg(&S.sf.alb[h.prim]);
          V3 fs = scale(scale(xyz(al), 0.0f), kInvPi);   // alpha_t = 0
          float alpha = h.alpha * opacity;
          V3 w = divs(scale(scale(fs, alpha / A.q_reflect), ct), pdf);
          no = h.pos + scale(-on, 1e-5f);
          nt = mul(thr, w);
          alive = russian_roulette(r, bounce, nt, A.rr_start);
        }
      }
      if (alive) A.qb.stage[slot] = make_ray(no, nd, nt, path, bounce, 0u);
    }
    A.qb.flags[slot] = (alive ? 1 : 0) | (dep ? 2 : 0);
  }
  block_count3(&A.st->photon_segments, slot < n_in ? 1u : 0u, &A.st->node_visits, ctr.nodes, &A.st->surfel_tests,
               ctr.tests);
  uint32_t ca = __syncthreads_count(alive), cd = __syncthreads_count(dep);
  if (threadIdx.x == 0) A.qb.tile_counts[blockIdx.x] = make_uint2(ca, cd);
}

// Dynamic shared memory of a traversal kernel: the staged top nodes, then
// PALE_SMEM_STACK stack entries (8 B) per thread of the block.
static size_t top_smem(const SceneView& s) {
  return (size_t)s.top_nodes * sizeof(TravNode) + (size_t)PALE_SMEM_STACK * kBlock * sizeof(uint2);
}
static size_t top_smem(const SceneTable& t, int threads = kBlock) {
  return (size_t)t.n * t.staged * sizeof(TravNode) + (size_t)PALE_SMEM_STACK * threads * sizeof(uint2);
}

// Launch of a persistent walk kernel with the block size `threads` (64,
// 128 or 256): one resident wave of blocks (occupancy x SMs), at most
// `limit` blocks of 256-thread equivalents.
template <typename KernelT, typename Args>
static void launch_walk(KernelT kernel, int threads, const Args& a, uint32_t arg, size_t smem, uint32_t limit,
                        cudaStream_t s) {
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // the staged nodes of a call of several scenes and the shared stack reach
  // 48 KB, and the kernel's own static shared memory comes on top: allow
  // the dynamic part past the default limit
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
  const uint64_t grid = std::min<uint64_t>((uint64_t)limit * (kBlock / threads),
                                           (uint64_t)std::max(1, sms * std::max(1, per_sm)));
  kernel<<<(uint32_t)std::max<uint64_t>(1, grid), threads, smem, s>>>(a, arg);
  note_launch();
}

void photon_emit(const PhotonArgs& a, cudaStream_t s) {
  const uint32_t nb = blocks_for(a.photons_per_launch);
  if (nb == 0) return;
  k_photon_emit<<<nb, kBlock, 0, s>>>(a); note_launch();
  k_queue_scan<<<1, 1024, 0, s>>>(a.st, a.qb.tile_counts, a.qb.tile_offsets, 0, 1, a.photons_per_launch, 0,
                                  a.ps.capacity); note_launch();
  k_queue_scatter<0><<<nb, kBlock, 0, s>>>(a.st, a.qb, 0, 1, a.photons_per_launch, a.ps, EventBufs{}); note_launch();
}

void photon_bounce(const PhotonArgs& a, uint32_t parity, cudaStream_t s) {
  const uint32_t nb = blocks_for(a.qb.capacity);
  k_photon_bounce<<<nb, kBlock, top_smem(a.scene), s>>>(a, parity); note_launch();
  k_queue_scan<<<1, 1024, 0, s>>>(a.st, a.qb.tile_counts, a.qb.tile_offsets, parity, 0, 0, 0, a.ps.capacity); note_launch();
  k_queue_scatter<0><<<nb, kBlock, 0, s>>>(a.st, a.qb, parity, 0, 0, a.ps, EventBufs{}); note_launch();
}

// ------------------------------------------------------------ photon grid
__global__ void k_stored(RunState* st, uint64_t cap, uint32_t* d_stored, uint32_t* d_attempts) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    uint64_t a = st->photon_attempts;
    *d_stored = (uint32_t)(a < cap ? a : cap);
    *d_attempts = (uint32_t)a;
  }
}

// computePhotonCellIdsAndPermutation + countPhotonsPerCell
// (PrimalKernels.cpp:796-855).
__global__ void k_cell_ids(GridView G, const float4* __restrict__ pa, const uint32_t* __restrict__ d_stored,
                           uint32_t* __restrict__ cell_id, uint32_t* __restrict__ sort_keys,
                           uint32_t* __restrict__ sorted, uint32_t* __restrict__ cell_count) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= *d_stored) return;
  int c[3];
  world_to_cell(G, xyz(pa[i]), c);
  uint32_t id = (uint32_t)((c[2] * G.res[1] + c[1]) * G.res[0] + c[0]);
  cell_id[i] = id;
  sort_keys[i] = id;
  sorted[i] = i;
  atomicAdd(&cell_count[id], 1u);
}

__global__ void k_gather_sorted(const uint32_t* __restrict__ sorted, const uint32_t* __restrict__ d_stored,
                                const float4* __restrict__ a, const float4* __restrict__ b,
                                const float* __restrict__ c, float4* __restrict__ sa, float4* __restrict__ sb,
                                float* __restrict__ sc) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= *d_stored) return;
  uint32_t j = sorted[i];
  sa[i] = a[j];
  sb[i] = b[j];
  sc[i] = c[j];
}

void grid_build(const SceneView& sv, RunState* st, const PhotonStore& ps, const GridBufs& g, uint32_t cells,
                int key_bits, cudaStream_t s) {
  const uint32_t cap = (uint32_t)ps.capacity;
  k_stored<<<1, 32, 0, s>>>(st, ps.capacity, g.d_stored, g.d_attempts); note_launch();
  cudaMemsetAsync(g.cell_count, 0, ((size_t)cells + 1) * 4, s);
  uint32_t* sort_keys = g.keys_tmp;            // first half: keys, second: ping-pong
  uint32_t* sort_keys_tmp = g.keys_tmp + cap;
  k_cell_ids<<<blocks_for(cap), kBlock, 0, s>>>(sv.grid, ps.a, g.d_stored, g.cell_id, sort_keys, g.sorted,
                                                g.cell_count); note_launch();
  exclusive_scan(g.cell_count, g.cell_off, cells + 1, g.scan_temp, nullptr, s);
  radix_sort_pairs(sort_keys, g.sorted, sort_keys_tmp, g.vals_tmp, g.d_stored, cap, key_bits, g.sort_temp, s);
  k_gather_sorted<<<blocks_for(cap), kBlock, 0, s>>>(g.sorted, g.d_stored, ps.a, ps.b, ps.c, g.pa, g.pb, g.pc); note_launch();
}

// ---------------------------------------------------------- primary rays
// makePrimaryRayFromPixelJitteredFov (KernelHelpers.h:764-796).
__device__ __forceinline__ void primary_ray(const CameraRec& C, float px, float py, float jx, float jy, V3& o,
                                            V3& d) {
  float u = (px + 0.5f + jx);
  float v = (py + 0.5f + jy);
  float vf = C.height - v;
  float ndcX = (2.0f * u / C.width - 1.0f);
  float ndcY = (2.0f * vf / C.height - 1.0f);
  V3 dc = normalize(v3(ndcX * C.half_w / C.fx, ndcY * C.half_h / C.fy, -1.0f));
  d = xform_dir(C.inv_view, dc);
  float h[4];
  m4mul(C.inv_view, 0.f, 0.f, 0.f, 1.f, h);
  float invW = 1.f / h[3];
  o = v3(h[0] * invW, h[1] * invW, h[2] * invW);
}

// -------------------------------------------------------- camera gather
// launchCameraGatherKernel (PrimalKernels.cpp:500-653) as a wavefront.  A
// camera path is one (pixel, gather pass); it walks the surfel layers of its
// ray front to back, compositing L += T*alpha*Lo, T *= 1 - alpha, until a
// mesh (emitter or diffuse lookup) or a miss ends it.  The reference traces
// every layer from the root: the closest hit from the previous hit point
// advanced by 1e-4.  Here one traversal per round collects the K closest
// surfels and the round walks them in order, re-intersecting each from the
// chained origin exactly as that layer's trace would (the first is that
// trace's own hit; a surfel that is not hit from the chained origin, e.g.
// within 1e-4 behind the previous layer, is passed over as the layered walk
// passes over it); a round that used all K continues from the last one.
// Every layer's photon lookup becomes a record; k_cg_lookup gives each
// record a warp, and k_cg_compose adds a path's contributions in layer order,
// so the sums are the layered walk's.  The walk draws no random numbers, so
// queue order does not matter.  Each finished path writes its radiance to
// res[path]; k_cg_finalize then adds the passes of a pixel in pass order,
// cur + fb, as the reference's sequence of launches does, and applies
// launchPostProcessKernel (PostprocessKernel.cpp:11-106).

__device__ __forceinline__ uint32_t find_camera(const FrameArgs& A, uint32_t gp) {
  return view_of_pixel(A.cams, A.ncams, gp);
}

// The view of chunk path `path`: the last view whose first path of the
// chunk is <= path.  view_start is non-decreasing; a view without a pass in
// the chunk has an empty range (its start is the next view's), so the last
// view at or below `path` is the one that holds it.
__device__ __forceinline__ uint32_t view_of_path(const FrameArgs& A, uint32_t path) {
  uint32_t lo = 0, hi = A.ncams - 1;
  while (lo < hi) {
    const uint32_t mid = (lo + hi + 1) >> 1;
    if (A.view_start[mid] <= path) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Primary rays of the chunk: view v's pass p at paths view_start[v] +
// (p - p0(v)) * pixels(v) + pixel.
__global__ void k_cg_init(FrameArgs A, uint32_t n) {
  const uint32_t path = blockIdx.x * kBlock + threadIdx.x;
  if (path == 0) A.counts[0] = n;
  if (path == 0 && A.vs.base) {
    A.vs.base[0] = A.vs.rec_start;
    A.vs.base[kVertexBases] = A.vs.ent_start;
    *A.vs.overflow = 0u;
  }
  if (path >= n) return;
  const uint32_t v = view_of_path(A, path);
  const CameraRec& C = A.cams[v];
  const uint32_t npix = C.w * C.h;
  const uint32_t local = path - A.view_start[v];
  const uint32_t pass = A.view_start[A.ncams + v] + local / npix, pix = local % npix;
  const SceneSeeds& SS = A.sseeds[C.scene];
  const uint64_t cseed = SS.seeds[*SS.cursor + C.seed_slot];
  const uint64_t base = A.rng_mode == 1 ? per_item_seed(cseed, pass) : cseed;
  Rng r(per_item_seed(base, pix));
  float jx = r.next_float() - 0.5f, jy = r.next_float() - 0.5f;
  V3 o, d;
  primary_ray(C, (float)(pix % C.w), (float)(pix / C.w), jx, jy, o, d);
  RayRec rec;
  rec.o = make_float4(o.x, o.y, o.z, __uint_as_float(path));
  rec.d = make_float4(d.x, d.y, d.z, 1.0f);
  rec.t = make_float4(0.f, 0.f, 0.f, 0.f);
  A.paths[0][path] = rec;
}

// Lookup record (2 x float4): (position, weight) (lookup normal, index |
// kind << 30), weight = T * alpha for a surfel layer, T for the diffuse mesh
// that ends a path.  k_cg_lookup overwrites the first float4 with the
// layer's radiance contribution.  Unused slots of an entry's range are
// kRecNone with zero contribution.
// The index word also holds the record's scene: index (27 bits) | scene
// << 27 | kind << 30.
enum : uint32_t { kRecSurfel = 0, kRecMesh = 1, kRecNone = 2 };
constexpr uint32_t kRecIndexMask = 0x07FFFFFFu;

__device__ __forceinline__ void put_record(float4* q, uint32_t r, V3 pos, float w, V3 nrm, uint32_t idx,
                                           uint32_t kind, uint32_t sid) {
  q[2 * (size_t)r] = make_float4(pos.x, pos.y, pos.z, w);
  q[2 * (size_t)r + 1] = make_float4(nrm.x, nrm.y, nrm.z, __uint_as_float(idx | (sid << 27) | (kind << 30)));
}

// Vertex-store slot of record / entry `i` of round `round` (kInvalid when
// the store is not written or the slot lies past its capacity).
__device__ __forceinline__ uint32_t vs_rec_slot(const FrameArgs& A, uint32_t round, uint32_t i) {
  if (!A.vs.write) return kInvalid;
  const uint64_t g = (uint64_t)A.vs.base[round] + i;
  if (g >= A.vs.rec_cap) {
    atomicOr(A.vs.overflow, 1u);
    return kInvalid;
  }
  return (uint32_t)g;
}

__device__ __forceinline__ uint32_t vs_ent_slot(const FrameArgs& A, uint32_t round, uint32_t i) {
  if (!A.vs.write) return kInvalid;
  const uint64_t g = (uint64_t)A.vs.base[kVertexBases + round] + i;
  if (g >= A.vs.ent_cap) {
    atomicOr(A.vs.overflow, 1u);
    return kInvalid;
  }
  return (uint32_t)g;
}

// Round step 1: one lane per queue entry (a live path).
// Round step 1a: the mesh pass of every queue entry (one thread per entry):
// its closest mesh hit and its surfel walk's record, whose limit is the
// mesh distance plus intersect_scene's margin.
__global__ void k_cg_mesh(FrameArgs A, uint32_t round) {
  const uint32_t n = A.counts[round];
  if (blockIdx.x == 0 && threadIdx.x == 0) A.st->walk_next = 0u;
  const RayRec* __restrict__ in = A.paths[round & 1];
  for (uint32_t slot = blockIdx.x * kBlock + threadIdx.x; slot < n; slot += gridDim.x * kBlock) {
    const float4 ro = in[slot].o;
    const uint32_t sid = A.cams[view_of_path(A, __float_as_uint(ro.w))].scene;
    const SceneView& S = A.scenes.s[sid];
    const V3 o = xyz(ro), d = xyz(in[slot].d);
    const V3 invw = safe_inv(d);
    float best_m;
    const Hit hm = intersect_meshes(S, o, d, invw, best_m);
    float limit = -1.0f;
    if (S.has_pc && S.node_count > 0 &&
        entered(slab_entry(o, invw, S.pc_lo.x, S.pc_lo.y, S.pc_lo.z, S.pc_hi.x, S.pc_hi.y, S.pc_hi.z, best_m),
                best_m))
      limit = best_m < 3.0e38f ? best_m * 1.00001f + 1e-6f : __int_as_float(0x7f800000);
    A.mhit[slot] = make_float4(hm.pos.x, hm.pos.y, hm.pos.z, __int_as_float(hm.inst));
    const V3 dd = normalize(d);
    A.walk[2 * (size_t)slot] = make_float4(o.x, o.y, o.z, limit);
    A.walk[2 * (size_t)slot + 1] = make_float4(dd.x, dd.y, dd.z, __uint_as_float(sid));
  }
}

// Round step 1b: the K-closest-surfel walks, on a persistent grid whose
// lanes take the next queue entries every kRefillSteps node visits once
// their walk has ended (as k_adj_walk does for the adjoint's closest hits).
// A walk ends with one store of its hit count and surfels.
// kMulti: the call renders several scenes (each lane's scene from its walk
// record); a one-scene call reads the table's first entry, whose fields the
// compiler takes straight from the kernel parameters.
// kThreads: threads per block (the autotuner's choice of 64, 128 or 256);
// the register budget per thread stays the one of kRoundMinBlocks blocks
// of kBlock threads.
template <int K, bool kMulti, int kThreads>
__global__ void __launch_bounds__(kThreads, kRoundMinBlocks * (kBlock / kThreads))
    k_cg_walk(FrameArgs A, uint32_t round) {
  extern __shared__ TravNode s_top[];
  stage_top_nodes(A.scenes, s_top);
  const uint32_t n = A.counts[round];
  const int lane = threadIdx.x & 31;
  TravStack stk(s_top, A.scenes.n * A.scenes.staged);
#if PALE_KHIT_SMEM
  KHitWalkS<K> w;
  // the hit lists after the staged nodes and the shared part of the stacks
  w.bind(reinterpret_cast<uint2*>(s_top + A.scenes.n * A.scenes.staged) + (size_t)PALE_SMEM_STACK * kThreads +
         threadIdx.x);
#else
  KHitWalk<K> w;
#endif
  TraceCounters ctr{0, 0};
  uint32_t sid = 0;          // scene of this lane's walk
  uint32_t cur = kInvalid;   // queue entry of this lane's walk
  bool more = true;          // uniform in the warp: the cursor has entries left
  for (;;) {
    const unsigned need = __ballot_sync(0xffffffffu, cur == kInvalid);
    if (need && more) {
      const int leader = __ffs(need) - 1;
      uint32_t b0 = 0;
      if (lane == leader) b0 = atomicAdd(&A.st->walk_next, (uint32_t)__popc(need));
      b0 = __shfl_sync(0xffffffffu, b0, leader);
      if ((uint64_t)b0 + __popc(need) >= n) more = false;
      if (cur == kInvalid) {
        const uint32_t t = b0 + __popc(need & ((1u << lane) - 1u));
        if (t < n) {
          const float4 wa = A.walk[2 * (size_t)t], wb = A.walk[2 * (size_t)t + 1];
          if (wa.w >= 0.0f) {
            cur = t;
            if (kMulti) sid = __float_as_uint(wb.w);
            w.init(xyz(wa), xyz(wb), 1e-5f, wa.w);
          }
        }
      }
    }
    if (!__any_sync(0xffffffffu, cur != kInvalid)) {
      if (!more) break;
      continue;
    }
    for (int it = 0; it < kRefillSteps; ++it) {
      if (!__any_sync(0xffffffffu, cur != kInvalid)) break;
      const uint32_t sc = kMulti ? sid : 0u;
      if (warp_step(w, cur != kInvalid, A.scenes.s[sc], s_top + sc * A.scenes.staged, stk, ctr, A.st) ||
          cur == kInvalid)
        continue;
      uint32_t rw[kKHitWords];
      rw[0] = w.count;
#pragma unroll
#if PALE_KHIT_SMEM
      for (int k = 0; k < K; ++k) rw[1 + k] = w.prim(k);
#else
      for (int k = 0; k < K; ++k) rw[1 + k] = w.prim_out[k];
#endif
#pragma unroll
      for (int k = K + 1; k < kKHitWords; ++k) rw[k] = 0u;
      uint4* dst = reinterpret_cast<uint4*>(A.khit + (size_t)kKHitWords * cur);
#pragma unroll
      for (int q = 0; q < kKHitWords / 4; ++q) dst[q] = make_uint4(rw[4 * q], rw[4 * q + 1], rw[4 * q + 2], rw[4 * q + 3]);
      cur = kInvalid;
    }
  }
  warp_count(&A.st->node_visits, ctr.nodes);
  warp_count(&A.st->surfel_tests, ctr.tests);
  warp_count(&A.st->gather_node_visits, ctr.nodes);
  warp_count(&A.st->gather_surfel_tests, ctr.tests);
}

// Round step 1c: the layers of each entry from its walk's hits, re-tested
// from the chained origin, and the path's end.
template <int K>
__global__ void __launch_bounds__(kBlock, kTraceMinBlocks) k_cg_round(FrameArgs A, uint32_t round) {
  const uint32_t n = A.counts[round];
  const RayRec* __restrict__ in = A.paths[round & 1];
  RayRec* __restrict__ out = A.paths[(round + 1) & 1];
  const int lane = threadIdx.x & 31;
  const float inf = __int_as_float(0x7f800000);
  uint32_t segs = 0;
  for (uint32_t b = blockIdx.x * kBlock; b < n; b += gridDim.x * kBlock) {
    const uint32_t slot = b + threadIdx.x;
    const bool live = slot < n;
    RayRec rec{};
    uint32_t pl[K];
#pragma unroll
    for (int k = 0; k < K; ++k) pl[k] = 0;
    uint32_t count = 0, nslots = 0;
    Hit hm{};
    hm.inst = -1;
    V3 o{}, d{}, invw{}, dd{};
    uint32_t sid = 0;
    if (live) {
      rec = in[slot];
      sid = __float_as_uint(A.walk[2 * (size_t)slot + 1].w);
      o = xyz(rec.o);
      d = xyz(rec.d);
      invw = safe_inv(d);
      const float4 mh = A.mhit[slot];
      hm.inst = __float_as_int(mh.w);
      hm.pos = xyz(mh);
      if (A.walk[2 * (size_t)slot].w >= 0.0f) {
        dd = normalize(d);
        uint32_t rw[kKHitWords];
        const uint4* src = reinterpret_cast<const uint4*>(A.khit + (size_t)kKHitWords * slot);
#pragma unroll
        for (int q = 0; q < kKHitWords / 4; ++q) {
          const uint4 v = src[q];
          rw[4 * q] = v.x;
          rw[4 * q + 1] = v.y;
          rw[4 * q + 2] = v.z;
          rw[4 * q + 3] = v.w;
        }
        count = rw[0];
#pragma unroll
        for (int k = 0; k < K; ++k) pl[k] = rw[1 + k];
      }
      nslots = count + (count < (uint32_t)K ? 1u : 0u);
    }
    // record range of this entry: warp scan of the slot counts, one atomic
    uint32_t incl = nslots;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t v = __shfl_up_sync(0xffffffffu, incl, off);
      if (lane >= off) incl += v;
    }
    const uint32_t wtotal = __shfl_sync(0xffffffffu, incl, 31);
    uint32_t base = 0;
    if (lane == 0 && wtotal) base = atomicAdd(&A.counts[kMaxLayers + 2 + round], wtotal);
    base = __shfl_sync(0xffffffffu, base, 0);
    const uint32_t first = base + incl - nslots;

    bool cont = false;
    uint32_t flags = 0;
    V3 c_em = v3(0.f, 0.f, 0.f);
    V3 oc = o;
    float T = rec.d.w;
    uint32_t layer = __float_as_uint(rec.t.w);
    uint32_t used = 0;
    const SceneView& S = A.scenes.s[sid];
    if (live) {
      bool ended = false, mesh_first = false;
      for (uint32_t i = 0; i < count && !ended; ++i) {
        float th, a;
        V3 x;
        if (!surfel_hit(S.sf, pl[i], oc, dd, 1e-5f, inf, th, x, a)) continue;
        // the mesh wins when it is nearer than this surfel from the chained origin
        const float tw = dot(x - oc, d);
        const float tm = hm.inst >= 0 ? dot(hm.pos - oc, d) : inf;
        if (!(tw > 0.0f && tw < tm)) {
          mesh_first = true;
          break;
        }
        ++segs;
        const float ae = __ldg(&S.sf.n[pl[i]]).w * a;
        V3 nrm = xyz(__ldg(&S.sf.cn[pl[i]]));
        if (dot(nrm, -d) < 0.0f) nrm = -nrm;
        put_record(A.qrec, first + used, x, T * ae, nrm, pl[i], kRecSurfel, sid);
        const uint32_t vr = vs_rec_slot(A, round, first + used);
        if (vr != kInvalid) A.vs.rec_xa[vr] = make_float4(x.x, x.y, x.z, a);
        ++used;
        T *= (1.0f - ae);
        if (layer + 1 >= (uint32_t)kMaxLayers) {
          flag_error(A.st, kErrLayerCap);
          ended = true;
          break;
        }
        ++layer;
        oc = x + scale(d, 1e-4f);
      }
      if (!ended) {
        if (count == (uint32_t)K && !mesh_first) {
          cont = true;   // more surfels may lie beyond the K-th
        } else {
          // the layer that ends the path, traced from the chained origin
          ++segs;
          float bm;
          const Hit h2 = intersect_meshes(S, oc, d, invw, bm);
          if (h2.inst >= 0) {
            const uint32_t mi = __ldg(&S.mesh.material[h2.inst]);
            const float4 mat = __ldg(&S.mesh.materials[mi]);
            if (mat.w > 0.f) {
              V3 Le = scale(xyz(mat), mat.w);
              Le = v3(fminf(Le.x, 1.0f), fminf(Le.y, 1.0f), fminf(Le.z, 1.0f));
              c_em = scale(Le, T);
              flags = 1;
              const uint32_t ve = vs_ent_slot(A, round, slot);
              if (ve != kInvalid) A.vs.ent_l[ve] = make_float4(Le.x, Le.y, Le.z, 0.f);
            } else {
              put_record(A.qrec, first + used, h2.pos, T, hit_normal(S, h2), mi, kRecMesh, sid);
              ++used;
            }
          }
        }
      }
      for (uint32_t r = used; r < nslots; ++r)
        put_record(A.qrec, first + r, v3(0.f, 0.f, 0.f), 0.f, v3(0.f, 0.f, 0.f), 0u, kRecNone, 0u);
      A.info_b[slot] = make_float4(c_em.x, c_em.y, c_em.z, 0.f);
    }
    // next-round queue entries for the paths that continue
    const unsigned cb = __ballot_sync(0xffffffffu, cont);
    uint32_t nbase = 0;
    if (cb) {
      if (lane == __ffs(cb) - 1) nbase = atomicAdd(&A.counts[round + 1], (uint32_t)__popc(cb));
      nbase = __shfl_sync(0xffffffffu, nbase, __ffs(cb) - 1);
    }
    if (live) {
      uint32_t next = kInvalid;
      if (cont) {
        next = nbase + __popc(cb & ((1u << lane) - 1u));
        RayRec nr;
        nr.o = make_float4(oc.x, oc.y, oc.z, rec.o.w);
        nr.d = make_float4(d.x, d.y, d.z, T);
        nr.t = make_float4(0.f, 0.f, 0.f, __uint_as_float(layer));   // radiance added by k_cg_compose
        out[next] = nr;
      }
      A.info_a[slot] = make_uint4(first, nslots | (flags << 8), __float_as_uint(rec.o.w), next);
      const uint32_t ve = vs_ent_slot(A, round, slot);
      if (ve != kInvalid) {
        // the entry's first record and the next round's entry as store slots
        const uint32_t rb = A.vs.base[round], eb = A.vs.base[kVertexBases + round];
        A.vs.ent_d[ve] = rec.d;
        A.vs.ent_b[ve] = make_uint4(rb + first, used | (flags << 8), next != kInvalid ? eb + n + next : kInvalid,
                                    __float_as_uint(rec.o.w));
      }
    }
  }
  warp_count(&A.st->gather_segments, segs);
}

// Round step 2: one warp per lookup record (warps stride over the records,
// so in deep rounds every lookup has a warp of its own).  Lane 0 writes the
// layer's contribution Lo * weight over the record's first float4.
template <bool kMulti>
__global__ void __launch_bounds__(kBlock, kLookupMinBlocks) k_cg_lookup(FrameArgs A, uint32_t round) {
  __shared__ float4 s_terms[kBlock];
  __shared__ GatherConst s_gc[kMaxScenes];
  if (threadIdx.x < A.scenes.n) s_gc[threadIdx.x] = gather_const(A.scenes.s[threadIdx.x].grid);
  __syncthreads();
  const uint32_t n = A.counts[kMaxLayers + 2 + round];
  const int lane = threadIdx.x & 31;
  float4* terms = s_terms + (threadIdx.x & ~31u);
  const uint32_t warps = gridDim.x * (kBlock / 32);
  uint32_t queries = 0, scanned = 0;
  // lanes 0-7 hold the 8 floats of the next record, loaded one record ahead
  uint32_t i = blockIdx.x * (kBlock / 32) + (threadIdx.x >> 5);
  float pre = (i < n && lane < 8) ? reinterpret_cast<const float*>(A.qrec + 2 * (size_t)i)[lane] : 0.f;
  for (; i < n; i += warps) {
    const float cur = pre;
    if (i + warps < n && lane < 8) pre = reinterpret_cast<const float*>(A.qrec + 2 * (size_t)(i + warps))[lane];
    auto field = [&](int f) { return __shfl_sync(0xffffffffu, cur, f); };
    const float4 ra = make_float4(field(0), field(1), field(2), field(3));
    const float4 rb = make_float4(field(4), field(5), field(6), field(7));
    const uint32_t word = __float_as_uint(rb.w);
    const uint32_t kind = word >> 30, idx = word & kRecIndexMask, sid = kMulti ? (word >> 27) & 7u : 0u;
    if (kind == kRecNone) continue;
    const SceneView& S = A.scenes.s[sid];
    // the reflectance, loaded before the gather so that its latency overlaps it
    float4 refl = make_float4(0.f, 0.f, 0.f, 0.f);
    if (lane == 0) refl = kind == kRecSurfel ? __ldg(&S.sf.alb[idx]) : __ldg(&S.mesh.materials[idx]);
    uint32_t cnt = 0;
    const V3 E = gather_irradiance_warp<false>(S.grid, s_gc[sid], xyz(ra), xyz(rb), terms, cnt);
    if (lane == 0) {
      ++queries;
      scanned += cnt;
      V3 Lo;
      if (kind == kRecSurfel) {
        Lo = mul(E, scale(scale(xyz(refl), refl.w), kInvPi));
      } else {
        Lo = mul(scale(xyz(refl), kInvPi), E);
      }
      const V3 c = scale(Lo, ra.w);
      A.qrec[2 * (size_t)i] = make_float4(c.x, c.y, c.z, 0.f);
      const uint32_t vr = vs_rec_slot(A, round, i);
      if (vr != kInvalid) A.vs.rec_ew[vr] = make_float4(E.x, E.y, E.z, rb.w);
    }
  }
  warp_count(&A.st->gather_queries, queries);
  warp_count(&A.st->photons_scanned, scanned);
  warp_count(&A.st->gather_photons_scanned, scanned);
}

// Round step 3: one lane per entry adds its layers' contributions in order
// (then an emitter's), as the layered walk's acc = acc + c does, and hands
// the sum to the path's next-round entry or to res[path].
__global__ void k_cg_compose(FrameArgs A, uint32_t round) {
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e == 0 && A.vs.base) {
    // the next round's slots follow this round's records and entries
    A.vs.base[round + 1] = A.vs.base[round] + A.counts[kMaxLayers + 2 + round];
    A.vs.base[kVertexBases + round + 1] = A.vs.base[kVertexBases + round] + A.counts[round];
  }
  if (e >= A.counts[round]) return;
  const RayRec* __restrict__ in = A.paths[round & 1];
  RayRec* __restrict__ out = A.paths[(round + 1) & 1];
  const uint4 ia = A.info_a[e];
  V3 acc = xyz(in[e].t);
  const uint32_t nslots = ia.y & 0xFFu;
  for (uint32_t r = 0; r < nslots; ++r) acc = acc + xyz(A.qrec[2 * (size_t)(ia.x + r)]);
  if (ia.y & 0x100u) acc = acc + xyz(A.info_b[e]);
  if (ia.w != kInvalid) {
    out[ia.w].t = make_float4(acc.x, acc.y, acc.z, out[ia.w].t.w);
  } else {
    A.res[ia.z] = make_float4(acc.x, acc.y, acc.z, 0.f);
  }
}

// fb += res/passes over the view's passes of the chunk [p0(v), p1(v)), in
// pass order; the chunk that holds a view's last pass writes its RAW image
// and the post-processed LDR image.
__global__ void k_cg_finalize(FrameArgs A) {
  const uint32_t gp = blockIdx.x * kBlock + threadIdx.x;
  if (gp >= A.total_pixels) return;
  const uint32_t v = find_camera(A, gp);
  const CameraRec& C = A.cams[v];
  const uint32_t P = C.passes;
  const uint32_t p0 = A.view_start[A.ncams + v], p1 = A.view_start[2 * A.ncams + v];
  if (P == 0 || p0 >= p1) return;                   // no pass of this view in the chunk
  const uint32_t npix = C.w * C.h, pix = gp - C.pixel_offset;
  const bool last = p1 >= P;
  float4 f = p0 == 0 ? make_float4(0.f, 0.f, 0.f, 0.f) : A.fb[gp];
  float fb[4] = {f.x, f.y, f.z, f.w};
  const float inv = 1.f / (float)P;
  for (uint32_t p = p0; p < p1; ++p) {
    const float4 a = A.res[(size_t)A.view_start[v] + (size_t)(p - p0) * npix + pix];
    float cur[4] = {a.x * inv, a.y * inv, a.z * inv, 1.0f * inv};
#pragma unroll
    for (int k = 0; k < 4; ++k) fb[k] = cur[k] + fb[k];
  }
  if (!last) {
    A.fb[gp] = make_float4(fb[0], fb[1], fb[2], fb[3]);
    return;
  }
  const size_t o4 = 4 * (size_t)gp;
  if (A.raw) *reinterpret_cast<float4*>(A.raw + o4) = make_float4(fb[0], fb[1], fb[2], fb[3]);
  if (A.ldr || A.dldi) {
    float ig = (A.gamma > 0.0f) ? (1.0f / A.gamma) : 1.0f;
    float l[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float x = fb[c] * A.exposure;
      x = fmaxf(x, 0.0f);
      x = powf(x, ig);
      l[c] = clampf(x, 0.0f, 1.0f);
    }
    if (A.ldr) *reinterpret_cast<float4*>(A.ldr + o4) = make_float4(l[0], l[1], l[2], 1.0f);
    if (A.dldi) {
      // compute_l2_grad (python/losses.py:27-45) per camera: the residual
      // over the camera's number of RGB values, in float32
      const float size = (float)(3u * C.w * C.h);
      const float* t = A.target + (size_t)A.target_channels * gp;
      *reinterpret_cast<float4*>(A.dldi + o4) =
          make_float4((l[0] - t[0]) / size, (l[1] - t[1]) / size, (l[2] - t[2]) / size, 0.0f);
    }
  }
}

// compute_l2_loss (python/losses.py:10-24) per selected camera: block
// (chunk, camera) sums its strided share of the camera's squared RGB
// residuals in double; k_loss_final adds the chunks in order.
__global__ void k_loss_partials(FrameArgs A, double* __restrict__ partials) {
  __shared__ double s_part[kBlock / 32];
  const uint32_t ci = blockIdx.y;
  const CameraRec& C = A.cams[ci];
  const uint32_t npix = C.w * C.h;
  double acc = 0.0;
  for (uint32_t p = blockIdx.x * kBlock + threadIdx.x; p < npix; p += gridDim.x * kBlock) {
    const size_t gp = (size_t)C.pixel_offset + p;
    const float4 l = *reinterpret_cast<const float4*>(A.ldr + 4 * gp);
    const float* t = A.target + (size_t)A.target_channels * gp;
    const float d0 = l.x - t[0], d1 = l.y - t[1], d2 = l.z - t[2];
    acc += (double)(d0 * d0) + (double)(d1 * d1) + (double)(d2 * d2);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < kBlock / 32; ++w) s += s_part[w];
    partials[(size_t)ci * gridDim.x + blockIdx.x] = s;
  }
}

__global__ void k_loss_final(FrameArgs A, const double* __restrict__ partials, uint32_t chunks,
                             double* __restrict__ loss) {
  const uint32_t ci = blockIdx.x * blockDim.x + threadIdx.x;
  if (ci >= A.ncams) return;
  double s = 0.0;
  for (uint32_t k = 0; k < chunks; ++k) s += partials[(size_t)ci * chunks + k];
  const CameraRec& C = A.cams[ci];
  loss[ci] = 0.5 * s / (3.0 * (double)C.w * (double)C.h);
}

void image_loss(const FrameArgs& a, double* partials, double* loss, cudaStream_t s) {
  if (a.ncams == 0) return;
  k_loss_partials<<<dim3(kLossChunks, a.ncams), kBlock, 0, s>>>(a, partials); note_launch();
  k_loss_final<<<(a.ncams + 63) / 64, 64, 0, s>>>(a, partials, kLossChunks, loss); note_launch();
}

std::vector<GatherChunk> gather_chunks(const std::vector<CameraRec>& views, uint32_t path_capacity) {
  const size_t nv = views.size();
  std::vector<GatherChunk> out;
  GatherChunk cur;
  std::vector<uint32_t> p0(nv, 0u), p1(nv, 0u);
  std::vector<char> in(nv, 0);
  uint64_t used = 0;
  auto close = [&]() {
    cur.n = (uint32_t)used;
    cur.table.assign(3 * nv, 0u);
    // paths in view order; a view absent from the chunk gets an empty
    // range at the next view's start
    uint64_t acc = 0;
    for (size_t v = 0; v < nv; ++v) {
      cur.table[v] = (uint32_t)acc;
      if (in[v]) {
        cur.table[nv + v] = p0[v];
        cur.table[2 * nv + v] = p1[v];
        acc += (uint64_t)views[v].w * views[v].h * (p1[v] - p0[v]);
      }
    }
    out.push_back(cur);
    cur = GatherChunk{};
    std::fill(in.begin(), in.end(), 0);
    used = 0;
  };
  for (size_t v = 0; v < nv; ++v) {
    const uint64_t npix = (uint64_t)views[v].w * views[v].h;
    const uint32_t end = views[v].pass_end;
    uint32_t r = views[v].pass_begin;
    while (r < end) {
      uint64_t fit = used < path_capacity ? (path_capacity - used) / npix : 0;
      if (fit == 0) {
        if (used) {
          close();
          continue;
        }
        fit = 1;   // one pass of a view always goes
      }
      const uint32_t take = (uint32_t)std::min<uint64_t>(fit, end - r);
      in[v] = 1;
      p0[v] = r;
      p1[v] = r + take;
      used += npix * take;
      r += take;
      if (r < end) close();   // the chunk is full
    }
  }
  if (used) close();
  return out;
}

namespace {

// The launch shapes of the camera gather's kernels.
struct GatherShape {
  uint32_t grid_r = 1, grid_l = 1;
  int wt = kBlock;
  size_t smem = 0;
};

template <bool kMulti>
GatherShape gather_shape(const FrameArgs& a) {
  GatherShape g;
  // persistent grids: every SM filled once
  int dev = 0, sms = 148, per_sm_l = 1, per_sm_r = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  g.wt = a.walk_block == 64 || a.walk_block == 128 ? (int)a.walk_block : kBlock;
  g.smem = top_smem(a.scenes, g.wt) + (PALE_KHIT_SMEM ? (size_t)kGatherHits * g.wt * sizeof(uint2) : 0);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_r, k_cg_round<kGatherHits>, kBlock, 0);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_l, k_cg_lookup<kMulti>, kBlock, 0);
  g.grid_r = (uint32_t)std::max(1, sms * std::max(1, per_sm_r));
  g.grid_l = (uint32_t)std::max(1, sms * std::max(1, per_sm_l));
  return g;
}

// The rounds of one chunk of n paths (its view_start already on the
// device); returns the rounds run.
template <bool kMulti>
uint32_t gather_rounds(const FrameArgs& a, const GatherShape& g, uint32_t n, cudaStream_t s) {
  cudaMemsetAsync(a.counts, 0, 2 * (kMaxLayers + 2) * sizeof(uint32_t), s);
  k_cg_init<<<blocks_for(n), kBlock, 0, s>>>(a, n); note_launch();
  // every round consumes at least one layer of each live path, so
  // kMaxLayers rounds bound the walk (the layer cap ends longer ones)
  uint32_t round = 0, live = n;
  while (round < (uint32_t)kMaxLayers && live) {
    for (uint32_t group = 0; group < 16 && round < (uint32_t)kMaxLayers; ++group, ++round) {
      if (a.timer) a.timer->begin(kTimeTrace, s);
      k_cg_mesh<<<g.grid_r, kBlock, 0, s>>>(a, round); note_launch();
      if (g.wt == 64) launch_walk(k_cg_walk<kGatherHits, kMulti, 64>, 64, a, round, g.smem, ~0u, s);
      else if (g.wt == 128) launch_walk(k_cg_walk<kGatherHits, kMulti, 128>, 128, a, round, g.smem, ~0u, s);
      else launch_walk(k_cg_walk<kGatherHits, kMulti, 256>, 256, a, round, g.smem, ~0u, s);
      k_cg_round<kGatherHits><<<g.grid_r, kBlock, 0, s>>>(a, round); note_launch();
      if (a.timer) a.timer->end(s);
      if (a.timer) a.timer->begin(kTimeLookup, s);
      k_cg_lookup<kMulti><<<g.grid_l, kBlock, 0, s>>>(a, round); note_launch();
      if (a.timer) a.timer->end(s);
      // queues only shrink, so `live` bounds the entries of every round of the group
      k_cg_compose<<<blocks_for(live), kBlock, 0, s>>>(a, round); note_launch();
    }
    // the host reads the queue length after each group of 16 rounds
    cudaMemcpyAsync(&live, a.counts + round, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
  }
  return round;
}

template <bool kMulti>
void camera_gather_impl(const FrameArgs& a0, const std::vector<CameraRec>& views, uint32_t* d_view_start,
                        cudaStream_t s, VertexPlan* plan) {
  FrameArgs a = a0;
  a.view_start = d_view_start;
  const GatherShape g = gather_shape<kMulti>(a);
  const auto chunks = gather_chunks(views, a.path_capacity);
  if (plan) plan->chunks.assign(chunks.size(), VertexChunk{});
  uint32_t rec_used = 0, ent_used = 0;   // stored slots so far
  bool room = plan && plan->store;
  for (size_t c = 0; c < chunks.size(); ++c) {
    const uint32_t n = chunks[c].n;
    cudaMemcpyAsync(d_view_start, chunks[c].table.data(), chunks[c].table.size() * sizeof(uint32_t),
                    cudaMemcpyHostToDevice, s);
    if (plan) {
      // write the chunk after the stored ones while the store has room;
      // otherwise only count its slots
      a.vs.write = room ? 1 : 0;
      a.vs.rec_start = room ? rec_used : 0u;
      a.vs.ent_start = room ? ent_used : 0u;
    }
    const uint32_t rounds = gather_rounds<kMulti>(a, g, n, s);
    if (plan) {
      VertexChunk& vc = plan->chunks[c];
      vc.n = n;
      vc.rounds = rounds;
      vc.rec_start = a.vs.rec_start;
      vc.ent_start = a.vs.ent_start;
      vc.table = chunks[c].table;
      uint32_t tail[3] = {0, 0, 0};
      cudaMemcpyAsync(plan->d_chunk_base + c * 2 * kVertexBases, a.vs.base, 2 * kVertexBases * sizeof(uint32_t),
                      cudaMemcpyDeviceToDevice, s);
      cudaMemcpyAsync(&tail[0], a.vs.base + rounds, 4, cudaMemcpyDeviceToHost, s);
      cudaMemcpyAsync(&tail[1], a.vs.base + kVertexBases + rounds, 4, cudaMemcpyDeviceToHost, s);
      cudaMemcpyAsync(&tail[2], a.vs.overflow, 4, cudaMemcpyDeviceToHost, s);
      cudaStreamSynchronize(s);
      vc.recs = tail[0] - vc.rec_start;
      vc.ents = tail[1] - vc.ent_start;
      vc.stored = a.vs.write && tail[2] == 0u;
      if (vc.stored) {
        rec_used = tail[0];
        ent_used = tail[1];
      }
      // a chunk that did not fit leaves the store where it was: a later,
      // smaller chunk may still fit (its slots overwrite the dropped ones)
    }
    k_cg_finalize<<<blocks_for(a.total_pixels), kBlock, 0, s>>>(a); note_launch();
  }
}

}  // namespace

void camera_gather(const FrameArgs& a, const std::vector<CameraRec>& views, uint32_t* d_view_start,
                   cudaStream_t s, VertexPlan* plan) {
  if (a.total_pixels == 0 || views.empty()) return;
  if (a.scenes.n > 1) camera_gather_impl<true>(a, views, d_view_start, s, plan);
  else camera_gather_impl<false>(a, views, d_view_start, s, plan);
}

// ------------------------------------------------------------- adjoint
enum : uint32_t { kKindNone = 0, kKindNull = 1, kKindReflect = 2, kKindTransmit = 3, kKindProjection = 4 };

// launchRayGenAdjointKernel (AdjointKernels.cpp:15-84) + the per-spp
// reset of the pending states (SyclBridge.cpp:222), for every job of a batch.
__device__ __forceinline__ uint32_t find_job(const AdjointArgs& A, uint32_t path) {
  uint32_t lo = 0, hi = A.njobs - 1;
  while (lo < hi) {
    const uint32_t mid = (lo + hi + 1) >> 1;
    if (A.jobs[mid].path_start <= path) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ uint64_t adjoint_base(const AdjointArgs& A, uint32_t job, uint32_t word) {
  return A.rng_mode == 1 ? (uint64_t)A.seeds[A.jobs[job].seed_index + word] : (uint64_t)A.fixed_seed;
}

__global__ void k_adj_raygen(AdjointArgs A, uint32_t npaths) {
  const uint32_t path = blockIdx.x * kBlock + threadIdx.x;
  if (path == 0) A.st->active[0] = npaths;
  if (path < kMaxJobsPerBatch) {
    A.job_count[path] = 0u;
    A.job_count[kMaxJobsPerBatch + path] = 0u;
    A.job_start[path] = path < A.njobs ? A.jobs[path].path_start : 0u;
  }
  if (path >= npaths) return;
  const uint32_t job = find_job(A, path);
  const AdjJob J = A.jobs[job];
  const CameraRec& C = A.cams[J.cam];
  const uint32_t p = path - J.path_start;
  Rng r(per_item_seed(adjoint_base(A, job, 0), p));
  float jx = r.next_float() - 0.5f, jy = r.next_float() - 0.5f;
  V3 o, d;
  primary_ray(C, (float)(p % C.w), (float)(p / C.w), jx, jy, o, d);
  const uint32_t pixel = C.pixel_offset + p;
  const float4 g = *reinterpret_cast<const float4*>(A.dldi + 4 * (size_t)pixel);
  A.qb.q[0][path] = make_ray(o, d, v3(g.x, g.y, g.z), path, job << 8, pixel);
  A.pend.a[path] = make_float4(0.f, 0.f, 0.f, 0.f);
  A.pend.b[path] = make_float4(0.f, 0.f, 0.f, __uint_as_float(kKindNone));
  A.pend.c[path] = make_uint4(kInvalid, kInvalid, 0u, 0u);
}

// Queue start of every job after a compaction: exclusive scan of the
// survivor counts, which are cleared for the bounce after next.
__global__ void __launch_bounds__(kMaxJobsPerBatch) k_job_scan(AdjointArgs A, uint32_t parity) {
  __shared__ uint32_t s_w[32];
  uint32_t* cnt = A.job_count + (size_t)(parity ^ 1u) * kMaxJobsPerBatch;
  uint32_t* start = A.job_start + (size_t)(parity ^ 1u) * kMaxJobsPerBatch;
  const uint32_t j = threadIdx.x;
  const int lane = j & 31, wid = j >> 5;
  const uint32_t c = j < A.njobs ? cnt[j] : 0u;
  uint32_t x = c;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_w[wid] = x;
  __syncthreads();
  if (wid == 0) {
    uint32_t w = s_w[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    s_w[lane] = w;
  }
  __syncthreads();
  start[j] = (wid > 0 ? s_w[wid - 1] : 0u) + x - c;
  cnt[j] = 0u;
}

// Sort key of a queued ray: direction octant (3 bits) over the Morton code
// of its origin on a 512^3 lattice over the photon grid's box (27 bits).
__device__ __forceinline__ uint32_t spread9(uint32_t v) {
  v &= 0x1FFu;
  v = (v | (v << 16)) & 0x030000FFu;
  v = (v | (v << 8)) & 0x0300F00Fu;
  v = (v | (v << 4)) & 0x030C30C3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

// Sort key of a ray: (direction octant, 27-bit Morton code of the origin in
// its scene's grid box); with several scenes, (scene, octant, 24-bit Morton
// code), so that the rays of one scene stay together.
__global__ void k_adj_keys(AdjointArgs A, uint32_t parity) {
  const uint32_t t = blockIdx.x * kBlock + threadIdx.x;
  if (t >= A.st->active[parity]) return;
  const RayRec ry = A.qb.q[parity][t];
  const uint32_t sid = A.cams[A.jobs[__float_as_uint(ry.d.w) >> 8].cam].scene;
  const GridView& G = A.scenes.s[sid].grid;
  uint32_t q[3];
  const float o[3] = {ry.o.x, ry.o.y, ry.o.z}, lo[3] = {G.origin.x, G.origin.y, G.origin.z},
              ext[3] = {G.cell.x * G.res[0], G.cell.y * G.res[1], G.cell.z * G.res[2]};
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float f = (o[k] - lo[k]) / fmaxf(ext[k], 1e-30f) * 512.0f;
    q[k] = (uint32_t)fminf(fmaxf(f, 0.0f), 511.0f);
  }
  const uint32_t oct = (ry.d.x < 0.f ? 1u : 0u) | (ry.d.y < 0.f ? 2u : 0u) | (ry.d.z < 0.f ? 4u : 0u);
  const uint32_t morton = (spread9(q[0]) << 2) | (spread9(q[1]) << 1) | spread9(q[2]);
  A.sort_keys[t] = A.scenes.n > 1 ? (sid << 27) | (oct << 24) | (morton >> 3) : (oct << 27) | morton;
  A.perm[t] = t;
}

// Per 256-slot tile of the input queue: survivors and events, for the
// slot-ordered compaction.
__global__ void k_adj_tile_counts(AdjointArgs A, uint32_t parity) {
  const uint32_t n_in = A.st->active[parity];
  if ((uint64_t)blockIdx.x * kBlock >= n_in) return;
  const uint32_t slot = blockIdx.x * kBlock + threadIdx.x;
  const uint8_t f = slot < n_in ? A.qb.flags[slot] : 0;
  const uint32_t ca = __syncthreads_count(f & 1), ce = __syncthreads_count(f & 2);
  if (threadIdx.x == 0) A.qb.tile_counts[blockIdx.x] = make_uint2(ca, ce);
}

// intersectScene of the adjoint bounce (AdjointKernels.cpp:87-386 traces
// with it) in three steps: k_adj_mesh, k_adj_walk, and k_adj_bounce reading
// their records.  Step 1: the mesh pass of every ray, one thread per ray in
// the order of the bounce: the closest mesh hit, and the surfel walk's
// record with its limit (the mesh distance plus intersect_scene's margin)
// when the ray enters the surfel cloud's box before the mesh hit.
__global__ void k_adj_mesh(AdjointArgs A, uint32_t parity, int sorted) {
  const uint32_t n_in = A.st->active[parity];
  const uint32_t t = blockIdx.x * kBlock + threadIdx.x;
  if (t == 0) A.st->walk_next = 0u;
  if (t >= n_in) return;
  const uint32_t slot = sorted ? A.perm[t] : t;
  const float4 rd = A.qb.q[parity][slot].d;
  const uint32_t sid = A.cams[A.jobs[__float_as_uint(rd.w) >> 8].cam].scene;
  const SceneView& S = A.scenes.s[sid];
  const V3 o = xyz(A.qb.q[parity][slot].o), d = xyz(rd);
  const V3 invw = safe_inv(d);
  float best;
  const Hit h = intersect_meshes(S, o, d, invw, best);
  float limit = -1.0f;
  if (S.has_pc && S.node_count > 0 &&
      entered(slab_entry(o, invw, S.pc_lo.x, S.pc_lo.y, S.pc_lo.z, S.pc_hi.x, S.pc_hi.y, S.pc_hi.z, best), best))
    limit = best < 3.0e38f ? best * 1.00001f + 1e-6f : __int_as_float(0x7f800000);
  A.hits[3 * (size_t)slot] = make_float4(h.pos.x, h.pos.y, h.pos.z, best);
  A.hits[3 * (size_t)slot + 1] = make_float4(h.alpha, __int_as_float(h.inst), __uint_as_float(h.prim), 0.0f);
  A.hits[3 * (size_t)slot + 2] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  const V3 dd = normalize(d);
  // the slot (below 2^24) with the scene in the top bits
  A.walkq[2 * (size_t)t] = make_float4(o.x, o.y, o.z, limit);
  A.walkq[2 * (size_t)t + 1] = make_float4(dd.x, dd.y, dd.z, __uint_as_float(slot | (sid << 24)));
}

// Step 2: the closest-surfel walks (surfel_closest's) of the rays that
// enter the cloud, on a persistent grid.  Each lane walks one ray at a
// time; every kRefillSteps node visits the lanes whose walk has ended take
// the next rays (one atomic per warp on a cursor over the bounce's order,
// one load of the walk record each), so that a warp's lanes stay busy
// while walks of very different lengths end.  A walk that finds a surfel
// ends with one store of it and its distance in the ray's hit record; the
// hits do not depend on the schedule.
template <bool kMulti, int kThreads>
__global__ void __launch_bounds__(kThreads, kWalkMinBlocks * (kBlock / kThreads))
    k_adj_walk(AdjointArgs A, uint32_t parity) {
  extern __shared__ TravNode s_top[];
  stage_top_nodes(A.scenes, s_top);
  const uint32_t n_in = A.st->active[parity];
  const int lane = threadIdx.x & 31;
  TravStack stk(s_top, A.scenes.n * A.scenes.staged);
  ClosestWalk w;
  TraceCounters ctr{0, 0};
  uint32_t sid = 0;          // scene of this lane's ray
  uint32_t cur = kInvalid;   // queue slot of this lane's ray
  bool more = true;          // uniform in the warp: the cursor has rays left
  for (;;) {
    const unsigned need = __ballot_sync(0xffffffffu, cur == kInvalid);
    if (need && more) {
      const int leader = __ffs(need) - 1;
      uint32_t b0 = 0;
      if (lane == leader) b0 = atomicAdd(&A.st->walk_next, (uint32_t)__popc(need));
      b0 = __shfl_sync(0xffffffffu, b0, leader);
      if ((uint64_t)b0 + __popc(need) >= n_in) more = false;
      if (cur == kInvalid) {
        const uint32_t t = b0 + __popc(need & ((1u << lane) - 1u));
        if (t < n_in) {
          const float4 wa = A.walkq[2 * (size_t)t], wb = A.walkq[2 * (size_t)t + 1];
          if (wa.w >= 0.0f) {
            const uint32_t word = __float_as_uint(wb.w);
            cur = word & 0x00FFFFFFu;
            if (kMulti) sid = word >> 24;
            w.init(xyz(wa), xyz(wb), 1e-5f, wa.w);
          }
        }
      }
    }
    if (!__any_sync(0xffffffffu, cur != kInvalid)) {
      if (!more) break;
      continue;
    }
    for (int it = 0; it < kRefillSteps; ++it) {
      if (!__any_sync(0xffffffffu, cur != kInvalid)) break;
      const uint32_t sc = kMulti ? sid : 0u;
      if (warp_step(w, cur != kInvalid, A.scenes.s[sc], s_top + sc * A.scenes.staged, stk, ctr, A.st) ||
          cur == kInvalid)
        continue;
      if (w.hit) A.hits[3 * (size_t)cur + 2] = make_float4(__uint_as_float(w.prim), w.best, 1.0f, 0.0f);
      cur = kInvalid;
    }
  }
  block_count3(&A.st->node_visits, ctr.nodes, &A.st->surfel_tests, ctr.tests, nullptr, 0u);
}

// Step 3, launchAdjointIntersectKernel (AdjointKernels.cpp:87-386) after
// its intersection, in slot order (every access coalesced; the sorted
// order only serves the walks).  The hit is intersect_scene's: the walk's
// surfel when its world distance is below the mesh hit's, else the mesh hit.
__global__ void __launch_bounds__(kBlock, kTraceMinBlocks) k_adj_bounce(AdjointArgs A, uint32_t parity, uint32_t bounce_index) {
  const uint32_t n_in = A.st->active[parity];
  if ((uint64_t)blockIdx.x * kBlock >= n_in) return;
  const uint32_t slot = blockIdx.x * kBlock + threadIdx.x;
  bool alive = false, has_ev = false;
  uint32_t job = kInvalid;
  if (slot < n_in) {
    const float4 ro = A.qb.q[parity][slot].o, rd = A.qb.q[parity][slot].d;
    const SceneView& S = A.scenes.s[A.cams[A.jobs[__float_as_uint(rd.w) >> 8].cam].scene];
    const V3 d = xyz(rd);
    Hit h;
    {
      const float4 ha = A.hits[3 * (size_t)slot], hb = A.hits[3 * (size_t)slot + 1];
      const float4 wr = A.hits[3 * (size_t)slot + 2];
      h.pos = xyz(ha);
      h.inst = __float_as_int(hb.y);
      h.prim = __float_as_uint(hb.z);
      h.alpha = hb.x;
      h.t = h.inst >= 0 ? ha.w : 3.402823466e+38f;
      const float best = ha.w;
      if (wr.z != 0.0f) {
        const V3 o = xyz(ro);
        const uint32_t prim = __float_as_uint(wr.x);
        V3 x;
        float a;
        surfel_eval(S.sf, prim, o, normalize(d), wr.y, x, a);
        const float tw = dot(x - o, d);
        if (tw > 0.0f && tw < best) {
          h.inst = (int)S.mesh.instances;
          h.t = tw;
          h.pos = x;
          h.prim = prim;
          h.alpha = a;
        }
      }
    }
    const float4 rt = A.qb.q[parity][slot].t;
    const uint32_t jb = __float_as_uint(rd.w);
    job = jb >> 8;
    // the RNG key is the slot the ray holds in its own job's queue
    const uint32_t jslot = slot - A.job_start[(size_t)parity * kMaxJobsPerBatch + job];
    Rng r(per_item_seed(adjoint_base(A, job, 1u + bounce_index), jslot));
    const V3 thr = xyz(rt);
    const uint32_t path = __float_as_uint(ro.w), bounce = (jb & 0xFFu) + 1u;
    const uint32_t pixel = __float_as_uint(rt.w);
    if (h.inst >= 0) {
      const bool is_mesh = h.inst < (int)S.mesh.instances;
      V3 nrm = hit_normal(S, h);
      V3 on, dir;
      float pdf = 0.f;
      if (is_mesh) {
        sample_cosine(r, nrm, dir, pdf);
        on = nrm;
      } else {
        float sc = dot(nrm, -d);
        on = scale(nrm, (float)(sc >= 0.0f ? 1 : -1));
        sample_uniform_hemi(r, on, dir, pdf);
      }
      // complete the pending interaction with this hit as its endpoint
      const float4 pa = A.pend.a[path], pb = A.pend.b[path];
      const uint4 pc = A.pend.c[path];
      const uint32_t pkind = __float_as_uint(pb.w);
      EventRec ev;
      if ((pkind == kKindReflect && !is_mesh) || pkind == kKindNull) {
        const bool refl = pkind == kKindReflect;
        V3 pthr = scale(xyz(pb), refl ? A.q_reflect : A.q_null);
        float endcos = fmaxf(0.0f, dot(dir, on));
        uint32_t mat = kInvalid;
        if (refl) mat = __ldg(&S.mesh.material[pc.y]);
        else if (is_mesh) mat = __ldg(&S.mesh.material[h.inst]);
        ev.a = f4(h.pos, refl ? h.alpha : pa.w);
        ev.b = f4(on, refl ? pdf : endcos);
        ev.c = f4(pthr, __uint_as_float(job));
        ev.d = make_uint4(pkind, refl ? h.prim : pc.x, mat, pc.z);
        // the target surfel's hit: the endpoint (reflect) or the pending
        // null surfel, on the same line (a null continuation keeps d)
        ev.e = f4(refl ? h.pos : xyz(pa), 0.f);
        ev.f = f4(normalize(d), 0.f);
        has_ev = true;
        A.pend.b[path] = make_float4(0.f, 0.f, 0.f, __uint_as_float(kKindNone));
        A.pend.a[path] = make_float4(0.f, 0.f, 0.f, 0.f);
        A.pend.c[path] = make_uint4(kInvalid, pc.y, 0u, 0u);
      }
      V3 no, nd, nt;
      if (is_mesh) {
        const float4 mat = __ldg(&S.mesh.materials[__ldg(&S.mesh.material[h.inst])]);
        no = h.pos + scale(nrm, 1e-6f);
        nd = dir;
        nt = mul(thr, xyz(mat));
        alive = russian_roulette(r, bounce, nt, A.rr_start);
        if (alive) {
          V3 pt = mul(thr, xyz(mat));
          A.pend.a[path] = f4(h.pos, 0.0f);
          A.pend.b[path] = f4(pt, __uint_as_float(kKindReflect));
          A.pend.c[path] = make_uint4(kInvalid, (uint32_t)h.inst, pixel, 0u);
        }
      } else {
        const float opacity = __ldg(&S.sf.n[h.prim]).w;
        float u = r.next_float();
        if (u < A.q_null) {
          float att = 1.0f - h.alpha * opacity;
          float w = att / A.q_null;
          no = h.pos + scale(d, 1e-5f);
          nd = d;
          nt = scale(thr, w);
          alive = russian_roulette(r, bounce, nt, A.rr_start);
          if (alive) {
            A.pend.a[path] = f4(h.pos, h.alpha);
            A.pend.b[path] = f4(divs(thr, A.q_null), __uint_as_float(kKindNull));
            A.pend.c[path] = make_uint4(h.prim, kInvalid, pixel, 0u);
          }
        } else if (u < A.q_null + A.q_reflect) {
          const float4 al = __ldg(&S.sf.alb[h.prim]);
          V3 fs = scale(scale(xyz(al), al.w), kInvPi);
          float ct = fmaxf(0.0f, dot(dir, on));
          float alpha = h.alpha * opacity;
          V3 m = divs(scale(scale(fs, ct), alpha / A.q_reflect), pdf);
          no = h.pos + scale(on, 1e-5f);
          nd = dir;
          nt = mul(thr, m);
          alive = russian_roulette(r, bounce, nt, A.rr_start);
          if (alive && bounce_index == 0) {
            ev.a = f4(h.pos, h.alpha);
            ev.b = f4(on, 0.f);
            ev.c = f4(divs(thr, A.q_reflect), __uint_as_float(job));
            ev.d = make_uint4(kKindProjection, h.prim, kInvalid, pixel);
            ev.e = f4(h.pos, 0.f);
            ev.f = f4(normalize(d), 0.f);
            has_ev = true;
          }
        } else if (u < A.q_null + A.q_reflect + A.q_transmit) {
          float alpha = h.alpha * opacity;
          float w = (alpha * 0.0f) / A.q_transmit;   // alpha_t = 0
          V3 t2 = scale(thr, w);
          V3 on2 = on;
          float pdf2;
          sample_uniform_hemi(r, on2, nd, pdf2);
          const float4 al = __ldg(&S.sf.alb[h.prim]);
          no = h.pos + scale(-on2, 1e-5f);
          nt = mul(t2, xyz(al));
          alive = russian_roulette(r, bounce, nt, A.rr_start);
        }
      }
      // a view's rays end after its own number of bounces
      if (alive && bounce >= A.cams[A.jobs[job].cam].depth) alive = false;
      if (alive) A.qb.stage[slot] = make_ray(no, nd, nt, path, bounce | (job << 8), pixel);
      if (has_ev) A.ev.stage[slot] = ev;
    }
    A.qb.flags[slot] = (alive ? 1 : 0) | (has_ev ? 2 : 0);
  }
  {
    // survivors per job, one atomic per job present in the warp
    const uint32_t key = alive ? job : kInvalid;
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    if (alive && (threadIdx.x & 31) == __ffs(peers) - 1)
      atomicAdd(&A.job_count[(size_t)(parity ^ 1u) * kMaxJobsPerBatch + job], (uint32_t)__popc(peers));
  }
  block_count3(&A.st->adjoint_segments, slot < n_in ? 1u : 0u, nullptr, 0u, nullptr, 0u);
}

// Derivatives of eta * alpha_geom for the hit at x on surfel k along the
// unit direction d, with alpha_geom = (1 - r^2)^B, B = 4 e^beta,
// r^2 = u^2 + v^2, u = U.(x - p) / s_u, v = V.(x - p) / s_v, and x on the
// plane through p with normal n = U x V / |U x V| (x = o + t d,
// t = n.(p - o) / (n.d)).  These are the reference's helpers
// computeDuvDPositionFull, computeFullDuDvWrtTangents, computeDuvDScale and
// computeDAlphaDb (AdjointGradientKernels.h:212-272, 321-368, 440-451)
// chained through d alpha_geom / d r^2 = -B alpha_geom / (1 - r^2):
//   du/dp = ((U.d) / (n.d) n - U) / s_u,
//   du/dU = (r + (U.d) dt/dU) / s_u,  dv/dU = (V.d) dt/dU / s_v,
//   dt/dU = (r x V) / ((U x V).d),    dt/dV = (U x r) / ((U x V).d),
//   du/ds_u = -u / s_u,  d alpha_geom / d beta = alpha_geom B ln(1 - r^2).
// U and V are the tangents as given (the intersection does not normalize
// them); zero at the rim (r^2 >= 1) and for rays in the surfel's plane.
struct AlphaGrad {
  float beta;
  V3 pos, tu, tv;
  float su, sv;
};

__device__ __forceinline__ AlphaGrad alpha_grad(const SurfelView& S, uint32_t k, V3 x, V3 d) {
  AlphaGrad g;
  g.beta = 0.f;
  g.pos = g.tu = g.tv = v3(0.f, 0.f, 0.f);
  g.su = g.sv = 0.f;
  const float4 pe = __ldg(&S.pe[k]), n4 = __ldg(&S.n[k]), u4 = __ldg(&S.u[k]), v4 = __ldg(&S.v[k]);
  const V3 p = xyz(pe), U = xyz(u4), V = xyz(v4);
  const float B = pe.w, eta = n4.w, su = u4.w, sv = v4.w;
  const V3 r = x - p;
  const float u = dot(U, r) / su, v = dot(V, r) / sv;
  const float one = 1.0f - (u * u + v * v);
  if (!(one > 0.0f)) return g;
  const float alpha = powf(one, B);
  g.beta = eta * alpha * B * logf(one);
  const V3 m = cross(U, V);
  const V3 n = normalize(m);
  const float nd = dot(n, d), md = dot(m, d);
  if (fabsf(nd) < 1e-6f) return g;
  const float k2 = -2.0f * eta * B * alpha / one;   // d(eta alpha) / d(u) = k2 * u, d/dv = k2 * v
  const float ud = dot(U, d), vd = dot(V, d);
  const V3 dudp = scale(scale(n, ud / nd) - U, 1.0f / su);
  const V3 dvdp = scale(scale(n, vd / nd) - V, 1.0f / sv);
  g.pos = scale(scale(dudp, u) + scale(dvdp, v), k2);
  const V3 gU = scale(cross(r, V), 1.0f / md), gV = scale(cross(U, r), 1.0f / md);
  const V3 dudU = scale(r + scale(gU, ud), 1.0f / su), dvdU = scale(gU, vd / sv);
  const V3 dudV = scale(gV, ud / su), dvdV = scale(r + scale(gV, vd), 1.0f / sv);
  g.tu = scale(scale(dudU, u) + scale(dvdU, v), k2);
  g.tv = scale(scale(dudV, u) + scale(dvdV, v), k2);
  g.su = k2 * u * (-u / su);
  g.sv = k2 * v * (-v / sv);
  return g;
}

// The gather estimator's sweep over the entries of one round (rounds are
// swept last to first, so an entry finds the radiance behind its last
// layer in the next round's entry).  A camera path composites its layers
// front to back, I = sum_k T_k a_k Lo_k + T_end L_end with
// T_{k+1} = T_k (1 - a_k), a_k = opacity alpha_geom(x_k) and
// Lo_k = E(x_k) albedo alpha_r / pi; with Lb_k the radiance behind layer k
// (composited back to front, Lb = a Lo + (1 - a) Lb), dI/da_k =
// T_k (Lo_k - Lb_k).  The loss gradient of layer k, w = dL/dI . dI/da_k
// over the view's passes, goes to the opacity as w alpha_geom, to beta,
// position, tangents and scales as w d(a_k)/d(theta) (alpha_grad, the
// derivatives of the hit's alpha_geom) and to the albedo as
// dL/dI T_k a_k alpha_r E / pi per channel.  E(x_k) is the photon map's
// and held; the transmittance T_k is recomputed from the entry's with the
// forward's float operations.
__device__ __forceinline__ float* sweep_target(const SceneGrads& G, uint32_t k, int c) {
  switch (c) {
    case 0: return G.opacity + k;
    case 1: return G.all.beta + k;
    case 2: case 3: case 4: return G.all.position + 3 * (size_t)k + (c - 2);
    case 5: case 6: case 7: return G.all.tangent_u + 3 * (size_t)k + (c - 5);
    case 8: case 9: case 10: return G.all.tangent_v + 3 * (size_t)k + (c - 8);
    case 11: case 12: return G.all.scale + 2 * (size_t)k + (c - 11);
    default: return G.all.albedo + 3 * (size_t)k + (c - 13);
  }
}

constexpr int kSweepTerms = 16;   // opacity, beta, position 3, tangent_u 3, tangent_v 3, scale 2, albedo 3

// One thread per entry; the layers of a warp's entries are visited by layer
// index, deepest first, and the terms of lanes whose layer at that index
// is the same surfel are added up inside the warp (__match_any_sync on the
// scene and surfel, the lowest lane sums in lane order from shared memory)
// before one atomicAdd per component, the components spread over lanes.
// Neighbouring camera paths cross the same front surfels, so the first
// layers of a warp share targets.
__global__ void __launch_bounds__(kBlock) k_vs_sweep(FrameArgs A, SweepArgs W, const uint32_t* __restrict__ base,
                                                     uint32_t round) {
  __shared__ float s_val[kBlock / 32][kSweepTerms][33];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const uint32_t e1 = base[kVertexBases + round + 1];
  const uint32_t e = base[kVertexBases + round] + blockIdx.x * kBlock + threadIdx.x;
  bool valid = e < e1;
  if (valid && e >= A.vs.ent_cap) {   // slots past the store: never written
    flag_error(A.st, kErrBounds);
    valid = false;
  }
  if (!__any_sync(0xffffffffu, valid)) return;
  const int nterms = W.all_grads ? kSweepTerms : 1;
  float4 dT = make_float4(0.f, 0.f, 0.f, 1.f);
  uint4 b = make_uint4(0u, 0u, kInvalid, 0u);
  uint32_t sid = 0, route = 0, gp = 0;   // route: the gradient arrays' index (view or scene)
  float inv = 0.f;
  if (valid) {
    b = A.vs.ent_b[e];
    const uint32_t v = view_of_path(A, b.w);
    const CameraRec& C = A.cams[v];
    sid = C.scene;
    route = W.view_grads ? v : sid;
    if (W.view_grads && !W.view_grads[v].opacity) valid = false;   // a view without gradients
    dT = A.vs.ent_d[e];
    gp = C.pixel_offset + (b.w - A.view_start[v]) % (C.w * C.h);
    inv = 1.0f / (float)C.passes;
  }
  if (valid && ((uint64_t)b.x + (b.y & 0xFFu) > A.vs.rec_cap || (b.z != kInvalid && b.z >= A.vs.ent_cap))) {
    flag_error(A.st, kErrBounds);
    valid = false;
  }
  if (!valid) b = make_uint4(0u, 0u, kInvalid, 0u);
  const SceneView& S = A.scenes.s[sid];
  const uint32_t used = b.y & 0xFFu, first = b.x;
  const V3 g = valid ? xyz(*reinterpret_cast<const float4*>(W.dldi + 4 * (size_t)gp)) : v3(0.f, 0.f, 0.f);
  V3 Lb = v3(0.f, 0.f, 0.f);
  if (valid && b.z != kInvalid) Lb = xyz(A.vs.ent_l[b.z]);
  else if (valid && ((b.y >> 8) & 1u)) Lb = xyz(A.vs.ent_l[e]);
  float Ts[kGatherHits], as[kGatherHits];
  int ns = 0;
  float T = dT.w;
#pragma unroll
  for (int i = 0; i <= kGatherHits; ++i) {
    Ts[i < kGatherHits ? i : 0] = 0.f;
    as[i < kGatherHits ? i : 0] = 0.f;
  }
#pragma unroll
  for (int i = 0; i <= kGatherHits; ++i) {
    if (i < (int)used) {
      const float4 ew = A.vs.rec_ew[first + i];
      const uint32_t word = __float_as_uint(ew.w);
      const uint32_t kind = word >> 30, idx = word & kRecIndexMask;
      if (kind == kRecSurfel && i < kGatherHits) {
        const float ae = __ldg(&S.sf.n[idx]).w * A.vs.rec_xa[first + i].w;
        Ts[i < kGatherHits ? i : 0] = T;
        as[i < kGatherHits ? i : 0] = ae;
        T *= (1.0f - ae);
        ns = i + 1;
      } else if (kind == kRecMesh) {
        const float4 mat = __ldg(&S.mesh.materials[idx]);
        Lb = mul(scale(xyz(mat), kInvPi), xyz(ew));
      }
    }
  }
  const V3 dd = normalize(xyz(dT));
  float (*val)[33] = s_val[wid];
#pragma unroll
  for (int i = kGatherHits - 1; i >= 0; --i) {
    if (!__any_sync(0xffffffffu, i < ns)) continue;
    uint32_t k = kInvalid;
    float t[kSweepTerms];
#pragma unroll
    for (int c = 0; c < kSweepTerms; ++c) t[c] = 0.f;
    if (i < ns) {
      const float4 xa = A.vs.rec_xa[first + i], ew = A.vs.rec_ew[first + i];
      k = __float_as_uint(ew.w) & kRecIndexMask;
      const float4 al = __ldg(&S.sf.alb[k]);
      const V3 E = xyz(ew);
      const V3 Lo = mul(E, scale(scale(xyz(al), al.w), kInvPi));
      const float w = inv * dot(g, scale(Lo - Lb, Ts[i]));
      t[0] = w * xa.w;
      if (W.all_grads) {
        if (w != 0.f) {
          const AlphaGrad ag = alpha_grad(S.sf, k, xyz(xa), dd);
          t[1] = w * ag.beta;
          t[2] = w * ag.pos.x; t[3] = w * ag.pos.y; t[4] = w * ag.pos.z;
          t[5] = w * ag.tu.x; t[6] = w * ag.tu.y; t[7] = w * ag.tu.z;
          t[8] = w * ag.tv.x; t[9] = w * ag.tv.y; t[10] = w * ag.tv.z;
          t[11] = w * ag.su; t[12] = w * ag.sv;
        }
        const float ka = inv * Ts[i] * as[i] * al.w * kInvPi;
        t[13] = g.x * ka * E.x;
        t[14] = g.y * ka * E.y;
        t[15] = g.z * ka * E.z;
      }
      Lb = scale(Lo, as[i]) + scale(Lb, 1.0f - as[i]);
    }
    for (int c = 0; c < nterms; ++c) val[c][lane] = t[c];
    __syncwarp();
    const unsigned grp = __match_any_sync(0xffffffffu, ((unsigned long long)route << 32) | k);
    const bool leader = k != kInvalid && lane == __ffs(grp) - 1;
    if (leader && __popc(grp) > 1) {
      for (int c = 0; c < nterms; ++c) {
        float acc = 0.f;
        for (unsigned r = grp; r; r &= r - 1u) acc += val[c][__ffs(r) - 1];
        val[c][lane] = acc;
      }
    }
    __syncwarp();
    for (unsigned lm = __ballot_sync(0xffffffffu, leader); lm; lm &= lm - 1u) {
      const int L = __ffs(lm) - 1;
      const uint32_t kL = __shfl_sync(0xffffffffu, k, L);
      const uint32_t rL = __shfl_sync(0xffffffffu, route, L);
      if (lane < nterms) {
        const float x = val[lane][L];
        if (x != 0.f) atomicAdd(sweep_target(W.view_grads ? W.view_grads[rL] : W.grads[rL], kL, lane), x);
      }
    }
    __syncwarp();
  }
  if (valid) A.vs.ent_l[e] = make_float4(Lb.x, Lb.y, Lb.z, 0.f);
}

void gather_backward(const FrameArgs& a0, const std::vector<CameraRec>& views, const VertexPlan& plan,
                     const SweepArgs& w, const VertexStore& scratch, cudaStream_t s) {
  const bool multi = a0.scenes.n > 1;
  const GatherShape g = multi ? gather_shape<true>(a0) : gather_shape<false>(a0);
  for (size_t c = 0; c < plan.chunks.size(); ++c) {
    const VertexChunk& vc = plan.chunks[c];
    FrameArgs a = a0;
    cudaMemcpyAsync(const_cast<uint32_t*>(a.view_start), vc.table.data(), vc.table.size() * sizeof(uint32_t),
                    cudaMemcpyHostToDevice, s);
    const uint32_t* bases = plan.d_chunk_base + c * 2 * kVertexBases;
    uint32_t rounds = vc.rounds;
    if (!vc.stored) {
      // replay: the chunk's rounds again, with the forward's seeds, into
      // the scratch store from its first slot
      a.vs = scratch;
      a.vs.write = 1;
      a.vs.rec_start = 0;
      a.vs.ent_start = 0;
      rounds = multi ? gather_rounds<true>(a, g, vc.n, s) : gather_rounds<false>(a, g, vc.n, s);
      bases = a.vs.base;
    }
    // timed as the adjoint's transport (this estimator has none)
    if (a.timer) a.timer->begin(kTimeTransport, s);
    for (uint32_t r = rounds; r-- > 0;) {
      k_vs_sweep<<<blocks_for(vc.n), kBlock, 0, s>>>(a, w, bases, r); note_launch();
    }
    if (a.timer) a.timer->end(s);
  }
}

// launchAdjointTransportKernel (AdjointKernels.cpp:389-509).  A warp takes
// the events of a tile of 32 (warps stride over the tiles), lane i the
// i-th: every lane loads its own event record (one coalesced load), the
// warp does the photon lookups of the tile's events one after another
// (gather_irradiance_warp, each lookup's 32 photon rounds spread over the
// lanes) and the lane of each event keeps its irradiance; then every lane
// evaluates its own event's terms (the opacity term as the reference
// computes it; with gradients = "all" also the other six groups) at the
// same time.  Events with the same target surfel are added up inside the
// warp before they reach memory (__match_any_sync groups the lanes by
// scene and target; the lowest lane of a group sums the group's terms in lane order
// from shared memory), and each group's terms go out with one atomicAdd
// per component, the components of one group spread over lanes.
constexpr int kTransportTerms = 16;   // opacity, beta, position 3, tangent_u 3, tangent_v 3, scale 2, albedo 3 - 1

__global__ void __launch_bounds__(kBlock, kTransportMinBlocks) k_transport(AdjointArgs A) {
  __shared__ float4 s_terms[kBlock];                        // per warp: the lookups' row compaction
  __shared__ float s_val[kBlock / 32][kTransportTerms + 1][33];   // per warp: the lanes' terms
  __shared__ GatherConst s_gc[kMaxScenes];
  if (threadIdx.x < A.scenes.n) s_gc[threadIdx.x] = gather_const(A.scenes.s[threadIdx.x].grid);
  __syncthreads();
  const uint32_t count = A.st->event_count;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  float4* terms = s_terms + (threadIdx.x & ~31u);
  const uint32_t warps = gridDim.x * (kBlock / 32);
  const uint32_t tiles = (count + 31u) / 32u;
  const int nterms = A.all_grads ? kTransportTerms + 1 : 1;
  uint32_t events = 0, queries = 0, scanned = 0;
  for (uint32_t tile = blockIdx.x * (kBlock / 32) + wid; tile < tiles; tile += warps) {
    const uint32_t e = tile * 32u + lane;
    const bool valid = e < count;
    // the lookup's point and normal and the event's kind and indices now;
    // the throughput (and the alpha-gradient point) after the lookups
    const EventRec* src = A.ev.list + (valid ? e : 0u);
    EventRec ev;
    uint32_t sid = 0, passes = 1;   // the event's scene and its view's passes
    if (valid) {
      ev.a = src->a;
      ev.b = src->b;
      ev.d = src->d;
      const CameraRec& C = A.cams[A.jobs[__float_as_uint(src->c.w)].cam];
      sid = C.scene;
      passes = C.passes;
    } else {
      ev.a = ev.b = make_float4(0.f, 0.f, 0.f, 0.f);
      ev.d = make_uint4(kInvalid, kInvalid, kInvalid, 0u);
    }
    const uint32_t kind = ev.d.x;
    // a null event ending on a surfel has no material (the reference reads
    // materials[0xFFFFFFFF], AdjointKernels.cpp:446-447): no contribution
    const bool need =
        valid && (kind == kKindProjection || kind == kKindReflect || (kind == kKindNull && ev.d.z != kInvalid));
    V3 E = v3(0.f, 0.f, 0.f);
    for (unsigned m = __ballot_sync(0xffffffffu, need); m; m &= m - 1u) {
      const int j = __ffs(m) - 1;
      const V3 xj = v3(__shfl_sync(0xffffffffu, ev.a.x, j), __shfl_sync(0xffffffffu, ev.a.y, j),
                       __shfl_sync(0xffffffffu, ev.a.z, j));
      const V3 nj = v3(__shfl_sync(0xffffffffu, ev.b.x, j), __shfl_sync(0xffffffffu, ev.b.y, j),
                       __shfl_sync(0xffffffffu, ev.b.z, j));
      const uint32_t sj = __shfl_sync(0xffffffffu, sid, j);
      uint32_t cnt = 0;
      const V3 Ej = gather_irradiance_warp<true>(A.scenes.s[sj].grid, s_gc[sj], xj, nj, terms, cnt);
      if (lane == j) {
        E = Ej;
        scanned += cnt;
        ++queries;
      }
    }
    // this lane's event
    const SceneView& S = A.scenes.s[sid];
    const float inv_spp = 1.0f / (float)passes;
    float g = 0.f;        // opacity term, as the reference computes it
    float W = 0.f;        // the event's weight: g = W * alpha_geom
    V3 dalb = v3(0.f, 0.f, 0.f);
    uint32_t target = kInvalid;
    if (valid) {
      ++events;
      const V3 thr = xyz(src->c);
      if (kind == kKindProjection) {
        target = ev.d.y;
        const float4 al = __ldg(&S.sf.alb[target < S.sf.count ? target : 0u]);
        V3 fr = scale(scale(xyz(al), al.w), kInvPi);
        V3 Lo = mul(fr, E);
        g = vsum(mul(scale(thr, ev.a.w), Lo)) * inv_spp;
        if (A.all_grads && target < S.sf.count) {
          W = vsum(mul(thr, Lo)) * inv_spp;
          // d/d albedo of eta alpha_geom (alpha_r albedo / pi) E, per channel
          const float eta = __ldg(&S.sf.n[target]).w;
          dalb = scale(mul(thr, E), eta * ev.a.w * al.w * kInvPi * inv_spp);
        }
      } else if (kind == kKindNull) {
        target = ev.d.y;
        if (ev.d.z != kInvalid) {
          const float4 mat = __ldg(&S.mesh.materials[ev.d.z]);
          V3 Lr = scale(mul(E, xyz(mat)), kInvPi);
          V3 Le = v3(0.f, 0.f, 0.f);
          if (mat.w > 0.f) {
            float area = A.light0_valid ? A.light0_area : 0.f;
            Le = scale(scale(xyz(mat), mat.w / (kPi * area)), ev.b.w);
          }
          V3 Lo = Le + Lr;
          g = vsum(mul(scale(thr, -ev.a.w * A.null_scale), Lo)) * inv_spp;
          if (A.all_grads) W = -vsum(mul(thr, Lo)) * A.null_scale * inv_spp;
        }
      } else if (kind == kKindReflect) {
        target = ev.d.y;
        const float4 mat = __ldg(&S.mesh.materials[ev.d.z]);
        V3 Lo = scale(mul(E, xyz(mat)), kInvPi);
        V3 p = divs(thr, ev.b.w);
        g = vsum(scale(mul(p, Lo), ev.a.w)) * inv_spp;
        if (A.all_grads) W = vsum(mul(p, Lo)) * inv_spp;
      }
      if (target != kInvalid && target >= S.sf.count) {
        flag_error(A.st, kErrBounds);
        target = kInvalid;
      }
      if (target != kInvalid && A.debug_opacity) {
        float* px = A.debug_opacity + 4 * (size_t)ev.d.w;
        atomicAdd(px + 0, g);
        atomicAdd(px + 1, g);
        atomicAdd(px + 2, g);
        px[3] = 1.0f;
      }
    }
    // the lane's terms, in the order of kTransportTerms
    float (*val)[33] = s_val[wid];
    val[0][lane] = g;
    if (A.all_grads) {
      AlphaGrad ag{};
      if (target != kInvalid && W != 0.f) ag = alpha_grad(S.sf, target, xyz(src->e), xyz(src->f));
      const bool w0 = target != kInvalid && W != 0.f;
      val[1][lane] = w0 ? W * ag.beta : 0.f;
      val[2][lane] = w0 ? W * ag.pos.x : 0.f;
      val[3][lane] = w0 ? W * ag.pos.y : 0.f;
      val[4][lane] = w0 ? W * ag.pos.z : 0.f;
      val[5][lane] = w0 ? W * ag.tu.x : 0.f;
      val[6][lane] = w0 ? W * ag.tu.y : 0.f;
      val[7][lane] = w0 ? W * ag.tu.z : 0.f;
      val[8][lane] = w0 ? W * ag.tv.x : 0.f;
      val[9][lane] = w0 ? W * ag.tv.y : 0.f;
      val[10][lane] = w0 ? W * ag.tv.z : 0.f;
      val[11][lane] = w0 ? W * ag.su : 0.f;
      val[12][lane] = w0 ? W * ag.sv : 0.f;
      val[13][lane] = dalb.x;
      val[14][lane] = dalb.y;
      val[15][lane] = dalb.z;
      val[16][lane] = 0.f;
    }
    __syncwarp();
    // same-target lanes form a group; its lowest lane sums the group's terms
    const unsigned grp = __match_any_sync(0xffffffffu, ((unsigned long long)sid << 32) | target);
    const bool leader = target != kInvalid && lane == __ffs(grp) - 1;
    if (leader && __popc(grp) > 1) {
      for (int c = 0; c < nterms; ++c) {
        float acc = 0.f;
        for (unsigned r = grp; r; r &= r - 1u) acc += val[c][__ffs(r) - 1];
        val[c][lane] = acc;
      }
    }
    __syncwarp();
    // one atomicAdd per component of each group: the group leaders in turn,
    // the components over lanes
    for (unsigned lm = __ballot_sync(0xffffffffu, leader); lm; lm &= lm - 1u) {
      const int L = __ffs(lm) - 1;
      const uint32_t t = __shfl_sync(0xffffffffu, target, L);
      const SceneGrads& G = A.sgrads[__shfl_sync(0xffffffffu, sid, L)];
      if (lane < nterms) {
        const float v = val[lane][L];
        float* dst = nullptr;
        switch (lane) {
          case 0: dst = G.opacity + t; break;
          case 1: dst = G.all.beta + t; break;
          case 2: case 3: case 4: dst = G.all.position + 3 * (size_t)t + (lane - 2); break;
          case 5: case 6: case 7: dst = G.all.tangent_u + 3 * (size_t)t + (lane - 5); break;
          case 8: case 9: case 10: dst = G.all.tangent_v + 3 * (size_t)t + (lane - 8); break;
          case 11: case 12: dst = G.all.scale + 2 * (size_t)t + (lane - 11); break;
          case 13: case 14: case 15: dst = G.all.albedo + 3 * (size_t)t + (lane - 13); break;
          default: break;
        }
        if (dst && (lane == 0 || v != 0.f)) atomicAdd(dst, v);
      }
    }
    __syncwarp();
  }
  warp_count(&A.st->gradient_events, events);
  warp_count(&A.st->gather_queries, queries);
  warp_count(&A.st->photons_scanned, scanned);
}

void adjoint_raygen(const AdjointArgs& a, uint32_t npaths, cudaStream_t s) {
  k_adj_raygen<<<blocks_for(std::max<uint32_t>(npaths, kMaxJobsPerBatch)), kBlock, 0, s>>>(a, npaths); note_launch();
}

// One bounce of every job of the batch; npaths bounds the live queue.
void adjoint_bounce(const AdjointArgs& a, uint32_t bounce, uint32_t npaths, cudaStream_t s) {
  const uint32_t nb = blocks_for(npaths);
  if (nb == 0) return;
  const uint32_t parity = bounce & 1u;
  // the first bounce traces camera rays in pixel order, already coherent
  const int sorted = bounce > 0 && a.perm && npaths <= a.sort_capacity;
  if (sorted) {
    k_adj_keys<<<nb, kBlock, 0, s>>>(a, parity); note_launch();
    radix_sort_pairs(a.sort_keys, a.perm, a.sort_keys_tmp, a.perm_tmp, &a.st->active[parity], npaths, 30,
                     a.sort_temp, s);
  }
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const bool multi = a.scenes.n > 1;
  const int wt = a.walk_block == 64 || a.walk_block == 128 ? (int)a.walk_block : kBlock;
  const size_t smem = top_smem(a.scenes, wt);
  if (a.timer) a.timer->begin(kTimeAdjBounce, s);
  k_adj_mesh<<<nb, kBlock, 0, s>>>(a, parity, sorted); note_launch();
  // the walk's persistent grid: every SM filled once, no more blocks than rays need
  if (multi) {
    if (wt == 64) launch_walk(k_adj_walk<true, 64>, 64, a, parity, smem, nb, s);
    else if (wt == 128) launch_walk(k_adj_walk<true, 128>, 128, a, parity, smem, nb, s);
    else launch_walk(k_adj_walk<true, 256>, 256, a, parity, smem, nb, s);
  } else {
    if (wt == 64) launch_walk(k_adj_walk<false, 64>, 64, a, parity, smem, nb, s);
    else if (wt == 128) launch_walk(k_adj_walk<false, 128>, 128, a, parity, smem, nb, s);
    else launch_walk(k_adj_walk<false, 256>, 256, a, parity, smem, nb, s);
  }
  k_adj_bounce<<<nb, kBlock, 0, s>>>(a, parity, bounce); note_launch();
  if (a.timer) a.timer->end(s);
  k_adj_tile_counts<<<nb, kBlock, 0, s>>>(a, parity); note_launch();
  k_queue_scan<<<1, 1024, 0, s>>>(a.st, a.qb.tile_counts, a.qb.tile_offsets, parity, 0, 0, 1, 0); note_launch();
  k_job_scan<<<1, kMaxJobsPerBatch, 0, s>>>(a, parity); note_launch();
  k_queue_scatter<1><<<nb, kBlock, 0, s>>>(a.st, a.qb, parity, 0, 0, PhotonStore{}, a.ev); note_launch();
  // a warp per tile of 32 events: a grid that fills every SM once
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_transport, kBlock, 0);
  if (a.timer) a.timer->begin(kTimeTransport, s);
  k_transport<<<(uint32_t)std::max(1, sms * std::max(1, per_sm)), kBlock, 0, s>>>(a); note_launch();
  if (a.timer) a.timer->end(s);
}

// ------------------------------------------------------ component queries
__global__ void __launch_bounds__(kBlock) k_trace_rays(SceneView S, RunState* st, uint32_t n,
                                                       const float* __restrict__ o, const float* __restrict__ d,
                                                       int32_t* inst, int32_t* prim, float* t, float* alpha,
                                                       float* pos) {
  extern __shared__ TravNode s_top[];
  stage_top_nodes(S, s_top);
  uint32_t i = blockIdx.x * kBlock + threadIdx.x;
  TraceCounters ctr{0, 0};
  if (i < n) {
    Hit h = intersect_scene(S, s_top, v3(o[3 * i], o[3 * i + 1], o[3 * i + 2]),
                            v3(d[3 * i], d[3 * i + 1], d[3 * i + 2]), ctr, st);
    inst[i] = h.inst;
    prim[i] = h.inst >= 0 ? (int32_t)h.prim : -1;
    t[i] = h.inst >= 0 ? h.t : 3.402823466e+38f;
    alpha[i] = h.inst >= 0 ? h.alpha : 0.f;
    if (pos) {
      pos[3 * i] = h.pos.x;
      pos[3 * i + 1] = h.pos.y;
      pos[3 * i + 2] = h.pos.z;
    }
  }
  block_count3(&st->node_visits, ctr.nodes, &st->surfel_tests, ctr.tests, nullptr, 0u);
}

void trace_rays(const SceneView& sv, RunState* st, uint32_t n, const float* o, const float* d, int32_t* inst,
                int32_t* prim, float* t, float* alpha, float* pos, cudaStream_t s) {
  if (n == 0) return;
  k_trace_rays<<<blocks_for(n), kBlock, top_smem(sv), s>>>(sv, st, n, o, d, inst, prim, t, alpha, pos); note_launch();
}

// Transmit-mode scene query, one ray per thread: the closest mesh hit and
// the surfel cloud's transmissivity (intersect_scene_transmit).  The walk
// is bounded at 2^16 surfel hits per ray.
__global__ void __launch_bounds__(kBlock) k_trace_transmittance(SceneView S, RunState* st, uint32_t n,
                                                                const float* __restrict__ o,
                                                                const float* __restrict__ d, int32_t* inst,
                                                                float* t, float* transmit) {
  extern __shared__ TravNode s_top[];
  stage_top_nodes(S, s_top);
  uint32_t i = blockIdx.x * kBlock + threadIdx.x;
  TraceCounters ctr{0, 0};
  if (i < n) {
    float T = 1.0f;
    Hit h = intersect_scene_transmit(S, s_top, v3(o[3 * i], o[3 * i + 1], o[3 * i + 2]),
                                     v3(d[3 * i], d[3 * i + 1], d[3 * i + 2]), T, 1u << 16, ctr, st);
    inst[i] = h.inst;
    t[i] = h.inst >= 0 ? h.t : 3.402823466e+38f;
    transmit[i] = T;
  }
  block_count3(&st->node_visits, ctr.nodes, &st->surfel_tests, ctr.tests, nullptr, 0u);
}

void trace_transmittance(const SceneView& sv, RunState* st, uint32_t n, const float* o, const float* d,
                         int32_t* inst, float* t, float* transmit, cudaStream_t s) {
  if (n == 0) return;
  k_trace_transmittance<<<blocks_for(n), kBlock, top_smem(sv), s>>>(sv, st, n, o, d, inst, t, transmit);
  note_launch();
}

__global__ void k_gather_points(SceneView S, uint32_t n, const float* __restrict__ p, const float* __restrict__ nrm,
                                float* E) {
  __shared__ float4 s_terms[kBlock];
  const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const bool in = i < n;
  const GatherConst GC = gather_const(S.grid);
  V3 x = v3(0.f, 0.f, 0.f), nv = v3(0.f, 0.f, 0.f), e = v3(0.f, 0.f, 0.f);
  if (in) {
    x = v3(p[3 * i], p[3 * i + 1], p[3 * i + 2]);
    nv = v3(nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2]);
  }
  unsigned qm = __ballot_sync(0xffffffffu, in);
  while (qm) {
    const int src = __ffs(qm) - 1;
    qm &= qm - 1u;
    const V3 qx = v3(__shfl_sync(0xffffffffu, x.x, src), __shfl_sync(0xffffffffu, x.y, src),
                     __shfl_sync(0xffffffffu, x.z, src));
    const V3 qv = v3(__shfl_sync(0xffffffffu, nv.x, src), __shfl_sync(0xffffffffu, nv.y, src),
                     __shfl_sync(0xffffffffu, nv.z, src));
    uint32_t cnt = 0;
    const V3 r = gather_irradiance_warp<false>(S.grid, GC, qx, qv, s_terms + (threadIdx.x & ~31u), cnt);
    if (lane == src) e = r;
  }
  if (!in) return;
  E[3 * i] = e.x;
  E[3 * i + 1] = e.y;
  E[3 * i + 2] = e.z;
}

void gather_points(const SceneView& sv, uint32_t n, const float* p, const float* nrm, float* E, cudaStream_t s) {
  if (n == 0) return;
  k_gather_points<<<blocks_for(n), kBlock, 0, s>>>(sv, n, p, nrm, E); note_launch();
}

__global__ void k_load_photons(uint32_t n, const float* __restrict__ pos, const float* __restrict__ pw,
                               const float* __restrict__ dir, PhotonStore ps) {
  uint32_t i = blockIdx.x * kBlock + threadIdx.x;
  if (i >= n) return;
  ps.a[i] = make_float4(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], pw[3 * i]);
  ps.b[i] = make_float4(dir[3 * i], dir[3 * i + 1], dir[3 * i + 2], pw[3 * i + 1]);
  ps.c[i] = pw[3 * i + 2];
}

void load_photon_arrays(uint32_t n, const float* pos, const float* pw, const float* dir, const PhotonStore& ps,
                        cudaStream_t s) {
  if (n == 0) return;
  k_load_photons<<<blocks_for(n), kBlock, 0, s>>>(n, pos, pw, dir, ps); note_launch();
}

// ----------------------------------------------------------- KernelTimer
void KernelTimer::begin(int k, cudaStream_t s) {
  if (2 * used + 2 > pool.size()) {
    cudaEvent_t a = nullptr, b = nullptr;
    if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) {
      if (a) cudaEventDestroy(a);
      open = false;
      return;
    }
    pool.push_back(a);
    pool.push_back(b);
  }
  if (kind.size() <= used) kind.resize(used + 1);
  kind[used] = k;
  cudaEventRecord(pool[2 * used], s);
  open = true;
}

void KernelTimer::end(cudaStream_t s) {
  if (!open) return;
  cudaEventRecord(pool[2 * used + 1], s);
  ++used;
  open = false;
}

void KernelTimer::collect(float* ms, uint32_t* n) {
  for (size_t i = 0; i < used; ++i) {
    float t = 0.f;
    if (cudaEventElapsedTime(&t, pool[2 * i], pool[2 * i + 1]) == cudaSuccess) {
      ms[kind[i]] += t;
      n[kind[i]] += 1;
    }
  }
  used = 0;
}

KernelTimer::~KernelTimer() {
  for (cudaEvent_t e : pool) cudaEventDestroy(e);
}

}  // namespace pale
