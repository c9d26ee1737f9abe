// api.cu -- host implementation of the C-ABI in include/pale_b200.h.
//
// A pale_handle owns every device buffer of one renderer: meshes, cameras,
// the surfel parameters in BVH order with their derived arrays and LBVH,
// the photon store and grid, the ray queues and the adjoint state.  Each
// entry point runs on the handle's own stream and returns a status code;
// nothing throws across the boundary.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/pale_b200.h"
#include "kernels.h"

using namespace pale;

namespace pale {
static thread_local uint64_t g_launches = 0;
void note_launch() { ++g_launches; }
uint64_t launches_issued() { return g_launches; }
}  // namespace pale

namespace {

thread_local std::string g_create_error;

}  // namespace

void pale::set_thread_error(const std::string& msg) { g_create_error = msg; }

namespace {

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct ArgError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

#define CK(x)                                                                                       \
  do {                                                                                              \
    cudaError_t e_ = (x);                                                                           \
    if (e_ != cudaSuccess)                                                                          \
      throw CudaError(std::string(#x) + " failed: " + cudaGetErrorString(e_) + " (" __FILE__ ":" + \
                      std::to_string(__LINE__) + ")");                                              \
  } while (0)

template <typename T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  void alloc(size_t count) {
    free();
    if (count == 0) count = 1;
    CK(cudaMalloc(&p, count * sizeof(T)));
    n = count;
  }
  void ensure(size_t count) {
    if (count > n || !p) alloc(count);
  }
  void free() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  ~DBuf() { free(); }
};

struct PointsBufs {
  DBuf<float> pos, tu, tv, sc, alb, op, beta, shape;
  void alloc(uint32_t n) {
    pos.ensure(3 * (size_t)n); tu.ensure(3 * (size_t)n); tv.ensure(3 * (size_t)n); sc.ensure(2 * (size_t)n);
    alb.ensure(3 * (size_t)n); op.ensure(n); beta.ensure(n); shape.ensure(n);
  }
  PointsDev view() const { return PointsDev{pos.p, tu.p, tv.p, sc.p, alb.p, op.p, beta.p, shape.p}; }
};

uint32_t next_pow2(uint32_t v) {
  uint32_t c = 1;
  while (c < v) c <<= 1;
  return c;
}

// Pinned host memory that stages the copies between a caller's (pageable)
// host buffers and the device: the device side of a copy runs at the
// pinned-memory rate and the host side is split over threads, where a
// pageable cudaMemcpyAsync copies through the driver's staging on one.
struct HostStage {
  char* p = nullptr;
  size_t n = 0;
  bool in_flight = false;   // a host-to-device copy from it may still run
  // At least `bytes` of pinned memory; false (and no stage) when the host
  // cannot pin that much, and the copies then go through pageable memory.
  bool ensure(size_t bytes, cudaStream_t s) {
    if (bytes <= n && p) return true;
    if (in_flight) CK(cudaStreamSynchronize(s));
    in_flight = false;
    if (p) cudaFreeHost(p);
    p = nullptr;
    n = 0;
    if (cudaMallocHost(&p, bytes) != cudaSuccess) {
      cudaGetLastError();   // the failed allocation is not sticky; clear it
      p = nullptr;
      return false;
    }
    n = bytes;
    return true;
  }
  ~HostStage() {
    if (p) cudaFreeHost(p);
  }
};

// Copies of at least this many bytes in total go through the stage.
constexpr size_t kStageMinBytes = 4u << 20;

// Threads of a staged host copy: PALE_COPY_THREADS, else up to 8.
unsigned copy_threads() {
  static const unsigned t = [] {
    const char* e = std::getenv("PALE_COPY_THREADS");
    const long v = e ? std::strtol(e, nullptr, 10) : 0;
    if (v > 0) return (unsigned)std::min<long>(v, 64);
    return std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
  }();
  return t;
}

struct HostPiece {
  char* dst;
  const char* src;
  size_t bytes;
};

// memcpy of every piece, the pieces' bytes split evenly over the threads
// (each thread a contiguous range of the concatenated pieces).
void host_copy(const std::vector<HostPiece>& pieces) {
  size_t total = 0;
  for (const HostPiece& q : pieces) total += q.bytes;
  const unsigned nt = (unsigned)std::min<size_t>(copy_threads(), std::max<size_t>(1, total / (1u << 20)));
  auto range = [&](size_t a, size_t b) {   // bytes [a, b) of the concatenation
    size_t off = 0;
    for (const HostPiece& q : pieces) {
      const size_t lo = std::max(a, off), hi = std::min(b, off + q.bytes);
      if (lo < hi) std::memcpy(q.dst + (lo - off), q.src + (lo - off), hi - lo);
      off += q.bytes;
    }
  };
  if (nt <= 1) {
    range(0, total);
    return;
  }
  const size_t per = (total + nt - 1) / nt;
  std::vector<std::thread> th;
  th.reserve(nt);
  for (unsigned t = 0; t < nt; ++t) {
    const size_t a = std::min(total, (size_t)t * per), b = std::min(total, a + per);
    if (a < b) th.emplace_back(range, a, b);
  }
  for (std::thread& x : th) x.join();
}

}  // namespace

struct pale_handle {
  pale_settings st{};
  cudaStream_t stream = nullptr;
  std::string err;
  // meshes
  uint32_t n_inst = 0, n_tris = 0;
  DBuf<float> o2w, w2o;
  DBuf<float4> inst_box, tri, wtri, materials;
  DBuf<uint2> wtri_range;
  DBuf<uint2> tri_range;
  DBuf<uint32_t> inst_mat;
  std::vector<float> h_inst_box;   // lo.xyz hi.xyz per instance
  // lights
  uint32_t n_lights = 0;
  DBuf<uint4> light_rec;
  DBuf<float4> light_col;
  DBuf<float> light_area, light_cdf;
  DBuf<uint32_t> light_tri;
  float light0_area = 0.f;
  // cameras
  std::vector<CameraRec> cams;
  std::vector<std::string> cam_names;
  DBuf<CameraRec> d_cams;
  DBuf<uint32_t> d_view_start;   // the current gather chunk's view table (3 words per view)
  // surfels
  uint32_t np = 0;
  PointsBufs asset, collected, params;
  DBuf<float4> sf_pe, sf_n, sf_u, sf_v, sf_cn, sf_alb;
  DBuf<float> aabb_lo, aabb_hi, bounds_part, bounds;
  DBuf<uint32_t> codes, order, codes_tmp, order_tmp, sort_temp, rfirst, rlast, parent, leaf_parent, visits, d_n;
  DBuf<int32_t> lc, rc;
  DBuf<float> box;
  DBuf<BvhNode> nodes;
  DBuf<BvhNodeH> hnodes;   // traversal copy (half boxes) when PALE_HALF_NODES
  uint32_t node_count = 0, top = 0;
  float pc_lo[3] = {0, 0, 0}, pc_hi[3] = {0, 0, 0};
  // photon grid
  float radius = 0.01f, origin[3] = {0, 0, 0}, cell = 0.005f;
  int res[3] = {1, 1, 1};
  uint32_t cells = 1;
  int key_bits = 8;
  uint64_t photon_cap = 0;
  DBuf<float4> ph_a, ph_b, ph_sa, ph_sb, g_pa, g_pb;
  DBuf<float> ph_c, ph_sc, g_pc;
  DBuf<uint32_t> g_cell_id, g_sorted, g_keys, g_vals_tmp, g_sort_temp, g_cell_count, g_cell_off, g_scan_temp,
      g_stored, g_attempts;
  // queues
  uint32_t qcap = 0;
  DBuf<RayRec> q0, q1, qstage;
  DBuf<uint8_t> qflags;
  DBuf<uint2> tile_counts, tile_offsets;
  DBuf<float4> pend_a, pend_b;
  DBuf<uint4> pend_c;
  DBuf<EventRec> ev_stage, ev_list;
  DBuf<float4> adj_hits;   // hit record per adjoint queue slot (3 float4)
  DBuf<float4> adj_walkq;  // walk record per sorted position (2 float4)
  // adjoint batches
  uint32_t adj_cap = 0;
  DBuf<uint32_t> adj_keys, adj_perm, adj_keys_tmp, adj_perm_tmp, adj_sort_temp;   // ray order of a bounce
  DBuf<AdjJob> d_jobs;
  DBuf<CameraRec> d_adj_cams;
  DBuf<uint32_t> job_count, job_start;
  // camera-gather wavefront
  uint32_t path_cap = 0;
  KernelTimer timer;          // device time of the hot kernels of the last call
  DBuf<RayRec> cg_paths, cg_paths2;
  DBuf<float4> cg_qrec, cg_info_b;
  DBuf<uint4> cg_info_a;
  DBuf<float4> cg_mhit, cg_walk;   // per round entry: mesh hit, walk record
  DBuf<uint32_t> cg_khit;          // per round entry: K-hit walk result
  DBuf<uint32_t> cg_counts;
  DBuf<float4> cg_res, cg_fb;
  // run state, seeds, images, gradients
  DBuf<RunState> run;
  DBuf<uint32_t> seeds_fwd, seeds_adj;
  DBuf<uint32_t> cam_cursor;   // seed cursor after the last photon pass
  DBuf<float> img_raw, img_ldr, dldi, dbg, target;
  DBuf<double> loss_part, loss;
  PointsBufs grads;
  // gather estimator: the vertex store (chunks of the last forward that
  // fit), the replay scratch (the largest chunk replayed), and what the
  // last forward rendered: its views, scenes and their BVH and photon-map
  // generations, which its backward must find unchanged
  VertexPlan vplan;
  std::vector<CameraRec> vviews;
  std::vector<pale_handle*> vscenes;
  std::vector<uint64_t> vgens;
  DBuf<float4> vs_rec_xa, vs_rec_ew, vs_ent_d, vs_ent_l, sc_rec_xa, sc_rec_ew, sc_ent_d, sc_ent_l;
  DBuf<uint4> vs_ent_b, sc_ent_b;
  DBuf<uint32_t> vs_base, vs_overflow, vs_chunk_base;
  DBuf<SceneGrads> vs_view_grads;   // per view gradient arrays of a per-view backward
  uint64_t photon_gen = 0;     // photon maps traced or loaded so far
  uint64_t params_gen = 0;     // surfel parameter writes so far
  uint64_t bvh_gen = 0;        // BVH builds so far
  uint64_t grads_gen = ~0ull;  // build the gradients belong to
  // optimizer state (BVH order; starts over after every build)
  PointsBufs opt_m, opt_v;
  DBuf<uint32_t> opt_steps;
  uint64_t opt_gen = ~0ull, opt_t = 0;
  uint32_t opt_type = ~0u;
  // density control scratch
  DBuf<uint32_t> dc_keys, dc_vals, dc_keys_tmp, dc_vals_tmp, dc_sort_temp, dc_flags, dc_dst, dc_list, dc_word, dc_aux;
  PointsBufs dc_points;
  HostStage stage;            // staging of large host copies
  pale_stats stats{};
  uint64_t launches_last = 0;  // kernels launched by the last render call
  int stats_pending = 0;   // a render ran without reading its run state yet
  int timed = 0;           // 1 forward events, 2 adjoint events pending
  cudaStream_t own_stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr;

  ~pale_handle() {
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (ev2) cudaEventDestroy(ev2);
    if (own_stream) cudaStreamDestroy(own_stream);
  }

  SceneView view() const {
    SceneView s{};
    s.mesh.o2w = o2w.p;
    s.mesh.w2o = w2o.p;
    s.mesh.box = inst_box.p;
    s.mesh.tri_range = tri_range.p;
    s.mesh.tri = tri.p;
    s.mesh.wtri = wtri.p;
    s.mesh.wtri_range = wtri_range.p;
    s.mesh.material = inst_mat.p;
    s.mesh.materials = materials.p;
    s.mesh.instances = n_inst;
    s.sf = SurfelView{sf_pe.p, sf_n.p, sf_u.p, sf_v.p, sf_cn.p, sf_alb.p, np};
#if PALE_HALF_NODES
    s.nodes = hnodes.p;
#else
    s.nodes = nodes.p;
#endif
    s.node_count = np ? node_count : 0;
    s.top_nodes = np ? std::min(top, node_count) : 0;
    s.pc_lo = v3(pc_lo[0], pc_lo[1], pc_lo[2]);
    s.pc_hi = v3(pc_hi[0], pc_hi[1], pc_hi[2]);
    s.has_pc = np > 0;
    s.lights = LightView{n_lights, light_rec.p, light_col.p, light_area.p, light_cdf.p, light_tri.p};
    GridView& g = s.grid;
    g.radius = radius;
    g.origin = v3(origin[0], origin[1], origin[2]);
    g.cell = v3(cell, cell, cell);
    g.res[0] = res[0]; g.res[1] = res[1]; g.res[2] = res[2];
    g.cells = cells;
    g.cell_off = g_cell_off.p;
    g.pa = g_pa.p;
    g.pb = g_pb.p;
    g.pc = g_pc.p;
    g.attempts = g_attempts.p;
    g.capacity = photon_cap;
    return s;
  }
};

namespace {

void check_points(const pale_points* p, const char* what) {
  if (!p) throw ArgError(std::string(what) + ": null point block");
  if (p->count && (!p->position || !p->tangent_u || !p->tangent_v || !p->scale || !p->albedo || !p->opacity ||
                   !p->beta))
    throw ArgError(std::string(what) + ": missing point field");
}

void upload_points(pale_handle* h, const pale_points* p, PointsBufs& dst, cudaStream_t s) {
  const uint32_t n = p->count;
  dst.alloc(n);
  if (!n) return;
  CK(cudaMemcpyAsync(dst.pos.p, p->position, 12ull * n, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(dst.tu.p, p->tangent_u, 12ull * n, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(dst.tv.p, p->tangent_v, 12ull * n, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(dst.sc.p, p->scale, 8ull * n, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(dst.alb.p, p->albedo, 12ull * n, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(dst.op.p, p->opacity, 4ull * n, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(dst.beta.p, p->beta, 4ull * n, cudaMemcpyHostToDevice, s));
  if (p->shape) CK(cudaMemcpyAsync(dst.shape.p, p->shape, 4ull * n, cudaMemcpyHostToDevice, s));
  else CK(cudaMemsetAsync(dst.shape.p, 0, 4ull * n, s));
  (void)h;
}

void build_from_device_asset(pale_handle* h);

// Builds the LBVH and surfel arrays from asset-order points.
void build_surfels(pale_handle* h, const pale_points* asset) {
  h->np = asset->count;
  upload_points(h, asset, h->asset, h->stream);
  build_from_device_asset(h);
}

// Builds the LBVH and surfel arrays from the device copy of the asset
// (h->asset, h->np points).
void build_from_device_asset(pale_handle* h) {
  cudaStream_t s = h->stream;
  const uint32_t n = h->np;
  h->collected.alloc(n);
  h->params.alloc(n);
  h->sf_pe.ensure(n); h->sf_n.ensure(n); h->sf_u.ensure(n); h->sf_v.ensure(n); h->sf_cn.ensure(n);
  h->sf_alb.ensure(n);
  h->grads.alloc(n);
  ++h->bvh_gen;
  if (n == 0) {
    h->node_count = 0;
    return;
  }
  h->aabb_lo.ensure(3 * (size_t)n); h->aabb_hi.ensure(3 * (size_t)n);
  h->bounds_part.ensure(12 * 148 * 4); h->bounds.ensure(12);
  h->codes.ensure(n); h->order.ensure(n); h->codes_tmp.ensure(n); h->order_tmp.ensure(n);
  h->sort_temp.ensure(radix_temp_words(n));
  h->lc.ensure(n); h->rc.ensure(n); h->rfirst.ensure(n); h->rlast.ensure(n); h->parent.ensure(n);
  h->leaf_parent.ensure(n); h->visits.ensure(n); h->box.ensure(6 * (size_t)n);
  h->d_n.ensure(1);
  const uint32_t leaf = std::max(1u, std::min(8u, h->st.leaf_size ? h->st.leaf_size : 1u));
  h->top = kTopNodes;
  h->node_count = (n <= leaf) ? 1 : h->top + (n - 1);
  if (n <= leaf) h->top = 0;
  h->nodes.ensure(h->node_count);
  CK(cudaMemcpyAsync(h->d_n.p, &n, 4, cudaMemcpyHostToDevice, s));
  LbvhArgs A{};
  A.n = n;
  A.d_n = h->d_n.p;
  A.leaf_size = leaf;
  A.top = h->top;
  A.asset = h->asset.view();
  A.collected = h->collected.view();
  A.params = h->params.view();
  A.derived = SurfelArrays{h->sf_pe.p, h->sf_n.p, h->sf_u.p, h->sf_v.p, h->sf_cn.p, h->sf_alb.p};
  A.lo = h->aabb_lo.p; A.hi = h->aabb_hi.p;
  A.bounds_part = h->bounds_part.p; A.bounds = h->bounds.p;
  A.codes = h->codes.p; A.order = h->order.p; A.codes_tmp = h->codes_tmp.p; A.order_tmp = h->order_tmp.p;
  A.sort_temp = h->sort_temp.p;
  A.lc = h->lc.p; A.rc = h->rc.p; A.rfirst = h->rfirst.p; A.rlast = h->rlast.p; A.parent = h->parent.p;
  A.leaf_parent = h->leaf_parent.p; A.visits = h->visits.p; A.box = h->box.p;
  A.nodes = h->nodes.p;
  A.err = &h->run.p->error;
  CK(cudaMemsetAsync(h->run.p, 0, sizeof(RunState), s));
  lbvh_build(A, s);
#if PALE_HALF_NODES
  h->hnodes.ensure(h->node_count);
  half_nodes(h->nodes.p, h->node_count, h->hnodes.p, s);
#endif
  CK(cudaGetLastError());
  float b[12];
  uint32_t err = 0;
  CK(cudaMemcpyAsync(b, h->bounds.p, sizeof(b), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(&err, &h->run.p->error, 4, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (err) throw std::runtime_error("LBVH build failed a consistency check (device error flags " +
                                    std::to_string(err) + ")");
  for (int k = 0; k < 3; ++k) {
    h->pc_lo[k] = b[6 + k];
    h->pc_hi[k] = b[9 + k];
  }
}

// Photon store (deposit order) and the sorted copy of the grid.
void alloc_photon_store(pale_handle* h, uint64_t cap) {
  h->photon_cap = cap;
  const size_t pc = (size_t)cap;
  h->ph_a.alloc(pc); h->ph_b.alloc(pc); h->ph_c.alloc(pc);
  h->g_pa.alloc(pc); h->g_pb.alloc(pc); h->g_pc.alloc(pc);
  h->g_cell_id.alloc(pc); h->g_sorted.alloc(pc); h->g_keys.alloc(2 * pc); h->g_vals_tmp.alloc(pc);
  h->g_sort_temp.alloc(radix_temp_words((uint32_t)pc));
}

// Host restatement of toWorldPoint with the device's operation order.
V3 host_xform_point(const float* M, V3 p) { return xform_point(M, p); }

// Ray queues (ping-pong, staging, flags, per-tile counts) of at least n
// slots: the photon passes need photons_per_launch, the adjoint its batch.
void size_queues(pale_handle* h, size_t n) {
  if (h->q0.n >= n) return;
  h->q0.alloc(n); h->q1.alloc(n); h->qstage.alloc(n); h->qflags.alloc(n);
  h->tile_counts.alloc(n / kBlock + 1); h->tile_offsets.alloc(n / kBlock + 1);
}

// The wavefront buffers of camera-gather and adjoint calls whose views hold
// all_pix pixels, the largest view max_pix (grown, never shrunk):
// - adjoint: the (view, pass) jobs of a call trace together, up to 2^24
//   paths per batch (about 5.4 GB of queues and events), or the
//   adjoint_batch_paths setting;
// - camera gather: every pass of every pixel in flight when that fits in
//   2^25 paths (3.2 GB of path queues, 8.6 GB of lookup records, 1 GB of
//   per-entry state), or the gather_batch_paths setting, else chunks of
//   whole passes; at least every pixel once.
void size_wavefronts(pale_handle* h, uint64_t all_pix, uint32_t max_pix) {
  const pale_settings& st = h->st;
  if (all_pix >= (1ull << 31)) throw ArgError("too many camera pixels");
  if (max_pix >= (1u << 24)) throw ArgError("a view of 2^24 pixels or more");
  const size_t qc = h->qcap;
  const uint64_t adj_want = all_pix * std::max<uint32_t>(1u, st.adjoint_passes);
  const uint64_t adj_limit = std::min<uint64_t>(st.adjoint_batch_paths ? st.adjoint_batch_paths : (1ull << 24),
                                                (1ull << 24));
  const uint32_t adj_cap = (uint32_t)std::max<uint64_t>(max_pix, std::min<uint64_t>(adj_want, adj_limit));
  if (adj_cap > h->adj_cap) {
    h->adj_cap = adj_cap;
    const size_t qa = std::max<size_t>(qc, h->adj_cap);
    h->adj_keys.alloc(h->adj_cap); h->adj_perm.alloc(h->adj_cap);
    h->adj_keys_tmp.alloc(h->adj_cap); h->adj_perm_tmp.alloc(h->adj_cap);
    h->adj_sort_temp.alloc(radix_temp_words(h->adj_cap));
    size_queues(h, qa);
    h->pend_a.alloc(qa); h->pend_b.alloc(qa); h->pend_c.alloc(qa);
    h->ev_stage.alloc(qa); h->ev_list.alloc(qa);
    h->adj_hits.alloc(3 * qa);
    h->adj_walkq.alloc(2 * qa);
  }
  const uint64_t want = all_pix * std::max<uint32_t>(1u, st.gather_passes);
  const uint64_t cg_limit = st.gather_batch_paths ? st.gather_batch_paths : (1ull << 25);
  const uint32_t path_cap =
      (uint32_t)std::max<uint64_t>(std::max<uint64_t>(all_pix, 1), std::min<uint64_t>(want, cg_limit));
  if (path_cap > h->path_cap) {
    h->path_cap = path_cap;
    h->cg_paths.alloc(h->path_cap); h->cg_paths2.alloc(h->path_cap);
    h->cg_qrec.alloc(2 * (size_t)kGatherHits * h->path_cap); h->cg_res.alloc(h->path_cap);
    h->cg_info_a.alloc(h->path_cap); h->cg_info_b.alloc(h->path_cap);
    h->cg_mhit.alloc(h->path_cap); h->cg_walk.alloc(2 * (size_t)h->path_cap);
    h->cg_khit.alloc((size_t)kKHitWords * h->path_cap);
  }
  h->cg_fb.ensure(std::max<uint64_t>(all_pix, 1));
}

void setup_scene(pale_handle* h, const pale_scene_desc* d) {
  cudaStream_t s = h->stream;
  h->run.alloc(1);
  CK(cudaMemsetAsync(h->run.p, 0, sizeof(RunState), s));
  // ---- meshes: per instance transforms, world boxes, triangles
  h->n_inst = d->num_instances;
  h->n_tris = d->num_triangles;
  for (uint32_t i = 0; i < d->num_instances; ++i) {
    if (d->instance_mesh[i] >= d->num_meshes) throw ArgError("instance mesh index out of range");
    if (d->instance_material[i] >= d->num_materials) throw ArgError("instance material index out of range");
  }
  for (uint32_t t = 0; t < 3 * d->num_triangles; ++t)
    if (d->triangles[t] >= d->num_vertices) throw ArgError("triangle vertex index out of range");
  for (uint32_t m = 0; m < d->num_meshes; ++m)
    if ((uint64_t)d->mesh_ranges[2 * m] + d->mesh_ranges[2 * m + 1] > d->num_triangles)
      throw ArgError("mesh range out of range");
  std::vector<float4> tri(3 * (size_t)std::max(1u, d->num_triangles));
  for (uint32_t t = 0; t < d->num_triangles; ++t)
    for (int c = 0; c < 3; ++c) {
      const float* v = d->vertices + 3 * d->triangles[3 * t + c];
      tri[3 * t + c] = make_float4(v[0], v[1], v[2], 0.f);
    }
  std::vector<uint2> rng(std::max(1u, h->n_inst));
  std::vector<float4> box(2 * (size_t)std::max(1u, h->n_inst));
  h->h_inst_box.assign(6 * (size_t)h->n_inst, 0.f);
  for (uint32_t i = 0; i < h->n_inst; ++i) {
    uint32_t m = d->instance_mesh[i];
    uint32_t first = d->mesh_ranges[2 * m], cnt = d->mesh_ranges[2 * m + 1];
    rng[i] = make_uint2(first, cnt);
    V3 bl = v3(INFINITY, INFINITY, INFINITY), bh = v3(-INFINITY, -INFINITY, -INFINITY);
    for (uint32_t k = 0; k < cnt; ++k)
      for (int c = 0; c < 3; ++c) {
        const float* v = d->vertices + 3 * d->triangles[3 * (first + k) + c];
        bl = vmin(bl, v3(v[0], v[1], v[2]));
        bh = vmax(bh, v3(v[0], v[1], v[2]));
      }
    // buildTLAS world box: the 8 transformed corners (SceneBuild.cpp:562-581)
    V3 wl = v3(3.402823466e+38f, 3.402823466e+38f, 3.402823466e+38f);
    V3 wh = v3(-3.402823466e+38f, -3.402823466e+38f, -3.402823466e+38f);
    for (int c = 0; c < 8; ++c) {
      V3 p = v3((c & 4) ? bh.x : bl.x, (c & 2) ? bh.y : bl.y, (c & 1) ? bh.z : bl.z);
      V3 pw = host_xform_point(d->instance_object_to_world + 16 * i, p);
      wl = vmin(wl, pw);
      wh = vmax(wh, pw);
    }
    box[2 * i] = make_float4(wl.x, wl.y, wl.z, 0.f);
    box[2 * i + 1] = make_float4(wh.x, wh.y, wh.z, 0.f);
    float* hb = &h->h_inst_box[6 * i];
    hb[0] = wl.x; hb[1] = wl.y; hb[2] = wl.z; hb[3] = wh.x; hb[4] = wh.y; hb[5] = wh.z;
  }
  // world-space copies of every instance's triangles (the vertices of the
  // mesh-hit normals, buildIntersectionNormal)
  std::vector<float4> wtri;
  std::vector<uint2> wrng(std::max(1u, h->n_inst));
  for (uint32_t i = 0; i < h->n_inst; ++i) {
    wrng[i] = make_uint2((uint32_t)(wtri.size() / 3), rng[i].y);
    for (uint32_t k = 0; k < rng[i].y; ++k)
      for (int c = 0; c < 3; ++c) {
        const float4 v = tri[3 * (rng[i].x + k) + c];
        const V3 pw = host_xform_point(d->instance_object_to_world + 16 * i, v3(v.x, v.y, v.z));
        wtri.push_back(make_float4(pw.x, pw.y, pw.z, 0.f));
      }
  }
  if (wtri.empty()) wtri.assign(3, make_float4(0.f, 0.f, 0.f, 0.f));
  h->wtri.alloc(wtri.size());
  h->wtri_range.alloc(wrng.size());
  CK(cudaMemcpyAsync(h->wtri.p, wtri.data(), wtri.size() * sizeof(float4), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(h->wtri_range.p, wrng.data(), wrng.size() * sizeof(uint2), cudaMemcpyHostToDevice, s));
  h->o2w.alloc(16 * (size_t)std::max(1u, h->n_inst));
  h->w2o.alloc(16 * (size_t)std::max(1u, h->n_inst));
  h->inst_box.alloc(box.size());
  h->tri_range.alloc(rng.size());
  h->tri.alloc(tri.size());
  h->inst_mat.alloc(std::max(1u, h->n_inst));
  h->materials.alloc(std::max(1u, d->num_materials));
  if (h->n_inst) {
    CK(cudaMemcpyAsync(h->o2w.p, d->instance_object_to_world, 64ull * h->n_inst, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(h->w2o.p, d->instance_world_to_object, 64ull * h->n_inst, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(h->inst_mat.p, d->instance_material, 4ull * h->n_inst, cudaMemcpyHostToDevice, s));
  }
  CK(cudaMemcpyAsync(h->inst_box.p, box.data(), box.size() * sizeof(float4), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(h->tri_range.p, rng.data(), rng.size() * sizeof(uint2), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(h->tri.p, tri.data(), tri.size() * sizeof(float4), cudaMemcpyHostToDevice, s));
  std::vector<float4> mats(std::max(1u, d->num_materials));
  for (uint32_t k = 0; k < d->num_materials; ++k)
    mats[k] = make_float4(d->materials[4 * k], d->materials[4 * k + 1], d->materials[4 * k + 2], d->materials[4 * k + 3]);
  CK(cudaMemcpyAsync(h->materials.p, mats.data(), mats.size() * sizeof(float4), cudaMemcpyHostToDevice, s));

  // ---- lights: world-area CDF per emissive instance (SceneBuild.cpp:263-343)
  std::vector<uint4> lrec;
  std::vector<float4> lcol;
  std::vector<float> larea, lcdf;
  std::vector<uint32_t> ltri;
  for (uint32_t i = 0; i < h->n_inst; ++i) {
    const float* mat = d->materials + 4 * d->instance_material[i];
    if (!(mat[3] > 0.f)) continue;
    uint32_t m = d->instance_mesh[i];
    uint32_t first = d->mesh_ranges[2 * m], cnt = d->mesh_ranges[2 * m + 1];
    if (cnt == 0) continue;
    const float* O2W = d->instance_object_to_world + 16 * i;
    std::vector<float> areas(cnt);
    float total = 0.f;
    for (uint32_t k = 0; k < cnt; ++k) {
      const uint32_t* tr = d->triangles + 3 * (first + k);
      auto P = [&](int c) { const float* v = d->vertices + 3 * tr[c]; return host_xform_point(O2W, v3(v[0], v[1], v[2])); };
      V3 w0 = P(0), w1 = P(1), w2 = P(2);
      areas[k] = 0.5f * length(cross(w1 - w0, w2 - w0));
      total += areas[k];
    }
    if (total <= 0.f) continue;
    uint32_t off = (uint32_t)lcdf.size();
    float run = 0.f;
    for (uint32_t k = 0; k < cnt; ++k) {
      run += areas[k];
      lcdf.push_back(run / total);
      ltri.push_back(first + k);
    }
    lcdf[off + cnt - 1] = 1.0f;
    lrec.push_back(make_uint4(i, off, cnt, 0));
    lcol.push_back(make_float4(mat[0], mat[1], mat[2], mat[3]));
    larea.push_back(total);
  }
  h->n_lights = (uint32_t)lrec.size();
  h->light0_area = h->n_lights ? larea[0] : 0.f;
  h->light_rec.alloc(std::max<size_t>(1, lrec.size()));
  h->light_col.alloc(std::max<size_t>(1, lcol.size()));
  h->light_area.alloc(std::max<size_t>(1, larea.size()));
  h->light_cdf.alloc(std::max<size_t>(1, lcdf.size()));
  h->light_tri.alloc(std::max<size_t>(1, ltri.size()));
  if (h->n_lights) {
    CK(cudaMemcpyAsync(h->light_rec.p, lrec.data(), lrec.size() * sizeof(uint4), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(h->light_col.p, lcol.data(), lcol.size() * sizeof(float4), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(h->light_area.p, larea.data(), larea.size() * 4, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(h->light_cdf.p, lcdf.data(), lcdf.size() * 4, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(h->light_tri.p, ltri.data(), ltri.size() * 4, cudaMemcpyHostToDevice, s));
  }

  // ---- cameras (makePrimaryRayFromPixelJitteredFov constants)
  h->cams.resize(d->num_cameras);
  h->cam_names.resize(d->num_cameras);
  uint32_t max_pix = 0;
  uint64_t all_pix = 0;
  for (uint32_t c = 0; c < d->num_cameras; ++c) {
    CameraRec& C = h->cams[c];
    std::memset(&C, 0, sizeof(C));
    std::memcpy(C.inv_view, d->camera_inv_view + 16 * c, 64);
    C.w = d->camera_size[2 * c];
    C.h = d->camera_size[2 * c + 1];
    if (C.w == 0 || C.h == 0) throw ArgError("camera with zero size");
    C.width = (float)C.w;
    C.height = (float)C.h;
    C.half_w = 0.5f * C.width;
    C.half_h = 0.5f * C.height;
    C.fy = 0.5f * C.height / std::tan(0.5f * (d->camera_fovy_deg[c] * 0.01745329251994329576923690768489f));
    C.fx = C.fy * (C.width / C.height);
    max_pix = std::max(max_pix, C.w * C.h);
    all_pix += (uint64_t)C.w * C.h;
    char nm[17];
    std::memset(nm, 0, sizeof(nm));
    if (d->camera_names) std::memcpy(nm, d->camera_names + 16 * c, 16);
    h->cam_names[c] = nm;
  }
  h->d_cams.alloc(std::max<size_t>(1, d->num_cameras));

  // ---- surfels + LBVH
  build_surfels(h, &d->points);

  // ---- photon grid from the scene box (configurePhotonGrid, PathTracer.cpp:184-221)
  V3 lo = v3(INFINITY, INFINITY, INFINITY), hi = v3(-INFINITY, -INFINITY, -INFINITY);
  for (uint32_t i = 0; i < h->n_inst; ++i) {
    const float* b = &h->h_inst_box[6 * i];
    lo = vmin(lo, v3(b[0], b[1], b[2]));
    hi = vmax(hi, v3(b[3], b[4], b[5]));
  }
  if (h->np) {
    lo = vmin(lo, v3(h->pc_lo[0], h->pc_lo[1], h->pc_lo[2]));
    hi = vmax(hi, v3(h->pc_hi[0], h->pc_hi[1], h->pc_hi[2]));
  }
  if (!(lo.x <= hi.x)) throw ArgError("scene is empty");
  h->radius = h->st.gather_radius;
  const float cs = 0.5f * h->radius;
  h->cell = cs;
  V3 pad = v3(h->radius, h->radius, h->radius);
  V3 org = lo - pad, gmax = hi + pad, ext = gmax - org;
  h->origin[0] = org.x; h->origin[1] = org.y; h->origin[2] = org.z;
  const float safe = std::fmax(cs, 1e-6f);
  h->res[0] = (int)std::ceil(ext.x / safe);
  h->res[1] = (int)std::ceil(ext.y / safe);
  h->res[2] = (int)std::ceil(ext.z / safe);
  uint64_t tot = (uint64_t)h->res[0] * h->res[1] * h->res[2];
  // the cell-offset scan handles up to 2^28 cells
  if (tot == 0 || tot >= (1ull << 28)) throw ArgError("Photon grid resolution too high; increase r or tighten AABB.");
  h->cells = (uint32_t)tot;
  h->key_bits = 1;
  while (h->key_bits < 32 && ((uint64_t)1 << h->key_bits) < tot) ++h->key_bits;

  // ---- photon store (PathTracer.cpp:123-144): photons x passes x bounces,
  // clamped to 10 GiB of the reference's 64-byte records
  const pale_settings& st = h->st;
  uint64_t req = (uint64_t)st.photons_per_launch * st.forward_passes * st.max_bounces;
  uint64_t mx = (10ull << 30) / 64ull;
  alloc_photon_store(h, std::max<uint64_t>(1, std::min(req, mx)));
  h->g_cell_count.alloc((size_t)h->cells + 1);
  h->g_cell_off.alloc((size_t)h->cells + 1);
  h->g_scan_temp.alloc(scan_temp_words(h->cells + 1));
  h->g_stored.alloc(1);
  h->g_attempts.alloc(1);
  h->cam_cursor.alloc(1);
  CK(cudaMemsetAsync(h->cam_cursor.p, 0, 4, s));
  CK(cudaMemsetAsync(h->g_stored.p, 0, 4, s));
  CK(cudaMemsetAsync(h->g_attempts.p, 0, 4, s));
  CK(cudaMemsetAsync(h->g_cell_off.p, 0, ((size_t)h->cells + 1) * 4, s));

  // ---- queues: next power of two >= max(photons per launch, pixels)
  h->qcap = next_pow2(std::max(std::max(st.photons_per_launch, max_pix), 256u));
  const size_t qc = h->qcap;
  h->ph_sa.alloc(qc); h->ph_sb.alloc(qc); h->ph_sc.alloc(qc);
  h->job_count.alloc(2 * kMaxJobsPerBatch);
  h->job_start.alloc(2 * kMaxJobsPerBatch);
  h->cg_counts.alloc(2 * (kMaxLayers + 2));
  // the photon queues now; the camera-gather and adjoint wavefronts when a
  // call first renders through this handle (size_wavefronts), so that a
  // scene that only lends its data to batched calls holds none
  size_queues(h, qc);
  (void)all_pix;
  CK(cudaMemsetAsync(h->run.p, 0, sizeof(RunState), s));
  CK(cudaStreamSynchronize(s));
}

std::vector<uint32_t> mt_table(uint64_t seed, size_t n) {
  std::mt19937_64 g(seed);
  std::vector<uint32_t> t(n);
  for (size_t i = 0; i < n; ++i) t[i] = (uint32_t)g();
  return t;
}

int fail(pale_handle* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  else g_create_error = msg;
  return code;
}

template <typename F>
int guarded(pale_handle* h, F&& f) {
  try {
    return f();
  } catch (const ArgError& e) {
    return fail(h, PALE_ERR_ARGUMENT, e.what());
  } catch (const CudaError& e) {
    return fail(h, PALE_ERR_CUDA, e.what());
  } catch (const std::exception& e) {
    return fail(h, PALE_ERR_STATE, e.what());
  }
}

// Reads the run state of the last render (synchronising its stream) into
// h->stats, with the device times of the recorded events; throws when a
// kernel raised an error flag.
void copy_stats(pale_handle* h) {
  h->stats_pending = 0;
  RunState rs;
  CK(cudaMemcpyAsync(&rs, h->run.p, sizeof(rs), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (h->timed == 1) {
    float a = 0.f, b = 0.f;
    CK(cudaEventElapsedTime(&a, h->ev0, h->ev1));
    CK(cudaEventElapsedTime(&b, h->ev1, h->ev2));
    h->stats.photon_ms = a;
    h->stats.gather_ms = b;
    h->stats.forward_ms = a + b;
  } else if (h->timed == 2) {
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    h->stats.backward_ms = ms;
  }
  h->timed = 0;
  for (int k = 0; k < kTimedKernels; ++k) {
    h->stats.timed_ms[k] = 0.f;
    h->stats.timed_launches[k] = 0;
  }
  h->timer.collect(h->stats.timed_ms, h->stats.timed_launches);
  h->stats.photon_segments = rs.photon_segments;
  h->stats.gather_segments = rs.gather_segments;
  h->stats.adjoint_segments = rs.adjoint_segments;
  h->stats.photons_stored = std::min<uint64_t>(rs.photon_attempts, h->photon_cap);
  h->stats.gradient_events = rs.gradient_events;
  h->stats.gather_queries = rs.gather_queries;
  h->stats.node_visits = rs.node_visits;
  h->stats.surfel_tests = rs.surfel_tests;
  h->stats.photons_scanned = rs.photons_scanned;
  h->stats.gather_node_visits = rs.gather_node_visits;
  h->stats.gather_surfel_tests = rs.gather_surfel_tests;
  h->stats.gather_photons_scanned = rs.gather_photons_scanned;
  h->stats.kernel_launches = h->launches_last;
  if (rs.error) {
    char buf[128];
    std::snprintf(buf, sizeof(buf), "device error flags 0x%x (1 stack, 2 layer cap, 4 photon capacity, 8 bounds, 16 queue)",
                  rs.error);
    throw std::runtime_error(buf);
  }
}

// The stream a device entry point runs on: the caller's, where NULL is the
// default stream (the legacy stream), so that the work is ordered with the
// caller's default-stream work.
cudaStream_t caller_stream(void* stream) { return stream ? (cudaStream_t)stream : cudaStreamLegacy; }

// Makes `s` the stream of the following work, ordered after everything
// already queued on the previous stream of this handle.
void use_stream(pale_handle* h, cudaStream_t s) {
  if (s == h->stream) return;
  cudaEvent_t e;
  CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  CK(cudaEventRecord(e, h->stream));
  CK(cudaStreamWaitEvent(s, e, 0));
  CK(cudaEventDestroy(e));
  h->stream = s;
}

void validate_cams(pale_handle* h, uint32_t nsel, const uint32_t* idx) {
  if (nsel && !idx) throw ArgError("camera index list is null");
  for (uint32_t i = 0; i < nsel; ++i)
    if (idx[i] >= h->cams.size()) throw ArgError("camera index out of range");
}

// Optional image loss of a forward pass (device pointers).
struct LossReq {
  const float* target;
  uint32_t channels;
  float* dldi;     // may be null
  double* loss;    // may be null
};

// One view of a render call: a camera of one of the call's scenes, with its
// passes (gather and adjoint) and adjoint bounces.
struct ViewReq {
  uint32_t scene;    // index into the call's scene list
  uint32_t cam;      // camera index in that scene
  uint32_t passes;
  uint32_t depth;
  uint32_t first = 0, count = 0;   // forward slices: passes [first, first + count) (0, 0: all)
};

// The views of a one-scene call: the selected cameras with the scene's
// gather passes (forward) or adjoint passes (adjoint) and its bounces.
std::vector<ViewReq> all_passes(pale_handle* h, uint32_t nsel, const uint32_t* idx, bool adjoint) {
  std::vector<ViewReq> v(nsel);
  const uint32_t passes = adjoint ? h->st.adjoint_passes : h->st.gather_passes;
  for (uint32_t i = 0; i < nsel; ++i) v[i] = ViewReq{0u, idx[i], passes, h->st.adjoint_bounces, 0u, 0u};
  return v;
}

// adjoint: the views' passes are adjoint passes (at most the scene's
// adjoint_passes), else gather passes (at most its gather_passes).
// allow_twice: one scene may fill several entries of the list (an adjoint
// call whose entries have gradient arrays of their own).
void check_views(const std::vector<pale_handle*>& scenes, const std::vector<ViewReq>& views, bool adjoint,
                 bool allow_twice = false) {
  if (scenes.empty() || scenes.size() > kMaxScenes) throw ArgError("a call renders 1 to 8 scenes");
  for (size_t k = 0; k < scenes.size(); ++k) {
    if (!scenes[k]) throw ArgError("null scene handle");
    for (size_t j = 0; j < k && !allow_twice; ++j)
      if (scenes[j] == scenes[k]) throw ArgError("a scene appears twice in the scene list");
  }
  for (const ViewReq& v : views) {
    if (v.scene >= scenes.size()) throw ArgError("view scene index out of range");
    pale_handle* h = scenes[v.scene];
    if (v.cam >= h->cams.size()) throw ArgError("camera index out of range");
    if (v.passes == 0 || v.passes > (adjoint ? h->st.adjoint_passes : h->st.gather_passes))
      throw ArgError(adjoint ? "view passes must be 1 .. the scene's adjoint_passes"
                             : "view passes must be 1 .. the scene's gather_passes");
    if (v.depth > h->st.adjoint_bounces) throw ArgError("view depth above the scene's adjoint bounces");
    if (v.first || v.count) {
      if (adjoint) throw ArgError("an adjoint call renders every pass of its views");
      if (v.count == 0 || v.first >= v.passes || v.count > v.passes - v.first)
        throw ArgError("view pass range outside its passes");
    }
  }
}

// The camera seeds a scene's forward render uses: one per camera of the
// scene (camera_seeds = camera) or one per view of the scene in the call
// (the reference's order of the selection).
std::vector<uint32_t> seed_slots(const std::vector<pale_handle*>& scenes, const std::vector<ViewReq>& views) {
  std::vector<uint32_t> slot(views.size()), rank(scenes.size(), 0u);
  for (size_t i = 0; i < views.size(); ++i) {
    const uint32_t k = views[i].scene;
    slot[i] = scenes[k]->st.camera_seeds == PALE_CAMERA_SEEDS_CAMERA ? views[i].cam : rank[k];
    ++rank[k];
  }
  return slot;
}

// The seed table of a scene's forward render (submitPhotonMappingKernel's
// stream: passes x (1 + bounces) photon seeds, then the camera seeds).
void forward_seeds(pale_handle* h, size_t cam_words) {
  const pale_settings& st = h->st;
  const size_t words = std::max<size_t>(cam_words, h->cams.size());
  std::vector<uint32_t> seeds = mt_table(st.seed, (size_t)st.forward_passes * (1 + st.max_bounces) + words + 1);
  h->seeds_fwd.ensure(seeds.size());
  CK(cudaMemcpyAsync(h->seeds_fwd.p, seeds.data(), seeds.size() * 4, cudaMemcpyHostToDevice, h->stream));
}

// The photon passes and the photon grid of scene h on its stream
// (submitPhotonMappingKernel, SyclBridge.cpp:82-138); the seed cursor
// where the camera seeds start is kept in h->cam_cursor.
void trace_photon_map(pale_handle* h) {
  cudaStream_t s = h->stream;
  const pale_settings& st = h->st;
  PhotonArgs P{};
  P.scene = h->view();
  P.st = h->run.p;
  P.seeds = h->seeds_fwd.p;
  P.qb = QueueBufs{{h->q0.p, h->q1.p}, h->qstage.p, h->qflags.p, h->tile_counts.p, h->tile_offsets.p, h->qcap};
  P.ps = PhotonStore{h->ph_a.p, h->ph_b.p, h->ph_c.p, h->ph_sa.p, h->ph_sb.p, h->ph_sc.p, h->photon_cap};
  P.photons_per_launch = st.photons_per_launch;
  P.inv_emitted = 1.0f / (float)(st.photons_per_launch * st.forward_passes);
  P.rr_start = st.rr_start;
  P.q_null = st.q_null;
  P.q_reflect = st.q_reflect;
  P.q_transmit = st.q_transmit;
  if (st.photons_per_launch > h->qcap) throw ArgError("photons per launch exceed the queue capacity");
  for (uint32_t pass = 0; pass < st.forward_passes; ++pass) {
    photon_emit(P, s);
    for (uint32_t b = 0; b < st.max_bounces; ++b) photon_bounce(P, b & 1u, s);
  }
  GridBufs G{};
  G.cell_id = h->g_cell_id.p;
  G.sorted = h->g_sorted.p;
  G.keys_tmp = h->g_keys.p;
  G.vals_tmp = h->g_vals_tmp.p;
  G.sort_temp = h->g_sort_temp.p;
  G.cell_count = h->g_cell_count.p;
  G.cell_off = h->g_cell_off.p;
  G.scan_temp = h->g_scan_temp.p;
  G.pa = h->g_pa.p;
  G.pb = h->g_pb.p;
  G.pc = h->g_pc.p;
  G.d_stored = h->g_stored.p;
  G.d_attempts = h->g_attempts.p;
  grid_build(P.scene, h->run.p, P.ps, G, h->cells, h->key_bits, s);
  CK(cudaMemcpyAsync(h->cam_cursor.p, &h->run.p->seed_cursor, sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
  ++h->photon_gen;
}

// The scene table of a call: every scene's view, with the same number of
// LBVH top nodes staged per scene (256 shared among them).
SceneTable scene_table(const std::vector<pale_handle*>& scenes) {
  SceneTable T{};
  T.n = (uint32_t)scenes.size();
  // each scene's slot: its top nodes up to kTopNodes, within 1024 nodes
  // (32 KB of shared memory) for the whole table
  const uint32_t slot = std::min<uint32_t>(kTopNodes, std::max<uint32_t>(32u, kStagedNodesPerCall / T.n));
  for (uint32_t k = 0; k < T.n; ++k) {
    T.s[k] = scenes[k]->view();
    T.s[k].top_nodes = std::min(T.s[k].top_nodes, slot);
  }
  T.staged = slot;
  return T;
}

// The views' camera records, packed in call order.
std::vector<CameraRec> view_records(const std::vector<pale_handle*>& scenes, const std::vector<ViewReq>& views,
                                    uint32_t& total, uint32_t& max_pix) {
  const std::vector<uint32_t> slots = seed_slots(scenes, views);
  std::vector<CameraRec> sel(views.size());
  total = 0;
  max_pix = 0;
  for (size_t i = 0; i < views.size(); ++i) {
    const ViewReq& v = views[i];
    sel[i] = scenes[v.scene]->cams[v.cam];
    sel[i].pixel_offset = total;
    sel[i].seed_slot = slots[i];
    sel[i].passes = v.passes;
    sel[i].scene = v.scene;
    sel[i].depth = v.depth ? v.depth : scenes[v.scene]->st.adjoint_bounces;
    sel[i].pass_begin = v.count ? v.first : 0u;
    sel[i].pass_end = v.count ? v.first + v.count : v.passes;
    total += sel[i].w * sel[i].h;
    max_pix = std::max(max_pix, sel[i].w * sel[i].h);
  }
  return sel;
}

// The camera gather's arguments for the views whose records are in
// h->d_cams (h = scenes[0], whose wavefront buffers the gather uses).
FrameArgs frame_args(const std::vector<pale_handle*>& scenes, uint32_t nsel, uint32_t total) {
  pale_handle* h = scenes[0];
  FrameArgs F{};
  F.scenes = scene_table(scenes);
  for (size_t k = 0; k < scenes.size(); ++k) F.sseeds[k] = SceneSeeds{scenes[k]->seeds_fwd.p, scenes[k]->cam_cursor.p};
  F.st = h->run.p;
  F.cams = h->d_cams.p;
  F.ncams = nsel;
  F.total_pixels = total;
  F.rng_mode = h->st.rng_mode;
  F.exposure = h->st.exposure;
  F.gamma = h->st.gamma;
  F.paths[0] = h->cg_paths.p;
  F.paths[1] = h->cg_paths2.p;
  F.qrec = h->cg_qrec.p;
  F.info_a = h->cg_info_a.p;
  F.info_b = h->cg_info_b.p;
  F.mhit = h->cg_mhit.p;
  F.walk = h->cg_walk.p;
  F.khit = h->cg_khit.p;
  F.counts = h->cg_counts.p;
  F.res = h->cg_res.p;
  F.fb = h->cg_fb.p;
  F.path_capacity = h->path_cap;
  F.walk_block = h->st.walk_block;
  F.timer = &h->timer;
  return F;
}

// Bytes of the vertex store per record slot and per entry slot.
constexpr uint64_t kRecSlotBytes = 2 * sizeof(float4), kEntSlotBytes = 2 * sizeof(float4) + sizeof(uint4);

// Before a forward with the gather estimator: the store grows to hold every
// chunk of the previous forward (with 1/16 to spare) in the "checkpoint"
// mode; in "auto" to that or to the budget (vertex_store_bytes; 0 = half
// the device memory free now), whichever is smaller, which then holds the
// first chunks.  A training loop renders the same views every iteration, so
// from its second iteration on the chunks that fit are kept.
void vertex_store_grow(pale_handle* h) {
  const pale_settings& st = h->st;
  if (st.vertex_store == PALE_VERTICES_REPLAY) return;
  uint64_t recs = 0, ents = 0;
  for (const VertexChunk& c : h->vplan.chunks) {
    recs += c.recs;
    ents += c.ents;
  }
  recs += recs / 16 + 1024;
  ents += ents / 16 + 1024;
  recs = std::min<uint64_t>(recs, 0xFFFFFFFFull);   // slots are 32-bit: the chunks past them are replayed
  ents = std::min<uint64_t>(ents, 0xFFFFFFFFull);
  if (st.vertex_store == PALE_VERTICES_AUTO) {
    // within the budget: as large a share of the need as it holds
    uint64_t budget = st.vertex_store_bytes;
    if (!budget) {
      size_t free_b = 0, total_b = 0;
      CK(cudaMemGetInfo(&free_b, &total_b));
      budget = free_b / 2 + h->vs_rec_xa.n * kRecSlotBytes + h->vs_ent_d.n * kEntSlotBytes;
    }
    const uint64_t bytes = recs * kRecSlotBytes + ents * kEntSlotBytes;
    if (bytes > budget) {
      const double f = (double)budget / (double)bytes;
      recs = (uint64_t)(recs * f);
      ents = (uint64_t)(ents * f);
    }
  }
  if (recs <= h->vs_rec_xa.n && ents <= h->vs_ent_d.n) return;
  CK(cudaStreamSynchronize(h->stream));
  h->vs_rec_xa.alloc(recs); h->vs_rec_ew.alloc(recs);
  h->vs_ent_d.alloc(ents); h->vs_ent_b.alloc(ents); h->vs_ent_l.alloc(ents);
}

uint64_t vertex_bytes(const pale_handle* h) {
  return h->vs_rec_xa.n * kRecSlotBytes + h->vs_ent_d.n * kEntSlotBytes + h->sc_rec_xa.n * kRecSlotBytes +
         h->sc_ent_d.n * kEntSlotBytes;
}

// The forward render of `views` into packed device images, on the stream
// of scenes[0], whose wavefront buffers the call uses; the other scenes
// lend their scene data (surfels, LBVH, meshes, photon grid).  With
// trace_photons every scene first traces its photon map; without, the
// camera gather runs on the current photon maps (the last forward's or
// loaded photons) with the camera seeds the last forward used.
uint32_t render_views(const std::vector<pale_handle*>& scenes, const std::vector<ViewReq>& views, float* d_raw,
                      float* d_ldr, bool sync, bool trace_photons, const LossReq* lq, float* d_partial = nullptr) {
  pale_handle* h = scenes[0];
  cudaStream_t s = h->stream;
  h->timer.used = 0;
  const uint64_t launches0 = launches_issued();
  check_views(scenes, views, false);
  bool sliced = false;
  for (const ViewReq& v : views) sliced = sliced || v.count != 0;
  if (sliced && !d_partial) throw ArgError("views rendered in slices need the running sums (d_partial)");
  if (sliced && trace_photons)
    throw ArgError("views rendered in slices keep one photon map: trace it first, then render without trace_photons");
  uint32_t total = 0, max_pix = 0;
  std::vector<CameraRec> sel = view_records(scenes, views, total, max_pix);
  size_wavefronts(h, total, max_pix);
  const uint32_t nsel = (uint32_t)sel.size();
  h->d_cams.ensure(std::max<size_t>(1, nsel));
  h->d_view_start.ensure(3 * std::max<size_t>(1, nsel));   // the gather chunks' view tables
  if (nsel) CK(cudaMemcpyAsync(h->d_cams.p, sel.data(), nsel * sizeof(CameraRec), cudaMemcpyHostToDevice, s));
  // photon maps of the scenes that some view renders (a scene of the list
  // without views, such as a handle that only lends its wavefront buffers,
  // is left alone)
  std::vector<char> used(scenes.size(), 0);
  for (const ViewReq& v : views) used[v.scene] = 1;
  CK(cudaMemsetAsync(h->run.p, 0, sizeof(RunState), s));
  CK(cudaEventRecord(h->ev0, s));
  for (size_t k = 0; k < scenes.size(); ++k) {
    pale_handle* sk = scenes[k];
    if (!used[k]) continue;
    forward_seeds(sk, views.size());
    if (trace_photons) {
      if (sk != h) CK(cudaMemsetAsync(sk->run.p, 0, sizeof(RunState), s));
      trace_photon_map(sk);
    }
  }
  CK(cudaEventRecord(h->ev1, s));
  FrameArgs F = frame_args(scenes, nsel, total);
  F.raw = d_raw;
  F.ldr = d_ldr;
  if (d_partial) F.fb = reinterpret_cast<float4*>(d_partial);   // the caller's running sums
  if (lq) {
    F.target = lq->target;
    F.target_channels = lq->channels;
    F.dldi = lq->dldi;
  }
  VertexPlan* plan = nullptr;
  if (h->st.estimator == PALE_ESTIMATOR_GATHER && !sliced) {
    // keep the path vertices: in the store while the chunks fit, else only
    // their counts (the backward replays those chunks)
    plan = &h->vplan;
    vertex_store_grow(h);
    const size_t nchunks = gather_chunks(sel, h->path_cap).size();
    h->vs_base.ensure(2 * kVertexBases);
    h->vs_overflow.ensure(1);
    h->vs_chunk_base.ensure(std::max<size_t>(1, nchunks) * 2 * kVertexBases);
    plan->d_chunk_base = h->vs_chunk_base.p;
    plan->store = h->st.vertex_store != PALE_VERTICES_REPLAY && h->vs_rec_xa.p && h->vs_ent_d.p;
    F.vs = VertexStore{h->vs_rec_xa.p, h->vs_rec_ew.p, h->vs_ent_d.p, h->vs_ent_b.p, h->vs_ent_l.p, h->vs_base.p,
                       h->vs_overflow.p, (uint32_t)h->vs_rec_xa.n, (uint32_t)h->vs_ent_d.n, 0u, 0u, 0};
    h->vviews.clear();   // valid again once the gather has run
  }
  if (h->st.estimator == PALE_ESTIMATOR_GATHER && sliced) h->vviews.clear();   // nothing to differentiate
  camera_gather(F, sel, h->d_view_start.p, s, plan);
  if (plan) {
    h->vviews = sel;
    h->vscenes = scenes;
    h->vgens.clear();
    for (pale_handle* sk : scenes) {
      h->vgens.push_back(sk->bvh_gen);
      h->vgens.push_back(sk->photon_gen);
      h->vgens.push_back(sk->params_gen);
    }
  }
  if (lq && lq->loss) {
    h->loss_part.ensure((size_t)std::max(1u, nsel) * kLossChunks);
    image_loss(F, h->loss_part.p, lq->loss, s);
  }
  CK(cudaEventRecord(h->ev2, s));
  CK(cudaGetLastError());
  h->launches_last = launches_issued() - launches0;
  h->timed = 1;
  h->stats_pending = 1;
  if (sync) copy_stats(h);
  return total;
}

uint32_t forward(pale_handle* h, uint32_t nsel, const uint32_t* idx, float* d_raw, float* d_ldr, bool sync,
                 bool trace_photons = true, const LossReq* lq = nullptr) {
  validate_cams(h, nsel, idx);
  return render_views({h}, all_passes(h, nsel, idx, false), d_raw, d_ldr, sync, trace_photons, lq);
}

void zero_grads(pale_handle* h, cudaStream_t s) {
  const size_t n = h->np ? h->np : 1;
  PointsBufs& g = h->grads;
  h->grads_gen = h->bvh_gen;
  CK(cudaMemsetAsync(g.pos.p, 0, 12 * n, s));
  CK(cudaMemsetAsync(g.tu.p, 0, 12 * n, s));
  CK(cudaMemsetAsync(g.tv.p, 0, 12 * n, s));
  CK(cudaMemsetAsync(g.sc.p, 0, 8 * n, s));
  CK(cudaMemsetAsync(g.alb.p, 0, 12 * n, s));
  CK(cudaMemsetAsync(g.op.p, 0, 4 * n, s));
  CK(cudaMemsetAsync(g.beta.p, 0, 4 * n, s));
  CK(cudaMemsetAsync(g.shape.p, 0, 4 * n, s));
}

// The gather estimator's backward: the derivative of the last forward
// render of the same views (h = scenes[0] holds its vertex plan), swept
// from the vertex store where its chunks were kept and replayed into the
// scratch store where they were not.
void gather_adjoint(const std::vector<pale_handle*>& scenes, const std::vector<CameraRec>& sel, uint32_t total,
                    const float* d_dldi, const SceneGrads* grads, bool all, const SceneGrads* d_view_grads = nullptr) {
  pale_handle* h = scenes[0];
  cudaStream_t s = h->stream;
  bool same = !h->vviews.empty() && h->vviews.size() == sel.size() && h->vscenes == scenes &&
              std::memcmp(h->vviews.data(), sel.data(), sel.size() * sizeof(CameraRec)) == 0;
  for (size_t k = 0; same && k < scenes.size(); ++k)
    same = h->vgens[3 * k] == scenes[k]->bvh_gen && h->vgens[3 * k + 1] == scenes[k]->photon_gen &&
           h->vgens[3 * k + 2] == scenes[k]->params_gen;
  if (!same)
    throw ArgError("the gather estimator differentiates the last forward render: render the same views, with "
                   "the same points and photon maps, right before the backward");
  const uint32_t nsel = (uint32_t)sel.size();
  CK(cudaMemcpyAsync(h->d_cams.p, sel.data(), nsel * sizeof(CameraRec), cudaMemcpyHostToDevice, s));
  FrameArgs F = frame_args(scenes, nsel, total);
  F.view_start = h->d_view_start.p;
  // the replay scratch: the largest chunk that was not stored
  uint64_t recs = 0, ents = 0;
  for (const VertexChunk& c : h->vplan.chunks)
    if (!c.stored) {
      recs = std::max<uint64_t>(recs, c.recs);
      ents = std::max<uint64_t>(ents, c.ents);
    }
  if (recs || ents) {
    recs = std::max<uint64_t>(recs, 1);
    ents = std::max<uint64_t>(ents, 1);
    h->sc_rec_xa.ensure(recs); h->sc_rec_ew.ensure(recs);
    h->sc_ent_d.ensure(ents); h->sc_ent_b.ensure(ents); h->sc_ent_l.ensure(ents);
  } else if (h->sc_rec_xa.p) {
    // every chunk is in the store: the scratch of an earlier replay goes
    CK(cudaStreamSynchronize(s));
    h->sc_rec_xa.free(); h->sc_rec_ew.free();
    h->sc_ent_d.free(); h->sc_ent_b.free(); h->sc_ent_l.free();
  }
  h->vs_base.ensure(2 * kVertexBases);
  h->vs_overflow.ensure(1);
  F.vs = VertexStore{h->vs_rec_xa.p, h->vs_rec_ew.p, h->vs_ent_d.p, h->vs_ent_b.p, h->vs_ent_l.p, h->vs_base.p,
                     h->vs_overflow.p, (uint32_t)h->vs_rec_xa.n, (uint32_t)h->vs_ent_d.n, 0u, 0u, 0};
  VertexStore scratch{h->sc_rec_xa.p, h->sc_rec_ew.p, h->sc_ent_d.p, h->sc_ent_b.p, h->sc_ent_l.p, h->vs_base.p,
                      h->vs_overflow.p, (uint32_t)h->sc_rec_xa.n, (uint32_t)h->sc_ent_d.n, 0u, 0u, 1};
  SweepArgs W{};
  W.dldi = d_dldi;
  for (size_t k = 0; k < scenes.size(); ++k) W.grads[k] = grads[k];
  W.all_grads = all ? 1 : 0;
  W.view_grads = d_view_grads;
  gather_backward(F, sel, h->vplan, W, scratch, s);
  uint32_t stored = 0;
  uint64_t recs_all = 0, ents_all = 0;
  for (const VertexChunk& c : h->vplan.chunks) {
    stored += c.stored ? 1u : 0u;
    recs_all += c.recs;
    ents_all += c.ents;
  }
  h->stats.vertex_records = recs_all;
  h->stats.vertex_entries = ents_all;
  h->stats.vertex_chunks_stored = stored;
  h->stats.vertex_chunks_replayed = (uint32_t)h->vplan.chunks.size() - stored;
  h->stats.vertex_bytes = vertex_bytes(h);
}

// The adjoint pass of `views` reading packed dL/dI at d_dldi (device), on
// the stream and with the wavefront buffers of scenes[0]; each scene's
// gradients accumulate in its own arrays (BVH order).  All scenes share
// the rng mode, the null weighting and the gradient groups of scenes[0].
// out: null, or per entry of `scenes` DEVICE gradient arrays (every field
// but shape non-null) that the entry's gradients accumulate in, zeroed
// first, instead of the scene's own arrays; then one scene may fill
// several entries (one per request of a server).
void adjoint_views(const std::vector<pale_handle*>& scenes, const std::vector<ViewReq>& views, const float* d_dldi,
                   float* d_dbg, bool sync, const pale_points* out = nullptr) {
  pale_handle* h = scenes[0];
  cudaStream_t s = h->stream;
  h->timer.used = 0;
  const uint64_t launches0 = launches_issued();
  const pale_settings& st = h->st;
  // the gather estimator differentiates a forward render: its views carry
  // gather passes
  check_views(scenes, views, st.estimator != PALE_ESTIMATOR_GATHER, out != nullptr);
  uint32_t total = 0, max_pix = 0;
  std::vector<CameraRec> sel = view_records(scenes, views, total, max_pix);
  size_wavefronts(h, total, max_pix);
  // decorrelated seeds: per scene one block of (1 + bounces) per (camera,
  // pass), camera-major with the scene's passes as the stride; a camera is
  // its position among the scene's views in the call, or with camera_seeds
  // = camera its scene index, so that its gradient does not depend on which
  // other cameras the call holds.  The scenes' tables are concatenated.
  std::vector<uint32_t> seeds;
  std::vector<size_t> seed_base(scenes.size());
  std::vector<uint32_t> nviews(scenes.size(), 0u);
  for (const ViewReq& v : views) ++nviews[v.scene];
  for (size_t k = 0; k < scenes.size(); ++k) {
    const pale_settings& sk = scenes[k]->st;
    const bool by_camera = sk.camera_seeds == PALE_CAMERA_SEEDS_CAMERA;
    const size_t seed_cams = by_camera ? scenes[k]->cams.size() : nviews[k];
    std::vector<uint32_t> t = mt_table(st.rng_mode == PALE_RNG_DECORRELATED ? sk.seed : 42ull,
                                       seed_cams * sk.adjoint_passes * (1 + sk.adjoint_bounces) + 1);
    seed_base[k] = seeds.size();
    seeds.insert(seeds.end(), t.begin(), t.end());
  }
  h->seeds_adj.ensure(seeds.size());
  CK(cudaMemcpyAsync(h->seeds_adj.p, seeds.data(), seeds.size() * 4, cudaMemcpyHostToDevice, s));
  AdjointArgs A{};
  for (size_t k = 0; k < scenes.size(); ++k) {
    pale_handle* sk = scenes[k];
    if (!out) {
      zero_grads(sk, s);
      A.sgrads[k] = SceneGrads{sk->grads.op.p, sk->grads.view()};
      continue;
    }
    const pale_points& g = out[k];
    if (!g.position || !g.tangent_u || !g.tangent_v || !g.scale || !g.albedo || !g.opacity || !g.beta)
      throw ArgError("gradient outputs need every field but shape");
    const size_t n = sk->np;
    for (float* f : {g.position, g.tangent_u, g.tangent_v, g.albedo}) CK(cudaMemsetAsync(f, 0, 12 * n, s));
    CK(cudaMemsetAsync(g.scale, 0, 8 * n, s));
    CK(cudaMemsetAsync(g.opacity, 0, 4 * n, s));
    CK(cudaMemsetAsync(g.beta, 0, 4 * n, s));
    if (g.shape) CK(cudaMemsetAsync(g.shape, 0, 4 * n, s));
    PointsDev pd{g.position, g.tangent_u, g.tangent_v, g.scale, g.albedo, g.opacity, g.beta, g.shape};
    A.sgrads[k] = SceneGrads{g.opacity, pd};
  }
  CK(cudaMemsetAsync(h->run.p, 0, sizeof(RunState), s));
  CK(cudaEventRecord(h->ev0, s));
  if (st.estimator == PALE_ESTIMATOR_GATHER) {
    gather_adjoint(scenes, sel, total, d_dldi, A.sgrads, st.gradients == PALE_GRADIENTS_ALL);
    CK(cudaEventRecord(h->ev1, s));
    CK(cudaGetLastError());
    h->launches_last = launches_issued() - launches0;
    h->timed = 2;
    h->stats_pending = 1;
    if (sync) copy_stats(h);
    return;
  }
  A.scenes = scene_table(scenes);
  A.st = h->run.p;
  A.seeds = h->seeds_adj.p;
  A.qb = QueueBufs{{h->q0.p, h->q1.p}, h->qstage.p, h->qflags.p, h->tile_counts.p, h->tile_offsets.p,
                   std::max(h->qcap, h->adj_cap)};
  A.pend = PendingBufs{h->pend_a.p, h->pend_b.p, h->pend_c.p};
  A.ev = EventBufs{h->ev_stage.p, h->ev_list.p};
  A.dldi = d_dldi;
  A.all_grads = st.gradients == PALE_GRADIENTS_ALL;
  A.debug_opacity = d_dbg;
  A.rr_start = st.rr_start;
  A.q_null = st.q_null;
  A.q_reflect = st.q_reflect;
  A.q_transmit = st.q_transmit;
  A.fixed_seed = st.random_number;
  A.rng_mode = st.rng_mode;
  A.null_scale = st.null_weight == PALE_NULL_WEIGHT_UNBIASED ? 1.0f / st.q_null : 1.0f;
  A.light0_valid = h->n_lights > 0;
  A.light0_area = h->light0_area;
  A.timer = &h->timer;
  A.sort_keys = h->adj_keys.p;
  A.perm = h->adj_perm.p;
  A.sort_keys_tmp = h->adj_keys_tmp.p;
  A.perm_tmp = h->adj_perm_tmp.p;
  A.sort_temp = h->adj_sort_temp.p;
  A.sort_capacity = h->adj_cap;
  A.hits = h->adj_hits.p;
  A.walkq = h->adj_walkq.p;
  A.walk_block = st.walk_block;
  // jobs in the reference's order (view-major, then pass), packed into
  // batches of at most adj_cap paths and kMaxJobsPerBatch jobs
  const std::vector<uint32_t> slots = seed_slots(scenes, views);
  std::vector<AdjJob> jobs;
  std::vector<std::pair<uint32_t, uint32_t>> batches;  // (first job, paths)
  uint32_t in_batch = 0, first = 0, max_depth = 0;
  for (uint32_t i = 0; i < (uint32_t)sel.size(); ++i) {
    const uint32_t npix = sel[i].w * sel[i].h;
    const pale_settings& sk = scenes[sel[i].scene]->st;
    const uint32_t stride = 1u + sk.adjoint_bounces;
    max_depth = std::max(max_depth, sel[i].depth);
    for (uint32_t spp = 0; spp < sel[i].passes; ++spp) {
      const uint32_t j = (uint32_t)jobs.size();
      if (in_batch + npix > h->adj_cap || j - first == kMaxJobsPerBatch) {
        batches.emplace_back(first, in_batch);
        first = j;
        in_batch = 0;
      }
      const size_t seed_index = seed_base[sel[i].scene] + ((size_t)slots[i] * sk.adjoint_passes + spp) * stride;
      jobs.push_back(AdjJob{i, in_batch, npix, (uint32_t)seed_index});
      in_batch += npix;
    }
  }
  if (!jobs.empty()) batches.emplace_back(first, in_batch);
  h->d_adj_cams.ensure(std::max<size_t>(1, sel.size()));
  h->d_jobs.ensure(std::max<size_t>(1, jobs.size()));
  if (!sel.empty())
    CK(cudaMemcpyAsync(h->d_adj_cams.p, sel.data(), sel.size() * sizeof(CameraRec), cudaMemcpyHostToDevice, s));
  if (!jobs.empty())
    CK(cudaMemcpyAsync(h->d_jobs.p, jobs.data(), jobs.size() * sizeof(AdjJob), cudaMemcpyHostToDevice, s));
  A.cams = h->d_adj_cams.p;
  A.job_count = h->job_count.p;
  A.job_start = h->job_start.p;
  for (size_t bi = 0; bi < batches.size(); ++bi) {
    const uint32_t j0 = batches[bi].first;
    const uint32_t j1 = bi + 1 < batches.size() ? batches[bi + 1].first : (uint32_t)jobs.size();
    A.jobs = h->d_jobs.p + j0;
    A.njobs = j1 - j0;
    const uint32_t npaths = batches[bi].second;
    adjoint_raygen(A, npaths, s);
    for (uint32_t b = 0; b < max_depth; ++b) adjoint_bounce(A, b, npaths, s);
  }
  CK(cudaEventRecord(h->ev1, s));
  CK(cudaGetLastError());
  h->launches_last = launches_issued() - launches0;
  h->timed = 2;
  h->stats_pending = 1;
  if (sync) copy_stats(h);
}

void backward(pale_handle* h, uint32_t nsel, const uint32_t* idx, const float* d_dldi, float* d_dbg, bool sync) {
  validate_cams(h, nsel, idx);
  adjoint_views({h}, all_passes(h, nsel, idx, h->st.estimator != PALE_ESTIMATOR_GATHER), d_dldi, d_dbg, sync);
}

// Host-to-device copy from a caller's buffer on the handle's stream,
// staged when large.  The stage holds the data until the copy has run: a
// later staged copy into the stage waits for it.
void copy_in(pale_handle* h, void* dev, const void* host, size_t bytes) {
  if (!bytes) return;
  cudaStream_t s = h->stream;
  if (bytes < kStageMinBytes) {
    CK(cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, s));
    return;
  }
  if (h->stage.in_flight) {
    CK(cudaStreamSynchronize(s));
    h->stage.in_flight = false;
  }
  if (!h->stage.ensure(bytes, s)) {
    CK(cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, s));
    return;
  }
  host_copy({HostPiece{h->stage.p, static_cast<const char*>(host), bytes}});
  CK(cudaMemcpyAsync(dev, h->stage.p, bytes, cudaMemcpyHostToDevice, s));
  h->stage.in_flight = true;
}

struct DeviceOut {
  void* host;        // null: skipped
  const void* dev;
  size_t bytes;
};

// Device-to-host copies into callers' buffers: enqueued on the handle's
// stream (through the stage when they add up to kStageMinBytes or more),
// then the run state is read (with `stats`) and the stream synchronised.
void copy_out(pale_handle* h, const std::vector<DeviceOut>& outs, bool stats) {
  cudaStream_t s = h->stream;
  auto slot = [](size_t b) { return (b + 255) & ~size_t(255); };
  size_t total = 0;
  for (const DeviceOut& o : outs)
    if (o.host && o.bytes) total += slot(o.bytes);
  const bool staged = total >= kStageMinBytes && h->stage.ensure(total, s);
  std::vector<HostPiece> pieces;
  if (staged) {
    // (the copies into the stage run after any copy out of it: same stream)
    size_t off = 0;
    for (const DeviceOut& o : outs) {
      if (!o.host || !o.bytes) continue;
      CK(cudaMemcpyAsync(h->stage.p + off, o.dev, o.bytes, cudaMemcpyDeviceToHost, s));
      pieces.push_back(HostPiece{static_cast<char*>(o.host), h->stage.p + off, o.bytes});
      off += slot(o.bytes);
    }
  } else {
    for (const DeviceOut& o : outs)
      if (o.host && o.bytes) CK(cudaMemcpyAsync(o.host, o.dev, o.bytes, cudaMemcpyDeviceToHost, s));
  }
  if (stats) copy_stats(h);
  CK(cudaStreamSynchronize(s));
  h->stage.in_flight = false;
  if (staged) host_copy(pieces);
}

void download_points(pale_handle* h, const PointsBufs& src, pale_points* out) {
  const size_t n = h->np;
  if (!n) return;
  copy_out(h, {DeviceOut{out->position, src.pos.p, 12 * n}, DeviceOut{out->tangent_u, src.tu.p, 12 * n},
               DeviceOut{out->tangent_v, src.tv.p, 12 * n}, DeviceOut{out->scale, src.sc.p, 8 * n},
               DeviceOut{out->albedo, src.alb.p, 12 * n}, DeviceOut{out->opacity, src.op.p, 4 * n},
               DeviceOut{out->beta, src.beta.p, 4 * n}, DeviceOut{out->shape, src.shape.p, 4 * n}},
           false);
}

// dst := src for the current point count (device to device, enqueued).
void copy_points(pale_handle* h, const PointsBufs& src, PointsBufs& dst, cudaStream_t s) {
  const size_t n = h->np;
  if (!n) return;
  CK(cudaMemcpyAsync(dst.pos.p, src.pos.p, 12 * n, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemcpyAsync(dst.tu.p, src.tu.p, 12 * n, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemcpyAsync(dst.tv.p, src.tv.p, 12 * n, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemcpyAsync(dst.sc.p, src.sc.p, 8 * n, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemcpyAsync(dst.alb.p, src.alb.p, 12 * n, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemcpyAsync(dst.op.p, src.op.p, 4 * n, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemcpyAsync(dst.beta.p, src.beta.p, 4 * n, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemcpyAsync(dst.shape.p, src.shape.p, 4 * n, cudaMemcpyDeviceToDevice, s));
}

void zero_point_bufs(pale_handle* h, PointsBufs& b, cudaStream_t s) {
  const size_t n = h->np;
  if (!n) return;
  CK(cudaMemsetAsync(b.pos.p, 0, 12 * n, s));
  CK(cudaMemsetAsync(b.tu.p, 0, 12 * n, s));
  CK(cudaMemsetAsync(b.tv.p, 0, 12 * n, s));
  CK(cudaMemsetAsync(b.sc.p, 0, 8 * n, s));
  CK(cudaMemsetAsync(b.alb.p, 0, 12 * n, s));
  CK(cudaMemsetAsync(b.op.p, 0, 4 * n, s));
  CK(cudaMemsetAsync(b.beta.p, 0, 4 * n, s));
}

void check_optimizer(const pale_optimizer* o) {
  if (!o) throw ArgError("pale_optimizer_step: null optimizer description");
  if (o->type > PALE_OPT_MASKED_ADAM) throw ArgError("Unknown optimizer type " + std::to_string(o->type));
  if (o->flags & ~PALE_OPT_SURFEL_MASK) throw ArgError("Unknown optimizer flags");
  for (int g = 0; g < 6; ++g)
    if (!(o->lr[g] >= 0.0) || !std::isfinite(o->lr[g])) throw ArgError("Invalid learning rate");
  if (o->type != PALE_OPT_SGD) {
    if (!(o->beta1 >= 0.0 && o->beta1 < 1.0 && o->beta2 >= 0.0 && o->beta2 < 1.0))
      throw ArgError("Invalid betas");
    if (!(o->eps > 0.0)) throw ArgError("Invalid eps");
  } else if (!(o->momentum >= 0.0)) {
    throw ArgError("Invalid momentum");
  }
}

}  // namespace

// ===================================================================== ABI
extern "C" {

void pale_default_settings(pale_settings* s) {
  if (!s) return;
  std::memset(s, 0, sizeof(*s));
  s->photons_per_launch = 1000000u;
  s->max_bounces = 6;
  s->forward_passes = 6;
  s->gather_passes = 6;
  s->adjoint_bounces = 6;
  s->adjoint_passes = 6;
  s->seed = 42;
  s->random_number = 42;
  s->rr_start = 6;
  s->q_null = 0.5f;
  s->q_reflect = 0.5f;
  s->q_transmit = 0.0f;
  s->gather_radius = 0.01f;
  s->leaf_size = 1;
  s->rng_mode = PALE_RNG_REFERENCE;
  s->null_weight = PALE_NULL_WEIGHT_REFERENCE;
  s->gradients = PALE_GRADIENTS_OPACITY;
  s->debug_images = 0;
  s->exposure = 1.0f;
  s->gamma = 2.2f;
}

const char* pale_version(void) { return "pale_b200 0.1 (sm_100a)"; }

const char* pale_last_error(const pale_handle* h) { return h ? h->err.c_str() : g_create_error.c_str(); }

int pale_create(const pale_scene_desc* desc, const pale_settings* settings, pale_handle** out) {
  if (!desc || !settings || !out) return fail(nullptr, PALE_ERR_ARGUMENT, "pale_create: null argument");
  *out = nullptr;
  pale_handle* h = new pale_handle();
  int rc = guarded(nullptr, [&]() {
    h->st = *settings;
    if (h->st.forward_passes == 0 || h->st.photons_per_launch == 0) throw ArgError("photons and forward passes must be > 0");
    if (h->st.gather_passes == 0 || h->st.adjoint_passes == 0) throw ArgError("gather and adjoint passes must be > 0");
    if (!(h->st.gather_radius > 0.f)) throw ArgError("gather radius must be > 0");
    if (h->st.adjoint_bounces > 255) throw ArgError("at most 255 adjoint bounces are supported");
    if (h->st.null_weight > PALE_NULL_WEIGHT_UNBIASED) throw ArgError("null_weight must be reference or unbiased");
    if (h->st.gradients > PALE_GRADIENTS_ALL) throw ArgError("gradients must be opacity or all");
    if (h->st.camera_seeds > PALE_CAMERA_SEEDS_CAMERA) throw ArgError("camera_seeds must be selection or camera");
    if (h->st.walk_block != 0 && h->st.walk_block != 64 && h->st.walk_block != 128 && h->st.walk_block != 256)
      throw ArgError("walk_block must be 64, 128 or 256");
    if (h->st.estimator > PALE_ESTIMATOR_GATHER) throw ArgError("estimator must be 0 (reference) or 1 (gather)");
    if (h->st.vertex_store > PALE_VERTICES_REPLAY)
      throw ArgError("vertex_store must be 0 (auto), 1 (checkpoint) or 2 (replay)");
    if (h->st.null_weight == PALE_NULL_WEIGHT_UNBIASED && !(h->st.q_null > 0.f))
      throw ArgError("unbiased null weighting needs q_null > 0");
    check_points(&desc->points, "pale_create");
    if (desc->points.count >= (1u << 28)) throw ArgError("at most 2^28 surfels are supported");
    CK(cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking));
    h->stream = h->own_stream;
    CK(cudaEventCreate(&h->ev0));
    CK(cudaEventCreate(&h->ev1));
    CK(cudaEventCreate(&h->ev2));
    setup_scene(h, desc);
    return PALE_OK;
  });
  if (rc != PALE_OK) {
    delete h;
    return rc;
  }
  *out = h;
  return PALE_OK;
}

int pale_destroy(pale_handle* h) {
  if (!h) return PALE_OK;
  if (h->stream) cudaStreamSynchronize(h->stream);
  delete h;
  return PALE_OK;
}

int pale_point_count(const pale_handle* h, uint32_t* count) {
  if (!h || !count) return PALE_ERR_ARGUMENT;
  *count = h->np;
  return PALE_OK;
}

int pale_camera_count(const pale_handle* h, uint32_t* count) {
  if (!h || !count) return PALE_ERR_ARGUMENT;
  *count = (uint32_t)h->cams.size();
  return PALE_OK;
}

int pale_camera_info(const pale_handle* h, uint32_t index, char name[16], uint32_t* width, uint32_t* height) {
  if (!h || index >= h->cams.size()) return PALE_ERR_ARGUMENT;
  if (name) {
    std::memset(name, 0, 16);
    std::strncpy(name, h->cam_names[index].c_str(), 15);
  }
  if (width) *width = h->cams[index].w;
  if (height) *height = h->cams[index].h;
  return PALE_OK;
}

int pale_render_forward(pale_handle* h, uint32_t nsel, const uint32_t* idx, float* ldr, float* raw) {
  if (!h) return PALE_ERR_ARGUMENT;
  return guarded(h, [&]() {
    validate_cams(h, nsel, idx);
    size_t pix = 0;
    for (uint32_t i = 0; i < nsel; ++i) pix += (size_t)h->cams[idx[i]].w * h->cams[idx[i]].h;
    use_stream(h, h->own_stream);
    h->img_raw.ensure(4 * std::max<size_t>(1, pix));
    h->img_ldr.ensure(4 * std::max<size_t>(1, pix));
    forward(h, nsel, idx, h->img_raw.p, h->img_ldr.p, true);
    copy_out(h, {DeviceOut{raw, h->img_raw.p, 16 * pix}, DeviceOut{ldr, h->img_ldr.p, 16 * pix}}, false);
    return PALE_OK;
  });
}

int pale_render_gather(pale_handle* h, uint32_t nsel, const uint32_t* idx, float* ldr, float* raw) {
  if (!h) return PALE_ERR_ARGUMENT;
  return guarded(h, [&]() {
    validate_cams(h, nsel, idx);
    size_t pix = 0;
    for (uint32_t i = 0; i < nsel; ++i) pix += (size_t)h->cams[idx[i]].w * h->cams[idx[i]].h;
    use_stream(h, h->own_stream);
    h->img_raw.ensure(4 * std::max<size_t>(1, pix));
    h->img_ldr.ensure(4 * std::max<size_t>(1, pix));
    forward(h, nsel, idx, h->img_raw.p, h->img_ldr.p, true, false);
    copy_out(h, {DeviceOut{raw, h->img_raw.p, 16 * pix}, DeviceOut{ldr, h->img_ldr.p, 16 * pix}}, false);
    return PALE_OK;
  });
}

int pale_render_forward_device(pale_handle* h, uint32_t nsel, const uint32_t* idx, float* d_ldr, float* d_raw,
                               void* stream) {
  if (!h) return PALE_ERR_ARGUMENT;
  return guarded(h, [&]() {
    validate_cams(h, nsel, idx);
    size_t pix = 0;
    for (uint32_t i = 0; i < nsel; ++i) pix += (size_t)h->cams[idx[i]].w * h->cams[idx[i]].h;
    use_stream(h, caller_stream(stream));
    h->img_raw.ensure(4 * std::max<size_t>(1, pix));
    forward(h, nsel, idx, d_raw ? d_raw : h->img_raw.p, d_ldr, false);
    return PALE_OK;
  });
}

int pale_render_forward_loss(pale_handle* h, uint32_t nsel, const uint32_t* idx, const float* target,
                             uint32_t channels, float* ldr, float* raw, float* dldi, double* loss) {
  if (!h) return PALE_ERR_ARGUMENT;
  return guarded(h, [&]() {
    validate_cams(h, nsel, idx);
    if (!target && nsel) throw ArgError("target image is null");
    if (channels != 3 && channels != 4) throw ArgError("target images need 3 or 4 channels");
    if (nsel > 65535) throw ArgError("at most 65535 cameras per call");
    size_t pix = 0;
    for (uint32_t i = 0; i < nsel; ++i) pix += (size_t)h->cams[idx[i]].w * h->cams[idx[i]].h;
    use_stream(h, h->own_stream);
    const size_t p1 = std::max<size_t>(1, pix);
    h->img_raw.ensure(4 * p1);
    h->img_ldr.ensure(4 * p1);
    h->dldi.ensure(4 * p1);
    h->target.ensure(channels * p1);
    h->loss.ensure(std::max(1u, nsel));
    // the stage at the size of the call's largest staged copy, allocated once
    const size_t out_bytes = (raw ? 16 * pix : 0) + (ldr ? 16 * pix : 0) + (dldi ? 16 * pix : 0) + 4096;
    if (out_bytes >= kStageMinBytes) (void)h->stage.ensure(std::max<size_t>(out_bytes, 4ull * channels * pix), h->stream);
    copy_in(h, h->target.p, target, 4ull * channels * pix);
    LossReq lq{h->target.p, channels, h->dldi.p, h->loss.p};
    forward(h, nsel, idx, h->img_raw.p, h->img_ldr.p, false, true, &lq);
    copy_out(h, {DeviceOut{raw, h->img_raw.p, 16 * pix}, DeviceOut{ldr, h->img_ldr.p, 16 * pix},
                 DeviceOut{dldi, h->dldi.p, 16 * pix}, DeviceOut{nsel ? loss : nullptr, h->loss.p, 8ull * nsel}},
             true);
    return PALE_OK;
  });
}

int pale_render_forward_loss_device(pale_handle* h, uint32_t nsel, const uint32_t* idx, const float* d_target,
                                    uint32_t channels, float* d_ldr, float* d_raw, float* d_dldi, double* d_loss,
                                    void* stream) {
  if (!h) return PALE_ERR_ARGUMENT;
  return guarded(h, [&]() {
    validate_cams(h, nsel, idx);
    if (!d_target && nsel) throw ArgError("target image is null");
    if (channels != 3 && channels != 4) throw ArgError("target images need 3 or 4 channels");
    if (nsel > 65535) throw ArgError("at most 65535 cameras per call");
    size_t pix = 0;
    for (uint32_t i = 0; i < nsel; ++i) pix += (size_t)h->cams[idx[i]].w * h->cams[idx[i]].h;
    use_stream(h, caller_stream(stream));
    h->img_raw.ensure(4 * std::max<size_t>(1, pix));
    if (!d_ldr && d_loss) {
      h->img_ldr.ensure(4 * std::max<size_t>(1, pix));
      d_ldr = h->img_ldr.p;
    }
    LossReq lq{d_target, channels, d_dldi, d_loss};
    forward(h, nsel, idx, d_raw ? d_raw : h->img_raw.p, d_ldr, false, true, &lq);
    return PALE_OK;
  });
}

int pale_render_backward(pale_handle* h, uint32_t nsel, const uint32_t* idx, const float* dldi, pale_points* grads,
                         float* debug_opacity) {
  if (!h) return PALE_ERR_ARGUMENT;
  return guarded(h, [&]() {
    validate_cams(h, nsel, idx);
    if (!dldi && nsel) throw ArgError("dL/dI is null");
    size_t pix = 0;
    for (uint32_t i = 0; i < nsel; ++i) pix += (size_t)h->cams[idx[i]].w * h->cams[idx[i]].h;
    use_stream(h, h->own_stream);
    h->dldi.ensure(4 * std::max<size_t>(1, pix));
    copy_in(h, h->dldi.p, dldi, 16 * pix);
    float* dbg = nullptr;
    if (debug_opacity && h->st.debug_images) {
      h->dbg.ensure(4 * std::max<size_t>(1, pix));
      CK(cudaMemsetAsync(h->dbg.p, 0, 16 * pix, h->stream));
      dbg = h->dbg.p;
    }
    backward(h, nsel, idx, h->dldi.p, dbg, true);
    if (grads) download_points(h, h->grads, grads);
    if (debug_opacity) {
      if (dbg) CK(cudaMemcpyAsync(debug_opacity, dbg, 16 * pix, cudaMemcpyDeviceToHost, h->stream));
      else std::memset(debug_opacity, 0, 16 * pix);
    }
    CK(cudaStreamSynchronize(h->stream));
    return PALE_OK;
  });
}

int pale_render_backward_device(pale_handle* h, uint32_t nsel, const uint32_t* idx, const float* d_dldi,
                                pale_points* d_grads, void* stream) {
  if (!h) return PALE_ERR_ARGUMENT;
  return guarded(h, [&]() {
    validate_cams(h, nsel, idx);
    use_stream(h, caller_stream(stream));
    backward(h, nsel, idx, d_dldi, nullptr, false);
    if (d_grads) {
      const size_t n = h->np;
      cudaStream_t s = h->stream;
      auto cp = [&](float* dst, const float* src, size_t bytes) {
        if (dst && n) CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, s));
      };
      cp(d_grads->position, h->grads.pos.p, 12 * n);
      cp(d_grads->tangent_u, h->grads.tu.p, 12 * n);
      cp(d_grads->tangent_v, h->grads.tv.p, 12 * n);
      cp(d_grads->scale, h->grads.sc.p, 8 * n);
      cp(d_grads->albedo, h->grads.alb.p, 12 * n);
      cp(d_grads->opacity, h->grads.op.p, 4 * n);
      cp(d_grads->beta, h->grads.beta.p, 4 * n);
      cp(d_grads->shape, h->grads.shape.p, 4 * n);
    }
    return PALE_OK;
  });
}

namespace {
std::vector<pale_handle*> scene_list(uint32_t n, pale_handle* const* scenes) {
  if (!scenes || n == 0 || n > kMaxScenes) throw ArgError("a call renders 1 to 8 scenes");
  return std::vector<pale_handle*>(scenes, scenes + n);
}

std::vector<ViewReq> view_list(uint32_t n, const pale_view* views) {
  if (n && !views) throw ArgError("view list is null");
  std::vector<ViewReq> v(n);
  for (uint32_t i = 0; i < n; ++i)
    v[i] = ViewReq{views[i].scene, views[i].camera, views[i].passes, views[i].depth, views[i].first_pass,
                   views[i].pass_count};
  return v;
}

}  // namespace

int pale_render_views_loss_device(uint32_t num_scenes, pale_handle* const* scenes, int trace_photons,
                                  uint32_t num_views, const pale_view* views, const float* d_target,
                                  uint32_t channels, float* d_ldr, float* d_raw, float* d_dldi, double* d_loss,
                                  float* d_partial, void* stream) {
  if (!scenes || num_scenes == 0 || !scenes[0]) return fail(nullptr, PALE_ERR_ARGUMENT, "no scenes");
  pale_handle* h = scenes[0];
  return guarded(h, [&]() {
    std::vector<pale_handle*> sc = scene_list(num_scenes, scenes);
    std::vector<ViewReq> vw = view_list(num_views, views);
    check_views(sc, vw, false);
    if ((d_dldi || d_loss) && !d_target && num_views) throw ArgError("target image is null");
    if (d_target && channels != 3 && channels != 4) throw ArgError("target images need 3 or 4 channels");
    size_t pix = 0;
    for (const ViewReq& v : vw) pix += (size_t)sc[v.scene]->cams[v.cam].w * sc[v.scene]->cams[v.cam].h;
    const cudaStream_t s = caller_stream(stream);
    for (pale_handle* sk : sc) use_stream(sk, s);
    h->img_raw.ensure(4 * std::max<size_t>(1, pix));
    if (!d_ldr && (d_loss || d_dldi)) {
      h->img_ldr.ensure(4 * std::max<size_t>(1, pix));
      d_ldr = h->img_ldr.p;
    }
    LossReq lq{d_target, channels, d_dldi, d_loss};
    render_views(sc, vw, d_raw ? d_raw : h->img_raw.p, d_ldr, false, trace_photons != 0, d_target ? &lq : nullptr,
                 d_partial);
    return PALE_OK;
  });
}

int pale_trace_photon_map(pale_handle* h, void* stream) {
  if (!h) return PALE_ERR_ARGUMENT;
  return guarded(h, [&]() {
    use_stream(h, caller_stream(stream));
    forward_seeds(h, h->cams.size());
    CK(cudaMemsetAsync(h->run.p, 0, sizeof(RunState), h->stream));
    trace_photon_map(h);
    CK(cudaGetLastError());
    return PALE_OK;
  });
}

int pale_render_views_backward_device(uint32_t num_scenes, pale_handle* const* scenes, uint32_t num_views,
                                      const pale_view* views, const float* d_dldi, pale_points* d_grads,
                                      void* stream) {
  if (!scenes || num_scenes == 0 || !scenes[0]) return fail(nullptr, PALE_ERR_ARGUMENT, "no scenes");
  pale_handle* h = scenes[0];
  return guarded(h, [&]() {
    std::vector<pale_handle*> sc = scene_list(num_scenes, scenes);
    std::vector<ViewReq> vw = view_list(num_views, views);
    if (num_views && !d_dldi) throw ArgError("dL/dI is null");
    const cudaStream_t s = caller_stream(stream);
    for (pale_handle* sk : sc) use_stream(sk, s);
    adjoint_views(sc, vw, d_dldi, nullptr, false, d_grads);
    return PALE_OK;
  });
}

int pale_render_views_gradients_device(uint32_t num_scenes, pale_handle* const* scenes, uint32_t num_views,
                                       const pale_view* views, const float* d_dldi, const pale_points* d_grads,
                                       void* stream) {
  if (!scenes || num_scenes == 0 || !scenes[0]) return fail(nullptr, PALE_ERR_ARGUMENT, "no scenes");
  pale_handle* h = scenes[0];
  return guarded(h, [&]() {
    if (h->st.estimator != PALE_ESTIMATOR_GATHER)
      throw ArgError("per-view gradients need the gather estimator (scenes[0]'s settings)");
    std::vector<pale_handle*> sc = scene_list(num_scenes, scenes);
    std::vector<ViewReq> vw = view_list(num_views, views);
    if (num_views && (!d_dldi || !d_grads)) throw ArgError("dL/dI or the gradient outputs are null");
    const cudaStream_t cs = caller_stream(stream);
    for (pale_handle* sk : sc) use_stream(sk, cs);
    cudaStream_t s = h->stream;
    h->timer.used = 0;
    const uint64_t launches0 = launches_issued();
    check_views(sc, vw, false);
    uint32_t total = 0, max_pix = 0;
    std::vector<CameraRec> sel = view_records(sc, vw, total, max_pix);
    std::vector<SceneGrads> vg(std::max<size_t>(1, vw.size()));
    for (size_t i = 0; i < vw.size(); ++i) {
      const pale_points& g = d_grads[i];
      if (!g.opacity) continue;   // no gradients for this view
      if (!g.position || !g.tangent_u || !g.tangent_v || !g.scale || !g.albedo || !g.beta)
        throw ArgError("gradient outputs need every field but shape");
      const size_t n = sc[vw[i].scene]->np;
      for (float* f : {g.position, g.tangent_u, g.tangent_v, g.albedo}) CK(cudaMemsetAsync(f, 0, 12 * n, s));
      CK(cudaMemsetAsync(g.scale, 0, 8 * n, s));
      CK(cudaMemsetAsync(g.opacity, 0, 4 * n, s));
      CK(cudaMemsetAsync(g.beta, 0, 4 * n, s));
      if (g.shape) CK(cudaMemsetAsync(g.shape, 0, 4 * n, s));
      vg[i] = SceneGrads{g.opacity, PointsDev{g.position, g.tangent_u, g.tangent_v, g.scale, g.albedo, g.opacity,
                                              g.beta, g.shape}};
    }
    h->vs_view_grads.ensure(vg.size());
    CK(cudaMemcpyAsync(h->vs_view_grads.p, vg.data(), vg.size() * sizeof(SceneGrads), cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(h->run.p, 0, sizeof(RunState), s));
    CK(cudaEventRecord(h->ev0, s));
    SceneGrads none[kMaxScenes] = {};
    gather_adjoint(sc, sel, total, d_dldi, none, h->st.gradients == PALE_GRADIENTS_ALL, h->vs_view_grads.p);
    CK(cudaEventRecord(h->ev1, s));
    CK(cudaGetLastError());
    h->launches_last = launches_issued() - launches0;
    h->timed = 2;
    h->stats_pending = 1;
    return PALE_OK;
  });
}

int pale_get_points(pale_handle* h, pale_points* out) {
  if (!h || !out) return PALE_ERR_ARGUMENT;
  return guarded(h, [&]() {
    use_stream(h, h->own_stream);
    download_points(h, h->params, out);
    return PALE_OK;
  });
}

int pale_get_order(pale_handle* h, uint32_t* order) {
  if (!h || !order) return PALE_ERR_ARGUMENT;
  return guarded(h, [&]() {
    use_stream(h, h->own_stream);
    if (h->np) CK(cudaMemcpyAsync(order, h->order.p, 4ull * h->np, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return PALE_OK;
  });
}

int pale_apply_points(pale_handle* h, const pale_points* p) {
  if (!h) return PALE_ERR_ARGUMENT;
  return guarded(h, [&]() {
    check_points(p, "pale_apply_points");
    if (p->count != h->np) throw ArgError("apply_point_optimization expects consistent point count");
    use_stream(h, h->own_stream);
    cudaStream_t s = h->stream;
    const size_t n = h->np;
    if (!n) return PALE_OK;
    PointsBufs& d = h->params;
    CK(cudaMemcpyAsync(d.pos.p, p->position, 12 * n, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(d.tu.p, p->tangent_u, 12 * n, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(d.tv.p, p->tangent_v, 12 * n, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(d.sc.p, p->scale, 8 * n, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(d.alb.p, p->albedo, 12 * n, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(d.op.p, p->opacity, 4 * n, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(d.beta.p, p->beta, 4 * n, cudaMemcpyHostToDevice, s));
    derive_surfels(d.view(), h->np, SurfelArrays{h->sf_pe.p, h->sf_n.p, h->sf_u.p, h->sf_v.p, h->sf_cn.p, h->sf_alb.p},
                   s);
    ++h->params_gen;
    copy_points(h, d, h->asset, s);   // the asset mirrors the written parameters
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s));
    return PALE_OK;
  });
}

int pale_apply_points_device(pale_handle* h, const pale_points* p, void* stream) {
  if (!h) return PALE_ERR_ARGUMENT;
  return guarded(h, [&]() {
    check_points(p, "pale_apply_points_device");
    if (p->count != h->np) throw ArgError("apply_point_optimization expects consistent point count");
    use_stream(h, caller_stream(stream));
    cudaStream_t s = h->stream;
    const size_t n = h->np;
    if (!n) return PALE_OK;
    PointsBufs& d = h->params;
    auto cp = [&](float* dst, const float* src, size_t bytes) {
      if (dst != src) CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, s));
    };
    cp(d.pos.p, p->position, 12 * n);
    cp(d.tu.p, p->tangent_u, 12 * n);
    cp(d.tv.p, p->tangent_v, 12 * n);
    cp(d.sc.p, p->scale, 8 * n);
    cp(d.alb.p, p->albedo, 12 * n);
    cp(d.op.p, p->opacity, 4 * n);
    cp(d.beta.p, p->beta, 4 * n);
    derive_surfels(d.view(), h->np, SurfelArrays{h->sf_pe.p, h->sf_n.p, h->sf_u.p, h->sf_v.p, h->sf_cn.p, h->sf_alb.p},
                   s);
    ++h->params_gen;
    copy_points(h, d, h->asset, s);
    CK(cudaGetLastError());
    return PALE_OK;
  });
}

int pale_rebuild(pale_handle* h, const pale_points* asset) {
  if (!h) return PALE_ERR_ARGUMENT;
  return guarded(h, [&]() {
    use_stream(h, h->own_stream);
    if (!asset) {
      build_from_device_asset(h);
      return PALE_OK;
    }
    check_points(asset, "pale_rebuild");
    if (asset->count >= (1u << 28)) throw ArgError("at most 2^28 surfels are supported");
    build_surfels(h, asset);
    return PALE_OK;
  });
}

int pale_get_asset(pale_handle* h, pale_points* out) {
  if (!h || !out) return PALE_ERR_ARGUMENT;
  return guarded(h, [&]() {
    use_stream(h, h->own_stream);
    out->count = h->np;
    download_points(h, h->asset, out);
    return PALE_OK;
  });
}

namespace {

float host_key_to_float(uint32_t k) {
  const uint32_t b = (k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k;
  float f;
  std::memcpy(&f, &b, 4);
  return f;
}

void density_scratch(pale_handle* h, uint32_t n) {
  h->dc_keys.ensure(n); h->dc_vals.ensure(n); h->dc_keys_tmp.ensure(n); h->dc_vals_tmp.ensure(n);
  h->dc_sort_temp.ensure(radix_temp_words(n)); h->dc_flags.ensure(n); h->dc_dst.ensure(n); h->dc_list.ensure(n);
  h->dc_word.ensure(scan_temp_words(n));
  h->dc_aux.ensure(4);
}

// Stable radix sort of (dc_keys, dc_vals) over n entries (four passes: the
// result ends in dc_keys / dc_vals).
void density_sort(pale_handle* h, uint32_t n, cudaStream_t s) {
  CK(cudaMemcpyAsync(h->dc_aux.p, &n, 4, cudaMemcpyHostToDevice, s));
  radix_sort_pairs(h->dc_keys.p, h->dc_vals.p, h->dc_keys_tmp.p, h->dc_vals_tmp.p, h->dc_aux.p, n, 32,
                   h->dc_sort_temp.p, s);
}

// Exclusive scan of dc_flags into dc_dst; returns the number of flags set.
uint32_t density_scan(pale_handle* h, uint32_t n, cudaStream_t s) {
  uint32_t total = 0;
  exclusive_scan(h->dc_flags.p, h->dc_dst.p, n, h->dc_word.p, h->dc_aux.p + 1, s);
  CK(cudaMemcpyAsync(&total, h->dc_aux.p + 1, 4, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return total;
}

// Replaces the asset by dc_points[0, m) and rebuilds.
void density_commit(pale_handle* h, uint32_t m, cudaStream_t s) {
  h->np = m;
  h->asset.alloc(m);
  copy_points(h, h->dc_points, h->asset, s);
  build_from_device_asset(h);
}

void indices_to_host(pale_handle* h, const uint32_t* d_idx, uint32_t k, int64_t* out, bool sort, cudaStream_t s) {
  std::vector<uint32_t> idx(k);
  if (k) CK(cudaMemcpyAsync(idx.data(), d_idx, 4ull * k, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (sort) std::sort(idx.begin(), idx.end());
  for (uint32_t j = 0; j < k; ++j) out[j] = idx[j];
}

}  // namespace

int pale_prune_by_opacity(pale_handle* h, float min_opacity, uint32_t use_quantile, double max_fraction,
                          uint32_t min_keep, uint32_t* removed_count, int64_t* removed) {
  if (!h) return PALE_ERR_ARGUMENT;
  return guarded(h, [&]() {
    use_stream(h, h->own_stream);
    cudaStream_t s = h->stream;
    const uint32_t n = h->np;
    if (removed_count) *removed_count = 0;
    if (n == 0) return PALE_OK;
    density_scratch(h, n);
    opacity_sort_keys(h->asset.op.p, n, h->dc_keys.p, h->dc_vals.p, s);
    density_sort(h, n, s);
    float thr = min_opacity;
    if (use_quantile) {
      // np.quantile(opa, q) with the default "linear" method: virtual index
      // (n - 1) q, the last value from n - 1 on, numpy's two-sided lerp
      const double q = std::max(0.0, std::min(1.0, (double)min_opacity));
      const double vi = (double)(n - 1) * q;
      uint32_t lo = (uint32_t)std::floor(vi), hi = lo + 1;
      const double g = vi - std::floor(vi);
      if (vi >= (double)(n - 1)) lo = hi = n - 1;
      uint32_t k2[2] = {0, 0};
      CK(cudaMemcpyAsync(&k2[0], h->dc_keys.p + lo, 4, cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(&k2[1], h->dc_keys.p + hi, 4, cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      const float a = host_key_to_float(k2[0]), b = host_key_to_float(k2[1]);
      const float diff = b - a;
      const double t = g >= 0.5 ? (double)b - (double)diff * (1.0 - g) : (double)a + (double)diff * g;
      thr = (float)t;
    }
    // opa <= threshold in float32, as numpy compares a float32 array with a Python float
    count_le(h->asset.op.p, n, thr, h->dc_aux.p + 2, s);
    uint32_t count = 0;
    CK(cudaMemcpyAsync(&count, h->dc_aux.p + 2, 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    const int64_t by_fraction = (int64_t)(max_fraction * (double)n);
    const int64_t by_min = std::max<int64_t>(0, (int64_t)n - (int64_t)min_keep);
    const int64_t max_prune = std::min(by_fraction, by_min);
    if (count == 0 || max_prune <= 0) return PALE_OK;
    // the candidates are the `count` lowest opacities, a prefix of the sort;
    // above the cap the lowest max_prune of them (ties: lower index first)
    const uint32_t k = (uint32_t)std::min<int64_t>(count, max_prune);
    if (removed) indices_to_host(h, h->dc_vals.p, k, removed, true, s);
    fill_u32(h->dc_flags.p, n, 1u, s);
    mark_indices(h->dc_vals.p, k, n, h->dc_flags.p, 0u, s);
    const uint32_t kept = density_scan(h, n, s);
    h->dc_points.alloc(std::max(1u, kept));
    compact_points(h->asset.view(), h->dc_flags.p, h->dc_dst.p, n, h->dc_points.view(), s);
    density_commit(h, kept, s);
    if (removed_count) *removed_count = k;
    return PALE_OK;
  });
}

int pale_densify_long_axis_split(pale_handle* h, const float* d_importance, int64_t max_new_points,
                                 double split_distance, double minor_axis_shrink, double opacity_reduction,
                                 float min_long_axis_scale, float grad_threshold, uint32_t* parent_count,
                                 int64_t* parents_out) {
  if (!h) return PALE_ERR_ARGUMENT;
  return guarded(h, [&]() {
    use_stream(h, h->own_stream);
    cudaStream_t s = h->stream;
    const uint32_t n = h->np;
    if (parent_count) *parent_count = 0;
    if (n == 0) return PALE_OK;
    if (max_new_points >= 0 && max_new_points / 2 <= 0) return PALE_OK;
    if ((uint64_t)n + 2ull * n >= (1ull << 28)) throw ArgError("at most 2^28 surfels are supported");
    density_scratch(h, n);
    split_candidates(h->asset.view(), n, d_importance, min_long_axis_scale, grad_threshold,
                     d_importance && grad_threshold > 0.0f ? 1 : 0, h->dc_flags.p, h->dc_keys.p, h->dc_vals.p, s);
    uint32_t np = density_scan(h, n, s);
    if (np == 0) return PALE_OK;
    if (max_new_points >= 0 && (int64_t)np > max_new_points / 2) {
      // the budget binds: the highest scores (ties: lower index first)
      np = (uint32_t)(max_new_points / 2);
      density_sort(h, n, s);
      fill_u32(h->dc_flags.p, n, 0u, s);
      mark_indices(h->dc_vals.p, np, n, h->dc_flags.p, 1u, s);
      density_scan(h, n, s);
    }
    // parents in increasing index order
    flagged_list(h->dc_flags.p, h->dc_dst.p, n, h->dc_list.p, s);
    if (parents_out) indices_to_host(h, h->dc_list.p, np, parents_out, false, s);
    // survivors in order, then two children per parent
    fill_u32(h->dc_flags.p, n, 1u, s);
    mark_indices(h->dc_list.p, np, n, h->dc_flags.p, 0u, s);
    const uint32_t kept = density_scan(h, n, s);
    h->dc_points.alloc(kept + 2 * np);
    compact_points(h->asset.view(), h->dc_flags.p, h->dc_dst.p, n, h->dc_points.view(), s);
    split_children(h->asset.view(), h->dc_list.p, np, kept, h->dc_points.view(), split_distance, minor_axis_shrink,
                   opacity_reduction, s);
    density_commit(h, kept + 2 * np, s);
    if (parent_count) *parent_count = np;
    return PALE_OK;
  });
}

int pale_optimizer_reset(pale_handle* h) {
  if (!h) return PALE_ERR_ARGUMENT;
  h->opt_gen = ~0ull;
  return PALE_OK;
}

int pale_optimizer_step(pale_handle* h, const pale_optimizer* o, const pale_points* d_grads, void* stream) {
  if (!h) return PALE_ERR_ARGUMENT;
  return guarded(h, [&]() {
    check_optimizer(o);
    PointsDev grads = h->grads.view();
    if (d_grads) {
      if (d_grads->count != h->np) throw ArgError("pale_optimizer_step: gradient count differs from the point count");
      if (h->np && (!d_grads->position || !d_grads->tangent_u || !d_grads->tangent_v || !d_grads->scale ||
                    !d_grads->albedo || !d_grads->opacity || !d_grads->beta))
        throw ArgError("pale_optimizer_step: missing gradient field");
      grads = PointsDev{d_grads->position, d_grads->tangent_u, d_grads->tangent_v, d_grads->scale,
                        d_grads->albedo, d_grads->opacity, d_grads->beta, nullptr};
    } else if (h->grads_gen != h->bvh_gen) {
      throw ArgError("pale_optimizer_step: no adjoint pass since the last BVH build");
    }
    use_stream(h, caller_stream(stream));
    cudaStream_t s = h->stream;
    const uint32_t n = h->np;
    if (h->opt_gen != h->bvh_gen || h->opt_type != o->type) {
      // a fresh optimizer: zero moments and step counts
      h->opt_m.alloc(n);
      h->opt_v.alloc(n);
      h->opt_steps.ensure(std::max(1u, n));
      zero_point_bufs(h, h->opt_m, s);
      zero_point_bufs(h, h->opt_v, s);
      if (n) CK(cudaMemsetAsync(h->opt_steps.p, 0, 4ull * n, s));
      h->opt_gen = h->bvh_gen;
      h->opt_type = o->type;
      h->opt_t = 0;
    }
    ++h->opt_t;
    OptArgs A{};
    A.n = n;
    A.grads = grads;
    A.params = h->params.view();
    A.asset = h->asset.view();
    A.m = h->opt_m.view();
    A.v = h->opt_v.view();
    A.steps = h->opt_steps.p;
    A.mode = o->type;
    A.use_mask = (o->type == PALE_OPT_MASKED_ADAM && (o->flags & PALE_OPT_SURFEL_MASK)) ? 1u : 0u;
    A.first = h->opt_t == 1;
    // Python-float scalars of the torch step (bias corrections in double),
    // each rounded to float once where torch hands it to a float32 kernel.
    const double t = (double)h->opt_t;
    const double bc1 = 1.0 - std::pow(o->beta1, t);
    const double bc2 = 1.0 - std::pow(o->beta2, t);
    for (int g = 0; g < 6; ++g) {
      A.lr[g] = (float)o->lr[g];
      A.step_size[g] = o->type == PALE_OPT_SGD ? (float)o->lr[g] : (float)(o->lr[g] / bc1);
    }
    A.beta1 = (float)o->beta1;
    A.beta2 = (float)o->beta2;
    A.one_minus_beta1 = (float)(1.0 - o->beta1);
    A.one_minus_beta2 = (float)(1.0 - o->beta2);
    A.bc2_sqrt = (float)std::sqrt(bc2);
    A.eps = (float)o->eps;
    A.momentum = (float)o->momentum;
    A.opacity_reset = o->opacity_reset;
    for (int c = 0; c < 3; ++c) A.ref[c] = o->reference_dir[c];
    optimizer_step(A, s);
    derive_surfels(h->params.view(), n,
                   SurfelArrays{h->sf_pe.p, h->sf_n.p, h->sf_u.p, h->sf_v.p, h->sf_cn.p, h->sf_alb.p}, s);
    ++h->params_gen;
    CK(cudaGetLastError());
    return PALE_OK;
  });
}

int pale_trace_rays(pale_handle* h, uint32_t n, const float* o, const float* d, int32_t* inst, int32_t* prim,
                    float* t, float* alpha, float* pos) {
  if (!h) return PALE_ERR_ARGUMENT;
  return guarded(h, [&]() {
    if (n && (!o || !d || !inst || !prim || !t || !alpha)) throw ArgError("pale_trace_rays: null array");
    if (!n) return PALE_OK;
    use_stream(h, h->own_stream);
    cudaStream_t s = h->stream;
    DBuf<float> dO, dD, dT, dA, dP;
    DBuf<int32_t> dI, dR;
    dO.alloc(3ull * n); dD.alloc(3ull * n); dT.alloc(n); dA.alloc(n); dP.alloc(3ull * n); dI.alloc(n); dR.alloc(n);
    CK(cudaMemcpyAsync(dO.p, o, 12ull * n, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(dD.p, d, 12ull * n, cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(h->run.p, 0, sizeof(RunState), s));
    trace_rays(h->view(), h->run.p, n, dO.p, dD.p, dI.p, dR.p, dT.p, dA.p, dP.p, s);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(inst, dI.p, 4ull * n, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(prim, dR.p, 4ull * n, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(t, dT.p, 4ull * n, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(alpha, dA.p, 4ull * n, cudaMemcpyDeviceToHost, s));
    if (pos) CK(cudaMemcpyAsync(pos, dP.p, 12ull * n, cudaMemcpyDeviceToHost, s));
    h->timed = 0;
    h->launches_last = 1;
    copy_stats(h);
    return PALE_OK;
  });
}

int pale_trace_transmittance(pale_handle* h, uint32_t n, const float* o, const float* d, int32_t* inst, float* t,
                             float* transmit) {
  if (!h) return PALE_ERR_ARGUMENT;
  return guarded(h, [&]() {
    if (n && (!o || !d || !inst || !t || !transmit)) throw ArgError("pale_trace_transmittance: null array");
    if (!n) return PALE_OK;
    use_stream(h, h->own_stream);
    cudaStream_t s = h->stream;
    DBuf<float> dO, dD, dT, dX;
    DBuf<int32_t> dI;
    dO.alloc(3ull * n); dD.alloc(3ull * n); dT.alloc(n); dX.alloc(n); dI.alloc(n);
    CK(cudaMemcpyAsync(dO.p, o, 12ull * n, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(dD.p, d, 12ull * n, cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(h->run.p, 0, sizeof(RunState), s));
    trace_transmittance(h->view(), h->run.p, n, dO.p, dD.p, dI.p, dT.p, dX.p, s);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(inst, dI.p, 4ull * n, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(t, dT.p, 4ull * n, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(transmit, dX.p, 4ull * n, cudaMemcpyDeviceToHost, s));
    h->timed = 0;
    h->launches_last = 1;
    copy_stats(h);
    return PALE_OK;
  });
}

int pale_gather_irradiance(pale_handle* h, uint32_t n, const float* pts, const float* nrm, float* E) {
  if (!h) return PALE_ERR_ARGUMENT;
  return guarded(h, [&]() {
    if (n && (!pts || !nrm || !E)) throw ArgError("pale_gather_irradiance: null array");
    if (!n) return PALE_OK;
    use_stream(h, h->own_stream);
    cudaStream_t s = h->stream;
    DBuf<float> dP, dN, dE;
    dP.alloc(3ull * n); dN.alloc(3ull * n); dE.alloc(3ull * n);
    CK(cudaMemcpyAsync(dP.p, pts, 12ull * n, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(dN.p, nrm, 12ull * n, cudaMemcpyHostToDevice, s));
    gather_points(h->view(), n, dP.p, dN.p, dE.p, s);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(E, dE.p, 12ull * n, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return PALE_OK;
  });
}

int pale_load_photons(pale_handle* h, uint32_t n, const float* pos, const float* pw, const float* dir) {
  if (!h) return PALE_ERR_ARGUMENT;
  return guarded(h, [&]() {
    if (n && (!pos || !pw || !dir)) throw ArgError("pale_load_photons: null array");
    use_stream(h, h->own_stream);
    cudaStream_t s = h->stream;
    if (n > (1u << 30)) throw ArgError("at most 2^30 photons can be loaded");
    if (n > h->photon_cap) {
      CK(cudaStreamSynchronize(s));
      alloc_photon_store(h, n);
    }
    DBuf<float> dP, dW, dD;
    dP.alloc(3ull * n); dW.alloc(3ull * n); dD.alloc(3ull * n);
    if (n) {
      CK(cudaMemcpyAsync(dP.p, pos, 12ull * n, cudaMemcpyHostToDevice, s));
      CK(cudaMemcpyAsync(dW.p, pw, 12ull * n, cudaMemcpyHostToDevice, s));
      CK(cudaMemcpyAsync(dD.p, dir, 12ull * n, cudaMemcpyHostToDevice, s));
    }
    PhotonStore ps{h->ph_a.p, h->ph_b.p, h->ph_c.p, h->ph_sa.p, h->ph_sb.p, h->ph_sc.p, h->photon_cap};
    load_photon_arrays(n, dP.p, dW.p, dD.p, ps, s);
    ++h->photon_gen;
    CK(cudaMemsetAsync(h->run.p, 0, sizeof(RunState), s));
    CK(cudaMemcpyAsync(&h->run.p->photon_attempts, &n, 4, cudaMemcpyHostToDevice, s));
    GridBufs G{};
    G.cell_id = h->g_cell_id.p; G.sorted = h->g_sorted.p; G.keys_tmp = h->g_keys.p; G.vals_tmp = h->g_vals_tmp.p;
    G.sort_temp = h->g_sort_temp.p; G.cell_count = h->g_cell_count.p; G.cell_off = h->g_cell_off.p;
    G.scan_temp = h->g_scan_temp.p; G.pa = h->g_pa.p; G.pb = h->g_pb.p; G.pc = h->g_pc.p; G.d_stored = h->g_stored.p;
    G.d_attempts = h->g_attempts.p;
    grid_build(h->view(), h->run.p, ps, G, h->cells, h->key_bits, s);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s));
    return PALE_OK;
  });
}

int pale_get_photons(pale_handle* h, uint32_t* count, float* position, float* power, float* direction,
                     uint32_t* cell_id, uint32_t* sorted, float* grid_info) {
  if (!h || !count) return PALE_ERR_ARGUMENT;
  return guarded(h, [&]() {
    use_stream(h, h->own_stream);
    cudaStream_t s = h->stream;
    uint32_t n = 0;
    CK(cudaMemcpyAsync(&n, h->g_stored.p, 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    *count = n;
    if (n && (position || power || direction)) {
      std::vector<float4> a(n), b(n);
      std::vector<float> c(n);
      CK(cudaMemcpyAsync(a.data(), h->ph_a.p, 16ull * n, cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(b.data(), h->ph_b.p, 16ull * n, cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(c.data(), h->ph_c.p, 4ull * n, cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      for (uint32_t i = 0; i < n; ++i) {
        if (position) { position[3 * i] = a[i].x; position[3 * i + 1] = a[i].y; position[3 * i + 2] = a[i].z; }
        if (power) { power[3 * i] = a[i].w; power[3 * i + 1] = b[i].w; power[3 * i + 2] = c[i]; }
        if (direction) { direction[3 * i] = b[i].x; direction[3 * i + 1] = b[i].y; direction[3 * i + 2] = b[i].z; }
      }
    }
    if (n && cell_id) CK(cudaMemcpyAsync(cell_id, h->g_cell_id.p, 4ull * n, cudaMemcpyDeviceToHost, s));
    if (n && sorted) CK(cudaMemcpyAsync(sorted, h->g_sorted.p, 4ull * n, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (grid_info) {
      grid_info[0] = h->origin[0]; grid_info[1] = h->origin[1]; grid_info[2] = h->origin[2];
      grid_info[3] = h->cell;
      grid_info[4] = (float)h->res[0]; grid_info[5] = (float)h->res[1]; grid_info[6] = (float)h->res[2];
    }
    return PALE_OK;
  });
}

int pale_get_bvh(pale_handle* h, uint32_t* codes, uint32_t* node_count, float* nodes, uint32_t max_nodes) {
  if (!h) return PALE_ERR_ARGUMENT;
  return guarded(h, [&]() {
    use_stream(h, h->own_stream);
    cudaStream_t s = h->stream;
    if (node_count) *node_count = h->np ? h->node_count : 0;
    if (codes && h->np) CK(cudaMemcpyAsync(codes, h->codes.p, 4ull * h->np, cudaMemcpyDeviceToHost, s));
    if (nodes && h->np) {
      uint32_t k = std::min(max_nodes, h->node_count);
      CK(cudaMemcpyAsync(nodes, h->nodes.p, 64ull * k, cudaMemcpyDeviceToHost, s));
    }
    CK(cudaStreamSynchronize(s));
    return PALE_OK;
  });
}

int pale_get_stats(pale_handle* h, pale_stats* out) {
  if (!h || !out) return PALE_ERR_ARGUMENT;
  return guarded(h, [&]() {
    if (h->stats_pending) copy_stats(h);
    *out = h->stats;
    return PALE_OK;
  });
}

}  // extern "C"
