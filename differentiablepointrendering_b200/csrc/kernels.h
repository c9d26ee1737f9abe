// kernels.h -- launch wrappers shared by the build, render and API units.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "common.cuh"

namespace pale {

// Per-point parameter arrays on the device (structure of arrays).
struct PointsDev {
  float* position;
  float* tangent_u;
  float* tangent_v;
  float* scale;
  float* albedo;
  float* opacity;
  float* beta;
  float* shape;
};

struct SurfelArrays {
  float4 *pe, *n, *u, *v, *cn, *alb;
};

struct LbvhArgs {
  uint32_t n;
  const uint32_t* d_n;      // device copy of n (radix sort)
  uint32_t leaf_size;
  uint32_t top;
  PointsDev asset;          // asset-order input
  PointsDev collected;      // asset-order collected
  PointsDev params;         // BVH-order output
  SurfelArrays derived;
  float *lo, *hi;           // asset-order boxes
  float *bounds_part, *bounds;   // bounds[0..5] centroid lo/hi, [6..11] box lo/hi
  uint32_t *codes, *order, *codes_tmp, *order_tmp, *sort_temp;
  int32_t *lc, *rc;
  uint32_t *rfirst, *rlast, *parent, *leaf_parent, *visits;
  float* box;
  BvhNode* nodes;
  uint32_t* err;            // device error word
};

size_t scan_temp_words(uint32_t n);
void exclusive_scan(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* temp, uint32_t* total,
                    cudaStream_t s);
size_t radix_temp_words(uint32_t n_max);
void radix_sort_pairs(uint32_t* keys, uint32_t* vals, uint32_t* keys_tmp, uint32_t* vals_tmp, const uint32_t* d_n,
                      uint32_t n_max, int bits, uint32_t* temp, cudaStream_t s);
void lbvh_build(const LbvhArgs& a, cudaStream_t s);
// The traversal copy of n nodes (BvhNodeH: boxes rounded outwards to half).
void half_nodes(const BvhNode* in, uint32_t n, BvhNodeH* out, cudaStream_t s);
void derive_surfels(const PointsDev& p, uint32_t n, const SurfelArrays& d, cudaStream_t s);

// One optimizer step on the device (optim.cu), in BVH order like the
// parameters and gradients it reads.  Moments have the parameter layout.
enum OptMode : uint32_t { kOptAdam = 0, kOptSgd = 1, kOptMaskedAdam = 2 };
struct OptArgs {
  uint32_t n;
  PointsDev grads;         // gradients of the last adjoint pass
  PointsDev params;        // updated in place
  PointsDev asset;         // receives a copy of the updated parameters
  PointsDev m, v;          // first / second moments (SGD: m = momentum buffer)
  uint32_t* steps;         // masked Adam: per-surfel step counts
  uint32_t mode;           // OptMode
  uint32_t use_mask;       // masked Adam: only surfels with a nonzero gradient
  uint32_t first;          // SGD: first step (momentum buffer = gradient)
  float lr[6];             // groups: position, tangents, scale, albedo, opacity, beta
  float step_size[6];      // Adam: lr / (1 - beta1^t); SGD: lr
  float beta1, beta2, one_minus_beta1, one_minus_beta2, bc2_sqrt, eps, momentum;
  float opacity_reset;     // >= 0: every opacity set to it after the step
  float ref[3];            // tangent frames: normal oriented towards ref
};
void optimizer_step(const OptArgs& a, cudaStream_t s);

// Density control helpers (density.cu).
void opacity_sort_keys(const float* op, uint32_t n, uint32_t* keys, uint32_t* vals, cudaStream_t s);
void count_le(const float* v, uint32_t n, float thr, uint32_t* count, cudaStream_t s);
void fill_u32(uint32_t* a, uint32_t n, uint32_t value, cudaStream_t s);
void mark_indices(const uint32_t* idx, uint32_t k, uint32_t n, uint32_t* flags, uint32_t value, cudaStream_t s);
void compact_points(const PointsDev& src, const uint32_t* keep, const uint32_t* dst, uint32_t n, const PointsDev& out,
                    cudaStream_t s);
void flagged_list(const uint32_t* flag, const uint32_t* dst, uint32_t n, uint32_t* list, cudaStream_t s);
void split_candidates(const PointsDev& a, uint32_t n, const float* importance, float min_long, float grad_threshold,
                      int use_threshold, uint32_t* cand, uint32_t* keys, uint32_t* vals, cudaStream_t s);
void split_children(const PointsDev& a, const uint32_t* parents, uint32_t np, uint32_t base, const PointsDev& out,
                    double split, double shrink, double reduction, cudaStream_t s);

// Device time of the hot kernels: a pair of CUDA events around every launch
// of a timed kernel, summed per kernel after the stream is synchronised.
// Host-side only (kernels receive the pointer inside their argument
// structs but never touch it).
enum TimedKernel : int { kTimeTrace = 0, kTimeLookup = 1, kTimeAdjBounce = 2, kTimeTransport = 3, kTimedKernels = 4 };

struct KernelTimer {
  std::vector<cudaEvent_t> pool;   // start, end, start, end, ...
  std::vector<int> kind;
  size_t used = 0;
  bool open = false;
  void begin(int k, cudaStream_t s);
  void end(cudaStream_t s);
  // Adds the elapsed times of the recorded pairs to ms[] / n[] and starts over.
  void collect(float* ms, uint32_t* n);
  ~KernelTimer();
};

// ------------------------------------------------------------ rendering
struct QueueBufs {
  RayRec* q[2];           // ping-pong ray queues
  RayRec* stage;          // per-slot staging of the next ray
  uint8_t* flags;         // per-slot: 1 alive, 2 deposit / event
  uint2* tile_counts;     // per 256-slot tile: (alive, deposit|event)
  uint2* tile_offsets;
  uint32_t capacity;
};

struct PhotonStore {
  float4* a;              // deposit order: position, power.r
  float4* b;              // incoming direction, power.g
  float* c;               // power.b
  float4 *sa, *sb;        // staging per slot
  float* sc;
  uint64_t capacity;
};

struct GridBufs {
  uint32_t* cell_id;      // per stored photon (deposit order)
  uint32_t* sorted;       // sorted position -> deposit index
  uint32_t *keys_tmp, *vals_tmp, *sort_temp;
  uint32_t* cell_count;   // cells + 1
  uint32_t* cell_off;     // cells + 1
  uint32_t* scan_temp;
  float4 *pa, *pb;        // sorted photons
  float* pc;
  uint32_t* d_stored;     // photons stored (device)
  uint32_t* d_attempts;   // deposits attempted, read by the lookups
};

// Adjoint pending interaction per path (PendingAdjointState,
// GPUDataStructures.h:319-336): (position, alpha) (throughput, kind)
// (primitive, instance, pixel, -).
struct PendingBufs {
  float4* a;
  float4* b;
  uint4* c;
};

// Completed gradient event (CompletedGradientEvent, :338-369), reduced to
// what the transport step needs.
struct EventRec {
  float4 a;   // gather position, alpha (alpha_geom or endpoint alpha_geom)
  float4 b;   // gather normal, endpoint pdf or endpoint cosine
  float4 c;   // path throughput, -
  uint4 d;    // kind, target surfel, material, pixel
  float4 e;   // hit position on the target surfel (its alpha term's point), -
  float4 f;   // unit ray direction at that hit, -
};

struct EventBufs {
  EventRec* stage;        // per slot
  EventRec* list;         // compacted, slot order
};

// The scenes of one render call.  A call renders views (a camera of a scene
// and its number of passes); the views of every scene trace as one
// wavefront, each path finding its scene's surfels, LBVH, meshes and photon
// grid through the view's scene index.  The traversal kernels stage each
// scene's first top_nodes LBVH nodes in shared memory, scene k's in the
// slot [k * staged, (k + 1) * staged) (top_nodes <= staged; a small scene
// stages fewer), at most kStagedNodesPerCall nodes for the whole table:
// 16 KB, so that the camera walk (with its 16 KB stack and 16 KB hit list
// per 256-thread block) keeps 4 resident blocks in a call of many scenes.
#ifndef PALE_STAGED_NODES_PER_CALL
#define PALE_STAGED_NODES_PER_CALL 512
#endif
constexpr uint32_t kMaxScenes = 8;
constexpr uint32_t kStagedNodesPerCall = PALE_STAGED_NODES_PER_CALL;

struct SceneTable {
  SceneView s[kMaxScenes];
  uint32_t n;
  uint32_t staged;
};

// Where the camera seeds of a scene's forward render start: the scene's
// seed table and the device word holding the cursor position after its
// photon passes.
struct SceneSeeds {
  const uint32_t* seeds;
  const uint32_t* cursor;
};

// Gradient arrays of a scene (BVH order).
struct SceneGrads {
  float* opacity;
  PointsDev all;          // all seven groups, written when all_grads
};

// The camera gather's path vertices, for the gather estimator (the exact
// derivative of the gathered image with the photon map held).  Every queue
// entry of a round (a live camera path) and every lookup record of its
// layers get a slot: records at base[r] + (the record's index in round r),
// entries at base[kVertexBases + r] + (the entry's index in round r).  The
// bases are kept whenever `base` is set (the record and entry counts of a
// chunk); slots are written when `write` is set and dropped, with
// *overflow set, past the capacities.
constexpr uint32_t kVertexBases = kMaxLayers + 1;

struct VertexStore {
  float4* rec_xa;       // surfel layer: hit point, alpha_geom
  float4* rec_ew;       // irradiance at the layer (or at the mesh that ends the path), index word
  float4* ent_d;        // ray direction, transmittance in front of the entry's first layer
  uint4* ent_b;         // first record, records | emitter << 8, next round's entry or kInvalid, path
  float4* ent_l;        // emitter radiance (unattenuated); the sweep's radiance behind the entry's front
  uint32_t* base;       // 2 * kVertexBases words
  uint32_t* overflow;
  uint32_t rec_cap, ent_cap;
  uint32_t rec_start, ent_start;   // where the chunk's first round starts
  int write;
};

struct FrameArgs {
  SceneTable scenes;
  SceneSeeds sseeds[kMaxScenes];
  RunState* st;
  const CameraRec* cams;  // the views, in packing order (pixel_offset increasing)
  uint32_t ncams;
  uint32_t total_pixels;
  float* raw;             // packed H*W*4 per camera
  float* ldr;
  // the current chunk's view table (3 words per view): view_start[v], the
  // first path of view v in the chunk (non-decreasing; a view without a
  // pass in the chunk has an empty range), then view_start[ncams + v] and
  // view_start[2 ncams + v], the view's passes [p0, p1) in the chunk, at
  // paths view_start[v] + (pass - p0) * pixels + pixel
  const uint32_t* view_start;
  uint32_t walk_block;     // threads per block of the persistent walks (host side)
  uint32_t rng_mode;
  float exposure, gamma;
  // wavefront buffers: path queues (ping-pong by round), lookup records (2
  // float4 each, up to kGatherHits per queue entry), per-entry record range
  // and end state, queue lengths per round (kMaxLayers + 2 words) followed
  // by record counts per round (as many), per-path radiance, running
  // framebuffer
  RayRec* paths[2];
  float4* qrec;
  uint4* info_a;
  float4* info_b;
  uint32_t* counts;
  float4* res;
  float4* fb;
  uint32_t path_capacity;  // >= total_pixels
  // per queue entry of a round: the closest mesh hit (position, instance
  // bits), the surfel walk's record (origin, limit or -1 when the path does
  // not enter the surfel cloud's box) (unit direction), and the walk's
  // result: the hit count and the surfels of the K closest hits
  // (kKHitWords words)
  float4* mhit;
  float4* walk;
  uint32_t* khit;
  KernelTimer* timer;      // host side, may be null
  // optional L2 image loss: target packed like the images with
  // target_channels floats per pixel; dL/dI (float4 per pixel) written by
  // the post-process
  const float* target;
  uint32_t target_channels;
  float* dldi;
  // the gather estimator's vertex store (base null: not kept)
  VertexStore vs;
};

// LBVH nodes duplicated in breadth-first order at the front of the node
// array and staged in shared memory by every traversal kernel.
#ifndef PALE_TOP_NODES
#define PALE_TOP_NODES 256
#endif
constexpr uint32_t kTopNodes = PALE_TOP_NODES;

// Surfel layers collected per traversal of the camera gather.
#ifndef PALE_GATHER_HITS
#define PALE_GATHER_HITS 8
#endif
constexpr int kGatherHits = PALE_GATHER_HITS;
// The camera walk's hit list in shared memory (1) or registers (0).
#ifndef PALE_KHIT_SMEM
#define PALE_KHIT_SMEM 1
#endif
// Words of a K-hit walk result: the count and K surfels, padded to uint4s.
constexpr int kKHitWords = (kGatherHits + 4) / 4 * 4;
// Resident blocks per SM the record kernels around the walks (camera
// layer records, adjoint shading) are compiled for (their register budget:
// 65536 / (kBlock * blocks)).
#ifndef PALE_TRACE_MIN_BLOCKS
#define PALE_TRACE_MIN_BLOCKS 4
#endif
constexpr int kTraceMinBlocks = PALE_TRACE_MIN_BLOCKS;
// The camera gather's 8-hit walk: 4 resident blocks with its hit list in
// shared memory (3 with the list in registers, which need them more than
// the fourth block).
#ifndef PALE_ROUND_MIN_BLOCKS
#define PALE_ROUND_MIN_BLOCKS (PALE_KHIT_SMEM ? 4 : 3)
#endif
constexpr int kRoundMinBlocks = PALE_ROUND_MIN_BLOCKS;
// The same for the warp-per-lookup kernels (camera lookups, transport).
#ifndef PALE_LOOKUP_MIN_BLOCKS
#define PALE_LOOKUP_MIN_BLOCKS 4
#endif
constexpr int kLookupMinBlocks = PALE_LOOKUP_MIN_BLOCKS;
// The persistent walks (adjoint closest hit, camera 8 hits): lanes whose
// walk has ended take a new ray every PALE_REFILL_STEPS node visits;
// PALE_WALK_MIN_BLOCKS is the adjoint walk's register budget.
// A persistent walk's lanes standing at leaves test them together once at
// least PALE_LEAF_BATCH lanes of the warp do (or every walking lane).
#ifndef PALE_LEAF_BATCH
#define PALE_LEAF_BATCH 8
#endif
constexpr int kLeafBatch = PALE_LEAF_BATCH;

#ifndef PALE_REFILL_STEPS
#define PALE_REFILL_STEPS 16
#endif
constexpr int kRefillSteps = PALE_REFILL_STEPS;
#ifndef PALE_WALK_MIN_BLOCKS
#define PALE_WALK_MIN_BLOCKS 4
#endif
constexpr int kWalkMinBlocks = PALE_WALK_MIN_BLOCKS;
// The adjoint transport kernel: its event record and gradient terms spill
// at 64 registers.
#ifndef PALE_TRANSPORT_MIN_BLOCKS
#define PALE_TRANSPORT_MIN_BLOCKS 3
#endif
constexpr int kTransportMinBlocks = PALE_TRANSPORT_MIN_BLOCKS;

// Per-camera L2 loss 0.5 mean((ldr - target)^2) over the RGB values of
// each camera of a finished frame (needs a.ldr and a.target), summed in
// double in a fixed order: partials[ncams * kLossChunks], loss[ncams].
constexpr uint32_t kLossChunks = 64;
void image_loss(const FrameArgs& a, double* partials, double* loss, cudaStream_t s);

struct PhotonArgs {
  SceneView scene;
  RunState* st;
  const uint32_t* seeds;
  QueueBufs qb;
  PhotonStore ps;
  uint32_t photons_per_launch;
  float inv_emitted;
  uint32_t rr_start;
  float q_null, q_reflect, q_transmit;
};

// One adjoint job: every pixel of one selected camera for one pass.  The
// jobs of a batch trace as one wavefront; their rays stay grouped by job in
// the queues (stable compaction), and a ray's random stream is keyed by its
// rank inside its own job, as when each job runs alone.
struct AdjJob {
  uint32_t cam;           // index into the selected cameras
  uint32_t path_start;    // first path of the job in the batch
  uint32_t npix;
  uint32_t seed_index;    // first of the job's 1 + bounces seed-table words
};

constexpr uint32_t kMaxJobsPerBatch = 1024;

struct AdjointArgs {
  SceneTable scenes;
  SceneGrads sgrads[kMaxScenes];
  RunState* st;
  const uint32_t* seeds;
  QueueBufs qb;
  PendingBufs pend;
  EventBufs ev;
  const float* dldi;       // packed H*W*4 per camera
  uint32_t all_grads;
  float* debug_opacity;    // packed H*W*4 per camera or null
  const CameraRec* cams;   // selected cameras, packed pixel offsets
  const AdjJob* jobs;      // jobs of this batch
  uint32_t njobs;
  uint32_t* job_count;     // [2][kMaxJobsPerBatch] survivors per job
  uint32_t* job_start;     // [2][kMaxJobsPerBatch] queue start per job
  uint32_t rr_start;
  float q_null, q_reflect, q_transmit;
  uint32_t fixed_seed;     // reference mode: settings.random.number
  uint32_t rng_mode;
  float null_scale;        // NullTransmittance weight: 1 or 1 / q_null
  uint32_t light0_valid;
  float light0_area;
  KernelTimer* timer;      // host side, may be null
  // Bounces after the first trace their rays in the order of a sort by
  // (direction octant, origin Morton code): thread t takes queue slot
  // perm[t].  Each ray keeps its slot for its random stream and its
  // outputs, so the results do not depend on the order.  Null: slot order.
  uint32_t* sort_keys;     // 4 arrays of the queue capacity: keys, perm,
  uint32_t* perm;          //   and the sort's ping-pong copies
  uint32_t* sort_keys_tmp;
  uint32_t* perm_tmp;
  uint32_t* sort_temp;     // radix_temp_words(queue capacity)
  uint32_t sort_capacity;
  // Per queue slot, 3 float4: the closest mesh hit (position and distance,
  // +inf on a miss; alpha, instance bits, primitive bits) and the surfel
  // walk's result (surfel bits, distance, 1 on a hit), which the mesh pass
  // sets to no hit.  Per sorted position t (the order the walk takes the
  // rays in), the walk's record, 2 float4: (origin, walk limit or -1 when
  // the ray does not enter the surfel cloud's box) (unit direction, slot
  // bits).
  float4* hits;
  float4* walkq;
  uint32_t walk_block;     // threads per block of the persistent walks (host side)
};

void photon_emit(const PhotonArgs& a, cudaStream_t s);
void photon_bounce(const PhotonArgs& a, uint32_t parity, cudaStream_t s);
void grid_build(const SceneView& sv, RunState* st, const PhotonStore& ps, const GridBufs& g, uint32_t cells,
                int key_bits, cudaStream_t s);
// The camera gather of the views `views` (host copy of a.cams; every view
// passes >= 1); d_view_start holds 3 * views.size() words of device scratch
// (the chunks' view tables).
void camera_gather(const FrameArgs& a, const std::vector<CameraRec>& views, uint32_t* d_view_start,
                   cudaStream_t s, struct VertexPlan* plan = nullptr);

// One chunk of a camera gather: its paths and its view table (as
// FrameArgs::view_start).  The (view, pass) jobs are packed in view order,
// each view's passes in pass order, whole passes into a chunk while its
// paths fit the path capacity (one pass at least), so that every chunk but
// the last is full and a view's passes may span chunks.
struct GatherChunk {
  uint32_t n = 0;
  std::vector<uint32_t> table;
};
std::vector<GatherChunk> gather_chunks(const std::vector<CameraRec>& views, uint32_t path_capacity);

// Host record of a camera gather kept for the gather estimator: per chunk
// its paths, rounds, where its slots start and how many it used, whether
// they were stored, and its view table; d_chunk_base holds each chunk's
// 2 * kVertexBases bases.
struct VertexChunk {
  uint32_t n = 0, rounds = 0;
  uint32_t rec_start = 0, ent_start = 0, recs = 0, ents = 0;
  bool stored = false;
  std::vector<uint32_t> table;   // the chunk's view table
};

struct VertexPlan {
  bool store = false;          // write the chunks' slots while they fit
  std::vector<VertexChunk> chunks;
  uint32_t* d_chunk_base = nullptr;   // chunks.size() * 2 * kVertexBases words
};

// The gather estimator's backward over the chunks of `plan`: each stored
// chunk is swept from the store; any other is replayed (its rounds traced
// again with the forward's seeds, its slots written from 0) and swept.
// a: the forward's frame arguments with a.vs the store and a.view_start the
// device table; scratch: the store replayed chunks are written to (big
// enough for the largest chunk not stored).  The sweep reads dL/dI (float4
// per packed pixel) and accumulates into the scenes' gradient arrays.
struct SweepArgs {
  const float* dldi;
  SceneGrads grads[kMaxScenes];
  // optional (device): per view the arrays its gradients go to instead of
  // its scene's; a view whose opacity array is null is not swept
  const SceneGrads* view_grads;
  int all_grads;
};
void gather_backward(const FrameArgs& a, const std::vector<CameraRec>& views, const VertexPlan& plan,
                     const SweepArgs& w, const VertexStore& scratch, cudaStream_t s);
void adjoint_raygen(const AdjointArgs& a, uint32_t npaths, cudaStream_t s);
void adjoint_bounce(const AdjointArgs& a, uint32_t bounce, uint32_t npaths, cudaStream_t s);

// Component queries.
void trace_rays(const SceneView& sv, RunState* st, uint32_t n, const float* o, const float* d, int32_t* inst,
                int32_t* prim, float* t, float* alpha, float* pos, cudaStream_t s);
void trace_transmittance(const SceneView& sv, RunState* st, uint32_t n, const float* o, const float* d,
                         int32_t* inst, float* t, float* transmit, cudaStream_t s);
void gather_points(const SceneView& sv, uint32_t n, const float* p, const float* nrm, float* E, cudaStream_t s);
void load_photon_arrays(uint32_t n, const float* pos, const float* pw, const float* dir, const PhotonStore& ps,
                        cudaStream_t s);

}  // namespace pale

namespace pale {
// Counts kernel launches issued by this thread (reported in pale_stats).
void note_launch();
uint64_t launches_issued();
// Error text returned by pale_last_error(NULL) on this thread.
void set_thread_error(const std::string& msg);
}  // namespace pale
