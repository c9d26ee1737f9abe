/*
 * pale_b200.h -- C-ABI of the B200-native adjoint renderer for beta surfels.
 *
 * This is the drop-in boundary for Pale's `pale.Renderer` pybind11 module
 * (Pale/pale_bindings.cpp:1613-1650).  Every entry point takes plain pointers
 * and sizes; no C++ or torch types cross it and no exception escapes it.
 *
 * Return codes: 0 = ok, >0 = recoverable (capacity exceeded, iteration cap
 * hit inside a kernel), <0 = fatal (bad argument, CUDA error).  After a
 * non-zero return, pale_last_error() describes the failure.
 *
 * Orders of surfels: the "asset order" is the order the caller supplies
 * points in (PLY file order); the "BVH order" is the leaf order of the
 * device LBVH.  As in the reference (SceneBuild.cpp:710-731,
 * pale_bindings.cpp:734-757) every per-point array that comes back
 * (parameters, gradients) is in BVH order; pale_get_order() gives the map
 * order[bvh_index] = asset_index.
 *
 * Host buffers: the render calls that take host pointers copy 4 MB and
 * more at a time through pinned memory the handle holds (allocated at the
 * size of the largest such copy; without it, when the host cannot pin that
 * much, they copy from pageable memory), the host side of each copy split
 * over threads: the environment variable PALE_COPY_THREADS, read once,
 * sets how many (default: up to 8).
 */
#ifndef PALE_B200_H
#define PALE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PALE_OK 0
#define PALE_ERR_CAPACITY 1      /* a queue or photon store overflowed       */
#define PALE_ERR_DEVICE_FLAG 2   /* a kernel bounds check or loop cap fired  */
#define PALE_ERR_ARGUMENT (-1)
#define PALE_ERR_CUDA (-2)
#define PALE_ERR_STATE (-3)

#define PALE_RNG_REFERENCE 0     /* reproduce the reference's seeding        */
#define PALE_RNG_DECORRELATED 1  /* fresh seed per gather pass / adjoint spp */

typedef struct pale_handle pale_handle;

/* Renderer settings.  Field <- settings-dict key of the reference
 * (pale_bindings.cpp:123-139; PathTracerSettings, GPUDataStructures.h:407-422).
 * Fill with pale_default_settings() first. */
/* Weight of the adjoint's NullTransmittance gradient events.  The
 * reference completes a pending null event with throughput
 * (p / qNull) * qNull = p (AdjointKernels.cpp:171-204, 314-323), but a path
 * only takes the null branch with probability qNull, so the events' expected
 * sum is qNull times the occlusion term of d(image)/d(opacity).  REFERENCE
 * keeps that weighting (gradients identical to the reference's); UNBIASED
 * divides the term by qNull. */
#define PALE_NULL_WEIGHT_REFERENCE 0u
#define PALE_NULL_WEIGHT_UNBIASED 1u

/* Gradient groups the adjoint pass writes.  OPACITY is the reference's
 * live adjoint (AdjointKernels.cpp:389-509; the other six groups are zero,
 * SyclBridge.cpp:172-179).  ALL also writes beta, position, tangents and
 * scale through each event surfel's alpha_geom = (1 - r^2)^(4 e^beta),
 * r^2 = u^2 + v^2 at the ray-plane hit, and albedo through ProjectionScatter
 * events (the derivatives of AdjointGradientKernels.h:212-451, 757-808). */
#define PALE_GRADIENTS_OPACITY 0u
#define PALE_GRADIENTS_ALL 1u

/* Which seeds a camera uses: its camera-gather seed and, with decorrelated
 * seeds, its adjoint seeds.  SELECTION is the reference's: the camera's
 * position in the list a render call selects, so one camera rendered alone
 * and inside a larger selection draws different samples.  CAMERA keys the
 * seeds by the camera's index in the scene, so a camera's image and
 * gradient do not depend on which other cameras share the call (what a
 * server that merges requests needs, and ranks that split the cameras of
 * one scene). */
#define PALE_CAMERA_SEEDS_SELECTION 0u
#define PALE_CAMERA_SEEDS_CAMERA 1u

/* Which gradient the backward computes.  REFERENCE is the reference's
 * adjoint (AdjointKernels.cpp): its own paths from the camera, events at
 * their bounces, photon lookups at the events.  GATHER is the exact
 * derivative of the forward's camera-gather image with the photon map
 * held: the forward's camera paths (the same seeds) and their layers, each
 * layer k of a path getting dI/d(alpha_k) = T_k (Lo_k - Lb_k), Lb_k the
 * radiance composited behind it, chained to opacity, beta, position,
 * tangents, scales (through alpha_geom) and albedo.  A GATHER backward
 * differentiates the last forward render of the same views and fails with
 * PALE_ERR_ARGUMENT for any other. */
#define PALE_ESTIMATOR_REFERENCE 0u
#define PALE_ESTIMATOR_GATHER 1u

/* Where a GATHER backward finds the forward's path vertices (per layer its
 * hit point, alpha_geom and irradiance; per path segment its direction,
 * transmittance and links; 32 bytes per layer and 48 per segment).
 * CHECKPOINT keeps them from the forward in a store grown to the last
 * forward's need; REPLAY keeps none and the backward traces each chunk of
 * camera paths again with the forward's seeds (deterministic, so the
 * layers are the forward's) into a scratch store of one chunk; AUTO
 * checkpoints while the store fits vertex_store_bytes (0: half the free
 * device memory) and replays the chunks that do not fit. */
#define PALE_VERTICES_AUTO 0u
#define PALE_VERTICES_CHECKPOINT 1u
#define PALE_VERTICES_REPLAY 2u

typedef struct pale_settings {
    uint32_t photons_per_launch;   /* "photons"          (default 1e6)       */
    uint32_t max_bounces;          /* "bounces"          (6)                 */
    uint32_t forward_passes;       /* "forward_passes"   (6)                 */
    uint32_t gather_passes;        /* "gather_passes"    (6)                 */
    uint32_t adjoint_bounces;      /* "adjoint_bounces"  (6)                 */
    uint32_t adjoint_passes;       /* "adjoint_passes"   (6)                 */
    uint64_t seed;                 /* "seed"             (42)                */
    uint32_t random_number;        /* Random::number     (42) -- adjoint base */
    uint32_t rr_start;             /* russianRouletteStart (6)               */
    float q_null;                  /* AdjointSampleSettings (0.5/0.5/0)      */
    float q_reflect;
    float q_transmit;
    float gather_radius;           /* PathTracer.cpp:187 hard-codes 0.01     */
    uint32_t leaf_size;            /* surfels per LBVH leaf (1); the hits do
                                      not depend on it (the reference's
                                      BuildOptions use 4, SceneBuild.ixx:72) */
    uint32_t rng_mode;             /* PALE_RNG_*                             */
    uint32_t debug_images;         /* "debug_images"                         */
    float exposure;                /* SensorGPU::exposureCorrection (1.0)    */
    float gamma;                   /* SensorGPU::gammaCorrection   (2.2)     */
    uint32_t null_weight;          /* PALE_NULL_WEIGHT_*                     */
    uint32_t gradients;            /* PALE_GRADIENTS_*                       */
    uint32_t camera_seeds;         /* PALE_CAMERA_SEEDS_*                    */
    uint32_t gather_batch_paths;   /* camera paths in flight per gather chunk
                                      (0 = 2^25; at least every pixel once)  */
    uint32_t adjoint_batch_paths;  /* adjoint paths per batch of (camera,
                                      pass) jobs (0 = 2^24; at least the
                                      largest camera's pixels)               */
    uint32_t walk_block;           /* threads per block of the persistent
                                      BVH walks: 64, 128 or 256 (0 = 256)    */
    uint32_t estimator;            /* PALE_ESTIMATOR_* ("estimator")          */
    uint32_t vertex_store;         /* PALE_VERTICES_* ("vertices")            */
    uint64_t vertex_store_bytes;   /* AUTO's budget (0 = half the free memory) */
} pale_settings;

/* Per-point parameter block (structure of arrays, float32).
 * position/tangent_u/tangent_v/albedo: count*3, scale: count*2,
 * opacity/beta/shape: count.  For outputs, every pointer may be NULL to
 * skip that field. */
typedef struct pale_points {
    uint32_t count;
    float *position;
    float *tangent_u;
    float *tangent_v;
    float *scale;
    float *albedo;
    float *opacity;
    float *beta;
    float *shape;
} pale_points;

/* Scene description: triangle meshes, instances, materials, cameras and the
 * surfel cloud in asset order.  All matrices are 4x4 row-major float32 with
 * y = M x.  Mirrors the host data SceneBuild::build collects
 * (SceneBuild.cpp:72-392). */
typedef struct pale_scene_desc {
    uint32_t num_vertices;
    const float *vertices;          /* num_vertices*3, object space          */
    uint32_t num_triangles;
    const uint32_t *triangles;      /* num_triangles*3 vertex indices        */
    uint32_t num_meshes;
    const uint32_t *mesh_ranges;    /* num_meshes*2: first triangle, count   */
    uint32_t num_materials;
    const float *materials;         /* num_materials*4: base colour rgb, power */
    uint32_t num_instances;         /* mesh instances (the surfel cloud is one
                                       implicit extra instance after them)   */
    const uint32_t *instance_mesh;
    const uint32_t *instance_material;
    const float *instance_object_to_world;  /* num_instances*16             */
    const float *instance_world_to_object;  /* num_instances*16             */
    uint32_t num_cameras;
    const float *camera_inv_view;   /* num_cameras*16, camera -> world       */
    const float *camera_forward;    /* num_cameras*3                         */
    const float *camera_fovy_deg;   /* num_cameras                           */
    const uint32_t *camera_size;    /* num_cameras*2: width, height          */
    const char *camera_names;       /* num_cameras*16, NUL padded            */
    pale_points points;             /* asset-order surfels                   */
} pale_scene_desc;

/* Device-side counters of the last render call (for throughput metrics). */
typedef struct pale_stats {
    uint64_t photon_segments;       /* photon rays submitted to traversal    */
    uint64_t gather_segments;       /* camera-gather layer traversals        */
    uint64_t adjoint_segments;      /* adjoint rays submitted to traversal   */
    uint64_t photons_stored;        /* photons deposited in the map          */
    uint64_t gradient_events;       /* completed adjoint gradient events     */
    uint64_t gather_queries;        /* photon-map irradiance lookups         */
    uint64_t node_visits;           /* BVH nodes visited (instrumented only) */
    uint64_t surfel_tests;          /* ray/surfel tests (instrumented only)  */
    uint64_t photons_scanned;       /* photons scanned by lookups (instr.)   */
    uint64_t gather_node_visits;    /* ... of the camera-gather kernel alone */
    uint64_t gather_surfel_tests;
    uint64_t gather_photons_scanned;
    uint64_t kernel_launches;       /* kernels launched by the last call     */
    float forward_ms;               /* device time of the last forward pass  */
    float backward_ms;              /* device time of the last adjoint pass  */
    float photon_ms;                /* photon trace + grid build part        */
    float gather_ms;                /* camera gather part                    */
    float timed_ms[4];              /* device time of the hot kernels: camera
                                       trace, photon lookup, adjoint bounce,
                                       adjoint transport or the gather
                                       estimator's sweep (CUDA events around
                                       each launch or group of launches)     */
    uint32_t timed_launches[4];     /* ... and their launch counts           */
    uint64_t vertex_bytes;          /* vertex store + replay scratch held    */
    uint32_t vertex_chunks_stored;  /* last GATHER backward: chunks swept
                                       from the store ...                    */
    uint32_t vertex_chunks_replayed;/* ... and chunks traced again           */
    uint64_t vertex_records;        /* ... layer records and path segments   */
    uint64_t vertex_entries;        /*     it swept                          */
} pale_stats;

/* Fills *s with the reference's PathTracerSettings defaults. */
void pale_default_settings(pale_settings *s);

/* Library version string. */
const char *pale_version(void);

/* Error text of the last failing call on this handle; with handle == NULL
 * the last failure of pale_create on this thread. */
const char *pale_last_error(const pale_handle *h);

/* Creates a renderer on the current CUDA device: uploads meshes and cameras,
 * builds the surfel LBVH on the device, sizes the ray queues and configures
 * the photon grid from the scene bounds.  Replaces the constructor
 * PythonRenderer::PythonRenderer (pale_bindings.cpp:61-170) together with
 * PathTracer::setScene (PathTracer.cpp:22-53). */
int pale_create(const pale_scene_desc *desc, const pale_settings *settings,
                pale_handle **out);

/* Frees every device buffer of the handle.  (pale_bindings.cpp:172-177) */
int pale_destroy(pale_handle *h);

/* Number of surfels and cameras. */
int pale_point_count(const pale_handle *h, uint32_t *count);
int pale_camera_count(const pale_handle *h, uint32_t *count);
/* Camera name (16 bytes incl. NUL) and size.  (getCameraNames,
 * pale_bindings.cpp:1397-1403) */
int pale_camera_info(const pale_handle *h, uint32_t index, char name[16],
                     uint32_t *width, uint32_t *height);

/* Forward photon-mapped render of the selected cameras
 * (render_forward, pale_bindings.cpp:180-277; submitPhotonMappingKernel,
 * SyclBridge.cpp:82-166).  ldr_out / raw_out receive, per selected camera in
 * order, H*W*4 floats (row 0 = top).  Either may be NULL.  Host pointers. */
int pale_render_forward(pale_handle *h, uint32_t num_selected,
                        const uint32_t *camera_indices, float *ldr_out,
                        float *raw_out);

/* The camera gather alone (launchCameraGatherKernel + post-process) from
 * the current photon map: the last forward's, or photons given to
 * pale_load_photons.  The camera seeds are those the last forward used, so
 * right after pale_render_forward it returns the same images.  With the
 * photon map held fixed, finite differences of these images are what the
 * adjoint pass differentiates (it does not follow the photon map).  Host
 * pointers, layout as pale_render_forward.  No counterpart in the reference,
 * which always retraces the photons. */
int pale_render_gather(pale_handle *h, uint32_t num_selected,
                       const uint32_t *camera_indices, float *ldr_out,
                       float *raw_out);

/* Same render, but the LDR/RAW images are written to DEVICE pointers
 * (no host copies).  `stream` is a cudaStream_t; NULL is the default
 * (legacy) stream.  The call returns without waiting for the work, except
 * that the camera gather reads one queue length per 16 surfel layers. */
int pale_render_forward_device(pale_handle *h, uint32_t num_selected,
                               const uint32_t *camera_indices, float *d_ldr,
                               float *d_raw, void *stream);

/* Adjoint pass (render_backward, pale_bindings.cpp:279-731;
 * submitAdjointKernel, SyclBridge.cpp:169-294).  dldi holds, per selected
 * camera in order, H*W*4 floats of dL/dI (alpha ignored).  Gradients are
 * written in BVH order into *grads (fields may be NULL).  debug_opacity,
 * when not NULL, receives per camera H*W*4 floats of the opacity-gradient
 * debug image (DebugImages::framebufferOpacity).  Host pointers. */
int pale_render_backward(pale_handle *h, uint32_t num_selected,
                         const uint32_t *camera_indices, const float *dldi,
                         pale_points *grads, float *debug_opacity);

/* Forward pass plus the training loop's L2 image loss (compute_l2_grad and
 * compute_l2_loss, python/losses.py:10-45, per camera as
 * python/training.py:625-657 applies them): with the LDR image I of each
 * selected camera and the target T (RGB, packed like the images with
 * `channels` = 3 or 4 floats per pixel, alpha ignored), the post-process
 * writes dL/dI = (I - T) / (3 W H) (packed float4 per pixel, alpha 0) and
 * loss[c] = 0.5 mean((I - T)^2) over the camera's RGB values (double).
 * Host buffers; every output may be NULL. */
int pale_render_forward_loss(pale_handle *h, uint32_t num_selected,
                             const uint32_t *camera_indices,
                             const float *target, uint32_t channels,
                             float *ldr, float *raw, float *dldi,
                             double *loss);

/* Same with DEVICE pointers, enqueued on `stream` (NULL = the default
 * stream) without waiting; d_ldr, d_raw, d_dldi and d_loss may be NULL. */
int pale_render_forward_loss_device(pale_handle *h, uint32_t num_selected,
                                    const uint32_t *camera_indices,
                                    const float *d_target, uint32_t channels,
                                    float *d_ldr, float *d_raw, float *d_dldi,
                                    double *d_loss, void *stream);

/* Same adjoint pass with DEVICE pointers for dL/dI and the gradient fields,
 * enqueued on `stream` (NULL = the default stream) without waiting. */
int pale_render_backward_device(pale_handle *h, uint32_t num_selected,
                                const uint32_t *camera_indices,
                                const float *d_dldi, pale_points *d_grads,
                                void *stream);

/* One view of a batched render: a camera of one of the call's scenes with
 * its own number of passes and adjoint bounces. */
typedef struct pale_view {
    uint32_t scene;    /* index into the call's scene list                      */
    uint32_t camera;   /* camera index in that scene                            */
    uint32_t passes;   /* gather passes in a forward call, adjoint passes in an
                          adjoint call: 1 .. the scene's gather_passes /
                          adjoint_passes                                        */
    uint32_t depth;    /* adjoint bounces: 0 = the scene's adjoint_bounces, at
                          most that                                             */
    uint32_t first_pass;  /* forward calls: render passes [first_pass,
                          first_pass + pass_count) of `passes` (a view rendered
                          in slices over several calls, its running sums kept
                          in the caller's d_partial); 0 and 0: all of them       */
    uint32_t pass_count;
} pale_view;

/* Batched forward render with the L2 loss: the views of up to 8 scenes of
 * uneven resolution, passes and depth as ONE camera-gather wavefront (every
 * path finds its scene's surfels, LBVH, meshes and photon grid through its
 * view).  No counterpart in the reference, which renders one camera and
 * one pass per launch (SyclBridge.cpp:136-146).  With trace_photons every
 * scene first traces its own photon map; without, the views use the
 * current photon maps.  Images, dL/dI and losses are packed in view order
 * like pale_render_forward_loss_device's (d_target likewise); d_ldr, d_raw,
 * d_dldi and d_loss may be NULL.  Runs on `stream` (NULL = the default
 * stream) with the wavefront buffers of scenes[0], without waiting; a
 * camera's seeds follow the scenes' camera_seeds setting.  Errors are
 * reported through scenes[0] (pale_last_error).
 * Slices: a view with a pass range (first_pass, pass_count) renders only
 * those passes (with trace_photons 0: every slice on one photon map);
 * d_partial (DEVICE, float4 per packed pixel, needed when any
 * view has a range) holds the view's running sum of the passes before
 * first_pass on entry (ignored for first_pass 0) and of the passes up to
 * the range's end on return when the view is not finished; a view's images,
 * dL/dI and loss are written by the call that renders its last pass, and
 * are then the same, bit for bit, as those of one call over all passes. */
int pale_render_views_loss_device(uint32_t num_scenes, pale_handle *const *scenes,
                                  int trace_photons, uint32_t num_views,
                                  const pale_view *views, const float *d_target,
                                  uint32_t channels, float *d_ldr, float *d_raw,
                                  float *d_dldi, double *d_loss, float *d_partial,
                                  void *stream);

/* The photon passes and the photon grid of the scene alone (the first half
 * of render_forward, SyclBridge.cpp:82-138), enqueued on `stream` (NULL =
 * the default stream) without waiting: the photon map that gather-only
 * renders (pale_render_gather, or views rendered without trace_photons)
 * then use, e.g. a server's resident scene. */
int pale_trace_photon_map(pale_handle *h, void *stream);

/* The adjoint pass of the same views as ONE wavefront of (view, pass) jobs:
 * dL/dI packed in view order (DEVICE).  With d_grads NULL each scene's
 * gradients go to the scene's own gradient arrays (zeroed first), those
 * that pale_optimizer_step with NULL gradients applies; else
 * d_grads holds num_scenes entries of DEVICE arrays (BVH order, every field
 * but shape non-null) that entry k's gradients accumulate in after they
 * are zeroed, and one scene may then fill several entries, so that the
 * views of different requests of one scene keep separate gradients in one
 * wavefront.  The rng mode, null weighting and gradient groups are
 * scenes[0]'s. */
int pale_render_views_backward_device(uint32_t num_scenes, pale_handle *const *scenes,
                                      uint32_t num_views, const pale_view *views,
                                      const float *d_dldi, pale_points *d_grads,
                                      void *stream);

/* The gather estimator's backward (scenes[0]'s estimator must be
 * PALE_ESTIMATOR_GATHER) of the last pale_render_views_loss_device call
 * with the same scenes and views, with gradients per VIEW: d_grads holds
 * num_views entries of DEVICE arrays (BVH order of the view's scene, every
 * field but shape non-null) that view i's gradients go to after they are
 * zeroed; an entry whose opacity pointer is NULL gets none and its view is
 * not swept.  dL/dI packed in view order (DEVICE).  So the requests of a
 * server that share a scene keep separate gradients from one forward
 * wavefront.  No reference counterpart (one camera per call there). */
int pale_render_views_gradients_device(uint32_t num_scenes, pale_handle *const *scenes,
                                       uint32_t num_views, const pale_view *views,
                                       const float *d_dldi, const pale_points *d_grads,
                                       void *stream);

/* Current per-point parameters in BVH order (get_point_parameters,
 * pale_bindings.cpp:733-850). */
int pale_get_points(pale_handle *h, pale_points *out);

/* order[bvh_index] = asset_index of the last build. */
int pale_get_order(pale_handle *h, uint32_t *order);

/* Overwrites the BVH-ordered surfel parameters WITHOUT rebuilding the BVH
 * (apply_point_optimization, pale_bindings.cpp:853-1056: the BVH nodes stay
 * as they were).  params->count must equal the current count. */
int pale_apply_points(pale_handle *h, const pale_points *params);

/* Same with the seven fields as DEVICE pointers (BVH order; shape is
 * ignored), enqueued on `stream` (NULL = the default stream) without
 * waiting: the parameter tensors of a torch training loop go to the
 * renderer without a host round trip. */
int pale_apply_points_device(pale_handle *h, const pale_points *d_params, void *stream);

/* Rebuilds the LBVH from an asset-order point set of any size (rebuild_bvh,
 * pale_bindings.cpp:1058-1079; also behind add_points / remove_points /
 * set_point_* which edit the asset and rebuild).  asset_points == NULL
 * rebuilds from the renderer's own asset, which pale_apply_points and
 * pale_optimizer_step keep equal to the last written parameters, as
 * rebuild_bvh() does. */
int pale_rebuild(pale_handle *h, const pale_points *asset_points);

/* The renderer's asset (the point set the last BVH build started from, or
 * the parameters written since): count and the seven fields plus shape. */
int pale_get_asset(pale_handle *h, pale_points *out);

/* One optimizer step of the training loop on the device
 * (python/training.py:685-743): the gradients of the last adjoint pass go
 * through the optimizer (python/optimizers.py:11-66, :301-337), opacities
 * are reset if asked (training.py:707-711), the parameters are projected
 * onto their constraints (verify_parameters_inplane, training.py:326-343)
 * and written back without a BVH rebuild, as apply_point_optimization.
 * Optimizer state (moments, step counts) lives on the device in BVH order
 * and starts over after every BVH build, as training.py:730-749 creates a
 * new optimizer after rebuild_bvh.  Enqueued on `stream` (NULL = the
 * default stream) without waiting. */
#define PALE_OPT_ADAM 0u          /* torch.optim.Adam                        */
#define PALE_OPT_SGD 1u           /* torch.optim.SGD, momentum (0.8)        */
#define PALE_OPT_MASKED_ADAM 2u   /* MaskedAdam (optimizers.py:70-214)     */
#define PALE_OPT_SURFEL_MASK 1u   /* flags: MaskedAdam updates only surfels
                                     with a nonzero gradient entry, each with
                                     its own step count
                                     (compute_surfel_update_mask)           */
typedef struct pale_optimizer {
    uint32_t type;            /* PALE_OPT_*                                 */
    uint32_t flags;
    double lr[6];             /* position, tangents, scale, albedo, opacity,
                                 beta (config.py:46-51 defaults)           */
    double beta1, beta2, eps; /* Adam (0.9, 0.999, 1e-8)                    */
    double momentum;          /* SGD (0.8)                                  */
    float opacity_reset;      /* >= 0: every opacity set to this value after
                                 the update; < 0: no reset                  */
    float reference_dir[3];   /* tangent-frame normals oriented towards this
                                 direction (+Z)                             */
} pale_optimizer;

/* d_grads: the seven DEVICE gradient fields in BVH order (count = the
 * point count; shape is ignored), e.g. the adjoint's gradients plus a
 * regulariser's, or NULL for the gradients of the last adjoint pass. */
int pale_optimizer_step(pale_handle *h, const pale_optimizer *opt,
                        const pale_points *d_grads, void *stream);

/* Drops the optimizer state: the next step starts from zero moments. */
int pale_optimizer_reset(pale_handle *h);

/* Density control on the renderer's asset (the parameter order of the last
 * apply / optimizer step), each followed by the BVH rebuild.
 *
 * pale_prune_by_opacity: compute_prune_indices_by_opacity
 * (python/density_control.py:199-263) + remove_points
 * (pale_bindings.cpp:1081-1189): with use_quantile the threshold is the
 * `min_opacity` quantile of the opacities (numpy's default linear method),
 * else min_opacity itself; surfels with opacity <= threshold are removed,
 * at most min(floor(max_fraction * N), N - min_keep) of them, the lowest
 * first (ties: lower index first; numpy's default argsort leaves ties in no
 * defined order).  *removed_count gets their number and, when not NULL,
 * removed[] (capacity: the point count) their indices in increasing order. */
int pale_prune_by_opacity(pale_handle *h, float min_opacity, uint32_t use_quantile,
                          double max_fraction, uint32_t min_keep,
                          uint32_t *removed_count, int64_t *removed);

/* pale_densify_long_axis_split: densify_points_long_axis_split
 * (density_control.py:6-196) + remove_points(parents) + add_points(children)
 * (pale_bindings.cpp:1081-1395).  Candidates have max(s_u, s_v) >=
 * min_long_axis_scale and, with an importance array (DEVICE pointer, one
 * score per surfel in asset order, may be NULL) and grad_threshold > 0, a
 * score >= grad_threshold.  With max_new_points >= 0 at most
 * max_new_points / 2 parents are split, the highest scores (importance,
 * else the long-axis scale; ties: lower index first); max_new_points < 0
 * sets no budget.  Each parent is replaced by two children offset by
 * +-split_distance * 3 * s_long along its long tangent, with scales
 * (s_long (1 - split_distance), s_short * minor_axis_shrink) and opacity
 * clamp(opacity * opacity_reduction, 0, 1): the survivors keep their order
 * and the children follow, parent by parent (+ then -).  *parent_count gets
 * the number of parents and parents_out[] (capacity: the point count, may be
 * NULL) their indices in increasing order. */
int pale_densify_long_axis_split(pale_handle *h, const float *d_importance,
                                 int64_t max_new_points, double split_distance,
                                 double minor_axis_shrink, double opacity_reduction,
                                 float min_long_axis_scale, float grad_threshold,
                                 uint32_t *parent_count, int64_t *parents_out);

/* Closest-hit queries against the scene (intersectScene in FirstHit mode,
 * IntersectionKernels.h:954-1097).  Host arrays of n rays; outputs:
 * instance (-1 = miss), primitive (surfel in BVH order or triangle id),
 * world t, alpha_geom, hit position (n*3). */
int pale_trace_rays(pale_handle *h, uint32_t n, const float *origins,
                    const float *directions, int32_t *instance,
                    int32_t *primitive, float *t, float *alpha_geom,
                    float *hit_position);

/* Transmittance queries (intersectScene in Transmit mode,
 * IntersectionKernels.h:1066-1090, with intersectBLASPointCloudTransmit,
 * :837-948): for n host rays, the closest mesh hit (instance, -1 = miss;
 * world t, FLT_MAX on a miss) and the surfel cloud's transmissivity
 * T = prod(1 - opacity * alpha_geom) over the successive surfel hits along
 * the ray (stopping once T <= 0.001). */
int pale_trace_transmittance(pale_handle *h, uint32_t n, const float *origins,
                             const float *directions, int32_t *instance,
                             float *t, float *transmissivity);

/* Irradiance lookups in the current photon map
 * (gatherDiffuseIrradianceAtPoint, KernelHelpers.h:990-1037). */
int pale_gather_irradiance(pale_handle *h, uint32_t n, const float *points,
                           const float *normals, float *irradiance);

/* Replaces the photon map by caller photons (n records: position 3,
 * power 3, incoming direction 3) and rebuilds the grid.  Used to check the
 * grid build and lookups on identical inputs. */
int pale_load_photons(pale_handle *h, uint32_t n, const float *position,
                      const float *power, const float *direction);

/* Copies the photon map out: count, and (each may be NULL) the photons in
 * deposit order, the per-photon cell ids in deposit order, and the sorted
 * order (sorted[i] = deposit index) plus the grid geometry
 * (origin xyz, cell size, resolution xyz as floats). */
int pale_get_photons(pale_handle *h, uint32_t *count, float *position,
                     float *power, float *direction, uint32_t *cell_id,
                     uint32_t *sorted, float *grid_info);

/* Exports the LBVH: Morton codes and sorted order of the last build
 * (codes[i] / order[i] for sorted position i), the node count, and the
 * traversal nodes (each 16 words: child0 box lo/hi, child1 box lo/hi,
 * child words).  Any pointer may be NULL. */
int pale_get_bvh(pale_handle *h, uint32_t *codes, uint32_t *node_count,
                 float *nodes, uint32_t max_nodes);

/* Counters of the last render. */
int pale_get_stats(pale_handle *h, pale_stats *stats);

/* Largest surfel count pale_build_lbvh_noalloc accepts. */
#define PALE_NOALLOC_MAX_SURFELS 16384u

/* Node count of the LBVH over n surfels with the given leaf size (0 is
 * taken as 1): 0 for n = 0, 1 when n <= leaf_size, else T + n - 1 with T
 * the number of top nodes the library stages in shared memory (256 unless
 * it was built with another -DPALE_TOP_NODES).  The size of the nodes
 * buffer pale_build_lbvh_noalloc needs, and pale_get_bvh's node_count.
 * Host only; no counterpart in the reference. */
uint32_t pale_lbvh_node_count(uint32_t n, uint32_t leaf_size);

/* LBVH build that allocates nothing.  No counterpart in the reference (its
 * BVH is built on the CPU); it serves callers that cannot allocate device
 * memory around the call: code running while a CUDA graph is captured
 * (cudaMalloc cannot be captured), host applications whose own allocator
 * owns all device memory, and loops that cannot afford cudaMalloc's
 * implicit device synchronisation.
 *
 * Inputs (device, asset order, n <= PALE_NOALLOC_MAX_SURFELS): position n*3,
 * tangent_u n*3, tangent_v n*3, scale n*2.  Outputs (device, caller owned):
 * codes[n] and order[n] by sorted position, nodes as 16 floats per node
 * (pale_lbvh_node_count(n, leaf_size) nodes), and optionally the error
 * flags in *d_status (0 = ok; also cleared to 0 when n = 0).  The result
 * equals the LBVH that pale_create / pale_rebuild build (see pale_get_bvh,
 * pale_get_order).
 *
 * Temporaries live in one fixed device array of 2,731,904 bytes (2.6 MiB)
 * that every GPU loading the library holds until exit.  The first call on
 * a device looks up that array's device address (cudaGetSymbolAddress), so
 * make the first call on each device outside any stream capture; the
 * address is kept for the life of the process, so do not call this entry
 * point after cudaDeviceReset.  All calls share the array: calls that
 * overlap on the GPU race.  Work is enqueued on `stream` (a cudaStream_t,
 * NULL = default stream) without synchronising.  Returns PALE_ERR_ARGUMENT
 * (with pale_last_error(NULL) text) when n is above the maximum. */
int pale_build_lbvh_noalloc(const float *d_position, const float *d_tangent_u,
                            const float *d_tangent_v, const float *d_scale,
                            uint32_t n, uint32_t leaf_size, uint32_t *d_codes,
                            uint32_t *d_order, float *d_nodes,
                            uint32_t *d_status, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* PALE_B200_H */
