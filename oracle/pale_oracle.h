/*
 * pale_oracle.h -- CPU oracle for the adjoint surfel renderer.
 *
 * TEST INFRASTRUCTURE ONLY.  This library restates, in plain C, the
 * algorithm of Pale's SYCL renderer (Pale/Renderer/Kernels/ sources and headers,
 * Pale/Renderer/SceneBuild.cpp, Pale/Renderer/BVH.ixx,
 * Pale/Renderer/PathTracer.cpp) with the reference's work-queue semantics
 * executed in sequential order: every queue slot is the rank of the item
 * among the survivors of the previous step, exactly what the reference's
 * atomic appends produce when its parallel_for bodies run one after the
 * other.  Only tests, the smoke check and the CPU-baseline leg of the
 * benchmark may load it; the product never does.
 *
 * Parity pinning: the reference ships no golden vectors.  The oracle is
 * pinned (a) by the reference's own gradient check (fd_test.py +
 * batch_fd_check.py with tests.json: finite differences of the L2 loss
 * agree with the adjoint opacity gradient within |err| <= 1e-4 or
 * rel <= 0.05 on the `empty` and `simple_1` scenes), reproduced in
 * tests/test_oracle_fd.py, and (b) by known-answer values of its RNG and
 * seed-stream building blocks (SplitMix64, Xorshift128, mt19937_64).
 *
 * The struct layouts are identical to the ones in include/pale_b200.h so
 * that one set of host arrays can drive both.
 */
#ifndef PALE_ORACLE_H
#define PALE_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_settings {
    uint32_t photons_per_launch, max_bounces, forward_passes, gather_passes;
    uint32_t adjoint_bounces, adjoint_passes;
    uint64_t seed;
    uint32_t random_number, rr_start;
    float q_null, q_reflect, q_transmit, gather_radius;
    uint32_t leaf_size, rng_mode, debug_images;
    float exposure, gamma;
    uint32_t null_weight;   /* 0 reference, 1 unbiased (divide by q_null) */
    uint32_t gradients;     /* 0 opacity, 1 all seven groups */
    uint32_t camera_seeds;  /* 0 by position in the selection, 1 by camera index */
    uint32_t gather_batch_paths, adjoint_batch_paths, walk_block;   /* GPU batching: unused here */
    uint32_t estimator;     /* 0 the reference's adjoint (photon-path events),
                               1 the derivative of the camera gather with the
                               photon map held (render_backward) */
} orc_settings;

typedef struct orc_points {
    uint32_t count;
    float *position, *tangent_u, *tangent_v, *scale, *albedo, *opacity, *beta, *shape;
} orc_points;

typedef struct orc_scene_desc {
    uint32_t num_vertices; const float *vertices;
    uint32_t num_triangles; const uint32_t *triangles;
    uint32_t num_meshes; const uint32_t *mesh_ranges;
    uint32_t num_materials; const float *materials;
    uint32_t num_instances; const uint32_t *instance_mesh; const uint32_t *instance_material;
    const float *instance_object_to_world; const float *instance_world_to_object;
    uint32_t num_cameras; const float *camera_inv_view; const float *camera_forward;
    const float *camera_fovy_deg; const uint32_t *camera_size; const char *camera_names;
    orc_points points;
} orc_scene_desc;

typedef struct orc_stats {
    uint64_t photon_segments, gather_segments, adjoint_segments, photons_stored;
    uint64_t gradient_events, gather_queries, node_visits, surfel_tests, photons_scanned;
    uint64_t gather_node_visits, gather_surfel_tests, gather_photons_scanned, kernel_launches;
    float forward_ms, backward_ms, photon_ms, gather_ms;
    float timed_ms[4];
    uint32_t timed_launches[4];
} orc_stats;

typedef struct orc_scene orc_scene;

/* bvh_kind: 0 = the reference's median-split BVH (BVH.ixx:49-133),
 *           1 = restatement of the product's Morton LBVH (bit-exact check). */
orc_scene *orc_create(const orc_scene_desc *desc, const orc_settings *st, int bvh_kind);
void orc_destroy(orc_scene *s);
void orc_set_threads(int n);
uint32_t orc_point_count(const orc_scene *s);
int orc_get_order(const orc_scene *s, uint32_t *order);
int orc_get_points(const orc_scene *s, orc_points *out);
int orc_apply_points(orc_scene *s, const orc_points *p);
int orc_rebuild(orc_scene *s, const orc_points *asset);
int orc_render_forward(orc_scene *s, uint32_t nsel, const uint32_t *cams, float *ldr, float *raw);
int orc_render_gather(orc_scene *s, uint32_t nsel, const uint32_t *cams, float *ldr, float *raw);
int orc_render_backward(orc_scene *s, uint32_t nsel, const uint32_t *cams, const float *dldi,
                        orc_points *grads, float *debug_opacity);
/* The same with a number of passes per selected camera (and for the
 * adjoint a number of bounces, 0 = the settings'), the views of a batched
 * render. */
int orc_render_forward_views(orc_scene *s, uint32_t nsel, const uint32_t *cams, const uint32_t *passes,
                             float *ldr, float *raw);
int orc_render_backward_views(orc_scene *s, uint32_t nsel, const uint32_t *cams, const uint32_t *passes,
                              const uint32_t *depths, const float *dldi, orc_points *grads);
int orc_trace_rays(orc_scene *s, uint32_t n, const float *o, const float *d, int32_t *inst,
                   int32_t *prim, float *t, float *alpha, float *hitpos);
int orc_trace_transmittance(orc_scene *s, uint32_t n, const float *o, const float *d, int32_t *inst, float *t,
                            float *transmit);
int orc_gather_irradiance(orc_scene *s, uint32_t n, const float *pts, const float *nrm, float *E);
int orc_load_photons(orc_scene *s, uint32_t n, const float *pos, const float *pw, const float *dir);
int orc_get_photons(orc_scene *s, uint32_t *count, float *pos, float *pw, float *dir,
                    uint32_t *cell_id, uint32_t *sorted, float *grid_info);
int orc_get_stats(const orc_scene *s, orc_stats *out);

/* The built scene as plain arrays, for the harness that runs the
 * reference's own kernel code on it (oracle/ref_driver.cpp).  Pointers
 * point into the scene and stay valid until the next rebuild.  Layouts:
 *   points: 19 floats per surfel in BVH order (position[3], tangent_u[3],
 *           tangent_v[3], scale[2], albedo[3], alpha_t, alpha_r, opacity,
 *           beta, shape) after the reference's collection (unit tangents,
 *           clamped albedo/opacity, alpha_r = 1, alpha_t = 0);
 *   nodes:  10 words per node of the median-split BVH (lo[3], hi[3] as
 *           floats; left, right as int32 (-1 for a leaf), first, count as
 *           uint32; children of a node are consecutive);
 *   lights: 8 words per light (mesh instance, first CDF entry, triangle
 *           count as uint32; color[3], power, world area as floats) with
 *           per-triangle inclusive CDF values and global triangle ids. */
typedef struct orc_export {
    uint32_t np; const float *points; const uint32_t *order;
    uint32_t nnodes; const void *nodes;
    uint32_t nv; const float *verts; uint32_t nt; const uint32_t *tris;
    uint32_t nm; const uint32_t *mranges; uint32_t nmat; const float *mats;
    uint32_t ninst; const uint32_t *inst_mesh, *inst_mat; const float *o2w, *w2o;
    uint32_t nlights; const void *lights; const float *tri_cdf; const uint32_t *tri_global;
    uint32_t ncam; const float *cam_inv_view, *cam_forward, *cam_fovy; const uint32_t *cam_size;
    const char *cam_names;
    float radius, cell[3], origin[3]; int32_t res[3]; uint32_t ncells;
    uint64_t photon_capacity;
} orc_export;
int orc_export_scene(const orc_scene *s, orc_export *e);

/* LBVH restatement on raw arrays (no scene): positions and per-surfel
 * boxes in BVH-input order -> Morton codes / order by sorted position and
 * 16-word traversal nodes.  Returns the node count. */
uint32_t orc_lbvh_build(uint32_t n, const float *positions, const float *aabb_lo,
                        const float *aabb_hi, uint32_t leaf_size, uint32_t top_nodes,
                        uint32_t *codes, uint32_t *order, float *nodes, uint32_t max_nodes);
/* Per-surfel beta AABB (SceneBuild.cpp:395-444) of already-collected points. */
void orc_surfel_aabbs(uint32_t n, const float *pos, const float *tu, const float *tv,
                      const float *scale, float *lo, float *hi);

/* RNG building blocks (KernelHelpers.h:10-116; SyclBridge.cpp:83). */
uint64_t orc_per_item_seed(uint64_t base, uint64_t id);
void orc_xorshift_floats(uint64_t seed, uint32_t n, float *out);
void orc_xorshift128_raw(uint32_t x, uint32_t y, uint32_t z, uint32_t w, uint32_t n, uint32_t *out);
void orc_mt19937_64(uint64_t seed, uint32_t n, uint64_t *out);

#ifdef __cplusplus
}
#endif
#endif
