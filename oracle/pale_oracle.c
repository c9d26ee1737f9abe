/*
 * pale_oracle.c -- CPU oracle of the adjoint surfel renderer.
 *
 * TEST INFRASTRUCTURE ONLY (see pale_oracle.h).  Every function cites the
 * reference file:line it restates.  Floating-point expressions keep the
 * reference's evaluation order (vector / scalar is a multiply by the
 * reciprocal, normalize() multiplies by 1/sqrt of the squared length,
 * GPUDataTypes.h:272-276, 322-328); build with -ffp-contract=off.
 *
 * Queue semantics: a bounce kernel of the reference appends survivors with
 * an atomic counter and keys its RNG by the queue slot
 * (PrimalKernels.cpp:80-82, AdjointKernels.cpp:99-101).  Here each bounce
 * first evaluates every slot (independently, so OpenMP may run them in
 * parallel) into a staging record, then compacts the staging records in
 * slot order: slot = rank among survivors, the order a sequential run of
 * the reference produces.
 */
#include "pale_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define M_PIf_ 3.14159265358979323846f
#define M_1_PIf_ 0.318309886183790671538f
#define INVALID_U32 0xFFFFFFFFu

/* ------------------------------------------------------------------ math */
typedef struct { float x, y, z; } v3;

static inline v3 V3(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static inline v3 vadd(v3 a, v3 b) { return V3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 vsub(v3 a, v3 b) { return V3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 vmul(v3 a, v3 b) { return V3(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline v3 vscale(v3 a, float s) { return V3(a.x * s, a.y * s, a.z * s); }
/* float3 / float multiplies by the reciprocal (GPUDataTypes.h:272-276). */
static inline v3 vdivs(v3 a, float s) { float inv = 1.f / s; return V3(a.x * inv, a.y * inv, a.z * inv); }
static inline v3 vneg(v3 a) { return V3(-a.x, -a.y, -a.z); }
static inline float vdot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 vcross(v3 a, v3 b) {
    return V3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline float vlen(v3 a) { return sqrtf(vdot(a, a)); }
/* normalize(): v * rsqrt(sum of squares) (GPUDataTypes.h:322-328). */
static inline v3 vnorm(v3 a) {
    float s = a.x * a.x + a.y * a.y + a.z * a.z;
    float inv = 1.0f / sqrtf(s);
    return vscale(a, inv);
}
static inline v3 vmin(v3 a, v3 b) { return V3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
static inline v3 vmax(v3 a, v3 b) { return V3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }
static inline float vsum(v3 a) { return a.x + a.y + a.z; }
static inline float vcomp(v3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
static inline v3 vload(const float *p) { return V3(p[0], p[1], p[2]); }
static inline void vstore(float *p, v3 a) { p[0] = a.x; p[1] = a.y; p[2] = a.z; }
static inline float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }

/* Matrix * (v, w): each output is sycl::dot(row, v) (GPUDataTypes.h:50-60). */
static inline void m4mul(const float *M, float x, float y, float z, float w, float *o) {
    for (int r = 0; r < 4; ++r)
        o[r] = M[4 * r + 0] * x + M[4 * r + 1] * y + M[4 * r + 2] * z + M[4 * r + 3] * w;
}
/* toWorldPoint / toObjectSpace origin: (M*(p,1)).xyz / w  (KernelHelpers.h:217-246). */
static inline v3 xform_point(const float *M, v3 p) {
    float h[4];
    m4mul(M, p.x, p.y, p.z, 1.f, h);
    return vdivs(V3(h[0], h[1], h[2]), h[3]);
}
/* transformDirection: normalize((M*(d,0)).xyz)  (KernelHelpers.h:237-241). */
static inline v3 xform_dir(const float *M, v3 d) {
    float h[4];
    m4mul(M, d.x, d.y, d.z, 0.f, h);
    return vnorm(V3(h[0], h[1], h[2]));
}

/* ------------------------------------------------------------------- RNG */
/* SplitMix64 / Xorshift128 / makePerItemSeed1D (KernelHelpers.h:12-115). */
static inline uint64_t splitmix_next(uint64_t *s) {
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
uint64_t orc_per_item_seed(uint64_t base, uint64_t id) {
    uint64_t mixed = base ^ (0x9E3779B97F4A7C15ull + id);
    return splitmix_next(&mixed);
}
typedef struct { uint32_t x, y, z, w; } rng_t;
static inline rng_t rng_make(uint64_t seed) {
    rng_t r;
    uint64_t s = seed;
    r.x = (uint32_t)splitmix_next(&s);
    r.y = (uint32_t)splitmix_next(&s);
    r.z = (uint32_t)splitmix_next(&s);
    r.w = (uint32_t)splitmix_next(&s);
    if (!(r.x | r.y | r.z | r.w)) r.w = 0xA511E9B3u;
    return r;
}
static inline uint32_t rng_u32(rng_t *r) {
    uint32_t t = r->x ^ (r->x << 11);
    r->x = r->y; r->y = r->z; r->z = r->w;
    r->w = (r->w ^ (r->w >> 19)) ^ (t ^ (t >> 8));
    return r->w;
}
static inline float rng_f(rng_t *r) { return (float)(rng_u32(r) >> 8) * 0x1.0p-24f; }
void orc_xorshift_floats(uint64_t seed, uint32_t n, float *out) {
    rng_t r = rng_make(seed);
    for (uint32_t i = 0; i < n; ++i) out[i] = rng_f(&r);
}
/* Xorshift128 from an explicit state (the four-word constructor,
 * KernelHelpers.h:76-81). */
void orc_xorshift128_raw(uint32_t x, uint32_t y, uint32_t z, uint32_t w, uint32_t n, uint32_t *out) {
    rng_t r;
    r.x = x ? x : 0x1u;
    r.y = y ? y : 0x9E3779B9u;
    r.z = z ? z : 0x7F4A7C15u;
    r.w = w ? w : 0x94D049BBu;
    for (uint32_t i = 0; i < n; ++i) out[i] = rng_u32(&r);
}

/* mt19937_64 (Matsumoto & Nishimura 2004), the host seed stream of
 * SyclBridge.cpp:83,170 (std::mt19937_64). */
typedef struct { uint64_t mt[312]; int idx; } mt64_t;
static void mt_seed(mt64_t *m, uint64_t seed) {
    m->mt[0] = seed;
    for (int i = 1; i < 312; ++i)
        m->mt[i] = 6364136223846793005ull * (m->mt[i - 1] ^ (m->mt[i - 1] >> 62)) + (uint64_t)i;
    m->idx = 312;
}
static uint64_t mt_next(mt64_t *m) {
    if (m->idx >= 312) {
        for (int i = 0; i < 312; ++i) {
            uint64_t x = (m->mt[i] & 0xFFFFFFFF80000000ull) | (m->mt[(i + 1) % 312] & 0x7FFFFFFFull);
            uint64_t xa = x >> 1;
            if (x & 1ull) xa ^= 0xB5026F5AA96619E9ull;
            m->mt[i] = m->mt[(i + 156) % 312] ^ xa;
        }
        m->idx = 0;
    }
    uint64_t x = m->mt[m->idx++];
    x ^= (x >> 29) & 0x5555555555555555ull;
    x ^= (x << 17) & 0x71D67FFFEDA60000ull;
    x ^= (x << 37) & 0xFFF7EEE000000000ull;
    x ^= (x >> 43);
    return x;
}
void orc_mt19937_64(uint64_t seed, uint32_t n, uint64_t *out) {
    mt64_t m;
    mt_seed(&m, seed);
    for (uint32_t i = 0; i < n; ++i) out[i] = mt_next(&m);
}

/* ----------------------------------------------------------------- scene */
typedef struct {
    v3 p, tu, tv;
    float su, sv;
    v3 albedo;
    float alpha_t, alpha_r, opacity, beta, shape;
} point_t;   /* Point (GPUDataStructures.h:36-49) */

typedef struct { v3 lo, hi; int32_t left, right; uint32_t first, count; } node_t;

typedef struct { v3 pos, power, dir; } photon_t;   /* DevicePhotonSurface (:430-442) */

typedef struct {
    uint32_t mesh_instance;     /* index into mesh instances              */
    uint32_t tri_offset, tri_count;
    v3 color;
    float power, area;
} light_t;                      /* GPULightRecord (:149-159) */

typedef struct { v3 o, d, n, thr; uint32_t bounce, pixel, path; } ray_t;   /* RayState */

typedef struct {
    int hit;
    int inst;                   /* -1 miss; ninst = the surfel cloud */
    uint32_t prim;
    float t, alpha;
    v3 pos, normal;
} hit_t;                        /* WorldHit (:280-293) */

enum { PK_NONE = 0, PK_NULL = 1, PK_REFLECT = 2, PK_TRANSMIT = 3, PK_PROJECTION = 4 };

typedef struct { int kind; uint32_t prim, inst; float alpha; v3 pos, thr; uint32_t pixel; } pending_t;

typedef struct {
    int kind;
    uint32_t prim, inst;        /* surfel / pending instance             */
    float alpha;
    v3 pos, normal, thr;
    uint32_t pixel;
    int end_type;               /* 0 mesh, 1 surfel                      */
    uint32_t end_inst, end_prim;
    float end_alpha, end_pdf, end_cos;
    v3 end_pos, end_normal;
    v3 tpos, tdir;              /* hit on the target surfel, unit direction */
} event_t;                      /* CompletedGradientEvent (:338-369) */

struct orc_scene {
    orc_settings st;
    int bvh_kind;
    /* seed stream position after the last photon pass: where the camera
     * seeds of a gather-only render start */
    mt64_t cam_mt;
    int cam_mt_valid;
    /* meshes */
    uint32_t nv, nt, nm, nmat, ninst, ncam;
    float *verts; uint32_t *tris; uint32_t *mranges; float *mats;
    uint32_t *inst_mesh, *inst_mat; float *o2w, *w2o;
    v3 *inst_lo, *inst_hi;
    /* lights */
    uint32_t nlights; light_t *lights; float *tri_cdf; uint32_t *tri_global;
    /* cameras */
    float *cam_inv_view, *cam_forward, *cam_fovy; uint32_t *cam_size; char *cam_names;
    /* surfels in BVH order */
    uint32_t np; point_t *pts; uint32_t *order;
    node_t *nodes; uint32_t nnodes;
    v3 pc_lo, pc_hi; int has_pc;
    /* photon map */
    int grid_ready;
    float r; v3 cell, origin; int res[3]; uint32_t ncells;
    uint64_t cap; uint32_t attempts, stored;
    photon_t *ph; uint32_t *ph_cell; uint32_t *sorted; uint32_t *cell_off;
    photon_t *ph_sorted;
    /* queues */
    uint32_t qcap;
    orc_stats stats;
};

static int g_threads = 0;
void orc_set_threads(int n) { g_threads = n; }
static void apply_threads(void) {
#ifdef _OPENMP
    if (g_threads > 0) omp_set_num_threads(g_threads);
#endif
}

static double now_ms(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec * 1e3 + ts.tv_nsec * 1e-6;
}

static void *xdup(const void *src, size_t bytes) {
    void *p = malloc(bytes ? bytes : 1);
    if (src && bytes) memcpy(p, src, bytes);
    return p;
}

/* Surfel collection: normalize tangents, clamp albedo/opacity/shape,
 * alpha_r = 1, alpha_t = 0 (SceneBuild.cpp:203-215). */
static point_t collect_point(const orc_points *a, uint32_t i) {
    point_t q;
    q.p = vload(a->position + 3 * i);
    q.tu = vnorm(vload(a->tangent_u + 3 * i));
    q.tv = vnorm(vload(a->tangent_v + 3 * i));
    q.su = a->scale[2 * i];
    q.sv = a->scale[2 * i + 1];
    v3 al = vload(a->albedo + 3 * i);
    q.albedo = V3(clampf(al.x, 0.f, 1.f), clampf(al.y, 0.f, 1.f), clampf(al.z, 0.f, 1.f));
    q.opacity = clampf(a->opacity[i], 0.f, 1.f);
    q.alpha_r = 1.0f;
    q.alpha_t = 0.0f;
    q.beta = a->beta[i];
    q.shape = a->shape ? clampf(a->shape[i], -5.f, 5.f) : 0.f;
    return q;
}

/* surfelObjectAabbBeta (SceneBuild.cpp:395-444). */
static void surfel_aabb(v3 p, v3 tanU, v3 tanV, float su, float sv, v3 *lo, v3 *hi) {
    v3 tU = vnorm(tanU), tV = vnorm(tanV);
    v3 n = vnorm(vcross(tU, tV));
    float rU = 1.0001f * su, rV = 1.0001f * sv;
    float e[3];
    for (int a = 0; a < 3; ++a) {
        float cu = rU * vcomp(tU, a), cv = rV * vcomp(tV, a);
        float proj = sqrtf(cu * cu + cv * cv);
        e[a] = proj + 0.001f * fabsf(vcomp(n, a));
    }
    v3 ext = V3(e[0], e[1], e[2]);
    *lo = vsub(p, ext);
    *hi = vadd(p, ext);
}

void orc_surfel_aabbs(uint32_t n, const float *pos, const float *tu, const float *tv,
                      const float *scale, float *lo, float *hi) {
    for (uint32_t i = 0; i < n; ++i) {
        v3 l, h;
        surfel_aabb(vload(pos + 3 * i), vload(tu + 3 * i), vload(tv + 3 * i), scale[2 * i],
                    scale[2 * i + 1], &l, &h);
        vstore(lo + 3 * i, l);
        vstore(hi + 3 * i, h);
    }
}

/* ------------------------------------------- reference median-split BVH */
/* BasicBVH::buildFromBoxes / subdivideBoxes (BVH.ixx:49-133): median split
 * on centroids along the longest node axis, leaf when count <= leafSize.
 * std::nth_element leaves equal keys in an implementation-defined order;
 * here the range is sorted by (centroid, index), one valid outcome. */
static const float *g_sort_cent;
static int g_sort_axis;
static int cmp_axis(const void *a, const void *b) {
    uint32_t ia = *(const uint32_t *)a, ib = *(const uint32_t *)b;
    float ca = g_sort_cent[3 * ia + g_sort_axis], cb = g_sort_cent[3 * ib + g_sort_axis];
    if (ca < cb) return -1;
    if (ca > cb) return 1;
    return (ia < ib) ? -1 : (ia > ib);
}
typedef struct { node_t *v; uint32_t n, cap; } nodevec;
static uint32_t nv_push(nodevec *nv) {
    if (nv->n == nv->cap) {
        nv->cap = nv->cap ? 2 * nv->cap : 64;
        nv->v = (node_t *)realloc(nv->v, nv->cap * sizeof(node_t));
    }
    memset(&nv->v[nv->n], 0, sizeof(node_t));
    return nv->n++;
}
static void median_fit(node_t *nd, const uint32_t *ord, const v3 *lo, const v3 *hi) {
    v3 bl = V3(INFINITY, INFINITY, INFINITY), bh = V3(-INFINITY, -INFINITY, -INFINITY);
    for (uint32_t i = 0; i < nd->count; ++i) {
        uint32_t k = ord[nd->first + i];
        bl = vmin(bl, lo[k]);
        bh = vmax(bh, hi[k]);
    }
    nd->lo = bl;
    nd->hi = bh;
}
static void median_subdivide(nodevec *nv, uint32_t ni, uint32_t *ord, const float *cent,
                             const v3 *lo, const v3 *hi, uint32_t leaf) {
    node_t nd = nv->v[ni];
    if (nd.count <= leaf) return;
    v3 ext = vsub(nd.hi, nd.lo);
    int axis = (ext.y > ext.x && ext.y > ext.z) ? 1 : ((ext.z > ext.x && ext.z > ext.y) ? 2 : 0);
    g_sort_cent = cent;
    g_sort_axis = axis;
    qsort(ord + nd.first, nd.count, sizeof(uint32_t), cmp_axis);
    uint32_t leftCount = nd.count >> 1;
    if (leftCount == 0 || leftCount == nd.count) return;
    uint32_t l = nv_push(nv), r = nv_push(nv);
    nv->v[l].first = nd.first; nv->v[l].count = leftCount;
    nv->v[r].first = nd.first + leftCount; nv->v[r].count = nd.count - leftCount;
    nv->v[l].left = nv->v[l].right = -1;
    nv->v[r].left = nv->v[r].right = -1;
    nv->v[ni].left = (int32_t)l;
    nv->v[ni].right = (int32_t)r;
    nv->v[ni].count = 0;
    median_fit(&nv->v[l], ord, lo, hi);
    median_fit(&nv->v[r], ord, lo, hi);
    median_subdivide(nv, l, ord, cent, lo, hi, leaf);
    median_subdivide(nv, r, ord, cent, lo, hi, leaf);
}

/* --------------------------------------------- LBVH restatement (product) */
/* expandBits / Morton code as in Karras, "Maximizing parallelism in the
 * construction of BVHs, octrees and k-d trees" (HPG 2012). */
static inline uint32_t expand_bits(uint32_t v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}
static inline uint32_t quantize(float c, float lo, float ext) {
    float f = (ext > 0.f) ? (c - lo) / ext : 0.f;
    float q = f * 1024.0f;
    if (!(q > 0.f)) return 0u;
    if (q >= 1023.f) return 1023u;
    return (uint32_t)q;
}
static inline int clz64(uint64_t x) { return x ? __builtin_clzll(x) : 64; }
static inline int delta_key(const uint64_t *k, uint32_t n, int64_t i, int64_t j) {
    if (j < 0 || j >= (int64_t)n) return -1;
    return clz64(k[i] ^ k[j]);
}

#define LEAF_FLAG 0x80000000u
#define EMPTY_CHILD 0xFFFFFFFFu
static inline uint32_t leaf_word(uint32_t first, uint32_t count) {
    return LEAF_FLAG | ((count - 1u) << 28) | first;
}

uint32_t orc_lbvh_build(uint32_t n, const float *positions, const float *aabb_lo,
                        const float *aabb_hi, uint32_t leaf_size, uint32_t top_nodes,
                        uint32_t *codes_out, uint32_t *order_out, float *nodes_out,
                        uint32_t max_nodes) {
    if (n == 0) return 0;
    if (leaf_size < 1) leaf_size = 1;
    if (leaf_size > 8) leaf_size = 8;
    /* scene bounds of the centroids */
    v3 lo = V3(INFINITY, INFINITY, INFINITY), hi = V3(-INFINITY, -INFINITY, -INFINITY);
    for (uint32_t i = 0; i < n; ++i) {
        v3 p = vload(positions + 3 * i);
        lo = vmin(lo, p);
        hi = vmax(hi, p);
    }
    v3 ext = vsub(hi, lo);
    uint32_t *code = (uint32_t *)malloc(n * sizeof(uint32_t));
    for (uint32_t i = 0; i < n; ++i) {
        v3 p = vload(positions + 3 * i);
        code[i] = (expand_bits(quantize(p.x, lo.x, ext.x)) << 2) |
                  (expand_bits(quantize(p.y, lo.y, ext.y)) << 1) |
                  expand_bits(quantize(p.z, lo.z, ext.z));
    }
    /* stable LSD radix sort of (code, index), 8-bit digits */
    uint32_t *ord = (uint32_t *)malloc(n * sizeof(uint32_t));
    uint32_t *tmp = (uint32_t *)malloc(n * sizeof(uint32_t));
    for (uint32_t i = 0; i < n; ++i) ord[i] = i;
    for (int pass = 0; pass < 4; ++pass) {
        uint32_t cnt[257];
        memset(cnt, 0, sizeof(cnt));
        int sh = 8 * pass;
        for (uint32_t i = 0; i < n; ++i) cnt[((code[ord[i]] >> sh) & 255u) + 1]++;
        for (int b = 0; b < 256; ++b) cnt[b + 1] += cnt[b];
        for (uint32_t i = 0; i < n; ++i) tmp[cnt[(code[ord[i]] >> sh) & 255u]++] = ord[i];
        uint32_t *t = ord; ord = tmp; tmp = t;
    }
    uint64_t *key = (uint64_t *)malloc(n * sizeof(uint64_t));
    for (uint32_t i = 0; i < n; ++i) {
        key[i] = ((uint64_t)code[ord[i]] << 32) | i;
        if (codes_out) codes_out[i] = code[ord[i]];
        if (order_out) order_out[i] = ord[i];
    }
    uint32_t nodes_written = 0;
    uint32_t T = top_nodes;
    if (n <= leaf_size) {
        /* single leaf under one root node */
        v3 bl = V3(INFINITY, INFINITY, INFINITY), bh = V3(-INFINITY, -INFINITY, -INFINITY);
        for (uint32_t i = 0; i < n; ++i) {
            bl = vmin(bl, vload(aabb_lo + 3 * ord[i]));
            bh = vmax(bh, vload(aabb_hi + 3 * ord[i]));
        }
        if (nodes_out && max_nodes >= 1) {
            float *w = nodes_out;
            memset(w, 0, 16 * sizeof(float));
            w[0] = bl.x; w[1] = bl.y; w[2] = bl.z; w[3] = bh.x; w[4] = bh.y; w[5] = bh.z;
            w[6] = INFINITY; w[7] = INFINITY; w[8] = INFINITY;
            w[9] = -INFINITY; w[10] = -INFINITY; w[11] = -INFINITY;
            uint32_t c0 = leaf_word(0, n), c1 = EMPTY_CHILD;
            memcpy(&w[12], &c0, 4);
            memcpy(&w[13], &c1, 4);
        }
        nodes_written = 1;
        goto done;
    }
    {
        uint32_t ni = n - 1;
        int32_t *lc = (int32_t *)malloc(ni * sizeof(int32_t));  /* >=0 internal, <0: -(leaf+1) */
        int32_t *rc = (int32_t *)malloc(ni * sizeof(int32_t));
        uint32_t *rfirst = (uint32_t *)malloc(ni * sizeof(uint32_t));
        uint32_t *rlast = (uint32_t *)malloc(ni * sizeof(uint32_t));
        for (int64_t i = 0; i < (int64_t)ni; ++i) {
            int d = (delta_key(key, n, i, i + 1) - delta_key(key, n, i, i - 1)) >= 0 ? 1 : -1;
            int dmin = delta_key(key, n, i, i - d);
            int64_t lmax = 2;
            while (delta_key(key, n, i, i + lmax * d) > dmin) lmax *= 2;
            int64_t l = 0;
            for (int64_t t = lmax / 2; t >= 1; t /= 2)
                if (delta_key(key, n, i, i + (l + t) * d) > dmin) l += t;
            int64_t j = i + l * d;
            int dnode = delta_key(key, n, i, j);
            int64_t s = 0;
            int64_t div = 2;
            int64_t t = (l + div - 1) / div;
            while (1) {
                if (delta_key(key, n, i, i + (s + t) * d) > dnode) s += t;
                if (t == 1) break;
                div *= 2;
                t = (l + div - 1) / div;
            }
            int64_t gamma = i + s * d + (d < 0 ? d : 0);
            int64_t mn = i < j ? i : j, mx = i < j ? j : i;
            lc[i] = (mn == gamma) ? -(int32_t)(gamma + 1) : (int32_t)gamma;
            rc[i] = (mx == gamma + 1) ? -(int32_t)(gamma + 2) : (int32_t)(gamma + 1);
            rfirst[i] = (uint32_t)mn;
            rlast[i] = (uint32_t)mx;
        }
        /* bottom-up boxes (post-order; min/max are exact so any order agrees) */
        v3 *blo = (v3 *)malloc(ni * sizeof(v3));
        v3 *bhi = (v3 *)malloc(ni * sizeof(v3));
        uint32_t *stack = (uint32_t *)malloc(2 * ni * sizeof(uint32_t) + 16);
        uint8_t *state = (uint8_t *)calloc(ni, 1);
        int sp = 0;
        stack[sp++] = 0;
        while (sp) {
            uint32_t x = stack[sp - 1];
            if (!state[x]) {
                state[x] = 1;
                if (lc[x] >= 0) stack[sp++] = (uint32_t)lc[x];
                if (rc[x] >= 0) stack[sp++] = (uint32_t)rc[x];
                continue;
            }
            --sp;
            v3 l0, h0, l1, h1;
            if (lc[x] >= 0) { l0 = blo[lc[x]]; h0 = bhi[lc[x]]; }
            else { uint32_t p = ord[-lc[x] - 1]; l0 = vload(aabb_lo + 3 * p); h0 = vload(aabb_hi + 3 * p); }
            if (rc[x] >= 0) { l1 = blo[rc[x]]; h1 = bhi[rc[x]]; }
            else { uint32_t p = ord[-rc[x] - 1]; l1 = vload(aabb_lo + 3 * p); h1 = vload(aabb_hi + 3 * p); }
            blo[x] = vmin(l0, l1);
            bhi[x] = vmax(h0, h1);
        }
        /* top BFS copies, then all Karras nodes */
        int32_t *topmap = (int32_t *)malloc(ni * sizeof(int32_t));
        for (uint32_t i = 0; i < ni; ++i) topmap[i] = -1;
        uint32_t *topsrc = (uint32_t *)malloc((T + 1) * sizeof(uint32_t));
        uint32_t ntop = 0, head = 0;
        if (T > 0) { topsrc[ntop] = 0; topmap[0] = (int32_t)ntop; ntop++; }
        while (head < ntop) {
            uint32_t x = topsrc[head++];
            int32_t ch[2] = {lc[x], rc[x]};
            for (int c = 0; c < 2; ++c) {
                if (ch[c] < 0) continue;
                uint32_t y = (uint32_t)ch[c];
                if (rlast[y] - rfirst[y] + 1u <= leaf_size) continue;
                if (ntop >= T) continue;
                topmap[y] = (int32_t)ntop;
                topsrc[ntop++] = y;
            }
        }
        uint32_t total = T + ni;
        nodes_written = total;
        if (nodes_out) {
            for (uint32_t slot = 0; slot < total && slot < max_nodes; ++slot) {
                int is_top = slot < T;
                if (is_top && slot >= ntop) { memset(nodes_out + 16 * slot, 0, 64); continue; }
                uint32_t x = is_top ? topsrc[slot] : slot - T;
                float *w = nodes_out + 16 * slot;
                memset(w, 0, 16 * sizeof(float));
                int32_t ch[2] = {lc[x], rc[x]};
                for (int c = 0; c < 2; ++c) {
                    v3 bl, bh;
                    uint32_t word;
                    if (ch[c] < 0) {
                        uint32_t sp_ = (uint32_t)(-ch[c] - 1);
                        uint32_t p = ord[sp_];
                        bl = vload(aabb_lo + 3 * p);
                        bh = vload(aabb_hi + 3 * p);
                        word = leaf_word(sp_, 1);
                    } else {
                        uint32_t y = (uint32_t)ch[c];
                        bl = blo[y];
                        bh = bhi[y];
                        uint32_t cnt = rlast[y] - rfirst[y] + 1u;
                        if (cnt <= leaf_size) word = leaf_word(rfirst[y], cnt);
                        else if (is_top && topmap[y] >= 0) word = (uint32_t)topmap[y];
                        else word = T + y;
                    }
                    w[6 * c + 0] = bl.x; w[6 * c + 1] = bl.y; w[6 * c + 2] = bl.z;
                    w[6 * c + 3] = bh.x; w[6 * c + 4] = bh.y; w[6 * c + 5] = bh.z;
                    memcpy(&w[12 + c], &word, 4);
                }
            }
        }
        free(lc); free(rc); free(rfirst); free(rlast); free(blo); free(bhi);
        free(stack); free(state); free(topmap); free(topsrc);
    }
done:
    free(code); free(ord); free(tmp); free(key);
    return nodes_written;
}

/* Converts 16-word LBVH nodes into generic oracle nodes for traversal. */
static void lbvh_to_nodes(orc_scene *s, const float *w, uint32_t count) {
    /* generic node per 16-word node: the node's own box is the union of the
     * children; children are either other nodes or leaf ranges, which become
     * extra leaf nodes. */
    nodevec nv = {0};
    uint32_t *map = (uint32_t *)malloc(count * sizeof(uint32_t));
    for (uint32_t i = 0; i < count; ++i) map[i] = nv_push(&nv);
    for (uint32_t i = 0; i < count; ++i) {
        const float *x = w + 16 * i;
        uint32_t words[2];
        memcpy(&words[0], &x[12], 4);
        memcpy(&words[1], &x[13], 4);
        int32_t kids[2] = {-1, -1};
        for (int c = 0; c < 2; ++c) {
            if (words[c] == EMPTY_CHILD) continue;
            v3 bl = V3(x[6 * c], x[6 * c + 1], x[6 * c + 2]);
            v3 bh = V3(x[6 * c + 3], x[6 * c + 4], x[6 * c + 5]);
            if (words[c] & LEAF_FLAG) {
                uint32_t k = nv_push(&nv);
                nv.v[k].lo = bl; nv.v[k].hi = bh;
                nv.v[k].first = words[c] & 0x0FFFFFFFu;
                nv.v[k].count = ((words[c] >> 28) & 7u) + 1u;
                nv.v[k].left = nv.v[k].right = -1;
                kids[c] = (int32_t)k;
            } else {
                kids[c] = (int32_t)map[words[c]];
                nv.v[map[words[c]]].lo = bl;
                nv.v[map[words[c]]].hi = bh;
            }
        }
        nv.v[map[i]].left = kids[0];
        nv.v[map[i]].right = kids[1];
        nv.v[map[i]].count = 0;
    }
    /* root box = union of its children */
    if (count) {
        node_t *r = &nv.v[map[0]];
        v3 bl = V3(INFINITY, INFINITY, INFINITY), bh = V3(-INFINITY, -INFINITY, -INFINITY);
        if (r->left >= 0) { bl = vmin(bl, nv.v[r->left].lo); bh = vmax(bh, nv.v[r->left].hi); }
        if (r->right >= 0) { bl = vmin(bl, nv.v[r->right].lo); bh = vmax(bh, nv.v[r->right].hi); }
        r->lo = bl; r->hi = bh;
    }
    free(map);
    s->nodes = nv.v;
    s->nnodes = nv.n;
}

/* Builds the surfel BVH and the BVH-ordered point array from asset points
 * (buildPointCloudBLAS + reorder, SceneBuild.cpp:476-512, 710-761). */
static void build_points(orc_scene *s, const orc_points *a) {
    free(s->pts); free(s->order); free(s->nodes);
    s->pts = NULL; s->order = NULL; s->nodes = NULL; s->nnodes = 0;
    s->np = a ? a->count : 0;
    s->has_pc = s->np > 0;
    if (!s->np) return;
    point_t *col = (point_t *)malloc(s->np * sizeof(point_t));
    v3 *lo = (v3 *)malloc(s->np * sizeof(v3)), *hi = (v3 *)malloc(s->np * sizeof(v3));
    float *cent = (float *)malloc(3 * s->np * sizeof(float));
    for (uint32_t i = 0; i < s->np; ++i) {
        col[i] = collect_point(a, i);
        surfel_aabb(col[i].p, col[i].tu, col[i].tv, col[i].su, col[i].sv, &lo[i], &hi[i]);
        vstore(cent + 3 * i, col[i].p);
    }
    s->order = (uint32_t *)malloc(s->np * sizeof(uint32_t));
    /* the reference's median split always uses BuildOptions' leaf size 4
     * (SceneBuild.ixx:72-75); the LBVH restatement uses the settings' leaf
     * size, as the CUDA build does */
    uint32_t leaf = s->bvh_kind == 0 ? 4u : (s->st.leaf_size ? s->st.leaf_size : 1u);
    if (s->bvh_kind == 0) {
        nodevec nv = {0};
        for (uint32_t i = 0; i < s->np; ++i) s->order[i] = i;
        uint32_t root = nv_push(&nv);
        nv.v[root].first = 0; nv.v[root].count = s->np; nv.v[root].left = nv.v[root].right = -1;
        median_fit(&nv.v[root], s->order, lo, hi);
        median_subdivide(&nv, root, s->order, cent, lo, hi, leaf);
        s->nodes = nv.v;
        s->nnodes = nv.n;
    } else {
        float *flo = (float *)malloc(3 * s->np * sizeof(float)), *fhi = (float *)malloc(3 * s->np * sizeof(float));
        for (uint32_t i = 0; i < s->np; ++i) { vstore(flo + 3 * i, lo[i]); vstore(fhi + 3 * i, hi[i]); }
        uint32_t cnt = orc_lbvh_build(s->np, cent, flo, fhi, leaf, 0, NULL, s->order, NULL, 0);
        float *w = (float *)malloc((size_t)cnt * 16 * sizeof(float));
        orc_lbvh_build(s->np, cent, flo, fhi, leaf, 0, NULL, NULL, w, cnt);
        lbvh_to_nodes(s, w, cnt);
        free(w); free(flo); free(fhi);
    }
    s->pts = (point_t *)malloc(s->np * sizeof(point_t));
    s->pc_lo = V3(INFINITY, INFINITY, INFINITY);
    s->pc_hi = V3(-INFINITY, -INFINITY, -INFINITY);
    for (uint32_t i = 0; i < s->np; ++i) {
        s->pts[i] = col[s->order[i]];
        s->pc_lo = vmin(s->pc_lo, lo[i]);
        s->pc_hi = vmax(s->pc_hi, hi[i]);
    }
    free(col); free(lo); free(hi); free(cent);
}

/* ----------------------------------------------------------- intersection */
/* safeInvDir (KernelHelpers.h:140-148). */
static inline v3 safe_inv(v3 d) {
    return V3(fabsf(d.x) < 1e-6f ? 1e30f : 1.f / d.x, fabsf(d.y) < 1e-6f ? 1e30f : 1.f / d.y,
              fabsf(d.z) < 1e-6f ? 1e30f : 1.f / d.z);
}
/* slabIntersectAABB (KernelHelpers.h:150-214). */
static inline int slab(v3 o, v3 inv, v3 lo, v3 hi, float tmax_limit, float *tentry, float clamp) {
    v3 t0 = vmul(vsub(lo, o), inv), t1 = vmul(vsub(hi, o), inv);
    float tmin = fmaxf(fmaxf(fminf(t0.x, t1.x), fminf(t0.y, t1.y)), fminf(t0.z, t1.z));
    float tmax = fminf(fminf(fmaxf(t0.x, t1.x), fmaxf(t0.y, t1.y)), fmaxf(t0.z, t1.z));
    if (tmin > tmax) return 0;
    if (tmax < 0.0f) return 0;
    if (tmin > tmax_limit) return 0;
    *tentry = fmaxf(tmin, clamp);
    return 1;
}
/* intersectTriangle (KernelHelpers.h:248-277). */
static inline int tri_hit(v3 o, v3 d, v3 v0, v3 v1, v3 v2, float *t_out, float tmin) {
    v3 e1 = vsub(v1, v0), e2 = vsub(v2, v0);
    v3 h = vcross(d, e2);
    float a = vdot(e1, h);
    if (fabsf(a) < 1.0e-4f) return 0;
    float f = 1.0f / a;
    v3 s = vsub(o, v0);
    float u = f * vdot(s, h);
    if (u < 0.0f || u > 1.0f) return 0;
    v3 q = vcross(s, e1);
    float v = f * vdot(d, q);
    if (v < 0.0f || u + v > 1.0f) return 0;
    float t = f * vdot(e2, q);
    if (t <= tmin) return 0;
    *t_out = t;
    return 1;
}
/* intersectSurfel + opacityBeta + phiInverse (KernelHelpers.h:506-669). */
static inline int surfel_hit(v3 o, v3 d, const point_t *sf, float tmin, float tmax, float *t_out,
                             v3 *x_out, float *alpha_out) {
    v3 uT = vnorm(sf->tu);
    v3 vT = vnorm(vsub(sf->tv, vscale(uT, vdot(uT, sf->tv))));
    v3 n = vnorm(vcross(uT, vT));
    float nd = vdot(n, d);
    if (fabsf(nd) < 1e-6f) return 0;
    float th = vdot(n, vsub(sf->p, o)) / nd;
    if (th <= tmin || th >= tmax) return 0;
    v3 x = vadd(o, vscale(d, th));
    v3 r = vsub(x, sf->p);
    float u = vdot(sf->tu, r) / sf->su;
    float v = vdot(sf->tv, r) / sf->sv;
    float r2 = u * u + v * v;
    if (r2 >= 1.0f) return 0;
    float base = 1.0f - r2;
    float ex = 4.0f * expf(sf->beta);
    *alpha_out = powf(base, ex);
    *t_out = th;
    *x_out = x;
    return 1;
}

typedef struct { uint64_t nodes, tests; } trav_ctr;

/* intersectBLASPointCloudFirstHit (IntersectionKernels.h:585-675): the
 * closest surfel with t in (tmin, inf); tmin is 1e-5 (rayEpsilon) except
 * in the transmittance walk below. */
static int blas_firsthit_from(const orc_scene *s, v3 o, v3 d, float tmin, uint32_t *prim, float *t, v3 *x,
                              float *alpha, trav_ctr *ctr) {
    if (!s->nnodes) return 0;
    v3 inv = safe_inv(d);
    float best = INFINITY;
    int hit = 0;
    int32_t stack[512];
    int sp = 0;
    stack[sp++] = 0;
    while (sp) {
        const node_t *nd = &s->nodes[stack[--sp]];
        float te;
        if (!slab(o, inv, nd->lo, nd->hi, best, &te, 1e-6f)) continue;
        if (ctr) ctr->nodes++;
        if (nd->count == 0) {
            int32_t L = nd->left, R = nd->right;
            float tl = INFINITY, tr = INFINITY;
            int hl = L >= 0 && slab(o, inv, s->nodes[L].lo, s->nodes[L].hi, best, &tl, 1e-6f);
            int hr = R >= 0 && slab(o, inv, s->nodes[R].lo, s->nodes[R].hi, best, &tr, 1e-6f);
            if (hl && hr) {
                if (tl <= tr) { stack[sp++] = R; stack[sp++] = L; }
                else { stack[sp++] = L; stack[sp++] = R; }
            } else if (hl) stack[sp++] = L;
            else if (hr) stack[sp++] = R;
            if (sp > 500) sp = 500;
            continue;
        }
        for (uint32_t k = 0; k < nd->count; ++k) {
            uint32_t idx = nd->first + k;
            float th, a;
            v3 xx;
            if (ctr) ctr->tests++;
            if (!surfel_hit(o, d, &s->pts[idx], tmin, best, &th, &xx, &a)) continue;
            hit = 1;
            best = th;
            *prim = idx;
            *x = xx;
            *alpha = a;
        }
    }
    if (hit) *t = best;
    return hit;
}

static int blas_firsthit(const orc_scene *s, v3 o, v3 d, uint32_t *prim, float *t, v3 *x,
                         float *alpha, trav_ctr *ctr) {
    return blas_firsthit_from(s, o, d, 1e-5f, prim, t, x, alpha, ctr);
}

/* intersectBLASPointCloudTransmit (IntersectionKernels.h:837-948): walks the
 * successive closest surfels along the whole ray from the same origin
 * (t in (tMin, inf), tMin = t_hit + 1e-4 after each hit; the reference
 * rejects t <= tMin after intersectSurfel's t > 1e-5, and tMin >= 1e-5) and
 * returns T = prod(1 - opacity * alpha_geom), stopping once T <= 0.001. */
static float blas_transmit(const orc_scene *s, v3 o, v3 d, trav_ctr *ctr) {
    float T = 1.0f, tmin = 1e-5f;
    for (uint32_t guard = 0; guard < (1u << 22); ++guard) {
        uint32_t prim;
        float t, a;
        v3 x;
        if (!blas_firsthit_from(s, o, d, tmin, &prim, &t, &x, &a, ctr)) break;
        float alpha_eff = s->pts[prim].opacity * a;
        T *= 1.0f - alpha_eff;
        tmin = t + 1e-4f;
        if (T <= 0.001f) break;
    }
    return T;
}

/* intersectScene in FirstHit mode (IntersectionKernels.h:954-1097):
 * closest world-space hit over the mesh instances (object-space
 * Moller-Trumbore, intersectBLASMesh :37-105) and the surfel cloud. */
static hit_t intersect_scene_mode(const orc_scene *s, v3 o, v3 d, trav_ctr *ctr, float *transmit) {
    hit_t h;
    memset(&h, 0, sizeof(h));
    h.inst = -1;
    h.t = FLT_MAX;
    float best = INFINITY;
    v3 invw = safe_inv(d);
    for (uint32_t i = 0; i < s->ninst; ++i) {
        float te;
        if (!slab(o, invw, s->inst_lo[i], s->inst_hi[i], best, &te, 0.f)) continue;
        const float *W2O = s->w2o + 16 * i, *O2W = s->o2w + 16 * i;
        v3 oo = xform_point(W2O, o);
        v3 dd = xform_dir(W2O, d);
        uint32_t m = s->inst_mesh[i];
        uint32_t first = s->mranges[2 * m], cnt = s->mranges[2 * m + 1];
        float bt = INFINITY;
        int any = 0;
        uint32_t bprim = 0;
        for (uint32_t k = 0; k < cnt; ++k) {
            const uint32_t *tr = s->tris + 3 * (first + k);
            float t;
            if (tri_hit(oo, dd, vload(s->verts + 3 * tr[0]), vload(s->verts + 3 * tr[1]),
                        vload(s->verts + 3 * tr[2]), &t, 1e-4f) && t < bt && t > 0.0f) {
                bt = t;
                any = 1;
                bprim = first + k;
            }
        }
        if (!any) continue;
        v3 hw = xform_point(O2W, vadd(oo, vscale(dd, bt)));
        float tw = vdot(vsub(hw, o), d);
        if (tw > 0.0f && tw < best) {
            best = tw;
            h.hit = 1;
            h.t = tw;
            h.pos = hw;
            h.inst = (int)i;
            h.prim = bprim;
            h.alpha = 0.0f;
        }
    }
    if (s->has_pc) {
        float te;
        if (slab(o, invw, s->pc_lo, s->pc_hi, best, &te, 0.f)) {
            /* the surfel cloud's instance transform is the identity, so the
             * object-space ray is (o, normalize(d)) (toObjectSpace, :217-227) */
            v3 dd = vnorm(d);
            uint32_t prim;
            float t, a;
            v3 x;
            /* Transmit mode (:1066-1090): the cloud adds no surface hit, only
             * its transmissivity over the whole ray */
            if (transmit) *transmit = blas_transmit(s, o, dd, ctr);
            else if (blas_firsthit(s, o, dd, &prim, &t, &x, &a, ctr)) {
                float tw = vdot(vsub(x, o), d);
                if (tw > 0.0f && tw < best) {
                    best = tw;
                    h.hit = 1;
                    h.t = tw;
                    h.pos = x;
                    h.inst = (int)s->ninst;
                    h.prim = prim;
                    h.alpha = a;
                }
            }
        }
    }
    if (h.hit) {
        /* buildIntersectionNormal (KernelHelpers.h:480-503) */
        if (h.inst < (int)s->ninst) {
            const float *O2W = s->o2w + 16 * h.inst;
            const uint32_t *tr = s->tris + 3 * h.prim;
            v3 p0 = xform_point(O2W, vload(s->verts + 3 * tr[0]));
            v3 p1 = xform_point(O2W, vload(s->verts + 3 * tr[1]));
            v3 p2 = xform_point(O2W, vload(s->verts + 3 * tr[2]));
            h.normal = vnorm(vcross(vsub(p1, p0), vsub(p2, p0)));
        } else {
            const point_t *sf = &s->pts[h.prim];
            h.normal = vnorm(vcross(sf->tu, sf->tv));
        }
    }
    return h;
}

static hit_t intersect_scene(const orc_scene *s, v3 o, v3 d, trav_ctr *ctr) {
    return intersect_scene_mode(s, o, d, ctr, NULL);
}

/* ---------------------------------------------------------------- sampling */
/* sampleCosineHemisphere (rng first) (KernelHelpers.h:317-337). */
static void sample_cosine(rng_t *r, v3 n, v3 *out, float *pdf) {
    float u1 = rng_f(r), u2 = rng_f(r);
    float z = sqrtf(1.f - u1);
    float rr = sqrtf(1 - (z * z));
    float phi = 2.f * M_PIf_ * u2;
    float x = rr * cosf(phi), y = rr * sinf(phi);
    v3 up = fabsf(n.z) < .999f ? V3(0, 0, 1) : V3(1, 0, 0);
    v3 tang = vnorm(vcross(up, n));
    v3 bit = vcross(n, tang);
    *out = vnorm(vadd(vadd(vscale(tang, x), vscale(bit, y)), vscale(n, z)));
    *pdf = fmaxf(0.f, vdot(*out, n)) / M_PIf_;
}
/* sampleUniformHemisphereAroundNormal (KernelHelpers.h:541-611). */
static void sample_uniform_hemi(rng_t *r, v3 normal, v3 *out, float *pdf) {
    v3 n = vnorm(normal);
    float u1 = rng_f(r), u2 = rng_f(r);
    float z = u1;
    float phi = 2.0f * M_PIf_ * u2;
    float rr = sqrtf(fmaxf(0.0f, 1.0f - z * z));
    float x = rr * cosf(phi), y = rr * sinf(phi);
    float sign = copysignf(1.0f, n.z);
    float a = -1.0f / (sign + n.z);
    float b = n.x * n.y * a;
    v3 T = V3(1.0f + sign * n.x * n.x * a, sign * b, -sign * n.x);
    v3 B = V3(b, sign + n.y * n.y * a, -n.y);
    *out = vnorm(vadd(vadd(vscale(T, x), vscale(B, y)), vscale(n, z)));
    *pdf = 1.0f / (2.0f * M_PIf_);
}
/* applyRussianRoulette (KernelHelpers.h:1612-1657). */
static int russian_roulette(rng_t *r, uint32_t bounce, v3 *thr, uint32_t start) {
    if (bounce < start) return 1;
    if (!isfinite(thr->x) || !isfinite(thr->y) || !isfinite(thr->z)) return 0;
    float lum = 0.2126f * thr->x + 0.7152f * thr->y + 0.0722f * thr->z;
    float p = clampf(lum, 0.0f, 0.99f);
    if (rng_f(r) > p) return 0;
    float comp = 1.0f / p;
    comp = fminf(comp, 10.0f);
    *thr = vscale(*thr, comp);
    return 1;
}
/* sampleMeshAreaLight (KernelHelpers.h:340-449). */
static int sample_light(const orc_scene *s, rng_t *r, v3 *pos, v3 *nrm, v3 *dir, v3 *power,
                        uint32_t *li) {
    if (s->nlights == 0) return 0;
    float ul = rng_f(r);
    uint32_t l = (uint32_t)(ul * (float)s->nlights);
    if (l > s->nlights - 1u) l = s->nlights - 1u;
    const light_t *L = &s->lights[l];
    if (L->tri_count == 0u || L->area <= 0.0f) return 0;
    float ut = rng_f(r);
    uint32_t lo = 0, hi = L->tri_count - 1u;
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1u;
        if (ut <= s->tri_cdf[L->tri_offset + mid]) hi = mid;
        else lo = mid + 1u;
    }
    uint32_t tri = s->tri_global[L->tri_offset + lo];
    const uint32_t *tr = s->tris + 3 * tri;
    v3 p0 = vload(s->verts + 3 * tr[0]), p1 = vload(s->verts + 3 * tr[1]), p2 = vload(s->verts + 3 * tr[2]);
    float u1 = rng_f(r), u2 = rng_f(r);
    float su1 = sqrtf(u1);
    float b0 = 1.0f - su1, b1 = su1 * (1.0f - u2), b2 = su1 * u2;
    v3 xo = vadd(vadd(vscale(p0, b0), vscale(p1, b1)), vscale(p2, b2));
    const float *O2W = s->o2w + 16 * L->mesh_instance;
    v3 w0 = xform_point(O2W, p0), w1 = xform_point(O2W, p1), w2 = xform_point(O2W, p2);
    v3 e0 = vsub(w1, w0), e1 = vsub(w2, w0);
    v3 nw = V3(e0.y * e1.z - e0.z * e1.y, e0.z * e1.x - e0.x * e1.z, e0.x * e1.y - e0.y * e1.x);
    float nl = sqrtf(vdot(nw, nw));
    if (nl <= 0.0f) return 0;
    nw = vdivs(nw, nl);
    float pdf;
    sample_cosine(r, nw, dir, &pdf);
    *pos = xform_point(O2W, xo);
    *nrm = nw;
    *power = vscale(L->color, L->power);
    *li = l;
    return 1;
}

/* ------------------------------------------------------------- photon map */
/* worldToCellClamped / linearCellIndex (KernelHelpers.h:900-987). */
static inline void world_to_cell(const orc_scene *s, v3 p, int c[3]) {
    v3 l = vsub(p, s->origin);
    float f[3] = {l.x / s->cell.x, l.y / s->cell.y, l.z / s->cell.z};
    for (int a = 0; a < 3; ++a) {
        int v = (int)floorf(f[a]);
        if (v < 0) v = 0;
        if (v > s->res[a] - 1) v = s->res[a] - 1;
        c[a] = v;
    }
}
static inline uint32_t lin_cell(const orc_scene *s, int x, int y, int z) {
    return (uint32_t)((z * s->res[1] + y) * s->res[0] + x);
}
/* configurePhotonGrid (PathTracer.cpp:184-221), radius from settings. */
static int configure_grid(orc_scene *s) {
    v3 lo = V3(INFINITY, INFINITY, INFINITY), hi = V3(-INFINITY, -INFINITY, -INFINITY);
    for (uint32_t i = 0; i < s->ninst; ++i) { lo = vmin(lo, s->inst_lo[i]); hi = vmax(hi, s->inst_hi[i]); }
    if (s->has_pc) { lo = vmin(lo, s->pc_lo); hi = vmax(hi, s->pc_hi); }
    s->r = s->st.gather_radius;
    float cs = 0.5f * s->r;
    s->cell = V3(cs, cs, cs);
    v3 pad = V3(s->r, s->r, s->r);
    s->origin = vsub(lo, pad);
    v3 gmax = vadd(hi, pad);
    v3 ext = vsub(gmax, s->origin);
    float safe = fmaxf(cs, 1e-6f);
    s->res[0] = (int)ceilf(ext.x / safe);
    s->res[1] = (int)ceilf(ext.y / safe);
    s->res[2] = (int)ceilf(ext.z / safe);
    uint64_t tot = (uint64_t)s->res[0] * (uint64_t)s->res[1] * (uint64_t)s->res[2];
    if (tot == 0 || tot > 0xFFFFFFFFull) return -1;
    s->ncells = (uint32_t)tot;
    free(s->cell_off);
    s->cell_off = (uint32_t *)calloc((size_t)s->ncells + 1, sizeof(uint32_t));
    s->grid_ready = 1;
    return 0;
}
/* buildPhotonCellRangesAndOrdering (PrimalKernels.cpp:796-1018) with the
 * intra-cell order fixed to ascending deposit index (a counting sort). */
static void build_grid(orc_scene *s) {
    uint32_t n = s->stored;
    free(s->ph_cell); free(s->sorted); free(s->ph_sorted);
    s->ph_cell = (uint32_t *)malloc((n ? n : 1) * sizeof(uint32_t));
    s->sorted = (uint32_t *)malloc((n ? n : 1) * sizeof(uint32_t));
    s->ph_sorted = (photon_t *)malloc((n ? n : 1) * sizeof(photon_t));
    memset(s->cell_off, 0, ((size_t)s->ncells + 1) * sizeof(uint32_t));
    for (uint32_t i = 0; i < n; ++i) {
        int c[3];
        world_to_cell(s, s->ph[i].pos, c);
        s->ph_cell[i] = lin_cell(s, c[0], c[1], c[2]);
        s->cell_off[s->ph_cell[i] + 1]++;
    }
    for (uint32_t c = 0; c < s->ncells; ++c) s->cell_off[c + 1] += s->cell_off[c];
    uint32_t *fill = (uint32_t *)malloc(((size_t)s->ncells + 1) * sizeof(uint32_t));
    memcpy(fill, s->cell_off, ((size_t)s->ncells + 1) * sizeof(uint32_t));
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t k = fill[s->ph_cell[i]]++;
        s->sorted[k] = i;
        s->ph_sorted[k] = s->ph[i];
    }
    free(fill);
}
/* gatherDiffuseIrradianceAtPoint (KernelHelpers.h:990-1037). */
static v3 gather(const orc_scene *s, v3 x, v3 n, uint64_t *scanned) {
    float r = s->r, r2 = r * r;
    float invArea = 1.0f / (M_PIf_ * r2);
    int c0[3], c1[3];
    world_to_cell(s, vsub(x, V3(r, r, r)), c0);
    world_to_cell(s, vadd(x, V3(r, r, r)), c1);
    v3 E = V3(0, 0, 0);
    uint64_t sc = 0;
    for (int cz = c0[2]; cz <= c1[2]; ++cz)
        for (int cy = c0[1]; cy <= c1[1]; ++cy)
            for (int cx = c0[0]; cx <= c1[0]; ++cx) {
                uint32_t id = lin_cell(s, cx, cy, cz);
                for (uint32_t j = s->cell_off[id]; j < s->cell_off[id + 1]; ++j) {
                    const photon_t *ph = &s->ph_sorted[j];
                    sc++;
                    v3 dd = vsub(ph->pos, x);
                    float cosine = vdot(n, vneg(ph->dir));
                    if (cosine < 0.0f) continue;
                    float d2 = vdot(dd, dd);
                    if (d2 > r2) continue;
                    E = vadd(E, vscale(ph->power, invArea));
                }
            }
    if (scanned) *scanned += sc;
    uint32_t T = s->attempts;
    uint32_t D = (uint64_t)T < s->cap ? T : (uint32_t)s->cap;
    if (D == 0u) return V3(0, 0, 0);
    float scale = (float)T / (float)D;
    return vscale(E, scale);
}

/* ------------------------------------------------------------ scene setup */
orc_scene *orc_create(const orc_scene_desc *d, const orc_settings *st, int bvh_kind) {
    orc_scene *s = (orc_scene *)calloc(1, sizeof(orc_scene));
    s->st = *st;
    s->bvh_kind = bvh_kind;
    s->nv = d->num_vertices; s->nt = d->num_triangles; s->nm = d->num_meshes;
    s->nmat = d->num_materials; s->ninst = d->num_instances; s->ncam = d->num_cameras;
    s->verts = (float *)xdup(d->vertices, 3 * s->nv * sizeof(float));
    s->tris = (uint32_t *)xdup(d->triangles, 3 * s->nt * sizeof(uint32_t));
    s->mranges = (uint32_t *)xdup(d->mesh_ranges, 2 * s->nm * sizeof(uint32_t));
    s->mats = (float *)xdup(d->materials, 4 * s->nmat * sizeof(float));
    s->inst_mesh = (uint32_t *)xdup(d->instance_mesh, s->ninst * sizeof(uint32_t));
    s->inst_mat = (uint32_t *)xdup(d->instance_material, s->ninst * sizeof(uint32_t));
    s->o2w = (float *)xdup(d->instance_object_to_world, 16 * s->ninst * sizeof(float));
    s->w2o = (float *)xdup(d->instance_world_to_object, 16 * s->ninst * sizeof(float));
    s->cam_inv_view = (float *)xdup(d->camera_inv_view, 16 * s->ncam * sizeof(float));
    s->cam_forward = (float *)xdup(d->camera_forward, 3 * s->ncam * sizeof(float));
    s->cam_fovy = (float *)xdup(d->camera_fovy_deg, s->ncam * sizeof(float));
    s->cam_size = (uint32_t *)xdup(d->camera_size, 2 * s->ncam * sizeof(uint32_t));
    s->cam_names = (char *)xdup(d->camera_names, 16 * s->ncam);
    /* per-instance world AABB: 8 transformed corners of the mesh box
     * (buildTLAS, SceneBuild.cpp:555-582) */
    s->inst_lo = (v3 *)malloc((s->ninst + 1) * sizeof(v3));
    s->inst_hi = (v3 *)malloc((s->ninst + 1) * sizeof(v3));
    for (uint32_t i = 0; i < s->ninst; ++i) {
        uint32_t m = s->inst_mesh[i];
        uint32_t first = s->mranges[2 * m], cnt = s->mranges[2 * m + 1];
        v3 bl = V3(INFINITY, INFINITY, INFINITY), bh = V3(-INFINITY, -INFINITY, -INFINITY);
        for (uint32_t k = 0; k < cnt; ++k)
            for (int c = 0; c < 3; ++c) {
                v3 p = vload(s->verts + 3 * s->tris[3 * (first + k) + c]);
                bl = vmin(bl, p);
                bh = vmax(bh, p);
            }
        v3 wl = V3(FLT_MAX, FLT_MAX, FLT_MAX), wh = V3(-FLT_MAX, -FLT_MAX, -FLT_MAX);
        for (int c = 0; c < 8; ++c) {
            v3 p = V3((c & 4) ? bh.x : bl.x, (c & 2) ? bh.y : bl.y, (c & 1) ? bh.z : bl.z);
            v3 pw = xform_point(s->o2w + 16 * i, p);
            wl = vmin(wl, pw);
            wh = vmax(wh, pw);
        }
        s->inst_lo[i] = wl;
        s->inst_hi[i] = wh;
    }
    /* lights: world-area CDF per emissive mesh instance (SceneBuild.cpp:263-343) */
    s->lights = (light_t *)calloc(s->ninst + 1, sizeof(light_t));
    s->tri_cdf = (float *)calloc(s->nt * (s->ninst + 1) + 1, sizeof(float));
    s->tri_global = (uint32_t *)calloc(s->nt * (s->ninst + 1) + 1, sizeof(uint32_t));
    uint32_t off = 0;
    for (uint32_t i = 0; i < s->ninst; ++i) {
        const float *mat = s->mats + 4 * s->inst_mat[i];
        if (!(mat[3] > 0.f)) continue;
        uint32_t m = s->inst_mesh[i];
        uint32_t first = s->mranges[2 * m], cnt = s->mranges[2 * m + 1];
        if (cnt == 0) continue;
        float total = 0.0f;
        float *areas = (float *)malloc(cnt * sizeof(float));
        for (uint32_t k = 0; k < cnt; ++k) {
            const uint32_t *tr = s->tris + 3 * (first + k);
            v3 w0 = xform_point(s->o2w + 16 * i, vload(s->verts + 3 * tr[0]));
            v3 w1 = xform_point(s->o2w + 16 * i, vload(s->verts + 3 * tr[1]));
            v3 w2 = xform_point(s->o2w + 16 * i, vload(s->verts + 3 * tr[2]));
            areas[k] = 0.5f * vlen(vcross(vsub(w1, w0), vsub(w2, w0)));
            total += areas[k];
        }
        if (total <= 0.0f) { free(areas); continue; }
        float run = 0.0f;
        for (uint32_t k = 0; k < cnt; ++k) {
            run += areas[k];
            s->tri_cdf[off + k] = run / total;
            s->tri_global[off + k] = first + k;
        }
        s->tri_cdf[off + cnt - 1] = 1.0f;
        light_t *L = &s->lights[s->nlights++];
        L->mesh_instance = i;
        L->tri_offset = off;
        L->tri_count = cnt;
        L->color = V3(mat[0], mat[1], mat[2]);
        L->power = mat[3];
        L->area = total;
        off += cnt;
        free(areas);
    }
    build_points(s, &d->points);
    /* photon store: photons x passes x bounces, clamped to 10 GiB of 64-byte
     * records (PathTracer.cpp:123-144) */
    uint64_t req = (uint64_t)st->photons_per_launch * (uint64_t)st->forward_passes * st->max_bounces;
    uint64_t mx = (10ull << 30) / 64ull;
    s->cap = req < mx ? req : mx;
    s->ph = (photon_t *)malloc((s->cap ? s->cap : 1) * sizeof(photon_t));
    if (configure_grid(s) != 0) { orc_destroy(s); return NULL; }
    s->stored = s->attempts = 0;
    build_grid(s);
    return s;
}

void orc_destroy(orc_scene *s) {
    if (!s) return;
    free(s->verts); free(s->tris); free(s->mranges); free(s->mats); free(s->inst_mesh);
    free(s->inst_mat); free(s->o2w); free(s->w2o); free(s->inst_lo); free(s->inst_hi);
    free(s->lights); free(s->tri_cdf); free(s->tri_global); free(s->cam_inv_view);
    free(s->cam_forward); free(s->cam_fovy); free(s->cam_size); free(s->cam_names);
    free(s->pts); free(s->order); free(s->nodes); free(s->ph); free(s->ph_cell);
    free(s->sorted); free(s->cell_off); free(s->ph_sorted);
    free(s);
}

uint32_t orc_point_count(const orc_scene *s) { return s->np; }
int orc_get_order(const orc_scene *s, uint32_t *order) {
    if (s->np) memcpy(order, s->order, s->np * sizeof(uint32_t));
    return 0;
}
int orc_get_points(const orc_scene *s, orc_points *o) {
    for (uint32_t i = 0; i < s->np; ++i) {
        const point_t *q = &s->pts[i];
        if (o->position) vstore(o->position + 3 * i, q->p);
        if (o->tangent_u) vstore(o->tangent_u + 3 * i, q->tu);
        if (o->tangent_v) vstore(o->tangent_v + 3 * i, q->tv);
        if (o->scale) { o->scale[2 * i] = q->su; o->scale[2 * i + 1] = q->sv; }
        if (o->albedo) vstore(o->albedo + 3 * i, q->albedo);
        if (o->opacity) o->opacity[i] = q->opacity;
        if (o->beta) o->beta[i] = q->beta;
        if (o->shape) o->shape[i] = q->shape;
    }
    return 0;
}
/* apply_point_optimization: raw values into the BVH-ordered points, BVH
 * left untouched (pale_bindings.cpp:853-1056). */
int orc_apply_points(orc_scene *s, const orc_points *p) {
    if (p->count != s->np) return -1;
    for (uint32_t i = 0; i < s->np; ++i) {
        point_t *q = &s->pts[i];
        q->p = vload(p->position + 3 * i);
        q->tu = vload(p->tangent_u + 3 * i);
        q->tv = vload(p->tangent_v + 3 * i);
        q->su = p->scale[2 * i];
        q->sv = p->scale[2 * i + 1];
        q->albedo = vload(p->albedo + 3 * i);
        q->opacity = p->opacity[i];
        q->beta = p->beta[i];
    }
    return 0;
}
int orc_rebuild(orc_scene *s, const orc_points *asset) {
    build_points(s, asset);
    return 0;
}

/* --------------------------------------------------------- camera rays */
/* makePrimaryRayFromPixelJitteredFov (KernelHelpers.h:764-796). */
static void primary_ray(const orc_scene *s, uint32_t cam, float px, float py, float jx, float jy,
                        v3 *o, v3 *d) {
    const uint32_t W = s->cam_size[2 * cam], H = s->cam_size[2 * cam + 1];
    const float width = (float)W, height = (float)H;
    float u = (px + 0.5f + jx);
    float v = (py + 0.5f + jy);
    float vf = height - v;
    float ndcX = (2.0f * u / width - 1.0f);
    float ndcY = (2.0f * vf / height - 1.0f);
    float f_y = 0.5f * height / tanf(0.5f * (s->cam_fovy[cam] * 0.01745329251994329576923690768489f));
    float f_x = f_y * (width / height);
    v3 dc = vnorm(V3(ndcX * (0.5f * width) / f_x, ndcY * (0.5f * height) / f_y, -1.0f));
    const float *M = s->cam_inv_view + 16 * cam;
    *d = xform_dir(M, dc);
    float h[4];
    m4mul(M, 0.f, 0.f, 0.f, 1.f, h);
    float invW = 1.f / h[3];
    *o = V3(h[0] * invW, h[1] * invW, h[2] * invW);
}

/* ------------------------------------------------------- forward pass */
typedef struct {
    int alive;
    ray_t next;
    int dep;
    photon_t ph;
} pstage_t;

/* launchIntersectKernel body for one queue slot (PrimalKernels.cpp:65-321). */
static void photon_bounce(const orc_scene *s, uint64_t base, uint32_t slot, const ray_t *ray,
                          pstage_t *out, trav_ctr *ctr) {
    const orc_settings *st = &s->st;
    rng_t r = rng_make(orc_per_item_seed(base, slot));
    out->alive = 0;
    out->dep = 0;
    hit_t h = intersect_scene(s, ray->o, ray->d, ctr);
    if (!h.hit) return;
    ray_t nx;
    memset(&nx, 0, sizeof(nx));
    nx.bounce = ray->bounce + 1;
    nx.pixel = ray->pixel;
    nx.path = ray->path;
    if (h.inst < (int)s->ninst) {
        /* depositPhotonSurface (KernelHelpers.h:1688-1727) */
        out->dep = 1;
        out->ph.pos = h.pos;
        out->ph.dir = ray->d;
        out->ph.power = ray->thr;
        const float *mat = s->mats + 4 * s->inst_mat[h.inst];
        v3 dir;
        float pdf;
        sample_cosine(&r, h.normal, &dir, &pdf);
        nx.o = vadd(h.pos, vscale(h.normal, 1e-6f));
        nx.d = dir;
        nx.n = h.normal;
        nx.thr = vmul(ray->thr, V3(mat[0], mat[1], mat[2]));
        if (!russian_roulette(&r, nx.bounce, &nx.thr, st->rr_start)) return;
        out->alive = 1;
        out->next = nx;
        return;
    }
    const point_t *sf = &s->pts[h.prim];
    float u = rng_f(&r);
    if (u < st->q_null) {
        float att = 1.0f - h.alpha * sf->opacity;
        float w = att / st->q_null;
        nx.o = vadd(h.pos, vscale(ray->d, 1e-5f));
        nx.d = ray->d;
        nx.n = h.normal;
        nx.thr = vscale(ray->thr, w);
        if (!russian_roulette(&r, nx.bounce, &nx.thr, st->rr_start)) return;
        out->alive = 1;
        out->next = nx;
    } else if (u < st->q_null + st->q_reflect) {
        v3 cn = vnorm(vcross(sf->tu, sf->tv));
        float sc = vdot(cn, vneg(ray->d));
        v3 on = vscale(cn, (float)(sc >= 0.0f ? 1 : -1));
        out->dep = 1;
        out->ph.pos = h.pos;
        out->ph.dir = ray->d;
        out->ph.power = vdivs(ray->thr, st->q_reflect);
        v3 dir;
        float pdf;
        sample_uniform_hemi(&r, on, &dir, &pdf);
        float ct = fmaxf(0.0f, vdot(dir, on));
        v3 fs = vscale(vscale(sf->albedo, sf->alpha_r), M_1_PIf_);
        float alpha = h.alpha * sf->opacity;
        v3 w = vdivs(vscale(vscale(fs, alpha / st->q_reflect), ct), pdf);
        nx.o = vadd(h.pos, vscale(on, 1e-5f));
        nx.d = dir;
        nx.n = on;
        nx.thr = vmul(ray->thr, w);
        if (!russian_roulette(&r, nx.bounce, &nx.thr, st->rr_start)) return;
        out->alive = 1;
        out->next = nx;
    } else if (u < st->q_null + st->q_reflect + st->q_transmit) {
        v3 cn = vnorm(vcross(sf->tu, sf->tv));
        float sc = vdot(cn, vneg(ray->d));
        v3 on = vscale(cn, (float)(sc >= 0.0f ? 1 : -1));
        v3 dir;
        float pdf;
        sample_uniform_hemi(&r, on, &dir, &pdf);
        float ct = fmaxf(0.0f, vdot(dir, on));
        v3 fs = vscale(vscale(sf->albedo, sf->alpha_t), M_1_PIf_);
        float alpha = h.alpha * sf->opacity;
        /* the reference divides by qReflect here (PrimalKernels.cpp:297) */
        v3 w = vdivs(vscale(vscale(fs, alpha / st->q_reflect), ct), pdf);
        nx.o = vadd(h.pos, vscale(vneg(on), 1e-5f));
        nx.d = dir;
        nx.n = vneg(on);
        nx.thr = vmul(ray->thr, w);
        if (!russian_roulette(&r, nx.bounce, &nx.thr, st->rr_start)) return;
        out->alive = 1;
        out->next = nx;
    }
}

/* submitPhotonMappingKernel photon part (SyclBridge.cpp:82-131). */
static void photon_pass(orc_scene *s, mt64_t *mt) {
    const orc_settings *st = &s->st;
    uint32_t P = st->photons_per_launch;
    uint32_t qcap = P ? P : 1;
    ray_t *q = (ray_t *)malloc(qcap * sizeof(ray_t)), *q2 = (ray_t *)malloc(qcap * sizeof(ray_t));
    pstage_t *stg = (pstage_t *)malloc(qcap * sizeof(pstage_t));
    s->attempts = s->stored = 0;
    const uint32_t emitted = st->photons_per_launch * st->forward_passes;
    const float invEmitted = 1.0f / (float)emitted;
    for (uint32_t pass = 0; pass < st->forward_passes; ++pass) {
        uint32_t base = (uint32_t)mt_next(mt);
        /* launchRayGenEmitterKernel (PrimalKernels.cpp:13-62) */
        uint32_t n = 0;
        for (uint32_t g = 0; g < P; ++g) {
            rng_t r = rng_make(orc_per_item_seed(base, g));
            if (s->nlights == 0) continue;
            v3 pos, nrm, dir, pw;
            uint32_t li;
            if (!sample_light(s, &r, &pos, &nrm, &dir, &pw, &li)) continue;
            ray_t ry;
            memset(&ry, 0, sizeof(ry));
            ry.o = pos;
            ry.d = dir;
            ry.n = nrm;
            ry.thr = vscale(vscale(pw, (float)s->nlights), invEmitted);
            ry.path = g;
            q[n++] = ry;
        }
        uint32_t active = n;
        for (uint32_t b = 0; b < st->max_bounces && active > 0; ++b) {
            uint32_t bs = (uint32_t)mt_next(mt);
            s->stats.photon_segments += active;
            uint64_t nodes = 0, tests = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : nodes, tests)
            for (int64_t k = 0; k < (int64_t)active; ++k) {
                trav_ctr c = {0, 0};
                photon_bounce(s, bs, (uint32_t)k, &q[k], &stg[k], &c);
                nodes += c.nodes;
                tests += c.tests;
            }
            s->stats.node_visits += nodes;
            s->stats.surfel_tests += tests;
            uint32_t m = 0;
            for (uint32_t k = 0; k < active; ++k) {
                if (stg[k].dep) {
                    uint32_t a = s->attempts++;
                    if (a < s->cap) s->ph[s->stored++] = stg[k].ph;
                }
                if (stg[k].alive) q2[m++] = stg[k].next;
            }
            ray_t *t = q; q = q2; q2 = t;
            active = m;
        }
    }
    s->stats.photons_stored = s->stored;
    free(q); free(q2); free(stg);
}

/* launchCameraGatherKernel for one pixel and pass (PrimalKernels.cpp:500-653). */
static v3 gather_pixel(const orc_scene *s, uint32_t cam, uint64_t base, uint32_t pix,
                       uint64_t *segs, uint64_t *queries, uint64_t *scanned, trav_ctr *ctr) {
    const uint32_t W = s->cam_size[2 * cam];
    rng_t r = rng_make(orc_per_item_seed(base, pix));
    v3 acc = V3(0, 0, 0);
    float jx = rng_f(&r) - 0.5f, jy = rng_f(&r) - 0.5f;
    v3 o, d;
    primary_ray(s, cam, (float)(pix % W), (float)(pix / W), jx, jy, &o, &d);
    float T = 1.0f;
    for (int layer = 0; layer < 65536; ++layer) {
        (*segs)++;
        hit_t h = intersect_scene(s, o, d, ctr);
        if (!h.hit) break;
        if (h.inst >= (int)s->ninst) {
            const point_t *sf = &s->pts[h.prim];
            v3 n = vnorm(vcross(sf->tu, sf->tv));
            if (vdot(n, vneg(d)) < 0.0f) n = vneg(n);
            (*queries)++;
            v3 E = gather(s, h.pos, n, scanned);
            v3 Lo = vmul(E, vscale(vscale(sf->albedo, sf->alpha_r), M_1_PIf_));
            float ae = sf->opacity * h.alpha;
            acc = vadd(acc, vscale(Lo, T * ae));
            T *= (1.0f - ae);
            o = vadd(h.pos, vscale(d, 1e-4f));
            continue;
        }
        const float *mat = s->mats + 4 * s->inst_mat[h.inst];
        v3 base_c = V3(mat[0], mat[1], mat[2]);
        if (mat[3] > 0.f) {
            v3 Le = vscale(base_c, mat[3]);
            Le = V3(fminf(Le.x, 1.0f), fminf(Le.y, 1.0f), fminf(Le.z, 1.0f));
            acc = vadd(acc, vscale(Le, T));
        } else {
            (*queries)++;
            v3 E = gather(s, h.pos, h.normal, scanned);
            v3 Lo = vmul(vscale(base_c, M_1_PIf_), E);
            acc = vadd(acc, vscale(Lo, T));
        }
        break;
    }
    return acc;
}

/* launchPostProcessKernel (PostprocessKernel.cpp:11-106): LDR floats. */
static void postprocess(const orc_scene *s, const float *raw, float *ldr, uint32_t npix) {
    float invGamma = (s->st.gamma > 0.0f) ? (1.0f / s->st.gamma) : 1.0f;
    for (uint32_t i = 0; i < npix; ++i) {
        for (int c = 0; c < 3; ++c) {
            float x = raw[4 * i + c] * s->st.exposure;
            x = fmaxf(x, 0.0f);
            x = powf(x, invGamma);
            ldr[4 * i + c] = clampf(x, 0.0f, 1.0f);
        }
        ldr[4 * i + 3] = 1.0f;
    }
}

static void gather_cameras(orc_scene *s, mt64_t mt, uint32_t nsel, const uint32_t *cams, const uint32_t *passes,
                           float *ldr, float *raw);

int orc_render_forward(orc_scene *s, uint32_t nsel, const uint32_t *cams, float *ldr, float *raw) {
    apply_threads();
    memset(&s->stats, 0, sizeof(s->stats));
    double t0 = now_ms();
    mt64_t mt;
    mt_seed(&mt, s->st.seed);
    photon_pass(s, &mt);
    build_grid(s);
    s->cam_mt = mt;
    s->cam_mt_valid = 1;
    double t1 = now_ms();
    gather_cameras(s, mt, nsel, cams, NULL, ldr, raw);
    double t2 = now_ms();
    s->stats.photon_ms = (float)(t1 - t0);
    s->stats.gather_ms = (float)(t2 - t1);
    s->stats.forward_ms = (float)(t2 - t0);
    return 0;
}

/* The camera gather alone, from the current photon map (the last forward's
 * or loaded ones), with the camera seeds a forward render uses. */
int orc_render_gather(orc_scene *s, uint32_t nsel, const uint32_t *cams, float *ldr, float *raw) {
    apply_threads();
    memset(&s->stats, 0, sizeof(s->stats));
    mt64_t mt;
    if (s->cam_mt_valid) mt = s->cam_mt;
    else mt_seed(&mt, s->st.seed);
    double t1 = now_ms();
    gather_cameras(s, mt, nsel, cams, NULL, ldr, raw);
    s->stats.gather_ms = (float)(now_ms() - t1);
    s->stats.forward_ms = s->stats.gather_ms;
    return 0;
}

/* passes: per selected camera (a view's own number of gather passes), or
 * NULL for the settings' gather_passes. */
static void gather_cameras(orc_scene *s, mt64_t mt, uint32_t nsel, const uint32_t *cams, const uint32_t *passes,
                           float *ldr, float *raw) {
    size_t off = 0;
    /* camera seeds: one draw per selected camera in selection order (the
     * reference), or one per scene camera, indexed by the camera */
    const uint32_t nseed = s->st.camera_seeds == 1 ? s->ncam : nsel;
    uint32_t *cam_seed = (uint32_t *)malloc((nseed ? nseed : 1) * sizeof(uint32_t));
    for (uint32_t k = 0; k < nseed; ++k) cam_seed[k] = (uint32_t)mt_next(&mt);
    for (uint32_t ci = 0; ci < nsel; ++ci) {
        uint32_t cam = cams[ci];
        uint32_t W = s->cam_size[2 * cam], H = s->cam_size[2 * cam + 1], npix = W * H;
        uint64_t cseed = cam_seed[s->st.camera_seeds == 1 ? cam : ci];
        float *fb = (float *)calloc((size_t)npix * 4, sizeof(float));
        const uint32_t npass = passes ? passes[ci] : s->st.gather_passes;
        float spp = (float)npass;
        uint64_t segs = 0, queries = 0, scanned = 0, nodes = 0, tests = 0;
        for (uint32_t pass = 0; pass < npass; ++pass) {
            uint64_t base = s->st.rng_mode == 1 ? orc_per_item_seed(cseed, pass) : cseed;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : segs, queries, scanned, nodes, tests)
            for (int64_t p = 0; p < (int64_t)npix; ++p) {
                trav_ctr c = {0, 0};
                uint64_t sg = 0, qu = 0, sc = 0;
                v3 a = gather_pixel(s, cam, base, (uint32_t)p, &sg, &qu, &sc, &c);
                float inv = 1.f / spp;
                float cur[4] = {a.x * inv, a.y * inv, a.z * inv, 1.0f * inv};
                for (int k = 0; k < 4; ++k) fb[4 * p + k] = cur[k] + fb[4 * p + k];
                segs += sg; queries += qu; scanned += sc; nodes += c.nodes; tests += c.tests;
            }
        }
        s->stats.gather_segments += segs;
        s->stats.gather_queries += queries;
        s->stats.photons_scanned += scanned;
        s->stats.node_visits += nodes;
        s->stats.surfel_tests += tests;
        s->stats.gather_photons_scanned += scanned;
        s->stats.gather_node_visits += nodes;
        s->stats.gather_surfel_tests += tests;
        if (raw) memcpy(raw + off, fb, (size_t)npix * 4 * sizeof(float));
        if (ldr) postprocess(s, fb, ldr + off, npix);
        off += (size_t)npix * 4;
        free(fb);
    }
    free(cam_seed);
}

/* --------------------------------------------------------- adjoint pass */
typedef struct {
    int alive;
    ray_t next;
    int has_event;
    event_t ev;
    int set_pending;
    pending_t pend;
    int clear_pending;
} astage_t;

/* launchAdjointIntersectKernel for one slot (AdjointKernels.cpp:87-386). */
static void adjoint_bounce(const orc_scene *s, uint64_t base, uint32_t slot, uint32_t bounce,
                           const ray_t *ray, const pending_t *pend, astage_t *out, trav_ctr *ctr) {
    const orc_settings *st = &s->st;
    rng_t r = rng_make(orc_per_item_seed(base, slot));
    out->alive = out->has_event = out->set_pending = out->clear_pending = 0;
    hit_t h = intersect_scene(s, ray->o, ray->d, ctr);
    if (!h.hit) return;
    int is_mesh = h.inst < (int)s->ninst;
    v3 on, dir;
    float pdf = 0.0f;
    if (is_mesh) {
        sample_cosine(&r, h.normal, &dir, &pdf);
        on = h.normal;
    } else {
        const point_t *sf = &s->pts[h.prim];
        v3 cn = vnorm(vcross(sf->tu, sf->tv));
        float sc = vdot(cn, vneg(ray->d));
        on = vscale(cn, (float)(sc >= 0.0f ? 1 : -1));
        sample_uniform_hemi(&r, on, &dir, &pdf);
    }
    /* complete the pending interaction with this hit as its endpoint */
    if ((pend->kind == PK_REFLECT && !is_mesh) || pend->kind == PK_NULL) {
        event_t *e = &out->ev;
        memset(e, 0, sizeof(*e));
        e->kind = pend->kind;
        e->prim = pend->prim;
        e->inst = pend->inst;
        e->alpha = pend->alpha;
        e->pos = pend->pos;
        e->thr = vscale(pend->thr, pend->kind == PK_REFLECT ? st->q_reflect : st->q_null);
        e->pixel = pend->pixel;
        e->end_alpha = h.alpha;
        e->end_inst = (uint32_t)h.inst;
        e->end_prim = h.prim;
        e->end_pos = h.pos;
        e->end_normal = on;
        e->end_pdf = pdf;
        e->end_type = is_mesh ? 0 : 1;
        e->end_cos = fmaxf(0.0f, vdot(dir, on));
        /* the target surfel's hit: the endpoint (reflect) or the pending null
         * surfel, on the same line (a null continuation keeps d) */
        e->tpos = pend->kind == PK_REFLECT ? h.pos : pend->pos;
        e->tdir = vnorm(ray->d);
        out->has_event = 1;
        out->clear_pending = 1;
    }
    ray_t nx;
    memset(&nx, 0, sizeof(nx));
    nx.bounce = ray->bounce + 1;
    nx.pixel = ray->pixel;
    nx.path = ray->path;
    if (is_mesh) {
        const float *mat = s->mats + 4 * s->inst_mat[h.inst];
        v3 mul = V3(mat[0], mat[1], mat[2]);
        nx.o = vadd(h.pos, vscale(h.normal, 1e-6f));
        nx.d = dir;
        nx.n = h.normal;
        nx.thr = vmul(ray->thr, mul);
        if (!russian_roulette(&r, nx.bounce, &nx.thr, st->rr_start)) return;
        pending_t *p = &out->pend;
        p->kind = PK_REFLECT;
        p->prim = INVALID_U32;
        p->inst = (uint32_t)h.inst;
        p->alpha = 0.0f;
        p->pos = h.pos;
        p->thr = vmul(ray->thr, mul);
        p->pixel = ray->pixel;
        out->set_pending = 1;
        out->alive = 1;
        out->next = nx;
        return;
    }
    const point_t *sf = &s->pts[h.prim];
    float u = rng_f(&r);
    if (u < st->q_null) {
        float att = 1.0f - h.alpha * sf->opacity;
        float w = att / st->q_null;
        nx.o = vadd(h.pos, vscale(ray->d, 1e-5f));
        nx.d = ray->d;
        nx.n = h.normal;
        nx.thr = vscale(ray->thr, w);
        if (!russian_roulette(&r, nx.bounce, &nx.thr, st->rr_start)) return;
        pending_t *p = &out->pend;
        p->kind = PK_NULL;
        p->prim = h.prim;
        p->inst = INVALID_U32;
        p->alpha = h.alpha;
        p->pos = h.pos;
        p->thr = vdivs(ray->thr, st->q_null);
        p->pixel = ray->pixel;
        out->set_pending = 1;
        out->alive = 1;
        out->next = nx;
    } else if (u < st->q_null + st->q_reflect) {
        v3 fs = vscale(vscale(sf->albedo, sf->alpha_r), M_1_PIf_);
        float ct = fmaxf(0.0f, vdot(dir, on));
        float alpha = h.alpha * sf->opacity;
        v3 mul = vdivs(vscale(vscale(fs, ct), alpha / st->q_reflect), pdf);
        nx.o = vadd(h.pos, vscale(on, 1e-5f));
        nx.d = dir;
        nx.n = on;
        nx.thr = vmul(ray->thr, mul);
        if (!russian_roulette(&r, nx.bounce, &nx.thr, st->rr_start)) return;
        if (bounce == 0) {
            event_t *e = &out->ev;
            memset(e, 0, sizeof(*e));
            e->kind = PK_PROJECTION;
            e->prim = h.prim;
            e->alpha = h.alpha;
            e->pos = h.pos;
            e->normal = on;
            e->thr = vdivs(ray->thr, st->q_reflect);
            e->pixel = ray->pixel;
            e->tpos = h.pos;
            e->tdir = vnorm(ray->d);
            out->has_event = 1;
        }
        out->alive = 1;
        out->next = nx;
    } else if (u < st->q_null + st->q_reflect + st->q_transmit) {
        float alpha = h.alpha * sf->opacity;
        float w = (alpha * sf->alpha_t) / st->q_transmit;
        v3 thr = vscale(ray->thr, w);
        v3 cn = vnorm(vcross(sf->tu, sf->tv));
        float sc = vdot(cn, vneg(ray->d));
        v3 on2 = vscale(cn, (float)(sc >= 0.0f ? 1 : -1));
        v3 d2;
        float pdf2;
        sample_uniform_hemi(&r, on2, &d2, &pdf2);
        nx.o = vadd(h.pos, vscale(vneg(on2), 1e-5f));
        nx.d = d2;
        nx.n = vneg(on2);
        nx.thr = vmul(thr, sf->albedo);
        if (!russian_roulette(&r, nx.bounce, &nx.thr, st->rr_start)) return;
        out->alive = 1;
        out->next = nx;
    }
}

/* Derivatives of eta * alpha_geom for the hit at x on surfel sf along the
 * unit direction d: alpha_geom = (1 - r^2)^B, B = 4 e^beta, r^2 = u^2 + v^2,
 * u = tu.(x - p) / su, v = tv.(x - p) / sv, x on the plane through p with
 * normal n = tu x tv / |tu x tv|.  The chain of AdjointGradientKernels.h
 * (computeDuvDPositionFull :212-272, computeFullDuDvWrtTangents :321-355,
 * computeDuvDScale :361-368, computeDAlphaDb :440-451) through
 * d alpha_geom / d r^2 = -B alpha_geom / (1 - r^2).  out: beta, position[3],
 * tangent_u[3], tangent_v[3], scale[2]; zero at the rim and in-plane. */
static void alpha_grad(const point_t *sf, v3 x, v3 d, float out[12]) {
    memset(out, 0, 12 * sizeof(float));
    const v3 U = sf->tu, V = sf->tv, r = vsub(x, sf->p);
    const float B = 4.0f * expf(sf->beta), eta = sf->opacity, su = sf->su, sv = sf->sv;
    const float u = vdot(U, r) / su, v = vdot(V, r) / sv;
    const float one = 1.0f - (u * u + v * v);
    if (!(one > 0.0f)) return;
    const float alpha = powf(one, B);
    out[0] = eta * alpha * B * logf(one);
    const v3 m = vcross(U, V), n = vnorm(m);
    const float nd = vdot(n, d), md = vdot(m, d);
    if (fabsf(nd) < 1e-6f) return;
    const float k2 = -2.0f * eta * B * alpha / one;
    const float ud = vdot(U, d), vd = vdot(V, d);
    const v3 dudp = vscale(vsub(vscale(n, ud / nd), U), 1.0f / su);
    const v3 dvdp = vscale(vsub(vscale(n, vd / nd), V), 1.0f / sv);
    const v3 gp = vscale(vadd(vscale(dudp, u), vscale(dvdp, v)), k2);
    const v3 gU = vscale(vcross(r, V), 1.0f / md), gV = vscale(vcross(U, r), 1.0f / md);
    const v3 dudU = vscale(vadd(r, vscale(gU, ud)), 1.0f / su), dvdU = vscale(gU, vd / sv);
    const v3 dudV = vscale(gV, ud / su), dvdV = vscale(vadd(r, vscale(gV, vd)), 1.0f / sv);
    const v3 gtu = vscale(vadd(vscale(dudU, u), vscale(dvdU, v)), k2);
    const v3 gtv = vscale(vadd(vscale(dudV, u), vscale(dvdV, v)), k2);
    vstore(out + 1, gp);
    vstore(out + 4, gtu);
    vstore(out + 7, gtv);
    out[10] = k2 * u * (-u / su);
    out[11] = k2 * v * (-v / sv);
}

/* launchAdjointTransportKernel for one event (AdjointKernels.cpp:389-509).
 * Returns the opacity-gradient contribution and its surfel index; *W gets
 * the event's weight (opacity term = W alpha_geom) and dalb the albedo term
 * of a ProjectionScatter event. */
static float transport_event(const orc_scene *s, const event_t *e, float invSpp, uint32_t *target,
                             uint64_t *queries, uint64_t *scanned, float *W, v3 *dalb) {
    *W = 0.0f;
    *dalb = V3(0, 0, 0);
    if (e->kind == PK_PROJECTION) {
        const point_t *sf = &s->pts[e->prim];
        (*queries)++;
        v3 E = gather(s, e->pos, e->normal, scanned);
        v3 fr = vscale(vscale(sf->albedo, sf->alpha_r), M_1_PIf_);
        v3 Lo = vmul(fr, E);
        v3 g = vmul(vscale(e->thr, e->alpha), Lo);
        *target = e->prim;
        *W = vsum(vmul(e->thr, Lo)) * invSpp;
        *dalb = vscale(vmul(e->thr, E), sf->opacity * e->alpha * sf->alpha_r * M_1_PIf_ * invSpp);
        return vsum(g) * invSpp;
    }
    if (e->kind == PK_NULL) {
        *target = e->prim;
        /* A surfel endpoint has no material: the reference reads
         * materials[0xFFFFFFFF] here (AdjointKernels.cpp:446-447); the
         * oracle treats the missing material as black and non-emissive. */
        if (e->end_type != 0) return 0.0f;
        const float *mat = s->mats + 4 * s->inst_mat[e->end_inst];
        v3 bc = V3(mat[0], mat[1], mat[2]);
        (*queries)++;
        v3 Lr = vscale(vmul(gather(s, e->end_pos, e->end_normal, scanned), bc), M_1_PIf_);
        v3 Le = V3(0, 0, 0);
        if (mat[3] > 0.f) {
            float area = s->nlights ? s->lights[0].area : 0.f;
            Le = vscale(vscale(bc, mat[3] / (M_PIf_ * area)), e->end_cos);
        }
        v3 Lo = vadd(Le, Lr);
        /* the reference's weighting: thr, on a branch taken with
         * probability q_null; null_weight 1 divides by q_null */
        float scale = s->st.null_weight == 1 ? 1.0f / s->st.q_null : 1.0f;
        float w = -e->alpha * scale;
        v3 g = vmul(vscale(e->thr, w), Lo);
        *W = -vsum(vmul(e->thr, Lo)) * scale * invSpp;
        return vsum(g) * invSpp;
    }
    if (e->kind == PK_REFLECT) {
        const float *mat = s->mats + 4 * s->inst_mat[e->inst];
        v3 bc = V3(mat[0], mat[1], mat[2]);
        (*queries)++;
        v3 Lo = vscale(vmul(gather(s, e->end_pos, e->end_normal, scanned), bc), M_1_PIf_);
        v3 p = vdivs(e->thr, e->end_pdf);
        v3 g = vscale(vmul(p, Lo), e->end_alpha);
        *target = e->end_prim;
        *W = vsum(vmul(p, Lo)) * invSpp;
        return vsum(g) * invSpp;
    }
    *target = INVALID_U32;
    return 0.0f;
}

static int render_backward_views(orc_scene *s, uint32_t nsel, const uint32_t *cams, const uint32_t *passes,
                                 const uint32_t *depths, const float *dldi, orc_points *grads, float *debug_opacity);

int orc_render_backward(orc_scene *s, uint32_t nsel, const uint32_t *cams, const float *dldi,
                        orc_points *grads, float *debug_opacity) {
    return render_backward_views(s, nsel, cams, NULL, NULL, dldi, grads, debug_opacity);
}

int orc_render_forward_views(orc_scene *s, uint32_t nsel, const uint32_t *cams, const uint32_t *passes,
                             float *ldr, float *raw) {
    apply_threads();
    memset(&s->stats, 0, sizeof(s->stats));
    mt64_t mt;
    mt_seed(&mt, s->st.seed);
    photon_pass(s, &mt);
    build_grid(s);
    s->cam_mt = mt;
    s->cam_mt_valid = 1;
    gather_cameras(s, mt, nsel, cams, passes, ldr, raw);
    return 0;
}

int orc_render_backward_views(orc_scene *s, uint32_t nsel, const uint32_t *cams, const uint32_t *passes,
                              const uint32_t *depths, const float *dldi, orc_points *grads) {
    return render_backward_views(s, nsel, cams, passes, depths, dldi, grads, NULL);
}

/* ------------------------------------------ gather estimator (estimator 1)
 * The exact derivative of the camera gather's image (gather_pixel) with the
 * photon map held: a camera path composites its surfel layers front to back,
 *   I = sum_k T_k a_k Lo_k + T_end L_end,  T_{k+1} = T_k (1 - a_k),
 * with a_k = opacity_k alpha_geom_k, Lo_k = E(x_k) albedo_k alpha_r / pi and
 * L_end the emitter (clamped) or the lit mesh that ends the path.  With Lb_k
 * the radiance behind layer k, composited back to front
 * (Lb = a Lo + (1 - a) Lb), dI/da_k = T_k (Lo_k - Lb_k); the opacity gets
 * dI/da_k alpha_geom_k, the parameters of alpha_geom (beta, position,
 * tangents, scales) dI/da_k d(a_k)/d(theta) (alpha_grad), the albedo
 * T_k a_k alpha_r E(x_k) / pi per channel.  The irradiance E(x_k) is held:
 * moving a surfel out of its plane also moves x_k against the photons,
 * which this derivative does not follow.  Every pixel and pass replays the
 * forward's camera path (same seeds), so the layers are the forward's. */
typedef struct { uint32_t prim; v3 x, E; float a, T, ageom; } glayer_t;

static void gather_pixel_grad(const orc_scene *s, uint32_t cam, uint64_t base, uint32_t pix, v3 g, float inv,
                              glayer_t **buf, uint32_t *cap, float *gop, float *gall, int all) {
    const uint32_t W = s->cam_size[2 * cam];
    rng_t r = rng_make(orc_per_item_seed(base, pix));
    float jx = rng_f(&r) - 0.5f, jy = rng_f(&r) - 0.5f;
    v3 o, d;
    primary_ray(s, cam, (float)(pix % W), (float)(pix / W), jx, jy, &o, &d);
    float T = 1.0f;
    uint32_t nl = 0;
    v3 Lend = V3(0, 0, 0);
    uint64_t dummy = 0;
    trav_ctr ctr = {0, 0};
    for (int layer = 0; layer < 65536; ++layer) {
        hit_t h = intersect_scene(s, o, d, &ctr);
        if (!h.hit) break;
        if (h.inst >= (int)s->ninst) {
            const point_t *sf = &s->pts[h.prim];
            v3 n = vnorm(vcross(sf->tu, sf->tv));
            if (vdot(n, vneg(d)) < 0.0f) n = vneg(n);
            if (nl == *cap) {
                *cap = *cap ? 2 * *cap : 64;
                *buf = (glayer_t *)realloc(*buf, *cap * sizeof(glayer_t));
            }
            glayer_t *L = *buf + nl++;
            L->prim = h.prim;
            L->x = h.pos;
            L->E = gather(s, h.pos, n, &dummy);
            L->ageom = h.alpha;
            L->a = sf->opacity * h.alpha;
            L->T = T;
            T *= (1.0f - L->a);
            o = vadd(h.pos, vscale(d, 1e-4f));
            continue;
        }
        const float *mat = s->mats + 4 * s->inst_mat[h.inst];
        v3 base_c = V3(mat[0], mat[1], mat[2]);
        if (mat[3] > 0.f) {
            v3 Le = vscale(base_c, mat[3]);
            Lend = V3(fminf(Le.x, 1.0f), fminf(Le.y, 1.0f), fminf(Le.z, 1.0f));
        } else {
            Lend = vmul(vscale(base_c, M_1_PIf_), gather(s, h.pos, h.normal, &dummy));
        }
        break;
    }
    const v3 dn = vnorm(d);
    v3 Lb = Lend;
    for (uint32_t k = nl; k-- > 0;) {
        const glayer_t *L = *buf + k;
        const point_t *sf = &s->pts[L->prim];
        const v3 fr = vscale(vscale(sf->albedo, sf->alpha_r), M_1_PIf_);
        const v3 Lo = vmul(L->E, fr);
        const float w = inv * vdot(g, vscale(vsub(Lo, Lb), L->T));   /* dLoss / da_k */
        float terms[16];
        terms[0] = w * L->ageom;
        int nt = 1;
        if (all) {
            float ag[12];
            alpha_grad(sf, L->x, dn, ag);
            for (int c = 0; c < 12; ++c) terms[1 + c] = w * ag[c];
            const float ka = inv * L->T * L->a * sf->alpha_r * M_1_PIf_;
            terms[13] = g.x * ka * L->E.x;
            terms[14] = g.y * ka * L->E.y;
            terms[15] = g.z * ka * L->E.z;
            nt = 16;
        }
#pragma omp atomic
        gop[L->prim] += terms[0];
        for (int c = 1; c < nt; ++c) {
#pragma omp atomic
            gall[15 * (size_t)L->prim + c - 1] += terms[c];
        }
        Lb = vadd(vscale(Lo, L->a), vscale(Lb, 1.0f - L->a));
    }
}

static void gather_backward(orc_scene *s, uint32_t nsel, const uint32_t *cams, const uint32_t *passes,
                            const float *dldi, float *gop, float *gall, int all) {
    mt64_t mt;
    if (s->cam_mt_valid) mt = s->cam_mt;
    else mt_seed(&mt, s->st.seed);
    const uint32_t nseed = s->st.camera_seeds == 1 ? s->ncam : nsel;
    uint32_t *cam_seed = (uint32_t *)malloc((nseed ? nseed : 1) * sizeof(uint32_t));
    for (uint32_t k = 0; k < nseed; ++k) cam_seed[k] = (uint32_t)mt_next(&mt);
    size_t off = 0;
    for (uint32_t ci = 0; ci < nsel; ++ci) {
        const uint32_t cam = cams[ci];
        const uint32_t npix = s->cam_size[2 * cam] * s->cam_size[2 * cam + 1];
        const uint64_t cseed = cam_seed[s->st.camera_seeds == 1 ? cam : ci];
        const uint32_t npass = passes ? passes[ci] : s->st.gather_passes;
        const float inv = 1.0f / (float)npass;
        const float *img = dldi + off;
        for (uint32_t pass = 0; pass < npass; ++pass) {
            const uint64_t b = s->st.rng_mode == 1 ? orc_per_item_seed(cseed, pass) : cseed;
#pragma omp parallel
            {
                glayer_t *buf = NULL;
                uint32_t cap = 0;
#pragma omp for schedule(dynamic, 64)
                for (int64_t p = 0; p < (int64_t)npix; ++p) {
                    const v3 g = V3(img[4 * p], img[4 * p + 1], img[4 * p + 2]);
                    gather_pixel_grad(s, cam, b, (uint32_t)p, g, inv, &buf, &cap, gop, gall, all);
                }
                free(buf);
            }
        }
        off += (size_t)npix * 4;
    }
    free(cam_seed);
}

/* passes / depths: per selected camera (a view's own passes and adjoint
 * bounces; depth 0 = the settings'), or NULL for the settings. */
static int render_backward_views(orc_scene *s, uint32_t nsel, const uint32_t *cams, const uint32_t *passes,
                                 const uint32_t *depths, const float *dldi, orc_points *grads, float *debug_opacity) {
    apply_threads();
    memset(&s->stats, 0, sizeof(s->stats));
    double t0 = now_ms();
    const orc_settings *st = &s->st;
    float *gop = (float *)calloc(s->np ? s->np : 1, sizeof(float));
    /* gradients == 1: per surfel beta, position[3], tangent_u[3],
     * tangent_v[3], scale[2], albedo[3] */
    const int all = st->gradients == 1;
    float *gall = all ? (float *)calloc((size_t)(s->np ? s->np : 1) * 15, sizeof(float)) : NULL;
    /* adjoint seed table: per (camera, pass) one draw for the ray
     * generation and one per bounce, camera-major; the camera is its
     * position in the selection, or with camera_seeds its scene index */
    mt64_t mt;
    mt_seed(&mt, st->rng_mode == 1 ? st->seed : 42ull);
    const uint32_t seed_cams = st->camera_seeds == 1 ? s->ncam : nsel;
    const size_t per_job = (size_t)st->adjoint_bounces + 1;
    const size_t nseeds = (size_t)seed_cams * st->adjoint_passes * per_job;
    uint32_t *seed_tab = (uint32_t *)malloc((nseeds ? nseeds : 1) * sizeof(uint32_t));
    for (size_t k = 0; k < nseeds; ++k) seed_tab[k] = (uint32_t)mt_next(&mt);
    size_t off = 0;

    if (st->estimator == 1) {
        gather_backward(s, nsel, cams, passes, dldi, gop, gall, all);
        nsel = 0;
    }
    for (uint32_t ci = 0; ci < nsel; ++ci) {
        uint32_t cam = cams[ci];
        uint32_t W = s->cam_size[2 * cam], H = s->cam_size[2 * cam + 1], npix = W * H;
        const float *img = dldi + off;
        ray_t *q = (ray_t *)malloc(npix * sizeof(ray_t)), *q2 = (ray_t *)malloc(npix * sizeof(ray_t));
        astage_t *stg = (astage_t *)malloc(npix * sizeof(astage_t));
        pending_t *pend = (pending_t *)malloc(npix * sizeof(pending_t));
        float *dbg = debug_opacity ? debug_opacity + off : NULL;
        if (dbg) memset(dbg, 0, (size_t)npix * 4 * sizeof(float));
        const uint32_t npass = passes ? passes[ci] : st->adjoint_passes;
        const uint32_t depth = depths && depths[ci] ? depths[ci] : st->adjoint_bounces;
        const float invSpp = 1.0f / (float)npass;
        for (uint32_t spp = 0; spp < npass; ++spp) {
            /* decorrelated mode: one seed for the ray generation and one per
               bounce of every pass, drawn whether or not the bounce has work */
            const uint32_t *blk = seed_tab + ((size_t)(st->camera_seeds == 1 ? cam : ci) * st->adjoint_passes + spp) * per_job;
            uint32_t sspp = blk[0];
            uint64_t rbase = st->rng_mode == 1 ? sspp : st->random_number;
            uint32_t *sbounce = (uint32_t *)malloc((st->adjoint_bounces + 1) * sizeof(uint32_t));
            for (uint32_t b = 0; b < st->adjoint_bounces; ++b) sbounce[b] = blk[1 + b];
            /* launchRayGenAdjointKernel (AdjointKernels.cpp:15-84) */
            for (uint32_t p = 0; p < npix; ++p) {
                rng_t r = rng_make(orc_per_item_seed(rbase, p));
                float jx = rng_f(&r) - 0.5f, jy = rng_f(&r) - 0.5f;
                ray_t ry;
                memset(&ry, 0, sizeof(ry));
                primary_ray(s, cam, (float)(p % W), (float)(p / W), jx, jy, &ry.o, &ry.d);
                ry.thr = V3(img[4 * p], img[4 * p + 1], img[4 * p + 2]);
                ry.pixel = p;
                ry.path = p;
                q[p] = ry;
                memset(&pend[p], 0, sizeof(pending_t));
                pend[p].prim = INVALID_U32;
                pend[p].inst = INVALID_U32;
            }
            uint32_t active = npix;
            for (uint32_t b = 0; b < depth && active > 0; ++b) {
                uint64_t bbase = st->rng_mode == 1 ? sbounce[b] : st->random_number;
                s->stats.adjoint_segments += active;
                uint64_t nodes = 0, tests = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : nodes, tests)
                for (int64_t k = 0; k < (int64_t)active; ++k) {
                    trav_ctr c = {0, 0};
                    adjoint_bounce(s, bbase, (uint32_t)k, b, &q[k], &pend[q[k].path], &stg[k], &c);
                    nodes += c.nodes;
                    tests += c.tests;
                }
                s->stats.node_visits += nodes;
                s->stats.surfel_tests += tests;
                /* pending updates (each path owns its slot; no conflicts) */
                for (uint32_t k = 0; k < active; ++k) {
                    uint32_t path = q[k].path;
                    if (stg[k].clear_pending) {
                        pend[path].kind = PK_NONE;
                        pend[path].prim = INVALID_U32;
                        pend[path].alpha = 0.0f;
                        pend[path].pos = V3(0, 0, 0);
                        pend[path].thr = V3(0, 0, 0);
                        pend[path].pixel = 0;
                    }
                    if (stg[k].set_pending) pend[path] = stg[k].pend;
                }
                /* transport in slot order of the events */
                uint32_t nev = 0;
                for (uint32_t k = 0; k < active; ++k) nev += stg[k].has_event;
                s->stats.gradient_events += nev;
                float *contrib = (float *)malloc((active ? active : 1) * sizeof(float));
                uint32_t *tgt = (uint32_t *)malloc((active ? active : 1) * sizeof(uint32_t));
                float *terms = all ? (float *)calloc((size_t)(active ? active : 1) * 15, sizeof(float)) : NULL;
                uint64_t queries = 0, scanned = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : queries, scanned)
                for (int64_t k = 0; k < (int64_t)active; ++k) {
                    tgt[k] = INVALID_U32;
                    contrib[k] = 0.f;
                    if (!stg[k].has_event) continue;
                    uint64_t qu = 0, sc = 0;
                    float W;
                    v3 dalb;
                    contrib[k] = transport_event(s, &stg[k].ev, invSpp, &tgt[k], &qu, &sc, &W, &dalb);
                    queries += qu;
                    scanned += sc;
                    if (all && tgt[k] != INVALID_U32 && W != 0.0f) {
                        float ag[12];
                        alpha_grad(&s->pts[tgt[k]], stg[k].ev.tpos, stg[k].ev.tdir, ag);
                        for (int c = 0; c < 12; ++c) terms[15 * k + c] = W * ag[c];
                    }
                    if (all && tgt[k] != INVALID_U32) vstore(terms + 15 * k + 12, dalb);
                }
                s->stats.gather_queries += queries;
                s->stats.photons_scanned += scanned;
                for (uint32_t k = 0; k < active; ++k) {
                    if (!stg[k].has_event || tgt[k] == INVALID_U32) continue;
                    gop[tgt[k]] += contrib[k];
                    if (all)
                        for (int c = 0; c < 15; ++c) gall[15 * (size_t)tgt[k] + c] += terms[15 * k + c];
                    if (dbg && st->debug_images) {
                        uint32_t px = stg[k].ev.pixel;
                        for (int c = 0; c < 3; ++c) dbg[4 * px + c] += contrib[k];
                        dbg[4 * px + 3] = 1.0f;
                    }
                }
                free(contrib);
                free(tgt);
                free(terms);
                uint32_t m = 0;
                for (uint32_t k = 0; k < active; ++k)
                    if (stg[k].alive) q2[m++] = stg[k].next;
                ray_t *t = q; q = q2; q2 = t;
                active = m;
            }
            free(sbounce);
        }
        free(q); free(q2); free(stg); free(pend);
        off += (size_t)npix * 4;
    }
    if (grads) {
        uint32_t n = s->np;
        if (grads->position) memset(grads->position, 0, 3 * n * sizeof(float));
        if (grads->tangent_u) memset(grads->tangent_u, 0, 3 * n * sizeof(float));
        if (grads->tangent_v) memset(grads->tangent_v, 0, 3 * n * sizeof(float));
        if (grads->scale) memset(grads->scale, 0, 2 * n * sizeof(float));
        if (grads->albedo) memset(grads->albedo, 0, 3 * n * sizeof(float));
        if (grads->beta) memset(grads->beta, 0, n * sizeof(float));
        if (grads->shape) memset(grads->shape, 0, n * sizeof(float));
        if (grads->opacity) memcpy(grads->opacity, gop, n * sizeof(float));
        if (all) {
            for (uint32_t i = 0; i < n; ++i) {
                const float *g = gall + 15 * (size_t)i;
                if (grads->beta) grads->beta[i] = g[0];
                for (int c = 0; c < 3; ++c) {
                    if (grads->position) grads->position[3 * i + c] = g[1 + c];
                    if (grads->tangent_u) grads->tangent_u[3 * i + c] = g[4 + c];
                    if (grads->tangent_v) grads->tangent_v[3 * i + c] = g[7 + c];
                    if (grads->albedo) grads->albedo[3 * i + c] = g[12 + c];
                }
                if (grads->scale) {
                    grads->scale[2 * i] = g[10];
                    grads->scale[2 * i + 1] = g[11];
                }
            }
        }
    }
    free(gop);
    free(gall);
    free(seed_tab);
    s->stats.backward_ms = (float)(now_ms() - t0);
    return 0;
}

/* ---------------------------------------------------- component queries */
int orc_trace_rays(orc_scene *s, uint32_t n, const float *o, const float *d, int32_t *inst,
                   int32_t *prim, float *t, float *alpha, float *hitpos) {
    apply_threads();
    uint64_t nodes = 0, tests = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : nodes, tests)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        trav_ctr c = {0, 0};
        hit_t h = intersect_scene(s, vload(o + 3 * i), vload(d + 3 * i), &c);
        nodes += c.nodes;
        tests += c.tests;
        inst[i] = h.hit ? h.inst : -1;
        prim[i] = h.hit ? (int32_t)h.prim : -1;
        t[i] = h.hit ? h.t : FLT_MAX;
        alpha[i] = h.hit ? h.alpha : 0.f;
        if (hitpos) vstore(hitpos + 3 * i, h.hit ? h.pos : V3(0, 0, 0));
    }
    memset(&s->stats, 0, sizeof(s->stats));
    s->stats.node_visits = nodes;
    s->stats.surfel_tests = tests;
    return 0;
}
/* intersectScene in Transmit mode: closest mesh hit (instance, world t;
 * -1 and FLT_MAX on a miss) and the surfel cloud's transmissivity. */
int orc_trace_transmittance(orc_scene *s, uint32_t n, const float *o, const float *d, int32_t *inst, float *t,
                            float *transmit) {
    apply_threads();
    uint64_t nodes = 0, tests = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : nodes, tests)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        trav_ctr c = {0, 0};
        float T = 1.0f;
        hit_t h = intersect_scene_mode(s, vload(o + 3 * i), vload(d + 3 * i), &c, &T);
        nodes += c.nodes;
        tests += c.tests;
        inst[i] = h.hit ? h.inst : -1;
        t[i] = h.hit ? h.t : FLT_MAX;
        transmit[i] = T;
    }
    memset(&s->stats, 0, sizeof(s->stats));
    s->stats.node_visits = nodes;
    s->stats.surfel_tests = tests;
    return 0;
}
int orc_gather_irradiance(orc_scene *s, uint32_t n, const float *pts, const float *nrm, float *E) {
    apply_threads();
    uint64_t scanned = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : scanned)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        uint64_t sc = 0;
        vstore(E + 3 * i, gather(s, vload(pts + 3 * i), vload(nrm + 3 * i), &sc));
        scanned += sc;
    }
    memset(&s->stats, 0, sizeof(s->stats));
    s->stats.gather_queries = n;
    s->stats.photons_scanned = scanned;
    return 0;
}
int orc_load_photons(orc_scene *s, uint32_t n, const float *pos, const float *pw, const float *dir) {
    if (n > s->cap) {
        free(s->ph);
        s->cap = n;
        s->ph = (photon_t *)malloc(n * sizeof(photon_t));
    }
    for (uint32_t i = 0; i < n; ++i) {
        s->ph[i].pos = vload(pos + 3 * i);
        s->ph[i].power = vload(pw + 3 * i);
        s->ph[i].dir = vload(dir + 3 * i);
    }
    s->stored = s->attempts = n;
    build_grid(s);
    return 0;
}
int orc_get_photons(orc_scene *s, uint32_t *count, float *pos, float *pw, float *dir,
                    uint32_t *cell_id, uint32_t *sorted, float *grid_info) {
    *count = s->stored;
    for (uint32_t i = 0; i < s->stored; ++i) {
        if (pos) vstore(pos + 3 * i, s->ph[i].pos);
        if (pw) vstore(pw + 3 * i, s->ph[i].power);
        if (dir) vstore(dir + 3 * i, s->ph[i].dir);
        if (cell_id) cell_id[i] = s->ph_cell[i];
        if (sorted) sorted[i] = s->sorted[i];
    }
    if (grid_info) {
        grid_info[0] = s->origin.x; grid_info[1] = s->origin.y; grid_info[2] = s->origin.z;
        grid_info[3] = s->cell.x;
        grid_info[4] = (float)s->res[0]; grid_info[5] = (float)s->res[1]; grid_info[6] = (float)s->res[2];
    }
    return 0;
}
_Static_assert(sizeof(point_t) == 19 * 4, "point record");
_Static_assert(sizeof(node_t) == 10 * 4, "node record");
_Static_assert(sizeof(light_t) == 8 * 4, "light record");

int orc_export_scene(const orc_scene *s, orc_export *e) {
    memset(e, 0, sizeof(*e));
    e->np = s->np; e->points = (const float *)s->pts; e->order = s->order;
    e->nnodes = s->nnodes; e->nodes = s->nodes;
    e->nv = s->nv; e->verts = s->verts; e->nt = s->nt; e->tris = s->tris;
    e->nm = s->nm; e->mranges = s->mranges; e->nmat = s->nmat; e->mats = s->mats;
    e->ninst = s->ninst; e->inst_mesh = s->inst_mesh; e->inst_mat = s->inst_mat;
    e->o2w = s->o2w; e->w2o = s->w2o;
    e->nlights = s->nlights; e->lights = s->lights; e->tri_cdf = s->tri_cdf; e->tri_global = s->tri_global;
    e->ncam = s->ncam; e->cam_inv_view = s->cam_inv_view; e->cam_forward = s->cam_forward;
    e->cam_fovy = s->cam_fovy; e->cam_size = s->cam_size; e->cam_names = s->cam_names;
    e->radius = s->r;
    e->cell[0] = s->cell.x; e->cell[1] = s->cell.y; e->cell[2] = s->cell.z;
    e->origin[0] = s->origin.x; e->origin[1] = s->origin.y; e->origin[2] = s->origin.z;
    for (int a = 0; a < 3; ++a) e->res[a] = s->res[a];
    e->ncells = s->ncells;
    e->photon_capacity = s->cap;
    return s->bvh_kind == 0 ? 0 : 1;
}

int orc_get_stats(const orc_scene *s, orc_stats *out) {
    *out = s->stats;
    return 0;
}
