// Runs the reference renderer's own kernel code on the CPU.
//
// TEST INFRASTRUCTURE ONLY.  oracle/build_ref.py compiles this file with the
// reference's unmodified kernel sources (Pale/Renderer/Kernels/
// PrimalKernels.cpp, AdjointKernels.cpp, PostprocessKernel.cpp) against the
// host SYCL subset in oracle/ref_shim/ into oracle/_ref/libpale_ref.so.  The
// tests use it to pin the C oracle (oracle/pale_oracle.c) to the
// reference's kernels; the benchmark's CPU baseline times it.
//
// What is the reference's and what is restated here:
//   * every device function and kernel body is the reference's own source;
//   * the host flow is restated from Pale/Renderer/Kernels/SyclBridge.cpp
//     (submitPhotonMappingKernel :82-166, submitAdjointKernel :169-294),
//     Pale/Renderer/PathTracer.cpp (buffer capacities :56-172, grid set-up
//     :184-271, renderForward/renderBackward :289-356) and
//     Pale/pale_bindings.cpp (sensor selection, dL/dI upload, downloads),
//     because SyclBridge.cpp imports a C++20 logging module and PathTracer
//     is a C++20 module;
//   * the scene (SceneBuild.cpp: an EnTT scene graph and C++20 modules) is
//     taken from the C oracle's restatement of the build: surfels in BVH
//     order, the median-split BVH, per-instance transforms, the light CDF,
//     the cameras and the photon-grid geometry (orc_export_scene).  Each
//     mesh's bottom-level BVH is one leaf over all of its triangles (the
//     reference's build with leaf size 4 makes that one leaf for the
//     two-triangle quads these scenes use).
// The gather radius comes from the settings (the reference hard-codes 0.01
// in PathTracer.cpp:187).
//
// Known out-of-bounds read in the reference: a NullTransmittance event whose
// endpoint is a surfel reads scene.materials[0xFFFFFFFF] (AdjointKernels.cpp
// :446-447; point-cloud instances carry kInvalidMaterialIndex).  The
// material array is placed at the start of a reserved 2^32-entry virtual
// range whose untouched pages read as zero, so that entry is a black,
// non-emissive material: the meaning the C oracle and the CUDA renderer give
// it.  No reference source is edited.
#include <omp.h>
#include <sys/mman.h>

#include <sycl/sycl.hpp>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "Renderer/GPUDataStructures.h"
#include "Renderer/Kernels/AdjointKernels.h"
#include "Renderer/Kernels/IntersectionKernels.h"
#include "Renderer/Kernels/KernelHelpers.h"
#include "Renderer/Kernels/PostprocessKernel.h"
#include "Renderer/Kernels/PrimalKernels.h"
#include "Renderer/RenderPackage.h"
#include "pale_oracle.h"

using namespace Pale;

namespace {

struct OracleNode {
  float lo[3], hi[3];
  int32_t left, right;
  uint32_t first, count;
};
struct OracleLight {
  uint32_t mesh_instance, tri_offset, tri_count;
  float color[3], power, area;
};
static_assert(sizeof(OracleNode) == 40 && sizeof(OracleLight) == 32, "oracle export layouts");

float4x4 rows16(const float* m) {
  float4x4 out;
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) out.row[r][c] = m[4 * r + c];
  return out;
}

}  // namespace

struct ref_scene {
  orc_scene* oracle = nullptr;
  orc_settings st{};
  PathTracerSettings settings{};
  sycl::queue queue;
  // scene buffers (GPUSceneBuffers points into these)
  std::vector<BVHNode> blasNodes;
  std::vector<BLASRange> blasRanges;
  std::vector<TLASNode> tlasNodes;
  std::vector<Triangle> triangles;
  std::vector<Vertex> vertices;
  std::vector<Transform> transforms;
  GPUMaterial* materials = nullptr;   // reserved 2^32-entry range, see the header
  size_t materialsBytes = 0;
  std::vector<Point> points;
  std::vector<InstanceRecord> instances;
  std::vector<GPULightRecord> lights;
  std::vector<GPUEmissiveTriangle> emissive;
  GPUSceneBuffers scene{};
  // cameras
  std::vector<CameraGPU> cameras;
  std::vector<std::string> cameraNames;
  // queues and photon map (PathTracer::allocateIntermediates / allocatePhotonMap)
  uint32_t rayCapacity = 0;
  std::vector<RayState> primaryRays, extensionRays;
  std::vector<WorldHit> hitRecords;
  std::vector<HitInfoContribution> contributions;
  std::vector<CompletedGradientEvent> events;
  std::vector<PendingAdjointState> pending;
  uint32_t counters[4] = {0, 0, 0, 0};   // primary, contributions, completed events, extension out
  uint32_t photonCount = 0;
  std::vector<DevicePhotonSurface> photons;
  std::vector<uint32_t> cellStart, cellEnd, cellCount, cellWriteOffset, photonCellId, photonIndex,
      sortedPhotonIndex, blockSums, blockPrefix;
  RenderIntermediatesGPU intermediates{};
  // per-call outputs
  std::vector<float> gradOpacity;
  std::vector<float3> gradPosition, gradTanU, gradTanV, gradAlbedo;
  std::vector<float2> gradScale;
  std::vector<float> gradBeta, gradShape;
  // segment counts of the last call (host-visible queue sizes) and the
  // wall time of its parts
  uint64_t photonSegments = 0, adjointSegments = 0;
  double photonMs = 0, gatherMs = 0, adjointMs = 0;
};

namespace {

void build_buffers(ref_scene* s) {
  orc_export e;
  orc_export_scene(s->oracle, &e);
  const OracleNode* onodes = static_cast<const OracleNode*>(e.nodes);
  const OracleLight* olights = static_cast<const OracleLight*>(e.lights);

  // vertices and triangles (SceneBuild's Vertex/Triangle; normals unused by the kernels)
  s->vertices.assign(e.nv, Vertex{});
  for (uint32_t i = 0; i < e.nv; ++i) s->vertices[i].pos = float3{e.verts[3 * i], e.verts[3 * i + 1], e.verts[3 * i + 2]};
  s->triangles.assign(e.nt, Triangle{});
  for (uint32_t t = 0; t < e.nt; ++t) {
    Triangle& tr = s->triangles[t];
    tr.v0 = e.tris[3 * t];
    tr.v1 = e.tris[3 * t + 1];
    tr.v2 = e.tris[3 * t + 2];
    tr.centroid = (s->vertices[tr.v0].pos + s->vertices[tr.v1].pos + s->vertices[tr.v2].pos) * (1.0f / 3.0f);
  }
  // bottom-level BVHs: one leaf per mesh, then the surfel cloud's nodes
  s->blasNodes.clear();
  s->blasRanges.clear();
  for (uint32_t m = 0; m < e.nm; ++m) {
    const uint32_t first = e.mranges[2 * m], cnt = e.mranges[2 * m + 1];
    BVHNode nd{};
    float3 lo{FLT_MAX, FLT_MAX, FLT_MAX}, hi{-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (uint32_t k = 0; k < cnt; ++k) {
      const Triangle& tr = s->triangles[first + k];
      for (uint32_t v : {tr.v0, tr.v1, tr.v2}) {
        lo = min(lo, s->vertices[v].pos);
        hi = max(hi, s->vertices[v].pos);
      }
    }
    nd.aabbMin = lo;
    nd.aabbMax = hi;
    nd.leftFirst = first;
    nd.triCount = cnt;
    s->blasRanges.push_back(BLASRange{static_cast<uint32_t>(s->blasNodes.size()), 1u});
    s->blasNodes.push_back(nd);
  }
  const uint32_t pcRange = static_cast<uint32_t>(s->blasRanges.size());
  if (e.np) {
    const uint32_t base = static_cast<uint32_t>(s->blasNodes.size());
    s->blasRanges.push_back(BLASRange{base, e.nnodes});
    for (uint32_t i = 0; i < e.nnodes; ++i) {
      const OracleNode& o = onodes[i];
      BVHNode nd{};
      nd.aabbMin = float3{o.lo[0], o.lo[1], o.lo[2]};
      nd.aabbMax = float3{o.hi[0], o.hi[1], o.hi[2]};
      if (o.count == 0) {
        nd.leftFirst = static_cast<uint32_t>(o.left);   // children at left, left + 1
        nd.triCount = 0;
      } else {
        nd.leftFirst = o.first;
        nd.triCount = o.count;
      }
      s->blasNodes.push_back(nd);
    }
  }
  // surfels in BVH order
  s->points.assign(e.np, Point{});
  for (uint32_t i = 0; i < e.np; ++i) {
    const float* q = e.points + 19 * i;
    Point& p = s->points[i];
    p.position = float3{q[0], q[1], q[2]};
    p.tanU = float3{q[3], q[4], q[5]};
    p.tanV = float3{q[6], q[7], q[8]};
    p.scale = float2{q[9], q[10]};
    p.albedo = float3{q[11], q[12], q[13]};
    p.alpha_t = q[14];
    p.alpha_r = q[15];
    p.opacity = q[16];
    p.beta = q[17];
    p.shape = q[18];
    p.pointId = e.order ? e.order[i] : i;
  }
  // transforms: one per mesh instance, then the identity of the surfel cloud
  s->transforms.assign(e.ninst + 1, Transform{});
  for (uint32_t i = 0; i < e.ninst; ++i) {
    s->transforms[i].objectToWorld = rows16(e.o2w + 16 * i);
    s->transforms[i].worldToObject = rows16(e.w2o + 16 * i);
  }
  s->transforms[e.ninst].objectToWorld = identity4x4();
  s->transforms[e.ninst].worldToObject = identity4x4();
  // materials (see the header for the reserved range)
  if (s->materials) munmap(s->materials, s->materialsBytes);
  s->materialsBytes = (size_t(1) << 32) * sizeof(GPUMaterial);
  void* mem = mmap(nullptr, s->materialsBytes, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS | MAP_NORESERVE,
                   -1, 0);
  if (mem == MAP_FAILED) throw std::runtime_error("reserving the material range failed");
  s->materials = static_cast<GPUMaterial*>(mem);
  for (uint32_t m = 0; m < e.nmat; ++m) {
    GPUMaterial gm{};
    gm.baseColor = float3{e.mats[4 * m], e.mats[4 * m + 1], e.mats[4 * m + 2]};
    gm.power = e.mats[4 * m + 3];
    gm.diffuse = 1.0f;
    s->materials[m] = gm;
  }
  // instances: the meshes in the scene's order, then the surfel cloud
  s->instances.clear();
  for (uint32_t i = 0; i < e.ninst; ++i) {
    InstanceRecord r{};
    r.geometryType = GeometryType::Mesh;
    r.geometryIndex = e.inst_mesh[i];
    r.materialIndex = e.inst_mat[i];
    r.transformIndex = i;
    r.blasRangeIndex = e.inst_mesh[i];
    copyName(r.name, "mesh" + std::to_string(i));
    s->instances.push_back(r);
  }
  if (e.np) {
    InstanceRecord r{};
    r.geometryType = GeometryType::PointCloud;
    r.geometryIndex = 0;
    r.materialIndex = kInvalidMaterialIndex;
    r.transformIndex = e.ninst;
    r.blasRangeIndex = pcRange;
    copyName(r.name, "points");
    s->instances.push_back(r);
  }
  // top level: SceneBuild::buildTLAS (SceneBuild.cpp:555-640), restated
  struct Box {
    float3 bmin, bmax;
    uint32_t inst;
  };
  std::vector<Box> boxes;
  for (uint32_t i = 0; i < s->instances.size(); ++i) {
    const InstanceRecord& inst = s->instances[i];
    const Transform& xf = s->transforms[inst.transformIndex];
    const BVHNode& root = s->blasNodes[s->blasRanges[inst.blasRangeIndex].firstNode];
    float3 wmin{FLT_MAX, FLT_MAX, FLT_MAX}, wmax{-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int c = 0; c < 8; ++c) {
      const float3 pObj{(c & 4) ? root.aabbMax.x() : root.aabbMin.x(), (c & 2) ? root.aabbMax.y() : root.aabbMin.y(),
                        (c & 1) ? root.aabbMax.z() : root.aabbMin.z()};
      const float3 pW = toWorldPoint(pObj, xf);
      wmin = min(wmin, pW);
      wmax = max(wmax, pW);
    }
    boxes.push_back({wmin, wmax, i});
  }
  s->tlasNodes.clear();
  std::function<uint32_t(uint32_t, uint32_t)> build = [&](uint32_t start, uint32_t end) -> uint32_t {
    const uint32_t n = static_cast<uint32_t>(s->tlasNodes.size());
    s->tlasNodes.emplace_back();
    float3 bmin{FLT_MAX, FLT_MAX, FLT_MAX}, bmax{-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (uint32_t i = start; i < end; ++i) {
      bmin = min(bmin, boxes[i].bmin);
      bmax = max(bmax, boxes[i].bmax);
    }
    s->tlasNodes[n].aabbMin = bmin;
    s->tlasNodes[n].aabbMax = bmax;
    const uint32_t count = end - start;
    if (count == 1) {
      s->tlasNodes[n].count = 1;
      s->tlasNodes[n].leftChild = boxes[start].inst;
      s->tlasNodes[n].rightChild = 0;
      return n;
    }
    s->tlasNodes[n].count = 0;
    float3 cmin{FLT_MAX, FLT_MAX, FLT_MAX}, cmax{-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (uint32_t i = start; i < end; ++i) {
      const float3 cent = (boxes[i].bmin + boxes[i].bmax) * 0.5f;
      cmin = min(cmin, cent);
      cmax = max(cmax, cent);
    }
    const float3 ext = cmax - cmin;
    const int axis = (ext.x() > ext.y() && ext.x() > ext.z()) ? 0 : (ext.y() > ext.z()) ? 1 : 2;
    const float pivot = (cmin[axis] + cmax[axis]) * 0.5f;
    auto mid_it = std::partition(boxes.begin() + start, boxes.begin() + end, [&](const Box& b) {
      const float3 cc = (b.bmin + b.bmax) * 0.5f;
      return cc[axis] < pivot;
    });
    uint32_t mid = static_cast<uint32_t>(mid_it - boxes.begin());
    if (mid == start || mid == end) mid = start + count / 2;
    const uint32_t l = build(start, mid);
    const uint32_t r = build(mid, end);
    s->tlasNodes[n].leftChild = l;
    s->tlasNodes[n].rightChild = r;
    return n;
  };
  if (!boxes.empty()) build(0, static_cast<uint32_t>(boxes.size()));
  // lights (SceneBuild::collectLights, SceneBuild.cpp:263-343)
  s->lights.clear();
  s->emissive.clear();
  for (uint32_t l = 0; l < e.nlights; ++l) {
    const OracleLight& o = olights[l];
    GPULightRecord r{};
    r.lightType = 0;
    r.geometryIndex = e.inst_mesh[o.mesh_instance];
    r.transformIndex = o.mesh_instance;
    r.materialIndex = e.inst_mat[o.mesh_instance];
    r.triangleOffset = o.tri_offset;
    r.triangleCount = o.tri_count;
    r.color = float3{o.color[0], o.color[1], o.color[2]};
    r.power = o.power;
    r.totalAreaWorld = o.area;
    s->lights.push_back(r);
  }
  uint32_t ntri = 0;
  for (uint32_t l = 0; l < e.nlights; ++l) ntri = std::max(ntri, olights[l].tri_offset + olights[l].tri_count);
  for (uint32_t k = 0; k < ntri; ++k) s->emissive.push_back(GPUEmissiveTriangle{e.tri_global[k], 0.0f, e.tri_cdf[k]});
  // cameras: what makePrimaryRayFromPixelJitteredFov and the gather read
  s->cameras.assign(e.ncam, CameraGPU{});
  s->cameraNames.clear();
  for (uint32_t c = 0; c < e.ncam; ++c) {
    CameraGPU& cam = s->cameras[c];
    cam.invView = rows16(e.cam_inv_view + 16 * c);
    cam.forward = float3{e.cam_forward[3 * c], e.cam_forward[3 * c + 1], e.cam_forward[3 * c + 2]};
    cam.pos = float3{cam.invView.row[0][3], cam.invView.row[1][3], cam.invView.row[2][3]};
    cam.width = e.cam_size[2 * c];
    cam.height = e.cam_size[2 * c + 1];
    cam.fovy = e.cam_fovy[c];
    std::string name(e.cam_names + 16 * c, strnlen(e.cam_names + 16 * c, 16));
    std::snprintf(cam.name, sizeof(cam.name), "%s", name.c_str());
    s->cameraNames.push_back(name);
  }
  // scene buffers
  GPUSceneBuffers& g = s->scene;
  g = GPUSceneBuffers{};
  g.blasNodes = s->blasNodes.data();
  g.blasRanges = s->blasRanges.data();
  g.tlasNodes = s->tlasNodes.data();
  g.triangles = s->triangles.data();
  g.vertices = s->vertices.data();
  g.transforms = s->transforms.data();
  g.materials = s->materials;
  g.points = s->points.data();
  g.instances = s->instances.data();
  g.blasNodeCount = static_cast<uint32_t>(s->blasNodes.size());
  g.tlasNodeCount = static_cast<uint32_t>(s->tlasNodes.size());
  g.triangleCount = e.nt;
  g.vertexCount = e.nv;
  g.pointCount = e.np;
  g.lights = s->lights.data();
  g.emissiveTriangles = s->emissive.data();
  g.lightCount = static_cast<uint32_t>(s->lights.size());
  g.emissiveTriangleCount = static_cast<uint32_t>(s->emissive.size());

  // ray queues: next power of two >= max(photons per launch, largest camera)
  uint32_t need = std::max<uint32_t>(1u, s->st.photons_per_launch);
  for (const CameraGPU& cam : s->cameras) need = std::max<uint32_t>(need, cam.width * cam.height);
  uint32_t cap = 1;
  while (cap < need) cap <<= 1;
  s->rayCapacity = cap;
  s->primaryRays.assign(cap, RayState{});
  s->extensionRays.assign(cap, RayState{});
  s->hitRecords.assign(cap, WorldHit{});
  s->contributions.assign(cap, HitInfoContribution{});
  s->events.assign(cap, CompletedGradientEvent{});
  s->pending.assign(cap, PendingAdjointState{});
  RenderIntermediatesGPU& I = s->intermediates;
  I = RenderIntermediatesGPU{};
  I.primaryRays = s->primaryRays.data();
  I.extensionRaysA = s->extensionRays.data();
  I.hitRecords = s->hitRecords.data();
  I.hitContribution = s->contributions.data();
  I.maxHitContributionCount = cap;
  I.countContributions = &s->counters[1];
  I.completedGradientEvents = s->events.data();
  I.maxCompletedGradientEventCount = cap;
  I.countCompletedGradientEvents = &s->counters[2];
  I.pendingAdjointStates = s->pending.data();
  I.maxPendingAdjointStateCount = cap;
  I.countPrimary = &s->counters[0];
  I.countExtensionOut = &s->counters[3];
  // photon map and grid (PathTracer::allocatePhotonMap, configurePhotonGrid)
  DeviceSurfacePhotonMapGrid& G = I.map;
  const uint32_t pcap = static_cast<uint32_t>(e.photon_capacity);
  s->photons.assign(std::max<uint32_t>(1u, pcap), DevicePhotonSurface{});
  G.photons = s->photons.data();
  G.photonCapacity = pcap;
  G.photonCountDevicePtr = &s->photonCount;
  G.gatherRadiusWorld = e.radius;
  G.cellSizeWorld = float3{e.cell[0], e.cell[1], e.cell[2]};
  G.gridOriginWorld = float3{e.origin[0], e.origin[1], e.origin[2]};
  G.gridResolution = sycl::int3{e.res[0], e.res[1], e.res[2]};
  G.totalCellCount = e.ncells;
  const uint32_t blocks = (e.ncells + 1023u) / 1024u;
  s->cellStart.assign(e.ncells, 0);
  s->cellEnd.assign(e.ncells, 0);
  s->cellCount.assign(e.ncells, 0);
  s->cellWriteOffset.assign(e.ncells, 0);
  s->photonCellId.assign(std::max<uint32_t>(1u, pcap), 0);
  s->photonIndex.assign(std::max<uint32_t>(1u, pcap), 0);
  s->sortedPhotonIndex.assign(std::max<uint32_t>(1u, pcap), 0);
  s->blockSums.assign(std::max<uint32_t>(1u, blocks), 0);
  s->blockPrefix.assign(std::max<uint32_t>(1u, blocks), 0);
  G.allocatedCellCount = e.ncells;
  G.allocatedPhotonCapacity = pcap;
  G.allocatedBlockCount = blocks;
  G.cellStart = s->cellStart.data();
  G.cellEnd = s->cellEnd.data();
  G.cellCount = s->cellCount.data();
  G.cellWriteOffset = s->cellWriteOffset.data();
  G.photonCellId = s->photonCellId.data();
  G.photonIndex = s->photonIndex.data();
  G.sortedPhotonIndex = s->sortedPhotonIndex.data();
  G.blockSums = s->blockSums.data();
  G.blockPrefix = s->blockPrefix.data();
}

PathTracerSettings to_settings(const orc_settings& st) {
  PathTracerSettings p{};
  p.integratorKind = IntegratorKind::photonMapping;
  p.photonsPerLaunch = st.photons_per_launch;
  p.random.seed = st.seed;
  p.random.number = st.random_number;
  p.maxBounces = st.max_bounces;
  p.numForwardPasses = st.forward_passes;
  p.numGatherPasses = st.gather_passes;
  p.maxAdjointBounces = st.adjoint_bounces;
  p.adjointSamplesPerPixel = st.adjoint_passes;
  p.russianRouletteStart = st.rr_start;
  p.renderDebugGradientImages = false;
  p.sampling.qNull = st.q_null;
  p.sampling.qReflect = st.q_reflect;
  p.sampling.qTransmit = st.q_transmit;
  p.sampling.qAbsorb = 1.0f - st.q_null - st.q_reflect - st.q_transmit;
  return p;
}

// Sensors of the selected cameras (pale_bindings.cpp:180-192), each with
// its own raw, LDR and RGBA8 framebuffers.
struct SensorSet {
  std::vector<SensorGPU> sensors;
  std::vector<std::vector<float4>> raw;
  std::vector<std::vector<float>> ldr;
  std::vector<std::vector<sycl::uchar4>> rgba8;
  std::vector<DebugImages> debug;
};

void make_sensors(ref_scene* s, uint32_t nsel, const uint32_t* cams, SensorSet& out) {
  out.sensors.resize(nsel);
  out.raw.resize(nsel);
  out.ldr.resize(nsel);
  out.rgba8.resize(nsel);
  out.debug.assign(nsel, DebugImages{});
  for (uint32_t i = 0; i < nsel; ++i) {
    const CameraGPU& cam = s->cameras[cams[i]];
    const size_t npix = size_t(cam.width) * cam.height;
    out.raw[i].assign(npix, float4{0.0f});
    out.ldr[i].assign(4 * npix, 0.0f);
    out.rgba8[i].assign(npix, sycl::uchar4{});
    SensorGPU& sg = out.sensors[i];
    sg.camera = cam;
    sg.framebuffer = out.raw[i].data();
    sg.width = cam.width;
    sg.height = cam.height;
    sg.gammaCorrection = s->st.gamma;
    sg.exposureCorrection = s->st.exposure;
    sg.ldrFramebuffer = out.ldr[i].data();
    sg.outputFramebuffer = out.rgba8[i].data();
    std::snprintf(sg.name, sizeof(sg.name), "%s", cam.name);
  }
}

RenderPackage make_package(ref_scene* s, SensorSet& ss) {
  RenderPackage pkg{};
  pkg.queue = s->queue;
  pkg.settings = s->settings;
  pkg.scene = s->scene;
  pkg.intermediates = s->intermediates;
  pkg.sensors = ss.sensors;
  pkg.numSensors = static_cast<uint32_t>(ss.sensors.size());
  pkg.debugImages = ss.debug.data();
  return pkg;
}

// submitPhotonMappingKernel (SyclBridge.cpp:82-166): the photon passes
// and the grid; with `gather` also the per-camera gather and the
// post-process.  Returns the seed stream where the camera seeds start.
std::mt19937_64 photon_mapping(ref_scene* s, RenderPackage& pkg, bool gather) {
  const double t0 = omp_get_wtime();
  std::mt19937_64 seedGen(pkg.random.seed);
  pkg.queue.fill(pkg.intermediates.map.photonCountDevicePtr, 0u, 1).wait();
  s->photonSegments = 0;
  for (uint32_t forwardPass = 0; forwardPass < pkg.settings.numForwardPasses; forwardPass++) {
    pkg.random.number = seedGen();
    pkg.queue.fill(pkg.intermediates.countPrimary, 0u, 1).wait();
    launchRayGenEmitterKernel(pkg);
    uint32_t activeCount = 0;
    pkg.queue.memcpy(&activeCount, pkg.intermediates.countPrimary, sizeof(uint32_t)).wait();
    for (uint32_t bounce = 0; bounce < pkg.settings.maxBounces && activeCount > 0; ++bounce) {
      pkg.random.number = seedGen();
      pkg.queue.fill(pkg.intermediates.countExtensionOut, static_cast<uint32_t>(0), 1);
      pkg.queue.fill(pkg.intermediates.hitRecords, WorldHit(), activeCount);
      pkg.queue.wait();
      s->photonSegments += activeCount;
      launchIntersectKernel(pkg, activeCount);
      uint32_t nextCount = 0;
      pkg.queue.memcpy(&nextCount, pkg.intermediates.countExtensionOut, sizeof(uint32_t)).wait();
      pkg.queue.memcpy(pkg.intermediates.primaryRays, pkg.intermediates.extensionRaysA, nextCount * sizeof(RayState));
      pkg.queue.wait();
      activeCount = nextCount;
    }
  }
  uint32_t photonMapCount = 0;
  pkg.queue.memcpy(&photonMapCount, pkg.intermediates.map.photonCountDevicePtr, sizeof(uint32_t)).wait();
  const uint32_t photonCount = std::min(photonMapCount, pkg.intermediates.map.photonCapacity);
  buildPhotonCellRangesAndOrdering(pkg.queue, pkg.intermediates.map, photonCount);
  const double t1 = omp_get_wtime();
  s->photonMs = (t1 - t0) * 1e3;
  s->gatherMs = 0;
  if (gather) {
    for (size_t cameraIndex = 0; cameraIndex < pkg.numSensors; ++cameraIndex) {
      pkg.random.number = seedGen();
      launchCameraGatherKernel(pkg, static_cast<uint32_t>(cameraIndex));
      pkg.queue.wait();
    }
    launchPostProcessKernel(pkg);
    s->gatherMs = (omp_get_wtime() - t1) * 1e3;
  }
  return seedGen;
}

}  // namespace

extern "C" {

void ref_set_threads(int n) { sycl_shim_set_threads(n); }

ref_scene* ref_create(const orc_scene_desc* desc, const orc_settings* st) {
  ref_scene* s = new ref_scene();
  s->st = *st;
  s->settings = to_settings(*st);
  s->oracle = orc_create(desc, st, 0);
  if (!s->oracle) {
    delete s;
    return nullptr;
  }
  try {
    build_buffers(s);
  } catch (const std::exception& ex) {
    std::fprintf(stderr, "ref_create: %s\n", ex.what());
    orc_destroy(s->oracle);
    delete s;
    return nullptr;
  }
  return s;
}

void ref_destroy(ref_scene* s) {
  if (!s) return;
  if (s->materials) munmap(s->materials, s->materialsBytes);
  orc_destroy(s->oracle);
  delete s;
}

uint32_t ref_point_count(const ref_scene* s) { return static_cast<uint32_t>(s->points.size()); }

int ref_get_order(const ref_scene* s, uint32_t* order) {
  for (size_t i = 0; i < s->points.size(); ++i) order[i] = static_cast<uint32_t>(s->points[i].pointId);
  return 0;
}

// render_forward over the selected cameras: LDR and raw RGBA per camera,
// concatenated (W*H*4 floats each), as the C oracle's orc_render_forward.
int ref_render_forward(ref_scene* s, uint32_t nsel, const uint32_t* cams, float* ldr, float* raw) {
  SensorSet ss;
  make_sensors(s, nsel, cams, ss);
  RenderPackage pkg = make_package(s, ss);
  pkg.random.seed = s->st.seed;   // renderForward: .random.seed = m_sessionSeed
  photon_mapping(s, pkg, true);
  size_t off = 0;
  for (uint32_t i = 0; i < nsel; ++i) {
    const size_t npix = ss.raw[i].size();
    for (size_t p = 0; p < npix; ++p)
      for (int c = 0; c < 4; ++c) {
        if (raw) raw[off + 4 * p + c] = ss.raw[i][p][c];
      }
    if (ldr) std::memcpy(ldr + off, ss.ldr[i].data(), 4 * npix * sizeof(float));
    off += 4 * npix;
  }
  return 0;
}

// The photon pass and grid alone (timing of the forward's first half).
int ref_trace_photons(ref_scene* s) {
  SensorSet ss;
  RenderPackage pkg = make_package(s, ss);
  pkg.random.seed = s->st.seed;
  photon_mapping(s, pkg, false);
  return 0;
}

// Number of scene traversals (ray segments) that the camera gather of the
// given cameras submits, for the throughput metric: the layer loop of
// launchCameraGatherKernel (PrimalKernels.cpp:500-653) with the same seeds
// and the reference's own intersectScene, without the photon lookups.  It
// runs the photon pass first, which decides where the camera seeds start.
uint64_t ref_count_gather_segments(ref_scene* s, uint32_t nsel, const uint32_t* cams) {
  SensorSet ss;
  make_sensors(s, nsel, cams, ss);
  RenderPackage pkg = make_package(s, ss);
  pkg.random.seed = s->st.seed;
  std::mt19937_64 seedGen = photon_mapping(s, pkg, false);
  std::vector<uint64_t> perCamera(nsel, 0);
  for (uint32_t ci = 0; ci < nsel; ++ci) {
    const uint64_t baseSeed = static_cast<uint32_t>(seedGen());
    const CameraGPU cam = ss.sensors[ci].camera;
    const uint32_t W = cam.width, npix = cam.width * cam.height;
    const GPUSceneBuffers scene = s->scene;
    std::vector<uint64_t> layers(npix, 0);
    sycl_shim::run_range(npix, [&](size_t p) {
      rng::Xorshift128 rng(rng::makePerItemSeed1D(baseSeed, p));
      const float jx = rng.nextFloat() - 0.5f;
      const float jy = rng.nextFloat() - 0.5f;
      Ray ray = makePrimaryRayFromPixelJitteredFov(cam, static_cast<float>(p % W), static_cast<float>(p / W), jx, jy);
      uint64_t n = 0;
      while (true) {
        WorldHit hit{};
        ++n;
        intersectScene(ray, &hit, scene, rng, SurfelIntersectMode::FirstHit);
        if (!hit.hit) break;
        if (scene.instances[hit.instanceIndex].geometryType != GeometryType::PointCloud) break;
        ray.origin = hit.hitPositionW + (ray.direction * 1e-4f);
      }
      layers[p] = n;
    });
    for (uint64_t v : layers) perCamera[ci] += v;
  }
  uint64_t total = 0;
  for (uint64_t v : perCamera) total += v;
  return total * s->st.gather_passes;   // every gather pass of a camera uses its one seed
}

int ref_render_backward(ref_scene* s, uint32_t nsel, const uint32_t* cams, const float* dldi, float* grad_opacity) {
  SensorSet ss;
  make_sensors(s, nsel, cams, ss);
  // upload dL/dI as the sensor framebuffers (pale_bindings.cpp:358-392)
  size_t off = 0;
  for (uint32_t i = 0; i < nsel; ++i) {
    const size_t npix = ss.raw[i].size();
    for (size_t p = 0; p < npix; ++p)
      ss.raw[i][p] = float4{dldi[off + 4 * p], dldi[off + 4 * p + 1], dldi[off + 4 * p + 2], 1.0f};
    off += 4 * npix;
  }
  const size_t n = s->points.size();
  s->gradPosition.assign(std::max<size_t>(1, n), float3{0.0f});
  s->gradTanU.assign(std::max<size_t>(1, n), float3{0.0f});
  s->gradTanV.assign(std::max<size_t>(1, n), float3{0.0f});
  s->gradAlbedo.assign(std::max<size_t>(1, n), float3{0.0f});
  s->gradScale.assign(std::max<size_t>(1, n), float2{0.0f});
  s->gradOpacity.assign(std::max<size_t>(1, n), 0.0f);
  s->gradBeta.assign(std::max<size_t>(1, n), 0.0f);
  s->gradShape.assign(std::max<size_t>(1, n), 0.0f);
  RenderPackage pkg = make_package(s, ss);   // renderBackward: Random{} (seed 42)
  pkg.gradients.gradPosition = s->gradPosition.data();
  pkg.gradients.gradTanU = s->gradTanU.data();
  pkg.gradients.gradTanV = s->gradTanV.data();
  pkg.gradients.gradScale = s->gradScale.data();
  pkg.gradients.gradAlbedo = s->gradAlbedo.data();
  pkg.gradients.gradOpacity = s->gradOpacity.data();
  pkg.gradients.gradBeta = s->gradBeta.data();
  pkg.gradients.gradShape = s->gradShape.data();
  pkg.gradients.numPoints = n;

  // submitAdjointKernel (SyclBridge.cpp:169-294)
  const double t0 = omp_get_wtime();
  std::mt19937_64 seedGen(pkg.random.seed);
  s->adjointSegments = 0;
  pkg.queue.fill(pkg.intermediates.countPrimary, 0u, 1).wait();
  pkg.queue.fill(pkg.gradients.gradPosition, float3{0, 0, 0}, pkg.gradients.numPoints).wait();
  pkg.queue.fill(pkg.gradients.gradTanU, float3{0, 0, 0}, pkg.gradients.numPoints).wait();
  pkg.queue.fill(pkg.gradients.gradTanV, float3{0, 0, 0}, pkg.gradients.numPoints).wait();
  pkg.queue.fill(pkg.gradients.gradScale, float2{0, 0}, pkg.gradients.numPoints).wait();
  pkg.queue.fill(pkg.gradients.gradAlbedo, float3{0}, pkg.gradients.numPoints).wait();
  pkg.queue.fill(pkg.gradients.gradOpacity, 0.0f, pkg.gradients.numPoints).wait();
  pkg.queue.fill(pkg.gradients.gradBeta, 0.0f, pkg.gradients.numPoints).wait();
  for (size_t cameraIndex = 0; cameraIndex < pkg.numSensors; ++cameraIndex) {
    const int samplesPerPixel = static_cast<int>(pkg.settings.adjointSamplesPerPixel);
    for (int spp = 0; spp < samplesPerPixel; ++spp) {
      pkg.random.number = seedGen();
      pkg.queue.fill(pkg.intermediates.countPrimary, 0u, 1).wait();
      launchRayGenAdjointKernel(pkg, spp, static_cast<uint32_t>(cameraIndex));
      const uint32_t raysPerFrame = pkg.sensors[cameraIndex].width * pkg.sensors[cameraIndex].height;
      uint32_t activeCount = raysPerFrame;
      pkg.queue.fill(pkg.intermediates.pendingAdjointStates, PendingAdjointState(), activeCount);
      pkg.queue.fill(pkg.intermediates.completedGradientEvents, CompletedGradientEvent(), activeCount);
      for (uint32_t bounce = 0; bounce < pkg.settings.maxAdjointBounces && activeCount > 0; ++bounce) {
        pkg.random.number = seedGen();
        pkg.queue.fill(pkg.intermediates.countExtensionOut, static_cast<uint32_t>(0), 1);
        pkg.queue.fill(pkg.intermediates.countCompletedGradientEvents, static_cast<uint32_t>(0), 1);
        pkg.queue.fill(pkg.intermediates.hitRecords, WorldHit(), activeCount);
        pkg.queue.wait();
        s->adjointSegments += activeCount;
        launchAdjointIntersectKernel(pkg, activeCount, bounce);
        uint32_t completed = 0;
        pkg.queue.memcpy(&completed, pkg.intermediates.countCompletedGradientEvents, sizeof(uint32_t)).wait();
        completed = sycl::min(completed, pkg.intermediates.maxPendingAdjointStateCount);
        if (completed) launchAdjointTransportKernel(pkg, completed, static_cast<uint32_t>(cameraIndex));
        uint32_t nextCount = 0;
        pkg.queue.memcpy(&nextCount, pkg.intermediates.countExtensionOut, sizeof(uint32_t)).wait();
        pkg.queue.memcpy(pkg.intermediates.primaryRays, pkg.intermediates.extensionRaysA, nextCount * sizeof(RayState));
        pkg.queue.wait();
        activeCount = nextCount;
      }
    }
  }
  s->adjointMs = (omp_get_wtime() - t0) * 1e3;
  if (grad_opacity && n) std::memcpy(grad_opacity, s->gradOpacity.data(), n * sizeof(float));
  return 0;
}

// Photon records in deposit order (position, power, incoming direction,
// 3 floats each), their grid cell ids and the cell-sorted photon indices.
int ref_get_photons(const ref_scene* s, uint32_t* count, float* pos, float* power, float* dir, uint32_t* cell_id,
                    uint32_t* sorted) {
  const uint32_t n = std::min(s->photonCount, s->intermediates.map.photonCapacity);
  if (count) *count = n;
  for (uint32_t i = 0; i < n; ++i) {
    const DevicePhotonSurface& p = s->photons[i];
    for (int c = 0; c < 3; ++c) {
      if (pos) pos[3 * i + c] = p.position[c];
      if (power) power[3 * i + c] = p.power[c];
      if (dir) dir[3 * i + c] = p.incomingDirection[c];
    }
    if (cell_id) cell_id[i] = s->photonCellId[i];
    if (sorted) sorted[i] = s->sortedPhotonIndex[i];
  }
  return 0;
}

void ref_get_segments(const ref_scene* s, uint64_t* photon, uint64_t* adjoint) {
  if (photon) *photon = s->photonSegments;
  if (adjoint) *adjoint = s->adjointSegments;
}

// Wall time of the last calls: photon pass + grid, camera gather +
// post-process (last forward), adjoint pass (last backward).
void ref_get_times(const ref_scene* s, double* photon_ms, double* gather_ms, double* adjoint_ms) {
  if (photon_ms) *photon_ms = s->photonMs;
  if (gather_ms) *gather_ms = s->gatherMs;
  if (adjoint_ms) *adjoint_ms = s->adjointMs;
}

}  // extern "C"
