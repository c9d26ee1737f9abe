"""Scene descriptions for the adjoint surfel renderer.

A :class:`SceneArrays` holds the host-side data that ``SceneBuild::build``
collects in the reference (Pale/Renderer/SceneBuild.cpp:72-392): triangle
meshes with per-instance transforms and materials, pinhole cameras, and a
beta-surfel cloud in asset (file) order.  It is filled either by

* :func:`load_mitsuba_scene` -- the Mitsuba-XML subset Pale reads
  (Pale/Scene/SceneSerializer.cpp:71-356, Pale/Asset/MaterialBakerMitsuba.ixx)
  plus OBJ meshes and the custom surfel PLY schema
  (Pale/Asset/PLYPointLoader.ixx:156-188), or
* :func:`make_box_scene` -- the seeded synthetic Cornell-style box used for
  the throughput workloads (five 1x1 diffuse walls around [-0.5,0.5]^3 with
  the -y side open, a 0.25x0.25 area emitter under the ceiling, and
  uniformly placed surfels in [-0.4,0.4]^3).

All matrices are row-major float32 with y = M x.
"""
from __future__ import annotations

import dataclasses
import math
import os
import xml.etree.ElementTree as ET
from typing import Dict, List, Optional, Sequence

import numpy as np

POINT_FIELDS = ("position", "tangent_u", "tangent_v", "scale", "albedo", "opacity", "beta", "shape")
POINT_WIDTH = {"position": 3, "tangent_u": 3, "tangent_v": 3, "scale": 2, "albedo": 3,
               "opacity": 1, "beta": 1, "shape": 1}


def empty_points(n: int = 0) -> Dict[str, np.ndarray]:
    out = {}
    for k in POINT_FIELDS:
        w = POINT_WIDTH[k]
        out[k] = np.zeros((n, w) if w > 1 else (n,), np.float32)
    return out


def as_points(d: Dict[str, np.ndarray]) -> Dict[str, np.ndarray]:
    """Returns contiguous float32 copies with the canonical shapes."""
    n = int(np.asarray(d["position"]).reshape(-1, 3).shape[0])
    out = {}
    for k in POINT_FIELDS:
        w = POINT_WIDTH[k]
        if k not in d or d[k] is None:
            v = np.zeros((n, w) if w > 1 else (n,), np.float32)
        else:
            v = np.ascontiguousarray(np.asarray(d[k], np.float32).reshape((n, w) if w > 1 else (n,)))
        out[k] = v
    return out


@dataclasses.dataclass
class SceneArrays:
    vertices: np.ndarray            # (V,3) f32, object space
    triangles: np.ndarray           # (T,3) u32
    mesh_ranges: np.ndarray         # (M,2) u32 first triangle, count
    materials: np.ndarray           # (K,4) f32 base colour rgb, power
    instance_mesh: np.ndarray       # (I,) u32
    instance_material: np.ndarray   # (I,) u32
    object_to_world: np.ndarray     # (I,4,4) f32
    world_to_object: np.ndarray     # (I,4,4) f32
    camera_inv_view: np.ndarray     # (C,4,4) f32 camera -> world
    camera_forward: np.ndarray      # (C,3) f32
    camera_fovy: np.ndarray         # (C,) f32 degrees
    camera_size: np.ndarray         # (C,2) u32 width, height
    camera_names: List[str]
    camera_adjoint: np.ndarray      # (C,) bool: camera takes part in the adjoint pass
    points: Dict[str, np.ndarray]   # asset-order surfels
    instance_names: List[str] = dataclasses.field(default_factory=list)

    @property
    def num_points(self) -> int:
        return int(self.points["position"].shape[0])

    def with_points(self, points: Dict[str, np.ndarray]) -> "SceneArrays":
        return dataclasses.replace(self, points=as_points(points))

    def with_cameras(self, idx: Sequence[int]) -> "SceneArrays":
        idx = list(idx)
        return dataclasses.replace(
            self, camera_inv_view=self.camera_inv_view[idx], camera_forward=self.camera_forward[idx],
            camera_fovy=self.camera_fovy[idx], camera_size=self.camera_size[idx],
            camera_names=[self.camera_names[i] for i in idx], camera_adjoint=self.camera_adjoint[idx])


# --------------------------------------------------------------- transforms
def _rotation(axis, angle_deg: float) -> np.ndarray:
    axis = np.asarray(axis, np.float64)
    n = np.linalg.norm(axis)
    R = np.eye(4)
    if n == 0.0:
        return R
    x, y, z = axis / n
    a = math.radians(angle_deg)
    c, s, C = math.cos(a), math.sin(a), 1.0 - math.cos(a)
    R[:3, :3] = [[c + x * x * C, x * y * C - z * s, x * z * C + y * s],
                 [y * x * C + z * s, c + y * y * C, y * z * C - x * s],
                 [z * x * C - y * s, z * y * C + x * s, c + z * z * C]]
    return R


def trs(translate=(0, 0, 0), axis=(1, 0, 0), angle_deg=0.0, scale=(1, 1, 1)) -> np.ndarray:
    """translate * rotate * scale (TransformComponent::getTransform,
    Pale/Scene/Components.ixx:68-73), float64."""
    T = np.eye(4)
    T[:3, 3] = translate
    S = np.diag([scale[0], scale[1], scale[2], 1.0])
    return T @ _rotation(axis, angle_deg) @ S


def look_at(eye, target, up) -> np.ndarray:
    """World -> camera view matrix of glm::lookAt (right handed, -Z forward)."""
    eye, target, up = (np.asarray(v, np.float64) for v in (eye, target, up))
    f = target - eye
    f /= np.linalg.norm(f)
    s = np.cross(f, up)
    s /= np.linalg.norm(s)
    u = np.cross(s, f)
    V = np.eye(4)
    V[0, :3], V[1, :3], V[2, :3] = s, u, -f
    V[0, 3], V[1, 3], V[2, 3] = -s @ eye, -u @ eye, f @ eye
    return V


def fov_y_degrees(fov: float, axis: str, width: int, height: int) -> float:
    """computeFovYDegrees (Pale/Scene/SceneSerializer.cpp:71-85)."""
    aspect = float(width) / float(height)
    if axis == "y":
        return float(fov)
    if axis == "x" or width <= height:
        fy = 2.0 * math.atan(math.tan(math.radians(fov) * 0.5) / aspect)
        return math.degrees(fy)
    return float(fov)


# ----------------------------------------------------------- scene builder
class _Builder:
    def __init__(self):
        self.vertices: List[np.ndarray] = []
        self.triangles: List[np.ndarray] = []
        self.mesh_ranges: List[tuple] = []
        self.mesh_index: Dict[str, int] = {}
        self.nv = 0
        self.nt = 0
        self.materials: List[tuple] = []
        self.inst_mesh: List[int] = []
        self.inst_mat: List[int] = []
        self.o2w: List[np.ndarray] = []
        self.inst_names: List[str] = []
        self.cams: List[dict] = []

    def add_mesh(self, key: str, verts: np.ndarray, tris: np.ndarray) -> int:
        if key in self.mesh_index:
            return self.mesh_index[key]
        verts = np.asarray(verts, np.float32).reshape(-1, 3)
        tris = np.asarray(tris, np.uint32).reshape(-1, 3) + self.nv
        self.vertices.append(verts)
        self.triangles.append(tris)
        self.mesh_ranges.append((self.nt, tris.shape[0]))
        self.nv += verts.shape[0]
        self.nt += tris.shape[0]
        self.mesh_index[key] = len(self.mesh_ranges) - 1
        return self.mesh_index[key]

    def add_material(self, rgb, power=0.0) -> int:
        self.materials.append((float(rgb[0]), float(rgb[1]), float(rgb[2]), float(power)))
        return len(self.materials) - 1

    def add_instance(self, mesh: int, material: int, o2w: np.ndarray, name: str = ""):
        self.inst_mesh.append(mesh)
        self.inst_mat.append(material)
        self.o2w.append(np.asarray(o2w, np.float64))
        self.inst_names.append(name)

    def add_camera(self, name, eye, target, up, fovy_deg, width, height, adjoint=True):
        view = look_at(eye, target, up)
        inv = np.linalg.inv(view)
        fwd = inv[:3, :3] @ np.array([0.0, 0.0, -1.0])
        fwd /= np.linalg.norm(fwd)
        self.cams.append(dict(name=name, inv=inv, fwd=fwd, fovy=fovy_deg, w=int(width), h=int(height),
                              adjoint=bool(adjoint)))

    def finish(self, points: Dict[str, np.ndarray]) -> SceneArrays:
        o2w = np.stack(self.o2w) if self.o2w else np.zeros((0, 4, 4))
        w2o = np.stack([np.linalg.inv(m) for m in self.o2w]) if self.o2w else np.zeros((0, 4, 4))
        cams = self.cams
        return SceneArrays(
            vertices=np.concatenate(self.vertices).astype(np.float32) if self.vertices else np.zeros((0, 3), np.float32),
            triangles=np.concatenate(self.triangles).astype(np.uint32) if self.triangles else np.zeros((0, 3), np.uint32),
            mesh_ranges=np.asarray(self.mesh_ranges, np.uint32).reshape(-1, 2),
            materials=np.asarray(self.materials, np.float32).reshape(-1, 4),
            instance_mesh=np.asarray(self.inst_mesh, np.uint32),
            instance_material=np.asarray(self.inst_mat, np.uint32),
            object_to_world=o2w.astype(np.float32),
            world_to_object=w2o.astype(np.float32),
            camera_inv_view=np.asarray([c["inv"] for c in cams], np.float32).reshape(-1, 4, 4),
            camera_forward=np.asarray([c["fwd"] for c in cams], np.float32).reshape(-1, 3),
            camera_fovy=np.asarray([c["fovy"] for c in cams], np.float32),
            camera_size=np.asarray([(c["w"], c["h"]) for c in cams], np.uint32).reshape(-1, 2),
            camera_names=[c["name"] for c in cams],
            camera_adjoint=np.asarray([c["adjoint"] for c in cams], bool),
            points=as_points(points),
            instance_names=list(self.inst_names),
        )


# The unit quad of Assets/meshes/rectangle.obj: corners (+-1, +-1, 0), faces
# (2,3,1) and (2,4,3), front normal +z.
QUAD_VERTS = np.array([[-1, -1, 0], [1, -1, 0], [-1, 1, 0], [1, 1, 0]], np.float32)
QUAD_TRIS = np.array([[1, 2, 0], [1, 3, 2]], np.uint32)


# -------------------------------------------------------- synthetic scenes
def make_surfels(n: int, seed: int = 1234, lo: float = -0.4, hi: float = 0.4) -> Dict[str, np.ndarray]:
    """Seeded beta surfels: position U[lo,hi]^3, normal uniform on S^2,
    tangent from a Frisvad basis rotated by a uniform in-plane angle,
    tv = n x tu, scales lognormal(ln 0.01, 0.3), albedo U[0.2,0.9]^3,
    opacity U[0.3,1], beta U[-1,1]."""
    rng = np.random.default_rng(seed)
    pos = rng.uniform(lo, hi, (n, 3))
    z = rng.uniform(-1.0, 1.0, n)
    phi = rng.uniform(0.0, 2 * np.pi, n)
    r = np.sqrt(np.maximum(0.0, 1 - z * z))
    nrm = np.stack([r * np.cos(phi), r * np.sin(phi), z], 1)
    sign = np.where(nrm[:, 2] >= 0, 1.0, -1.0)
    a = -1.0 / (sign + nrm[:, 2])
    b = nrm[:, 0] * nrm[:, 1] * a
    t0 = np.stack([1 + sign * nrm[:, 0] ** 2 * a, sign * b, -sign * nrm[:, 0]], 1)
    b0 = np.stack([b, sign + nrm[:, 1] ** 2 * a, -nrm[:, 1]], 1)
    ang = rng.uniform(0.0, 2 * np.pi, n)[:, None]
    tu = np.cos(ang) * t0 + np.sin(ang) * b0
    tu /= np.linalg.norm(tu, axis=1, keepdims=True)
    tv = np.cross(nrm, tu)
    scale = np.exp(rng.normal(math.log(0.01), 0.3, (n, 2)))
    albedo = rng.uniform(0.2, 0.9, (n, 3))
    opacity = rng.uniform(0.3, 1.0, n)
    beta = rng.uniform(-1.0, 1.0, n)
    return as_points(dict(position=pos, tangent_u=tu, tangent_v=tv, scale=scale, albedo=albedo,
                          opacity=opacity, beta=beta, shape=np.zeros(n)))


def jitter_target(points: Dict[str, np.ndarray], seed: int = 5678, pos_sigma=0.005,
                  albedo_sigma=0.05) -> Dict[str, np.ndarray]:
    """Target cloud: positions += N(0, 0.005), albedo += N(0, 0.05) clamped."""
    rng = np.random.default_rng(seed)
    out = {k: v.copy() for k, v in points.items()}
    out["position"] = (out["position"] + rng.normal(0, pos_sigma, out["position"].shape)).astype(np.float32)
    out["albedo"] = np.clip(out["albedo"] + rng.normal(0, albedo_sigma, out["albedo"].shape), 0, 1).astype(np.float32)
    return out


def ring_cameras(count: int, radius: float = 1.5, height: float = 0.0, offset: float = 0.0):
    """Eye positions on a horizontal circle; camera 0 (offset 0) looks
    through the open -y side of the box.  `offset` rotates the ring by a
    fraction of the camera spacing."""
    eyes = []
    for k in range(count):
        th = 2.0 * math.pi * (k + offset) / count
        eyes.append((radius * math.sin(th), -radius * math.cos(th), height))
    return eyes


def make_box_scene(n_surfels: int, cameras: int = 1, resolution: int = 256, fovy: float = 40.0,
                   seed: int = 1234, radiance: float = 15.0,
                   points: Optional[Dict[str, np.ndarray]] = None, ring_offset: float = 0.0,
                   resolutions: Optional[Sequence[int]] = None) -> SceneArrays:
    """The synthetic box of the throughput workloads.

    Cameras: `cameras` positions on the ring, each at `resolution`, or with
    `resolutions` one camera per (position, resolution), camera index
    position * len(resolutions) + k, named camera{position}_{resolution}.

    Walls are instances of the rectangle quad (front faces inward), albedo
    0.8 (floor, ceiling, back), 0.6/0.1/0.1 (x = -0.5) and 0.1/0.6/0.1
    (x = +0.5).  The emitter is a 0.25x0.25 quad at z = 0.499 facing -z;
    Pale parametrises emitters by power with L_e = power/(pi*A), so a
    radiance of 15 is power 15*pi*0.0625.
    """
    B = _Builder()
    quad = B.add_mesh("rectangle", QUAD_VERTS, QUAD_TRIS)
    white = B.add_material((0.8, 0.8, 0.8))
    red = B.add_material((0.6, 0.1, 0.1))
    green = B.add_material((0.1, 0.6, 0.1))
    light = B.add_material((1.0, 1.0, 1.0), power=radiance * math.pi * 0.0625)
    h = (0.5, 0.5, 1.0)
    B.add_instance(quad, white, trs((0, 0, -0.5), scale=h), "floor")
    B.add_instance(quad, white, trs((0, 0, 0.5), (1, 0, 0), 180.0, h), "ceiling")
    B.add_instance(quad, white, trs((0, 0.5, 0), (1, 0, 0), 90.0, h), "back")
    B.add_instance(quad, red, trs((-0.5, 0, 0), (0, 1, 0), 90.0, h), "left")
    B.add_instance(quad, green, trs((0.5, 0, 0), (0, 1, 0), -90.0, h), "right")
    B.add_instance(quad, light, trs((0, 0, 0.499), (1, 0, 0), 180.0, (0.125, 0.125, 1.0)), "light")
    for k, eye in enumerate(ring_cameras(cameras, offset=ring_offset)):
        if resolutions:
            for res in resolutions:
                B.add_camera(f"camera{k}_{res}", eye, (0, 0, 0), (0, 0, 1), fovy, res, res)
        else:
            B.add_camera(f"camera{k}", eye, (0, 0, 0), (0, 0, 1), fovy, resolution, resolution)
    if points is None:
        points = make_surfels(n_surfels, seed)
    return B.finish(points)


# ------------------------------------------------------------- file I/O
def load_obj(path: str):
    """Positions and triangle fans of a Wavefront OBJ file."""
    verts, tris = [], []
    with open(path, "r") as f:
        for line in f:
            p = line.split()
            if not p:
                continue
            if p[0] == "v":
                verts.append([float(x) for x in p[1:4]])
            elif p[0] == "f":
                idx = []
                for tok in p[1:]:
                    i = int(tok.split("/")[0])
                    idx.append(i - 1 if i > 0 else len(verts) + i)
                for k in range(1, len(idx) - 1):
                    tris.append([idx[0], idx[k], idx[k + 1]])
    return np.asarray(verts, np.float32).reshape(-1, 3), np.asarray(tris, np.uint32).reshape(-1, 3)


_PLY_TYPES = {"char": "i1", "int8": "i1", "uchar": "u1", "uint8": "u1", "short": "i2", "int16": "i2",
              "ushort": "u2", "uint16": "u2", "int": "i4", "int32": "i4", "uint": "u4", "uint32": "u4",
              "float": "f4", "float32": "f4", "double": "f8", "float64": "f8"}


def read_ply_vertices(path: str) -> Dict[str, np.ndarray]:
    """Vertex properties of an ascii or binary_little_endian PLY file."""
    with open(path, "rb") as f:
        header = []
        while True:
            line = f.readline()
            if not line:
                raise RuntimeError(f"PLY header of {path} is truncated")
            s = line.decode("ascii", "replace").strip()
            header.append(s)
            if s == "end_header":
                break
        body = f.read()
    fmt, count, props, cur = None, 0, [], None
    for s in header:
        p = s.split()
        if not p:
            continue
        if p[0] == "format":
            fmt = p[1]
        elif p[0] == "element":
            cur = p[1]
            if cur == "vertex":
                count = int(p[2])
        elif p[0] == "property" and cur == "vertex" and p[1] != "list":
            props.append((p[2], _PLY_TYPES[p[1]]))
    if fmt == "ascii":
        vals = []
        for line in body.decode("ascii", "replace").splitlines():
            line = line.split("#")[0].strip()
            if line:
                vals.append([float(x) for x in line.split()[: len(props)]])
            if len(vals) == count:
                break
        arr = np.asarray(vals, np.float64).reshape(count, len(props))
        return {name: arr[:, i].astype(np.float32) for i, (name, _) in enumerate(props)}
    if fmt != "binary_little_endian":
        raise RuntimeError(f"unsupported PLY format {fmt}")
    dt = np.dtype([(name, "<" + t) for name, t in props])
    rec = np.frombuffer(body, dt, count)
    return {name: rec[name].astype(np.float32) for name, _ in props}


_CUSTOM = ("x", "y", "z", "tu_x", "tu_y", "tu_z", "tv_x", "tv_y", "tv_z", "su", "sv",
           "albedo_r", "albedo_g", "albedo_b", "opacity")


_SPLAT = ("x", "y", "z", "f_dc_0", "f_dc_1", "f_dc_2", "opacity", "scale_0", "scale_1",
          "rot_0", "rot_1", "rot_2", "rot_3")


def _norm_rows(a: np.ndarray) -> np.ndarray:
    return a / np.sqrt(np.sum(a * a, axis=1, keepdims=True, dtype=np.float32))


def canonical_frames(tu: np.ndarray, tv: np.ndarray):
    """canonicalizeFrameFaceUp (PLYPointLoader.ixx:71-97): unit tangents,
    Gram-Schmidt of the second against the first (the y axis, or x when the
    first is near y, for a degenerate pair), and the second flipped so that
    the normal tu x tv has z >= 0."""
    tu = _norm_rows(tu.astype(np.float32))
    tv = _norm_rows(tv.astype(np.float32))
    ortho = tv - np.sum(tv * tu, axis=1, keepdims=True) * tu
    bad = np.sum(ortho * ortho, axis=1) < np.float32(1e-6)
    if bad.any():
        alt = np.where((np.abs(tu[:, 1]) < 0.9)[:, None], np.array([0, 1, 0], np.float32),
                       np.array([1, 0, 0], np.float32))
        alt = alt - np.sum(alt * tu, axis=1, keepdims=True) * tu
        ortho = np.where(bad[:, None], alt, ortho)
    tv = _norm_rows(ortho)
    flip = np.cross(tu, tv)[:, 2] < 0
    tv = np.where(flip[:, None], -tv, tv)
    return tu.astype(np.float32), tv.astype(np.float32)


def _splat_points(v: Dict[str, np.ndarray]) -> Dict[str, np.ndarray]:
    """The Gaussian-splat schema as surfels (PLYPointLoader.ixx:294-388):
    radii 2 exp(scale_0/1), opacity sigmoid(opacity) (arguments clamped to
    [-20, 20]), albedo 0.8 (the loader computes the DC colour but keeps a
    constant albedo), tangents the first two columns of the normalised
    rotation quaternion (w, x, y, z), then orthonormalised (the second
    falls back to +y when it vanishes); beta and shape 0."""
    n = v["x"].shape[0]
    f = lambda k: v[k].astype(np.float32)
    c = lambda x: np.clip(x, np.float32(-20), np.float32(20))
    q = np.stack([f("rot_0"), f("rot_1"), f("rot_2"), f("rot_3")], 1)
    q = q / np.sqrt(np.sum(q * q, axis=1, keepdims=True, dtype=np.float32))
    w, x, y, z = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    one, two = np.float32(1), np.float32(2)
    tu = np.stack([one - two * (y * y + z * z), two * (x * y + w * z), two * (x * z - w * y)], 1)
    tv = np.stack([two * (x * y - w * z), one - two * (x * x + z * z), two * (y * z + w * x)], 1)
    lu = np.sum(tu * tu, axis=1, keepdims=True)
    tu = np.where(lu > 0, tu / np.sqrt(np.where(lu > 0, lu, 1)), tu)
    tv = tv - np.sum(tv * tu, axis=1, keepdims=True) * tu
    lv = np.sum(tv * tv, axis=1, keepdims=True)
    tv = np.where(lv > 0, tv / np.sqrt(np.where(lv > 0, lv, 1)), np.array([[0, 1, 0]], np.float32))
    scale = np.stack([np.exp(c(f("scale_0"))), np.exp(c(f("scale_1")))], 1) * two
    opacity = one / (one + np.exp(-c(f("opacity"))))
    return as_points(dict(position=np.stack([f("x"), f("y"), f("z")], 1), tangent_u=tu, tangent_v=tv,
                          scale=scale, albedo=np.full((n, 3), 0.8, np.float32), opacity=opacity,
                          beta=np.zeros(n, np.float32), shape=np.zeros(n, np.float32)))


def load_surfel_ply(path: str) -> Dict[str, np.ndarray]:
    """PLYPointLoader (PLYPointLoader.ixx:144-390): the custom surfel schema
    (:156-161; tangent frames canonicalised face up, albedo clamped to
    [0, 1]; beta and shape default to 0 when absent) or the Gaussian-splat
    schema (:163-167, converted as _splat_points describes)."""
    v = read_ply_vertices(path)
    if all(k in v for k in _CUSTOM):
        n = v["x"].shape[0]
        st = lambda *ks: np.stack([v[k] for k in ks], 1).astype(np.float32)
        tu, tv = canonical_frames(st("tu_x", "tu_y", "tu_z"), st("tv_x", "tv_y", "tv_z"))
        return as_points(dict(position=st("x", "y", "z"), tangent_u=tu, tangent_v=tv, scale=st("su", "sv"),
                              albedo=np.clip(st("albedo_r", "albedo_g", "albedo_b"), 0, 1), opacity=v["opacity"],
                              beta=v.get("beta", np.zeros(n, np.float32)),
                              shape=v.get("shape", np.zeros(n, np.float32))))
    if all(k in v for k in _SPLAT):
        return _splat_points(v)
    raise RuntimeError(f"{path}: unsupported vertex schema")


def write_surfel_ply(path: str, points: Dict[str, np.ndarray]):
    """Writes the custom surfel schema as binary_little_endian."""
    p = as_points(points)
    n = p["position"].shape[0]
    names = list(_CUSTOM) + ["beta", "shape"]
    cols = np.concatenate([p["position"], p["tangent_u"], p["tangent_v"], p["scale"], p["albedo"],
                           p["opacity"][:, None], p["beta"][:, None], p["shape"][:, None]], 1)
    head = ["ply", "format binary_little_endian 1.0", f"element vertex {n}"]
    head += [f"property float {k}" for k in names] + ["end_header"]
    with open(path, "wb") as f:
        f.write(("\n".join(head) + "\n").encode("ascii"))
        f.write(np.ascontiguousarray(cols, "<f4").tobytes())


def _floats(s: str):
    return [float(x) for x in s.replace(",", " ").split()]


def load_mitsuba_scene(asset_root: str, scene_xml: str, points: Dict[str, np.ndarray]) -> SceneArrays:
    """The Mitsuba-XML subset of SceneSerializer::deserialize: perspective
    sensors with fov / fov_axis / lookat / film size / adjoint_source, diffuse
    bsdfs, obj/ply shapes with to_world translate/rotate/scale and area
    emitters with colour and power."""
    path = scene_xml if os.path.isabs(scene_xml) else os.path.join(asset_root, scene_xml)
    root = ET.parse(path).getroot()
    B = _Builder()

    def child_by(node, tag, name):
        for c in node.findall(tag):
            if c.get("name") == name:
                return c
        return None

    for sensor in root.findall("sensor"):
        film = sensor.find("film")
        W = int(child_by(film, "integer", "width").get("value"))
        H = int(child_by(film, "integer", "height").get("value"))
        fov_n = child_by(sensor, "float", "fov")
        fov = float(fov_n.get("value")) if fov_n is not None else 45.0
        ax_n = child_by(sensor, "string", "fov_axis")
        axis = ax_n.get("value") if ax_n is not None else "smaller"
        la = sensor.find("transform").find("lookat")
        adj = True
        for tag in ("boolean", "float"):
            n = child_by(sensor, tag, "adjoint_source")
            if n is not None:
                v = n.get("value", "").strip().lower()
                adj = v in ("true", "1", "yes", "on") or (v not in ("false", "0", "no", "off") and
                                                         _try_float(v, 1.0) != 0.0)
        B.add_camera(sensor.get("id", f"camera{len(B.cams)}"), _floats(la.get("origin")),
                     _floats(la.get("target")), _floats(la.get("up")),
                     fov_y_degrees(fov, axis, W, H), W, H, adj)

    bsdfs = {}
    for b in root.findall("bsdf"):
        rgb = child_by(b, "rgb", "reflectance")
        bsdfs[b.get("id")] = _floats(rgb.get("value")) if rgb is not None else [0.5, 0.5, 0.5]

    for shape in root.findall("shape"):
        kind = shape.get("type", "")
        fn = child_by(shape, "string", "filename")
        if fn is None:
            continue
        mesh_path = os.path.join(asset_root, fn.get("value"))
        if kind == "obj":
            verts, tris = load_obj(mesh_path)
        else:
            raise RuntimeError(f"shape type {kind} is not supported")
        mesh = B.add_mesh(mesh_path, verts, tris)
        t, axis, ang, sc = (0, 0, 0), (1, 0, 0), 0.0, (1, 1, 1)
        tw = child_by(shape, "transform", "to_world")
        if tw is not None:
            for c in tw:
                g = lambda k, d: float(c.get(k, d))
                if c.tag == "translate":
                    t = (g("x", 0), g("y", 0), g("z", 0))
                elif c.tag == "scale":
                    sc = (g("x", 1), g("y", 1), g("z", 1))
                elif c.tag == "rotate":
                    axis, ang = (g("x", 0), g("y", 0), g("z", 0)), g("angle", 0)
        em = shape.find("emitter")
        if em is not None and em.get("type", "area") == "area":
            col = child_by(em, "rgb", "color")
            pw = child_by(em, "float", "power")
            mat = B.add_material(_floats(col.get("value")) if col is not None else (0.5, 0.5, 0.5),
                                 float(pw.get("value")) if pw is not None else 0.0)
        else:
            ref = shape.find("ref")
            inline = shape.find("bsdf")
            if ref is not None and ref.get("id") in bsdfs:
                rgb = bsdfs[ref.get("id")]
            elif inline is not None and child_by(inline, "rgb", "reflectance") is not None:
                rgb = _floats(child_by(inline, "rgb", "reflectance").get("value"))
            else:
                rgb = [0.5, 0.5, 0.5]
            mat = B.add_material(rgb, 0.0)
        B.add_instance(mesh, mat, trs(t, axis, ang, sc), shape.get("id", ""))
    return B.finish(points)


def _try_float(s: str, default: float) -> float:
    try:
        return float(s)
    except ValueError:
        return default


def resolve_point_cloud(asset_root: str, point_cloud_file: str) -> str:
    """Pale imports the point cloud from <assetRoot>/PointClouds/<file>
    (pale_bindings.cpp:90-96); a path relative to the asset root or an
    absolute path is accepted too."""
    name = point_cloud_file or "initial.ply"
    for cand in (os.path.join(asset_root, "PointClouds", name), os.path.join(asset_root, name), name):
        if os.path.isfile(cand):
            return cand
    raise FileNotFoundError(f"point cloud {name} not found under {asset_root}")
