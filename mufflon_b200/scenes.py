"""Procedural scenes for the path-tracer workloads (seeded, synthetic).

The reference quotes no public scene corpus for this path (its ``testscenes``
submodule is empty), so every workload is generated here from a seed:

* ``cornell_box``       -- 5 wall quads, two 12-triangle boxes with a random
                           yaw, one emissive ceiling quad (radiance 15),
                           Lambert albedo U[0.2, 0.8]^3 per object; 256x256.
* ``displaced_icosphere`` -- icosphere subdivided ``subdiv`` times (8 gives
                           1 310 720 triangles), radius 1, radial displacement
                           1 + 0.05 * n(p) with seeded 3-octave value noise,
                           GGX/Smith Torrance material with roughness
                           U[0.1, 0.5], a Lambert ground quad, one point light
                           and a monochrome environment; 1920x1080.
* ``instanced_scene``   -- 10 noise-displaced spheres and tori (triangle
                           counts log-uniform), many randomly rotated and
                           scaled instances in a 100^3 box and one object of
                           analytic spheres.
* ``displaced_plane``   -- a noise-displaced grid of quads split into
                           triangles (batched workload).

A scene is a :class:`SceneSpec` of flat numpy arrays. The same spec feeds the
library through its C API (``mufflon_b200.bindings``) and the CPU oracle.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional

import numpy as np

MAT_LAMBERT = 0
MAT_TORRANCE = 1
MAT_EMISSIVE = 2


@dataclasses.dataclass
class LodSpec:
    vertices: np.ndarray            # (V, 3) float32
    normals: np.ndarray             # (V, 3) float32
    uvs: np.ndarray                 # (V, 2) float32
    triangles: np.ndarray           # (T, 3) uint32
    quads: np.ndarray               # (Q, 4) uint32
    face_materials: np.ndarray      # (T + Q,) uint16
    spheres: np.ndarray             # (S, 4) float32 center xyz, radius
    sphere_materials: np.ndarray    # (S,) uint16
    name: str = "object"

    @property
    def num_prims(self) -> int:
        return len(self.triangles) + len(self.quads) + len(self.spheres)


@dataclasses.dataclass
class MaterialSpec:
    type: int
    albedo: tuple = (0.5, 0.5, 0.5)
    roughness: tuple = (0.3, 0.3)
    radiance: tuple = (0.0, 0.0, 0.0)
    scale: tuple = (1.0, 1.0, 1.0)
    albedo_texture: int = -1
    name: str = "material"
    shadowing: int = 1                  # Torrance: 1 Smith, 0 V-cavity (core_interface.h ShadowingModel)
    alpha_texture: int = -1             # cut-out texture (first channel < 0.5 is transparent), -1: opaque


@dataclasses.dataclass
class SceneSpec:
    lods: List[LodSpec]
    world_to_instance: np.ndarray   # (I, 12) float32
    instance_lod: np.ndarray        # (I,) uint32
    materials: List[MaterialSpec]
    point_lights: np.ndarray        # (L, 6) float32 position, intensity
    background: Optional[tuple]     # ((r, g, b) color, (r, g, b) scale) or None
    cam_pos: tuple
    cam_dir: tuple
    cam_up: tuple
    vfov: float                     # radians
    width: int
    height: int
    textures: list = dataclasses.field(default_factory=list)  # (H, W, 4) float32 arrays
    name: str = "scene"

    @property
    def num_prims(self) -> int:
        return sum(l.num_prims for l in self.lods)


def _empty_spheres():
    return np.zeros((0, 4), np.float32), np.zeros((0,), np.uint16)


def _lod(vertices, normals, uvs, tris=None, quads=None, mats=None, spheres=None, sphere_mats=None, name="object"):
    tris = np.zeros((0, 3), np.uint32) if tris is None else np.asarray(tris, np.uint32).reshape(-1, 3)
    quads = np.zeros((0, 4), np.uint32) if quads is None else np.asarray(quads, np.uint32).reshape(-1, 4)
    if spheres is None:
        spheres, sphere_mats = _empty_spheres()
    mats = np.zeros((len(tris) + len(quads),), np.uint16) if mats is None else np.asarray(mats, np.uint16)
    return LodSpec(np.ascontiguousarray(vertices, np.float32), np.ascontiguousarray(normals, np.float32),
                   np.ascontiguousarray(uvs, np.float32), np.ascontiguousarray(tris), np.ascontiguousarray(quads),
                   np.ascontiguousarray(mats), np.ascontiguousarray(spheres, np.float32),
                   np.ascontiguousarray(sphere_mats, np.uint16), name)


def identity34():
    return np.array([1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0], np.float32)


def _quad(p0, p1, p2, p3):
    """Four corners of a quad with the normal cross(p1 - p0, p3 - p0)."""
    p = np.array([p0, p1, p2, p3], np.float32)
    n = np.cross(p[1] - p[0], p[3] - p[0])
    n = n / np.linalg.norm(n)
    return p, np.tile(n, (4, 1)).astype(np.float32)


def _box_mesh(half):
    """Axis-aligned box centred at the origin, 6 faces x 2 triangles, outward winding."""
    hx, hy, hz = half
    c = np.array([[-hx, -hy, -hz], [hx, -hy, -hz], [hx, hy, -hz], [-hx, hy, -hz],
                  [-hx, -hy, hz], [hx, -hy, hz], [hx, hy, hz], [-hx, hy, hz]], np.float32)
    faces = [(0, 3, 2, 1), (4, 5, 6, 7), (0, 1, 5, 4), (3, 7, 6, 2), (0, 4, 7, 3), (1, 2, 6, 5)]
    verts, norms, uvs, tris = [], [], [], []
    for f in faces:
        p = c[list(f)]
        n = np.cross(p[1] - p[0], p[3] - p[0])
        n /= np.linalg.norm(n)
        base = len(verts)
        verts += list(p)
        norms += [n] * 4
        uvs += [(0, 0), (1, 0), (1, 1), (0, 1)]
        tris += [(base, base + 1, base + 2), (base, base + 2, base + 3)]
    return (np.array(verts, np.float32), np.array(norms, np.float32), np.array(uvs, np.float32),
            np.array(tris, np.uint32))


def _w2i_from_rt(rot, trans, scale=1.0):
    """World-to-instance matrix (3x4 row-major) of x_world = R * (s * x_obj) + t."""
    R = np.asarray(rot, np.float64)
    inv_r = R.T / scale
    inv_t = -inv_r @ np.asarray(trans, np.float64)
    m = np.concatenate([inv_r, inv_t[:, None]], axis=1)
    return m.astype(np.float32).reshape(12)


def cornell_box(seed: int = 0, width: int = 256, height: int = 256) -> SceneSpec:
    rng = np.random.default_rng(seed)
    mats = []
    for i in range(5):  # walls(floor/ceiling/back), left, right, box0, box1
        mats.append(MaterialSpec(MAT_LAMBERT, albedo=tuple(float(x) for x in rng.uniform(0.2, 0.8, 3)), name=f"lambert{i}"))
    mats.append(MaterialSpec(MAT_EMISSIVE, radiance=(15.0, 15.0, 15.0), name="light"))
    # walls: inward-facing quads
    walls = [
        _quad((-1, -1, -1), (-1, -1, 1), (1, -1, 1), (1, -1, -1)),   # floor, normal +y
        _quad((-1, 1, -1), (1, 1, -1), (1, 1, 1), (-1, 1, 1)),       # ceiling, normal -y
        _quad((-1, -1, -1), (1, -1, -1), (1, 1, -1), (-1, 1, -1)),   # back, normal +z
        _quad((-1, -1, -1), (-1, 1, -1), (-1, 1, 1), (-1, -1, 1)),   # left, normal +x
        _quad((1, -1, -1), (1, -1, 1), (1, 1, 1), (1, 1, -1)),       # right, normal -x
    ]
    wv = np.concatenate([w[0] for w in walls])
    wn = np.concatenate([w[1] for w in walls])
    wuv = np.tile(np.array([(0, 0), (1, 0), (1, 1), (0, 1)], np.float32), (5, 1))
    wq = np.arange(20, dtype=np.uint32).reshape(5, 4)
    lods = [_lod(wv, wn, wuv, quads=wq, mats=np.array([0, 0, 0, 1, 2], np.uint16), name="walls")]
    w2i = [identity34()]
    inst_lod = [0]
    for b in range(2):
        edge = rng.uniform(0.3, 0.7, 3)
        yaw = float(rng.uniform(0.0, 2.0 * math.pi))
        v, n, uv, t = _box_mesh(edge / 2.0)
        lods.append(_lod(v, n, uv, tris=t, mats=np.full(12, 3 + b, np.uint16), name=f"box{b}"))
        cx = -0.45 + 0.9 * b + float(rng.uniform(-0.1, 0.1))
        cz = float(rng.uniform(-0.5, 0.3))
        rot = np.array([[math.cos(yaw), 0, math.sin(yaw)], [0, 1, 0], [-math.sin(yaw), 0, math.cos(yaw)]])
        w2i.append(_w2i_from_rt(rot, (cx, -1.0 + edge[1] / 2.0, cz)))
        inst_lod.append(len(lods) - 1)
    # ceiling light, facing down, just below the ceiling
    a, y = 0.25, 0.998
    lp, ln = _quad((-a, y, -a), (a, y, -a), (a, y, a), (-a, y, a))
    lods.append(_lod(lp, ln, np.array([(0, 0), (1, 0), (1, 1), (0, 1)], np.float32),
                     quads=np.arange(4, dtype=np.uint32).reshape(1, 4), mats=np.array([5], np.uint16), name="light"))
    w2i.append(identity34())
    inst_lod.append(len(lods) - 1)
    return SceneSpec(lods, np.array(w2i, np.float32), np.array(inst_lod, np.uint32), mats,
                     np.zeros((0, 6), np.float32), None,
                     (0.0, 0.0, 3.6), (0.0, 0.0, -1.0), (0.0, 1.0, 0.0), math.radians(40.0),
                     width, height, name="cornell_box")


def smooth_noise_texture(seed: int, size: int = 512, lo: float = 0.1, hi: float = 0.9) -> np.ndarray:
    """(size, size, 4) float32 RGBA texture: seeded Gaussian noise, low-pass
    filtered (periodic), scaled per channel to [lo, hi]; alpha 1."""
    rng = np.random.default_rng(seed)
    f = np.fft.fftfreq(size)
    fx, fy = np.meshgrid(f, f)
    lowpass = np.exp(-(fx ** 2 + fy ** 2) / (2 * (4.0 / size) ** 2))
    out = np.ones((size, size, 4), np.float32)
    for c in range(3):
        v = np.real(np.fft.ifft2(np.fft.fft2(rng.normal(size=(size, size))) * lowpass))
        v = (v - v.min()) / max(v.max() - v.min(), 1e-12)
        out[..., c] = (lo + (hi - lo) * v).astype(np.float32)
    return out


def cornell_box_textured(seed: int = 0, width: int = 512, height: int = 512, texture=None,
                         texture_size: int = 512) -> SceneSpec:
    """The Cornell box with its back wall in its own Lambert material whose
    albedo is texture 0 ((H, W, 4) float32; default a constant 0.5)."""
    spec = cornell_box(seed, width, height)
    tex = np.full((texture_size, texture_size, 4), 0.5, np.float32) if texture is None else np.asarray(texture, np.float32)
    tex = np.ascontiguousarray(tex)
    tex[..., 3] = 1.0
    walls = spec.lods[0]
    mats = walls.face_materials.copy()
    mats[2] = len(spec.materials)  # the back wall quad
    lods = [dataclasses.replace(walls, face_materials=mats)] + spec.lods[1:]
    materials = spec.materials + [MaterialSpec(MAT_LAMBERT, albedo=(0.5, 0.5, 0.5), albedo_texture=0, name="back_wall")]
    return dataclasses.replace(spec, lods=lods, materials=materials, textures=[tex], name="cornell_box_textured")


# ------------------------------------------------------------------ meshes
def value_noise3(p: np.ndarray, seed: int, octaves: int = 3) -> np.ndarray:
    """Seeded 3-octave value noise in [-1, 1] (trilinear lattice interpolation)."""
    rng = np.random.default_rng(seed)
    table = rng.uniform(-1.0, 1.0, 4096)
    perm = rng.permutation(4096)
    total = np.zeros(len(p), np.float64)
    amp, freq, norm = 1.0, 2.0, 0.0
    for _ in range(octaves):
        q = p * freq
        i = np.floor(q).astype(np.int64)
        f = q - i
        f = f * f * (3.0 - 2.0 * f)

        def lat(dx, dy, dz):
            h = perm[(i[:, 0] + dx) & 4095]
            h = perm[(h + i[:, 1] + dy) & 4095]
            h = perm[(h + i[:, 2] + dz) & 4095]
            return table[h]

        c00 = lat(0, 0, 0) * (1 - f[:, 0]) + lat(1, 0, 0) * f[:, 0]
        c10 = lat(0, 1, 0) * (1 - f[:, 0]) + lat(1, 1, 0) * f[:, 0]
        c01 = lat(0, 0, 1) * (1 - f[:, 0]) + lat(1, 0, 1) * f[:, 0]
        c11 = lat(0, 1, 1) * (1 - f[:, 0]) + lat(1, 1, 1) * f[:, 0]
        c0 = c00 * (1 - f[:, 1]) + c10 * f[:, 1]
        c1 = c01 * (1 - f[:, 1]) + c11 * f[:, 1]
        total += amp * (c0 * (1 - f[:, 2]) + c1 * f[:, 2])
        norm += amp
        amp *= 0.5
        freq *= 2.0
    return total / norm


def icosphere(subdiv: int):
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t],
                  [0, -1, -t], [0, 1, -t], [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4],
                  [11, 10, 2], [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8],
                  [3, 8, 9], [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], np.int64)
    for _ in range(subdiv):
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        es = np.sort(e, axis=1)
        key = es[:, 0] * (len(v) + 1) + es[:, 1]
        uniq, inv = np.unique(key, return_inverse=True)
        a = uniq // (len(v) + 1)
        b = uniq % (len(v) + 1)
        mid = v[a] + v[b]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        mid_idx = inv + len(v)
        nf = len(f)
        m01, m12, m20 = mid_idx[:nf], mid_idx[nf:2 * nf], mid_idx[2 * nf:]
        v = np.concatenate([v, mid])
        f = np.concatenate([np.stack([f[:, 0], m01, m20], 1), np.stack([f[:, 1], m12, m01], 1),
                            np.stack([f[:, 2], m20, m12], 1), np.stack([m01, m12, m20], 1)])
    return v, f


def vertex_normals(v: np.ndarray, f: np.ndarray) -> np.ndarray:
    fn = np.cross(v[f[:, 1]] - v[f[:, 0]], v[f[:, 2]] - v[f[:, 0]])
    n = np.zeros_like(v)
    for k in range(3):
        np.add.at(n, f[:, k], fn)
    n /= np.maximum(np.linalg.norm(n, axis=1, keepdims=True), 1e-30)
    return n


def spherical_uv(v: np.ndarray) -> np.ndarray:
    n = v / np.linalg.norm(v, axis=1, keepdims=True)
    u = np.arctan2(n[:, 2], n[:, 0]) / (2 * math.pi) + 0.5
    w = np.arccos(np.clip(-n[:, 1], -1, 1)) / math.pi
    return np.stack([u, w], 1)


def displaced_sphere_mesh(subdiv: int, seed: int, amplitude: float = 0.05):
    v, f = icosphere(subdiv)
    d = 1.0 + amplitude * value_noise3(v * 1.5, seed)
    v = v * d[:, None]
    return v, f


def torus_mesh(n_major: int, n_minor: int, R: float = 1.0, r: float = 0.35, seed: int = 0, amplitude: float = 0.03):
    i = np.arange(n_major)
    j = np.arange(n_minor)
    th, ph = np.meshgrid(i * 2 * math.pi / n_major, j * 2 * math.pi / n_minor, indexing="ij")
    x = (R + r * np.cos(ph)) * np.cos(th)
    z = (R + r * np.cos(ph)) * np.sin(th)
    y = r * np.sin(ph)
    v = np.stack([x, y, z], -1).reshape(-1, 3)
    d = 1.0 + amplitude * value_noise3(v * 2.0, seed)
    v = v * d[:, None]
    a = (i[:, None] * n_minor + j[None, :])
    b = (((i + 1) % n_major)[:, None] * n_minor + j[None, :])
    c = (((i + 1) % n_major)[:, None] * n_minor + ((j + 1) % n_minor)[None, :])
    e = (i[:, None] * n_minor + ((j + 1) % n_minor)[None, :])
    f = np.concatenate([np.stack([a, e, c], -1).reshape(-1, 3), np.stack([a, c, b], -1).reshape(-1, 3)])
    return v, f


def displaced_icosphere(seed: int = 0, subdiv: int = 8, width: int = 1920, height: int = 1080) -> SceneSpec:
    rng = np.random.default_rng(seed)
    v, f = displaced_sphere_mesh(subdiv, seed)
    n = vertex_normals(v, f)
    uv = spherical_uv(v)
    rough = float(rng.uniform(0.1, 0.5))
    mats = [MaterialSpec(MAT_TORRANCE, albedo=tuple(float(x) for x in rng.uniform(0.2, 0.8, 3)),
                         roughness=(rough, rough), name="ggx"),
            MaterialSpec(MAT_LAMBERT, albedo=tuple(float(x) for x in rng.uniform(0.2, 0.8, 3)), name="ground")]
    sphere = _lod(v, n, uv, tris=f.astype(np.uint32), mats=np.zeros(len(f), np.uint16), name="icosphere")
    gy, gs = -1.2, 12.0
    gp, gn = _quad((-gs, gy, -gs), (-gs, gy, gs), (gs, gy, gs), (gs, gy, -gs))
    ground = _lod(gp, gn, np.array([(0, 0), (1, 0), (1, 1), (0, 1)], np.float32),
                  quads=np.arange(4, dtype=np.uint32).reshape(1, 4), mats=np.array([1], np.uint16), name="ground")
    lights = np.array([[3.0, 4.0, 2.5, 40.0, 38.0, 35.0]], np.float32)
    return SceneSpec([sphere, ground], np.array([identity34(), identity34()], np.float32),
                     np.array([0, 1], np.uint32), mats, lights, ((0.25, 0.3, 0.4), (1.0, 1.0, 1.0)),
                     (0.0, 0.35, 3.4), (0.0, -0.1, -1.0), (0.0, 1.0, 0.0), math.radians(45.0),
                     width, height, name="displaced_icosphere")


def _random_rotation(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def instanced_scene(seed: int = 0, num_meshes: int = 10, num_instances: int = 4096, num_spheres: int = 20000,
                    tri_range=(10_000, 200_000), width: int = 1920, height: int = 1080) -> SceneSpec:
    rng = np.random.default_rng(seed)
    lods = []
    mats = []
    for m in range(num_meshes):
        target = math.exp(rng.uniform(math.log(tri_range[0]), math.log(tri_range[1])))
        if m % 2 == 0:
            sub = max(2, int(round(math.log(target / 20.0, 4))))
            v, f = displaced_sphere_mesh(sub, seed * 131 + m)
        else:
            nm = max(8, int(math.sqrt(target / 2.0 * 2.5)))
            nn = max(6, int(target / 2.0 / nm))
            v, f = torus_mesh(nm, nn, seed=seed * 131 + m)
        n = vertex_normals(v, f)
        uv = spherical_uv(v)
        if rng.uniform() < 0.5:
            r = float(rng.uniform(0.1, 0.5))
            mats.append(MaterialSpec(MAT_TORRANCE, albedo=tuple(float(x) for x in rng.uniform(0.2, 0.8, 3)), roughness=(r, r)))
        else:
            mats.append(MaterialSpec(MAT_LAMBERT, albedo=tuple(float(x) for x in rng.uniform(0.2, 0.8, 3))))
        lods.append(_lod(v, n, uv, tris=f.astype(np.uint32), mats=np.full(len(f), m, np.uint16), name=f"mesh{m}"))
    mats.append(MaterialSpec(MAT_LAMBERT, albedo=(0.6, 0.6, 0.6), name="spheres"))
    sph = np.concatenate([rng.uniform(0.0, 100.0, (num_spheres, 3)), rng.uniform(0.1, 1.0, (num_spheres, 1))], 1)
    lods.append(_lod(np.zeros((0, 3)), np.zeros((0, 3)), np.zeros((0, 2)), spheres=sph.astype(np.float32),
                     sphere_mats=np.full(num_spheres, num_meshes, np.uint16), name="spheres"))
    w2i, inst_lod = [], []
    for i in range(num_instances):
        rot = _random_rotation(rng)
        s = float(rng.uniform(0.5, 3.0))
        t = rng.uniform(0.0, 100.0, 3)
        w2i.append(_w2i_from_rt(rot, t, s))
        inst_lod.append(int(rng.integers(0, num_meshes)))
    w2i.append(identity34())
    inst_lod.append(num_meshes)
    cam = tuple(float(x) for x in rng.uniform(20.0, 80.0, 3))
    d = rng.normal(size=3)
    d /= np.linalg.norm(d)
    lights = np.array([[50.0, 50.0, 50.0, 4000.0, 4000.0, 4000.0]], np.float32)
    return SceneSpec(lods, np.array(w2i, np.float32), np.array(inst_lod, np.uint32), mats, lights,
                     ((0.3, 0.35, 0.45), (1.0, 1.0, 1.0)), cam, tuple(float(x) for x in d), (0.0, 1.0, 0.0),
                     math.radians(60.0), width, height, name="instanced_scene")


def displaced_plane(seed: int = 0, n: int = 224, width: int = 512, height: int = 512) -> SceneSpec:
    """n x n grid, 2 n^2 triangles (224 -> 100 352), displaced by value noise."""
    rng = np.random.default_rng(seed)
    xs = np.linspace(-5, 5, n + 1)
    X, Z = np.meshgrid(xs, xs, indexing="ij")
    P = np.stack([X, np.zeros_like(X), Z], -1).reshape(-1, 3)
    P[:, 1] = 0.3 * value_noise3(P * 0.4, seed)
    i = np.arange(n)
    a = (i[:, None] * (n + 1) + i[None, :])
    b = a + 1
    c = a + n + 2
    d = a + n + 1
    f = np.concatenate([np.stack([a, b, c], -1).reshape(-1, 3), np.stack([a, c, d], -1).reshape(-1, 3)])
    v = P
    nrm = vertex_normals(v, f)
    uv = np.stack([X.reshape(-1) / 10 + 0.5, Z.reshape(-1) / 10 + 0.5], 1)
    mats = [MaterialSpec(MAT_LAMBERT, albedo=tuple(float(x) for x in rng.uniform(0.2, 0.8, 3)))]
    lod = _lod(v, nrm, uv, tris=f.astype(np.uint32), mats=np.zeros(len(f), np.uint16), name="plane")
    lights = np.array([[0.0, 6.0, 0.0, 60.0, 60.0, 60.0]], np.float32)
    return SceneSpec([lod], np.array([identity34()], np.float32), np.array([0], np.uint32), mats, lights,
                     ((0.2, 0.2, 0.25), (1.0, 1.0, 1.0)), (0.0, 4.0, 8.0), (0.0, -0.5, -1.0), (0.0, 1.0, 0.0),
                     math.radians(50.0), width, height, name="displaced_plane")


def alpha_cutouts(seed: int = 0, width: int = 128, height: int = 128, background: bool = True) -> SceneSpec:
    """The Cornell box with cut-out surfaces (materials with an alpha texture, MaterialParams.alpha): a
    checkerboard quad panel, a strongly twisted (non-planar) quad, a triangle fence with stripes, and
    striped spheres in two instances (one rotated and scaled). Every cut-out kind of the reference's
    alpha test (intersection.cu:181-316) is hit, including the second root of quads and spheres."""
    spec = cornell_box(seed, width, height)
    rng = np.random.default_rng(seed + 101)
    checker = np.zeros((8, 8, 4), np.float32)
    checker[..., 0] = (np.add.outer(np.arange(8), np.arange(8)) % 2).astype(np.float32)
    stripes = np.zeros((1, 12, 4), np.float32)
    stripes[0, :, 0] = (np.arange(12) % 3 != 0).astype(np.float32) * 0.9
    spec.textures = [checker, stripes]
    base = len(spec.materials)
    spec.materials += [
        MaterialSpec(MAT_LAMBERT, albedo=tuple(float(x) for x in rng.uniform(0.3, 0.9, 3)), alpha_texture=0, name="panel"),
        MaterialSpec(MAT_TORRANCE, albedo=(0.8, 0.7, 0.5), roughness=(0.3, 0.3), alpha_texture=1, name="striped_glossy"),
        MaterialSpec(MAT_LAMBERT, albedo=(0.3, 0.6, 0.8), alpha_texture=1, name="fence"),
    ]
    uv4 = np.array([(0, 0), (1, 0), (1, 1), (0, 1)], np.float32)
    # checkerboard panel and a twisted quad
    pp, pn = _quad((-0.6, -0.7, 0.1), (0.6, -0.7, 0.1), (0.6, 0.5, 0.1), (-0.6, 0.5, 0.1))
    tw = np.array([(-0.9, 0.55, -0.6), (-0.1, 0.55, -0.2), (-0.1, 0.95, -0.9), (-0.9, 0.95, 0.2)], np.float32)
    tn = np.tile(np.array([0, 0, 1], np.float32), (4, 1))
    spec.lods.append(_lod(np.concatenate([pp, tw]), np.concatenate([pn, tn]), np.concatenate([uv4, uv4 * 3.0]),
                          quads=np.arange(8, dtype=np.uint32).reshape(2, 4),
                          mats=np.array([base, base], np.uint16), name="panels"))
    # triangle fence: 4 x 3 cells, two triangles each, uv along x
    nx, ny = 4, 3
    xs, ys = np.linspace(-0.9, 0.9, nx + 1), np.linspace(-1.0, -0.2, ny + 1)
    gv = np.array([(x, y, 0.55) for y in ys for x in xs], np.float32)
    guv = np.array([(4.0 * i / nx, j / ny) for j in range(ny + 1) for i in range(nx + 1)], np.float32)
    tris = []
    for j in range(ny):
        for i in range(nx):
            a0 = j * (nx + 1) + i
            tris += [(a0, a0 + 1, a0 + nx + 2), (a0, a0 + nx + 2, a0 + nx + 1)]
    spec.lods.append(_lod(gv, np.tile(np.array([0, 0, 1], np.float32), (len(gv), 1)), guv, tris=tris,
                          mats=np.full(len(tris), base + 2, np.uint16), name="fence"))
    # striped spheres, the object in two instances
    sph = np.array([(0.45, -0.55, -0.2, 0.3), (-0.5, -0.6, 0.35, 0.22), (0.2, 0.3, -0.4, 0.18)], np.float32)
    spec.lods.append(_lod(np.zeros((0, 3), np.float32), np.zeros((0, 3), np.float32), np.zeros((0, 2), np.float32),
                          spheres=sph, sphere_mats=np.full(3, base + 1, np.uint16), name="spheres"))
    yaw = 0.7
    rot = np.array([[math.cos(yaw), 0, math.sin(yaw)], [0, 1, 0], [-math.sin(yaw), 0, math.cos(yaw)]])
    spec.world_to_instance = np.concatenate([spec.world_to_instance,
                                             np.array([identity34(), identity34(), identity34(),
                                                       _w2i_from_rt(rot, (0.1, 0.35, 0.3), 0.6)], np.float32)])
    n = len(spec.lods)
    spec.instance_lod = np.concatenate([spec.instance_lod, np.array([n - 3, n - 2, n - 1, n - 1], np.uint32)])
    if background:
        spec.background = ((0.2, 0.25, 0.3), (1.0, 1.0, 1.0))
    spec.name = "alpha_cutouts"
    return spec


def emissive_panels(seed: int = 0, num_instances: int = 4, quads_per_instance: int = 16, num_point_lights: int = 1,
                    width: int = 96, height: int = 64, emissive_triangles: int = 0,
                    emissive_spheres: int = 0) -> SceneSpec:
    """Many small emissive quads: a ground quad, and `num_instances` instances
    (one of them mirrored) of a panel set holding non-emissive triangles,
    `quads_per_instance` emissive quads of three radiances and some
    non-emissive quads; plus point lights. With `emissive_triangles` > 0 the
    panel set also holds that many emissive triangles, and with `emissive_spheres` > 0
    that many emissive spheres (next to two spheres that do not emit). The light tree
    then has num_instances * (quads_per_instance + emissive_triangles + emissive_spheres)
    + num_point_lights leaves."""
    rng = np.random.default_rng(seed)
    mats = [MaterialSpec(MAT_LAMBERT, albedo=(0.6, 0.6, 0.55), name="ground"),
            MaterialSpec(MAT_LAMBERT, albedo=(0.3, 0.5, 0.7), name="frame")]
    for k in range(3):
        mats.append(MaterialSpec(MAT_EMISSIVE, radiance=tuple(float(x) for x in rng.uniform(2.0, 12.0, 3)), name=f"emit{k}"))
    gp, gn = _quad((-20, 0, -20), (-20, 0, 20), (20, 0, 20), (20, 0, -20))
    ground = _lod(gp, gn, np.array([(0, 0), (1, 0), (1, 1), (0, 1)], np.float32),
                  quads=np.arange(4, dtype=np.uint32).reshape(1, 4), mats=np.array([0], np.uint16), name="ground")
    # the panel set: frame triangles first, then emissive and frame quads interleaved
    verts, norms, uvs, tris, quads, qmats = [], [], [], [], [], []
    for t in range(3 + emissive_triangles):
        c = rng.uniform(-1.5, 1.5, 3) + (np.array([0.0, 2.0, 0.0]) if t >= 3 else 0.0)
        p = (c + rng.normal(scale=0.3, size=(3, 3))).astype(np.float32)
        n = np.cross(p[1] - p[0], p[2] - p[0])
        n /= np.linalg.norm(n)
        base = len(verts)
        verts += list(p)
        norms += [n] * 3
        uvs += [(0, 0), (1, 0), (0, 1)]
        tris.append((base, base + 1, base + 2))
    num_frame = max(1, quads_per_instance // 4)
    kinds = [2 + int(rng.integers(0, 3)) for _ in range(quads_per_instance)] + [1] * num_frame
    rng.shuffle(kinds)
    for kind in kinds:
        c = rng.uniform(-1.5, 1.5, 3) + np.array([0.0, 2.0, 0.0])
        a, b = rng.normal(size=3), rng.normal(size=3)
        a /= np.linalg.norm(a)
        b = b - a * np.dot(a, b)
        b /= np.linalg.norm(b)
        s = rng.uniform(0.03, 0.12, 2)
        p = np.array([c - s[0] * a - s[1] * b, c + s[0] * a - s[1] * b, c + s[0] * a + s[1] * b,
                      c - s[0] * a + s[1] * b], np.float32)
        n = np.cross(p[1] - p[0], p[3] - p[0])
        n /= np.linalg.norm(n)
        base = len(verts)
        verts += list(p)
        norms += [n] * 4
        uvs += [(0, 0), (1, 0), (1, 1), (0, 1)]
        quads.append((base, base + 1, base + 2, base + 3))
        qmats.append(kind)
    sph, smats = _empty_spheres()
    if emissive_spheres:
        c = rng.uniform(-1.8, 1.8, (emissive_spheres + 2, 3)) + np.array([0.0, 2.2, 0.0])
        r = rng.uniform(0.08, 0.35, (emissive_spheres + 2, 1))
        sph = np.concatenate([c, r], 1).astype(np.float32)
        smats = np.array([1] + [2 + k % 3 for k in range(emissive_spheres)] + [1], np.uint16)
    panel = _lod(np.array(verts, np.float32), np.array(norms, np.float32), np.array(uvs, np.float32),
                 tris=np.array(tris, np.uint32), quads=np.array(quads, np.uint32),
                 mats=np.array([1] * 3 + [2 + t % 3 for t in range(emissive_triangles)] + qmats, np.uint16),
                 spheres=sph, sphere_mats=smats, name="panels")
    w2i, inst_lod = [identity34()], [0]
    for i in range(num_instances):
        rot = _random_rotation(rng)
        if i == 0:
            rot = rot @ np.diag([1.0, 1.0, -1.0])  # a mirroring instance
        w2i.append(_w2i_from_rt(rot, rng.uniform(-8.0, 8.0, 3) * np.array([1.0, 0.0, 1.0]) + np.array([0.0, 0.5, 0.0]),
                                float(rng.uniform(0.7, 1.5))))
        inst_lod.append(1)
    lights = np.array([np.concatenate([rng.uniform(-6, 6, 3) * np.array([1.0, 0.0, 1.0]) + np.array([0.0, 6.0, 0.0]),
                                       rng.uniform(20.0, 60.0, 3)]) for _ in range(num_point_lights)],
                      np.float32).reshape(-1, 6)
    return SceneSpec([ground, panel], np.array(w2i, np.float32), np.array(inst_lod, np.uint32), mats, lights, None,
                     (0.0, 6.0, 16.0), (0.0, -0.35, -1.0), (0.0, 1.0, 0.0), math.radians(50.0), width, height,
                     name="emissive_panels")
