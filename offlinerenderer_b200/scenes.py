"""Procedural, seeded scenes for the benchmark configurations.

Every scene is a flat triangle soup in the form libWR's ``Scene::addTriangleMesh``
accumulates it (libWR/src/internal/scene.cpp:190-244): float32 xyz vertices,
optional per-vertex normals and uvs, uint32 index triplets, one material id per
triangle, a list of 64-byte material records and RGBA8 textures (1-based ids).

Scenes:
  * ``cornell(...)``         -- the plain Cornell box (36 triangles).
  * ``material_showcase()``  -- the Cornell room + three subdivision-4 icospheres
    (glass, GGX metal, rough glass), a 1024^2 checker floor and a value-noise
    normal map.
  * ``scale_test()``         -- 1024^2 fBm heightfield + 250 icospheres + 64
    emissive triangles (about 2.4M triangles).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

LAMBERTIAN, EMISSIVE, GLASS, GGX_REFLECTION, GGX_TRANSMISSION = 0, 1, 2, 3, 4

# 64-byte material record (libWR/src/internal/gpu_types.h:28-37 field meaning).
MATERIAL_DTYPE = np.dtype(
    [
        ("albedo", "<f4", 4),
        ("emission", "<f4", 4),
        ("ior", "<f4"),
        ("type", "<u4"),
        ("roughness", "<f4"),
        ("metallic", "<f4"),
        ("albedoTextureId", "<u4"),
        ("normalTextureId", "<u4"),
        ("pad", "<u4", 2),
    ]
)
assert MATERIAL_DTYPE.itemsize == 64


def _radians(deg: float) -> np.float32:
    # glm::radians for float: degrees * float(pi/180)
    return np.float32(np.float32(deg) * np.float32(0.01745329251994329576923690768489))


@dataclasses.dataclass
class Camera:
    position: tuple = (0.0, 0.0, 0.0)
    target: tuple = (0.0, 0.0, -1.0)
    up: tuple = (0.0, 1.0, 0.0)
    fovY: float = float(_radians(45.0))
    aspect: float = 1.0
    focalDistance: float = 0.0
    lensRadius: float = 0.0


@dataclasses.dataclass
class RenderSettings:
    width: int
    height: int
    spp: int
    maxBounces: int = 8
    russianRouletteDepth: float = 3.0
    useNEE: bool = True
    fireflyClamp: float = 0.0
    seed: int = 0


@dataclasses.dataclass
class SceneData:
    vertices: np.ndarray  # (V,3) f32
    indices: np.ndarray  # (T,3) u32
    tri_material: np.ndarray  # (T,) u32
    materials: np.ndarray  # (M,) MATERIAL_DTYPE
    normals: np.ndarray | None = None  # (V,3) f32
    uvs: np.ndarray | None = None  # (V,2) f32
    textures: list = dataclasses.field(default_factory=list)  # (H,W,4) u8, id = index+1
    env: tuple = (0.0, 0.0, 0.0)
    env_map: np.ndarray | None = None  # (H, W, 4) f32 lat-long map, row 0 = +y pole
    camera: Camera | None = None
    settings: RenderSettings | None = None
    name: str = ""

    @property
    def num_triangles(self) -> int:
        return int(self.indices.shape[0])


class _Builder:
    """Accumulates meshes the way Scene::addTriangleMesh does (indices rebased,
    absent normals/uvs zero-padded)."""

    def __init__(self):
        self.v, self.n, self.uv, self.i, self.m = [], [], [], [], []
        self.has_n = self.has_uv = False
        self.nv = 0
        self.mats = []
        self.textures = []

    def material(self, type_, albedo=(0, 0, 0), emission=(0, 0, 0), ior=1.0, roughness=0.0, metallic=0.0,
                 albedo_tex=0, normal_tex=0) -> int:
        rec = np.zeros((), MATERIAL_DTYPE)
        rec["albedo"][:3] = albedo
        rec["emission"][:3] = emission
        rec["ior"] = ior
        rec["type"] = type_
        rec["roughness"] = roughness
        rec["metallic"] = metallic
        rec["albedoTextureId"] = albedo_tex
        rec["normalTextureId"] = normal_tex
        self.mats.append(rec)
        return len(self.mats) - 1

    # Material constructors with libWR's defaults (scene.cpp:91-168).
    def lambertian(self, albedo, tex=0):
        return self.material(LAMBERTIAN, albedo=albedo, ior=1.0, roughness=1.0, albedo_tex=tex)

    def emissive(self, emission):
        return self.material(EMISSIVE, emission=emission, ior=1.0)

    def glass(self, albedo, ior):
        return self.material(GLASS, albedo=albedo, ior=ior)

    def ggx(self, albedo, roughness, metallic=0.0):
        return self.material(GGX_REFLECTION, albedo=albedo, ior=1.5, roughness=roughness, metallic=metallic)

    def ggx_transmission(self, albedo, roughness, ior):
        return self.material(GGX_TRANSMISSION, albedo=albedo, ior=ior, roughness=roughness)

    def texture(self, rgba: np.ndarray) -> int:
        self.textures.append(np.ascontiguousarray(rgba, dtype=np.uint8))
        return len(self.textures)

    def mesh(self, verts, inds, mat, normals=None, uvs=None):
        verts = np.asarray(verts, np.float32).reshape(-1, 3)
        inds = np.asarray(inds, np.uint32).reshape(-1, 3)
        nv = verts.shape[0]
        self.v.append(verts)
        if normals is not None:
            self.has_n = True
            self.n.append(np.asarray(normals, np.float32).reshape(-1, 3))
        else:
            self.n.append(np.zeros((nv, 3), np.float32))
        if uvs is not None:
            self.has_uv = True
            self.uv.append(np.asarray(uvs, np.float32).reshape(-1, 2))
        else:
            self.uv.append(np.zeros((nv, 2), np.float32))
        self.i.append(inds + np.uint32(self.nv))
        self.m.append(np.full(inds.shape[0], mat, np.uint32))
        self.nv += nv

    def build(self, **kw) -> SceneData:
        return SceneData(
            vertices=np.ascontiguousarray(np.concatenate(self.v), np.float32),
            indices=np.ascontiguousarray(np.concatenate(self.i), np.uint32),
            tri_material=np.ascontiguousarray(np.concatenate(self.m), np.uint32),
            materials=np.array(self.mats, MATERIAL_DTYPE),
            normals=np.ascontiguousarray(np.concatenate(self.n)) if self.has_n else None,
            uvs=np.ascontiguousarray(np.concatenate(self.uv)) if self.has_uv else None,
            textures=list(self.textures),
            **kw,
        )


def _quad(b: _Builder, p0, p1, p2, p3, mat, uvs=None):
    b.mesh([p0, p1, p2, p3], [0, 1, 2, 0, 2, 3], mat, uvs=uvs)


def _box(b: _Builder, cx, cz, sx, sy, sz, angle_deg, mat):
    """Axis-aligned box resting on y=0, rotated about y through its centre; 12 triangles."""
    a = math.radians(angle_deg)
    ca, sa = math.cos(a), math.sin(a)
    corners = []
    for y in (0.0, sy):
        for dx, dz in ((-1, -1), (1, -1), (1, 1), (-1, 1)):
            x, z = dx * sx / 2, dz * sz / 2
            corners.append((cx + ca * x + sa * z, y, cz - sa * x + ca * z))
    # bottom 0-3, top 4-7 (counter-clockwise seen from +y for the top)
    faces = [(0, 3, 2, 1), (4, 5, 6, 7), (0, 1, 5, 4), (1, 2, 6, 5), (2, 3, 7, 6), (3, 0, 4, 7)]
    idx = []
    for f in faces:
        idx += [f[0], f[1], f[2], f[0], f[2], f[3]]
    b.mesh(corners, idx, mat)


def icosphere(subdiv: int):
    """Unit icosphere: 20 * 4^subdiv triangles; returns (verts (V,3) f64, idx (T,3))."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    v = [np.array(p, np.float64) / np.linalg.norm(p) for p in v]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
         (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
         (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdiv):
        cache = {}

        def mid(a, b):
            key = (a, b) if a < b else (b, a)
            if key not in cache:
                p = v[a] + v[b]
                v.append(p / np.linalg.norm(p))
                cache[key] = len(v) - 1
            return cache[key]

        nf = []
        for a, b, c in f:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        f = nf
    return np.array(v, np.float64), np.array(f, np.uint32)


_ICO_CACHE: dict = {}


def _sphere(b: _Builder, center, radius, subdiv, mat, smooth=True):
    if subdiv not in _ICO_CACHE:
        _ICO_CACHE[subdiv] = icosphere(subdiv)
    unit, idx = _ICO_CACHE[subdiv]
    verts = (unit * radius + np.asarray(center, np.float64)).astype(np.float32)
    b.mesh(verts, idx, mat, normals=unit.astype(np.float32) if smooth else None)


def _room(b: _Builder, white, red, green, light, floor_mat=None, floor_uvs=False):
    fm = white if floor_mat is None else floor_mat
    uvs = [(0, 0), (1, 0), (1, 1), (0, 1)] if floor_uvs else None
    _quad(b, (0, 0, 0), (1, 0, 0), (1, 0, 1), (0, 0, 1), fm, uvs=uvs)  # floor
    _quad(b, (0, 1, 0), (0, 1, 1), (1, 1, 1), (1, 1, 0), white)  # ceiling
    _quad(b, (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1), white)  # back wall
    # The camera's right vector is -x, so the image-left wall is x=1.
    _quad(b, (1, 0, 0), (1, 1, 0), (1, 1, 1), (1, 0, 1), red)  # left wall
    _quad(b, (0, 0, 0), (0, 0, 1), (0, 1, 1), (0, 1, 0), green)
    # Ceiling light wound like libWR's (cornell_box_var_test.cpp:64-70): normal -y.
    ly = 0.999
    _quad(b, (0.35, ly, 0.35), (0.65, ly, 0.35), (0.65, ly, 0.65), (0.35, ly, 0.65), light)


def _cornell_camera(w, h) -> Camera:
    return Camera(position=(0.5, 0.5, -1.4), target=(0.5, 0.5, 0.0), up=(0.0, 1.0, 0.0), fovY=float(_radians(40.0)),
                  aspect=float(np.float32(w) / np.float32(h)))


def cornell(width=256, height=256, spp=64, seed=1) -> SceneData:
    """Plain Cornell box: 10 room triangles, a 2-triangle light (17,12,4), a tall
    (0.3x0.6x0.3, +15 deg) and a short (0.3^3, -18 deg) white box; 36 triangles."""
    b = _Builder()
    white = b.lambertian((0.73, 0.73, 0.73))
    red = b.lambertian((0.63, 0.065, 0.05))
    green = b.lambertian((0.14, 0.45, 0.09))
    light = b.emissive((17.0, 12.0, 4.0))
    _room(b, white, red, green, light)
    _box(b, 0.66, 0.64, 0.3, 0.6, 0.3, 15.0, white)
    _box(b, 0.34, 0.36, 0.3, 0.3, 0.3, -18.0, white)
    return b.build(camera=_cornell_camera(width, height),
                   settings=RenderSettings(width, height, spp, maxBounces=8, russianRouletteDepth=3.0, seed=seed),
                   name=f"cornell_{width}x{height}_{spp}spp")


def checker_texture(size=1024, cell=32, a=(235, 235, 235), b=(40, 40, 40)) -> np.ndarray:
    y, x = np.mgrid[0:size, 0:size]
    odd = ((x // cell) + (y // cell)) % 2 == 1
    tex = np.empty((size, size, 4), np.uint8)
    tex[...] = (*a, 255)
    tex[odd] = (*b, 255)
    return tex


def value_noise_normal_map(size=1024, cells=32, strength=0.6, seed=1) -> np.ndarray:
    """Tangent-space normal map from the gradient of seeded, bilinearly interpolated
    value noise on a ``cells`` x ``cells`` lattice (wrapping)."""
    rng = np.random.default_rng(seed)
    lat = rng.random((cells, cells))
    t = (np.arange(size) + 0.5) * cells / size
    i0 = np.floor(t).astype(int) % cells
    i1 = (i0 + 1) % cells
    f = t - np.floor(t)
    f = f * f * (3 - 2 * f)
    v00 = lat[np.ix_(i0, i0)]
    v10 = lat[np.ix_(i0, i1)]
    v01 = lat[np.ix_(i1, i0)]
    v11 = lat[np.ix_(i1, i1)]
    fx = f[None, :]
    fy = f[:, None]
    h = (v00 * (1 - fx) + v10 * fx) * (1 - fy) + (v01 * (1 - fx) + v11 * fx) * fy
    # slope in height per unit uv, scaled so a lattice step tilts by ~``strength``
    gy, gx = np.gradient(h)
    k = strength * size / cells
    n = np.stack([-gx * k, -gy * k, np.ones_like(h)], -1)
    n /= np.linalg.norm(n, axis=-1, keepdims=True)
    tex = np.empty((size, size, 4), np.uint8)
    tex[..., :3] = np.clip(np.round((n * 0.5 + 0.5) * 255), 0, 255).astype(np.uint8)
    tex[..., 3] = 255
    return tex


def material_showcase(width=512, height=512, spp=256, seed=1, tex_size=1024) -> SceneData:
    """Cornell room + ideal-glass, GGX-metal and rough-glass icospheres (subdiv 4,
    r=0.15) on a checker-textured, normal-mapped floor."""
    b = _Builder()
    checker = b.texture(checker_texture(tex_size, max(1, tex_size // 32)))
    nmap = b.texture(value_noise_normal_map(tex_size, 32, seed=seed))
    white = b.lambertian((0.73, 0.73, 0.73))
    red = b.lambertian((0.63, 0.065, 0.05))
    green = b.lambertian((0.14, 0.45, 0.09))
    light = b.emissive((17.0, 12.0, 4.0))
    floor = b.lambertian((0.73, 0.73, 0.73), checker)
    b.mats[floor]["normalTextureId"] = nmap
    glass = b.glass((0.999, 0.999, 0.999), 1.5)
    metal = b.ggx((0.95, 0.64, 0.54), 0.3, 1.0)
    rough_glass = b.ggx_transmission((0.999, 0.999, 0.999), 0.2, 1.5)
    _room(b, white, red, green, light, floor_mat=floor, floor_uvs=True)
    _sphere(b, (0.75, 0.15, 0.45), 0.15, 4, glass)
    _sphere(b, (0.5, 0.15, 0.62), 0.15, 4, metal)
    _sphere(b, (0.25, 0.15, 0.45), 0.15, 4, rough_glass)
    return b.build(camera=_cornell_camera(width, height),
                   settings=RenderSettings(width, height, spp, maxBounces=16, russianRouletteDepth=3.0, seed=seed),
                   name=f"showcase_{width}x{height}_{spp}spp")


def _fbm(n, octaves, seed):
    rng = np.random.default_rng(seed)
    h = np.zeros((n, n))
    amp, total = 1.0, 0.0
    for o in range(octaves):
        cells = 4 * 2 ** o
        lat = rng.random((cells + 1, cells + 1))
        t = np.linspace(0, cells, n, endpoint=False)
        i0 = np.floor(t).astype(int)
        f = t - i0
        f = f * f * (3 - 2 * f)
        v00 = lat[np.ix_(i0, i0)]
        v10 = lat[np.ix_(i0, i0 + 1)]
        v01 = lat[np.ix_(i0 + 1, i0)]
        v11 = lat[np.ix_(i0 + 1, i0 + 1)]
        fx, fy = f[None, :], f[:, None]
        h += amp * ((v00 * (1 - fx) + v10 * fx) * (1 - fy) + (v01 * (1 - fx) + v11 * fx) * fy)
        total += amp
        amp *= 0.5
    return h / total


def scale_test(width=1920, height=1080, spp=64, seed=1, grid=1024, spheres=250, lights=64) -> SceneData:
    """Heightfield (grid x grid vertices, fBm 4 octaves, amplitude 0.1) + icospheres
    (subdiv 3) at uniform positions, radii U[0.01,0.05], materials drawn from the
    five BSDF kinds, and 64 small emissive triangles with |E| in U(5,50)."""
    rng = np.random.default_rng(seed)
    b = _Builder()
    ground = b.lambertian((0.5, 0.5, 0.5))
    h = _fbm(grid, 4, seed) * 0.1
    xs = np.linspace(0.0, 1.0, grid, dtype=np.float64)
    gx, gz = np.meshgrid(xs, xs)
    verts = np.stack([gx, h, gz], -1).reshape(-1, 3).astype(np.float32)
    r = np.arange(grid - 1)
    i00 = (r[:, None] * grid + r[None, :]).reshape(-1)
    i10, i01, i11 = i00 + 1, i00 + grid, i00 + grid + 1
    tris = np.stack([np.stack([i00, i01, i11], -1), np.stack([i00, i11, i10], -1)], 1).reshape(-1, 3)
    b.mesh(verts, tris.astype(np.uint32), ground)
    for _ in range(spheres):
        kind = int(rng.integers(0, 5))
        alb = tuple(rng.uniform(0.1, 0.9, 3))
        if kind == 0:
            m = b.lambertian(alb)
        elif kind == 1:
            m = b.glass((0.999, 0.999, 0.999), float(rng.uniform(1.3, 1.7)))
        elif kind == 2:
            m = b.ggx(alb, float(rng.uniform(0.05, 0.8)), 1.0)
        elif kind == 3:
            m = b.ggx(alb, float(rng.uniform(0.05, 0.8)), 0.0)
        else:
            m = b.ggx_transmission((0.999, 0.999, 0.999), float(rng.uniform(0.05, 0.8)), float(rng.uniform(1.3, 1.7)))
        rad = float(rng.uniform(0.01, 0.05))
        x, z = rng.uniform(0.05, 0.95, 2)
        gi = min(grid - 1, int(round(z * (grid - 1)))), min(grid - 1, int(round(x * (grid - 1))))
        _sphere(b, (x, h[gi] + rad, z), rad, 3, m)
    for _ in range(lights):
        e = float(rng.uniform(5.0, 50.0))
        col = rng.uniform(0.5, 1.0, 3)
        col = col / np.linalg.norm(col) * e
        m = b.emissive(tuple(col))
        c = np.array([rng.uniform(0.05, 0.95), rng.uniform(0.2, 0.5), rng.uniform(0.05, 0.95)])
        s = rng.uniform(0.01, 0.03)
        # wound so the geometric normal faces down (-y), like the Cornell light
        p0, p1, p2 = c + (-s, 0, -s), c + (s, 0, -s), c + (0, 0, s)
        b.mesh([p0, p1, p2], [0, 1, 2], m)
    cam = Camera(position=(0.5, 0.55, -0.35), target=(0.5, 0.05, 0.55), up=(0.0, 1.0, 0.0),
                 fovY=float(_radians(55.0)), aspect=float(np.float32(width) / np.float32(height)))
    return b.build(env=(0.12, 0.12, 0.15), camera=cam,
                   settings=RenderSettings(width, height, spp, maxBounces=8, russianRouletteDepth=3.0, seed=seed),
                   name=f"scale_{width}x{height}_{spp}spp")


def _random_material(b: _Builder, rng):
    """One of the five BSDF kinds, parameters drawn as in the scale test."""
    kind = int(rng.integers(0, 5))
    alb = tuple(rng.uniform(0.1, 0.9, 3))
    if kind == 0:
        return b.lambertian(alb)
    if kind == 1:
        return b.glass((0.999, 0.999, 0.999), float(rng.uniform(1.3, 1.7)))
    if kind == 2:
        return b.ggx(alb, float(rng.uniform(0.05, 0.8)), 1.0)
    if kind == 3:
        return b.ggx(alb, float(rng.uniform(0.05, 0.8)), 0.0)
    return b.ggx_transmission((0.999, 0.999, 0.999), float(rng.uniform(0.05, 0.8)), float(rng.uniform(1.3, 1.7)))


def cornell_variant(seed: int, max_tris: int = 60000) -> SceneData:
    """One scene of the batched-scenes workload: the Cornell room with both boxes
    rotated by U(-45, 45) degrees and 0-8 icospheres (subdivision 2-5, random
    materials as in the scale test), the subdivision lowered where needed to keep
    the scene within `max_tris`; resolution from {128^2, 256^2, 512^2, 1024^2} and
    spp from {4, 16, 64, 256}, both drawn from the seed."""
    rng = np.random.default_rng(10_000 + seed)
    b = _Builder()
    white = b.lambertian((0.73, 0.73, 0.73))
    red = b.lambertian((0.63, 0.065, 0.05))
    green = b.lambertian((0.14, 0.45, 0.09))
    light = b.emissive((17.0, 12.0, 4.0))
    _room(b, white, red, green, light)
    _box(b, 0.66, 0.64, 0.3, 0.6, 0.3, float(rng.uniform(-45, 45)), white)
    _box(b, 0.34, 0.36, 0.3, 0.3, 0.3, float(rng.uniform(-45, 45)), white)
    tris = 36
    for _ in range(int(rng.integers(0, 9))):
        sub = int(rng.integers(2, 6))
        while sub > 2 and tris + 20 * 4 ** sub > max_tris:
            sub -= 1
        if tris + 20 * 4 ** sub > max_tris:
            break
        r = float(rng.uniform(0.05, 0.12))
        c = (float(rng.uniform(0.15, 0.85)), float(rng.uniform(0.05, 0.7)) + r, float(rng.uniform(0.15, 0.85)))
        _sphere(b, c, r, sub, _random_material(b, rng))
        tris += 20 * 4 ** sub
    res = int(rng.choice([128, 256, 512, 1024]))
    spp = int(rng.choice([4, 16, 64, 256]))
    return b.build(camera=_cornell_camera(res, res),
                   settings=RenderSettings(res, res, spp, maxBounces=8, russianRouletteDepth=3.0, seed=seed + 1),
                   name=f"cornell_variant_{seed}")
