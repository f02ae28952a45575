"""ctypes binding of the CPU oracle -- test infrastructure only.

Imported by tests/, by the smoke check and by bench.py's CPU-baseline leg; never
by the product package.  ``Oracle`` wraps liborc.so (the restated render path);
``Reference`` wraps _ref/libref.so (the reference's own shading headers compiled
on the host, driven by the same CPU traversal).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, "liborc.so")
REF_LIB = os.path.join(HERE, "_ref", "libref.so")

BSDF_IN = 20  # floats per bsdf input record
BSDF_OUT = 34  # doubles per bsdf output record


class _Material(C.Structure):
    _fields_ = [("albedo", C.c_float * 4), ("emission", C.c_float * 4), ("ior", C.c_float), ("type", C.c_uint32),
                ("roughness", C.c_float), ("metallic", C.c_float), ("albedoTextureId", C.c_uint32),
                ("normalTextureId", C.c_uint32), ("pad", C.c_uint32 * 2)]


class _Texture(C.Structure):
    _fields_ = [("rgba", C.c_void_p), ("width", C.c_uint32), ("height", C.c_uint32)]


class _SceneDesc(C.Structure):
    _fields_ = [("vertices", C.c_void_p), ("normals", C.c_void_p), ("uvs", C.c_void_p), ("indices", C.c_void_p),
                ("triMaterial", C.c_void_p), ("numVertices", C.c_uint32), ("numTriangles", C.c_uint32),
                ("materials", C.c_void_p), ("numMaterials", C.c_uint32), ("textures", C.c_void_p),
                ("numTextures", C.c_uint32), ("envRadiance", C.c_float * 3)]


class _Camera(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("target", C.c_float * 3), ("up", C.c_float * 3), ("fovY", C.c_float),
                ("aspect", C.c_float), ("focalDistance", C.c_float), ("lensRadius", C.c_float)]


class _Params(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("spp", C.c_uint32), ("useNEE", C.c_uint32),
                ("maxBounces", C.c_uint32), ("rrStartDepth", C.c_float), ("fireflyClamp", C.c_float),
                ("seed", C.c_uint32), ("maxIterations", C.c_uint32), ("drawOrder", C.c_uint32),
                ("sampleBegin", C.c_uint32), ("pixelBegin", C.c_uint32), ("pixelEnd", C.c_uint32)]


class _Stats(C.Structure):
    _fields_ = [("extensionRays", C.c_uint64), ("shadowRays", C.c_uint64), ("paths", C.c_uint64)]


def _ptr(a):
    return None if a is None else a.ctypes.data


def build(force: bool = False) -> None:
    """Builds liborc.so (and _ref/libref.so where the reference checkout exists)."""
    if force or not os.path.exists(PORT_LIB):
        subprocess.run(["make", "-s", "-C", HERE], check=True)


def make_camera(cam) -> _Camera:
    c = _Camera()
    c.position[:] = cam.position
    c.target[:] = cam.target
    c.up[:] = cam.up
    c.fovY, c.aspect, c.focalDistance, c.lensRadius = cam.fovY, cam.aspect, cam.focalDistance, cam.lensRadius
    return c


def make_params(st, spp=None, max_iterations=8, draw_order=0, sample_begin=0, pixel_begin=0, pixel_end=0) -> _Params:
    p = _Params()
    p.width, p.height = st.width, st.height
    p.spp = st.spp if spp is None else spp
    p.useNEE = 1 if st.useNEE else 0
    p.maxBounces = st.maxBounces
    p.rrStartDepth = st.russianRouletteDepth
    p.fireflyClamp = st.fireflyClamp
    p.seed = st.seed
    p.maxIterations = max_iterations
    p.drawOrder = draw_order
    p.sampleBegin = sample_begin
    p.pixelBegin, p.pixelEnd = pixel_begin, pixel_end
    return p


class _Base:
    _prefix = "orc"

    def __init__(self, path):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = C.CDLL(path)
        pf = self._prefix
        self._create = getattr(self.lib, f"{pf}_scene_create")
        self._create.restype = C.c_void_p
        self._create.argtypes = [C.POINTER(_SceneDesc)]
        self._destroy = getattr(self.lib, f"{pf}_scene_destroy")
        self._destroy.argtypes = [C.c_void_p]
        self._render = getattr(self.lib, f"{pf}_render")
        self._render.argtypes = [C.c_void_p, C.POINTER(_Camera), C.POINTER(_Params), C.c_void_p, C.c_void_p,
                                 C.c_void_p, C.c_int, C.POINTER(_Stats)]

    def scene(self, sd) -> "OracleScene":
        return OracleScene(self, sd)


class OracleScene:
    def __init__(self, owner: _Base, sd):
        self.owner = owner
        self.sd = sd
        self._keep = [sd.vertices, sd.indices, sd.tri_material, sd.materials, sd.normals, sd.uvs] + list(sd.textures)
        texs = (_Texture * max(1, len(sd.textures)))()
        for i, t in enumerate(sd.textures):
            texs[i].rgba = t.ctypes.data
            texs[i].height, texs[i].width = t.shape[0], t.shape[1]
        self._texs = texs
        d = _SceneDesc()
        d.vertices, d.normals, d.uvs = _ptr(sd.vertices), _ptr(sd.normals), _ptr(sd.uvs)
        d.indices, d.triMaterial = _ptr(sd.indices), _ptr(sd.tri_material)
        d.numVertices, d.numTriangles = sd.vertices.shape[0], sd.indices.shape[0]
        d.materials, d.numMaterials = _ptr(sd.materials), sd.materials.shape[0]
        d.textures, d.numTextures = C.cast(texs, C.c_void_p), len(sd.textures)
        d.envRadiance[:] = sd.env
        self._desc = d
        self.handle = owner._create(C.byref(d))

    def __del__(self):
        h = getattr(self, "handle", None)
        if h:
            self.owner._destroy(h)
            self.handle = None

    def render(self, camera=None, settings=None, spp=None, threads=0, **kw):
        """Returns (rgb (H,W,3) = sum/spp, albedo sum, normal sum, stats dict)."""
        cam = make_camera(camera or self.sd.camera)
        st = settings or self.sd.settings
        p = make_params(st, spp=spp, **kw)
        n = st.width * st.height
        rgb = np.zeros((n, 3), np.float32)
        alb = np.zeros((n, 3), np.float32)
        nrm = np.zeros((n, 3), np.float32)
        stats = _Stats()
        self.owner._render(self.handle, C.byref(cam), C.byref(p), rgb.ctypes.data, alb.ctypes.data, nrm.ctypes.data,
                           threads, C.byref(stats))
        shape = (st.height, st.width, 3)
        return rgb.reshape(shape), alb.reshape(shape), nrm.reshape(shape), {
            "extension_rays": stats.extensionRays, "shadow_rays": stats.shadowRays, "paths": stats.paths}

    # ray queries (oracle port only)
    def closest(self, rays: np.ndarray, mode: int = 0, threads: int = 0):
        rays = np.ascontiguousarray(rays, np.float32)
        n = rays.shape[0]
        t = np.zeros(n, np.float32)
        prim = np.zeros(n, np.uint32)
        self.owner.lib.orc_closest(C.c_void_p(self.handle), C.c_void_p(rays.ctypes.data), C.c_uint32(n), C.c_int(mode),
                                   C.c_void_p(t.ctypes.data), C.c_void_p(prim.ctypes.data), C.c_int(threads))
        return t, prim

    def occluded(self, rays: np.ndarray, threads: int = 0):
        rays = np.ascontiguousarray(rays, np.float32)
        n = rays.shape[0]
        out = np.zeros(n, np.uint32)
        self.owner.lib.orc_occluded(C.c_void_p(self.handle), C.c_void_p(rays.ctypes.data), C.c_uint32(n),
                                    C.c_void_p(out.ctypes.data), C.c_int(threads))
        return out

    def light_cdf(self):
        lib = self.owner.lib
        lib.orc_scene_num_emissive.restype = C.c_uint32
        n = lib.orc_scene_num_emissive(C.c_void_p(self.handle))
        tris = np.zeros(n, np.uint32)
        cdf = np.zeros(n, np.float32)
        lib.orc_scene_light_cdf(C.c_void_p(self.handle), C.c_void_p(tris.ctypes.data), C.c_void_p(cdf.ctypes.data))
        return tris, cdf


class Oracle(_Base):
    """The oracle's restatement of the reference render path (liborc.so)."""

    _prefix = "orc"

    def __init__(self, path: str = PORT_LIB):
        super().__init__(path)

    def bsdf(self, inp: np.ndarray, prec: int = 0) -> np.ndarray:
        inp = np.ascontiguousarray(inp, np.float32).reshape(-1, BSDF_IN)
        out = np.zeros((inp.shape[0], BSDF_OUT), np.float64)
        self.lib.orc_bsdf_batch(C.c_void_p(inp.ctypes.data), C.c_uint32(inp.shape[0]), C.c_int(prec),
                                C.c_void_p(out.ctypes.data))
        return out

    def rng(self, seeds, dims):
        seeds = np.ascontiguousarray(seeds, np.uint32)
        dims = np.ascontiguousarray(dims, np.uint32)
        h = np.zeros(seeds.shape[0], np.uint32)
        u = np.zeros(seeds.shape[0], np.float32)
        self.lib.orc_rng_batch(C.c_void_p(seeds.ctypes.data), C.c_void_p(dims.ctypes.data), C.c_uint32(seeds.shape[0]),
                               C.c_void_p(h.ctypes.data), C.c_void_p(u.ctypes.data))
        return h, u

    def cdf_sample(self, cdf, u):
        cdf = np.ascontiguousarray(cdf, np.float32)
        u = np.ascontiguousarray(u, np.float32)
        out = np.zeros(u.shape[0], np.uint32)
        self.lib.orc_cdf_batch(C.c_void_p(cdf.ctypes.data), C.c_uint32(cdf.shape[0]), C.c_void_p(u.ctypes.data),
                               C.c_uint32(u.shape[0]), C.c_void_p(out.ctypes.data))
        return out

    def tonemap(self, rgb: np.ndarray) -> np.ndarray:
        rgb = np.ascontiguousarray(rgb, np.float32)
        out = np.zeros(rgb.shape, np.uint8)
        self.lib.orc_tonemap(C.c_void_p(rgb.ctypes.data), C.c_uint32(rgb.size // 3), C.c_void_p(out.ctypes.data))
        return out

    def texture(self, rgba: np.ndarray, uv: np.ndarray) -> np.ndarray:
        rgba = np.ascontiguousarray(rgba, np.uint8)
        uv = np.ascontiguousarray(uv, np.float32).reshape(-1, 2)
        t = _Texture(rgba.ctypes.data, rgba.shape[1], rgba.shape[0])
        out = np.zeros((uv.shape[0], 4), np.float32)
        self.lib.orc_texture_batch(C.byref(t), C.c_void_p(uv.ctypes.data), C.c_uint32(uv.shape[0]),
                                   C.c_void_p(out.ctypes.data))
        return out

    def bvh8_validate(self, nodes: np.ndarray, tris: np.ndarray):
        """Structural check of an exported 8-wide BVH; returns (code, depth, internal, leaf)."""
        nodes = np.ascontiguousarray(nodes, np.uint32)
        tris = np.ascontiguousarray(tris, np.float32)
        out = np.zeros(3, np.uint32)
        self.lib.orc_bvh8_validate.restype = C.c_int
        rc = self.lib.orc_bvh8_validate(C.c_void_p(nodes.ctypes.data), C.c_uint32(nodes.shape[0]),
                                        C.c_void_p(tris.ctypes.data), C.c_uint32(tris.shape[0]),
                                        C.c_void_p(out.ctypes.data))
        return int(rc), int(out[0]), int(out[1]), int(out[2])

    def bvh8_trace(self, nodes: np.ndarray, tris: np.ndarray, rays: np.ndarray):
        """Closest hit through an exported 8-wide BVH: (t, prim, node visits, triangle tests)."""
        nodes = np.ascontiguousarray(nodes, np.uint32)
        tris = np.ascontiguousarray(tris, np.float32)
        rays = np.ascontiguousarray(rays, np.float32)
        n = rays.shape[0]
        t = np.zeros(n, np.float32)
        p = np.zeros(n, np.uint32)
        v = np.zeros(n, np.uint32)
        k = np.zeros(n, np.uint32)
        self.lib.orc_bvh8_trace(C.c_void_p(nodes.ctypes.data), C.c_uint32(nodes.shape[0]), C.c_void_p(tris.ctypes.data),
                                C.c_uint32(tris.shape[0]), C.c_void_p(rays.ctypes.data), C.c_uint32(n),
                                C.c_void_p(t.ctypes.data), C.c_void_p(p.ctypes.data), C.c_void_p(v.ctypes.data),
                                C.c_void_p(k.ctypes.data))
        return t, p, v, k

    def compact(self, stage, idx):
        stage = np.ascontiguousarray(stage, np.uint32)
        idx = np.ascontiguousarray(idx, np.uint32)
        out = np.zeros(idx.shape[0], np.uint32)
        self.lib.orc_compact.restype = C.c_uint32
        n = self.lib.orc_compact(C.c_void_p(stage.ctypes.data), C.c_void_p(idx.ctypes.data), C.c_uint32(idx.shape[0]),
                                 C.c_void_p(out.ctypes.data))
        return out[:n]

    def camera_rays(self, camera, width, height, pixels, samples, seed=0):
        pixels = np.ascontiguousarray(pixels, np.uint32)
        samples = np.ascontiguousarray(samples, np.uint32)
        out = np.zeros((pixels.shape[0], 8), np.float32)
        cam = make_camera(camera)
        self.lib.orc_camera_rays(C.byref(cam), C.c_uint32(width), C.c_uint32(height), C.c_void_p(pixels.ctypes.data),
                                 C.c_void_p(samples.ctypes.data), C.c_uint32(pixels.shape[0]), C.c_uint32(seed),
                                 C.c_void_p(out.ctypes.data))
        return out


class Reference(_Base):
    """The reference's shading headers compiled on the host (_ref/libref.so)."""

    _prefix = "ref"

    def __init__(self, path: str = REF_LIB):
        super().__init__(path)

    def bsdf(self, inp: np.ndarray) -> np.ndarray:
        inp = np.ascontiguousarray(inp, np.float32).reshape(-1, BSDF_IN)
        out = np.zeros((inp.shape[0], BSDF_OUT), np.float64)
        self.lib.ref_bsdf_batch(C.c_void_p(inp.ctypes.data), C.c_uint32(inp.shape[0]), C.c_void_p(out.ctypes.data))
        return out

    def rng(self, seeds, dims):
        seeds = np.ascontiguousarray(seeds, np.uint32)
        dims = np.ascontiguousarray(dims, np.uint32)
        h = np.zeros(seeds.shape[0], np.uint32)
        u = np.zeros(seeds.shape[0], np.float32)
        self.lib.ref_rng_batch(C.c_void_p(seeds.ctypes.data), C.c_void_p(dims.ctypes.data), C.c_uint32(seeds.shape[0]),
                               C.c_void_p(h.ctypes.data), C.c_void_p(u.ctypes.data))
        return h, u

    def cdf_sample(self, cdf, u):
        cdf = np.ascontiguousarray(cdf, np.float32)
        u = np.ascontiguousarray(u, np.float32)
        out = np.zeros(u.shape[0], np.uint32)
        self.lib.ref_cdf_batch(C.c_void_p(cdf.ctypes.data), C.c_uint32(cdf.shape[0]), C.c_void_p(u.ctypes.data),
                               C.c_uint32(u.shape[0]), C.c_void_p(out.ctypes.data))
        return out

    def camera_basis(self, camera) -> np.ndarray:
        out = np.zeros(12, np.float32)
        cam = make_camera(camera)
        self.lib.ref_camera_basis(C.byref(cam), C.c_void_p(out.ctypes.data))
        return out

    def save_png(self, path: str, rgb: np.ndarray) -> None:
        rgb = np.ascontiguousarray(rgb, np.float32)
        h, w = rgb.shape[0], rgb.shape[1]
        self.lib.ref_save_png(path.encode(), C.c_void_p(rgb.ctypes.data), C.c_uint32(w), C.c_uint32(h))


def random_bsdf_inputs(n: int, seed: int = 0) -> np.ndarray:
    """Seeded BSDF test records: unit wo/wi/n in the upper hemisphere of n mostly,
    roughness in [0.05, 1], metallic in {0, 1, U}, ior in [1.1, 2.0]."""
    rng = np.random.default_rng(seed)

    def unit(k):
        v = rng.normal(size=(k, 3))
        return v / np.linalg.norm(v, axis=1, keepdims=True)

    nrm = unit(n)
    wo = unit(n)
    wi = unit(n)
    flip = (wo * nrm).sum(1) < 0
    wo[flip & (rng.random(n) < 0.9)] *= -1
    flip = (wi * nrm).sum(1) < 0
    wi[flip & (rng.random(n) < 0.9)] *= -1
    rec = np.zeros((n, BSDF_IN), np.float32)
    rec[:, 0:3] = wo
    rec[:, 3:6] = wi
    rec[:, 6:9] = nrm
    rec[:, 9:12] = rng.uniform(0.05, 1.0, (n, 3))
    rec[:, 12] = rng.uniform(0.05, 1.0, n)
    m = rng.random(n)
    rec[:, 13] = np.where(m < 0.4, 0.0, np.where(m < 0.8, 1.0, rng.random(n)))
    rec[:, 14] = rng.uniform(1.1, 2.0, n)
    rec[:, 15:18] = rng.random((n, 3))
    rec[:, 18] = rng.integers(0, 12, n)
    rec[:, 19] = rng.choice([0.0, 3.0, 5.0], n)
    return rec
