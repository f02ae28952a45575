"""Python binding of libwrk.so (the C ABI in include/wrk.h), via ctypes.

Mirrors libWR's public API (trianglestrip/OfflineRenderer, libWR/include/wr/*.h):
``Scene`` with addLambertianMaterial / addEmissiveMaterial / addGlassMaterial /
addGGXReflectionMaterial / addGGXTransmissionMaterial / setMaterialNormalMap /
addTriangleMesh / setEnvironmentRadiance / finalize, and ``Renderer.render``.
Errors raise ``WrkError`` (a RuntimeError, libWR's convention).  There is no CPU
path: if libwrk.so is missing or no GPU is present, calls fail loudly.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import os

import numpy as np

from . import scenes as _scenes

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libwrk.so")

WRK_FLAG_RAW_GUIDES = 1
WRK_FLAG_STAGE_TIMING = 2
WRK_FLAG_ENV_MAP = 8
STAGES = ["control", "generate", "trace_extension", "trace_shadow", "shade_lambert", "shade_dielectric", "shade_ggx",
          "shade_emissive", "shade_lambert_resume"]
BUCKETS = ["lambert", "dielectric", "ggx", "other", "lambert_resume"]


class WrkError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"wrk error {code}: {msg}")
        self.code = code


class Material(C.Structure):
    _fields_ = [("albedo", C.c_float * 4), ("emission", C.c_float * 4), ("ior", C.c_float), ("type", C.c_uint32),
                ("roughness", C.c_float), ("metallic", C.c_float), ("albedoTextureId", C.c_uint32),
                ("normalTextureId", C.c_uint32), ("pad", C.c_uint32 * 2)]


class CameraC(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("target", C.c_float * 3), ("up", C.c_float * 3), ("fovY", C.c_float),
                ("aspect", C.c_float), ("focalDistance", C.c_float), ("lensRadius", C.c_float)]


class RenderParamsC(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("spp", C.c_uint32), ("useNEE", C.c_uint32),
                ("maxBounces", C.c_uint32), ("russianRouletteDepth", C.c_float), ("fireflyClamp", C.c_float),
                ("seed", C.c_uint32), ("maxIterations", C.c_uint32), ("flags", C.c_uint32),
                ("sampleOffset", C.c_uint32)]


class RenderStatsC(C.Structure):
    _fields_ = [("paths", C.c_uint64), ("extensionRays", C.c_uint64), ("shadowRays", C.c_uint64),
                ("iterations", C.c_uint32), ("deviceErrors", C.c_uint32), ("gpuMs", C.c_float),
                ("totalMs", C.c_float), ("stageMs", C.c_float * 9), ("stageLaunches", C.c_uint32 * 9),
                ("bucketPaths", C.c_uint64 * 5), ("shadowTraced", C.c_uint64)]


class BvhInfoC(C.Structure):
    _fields_ = [("numTriangles", C.c_uint32), ("numNodes", C.c_uint32), ("numBinaryNodes", C.c_uint32),
                ("depth", C.c_uint32), ("numEmissive", C.c_uint32), ("buildMs", C.c_float), ("sahCost", C.c_float)]


class ServerConfigC(C.Structure):
    _fields_ = [("capacity", C.c_uint32), ("maxRequests", C.c_uint32), ("poolBytes", C.c_uint64),
                ("chunk", C.c_uint32), ("shadeBlock", C.c_uint32)]


class ServerStatusC(C.Structure):
    _fields_ = [("queued", C.c_uint32), ("running", C.c_uint32), ("ready", C.c_uint32), ("iterations", C.c_uint64),
                ("lastChunkMs", C.c_float), ("poolFreeBytes", C.c_uint64)]


class RequestInfoC(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("spp", C.c_uint32), ("denoised", C.c_uint32),
                ("submitMs", C.c_double), ("admitMs", C.c_double), ("readyMs", C.c_double),
                ("iterations", C.c_uint32)]


class TuneTrialC(C.Structure):
    _fields_ = [("capacity", C.c_uint32), ("chunk", C.c_uint32), ("shadeBlock", C.c_uint32), ("ms", C.c_float)]


class TuneResultC(C.Structure):
    _fields_ = [("capacity", C.c_uint32), ("chunk", C.c_uint32), ("shadeBlock", C.c_uint32), ("bestMs", C.c_float),
                ("numTrials", C.c_uint32), ("trials", TuneTrialC * 32)]


WRK_FLAG_DENOISE = 4

# Every entry point include/wrk.h declares, with its ctypes signature.
_VP, _U32, _U64, _I, _F = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int, C.c_float
SIGNATURES = {
    "wrk_last_error": ([], C.c_char_p),
    "wrk_version": ([], _I),
    "wrk_device_count": ([C.POINTER(C.c_int)], _I),
    "wrk_malloc": ([_I, _U64, C.POINTER(_VP)], _I),
    "wrk_free": ([_VP], _I),
    "wrk_memcpy_htod": ([_VP, _VP, _U64], _I),
    "wrk_memcpy_dtoh": ([_VP, _VP, _U64], _I),
    "wrk_synchronize": ([_I], _I),
    "wrk_scene_create": ([_I, C.POINTER(_VP)], _I),
    "wrk_scene_destroy": ([_VP], _I),
    "wrk_scene_set_geometry": ([_VP, _VP, _U32, _VP, _VP, _VP, _U32, _VP], _I),
    "wrk_scene_set_materials": ([_VP, _VP, _U32], _I),
    "wrk_scene_add_texture": ([_VP, _VP, _U32, _U32, C.POINTER(_U32)], _I),
    "wrk_scene_set_environment": ([_VP, _VP], _I),
    "wrk_scene_set_environment_map": ([_VP, _VP, _U32, _U32], _I),
    "wrk_scene_finalize": ([_VP], _I),
    "wrk_scene_bvh_info": ([_VP, C.POINTER(BvhInfoC)], _I),
    "wrk_scene_light_cdf": ([_VP, _VP, _VP, _U32, C.POINTER(_U32)], _I),
    "wrk_scene_buffers_get": ([_VP, _VP], _I),
    "wrk_scene_bvh_export": ([_VP, _VP, _VP], _I),
    "wrk_renderer_create": ([_I, _U32, C.POINTER(_VP)], _I),
    "wrk_renderer_destroy": ([_VP], _I),
    "wrk_render": ([_VP, _VP, C.POINTER(CameraC), C.POINTER(RenderParamsC), _VP, _VP, _VP,
                    C.POINTER(RenderStatsC)], _I),
    "wrk_render_device": ([_VP, _VP, C.POINTER(CameraC), C.POINTER(RenderParamsC), _VP, _VP, _VP,
                           C.POINTER(RenderStatsC)], _I),
    "wrk_trace_closest": ([_VP, _VP, _U32, _VP, _VP], _I),
    "wrk_trace_occluded": ([_VP, _VP, _U32, _VP], _I),
    "wrk_compact": ([_VP, _VP, _U32, _VP, _VP], _I),
    "wrk_compact_noalloc": ([_VP, _VP, _U32, _VP, _VP], _I),
    "wrk_cdf_sample": ([_VP, _U32, _VP, _U32, _VP], _I),
    "wrk_rng_batch": ([_VP, _VP, _U32, _VP, _VP], _I),
    "wrk_bsdf_batch": ([_VP, _U32, _VP], _I),
    "wrk_texture_batch": ([_VP, _U32, _VP, _U32, _VP], _I),
    "wrk_camera_rays": ([C.POINTER(CameraC), _U32, _U32, _VP, _VP, _U32, _U32, _VP], _I),
    "wrk_tonemap_aces": ([_VP, _U32, _VP], _I),
    "wrk_image_save_png": ([C.c_char_p, _VP, _U32, _U32], _I),
    "wrk_png_write": ([C.c_char_p, _VP, _U32, _U32], _I),
    "wrk_exr_write": ([C.c_char_p, _VP, _U32, _U32], _I),
    "wrk_hdr_write": ([C.c_char_p, _VP, _U32, _U32], _I),
    "wrk_renderer_set_launch": ([_VP, _U32, _U32], _I),
    "wrk_server_create": ([_I, _VP, C.POINTER(_VP)], _I),
    "wrk_server_destroy": ([_VP], _I),
    "wrk_server_set_denoiser": ([_VP, _VP], _I),
    "wrk_server_submit": ([_VP, _VP, C.POINTER(CameraC), C.POINTER(RenderParamsC), C.POINTER(_U64)], _I),
    "wrk_server_step": ([_VP, _VP], _I),
    "wrk_server_poll": ([_VP, _U64, C.POINTER(C.c_int)], _I),
    "wrk_server_wait": ([_VP, _U64], _I),
    "wrk_server_result": ([_VP, _U64, _VP, _VP, _VP, _VP], _I),
    "wrk_server_result_device": ([_VP, _U64, _VP, _VP, _VP, _VP], _I),
    "wrk_autotune": ([_I, _VP, C.POINTER(CameraC), C.POINTER(RenderParamsC), _VP], _I),
    "wrk_conv3x3_forward": ([_VP, _U32, _U32, _U32, _U32, _VP, _VP, _U32, _U32, _VP], _I),
    "wrk_conv3x3_wgrad": ([_VP, _VP, _U32, _U32, _U32, _U32, _U32, _VP], _I),
    "wrk_denoiser_create": ([_I, _U32, C.POINTER(_VP)], _I),
    "wrk_denoiser_destroy": ([_VP], _I),
    "wrk_denoiser_num_params": ([_VP, C.POINTER(_U64)], _I),
    "wrk_denoiser_get_params": ([_VP, _VP, _U64], _I),
    "wrk_denoiser_set_params": ([_VP, _VP, _U64], _I),
    "wrk_denoiser_gradients": ([_VP, _VP, _VP, _VP, _VP, _U32, _U32, _U32, _VP, C.POINTER(_F)], _I),
    "wrk_denoiser_train_step": ([_VP, _VP, _VP, _VP, _VP, _U32, _U32, _U32, _F, C.POINTER(_F)], _I),
    "wrk_denoiser_infer": ([_VP, _VP, _VP, _VP, _U32, _U32, _U32, _VP], _I),
    "wrk_denoiser_last_ms": ([_VP, C.POINTER(_F)], _I),
    "wrk_denoiser_grads_copy": ([_VP, _VP], _I),
    "wrk_denoiser_grads_set": ([_VP, _VP], _I),
    "wrk_denoiser_apply": ([_VP, _F], _I),
    "wrk_denoiser_load": ([_VP, C.c_char_p], _I),
}

_lib = None


def lib() -> C.CDLL:
    """Loads libwrk.so (built in-tree by offlinerenderer_b200.build); raises if absent."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m offlinerenderer_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def _check(rc: int) -> None:
    if rc != 0:
        raise WrkError(rc, lib().wrk_last_error().decode())


def device_count() -> int:
    n = C.c_int(0)
    _check(lib().wrk_device_count(C.byref(n)))
    return n.value


class DeviceArray:
    """Device memory from wrk_malloc holding one numpy-typed array."""

    def __init__(self, shape, dtype, device: int = 0):
        self.shape = tuple(np.atleast_1d(shape)) if not isinstance(shape, tuple) else shape
        self.dtype = np.dtype(dtype)
        self.nbytes = int(np.prod(self.shape)) * self.dtype.itemsize
        p = C.c_void_p()
        _check(lib().wrk_malloc(device, max(1, self.nbytes), C.byref(p)))
        self.ptr = p.value

    @classmethod
    def from_numpy(cls, a: np.ndarray, device: int = 0) -> "DeviceArray":
        a = np.ascontiguousarray(a)
        d = cls(a.shape, a.dtype, device)
        if d.nbytes:
            _check(lib().wrk_memcpy_htod(d.ptr, a.ctypes.data, d.nbytes))
        return d

    def numpy(self) -> np.ndarray:
        out = np.empty(self.shape, self.dtype)
        if self.nbytes:
            _check(lib().wrk_memcpy_dtoh(out.ctypes.data, self.ptr, self.nbytes))
        return out

    def __del__(self):
        p = getattr(self, "ptr", None)
        if p and _lib is not None:
            _lib.wrk_free(p)
            self.ptr = None


class TensorPtr:
    """A torch CUDA tensor passed where the binding takes a DeviceArray.  The library
    works on its own CUDA streams, so the work torch queued to produce the tensor is
    waited for here, before the library reads it."""

    def __init__(self, t):
        import torch

        if t.is_cuda:
            torch.cuda.current_stream(t.device).synchronize()
        self.t = t
        self.ptr = t.data_ptr()


def camera_struct(cam) -> CameraC:
    c = CameraC()
    c.position[:] = tuple(cam.position)
    c.target[:] = tuple(cam.target)
    c.up[:] = tuple(cam.up)
    c.fovY, c.aspect = cam.fovY, cam.aspect
    c.focalDistance, c.lensRadius = cam.focalDistance, cam.lensRadius
    return c


def params_struct(st, spp=None, max_iterations=8, raw_guides=False, seed=None, sample_offset=0,
                  stage_timing=False, env_map=False) -> RenderParamsC:
    p = RenderParamsC()
    p.width, p.height = st.width, st.height
    p.spp = st.spp if spp is None else spp
    p.useNEE = 1 if st.useNEE else 0
    p.maxBounces = st.maxBounces
    p.russianRouletteDepth = st.russianRouletteDepth
    p.fireflyClamp = st.fireflyClamp
    p.seed = st.seed if seed is None else seed
    p.maxIterations = max_iterations
    p.flags = ((WRK_FLAG_RAW_GUIDES if raw_guides else 0) | (WRK_FLAG_STAGE_TIMING if stage_timing else 0)
               | (WRK_FLAG_ENV_MAP if env_map else 0))
    p.sampleOffset = sample_offset
    return p


def _stats_dict(stats: "RenderStatsC") -> dict:
    d = {k: getattr(stats, k) for k, _ in RenderStatsC._fields_ if k not in ("stageMs", "stageLaunches", "bucketPaths")}
    d["bucketPaths"] = {n: stats.bucketPaths[i] for i, n in enumerate(BUCKETS)}
    d["stageMs"] = {n: stats.stageMs[i] for i, n in enumerate(STAGES)}
    d["stageLaunches"] = {n: stats.stageLaunches[i] for i, n in enumerate(STAGES)}
    return d


class Scene:
    """wr::Scene: materials and meshes are accumulated on the host; finalize()
    uploads them, builds the light CDF and the GPU BVH."""

    def __init__(self, device: int = 0):
        self.device = device
        self._b = _scenes._Builder()
        self._env = (0.0, 0.0, 0.0)
        self.handle = None

    # material creation with libWR's defaults (scene.cpp:91-168)
    def addLambertianMaterial(self, albedo, albedoTextureId: int = 0) -> int:
        return self._b.lambertian(tuple(albedo), albedoTextureId)

    def addEmissiveMaterial(self, emission) -> int:
        return self._b.emissive(tuple(emission))

    def addGlassMaterial(self, albedo, ior: float) -> int:
        return self._b.glass(tuple(albedo), ior)

    def addGGXReflectionMaterial(self, albedo, roughness: float, metallic: float = 0.0) -> int:
        return self._b.ggx(tuple(albedo), roughness, metallic)

    def addGGXTransmissionMaterial(self, albedo, roughness: float, ior: float) -> int:
        return self._b.ggx_transmission(tuple(albedo), roughness, ior)

    def setMaterialNormalMap(self, materialId: int, normalTextureId: int) -> None:
        if materialId >= len(self._b.mats):
            raise WrkError(1, "Invalid material ID")
        self._b.mats[materialId]["normalTextureId"] = normalTextureId

    def addTexture(self, rgba: np.ndarray) -> int:
        """RGBA8 (H, W, 4) texture; returns the 1-based id (Texture2D::create)."""
        return self._b.texture(rgba)

    def addTriangleMesh(self, vertices, indices, materialId: int, normals=None, uvs=None) -> None:
        self._b.mesh(vertices, indices, materialId, normals=normals, uvs=uvs)

    def setEnvironmentRadiance(self, rgb) -> None:
        self._env = tuple(float(x) for x in rgb)

    def setEnvironmentMap(self, rgba: np.ndarray) -> None:
        """(H, W, 4) float lat-long map (Scene::setEnvironmentMap takes a .hdr path;
        the decoded texels are passed here); used by renders with env_map=True."""
        self._env_map = np.ascontiguousarray(rgba, np.float32)

    @classmethod
    def from_data(cls, sd: "_scenes.SceneData", device: int = 0) -> "Scene":
        s = cls(device)
        s._data = sd
        s._finalize_data(sd)
        return s

    def finalize(self) -> None:
        if self.handle is not None:
            return
        if not self._b.v:
            raise WrkError(1, "Scene has no geometry")
        sd = self._b.build(env=self._env, env_map=getattr(self, "_env_map", None))
        self._data = sd
        self._finalize_data(sd)

    def _finalize_data(self, sd) -> None:
        L = lib()
        h = C.c_void_p()
        _check(L.wrk_scene_create(self.device, C.byref(h)))
        self.handle = h.value
        v = np.ascontiguousarray(sd.vertices, np.float32)
        idx = np.ascontiguousarray(sd.indices, np.uint32)
        tm = np.ascontiguousarray(sd.tri_material, np.uint32)
        nrm = None if sd.normals is None else np.ascontiguousarray(sd.normals, np.float32)
        uv = None if sd.uvs is None else np.ascontiguousarray(sd.uvs, np.float32)
        _check(L.wrk_scene_set_geometry(self.handle, v.ctypes.data, v.shape[0], None if nrm is None else nrm.ctypes.data,
                                        None if uv is None else uv.ctypes.data, idx.ctypes.data, idx.shape[0],
                                        tm.ctypes.data))
        mats = np.ascontiguousarray(sd.materials)
        _check(L.wrk_scene_set_materials(self.handle, mats.ctypes.data, mats.shape[0]))
        for t in sd.textures:
            t = np.ascontiguousarray(t, np.uint8)
            tid = C.c_uint32()
            _check(L.wrk_scene_add_texture(self.handle, t.ctypes.data, t.shape[1], t.shape[0], C.byref(tid)))
        env = np.asarray(sd.env, np.float32)
        _check(L.wrk_scene_set_environment(self.handle, env.ctypes.data))
        if sd.env_map is not None:
            em = np.ascontiguousarray(sd.env_map, np.float32)
            _check(L.wrk_scene_set_environment_map(self.handle, em.ctypes.data, em.shape[1], em.shape[0]))
        _check(L.wrk_scene_finalize(self.handle))

    def __del__(self):
        h = getattr(self, "handle", None)
        if h and _lib is not None:
            _lib.wrk_scene_destroy(h)
            self.handle = None

    def bvh_info(self) -> dict:
        info = BvhInfoC()
        _check(lib().wrk_scene_bvh_info(self.handle, C.byref(info)))
        return {k: getattr(info, k) for k, _ in BvhInfoC._fields_}

    def bvh_export(self):
        """(nodes (N,20) u32, tris (T,12) f32) of the 8-wide BVH as built on the device."""
        info = self.bvh_info()
        nodes = np.zeros((info["numNodes"], 20), np.uint32)
        tris = np.zeros((info["numTriangles"], 12), np.float32)
        _check(lib().wrk_scene_bvh_export(self.handle, nodes.ctypes.data, tris.ctypes.data))
        return nodes, tris

    def light_cdf(self):
        n = C.c_uint32()
        _check(lib().wrk_scene_light_cdf(self.handle, None, None, 0, C.byref(n)))
        tris = np.zeros(n.value, np.uint32)
        cdf = np.zeros(n.value, np.float32)
        _check(lib().wrk_scene_light_cdf(self.handle, tris.ctypes.data, cdf.ctypes.data, n.value, C.byref(n)))
        return tris, cdf

    def trace_closest(self, rays: np.ndarray):
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        n = rays.shape[0]
        dr = DeviceArray.from_numpy(rays, self.device)
        dt = DeviceArray((n,), np.float32, self.device)
        dp = DeviceArray((n,), np.uint32, self.device)
        _check(lib().wrk_trace_closest(self.handle, dr.ptr, n, dt.ptr, dp.ptr))
        return dt.numpy(), dp.numpy()

    def trace_occluded(self, rays: np.ndarray):
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        n = rays.shape[0]
        dr = DeviceArray.from_numpy(rays, self.device)
        do = DeviceArray((n,), np.uint32, self.device)
        _check(lib().wrk_trace_occluded(self.handle, dr.ptr, n, do.ptr))
        return do.numpy()

    def texture_batch(self, texture_id: int, uv: np.ndarray) -> np.ndarray:
        uv = np.ascontiguousarray(uv, np.float32).reshape(-1, 2)
        n = uv.shape[0]
        du = DeviceArray.from_numpy(uv, self.device)
        do = DeviceArray((n, 4), np.float32, self.device)
        _check(lib().wrk_texture_batch(self.handle, texture_id, du.ptr, n, do.ptr))
        return do.numpy()


@dataclasses.dataclass
class RenderResult:
    rgb: np.ndarray
    albedo: np.ndarray | None
    normal: np.ndarray | None
    stats: dict


class Renderer:
    """wr::Renderer: one CUDA stream and a pool of ``capacity`` path slots."""

    def __init__(self, device: int = 0, capacity: int = 0):
        self.device = device
        h = C.c_void_p()
        _check(lib().wrk_renderer_create(device, capacity, C.byref(h)))
        self.handle = h.value

    def __del__(self):
        h = getattr(self, "handle", None)
        if h and _lib is not None:
            _lib.wrk_renderer_destroy(h)
            self.handle = None

    def set_launch(self, chunk: int = 8, shade_block: int = 256) -> None:
        _check(lib().wrk_renderer_set_launch(self.handle, chunk, shade_block))

    def render(self, scene: Scene, camera=None, settings=None, spp=None, guides=True, raw_guides=False,
               max_iterations=8, seed=None, sample_offset=0, stage_timing=False, env_map=False,
               out=None) -> RenderResult:
        """Synchronous render into host buffers (rgb = sum/spp, as libWR returns it).

        out: optional (rgb, albedo, normal) float32 C-contiguous (height, width, 3)
        arrays to write into (albedo / normal may be None when guides is False), as
        libWR's caller-owned output buffer; pinned host memory makes the copy faster."""
        cam = camera_struct(camera or scene._data.camera)
        st = settings or scene._data.settings
        p = params_struct(st, spp=spp, max_iterations=max_iterations, raw_guides=raw_guides, seed=seed,
                          sample_offset=sample_offset, stage_timing=stage_timing, env_map=env_map)
        shape = (st.height, st.width, 3)
        if out is not None:
            rgb, alb, nrm = out
            for a in (rgb, alb, nrm):
                if a is not None and (a.shape != shape or a.dtype != np.float32 or not a.flags["C_CONTIGUOUS"]):
                    raise ValueError(f"output arrays must be float32, C-contiguous, shape {shape}")
            if not guides:
                alb = nrm = None
        else:
            rgb = np.zeros(shape, np.float32)
            alb = np.zeros(shape, np.float32) if guides else None
            nrm = np.zeros(shape, np.float32) if guides else None
        stats = RenderStatsC()
        _check(lib().wrk_render(self.handle, scene.handle, C.byref(cam), C.byref(p), rgb.ctypes.data,
                                None if alb is None else alb.ctypes.data, None if nrm is None else nrm.ctypes.data,
                                C.byref(stats)))
        return RenderResult(rgb, alb, nrm, _stats_dict(stats))

    def render_device(self, scene: Scene, d_rgb: DeviceArray, camera=None, settings=None, spp=None,
                      d_albedo: DeviceArray | None = None, d_normal: DeviceArray | None = None,
                      max_iterations=8, seed=None, sample_offset=0, stage_timing=False, d_rgb_ptr=None) -> dict:
        """Render into device buffers (inputs and outputs stay in HBM)."""
        cam = camera_struct(camera or scene._data.camera)
        st = settings or scene._data.settings
        p = params_struct(st, spp=spp, max_iterations=max_iterations, seed=seed, sample_offset=sample_offset,
                          stage_timing=stage_timing)
        stats = RenderStatsC()
        out_ptr = d_rgb_ptr if d_rgb_ptr is not None else d_rgb.ptr
        _check(lib().wrk_render_device(self.handle, scene.handle, C.byref(cam), C.byref(p), out_ptr,
                                       None if d_albedo is None else d_albedo.ptr,
                                       None if d_normal is None else d_normal.ptr, C.byref(stats)))
        return _stats_dict(stats)


# ---- kernel-level entry points (numpy in / numpy out) ----
def compact(stage: np.ndarray, idx: np.ndarray, device: int = 0) -> np.ndarray:
    ds = DeviceArray.from_numpy(np.asarray(stage, np.uint32), device)
    di = DeviceArray.from_numpy(np.asarray(idx, np.uint32), device)
    do = DeviceArray((max(1, len(idx)),), np.uint32, device)
    dc = DeviceArray((1,), np.uint32, device)
    _check(lib().wrk_compact(ds.ptr, di.ptr, len(idx), do.ptr, dc.ptr))
    return do.numpy()[: int(dc.numpy()[0])]


def cdf_sample(cdf: np.ndarray, u: np.ndarray, device: int = 0) -> np.ndarray:
    dc = DeviceArray.from_numpy(np.asarray(cdf, np.float32), device)
    du = DeviceArray.from_numpy(np.asarray(u, np.float32), device)
    do = DeviceArray((len(u),), np.uint32, device)
    _check(lib().wrk_cdf_sample(dc.ptr, len(cdf), du.ptr, len(u), do.ptr))
    return do.numpy()


def rng_batch(seeds: np.ndarray, dims: np.ndarray, device: int = 0):
    n = len(seeds)
    ds = DeviceArray.from_numpy(np.asarray(seeds, np.uint32), device)
    dd = DeviceArray.from_numpy(np.asarray(dims, np.uint32), device)
    dh = DeviceArray((n,), np.uint32, device)
    du = DeviceArray((n,), np.float32, device)
    _check(lib().wrk_rng_batch(ds.ptr, dd.ptr, n, dh.ptr, du.ptr))
    return dh.numpy(), du.numpy()


def bsdf_batch(records: np.ndarray, device: int = 0) -> np.ndarray:
    records = np.ascontiguousarray(records, np.float32).reshape(-1, 20)
    n = records.shape[0]
    di = DeviceArray.from_numpy(records, device)
    do = DeviceArray((n, 34), np.float32, device)
    _check(lib().wrk_bsdf_batch(di.ptr, n, do.ptr))
    return do.numpy()


def camera_rays(camera, width: int, height: int, pixels, samples, seed: int = 0, device: int = 0) -> np.ndarray:
    pixels = np.asarray(pixels, np.uint32)
    n = len(pixels)
    dp = DeviceArray.from_numpy(pixels, device)
    ds = DeviceArray.from_numpy(np.asarray(samples, np.uint32), device)
    do = DeviceArray((n, 8), np.float32, device)
    cam = camera_struct(camera)
    _check(lib().wrk_camera_rays(C.byref(cam), width, height, dp.ptr, ds.ptr, n, seed, do.ptr))
    return do.numpy()


def tonemap_aces(rgb: np.ndarray, device: int = 0) -> np.ndarray:
    rgb = np.ascontiguousarray(rgb, np.float32)
    npx = rgb.size // 3
    di = DeviceArray.from_numpy(rgb, device)
    do = DeviceArray(rgb.shape, np.uint8, device)
    _check(lib().wrk_tonemap_aces(di.ptr, npx, do.ptr))
    return do.numpy()


# ---- learned denoiser ----
def to_bf16_bits(a: np.ndarray) -> np.ndarray:
    """f32 -> bf16 bit patterns (round to nearest even), as uint16."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32)
    return ((u + (((u >> 16) & 1) + 0x7FFF)) >> 16).astype(np.uint16)


def from_bf16_bits(b: np.ndarray) -> np.ndarray:
    return (np.asarray(b, np.uint16).astype(np.uint32) << 16).view(np.float32)


def conv3x3(x: np.ndarray, w: np.ndarray, bias=None, relu=False, f32_out=True, device: int = 0) -> np.ndarray:
    """Tensor-core 3x3 convolution: x (B,H,W,Cin) and w (Cout,3,3,Cin) are rounded to
    bf16; returns (B,H,W,Cout) f32 (or the bf16 result widened to f32)."""
    B, H, W, Cin = x.shape
    Cout = w.shape[0]
    dx = DeviceArray.from_numpy(to_bf16_bits(x), device)
    dw = DeviceArray.from_numpy(to_bf16_bits(w), device)
    db = None if bias is None else DeviceArray.from_numpy(np.asarray(bias, np.float32), device)
    do = DeviceArray((B, H, W, Cout), np.float32 if f32_out else np.uint16, device)
    flags = (1 if relu else 0) | (2 if f32_out else 0)
    _check(lib().wrk_conv3x3_forward(dx.ptr, B, H, W, Cin, dw.ptr, None if db is None else db.ptr, Cout, flags,
                                     do.ptr))
    out = do.numpy()
    return out if f32_out else from_bf16_bits(out)


def conv3x3_wgrad(g: np.ndarray, x: np.ndarray, device: int = 0) -> np.ndarray:
    """dW (Cout,3,3,Cin) = sum_p g[p] x[p + tap] with g (B,H,W,Cout), x (B,H,W,Cin) in bf16."""
    B, H, W, Cin = x.shape
    Cout = g.shape[3]
    dg = DeviceArray.from_numpy(to_bf16_bits(g), device)
    dx = DeviceArray.from_numpy(to_bf16_bits(x), device)
    dw = DeviceArray.from_numpy(np.zeros((Cout, 3, 3, Cin), np.float32), device)
    _check(lib().wrk_conv3x3_wgrad(dg.ptr, dx.ptr, B, H, W, Cin, Cout, dw.ptr))
    return dw.numpy()


class Denoiser:
    """The learned U-Net denoiser (stands in for libWR's OptiX AI denoiser)."""

    def __init__(self, device: int = 0, seed: int = 1):
        self.device = device
        h = C.c_void_p()
        _check(lib().wrk_denoiser_create(device, seed, C.byref(h)))
        self.handle = h.value
        n = C.c_uint64()
        _check(lib().wrk_denoiser_num_params(self.handle, C.byref(n)))
        self.num_params = n.value

    def __del__(self):
        h = getattr(self, "handle", None)
        if h and _lib is not None:
            _lib.wrk_denoiser_destroy(h)
            self.handle = None

    def get_params(self) -> np.ndarray:
        out = np.zeros(self.num_params, np.float32)
        _check(lib().wrk_denoiser_get_params(self.handle, out.ctypes.data, self.num_params))
        return out

    def load(self, path: str) -> None:
        """Loads a WRKUNET1 weights file through the C ABI."""
        _check(lib().wrk_denoiser_load(self.handle, os.fsencode(path)))

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, np.float32)
        _check(lib().wrk_denoiser_set_params(self.handle, p.ctypes.data, p.size))

    @staticmethod
    def _ptr(a):
        return None if a is None else a.ptr

    def gradients(self, d_rgb, d_alb, d_nrm, d_target, B, H, W):
        g = np.zeros(self.num_params, np.float32)
        loss = C.c_float()
        _check(lib().wrk_denoiser_gradients(self.handle, d_rgb.ptr, self._ptr(d_alb), self._ptr(d_nrm), d_target.ptr,
                                            B, H, W, g.ctypes.data, C.byref(loss)))
        return loss.value, g

    def gradients_device(self, d_rgb, d_alb, d_nrm, d_target, B, H, W) -> float:
        """Forward + backward; the gradients stay on the device (grads_copy reads them)."""
        loss = C.c_float()
        _check(lib().wrk_denoiser_gradients(self.handle, d_rgb.ptr, self._ptr(d_alb), self._ptr(d_nrm),
                                            d_target.ptr, B, H, W, None, C.byref(loss)))
        return loss.value

    def grads_copy(self, d_out_ptr: int) -> None:
        _check(lib().wrk_denoiser_grads_copy(self.handle, d_out_ptr))

    def grads_set(self, d_in_ptr: int) -> None:
        _check(lib().wrk_denoiser_grads_set(self.handle, d_in_ptr))

    def apply(self, lr: float) -> None:
        _check(lib().wrk_denoiser_apply(self.handle, lr))

    def train_step(self, d_rgb, d_alb, d_nrm, d_target, B, H, W, lr: float) -> float:
        loss = C.c_float()
        _check(lib().wrk_denoiser_train_step(self.handle, d_rgb.ptr, self._ptr(d_alb), self._ptr(d_nrm), d_target.ptr,
                                             B, H, W, lr, C.byref(loss)))
        return loss.value

    def last_ms(self) -> float:
        """Device time of the last inference / training step."""
        ms = C.c_float()
        _check(lib().wrk_denoiser_last_ms(self.handle, C.byref(ms)))
        return ms.value

    def infer_device(self, d_rgb, d_alb, d_nrm, B, H, W, d_out) -> None:
        _check(lib().wrk_denoiser_infer(self.handle, d_rgb.ptr, self._ptr(d_alb), self._ptr(d_nrm), B, H, W,
                                        d_out.ptr))

    def infer(self, rgb: np.ndarray, albedo=None, normal=None) -> np.ndarray:
        """Denoise host images (H,W,3) or (B,H,W,3)."""
        rgb = np.asarray(rgb, np.float32)
        squeeze = rgb.ndim == 3
        r4 = rgb[None] if squeeze else rgb
        B, H, W, _ = r4.shape
        dr = DeviceArray.from_numpy(r4, self.device)
        da = None if albedo is None else DeviceArray.from_numpy(np.asarray(albedo, np.float32).reshape(r4.shape), self.device)
        dn = None if normal is None else DeviceArray.from_numpy(np.asarray(normal, np.float32).reshape(r4.shape), self.device)
        do = DeviceArray(r4.shape, np.float32, self.device)
        self.infer_device(dr, da, dn, B, H, W, do)
        out = do.numpy()
        return out[0] if squeeze else out


# ---- serving loop and autotuner ----
def _struct_dict(st) -> dict:
    return {k: getattr(st, k) for k, _ in st._fields_}


class Server:
    """Continuous-batching render server (wrk_server_*): requests of any size, spp,
    camera and scene share one set of wavefront queues on the device."""

    def __init__(self, device: int = 0, capacity: int = 0, max_requests: int = 0, pool_bytes: int = 0,
                 chunk: int = 0, shade_block: int = 0):
        self.device = device
        cfg = ServerConfigC(capacity, max_requests, pool_bytes, chunk, shade_block)
        h = C.c_void_p()
        _check(lib().wrk_server_create(device, C.byref(cfg), C.byref(h)))
        self.handle = h.value
        self._shapes = {}
        self._denoiser = None

    def __del__(self):
        h = getattr(self, "handle", None)
        if h and _lib is not None:
            _lib.wrk_server_destroy(h)
            self.handle = None

    def set_denoiser(self, dn: "Denoiser") -> None:
        self._denoiser = dn
        _check(lib().wrk_server_set_denoiser(self.handle, dn.handle))

    def submit(self, scene: Scene, camera=None, settings=None, spp=None, seed=None, sample_offset=0,
               max_iterations=8, denoise=False) -> int:
        cam = camera_struct(camera or scene._data.camera)
        st = settings or scene._data.settings
        p = params_struct(st, spp=spp, max_iterations=max_iterations, seed=seed, sample_offset=sample_offset)
        if denoise:
            p.flags |= WRK_FLAG_DENOISE
        t = C.c_uint64()
        _check(lib().wrk_server_submit(self.handle, scene.handle, C.byref(cam), C.byref(p), C.byref(t)))
        self._shapes[t.value] = (st.height, st.width)
        return t.value

    def step(self) -> dict:
        s = ServerStatusC()
        _check(lib().wrk_server_step(self.handle, C.byref(s)))
        return _struct_dict(s)

    def ready(self, ticket: int) -> bool:
        r = C.c_int()
        _check(lib().wrk_server_poll(self.handle, ticket, C.byref(r)))
        return bool(r.value)

    def wait(self, ticket: int) -> None:
        _check(lib().wrk_server_wait(self.handle, ticket))

    def result(self, ticket: int, guides: bool = True):
        """(rgb, albedo, normal, info) of a ready request; releases it."""
        h, w = self._shapes.pop(ticket)
        rgb = np.zeros((h, w, 3), np.float32)
        alb = np.zeros((h, w, 3), np.float32) if guides else None
        nrm = np.zeros((h, w, 3), np.float32) if guides else None
        info = RequestInfoC()
        _check(lib().wrk_server_result(self.handle, ticket, rgb.ctypes.data, None if alb is None else alb.ctypes.data,
                                       None if nrm is None else nrm.ctypes.data, C.byref(info)))
        return rgb, alb, nrm, _struct_dict(info)

    def result_device(self, ticket: int, d_rgb_ptr: int, d_albedo_ptr=None, d_normal_ptr=None) -> dict:
        self._shapes.pop(ticket, None)
        info = RequestInfoC()
        _check(lib().wrk_server_result_device(self.handle, ticket, d_rgb_ptr, d_albedo_ptr, d_normal_ptr,
                                              C.byref(info)))
        return _struct_dict(info)


def autotune(scene: Scene, camera=None, settings=None, spp=None, device: int = 0) -> dict:
    cam = camera_struct(camera or scene._data.camera)
    st = settings or scene._data.settings
    p = params_struct(st, spp=spp)
    r = TuneResultC()
    _check(lib().wrk_autotune(device, scene.handle, C.byref(cam), C.byref(p), C.byref(r)))
    return {"capacity": r.capacity, "chunk": r.chunk, "shadeBlock": r.shadeBlock, "bestMs": r.bestMs,
            "trials": [_struct_dict(r.trials[i]) for i in range(r.numTrials)]}


def save_exr(path: str, rgb: np.ndarray) -> None:
    """Write an (H, W, 3) float image as an uncompressed 32-bit float OpenEXR file."""
    rgb = np.ascontiguousarray(rgb, np.float32)
    h, w = rgb.shape[:2]
    _check(lib().wrk_exr_write(os.fsencode(path), rgb.ctypes.data, w, h))


def save_hdr(path: str, rgb: np.ndarray) -> None:
    """Write an (H, W, 3) float image as a Radiance RGBE (.hdr) file."""
    rgb = np.ascontiguousarray(rgb, np.float32)
    h, w = rgb.shape[:2]
    _check(lib().wrk_hdr_write(os.fsencode(path), rgb.ctypes.data, w, h))


def save_png(path: str, rgb: np.ndarray) -> None:
    """Tone map (ACES, on the GPU) and write an (H, W, 3) float image as a PNG."""
    rgb = np.ascontiguousarray(rgb, np.float32)
    h, w = rgb.shape[:2]
    _check(lib().wrk_image_save_png(os.fsencode(path), rgb.ctypes.data, w, h))
