"""The C ABI boundary without a GPU: libwrk.so loads, exports every entry point
include/wrk.h declares (and the drop-in C++ API), and fails loudly -- with an
error code and message, never a CPU fallback -- when no device is present."""
import ctypes as C
import os
import re
import subprocess

import pytest

from conftest import ROOT


def declared_entry_points():
    text = open(os.path.join(ROOT, "include", "wrk.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(wrk_\w+)\s*\(", text, re.M)))


def test_header_declares_entry_points():
    names = declared_entry_points()
    assert "wrk_render" in names and "wrk_trace_closest" in names and len(names) >= 30


def test_library_exports_every_declared_symbol(wrk_lib):
    L = C.CDLL(wrk_lib.LIB_PATH)
    missing = [n for n in declared_entry_points() if not hasattr(L, n)]
    assert not missing, missing


def test_binding_covers_every_declared_symbol(wrk_lib):
    assert set(declared_entry_points()) == set(wrk_lib.SIGNATURES)


def test_cpp_api_symbols_exported(wrk_lib):
    """The compiled part of the C++ API is exported, and none of it names Vec3,
    Camera, RenderParams or GLM: the members that take those are inline in
    include/wr, so one libwrk.so serves callers built with glm::vec3 (libWR's
    wr::Vec3) and with the GLM-free fallback."""
    out = subprocess.run(["nm", "-DC", "--defined-only", wrk_lib.LIB_PATH], capture_output=True, text=True).stdout
    for sym in ["wr::Scene::addTriangleMesh(std::span<float const", "wr::Scene::finalize(wr::SceneBuildConfig const&)",
                "wr::Renderer::renderNative(wr::Scene*, wrk_camera const&, wrk_render_params const&, float*, float*, "
                "float*, bool, char const*)",
                "wr::Context::createScene()", "wr::Texture2D::create(wr::Scene*",
                "wr::Scene::addMaterialRecord(wrk_material const&)",
                "wr::Scene::setEnvironmentRadianceRGB(float, float, float)"]:
        assert sym in out, sym
    wr_syms = [ln for ln in out.splitlines() if " wr::" in ln or " test_helpers::" in ln]
    assert wr_syms
    for ln in wr_syms:
        assert not re.search(r"Vec3|glm|wr::Camera|RenderParams", ln), ln


GLM_DIRS = [os.environ.get("WR_GLM_INCLUDE", ""), os.path.join(ROOT, "..", "reference", "libWR", "external")]


@pytest.mark.parametrize("glm", [False, True])
def test_cpp_api_compiles_and_links_with_and_without_glm(wrk_lib, tmp_path, glm):
    """A libWR-style program (GLM math on wr::Vec3, Camera's GLM helpers when GLM is
    present) compiles against include/wr and links against libwrk.so both ways."""
    flags = []
    if glm:
        found = [d for d in GLM_DIRS if d and os.path.exists(os.path.join(d, "glm", "glm.hpp"))]
        if not found:
            pytest.skip("GLM headers not found (set WR_GLM_INCLUDE)")
        flags = ["-I", found[0], "-DWR_EXPECT_GLM"]
    else:
        flags = ["-DWR_NO_GLM"]
    lib_dir = os.path.dirname(wrk_lib.LIB_PATH)
    r = subprocess.run(["g++", "-std=c++20", "-O1", "-I", os.path.join(ROOT, "include")] + flags +
                       [os.path.join(ROOT, "tests", "cpp", "api_types.cpp"), "-o", str(tmp_path / "api_types"),
                        "-L", lib_dir, "-lwrk", f"-Wl,-rpath,{lib_dir}"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_no_device_fails_loudly(wrk_lib):
    import ctypes

    if wrk_lib.device_count() > 0:
        pytest.skip("a GPU is visible; this checks the no-GPU error path")
    L = wrk_lib.lib()
    h = ctypes.c_void_p()
    rc = L.wrk_scene_create(0, ctypes.byref(h))
    assert rc == 4  # WRK_ERR_NO_DEVICE
    assert b"no CUDA device" in L.wrk_last_error()
    with pytest.raises(wrk_lib.WrkError):
        wrk_lib.Renderer()


def test_invalid_arguments_rejected_without_device(wrk_lib):
    L = wrk_lib.lib()
    assert L.wrk_device_count(None) == 1  # WRK_ERR_INVALID
    assert L.wrk_cdf_sample(None, 0, None, 0, None) == 1
