"""Texture files through world_add_texture (core_interface.h:469-477,
interface.cpp:1790-1861): PFM read by the core ("PF" RGB with alpha 0, "Pf"
one channel, as src/pfmloader/interface.cpp:74-160), one texture per path,
the per-texel callback, the name and size queries, and the failures. A scene
whose albedo texture comes from a file renders the same bits as the same
texels given from memory, and the oracle's image."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from mufflon_b200 import bindings, scenefile, scenes

pytestmark = pytest.mark.gpu


def _render(spec, **kw):
    d = bindings.DllInterface()
    try:
        bindings.load_scene_spec(d, spec, **kw)
        assert d.render_enable_renderer(0, 0)
        assert d.renderer_set_parameter_int("Max. path length", 5)
        d.render_enable_render_target("Radiance", False)
        d.render_enable_render_target("Hit ID", False)
        for _ in range(2):
            d.render_iterate()
        return d.get_target_image("Radiance").copy(), d.get_target_image("Hit ID").copy()
    finally:
        d.close()


def _textured(tmp_path):
    tex = scenes.smooth_noise_texture(5, 32)
    spec = scenes.cornell_box_textured(5, 48, 48, texture=tex)
    path = tmp_path / "albedo.pfm"
    scenefile.write_pfm(str(path), spec.textures[0])
    return spec, path


def test_file_texture_renders_like_memory_texture_and_oracle(tmp_path, oracle):
    spec, path = _textured(tmp_path)
    img_file, hid_file = _render(spec, texture_files=[path])
    tex = spec.textures[0].copy()
    tex[..., 3] = 0.0  # a PFM file has no alpha channel
    spec_mem = scenes.cornell_box_textured(5, 48, 48, texture=tex)
    spec_mem.textures[0][..., 3] = 0.0
    img_mem, hid_mem = _render(spec_mem)
    assert np.array_equal(hid_file, hid_mem)
    assert np.array_equal(img_file.view(np.uint32), img_mem.view(np.uint32))
    pt = oracle.OraclePathTracer(oracle.OracleScene(spec_mem), seed=0, max_path=5)
    pt.iterate()
    pt.iterate()
    ref = pt.target("Radiance")
    assert np.sqrt(np.mean((img_file - ref) ** 2)) / np.sqrt(np.mean(ref ** 2)) <= 1e-4


@pytest.fixture(scope="module")
def callbacks(tmp_path_factory):
    """tests/cpp/texture_callbacks.c as a shared library (ctypes cannot define a
    callback that returns a struct by value)."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    so = str(tmp_path_factory.mktemp("cb") / "libtexture_callbacks.so")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-shared", "-fPIC", "-I", os.path.join(root, "include"),
                    os.path.join(root, "tests", "cpp", "texture_callbacks.c"), "-o", so], check=True, capture_output=True)
    lib = ctypes.CDLL(so)
    lib.callbacks_calls.restype = ctypes.c_uint32
    lib.callbacks_formats.restype = ctypes.c_uint32
    lib.callbacks_layers.restype = ctypes.c_uint32
    lib.callbacks_xy_sum.restype = ctypes.c_uint64
    lib.callbacks_values.restype = ctypes.POINTER(ctypes.c_float)
    return lib


def _cb(lib, name):
    return ctypes.cast(getattr(lib, name), bindings.TextureCallback)


def test_callback_rewrites_every_texel(tmp_path, callbacks):
    spec, path = _textured(tmp_path)
    callbacks.callbacks_reset()
    img_cb, _ = _render(spec, texture_files=[path], texture_callback=_cb(callbacks, "halve_red_quarter_green"))
    h, w = spec.textures[0].shape[:2]
    assert callbacks.callbacks_calls() == w * h
    assert callbacks.callbacks_layers() == 1                 # layer 0 only
    assert callbacks.callbacks_formats() == 1 << 11          # FORMAT_RGBA32F
    assert callbacks.callbacks_xy_sum() == sum(x + 65536 * y for y in range(h) for x in range(w))
    seen = np.ctypeslib.as_array(callbacks.callbacks_values(), shape=(64, 4))
    flat = spec.textures[0].reshape(-1, 4)
    assert np.array_equal(seen[:, :3], flat[:64, :3]) and not seen[:, 3].any()  # row-major, alpha 0
    tex = spec.textures[0].copy()
    tex[..., 0] *= 0.5
    tex[..., 1] *= 0.25
    spec2 = scenes.cornell_box_textured(5, 48, 48, texture=tex)
    img_mem, _ = _render(spec2)
    assert np.array_equal(img_cb.view(np.uint32), img_mem.view(np.uint32))


def test_queries_and_failures(tmp_path, dll, callbacks):
    core, inst = dll.core, dll.muffInst
    rgb = np.random.default_rng(1).uniform(0, 1, (3, 5, 3)).astype(np.float32)
    p_rgb = tmp_path / "a.pfm"
    scenefile.write_pfm(str(p_rgb), rgb)
    gray = np.arange(6, dtype="<f4").reshape(2, 3)
    p_gray = tmp_path / "g.pfm"
    p_gray.write_bytes(b"Pf\n3 2\n-1.0\n" + gray.tobytes())
    big = (np.arange(6).reshape(2, 3) + 10).astype(">f4")  # a positive scale: big-endian data
    p_big = tmp_path / "b.pfm"
    p_big.write_bytes(b"Pf\n3 2\n1.0\n" + big.tobytes())
    nocb = bindings.TextureCallback()
    t = core.world_add_texture(inst, str(p_rgb).encode(), 0, 0, nocb, None)
    assert t
    assert core.world_add_texture(inst, str(p_rgb).encode(), 0, 0, nocb, None) == t  # one texture per path
    assert core.world_get_texture(inst, str(p_rgb).encode()) == t
    assert core.world_get_texture_name(t).decode() == str(p_rgb)
    size = bindings.IVec2()
    assert core.world_get_texture_size(t, ctypes.byref(size)) and (size.x, size.y) == (5, 3)
    for path, arr in ((p_gray, gray), (p_big, big)):
        callbacks.callbacks_reset()
        assert core.world_add_texture(inst, str(path).encode(), 0, 0, _cb(callbacks, "record_only"), None)
        assert callbacks.callbacks_formats() == 1 << 9  # FORMAT_R32F
        seen = np.ctypeslib.as_array(callbacks.callbacks_values(), shape=(64, 4))[:6]
        assert np.array_equal(seen[:, 0], arr.astype(np.float32).reshape(-1)) and not seen[:, 1:].any()
    # failures: no reader for the format, a missing file, a truncated file
    (tmp_path / "x.png").write_bytes(b"\x89PNG")
    assert not core.world_add_texture(inst, str(tmp_path / "x.png").encode(), 0, 0, nocb, None)
    assert "PFM" in dll.core_get_dll_error()
    assert not core.world_add_texture(inst, str(tmp_path / "missing.pfm").encode(), 0, 0, nocb, None)
    assert "cannot open" in dll.core_get_dll_error()
    (tmp_path / "short.pfm").write_bytes(b"PF\n4 4\n-1.0\n" + np.zeros(5, "<f4").tobytes())
    assert not core.world_add_texture(inst, str(tmp_path / "short.pfm").encode(), 0, 0, nocb, None)
    assert "shorter" in dll.core_get_dll_error()
    assert not core.world_get_texture(inst, b"nope.pfm")
