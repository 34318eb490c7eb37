"""The C-ABI library builds, loads without a GPU, and exports every function
declared in include/mufflon_core.h. No compute call is made here."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions(header="mufflon_core.h", macro="CORE_API"):
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    src = "\n".join(l for l in src.splitlines() if not l.lstrip().startswith("#"))
    return sorted(set(re.findall(macro + r"\s+[^;]*?\b(\w+)\s*\(", src)))


def test_header_declares_core_interface():
    names = declared_functions()
    for required in ["mufflon_initialize", "mufflon_destroy", "render_iterate", "render_enable_renderer",
                     "render_get_renderer_name", "mufflon_get_target_image", "renderer_set_parameter_int",
                     "world_create_object", "polygon_add_vertex", "polygon_add_triangle_material",
                     "polygon_add_quad_material", "world_create_instance", "world_add_pinhole_camera",
                     "world_add_light", "world_add_material", "world_add_texture_value",
                     "world_create_scenario", "scenario_declare_material_slot", "scenario_assign_material",
                     "world_finalize_scenario", "world_load_scenario", "instance_set_transformation_matrix",
                     "render_save_screenshot", "render_enable_render_target"]:
        assert required in names, required


def test_library_exports_all_declared_symbols(core_lib_path):
    lib = ctypes.CDLL(core_lib_path)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_struct_layouts_match_reference_abi():
    from mufflon_b200 import bindings as b
    # sizes of the reference's C structs on x86-64 (core_interface.h)
    assert ctypes.sizeof(b.Vec3) == 12
    assert ctypes.sizeof(b.Mat3x4) == 48
    assert ctypes.sizeof(b.ProcessTime) == 16
    assert ctypes.sizeof(b.LightHdl) == 4
    assert ctypes.sizeof(b.MaterialParams) == 88
    assert b.MaterialParams.inner.offset == 56


def test_product_fails_loudly_without_gpu(core_lib_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from mufflon_b200 import bindings
    with pytest.raises(bindings.MufflonError):
        bindings.DllInterface(core_lib_path)


def test_missing_library_raises(tmp_path):
    from mufflon_b200 import bindings
    with pytest.raises(RuntimeError):
        bindings.DllHolder(str(tmp_path / "nope.so"))


def test_loader_library_exports_all_declared_symbols(core_lib_path):
    names = declared_functions("mff_interface.h", "LOADER_API")
    for required in ["loader_initialize", "loader_destroy", "loader_load_json", "loader_get_dll_error",
                     "loader_load_lod", "loader_abort", "loader_get_loading_status"]:
        assert required in names, required
    ctypes.CDLL(core_lib_path, mode=ctypes.RTLD_GLOBAL)
    lib = ctypes.CDLL(os.path.join(os.path.dirname(core_lib_path), "libmufflon_loader.so"))
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_reference_header_names_compile_and_link(core_lib_path, tmp_path):
    """A C99 program written against core_interface.h + mff_interface.h (the
    flow of examples/example.c) compiles and links against both libraries."""
    from tests.conftest import build_c_example
    exe = build_c_example(core_lib_path, str(tmp_path))
    assert os.path.exists(exe)
