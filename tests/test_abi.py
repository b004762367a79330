"""The C ABI: the library loads without a GPU, exports every function that
include/cgs.h declares, and fails loudly (no CPU fallback) when no device is
present."""
import ctypes
import os
import re
import subprocess

import pytest

from cindergs_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "cgs.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(cgs_\w+)\(", text, re.M)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for required in ("cgs_ctx_create", "cgs_execute_frame", "cgs_scene_upload",
                     "cgs_tet_cages_upload", "cgs_cage_vertices_update", "cgs_readback_rgba8",
                     "cgs_scan_u32", "cgs_sort_pairs_u32", "cgs_sort_pairs_u64"):
        assert required in names


def test_library_exports_every_declared_symbol():
    lib = _abi.load()
    exported = subprocess.run(["nm", "-D", "--defined-only", _abi.LIB_PATH], check=True,
                              capture_output=True, text=True).stdout
    syms = {line.split()[-1] for line in exported.splitlines() if line.strip()}
    for name in declared_functions():
        assert name in syms, name
        assert getattr(lib, name) is not None
    # the Python binding covers the same set
    assert set(_abi.SIGNATURES) == set(declared_functions())


def test_struct_layouts_match_the_reference_uniform_blocks():
    assert ctypes.sizeof(_abi.CgsCamera) == 96        # CameraUniforms (camera.rs:9-36)
    assert ctypes.sizeof(_abi.CgsCompositor) == 48    # CompositorUniforms (rasterizer/mod.rs:16-37)


def test_version_string():
    assert b"sm_100a" in _abi.load().cgs_version()


def test_kernel_names():
    lib = _abi.load()
    assert [lib.cgs_kernel_name(i).decode() for i in range(_abi.KERNEL_COUNT)] == \
        _abi.KERNEL_NAMES


def test_no_gpu_means_an_error_not_a_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from cindergs_b200 import GpuPipelineState
    with pytest.raises(_abi.CgsError):
        GpuPipelineState(0)


def test_null_arguments_are_rejected_without_a_device():
    lib = _abi.load()
    assert lib.cgs_ctx_create(0, None, None) == _abi.CGS_E_ARG
    assert lib.cgs_ctx_destroy(None) == _abi.CGS_E_ARG
    assert lib.cgs_execute_frame(None, None, None, None, None) == _abi.CGS_E_ARG
    assert lib.cgs_sort_pairs_u32_noalloc(None, None, 5, 32, 3, None) == _abi.CGS_E_ARG
    assert lib.cgs_sort_pairs_u32_noalloc(None, None, 5, 0, 8, None) == _abi.CGS_E_ARG
