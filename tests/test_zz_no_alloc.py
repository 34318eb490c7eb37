"""The allocation-free sort entry point agrees with a stable sort and takes no
device memory.

mufflon_sort_pairs_device_noalloc exists for callers that cannot call
cudaMalloc (an engine that owns all device memory, a frame loop that must not
stall in cudaMalloc/cudaFree). It sorts device-resident pairs in place using a
fixed scratch array inside the library. This test does the documented set-up
(mufflon_initialize, which prepares the array on its device), hands the entry
point device buffers that the test itself allocates, and calls it twice in a
row, so that the second call starts from the first call's leftover scratch
contents. Each result is compared with numpy's stable argsort of the same keys
(an implementation independent of the library's radix sort) and with the
allocating mufflon_sort_pairs; the outputs are integers, so they must be
identical. The device's free memory must be the same before and after each
call. A size beyond the maximum must be rejected.

The file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_PAIRS = 1 << 20


def _lib(path):
    lib = ctypes.CDLL(path)
    lib.mufflon_sort_pairs_device_noalloc.restype = ctypes.c_uint32
    lib.mufflon_sort_pairs_device_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p]
    lib.mufflon_sort_pairs.restype = ctypes.c_uint32
    lib.mufflon_sort_pairs.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32]
    lib.mufflon_initialize.restype = ctypes.c_void_p
    lib.mufflon_destroy.argtypes = [ctypes.c_void_p]
    lib.core_get_dll_error.restype = ctypes.c_char_p
    return lib


def _input(n, seed):
    rng = np.random.default_rng(seed)
    keys = rng.integers(0, 1 << 63, n, dtype=np.uint64)
    keys[::3] = keys[0]                      # many equal keys: stability matters
    keys[: n // 5] = rng.integers(0, 64, n // 5).astype(np.uint64)
    vals = np.arange(n, dtype=np.int32)[::-1].copy()
    return keys, vals


def test_noalloc_sort_matches_stable_sort(core_lib_path):
    import torch
    lib = _lib(core_lib_path)
    inst = lib.mufflon_initialize()
    assert inst, lib.core_get_dll_error()
    try:
        stream = torch.cuda.current_stream()
        for call, n in enumerate([MAX_PAIRS, 300_007]):
            keys, vals = _input(n, 40 + call)
            order = np.argsort(keys, kind="stable")
            exp_k, exp_v = keys[order], vals[order]
            lib_k, lib_v = keys.copy(), vals.copy()
            assert lib.mufflon_sort_pairs(lib_k.ctypes.data, lib_v.ctypes.data, n), lib.core_get_dll_error()
            dk = torch.from_numpy(keys.view(np.int64)).cuda()
            dv = torch.from_numpy(vals).cuda()
            torch.cuda.synchronize()
            free_before = torch.cuda.mem_get_info()[0]
            ok = lib.mufflon_sort_pairs_device_noalloc(dk.data_ptr(), dv.data_ptr(), n, stream.cuda_stream)
            assert ok, lib.core_get_dll_error()
            torch.cuda.synchronize()
            free_after = torch.cuda.mem_get_info()[0]
            assert free_after == free_before, f"call {call}: free device memory {free_before} -> {free_after}"
            got_k = dk.cpu().numpy().view(np.uint64)
            got_v = dv.cpu().numpy()
            assert np.array_equal(got_k, exp_k), f"call {call}: keys differ from the stable sort"
            assert np.array_equal(got_v, exp_v), f"call {call}: values differ from the stable sort"
            assert np.array_equal(got_k, lib_k) and np.array_equal(got_v, lib_v), \
                f"call {call}: differs from mufflon_sort_pairs"
    finally:
        lib.mufflon_destroy(inst)


def test_noalloc_sort_rejects_oversized_input(core_lib_path):
    import torch
    lib = _lib(core_lib_path)
    dk = torch.zeros(4, dtype=torch.int64, device="cuda")
    dv = torch.zeros(4, dtype=torch.int32, device="cuda")
    assert not lib.mufflon_sort_pairs_device_noalloc(dk.data_ptr(), dv.data_ptr(), MAX_PAIRS + 1, None)
    assert b"exceeds the maximum" in lib.core_get_dll_error()
