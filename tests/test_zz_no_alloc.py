"""The allocation-free banded LU entry point (jfb_banded_lu_factor_noalloc).

Callers that cannot allocate device memory -- an XLA custom call or another
framework's operator whose device memory belongs to that framework's
allocator, a process whose caching pool already holds all of the GPU's memory
-- use this variant, which keeps its per-matrix pivot status in a fixed device
array of the library instead of allocating it.  Its factors must be those of
jfb_banded_lu_factor, call after call (the shared status array is cleared by
every call).
"""

import ctypes

import pytest
import torch

from jaxfun_b200 import _lib

pytestmark = pytest.mark.gpu

MAX_BATCH = 65536


def random_bands(seed, n_batch=96, p=4, q=12, n=41, device="cuda"):
    g = torch.Generator().manual_seed(seed)
    band = torch.randn((n_batch, p + q + 1, n), generator=g, dtype=torch.float64)
    band[:, p, :] += 4.0 * (p + q + 1)  # diagonally dominant: no pivoting needed
    return band.to(device).contiguous()


def stream_of(t):
    return ctypes.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)


def test_noalloc_matches_allocating_entry_point_on_consecutive_calls(cuda):
    lib = _lib.load()
    p, q, n = 4, 12, 41
    for seed in (0, 1):  # two calls in a row on different data
        band = random_bands(seed, p=p, q=q, n=n, device=cuda)
        ref, out = band.clone(), band.clone()
        nb = band.shape[0]
        _lib.call("jfb_banded_lu_factor", ref.data_ptr(), nb, p, q, n, stream_of(ref))
        first = ctypes.c_int32(-7)
        st = lib.jfb_banded_lu_factor_noalloc(out.data_ptr(), nb, p, q, n,
                                              ctypes.byref(first), stream_of(out))
        assert st == _lib.JFB_OK, lib.jfb_last_error()
        assert first.value == -1
        torch.testing.assert_close(out, ref, rtol=1e-14, atol=0.0)


def test_noalloc_reports_the_first_singular_matrix_then_recovers(cuda):
    lib = _lib.load()
    p, q, n = 2, 6, 17
    band = random_bands(2, n_batch=32, p=p, q=q, n=n, device=cuda)
    bad = band.clone()
    bad[9, p, 0] = 0.0   # zero first pivot of matrix 9
    bad[21, p, 0] = 0.0
    first = ctypes.c_int32(-7)
    st = lib.jfb_banded_lu_factor_noalloc(bad.data_ptr(), 32, p, q, n, ctypes.byref(first),
                                          stream_of(bad))
    assert st == _lib.JFB_ERR_SINGULAR
    assert first.value == 9
    # the status array is shared between calls; the next call must start clean
    good, ref = band.clone(), band.clone()
    st = lib.jfb_banded_lu_factor_noalloc(good.data_ptr(), 32, p, q, n, ctypes.byref(first),
                                          stream_of(good))
    assert st == _lib.JFB_OK and first.value == -1
    _lib.call("jfb_banded_lu_factor", ref.data_ptr(), 32, p, q, n, stream_of(ref))
    torch.testing.assert_close(good, ref, rtol=1e-14, atol=0.0)


def test_noalloc_rejects_batches_beyond_its_fixed_capacity(cuda):
    lib = _lib.load()
    band = random_bands(3, n_batch=1, device=cuda)
    st = lib.jfb_banded_lu_factor_noalloc(band.data_ptr(), MAX_BATCH + 1, 4, 12, 41, None,
                                          stream_of(band))
    assert st == _lib.JFB_ERR_ARG
    assert b"JFB_NOALLOC_LU_MAX_BATCH" in lib.jfb_last_error()


def test_noalloc_call_leaves_device_memory_unchanged(cuda):
    """The entry point's defining property: after a first call (which may
    load the library's kernels and with them the fixed status array), further
    calls take no device memory; the free memory the driver reports is the
    same before and after them."""
    lib = _lib.load()
    p, q, n = 4, 12, 41
    bands = [random_bands(seed, p=p, q=q, n=n, device=cuda) for seed in (4, 5, 6)]
    first = ctypes.c_int32(-7)
    st = lib.jfb_banded_lu_factor_noalloc(bands[0].data_ptr(), bands[0].shape[0], p, q, n,
                                          ctypes.byref(first), stream_of(bands[0]))
    assert st == _lib.JFB_OK
    torch.cuda.synchronize(cuda)
    free0, _ = torch.cuda.mem_get_info(cuda)
    for b in bands[1:]:
        st = lib.jfb_banded_lu_factor_noalloc(b.data_ptr(), b.shape[0], p, q, n,
                                              ctypes.byref(first), stream_of(b))
        assert st == _lib.JFB_OK and first.value == -1
    torch.cuda.synchronize(cuda)
    free1, _ = torch.cuda.mem_get_info(cuda)
    assert free1 == free0
