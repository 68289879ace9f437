"""vh_cornelius_surfaces_noalloc: the allocation-free Cornelius entry point.

It exists for callers that cannot let a library allocate device memory -- a
host framework whose own pool owns the whole GPU, or a per-event loop sharing
the GPU with other streams, where cudaMalloc would synchronise the device.  The
caller supplies every device buffer; the library's working memory is a fixed
device array, which limits a call to VH_NOALLOC_MAX_CUBES cubes.

The test calls it through the C ABI twice in a row on different inputs (3D
cubes, then 4D hypercubes, so leftovers from the first call would show in the
second) and checks counts and elements against the allocating entry point,
vh_cornelius_surfaces, bit for bit -- the tolerance every parity test here uses.
This file is named so pytest collects it last."""
import ctypes as C
import os
import sys

import numpy as np
import pytest

import vh

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import cornelius_kat as K  # noqa: E402

MAX_CUBES = 262144   # VH_NOALLOC_MAX_CUBES in include/vh_b200.h

f = vh.lib.vh_cornelius_surfaces_noalloc
f.restype = C.c_int
f.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_double, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
              C.c_void_p]


def _noalloc(dim, cubes, cap):
    import torch
    d_cubes = torch.from_numpy(np.ascontiguousarray(cubes, dtype=np.float64)).cuda()
    d_el = torch.full((cap, 2 * dim), -7.0, dtype=torch.float64, device="cuda")
    d_counts = torch.full((len(cubes),), -1, dtype=torch.int32, device="cuda")
    d_n = torch.full((1,), -2, dtype=torch.int32, device="cuda")
    dx = np.ones(dim)
    stream = torch.cuda.current_stream()
    rc = f(dim, d_cubes.data_ptr(), len(cubes), 0.5, dx.ctypes.data, d_el.data_ptr(), cap, d_counts.data_ptr(),
           d_n.data_ptr(), stream.cuda_stream)
    assert rc == 0, vh.lib.vh_last_error().decode()
    stream.synchronize()
    n = int(d_n.item())
    return d_el.cpu().numpy()[:max(n, 0)], d_counts.cpu().numpy(), n


def test_noalloc_matches_allocating_entry_point_twice_in_a_row():
    for dim in (3, 4):
        cubes = K.random_cubes(dim)
        ref_el, ref_counts = vh.cornelius_surfaces(dim, cubes, 0.5, np.ones(dim))
        el, counts, n = _noalloc(dim, cubes, cap=len(ref_el) + 16)
        assert n == len(ref_el)
        np.testing.assert_array_equal(counts, ref_counts)
        np.testing.assert_array_equal(el.view(np.uint64), ref_el.view(np.uint64))


def test_noalloc_truncates_to_cap_and_reports_the_total():
    """cap below the total: the first cap elements (cube order) are written and
    the total still comes back, so the caller sees the truncation"""
    cubes = K.random_cubes(3, 2000)
    ref_el, ref_counts = vh.cornelius_surfaces(3, cubes, 0.5, np.ones(3))
    cap = len(ref_el) // 3
    el, counts, n = _noalloc(3, cubes, cap=cap)
    assert n == len(ref_el) > cap
    np.testing.assert_array_equal(counts, ref_counts)
    np.testing.assert_array_equal(el[:cap].view(np.uint64), ref_el[:cap].view(np.uint64))


def test_noalloc_header_reset_between_calls():
    """no cubes gives zero elements; a call with fewer cubes after a larger one
    reports only its own elements (the shared header and counts start again)"""
    big = K.random_cubes(4, 3000)
    _noalloc(4, big, cap=1)
    el, counts, n = _noalloc(4, big[:0], cap=0)
    assert n == 0 and len(counts) == 0
    small = big[:200]
    ref_el, ref_counts = vh.cornelius_surfaces(4, small, 0.5, np.ones(4))
    el, counts, n = _noalloc(4, small, cap=len(ref_el) + 4)
    assert n == len(ref_el)
    np.testing.assert_array_equal(counts, ref_counts)
    np.testing.assert_array_equal(el.view(np.uint64), ref_el.view(np.uint64))


def test_noalloc_rejects_batches_over_the_limit():
    dummy = C.c_void_p(1)
    dx = np.ones(3)
    rc = f(3, dummy, MAX_CUBES + 1, 0.5, dx.ctypes.data, dummy, 1, dummy, dummy, None)
    assert rc == 1   # VH_ERR_ARG
    assert b"VH_NOALLOC_MAX_CUBES" in vh.lib.vh_last_error()
