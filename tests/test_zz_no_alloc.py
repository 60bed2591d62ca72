"""cpt_lbvh_build_static: the LBVH build for callers that cannot allocate.

Hosts such as an engine plugin whose application owns all device memory, or a
frame loop that must not call cudaMalloc (it can synchronize the device), build
through this entry point: its scratch is a fixed array inside the library, so the
call allocates nothing. These tests call it through the C ABI and require outputs
identical to the allocating entry point's (the build is integer/selection work:
bit-exact), on two calls in a row, and a clear rejection above its size limit.
The file sorts last so that a run stopping at the first failure has run the rest.
"""
import ctypes

import numpy as np
import pytest
import torch

import cpt
from cpt.device import DeviceLbvh, to_device

pytestmark = pytest.mark.gpu

MAX_TRIANGLES = 131072


def in_place_source(lb, tris):
    """The triangles copied into the output's own sorted-triangle array, which the
    build then permutes in place (as the reference permutes its scene's triangles)."""
    src = to_device(tris)
    torch.cuda.synchronize()
    lb.mem[: src.numel()].copy_(src)  # bvh.tris is the first array of the allocation
    assert lb.bvh.tris == lb.mem.data_ptr()
    return lb.bvh.tris


def static_build(tris, bits, check=True, in_place=False):
    lb = DeviceLbvh(len(tris), bits)  # outputs owned by the caller (torch memory); no scratch used
    src = to_device(tris)
    ptr = in_place_source(lb, tris) if in_place else src.data_ptr()
    box = cpt.scene_bounds(tris)
    rc = cpt.lib.cpt_lbvh_build_static(ptr, len(tris), box.ctypes.data, bits, ctypes.byref(lb.bvh),
                                       cpt.BUILD_CHECK if check else 0, torch.cuda.current_stream().cuda_stream)
    cpt.check(rc, "cpt_lbvh_build_static")
    torch.cuda.synchronize()
    return lb.download()


def allocating_build(tris, bits, in_place=False):
    lb = DeviceLbvh(len(tris), bits)
    src = to_device(tris)
    lb.build(in_place_source(lb, tris) if in_place else src, box=cpt.scene_bounds(tris), check_root=True)
    torch.cuda.synchronize()
    return lb.download()


def assert_identical(a, b):
    for k in a:
        assert np.ascontiguousarray(a[k]).tobytes() == np.ascontiguousarray(b[k]).tobytes(), k


@pytest.mark.parametrize("bits", [30, 63])
def test_static_build_equals_allocating_build_twice(cuda, bits):
    first = cpt.scene_random(MAX_TRIANGLES - 2, seed=31)[0]          # the largest accepted size
    second = cpt.scene_sphere_hairball(96, 64, 20_000, seed=32)[0]   # a different, smaller scene next
    for tris in (first, second):
        assert_identical(static_build(tris, bits), allocating_build(tris, bits))
    # and the first scene again after the second: nothing left over changes the result
    assert_identical(static_build(first, bits), allocating_build(first, bits))


@pytest.mark.parametrize("bits", [30, 63])
def test_static_build_in_place_at_the_limit(cuda, bits):
    """An in-place build (input = the output's triangle array) gathers from a copy of
    the triangles held in the fixed scratch, its largest piece (40 B per triangle):
    at the maximum size it must equal the allocating in-place build, twice."""
    tris = cpt.scene_random(MAX_TRIANGLES - 2, seed=33)[0]
    for _ in range(2):
        assert_identical(static_build(tris, bits, in_place=True), allocating_build(tris, bits, in_place=True))


def test_static_build_rejects_more_than_the_limit(cuda):
    n = MAX_TRIANGLES + 1
    lb_bvh = cpt.Bvh()
    rc = cpt.lib.cpt_lbvh_build_static(None, n, None, 63, ctypes.byref(lb_bvh), 0, None)
    assert rc == cpt.ERR_SCRATCH_TOO_SMALL
    tris = cpt.scene_random(1000, seed=1)[0]
    src = to_device(tris)
    lb = DeviceLbvh(len(tris), 30)
    rc = cpt.lib.cpt_lbvh_build_static(src.data_ptr(), 1, None, 30, ctypes.byref(lb.bvh), 0, None)
    assert rc == cpt.ERR_INVALID_ARGUMENT
