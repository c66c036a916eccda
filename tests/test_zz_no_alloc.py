"""The allocation-free FDMT entry point, bfs_fdmt_execute_noalloc.

This entry point is for callers that cannot allocate device memory where they
run the transform — for example a real-time receiver that reserves all of
its GPU memory at start-up and must not risk an allocation mid-observation,
or a host framework that owns the device allocator.  It runs the same kernels
as bfs_fdmt_execute with its scratch in a fixed 256 MiB array built into the
library, so these tests check, through the C ABI, that two calls in a row
give exactly what the allocating entry point gives (the FDMT is bit-exact, so
the tolerance is zero, as in the other FDMT tests), and that a problem too
large for the fixed array is refused with an error instead of running.

The file is named so pytest collects it last; it also passes on its own in a
fresh process (the first call on a device performs the one-time set-up).
"""
import ctypes

import numpy as np
import pytest
import torch

from cpp_projects_b200 import CFdmtGpu, _capi

pytestmark = pytest.mark.gpu


def _host_plan(fmin, fmax, nchan, ncols, max_dt, fuse=-1):
    desc = _capi.FdmtDesc(fmin=fmin, fmax=fmax, nchan=nchan, ncols=ncols, max_dt=max_dt,
                          fuse_depth=fuse)
    plan = ctypes.c_void_p()
    _capi.call("bfs_fdmt_plan_create_host", ctypes.byref(desc), ctypes.byref(plan))
    return plan


def _noalloc(plan, x, out):
    s = torch.cuda.current_stream()
    st = _capi.lib().bfs_fdmt_execute_noalloc(plan, ctypes.c_void_p(x.data_ptr()),
                                              ctypes.c_void_p(out.data_ptr()), 0,
                                              ctypes.c_void_p(s.cuda_stream))
    _capi.check(st)


@pytest.mark.parametrize("shape", [
    (1200.0, 1600.0, 512, 32768, 512),   # fused head + plain levels
    (1100.0, 1500.0, 100, 3001, 77),     # odd channel count: level-0 kernel + plain levels
])
def test_noalloc_matches_allocating_entry_point_on_two_calls(cuda, shape):
    fmin, fmax, nchan, ncols, max_dt = shape
    plan = _host_plan(*shape)
    try:
        need, cap = ctypes.c_size_t(), ctypes.c_size_t()
        _capi.call("bfs_fdmt_noalloc_scratch_bytes", plan, ctypes.byref(need), ctypes.byref(cap))
        assert need.value <= cap.value == 256 << 20
        ref = CFdmtGpu(fmin, fmax, nchan, ncols, max_dt)
        g = torch.Generator(cuda)
        for seed in (1, 2):  # the second call must not see the first call's data
            x = torch.randn((nchan, ncols), device=cuda, generator=g.manual_seed(seed))
            want = torch.empty((max_dt, ncols), device=cuda)
            ref.process_image(x, want)
            got = torch.full((max_dt, ncols), float("nan"), device=cuda)
            _noalloc(plan, x, got)
            torch.cuda.synchronize()
            assert torch.equal(got.view(torch.int32), want.view(torch.int32)), f"call {seed}"
    finally:
        _capi.lib().bfs_fdmt_plan_destroy(plan)


@pytest.mark.parametrize("shape", [
    (1200.0, 1600.0, 512, 32768, 512),
    (1100.0, 1500.0, 100, 3001, 77),
])
def test_noalloc_ones_mode_matches_allocating_entry_point_on_two_calls(cuda, shape):
    """b_ones != 0 (the normalisation image, no input): the allocating entry
    point may take its one-pass mask route; the allocation-free one runs the
    level kernels on an all-ones image.  Both must give the same bits."""
    fmin, fmax, nchan, ncols, max_dt = shape
    plan = _host_plan(*shape)
    try:
        ref = CFdmtGpu(fmin, fmax, nchan, ncols, max_dt)
        want = torch.empty((max_dt, ncols), device=cuda)
        ref.process_image(None, want, True)
        s = torch.cuda.current_stream()
        for call in (1, 2):
            got = torch.full((max_dt, ncols), float("nan"), device=cuda)
            st = _capi.lib().bfs_fdmt_execute_noalloc(plan, None, ctypes.c_void_p(got.data_ptr()), 1,
                                                      ctypes.c_void_p(s.cuda_stream))
            _capi.check(st)
            torch.cuda.synchronize()
            assert torch.equal(got.view(torch.int32), want.view(torch.int32)), f"call {call}"
    finally:
        _capi.lib().bfs_fdmt_plan_destroy(plan)


def test_noalloc_refuses_a_problem_larger_than_its_static_scratch(cuda):
    plan = _host_plan(1200.0, 1600.0, 4096, 131072, 4096)
    try:
        x = torch.zeros(1, device=cuda)
        out = torch.zeros(1, device=cuda)
        st = _capi.lib().bfs_fdmt_execute_noalloc(plan, ctypes.c_void_p(x.data_ptr()),
                                                  ctypes.c_void_p(out.data_ptr()), 0, None)
        assert st == _capi.BFS_ERR_ARG
        assert b"256 MiB" in _capi.lib().bfs_last_error()
    finally:
        _capi.lib().bfs_fdmt_plan_destroy(plan)
