"""vf_sort2_noalloc: the 2D sort by cell for callers that cannot allocate device memory while they run.

Some hosts budget every byte of device memory up front, and some run a real-time loop in which a
cudaMalloc or cudaFree would synchronise the device and stall a frame; for them the library has one
entry point whose scratch is a fixed array inside the library. This checks it through the C-ABI against
vf_sort2 (which allocates its scratch per call) on two calls in a row, the second on different particles
and a different grid, so the counts the first call leaves behind must have been cleared. The sort is
integer work, so the comparison is exact. This file is collected last so a failure here stops nothing
else."""
import ctypes

import numpy as np
import pytest

import vexfluid as vf
from _oracle import JavaRandom, Particles

pytestmark = pytest.mark.gpu

_f32p = ctypes.POINTER(ctypes.c_float)
_i32p = ctypes.POINTER(ctypes.c_int32)


def noalloc():
    fn = vf.lib().vf_sort2_noalloc
    fn.argtypes = [ctypes.c_int32, ctypes.c_int32, _f32p, _f32p, ctypes.c_int64, _i32p, _i32p]
    fn.restype = ctypes.c_int32
    return fn


def sort_noalloc(n, p: Particles):
    perm = np.empty(p.count(), np.int32)
    starts = np.empty((n - 1) * (n - 1) + 1, np.int32)
    rc = noalloc()(n, n, p.x.ctypes.data_as(_f32p), p.y.ctypes.data_as(_f32p), p.count(),
                   perm.ctypes.data_as(_i32p), starts.ctypes.data_as(_i32p))
    vf.check(rc)
    return perm, starts


def test_sort_without_allocation_matches_the_allocating_sort_twice():
    first_n, second_n = 260, 41
    first = Particles.jittered(first_n - 1, 1, JavaRandom(21)).shuffled(JavaRandom(22))
    second = Particles.jittered(second_n - 1, 3, JavaRandom(33)).shuffled(JavaRandom(34))
    for n, p in ((first_n, first), (second_n, second)):
        perm, starts = sort_noalloc(n, p)
        want_perm, want_starts = vf.sort2(n, n, p.x, p.y)
        assert np.array_equal(starts, want_starts)
        assert np.array_equal(perm, want_perm)


def test_sort_without_allocation_refuses_inputs_beyond_its_fixed_scratch():
    big = 1 << 18
    x = np.zeros(big + 1, np.float32)
    perm = np.empty(big + 1, np.int32)
    starts = np.empty(16, np.int32)
    rc = noalloc()(4, 4, x.ctypes.data_as(_f32p), x.ctypes.data_as(_f32p), big + 1, perm.ctypes.data_as(_i32p),
                   starts.ctypes.data_as(_i32p))
    assert rc == vf.VF_EINVAL and "fixed array" in vf.last_error()
    rc = noalloc()(1000, 1000, x.ctypes.data_as(_f32p), x.ctypes.data_as(_f32p), 10, perm.ctypes.data_as(_i32p),
                   starts.ctypes.data_as(_i32p))
    assert rc == vf.VF_EINVAL and "cells" in vf.last_error()
