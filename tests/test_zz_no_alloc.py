"""dfg_slice_gen_noalloc: slice generation for callers that cannot allocate
device memory while they run (their own pool allocator owns the device memory
budget, or a cudaMalloc / cudaFree would stall a real-time loop). It must give
what dfg_slice_gen gives, call after call, using only its fixed device array.

Collected last on purpose (file name), so a run that stops at the first
failure has already run every other test; it also passes alone in a fresh
process.
"""
import numpy as np
import pytest

from common import load_case

pytestmark = pytest.mark.gpu


def test_noalloc_slice_matches_allocating_entry_point_twice_in_a_row():
    from dragonfly_b200._lib import Context
    prob, _ = load_case("modes2")
    c = Context(0)
    c.set_detector(prob.qvals, prob.corr, prob.mask)
    c.set_model(prob.model1)
    # two calls in a row with different orientations and modes: the shared
    # array keeps the previous call's contents, which must not leak through
    for r, mode in ((5, 0), (211, 1)):
        ref = c.slice_gen(prob.quats[r], mode)
        got = c.slice_gen_noalloc(prob.quats[r], mode)
        np.testing.assert_array_equal(got, ref)  # slices are exact in the other tests too
    c.close()


def test_noalloc_rejects_detectors_beyond_its_scratch():
    from dragonfly_b200._lib import Context, DFGError
    import ctypes
    limit = 262144
    c = Context(0)
    n = limit + 1
    q = np.zeros((n, 3))
    q[:, 0] = np.linspace(-3., 3., n)
    c.set_detector(q, np.ones(n), np.zeros(n, np.uint8))
    c.set_model(np.ones((1, 9, 9, 9)))
    with pytest.raises(DFGError, match="more than the maximum"):
        c.slice_gen_noalloc(np.array([1., 0., 0., 0., 1.]))
    # the allocating entry point has no such limit
    assert c.slice_gen(np.array([1., 0., 0., 0., 1.])).shape == (n,)
    c.close()
