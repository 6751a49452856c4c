"""The allocation-free BSDF entry point (pt_bsdf_queries_host_noalloc) against the allocating one.

It serves callers that must not call cudaMalloc -- a host whose device memory is owned by its own
allocator, or a real-time thread where an allocation would synchronise the device -- by staging the
batch in one fixed 65536-query device array instead of per-call buffers.  This file is named so that
pytest collects it last; it passes alone in a fresh process and after the other tests.
"""
import numpy as np
import pytest

from oracle import oracle_ctypes as oc
from open_rendering_framework_b200 import _native as nat

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

MAX_QUERIES = 65536


def run(entry, wo, alpha, first, n_ggx):
    n = alpha.size
    wi = np.empty((3, n), np.float32)
    f, pdf, F = (np.empty(n, np.float32) for _ in range(3))
    nat.call(entry, oc.fp(wo), oc.fp(alpha), n, first, first + n_ggx, np.float32(1 / 1.5), oc.fp(wi), oc.fp(f), oc.fp(pdf), oc.fp(F))
    return wi, f, pdf, F


def same_bits(a, b):
    """Both entry points run the same kernel on the same inputs, so every output word -- NaNs
    included -- must be identical."""
    return bool(np.array_equal(np.ascontiguousarray(a).view(np.uint32), np.ascontiguousarray(b).view(np.uint32)))


def test_noalloc_matches_allocating_entry_on_two_calls_in_a_row():
    # two different batches back to back: the second call reuses the array the first one filled
    for first, n, n_ggx in ((0, 40000, 20000), (123457, MAX_QUERIES, 1000)):
        wo, alpha = oc.c1_inputs(n, first)
        got = run("pt_bsdf_queries_host_noalloc", wo, alpha, first, n_ggx)
        ref = run("pt_bsdf_queries_host", wo, alpha, first, n_ggx)
        for g, r in zip(got, ref):
            assert same_bits(g, r)


def test_noalloc_rejects_batches_beyond_the_array():
    wo, alpha = oc.c1_inputs(8)
    big = MAX_QUERIES + 1
    status = nat.lib().pt_bsdf_queries_host_noalloc(oc.fp(wo), oc.fp(alpha), big, 0, 0, np.float32(0.5), oc.fp(wo), oc.fp(alpha),
                                                   oc.fp(alpha), oc.fp(alpha))
    assert status == 1
    assert b"65536" in nat.lib().pt_last_error_message()
