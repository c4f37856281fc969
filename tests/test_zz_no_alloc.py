"""RtxQueryRaysStatic: ray queries that allocate no device memory.

Some callers cannot allocate device memory while they query the scene: code
running beside a CUDA graph capture, latency-critical loops where
cudaMalloc/cudaFree would synchronise the whole device, or hosts whose device
memory belongs to a pool the library must not touch. RtxQueryRaysStatic
serves them by staging rays and hits in a file-scope device array (at most
16384 rays per call) instead of cudaMalloc'd buffers.

This file checks, through the C ABI, that two calls in a row return exactly
what the allocating entry point RtxQueryRays returns (bit-exact, the tolerance
of every ray-query test here), and that counts beyond the array's capacity are
refused with a message. It is collected last on purpose, so a run that stops
at its first failure has run every other test already; it also passes alone
in a fresh process.
"""
import numpy as np
import pytest

import scenes
from native_api import QUERY_DTYPE, Session, load_library

pytestmark = pytest.mark.gpu


def test_static_queries_equal_allocating_queries():
    lib = load_library()
    s = Session(lib)
    try:
        rng = np.random.Generator(np.random.PCG64(2024))
        tris = np.concatenate([scenes.scattered_triangles(rng, 3000), scenes.edge_case_triangles()])
        s.initialize(tris, 8, 8)
        first = np.concatenate([scenes.random_rays(rng, 12000), scenes.edge_grid_rays()])
        second = scenes.random_rays(rng, 9000)
        for rays in (first, second):  # two calls in a row share the static array
            for any_hit in (False, True):
                expected = s.query(rays, any_hit=any_hit)
                got = s.query_static(rays, any_hit=any_hit)
                assert got.tobytes() == expected.tobytes()
                assert (got['index'] >= 0).any()
        # Exactly the capacity: the caller's raw records then end where the
        # array's counters begin.
        full = scenes.random_rays(rng, Session.STATIC_QUERY_CAPACITY)
        for any_hit in (False, True):
            assert s.query_static(full, any_hit=any_hit).tobytes() == s.query(full, any_hit=any_hit).tobytes()
    finally:
        s.close()


def test_static_queries_refuse_counts_beyond_capacity():
    lib = load_library()
    s = Session(lib)
    try:
        s.initialize(scenes.edge_case_triangles(), 8, 8)
        capacity = Session.STATIC_QUERY_CAPACITY
        rays = np.zeros(capacity + 1, QUERY_DTYPE)
        hits = np.zeros(capacity + 1, dtype=[('index', '<i4'), ('distance', '<f4'), ('u', '<f4'), ('v', '<f4')])
        assert not lib.RtxQueryRaysStatic(s.handle, rays.ctypes.data, capacity + 1, 0, hits.ctypes.data)
        assert b'16384' in lib.RtLastError(s.handle)
        assert lib.RtxQueryRaysStatic(s.handle, rays.ctypes.data, 0, 0, hits.ctypes.data)
    finally:
        s.close()
