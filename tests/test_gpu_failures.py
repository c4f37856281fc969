"""Failure detection, in the forms that fault no GPU. Needs a GPU.

  - traversal stack overflow: RTX_TUNE_STACK_LIMIT makes the traversal
    kernels' overflow check fire on ordinary rays; every entry point that
    traces returns 0 with "BVH traversal stack overflow", and the session
    stays usable (the next pass at the default limit is bit-exact);
  - the stack in use: on the reference's exponentially spaced set
    (Tools/verify_bvh.cu:132-138) a query needs all 8 stack entries a ray
    keeps in shared memory (7 overflow, 8 do not) and its answers are
    bit-exact; 33 identical triangles (the geometry of the reference's
    deliberate depth-32 chain, Tools/verify_bvh.cu:139) answer exactly as
    the reference's traversal does;
  - out of device memory: RtxDebugFailAllocation makes the n-th next device
    allocation fail on the host; for every allocation of RtInitialize, of
    the first RtRender, RtDenoise and RtxQueryRays in turn, the call returns
    0 with a message, and the same session then works bit-exactly;
  - invalid arguments (Tools/verify_native.py:158-165 and the other entry
    points' preconditions): rejected with 0 and a message, no device work.
"""
import ctypes as c

import numpy as np
import pytest

import scenes
from conftest import golden
from native_api import HIT_DTYPE, PIXELSUM_DTYPE, NativeError, Session
from test_oracle_golden import GEOMETRY, RAYS

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def disarm(lib):
    lib.RtxDebugFailAllocation(0)
    yield
    lib.RtxDebugFailAllocation(0)


def small_scene():
    tris, cam, st, _, _ = scenes.cornell_sphere()
    w, h = 48, 40
    cam.aspect = w / h
    st.raysPerPixel = 2
    return tris, cam, st, w, h


def camera_rays(cam, count, seed=9):
    """Rays from the camera towards random points of the box's interior,
    which reach the sphere's deep subtrees like the camera rays of a pass."""
    from native_api import QUERY_DTYPE
    rng = np.random.Generator(np.random.PCG64(seed))
    o = np.array([cam.origin.x, cam.origin.y, cam.origin.z])
    target = rng.uniform((-0.9, 0.1, -0.9), (0.9, 1.9, 0.9), (count, 3))
    d = target - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    q = np.zeros(count, QUERY_DTYPE)
    for k, ax in enumerate('xyz'):
        q['origin'][ax] = o[k]
        q['direction'][ax] = d[:, k]
    q['limit'] = np.float32(1e30)
    return q


def reference_pass(lib, tris, cam, st, w, h):
    with Session(lib) as s:
        s.initialize(tris, w, h)
        rgba, _ = s.render(cam, st)
        return rgba.copy(), s.accumulation()


@pytest.mark.parametrize('integrator', (0, 1))
def test_stack_overflow_is_reported_and_recoverable(lib, session, integrator):
    tris, cam, st, w, h = small_scene()
    expect_rgba, expect_sums = reference_pass(lib, tris, cam, st, w, h)
    session.initialize(tris, w, h)
    session.set_integrator(integrator)
    session.set_tuning(stack_limit=1)
    with pytest.raises(NativeError, match='stack overflow'):
        session.render(cam, st)
    assert session.sample_count() == 0
    with pytest.raises(NativeError, match='stack overflow'):
        session.render_device(cam, st)
    with pytest.raises(NativeError, match='stack overflow'):
        session.query(camera_rays(cam, 4000))
    with pytest.raises(NativeError, match='stack overflow'):
        session.render(cam, st, backend=0)  # the host backend shares the traversal
    for bad in (0, 49):
        assert not lib.RtxSetTuning(session.handle, Session.TUNE_STACK_LIMIT, bad)
    session.set_tuning(stack_limit=48)
    session.lib.RtReset(session.handle)
    rgba, _ = session.render(cam, st)
    assert rgba.tobytes() == expect_rgba.tobytes()
    assert session.accumulation().tobytes() == expect_sums.tobytes()


def test_all_shared_stack_entries_in_use_exponential_set(session):
    g = golden('bvh_exponential.npz')
    session.initialize(GEOMETRY['exponential'], 8, 8)
    session.set_tuning(stack_limit=7)
    with pytest.raises(NativeError, match='stack overflow'):
        session.query(RAYS)
    session.set_tuning(stack_limit=8)
    assert session.query(RAYS).tobytes() == g['closest'].tobytes()
    any_hit = session.query(RAYS, any_hit=True)
    assert ((any_hit['index'] >= 0) == (g['any_index'] >= 0)).all()


def test_identical_triangles_chain_case(session, oracle):
    tris = np.concatenate([scenes.edge_case_triangles()[:1]] * 33)
    sc = oracle.scene(tris)
    try:
        session.initialize(tris, 8, 8)
        got = session.query(RAYS)
        want, _ = oracle.query(sc, RAYS)
        brute, _ = oracle.query(sc, RAYS, brute=True)
        assert got.tobytes() == want.tobytes()
        assert (got['index'] == brute['index']).all()  # the smallest index wins among the 33 equal hits
        assert (got['index'][got['index'] >= 0] == 0).all()
        any_hit = session.query(RAYS, any_hit=True)
        assert ((any_hit['index'] >= 0) == (want['index'] >= 0)).all()
    finally:
        sc.close()


def _count_allocations(lib, action):
    """How many device allocations `action` makes: arm the failure at growing
    n until the action succeeds (n beyond its last allocation)."""
    for n in range(1, 200):
        lib.RtxDebugFailAllocation(n)
        ok = action()
        lib.RtxDebugFailAllocation(0)
        if ok:
            return n - 1
    raise AssertionError('more than 199 allocations')


def test_out_of_memory_every_allocation_of_initialize(lib):
    tris, cam, st, w, h = small_scene()
    expect_rgba, expect_sums = reference_pass(lib, tris, cam, st, w, h)
    arr = np.ascontiguousarray(tris)
    s = Session(lib)
    try:
        failures = []

        def init():
            ok = lib.RtInitialize(s.handle, arr.ctypes.data, len(arr), w, h)
            if not ok:
                failures.append(lib.RtLastError(s.handle).decode())
            return ok
        count = _count_allocations(lib, init)
        assert count >= 10  # scene records, upload tables, sampler tables, sums, BVH buffers ...
        assert len(failures) == count
        assert all(f for f in failures)
        assert any('memory' in f.lower() for f in failures)
        s.width, s.height = w, h
        rgba, _ = s.render(cam, st)
        assert rgba.tobytes() == expect_rgba.tobytes()
        assert s.accumulation().tobytes() == expect_sums.tobytes()
    finally:
        s.close()


@pytest.mark.parametrize('what', ('render', 'denoise', 'query'))
def test_out_of_memory_in_later_calls(lib, what):
    tris, cam, st, w, h = small_scene()
    expect_rgba, expect_sums = reference_pass(lib, tris, cam, st, w, h)
    rays = scenes.random_rays(np.random.Generator(np.random.PCG64(4)), 3000)
    s = Session(lib)
    try:
        s.initialize(tris, w, h)
        if what != 'render':
            s.render(cam, st)
        out = np.zeros(w * h * 4, np.uint8)
        ms = c.c_float()
        hits = np.zeros(len(rays), HIT_DTYPE)
        calls = {
            'render': lambda: lib.RtRender(s.handle, c.byref(cam), c.byref(st),
                                           out.ctypes.data_as(c.POINTER(c.c_ubyte)), out.size, 2, c.byref(ms)),
            'denoise': lambda: lib.RtDenoise(s.handle, out.ctypes.data_as(c.POINTER(c.c_ubyte)), out.size,
                                             c.byref(ms)),
            'query': lambda: lib.RtxQueryRays(s.handle, rays.ctypes.data, len(rays), 0, hits.ctypes.data),
        }
        lib.RtxDebugFailAllocation(1)
        assert not calls[what]()
        assert lib.RtLastError(s.handle)
        lib.RtxDebugFailAllocation(0)
        if what == 'render':
            assert s.sample_count() == 0
            s.lib.RtReset(s.handle)
            rgba, _ = s.render(cam, st)
            assert rgba.tobytes() == expect_rgba.tobytes()
            assert s.accumulation().tobytes() == expect_sums.tobytes()
        elif what == 'denoise':
            before = s.accumulation()
            den, _ = s.denoise()
            assert (den[3::4] == 255).all()
            assert s.accumulation().tobytes() == before.tobytes() == expect_sums.tobytes()
        else:
            assert calls['query']()
            assert hits.tobytes() == s.query(rays).tobytes()
    finally:
        s.close()


def test_invalid_arguments_rejected(lib, session):
    """Tools/verify_native.py:158-165 and the additive entry points."""
    tris, cam, st, w, h = small_scene()
    session.initialize(tris, w, h)
    out = np.zeros(w * h * 4, np.uint8)
    po = out.ctypes.data_as(c.POINTER(c.c_ubyte))
    ms = c.c_float()
    for backend in (-1, 4):
        assert not lib.RtRender(session.handle, c.byref(cam), c.byref(st), po, out.size, backend, c.byref(ms))
        assert lib.RtLastError(session.handle)
    assert not lib.RtRender(session.handle, c.byref(cam), c.byref(st), po, 4, 2, c.byref(ms))
    assert b'output buffer' in lib.RtLastError(session.handle)
    assert not lib.RtRender(session.handle, c.byref(cam), c.byref(st), po, out.size, 3, c.byref(ms))
    assert b'Embree' in lib.RtLastError(session.handle)
    assert not lib.RtDenoise(session.handle, po, out.size, c.byref(ms))  # nothing rendered yet
    assert b'render at least one pass' in lib.RtLastError(session.handle)
    session.render(cam, st)
    assert not lib.RtDenoise(session.handle, po, 4, c.byref(ms))
    sums = np.zeros(w * h - 1, PIXELSUM_DTYPE)
    assert not lib.RtxReadAccumulation(session.handle, sums.ctypes.data, sums.size)
    aovs = np.zeros(10 * (w * h - 1), np.float32)
    assert not lib.RtxReadAovs(session.handle, aovs.ctypes.data, w * h - 1)
    hits = np.zeros(4, HIT_DTYPE)
    assert not lib.RtxQueryRays(session.handle, None, 4, 0, hits.ctypes.data)
    assert not lib.RtxQueryRays(session.handle, RAYS.ctypes.data, -1, 0, hits.ctypes.data)
    assert not lib.RtxSetEnvironment(session.handle, 2, 0.0, 0.0, 0.0)
    assert not lib.RtxSetEnvironment(session.handle, 1, -1.0, 0.0, 0.0)
    assert not lib.RtxSetTuning(session.handle, 99, 1)
    assert not lib.RtxDebugFailAllocation(-1)
    nodes = np.zeros(1, dtype=[('b', 'u1', 32)])
    assert not lib.RtxExportBvh(session.handle, nodes.ctypes.data, 1, None, 0)
    assert session.sample_count() == st.raysPerPixel  # none of the rejected calls changed the accumulation
    lib.RtShutdown(session.handle)
    assert not lib.RtRender(session.handle, c.byref(cam), c.byref(st), po, out.size, 2, c.byref(ms))
    assert b'not initialised' in lib.RtLastError(session.handle)
