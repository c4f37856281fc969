"""The workload configurations at their stated sizes, against the reference's
own CUDA renderer (Native/renderer.cu renderKernel, built for sm_100a into
oracle/_ref) and the oracle. Needs a GPU.

  - plain method, small: the 5,132-triangle Cornell box at 256x256, 64 paths
    per pixel as 4 RtRender passes of 16, depth 4: node array and SAH cost
    equal to the reference builder's; accumulation and image after every
    pass byte-identical to the reference renderer's;
  - traversal and build at scale: one 16-path pass of the 1,003,532-triangle
    room at 1920x1080, depth 3, byte-identical to the reference renderer's;
    65,536 camera rays, their first diffuse bounce and shadow rays to the
    light, all queried on the same scene: index, t, u and v bit-exact
    against the oracle's traversal (and the reference's own traversal code
    where oracle/_ref is present);
  - batched multi-scene tracing: the 8-scene, 64-view batch (10K-2M
    triangles, 256^2 to 1024^2, 8 paths per pixel, depth 4) renders every
    view byte-identical to the reference renderer's render of that view.

Tolerance everywhere here: bit-exact (the reference builds with
--fmad=false, and so does this library's integrator).
"""
import math

import numpy as np
import pytest

import scenes
from native_api import QUERY_DTYPE, Batch

pytestmark = pytest.mark.gpu


def _reference_session(reference):
    from oracle_api import ReferenceSession
    return ReferenceSession(reference)


def test_config1_stated_size_bit_exact_vs_reference_cuda(session, oracle, reference):
    tris, cam, st, w, h = scenes.cornell_sphere()
    assert (len(tris), w, h, st.maxBounces) == (5132, 256, 256, 4)
    st.raysPerPixel = 16
    session.initialize(tris, w, h)
    sc = oracle.scene(tris)
    try:
        nodes, _ = session.export_bvh(len(tris))
        assert nodes.tobytes() == sc.nodes().tobytes()
        stats = session.bvh_stats()
        expected = oracle.sah_cost(sc.nodes())
        assert abs(stats['sahCost'] - expected) <= 1e-9 * expected
    finally:
        sc.close()
    ref = _reference_session(reference)
    try:
        ref.initialize(tris, w, h)
        for k in range(4):  # 64 paths per pixel: 4 passes of 16 (RtRender takes at most 16)
            ref_rgba, _ = ref.render(cam, st)
            rgba, _ = session.render(cam, st)
            assert rgba.tobytes() == ref_rgba.tobytes(), f'image after pass {k}'
            assert session.accumulation().tobytes() == ref.sums().tobytes(), f'sums after pass {k}'
        assert session.sample_count() == 64
    finally:
        ref.close()


@pytest.fixture(scope='module')
def room_1m():
    return scenes.displaced_sphere_room()


def test_config2_one_pass_bit_exact_vs_reference_cuda(session, reference, room_1m):
    tris, cam, st, w, h = room_1m
    assert (len(tris), w, h, st.maxBounces) == (1003532, 1920, 1080, 3)
    st.raysPerPixel = 16
    ref = _reference_session(reference)
    try:
        ref.initialize(tris, w, h)
        ref_rgba, _ = ref.render(cam, st)
        ref_sums = ref.sums()
    finally:
        ref.close()
    session.initialize(tris, w, h)
    rgba, _ = session.render(cam, st)
    assert rgba.tobytes() == ref_rgba.tobytes()
    assert session.accumulation().tobytes() == ref_sums.tobytes()
    stats = session.render_stats()
    assert stats['primaryRays'] == w * h * 16


def path_queries(tris, cam, w, h, count, rng, hits_of):
    """Rays of the kinds a pass traces: camera rays through random pixel
    positions, a diffuse bounce from each primary hit (origin on the
    surface, cosine-distributed about the geometric normal facing the
    incoming ray) and a shadow ray from each hit to a random point on a
    random emitter (limit = distance - 0.001, as Native/renderer.cu:261).
    hits_of(queries) returns the closest hits used to place the next kind."""
    px = 2.0 * (rng.integers(0, w, count) + rng.random(count)) / w - 1.0
    py = 2.0 * (rng.integers(0, h, count) + rng.random(count)) / h - 1.0
    vec = lambda v: np.array([v.x, v.y, v.z], np.float64)
    fwd, right, up = vec(cam.forward), vec(cam.right), vec(cam.up)
    d = fwd[None] + (px * cam.aspect * cam.tanHalfFov)[:, None] * right[None] + (py * cam.tanHalfFov)[:, None] * up[None]
    d /= np.linalg.norm(d, axis=1, keepdims=True)

    def make(o, dirs, limit):
        q = np.zeros(len(o), QUERY_DTYPE)
        for k, ax in enumerate('xyz'):
            q['origin'][ax] = o[:, k]
            q['direction'][ax] = dirs[:, k]
        q['limit'] = limit
        return q

    primary = make(np.broadcast_to(vec(cam.origin), (count, 3)).astype(np.float32), d.astype(np.float32),
                   np.float32(3.0e38))
    hits = hits_of(primary)
    hit = hits['index'] >= 0
    idx = hits['index'][hit]
    o = np.stack([primary['origin'][ax][hit] for ax in 'xyz'], 1).astype(np.float32)
    di = np.stack([primary['direction'][ax][hit] for ax in 'xyz'], 1).astype(np.float32)
    p = (o + di * hits['distance'][hit][:, None]).astype(np.float32)
    e1 = np.stack([tris['edge1'][ax][idx] for ax in 'xyz'], 1).astype(np.float64)
    e2 = np.stack([tris['edge2'][ax][idx] for ax in 'xyz'], 1).astype(np.float64)
    n = np.cross(e1, e2)
    n /= np.maximum(np.linalg.norm(n, axis=1, keepdims=True), 1e-30)
    n *= -np.sign(np.sum(n * di, axis=1, keepdims=True) + 1e-30)
    a = np.where(np.abs(n[:, 1:2]) < 0.999, np.array([[0.0, 1.0, 0.0]]), np.array([[1.0, 0.0, 0.0]]))
    t = np.cross(a, n)
    t /= np.linalg.norm(t, axis=1, keepdims=True)
    b = np.cross(n, t)
    u1, u2 = rng.random(len(p)), rng.random(len(p))
    r, phi = np.sqrt(u1), 2 * np.pi * u2
    bounce = (t * (r * np.cos(phi))[:, None] + b * (r * np.sin(phi))[:, None] + n * np.sqrt(1 - u1)[:, None])
    secondary = make(p, bounce.astype(np.float32), np.float32(3.0e38))
    lights = np.nonzero(tris['emission'] > 0)[0]
    pick = lights[rng.integers(0, len(lights), len(p))]
    s1, s2 = rng.random(len(p)), rng.random(len(p))
    flip = s1 + s2 > 1
    s1, s2 = np.where(flip, 1 - s1, s1), np.where(flip, 1 - s2, s2)
    lo = np.stack([tris['origin'][ax][pick] for ax in 'xyz'], 1).astype(np.float64)
    le1 = np.stack([tris['edge1'][ax][pick] for ax in 'xyz'], 1).astype(np.float64)
    le2 = np.stack([tris['edge2'][ax][pick] for ax in 'xyz'], 1).astype(np.float64)
    target = lo + le1 * s1[:, None] + le2 * s2[:, None]
    to = target - p
    dist = np.linalg.norm(to, axis=1)
    shadow = make(p, (to / dist[:, None]).astype(np.float32), (dist - 0.001).astype(np.float32))
    return primary, secondary, shadow


def test_config2_ray_queries_bit_exact(session, oracle, room_1m, request):
    """65,536 camera rays plus their secondary and shadow rays on the
    1,003,532-triangle room: closest hits bit-exact (index, t, u, v) and
    any-hit occlusion equal, against the oracle and, where present, the
    reference's own traversal."""
    tris, cam, _, w, h = room_1m
    session.initialize(tris, 64, 64)
    sc = oracle.scene(tris)
    try:
        rng = np.random.Generator(np.random.PCG64(65536))
        primary, secondary, shadow = path_queries(tris, cam, w, h, 65536, rng, lambda q: oracle.query(sc, q)[0])
        assert len(secondary) > 30000
        reference = None
        try:
            reference = request.getfixturevalue('reference')
        except pytest.skip.Exception:
            pass
        ref_scene = reference.scene(tris) if reference is not None else None
        try:
            for name, q in (('primary', primary), ('secondary', secondary), ('shadow', shadow)):
                got = session.query(q)
                want, _ = oracle.query(sc, q)
                assert got.tobytes() == want.tobytes(), name
                got_any = session.query(q, any_hit=True)
                want_any, _ = oracle.query(sc, q, any_hit=True)
                assert ((got_any['index'] >= 0) == (want_any['index'] >= 0)).all(), name
                if ref_scene is not None:
                    assert got.tobytes() == reference.query(ref_scene, q).tobytes(), name
            assert (session.query(secondary)['index'] >= 0).mean() > 0.5
            assert 0.05 < (session.query(shadow, any_hit=True)['index'] >= 0).mean() < 0.95
        finally:
            if ref_scene is not None:
                ref_scene.close()
    finally:
        sc.close()


def test_config3_batch_views_bit_exact_vs_reference_cuda(lib, reference):
    """The stated batch: every one of the 64 views, rendered in the shared
    batch frame, equals the reference renderer's render of that view alone."""
    scene_list, views, st = scenes.batch_workload()
    assert len(scene_list) == 8 and len(views) == 64 and (st.raysPerPixel, st.maxBounces) == (8, 4)
    with Batch(lib) as b:
        for tris in scene_list:
            b.add_scene(tris)
        for k, cam, w, h in views:
            b.add_view(k, cam, w, h)
        b.render(st)
        got = [(b.accumulation(v), b.image(v)) for v in range(len(views))]
    # One reference session per (scene, resolution); a new camera restarts
    # its accumulation (Native/renderer.cu:388-389).
    groups = {}
    for v, (k, cam, w, h) in enumerate(views):
        groups.setdefault((k, w, h), []).append(v)
    for (k, w, h), members in groups.items():
        ref = _reference_session(reference)
        try:
            ref.initialize(scene_list[k], w, h)
            for v in members:
                rgba, _ = ref.render(views[v][1], st)
                assert got[v][0].tobytes() == ref.sums().tobytes(), f'view {v} sums'
                assert got[v][1].tobytes() == rgba.tobytes(), f'view {v} image'
        finally:
            ref.close()
