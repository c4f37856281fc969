"""Batched multi-scene rendering (RtxBatch*) on a GPU.

A view rendered in a batch must accumulate exactly what the reference's own
CUDA renderer (Native/renderer.cu renderKernel, built for sm_100a into
oracle/_ref) accumulates for that scene, camera and settings alone: every
tuning (block size, queue capacity down to waves that span several views,
refill, graph replay or direct launches, 4- or 8-wide BVH) only changes the
schedule, so the PixelSum records and images are compared bit for bit. Where
oracle/_ref is absent the expectation is this library's RtRender (backend 2),
itself bit-identical to the reference renderer in tests/test_gpu_parity.py.
The constant environment is this library's addition, so its expectation is
always RtRender."""
import math

import numpy as np
import pytest

import scenes
from native_api import Batch, Session, Settings

pytestmark = pytest.mark.gpu


def views_of_two_scenes():
    """Two scenes and four views of three sizes (two views share a scene)."""
    room, cam0, _, _, _ = scenes.cornell_sphere()
    rng = np.random.default_rng(8)
    v0, v1, v2, normals = scenes.geodesic_sphere(12, 0.6, (0.2, 0.9, 0.3), 0.05, rng, smooth=True)
    other = np.concatenate([scenes.open_box((-1.5, 0.0, -1.5), (1.5, 2.5, 1.5), rng.uniform(0.2, 0.8, (5, 3)),
                                            0.3, 2.45, 20.0),
                            scenes.records(v0, v1, v2, color=(0.7, 0.4, 0.3), normals=normals, mesh=9),
                            scenes.cuboid((-0.7, 0.3, 0.4), (0.5, 0.6, 0.4), 0.5, color=(0.3, 0.6, 0.8), mesh=10)])
    cam1 = scenes.camera((0.3, 1.2, -1.3), (0.0, 0.8, 0.5), math.tan(math.radians(35)), 1.0)
    cam2 = scenes.camera((-0.4, 1.5, -3.0), (0.1, 0.9, 0.0), math.tan(math.radians(22)), 1.0)
    cam3 = scenes.camera((-0.4, 1.5, -3.0), (0.1, 0.9, 0.0), math.tan(math.radians(22)), 1.0)
    views = [(0, cam0, 37, 25), (1, cam1, 64, 48), (0, cam2, 50, 50), (1, cam3, 29, 41)]
    for _, cam, w, h in views:
        cam.aspect = w / h
    return [room, other], views


SETTINGS = Settings(4, 1.0, 0.0, 1.0, 0.5, 42, 4)


def session_reference(lib, tris, cam, w, h, frames, settings=SETTINGS, environment=None):
    s = Session(lib)
    try:
        s.initialize(tris, w, h)
        if environment is not None:
            s.set_environment(environment)
        for _ in range(frames):
            image, _ = s.render(cam, settings)
        return s.accumulation(), image.copy()
    finally:
        s.close()


def reference_renderer(tris, cam, w, h, frames, settings=SETTINGS):
    """The reference's CUDA renderer on one view (None where oracle/_ref is absent)."""
    from oracle_api import Reference, ReferenceSession, reference_available
    if not reference_available():
        return None
    ref = ReferenceSession(Reference())
    try:
        ref.initialize(tris, w, h)
        for _ in range(frames):
            image, _ = ref.render(cam, settings)
        return ref.sums(), image.copy()
    finally:
        ref.close()


@pytest.fixture(scope='module')
def reference(lib):
    scene_list, views = views_of_two_scenes()
    expect = []
    for k, cam, w, h in views:
        expect.append(reference_renderer(scene_list[k], cam, w, h, 2) or
                      session_reference(lib, scene_list[k], cam, w, h, 2))
    return scene_list, views, expect


def make_batch(lib, scene_list, views):
    b = Batch(lib)
    for tris in scene_list:
        b.add_scene(tris)
    for k, cam, w, h in views:
        b.add_view(k, cam, w, h)
    return b


@pytest.mark.parametrize('tuning', [
    {},
    {'graph': 0},
    {'capacity': 1024},                    # waves of 1,024 paths: many waves, most span two views
    {'block': 64, 'refill': 8},
    {'block': 256, 'refill': 32, 'capacity': 3000},
    {'width': 4},
    {'width': 4, 'graph': 0, 'capacity': 2048},
    {'pieces': 1},
    {'pieces': 4, 'width': 4},
    {'leaf': 4},
    {'leaf': 1, 'pieces': 2},
    {'lanes': 1},
    {'lanes': 2, 'capacity': 1024},       # two lanes, waves spanning views
    {'lanes': 3, 'capacity': 3000, 'graph': 0},
    {'lanes': 3, 'capacity': 10000},       # waves cross sample rows as well as views
    {'lanes': 1, 'capacity': 20000},
    {'persistent': 1},                     # one persistent launch per frame over a (view, tile) queue
    {'persistent': 1, 'graph': 0},
])
def test_batch_equals_single_view_renders(lib, reference, tuning):
    scene_list, views, expect = reference
    with make_batch(lib, scene_list, views) as b:
        b.set_tuning(**tuning)
        for _ in range(2):
            ms = b.render(SETTINGS)
            assert ms > 0
        assert b.sample_count() == 8
        for v, (acc, image) in enumerate(expect):
            assert b.accumulation(v).tobytes() == acc.tobytes(), (tuning, v)
            assert np.array_equal(b.image(v), image), (tuning, v)
        st = b.stats()
        assert st['views'] == 4 and st['scenes'] == 2 and st['graph'] == tuning.get('graph', 1)
        assert st['pixels'] == sum(w * h for _, _, w, h in views)
        assert st['paths'] == st['pixels'] * 4 and st['primaryRays'] == st['paths']
        assert st['width'] == tuning.get('width', 8) and st['block'] == tuning.get('block', 128)
        assert st['lanes'] == tuning.get('lanes', 2)
        assert st['kernelLaunches'] > 0


def test_settings_change_restarts_and_environment(lib, reference):
    scene_list, views, expect = reference
    with make_batch(lib, scene_list, views) as b:
        other = Settings(4, 1.0, 0.0, 1.0, 0.5, 7, 4)
        b.render(other)
        b.render(SETTINGS)              # new settings bytes: the accumulation restarts
        b.render(SETTINGS)
        assert b.sample_count() == 8
        assert b.accumulation(2).tobytes() == expect[2][0].tobytes()
        b.set_environment(0.2)
        b.render(SETTINGS)
        assert b.sample_count() == 4
        k, cam, w, h = views[1]
        acc, _ = session_reference(lib, scene_list[k], cam, w, h, 1, environment=0.2)
        assert b.accumulation(1).tobytes() == acc.tobytes()


def test_autotune_keeps_results(lib, reference):
    scene_list, views, expect = reference
    with make_batch(lib, scene_list, views) as b:
        tried = b.autotune(SETTINGS)
        assert len(tried) >= 9  # the current tuning, pieces 1 and 3, width 4, blocks 64 and 256, three refills
        assert {t['width'] for t in tried} == {4, 8} and {t['block'] for t in tried} >= {64, 128, 256}
        assert all(t['frameMs'] > 0 for t in tried)
        best = min(tried, key=lambda t: t['frameMs'])
        st = b.stats()
        assert (st['block'], st['refill'], st['width'], st['pieces'], st['lanes']) == \
            (best['block'], best['refill'], best['width'], best['pieces'], best['lanes'])
        assert {t['pieces'] for t in tried} == {1, 2, 3} and {t['lanes'] for t in tried} == {1, 2, 4}
        assert b.sample_count() == 0
        b.render(SETTINGS)
        b.render(SETTINGS)
        for v, (acc, _) in enumerate(expect):
            assert b.accumulation(v).tobytes() == acc.tobytes(), v


def test_batch_errors(lib):
    with Batch(lib) as b:
        with pytest.raises(Exception, match='add a scene'):
            b.render(SETTINGS)
        tris, cam, _, _, _ = scenes.cornell_sphere()
        with pytest.raises(Exception, match='scene id'):
            b.add_view(0, cam, 16, 16)
        k = b.add_scene(tris)
        with pytest.raises(Exception, match='scene id'):
            b.add_view(k + 1, cam, 16, 16)
        with pytest.raises(Exception, match='width'):
            b.add_view(k, cam, 5000, 16)
        b.add_view(k, cam, 16, 16)
        with pytest.raises(Exception, match='render first'):
            b.image(0)
        for key, value in (('block', 96), ('capacity', 10), ('refill', 0), ('graph', 2), ('width', 6), ('lanes', 5),
                           ('persistent', 2)):
            with pytest.raises(Exception, match='out of range'):
                b.set_tuning(**{key: value})
        bad = Settings(4, 1.0, 0.0, 1.0, 0.5, 42, 17)
        with pytest.raises(Exception, match='invalid settings'):
            b.render(bad)
        b.render(SETTINGS)
        assert b.image(0)[3::4].min() == 255
