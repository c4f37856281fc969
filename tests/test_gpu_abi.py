"""Behaviour of the C ABI on a GPU, after the reference's own end-to-end
checks (Tools/verify_native.py and Tools/verify_denoising.py), through ctypes
exactly as those scripts call the reference library. Needs a GPU.

Backend 3 (Embree) is not part of this library: where the reference's
agree() renders it, these tests check that it is rejected with a message."""
import ctypes as c
import math
import os

import numpy as np
import pytest

import scenes
from native_api import Camera, Settings, Vector

pytestmark = pytest.mark.gpu


class Driver:
    def __init__(self, lib):
        self.lib = lib
        self.session, self.preview = lib.RtCreate(), lib.RtCreate()
        self.lit = Settings(8, 1, 0, 3, 0, 42, 1)

    def close(self):
        self.lib.RtDestroy(self.session)
        self.lib.RtDestroy(self.preview)

    def check(self, ok, ctx=None):
        assert ok, self.lib.RtLastError(ctx or self.session).decode()

    def initialize(self, triangles, w, h, ctx=None):
        tris = np.ascontiguousarray(triangles)
        self.check(self.lib.RtInitialize(ctx or self.session, tris.ctypes.data, len(tris), w, h), ctx)

    def render(self, camera, w, h, backend=2, settings=None, ctx=None):
        output = (c.c_ubyte * (w * h * 4))()
        ms = c.c_float()
        self.check(self.lib.RtRender(ctx or self.session, c.byref(camera), c.byref(settings or self.lit), output,
                                     len(output), backend, c.byref(ms)), ctx)
        assert ms.value >= 0 and math.isfinite(ms.value)
        return bytes(output)

    def agree(self, camera, w, h, settings, samples=4):
        """Tools/verify_native.py:73-95 with backend 3 replaced by its rejection."""
        lib = self.lib

        def batch(backend):
            lib.RtReset(self.session)
            for _ in range(samples):
                image = self.render(camera, w, h, backend, settings)
            assert lib.RtSampleCount(self.session) == samples * settings.raysPerPixel
            return image
        cpu = batch(0)
        assert lib.RtCpuThreadCount(self.session) == 1
        multi = batch(1)
        threads = lib.RtCpuThreadCount(self.session)
        if len(os.sched_getaffinity(0)) > 1 and not os.environ.get('OMP_NUM_THREADS'):
            assert threads > 1
        gpu = batch(2)
        assert lib.RtCpuThreadCount(self.session) == 0
        assert max(abs(a - b) for a, b in zip(cpu, multi)) == 0  # same host code: identical
        assert max(abs(a - b) for a, b in zip(cpu, gpu)) <= 1
        output = (c.c_ubyte * (w * h * 4))()
        assert not lib.RtRender(self.session, c.byref(camera), c.byref(settings), output, len(output), 3,
                                c.byref(c.c_float()))
        assert b'Embree' in lib.RtLastError(self.session)
        return gpu

    def accumulate(self, camera, w, h, samples, settings=None):
        self.lib.RtReset(self.session)
        for _ in range(samples):
            image = self.render(camera, w, h, settings=settings)
        return image


def centre(image, w, h):
    offset = ((h // 2) * w + w // 2) * 4
    return tuple(image[offset:offset + 4])


def rmse(a, b):
    values = [(x - y) ** 2 for i, (x, y) in enumerate(zip(a, b)) if i % 4 != 3]
    return math.sqrt(sum(values) / len(values))


@pytest.fixture
def drv(lib):
    d = Driver(lib)
    yield d
    d.close()


def test_known_colour_culling_and_sizes(drv):
    """Tools/verify_native.py:122-134."""
    red = scenes.quad(-1, 1, -1, 1, 0, color=(1, 0, 0), emission=1)
    for w, h in ((37, 25), (17, 19)):
        camera = Camera(Vector(0, 0, -2), Vector(1, 0, 0), Vector(0, 1, 0), Vector(0, 0, 1), .5, w / h, 1, 0)
        for sided, inside, expected in ((0, False, (208, 0, 0, 255)), (1, False, (0, 0, 0, 255)),
                                        (1, True, (208, 0, 0, 255))):
            red['oneSided'] = sided
            camera.origin.z = 2 if inside else -2
            camera.forward.z = -1 if inside else 1
            drv.initialize(red, w, h)
            image = drv.agree(camera, w, h, drv.lit)
            assert centre(image, w, h) == expected
            assert all(alpha == 255 for alpha in image[3::4])


def test_independent_sessions_and_shutdown(drv):
    """Tools/verify_native.py:135-143."""
    lib = drv.lib
    red = scenes.quad(-1, 1, -1, 1, 0, color=(1, 0, 0), emission=1)
    camera = Camera(Vector(0, 0, -2), Vector(1, 0, 0), Vector(0, 1, 0), Vector(0, 0, 1), .5, 17 / 19, 1, 0)
    drv.initialize(red, 17, 19)
    reference = drv.render(camera, 17, 19)
    green = scenes.quad(-1, 1, -1, 1, 0, color=(0, 1, 0), emission=1)
    drv.initialize(green, 7, 9, drv.preview)
    other = Camera(Vector(0, 0, -2), Vector(1, 0, 0), Vector(0, 1, 0), Vector(0, 0, 1), .5, 7 / 9, 1, 0)
    assert centre(drv.render(other, 7, 9, ctx=drv.preview), 7, 9) == (0, 208, 0, 255)
    lib.RtShutdown(drv.preview)
    lib.RtReset(drv.session)
    assert drv.render(camera, 17, 19) == reference


def test_light_occlusion_convergence_mirror_sky(drv):
    """Tools/verify_native.py:145-176."""
    w, h = 33, 25
    camera = Camera(Vector(0, 0, -3), Vector(1, 0, 0), Vector(0, 1, 0), Vector(0, 0, 1), .3, w / h, 1, 0)
    floor = scenes.quad(-2, 2, -2, 2, 0)
    light = scenes.quad(.8, 1.2, -.2, .2, -2, emission=30)
    blocker = scenes.quad(.25, .75, -.5, .5, -1)
    drv.initialize(np.concatenate([floor, light]), w, h)
    unblocked = drv.agree(camera, w, h, drv.lit, 16)
    drv.initialize(np.concatenate([floor, light, blocker]), w, h)
    blocked = drv.agree(camera, w, h, drv.lit, 16)
    assert centre(unblocked, w, h)[0] > centre(blocked, w, h)[0] + 20
    one = drv.accumulate(camera, w, h, 1)
    sixteen = drv.accumulate(camera, w, h, 16)
    reference = drv.accumulate(camera, w, h, 256)
    assert rmse(sixteen, reference) < rmse(one, reference) * .6
    mirror = scenes.quad(-2, 2, -2, 2, 0, specular_probability=1, smoothness=1)
    behind = scenes.quad(-1, 1, -1, 1, -4, color=(0, 1, 0), emission=2)
    drv.initialize(np.concatenate([mirror, behind]), w, h)
    reflected = drv.agree(camera, w, h, drv.lit)
    assert centre(reflected, w, h)[1] > 230 and centre(reflected, w, h)[0] == 0
    drv.initialize(floor, w, h)
    assert centre(drv.agree(camera, w, h, drv.lit), w, h) == (0, 0, 0, 255)
    lit = Settings(8, 1, 0, 3, 1, 42, 1)
    assert centre(drv.agree(camera, w, h, lit, 16), w, h)[0] > 100
    camera.origin.x = 20
    empty = drv.agree(camera, w, h, lit)
    assert all(empty[i:i + 4] == bytes((0, 0, 0, 255)) for i in range(0, len(empty), 4))


def test_batching_cameras_and_resets(drv):
    """Tools/verify_native.py:177-213."""
    lib = drv.lib
    w, h = 33, 25
    camera = Camera(Vector(0, 0, -3), Vector(1, 0, 0), Vector(0, 1, 0), Vector(0, 0, 1), .3, w / h, 1, 0)
    drv.initialize(scenes.quad(-2, 2, -2, 2, 0), w, h)
    lit = Settings(8, 1, 0, 3, 1, 42, 1)
    separate = drv.accumulate(camera, w, h, 12, lit)
    for rays in (2, 4, 6):
        lit.raysPerPixel = rays
        batched = drv.agree(camera, w, h, lit, 12 // rays)
        assert max(abs(a - b) for a, b in zip(separate, batched)) <= 1
        assert lib.RtSampleCount(drv.session) == 12
    lit.raysPerPixel = 1
    camera.orthographic = 1
    drv.agree(camera, w, h, lit)
    camera.orthographic = 0
    lit.aperture = .2
    drv.agree(camera, w, h, lit)
    lib.RtReset(drv.session)
    a = drv.render(camera, w, h, settings=lit)
    drv.render(camera, w, h, settings=lit)
    assert lib.RtSampleCount(drv.session) == 2
    lib.RtReset(drv.session)
    assert drv.render(camera, w, h, settings=lit) == a and lib.RtSampleCount(drv.session) == 1
    camera.origin.x += .1
    drv.render(camera, w, h, settings=lit)
    assert lib.RtSampleCount(drv.session) == 1
    lit.exposure = 2
    drv.render(camera, w, h, settings=lit)
    assert lib.RtSampleCount(drv.session) == 1
    drv.render(camera, w, h, 1, settings=lit)
    assert lib.RtSampleCount(drv.session) == 1
    output = (c.c_ubyte * (w * h * 4))()
    for backend in (-1, 4):
        assert not lib.RtRender(drv.session, c.byref(camera), c.byref(lit), output, len(output), backend,
                                c.byref(c.c_float()))
    assert not lib.RtRender(drv.session, c.byref(camera), c.byref(lit), output, 4, 2, c.byref(c.c_float()))
    for bad in (Settings(0, 1, 0, 3, 1, 42, 1), Settings(33, 1, 0, 3, 1, 42, 1), Settings(8, 0, 0, 3, 1, 42, 1),
                Settings(8, 1, -1, 3, 1, 42, 1), Settings(8, 1, 0, 0, 1, 42, 1), Settings(8, 1, 0, 3, -1, 42, 1),
                Settings(8, 1, 0, 3, 1, 42, 0), Settings(8, 1, 0, 3, 1, 42, 17)):
        assert not lib.RtRender(drv.session, c.byref(camera), c.byref(bad), output, len(output), 2,
                                c.byref(c.c_float()))
    drv.render(camera, w, h, settings=lit)
    lib.RtShutdown(drv.session)
    assert not lib.RtRender(drv.session, c.byref(camera), c.byref(lit), output, len(output), 2, c.byref(c.c_float()))


def test_denoise_behaviour(drv):
    """Tools/verify_denoising.py: must render first, keeps the accumulation,
    sample count and version, agrees across backends, black stays black."""
    lib = drv.lib
    tris, camera, settings, _, _ = scenes.cornell_sphere()
    settings.raysPerPixel = 16
    ms = c.c_float()

    def denoise(ctx, output):
        before, version = lib.RtSampleCount(ctx), lib.RtAccumulationVersion(ctx)
        drv.check(lib.RtDenoise(ctx, output, len(output), c.byref(ms)), ctx)
        assert lib.RtSampleCount(ctx) == before and lib.RtAccumulationVersion(ctx) == version
        assert ms.value > 0
        return bytes(output)

    for w, h in ((97, 55), (37, 25)):
        camera.aspect = w / h
        drv.initialize(tris, w, h)
        output = (c.c_ubyte * (w * h * 4))()
        assert not lib.RtDenoise(drv.session, output, len(output), c.byref(ms)), 'must render before denoising'
        reference = None
        for backend in (0, 1, 2):
            lib.RtReset(drv.session)
            raw = drv.render(camera, w, h, backend, settings)
            sums_before = np.zeros(w * h * 10, np.float32)
            lib.RtxReadAccumulation(drv.session, sums_before.ctypes.data, w * h)
            out = (c.c_ubyte * (w * h * 4))()
            ai = np.frombuffer(denoise(drv.session, out), np.uint8).astype(int)
            sums_after = np.zeros_like(sums_before)
            lib.RtxReadAccumulation(drv.session, sums_after.ctypes.data, w * h)
            assert sums_before.tobytes() == sums_after.tobytes()
            assert (ai[3::4] == 255).all()
            if reference is None:
                reference = ai
            assert np.abs(ai - reference).max() <= 2, backend
        assert not lib.RtDenoise(drv.session, output, len(output) - 1, c.byref(ms))
    camera.origin.x = 10000
    drv.initialize(tris, 37, 25)
    camera.aspect = 37 / 25
    first = (c.c_ubyte * (37 * 25 * 4))()
    drv.render(camera, 37, 25, 2, settings)
    ai = denoise(drv.session, first)
    assert all(value == (255 if i % 4 == 3 else 0) for i, value in enumerate(ai))
    lib.RtShutdown(drv.session)
    assert not lib.RtDenoise(drv.session, first, len(first), c.byref(ms))


def test_constant_environment_extension(drv):
    """RtxSetEnvironment mode 1 lights bounces with a constant radiance and
    leaves primary misses black; it resets the accumulation; mode 0 is the
    reference's sky. CPU and CUDA backends agree within 1/255."""
    lib = drv.lib
    w, h = 33, 25
    camera = Camera(Vector(0, 0, -3), Vector(1, 0, 0), Vector(0, 1, 0), Vector(0, 0, 1), .3, w / h, 1, 0)
    floor = scenes.quad(-2, 2, -2, 2, 0)
    drv.initialize(floor, w, h)
    lit = Settings(8, 1, 0, 3, 0, 42, 1)
    dark = drv.agree(camera, w, h, lit, 8)
    assert centre(dark, w, h) == (0, 0, 0, 255)
    version = lib.RtAccumulationVersion(drv.session)
    assert lib.RtxSetEnvironment(drv.session, 1, 0.5, 0.5, 0.5)
    assert lib.RtAccumulationVersion(drv.session) == version + 1 and lib.RtSampleCount(drv.session) == 0
    bright = drv.agree(camera, w, h, lit, 8)
    assert centre(bright, w, h)[0] > 60
    camera.origin.x = 20
    empty = drv.agree(camera, w, h, lit)
    assert all(empty[i:i + 4] == bytes((0, 0, 0, 255)) for i in range(0, len(empty), 4))
    assert not lib.RtxSetEnvironment(drv.session, 2, 0, 0, 0)
    assert not lib.RtxSetEnvironment(drv.session, 1, -1, 0, 0)
    assert lib.RtxSetEnvironment(drv.session, 0, 0, 0, 0)
