"""The C ABI surface of libCudaRayTracer.so, checked without a GPU: it loads,
exports every entry point include/cuda_ray_tracer.h declares, keeps the
reference's record layouts, and handles null or uninitialised sessions the
way the reference does (Native/renderer.cu:309-318, 376-382, 437-439)."""
import ctypes as c
import re

import numpy as np

from conftest import ROOT
import native_api
from native_api import Camera, Settings, Vector

HEADER = ROOT / 'include' / 'cuda_ray_tracer.h'


def declared_functions():
    text = re.sub(r'/\*.*?\*/', '', HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r'\b(Rtx?[A-Za-z]+)\s*\(', text)))


def test_header_lists_reference_exports():
    names = declared_functions()
    reference13 = {'RtCreate', 'RtDestroy', 'RtShutdown', 'RtInitialize', 'RtRender', 'RtDenoise', 'RtReset',
                   'RtAccumulationVersion', 'RtSampleCount', 'RtEmbreeBuildMilliseconds', 'RtCpuThreadCount',
                   'RtBvhInfo', 'RtLastError'}
    assert reference13 <= set(names)
    assert set(names) == set(native_api.EXPORTS)


def test_library_exports_every_declared_symbol(lib):
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_record_layouts():
    assert c.sizeof(native_api.Triangle) == 116 and c.sizeof(Camera) == 64 and c.sizeof(Settings) == 28
    assert c.sizeof(native_api.PixelSum) == 40 and c.sizeof(native_api.BvhNode) == 32
    offsets = {name: getattr(native_api.Triangle, name).offset for name, _ in native_api.Triangle._fields_}
    assert offsets == {'origin': 0, 'edge1': 12, 'edge2': 24, 'color': 36, 'emission': 48, 'oneSided': 52,
                       'normal0': 56, 'normal1': 68, 'normal2': 80, 'mesh': 92, 'specularColor': 96,
                       'smoothness': 108, 'specularProbability': 112}
    assert native_api.TRIANGLE_DTYPE.itemsize == 116


def test_null_session(lib):
    assert lib.RtSampleCount(None) == 0
    assert lib.RtAccumulationVersion(None) == 0
    assert lib.RtCpuThreadCount(None) == 0
    assert lib.RtEmbreeBuildMilliseconds(None) == 0
    assert lib.RtLastError(None)
    out = (c.c_ubyte * 16)()
    ms = c.c_float()
    cam, st = Camera(), Settings(1, 1, 0, 1, 0, 42, 1)
    assert not lib.RtRender(None, c.byref(cam), c.byref(st), out, 16, 2, c.byref(ms))
    assert not lib.RtDenoise(None, out, 16, c.byref(ms))
    assert not lib.RtInitialize(None, None, 0, 1, 1)
    nodes, depth, build = c.c_int(7), c.c_int(7), c.c_float(7)
    lib.RtBvhInfo(None, c.byref(nodes), c.byref(depth), c.byref(build))
    assert (nodes.value, depth.value, build.value) == (0, 0, 0)
    lib.RtReset(None)
    lib.RtShutdown(None)
    lib.RtDestroy(None)


def test_uninitialised_session_rejects_work(lib):
    s = lib.RtCreate()
    try:
        out = (c.c_ubyte * 16)()
        ms = c.c_float()
        cam = Camera(Vector(0, 0, -2), Vector(1, 0, 0), Vector(0, 1, 0), Vector(0, 0, 1), .5, 1, 1, 0)
        st = Settings(1, 1, 0, 1, 0, 42, 1)
        assert not lib.RtRender(s, c.byref(cam), c.byref(st), out, 16, 2, c.byref(ms))
        assert b'not initialised' in lib.RtLastError(s)
        assert not lib.RtDenoise(s, out, 16, c.byref(ms))
        version = lib.RtAccumulationVersion(s)
        lib.RtReset(s)
        assert lib.RtAccumulationVersion(s) == version + 1 and lib.RtSampleCount(s) == 0
        # Invalid initialisation arguments are rejected before any device work.
        tri = np.zeros(1, native_api.TRIANGLE_DTYPE)
        for w, h in ((0, 1), (1, 0), (4097, 1), (1, 4097)):
            assert not lib.RtInitialize(s, tri.ctypes.data, 1, w, h)
        assert not lib.RtInitialize(s, tri.ctypes.data, 0, 8, 8)
    finally:
        lib.RtDestroy(s)
