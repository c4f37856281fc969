"""ctypes wrappers of the parity checkers (test infrastructure, never product code).

  Oracle     oracle/liboracle.so: the CPU restatement (oracle/oracle.cpp)
  Reference  oracle/_ref/libref.so: the reference's own Native/renderer.cu,
             compiled by oracle/Makefile where the reference sources exist

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.
"""
import ctypes as c
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_LIB = HERE / 'liboracle.so'
REFERENCE_LIB = HERE / '_ref' / 'libref.so'

VEC = [('x', '<f4'), ('y', '<f4'), ('z', '<f4')]
NODE_DTYPE = np.dtype([('low', VEC), ('first', '<i4'), ('high', VEC), ('count', '<i4')])
HIT_DTYPE = np.dtype([('index', '<i4'), ('distance', '<f4'), ('u', '<f4'), ('v', '<f4')])
PIXELSUM_DTYPE = np.dtype([('radiance', VEC), ('albedo', VEC), ('normal', VEC), ('covered', '<u4')])
LIGHT_DTYPE = np.dtype([('triangle', '<i4'), ('cumulativeArea', '<f4')])
SOBOL_DIMS = 260


class _Scene:
    def __init__(self, lib, prefix, triangles):
        self.lib, self.prefix = lib, prefix
        self.triangles = np.ascontiguousarray(triangles)
        self.handle = getattr(lib, prefix + 'scene_create')(self.triangles.ctypes.data, len(self.triangles))
        if not self.handle:
            raise RuntimeError('scene creation failed')

    def _f(self, name):
        return getattr(self.lib, self.prefix + name)

    def close(self):
        if self.handle:
            self._f('scene_destroy')(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def node_count(self):
        return self._f('scene_node_count')(self.handle)

    @property
    def depth(self):
        return self._f('scene_depth')(self.handle)

    def nodes(self):
        out = np.zeros(self.node_count, NODE_DTYPE)
        self._f('scene_nodes')(self.handle, out.ctypes.data)
        return out

    def order(self):
        out = np.zeros(len(self.triangles), np.int32)
        self._f('scene_order')(self.handle, out.ctypes.data)
        return out

    def lights(self):
        out = np.zeros(self._f('scene_light_count')(self.handle), LIGHT_DTYPE)
        self._f('scene_lights')(self.handle, out.ctypes.data)
        return out

    def light_area(self):
        return self._f('scene_light_area')(self.handle)

    def linear_triangles(self):
        out = np.zeros_like(self.triangles)
        self._f('scene_triangles')(self.handle, out.ctypes.data)
        return out


def _setup_common(lib, prefix):
    vp = c.c_void_p
    getattr(lib, prefix + 'scene_create').restype = vp
    getattr(lib, prefix + 'scene_create').argtypes = [vp, c.c_int]
    for name in ('scene_destroy',):
        getattr(lib, prefix + name).argtypes = [vp]
    for name in ('scene_node_count', 'scene_depth', 'scene_light_count'):
        getattr(lib, prefix + name).argtypes = [vp]
        getattr(lib, prefix + name).restype = c.c_int
    getattr(lib, prefix + 'scene_light_area').argtypes = [vp]
    getattr(lib, prefix + 'scene_light_area').restype = c.c_float
    for name in ('scene_nodes', 'scene_order', 'scene_lights', 'scene_triangles'):
        getattr(lib, prefix + name).argtypes = [vp, vp]
    getattr(lib, prefix + 'sobol').argtypes = [vp, vp, vp, c.c_int, c.c_int, vp]
    getattr(lib, prefix + 'sobol').restype = c.c_int
    getattr(lib, prefix + 'max_threads').restype = c.c_int


class Oracle:
    """The CPU restatement of the reference's hot path."""
    prefix = 'orc_'

    def __init__(self, path=ORACLE_LIB):
        if not Path(path).exists():
            raise FileNotFoundError(f'{path} missing: run `make -C {HERE} oracle`')
        self.lib = c.CDLL(str(path))
        _setup_common(self.lib, self.prefix)
        vp = c.c_void_p
        self.lib.orc_query.argtypes = [vp, vp, c.c_int, c.c_int, vp, c.c_int, vp, c.c_int]
        self.lib.orc_render.argtypes = [vp, vp, vp, c.c_int, c.c_int, c.c_uint, vp, vp, c.c_int, c.c_int, c.c_int, vp]
        self.lib.orc_render_pixels.argtypes = [vp, vp, vp, c.c_int, c.c_int, c.c_uint, vp, vp, vp, c.c_int, c.c_int, vp]
        self.lib.orc_sah_cost.argtypes = [vp, c.c_int]
        self.lib.orc_sah_cost.restype = c.c_double
        self.lib.orc_sobol_directions.argtypes = [vp]
        self.lib.orc_tonemap.argtypes = [c.c_float, c.c_float]
        self.lib.orc_tonemap.restype = c.c_ubyte

    def scene(self, triangles):
        return _Scene(self.lib, self.prefix, triangles)

    def max_threads(self):
        return self.lib.orc_max_threads()

    def sobol(self, pixel, sample, seed, ndim=SOBOL_DIMS):
        pixel, sample, seed = (np.ascontiguousarray(a, np.uint32) for a in (pixel, sample, seed))
        out = np.zeros((len(pixel), ndim), np.float32)
        if not self.lib.orc_sobol(pixel.ctypes.data, sample.ctypes.data, seed.ctypes.data, len(pixel), ndim,
                                  out.ctypes.data):
            raise RuntimeError('oracle sampler failed (cuRAND direction vectors unavailable?)')
        return out

    def sobol_directions(self):
        out = np.zeros(SOBOL_DIMS * 32, np.uint32)
        self.lib.orc_sobol_directions(out.ctypes.data)
        return out

    def sah_cost(self, nodes):
        nodes = np.ascontiguousarray(nodes, NODE_DTYPE)
        return self.lib.orc_sah_cost(nodes.ctypes.data, len(nodes))

    def query(self, scene, queries, any_hit=False, brute=False, threads=0):
        q = np.ascontiguousarray(queries)
        out = np.zeros(len(q), HIT_DTYPE)
        stats = np.zeros(4, np.int64)
        self.lib.orc_query(scene.handle, q.ctypes.data, len(q), int(any_hit), out.ctypes.data, int(brute),
                           stats.ctypes.data, threads or self.max_threads())
        return out, stats

    def render(self, scene, camera, settings, w, h, sample=0, sums=None, rows=None, threads=0):
        sums = np.zeros(w * h, PIXELSUM_DTYPE) if sums is None else sums
        rgba = np.zeros(w * h * 4, np.uint8)
        counts = np.zeros(11, np.int64)
        y0, y1 = rows if rows else (0, h)
        self.lib.orc_render(scene.handle, c.byref(camera), c.byref(settings), w, h, sample, sums.ctypes.data,
                            rgba.ctypes.data, y0, y1, threads or self.max_threads(), counts.ctypes.data)
        return sums, rgba, counts

    def render_pixels(self, scene, camera, settings, w, h, pixels, sample=0, threads=0):
        sums = np.zeros(w * h, PIXELSUM_DTYPE)
        rgba = np.zeros(w * h * 4, np.uint8)
        counts = np.zeros(11, np.int64)
        pixels = np.ascontiguousarray(pixels, np.int32)
        self.lib.orc_render_pixels(scene.handle, c.byref(camera), c.byref(settings), w, h, sample, sums.ctypes.data,
                                   rgba.ctypes.data, pixels.ctypes.data, len(pixels), threads or self.max_threads(),
                                   counts.ctypes.data)
        return sums, rgba, counts


class Reference:
    """The reference renderer's own code (Native/renderer.cu) behind thin wrappers."""
    prefix = 'refh_'

    def __init__(self, path=REFERENCE_LIB):
        if not Path(path).exists():
            raise FileNotFoundError(f'{path} missing: run `make -C {HERE} ref` where the reference sources exist')
        self.lib = c.CDLL(str(path))
        _setup_common(self.lib, self.prefix)
        vp = c.c_void_p
        self.lib.refh_scene_build_ms.argtypes = [vp]
        self.lib.refh_scene_build_ms.restype = c.c_float
        self.lib.refh_query.argtypes = [vp, vp, c.c_int, c.c_int, vp, c.c_int]
        self.lib.refh_render.argtypes = [vp, vp, vp, c.c_int, c.c_int, c.c_uint, vp, vp, c.c_int, c.c_int, c.c_int]

    def scene(self, triangles):
        return _Scene(self.lib, self.prefix, triangles)

    def max_threads(self):
        return self.lib.refh_max_threads()

    def build_ms(self, scene):
        return self.lib.refh_scene_build_ms(scene.handle)

    def sobol(self, pixel, sample, seed, ndim=SOBOL_DIMS):
        pixel, sample, seed = (np.ascontiguousarray(a, np.uint32) for a in (pixel, sample, seed))
        out = np.zeros((len(pixel), ndim), np.float32)
        if not self.lib.refh_sobol(pixel.ctypes.data, sample.ctypes.data, seed.ctypes.data, len(pixel), ndim,
                                   out.ctypes.data):
            raise RuntimeError('reference sampler failed')
        return out

    def query(self, scene, queries, any_hit=False, threads=0):
        q = np.ascontiguousarray(queries)
        out = np.zeros(len(q), HIT_DTYPE)
        self.lib.refh_query(scene.handle, q.ctypes.data, len(q), int(any_hit), out.ctypes.data,
                            threads or self.max_threads())
        return out

    def render(self, scene, camera, settings, w, h, sample=0, sums=None, rows=None, threads=0):
        sums = np.zeros(w * h, PIXELSUM_DTYPE) if sums is None else sums
        rgba = np.zeros(w * h * 4, np.uint8)
        y0, y1 = rows if rows else (0, h)
        self.lib.refh_render(scene.handle, c.byref(camera), c.byref(settings), w, h, sample, sums.ctypes.data,
                             rgba.ctypes.data, y0, y1, threads or self.max_threads())
        return sums, rgba


class ReferenceSession:
    """A session of the reference's own exported ABI (RtCreate ... RtRender) in
    oracle/_ref/libref.so. Backend 2 runs the reference's CUDA renderer
    (renderKernel, Native/renderer.cu:303) built for sm_100a; needs a GPU."""

    def __init__(self, reference):
        lib = reference.lib
        vp = c.c_void_p
        lib.RtCreate.restype = vp
        lib.RtDestroy.argtypes = [vp]
        lib.RtInitialize.argtypes = [vp, vp, c.c_int, c.c_int, c.c_int]
        lib.RtRender.argtypes = [vp, vp, vp, vp, c.c_int, c.c_int, vp]
        lib.RtLastError.argtypes = [vp]
        lib.RtLastError.restype = c.c_char_p
        lib.refh_session_sums.argtypes = [vp, vp, c.c_int]
        self.lib = lib
        self.handle = lib.RtCreate()
        self.w = self.h = 0

    def close(self):
        if self.handle:
            self.lib.RtDestroy(self.handle)
            self.handle = None

    def _check(self, ok):
        if not ok:
            raise RuntimeError(self.lib.RtLastError(self.handle).decode())

    def initialize(self, triangles, w, h):
        tris = np.ascontiguousarray(triangles)
        self._check(self.lib.RtInitialize(self.handle, tris.ctypes.data, len(tris), w, h))
        self.w, self.h = w, h

    def render(self, camera, settings, backend=2):
        out = np.zeros(self.w * self.h * 4, np.uint8)
        ms = c.c_float()
        self._check(self.lib.RtRender(self.handle, c.byref(camera), c.byref(settings), out.ctypes.data, out.size,
                                      backend, c.byref(ms)))
        return out, ms.value

    def sums(self):
        out = np.zeros(self.w * self.h, PIXELSUM_DTYPE)
        self._check(self.lib.refh_session_sums(self.handle, out.ctypes.data, out.size))
        return out


def reference_available():
    return REFERENCE_LIB.exists()
