"""ctypes bindings of libCudaRayTracer.so, mirroring the reference's Tools/native_api.py.

The structures, the size checks (116/64/28 bytes, Tools/native_api.py:26), the
RAYTRACER_LIBRARY override (:29), the argument types set by load_library
(:28-43) and unpack() for Unity JSON snapshots (:45-48) keep the reference's
names and meaning, so scripts written against the reference bind this library
unchanged. Additions: numpy record dtypes for bulk triangle arrays and the
additive Rtx* entry points declared in include/cuda_ray_tracer.h.
"""
import ctypes as c
import os
from pathlib import Path

import numpy as np


class Vector(c.Structure):
    _fields_ = [(axis, c.c_float) for axis in 'xyz']


class Triangle(c.Structure):
    _fields_ = [(name, Vector) for name in ('origin', 'edge1', 'edge2', 'color')]
    _fields_ += [('emission', c.c_float), ('oneSided', c.c_int)]
    _fields_ += [(name, Vector) for name in ('normal0', 'normal1', 'normal2')]
    _fields_ += [('mesh', c.c_int), ('specularColor', Vector), ('smoothness', c.c_float),
                 ('specularProbability', c.c_float)]


class Camera(c.Structure):
    _fields_ = [(name, Vector) for name in ('origin', 'right', 'up', 'forward')]
    _fields_ += [('tanHalfFov', c.c_float), ('aspect', c.c_float), ('orthographicSize', c.c_float),
                 ('orthographic', c.c_int)]


class Settings(c.Structure):
    _fields_ = [('maxBounces', c.c_int)]
    _fields_ += [(name, c.c_float) for name in ('exposure', 'aperture', 'focusDistance', 'skyStrength')]
    _fields_ += [('seed', c.c_uint), ('raysPerPixel', c.c_int)]


class PixelSum(c.Structure):
    _fields_ = [('radiance', Vector), ('albedo', Vector), ('normal', Vector), ('covered', c.c_uint)]


class BvhNode(c.Structure):
    _fields_ = [('low', Vector), ('first', c.c_int), ('high', Vector), ('count', c.c_int)]


class RtxQuery(c.Structure):
    _fields_ = [('origin', Vector), ('direction', Vector), ('limit', c.c_float)]


class RtxHit(c.Structure):
    _fields_ = [('index', c.c_int), ('distance', c.c_float), ('u', c.c_float), ('v', c.c_float)]


class RtxRenderStats(c.Structure):
    _fields_ = [('primaryRays', c.c_ulonglong), ('secondaryRays', c.c_ulonglong), ('shadowRays', c.c_ulonglong),
                ('paths', c.c_ulonglong), ('renderMs', c.c_float), ('extendMs', c.c_float),
                ('shadowMs', c.c_float), ('kernelLaunches', c.c_int), ('primaryMs', c.c_float),
                ('denoiseMs', c.c_float)]


class RtxBvhStats(c.Structure):
    _fields_ = [('binaryNodes', c.c_int), ('binaryDepth', c.c_int), ('wideNodes', c.c_int),
                ('wideDepth', c.c_int), ('buildMs', c.c_float), ('collapseMs', c.c_float),
                ('sahCost', c.c_double), ('uploadMs', c.c_float), ('distinctColours', c.c_int),
                ('lightCount', c.c_int), ('lightArea', c.c_float), ('pieces', c.c_int), ('pieceBuildMs', c.c_float)]


class RtxBatchTune(c.Structure):
    _fields_ = [('block', c.c_int), ('capacity', c.c_int), ('refill', c.c_int), ('width', c.c_int),
                ('frameMs', c.c_float), ('pieces', c.c_int), ('lanes', c.c_int)]


class RtxBatchStats(c.Structure):
    _fields_ = [('primaryRays', c.c_ulonglong), ('secondaryRays', c.c_ulonglong), ('shadowRays', c.c_ulonglong),
                ('paths', c.c_ulonglong), ('frameMs', c.c_float), ('buildMs', c.c_float),
                ('triangles', c.c_longlong), ('pixels', c.c_longlong), ('scenes', c.c_int), ('views', c.c_int),
                ('kernelLaunches', c.c_int), ('graph', c.c_int), ('block', c.c_int), ('capacity', c.c_int),
                ('refill', c.c_int), ('width', c.c_int), ('pieces', c.c_int), ('lanes', c.c_int)]


assert (c.sizeof(Triangle), c.sizeof(Camera), c.sizeof(Settings)) == (116, 64, 28)
assert (c.sizeof(RtxBatchTune), c.sizeof(RtxBatchStats)) == (28, 96)
assert (c.sizeof(PixelSum), c.sizeof(BvhNode), c.sizeof(RtxQuery), c.sizeof(RtxHit)) == (40, 32, 28, 16)

# numpy views of the same records, for scenes of millions of triangles.
VEC = [('x', '<f4'), ('y', '<f4'), ('z', '<f4')]
TRIANGLE_DTYPE = np.dtype([('origin', VEC), ('edge1', VEC), ('edge2', VEC), ('color', VEC),
                           ('emission', '<f4'), ('oneSided', '<i4'), ('normal0', VEC), ('normal1', VEC),
                           ('normal2', VEC), ('mesh', '<i4'), ('specularColor', VEC), ('smoothness', '<f4'),
                           ('specularProbability', '<f4')])
PIXELSUM_DTYPE = np.dtype([('radiance', VEC), ('albedo', VEC), ('normal', VEC), ('covered', '<u4')])
NODE_DTYPE = np.dtype([('low', VEC), ('first', '<i4'), ('high', VEC), ('count', '<i4')])
QUERY_DTYPE = np.dtype([('origin', VEC), ('direction', VEC), ('limit', '<f4')])
HIT_DTYPE = np.dtype([('index', '<i4'), ('distance', '<f4'), ('u', '<f4'), ('v', '<f4')])
assert (TRIANGLE_DTYPE.itemsize, PIXELSUM_DTYPE.itemsize, NODE_DTYPE.itemsize) == (116, 40, 32)

ROOT = Path(__file__).resolve().parent
LIBRARY = ROOT / 'libCudaRayTracer.so'
# Trained parameters of the learned denoiser (train_denoiser.py writes them).
DENOISER_WEIGHTS = ROOT / 'weights' / 'denoiser_unet.bin'

# Every symbol the header declares (include/cuda_ray_tracer.h).
EXPORTS = ('RtCreate', 'RtDestroy', 'RtShutdown', 'RtInitialize', 'RtRender', 'RtDenoise', 'RtReset',
           'RtAccumulationVersion', 'RtSampleCount', 'RtEmbreeBuildMilliseconds', 'RtCpuThreadCount',
           'RtBvhInfo', 'RtLastError', 'RtxQueryRays', 'RtxSobolSamples', 'RtxExportBvh', 'RtxBvhStatsGet',
           'RtxReadAccumulation', 'RtxRenderStatsGet', 'RtxRenderDevice', 'RtxSetIntegrator', 'RtxSetTuning',
           'RtxDebugFailAllocation', 'RtxSetConvPath', 'RtxDebugConvWaitProbe', 'RtxConvLaunchCounts',
           'RtxQueryRaysStatic', 'RtxSetEnvironment', 'RtxUnetCreate', 'RtxUnetDestroy', 'RtxUnetParamCount',
           'RtxUnetLastError', 'RtxUnetGetParams', 'RtxUnetSetParams', 'RtxUnetLossGrad', 'RtxUnetTrain',
           'RtxUnetInfer', 'RtxUnetSave', 'RtxUnetLoad', 'RtxSetDenoiser', 'RtxReadAovs', 'RtxReadDenoised',
           'RtxBatchCreate', 'RtxBatchDestroy', 'RtxBatchLastError', 'RtxBatchAddScene', 'RtxBatchAddView',
           'RtxBatchSetEnvironment', 'RtxBatchRender', 'RtxBatchReset', 'RtxBatchSampleCount', 'RtxBatchReadImage',
           'RtxBatchReadAccumulation', 'RtxBatchSetTuning', 'RtxBatchAutotune', 'RtxBatchStatsGet')


def load_library(path=None):
    """Loads the library and declares argument types (Tools/native_api.py:28-43)."""
    path = path or os.environ.get('RAYTRACER_LIBRARY', LIBRARY)
    path = Path(path).resolve()
    if not path.exists():
        raise FileNotFoundError(f'{path} is not built: run `make -C {ROOT}` (or __graft_entry__.build())')
    lib = c.CDLL(str(path))
    vp = c.c_void_p
    lib.RtCreate.restype = vp
    lib.RtDestroy.argtypes = lib.RtShutdown.argtypes = lib.RtReset.argtypes = lib.RtSampleCount.argtypes = [vp]
    lib.RtSampleCount.restype = c.c_uint
    lib.RtInitialize.argtypes = [vp, c.c_void_p, c.c_int, c.c_int, c.c_int]
    lib.RtRender.argtypes = [vp, c.POINTER(Camera), c.POINTER(Settings), c.POINTER(c.c_ubyte), c.c_int, c.c_int,
                             c.POINTER(c.c_float)]
    lib.RtLastError.argtypes = [vp]
    lib.RtLastError.restype = c.c_char_p
    lib.RtCpuThreadCount.argtypes = [vp]
    lib.RtDenoise.argtypes = [vp, c.POINTER(c.c_ubyte), c.c_int, c.POINTER(c.c_float)]
    lib.RtAccumulationVersion.argtypes = [vp]
    lib.RtAccumulationVersion.restype = c.c_uint
    lib.RtEmbreeBuildMilliseconds.argtypes = [vp]
    lib.RtEmbreeBuildMilliseconds.restype = c.c_float
    lib.RtBvhInfo.argtypes = [vp, c.POINTER(c.c_int), c.POINTER(c.c_int), c.POINTER(c.c_float)]
    lib.RtxQueryRays.argtypes = [vp, c.c_void_p, c.c_int, c.c_int, c.c_void_p]
    lib.RtxSobolSamples.argtypes = [c.c_void_p, c.c_void_p, c.c_void_p, c.c_int, c.c_int, c.c_void_p]
    lib.RtxExportBvh.argtypes = [vp, c.c_void_p, c.c_int, c.c_void_p, c.c_int]
    lib.RtxBvhStatsGet.argtypes = [vp, c.POINTER(RtxBvhStats)]
    lib.RtxReadAccumulation.argtypes = [vp, c.c_void_p, c.c_int]
    lib.RtxRenderStatsGet.argtypes = [vp, c.POINTER(RtxRenderStats)]
    lib.RtxRenderDevice.argtypes = [vp, c.POINTER(Camera), c.POINTER(Settings), c.POINTER(c.c_float)]
    lib.RtxSetIntegrator.argtypes = [vp, c.c_int]
    lib.RtxSetTuning.argtypes = [vp, c.c_int, c.c_int]
    lib.RtxDebugFailAllocation.argtypes = [c.c_int]
    lib.RtxSetConvPath.argtypes = [c.c_int]
    lib.RtxDebugConvWaitProbe.argtypes = []
    lib.RtxConvLaunchCounts.argtypes = [c.c_void_p, c.c_void_p]
    lib.RtxQueryRaysStatic.argtypes = [vp, c.c_void_p, c.c_int, c.c_int, c.c_void_p]
    lib.RtxSetEnvironment.argtypes = [vp, c.c_int, c.c_float, c.c_float, c.c_float]
    lib.RtxUnetCreate.restype = vp
    lib.RtxUnetCreate.argtypes = [c.c_uint]
    lib.RtxUnetDestroy.argtypes = [vp]
    lib.RtxUnetParamCount.argtypes = [vp]
    lib.RtxUnetParamCount.restype = c.c_longlong
    lib.RtxUnetLastError.argtypes = [vp]
    lib.RtxUnetLastError.restype = c.c_char_p
    lib.RtxUnetGetParams.argtypes = lib.RtxUnetSetParams.argtypes = [vp, c.c_void_p]
    lib.RtxUnetLossGrad.argtypes = [vp, c.c_void_p, c.c_void_p, c.c_int, c.c_int, c.c_int, c.c_void_p, c.c_void_p]
    lib.RtxUnetTrain.argtypes = [vp, c.c_void_p, c.c_void_p, c.c_int, c.c_int, c.c_int, c.c_int, c.c_int, c.c_float,
                                 c.c_uint, c.c_void_p]
    lib.RtxUnetInfer.argtypes = [vp, c.c_void_p, c.c_int, c.c_int, c.c_void_p]
    lib.RtxUnetSave.argtypes = [vp, c.c_char_p, c.c_int]
    lib.RtxUnetLoad.argtypes = [vp, c.c_char_p]
    lib.RtxSetDenoiser.argtypes = [vp, vp]
    lib.RtxReadAovs.argtypes = [vp, c.c_void_p, c.c_int]
    lib.RtxReadDenoised.argtypes = [vp, c.c_void_p, c.c_int]
    lib.RtxBatchCreate.restype = vp
    lib.RtxBatchCreate.argtypes = []
    lib.RtxBatchDestroy.argtypes = [vp]
    lib.RtxBatchLastError.argtypes = [vp]
    lib.RtxBatchLastError.restype = c.c_char_p
    lib.RtxBatchAddScene.argtypes = [vp, c.c_void_p, c.c_int]
    lib.RtxBatchAddView.argtypes = [vp, c.c_int, c.POINTER(Camera), c.c_int, c.c_int]
    lib.RtxBatchSetEnvironment.argtypes = [vp, c.c_int, c.c_float, c.c_float, c.c_float]
    lib.RtxBatchRender.argtypes = [vp, c.POINTER(Settings), c.POINTER(c.c_float)]
    lib.RtxBatchReset.argtypes = [vp]
    lib.RtxBatchSampleCount.argtypes = [vp]
    lib.RtxBatchSampleCount.restype = c.c_uint
    lib.RtxBatchReadImage.argtypes = [vp, c.c_int, c.c_void_p, c.c_int]
    lib.RtxBatchReadAccumulation.argtypes = [vp, c.c_int, c.c_void_p, c.c_int]
    lib.RtxBatchSetTuning.argtypes = [vp, c.c_int, c.c_int]
    lib.RtxBatchAutotune.argtypes = [vp, c.POINTER(Settings), c.POINTER(RtxBatchTune), c.c_int,
                                     c.POINTER(c.c_int)]
    lib.RtxBatchStatsGet.argtypes = [vp, c.POINTER(RtxBatchStats)]
    return lib


def unpack(structure, values):
    """Read Unity's JSON snapshot without changing its float inputs (Tools/native_api.py:45-48)."""
    return structure(**{name: Vector(**values[name]) if field is Vector else values[name]
                        for name, field in structure._fields_})


def triangles_array(records):
    """A contiguous TRIANGLE_DTYPE array from numpy records or a ctypes Triangle array."""
    if isinstance(records, np.ndarray):
        return np.ascontiguousarray(records, dtype=TRIANGLE_DTYPE)
    return np.frombuffer(bytes(records), dtype=TRIANGLE_DTYPE).copy()


class NativeError(RuntimeError):
    pass


class Session:
    """Thin owner of one native session (RtCreate/RtDestroy) with checked calls."""

    def __init__(self, lib=None):
        self.lib = lib or load_library()
        self.handle = self.lib.RtCreate()
        self.width = self.height = 0

    def close(self):
        if self.handle:
            self.lib.RtDestroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def error(self):
        return self.lib.RtLastError(self.handle).decode()

    def check(self, ok):
        if not ok:
            raise NativeError(self.error())

    def initialize(self, triangles, width, height):
        tris = triangles_array(triangles)
        self.check(self.lib.RtInitialize(self.handle, tris.ctypes.data, len(tris), width, height))
        self.width, self.height = width, height
        return self

    def render(self, camera, settings, backend=2, output=None):
        output = output if output is not None else np.zeros(self.width * self.height * 4, np.uint8)
        ms = c.c_float()
        self.check(self.lib.RtRender(self.handle, c.byref(camera), c.byref(settings),
                                     output.ctypes.data_as(c.POINTER(c.c_ubyte)), output.size, backend, c.byref(ms)))
        return output, ms.value

    def render_device(self, camera, settings):
        ms = c.c_float()
        self.check(self.lib.RtxRenderDevice(self.handle, c.byref(camera), c.byref(settings), c.byref(ms)))
        return ms.value

    def denoise(self, output=None):
        output = output if output is not None else np.zeros(self.width * self.height * 4, np.uint8)
        ms = c.c_float()
        self.check(self.lib.RtDenoise(self.handle, output.ctypes.data_as(c.POINTER(c.c_ubyte)), output.size,
                                      c.byref(ms)))
        return output, ms.value

    def accumulation(self):
        out = np.zeros(self.width * self.height, PIXELSUM_DTYPE)
        self.check(self.lib.RtxReadAccumulation(self.handle, out.ctypes.data, out.size))
        return out

    def query(self, queries, any_hit=False):
        q = np.ascontiguousarray(queries, dtype=QUERY_DTYPE)
        out = np.zeros(len(q), HIT_DTYPE)
        self.check(self.lib.RtxQueryRays(self.handle, q.ctypes.data, len(q), int(any_hit), out.ctypes.data))
        return out

    STATIC_QUERY_CAPACITY = 16384

    def query_static(self, queries, any_hit=False):
        """RtxQueryRaysStatic: the same answers as query(), staged without device allocation."""
        q = np.ascontiguousarray(queries, dtype=QUERY_DTYPE)
        out = np.zeros(len(q), HIT_DTYPE)
        self.check(self.lib.RtxQueryRaysStatic(self.handle, q.ctypes.data, len(q), int(any_hit), out.ctypes.data))
        return out

    def bvh_info(self):
        nodes, depth, ms = c.c_int(), c.c_int(), c.c_float()
        self.lib.RtBvhInfo(self.handle, c.byref(nodes), c.byref(depth), c.byref(ms))
        return nodes.value, depth.value, ms.value

    def bvh_stats(self):
        st = RtxBvhStats()
        self.check(self.lib.RtxBvhStatsGet(self.handle, c.byref(st)))
        return {name: getattr(st, name) for name, _ in st._fields_}

    def export_bvh(self, triangle_count):
        n = self.bvh_info()[0]
        nodes = np.zeros(n, NODE_DTYPE)
        order = np.zeros(triangle_count, np.int32)
        self.check(self.lib.RtxExportBvh(self.handle, nodes.ctypes.data, n, order.ctypes.data, triangle_count))
        return nodes, order

    def render_stats(self):
        st = RtxRenderStats()
        self.check(self.lib.RtxRenderStatsGet(self.handle, c.byref(st)))
        return {name: getattr(st, name) for name, _ in st._fields_}

    def set_integrator(self, mode):
        self.check(self.lib.RtxSetIntegrator(self.handle, mode))

    TUNE_PATHS_IN_FLIGHT, TUNE_POSTPONE, TUNE_REFILL, TUNE_PIECES, TUNE_LEAF, TUNE_LANES = 1, 2, 3, 4, 5, 6
    TUNE_STACK_LIMIT = 7

    def set_tuning(self, paths_in_flight=None, postpone=None, refill=None, pieces=None, leaf=None, lanes=None,
                   stack_limit=None):
        """pieces and leaf apply from the next initialize(); stack_limit below
        48 makes traversal fail with a stack overflow (the failure path)."""
        for key, value in ((self.TUNE_PATHS_IN_FLIGHT, paths_in_flight), (self.TUNE_POSTPONE, postpone),
                           (self.TUNE_REFILL, refill), (self.TUNE_PIECES, pieces), (self.TUNE_LEAF, leaf),
                           (self.TUNE_LANES, lanes), (self.TUNE_STACK_LIMIT, stack_limit)):
            if value is not None:
                self.check(self.lib.RtxSetTuning(self.handle, key, int(value)))

    def set_environment(self, constant=None):
        """None: the reference's sky gradient; a float or RGB triple: constant radiance."""
        if constant is None:
            self.check(self.lib.RtxSetEnvironment(self.handle, 0, 0.0, 0.0, 0.0))
        else:
            r, g, b = (constant,) * 3 if isinstance(constant, (int, float)) else constant
            self.check(self.lib.RtxSetEnvironment(self.handle, 1, r, g, b))

    def aovs(self):
        """Denoiser inputs of the current accumulation, shape (height, width, 10)."""
        out = np.zeros((self.height, self.width, 10), np.float32)
        self.check(self.lib.RtxReadAovs(self.handle, out.ctypes.data, self.width * self.height))
        return out

    def denoised_radiance(self):
        """Linear radiance of the last denoise(), (width*height, 3) float32."""
        out = np.zeros((self.width * self.height, 3), np.float32)
        self.check(self.lib.RtxReadDenoised(self.handle, out.ctypes.data, self.width * self.height))
        return out

    def set_denoiser(self, net):
        self.check(self.lib.RtxSetDenoiser(self.handle, net.handle if net is not None else None))

    def sample_count(self):
        return self.lib.RtSampleCount(self.handle)

    def version(self):
        return self.lib.RtAccumulationVersion(self.handle)


def sobol_samples(lib, pixel, sample, seed, ndim):
    """Device sampler values, shape (count, ndim)."""
    pixel = np.ascontiguousarray(pixel, np.uint32)
    sample = np.ascontiguousarray(sample, np.uint32)
    seed = np.ascontiguousarray(seed, np.uint32)
    out = np.zeros((len(pixel), ndim), np.float32)
    if not lib.RtxSobolSamples(pixel.ctypes.data, sample.ctypes.data, seed.ctypes.data, len(pixel), ndim,
                               out.ctypes.data):
        raise NativeError('RtxSobolSamples failed')
    return out


class Unet:
    """The learned denoiser (RtxUnet* entry points)."""

    def __init__(self, lib=None, seed=1):
        self.lib = lib or load_library()
        self.handle = self.lib.RtxUnetCreate(seed)
        if not self.handle:
            raise NativeError('RtxUnetCreate failed')

    def close(self):
        if self.handle:
            self.lib.RtxUnetDestroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, ok):
        if not ok:
            raise NativeError(self.lib.RtxUnetLastError(self.handle).decode())

    @property
    def param_count(self):
        return self.lib.RtxUnetParamCount(self.handle)

    def params(self):
        out = np.zeros(self.param_count, np.float32)
        self.check(self.lib.RtxUnetGetParams(self.handle, out.ctypes.data))
        return out

    def set_params(self, params):
        p = np.ascontiguousarray(params, np.float32)
        assert p.size == self.param_count
        self.check(self.lib.RtxUnetSetParams(self.handle, p.ctypes.data))

    def loss_grad(self, aovs, targets):
        a = np.ascontiguousarray(aovs, np.float32)
        t = np.ascontiguousarray(targets, np.float32)
        n, h, w = a.shape[:3]
        loss = np.zeros(1, np.float32)
        grads = np.zeros(self.param_count, np.float32)
        self.check(self.lib.RtxUnetLossGrad(self.handle, a.ctypes.data, t.ctypes.data, n, h, w, loss.ctypes.data,
                                            grads.ctypes.data))
        return float(loss[0]), grads

    def train(self, aovs, targets, steps, batch=16, lr=1e-3, seed=0):
        a = np.ascontiguousarray(aovs, np.float32)
        t = np.ascontiguousarray(targets, np.float32)
        n, h, w = a.shape[:3]
        losses = np.zeros(max(steps, 1), np.float32)
        self.check(self.lib.RtxUnetTrain(self.handle, a.ctypes.data, t.ctypes.data, n, h, w, steps, batch, lr, seed,
                                         losses.ctypes.data))
        return losses[:steps]

    def infer(self, aovs):
        a = np.ascontiguousarray(aovs, np.float32)
        h, w = a.shape[:2]
        out = np.zeros((h, w, 3), np.float32)
        self.check(self.lib.RtxUnetInfer(self.handle, a.ctypes.data, h, w, out.ctypes.data))
        return out

    def save(self, path, optimizer_state=False):
        self.check(self.lib.RtxUnetSave(self.handle, str(path).encode(), int(optimizer_state)))

    def load(self, path):
        self.check(self.lib.RtxUnetLoad(self.handle, str(path).encode()))


class Batch:
    """Many views of many scenes rendered together (RtxBatch* entry points)."""

    BLOCK, CAPACITY, REFILL, GRAPH, WIDTH, PIECES, LEAF, LANES, PERSISTENT = 1, 2, 3, 4, 5, 6, 7, 8, 9

    def __init__(self, lib=None):
        self.lib = lib or load_library()
        self.handle = self.lib.RtxBatchCreate()
        self.views = []

    def close(self):
        if self.handle:
            self.lib.RtxBatchDestroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def error(self):
        return self.lib.RtxBatchLastError(self.handle).decode()

    def check(self, ok):
        if not ok:
            raise NativeError(self.error())

    def add_scene(self, triangles):
        tris = triangles_array(triangles)
        k = self.lib.RtxBatchAddScene(self.handle, tris.ctypes.data, len(tris))
        self.check(k >= 0)
        return k

    def add_view(self, scene, camera, width, height):
        k = self.lib.RtxBatchAddView(self.handle, scene, c.byref(camera), width, height)
        self.check(k >= 0)
        self.views.append((width, height))
        return k

    def set_environment(self, constant=None):
        if constant is None:
            self.check(self.lib.RtxBatchSetEnvironment(self.handle, 0, 0.0, 0.0, 0.0))
        else:
            r, g, b = (constant,) * 3 if isinstance(constant, (int, float)) else constant
            self.check(self.lib.RtxBatchSetEnvironment(self.handle, 1, r, g, b))

    def render(self, settings):
        ms = c.c_float()
        self.check(self.lib.RtxBatchRender(self.handle, c.byref(settings), c.byref(ms)))
        return ms.value

    def reset(self):
        self.lib.RtxBatchReset(self.handle)

    def sample_count(self):
        return self.lib.RtxBatchSampleCount(self.handle)

    def image(self, view):
        w, h = self.views[view]
        out = np.zeros(w * h * 4, np.uint8)
        self.check(self.lib.RtxBatchReadImage(self.handle, view, out.ctypes.data, out.size))
        return out

    def accumulation(self, view):
        w, h = self.views[view]
        out = np.zeros(w * h, PIXELSUM_DTYPE)
        self.check(self.lib.RtxBatchReadAccumulation(self.handle, view, out.ctypes.data, out.size))
        return out

    def set_tuning(self, block=None, capacity=None, refill=None, graph=None, width=None, pieces=None, leaf=None,
                   lanes=None, persistent=None):
        for key, value in ((self.BLOCK, block), (self.CAPACITY, capacity), (self.REFILL, refill),
                           (self.GRAPH, graph), (self.WIDTH, width), (self.PIECES, pieces), (self.LEAF, leaf),
                           (self.LANES, lanes), (self.PERSISTENT, persistent)):
            if value is not None:
                self.check(self.lib.RtxBatchSetTuning(self.handle, key, int(value)))

    def autotune(self, settings, max_results=64):
        results = (RtxBatchTune * max_results)()
        count = c.c_int()
        self.check(self.lib.RtxBatchAutotune(self.handle, c.byref(settings), results, max_results, c.byref(count)))
        return [{name: getattr(r, name) for name, _ in RtxBatchTune._fields_} for r in results[:count.value]]

    def stats(self):
        st = RtxBatchStats()
        self.check(self.lib.RtxBatchStatsGet(self.handle, c.byref(st)))
        return {name: getattr(st, name) for name, _ in st._fields_}
