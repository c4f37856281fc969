"""The library's portable code (wide-BVH collapse, traversal, integrator),
compiled for the host, against the reference's fixtures. CPU only.

tests/hostcheck/host_check.cu includes the same headers the CUDA kernels are
built from; the binary tree it collapses comes from the oracle's builder
(equal to the reference's, tests/test_oracle_golden.py)."""
import ctypes as c
import subprocess
from pathlib import Path

import numpy as np
import pytest

import scenes
from conftest import ROOT, golden
from native_api import HIT_DTYPE, PIXELSUM_DTYPE
from test_oracle_golden import GEOMETRY, RAYS, SETS

HERE = Path(__file__).resolve().parent / 'hostcheck'
LIB = HERE / '_build' / 'libhostcheck.so'
SOURCES = [HERE / 'host_check.cu'] + sorted((ROOT / 'custom-ray-tracing-shader_b200' / 'csrc').glob('*.cuh'))


@pytest.fixture(scope='module')
def hc():
    if not LIB.exists() or any(p.stat().st_mtime > LIB.stat().st_mtime for p in SOURCES):
        LIB.parent.mkdir(exist_ok=True)
        subprocess.run(['nvcc', '-O2', '--fmad=false', '-std=c++17', '-arch=sm_100a', '--shared',
                        '-Xcompiler=-fPIC', str(HERE / 'host_check.cu'), '-o', str(LIB)], check=True)
    lib = c.CDLL(str(LIB))
    vp = c.c_void_p
    lib.hc_collapse.argtypes = [vp, vp, vp, c.c_int, vp, c.c_int, vp, vp, c.c_int, c.c_int]
    lib.hc_query.argtypes = [vp, vp, vp, c.c_int, c.c_int, vp, vp, vp, c.c_int]
    lib.hc_render.argtypes = [vp, vp, c.c_int, c.c_float, vp, vp, vp, vp, vp, c.c_int, c.c_int, c.c_uint, vp, vp, vp]
    return lib


def collapse(hc, scene, group=3, width=8):
    nodes, order, lin = scene.nodes(), scene.order(), scene.linear_triangles()
    n = len(lin)
    cap = 2 * n + 8
    wide = np.zeros(cap * 20, np.uint32)
    packed = np.zeros(n * 12, np.float32)
    res = np.zeros(4, np.int32)
    assert hc.hc_collapse(nodes.ctypes.data, order.ctypes.data, lin.ctypes.data, n, wide.ctypes.data, cap,
                          packed.ctypes.data, res.ctypes.data, group, width)
    assert res[3] == n, 'every triangle packed exactly once'
    return wide, packed, res


@pytest.mark.parametrize('group,width', ((1, 8), (2, 8), (3, 8), (3, 4), (1, 4)))
@pytest.mark.parametrize('name', SETS)
def test_wide_traversal_matches_reference(hc, oracle, name, group, width):
    g = golden(f'bvh_{name}.npz')
    sc = oracle.scene(GEOMETRY[name])
    wide, packed, res = collapse(hc, sc, group, width)
    W = wide[:res[0] * 20].reshape(-1, 20)
    children = np.array([[m != 0 for m in node.view(np.uint8)[24:32]] for node in W[:200]])
    assert children.sum(axis=1).max() <= width
    assert res[1] <= 48
    for any_hit in (0, 1):
        out = np.zeros(len(RAYS), HIT_DTYPE)
        stats = np.zeros(3, np.uint64)
        hc.hc_query(wide.ctypes.data, packed.ctypes.data, np.ascontiguousarray(RAYS).ctypes.data, len(RAYS), any_hit,
                    out.ctypes.data, stats.ctypes.data, None, 0)
        assert stats[2] == 0
        if any_hit:
            assert ((out['index'] >= 0) == (g['any_index'] >= 0)).all()
        else:
            assert out.tobytes() == g['closest'].tobytes()


def test_wide_nodes_quantised_conservatively(hc, oracle):
    """Every child box, dequantised the way traversal does it, contains the
    padded boxes of the triangles below it."""
    sc = oracle.scene(GEOMETRY['scatter'])
    wide, packed, res = collapse(hc, sc)
    W = wide[:res[0] * 20].reshape(-1, 20)
    P = packed.reshape(-1, 3, 4)
    for node in W[:64]:
        p = node[:3].view(np.float32)
        e = node[3] & 0xFF, (node[3] >> 8) & 0xFF, (node[3] >> 16) & 0xFF
        scale = np.array([np.uint32(x << 23).view(np.float32) for x in e], np.float32)
        meta = node[6:8].view(np.uint8)
        q = node[8:20].view(np.uint8).reshape(6, 8)
        tri_base = int(node[5])
        for s in range(8):
            m = int(meta[s])
            if m == 0 or (m & 0x18) == 0x18:
                continue
            lo = p + q[0:3, s].astype(np.float32) * scale
            hi = p + q[3:6, s].astype(np.float32) * scale
            bits = m >> 5
            off = m & 0x1F
            for k in range(3):
                if bits >> k & 1:
                    t = P[tri_base + off + k]
                    o = t[0, :3]
                    e1 = np.array([t[0, 3], t[1, 0], t[1, 1]], np.float32)
                    e2 = np.array([t[1, 2], t[1, 3], t[2, 0]], np.float32)
                    for v in (o, o + e1, o + e2):
                        assert (v >= lo).all() and (v <= hi).all()


def test_integrator_matches_reference(hc, oracle):
    g = golden('render_cornell.npz')
    tris, cam, st, _, _ = scenes.cornell_sphere()
    sc = oracle.scene(tris)
    wide, packed, _ = collapse(hc, sc)
    W, H = int(g['width']), int(g['height'])
    cam.aspect = W / H
    st.raysPerPixel = int(g['rays_per_pixel'])
    lights, lin, dirs = sc.lights(), sc.linear_triangles(), oracle.sobol_directions()
    sums = np.zeros(W * H, PIXELSUM_DTYPE)
    rgba = np.zeros(W * H * 4, np.uint8)
    counts = np.zeros(3, np.uint64)
    for sample, key in ((0, '1'), (3, '2')):
        assert hc.hc_render(lin.ctypes.data, lights.ctypes.data, len(lights), c.c_float(sc.light_area()),
                            wide.ctypes.data, packed.ctypes.data, dirs.ctypes.data, c.byref(cam), c.byref(st), W, H,
                            sample, sums.ctypes.data, rgba.ctypes.data, counts.ctypes.data)
        assert sums.tobytes() == g['sums' + key].tobytes()
        assert rgba.tobytes() == g['rgba' + key].tobytes()


def test_integrator_features_match_reference(hc, oracle):
    import make_golden
    g = golden('render_features.npz')
    feat = make_golden.feature_scene()
    sc = oracle.scene(feat['triangles'])
    wide, packed, _ = collapse(hc, sc)
    lights, lin, dirs = sc.lights(), sc.linear_triangles(), oracle.sobol_directions()
    W, H = feat['width'], feat['height']
    for key, (cam, st) in feat['views'].items():
        sums = np.zeros(W * H, PIXELSUM_DTYPE)
        rgba = np.zeros(W * H * 4, np.uint8)
        counts = np.zeros(3, np.uint64)
        assert hc.hc_render(lin.ctypes.data, lights.ctypes.data, len(lights), c.c_float(sc.light_area()),
                            wide.ctypes.data, packed.ctypes.data, dirs.ctypes.data, c.byref(cam), c.byref(st), W, H, 0,
                            sums.ctypes.data, rgba.ctypes.data, counts.ctypes.data)
        assert sums.tobytes() == g[key + '_sums'].tobytes(), key
