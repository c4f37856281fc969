"""Scene input and output: the reference's snapshot files and meshes.

- load_snapshot / save_snapshot: the JSON snapshot the Unity front end writes
  (RayTraceSession.SaveSnapshot, UnityRayTracer/Assets/RayTracing/
  RayTraceSession.cs:170-184: triangles, camera, settings, width, height) and
  the reference's tools read, plain or gzip-compressed
  (Tools/verify_quality.py:31-33, Tools/benchmark_native.py:33-36). Floats
  are read as the tools read them (Tools/native_api.py:45-48: each JSON
  number rounded to float32), so a loaded scene holds the same bytes.
- load_obj: Wavefront OBJ meshes (v, vn, f with v, v/vt, v//vn, v/vt/vn
  corners, negative indices, polygons as triangle fans). unity_axes=True
  applies Unity's import conventions (x negated, winding reversed), under
  which the reference's Dragon_80K.obj becomes the mesh of its dragon room.
- load_mesh_json: the {vertices, triangles} files Tools/generate_suzanne.py
  writes (UnityRayTracer/Assets/RayTracing/Models/Suzanne.json).
- recalculate_normals: area-weighted vertex normals (the sum of the faces'
  cross products, normalised), as the Suzanne asset gets them
  (Editor/FirstSceneBuilder.cs:26).
- object_triangles: one object's Triangle records the way
  RayTraceSession.CollectTriangles builds them (RayTraceSession.cs:95-133):
  corners through the object's transform, edges from the first corner,
  triangles whose normalised face normal vanishes dropped, normals through
  the inverse transpose, material fields copied. Arithmetic in float32 like
  Unity's.

Command line, after Tools/benchmark_native.py (one JSON line per case):
  python scene_io.py SNAPSHOT [--sizes 320x180,1280x720] [--bounces 3,8]
                              [--backend 2] [--passes 5]
"""
import argparse
import gzip
import json
import math
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
if str(HERE) not in sys.path:
    sys.path.insert(0, str(HERE))

from native_api import TRIANGLE_DTYPE, Camera, Settings, Vector, triangles_array  # noqa: E402

_VECTOR_FIELDS = ('origin', 'edge1', 'edge2', 'color', 'normal0', 'normal1', 'normal2', 'specularColor')
_SCALAR_FIELDS = (('emission', float), ('oneSided', int), ('mesh', int), ('smoothness', float),
                  ('specularProbability', float))


def _read_json(path):
    data = Path(path).read_bytes()
    if str(path).endswith('.gz'):
        data = gzip.decompress(data)
    return json.loads(data)


def _struct(cls, values):
    """A ctypes record from a JSON object, floats rounded to float32 by ctypes."""
    kwargs = {}
    for name, field in cls._fields_:
        v = values[name]
        kwargs[name] = Vector(v['x'], v['y'], v['z']) if field is Vector else v
    return cls(**kwargs)


def triangles_from_json(items):
    """TRIANGLE_DTYPE array from the snapshot's list of triangle objects."""
    n = len(items)
    out = np.zeros(n, TRIANGLE_DTYPE)
    for name in _VECTOR_FIELDS:
        arr = np.array([(t[name]['x'], t[name]['y'], t[name]['z']) for t in items], np.float64).reshape(n, 3)
        arr = arr.astype(np.float32)
        for k, axis in enumerate('xyz'):
            out[name][axis] = arr[:, k]
    for name, kind in _SCALAR_FIELDS:
        values = np.array([t[name] for t in items], np.float64 if kind is float else np.int64)
        out[name] = values.astype(np.float32 if kind is float else np.int32)
    return out


def load_snapshot(path):
    """(triangles, camera, settings, width, height) of a snapshot file."""
    scene = _read_json(path)
    return (triangles_from_json(scene['triangles']), _struct(Camera, scene['camera']),
            _struct(Settings, scene['settings']), int(scene['width']), int(scene['height']))


def _num(x):
    return float(x)


def _vector_json(v):
    return {'x': _num(v[0]), 'y': _num(v[1]), 'z': _num(v[2])}


def _struct_json(s):
    out = {}
    for name, field in s._fields_:
        v = getattr(s, name)
        out[name] = _vector_json((v.x, v.y, v.z)) if field is Vector else v
    return out


def save_snapshot(path, triangles, camera, settings, width, height):
    """Writes the snapshot format (gzip when the name ends in .gz); every
    float is written as the decimal of its float32 value, so loading gives
    the same bytes back."""
    tris = triangles_array(triangles)
    items = []
    for t in tris:
        item = {}
        for name in ('origin', 'edge1', 'edge2', 'color'):
            item[name] = _vector_json(t[name].tolist())
        item['emission'] = _num(t['emission'])
        item['oneSided'] = int(t['oneSided'])
        for name in ('normal0', 'normal1', 'normal2'):
            item[name] = _vector_json(t[name].tolist())
        item['mesh'] = int(t['mesh'])
        item['specularColor'] = _vector_json(t['specularColor'].tolist())
        item['smoothness'] = _num(t['smoothness'])
        item['specularProbability'] = _num(t['specularProbability'])
        items.append(item)
    data = json.dumps({'triangles': items, 'camera': _struct_json(camera), 'settings': _struct_json(settings),
                       'width': int(width), 'height': int(height)}, separators=(',', ':')).encode()
    Path(path).write_bytes(gzip.compress(data) if str(path).endswith('.gz') else data)


# ---- meshes ----

def load_obj(path, unity_axes=False):
    """(vertices (V,3), indices (T,3), corner normals (T,3,3) or None)."""
    verts, normals, tris, tri_normals = [], [], [], []
    have_normals = True
    with open(path) as f:
        for line in f:
            parts = line.split()
            if not parts:
                continue
            if parts[0] == 'v':
                verts.append([float(x) for x in parts[1:4]])
            elif parts[0] == 'vn':
                normals.append([float(x) for x in parts[1:4]])
            elif parts[0] == 'f':
                corners = []
                for c in parts[1:]:
                    fields = c.split('/')
                    vi = int(fields[0])
                    vi = vi - 1 if vi > 0 else len(verts) + vi
                    ni = None
                    if len(fields) >= 3 and fields[2]:
                        ni = int(fields[2])
                        ni = ni - 1 if ni > 0 else len(normals) + ni
                    corners.append((vi, ni))
                for k in range(1, len(corners) - 1):
                    tri = (corners[0], corners[k], corners[k + 1])
                    tris.append([c[0] for c in tri])
                    if any(c[1] is None for c in tri):
                        have_normals = False
                    else:
                        tri_normals.append([c[1] for c in tri])
    v = np.array(verts, np.float64).reshape(-1, 3)
    idx = np.array(tris, np.int64).reshape(-1, 3)
    n = None
    if have_normals and len(tri_normals) == len(tris) and len(tris):
        n = np.array(normals, np.float64)[np.array(tri_normals, np.int64)]
    if unity_axes:
        v = v * np.array([-1.0, 1.0, 1.0])
        idx = idx[:, [0, 2, 1]]
        if n is not None:
            n = n[:, [0, 2, 1]] * np.array([-1.0, 1.0, 1.0])
    return v, idx, n


def load_mesh_json(path):
    """(vertices (V,3), indices (T,3)) of a {vertices, triangles} mesh file."""
    data = _read_json(path)
    v = np.array([(p['x'], p['y'], p['z']) for p in data['vertices']], np.float64)
    return v, np.array(data['triangles'], np.int64).reshape(-1, 3)


def recalculate_normals(vertices, indices):
    """Corner normals (T,3,3): each vertex gets its faces' summed cross
    products, normalised."""
    v = np.asarray(vertices, np.float64)
    face = np.cross(v[indices[:, 1]] - v[indices[:, 0]], v[indices[:, 2]] - v[indices[:, 0]])
    vn = np.zeros_like(v)
    for k in range(3):
        np.add.at(vn, indices[:, k], face)
    vn /= np.maximum(np.linalg.norm(vn, axis=1, keepdims=True), 1e-30)
    return vn[indices]


def quaternion_matrix(x, y, z, w):
    """Rotation matrix of a unit quaternion (x, y, z, w)."""
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def euler_quaternion(x_deg, y_deg, z_deg):
    """Unity's Quaternion.Euler: rotation about z, then x, then y (degrees)."""
    def axis(a, deg):
        h = math.radians(deg) / 2
        q = [0.0, 0.0, 0.0, math.cos(h)]
        q[a] = math.sin(h)
        return q

    def mul(p, q):
        px, py, pz, pw = p
        qx, qy, qz, qw = q
        return [pw * qx + px * qw + py * qz - pz * qy, pw * qy - px * qz + py * qw + pz * qx,
                pw * qz + px * qy - py * qx + pz * qw, pw * qw - px * qx - py * qy - pz * qz]
    return tuple(mul(mul(axis(1, y_deg), axis(0, x_deg)), axis(2, z_deg)))


def _normalized32(v):
    """Unity's Vector3.normalized in float32: zero when the length is <= 1e-5."""
    length = np.sqrt((v * v).sum(axis=1, dtype=np.float32)).astype(np.float32)
    ok = length > np.float32(1e-5)
    out = np.zeros_like(v)
    out[ok] = v[ok] / length[ok, None]
    return out


def object_triangles(vertices, indices, normals=None, position=(0, 0, 0), rotation=(0, 0, 0, 1), scale=1.0,
                     color=(1, 1, 1), emission=0.0, one_sided=False, mesh=0, specular_color=(1, 1, 1),
                     smoothness=0.0, specular_probability=0.0):
    """Triangle records of one object (RayTraceSession.cs:104-129). rotation
    is a quaternion (x, y, z, w); scale a number or three; normals (T,3,3)
    corner normals in object space or None for face normals."""
    f32 = np.float32
    s = np.broadcast_to(np.asarray(scale, np.float64), (3,))
    m = (quaternion_matrix(*rotation) * s[None, :]).astype(f32)
    t = np.asarray(position, f32)
    v = np.asarray(vertices, f32)
    world = (v[:, 0:1] * m[:, 0] + v[:, 1:2] * m[:, 1] + v[:, 2:3] * m[:, 2]) + t
    a, b, c = world[indices[:, 0]], world[indices[:, 1]], world[indices[:, 2]]
    e1, e2 = b - a, c - a
    face = _normalized32(np.cross(e1, e2).astype(f32))
    keep = (face * face).sum(axis=1, dtype=f32) >= f32(0.5)
    out = np.zeros(int(keep.sum()), TRIANGLE_DTYPE)

    def put(name, arr):
        arr = np.broadcast_to(np.asarray(arr, f32), (len(out), 3))
        for k, axis in enumerate('xyz'):
            out[name][axis] = arr[:, k]
    put('origin', a[keep])
    put('edge1', e1[keep])
    put('edge2', e2[keep])
    put('color', color)
    put('specularColor', specular_color)
    if normals is None:
        for name in ('normal0', 'normal1', 'normal2'):
            put(name, face[keep])
    else:
        nm = np.linalg.inv(quaternion_matrix(*rotation) * s[None, :]).T.astype(f32)
        for k, name in enumerate(('normal0', 'normal1', 'normal2')):
            n = np.asarray(normals[:, k], f32)
            put(name, _normalized32((n[:, 0:1] * nm[:, 0] + n[:, 1:2] * nm[:, 1] + n[:, 2:3] * nm[:, 2]))[keep])
    out['emission'] = emission
    out['oneSided'] = 1 if one_sided else 0
    out['mesh'] = mesh
    out['smoothness'] = smoothness
    out['specularProbability'] = specular_probability
    return out


def main(argv=None):
    from native_api import Session, load_library
    ap = argparse.ArgumentParser(description='Render a snapshot file and print timings (one JSON line per case).')
    ap.add_argument('snapshot', type=Path)
    ap.add_argument('--sizes', default='320x180,1280x720')
    ap.add_argument('--bounces', default='3,8')
    ap.add_argument('--backend', type=int, default=2, choices=(0, 1, 2))
    ap.add_argument('--passes', type=int, default=5, help='measured passes after one warm-up')
    ap.add_argument('--image', type=Path, default=None, help='write the last image as a binary PPM')
    args = ap.parse_args(argv)
    tris, cam, settings, _, _ = load_snapshot(args.snapshot)
    lib = load_library()
    for size in args.sizes.split(','):
        w, h = map(int, size.split('x'))
        cam.aspect = w / h
        for bounces in map(int, args.bounces.split(',')):
            settings.maxBounces = bounces
            with Session(lib) as s:
                t0 = time.perf_counter()
                s.initialize(tris, w, h)
                init_ms = (time.perf_counter() - t0) * 1e3
                nodes, depth, build_ms = s.bvh_info()
                image, _ = s.render(cam, settings, args.backend)
                times = []
                for _ in range(args.passes):
                    image, ms = s.render(cam, settings, args.backend)
                    times.append(ms)
                print(json.dumps({'width': w, 'height': h, 'bounces': bounces, 'backend': args.backend,
                                  'triangles': len(tris), 'initialize_ms': init_ms,
                                  'bvh': {'nodes': nodes, 'depth': depth, 'build_ms': build_ms},
                                  'compute_ms': times, 'samples': s.sample_count()}), flush=True)
                if args.image:
                    rgb = image.reshape(h, w, 4)[::-1, :, :3]  # rows are stored bottom-up
                    args.image.write_bytes(b'P6\n%d %d\n255\n' % (w, h) + rgb.tobytes())


if __name__ == '__main__':
    main()
