"""Seeded synthetic scenes for the renderer's workloads and checks.

Every generator is deterministic for a given seed (numpy PCG64 streams) and
returns triangles as TRIANGLE_DTYPE records in the ABI layout, with colours
given sRGB-encoded as the ABI expects (the library linearises them at
RtInitialize, as the reference does at Native/renderer.cu:347).

Workloads:
  cornell_sphere()   - 10-triangle open box + 2-triangle ceiling light
                       (emission 15) around a level-4 icosphere (5,120
                       triangles, radius 0.3, +-2% seeded normal
                       displacement); per-object albedo uniform in
                       [0.2, 0.8]^3; 256x256, max depth 4.
  displaced_sphere_room() - the same kind of room (10 walls + 2 light
                       triangles) around a geodesic sphere with f = 224
                       subdivisions per icosahedron edge (1,003,520
                       triangles, the geodesic count closest to one million)
                       and +-5% radial noise; 1920x1080, max depth 3,
                       diffuse only.
  end_to_end_room()  - four smoothly displaced spheres (1,997,120 triangles)
                       in the same kind of room with a shaded uplight,
                       1920x1080, max depth 5, constant 0.1 environment.
Check scenes mirror the geometry categories of the reference's own
verifiers (Tools/verify_native.py, Tools/verify_bvh.cu).
"""
import math

import numpy as np

from native_api import Camera, Settings, Vector, TRIANGLE_DTYPE

_PHI = (1.0 + 5.0 ** 0.5) / 2.0
_ICO_V = np.array([(-1, _PHI, 0), (1, _PHI, 0), (-1, -_PHI, 0), (1, -_PHI, 0), (0, -1, _PHI), (0, 1, _PHI),
                   (0, -1, -_PHI), (0, 1, -_PHI), (_PHI, 0, -1), (_PHI, 0, 1), (-_PHI, 0, -1), (-_PHI, 0, 1)],
                  dtype=np.float64)
_ICO_F = np.array([(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
                   (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5),
                   (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)], dtype=np.int64)


def records(v0, v1, v2, color=(1, 1, 1), emission=0.0, one_sided=0, normals=None, mesh=0, specular_color=(1, 1, 1),
            smoothness=0.0, specular_probability=0.0):
    """Triangle records from corner arrays (N,3); edges are float32 differences."""
    v0 = np.asarray(v0, np.float32).reshape(-1, 3)
    v1 = np.asarray(v1, np.float32).reshape(-1, 3)
    v2 = np.asarray(v2, np.float32).reshape(-1, 3)
    n = len(v0)
    out = np.zeros(n, TRIANGLE_DTYPE)
    e1 = v1 - v0
    e2 = v2 - v0

    def put(field, arr):
        arr = np.broadcast_to(np.asarray(arr, np.float32), (n, 3))
        out[field]['x'], out[field]['y'], out[field]['z'] = arr[:, 0], arr[:, 1], arr[:, 2]

    put('origin', v0)
    put('edge1', e1)
    put('edge2', e2)
    put('color', color)
    put('specularColor', specular_color)
    if normals is None:
        fn = np.cross(e1.astype(np.float64), e2.astype(np.float64))
        fn /= np.maximum(np.linalg.norm(fn, axis=1, keepdims=True), 1e-30)
        normals = (fn, fn, fn)
    for k, name in enumerate(('normal0', 'normal1', 'normal2')):
        put(name, normals[k])
    out['emission'] = emission
    out['oneSided'] = one_sided
    out['mesh'] = mesh
    out['smoothness'] = smoothness
    out['specularProbability'] = specular_probability
    return out


def quad(x0, x1, y0, y1, z, **kwargs):
    """Two triangles covering [x0,x1]x[y0,y1] at depth z (Tools/verify_native.py:105-107)."""
    a, b, c, d = (x0, y0, z), (x1, y0, z), (x1, y1, z), (x0, y1, z)
    return records([a, a], [b, c], [c, d], **kwargs)


def box_quad(p, u, v, **kwargs):
    """Two triangles of the parallelogram p, p+u, p+u+v, p+v (winding p->p+u->p+u+v)."""
    p, u, v = (np.asarray(x, np.float64) for x in (p, u, v))
    return records([p, p], [p + u, p + u + v], [p + u + v, p + v], **kwargs)


def geodesic_sphere(subdivisions, radius, center, noise, rng, smooth=False):
    """Icosahedron with every face split into subdivisions^2 triangles, projected
    to a sphere; each distinct vertex is moved along its radius by a factor
    (1 + U(-noise, noise)) (independent per vertex), or with smooth=True by
    (1 + noise * n(p)) where n is a seeded sum of eight random plane waves
    scaled to [-1, 1]. Returns corner arrays and smooth vertex normals."""
    f = int(subdivisions)
    ico = _ICO_V / np.linalg.norm(_ICO_V, axis=1, keepdims=True)
    ii, jj = np.meshgrid(np.arange(f + 1), np.arange(f + 1), indexing='ij')
    keep = ii + jj <= f
    ii, jj = ii[keep], jj[keep]
    local = {(int(a), int(b)): k for k, (a, b) in enumerate(zip(ii, jj))}
    up_a = [(a, b) for a in range(f) for b in range(f - a)]
    dn_a = [(a, b) for a in range(f - 1) for b in range(f - 1 - a)]
    up = np.array([[local[(a, b)], local[(a + 1, b)], local[(a, b + 1)]] for a, b in up_a], np.int64)
    dn = np.array([[local[(a + 1, b)], local[(a + 1, b + 1)], local[(a, b + 1)]] for a, b in dn_a], np.int64)
    tri_local = np.concatenate([up, dn]) if len(dn) else up
    pts = []
    tris = []
    for face_index, (A, B, C) in enumerate(_ICO_F):
        a, b, c = ico[A], ico[B], ico[C]
        p = a[None, :] + (b - a)[None, :] * (ii[:, None] / f) + (c - a)[None, :] * (jj[:, None] / f)
        pts.append(p / np.linalg.norm(p, axis=1, keepdims=True))
        tris.append(tri_local + face_index * len(ii))
    pts = np.concatenate(pts)
    tris = np.concatenate(tris)
    keys = np.round(pts * (1 << 24)).astype(np.int64)
    _, first, inverse = np.unique(keys, axis=0, return_index=True, return_inverse=True)
    unique_pts = pts[first]
    if smooth:
        waves = rng.normal(size=(8, 3)) * rng.uniform(2.0, 6.0, (8, 1))
        phases = rng.uniform(0, 2 * np.pi, 8)
        field = np.sin(unique_pts @ waves.T + phases).sum(axis=1)
        scale_f = 1.0 + noise * field / max(np.abs(field).max(), 1e-12)
    else:
        scale_f = 1.0 + rng.uniform(-noise, noise, len(unique_pts))
    verts = unique_pts * (radius * scale_f)[:, None] + np.asarray(center, np.float64)[None, :]
    corners = inverse.reshape(-1)[tris]
    # Area-weighted vertex normals.
    v0, v1, v2 = verts[corners[:, 0]], verts[corners[:, 1]], verts[corners[:, 2]]
    fn = np.cross(v1 - v0, v2 - v0)
    vn = np.zeros_like(verts)
    for k in range(3):
        for axis in range(3):
            vn[:, axis] += np.bincount(corners[:, k], weights=fn[:, axis], minlength=len(verts))
    vn /= np.maximum(np.linalg.norm(vn, axis=1, keepdims=True), 1e-30)
    return v0, v1, v2, (vn[corners[:, 0]], vn[corners[:, 1]], vn[corners[:, 2]])


def open_box(lo, hi, colors, light_half, light_y, emission):
    """Five inward-facing walls (floor, ceiling, back, left, right: 10
    triangles, open at z = lo.z) and a 2-triangle ceiling light facing down."""
    x0, y0, z0 = lo
    x1, y1, z1 = hi
    walls = [
        box_quad((x0, y0, z0), (0, 0, z1 - z0), (x1 - x0, 0, 0), color=colors[0], mesh=1),   # floor, normal +y
        box_quad((x0, y1, z0), (x1 - x0, 0, 0), (0, 0, z1 - z0), color=colors[1], mesh=2),   # ceiling, normal -y
        box_quad((x0, y0, z1), (0, y1 - y0, 0), (x1 - x0, 0, 0), color=colors[2], mesh=3),   # back, normal -z
        box_quad((x0, y0, z0), (0, y1 - y0, 0), (0, 0, z1 - z0), color=colors[3], mesh=4),   # left, normal +x
        box_quad((x1, y0, z0), (0, 0, z1 - z0), (0, y1 - y0, 0), color=colors[4], mesh=5),   # right, normal -x
    ]
    cx, cz = 0.5 * (x0 + x1), 0.5 * (z0 + z1)
    h = light_half
    light = box_quad((cx - h, light_y, cz - h), (2 * h, 0, 0), (0, 0, 2 * h), color=(1, 1, 1), emission=emission,
                     mesh=6)
    return np.concatenate(walls + [light])


def camera(origin, target, tan_half_fov, aspect, up=(0.0, 1.0, 0.0)):
    o = np.asarray(origin, np.float64)
    fwd = np.asarray(target, np.float64) - o
    fwd /= np.linalg.norm(fwd)
    right = np.cross(np.asarray(up, np.float64), fwd)
    right /= np.linalg.norm(right)
    upv = np.cross(fwd, right)
    v = lambda a: Vector(*(float(x) for x in a))
    return Camera(v(o), v(right), v(upv), v(fwd), float(tan_half_fov), float(aspect), 1.0, 0)


def cornell_sphere(seed=7, width=256, height=256, bounces=4):
    """Config 'plain method, small': 5,132 triangles, 256x256, depth 4."""
    rng = np.random.Generator(np.random.PCG64(seed))
    colors = rng.uniform(0.2, 0.8, (6, 3))
    room = open_box((-1.0, 0.0, -1.0), (1.0, 2.0, 1.0), colors[:5], 0.25, 1.98, 15.0)
    v0, v1, v2, normals = geodesic_sphere(16, 0.3, (0.0, 0.55, 0.1), 0.02, rng)
    sphere = records(v0, v1, v2, color=colors[5], normals=normals, mesh=7)
    tris = np.concatenate([room, sphere])
    cam = camera((0.0, 1.0, -3.4), (0.0, 1.0, 0.0), math.tan(math.radians(19.0)), width / height)
    settings = Settings(bounces, 1.0, 0.0, 1.0, 0.0, 42, 1)
    return tris, cam, settings, width, height


def displaced_sphere_room(seed=11, width=1920, height=1080, bounces=3, subdivisions=224):
    """Config 'traversal and build at scale': 1,003,520 + 12 triangles, 1920x1080, depth 3."""
    rng = np.random.Generator(np.random.PCG64(seed))
    colors = rng.uniform(0.2, 0.8, (6, 3))
    room = open_box((-2.5, 0.0, -2.5), (2.5, 4.0, 2.5), colors[:5], 0.6, 3.98, 15.0)
    v0, v1, v2, normals = geodesic_sphere(subdivisions, 1.3, (0.0, 1.45, 0.3), 0.05, rng)
    sphere = records(v0, v1, v2, color=colors[5], normals=normals, mesh=7)
    tris = np.concatenate([room, sphere])
    cam = camera((0.0, 2.0, -7.0), (0.0, 1.6, 0.0), math.tan(math.radians(24.0)), width / height)
    settings = Settings(bounces, 1.0, 0.0, 1.0, 0.0, 42, 1)
    return tris, cam, settings, width, height


def end_to_end_room(seed=17, width=1920, height=1080, bounces=5, subdivisions=158, light_half=0.4, emission=40.0,
                    eye=(0.0, 2.0, -2.8), target=(0.0, 1.5, 2.0), half_fov_deg=38.0, light_y=3.5, shade=True,
                    exposure=1.5):
    """Config 'end-to-end equal quality': four displaced geodesic spheres of
    20 * 158^2 = 499,280 triangles each (smooth +-5% radial displacement,
    different radii and albedo) in the 12-triangle room with one quad light
    and a 2-triangle shade under it, so the room is lit through the ceiling
    (mostly indirect light): 1,997,134 triangles, 1920x1080, max depth 5,
    camera inside the room. The workload's constant 0.1 environment is set
    on the session with RtxSetEnvironment."""
    rng = np.random.Generator(np.random.PCG64(seed))
    colors = rng.uniform(0.2, 0.8, (9, 3))
    room = open_box((-3.0, 0.0, -3.0), (3.0, 4.0, 3.0), colors[:5], light_half, light_y, emission)
    parts = [room]
    if shade:
        # A diffuse shade just under the (two-sided) light: the room below is
        # lit only through the ceiling, by indirect light.
        h = 1.5 * light_half
        parts.append(box_quad((-h, light_y - 0.05, -h), (2 * h, 0, 0), (0, 0, 2 * h), color=(0.8, 0.8, 0.8), mesh=20))
    layout = (((-1.4, 0.8, 0.6), 0.8), ((1.3, 0.9, 1.0), 0.9), ((-0.2, 0.55, -1.0), 0.55), ((0.6, 2.2, 1.6), 0.6))
    for k, (center, radius) in enumerate(layout):
        v0, v1, v2, normals = geodesic_sphere(subdivisions, radius, center, 0.05, rng, smooth=True)
        parts.append(records(v0, v1, v2, color=colors[5 + k], normals=normals, mesh=8 + k))
    tris = np.concatenate(parts)
    cam = camera(eye, target, math.tan(math.radians(half_fov_deg)), width / height)
    settings = Settings(bounces, exposure, 0.0, 1.0, 0.0, 42, 1)
    return tris, cam, settings, width, height


def cuboid(center, size, yaw, **kwargs):
    """Closed box of 12 triangles with outward windings, rotated by yaw about +y."""
    cx, cy, cz = center
    sx, sy, sz = (0.5 * v for v in size)
    c, s = math.cos(yaw), math.sin(yaw)
    ex, ez = np.array([c, 0, -s]) * sx, np.array([s, 0, c]) * sz
    ey = np.array([0.0, sy, 0.0])
    o = np.array([cx, cy, cz], np.float64)
    faces = []
    for axis, pair in ((ex, (ey, ez)), (ey, (ez, ex)), (ez, (ex, ey))):
        for sign in (1, -1):
            u, v = (2 * e for e in (pair if sign > 0 else pair[::-1]))
            p = o + sign * axis - 0.5 * u - 0.5 * v
            faces.append(box_quad(p, u, v, **kwargs))
    return np.concatenate(faces)


def random_room(seed, width=256, height=256, triangles=None):
    """Training scene for the learned denoiser (not a benchmark workload):
    an open room of random size and wall colours lit by a ceiling quad
    light (random size, height and power, half the time under a diffuse
    shade, sometimes with a second small light), two to seven objects
    (faceted or smooth displaced spheres, boxes; a quarter of them glossy),
    a random camera inside the room, depth 3 to 6. With `triangles` given,
    the spheres share that budget (20 f^2 triangles each; at least one
    object is a sphere), so the room has about that many triangles.
    Returns the triangles, camera, settings and the environment (None: the
    sky gradient, else a constant radiance)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    hx, top, hz = rng.uniform(1.5, 4.0), rng.uniform(2.2, 4.5), rng.uniform(1.5, 4.0)
    colors = rng.uniform(0.08, 0.9, (5, 3))
    light_half = rng.uniform(0.15, 0.8)
    light_y = top - rng.uniform(0.02, 0.5)
    emission = float(rng.uniform(6.0, 60.0))
    parts = [open_box((-hx, 0.0, -hz), (hx, top, hz), colors, light_half, light_y, emission)]
    if rng.random() < 0.5:
        h = light_half * rng.uniform(1.2, 2.0)
        parts.append(box_quad((-h, light_y - rng.uniform(0.03, 0.3), -h), (2 * h, 0, 0), (0, 0, 2 * h),
                              color=rng.uniform(0.3, 0.9, 3), mesh=20))
    if rng.random() < 0.3:
        q = rng.uniform(0.05, 0.25)
        lx, lz = rng.uniform(-hx + q, hx - q), rng.uniform(-hz + q, hz - q)
        parts.append(box_quad((lx - q, top - 0.01, lz - q), (2 * q, 0, 0), (0, 0, 2 * q), emission=emission,
                              mesh=21))
    objects = int(rng.integers(2, 8))
    kinds = rng.random(objects) < 0.6  # True: a sphere
    if triangles is not None and not kinds.any():
        kinds[0] = True
    shares = None
    if triangles is not None:
        boxes = int((~kinds).sum())
        budget = max(triangles - sum(len(p) for p in parts) - 12 * boxes, 20 * int(kinds.sum()))
        shares = iter(rng.dirichlet(np.ones(int(kinds.sum()))) * budget)
    for k in range(objects):
        size = rng.uniform(0.2, 0.35 * min(hx, hz, top))
        center = (rng.uniform(-hx + size, hx - size), rng.uniform(size, top - size), rng.uniform(-hz + size, hz - size))
        material = dict(color=rng.uniform(0.05, 0.95, 3), mesh=30 + k)
        if rng.random() < 0.25:
            material.update(smoothness=float(rng.uniform(0.6, 1.0)), specular_probability=float(rng.uniform(0.1, 0.6)),
                            specular_color=rng.uniform(0.6, 1.0, 3))
        if kinds[k]:
            f = int(rng.integers(3, 40)) if shares is None else max(1, int(round(math.sqrt(next(shares) / 20.0))))
            v0, v1, v2, normals = geodesic_sphere(f, size, center, rng.uniform(0, 0.1), rng,
                                                  smooth=bool(rng.random() < 0.5))
            parts.append(records(v0, v1, v2, normals=normals if rng.random() < 0.7 else None, **material))
        else:
            dims = rng.uniform(0.5, 1.8, 3) * size
            center = (center[0], 0.5 * dims[1] if rng.random() < 0.6 else center[1], center[2])
            parts.append(cuboid(center, dims, rng.uniform(0, math.pi), **material))
    tris = np.concatenate(parts)
    eye = (rng.uniform(-0.7, 0.7) * hx, rng.uniform(0.4, top - 0.3), -hz + rng.uniform(0.1, 0.6) * hz)
    target = (rng.uniform(-0.6, 0.6) * hx, rng.uniform(0.2, 0.8) * top, rng.uniform(0.0, 0.9) * hz)
    cam = camera(eye, target, math.tan(math.radians(rng.uniform(22.0, 45.0))), width / height)
    settings = Settings(int(rng.integers(3, 7)), float(rng.uniform(0.7, 2.0)), 0.0, 1.0,
                        float(rng.uniform(0.0, 1.0)), 42, 1)
    environment = None if rng.random() < 0.4 else float(rng.uniform(0.0, 0.3))
    return tris, cam, settings, environment


def random_scene(seed, triangles):
    """A room (12 triangles with its light) holding displaced geodesic spheres
    and boxes with random transforms, about `triangles` triangles in all:
    one to six spheres share the budget (20 f^2 triangles each), plus up to
    six boxes of 12."""
    rng = np.random.Generator(np.random.PCG64(seed))
    colors = rng.uniform(0.2, 0.8, (5, 3))
    room = open_box((-4.0, 0.0, -4.0), (4.0, 4.0, 4.0), colors, rng.uniform(0.3, 0.8), 3.98, rng.uniform(10.0, 30.0))
    parts = [room]
    boxes = int(rng.integers(0, 7))
    for k in range(boxes):
        size = rng.uniform(0.3, 1.2, 3)
        center = (rng.uniform(-3.0, 3.0), rng.uniform(0.2, 3.0), rng.uniform(-3.0, 3.0))
        parts.append(cuboid(center, size, rng.uniform(0, math.pi), color=rng.uniform(0.1, 0.9, 3), mesh=20 + k))
    budget = max(triangles - 12 - 12 * boxes, 20)
    spheres = int(rng.integers(1, 7))
    shares = rng.dirichlet(np.ones(spheres)) * budget
    for k, share in enumerate(shares):
        f = max(1, int(round(math.sqrt(share / 20.0))))
        radius = rng.uniform(0.3, 1.3)
        center = (rng.uniform(-2.5, 2.5), rng.uniform(radius, 4.0 - radius), rng.uniform(-2.5, 2.5))
        v0, v1, v2, normals = geodesic_sphere(f, radius, center, rng.uniform(0.0, 0.08), rng,
                                              smooth=bool(rng.random() < 0.5))
        # Random anisotropic scale and rotation about the centre.
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        w, x, y, z = q
        rot = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])
        m = rot * rng.uniform(0.7, 1.3, 3)[None, :]
        c = np.asarray(center)
        v0, v1, v2 = ((v - c) @ m.T + c for v in (v0, v1, v2))
        inv_t = np.linalg.inv(m).T
        normals = tuple(n @ inv_t.T / np.linalg.norm(n @ inv_t.T, axis=1, keepdims=True) for n in normals)
        parts.append(records(v0, v1, v2, color=rng.uniform(0.1, 0.9, 3), normals=normals, mesh=40 + k))
    return np.concatenate(parts)


def batch_workload(seed=23, scene_count=8, cameras=64, low=10_000, high=2_000_000,
                   resolutions=(256, 512, 1024)):
    """Config 'batched multi-scene tracing': scene_count scenes (random_scene)
    with triangle counts log-uniform in [low, high], `cameras` cameras spread
    evenly over them, each at a square resolution drawn uniformly from
    `resolutions`, looking into the room from random points. Returns the
    scenes, the views as (scene, camera, width, height) and the settings
    (depth 4, 8 paths per pixel)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    counts = np.exp(rng.uniform(math.log(low), math.log(high), scene_count)).astype(int)
    scene_list = [random_scene(seed * 1000 + k, int(t)) for k, t in enumerate(counts)]
    views = []
    for i in range(cameras):
        k = i % scene_count
        size = int(rng.choice(resolutions))
        eye = (rng.uniform(-3.0, 3.0), rng.uniform(0.8, 3.2), rng.uniform(-3.8, -2.5))
        target = (rng.uniform(-1.5, 1.5), rng.uniform(0.5, 2.5), rng.uniform(-1.0, 2.5))
        views.append((k, camera(eye, target, math.tan(math.radians(rng.uniform(25.0, 45.0))), 1.0), size, size))
    settings = Settings(4, 1.0, 0.0, 1.0, 0.5, 42, 8)
    return scene_list, views, settings


# ---- check geometry, after the categories of Tools/verify_bvh.cu:115-139 ----

def _tri(a, b, c, one_sided=0):
    return records([a], [b], [c], color=(1, 1, 1), one_sided=one_sided)


def edge_case_triangles():
    """Shared edges, a one-sided face, a duplicate and a zero-area triangle."""
    t0 = _tri((-1, -1, 0), (1, -1, 0), (1, 1, 0))
    t1 = _tri((-1, -1, 0), (1, 1, 0), (-1, 1, 0), one_sided=1)
    zero = _tri((0, 0, 0), (0, 0, 0), (0, 0, 0))
    return np.concatenate([t0, t1, t0, zero])


def scattered_triangles(rng, count=3000):
    a = rng.uniform(-10, 10, (count, 3)).astype(np.float32)
    b = a + np.array([.2, .3, 0], np.float32)
    c = a + np.array([0, .1, .4], np.float32)
    out = records(a, b, c, color=(1, 1, 1))
    out['oneSided'] = np.arange(count) % 2
    return out


def overlapping_triangles(count=256):
    return np.concatenate([_tri((-1, -1, 0), (1, -1, 0), (1, 1, 0))] * count)


def exponential_triangles():
    xs = []
    for i in range(200):
        x = 1.5 ** i
        if not np.isfinite(np.float32(x)):
            break
        xs.append(x)
    xs = np.array(xs, np.float64)
    a = np.stack([xs, -np.ones_like(xs), np.zeros_like(xs)], 1)
    b = np.stack([xs, np.ones_like(xs), np.zeros_like(xs)], 1)
    c = np.stack([xs, np.zeros_like(xs), np.ones_like(xs)], 1)
    return records(a, b, c, color=(1, 1, 1))


def random_rays(rng, count=12000):
    """Rays like Tools/verify_bvh.cu:105-114: random origins in [-10,10]^3, unit
    directions with every 4th axis-aligned and every 5th carrying a 1e-40
    (subnormal) x component; odd rays unbounded (1e30), even ones finite."""
    from native_api import QUERY_DTYPE
    q = np.zeros(count, QUERY_DTYPE)
    o = rng.uniform(-10, 10, (count, 3)).astype(np.float32)
    d = rng.uniform(-10, 10, (count, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    d = d.astype(np.float32)
    i = np.arange(count)
    axis = i % 3
    aligned = i % 4 == 0
    d[aligned] = 0
    d[aligned, axis[aligned]] = 1
    d[i % 5 == 0, 0] = np.float32(1e-40)
    limit = np.where(i % 2 == 1, np.float32(1e30), np.abs(rng.uniform(-10, 10, count)).astype(np.float32))
    for k, ax in enumerate('xyz'):
        q['origin'][ax] = o[:, k]
        q['direction'][ax] = d[:, k]
    q['limit'] = limit
    return q


def edge_grid_rays():
    """Axis-parallel rays from grid points on the test faces (Tools/verify_bvh.cu:120-122)."""
    from native_api import QUERY_DTYPE
    rows = []
    for z in (-1.0, 0.0, 1.0):
        for x in (-1.0, 0.0, 1.0):
            for d in ((0, 0, 1), (0, 0, -1), (0, 1, 0), (1e-40, 0, 1)):
                for limit in (.5, 1.0, 2.0, 1e30):
                    rows.append(((x, x, z), d, limit))
    q = np.zeros(len(rows), QUERY_DTYPE)
    for k, (o, d, limit) in enumerate(rows):
        q[k]['origin'] = tuple(np.float32(v) for v in o)
        q[k]['direction'] = tuple(np.float32(v) for v in d)
        q[k]['limit'] = np.float32(limit)
    return q


def concat_queries(*parts):
    return np.concatenate(parts)
