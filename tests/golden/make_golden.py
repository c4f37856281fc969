"""Generates the golden fixtures in this directory from the reference renderer itself.

Run from the repository root where the reference sources exist:
    make -C oracle            # builds oracle/_ref/libref.so from Native/renderer.cu
    python tests/golden/make_golden.py [snapshot]
Every array here is produced by the reference's own host code (BvhBuilder,
collision, PathSampler, pixel) through oracle/_ref/libref.so, on the seeded
scenes of custom-ray-tracing-shader_b200/scenes.py. The tests compare the
oracle and the CUDA library against these files, so they also run where the
reference is absent.
"""
import hashlib
import os
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / 'custom-ray-tracing-shader_b200'))
sys.path.insert(0, str(ROOT / 'oracle'))

import scenes  # noqa: E402
from oracle_api import Reference  # noqa: E402

OUT = Path(__file__).resolve().parent
# Where the reference's sources lie (the REFERENCE_ROOT environment variable);
# tests that read the reference's own files take it from here and skip when it
# is absent.
REFERENCE_ROOT = Path(os.environ.get('REFERENCE_ROOT', '/root/reference'))


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def geometry_sets():
    rng = np.random.Generator(np.random.PCG64(719393))
    rays = np.concatenate([scenes.random_rays(rng, 12000), scenes.edge_grid_rays()])
    cornell = scenes.cornell_sphere()[0]
    return rays, {
        'edges': scenes.edge_case_triangles(),
        'scatter': scenes.scattered_triangles(rng),
        'overlap': scenes.overlapping_triangles(),
        'exponential': scenes.exponential_triangles(),
        'cornell': cornell,
    }


def main():
    ref = Reference()
    # Sampler: the reference's own check set (Tools/verify_sampling.cu:26-39) as a
    # hash, plus a stored slice.
    i = np.arange(4096)
    full = ref.sobol(i // 1024, i % 1024, np.full(4096, 42))
    pix = np.array([0, 177, 4095, 123456], np.uint32).repeat(64)
    smp = np.tile(np.arange(64, dtype=np.uint32), 4) * 37 + 5
    seeds = np.where(np.arange(256) % 2, 1234, 42).astype(np.uint32)
    part = ref.sobol(pix, smp, seeds)
    np.savez_compressed(OUT / 'sobol.npz', full_sha256=sha(full), pixel=pix, sample=smp, seed=seeds, values=part)

    # BVH and ray queries.
    rays, sets = geometry_sets()
    bvh = {}
    for name, tris in sets.items():
        sc = ref.scene(tris)
        nodes, order = sc.nodes(), sc.order()
        closest = ref.query(sc, rays, False)
        anyhit = ref.query(sc, rays, True)
        bvh[name] = dict(triangles_sha256=sha(tris), node_count=sc.node_count, depth=sc.depth,
                         nodes_sha256=sha(nodes), order_sha256=sha(order))
        np.savez_compressed(OUT / f'bvh_{name}.npz', nodes=nodes, order=order, closest=closest,
                            any_index=anyhit['index'], triangles_sha256=sha(tris), rays_sha256=sha(rays),
                            depth=sc.depth)
        sc.close()

    # Renders: two progressive passes of the small Cornell scene, and one pass
    # with every camera/material feature the integrator has.
    tris, cam, settings, w, h = scenes.cornell_sphere()
    sc = ref.scene(tris)
    W, H = 48, 40
    cam.aspect = W / H
    settings.raysPerPixel = 3
    sums1, rgba1 = ref.render(sc, cam, settings, W, H, sample=0)
    sums2, rgba2 = ref.render(sc, cam, settings, W, H, sample=3, sums=sums1.copy())
    np.savez_compressed(OUT / 'render_cornell.npz', sums1=sums1, rgba1=rgba1, sums2=sums2, rgba2=rgba2, width=W,
                        height=H, rays_per_pixel=3, triangles_sha256=sha(tris))
    sc.close()
    feat = feature_scene()
    sc = ref.scene(feat['triangles'])
    out = {}
    for key, (cam, st) in feat['views'].items():
        s, rgba = ref.render(sc, cam, st, feat['width'], feat['height'], sample=0)
        out[key + '_sums'] = s
        out[key + '_rgba'] = rgba
    np.savez_compressed(OUT / 'render_features.npz', width=feat['width'], height=feat['height'],
                        triangles_sha256=sha(feat['triangles']), **out)
    print('golden fixtures written to', OUT)


def snapshot_fixture(reference_root=REFERENCE_ROOT):
    """The reference's Suzanne-room snapshot (Benchmarks/embree/scene.json,
    982 triangles) as scene_io loads it, with the size, depth and node-array
    hash of the reference builder's BVH for it."""
    import scene_io
    tris, cam, st, w, h = scene_io.load_snapshot(reference_root / 'Benchmarks/embree/scene.json')
    sc = Reference().scene(tris)
    np.savez_compressed(OUT / 'snapshot_room982.npz', triangles=tris, camera=np.frombuffer(bytes(cam), np.uint8),
                        settings=np.frombuffer(bytes(st), np.uint8), width=w, height=h, node_count=sc.node_count,
                        depth=sc.depth, nodes_sha256=sha(sc.nodes()), order_sha256=sha(sc.order()))
    sc.close()


def feature_scene():
    """Mirror, glossy Phong, one-sided faces, sky light, depth of field,
    orthographic and Russian roulette (depth 8) in one small scene."""
    from native_api import Settings
    rng = np.random.Generator(np.random.PCG64(99))
    colors = rng.uniform(0.2, 0.8, (6, 3))
    room = scenes.open_box((-1.0, 0.0, -1.0), (1.0, 2.0, 1.0), colors[:5], 0.3, 1.98, 12.0)
    v0, v1, v2, nrm = scenes.geodesic_sphere(4, 0.35, (-0.4, 0.4, 0.2), 0.02, rng)
    glossy = scenes.records(v0, v1, v2, color=colors[5], normals=nrm, mesh=8, specular_color=(.9, .8, .7),
                            smoothness=.8, specular_probability=.5)
    v0, v1, v2, nrm = scenes.geodesic_sphere(4, 0.3, (0.45, 0.35, -0.1), 0.0, rng)
    mirror = scenes.records(v0, v1, v2, color=(.5, .5, .5), normals=nrm, mesh=9, specular_color=(.95, .95, .95),
                            smoothness=1.0, specular_probability=1.0)
    cull = scenes.quad(-0.2, 0.2, 1.2, 1.6, 0.5, color=(0.3, 0.9, 0.3))
    cull['oneSided'] = 1
    tris = np.concatenate([room, glossy, mirror, cull])
    W, H = 40, 32
    base = scenes.camera((0.1, 1.0, -3.0), (0.0, 0.8, 0.0), 0.4, W / H)
    views = {}
    views['persp'] = (base, Settings(8, 1.0, 0.0, 1.0, 0.6, 1234, 4))
    dof = scenes.camera((0.1, 1.0, -3.0), (0.0, 0.8, 0.0), 0.4, W / H)
    views['dof'] = (dof, Settings(5, 1.3, 0.15, 3.0, 0.3, 42, 2))
    ortho = scenes.camera((0.0, 1.0, -3.0), (0.0, 1.0, 0.0), 0.4, W / H)
    ortho.orthographic = 1
    ortho.orthographicSize = 1.1
    views['ortho'] = (ortho, Settings(4, 0.8, 0.0, 1.0, 0.0, 7, 2))
    return dict(triangles=tris, views=views, width=W, height=H)


if __name__ == '__main__':
    if sys.argv[1:] == ['snapshot']:
        snapshot_fixture()   # only the snapshot fixture
    else:
        main()
        snapshot_fixture()
