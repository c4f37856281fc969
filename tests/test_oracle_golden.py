"""The oracle against fixtures produced by the reference itself (tests/golden),
and against the reference's own known answers. CPU only."""

import numpy as np
import pytest

import scenes
from conftest import golden, sha256
from native_api import Camera, Settings, Vector

SETS = ('edges', 'scatter', 'overlap', 'exponential', 'cornell')


def _sets():
    rng = np.random.Generator(np.random.PCG64(719393))
    rays = np.concatenate([scenes.random_rays(rng, 12000), scenes.edge_grid_rays()])
    return rays, {
        'edges': scenes.edge_case_triangles(),
        'scatter': scenes.scattered_triangles(rng),
        'overlap': scenes.overlapping_triangles(),
        'exponential': scenes.exponential_triangles(),
        'cornell': scenes.cornell_sphere()[0],
    }


RAYS, GEOMETRY = _sets()


def test_sobol_matches_reference_values(oracle):
    g = golden('sobol.npz')
    i = np.arange(4096)
    full = oracle.sobol(i // 1024, i % 1024, np.full(4096, 42))  # Tools/verify_sampling.cu:26-39
    assert sha256(full) == str(g['full_sha256'])
    part = oracle.sobol(g['pixel'], g['sample'], g['seed'])
    assert part.tobytes() == g['values'].tobytes()


def test_sobol_stratification(oracle):
    """Tools/verify_sampling.cu:16-25: every dimension in [0,1) and perfectly
    stratified over the first 16/64/256 samples, pixels {0,177} x seeds {42,1234}."""
    for pixel in (0, 177):
        for seed in (42, 1234):
            v = oracle.sobol(np.full(256, pixel), np.arange(256), np.full(256, seed))
            assert (v >= 0).all() and (v < 1).all()
            for count in (16, 64, 256):
                strata = np.floor(v[:count] * count).astype(np.int64)
                for d in range(v.shape[1]):
                    assert len(np.unique(strata[:, d])) == count, (pixel, seed, count, d)


@pytest.mark.parametrize('name', SETS)
def test_bvh_matches_reference(oracle, name):
    g = golden(f'bvh_{name}.npz')
    tris = GEOMETRY[name]
    assert sha256(tris) == str(g['triangles_sha256']), 'scene generator drifted'
    sc = oracle.scene(tris)
    assert sc.nodes().tobytes() == g['nodes'].tobytes()
    assert (sc.order() == g['order']).all()
    assert sc.depth == int(g['depth'])


@pytest.mark.parametrize('name', SETS)
def test_queries_match_reference(oracle, name):
    g = golden(f'bvh_{name}.npz')
    assert sha256(RAYS) == str(g['rays_sha256'])
    sc = oracle.scene(GEOMETRY[name])
    closest, _ = oracle.query(sc, RAYS, False)
    assert closest.tobytes() == g['closest'].tobytes()
    anyhit, _ = oracle.query(sc, RAYS, True)
    assert ((anyhit['index'] >= 0) == (g['any_index'] >= 0)).all()


@pytest.mark.parametrize('name', SETS)
def test_bvh_queries_equal_brute_force(oracle, name):
    """Tools/verify_bvh.cu:20-25: the BVH answers as the plain triangle loop does."""
    sc = oracle.scene(GEOMETRY[name])
    for any_hit in (False, True):
        fast, _ = oracle.query(sc, RAYS, any_hit)
        slow, _ = oracle.query(sc, RAYS, any_hit, brute=True)
        if any_hit:
            assert ((fast['index'] >= 0) == (slow['index'] >= 0)).all()
        else:
            assert (fast['index'] == slow['index']).all()
            hit = fast['index'] >= 0
            assert np.allclose(fast['distance'][hit], slow['distance'][hit], rtol=1e-5, atol=1e-5)


def test_bvh_structure(oracle):
    """Tools/verify_bvh.cu:42-66: every node reached once, every triangle in
    exactly one leaf, children inside parents, depth <= 32."""
    for name, tris in GEOMETRY.items():
        sc = oracle.scene(tris)
        nodes, order = sc.nodes(), sc.order()
        seen = np.zeros(len(nodes), np.int64)
        covered = np.zeros(len(tris), np.int64)
        stack = [(0, 0)]
        while stack:
            i, depth = stack.pop()
            seen[i] += 1
            assert depth <= 32
            n = nodes[i]
            if n['count'] > 0:
                covered[order[n['first']:n['first'] + n['count']]] += 1
            else:
                for ch in (n['first'], n['first'] + 1):
                    for ax in 'xyz':
                        assert nodes[ch]['low'][ax] >= n['low'][ax] and nodes[ch]['high'][ax] <= n['high'][ax]
                    stack.append((ch, depth + 1))
        assert (seen == 1).all() and (covered == 1).all(), name


def test_render_matches_reference(oracle):
    g = golden('render_cornell.npz')
    tris, cam, st, _, _ = scenes.cornell_sphere()
    assert sha256(tris) == str(g['triangles_sha256'])
    W, H = int(g['width']), int(g['height'])
    cam.aspect = W / H
    st.raysPerPixel = int(g['rays_per_pixel'])
    sc = oracle.scene(tris)
    s1, rgba1, _ = oracle.render(sc, cam, st, W, H)
    assert s1.tobytes() == g['sums1'].tobytes() and rgba1.tobytes() == g['rgba1'].tobytes()
    s2, rgba2, _ = oracle.render(sc, cam, st, W, H, sample=3, sums=s1.copy())
    assert s2.tobytes() == g['sums2'].tobytes() and rgba2.tobytes() == g['rgba2'].tobytes()


def test_render_features_match_reference(oracle):
    import make_golden
    g = golden('render_features.npz')
    feat = make_golden.feature_scene()
    assert sha256(feat['triangles']) == str(g['triangles_sha256'])
    sc = oracle.scene(feat['triangles'])
    for key, (cam, st) in feat['views'].items():
        s, rgba, _ = oracle.render(sc, cam, st, feat['width'], feat['height'])
        assert s.tobytes() == g[key + '_sums'].tobytes(), key
        assert rgba.tobytes() == g[key + '_rgba'].tobytes(), key
        assert rgba.reshape(-1, 4)[:, :3].max() > 0, key


def _centre(rgba, w, h):
    o = ((h // 2) * w + w // 2) * 4
    return tuple(int(v) for v in rgba[o:o + 4])


def test_known_answers(oracle):
    """Tools/verify_native.py:123-134: a frontal emissive red quad reads
    (208,0,0,255) at the centre; culled from behind when one-sided."""
    lit = Settings(8, 1, 0, 3, 0, 42, 1)
    for w, h in ((37, 25), (17, 19)):
        cam = Camera(Vector(0, 0, -2), Vector(1, 0, 0), Vector(0, 1, 0), Vector(0, 0, 1), .5, w / h, 1, 0)
        for sided, inside, expected in ((0, False, (208, 0, 0, 255)), (1, False, (0, 0, 0, 255)),
                                        (1, True, (208, 0, 0, 255))):
            red = scenes.quad(-1, 1, -1, 1, 0, color=(1, 0, 0), emission=1)
            red['oneSided'] = sided
            cam.origin.z = 2 if inside else -2
            cam.forward.z = -1 if inside else 1
            sc = oracle.scene(red)
            sums = None
            for k in range(4):
                sums, rgba, _ = oracle.render(sc, cam, lit, w, h, sample=k, sums=sums)
            assert _centre(rgba, w, h) == expected
            assert (rgba[3::4] == 255).all()


from make_golden import REFERENCE_ROOT  # noqa: E402
REFERENCE_SCENE = REFERENCE_ROOT / 'Benchmarks/embree/scene.json'


@pytest.mark.skipif(not REFERENCE_SCENE.exists(), reason='reference scene snapshots absent on this machine')
def test_published_bvh_counts(oracle):
    """The reference's recorded BVH for its 982-triangle room: 659 nodes, depth
    17 (Benchmarks/embree/native.json:128-129)."""
    import json
    from native_api import Triangle, unpack, triangles_array
    scene = json.loads(REFERENCE_SCENE.read_text())
    tris = (Triangle * len(scene['triangles']))(*(unpack(Triangle, t) for t in scene['triangles']))
    sc = oracle.scene(triangles_array(tris))
    assert (sc.node_count, sc.depth) == (659, 17)
