"""Scene loader (scene_io.py): snapshot files, OBJ and mesh JSON, and the
Triangle records of an object, against the reference's own files where they
exist (its two scene snapshots, the Suzanne mesh and the dragon OBJ) and
against hand-made files everywhere."""
import importlib.util

import numpy as np
import pytest

import scene_io
import scenes

from make_golden import REFERENCE_ROOT as REFERENCE  # noqa: E402
ROOM_SNAPSHOT = REFERENCE / 'Benchmarks/embree/scene.json'           # 982 triangles: Suzanne room
DRAGON_SNAPSHOT = REFERENCE / 'Benchmarks/quality/dragon/scene.json.gz'  # 87,165 triangles
SUZANNE = REFERENCE / 'UnityRayTracer/Assets/RayTracing/Models/Suzanne.json'
DRAGON_OBJ = REFERENCE / 'UnityRayTracer/Assets/RayTracing/Models/Dragon_80K.obj'
needs_reference = pytest.mark.skipif(not ROOM_SNAPSHOT.exists(), reason='reference files absent on this machine')


def vec(records, field):
    return np.stack([records[field][k] for k in 'xyz'], 1).astype(np.float64)


def test_snapshot_round_trip(tmp_path):
    tris, cam, st, w, h = scenes.cornell_sphere()
    cam.orthographic, cam.orthographicSize = 1, 2.5
    st.seed = 4000000000
    for name in ('scene.json', 'scene.json.gz'):
        scene_io.save_snapshot(tmp_path / name, tris, cam, st, w, h)
        t2, c2, s2, w2, h2 = scene_io.load_snapshot(tmp_path / name)
        assert t2.tobytes() == np.ascontiguousarray(tris).tobytes()
        assert bytes(c2) == bytes(cam) and bytes(s2) == bytes(st) and (w2, h2) == (w, h)
    assert (tmp_path / 'scene.json.gz').stat().st_size < (tmp_path / 'scene.json').stat().st_size


def test_obj_parsing(tmp_path):
    (tmp_path / 'm.obj').write_text('\n'.join([
        '# comment', 'o thing', 'v 0 0 0', 'v 1 0 0', 'v 1 1 0', 'v 0 1 0', 'vt 0 0', 'vn 0 0 1', 'vn 0 0 -1',
        'f 1/1/1 2/1/1 3/1/1 4/1/1',      # quad: a fan of two triangles
        'f -4//2 -2//2 -1//2', 's off', '']))
    v, idx, n = scene_io.load_obj(tmp_path / 'm.obj')
    assert v.shape == (4, 3) and idx.tolist() == [[0, 1, 2], [0, 2, 3], [0, 2, 3]]
    assert n.shape == (3, 3, 3) and n[0, 0].tolist() == [0, 0, 1] and n[2, 1].tolist() == [0, 0, -1]
    vu, iu, nu = scene_io.load_obj(tmp_path / 'm.obj', unity_axes=True)
    assert vu[1].tolist() == [-1, 0, 0] and iu[0].tolist() == [0, 2, 1]
    (tmp_path / 'p.obj').write_text('v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\n')
    _, idx, n = scene_io.load_obj(tmp_path / 'p.obj')
    assert idx.tolist() == [[0, 1, 2]] and n is None


def test_object_triangles_rules():
    """Transform order (scale, rotate, translate), face normals when the mesh
    has none, degenerate triangles dropped (RayTraceSession.cs:114-115),
    material fields copied."""
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [2, 0, 0], [0, 0, 1e-7]], np.float64)
    idx = np.array([[0, 1, 2], [0, 1, 3], [0, 1, 4]])  # a triangle, a line, a sliver below 1e-5
    q = scene_io.euler_quaternion(0, 90, 0)
    t = scene_io.object_triangles(v, idx, position=(1, 2, 3), rotation=q, scale=2.0, color=(.5, .25, 1),
                                  emission=3.0, one_sided=True, mesh=7, smoothness=.5, specular_probability=.25)
    assert len(t) == 1
    assert np.allclose(vec(t, 'origin')[0], (1, 2, 3)) and np.allclose(vec(t, 'edge1')[0], (0, 0, -2), atol=1e-6)
    assert np.allclose(vec(t, 'edge2')[0], (0, 2, 0), atol=1e-6)
    assert np.allclose(vec(t, 'normal0')[0], np.cross((0, 0, -1), (0, 1, 0)), atol=1e-6)
    assert t['oneSided'][0] == 1 and t['mesh'][0] == 7 and t['emission'][0] == 3.0
    assert np.allclose(vec(t, 'color')[0], (.5, .25, 1))
    # Unity's Quaternion.Euler applies z, then x, then y.
    qz, qx = scene_io.euler_quaternion(0, 0, 90), scene_io.euler_quaternion(90, 0, 0)
    both = scene_io.quaternion_matrix(*scene_io.euler_quaternion(90, 0, 90))
    assert np.allclose(both, scene_io.quaternion_matrix(*qx) @ scene_io.quaternion_matrix(*qz))


@needs_reference
@pytest.mark.parametrize('path', [ROOM_SNAPSHOT, DRAGON_SNAPSHOT], ids=['room982', 'dragon87165'])
def test_snapshots_load_like_the_reference_tools(path):
    """The same bytes as Tools/native_api.py's unpack (used by the reference's
    benchmark and quality tools) for triangles, camera and settings."""
    spec = importlib.util.spec_from_file_location('reference_native_api', REFERENCE / 'Tools/native_api.py')
    ref = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(ref)
    raw = scene_io._read_json(path)
    expect = (ref.Triangle * len(raw['triangles']))(*(ref.unpack(ref.Triangle, t) for t in raw['triangles']))
    tris, cam, st, w, h = scene_io.load_snapshot(path)
    assert tris.tobytes() == bytes(expect)
    assert bytes(cam) == bytes(ref.unpack(ref.Camera, raw['camera']))
    assert bytes(st) == bytes(ref.unpack(ref.Settings, raw['settings']))
    assert (w, h) == (raw['width'], raw['height'])


@needs_reference
def test_suzanne_object_matches_the_unity_snapshot():
    """Suzanne.json with area-weighted normals, yawed -15 degrees
    (Editor/FirstSceneBuilder.cs:26,50), gives the snapshot's 968 triangles
    within 2 float32 ulps; the position is the snapshot's own."""
    tris, *_ = scene_io.load_snapshot(ROOM_SNAPSHOT)
    monkey = tris[tris['mesh'] == 55492]
    v, idx = scene_io.load_mesh_json(SUZANNE)
    q = scene_io.euler_quaternion(0, -15, 0)
    r = scene_io.quaternion_matrix(*q)
    position = (vec(monkey, 'origin') - v[idx[:, 0]] @ r.T).mean(axis=0)
    mine = scene_io.object_triangles(v, idx, scene_io.recalculate_normals(v, idx), position=position, rotation=q)
    assert len(mine) == len(monkey) == 968
    for field in ('origin', 'edge1', 'edge2', 'normal0', 'normal1', 'normal2'):
        assert np.abs(vec(mine, field) - vec(monkey, field)).max() < 2.5e-7, field


@needs_reference
def test_dragon_obj_matches_the_unity_snapshot():
    """Dragon_80K.obj under Unity's axes with the dragon room's transform
    (Editor/DemoSceneBuilder.cs:124-126): the same 86,961 triangles (the
    degenerate-triangle rule drops the same 169) with the same corners in
    the same order and winding, within 2 ulps. Unity's importer reorders the
    triangles, so they are paired by centroid (a one-to-one pairing). Normals
    are the file's; the importer merges nearly equal vertex normals, so they
    agree to a dot product above 0.998."""
    from scipy.spatial import cKDTree
    tris, *_ = scene_io.load_snapshot(DRAGON_SNAPSHOT)
    dragon = tris[tris['mesh'] == 49556]
    v, idx, n = scene_io.load_obj(DRAGON_OBJ, unity_axes=True)
    assert len(idx) == 87130
    mine = scene_io.object_triangles(v, idx, n, position=(-.04, 1.43, -.02), rotation=(0, .48016095, 0, .8771804),
                                     scale=5.350002)
    assert len(mine) == len(dragon) == 86961

    def centroids(t):
        return vec(t, 'origin') + (vec(t, 'edge1') + vec(t, 'edge2')) / 3
    _, pair = cKDTree(centroids(mine)).query(centroids(dragon))
    assert len(np.unique(pair)) == len(pair)
    mine = mine[pair]
    for field in ('origin', 'edge1', 'edge2'):
        assert np.abs(vec(mine, field) - vec(dragon, field)).max() < 1e-6, field
    for field in ('normal0', 'normal1', 'normal2'):
        assert (np.sum(vec(mine, field) * vec(dragon, field), axis=1) > 0.998).all(), field


@needs_reference
@pytest.mark.parametrize('path,nodes,depth', [(ROOM_SNAPSHOT, 659, 17), (DRAGON_SNAPSHOT, 57839, 22)],
                         ids=['room982', 'dragon87165'])
def test_snapshot_bvh_counts_match_published(oracle, path, nodes, depth):
    """The reference's published BVH sizes for its snapshots
    (Benchmarks/embree/native.json:128-129, demos-native.json:264-265)."""
    tris, *_ = scene_io.load_snapshot(path)
    sc = oracle.scene(tris)
    try:
        assert (sc.node_count, sc.depth) == (nodes, depth)
    finally:
        sc.close()


def test_snapshot_fixture_pins_the_oracle(oracle):
    """The committed fixture of the reference's 982-triangle room: the
    oracle's builder gives the reference builder's node array for it."""
    from conftest import golden, sha256
    g = golden('snapshot_room982.npz')
    sc = oracle.scene(g['triangles'])
    try:
        assert (sc.node_count, sc.depth) == (int(g['node_count']), int(g['depth'])) == (659, 17)
        assert sha256(sc.nodes()) == str(g['nodes_sha256'])
    finally:
        sc.close()
