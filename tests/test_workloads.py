"""The seeded synthetic workloads (scenes.py) have the shapes of the
configurations they stand in for: triangle counts, lights and their emission,
albedo ranges, displacement amplitudes, resolutions, depths and paths per
pixel. CPU only."""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / 'custom-ray-tracing-shader_b200'))
import scenes  # noqa: E402


def vec(tris, field):
    return np.stack([tris[field][k] for k in 'xyz'], axis=1).astype(np.float64)


def radial_spread(tris, center):
    """Relative spread of corner distances from the sphere's center."""
    r = np.linalg.norm(vec(tris, 'origin') - np.asarray(center), axis=1)
    return r.min() / np.median(r), r.max() / np.median(r)


def test_plain_method_small():
    tris, cam, st, w, h = scenes.cornell_sphere()
    assert len(tris) == 5132 and (w, h) == (256, 256) and st.maxBounces == 4
    lights = tris[tris['emission'] > 0]
    assert len(lights) == 2 and np.all(lights['emission'] == 15.0)  # one quad light, emission 15
    sphere = tris[tris['mesh'] == 7]
    assert len(sphere) == 5120  # level-4 icosphere: 20 * 16^2
    lo, hi = radial_spread(sphere, (0.0, 0.55, 0.1))
    assert 0.97 < lo < 1.0 < hi < 1.03  # +-2% displacement of radius 0.3
    color = vec(tris[tris['emission'] == 0], 'color')  # albedo of every object in [0.2, 0.8]^3
    assert color.min() >= 0.2 and color.max() <= 0.8


def test_traversal_and_build_at_scale():
    tris, cam, st, w, h = scenes.displaced_sphere_room()
    assert len(tris) == 1003532 and (w, h) == (1920, 1080) and st.maxBounces == 3
    sphere = tris[tris['mesh'] == 7]
    assert len(sphere) == 1003520  # 20 * 224^2, about one million
    assert len(tris) - len(sphere) == 12  # the room with one quad light
    assert (tris['emission'] > 0).sum() == 2
    lo, hi = radial_spread(sphere, (0.0, 1.45, 0.3))
    assert 0.94 < lo < 1.0 < hi < 1.06  # +-5% radial noise
    assert np.all(tris['specularProbability'] == 0)  # diffuse only


def test_batched_multi_scene():
    scene_list, views, st = scenes.batch_workload()
    counts = [len(t) for t in scene_list]
    assert len(scene_list) == 8 and len(views) == 64
    assert all(10_000 <= n <= 2_100_000 for n in counts)
    assert {w for _, _, w, _ in views} <= {256, 512, 1024} and all(w == h for _, _, w, h in views)
    assert {k for k, _, _, _ in views} == set(range(8))
    assert st.raysPerPixel == 8 and st.maxBounces == 4


def test_end_to_end_equal_quality():
    tris, cam, st, w, h = scenes.end_to_end_room()
    assert len(tris) == 1997134 and (w, h) == (1920, 1080) and st.maxBounces == 5
    assert (tris['emission'] > 0).sum() == 2


def test_denoiser_training_set():
    """The learned denoiser's training configuration: 200 seeded rooms of 5K
    to 500K triangles (log-uniform), 5,000 crops of 128x128, 4-spp inputs
    with the ten AOV channels, 1024-spp targets, batch 32, 20K steps, Adam
    at lr 1e-3."""
    import inspect
    import train_denoiser as td
    plan = td.training_plan(200)
    budgets = np.array([b for _, b in plan])
    assert len(plan) == 200 and len({s for s, _ in plan}) == 200
    assert budgets.min() >= 5_000 and budgets.max() <= 500_000
    logs = np.log(budgets)
    assert abs(np.exp(logs.mean()) / 50_000 - 1) < 0.35          # geometric mean of a log-uniform [5K, 500K]
    assert budgets.min() < 8_000 and budgets.max() > 300_000
    src = inspect.getsource(td.main)
    for flag, value in (("'--scenes'", '200'), ("'--crops'", '5000'), ("'--crop'", '128'), ("'--input-spp'", '4'),
                        ("'--target-spp'", '1024'), ("'--steps'", '20000'), ("'--batch'", '32'), ("'--lr'", '1e-3')):
        line = next(l for l in src.splitlines() if flag in l)
        assert f'default={value}' in line, (flag, line)
    assert td.INPUTS_PER_ROOM * (384 // 128) ** 2 * 200 >= 5000
    for seed, budget in (plan[0], plan[int(np.argmax(budgets))], plan[int(np.argmin(budgets))]):
        tris, cam, st, env = scenes.random_room(seed, 384, 384, triangles=budget)
        assert abs(len(tris) / budget - 1) < 0.25, (seed, budget, len(tris))
        assert 3 <= st.maxBounces <= 6
