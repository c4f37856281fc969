"""Trains the learned denoiser (the RtxUnet* entry points) on images that
this library renders.

Data (the denoiser-training configuration): 200 seeded random rooms
(scenes.random_room) whose triangle counts are drawn log-uniformly from 5K to
500K; each is rendered at 384x384 once with 1024 paths per pixel (the
target: linear radiance, the colour AOV of RtxReadAovs) and three times with
4 paths per pixel and other sampler seeds (the inputs: all ten AOVs, 4-spp
radiance, albedo, normal, linear depth). Every image is cut into nine
128x128 crops, and 25 crops per room are kept: 5,000 crops. The network
trains with Adam at lr 1e-3 (cosine decay) for 20K steps at batch 32 on
random crops with random flips and an L1 loss on log(1 + radiance).
Held-out rooms (other seeds) report PSNR of the display values (exposure
tonemap and sRGB, as RtRender displays) for the input, the guided filter and
the network at 4 and 8 paths per pixel.

Usage:
  python train_denoiser.py [--scenes 200] [--crops 5000] [--holdout 12]
      [--size 384] [--input-spp 4] [--target-spp 1024] [--steps 20000]
      [--out weights/denoiser_unet.bin]
"""
import argparse
import json
import math
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
if str(HERE) not in sys.path:
    sys.path.insert(0, str(HERE))

import scenes  # noqa: E402
from native_api import DENOISER_WEIGHTS, Session, Settings, Unet, load_library  # noqa: E402

TRIANGLES = (5_000, 500_000)  # per room, log-uniform
INPUTS_PER_ROOM = 3            # 4-spp renders per room (other sampler seeds)


def training_plan(scenes_count, seed=1):
    """(room seed, triangle budget) of every training room."""
    rng = np.random.default_rng(seed)
    lo, hi = np.log(TRIANGLES[0]), np.log(TRIANGLES[1])
    return [(10_000 + i, int(round(np.exp(rng.uniform(lo, hi))))) for i in range(scenes_count)]


def display(radiance, exposure):
    """8-bit display values of linear radiance (Native/renderer.cu:86-90)."""
    c = 1.0 - np.exp(-np.maximum(radiance, 0.0) * exposure)
    c = np.where(c <= 0.0031308, 12.92 * c, 1.055 * np.power(c, 1 / 2.4) - 0.055)
    return np.floor(255.0 * np.minimum(c, 1.0) + 0.5)


def psnr(a, b):
    rmse = math.sqrt(float(np.mean((a.astype(np.float64) - b) ** 2)))
    return 20 * math.log10(255.0 / max(rmse, 1e-12))


def accumulate(session, camera, settings, spp, per_pass):
    """Render spp paths per pixel in passes of per_pass with one setting."""
    session.lib.RtReset(session.handle)
    settings.raysPerPixel = per_pass
    while session.sample_count() < spp:
        session.render_device(camera, settings)
    assert session.sample_count() == spp


def render_room(lib, seed, size, target_spp, input_spps, triangles=50_000):
    """(inputs [k][size][size][10], target [size][size][3], exposure, guided filter displays)."""
    tris, cam, st, env = scenes.random_room(seed, size, size, triangles=triangles)
    s = Session(lib)
    try:
        s.initialize(tris, size, size)
        s.set_environment(env)
        target_settings = Settings(st.maxBounces, st.exposure, st.aperture, st.focusDistance, st.skyStrength,
                                   1_000_003 + seed, 16)
        accumulate(s, cam, target_settings, target_spp, 16)
        target = s.aovs()[..., 0:3].copy()
        inputs, filtered = [], []
        for k, spp in enumerate(input_spps):
            settings = Settings(st.maxBounces, st.exposure, st.aperture, st.focusDistance, st.skyStrength,
                                7919 * seed + 101 * k + 5, 1)
            accumulate(s, cam, settings, spp, min(spp, 16))
            inputs.append(s.aovs())
            image, _ = s.denoise()
            filtered.append(image.reshape(size, size, 4)[..., :3].astype(np.float64))
        return np.stack(inputs), target, st.exposure, filtered
    finally:
        s.close()


def crops(images, crop):
    """(n, S, S, c) -> (n * (S / crop)^2, crop, crop, c)."""
    n, h, w, ch = images.shape
    t = images.reshape(n, h // crop, crop, w // crop, crop, ch).transpose(0, 1, 3, 2, 4, 5)
    return np.ascontiguousarray(t.reshape(-1, crop, crop, ch))


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split('\n\n')[0])
    ap.add_argument('--scenes', type=int, default=200, help='training rooms')
    ap.add_argument('--crops', type=int, default=5000, help='training crops in all (an equal share per room)')
    ap.add_argument('--holdout', type=int, default=12, help='validation rooms (other seeds)')
    ap.add_argument('--size', type=int, default=384, help='render resolution (square)')
    ap.add_argument('--crop', type=int, default=128)
    ap.add_argument('--input-spp', type=int, default=4)
    ap.add_argument('--target-spp', type=int, default=1024)
    ap.add_argument('--steps', type=int, default=20000)
    ap.add_argument('--batch', type=int, default=32)
    ap.add_argument('--lr', type=float, default=1e-3)
    ap.add_argument('--seed', type=int, default=1)
    ap.add_argument('--out', default=str(DENOISER_WEIGHTS))
    ap.add_argument('--log', default=None, help='write a JSON summary here')
    args = ap.parse_args(argv)
    assert args.size % args.crop == 0 and args.crop % 16 == 0
    per_room = -(-args.crops // args.scenes)
    assert per_room <= INPUTS_PER_ROOM * (args.size // args.crop) ** 2
    lib = load_library()

    t0 = time.perf_counter()
    train_in, train_t, budgets = [], [], []
    for seed, budget in training_plan(args.scenes, args.seed):
        inputs, target, _, _ = render_room(lib, seed, args.size, args.target_spp,
                                           (args.input_spp,) * INPUTS_PER_ROOM, budget)
        train_in.append(crops(inputs, args.crop)[:per_room])
        train_t.append(crops(np.repeat(target[None], len(inputs), 0), args.crop)[:per_room])
        budgets.append(budget)
    train_in, train_t = np.concatenate(train_in)[:args.crops], np.concatenate(train_t)[:args.crops]
    val = [render_room(lib, 900_000 + i, args.size, args.target_spp, (4, 8)) for i in range(args.holdout)]
    data_s = time.perf_counter() - t0
    print(f'data: {len(train_in)} crops of {args.crop}^2 from {args.scenes} rooms of '
          f'{min(budgets)}-{max(budgets)} triangles, {args.holdout} held out, {data_s:.1f} s', flush=True)

    net = Unet(lib, seed=args.seed)
    t1 = time.perf_counter()
    chunk, history = 500, []
    for start in range(0, args.steps, chunk):
        steps = min(chunk, args.steps - start)
        # Cosine decay to 5% of the initial rate.
        lr = args.lr * (0.05 + 0.95 * 0.5 * (1 + math.cos(math.pi * start / max(args.steps, 1))))
        losses = net.train(train_in, train_t, steps, args.batch, lr, seed=args.seed * 7_777 + start)
        history.append([start + steps, float(losses.mean())])
        print(f'step {start + steps}: loss {losses.mean():.4f} (lr {lr:.2e})', flush=True)
    train_s = time.perf_counter() - t1

    report = []
    for inputs, target, exposure, filtered in val:
        ref = display(target, exposure)
        for k, spp in enumerate((4, 8)):
            out = net.infer(inputs[k])
            report.append({'spp': spp, 'input_db': psnr(display(inputs[k][..., 0:3], exposure), ref),
                           'filter_db': psnr(filtered[k], ref), 'unet_db': psnr(display(out, exposure), ref)})
    summary = {'crops': len(train_in), 'crop': args.crop, 'rooms': args.scenes,
               'room_triangles': [min(budgets), max(budgets)], 'input_spp': args.input_spp,
               'target_spp': args.target_spp, 'render_size': args.size,
               'steps': args.steps, 'batch': args.batch, 'lr': args.lr, 'data_seconds': data_s,
               'train_seconds': train_s, 'ms_per_step': 1e3 * train_s / max(args.steps, 1), 'loss': history}
    for spp in (4, 8):
        rows = [r for r in report if r['spp'] == spp]
        summary[f'holdout_{spp}spp'] = {key: float(np.mean([r[key] for r in rows]))
                                        for key in ('input_db', 'filter_db', 'unet_db')}
    print(json.dumps(summary), flush=True)
    Path(args.out).parent.mkdir(parents=True, exist_ok=True)
    net.save(args.out)
    if args.log:
        Path(args.log).write_text(json.dumps(summary, indent=1))
    net.close()


if __name__ == '__main__':
    main()
