#!/usr/bin/env python3
"""Benchmark: Mrays/s of the progressive path tracer on its at-scale workload.

Workload (one step = one progressive pass of 16 paths per pixel):
  displaced_sphere_room - a seeded geodesic sphere of 1,003,520 triangles
  (+-5% radial noise) in a 12-triangle room with one quad light,
  1920x1080, 16 paths per pixel per step, maximum depth 3, diffuse only.
  Rays = closest-hit queries (primary + secondary) + shadow (any-hit)
  queries, counted on the device.

Line fields beyond the common contract:
  roofline      dominant traversal kernel against measured HBM bandwidth;
                algorithmic bytes per ray = 64 * interior nodes + 44 *
                triangles that the reference's binary-BVH traversal
                (Native/renderer.cu:136-178) visits for the same rays, counted
                by the oracle on a pixel sample of the workload
  cpu_baseline  the reference's own CPU backend (Native/renderer.cu compiled
                from its sources into oracle/_ref, else the oracle port) on a
                bounded row sample, all host threads
  build         GPU BVH build (binned SAH + wide collapse), Mtris/s
  reference_cuda  the reference's own CUDA renderer built for sm_100a, same
                scene and settings, when oracle/_ref is present
  config1       the small configuration (5,132-triangle Cornell box,
                256x256, 64 paths per pixel as 4 passes of 16, depth 4):
                this library's device time, and the reference's CPU loop on
                one core (its backend 0) over a bounded row sample

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
For N > 1 run under torch.distributed.run; each rank renders its own copy of
the workload on its own GPU (replicas, weak scaling) and the step time is the
maximum over ranks.
"""
import argparse
import ctypes as c
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / 'custom-ray-tracing-shader_b200'))
sys.path.insert(0, str(ROOT / 'oracle'))

WORKLOAD = 'displaced_sphere_room'
METRIC = 'Mrays/s'
SPP_PER_STEP = 16


def parse():
    p = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument('--gpus', type=int, default=1)
    p.add_argument('--steps', type=int, default=20)
    p.add_argument('--warmup', type=int, default=3)
    p.add_argument('--impl', choices=('ours', 'reference'), default='ours')
    p.add_argument('--integrator', choices=('auto', 'wavefront', 'megakernel'), default='auto')
    p.add_argument('--cpu-seconds', type=float, default=12.0, help='budget of the CPU-baseline sample')
    p.add_argument('--no-cpu-baseline', action='store_true')
    p.add_argument('--no-reference-cuda', action='store_true')
    p.add_argument('--resolution', default=None, help='WxH override, for small profiling cases')
    p.add_argument('--spp', type=int, default=SPP_PER_STEP, help='paths per pixel per step (1..16)')
    p.add_argument('--no-quality', dest='quality', action='store_false',
                   help='skip time to 35 dB PSNR vs a 4096-spp render of the 2M-triangle scene (1 GPU runs it by default)')
    p.add_argument('--quality-resolution', default=None, help='WxH override of the quality scene')
    p.add_argument('--oracle-spp', type=int, default=4096)
    p.add_argument('--no-batch', dest='batch', action='store_false',
                   help='skip batched multi-scene tracing (8 scenes, 64 views; 1 GPU runs it by default)')
    p.add_argument('--batch-frames', type=int, default=3)
    p.add_argument('--no-denoiser', dest='denoiser', action='store_false',
                   help='skip the learned-denoiser inference timing (1 GPU runs it by default)')
    p.add_argument('--pieces', type=int, default=None,
                   help='pieces per triangle of the traversal tree (RTX_TUNE_PIECES; default: the library default)')
    p.add_argument('--leaf', type=int, default=None,
                   help='leaf size of the traversal tree (RTX_TUNE_LEAF; default: the library default)')
    p.add_argument('--refill', type=int, default=None,
                   help='refill threshold of the persistent traversal (RTX_TUNE_REFILL; default: the library default)')
    p.add_argument('--paths', type=int, default=None,
                   help='paths per wave (RTX_TUNE_PATHS_IN_FLIGHT; default: the library default, 2^24)')
    p.add_argument('--lanes', type=int, default=None,
                   help="waves in flight, 1..4 (RTX_TUNE_LANES; default: the library default)")
    p.add_argument('--denoiser-only', action='store_true',
                   help='only time learned-denoiser inference at 1920x1080 (a small case for profiling)')
    p.add_argument('--conv-path', type=int, choices=(0, 1, 2), default=0,
                   help='convolution kernel of the denoiser (RtxSetConvPath): 0 pipelined where it fits, '
                        '1 single-role, 2 pipelined with tap-by-tap issue only')
    p.add_argument('--no-train-step', dest='train_step', action='store_false',
                   help='skip timing U-Net training steps (batch 32 of 128x128 crops; 1 GPU runs it by default)')
    p.add_argument('--train-steps', type=int, default=20, help='timed training steps')
    p.add_argument('--train-step-only', action='store_true', help='only time U-Net training steps (for profiling)')
    p.add_argument('--build-only', action='store_true',
                   help='only the BVH builds of the workload at RtInitialize (for profiling): a warm-up build, then '
                        '--steps timed builds')
    p.set_defaults(quality=True, batch=True, denoiser=True, train_step=True)
    return p.parse_args()


def dist_env():
    return int(os.environ.get('RANK', 0)), int(os.environ.get('LOCAL_RANK', 0)), int(os.environ.get('WORLD_SIZE', 1))


class Dist:
    """torch.distributed plumbing for N > 1 (barrier, max over ranks)."""

    def __init__(self, world):
        self.world = world
        self.pg = None
        if world > 1:
            import datetime
            import torch
            import torch.distributed as dist
            backend = 'nccl' if torch.cuda.is_available() else 'gloo'
            if backend == 'nccl':
                torch.cuda.set_device(0)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
            self.torch, self.dist, self.backend = torch, dist, backend

    def barrier(self):
        if self.world > 1:
            self.dist.barrier()

    def max(self, value):
        if self.world == 1:
            return value
        t = self.torch.tensor([float(value)], dtype=self.torch.float64,
                              device='cuda' if self.backend == 'nccl' else 'cpu')
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, value):
        if self.world == 1:
            return value
        t = self.torch.tensor([float(value)], dtype=self.torch.float64,
                              device='cuda' if self.backend == 'nccl' else 'cpu')
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.world > 1:
            self.dist.barrier()
            self.dist.destroy_process_group()


class Clocks:
    """nvidia-smi sampling during the timed region."""
    FIELDS = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
              'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
              'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, gpu_index):
        self.gpu_index = gpu_index
        self.proc = None
        self.skip = 0
        self.path = Path(os.environ.get('TMPDIR', '/tmp')) / f'bench_clocks_{os.getpid()}.csv'

    def start(self):
        """Starts sampling every 100 ms and returns once nvidia-smi writes
        samples (its start-up takes a while), so that the timed region that
        follows is covered; samples from before it are dropped."""
        self.skip = 0
        try:
            self.proc = subprocess.Popen(['nvidia-smi', '-i', str(self.gpu_index), f'--query-gpu={self.FIELDS}',
                                          '--format=csv,noheader,nounits', '-lms', '100'],
                                         stdout=open(self.path, 'w'), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        t0 = time.perf_counter()
        while time.perf_counter() - t0 < 5.0 and self.proc.poll() is None:
            lines = self.path.read_text().count('\n')
            if lines:
                self.skip = lines
                return
            time.sleep(0.02)

    def stop(self):
        if not self.proc:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['nvidia-smi unavailable']}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, sm_max, power, reasons = [], None, [], set()
        names = ('hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap')
        for line in self.path.read_text().splitlines()[self.skip:]:
            parts = [p.strip() for p in line.split(',')]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                sm_max = float(parts[2])
                power.append(float(parts[3]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower().startswith('active'):
                    reasons.add(name)
        self.path.unlink(missing_ok=True)
        if not sm:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['no samples']}
        under_load = [s for s, p in zip(sm, power) if p > 0.5 * max(power)] or sm
        return {'sm_mhz': statistics.median(under_load), 'sm_max_mhz': sm_max, 'reasons': sorted(reasons),
                'samples': len(sm)}


def measured_peaks():
    path = ROOT / 'MEASURED_PEAKS.json'
    if path.exists():
        data = json.loads(path.read_text())
        return float(data['hbm_gbs']), 'measured'
    return 6650.0, 'fallback'


def workload(args=None):
    import scenes
    kwargs = {}
    if args is not None and args.resolution:
        kwargs['width'], kwargs['height'] = (int(v) for v in args.resolution.lower().split('x'))
    tris, cam, settings, w, h = scenes.displaced_sphere_room(**kwargs)
    settings.raysPerPixel = args.spp if args is not None else SPP_PER_STEP
    return tris, cam, settings, w, h


def sample_rows(h, stride):
    return list(range(stride // 2, h, stride))


def algorithmic_bytes(tris, cam, settings, w, h, pixel_count=4096):
    """Bytes per closest and per shadow query of the reference's traversal,
    from the oracle's counters on a seeded pixel sample of the workload."""
    import numpy as np
    from oracle_api import Oracle
    o = Oracle()
    sc = o.scene(tris)
    rng = np.random.Generator(np.random.PCG64(5))
    pixels = rng.choice(w * h, pixel_count, replace=False)
    _, _, counts = o.render_pixels(sc, cam, settings, w, h, pixels)
    sc.close()
    closest_q, closest_int, closest_tri = counts[3], counts[4], counts[6]
    shadow_q, shadow_int, shadow_tri = counts[7], counts[8], counts[10]
    return {
        'closest': (64.0 * closest_int + 44.0 * closest_tri) / max(closest_q, 1),
        'shadow': (64.0 * shadow_int + 44.0 * shadow_tri) / max(shadow_q, 1),
        'sample_pixels': int(pixel_count),
        'interior_per_closest': float(closest_int / max(closest_q, 1)),
        'triangles_per_closest': float(closest_tri / max(closest_q, 1)),
    }


def cpu_baseline(tris, cam, settings, w, h, budget_s):
    """The reference's CPU backend on all host threads over a bounded row sample."""
    from oracle_api import Oracle, Reference, reference_available
    kind = 'reference' if reference_available() else 'port'
    impl = Reference() if kind == 'reference' else Oracle()
    threads = impl.max_threads()
    sc = impl.scene(tris)
    # Size the sample: one probe row, then enough evenly spaced rows for the budget.
    t0 = time.perf_counter()
    impl.render(sc, cam, settings, w, h, rows=(h // 2, h // 2 + 1), threads=threads)
    per_row = max(time.perf_counter() - t0, 1e-4)
    nrows = int(max(1, min(h, budget_s / per_row)))
    stride = max(1, h // nrows)
    rows = sample_rows(h, stride)
    t0 = time.perf_counter()
    for y in rows:
        impl.render(sc, cam, settings, w, h, rows=(y, y + 1), threads=threads)
    elapsed = time.perf_counter() - t0
    sc.close()
    # Ray count of the same rows, from the oracle's counters (identical paths).
    o = Oracle()
    osc = o.scene(tris)
    rays = 0
    for y in rows:
        _, _, counts = o.render(osc, cam, settings, w, h, rows=(y, y + 1))
        rays += int(counts[0] + counts[1] + counts[2])
    osc.close()
    return {
        'value': rays / elapsed / 1e6, 'unit': METRIC, 'cores': threads, 'kind': kind,
        'sample': f'{len(rows)} of {h} rows (every {stride}th) x {w} px x {settings.raysPerPixel} spp, '
                  f'{rays} rays in {elapsed:.2f} s',
        'seconds': elapsed, 'rays': rays,
    }


def guarded(fn, *args):
    """An auxiliary measurement that must not cost the bench line."""
    try:
        return fn(*args)
    except Exception as e:  # reported in the line instead
        return {'error': f'{type(e).__name__}: {e}'}


def config1_run(lib, budget_s=6.0):
    """Config 1 (scenes.cornell_sphere: 256x256, 64 paths per pixel as 4
    passes of 16, depth 4) on the GPU through the session, and the
    reference's CPU render loop on one thread (its backend 0,
    Native/renderer.cu:405-416) over evenly spaced rows of one 16-path pass,
    sized to about budget_s seconds. Rays of the CPU sample are counted by
    the oracle on the same rows (identical paths)."""
    import scenes
    from native_api import Session
    from oracle_api import Oracle, Reference, reference_available
    tris, cam, st, w, h = scenes.cornell_sphere()
    st.raysPerPixel = 16
    with Session(lib) as s:
        s.initialize(tris, w, h)
        s.render_device(cam, st)  # warm-up pass
        s.lib.RtReset(s.handle)
        ms, rays = 0.0, 0
        for _ in range(4):
            ms += s.render_device(cam, st)
            stats = s.render_stats()
            rays += int(stats['primaryRays'] + stats['secondaryRays'] + stats['shadowRays'])
        assert s.sample_count() == 64
    kind = 'reference' if reference_available() else 'port'
    impl = Reference() if kind == 'reference' else Oracle()
    sc = impl.scene(tris)
    t0 = time.perf_counter()
    impl.render(sc, cam, st, w, h, rows=(h // 2, h // 2 + 1), threads=1)
    per_row = max(time.perf_counter() - t0, 1e-4)
    stride = max(1, h // int(max(1, min(h, budget_s / per_row))))
    rows = sample_rows(h, stride)
    t0 = time.perf_counter()
    for y in rows:
        impl.render(sc, cam, st, w, h, rows=(y, y + 1), threads=1)
    elapsed = time.perf_counter() - t0
    sc.close()
    o = Oracle()
    osc = o.scene(tris)
    cpu_rays = 0
    for y in rows:
        _, _, counts = o.render(osc, cam, st, w, h, rows=(y, y + 1))
        cpu_rays += int(counts[0] + counts[1] + counts[2])
    osc.close()
    cpu_rate = cpu_rays / elapsed / 1e6
    gpu_rate = rays / ms / 1e3
    return {'workload': 'cornell_sphere 5,132 triangles, 256x256, 64 spp (4 passes of 16), depth 4',
            'gpu': {'device_ms': ms, 'mrays_per_s': gpu_rate, 'rays': rays},
            'cpu_single_core': {'value': cpu_rate, 'unit': METRIC, 'cores': 1, 'kind': kind,
                                'sample': f'{len(rows)} of {h} rows (every {stride}th) x {w} px x 16 spp, '
                                          f'{cpu_rays} rays in {elapsed:.2f} s',
                                'estimated_full_config_s': rays / (cpu_rate * 1e6) if cpu_rate > 0 else None},
            'speedup_vs_single_core': gpu_rate / cpu_rate if cpu_rate > 0 else None}


def reference_cuda(tris, cam, settings, w, h, rays_per_step, first_pass, steps=3):
    """The reference's own CUDA renderer (oracle/_ref, built for sm_100a).
    first_pass = (PixelSum records, RGBA8 image) of this library's first pass
    on the same session settings; parity is true when the reference's first
    pass accumulates the same bytes and shows the same image."""
    from oracle_api import Reference, ReferenceSession, reference_available
    if not reference_available():
        return None
    ref = ReferenceSession(Reference())
    try:
        ref.initialize(tris, w, h)
        times = []
        parity = None
        for k in range(steps + 1):
            rgba, ms = ref.render(cam, settings)
            times.append(ms)
            if k == 0:
                parity = (ref.sums().tobytes() == first_pass[0].tobytes() and
                          rgba.tobytes() == first_pass[1].tobytes())
        ms = statistics.median(times[1:])
        return {'value': rays_per_step / ms / 1e3, 'unit': METRIC, 'ms_per_step': ms, 'parity': parity,
                'note': 'Native/renderer.cu renderKernel built for sm_100a, same scene, settings and ray count; '
                        'parity: its first pass accumulates the same PixelSum bytes and RGBA8 image as this '
                        "library's"}
    finally:
        ref.close()


def psnr8(image, reference):
    """PSNR in dB of 8-bit RGB display values (alpha ignored)."""
    import numpy as np
    a = image.reshape(-1, 4)[:, :3].astype(np.float64)
    b = reference.reshape(-1, 4)[:, :3].astype(np.float64)
    mse = float(np.mean((a - b) ** 2))
    return (float('inf') if mse == 0 else float(20.0 * np.log10(255.0 / np.sqrt(mse)))), float(np.sqrt(mse))


def display_float(radiance, exposure):
    """The reference's display transform (Native/renderer.cu:86-90) before its
    8-bit quantisation: 1 - exp(-max(c, 0) * exposure), the sRGB curve,
    clamped to 1; float64."""
    import numpy as np
    c = 1.0 - np.exp(-np.maximum(np.asarray(radiance, np.float64), 0.0) * exposure)
    c = np.where(c <= 0.0031308, 12.92 * c, 1.055 * np.power(c, 1.0 / 2.4) - 0.055)
    return np.minimum(c, 1.0)


class QualityReference:
    """The 4096-path FP32 render of a scene: linear radiance per pixel
    (sum / samples) and its display values as floats."""

    def __init__(self, radiance, exposure, rgba):
        import numpy as np
        self.linear = np.asarray(radiance, np.float64)
        self.display = display_float(self.linear, exposure)
        self.exposure = exposure
        self.rgba = rgba

    def score(self, radiance, rgba=None):
        """PSNR (dB) of float display values, RMSE of linear HDR radiance and,
        given the RGBA8 image, the 8-bit PSNR of the reference's own quality
        tool (Tools/verify_quality.py:53-54)."""
        import numpy as np
        lin = np.asarray(radiance, np.float64)
        d = display_float(lin, self.exposure) - self.display
        rmse = float(np.sqrt(np.mean(d * d)))
        out = {'psnr_float_db': float('inf') if rmse == 0 else float(20.0 * np.log10(1.0 / rmse)),
               'rmse_display': rmse,
               'rmse_linear': float(np.sqrt(np.mean((lin - self.linear) ** 2)))}
        if rgba is not None:
            out['psnr_8bit_db'], out['rmse_8bit'] = psnr8(rgba, self.rgba)
        return out


def accumulated_radiance(session):
    import numpy as np
    acc = session.accumulation()
    samples = session.sample_count()
    return np.stack([acc['radiance'][k] for k in 'xyz'], 1).astype(np.float64) / samples


def quality_run(lib, args, target_db=35.0):
    """Time to reach target_db PSNR against a 4096-path FP32 render of the
    end-to-end scene (2M triangles, 1920x1080, depth 5, constant 0.1
    environment): plain progressive accumulation against 8 (or more) paths
    per pixel followed by RtDenoise, with the learned U-Net and with the
    guided filter.

    Quality: PSNR of the display values as floats (the reference's display
    transform before 8-bit quantisation) and RMSE of the linear HDR radiance,
    both against the FP32 accumulation of the 4096-path render (another
    sampler seed than the arms'); the 8-bit PSNR that the reference's own
    tool uses (Tools/verify_quality.py:53-54, against 2048 paths there) is
    reported beside them. The denoised arms are scored on RtxReadDenoised's
    linear radiance, the plain arm on its running sums.

    Time: each arm is re-run from a reset once its path count is known and
    timed on the host wall clock through the public calls (RtRender per pass,
    with its RGBA8 read-back, then RtDenoise with its read-back), after the
    buffers were allocated by earlier calls; the device time of the same calls
    (CUDA events) is reported beside it."""
    import numpy as np
    import scenes
    from native_api import DENOISER_WEIGHTS, Session, Settings, Unet
    kwargs = {}
    if args.quality_resolution:
        kwargs['width'], kwargs['height'] = (int(v) for v in args.quality_resolution.lower().split('x'))
    tris, cam, st, w, h = scenes.end_to_end_room(**kwargs)
    s = Session(lib)
    try:
        s.initialize(tris, w, h)
        s.set_environment(0.1)
        oracle_settings = Settings(st.maxBounces, st.exposure, st.aperture, st.focusDistance, st.skyStrength,
                                   20261023, 16)
        oracle_ms = 0.0
        passes = max(1, args.oracle_spp // 16)
        for _ in range(passes - 1):
            oracle_ms += s.render_device(cam, oracle_settings)
        oracle_rgba, ms = s.render(cam, oracle_settings)
        oracle_ms += ms
        ref = QualityReference(accumulated_radiance(s), st.exposure, oracle_rgba.copy())
        out = np.zeros(w * h * 4, np.uint8)

        def replay(spp, per_pass, denoise):
            """Wall and device time of spp paths per pixel from a reset through
            RtRender passes of per_pass, then RtDenoise when asked."""
            st.raysPerPixel = per_pass
            s.lib.RtReset(s.handle)
            device = 0.0
            t0 = time.perf_counter()
            while s.sample_count() < spp:
                _, ms = s.render(cam, st, output=out)
                device += ms
            if denoise:
                s.denoise(output=out)
            wall = (time.perf_counter() - t0) * 1e3
            if denoise:
                device += s.render_stats()['denoiseMs']
            return wall, device

        # Plain progressive accumulation, 4 paths per pixel per pass (one pass
        # size throughout: RtRender restarts when a setting changes,
        # renderer.cu:388-389): the first pass count that reaches the target,
        # found by scoring every 8th pass, then every pass of the last stretch
        # rendered again from a reset (the same paths: results are
        # deterministic).
        st.raysPerPixel = 4
        coarse = 8
        s.lib.RtReset(s.handle)
        s.render(cam, st, output=out)  # allocations of this pass size
        s.lib.RtReset(s.handle)
        curve, reached, upper = [], None, None
        while s.sample_count() < args.oracle_spp // 2:
            img, _ = s.render(cam, st, output=out)
            spp = s.sample_count()
            if spp % (4 * coarse) == 0 or spp >= args.oracle_spp // 2:
                q = ref.score(accumulated_radiance(s), img)
                curve.append([spp, round(q['psnr_float_db'], 3), round(q['psnr_8bit_db'], 3)])
                if q['psnr_float_db'] >= target_db:
                    upper = spp
                    break
        if upper is not None:
            s.lib.RtReset(s.handle)
            while s.sample_count() < max(0, upper - 4 * coarse):
                s.render(cam, st, output=out)
            while s.sample_count() < upper:
                img, _ = s.render(cam, st, output=out)
                q = ref.score(accumulated_radiance(s), img)
                if q['psnr_float_db'] >= target_db:
                    reached = dict(q, spp=s.sample_count())
                    break
        plain = dict(reached or {'spp': s.sample_count(), 'psnr_float_db': curve[-1][1] if curve else None},
                     reaches_target=reached is not None)
        if reached:
            plain['wall_ms'], plain['device_ms'] = replay(reached['spp'], 4, False)

        def denoised_arm(name):
            """8 paths per pixel, then more until the denoised image reaches
            the target (each budget rendered from a reset; above 16 paths a
            budget is several passes of 16)."""
            trials, arm = [], None
            for budget in (8, 16, 32, 64, 128, 256):
                per = min(16, budget)
                st.raysPerPixel = per
                s.lib.RtReset(s.handle)
                while s.sample_count() < budget:
                    img, _ = s.render(cam, st, output=out)
                raw = ref.score(accumulated_radiance(s), img)
                den, _ = s.denoise()
                q = ref.score(s.denoised_radiance(), den)
                trial = dict(q, spp=budget, raw_psnr_float_db=raw['psnr_float_db'])
                trial['wall_ms'], trial['device_ms'] = replay(budget, per, True)
                trials.append(trial)
                if q['psnr_float_db'] >= target_db:
                    arm = dict(trial, reaches_target=True)
                    break
            arm = arm or dict(trials[-1], reaches_target=False)
            arm['denoiser'] = name
            arm['at_8spp'] = trials[0]
            return arm

        st.raysPerPixel = 8
        s.lib.RtReset(s.handle)
        s.render(cam, st, output=out)
        s.denoise()  # the first call allocates the filter's buffers and loads its kernels
        filtered = denoised_arm('guided a-trous wavelet filter (RtDenoise without a network)')
        learned = None
        if DENOISER_WEIGHTS.exists():
            net = Unet(lib)
            try:
                net.load(DENOISER_WEIGHTS)
                s.set_denoiser(net)
                s.denoise()  # the first inference at this size allocates the activations
                learned = denoised_arm(f'learned U-Net ({net.param_count:,} parameters, BF16 tensor cores; '
                                       f'RtDenoise with RtxSetDenoiser)')
            finally:
                s.set_denoiser(None)
                net.close()
        result = {
            'workload': 'end_to_end_room', 'triangles': len(tris), 'width': w, 'height': h,
            'max_depth': st.maxBounces, 'environment': 0.1, 'exposure': st.exposure, 'target_db': target_db,
            'oracle_spp': passes * 16, 'oracle_device_ms': oracle_ms,
            'psnr_metric': ('20 log10(1 / RMSE) of display values as floats (Native/renderer.cu:86-90 before '
                            '8-bit quantisation) against the FP32 4096-path accumulation; rmse_linear on linear '
                            'HDR radiance; psnr_8bit_db is the reference tool\'s 8-bit metric'),
            'timing': 'wall_ms: host wall clock through RtRender passes (RGBA8 read-back each) and RtDenoise '
                      '(RGBA8 read-back), after allocation; device_ms: CUDA events of the same calls',
            'plain': plain, 'filter': filtered, 'learned': learned,
            'curve_every_4spp': curve[:: max(1, len(curve) // 32)],
        }
        for key, arm in (('filter', filtered), ('learned', learned)):
            if plain.get('reaches_target') and arm and arm['reaches_target']:
                result[f'speedup_{key}_vs_plain_wall'] = plain['wall_ms'] / arm['wall_ms']
                result[f'speedup_{key}_vs_plain_device'] = plain['device_ms'] / arm['device_ms']
        return result
    finally:
        s.close()


def batch_run(lib, args):
    """Batched multi-scene tracing: eight scenes of 10K-2M triangles (log-
    uniform), 64 views of 256^2, 512^2 or 1024^2, 8 paths per pixel, depth 4.
    The batch (one wave of paths across all views per traversal launch,
    frames replayed from a CUDA graph, launch shape and BVH width from the
    autotuner) against the same views rendered one by one through RtRender's
    device path (one session per scene and resolution). Rays: closest-hit
    plus shadow queries counted on the device."""
    import scenes
    from native_api import Batch, Session
    t0 = time.perf_counter()
    scene_list, views, st = scenes.batch_workload()
    gen_s = time.perf_counter() - t0
    b = Batch(lib)
    try:
        for tris in scene_list:
            b.add_scene(tris)
        for k, cam, w, h in views:
            b.add_view(k, cam, w, h)
        built = b.stats()
        t1 = time.perf_counter()
        tried = b.autotune(st)
        tune_s = time.perf_counter() - t1

        def frames(graph):
            b.set_tuning(graph=graph)
            b.reset()
            b.render(st)  # warm-up (and graph capture)
            ms = []
            rays = 0
            for _ in range(args.batch_frames):
                b.reset()  # samples 0..7 again: the paths (and rays) of the per-view renders
                ms.append(b.render(st))
                stats = b.stats()
                rays = stats['primaryRays'] + stats['secondaryRays'] + stats['shadowRays']
            best = min(ms)
            return {'frame_ms': best, 'mrays_per_s': rays / best / 1e3, 'rays_per_frame': rays,
                    'kernel_launches': stats['kernelLaunches']}
        graph = frames(1)
        launches = frames(0)
        tuned = b.stats()
        # One persistent launch per frame over a (view, tile) queue, the
        # reference's launch shape (RTX_BATCH_PERSISTENT).
        b.set_tuning(persistent=1)
        persistent = frames(1)
        b.set_tuning(persistent=0)
    finally:
        b.close()
    # Per-view launches: every view alone through the single-view device path.
    sessions = {}
    per_view_ms, per_view_rays = 0.0, 0
    try:
        for k, cam, w, h in views:
            s = sessions.get((k, w, h))
            if s is None:
                s = sessions[(k, w, h)] = Session(lib).initialize(scene_list[k], w, h)
                s.render_device(cam, st)  # warm-up of this session
            s.lib.RtReset(s.handle)  # samples 0..7, as in the batch frames
            per_view_ms += s.render_device(cam, st)
            r = s.render_stats()
            per_view_rays += r['primaryRays'] + r['secondaryRays'] + r['shadowRays']
    finally:
        for s in sessions.values():
            s.close()
    per_view = {'frame_ms': per_view_ms, 'mrays_per_s': per_view_rays / per_view_ms / 1e3,
                'rays_per_frame': per_view_rays}
    return {
        'workload': 'batch_workload (8 scenes, 64 views)', 'scenes': len(scene_list),
        'triangles': [len(t) for t in scene_list], 'views': len(views), 'pixels': built['pixels'],
        'spp_per_frame': st.raysPerPixel, 'max_depth': st.maxBounces,
        'build_ms': built['buildMs'], 'build_mtris_per_s': built['triangles'] / built['buildMs'] / 1e3,
        'generate_s': gen_s, 'autotune_s': tune_s, 'autotune': tried,
        'tuned': {k: tuned[k] for k in ('block', 'capacity', 'refill', 'width', 'pieces', 'lanes')},
        'batched_graph': graph, 'batched_launches': launches, 'persistent_launch': persistent,
        'per_view_launches': per_view,
        'speedup_vs_per_view': per_view['frame_ms'] / graph['frame_ms'],
        'same_rays': graph['rays_per_frame'] == per_view_rays,
    }


def unet_flops_per_pixel():
    """Forward FLOPs per (padded) pixel of the U-Net: 2 * 9 * cin * cout per
    3x3 layer at 1/4^level of the pixels, plus the 1x1 output layer."""
    widths, prev, table = (32, 48, 64, 96, 128), 16, []
    for level, w in enumerate(widths):
        table += [(prev, w, level), (w, w, level)]
        prev = w
    for level in (3, 2, 1, 0):
        w = widths[level]
        table += [(prev + w, w, level), (w, w, level)]
        prev = w
    return sum(2 * 9 * ci * co / 4 ** lv for ci, co, lv in table) + 2 * 32 * 3


def denoiser_run(lib, args, repeats=10):
    """Learned-denoiser inference at 1920x1080 through RtDenoise (AOV kernel,
    U-Net on BF16 tensor cores, tonemap, RGBA8 read-back): wall time per call
    and the tensor-core rate it implies against the measured bf16 peak."""
    import scenes
    from native_api import DENOISER_WEIGHTS, Session, Unet
    tris, cam, st, _, _ = scenes.cornell_sphere()
    w, h = 1920, 1080
    cam.aspect = w / h
    st.raysPerPixel = 8
    net = Unet(lib)
    s = Session(lib)
    try:
        net.load(DENOISER_WEIGHTS)
        s.initialize(tris, w, h)
        s.render(cam, st)
        s.set_denoiser(net)
        s.denoise()  # allocates the activations for this size
        times, device = [], []
        for _ in range(repeats):
            times.append(s.denoise()[1])
            device.append(s.render_stats()['denoiseMs'])
    finally:
        s.set_denoiser(None)
        s.close()
        net.close()
    ms = statistics.median(times)
    padded = ((h + 15) // 16 * 16) * ((w + 15) // 16 * 16)
    flops = unet_flops_per_pixel() * padded
    path = ROOT / 'MEASURED_PEAKS.json'
    peak, source = (float(json.loads(path.read_text())['bf16_tflops']), 'measured') if path.exists() else \
        (1590.0, 'fallback')
    device_ms = statistics.median(device)
    tflops = flops / (ms * 1e-3) / 1e12
    device_tflops = flops / (device_ms * 1e-3) / 1e12
    return {'workload': 'U-Net inference via RtDenoise, 1920x1080 (1920x1088 padded)', 'ms_per_call': ms,
            'min_ms': min(times), 'device_ms': device_ms, 'mflop_per_pixel': unet_flops_per_pixel() / 1e6,
            'gflop_per_call': flops / 1e9, 'tflops_whole_call': tflops,
            'roofline': {'bound': 'tensor', 'achieved': device_tflops, 'peak': peak, 'unit': 'TFLOP/s',
                         'frac': device_tflops / peak if peak else None, 'peak_source': f'{source} bf16_tflops',
                         'note': 'network FLOPs over the device time of RtDenoise\'s kernels (AOVs, U-Net, '
                                 'display; CUDA events), against the bf16 dense GEMM peak'}}


def train_step_run(lib, args, batch=32, size=128, crops=64, warmup=5):
    """U-Net training steps as configured for the denoiser (batch 32 of
    128x128 crops, Adam): forward, L1 loss on log radiance, backward (data
    and weight gradients on the tensor cores), Adam and the BF16 weight
    copies, driven by RtxUnetTrain on a seeded synthetic crop set resident on
    the device. ms_per_step = host wall time of RtxUnetTrain over the timed
    steps (it synchronises at its end) / steps."""
    import numpy as np
    from native_api import Unet
    rng = np.random.default_rng(31)
    yy, xx = np.mgrid[0:size, 0:size] / size
    target = (rng.uniform(0.1, 2.0, (crops, 1, 1, 3)) * (0.5 + 0.5 * np.sin(3 * xx + 2 * yy))[None, ..., None])
    aovs = np.empty((crops, size, size, 10), np.float32)
    aovs[..., 0:3] = target * rng.exponential(1.0, (crops, size, size, 3))
    aovs[..., 3:6] = rng.uniform(0, 1, (crops, 1, 1, 3))
    nrm = rng.normal(size=(crops, size, size, 3))
    aovs[..., 6:9] = nrm / np.linalg.norm(nrm, axis=-1, keepdims=True)
    aovs[..., 9] = 1.0 + 4.0 * yy[None]
    target = target.astype(np.float32)
    net = Unet(lib, seed=3)
    try:
        net.train(aovs, target, steps=warmup, batch=batch, lr=1e-3, seed=1)
        t0 = time.perf_counter()
        losses = net.train(aovs, target, steps=args.train_steps, batch=batch, lr=1e-3, seed=2)
        wall = time.perf_counter() - t0
    finally:
        net.close()
    ms = wall * 1e3 / args.train_steps
    flops = 3.0 * unet_flops_per_pixel() * batch * size * size  # forward, data gradient, weight gradient
    return {'workload': f'U-Net training step, batch {batch} of {size}x{size} crops, Adam (RtxUnetTrain)',
            'steps': args.train_steps, 'ms_per_step': ms, 'gflop_per_step': flops / 1e9,
            'tflops': flops / (ms * 1e-3) / 1e12, 'loss_first': float(losses[0]), 'loss_last': float(losses[-1]),
            'timing': 'host wall clock around RtxUnetTrain (synchronises at its end), after warm-up steps'}


def build_report(tris, bvh, init_wall_ms, peak, peak_kind):
    """GPU BVH build at RtInitialize. The traced tree (over triangle pieces
    when some triangle is split, else the reference's tree) is what
    RtInitialize builds; the reference's own tree is built on the first
    RtBvhInfo / RtxExportBvh / RtxBvhStatsGet when it is not the traced one.
    Roofline: algorithmic bytes per build triangle B_tri = (36 B of vertices
    + 8 B of index read/write) per binned-SAH level, ceil(log2(N / 4))
    levels, + 32 B per node of the reference's tree, against HBM bandwidth."""
    import math
    n = len(tris)
    pieces = bvh['pieces']
    reference_ms = bvh['buildMs'] + bvh['collapseMs']
    traced_ms = bvh['pieceBuildMs'] if pieces > 1 else reference_ms
    b_tri = 44.0 * math.ceil(math.log2(max(n / 4.0, 2.0))) + 32.0 * bvh['binaryNodes'] / n
    achieved = n * b_tri / (traced_ms * 1e-3) / 1e9
    return {
        'traced_tree': {'ms': traced_ms, 'mtris_per_s': n / traced_ms / 1e3, 'pieces_per_triangle': pieces,
                        'wide_nodes': bvh['wideNodes'], 'wide_depth': bvh['wideDepth'],
                        'built': 'at RtInitialize'},
        'reference_tree': {'ms': reference_ms, 'binned_sah_ms': bvh['buildMs'], 'collapse_ms': bvh['collapseMs'],
                           'mtris_per_s': n / reference_ms / 1e3, 'binary_nodes': bvh['binaryNodes'],
                           'binary_depth': bvh['binaryDepth'], 'sah_cost': bvh['sahCost'],
                           'built': ('on first RtBvhInfo/RtxExportBvh/RtxBvhStatsGet' if pieces > 1
                                     else 'at RtInitialize (it is the traced tree)')},
        'mtris_per_s': n / traced_ms / 1e3,
        'roofline': {'bound': 'hbm', 'bytes_per_triangle': b_tri, 'achieved': achieved, 'peak': peak,
                     'unit': 'GB/s', 'frac': achieved / peak,
                     'peak_source': f'{peak_kind} hbm_gbs', 'kernel': 'traced-tree build (all its kernels)'},
        'initialize_wall_ms': init_wall_ms, 'upload_ms': bvh['uploadMs'], 'distinct_colours': bvh['distinctColours'],
    }


def kernel_rates(integrator, per_kind, primary_ms, extend_ms, shadow_ms, lanes):
    """Mrays/s of each traversal kind over its own kernels' device time:
    primary (closest-hit at bounce 0), secondary (closest-hit at later
    bounces) and shadow (any-hit) queries. Wavefront integrator only; the
    megakernel interleaves all three in one launch. With two lanes of waves
    the launches overlap and these rates are lower bounds."""
    if integrator != 'wavefront' or extend_ms <= 0:
        return None
    rate = lambda rays, ms: rays / ms / 1e3 if ms > 0 else None
    return {'primary': rate(per_kind['primaryRays'], primary_ms),
            'secondary': rate(per_kind['secondaryRays'], extend_ms - primary_ms),
            'shadow': rate(per_kind['shadowRays'], shadow_ms),
            'lanes': lanes, 'bound': 'lower' if lanes > 1 else 'isolated'}


def l2_flusher():
    try:
        import torch
        if torch.cuda.is_available():
            buf = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device='cuda')  # 256 MB > 126 MB L2

            def flush():
                buf.fill_(1.0)
                torch.cuda.synchronize()
            return flush, 'flushed between steps (256 MB write)'
    except Exception:
        pass
    return (lambda: None), 'inputs larger than L2 (1.0M triangles: 116 MB records + 48 MB packed + 8.5 MB nodes)'


def build_only_run(lib, args):
    """The workload's BVH builds alone: RtInitialize of the workload scene
    after a warm-up build, `--steps` times, with the build report of the
    fastest (the traced tree; the reference's own tree is built on the
    first RtxBvhStatsGet, after the traced tree's time is taken)."""
    from native_api import Session
    tris, _, _, w, h = workload(args)
    peak, peak_kind = measured_peaks()
    reports = []
    for k in range(max(args.steps, 1) + 1):
        with Session(lib) as s:
            t0 = time.perf_counter()
            s.initialize(tris, 64, 64)
            wall = (time.perf_counter() - t0) * 1e3
            if k > 0:
                reports.append(build_report(tris, s.bvh_stats(), wall, peak, peak_kind))
    return min(reports, key=lambda r: r['traced_tree']['ms'])


def run_ours(args, rank, local_rank, world):
    import numpy as np
    from native_api import Session, load_library
    dist = Dist(world)
    lib = load_library()
    tris, cam, settings, w, h = workload(args)
    # Load every kernel once (CUDA loads modules lazily at first launch), so
    # the reported build time is the build's, not one-time module loading.
    import scenes
    with Session(lib) as warm:
        small = scenes.cornell_sphere(width=32, height=32)
        # Two diagonal slivers: the warm-up also builds a tree over triangle pieces.
        slivers = scenes.records([(0, 0, 0), (0, 0, 0)], [(1, 1, 1), (0.5, 0.3, 1.2)], [(1.01, 1, 1), (0.5, 0.31, 1.2)])
        warm.initialize(np.concatenate([small[0], slivers]), 32, 32)
        warm.render(small[1], small[2])
    s = Session(lib)
    if args.pieces is not None:
        s.set_tuning(pieces=args.pieces)
    if args.leaf is not None:
        s.set_tuning(leaf=args.leaf)
    if args.lanes is not None:
        s.set_tuning(lanes=args.lanes)
    if args.refill is not None:
        s.set_tuning(refill=args.refill)
    if args.paths is not None:
        s.set_tuning(paths_in_flight=args.paths)
    lanes = args.lanes if args.lanes is not None else 2  # RTX_TUNE_LANES default
    t_init = time.perf_counter()
    s.initialize(tris, w, h)
    init_wall_ms = (time.perf_counter() - t_init) * 1e3
    bvh = s.bvh_stats()
    # Integrator choice: both give identical sums; pick the faster on warm-up.
    candidates = {'wavefront': 0, 'megakernel': 1}
    if args.integrator != 'auto':
        candidates = {args.integrator: candidates[args.integrator]}
    flush, l2_note = l2_flusher()
    best, best_ms = None, None
    for name, mode in candidates.items():
        s.set_integrator(mode)
        times = []
        for _ in range(max(args.warmup, 1)):
            flush()
            times.append(s.render_device(cam, settings))
        ms = min(times)
        if best_ms is None or ms < best_ms:
            best, best_ms = name, ms
    s.set_integrator(candidates[best])
    for _ in range(args.warmup):
        flush()
        s.render_device(cam, settings)
    # Timed region: K passes, device time from CUDA events around each pass.
    gpu_index = int((os.environ.get('CUDA_VISIBLE_DEVICES') or str(local_rank)).split(',')[0]) if world > 1 else 0
    if world == 1 and os.environ.get('CUDA_VISIBLE_DEVICES'):
        gpu_index = int(os.environ['CUDA_VISIBLE_DEVICES'].split(',')[0])
    clocks = Clocks(gpu_index)
    rays = launches = 0
    device_ms = extend_ms = shadow_ms = primary_ms = 0.0
    per_kind = {'primaryRays': 0, 'secondaryRays': 0, 'shadowRays': 0}
    dist.barrier()
    clocks.start()
    wall0 = time.perf_counter()
    for _ in range(args.steps):
        flush()
        device_ms += s.render_device(cam, settings)
        st = s.render_stats()
        rays += st['primaryRays'] + st['secondaryRays'] + st['shadowRays']
        for k in per_kind:
            per_kind[k] += st[k]
        launches += st['kernelLaunches']
        extend_ms += st['extendMs']
        shadow_ms += st['shadowMs']
        primary_ms += st['primaryMs']
    wall = time.perf_counter() - wall0
    clock_info = clocks.stop()
    dist.barrier()
    t_max = dist.max(device_ms)
    total_rays = dist.sum(rays)
    value = total_rays / t_max / 1e3
    # End to end: RtRender through the C ABI into pinned host memory.
    out_buf, pinned = None, False
    try:
        import torch
        if torch.cuda.is_available():
            t = torch.empty(w * h * 4, dtype=torch.uint8, pin_memory=True)
            out_buf = np.frombuffer((c.c_ubyte * (w * h * 4)).from_address(t.data_ptr()), np.uint8)
            pinned = True
    except Exception:
        pass
    if out_buf is None:
        out_buf = np.zeros(w * h * 4, np.uint8)
    for _ in range(args.warmup):
        s.render(cam, settings, output=out_buf)
    dist.barrier()
    e2e_rays = 0
    e0 = time.perf_counter()
    for _ in range(args.steps):
        s.render(cam, settings, output=out_buf)
        st = s.render_stats()
        e2e_rays += st['primaryRays'] + st['secondaryRays'] + st['shadowRays']
    e2e_s = dist.max(time.perf_counter() - e0)
    e2e_value = dist.sum(e2e_rays) / e2e_s / 1e6
    # The dominant kernel alone: with one lane of waves no launch shares the
    # GPU, so its CUDA-event durations are the kernel's own (after the timed
    # region; every rank takes the same steps).
    isolated = None
    if best == 'wavefront' and lanes > 1:
        s.set_tuning(lanes=1)
        iso_ms, iso_rays = 0.0, 0
        iso_kind = {'primaryRays': 0, 'secondaryRays': 0, 'shadowRays': 0}
        iso_primary = iso_shadow = 0.0
        for _ in range(min(args.steps, 5)):
            flush()
            s.render_device(cam, settings)
            st = s.render_stats()
            iso_ms += st['extendMs']
            iso_primary += st['primaryMs']
            iso_shadow += st['shadowMs']
            iso_rays += st['primaryRays'] + st['secondaryRays']
            for k in iso_kind:
                iso_kind[k] += st[k]
        s.set_tuning(lanes=lanes)
        isolated = (iso_ms, iso_rays, kernel_rates(best, iso_kind, iso_primary, iso_ms, iso_shadow, 1))
    peak, peak_kind = measured_peaks()
    result = None
    if rank == 0:
        alg = algorithmic_bytes(tris, cam, settings, w, h)
        if best == 'wavefront':
            kernel = 'extendKernel (closest-hit traversal)'
            closest = per_kind['primaryRays'] + per_kind['secondaryRays']
            achieved = closest * alg['closest'] / (extend_ms / 1e3) / 1e9 if extend_ms > 0 else None
        else:
            kernel = 'megakernel (closest + shadow traversal and shading)'
            achieved = ((per_kind['primaryRays'] + per_kind['secondaryRays']) * alg['closest'] +
                        per_kind['shadowRays'] * alg['shadow']) / (device_ms / 1e3) / 1e9
        # DRAM traffic of the dominant kernel per launch, from the committed
        # ncu summary (bytes per ray of a capture of this kernel), scaled to
        # the rays of one launch here.
        closest_step = (per_kind['primaryRays'] + per_kind['secondaryRays']) / args.steps
        if best == 'wavefront':
            paths = w * h * settings.raysPerPixel
            waves = -(-paths // min(args.paths or (1 << 24), paths))  # RTX_TUNE_PATHS_IN_FLIGHT default 2^24
            launches_step = waves * settings.maxBounces  # one closest-hit launch per bounce of a wave
            rays_per_launch = closest_step / launches_step
        else:
            rays_per_launch = sum(per_kind.values()) / args.steps
        traffic = None
        tfile = ROOT / 'profiles' / 'traffic.json'
        if tfile.exists():
            tdata = json.loads(tfile.read_text()).get(best)
            if tdata:
                traffic = tdata['dram_bytes_per_ray'] * rays_per_launch
        iso = None
        if isolated and isolated[0] > 0:
            iso_achieved = isolated[1] * alg['closest'] / (isolated[0] / 1e3) / 1e9
            iso = {'achieved': iso_achieved, 'frac': iso_achieved / peak, 'lanes': 1,
                   'note': 'extendKernel timed with one lane of waves (no overlap), outside the timed region'}
        roofline = {'bound': 'hbm', 'kernel': kernel, 'achieved': achieved, 'peak': peak, 'unit': 'GB/s',
                    'frac': (achieved / peak) if achieved else None, 'traffic': traffic,
                    'peak_source': f'{peak_kind} hbm_gbs (MEASURED_PEAKS.json)' if peak_kind == 'measured' else
                                   'fallback 6.65 TB/s',
                    'bytes_per_closest_query': alg['closest'], 'bytes_per_shadow_query': alg['shadow'],
                    'model': '64 B per interior node + 44 B per triangle the reference traversal visits',
                    'launch_timing': ('CUDA events around each launch; two lanes of waves overlap, so a launch '
                                      'shares the GPU with the other lane for part of its duration and achieved is '
                                      'a lower bound' if lanes > 1 else 'CUDA events around each launch, one lane'),
                    'isolated': iso,
                    'sample_pixels': alg['sample_pixels']}
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            cpu = cpu_baseline(tris, cam, settings, w, h, args.cpu_seconds)
            cpu.pop('seconds', None)
            cpu.pop('rays', None)
        ref_cuda = None
        if world == 1 and not args.no_reference_cuda:
            # This library's first pass of the same settings, for the parity check.
            s.lib.RtReset(s.handle)
            first_rgba, _ = s.render(cam, settings)
            first_pass = (s.accumulation(), first_rgba.copy())
            try:
                ref_cuda = reference_cuda(tris, cam, settings, w, h, rays / args.steps, first_pass)
            except Exception as exc:
                ref_cuda = {'unavailable': str(exc)}
        result = {
            'metric': METRIC, 'value': value, 'unit': METRIC, 'n_gpus': world, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': t_max / args.steps, 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic (seeded procedural scene)',
            'config': {'workload': WORKLOAD, 'triangles': len(tris), 'width': w, 'height': h,
                       'spp_per_step': settings.raysPerPixel, 'max_depth': settings.maxBounces,
                       'integrator': best, 'l2': l2_note, 'parallelism': f'replicas x{world}'},
            'e2e': {'value': e2e_value, 'unit': METRIC, 'h2d_bytes_per_step': 64 + 28,
                    'd2h_bytes_per_step': w * h * 4, 'pinned_output': pinned},
            'gpu_launches': launches,
            'clocks': clock_info,
            'roofline': roofline,
            'cpu_baseline': cpu,
            'rays': {k: v // args.steps for k, v in per_kind.items()},
            'traversal_mrays_per_s': dict(kernel_rates(best, per_kind, primary_ms, extend_ms, shadow_ms, lanes) or {},
                                          isolated=isolated[2] if isolated else None),
            'wall_ms_per_step': wall * 1e3 / args.steps,
            'build': build_report(tris, bvh, init_wall_ms, peak, peak_kind),
            'reference_cuda': ref_cuda,
            'config1': guarded(config1_run, lib) if (not args.no_cpu_baseline and world == 1) else None,
            'time_to_35db': quality_run(lib, args) if (args.quality and world == 1) else None,
            'batch': batch_run(lib, args) if (args.batch and world == 1) else None,
            'denoiser': denoiser_run(lib, args) if (args.denoiser and world == 1) else None,
            'train_step': train_step_run(lib, args) if (args.train_step and world == 1) else None,
        }
    s.close()
    dist.close()
    return result


def run_reference(args, rank, world):
    """The reference's own CPU implementation on this machine's host cores."""
    if rank != 0:
        return None
    from oracle_api import Oracle, Reference, reference_available
    tris, cam, settings, w, h = workload(args)
    kind = 'reference' if reference_available() else 'port'
    impl = Reference() if kind == 'reference' else Oracle()
    threads = impl.max_threads()
    sc = impl.scene(tris)
    t0 = time.perf_counter()
    impl.render(sc, cam, settings, w, h, rows=(h // 2, h // 2 + 1), threads=threads)
    per_row = max(time.perf_counter() - t0, 1e-4)
    budget = max(0.5, 60.0 / max(1, args.steps + args.warmup))
    stride = max(1, int(h / max(1, budget / per_row)))
    rows = sample_rows(h, stride)
    for _ in range(args.warmup):
        for y in rows[:1]:
            impl.render(sc, cam, settings, w, h, rows=(y, y + 1), threads=threads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        for y in rows:
            impl.render(sc, cam, settings, w, h, rows=(y, y + 1), threads=threads)
        times.append(time.perf_counter() - t0)
    sc.close()
    o = Oracle()
    osc = o.scene(tris)
    rays = 0
    for y in rows:
        _, _, counts = o.render(osc, cam, settings, w, h, rows=(y, y + 1))
        rays += int(counts[0] + counts[1] + counts[2])
    osc.close()
    total = sum(times)
    value = rays * args.steps / total / 1e6
    sample = f'{len(rows)} of {h} rows (every {stride}th) x {w} px x {settings.raysPerPixel} spp per step'
    return {
        'impl': 'reference', 'metric': METRIC, 'value': value, 'unit': METRIC, 'n_gpus': world,
        'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': total * 1e3 / args.steps,
        'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32',
        'data': 'synthetic (seeded procedural scene)',
        'config': {'workload': WORKLOAD, 'triangles': len(tris), 'width': w, 'height': h,
                   'spp_per_step': settings.raysPerPixel, 'max_depth': settings.maxBounces,
                   'parallelism': 'host cores'},
        'cpu_baseline': {'value': value, 'unit': METRIC, 'cores': threads, 'kind': kind, 'sample': sample},
        'e2e': {'value': value, 'unit': METRIC, 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0},
    }


def main():
    args = parse()
    if args.conv_path:
        from native_api import load_library
        load_library().RtxSetConvPath(args.conv_path)
    rank, local_rank, world = dist_env()
    if world > 1 and args.impl == 'ours':
        os.environ['CUDA_VISIBLE_DEVICES'] = str(local_rank) if 'CUDA_VISIBLE_DEVICES' not in os.environ else \
            os.environ['CUDA_VISIBLE_DEVICES'].split(',')[local_rank]
    if args.denoiser_only:
        from native_api import load_library
        result = denoiser_run(load_library(), args) if rank == 0 else None
    elif args.train_step_only:
        from native_api import load_library
        result = train_step_run(load_library(), args) if rank == 0 else None
    elif args.build_only:
        from native_api import load_library
        result = build_only_run(load_library(), args) if rank == 0 else None
    elif args.impl == 'reference':
        result = run_reference(args, rank, world)
    else:
        result = run_ours(args, rank, local_rank, world)
    if rank == 0 and result is not None:
        print(json.dumps(result), flush=True)
        ref_cuda = result.get('reference_cuda') or {}
        if ref_cuda.get('parity') is False:
            sys.exit('parity failure: the reference CUDA renderer accumulated different bytes on the bench workload')


if __name__ == '__main__':
    main()
