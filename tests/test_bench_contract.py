"""bench.py's JSON line on CPU: the reference arm (the reference's own CPU
backend, or the oracle port where the reference is not compiled) prints one
line with the fields the benchmark contract names, on a small resolution of
the same 1,003,532-triangle workload; the per-kind rate helper of the GPU arm
is checked on made-up counts."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def test_reference_arm_json_line():
    cmd = [sys.executable, str(ROOT / 'bench.py'), '--impl', 'reference', '--steps', '1', '--warmup', '3',
           '--resolution', '64x48']
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line['impl'] == 'reference'
    for key in ('metric', 'value', 'unit', 'n_gpus', 'steps', 'warmup', 'ms_per_step', 'higher_is_better',
                'scaling', 'vs_baseline', 'dtype', 'data', 'config', 'cpu_baseline', 'e2e'):
        assert key in line, key
    assert line['metric'] == line['unit'] == 'Mrays/s' and line['value'] > 0 and line['higher_is_better']
    assert line['steps'] == 1 and line['warmup'] == 3 and line['n_gpus'] == 1
    cfg = line['config']
    assert cfg['workload'] == 'displaced_sphere_room' and cfg['triangles'] == 1003532
    assert (cfg['width'], cfg['height'], cfg['spp_per_step'], cfg['max_depth']) == (64, 48, 16, 3)
    cpu = line['cpu_baseline']
    assert cpu['kind'] in ('reference', 'port') and cpu['cores'] >= 1 and cpu['value'] == line['value']
    assert cpu['sample']
    e2e = line['e2e']
    assert e2e['value'] == line['value'] and e2e['unit'] == 'Mrays/s'
    assert e2e['h2d_bytes_per_step'] == 0 and e2e['d2h_bytes_per_step'] == 0


def test_kernel_rates():
    import bench
    kinds = {'primaryRays': 2_000_000, 'secondaryRays': 1_000_000, 'shadowRays': 3_000_000}
    r = bench.kernel_rates('wavefront', kinds, primary_ms=1.0, extend_ms=3.0, shadow_ms=2.0, lanes=2)
    assert (r['primary'], r['secondary'], r['shadow']) == (2000.0, 500.0, 1500.0)
    assert r['bound'] == 'lower' and r['lanes'] == 2
    assert bench.kernel_rates('wavefront', kinds, 1.0, 3.0, 2.0, 1)['bound'] == 'isolated'
    assert bench.kernel_rates('megakernel', kinds, 1.0, 3.0, 2.0, 1) is None
