"""The records of include/cuda_ray_tracer.h, compiled as C by the host
compiler, have the sizes and field offsets of their ctypes mirrors in
native_api (what Python callers bind): a field added to one side only, or a
changed type, fails here on the CPU."""
import shutil
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / 'custom-ray-tracing-shader_b200'))
import native_api  # noqa: E402

# C typedef name -> ctypes mirror
RECORDS = {
    'Triangle': native_api.Triangle,
    'CameraData': native_api.Camera,
    'RenderSettings': native_api.Settings,
    'PixelSum': native_api.PixelSum,
    'BvhNode': native_api.BvhNode,
    'RtxQuery': native_api.RtxQuery,
    'RtxHit': native_api.RtxHit,
    'RtxRenderStats': native_api.RtxRenderStats,
    'RtxBvhStats': native_api.RtxBvhStats,
    'RtxBatchTune': native_api.RtxBatchTune,
    'RtxBatchStats': native_api.RtxBatchStats,
}


@pytest.mark.skipif(shutil.which('gcc') is None, reason='no host C compiler')
def test_header_records_match_ctypes(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "cuda_ray_tracer.h"', 'int main(void) {']
    for cname, mirror in RECORDS.items():
        lines.append(f'    printf("{cname} size %zu\\n", sizeof({cname}));')
        for field, _ in mirror._fields_:
            lines.append(f'    printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ['    return 0;', '}']
    src = tmp_path / 'layouts.c'
    src.write_text('\n'.join(lines) + '\n')
    exe = tmp_path / 'layouts'
    build = subprocess.run(['gcc', '-std=c99', '-I', str(ROOT / 'include'), str(src), '-o', str(exe)],
                           capture_output=True, text=True)
    assert build.returncode == 0, build.stderr
    got = {}
    for line in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines():
        name, field, value = line.split()
        got[(name, field)] = int(value)
    for cname, mirror in RECORDS.items():
        assert got[(cname, 'size')] == native_api.c.sizeof(mirror), cname
        for field, _ in mirror._fields_:
            assert got[(cname, field)] == getattr(mirror, field).offset, (cname, field)
