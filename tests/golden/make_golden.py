#!/usr/bin/env python3
"""Regenerate the golden fixtures from the reference solver itself.

Runs the reference LBFlow binary (built from the reference sources by
`make -C oracle ref`) on every case of tests/cases.py:golden_cases() through
an input.prm written the way scripts/benchmarks.py writes one, and stores the
final post-collision populations (the .rst checkpoint) and the last VTI fields
as <case>.npz next to this script.  Run it in a checkout where oracle/_ref/
exists; the tests only read the .npz files.

    python tests/golden/make_golden.py
"""
import json
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(HERE.parent))
sys.path.insert(0, str(ROOT))
from cases import golden_cases, prm_text  # noqa: E402


def read_vti(path):
    """Minimal reader of the reference's appended-raw VTI (filevti.cpp:39-172)."""
    import struct
    import xml.etree.ElementTree as ET
    data = Path(path).read_bytes()
    pos = data.index(b'<AppendedData')
    doc = ET.fromstring(data[:pos] + b'</VTKFile>')
    begin = data.index(b'>_', pos) + 2
    out = {}
    for a in doc.find('ImageData').find('Piece').find('PointData').findall('DataArray'):
        off = begin + int(a.attrib['offset'])
        n = struct.unpack_from('<Q', data, off)[0] // 8
        out[a.attrib['Name']] = np.frombuffer(data, '<f8', n, off + 8).copy()
    return out


def main():
    exe = ROOT / 'oracle' / '_ref' / 'LBFlow'
    if not exe.exists():
        raise SystemExit('build the reference first: make -C oracle ref')
    index = {}
    for case in golden_cases():
        with tempfile.TemporaryDirectory() as d:
            d = Path(d)
            case['geometry'].tofile(d / 'geometry.raw')
            (d / 'input.prm').write_text(prm_text(case))
            r = subprocess.run([str(exe), 'input.prm'], cwd=d, capture_output=True, text=True)
            if r.returncode != 0:
                raise SystemExit(f'{case["name"]}: reference failed\n{r.stdout[-2000:]}')
            t = case['steps']
            f = np.fromfile(d / f'field.{t:010d}.rst', dtype='<f8')
            vti = read_vti(d / f'field.{t:010d}.vti') if t % case['write'] == 0 else {}
            timing = [json.loads(l[len('LBFlowTiming '):]) for l in r.stdout.splitlines()
                      if l.startswith('LBFlowTiming ')][0]
        np.savez_compressed(HERE / f'{case["name"]}.npz', populations=f, geometry=case['geometry'],
                            **{f'vti_{k}': v for k, v in vti.items()})
        index[case['name']] = dict(steps=t, fluid_nodes=timing['fluid_nodes'],
                                   total_voxels=timing['total_voxels'])
        print(case['name'], f.size, sorted(vti))
    (HERE / 'index.json').write_text(json.dumps(index, indent=1, sort_keys=True) + '\n')


if __name__ == '__main__':
    main()
