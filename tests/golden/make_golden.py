#!/usr/bin/env python3
"""Regenerate the golden fixtures from the reference solver itself.

Runs the reference LBFlow binary (built from the reference sources by
`make -C oracle ref`) on every case of tests/cases.py:golden_cases() through
an input.prm written the way scripts/benchmarks.py writes one, and stores the
final post-collision populations (the .rst checkpoint) and the last VTI fields
as <case>.npz next to this script.  Run it in a checkout where oracle/_ref/
exists; the tests only read the .npz files.

    python tests/golden/make_golden.py            # every case + the CLI contracts
    python tests/golden/make_golden.py NAME ...   # only the named cases
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
    only = set(sys.argv[1:])
    index = json.loads((HERE / 'index.json').read_text()) if only else {}
    for case in golden_cases():
        if only and case['name'] not in only:
            continue
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
    if not only:
        cli_contracts(exe)


def run_ref(exe, case, prm=None, extra=None):
    """Run the reference on a case; return (exit code, stdout, {file: bytes})."""
    with tempfile.TemporaryDirectory() as d:
        d = Path(d)
        case['geometry'].tofile(d / 'geometry.raw')
        (d / 'input.prm').write_text(prm if prm is not None else prm_text(case))
        if extra:
            extra(d)
        r = subprocess.run([str(exe), 'input.prm'], cwd=d, capture_output=True, text=True)
        files = {p.name: p.read_bytes() for p in d.iterdir() if p.name.startswith('field')}
        return r.returncode, r.stdout, files


def cli_contracts(exe):
    """Reference behaviour of the command line: error messages of invalid
    inputs, VTI headers, checkpoint sidecars and report lines."""
    from cases import (force_cases, channel_mrt, wall_color_2d, porous_scsp, wall_color_3d, zou_he_cases,
                       pressure_report_channel, entry_case)
    import re
    out = {'errors': {}, 'vti_header': {}, 'meta': {}, 'reports': {}}
    base = force_cases()[7]          # force-scsp-d3-MRT-tau1.4
    cbase = force_cases()[-1]        # force-color-d3-MRT-tau1.4
    text = prm_text(base)
    ctext = prm_text(cbase)
    def sub(t, key, val):
        return re.sub(rf'^{key} .*;$', f'{key} {val};', t, flags=re.M)
    invalid = {
        'zero-write': (base, sub(text, 'writeInterval', '0')),
        'invalid-tau': (base, sub(text, 'rexlationTime', '0.5')),
        'invalid-speed': (base, sub(text, 'latticeSpeed', '2')),
        'invalid-alpha': (cbase, sub(ctext, 'alpha0', '1.1')),
        'invalid-color-tau': (cbase, sub(ctext, 'rexlationTime', '.5 .5')),
        'tau-count': (base, sub(text, 'rexlationTime', '1 1')),
        'bad-model': (base, sub(text, 'fluidModel', '"foo"')),
        'shanchen': (base, sub(text, 'fluidModel', '"shanchen"')),
        'bad-equil': (base, sub(text, 'equilModel', '"BGK"')),
        'bad-directions': (base, sub(text, 'directions', '15')),
        'short-geometry': (base, sub(text, 'dimension', '5 6 8')),
        'missing-geometry': (base, sub(text, 'gridFile', '"nothere.raw"')),
        'undefined-label': (base, text.replace('75 "GV"', '76 "GV"')),
        'bad-label-type': (base, text.replace('75 "GV"', '75 "XX"')),
        'bad-force-dir': (base, text.replace('"1" "0"', '"0" "0"')),
        'missing-key': (base, text.replace('stopError 1e-08;', '')),
        'report-slice': (base, sub(sub(text, 'reportDir', '3'), 'reportSlice', '1 6')),
        'report-dir': (base, sub(text, 'reportDir', '19')),
        'sd-angle': (channel_mrt(), prm_text(channel_mrt()).replace('"SD" "90"', '"SD" "190"')),
    }
    for name, (case, prm) in invalid.items():
        code, stdout, _ = run_ref(exe, case, prm)
        assert code != 0 and 'Simulation finished!' not in stdout, name
        msg = [l for l in stdout.splitlines() if 'Failed to excute: ' in l][-1].split('Failed to excute: ', 1)[1]
        out['errors'][name] = dict(prm=prm, message=msg, geometry_case=case['name'])
    for case in (channel_mrt(), wall_color_2d('MRT')):
        code, stdout, files = run_ref(exe, case)
        vti = files[f'field.{case["steps"]:010d}.vti']
        out['vti_header'][case['name']] = vti[:vti.index(b'>_') + 2].decode()
        out['meta'][case['name']] = files[f'field.{case["steps"]:010d}.rst.meta'].decode()
    for case, rdir in ((dict(porous_scsp('MRT'), report=50, steps=300), 1),
                       (dict(wall_color_3d(0.7, 'MRT'), report=50, steps=200), 1),
                       (dict(zou_he_cases()[0], report=50, steps=300), 1),
                       (dict(pressure_report_channel(), report=2000), 1),
                       (dict(entry_case(1.5, 2, steps=400, write=400), report=100), 1)):
        code, stdout, _ = run_ref(exe, case, prm_text(case, report_dir=rdir))
        lines = [l for l in stdout.splitlines() if l.startswith(' - ') or l.startswith('Step ')]
        out['reports'][case['name']] = dict(report_dir=rdir, report=case['report'], steps=case['steps'],
                                            lines=lines)
    (HERE / 'cli_contracts.json').write_text(json.dumps(out, indent=1, sort_keys=True) + '\n')


if __name__ == '__main__':
    main()
