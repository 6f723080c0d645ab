"""The LBFlow command line on the B200 engine against the reference's behaviour.

The reference's outputs for the same inputs are in tests/golden/ (errors,
VTI headers, checkpoint sidecars, report lines, fields and checkpoints).
Contracts follow scripts/ci_smoke.py (forcing, restart, failure cases) and
scripts/benchmarks.py (Study.run: exit code, "Simulation finished!",
LBFlowTiming, VTI fields).
"""
import json
import math
import re
import struct
import subprocess
from pathlib import Path

import numpy as np
import pytest

from cases import (channel_mrt, drop_3d, golden_cases, porous_scsp, pressure_report_channel, prm_text,
                   wall_color_2d, wall_color_3d)
from conftest import GOLDEN, fluid_mask, load_golden

ROOT = Path(__file__).resolve().parent.parent
CONTRACTS = json.loads((GOLDEN / 'cli_contracts.json').read_text())


def lbflow():
    exe = ROOT / 'lbflow_b200' / 'lib' / 'LBFlow'
    if not exe.exists():
        import lbflow_b200.build as b
        b.build()
    return exe


def run_cli(tmp, case, prm=None, extra=None, start=None):
    tmp.mkdir(parents=True, exist_ok=True)
    np.asarray(case['geometry'], np.uint8).tofile(tmp / 'geometry.raw')
    text = prm if prm is not None else prm_text(case)
    if start is not None:
        text = re.sub(r'^startTime .*;$', f'startTime {start};', text, flags=re.M)
    (tmp / 'input.prm').write_text(text)
    if extra:
        extra(tmp)
    r = subprocess.run([str(lbflow()), 'input.prm'], cwd=tmp, capture_output=True, text=True, timeout=600)
    return r.returncode, r.stdout


def read_vti(path):
    data = Path(path).read_bytes()
    head = data[:data.index(b'>_') + 2].decode()
    begin = len(head)
    arrays = {}
    for m in re.finditer(r'Name="(\w+)"(?: NumberOfComponents="(\d+)")? format="appended" offset="(\d+)"', head):
        off = begin + int(m.group(3))
        n = struct.unpack_from('<Q', data, off)[0] // 8
        arrays[m.group(1)] = np.frombuffer(data, '<f8', n, off + 8).copy()
    return head, arrays


# ---- contracts that fail before any GPU work (run on CPU) -----------------------
@pytest.mark.parametrize('name', sorted(CONTRACTS['errors']))
def test_invalid_input_same_message(tmp_path, name):
    spec = CONTRACTS['errors'][name]
    case = next(c for c in golden_cases() if c['name'] == spec['geometry_case'])
    code, out = run_cli(tmp_path, case, spec['prm'])
    assert code != 0
    assert 'Simulation finished!' not in out
    last = out.strip().splitlines()[-1]
    assert last.endswith('0 Failed to excute: ' + spec['message']), last


def test_no_argument_and_missing_file(tmp_path):
    r = subprocess.run([str(lbflow())], capture_output=True, text=True)
    assert r.returncode != 0 and 'you must specify an input filename' in r.stderr
    r = subprocess.run([str(lbflow()), str(tmp_path / 'absent.prm')], capture_output=True, text=True)
    assert r.returncode != 0 and 'FilePrm::Load() - Input file does not exist.' in r.stdout


def test_unsupported_options_are_refused(tmp_path):
    case = channel_mrt()
    for key, val in (('wallGradient', '"tanh"'), ('recoloringModel', '"projection"')):
        text = prm_text(case).replace('wallGradient "legacy";', f'{key} {val};')
        code, out = run_cli(tmp_path / key, case, text)
        assert code != 0 and 'not supported by the B200 engine' in out
    text = prm_text(case).replace('75 "GV" "9.9999999999999995e-07" "1" "0"', '75 "HF" "N/A" "N/A" "0"')
    assert '"HF"' in text
    code, out = run_cli(tmp_path / 'hf', case, text)
    assert code != 0 and 'HF' in out


# ---- GPU runs -----------------------------------------------------------------
def _timing(out):
    lines = [l for l in out.splitlines() if l.startswith('LBFlowTiming ')]
    assert len(lines) == 1
    return json.loads(lines[0][len('LBFlowTiming '):])


@pytest.mark.gpu
@pytest.mark.parametrize('case', [c for c in golden_cases() if not c['name'].startswith('wall-color-2d')],
                         ids=lambda c: c['name'])
def test_cli_matches_reference_outputs(tmp_path, case):
    gold = load_golden(case['name'])
    code, out = run_cli(tmp_path, case)
    assert code == 0 and 'Simulation finished!' in out, out[-2000:]
    t = case['steps']
    timing = _timing(out)
    assert timing['completed_steps'] == t and timing['ranks'] == 1
    assert timing['fluid_nodes'] == fluid_mask(case).sum() and timing['total_voxels'] == case['geometry'].size
    f = np.fromfile(tmp_path / f'field.{t:010d}.rst')
    fl = np.tile(fluid_mask(case).ravel(), f.size // case['geometry'].size)
    ref = gold['populations']
    assert np.max(np.abs(f[fl] - ref[fl]) / np.maximum(np.abs(ref[fl]), 1e-3)) <= 1e-12
    _, arrays = read_vti(tmp_path / f'field.{t:010d}.vti')
    for k, v in arrays.items():
        want = gold[f'vti_{k}']
        assert v.shape == want.shape
        scale = 1.0 if k in ('density', 'r0', 'r1') else 1.0
        assert np.max(np.abs(v - want)) <= 1e-12 * scale, k


@pytest.mark.gpu
@pytest.mark.parametrize('case', [porous_scsp('MRT'), porous_scsp('SRT')], ids=lambda c: c['name'])
def test_cli_checkpoint_with_solid_populations(tmp_path, case):
    """`solidPopulations "stream";`: the checkpoint holds the reference's
    values at solid voxels too (the whole .rst against the reference's)."""
    gold = load_golden(case['name'])
    code, out = run_cli(tmp_path, case, prm=prm_text(case) + 'solidPopulations "stream";\n')
    assert code == 0 and 'Simulation finished!' in out, out[-2000:]
    f = np.fromfile(tmp_path / f'field.{case["steps"]:010d}.rst')
    ref = gold['populations']
    assert f.shape == ref.shape
    assert np.max(np.abs(f - ref) / np.maximum(np.abs(ref), 1e-3)) <= 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize('case', [channel_mrt(), wall_color_2d('MRT')], ids=lambda c: c['name'])
def test_vti_header_and_sidecar_bytes(tmp_path, case):
    code, out = run_cli(tmp_path, case)
    assert code == 0, out[-2000:]
    t = case['steps']
    head, _ = read_vti(tmp_path / f'field.{t:010d}.vti')
    assert head == CONTRACTS['vti_header'][case['name']]
    assert (tmp_path / f'field.{t:010d}.rst.meta').read_text() == CONTRACTS['meta'][case['name']]
    assert (tmp_path / f'field.{0:010d}.vti').exists()


def _numbers(line):
    return [float(x) for x in re.findall(r'[-+]?\d+\.\d+(?:e[-+]\d+)?', line)]


@pytest.mark.gpu
@pytest.mark.parametrize('name', sorted(CONTRACTS['reports']))
def test_report_lines_match_reference(tmp_path, name):
    spec = CONTRACTS['reports'][name]
    base = {c['name']: c for c in golden_cases() + [pressure_report_channel()]}[name]
    case = dict(base, report=spec['report'], steps=spec['steps'])
    code, out = run_cli(tmp_path, case, prm_text(case, report_dir=spec['report_dir']))
    assert code == 0, out[-2000:]
    lines = [l for l in out.splitlines() if l.startswith(' - ') or l.startswith('Step ')]
    want = spec['lines']
    assert len(lines) == len(want)
    for got, ref in zip(lines, want):
        if ref.startswith('Step '):
            assert got.split(' - ')[0] == ref.split(' - ')[0]
            continue
        assert re.sub(r'[-+]?\d+\.\d+(e[-+]\d+)?', '#', got) == re.sub(r'[-+]?\d+\.\d+(e[-+]\d+)?', '#', ref)
        for a, b in zip(_numbers(got), _numbers(ref)):
            assert math.isclose(a, b, rel_tol=2e-5, abs_tol=2e-6), (got, ref)


@pytest.mark.gpu
def test_pressure_study_acceptance(tmp_path):
    """scripts/porous_media.py:257-279: the pressure-driven slit reports the
    prescribed pressure drop between its report slices and the analytic slit
    permeability, each within 2e-4."""
    case = pressure_report_channel()
    code, out = run_cli(tmp_path, case, prm_text(case, report_dir=1))
    assert code == 0, out[-2000:]
    dp = float(re.findall(r' - dP = ([\deE+.-]+)', out)[-1])
    k = float(re.findall(r' - K = ([\deE+.-]+)', out)[-1])
    h, nx = case['h'], case['geometry'].shape[2]
    assert abs(dp / (case['dp'] * (nx - 3) / (nx - 1)) - 1) <= 2e-4
    assert abs(k / ((h ** 3 / 12 + h / 24) / (h + 2)) - 1) <= 2e-4


@pytest.mark.gpu
def test_restart_and_failure_contracts(tmp_path):
    """scripts/ci_smoke.py:50-116: resuming from the step-20 checkpoint gives the
    continuous run's fields bit for bit; corrupted checkpoints are refused."""
    n = 12
    z, y, x = np.mgrid[0:n, 0:n, 0:n]
    g = np.where((x - 5.5) ** 2 + (y - 5.5) ** 2 + (z - 5.5) ** 2 <= 9, 100, 0).astype(np.uint8)
    case = dict(drop_3d(), geometry=g, steps=40, write=20, restart=20)
    code, out = run_cli(tmp_path / 'cont', case)
    assert code == 0, out[-2000:]
    cp = tmp_path / 'cont' / 'field.0000000020'

    def copy_cp(src_rst, src_meta):
        def f(d):
            (d / 'field.0000000020.rst').write_bytes(src_rst)
            (d / 'field.0000000020.rst.meta').write_text(src_meta)
        return f
    rst = Path(str(cp) + '.rst').read_bytes()
    meta = Path(str(cp) + '.rst.meta').read_text()
    code, out = run_cli(tmp_path / 'resumed', case, extra=copy_cp(rst, meta), start=20)
    assert code == 0, out[-2000:]
    assert _timing(out)['completed_steps'] == 20
    _, a = read_vti(tmp_path / 'cont' / 'field.0000000040.vti')
    _, b = read_vti(tmp_path / 'resumed' / 'field.0000000040.vti')
    for k in a:
        assert np.array_equal(a[k].view(np.uint64), b[k].view(np.uint64)), k
    for name, (r, m) in {'missing-stage': (rst, 'NO_VALID_STAGE\n'),
                         'short-populations': (rst[:-8], meta),
                         'nonfinite-population': (struct.pack('<d', float('nan')) + rst[8:], meta)}.items():
        code, out = run_cli(tmp_path / name, case, extra=copy_cp(r, m), start=20)
        assert code != 0 and 'Simulation finished!' not in out, name
