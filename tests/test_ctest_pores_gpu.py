"""The reference's pore-flow CTest group (scripts/ctest_pores.py) run through
the LBFlow command-line binary: the two-slit bundle in 2D (single phase and
two phases with either viscosity ratio, scripts/porous_media.py:67-152), the
capillary-entry slit with PB boundaries on both sides and legacy walls
(:154-227) and the pressure-driven slit (test_cli.py). The acceptance checks
are the reference's, restated here: closed mass drift <= 5e-9, analytic
permeability and phase fluxes within 2e-6, phase fluxes summing to the
mixture Darcy velocity, and the late displacement of the entry slit going the
way the pressure ratio says."""
import math

import numpy as np
import pytest

from cases import entry_case, prm_text
from test_cli import read_vti, run_cli

pytestmark = pytest.mark.gpu


def bundle_case(taus):
    """bundle_cases at scale 1 in 2D: slits of width 8 and 16 in a 4 x 36 box."""
    h, ny, nx = 8, 36, 4
    widths = (h, 2 * h)
    force = 1e-6
    color = len(taus) == 2
    nu = [(t - 0.5) / 3 for t in taus]
    decay = max(widths[i] ** 2 / (nu[i % len(taus)] * math.pi ** 2) for i in (0, 1))
    steps = math.ceil(18 * decay / 1000) * 1000
    g = np.full((ny, nx), 255, np.uint8)
    g[4:4 + h, :] = 75
    g[8 + h:8 + 3 * h, :] = 76 if color else 75
    labels = {75: ('GV', force, 1, 0), 255: ('SD', 90.0, 0, 0)}
    if color:
        labels[76] = ('GV', force, 1, 1)
    return dict(name='bundle-' + '-'.join(map(str, taus)), geometry=g, labels=labels,
                model='color' if color else 'scsp', collision='MRT', tau=tuple(taus),
                rho=(1.0, 1.0) if color else (1.0,), alpha0=4 / 9, sigma=0.005, beta=0.7,
                steps=steps, write=steps // 2, widths=widths, force=force)


def fields(path, shape):
    """VTI arrays shaped (nz, ny, nx, components)."""
    _, arrays = read_vti(path)
    n = int(np.prod(shape))
    return {k: v.reshape(*shape, v.size // n) for k, v in arrays.items()}


def measure(a):
    """pore_measurement (porous_media.py:20-44)."""
    if 'v' in a:
        rho = a['r0'][..., 0] + a['r1'][..., 0]
        u = a['v']
    else:
        rho = a['density'][..., 0]
        u = a['velocity']
    pore = rho > 0
    m = dict(darcy=u.mean(axis=(0, 1, 2)), mass=rho.sum())
    if 'v' in a:
        phi = np.divide(a['r0'][..., 0], rho, out=np.zeros_like(rho), where=pore)
        fr = (phi, pore.astype(float) - phi)
        m['phase_mass'] = np.array([a['r0'].sum(), a['r1'].sum()])
        m['phase_flux'] = np.array([(f[..., None] * u).mean(axis=(0, 1, 2)) for f in fr])
        assert np.allclose(m['phase_flux'].sum(axis=0), m['darcy'], rtol=0, atol=1e-14)
    return m


def outputs(tmp, case):
    shape = (1,) + case['geometry'].shape if case['geometry'].ndim == 2 else case['geometry'].shape
    code, out = run_cli(tmp, case, prm_text(case))
    assert code == 0 and 'Simulation finished!' in out, out[-2000:]
    steps = range(0, case['steps'] + 1, case['write'])
    return [(t, fields(tmp / f'field.{t:010d}.vti', shape)) for t in steps]


@pytest.mark.parametrize('taus', [(1.0,), (0.6, 1.4), (1.4, 0.6)], ids=lambda t: '-'.join(map(str, t)))
def test_bundle_analytic_flux(tmp_path, taus):
    case = bundle_case(taus)
    hist = [(t, measure(a)) for t, a in outputs(tmp_path, case)]
    m0 = hist[0][1]
    for _, m in hist:       # closed mass audit (closed_history, porous_media.py:47-64)
        assert abs(m['mass'] - m0['mass']) / max(m0['mass'], 1.0) <= 5e-9
        if 'phase_mass' in m:
            assert np.all(np.abs(m['phase_mass'] - m0['phase_mass']) / np.maximum(m0['phase_mass'], 1.0) <= 5e-9)
    final = hist[-1][1]
    ny = case['geometry'].shape[0]
    weights = np.array([w ** 3 / 12 + w / 24 for w in case['widths']]) / ny
    nu = (np.array(taus) - 0.5) / 3
    if len(taus) == 1:
        k = nu[0] * final['darcy'][0] / case['force']
        assert abs(k / weights.sum() - 1) <= 2e-6
    else:
        q = final['phase_flux'][:, 0]
        assert np.max(np.abs(q / (case['force'] * weights / nu) - 1)) <= 2e-6


@pytest.mark.parametrize('ratio', [0.5, 1.5])
def test_capillary_entry_direction(tmp_path, ratio):
    """entry_study (porous_media.py:185-203): below the entry pressure
    (ratio 0.5) phase 0 recedes late in the run, above it (1.5) it advances."""
    case = entry_case(ratio, 2)
    h = case['height']
    lengths = []
    for _, a in outputs(tmp_path, case):
        rho = a['r0'][..., 0] + a['r1'][..., 0]
        phi = np.divide(a['r0'][..., 0], rho, out=np.zeros_like(rho), where=rho > 0)
        lengths.append(float(phi[0, 1:-1, 1:-1].sum() / h))
    late = lengths[-1] - lengths[-2]
    assert (ratio - 0.999) * late > 0
