"""Reduced-precision storage (FP32 collision, shifted FP16/BF16/FP32 populations)
against the FP64 plain path on a converged porous medium.

Bounds (relative error of the steady permeability K = nu <u_x> / g against
FP64): FP32 storage 1e-5, FP16 1e-3 (the accuracy a 16-bit time-to-permeability
run must reach), BF16 2e-2 (8-bit mantissa; reported, not a target).  FP16 and
BF16 round stochastically.  The FP64 path itself is pinned to the reference
elsewhere.
"""
import numpy as np
import pytest

from cases import porous_scsp

pytestmark = pytest.mark.gpu

BOUNDS = {'fp32': 1e-5, 'bfp16': 1e-4, 'fp16': 1e-3, 'bf16': 2e-2}


def _run(storage, case, steps):
    from lbflow_b200 import Engine
    from lbflow_b200.permeability import permeability
    with Engine(case['geometry'], case['labels'], model='scsp', collision=case['collision'],
                tau=case['tau'], rho=case['rho'], storage=storage) as e:
        e.initialize()
        e.step(steps, macros=True)
        e.check()
        r0, _, u = e.macros()
        return permeability(e, case['tau'][0], 1e-5), r0, u


@pytest.fixture(scope='module')
def medium():
    return porous_scsp('MRT', n=(48, 48, 48), seed=21)


@pytest.fixture(scope='module')
def fp64_ref(medium):
    return _run('fp64', medium, 6000)


@pytest.mark.parametrize('storage', ['fp32', 'bfp16', 'fp16', 'bf16'])
def test_reduced_precision_permeability(medium, fp64_ref, storage):
    K64, r64, u64 = fp64_ref
    K, r, u = _run(storage, medium, 6000)
    assert K > 0 and K64 > 0
    err = abs(K - K64) / K64
    print(f'{storage}: K = {K:.9e}, FP64 K = {K64:.9e}, relative error {err:.3e}')
    assert err < BOUNDS[storage]
    # Field-level agreement (fluid voxels), loose: reported for the record.
    fl = r64 > 0
    uerr = np.max(np.abs(u[:, fl] - u64[:, fl])) / np.max(np.abs(u64))
    print(f'{storage}: max |du| / max|u| = {uerr:.3e}')
    assert uerr < 50 * BOUNDS[storage]


@pytest.mark.parametrize('storage', ['fp32', 'bfp16', 'fp16', 'bf16'])
def test_reduced_precision_initial_state(storage):
    """t = 0 of the shifted storage expands back to the FP64 initial populations."""
    from lbflow_b200 import Engine
    case = porous_scsp('MRT', n=(16, 16, 12), seed=7)
    with Engine(case['geometry'], case['labels'], collision='MRT', tau=(1.0,), storage='fp64') as a, \
            Engine(case['geometry'], case['labels'], collision='MRT', tau=(1.0,), storage=storage) as b:
        a.initialize()
        b.initialize()
        fa, fb = a.populations(), b.populations()
        tol = {'fp32': 1e-7, 'bfp16': 1e-7, 'fp16': 1e-6, 'bf16': 1e-5}[storage]
        assert np.max(np.abs(fa - fb)) < tol


@pytest.mark.parametrize('storage', ['fp16', 'bfp16'])
def test_set_get_roundtrip_reduced_precision(storage):
    from lbflow_b200 import Engine
    case = porous_scsp('MRT', n=(16, 16, 12), seed=7)
    with Engine(case['geometry'], case['labels'], collision='MRT', tau=(1.0,), storage='fp64') as a, \
            Engine(case['geometry'], case['labels'], collision='MRT', tau=(1.0,), storage=storage) as b:
        a.initialize()
        a.step(50)
        f = a.populations()
        b.set_populations(f)
        g = b.populations()
        fl = case['geometry'] != 255
        w = np.array([12] + [2] * 6 + [1] * 12) / 36.0
        dev = np.abs(f - w[None, :, None, None, None])[:, :, fl].max()
        assert np.max(np.abs(g[:, :, fl] - f[:, :, fl])) <= dev * 1e-3 + 1e-9


def _color_porous(n=(64, 32, 32), seed=3):
    from lbflow_b200.geometry import porous_medium
    fluid = porous_medium(n, sigma=2.0, porosity=0.30, seed=seed)
    g = np.where(fluid, 76, 255).astype(np.uint8)
    g[:n[0] // 3][fluid[:n[0] // 3]] = 75
    labels = {75: ('GV', 2e-6, 5, 0), 76: ('GV', 2e-6, 5, 1), 255: ('SD', 60.0, 0, 0)}
    return g, labels


@pytest.mark.parametrize('steps', [1, 50, 400])
def test_color_fp32_storage_tracks_fp64(steps):
    """Two-phase color-gradient run with FP32 populations and arithmetic
    against FP64: no device error, phase-0 mass and the phase-weighted flux
    (porous_media.py:33-41) close to FP64."""
    from lbflow_b200 import Engine
    g, labels = _color_porous()
    out = {}
    for storage in ('fp64', 'fp32'):
        with Engine(g, labels, model='color', collision='MRT', tau=(1.0, 0.7), rho=(1.0, 1.0), alpha0=1 / 3,
                    sigma=1e-3, beta=0.7, storage=storage) as e:
            e.initialize()
            e.step(steps, macros=True)
            bits = e.status()
            r0, r1, u = e.macros()
            out[storage] = (bits, r0, r1, u)
    assert out['fp64'][0] == 0
    assert out['fp32'][0] == 0, f'device error word {out["fp32"][0]:#x}'
    m64, m32 = out['fp64'][1].sum(), out['fp32'][1].sum()
    assert abs(m32 - m64) <= 1e-5 * m64
    du = np.abs(out['fp32'][3] - out['fp64'][3]).max() / max(np.abs(out['fp64'][3]).max(), 1e-30)
    print(f'steps {steps}: phase-0 mass rel diff {abs(m32 - m64) / m64:.2e}, max |du|/max|u| {du:.2e}')
    assert du < 1e-2


# Bounds of the two-phase quantities after 2,000 steps on the two-phase
# workload's recipe (relative to FP64): phase-0 saturation, change of the
# phase-0 mass over the run, phase-fraction-weighted Darcy flux of each phase
# along the force (porous_media.py:33-41).
COLOR_BOUNDS = {
    'fp32': dict(saturation=1e-5, mass_drift=1e-4, flux=1e-2),
    'fp16': dict(saturation=2e-3, mass_drift=2e-3, flux=5e-2),
    'bf16': dict(saturation=1e-2, mass_drift=1e-2, flux=2e-1),
}


@pytest.fixture(scope='module')
def color_fp64():
    return _color_run('fp64')


def _color_run(storage, steps=2000):
    from lbflow_b200 import Engine
    g, labels = _color_porous(n=(96, 48, 48), seed=8)
    with Engine(g, labels, model='color', collision='MRT', tau=(1.0, 0.7), rho=(1.0, 1.0), alpha0=1 / 3,
                sigma=1e-3, beta=0.7, storage=storage) as e:
        e.initialize()
        s0 = e.flux_sums()
        e.step(steps, macros=True)
        e.check()
        s1 = e.flux_sums()
        nf = e.fluid_nodes
    return dict(saturation=s1[8] / nf, mass0=s0[6], mass1=s1[6], flux0=s1[5], flux1=s1[2] - s1[5])


@pytest.mark.parametrize('storage', ['fp32', 'fp16', 'bf16'])
def test_color_reduced_storage_phase_measures(color_fp64, storage):
    """FP32 populations, and the 16-bit total + component-share storage,
    against FP64 on a crop of the two-phase workload's recipe: saturation,
    phase-0 mass drift and both phases' weighted Darcy fluxes."""
    ref = color_fp64
    got = _color_run(storage)
    b = COLOR_BOUNDS[storage]
    e_sat = abs(got['saturation'] - ref['saturation']) / ref['saturation']
    drift = (got['mass1'] - got['mass0']) / got['mass0']
    drift64 = (ref['mass1'] - ref['mass0']) / ref['mass0']
    e_f0 = abs(got['flux0'] - ref['flux0']) / abs(ref['flux0'])
    e_f1 = abs(got['flux1'] - ref['flux1']) / abs(ref['flux1'])
    print(f'{storage}: saturation {e_sat:.2e}, phase-0 mass drift {drift:.2e} (fp64 {drift64:.2e}), '
          f'phase flux errors {e_f0:.2e} / {e_f1:.2e}')
    assert e_sat < b['saturation']
    assert abs(drift - drift64) < b['mass_drift']
    assert e_f0 < b['flux'] and e_f1 < b['flux']
