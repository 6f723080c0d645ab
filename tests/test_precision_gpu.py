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
