"""The C restatement oracle against the reference solver's own outputs.

The golden fixtures were produced by the reference LBFlow binary (see
tests/golden/make_golden.py).  The oracle must reproduce them bit for bit on
every fluid voxel -- that pins it before it is trusted as the engine's checker.
"""
import numpy as np
import pytest

from cases import golden_cases
from conftest import fluid_mask, load_golden
from oracle_port import Oracle

CASES = golden_cases()


def _vti_fields(case, gold):
    """Golden VTI arrays as dense (rho0, rho1, u[3]) in (nz, ny, nx)."""
    g = np.asarray(case['geometry'])
    shape = g.shape if g.ndim == 3 else (1,) + g.shape
    if 'vti_density' in gold:
        r0, r1, uv = gold['vti_density'], None, gold['vti_velocity']
    else:
        r0, r1, uv = gold['vti_r0'], gold['vti_r1'], gold['vti_v']
    n = int(np.prod(shape))
    comps = uv.size // n          # 2 in 2D (x, y), 3 in 3D (x, y, z)
    u = np.zeros((3, n))
    u[:comps] = uv.reshape(n, comps).T
    u = u.reshape(3, *shape)
    return r0.reshape(shape), (r1.reshape(shape) if r1 is not None else None), u


@pytest.mark.parametrize('case', CASES, ids=[c['name'] for c in CASES])
def test_oracle_bitwise_against_reference(case):
    gold = load_golden(case['name'])
    o = Oracle(case)
    o.start()
    o.step(case['steps'])
    fl = fluid_mask(case).ravel()
    f = o.populations().reshape(o.phases * o.q, -1)
    ref = gold['populations'].reshape(o.phases * o.q, -1)
    assert np.array_equal(f[:, fl], ref[:, fl])
    r0, r1, u = o.macros()
    g0, g1, gu = _vti_fields(case, gold)
    assert np.array_equal(r0.ravel(), g0.ravel())
    assert np.array_equal(u.reshape(3, -1), gu.reshape(3, -1))
    if r1 is not None:
        assert np.array_equal(r1.ravel(), g1.ravel())


@pytest.mark.parametrize('case', [c for c in CASES if c['name'].startswith('force-')],
                         ids=lambda c: c['name'])
def test_force_integration_kat(case):
    """scripts/benchmarks.py:176-188: u_x = 1e-4 +- 1e-12, transverse <= 1e-12 after 100 steps."""
    gold = load_golden(case['name'])
    _, _, u = _vti_fields(case, gold)
    assert np.max(np.abs(u[0] - 1e-4)) <= 1e-12
    assert np.max(np.abs(u[1:])) <= 1e-12


def test_channel_config1_poiseuille():
    """Config 1: the reference's profile is Poiseuille to the SRT halfway-wall offset."""
    case = golden_cases()[0]
    gold = load_golden(case['name'])
    _, _, u = _vti_fields(case, gold)
    ux = u[0].mean(axis=(0, 2))[1:-1]
    tau, F, h = 0.8, 1e-6, 8
    nu = (tau - 0.5) / 3
    y = np.arange(h) + 0.5
    ideal = F / (2 * nu) * y * (h - y)
    rel = np.linalg.norm(ux - ideal) / np.linalg.norm(ideal)
    assert rel < 0.012
    assert abs(u[0].mean() - 4.248e-5) / 4.248e-5 < 1e-3
