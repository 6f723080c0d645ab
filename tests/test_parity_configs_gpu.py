"""Parity of the CUDA engine with the oracle on the benchmark workloads' own
recipes, at sizes the oracle finishes in seconds.

- The 256^3 single-phase cube's recipe (sigma 3, porosity 0.22, MRT tau 1,
  g_x 1e-5, periodic) at 64^3, FP64, 1000 steps: populations within 1e-12
  relative, velocities within 1e-13 absolute, and the permeability
  K = nu <u_x> / g_x (scripts/rock_workflow.py:60-66, the mean over all
  voxels) within 1e-10 relative.  64 voxels in x are two occupancy words per
  row, so pulls cross word boundaries and the periodic wrap in x.
- A box whose x extent (80) is not a multiple of 32, so the last occupancy
  word of every row is partial: SRT, 1000 steps, same bars.
- The two-phase workload's recipe (sigma 2, porosity 0.30, the inlet third
  along z phase A, tau 1 / 0.7, A 1e-3, beta 0.7, 60-degree walls, g_z 2e-6)
  on a 32 x 32 x 64 crop, color MRT, 300 steps: populations within the color
  tolerance (10x the oracle's own response to a 1e-16 perturbation, never
  below 1e-12), and the pore measures of scripts/porous_media.py:20-44 --
  Darcy velocity, both phases' advective Darcy fluxes mean(phi_k u), phase
  masses and saturation -- within 1e-10 relative, from the engine's device
  reduction (lbf_flux_sums) against exactly rounded sums of the oracle's
  fields.
"""
import math

import numpy as np
import pytest

from conftest import fluid_mask
from oracle_port import Oracle
from test_parity_gpu import (assert_macros_close, assert_populations_close, engine_for,
                             population_tolerance)

pytestmark = pytest.mark.gpu


def cube_recipe(n=64, seed=0):
    from lbflow_b200.geometry import porous_medium
    fluid = porous_medium((n, n, n), sigma=3.0, porosity=0.22, seed=seed)
    return dict(name=f'cube-recipe-{n}', geometry=np.where(fluid, 75, 255).astype(np.uint8),
                labels={75: ('GV', 1e-5, 1, 0), 255: ('SD', 90.0, 0, 0)}, model='scsp', collision='MRT',
                tau=(1.0,), rho=(1.0,))


def ragged_box(seed=4):
    from lbflow_b200.geometry import porous_medium
    fluid = porous_medium((20, 36, 80), sigma=2.5, porosity=0.3, seed=seed)
    return dict(name='ragged-80x36x20', geometry=np.where(fluid, 75, 255).astype(np.uint8),
                labels={75: ('GV', 1e-5, 1, 0), 255: ('SD', 90.0, 0, 0)}, model='scsp', collision='SRT',
                tau=(0.8,), rho=(1.0,))


def color_recipe(nx=32, ny=32, nz=64, seed=0):
    from lbflow_b200.geometry import porous_medium
    fluid = porous_medium((nz, ny, nx), sigma=2.0, porosity=0.30, seed=seed)
    g = np.where(fluid, 76, 255).astype(np.uint8)
    inlet = nz // 3
    g[:inlet][fluid[:inlet]] = 75
    return dict(name=f'color-recipe-{nx}x{ny}x{nz}', geometry=g,
                labels={75: ('GV', 2e-6, 5, 0), 76: ('GV', 2e-6, 5, 1), 255: ('SD', 60.0, 0, 0)},
                model='color', collision='MRT', tau=(1.0, 0.7), rho=(1.0, 1.0), alpha0=1 / 3, sigma=1e-3,
                beta=0.7)


def pore_sums(r0, r1, u, fl):
    """The nine sums of lbf_flux_sums over the fluid voxels, exactly rounded:
    sum u (x, y, z), sum phi0 u, sum rho0, sum rho1, sum phi0 (phi0 = rho0/rho
    for two phases, 1 for one)."""
    r0f = r0[fl]
    uf = [u[c][fl] for c in range(3)]
    if r1 is not None:
        r1f = r1[fl]
        phi0 = r0f / (r0f + r1f)
    else:
        r1f = np.zeros(1)
        phi0 = np.ones_like(r0f)
    parts = uf + [phi0 * v for v in uf] + [r0f, r1f, phi0]
    return np.array([math.fsum(p.tolist()) for p in parts])


@pytest.mark.parametrize('make', [cube_recipe, ragged_box], ids=['cube-recipe-64', 'ragged-80x36x20'])
def test_single_phase_recipe_1000_steps(make):
    case = make()
    o = Oracle(case)
    o.start()
    o.step(1000)
    fl = fluid_mask(case)
    with engine_for(case) as e:
        e.initialize()
        e.step(1000, macros=True)
        e.check()
        assert_populations_close(e.populations(), o.populations(), fl)
        got, want = e.macros(), o.macros()
        assert_macros_close(got, want, fl)
        sums = e.flux_sums()
    nu = (case['tau'][0] - 0.5) / 3
    g = case['labels'][75][1]
    n = fl.size
    k_want = nu * math.fsum(want[2][0].ravel().tolist()) / n / g
    k_got = nu * sums[0] / n / g
    assert k_want > 0
    assert abs(k_got - k_want) <= 1e-10 * abs(k_want), (k_got, k_want)
    ref = pore_sums(*want, fl)
    assert abs(sums[6] - ref[6]) <= 1e-12 * ref[6]


def test_color_recipe_pore_measures():
    case = color_recipe()
    steps = 300
    o = Oracle(case)
    o.start()
    o.step(steps)
    fl = fluid_mask(case)
    rtol = population_tolerance(case, steps)
    with engine_for(case) as e:
        e.initialize()
        e.step(steps, macros=True)
        e.check()
        assert_populations_close(e.populations(), o.populations(), fl, rtol)
        want = o.macros()
        assert_macros_close(e.macros(), want, fl, rtol)
        got = e.flux_sums()
    ref = pore_sums(*want, fl)
    n = fl.size
    # Darcy velocity and the phases' advective fluxes, mean over all voxels
    # (porous_media.py:27-41): relative to the flow (z) component's magnitude.
    for k in (0, 3):
        scale = abs(ref[k + 2])
        assert scale > 0
        for c in range(3):
            assert abs(got[k + c] - ref[k + c]) <= 1e-10 * scale, (k, c, got[k + c], ref[k + c])
    flux1 = ref[:3] - ref[3:6]
    assert abs((got[2] - got[5]) - flux1[2]) <= 1e-10 * abs(ref[2])
    # Phase masses and the phase-0 saturation.
    for k in (6, 7, 8):
        assert abs(got[k] - ref[k]) <= 1e-12 * abs(ref[k]), (k, got[k], ref[k])
    # Mixture K from the Darcy velocity along the force, with the
    # saturation-weighted viscosity.
    s0 = ref[8] / fl.sum()
    nu = (s0 * (case['tau'][0] - 0.5) + (1 - s0) * (case['tau'][1] - 0.5)) / 3
    k_want, k_got = nu * ref[2] / n / 2e-6, nu * got[2] / n / 2e-6
    assert abs(k_got - k_want) <= 1e-10 * abs(k_want)
