"""CUDA engine (through the C ABI) against the reference outputs and the oracle.

Tolerances: the plain FP64 path must match populations to 1e-12 relative
(absolute 1e-15 for populations below 1e-3, e.g. an absent color component)
and densities to 1e-12 relative.  A velocity is a sum of O(0.1) populations
divided by the density, so the population tolerance bounds its error in
absolute lattice units: velocities must agree to 1e-13 (about 1e-8 of a
typical 1e-5 pore velocity), and the mean velocity that defines the
permeability K = nu <u_x> / g to 1e-10 relative.  Link classification is
compared bit for bit.

Some two-phase wall cases are ill-conditioned in the reference algorithm
itself: the geometric wall rotation branches on the sign and vanishing of the
wall-frame gradient (colorfluid.cpp:550-567), so a 1e-16 change of the state
can move a population by 1e-9 within ten steps.  For those the population
tolerance is 10x the oracle's own response to a 1e-16 perturbation (never
below 1e-12); oracle_sensitivity() measures it.
"""
import numpy as np
import pytest

from cases import golden_cases, porous_scsp, wall_color_3d, drop_3d
from conftest import fluid_mask, load_golden
from oracle_port import Oracle

pytestmark = pytest.mark.gpu
CASES = golden_cases()


def engine_for(case, storage='fp64'):
    from lbflow_b200 import Engine
    return Engine(case['geometry'], case['labels'], model=case['model'], collision=case['collision'],
                  tau=case['tau'], rho=case['rho'], alpha0=case.get('alpha0', 1 / 3),
                  sigma=case.get('sigma', 0.0), beta=case.get('beta', 0.0), storage=storage)


def oracle_sensitivity(case, steps, seeds=3):
    """Largest relative population change the oracle itself shows after
    `steps` steps when its t = 0 state is perturbed by 1e-16 (relative)."""
    base = Oracle(case)
    base.start()
    base.step(steps)
    ref = base.populations()
    fl = fluid_mask(case)
    fl = np.broadcast_to((fl if fl.ndim == 3 else fl[None])[None, None], ref.shape)
    worst = 0.0
    for seed in range(seeds):
        o = Oracle(case)
        o.start()
        f = o.populations()
        o.set_populations(f * (1 + 1e-16 * np.random.default_rng(seed).standard_normal(f.shape)))
        o.step(steps)
        g = o.populations()
        worst = max(worst, float(np.max(np.abs(g[fl] - ref[fl]) / np.maximum(np.abs(ref[fl]), 1e-3))))
    return worst


def population_tolerance(case, steps):
    if case['model'] != 'color':
        return 1e-12
    return max(1e-12, 10 * oracle_sensitivity(case, steps))


def assert_populations_close(f, ref, fl, rtol=1e-12):
    q = f.shape[0] * f.shape[1]
    a = f.reshape(q, -1)[:, fl.ravel()]
    b = ref.reshape(q, -1)[:, fl.ravel()]
    err = np.abs(a - b) / np.maximum(np.abs(b), 1e-3)
    assert err.max() <= rtol, f'max relative population error {err.max():.3e}'


def assert_macros_close(got, want, fl, rtol=1e-12):
    vtol = 1e-13 * max(1.0, rtol / 1e-12)
    r0, r1, u = got
    w0, w1, wu = want
    m = fl
    # Densities relative to the total density (a component may be absent).
    scale = np.abs(w0[m] + (w1[m] if w1 is not None else 0))
    assert np.max(np.abs(r0[m] - w0[m]) / scale) <= rtol
    if w1 is not None:
        assert np.max(np.abs(r1[m] - w1[m]) / scale) <= rtol
    assert np.max(np.abs(u[:, m] - wu[:, m])) <= vtol
    mean, want_mean = u[0].mean(), wu[0].mean()
    assert abs(mean - want_mean) <= 1e-10 * abs(want_mean) * max(1.0, rtol / 1e-12) + 1e-16


def golden_macros(case, gold):
    g = np.asarray(case['geometry'])
    shape = g.shape if g.ndim == 3 else (1,) + g.shape
    n = int(np.prod(shape))
    if 'vti_density' in gold:
        r0, r1, uv = gold['vti_density'], None, gold['vti_velocity']
    else:
        r0, r1, uv = gold['vti_r0'], gold['vti_r1'], gold['vti_v']
    comps = uv.size // n
    u = np.zeros((3, n))
    u[:comps] = uv.reshape(n, comps).T
    return r0.reshape(shape), (r1.reshape(shape) if r1 is not None else None), u.reshape(3, *shape)


@pytest.mark.parametrize('case', CASES, ids=[c['name'] for c in CASES])
def test_engine_matches_reference(case):
    gold = load_golden(case['name'])
    fl = fluid_mask(case)
    fl3 = fl if fl.ndim == 3 else fl[None]
    with engine_for(case) as e:
        e.initialize()
        e.step(case['steps'], macros=True)
        e.check()
        f = e.populations()
        ref = gold['populations'].reshape(f.shape)
        rtol = population_tolerance(case, case['steps'])
        assert_populations_close(f, ref, fl3, rtol)
        assert_macros_close(e.macros(), golden_macros(case, gold), fl3, rtol)


@pytest.mark.parametrize('case', [CASES[i] for i in (1, 2, 3, 5, 7, 9)], ids=lambda c: c['name'])
def test_link_classification_bitwise(case):
    with engine_for(case) as e:
        m = e.link_mask()
    want = Oracle(case).link_mask()
    assert np.array_equal(m, want)


@pytest.mark.parametrize('case', [CASES[1], CASES[2], CASES[3]], ids=lambda c: c['name'])
def test_initial_macros(case):
    o = Oracle(case)
    want = o.start()
    fl = fluid_mask(case)
    fl3 = fl if fl.ndim == 3 else fl[None]
    with engine_for(case) as e:
        e.initialize()
        assert_macros_close(e.macros(), want, fl3)
        assert_populations_close(e.populations(), o.populations(), fl3)


@pytest.mark.parametrize('case', [porous_scsp('MRT', n=(24, 20, 16), seed=11),
                                  porous_scsp('SRT', n=(24, 20, 16), seed=11),
                                  wall_color_3d(0.7, 'MRT'), drop_3d()],
                         ids=lambda c: c['name'])
def test_thousand_steps(case):
    """Plain FP64 path: populations within 1e-12 relative after 1000 steps."""
    o = Oracle(case)
    o.start()
    o.step(1000)
    fl = fluid_mask(case)
    fl3 = fl if fl.ndim == 3 else fl[None]
    with engine_for(case) as e:
        e.initialize()
        e.step(1000, macros=True)
        e.check()
        assert_populations_close(e.populations(), o.populations(), fl3)
        assert_macros_close(e.macros(), o.macros(), fl3)


@pytest.mark.parametrize('case', [CASES[2], CASES[7]], ids=lambda c: c['name'])
def test_restart_continues_exactly(case):
    """Load a checkpoint mid-run (loadRst) and continue: same as an unbroken run."""
    o = Oracle(case)
    o.start()
    o.step(20)
    mid = o.populations()
    o.step(15)
    fl = fluid_mask(case)
    fl3 = fl if fl.ndim == 3 else fl[None]
    with engine_for(case) as e:
        e.set_populations(mid)
        e.step(15, macros=True)
        assert_populations_close(e.populations(), o.populations(), fl3)
        assert_macros_close(e.macros(), o.macros(), fl3)


def test_reductions_match_numpy():
    """Convergence, report-slice and flux sums against numpy on the same fields."""
    case = porous_scsp('MRT', n=(24, 20, 16), seed=5)
    with engine_for(case) as e:
        e.initialize()
        e.step(50, macros=True)
        r0a, _, ua = e.macros()
        e.convergence(first=True)
        e.step(9)
        e.step(1, adjacent=True)
        _, _, uadj = e.macros()  # macros still from step 50
        e.step(1, macros=True)
        r0b, _, ub = e.macros()
        out = e.convergence()
        assert np.isclose(out[0], np.sum((ub - ua) ** 2), rtol=1e-12, atol=0)
        assert np.isclose(out[1], np.sum(ub ** 2), rtol=1e-12, atol=0)
        rep = e.report_sums(0, 1, 22)
        nz, ny, nx = ub.shape[1:]
        fl = fluid_mask(case)
        xs = np.arange(nx)
        sel = fl & ((xs >= 1) & (xs <= 22))[None, None, :]
        assert np.isclose(rep[0], ub[0][sel].sum(), rtol=1e-12)
        assert np.isclose(rep[1], r0b[sel].sum(), rtol=1e-12)
        assert rep[7] == (fl[:, :, 1]).sum() and rep[8] == (fl[:, :, 22]).sum()
        fx = e.flux_sums()
        assert np.isclose(fx[0], ub[0].sum(), rtol=1e-12)
        assert np.isclose(fx[6], r0b[fl].sum(), rtol=1e-12)


def test_mass_conservation_and_determinism():
    """Closed periodic medium: mass is conserved; two runs are bitwise identical."""
    case = porous_scsp('MRT', n=(64, 64, 64), seed=2)
    runs = []
    for _ in range(2):
        with engine_for(case) as e:
            e.initialize()
            m0 = e.flux_sums()[6]
            e.step(200, macros=True)
            m1 = e.flux_sums()[6]
            runs.append(e.populations())
        assert abs(m1 - m0) / m0 < 1e-13
    assert np.array_equal(runs[0], runs[1])


SOLID_CASES = [c for c in CASES if c['name'] in (
    'channel-mrt', 'porous-scsp-MRT', 'porous-scsp-SRT', 'porous-scsp-2d-MRT',
    'wall-color-3d-MRT-0.7', 'pb-porous-d3-MRT', 'entry-h16-ratio1.5-MRT', 'film-d3-MRT')]


@pytest.mark.parametrize('case', SOLID_CASES, ids=[c['name'] for c in SOLID_CASES])
def test_checkpoint_with_solid_populations_matches_reference(case):
    """lbf_keep_solid_populations: the whole population array, solid voxels
    included (the reference streams through them), against the reference's
    own checkpoint, at the same tolerance as the fluid voxels."""
    gold = load_golden(case['name'])
    with engine_for(case) as e:
        e.keep_solid_populations()
        e.initialize()
        e.step(case['steps'], macros=True)
        e.check()
        f = e.populations()
    ref = gold['populations'].reshape(f.shape)
    everywhere = np.ones(f.shape[2:], bool)
    solid = ~fluid_mask(case)
    solid = solid if solid.ndim == 3 else solid[None]
    assert np.any(ref[:, :, solid] != 0), 'the case has no streamed solid values'
    assert_populations_close(f, ref, everywhere, population_tolerance(case, case['steps']))


def test_solid_populations_survive_a_restart():
    """A checkpoint written with solid populations and loaded again continues
    exactly (loadRst semantics, solid voxels included)."""
    case = CASES[7]
    o = Oracle(case)
    o.start()
    o.step(20)
    mid = o.populations()
    o.step(15)
    with engine_for(case) as e:
        e.keep_solid_populations()
        e.set_populations(mid)
        e.step(15, macros=True)
        f = e.populations()
    assert_populations_close(f, o.populations(), np.ones(f.shape[2:], bool))
