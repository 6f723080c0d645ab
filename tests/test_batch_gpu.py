"""Batched geometries (lbf_batch_*) against one engine per geometry.

The batch kernel runs the same per-node update as the single-geometry kernel
on the same node order, so after the same steps every geometry's fields must
be bitwise identical to an independent engine's; per-geometry reductions must
agree with the engine's to 1e-12 relative (their summation order differs).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LABELS = {75: ('GV', 1e-5, 1, 0), 255: ('SD', 90.0, 0, 0)}


def _geometries(n=10, seed=4):
    from lbflow_b200.geometry import porous_medium
    rng = np.random.default_rng(seed)
    out, taus = [], []
    for k in range(n):
        shape = tuple(int(v) for v in rng.choice([16, 24, 32, 40], size=3))
        fluid = porous_medium(shape, sigma=float(rng.uniform(1.5, 3.0)), porosity=float(rng.uniform(0.25, 0.4)),
                              seed=100 + k)
        out.append(np.where(fluid, 75, 255).astype(np.uint8))
        taus.append(float(rng.uniform(0.6, 1.4)))
    return out, taus


def _engine_fields(g, tau, steps, storage='fp64'):
    from lbflow_b200 import Engine
    with Engine(g, LABELS, collision='MRT', tau=(tau,), storage=storage) as e:
        e.initialize()
        e.step(steps, macros=True)
        r, _, u = e.macros()
        return r, u, e.flux_sums()


@pytest.mark.parametrize('storage', ['fp64', 'fp32', 'fp16'])
def test_batch_matches_single_engines_bitwise(storage):
    """FP16 included: its stochastic rounding takes the same per-step seeds
    and per-node streams as the single engine, also inside graph replays."""
    from lbflow_b200.batch import Batch
    geoms, taus = _geometries()
    steps = 150   # exercises graph replays (64-step graphs) and explicit steps
    with Batch(geoms, taus, LABELS, collision='MRT', storage=storage) as b:
        b.initialize()
        b.step(steps, macros=True)
        b.check()
        fx = b.flux_sums()
        for k, (g, tau) in enumerate(zip(geoms, taus)):
            r, u = b.macros(k)
            re, ue, fe = _engine_fields(g, tau, steps, storage)
            assert np.array_equal(r, re) and np.array_equal(u, ue), k
            scale = np.maximum(np.abs(fe), 1e-300)
            assert np.all(np.abs(fx[k] - fe) <= 1e-12 * scale + 1e-300), k


def test_autotune_leaves_state_and_retire():
    from lbflow_b200.batch import Batch
    geoms, taus = _geometries(n=6, seed=9)
    with Batch(geoms, taus, LABELS) as b:
        b.initialize()
        b.step(20)
        choice = b.autotune(steps=4)
        assert choice['threads'] in (128, 256) and choice['ms_per_step'] > 0
        b.step(30, macros=True)
        for k in range(len(geoms)):
            r, u = b.macros(k)
            re, ue, _ = _engine_fields(geoms[k], taus[k], 50)
            assert np.array_equal(u, ue), k
        # Retire geometry 0: its fields stay; the others keep advancing exactly.
        r0, u0 = b.macros(0)
        active = np.ones(len(geoms), np.uint8)
        active[0] = 0
        b.set_active(active)
        b.step(40, macros=True)
        r0b, u0b = b.macros(0)
        assert np.array_equal(u0, u0b)
        for k in range(1, len(geoms)):
            _, u = b.macros(k)
            _, ue, _ = _engine_fields(geoms[k], taus[k], 90)
            assert np.array_equal(u, ue), k


def test_batch_convergence_matches_engine():
    """Per-geometry convergence sums equal the single-engine sums."""
    from lbflow_b200 import Engine
    from lbflow_b200.batch import Batch
    geoms, taus = _geometries(n=4, seed=2)
    with Batch(geoms, taus, LABELS) as b:
        b.initialize()
        b.step(100, macros=True)
        b.convergence(first=True)
        b.step(49, adjacent=True)
        b.step(1, macros=True)
        s = b.convergence()
    for k in range(len(geoms)):
        with Engine(geoms[k], LABELS, collision='MRT', tau=(taus[k],)) as e:
            e.initialize()
            e.step(100, macros=True)
            e.convergence(first=True)
            e.step(49, adjacent=True)
            e.step(1, macros=True)
            se = e.convergence()
        assert np.allclose(s[k, :3], se[:3], rtol=1e-12, atol=0), k
