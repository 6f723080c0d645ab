"""Run an engine to steady state and measure the body-force permeability.

converge() applies LBFlow's stopping rule (Simulator::updateConvergence,
solver/src/lbm/simulator.cpp:248-325) with the engine's device reductions: at
every report step the relative L2 change of the velocity field since the last
report, sqrt(sum (u - u_prev)^2 / sum u^2), and the same against the previous
step must be below `tol` (or their RMS below 1e-12) for three consecutive
reports.  permeability() is scripts/rock_workflow.py:60-66 /
porous_media.py:20-44: K = nu <u_x> / g_x with <u_x> averaged over all voxels
and nu = (tau - 1/2) / 3.
"""
import math
import time

import numpy as np


def permeability(engine, tau, g, axis=0):
    s = engine.flux_sums()
    mean = s[axis] / engine.N
    return (tau - 0.5) / 3.0 * mean / g


def converge(engine, tau, g, report=1000, tol=1e-6, max_steps=2_000_000, initialized=False,
             on_report=None, warm=None, patience=5, t0=None, accelerate=None, stall_floor=None):
    """Step to the reference's convergence criterion; returns a dict with the
    completed steps, wall seconds (device work included), K and the residual history.

    warm: optional callable that initialises the engine (a warm start).  The
    run then falls back to LBFlow's start from rest (engine.initialize) when
    the warm-started residual is non-finite, the device reports a numerical
    error, or the residual, still above `stall_floor` (default 100 * tol;
    16-bit storage needs a higher one, as its rounding noise keeps the
    residual near 1e-4), sets no new minimum for `patience` reports.  Steps
    and seconds count both attempts; `fallback` in the result says whether it
    happened.  t0: perf_counter value the seconds count from (default: the
    start of this call, after the engine's queued work).  accelerate:
    optional callable(t) run after the checks of every report (for example a
    warmstart.DarcyAccelerator); its work is inside the timed region."""
    engine.synchronize()
    if t0 is None:
        t0 = time.perf_counter()
    if warm is not None:
        warm()
    elif not initialized:
        engine.initialize()
    D = engine.dims
    count = D * engine.N
    t = 0
    stable = 0
    first = True
    history = []
    warm_active = warm is not None
    fallback = False
    best, since_best = math.inf, 0

    def restart():
        nonlocal first, stable, warm_active, fallback, best, since_best
        engine.initialize()
        first, stable, warm_active, fallback = True, 0, False, True
        best, since_best = math.inf, 0

    while t < max_steps:
        engine.step(report - 1, adjacent=True)
        engine.step(1, macros=True)
        t += report
        try:
            engine.check()
        except Exception:
            if not warm_active:
                raise
            restart()
            continue
        K = permeability(engine, tau, g)
        if accelerate is not None and accelerate(t):
            best, since_best = math.inf, 0       # a correction restarts the stall watch
        if first:
            engine.convergence(first=True)
            first = False
            history.append((t, float('nan'), float('nan'), K, time.perf_counter() - t0))
            continue
        s = engine.convergence()
        if not all(math.isfinite(v) for v in s[:3]):
            if warm_active:
                restart()
                continue
            raise RuntimeError('Invalid global velocity residual.')
        rms = math.sqrt(s[0] / count)
        res = math.sqrt(s[0] / s[1]) if s[1] > 0 else 0.0
        arms = math.sqrt(s[2] / count)
        ares = math.sqrt(s[2] / s[1]) if s[1] > 0 else 0.0
        ok = (rms <= 1e-12 or res < tol) and (arms <= 1e-12 or ares < tol)
        stable = stable + 1 if ok else 0
        history.append((t, res, ares, K, time.perf_counter() - t0))
        if on_report:
            on_report(t, res, ares)
        if stable >= 3:
            break
        if res < best:
            best, since_best = res, 0
        else:
            since_best += 1
        # A stall far above the tolerance means the warm start went wrong; near
        # the tolerance it is the storage precision's floor, which a restart
        # would not change.
        if warm_active and since_best >= patience and best > (stall_floor if stall_floor else 100 * tol):
            restart()
    engine.synchronize()
    seconds = time.perf_counter() - t0
    return dict(steps=t, seconds=seconds, K=permeability(engine, tau, g), converged=stable >= 3,
                history=history, fallback=fallback)


def time_to_band(history, K_ref, rel=1e-3):
    """First report after which K stays within rel of K_ref: (steps, seconds) or None."""
    hit = None
    for t, _, _, K, sec in history:
        if abs(K - K_ref) <= rel * abs(K_ref):
            if hit is None:
                hit = (t, sec)
        else:
            hit = None
    return hit
