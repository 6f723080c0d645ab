"""lbf_flux_sums_noalloc: the flux/mass sums for callers that cannot allocate.

Some callers cannot call cudaMalloc (a frozen or exhausted memory pool, an
allocator that owns the whole device), so this entry point takes the caller's
device arrays and writes the caller's device output, with its scratch in a
fixed array compiled into the library.  The test feeds it the engine's own
fields and checks it against lbf_flux_sums and against numpy sums of the same
downloaded arrays, within the relative 1e-12 used by the other reduction
tests, on two calls in a row (the second with new data, so stale scratch
contents would show), and checks that a call after the first one changes
neither the device's free memory nor torch's caching allocator.  The
argument checks, which need no GPU, are in test_abi.py.  It is collected last
on purpose.
"""
import ctypes

import numpy as np
import pytest

from cases import drop_3d, porous_scsp
from conftest import fluid_mask

pytestmark = pytest.mark.gpu


def _engine(case):
    from lbflow_b200 import Engine
    return Engine(case['geometry'], case['labels'], model=case['model'], collision=case['collision'],
                  tau=case['tau'], rho=case['rho'], alpha0=case.get('alpha0', 1 / 3),
                  sigma=case.get('sigma', 0.0), beta=case.get('beta', 0.0))


def _device_sums(u, r0, r1):
    """Call the entry point on device copies of compact node arrays."""
    import torch
    import lbflow_b200
    lib = lbflow_b200.library()
    n = r0.size
    stride = (n + 63) // 64 * 64
    du = torch.zeros((3, stride), dtype=torch.float64, device='cuda')
    du[:, :n] = torch.from_numpy(u)
    d0 = torch.zeros(stride, dtype=torch.float64, device='cuda')
    d0[:n] = torch.from_numpy(r0)
    d1 = None
    if r1 is not None:
        d1 = torch.zeros(stride, dtype=torch.float64, device='cuda')
        d1[:n] = torch.from_numpy(r1)
    out = torch.full((9,), float('nan'), dtype=torch.float64, device='cuda')
    stream = torch.cuda.current_stream()
    rc = lib.lbf_flux_sums_noalloc(ctypes.c_void_p(du.data_ptr()), ctypes.c_void_p(d0.data_ptr()),
                                   ctypes.c_void_p(d1.data_ptr()) if d1 is not None else None,
                                   n, stride, ctypes.c_void_p(out.data_ptr()),
                                   ctypes.c_void_p(stream.cuda_stream))
    assert rc == 0, lib.lbf_last_error(None).decode()
    stream.synchronize()
    return out.cpu().numpy()


def _compact(e, case):
    r0, r1, u = e.macros()
    fl = fluid_mask(case).ravel()
    uc = np.ascontiguousarray(u.reshape(3, -1)[:, fl])
    return uc, np.ascontiguousarray(r0.ravel()[fl]), (np.ascontiguousarray(r1.ravel()[fl]) if r1 is not None else None)


def _close(got, want, parts):
    # Relative 1e-12 of the summed magnitudes (a sum like sum(u_y) may cancel).
    scale = np.array([np.abs(p).sum() for p in parts])
    assert np.all(np.abs(got - want) <= 1e-12 * np.maximum(scale, 1e-300)), (got, want)


def _numpy_sums(parts):
    """The nine sums of lbf_flux_sums computed by numpy (math.fsum, exactly
    rounded) from the downloaded arrays."""
    import math
    return np.array([math.fsum(p.tolist()) for p in parts])


@pytest.mark.parametrize('case', [porous_scsp('MRT', n=(48, 40, 32), seed=3), drop_3d()],
                         ids=lambda c: c['name'])
def test_noalloc_matches_flux_sums_twice(case):
    with _engine(case) as e:
        e.initialize()
        for steps in (37, 11):
            e.step(steps, macros=True)
            want = e.flux_sums()
            uc, r0, r1 = _compact(e, case)
            got = _device_sums(uc, r0, r1)
            phi0 = r0 / (r0 + r1) if r1 is not None else np.ones_like(r0)
            parts = [uc[0], uc[1], uc[2], phi0 * uc[0], phi0 * uc[1], phi0 * uc[2], r0,
                     r1 if r1 is not None else np.zeros(1), phi0]
            _close(got, want, parts)
            _close(got, _numpy_sums(parts), parts)


def test_noalloc_allocates_nothing_after_the_first_call():
    """After a first call on the device (which loads the library's scratch
    array with the module), further calls leave the device's free memory and
    torch's caching allocator unchanged."""
    import torch
    rng = np.random.default_rng(4)
    n = 300_001
    u = rng.standard_normal((3, n)) * 1e-5
    r0 = 1.0 + 1e-3 * rng.standard_normal(n)
    _device_sums(u, r0, None)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    reserved0 = torch.cuda.memory_reserved()
    allocated0 = torch.cuda.memory_allocated()
    # Inputs prepared beforehand so that only the entry point runs in between.
    import lbflow_b200
    lib = lbflow_b200.library()
    stride = (n + 63) // 64 * 64
    du = torch.zeros((3, stride), dtype=torch.float64, device='cuda')
    du[:, :n] = torch.from_numpy(u)
    d0 = torch.zeros(stride, dtype=torch.float64, device='cuda')
    d0[:n] = torch.from_numpy(r0)
    out = torch.zeros(9, dtype=torch.float64, device='cuda')
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    reserved1 = torch.cuda.memory_reserved()
    stream = torch.cuda.current_stream()
    for _ in range(3):
        rc = lib.lbf_flux_sums_noalloc(ctypes.c_void_p(du.data_ptr()), ctypes.c_void_p(d0.data_ptr()), None,
                                       n, stride, ctypes.c_void_p(out.data_ptr()),
                                       ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, lib.lbf_last_error(None).decode()
    stream.synchronize()
    free2, _ = torch.cuda.mem_get_info()
    assert free2 == free1, (free1, free2)
    assert torch.cuda.memory_reserved() == reserved1
    assert reserved1 >= reserved0 and free0 >= free1 and torch.cuda.memory_allocated() >= allocated0
    parts = [u[0], u[1], u[2], u[0], u[1], u[2], r0, np.zeros(1), np.ones(n)]
    _close(out.cpu().numpy(), _numpy_sums(parts), parts)
