"""Device-written dense outputs (lbf_fields_dense_async,
lbf_populations_dense_async) against the host-gathered ones
(lbf_get_macros, lbf_get_populations): identical bytes, into page-locked
host memory and into device memory, for every storage and both models; the
non-finite check of a checkpoint; refusal of pageable memory."""
import ctypes

import numpy as np
import pytest
import torch

from cases import porous_scsp, wall_color_3d, entry_case
from test_parity_gpu import engine_for

pytestmark = pytest.mark.gpu


def vti_blocks(e):
    r0, r1, u = e.macros()
    parts = [r0.ravel()] + ([r1.ravel()] if r1 is not None else [])
    d = e.dims
    parts.append(u.reshape(3, -1)[:d].T.ravel())
    return np.concatenate(parts)


@pytest.mark.parametrize('case,storage', [(porous_scsp('MRT'), 'fp64'), (porous_scsp('MRT'), 'fp32'),
                                          (porous_scsp('SRT'), 'bfp16'), (porous_scsp('MRT'), 'fp16'),
                                          (wall_color_3d(0.7, 'MRT'), 'fp64'),
                                          (wall_color_3d(0.7, 'MRT'), 'fp32'),
                                          (entry_case(1.5, 2, steps=60, write=60), 'fp64')],
                         ids=lambda x: x if isinstance(x, str) else x['name'])
def test_dense_outputs_match_host_gather(case, storage):
    from lbflow_b200 import HostBuffer
    with engine_for(case, storage) as e:
        e.initialize()
        e.step(60, macros=True)
        e.check()
        want_f = e.populations().ravel()
        want_v = vti_blocks(e)
        with HostBuffer(want_v.size) as hv, HostBuffer(want_f.size) as hf:
            for _ in range(2):
                hv.array[:] = np.nan
                hf.array[:] = np.nan
                e.fields_dense_async(hv.ptr.value, want_v.size)
                e.populations_dense_async(hf.ptr.value, want_f.size)
                e.synchronize()
                assert np.array_equal(hv.array.view(np.uint64), want_v.view(np.uint64))
                assert np.array_equal(hf.array.view(np.uint64), want_f.view(np.uint64))
        dv = torch.full((want_v.size,), float('nan'), dtype=torch.float64, device='cuda')
        df = torch.full((want_f.size,), float('nan'), dtype=torch.float64, device='cuda')
        torch.cuda.synchronize()
        e.fields_dense_async(dv.data_ptr(), dv.numel())
        e.populations_dense_async(df.data_ptr(), df.numel())
        e.synchronize()
        assert np.array_equal(dv.cpu().numpy().view(np.uint64), want_v.view(np.uint64))
        assert np.array_equal(df.cpu().numpy().view(np.uint64), want_f.view(np.uint64))
        assert e.status() == 0


def test_dense_checkpoint_flags_non_finite_and_refuses_pageable():
    from lbflow_b200 import HostBuffer, LbfError
    case = porous_scsp('MRT')
    with engine_for(case) as e:
        e.initialize()
        f = e.populations()
        fl = np.argwhere(case['geometry'] != 255)[0]
        f[0, 3][tuple(fl)] = np.nan
        e.set_populations(f)
        with HostBuffer(f.size) as hf:
            e.populations_dense_async(hf.ptr.value, f.size)
            assert e.status() & 16
        pageable = np.zeros(f.size)
        with pytest.raises(LbfError, match='page-locked'):
            e.populations_dense_async(pageable.ctypes.data, f.size)
        with pytest.raises(LbfError, match='phases\\*Q\\*N'):
            e.populations_dense_async(pageable.ctypes.data, f.size - 1)
