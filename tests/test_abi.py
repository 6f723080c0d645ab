"""The C-ABI library: loads, exports what include/*.h declare, validates input (no GPU needed)."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    text = ''.join(p.read_text() for p in sorted((ROOT / 'include').glob('*.h')))
    return sorted(set(re.findall(r'\b(lbf_[a-z_]+)\s*\(', text)))


def test_library_exports_every_declared_symbol():
    import lbflow_b200
    lib = lbflow_b200.library()
    names = declared_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n


def _create(**over):
    import lbflow_b200 as L
    lib = L.library()
    cfg = dict(dims=3, nx=4, ny=4, nz=4, model=0, collision=1, storage=0, device=0)
    cfg.update(over)
    c = L._Config(cfg['dims'], cfg['nx'], cfg['ny'], cfg['nz'], cfg['model'], cfg['collision'],
                  cfg['storage'], cfg['device'], (ctypes.c_double * 2)(*over.get('tau', (1.0, 1.0))),
                  (ctypes.c_double * 2)(1.0, 1.0), 1 / 3, 0.0, 0.0)
    labels = L.make_labels(over.get('labels', {0: ('VD', 0, 0, 0)}))
    geom = over.get('geometry', np.zeros(64, np.uint8))
    h = ctypes.c_void_p()
    rc = lib.lbf_create(ctypes.byref(c), labels, geom.tobytes(), ctypes.byref(h))
    return rc, lib.lbf_last_error(None).decode()


@pytest.mark.parametrize('over,msg', [
    (dict(dims=4), 'dims'),
    (dict(nx=4096), 'grid dimensions'),
    (dict(model=7), 'fluid model'),
    (dict(collision=5), 'collision'),
    (dict(tau=(0.5, 1.0)), 'relaxation times must exceed 0.5'),
    (dict(labels={}), 'not defined'),
    (dict(labels={0: ('HF', 0.0, 0, 0)}), 'half-permeable films (HF) need the color model'),
    (dict(labels={0: ('AB', 0.0, 0, 0)}), 'only VD, GV, PB, VB, HF, BB and SD'),
    (dict(model=1, labels={0: ('PB', 1.0, 1, 2)}), 'phase'),
    (dict(labels={0: ('PB', 0.0, 1, 0)}), 'Pressure-boundary density must be positive'),
    (dict(labels={0: ('VB', 1e-3, 7, 0)}), 'axial direction'),
    (dict(labels={0: ('VB', 1e-3, 0, 0)}), 'non-rest lattice direction'),
    (dict(labels={0: ('VB', float('nan'), 1, 0)}), 'Non-finite boundary value'),
    (dict(labels={0: ('GV', 1e-6, 19, 0)}), 'body-force direction'),
    (dict(labels={0: ('VD', 0, 0, 1)}), 'phase'),
    (dict(model=1, storage=4), 'two-phase storage'),
])
def test_create_rejects_invalid_input(over, msg):
    rc, err = _create(**over)
    assert rc == -1
    assert msg in err


def test_null_arguments():
    import lbflow_b200 as L
    lib = L.library()
    assert lib.lbf_create(None, None, None, None) == -1
    assert lib.lbf_step(None, 1, 0) == -1
    assert lib.lbf_fluid_nodes(None) == 0


def test_darcy_pressure_rejects_bad_arguments():
    """Argument conversion and validation of lbf_darcy_pressure (no GPU work)."""
    import lbflow_b200 as L
    lib = L.library()
    it = ctypes.c_uint32(7)
    rc = lib.lbf_darcy_pressure(None, 8, 8, 8, 2.0, 1e-5, 1e-3, 10, None, ctypes.byref(it), None)
    assert rc == -1 and 'bad arguments' in lib.lbf_last_error(None).decode()
    rc = lib.lbf_darcy_pressure(ctypes.c_void_p(16), 8, 8, 8, 0.0, 1e-5, 1e-3, 10, ctypes.c_void_p(16),
                                ctypes.byref(it), None)
    assert rc == -1


def test_engine_block_and_density_entry_points_validate():
    import lbflow_b200 as L
    lib = L.library()
    out = (ctypes.c_double * 5)()
    assert lib.lbf_block_sums(None, 2, out, 5) == -1
    assert lib.lbf_add_density(None, None) == -1
    assert lib.lbf_initialize_equilibrium(None, None, 4, 0) == -1


@pytest.mark.parametrize('args,msg', [
    (dict(n=(1 << 24) + 1, stride=(1 << 24) + 1), 'exceeds the fixed scratch capacity'),
    (dict(u=None), 'must be device pointers'),
    (dict(rho0=None), 'must be device pointers'),
    (dict(out=None), 'must be device pointers'),
    (dict(n=100, stride=99), 'stride must be >= n'),
])
def test_noalloc_rejects_bad_arguments(args, msg):
    """lbf_flux_sums_noalloc refuses these before touching the GPU."""
    import lbflow_b200
    lib = lbflow_b200.library()
    a = dict(u=ctypes.c_void_p(16), rho0=ctypes.c_void_p(16), n=10, stride=10, out=ctypes.c_void_p(16))
    a.update(args)
    rc = lib.lbf_flux_sums_noalloc(a['u'], a['rho0'], None, a['n'], a['stride'], a['out'], None)
    assert rc == -1
    assert msg in lib.lbf_last_error(None).decode()


def test_keep_solid_populations_null_engine():
    import lbflow_b200
    lib = lbflow_b200.library()
    assert lib.lbf_keep_solid_populations(None) == -1
