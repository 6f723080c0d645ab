"""ctypes binding of the C restatement oracle (oracle/lbm_oracle.c).

Test infrastructure only: the tests use it as the checker of the CUDA engine.
"""
import ctypes
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
SO = ROOT / 'oracle' / '_build' / 'liblbm_oracle.so'
TYPES = {'VD': 0x1, 'GV': 0x2, 'PB': 0x4, 'VB': 0x8, 'AB': 0x10, 'BB': 0x20, 'HF': 0x40, 'SD': 0x80}


class Params(ctypes.Structure):
    _fields_ = [('dims', ctypes.c_int), ('nx', ctypes.c_int), ('ny', ctypes.c_int), ('nz', ctypes.c_int),
                ('color', ctypes.c_int), ('mrt', ctypes.c_int), ('tau', ctypes.c_double * 2),
                ('rho', ctypes.c_double * 2), ('alpha0', ctypes.c_double), ('sigma', ctypes.c_double),
                ('beta', ctypes.c_double)]


class Label(ctypes.Structure):
    _fields_ = [('type', ctypes.c_int), ('value', ctypes.c_double), ('dir', ctypes.c_int), ('phase', ctypes.c_int)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        src = [ROOT / 'oracle' / 'lbm_oracle.c', ROOT / 'oracle' / 'lbm_oracle.h']
        if not SO.exists() or any(p.stat().st_mtime > SO.stat().st_mtime for p in src):
            subprocess.run(['make', '-C', str(ROOT / 'oracle'), 'port'], check=True, capture_output=True)
        L = ctypes.CDLL(str(SO))
        V = ctypes.c_void_p
        L.lbo_create.restype = V
        L.lbo_create.argtypes = [ctypes.POINTER(Params), ctypes.POINTER(Label), ctypes.c_char_p]
        for n in ('lbo_initialize', 'lbo_collide', 'lbo_stream_macros'):
            getattr(L, n).argtypes = [V]
        L.lbo_step.argtypes = [V, ctypes.c_int]
        L.lbo_destroy.argtypes = [V]
        L.lbo_voxels.restype = ctypes.c_size_t
        L.lbo_voxels.argtypes = [V]
        for n in ('lbo_get_populations', 'lbo_set_populations', 'lbo_get_phi'):
            getattr(L, n).argtypes = [V, V]
        L.lbo_get_macros.argtypes = [V, V, V, V]
        L.lbo_link_mask.argtypes = [V, V]
        L.lbo_wall_angles.argtypes = [V, V, V]
        L.lbo_mrt_tables.argtypes = [ctypes.c_int, ctypes.c_double, V, V, V]
        _lib = L
    return _lib


class Oracle:
    """Dense CPU solver with the reference's layout and arithmetic."""

    def __init__(self, case):
        g = np.ascontiguousarray(case['geometry'], np.uint8)
        self.dims = 2 if g.ndim == 2 else 3
        if g.ndim == 2:
            ny, nx = g.shape
            nz = 1
        else:
            nz, ny, nx = g.shape
        self.shape = (nz, ny, nx)
        self.q = 9 if self.dims == 2 else 19
        self.color = case['model'] == 'color'
        self.phases = 2 if self.color else 1
        tau = tuple(case['tau']) + (case['tau'][-1],) * (2 - len(case['tau']))
        rho = tuple(case['rho']) + (case['rho'][-1],) * (2 - len(case['rho']))
        p = Params(self.dims, nx, ny, nz, int(self.color), int(case['collision'] == 'MRT'),
                   (ctypes.c_double * 2)(*tau), (ctypes.c_double * 2)(*rho), case.get('alpha0', 1 / 3),
                   case.get('sigma', 0.0), case.get('beta', 0.0))
        L = (Label * 256)()
        for k, (t, v, d, ph) in case['labels'].items():
            L[int(k)] = Label(TYPES[t], float(v), int(d), int(ph))
        self._labels = L
        h = lib().lbo_create(ctypes.byref(p), L, g.tobytes())
        if not h:
            raise ValueError('oracle rejected the case')
        self._h = ctypes.c_void_p(h)
        self.N = nx * ny * nz

    def __del__(self):
        if getattr(self, '_h', None):
            lib().lbo_destroy(self._h)
            self._h = None

    def _ck(self, rc):
        if rc != 0:
            raise RuntimeError(f'oracle error {rc}')

    def start(self):
        """t = 0: initialize, macros, body force, initial collision."""
        self._ck(lib().lbo_initialize(self._h))
        m = self.macros()
        self._ck(lib().lbo_collide(self._h))
        return m

    def step(self, n=1):
        self._ck(lib().lbo_step(self._h, n))

    def stream_macros(self):
        self._ck(lib().lbo_stream_macros(self._h))

    def collide(self):
        self._ck(lib().lbo_collide(self._h))

    def populations(self):
        f = np.empty(self.phases * self.q * self.N)
        lib().lbo_get_populations(self._h, f.ctypes.data)
        return f.reshape(self.phases, self.q, *self.shape)

    def set_populations(self, f):
        f = np.ascontiguousarray(f, np.float64).ravel()
        lib().lbo_set_populations(self._h, f.ctypes.data)

    def macros(self):
        r0, r1, u = np.empty(self.N), np.empty(self.N), np.empty(3 * self.N)
        lib().lbo_get_macros(self._h, r0.ctypes.data, r1.ctypes.data, u.ctypes.data)
        s = self.shape
        return r0.reshape(s), (r1.reshape(s) if self.color else None), u.reshape(3, *s)

    def phi(self):
        p = np.empty(self.N)
        lib().lbo_get_phi(self._h, p.ctypes.data)
        return p.reshape(self.shape)

    def link_mask(self):
        m = np.empty(self.N, np.uint32)
        lib().lbo_link_mask(self._h, m.ctypes.data)
        return m.reshape(self.shape)


def mrt_tables(q, tau):
    m, mi, s = np.empty(q * q), np.empty(q * q), np.empty(q)
    lib().lbo_mrt_tables(q, tau, m.ctypes.data, mi.ctypes.data, s.ctypes.data)
    return m.reshape(q, q), mi.reshape(q, q), s
