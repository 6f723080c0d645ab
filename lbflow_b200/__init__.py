"""lbflow_b200: B200 lattice Boltzmann engine behind LBFlow's solver interface.

The product is the CUDA library ``lib/liblbflow_b200.so`` (C ABI in
``include/lbflow.h``) and the ``lib/LBFlow`` command line that reads LBFlow's
``input.prm``.  This module is a thin ctypes binding of that C ABI for Python
callers, tests and the benchmark; it does no numerical work of its own and
there is no CPU fallback -- if the library cannot be loaded every call fails.
"""
import ctypes
import os
import threading
from pathlib import Path

import numpy as np

__all__ = ['Engine', 'HostBuffer', 'LbfError', 'library', 'library_path', 'LABEL_TYPES', 'ensure_built']

PKG = Path(__file__).resolve().parent
_LIB_PATH = PKG / 'lib' / 'liblbflow_b200.so'
_lock = threading.Lock()
_lib = None

LABEL_TYPES = {'VD': 0x1, 'GV': 0x2, 'PB': 0x4, 'VB': 0x8, 'AB': 0x10, 'BB': 0x20, 'HF': 0x40, 'SD': 0x80}
MODELS = {'scsp': 0, 'color': 1}
COLLISIONS = {'SRT': 0, 'MRT': 1}
STORAGES = {'fp64': 0, 'fp16': 1, 'bf16': 2, 'fp32': 3, 'bfp16': 4}
STEP_MACROS = 1
STEP_ADJACENT = 2
ERR_BITS = {1: 'Non-finite or non-positive fluid density.',
            2: 'Negative component density outside roundoff tolerance.',
            4: 'Invalid local relaxation time.',
            8: 'Non-finite fluid velocity.',
            16: 'Non-finite post-collision population; no restart will be written.'}


class LbfError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f'{message} (code {code})')
        self.code = code


class _Config(ctypes.Structure):
    _fields_ = [('dims', ctypes.c_uint32), ('nx', ctypes.c_uint32), ('ny', ctypes.c_uint32),
                ('nz', ctypes.c_uint32), ('model', ctypes.c_uint32), ('collision', ctypes.c_uint32),
                ('storage', ctypes.c_uint32), ('device', ctypes.c_int32),
                ('tau', ctypes.c_double * 2), ('rho', ctypes.c_double * 2),
                ('alpha0', ctypes.c_double), ('sigma', ctypes.c_double), ('beta', ctypes.c_double)]


class _Label(ctypes.Structure):
    _fields_ = [('type', ctypes.c_int32), ('dir', ctypes.c_int32), ('phase', ctypes.c_int32),
                ('reserved', ctypes.c_int32), ('value', ctypes.c_double)]


def library_path():
    return _LIB_PATH


def ensure_built():
    """Build the native library in-tree when it is missing (needs nvcc)."""
    if not _LIB_PATH.exists():
        from . import build
        build.build()
    return _LIB_PATH


def library():
    """Load the C-ABI library (raises if it is missing and cannot be built)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        path = ensure_built()
        lib = ctypes.CDLL(str(path))
        P, U32, U64, I = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int
        D = ctypes.POINTER(ctypes.c_double)
        sig = {
            'lbf_create': (I, [ctypes.POINTER(_Config), ctypes.POINTER(_Label), ctypes.c_char_p, ctypes.POINTER(P)]),
            'lbf_destroy': (None, [P]),
            'lbf_initialize': (I, [P]),
            'lbf_keep_solid_populations': (I, [P]),
            'lbf_initialize_equilibrium': (I, [P, P, U32, U32]),
            'lbf_block_sums': (I, [P, U32, D, ctypes.c_size_t]),
            'lbf_add_density': (I, [P, P]),
            'lbf_darcy_pressure': (I, [P, U32, U32, U32, ctypes.c_double, ctypes.c_double, ctypes.c_double, U32, P,
                                       ctypes.POINTER(U32), P]),
            'lbf_step': (I, [P, U32, U32]),
            'lbf_get_populations': (I, [P, D, ctypes.c_size_t]),
            'lbf_set_populations': (I, [P, D, ctypes.c_size_t]),
            'lbf_get_macros': (I, [P, D, D, D]),
            'lbf_convergence': (I, [P, I, D]),
            'lbf_report_sums': (I, [P, U32, U32, U32, D]),
            'lbf_flux_sums': (I, [P, D]),
            'lbf_link_mask': (I, [P, ctypes.POINTER(ctypes.c_uint32), ctypes.c_size_t]),
            'lbf_status': (I, [P, ctypes.POINTER(ctypes.c_uint32)]),
            'lbf_fluid_nodes': (U64, [P]),
            'lbf_device_bytes': (U64, [P]),
            'lbf_last_error': (ctypes.c_char_p, [P]),
            'lbf_synchronize': (I, [P]),
            'lbf_stream': (P, [P]),
            'lbf_flux_sums_noalloc': (I, [P, P, P, U32, U32, P, P]),
            'lbf_fields_dense_async': (I, [P, P, ctypes.c_size_t]),
            'lbf_populations_dense_async': (I, [P, P, ctypes.c_size_t]),
            'lbf_host_alloc': (I, [ctypes.c_size_t, ctypes.POINTER(P)]),
            'lbf_host_free': (None, [P]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if a is not None else None


def make_labels(labels):
    """labels: {label: (type_name, value, dir, phase)} -> ctypes array of 256."""
    arr = (_Label * 256)()
    for k, (t, value, d, ph) in labels.items():
        arr[int(k)] = _Label(LABEL_TYPES[t] if isinstance(t, str) else int(t), int(d), int(ph), 0, float(value))
    return arr


class HostBuffer:
    """Page-locked host memory the device can read and write (lbf_host_alloc),
    viewed as a numpy array (float64 by default): the destination of the
    engine's *_dense_async outputs, or a geometry to upload by DMA."""

    def __init__(self, count, dtype=np.float64):
        self._lib = library()
        self.ptr = ctypes.c_void_p()
        dtype = np.dtype(dtype)
        rc = self._lib.lbf_host_alloc(int(count) * dtype.itemsize, ctypes.byref(self.ptr))
        if rc != 0:
            raise LbfError(rc, self._lib.lbf_last_error(None).decode())
        self.count = int(count)
        raw = (ctypes.c_uint8 * (self.count * dtype.itemsize)).from_address(self.ptr.value)
        self.array = np.frombuffer(raw, dtype=dtype, count=self.count)

    def close(self):
        if self.ptr:
            self.array = None
            self._lib.lbf_host_free(self.ptr)
            self.ptr = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Engine:
    """One geometry on one GPU (see include/lbflow.h for the call contract).

    geometry: uint8 array shaped (nz, ny, nx) (or (ny, nx) in 2D) of labels.
    labels:   {label: (type, value, dir, phase)}, type one of LABEL_TYPES.
    """

    def __init__(self, geometry, labels, model='scsp', collision='MRT', tau=(1.0, 1.0),
                 rho=(1.0, 1.0), alpha0=1 / 3, sigma=0.0, beta=0.0, storage='fp64', device=0):
        self._lib = library()
        g = np.ascontiguousarray(geometry, dtype=np.uint8)
        if g.ndim == 2:
            g = g[None]
            dims = 2
        else:
            dims = 3
        nz, ny, nx = g.shape
        self.shape = (nz, ny, nx)
        self.dims = dims
        self.q = 9 if dims == 2 else 19
        self.phases = 2 if model == 'color' else 1
        self.N = nx * ny * nz
        tau = tuple(tau) + (tau[-1],) * (2 - len(tuple(tau)))
        rho = tuple(rho) + (rho[-1],) * (2 - len(tuple(rho)))
        cfg = _Config(dims, nx, ny, nz, MODELS[model], COLLISIONS[collision], STORAGES[storage], device,
                      (ctypes.c_double * 2)(*tau), (ctypes.c_double * 2)(*rho), alpha0, sigma, beta)
        self._labels = make_labels(labels)
        h = ctypes.c_void_p()
        # The library reads the N label bytes during the call: pass the
        # array's own buffer (page-locked if the caller allocated it so).
        rc = self._lib.lbf_create(ctypes.byref(cfg), self._labels, ctypes.cast(g.ctypes.data, ctypes.c_char_p),
                                  ctypes.byref(h))
        if rc != 0:
            raise LbfError(rc, self._lib.lbf_last_error(None).decode())
        self._h = h
        self.model, self.collision, self.storage = model, collision, storage

    # -- plumbing --------------------------------------------------------------
    def _ck(self, rc):
        if rc != 0:
            raise LbfError(rc, self._lib.lbf_last_error(self._h).decode())

    def close(self):
        if getattr(self, '_h', None):
            self._lib.lbf_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- the step loop ---------------------------------------------------------
    @property
    def fluid_nodes(self):
        return int(self._lib.lbf_fluid_nodes(self._h))

    @property
    def stream(self):
        """Raw cudaStream_t (as an int) of the engine's work queue."""
        return int(self._lib.lbf_stream(self._h) or 0)

    @property
    def device_bytes(self):
        return int(self._lib.lbf_device_bytes(self._h))

    def initialize(self):
        self._ck(self._lib.lbf_initialize(self._h))

    def keep_solid_populations(self):
        """Carry solid voxels' streamed populations (checkpoints identical to
        the reference's at solid voxels too); call before initialize."""
        self._ck(self._lib.lbf_keep_solid_populations(self._h))

    def block_sums(self, block, out=None):
        """Per-cube sums of the last written fields, (NBz, NBy, NBx, 5) of
        (sum rho, sum u_x, sum u_y, sum u_z, fluid voxels): a numpy array, or
        written into `out` (a contiguous float64 CUDA tensor of that shape)."""
        nz, ny, nx = (1,) + tuple(self.shape) if len(self.shape) == 2 else tuple(self.shape)
        bz = 1 if len(self.shape) == 2 else block
        shp = (nz // bz, ny // block, nx // block, 5)
        if out is not None:
            if (tuple(out.shape) != shp or str(out.dtype) != 'torch.float64' or not out.is_cuda
                    or not out.is_contiguous()):
                raise ValueError(f'out must be a contiguous float64 CUDA tensor of shape {shp}')
            ptr = ctypes.cast(ctypes.c_void_p(out.data_ptr()), ctypes.POINTER(ctypes.c_double))
            self._ck(self._lib.lbf_block_sums(self._h, int(block), ptr, out.numel()))
            return out
        res = np.zeros(shp)
        self._ck(self._lib.lbf_block_sums(self._h, int(block), _dptr(res), res.size))
        return res

    def add_density(self, drho):
        """Add w_q * drho to the current populations (contiguous float32 CUDA
        tensor shaped like the geometry): a density change at fixed momentum."""
        if (tuple(drho.shape) != tuple(self.shape) or str(drho.dtype) != 'torch.float32' or not drho.is_cuda
                or not drho.is_contiguous()):
            raise ValueError(f'drho must be a contiguous float32 CUDA tensor of shape {tuple(self.shape)}')
        self._ck(self._lib.lbf_add_density(self._h, ctypes.c_void_p(drho.data_ptr())))

    def initialize_equilibrium(self, fields):
        """Warm start from device fields: a contiguous float32 CUDA tensor of
        shape (nz, ny, nx, ld), ld >= 4, holding velocity x, y, z and density
        per voxel (2-D grids: (ny, nx, ld))."""
        shape = tuple(fields.shape)
        if (shape[:-1] != tuple(self.shape) or shape[-1] < 4 or str(fields.dtype) != 'torch.float32'
                or not fields.is_cuda or not fields.is_contiguous()):
            raise ValueError(f'fields must be a contiguous float32 CUDA tensor of shape {tuple(self.shape)} + (>=4,), '
                             f'got {shape} {fields.dtype} contiguous={fields.is_contiguous()}')
        self._ck(self._lib.lbf_initialize_equilibrium(self._h, ctypes.c_void_p(fields.data_ptr()), int(shape[-1]), 0))

    def step(self, n=1, macros=False, adjacent=False):
        flags = (STEP_MACROS if macros else 0) | (STEP_ADJACENT if adjacent else 0)
        self._ck(self._lib.lbf_step(self._h, int(n), flags))

    def synchronize(self):
        self._ck(self._lib.lbf_synchronize(self._h))

    def status(self):
        bits = ctypes.c_uint32()
        self._ck(self._lib.lbf_status(self._h, ctypes.byref(bits)))
        return bits.value

    def check(self):
        """Raise the reference's error text if the device error word is set."""
        bits = self.status()
        for b, msg in ERR_BITS.items():
            if bits & b:
                raise LbfError(-4, msg)

    # -- data in and out -------------------------------------------------------
    def populations(self):
        out = np.empty(self.phases * self.q * self.N)
        self._ck(self._lib.lbf_get_populations(self._h, _dptr(out), out.size))
        return out.reshape(self.phases, self.q, *self.shape)

    def set_populations(self, f):
        f = np.ascontiguousarray(f, dtype=np.float64).ravel()
        self._ck(self._lib.lbf_set_populations(self._h, _dptr(f), f.size))

    def fields_dense_async(self, address, count):
        """Enqueue the dense VTI-layout fields into device-writable memory at
        `address` (a HostBuffer's ptr or a CUDA tensor's data_ptr())."""
        self._ck(self._lib.lbf_fields_dense_async(self._h, ctypes.c_void_p(int(address)), int(count)))

    def populations_dense_async(self, address, count):
        """Enqueue the dense checkpoint-layout populations into
        device-writable memory at `address`."""
        self._ck(self._lib.lbf_populations_dense_async(self._h, ctypes.c_void_p(int(address)), int(count)))

    def macros(self):
        """(rho0, rho1 or None, u[3]) dense, shaped like the geometry."""
        r0 = np.empty(self.N)
        r1 = np.empty(self.N) if self.phases == 2 else None
        u = np.empty(3 * self.N)
        self._ck(self._lib.lbf_get_macros(self._h, _dptr(r0), _dptr(r1), _dptr(u)))
        shp = self.shape
        return r0.reshape(shp), (r1.reshape(shp) if r1 is not None else None), u.reshape(3, *shp)

    def convergence(self, first=False):
        out = np.zeros(6)
        self._ck(self._lib.lbf_convergence(self._h, 1 if first else 0, _dptr(out)))
        return out

    def report_sums(self, axis, lo, hi):
        out = np.zeros(10)
        self._ck(self._lib.lbf_report_sums(self._h, axis, lo, hi, _dptr(out)))
        return out

    def flux_sums(self):
        out = np.zeros(9)
        self._ck(self._lib.lbf_flux_sums(self._h, _dptr(out)))
        return out

    def link_mask(self):
        out = np.empty(self.N, dtype=np.uint32)
        self._ck(self._lib.lbf_link_mask(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), out.size))
        return out.reshape(self.shape)
