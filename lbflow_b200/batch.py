"""ctypes binding of the batched-geometry C ABI (lbf_batch_*, include/lbflow.h)."""
import ctypes
import math
import time

import numpy as np

from . import COLLISIONS, STORAGES, LbfError, library, make_labels

_SIGS = None


class _Geom(ctypes.Structure):
    _fields_ = [('nx', ctypes.c_uint32), ('ny', ctypes.c_uint32), ('nz', ctypes.c_uint32),
                ('labels', ctypes.c_void_p), ('tau', ctypes.c_double)]


def _lib():
    global _SIGS
    lib = library()
    if _SIGS is None:
        P, U32, I, D = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int, ctypes.POINTER(ctypes.c_double)
        sig = {
            'lbf_batch_create': (I, [P, U32, P, U32, U32, ctypes.c_int32, ctypes.c_double, ctypes.POINTER(P)]),
            'lbf_batch_destroy': (None, [P]),
            'lbf_batch_initialize': (I, [P]),
            'lbf_batch_step': (I, [P, U32, U32]),
            'lbf_batch_convergence': (I, [P, I, D]),
            'lbf_batch_flux_sums': (I, [P, D]),
            'lbf_batch_set_active': (I, [P, P]),
            'lbf_batch_autotune': (I, [P, U32, D]),
            'lbf_batch_get_macros': (I, [P, U32, D, D]),
            'lbf_batch_status': (I, [P, ctypes.POINTER(ctypes.c_uint32)]),
            'lbf_batch_synchronize': (I, [P]),
            'lbf_batch_fluid_nodes': (ctypes.c_uint64, [P, U32]),
            'lbf_batch_active_tiles': (U32, [P]),
            'lbf_batch_stream': (P, [P]),
            'lbf_batch_last_error': (ctypes.c_char_p, [P]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _SIGS = True
    return lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Batch:
    """Many single-phase D3Q19 geometries advanced in one launch per step.

    geometries: list of uint8 arrays shaped (nz, ny, nx); taus: one relaxation
    time per geometry; labels: shared {label: (type, value, dir, phase)}.
    """

    def __init__(self, geometries, taus, labels, collision='MRT', storage='fp64', device=0, rho0=1.0):
        self._lib = _lib()
        self._arrays = [np.ascontiguousarray(g, np.uint8) for g in geometries]
        self.shapes = [a.shape for a in self._arrays]
        self.taus = [float(t) for t in taus]
        self.count = len(self._arrays)
        geoms = (_Geom * self.count)()
        for k, a in enumerate(self._arrays):
            nz, ny, nx = a.shape
            geoms[k] = _Geom(nx, ny, nz, a.ctypes.data, self.taus[k])
        self._labels = make_labels(labels)
        h = ctypes.c_void_p()
        rc = self._lib.lbf_batch_create(geoms, self.count, self._labels, COLLISIONS[collision],
                                        STORAGES[storage], device, rho0, ctypes.byref(h))
        if rc != 0:
            raise LbfError(rc, self._lib.lbf_batch_last_error(None).decode())
        self._h = h

    def _ck(self, rc):
        if rc != 0:
            raise LbfError(rc, self._lib.lbf_batch_last_error(self._h).decode())

    def close(self):
        if getattr(self, '_h', None):
            self._lib.lbf_batch_destroy(self._h)
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

    def fluid_nodes(self, k=None):
        return int(self._lib.lbf_batch_fluid_nodes(self._h, 0xffffffff if k is None else k))

    @property
    def active_tiles(self):
        return int(self._lib.lbf_batch_active_tiles(self._h))

    @property
    def stream(self):
        return int(self._lib.lbf_batch_stream(self._h) or 0)

    def initialize(self):
        self._ck(self._lib.lbf_batch_initialize(self._h))

    def step(self, n=1, macros=False, adjacent=False):
        self._ck(self._lib.lbf_batch_step(self._h, int(n), (1 if macros else 0) | (2 if adjacent else 0)))

    def synchronize(self):
        self._ck(self._lib.lbf_batch_synchronize(self._h))

    def check(self):
        bits = ctypes.c_uint32()
        self._ck(self._lib.lbf_batch_status(self._h, ctypes.byref(bits)))
        if bits.value:
            raise LbfError(-4, f'device error word {bits.value:#x} (non-finite or non-positive density)')

    def convergence(self, first=False):
        out = np.zeros((self.count, 6))
        self._ck(self._lib.lbf_batch_convergence(self._h, 1 if first else 0, _dp(out)))
        return out

    def flux_sums(self):
        out = np.zeros((self.count, 9))
        self._ck(self._lib.lbf_batch_flux_sums(self._h, _dp(out)))
        return out

    def set_active(self, active):
        a = np.ascontiguousarray(active, np.uint8)
        self._ck(self._lib.lbf_batch_set_active(self._h, a.ctypes.data))

    def autotune(self, steps=10):
        out = np.zeros(4)
        self._ck(self._lib.lbf_batch_autotune(self._h, steps, _dp(out)))
        return dict(threads=int(out[0]), tile_nodes=int(out[1]), blocks128_per_sm=out[2], ms_per_step=out[3])

    def macros(self, k):
        nz, ny, nx = self.shapes[k]
        N = nx * ny * nz
        r, u = np.empty(N), np.empty(3 * N)
        self._ck(self._lib.lbf_batch_get_macros(self._h, k, _dp(r), _dp(u)))
        return r.reshape(nz, ny, nx), u.reshape(3, nz, ny, nx)

    def converge(self, g, report=1000, tol=1e-6, max_steps=200000, on_report=None):
        """Step every geometry to LBFlow's criterion (as permeability.converge)
        and retire each one when it converges.  Returns per-geometry steps,
        permeability K = nu <u_x> / g and the aggregate node updates."""
        self.initialize()
        active = np.ones(self.count, np.uint8)
        stable = np.zeros(self.count, int)
        steps = np.zeros(self.count, int)
        K = np.full(self.count, np.nan)
        updates = 0
        nodes = np.array([self.fluid_nodes(k) for k in range(self.count)], dtype=np.int64)
        N = np.array([np.prod(s) for s in self.shapes], dtype=float)
        count = 3 * N
        t = 0
        first = True
        self.synchronize()
        t0 = time.perf_counter()
        while t < max_steps and active.any():
            self.step(report - 1, adjacent=True)
            self.step(1, macros=True)
            t += report
            updates += int(nodes[active.astype(bool)].sum()) * report
            steps[active.astype(bool)] = t
            self.check()
            s = self.convergence(first=first)
            fx = self.flux_sums()
            for k in range(self.count):
                if not active[k]:
                    continue
                nu = (self.taus[k] - 0.5) / 3.0
                K[k] = nu * fx[k, 0] / N[k] / g
                if first:
                    continue
                rms = math.sqrt(s[k, 0] / count[k])
                res = math.sqrt(s[k, 0] / s[k, 1]) if s[k, 1] > 0 else 0.0
                arms = math.sqrt(s[k, 2] / count[k])
                ares = math.sqrt(s[k, 2] / s[k, 1]) if s[k, 1] > 0 else 0.0
                ok = (rms <= 1e-12 or res < tol) and (arms <= 1e-12 or ares < tol)
                stable[k] = stable[k] + 1 if ok else 0
            first = False
            done = (stable >= 3) & active.astype(bool)
            if done.any():
                active[done] = 0
                self.set_active(active)
            if on_report:
                on_report(t, int(active.sum()))
        self.synchronize()
        seconds = time.perf_counter() - t0
        return dict(steps=steps, K=K, converged=stable >= 3, seconds=seconds, updates=updates,
                    mlups=updates / seconds / 1e6)


# ---- several GPUs: the batch split into independent shards -------------------
def estimated_work(geometries, taus, labels):
    """Relative cost of converging each geometry: fluid voxels times steps,
    the steps scaling as the viscous time across the medium, L^2 / nu with L
    the longest edge (the slow pressure mode crosses the whole medium)."""
    from . import LABEL_TYPES
    fluid_types = {LABEL_TYPES[t] for t in ('VD', 'GV', 'PB', 'VB')}
    lut = np.zeros(256, bool)
    for k, (t, *_rest) in labels.items():
        lut[int(k)] = (LABEL_TYPES[t] if isinstance(t, str) else int(t)) in fluid_types
    work = []
    for g, tau in zip(geometries, taus):
        nf = int(lut[np.asarray(g, np.uint8)].sum())
        nu = (float(tau) - 0.5) / 3.0
        work.append(nf * max(g.shape) ** 2 / nu)
    return work


def partition(work, parts):
    """Longest-processing-time split of items with the given work into
    `parts` lists of indices: items in order of decreasing work, each to the
    currently lightest part (ties to the lower index, so every process that
    calls this with the same work gets the same split).  Each list is
    returned in ascending index order."""
    order = sorted(range(len(work)), key=lambda k: (-work[k], k))
    load = [0.0] * parts
    out = [[] for _ in range(parts)]
    for k in order:
        p = min(range(parts), key=lambda j: (load[j], j))
        out[p].append(k)
        load[p] += work[k]
    return [sorted(o) for o in out]


def converge_sharded(geometries, taus, labels, g, rank=0, world=1, device=0, collision='MRT', storage='fp64',
                     report=1000, tol=1e-6, max_steps=200000, group=None, batch_factory=None):
    """Converge a list of geometries split over `world` processes, one GPU
    each.  Geometries are independent, so there is no data-path collective:
    every rank runs its share (partition of estimated_work) in its own
    persistent batched launch, and only the per-geometry results (steps, K,
    convergence flag) and each rank's seconds are exchanged afterwards,
    host-side, with torch.distributed.all_gather_object on `group`.
    Returns the results in the original order, seconds = the slowest rank's
    wall time, and the aggregate node updates."""
    factory = batch_factory or Batch
    parts = partition(estimated_work(geometries, taus, labels), world)
    mine = parts[rank]
    local = dict(index=mine, steps=[], K=[], converged=[], seconds=0.0, updates=0, nodes=0)
    if mine:
        b = factory([geometries[k] for k in mine], [taus[k] for k in mine], labels, collision=collision,
                    storage=storage, device=device)
        try:
            r = b.converge(g, report=report, tol=tol, max_steps=max_steps)
            local.update(steps=[int(v) for v in r['steps']], K=[float(v) for v in r['K']],
                         converged=[bool(v) for v in r['converged']], seconds=float(r['seconds']),
                         updates=int(r['updates']), nodes=int(b.fluid_nodes()))
        finally:
            b.close()
    if world > 1:
        import torch.distributed as dist
        gathered = [None] * world
        dist.all_gather_object(gathered, local, group=group)
    else:
        gathered = [local]
    n = len(geometries)
    K = np.full(n, np.nan)
    steps = np.zeros(n, int)
    converged = np.zeros(n, bool)
    for part in gathered:
        for j, k in enumerate(part['index']):
            K[k], steps[k], converged[k] = part['K'][j], part['steps'][j], part['converged'][j]
    seconds = max(p['seconds'] for p in gathered)
    updates = sum(p['updates'] for p in gathered)
    return dict(K=K, steps=steps, converged=converged, seconds=seconds, updates=updates,
                mlups=updates / seconds / 1e6 if seconds > 0 else 0.0,
                nodes=sum(p['nodes'] for p in gathered), parts=[p['index'] for p in gathered],
                rank_seconds=[p['seconds'] for p in gathered])
