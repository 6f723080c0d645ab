"""Synthetic voxel geometries for the engine's workloads.

porous_medium() is the Gaussian-filtered-noise recipe used for every porous
workload: a seeded N(0,1) white-noise field, a periodic Gaussian filter of
width sigma voxels, a threshold at the quantile that gives the requested
porosity, then removal of fluid clusters not connected to the largest
periodic 6-connected fluid cluster.  These seeded synthetic media stand in for
scanned rock; scripts/rock_workflow.py applies the same solver to real crops.
"""
import numpy as np


def _largest_periodic_cluster(fluid):
    from scipy import ndimage as ndi
    lab, n = ndi.label(fluid)
    if n == 0:
        return fluid
    parent = np.arange(n + 1)

    def find(a):
        while parent[a] != a:
            parent[a] = parent[parent[a]]
            a = parent[a]
        return a

    # Union the clusters that touch across each periodic face.
    for ax in range(fluid.ndim):
        a = np.take(lab, 0, axis=ax)
        b = np.take(lab, -1, axis=ax)
        m = (a > 0) & (b > 0)
        for u, v in set(zip(a[m].tolist(), b[m].tolist())):
            ru, rv = find(u), find(v)
            if ru != rv:
                parent[ru] = rv
    roots = np.array([find(i) for i in range(n + 1)])
    merged = roots[lab]
    counts = np.bincount(merged.ravel())
    counts[0] = 0
    return merged == counts.argmax()


def porous_medium(shape, sigma, porosity, seed):
    """Boolean fluid mask of the given (nz, ny, nx) shape."""
    from scipy import ndimage as ndi
    rng = np.random.default_rng(seed)
    field = ndi.gaussian_filter(rng.standard_normal(shape), sigma, mode='wrap')
    fluid = field < np.quantile(field, porosity)
    return _largest_periodic_cluster(fluid)


def percolates(fluid, axis=-1):
    """True if a fluid path crosses the box from face to face along `axis`
    (x by default), with the other two axes periodic: the geometry then
    carries a non-zero flux under a body force along that axis."""
    from scipy import ndimage as ndi
    axis = axis % fluid.ndim
    lab, n = ndi.label(fluid)
    if n == 0:
        return False
    parent = np.arange(n + 1)

    def find(a):
        while parent[a] != a:
            parent[a] = parent[parent[a]]
            a = parent[a]
        return a

    for ax in range(fluid.ndim):
        if ax == axis:
            continue
        a = np.take(lab, 0, axis=ax)
        b = np.take(lab, -1, axis=ax)
        m = (a > 0) & (b > 0)
        for u, v in set(zip(a[m].tolist(), b[m].tolist())):
            ru, rv = find(u), find(v)
            if ru != rv:
                parent[ru] = rv
    lo = {find(int(v)) for v in np.unique(np.take(lab, 0, axis=axis)) if v}
    hi = {find(int(v)) for v in np.unique(np.take(lab, -1, axis=axis)) if v}
    return bool(lo & hi)


def labels_from_mask(fluid, fluid_label=75, solid_label=255):
    return np.where(fluid, fluid_label, solid_label).astype(np.uint8)


def channel(nx=8, ny=10, nz=4, fluid_label=75, solid_label=255):
    """The channel of examples/generate.py: solid planes at y = 0 and y = ny-1."""
    g = np.full((nz, ny, nx), fluid_label, np.uint8)
    g[:, 0, :] = solid_label
    g[:, ny - 1, :] = solid_label
    return g
