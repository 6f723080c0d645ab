"""Small solver cases shared by the golden-fixture script and the tests.

Each case is a dict with the geometry (uint8, shaped (nz, ny, nx) or (ny, nx)),
the label table, the model parameters and the step count.  The geometries
follow the reference's own test inputs: the channel of examples/generate.py,
the uniform body-force boxes of scripts/benchmarks.py:176-188, the drop of
scripts/ci_smoke.py:50-54, plus small porous media made with the
Gaussian-filtered-noise recipe (lbflow_b200.geometry).
"""
import numpy as np


def _labels_channel(force):
    return {75: ('GV', force, 1, 0), 255: ('SD', 90.0, 0, 0)}


def channel_config1():
    """Config 1: 8x10x4 channel, SD planes at y=0 and y=9, SRT tau=0.8, g_x=1e-6, 20000 steps."""
    nx, ny, nz = 8, 10, 4
    g = np.full((nz, ny, nx), 75, np.uint8)
    g[:, 0, :] = 255
    g[:, ny - 1, :] = 255
    return dict(name='channel-config1', geometry=g, labels=_labels_channel(1e-6), model='scsp',
                collision='SRT', tau=(0.8,), rho=(1.0,), steps=20000, write=20000)


def channel_mrt():
    """examples/generate.py channel: MRT tau=1, 1000 steps."""
    c = channel_config1()
    c.update(name='channel-mrt', collision='MRT', tau=(1.0,), steps=1000, write=1000)
    return c


def force_cases():
    """Uniform periodic GV boxes (scripts/benchmarks.py:176-188): u_x = 1e-4 after 100 steps."""
    out = []
    for model in ('scsp', 'color'):
        for ndim in (2, 3):
            for eq in ('SRT', 'MRT'):
                for tau in (0.6, 1.4):
                    nx, ny, nz = 8, 6, (1 if ndim == 2 else 4)
                    shape = (ny, nx) if ndim == 2 else (nz, ny, nx)
                    g = np.full(shape, 75, np.uint8)
                    ph = 1 if model == 'color' else 0
                    out.append(dict(name=f'force-{model}-d{ndim}-{eq}-tau{tau}', geometry=g,
                                    labels={75: ('GV', 1e-6, 1, ph)}, model=model, collision=eq,
                                    tau=(0.8, tau) if model == 'color' else (tau,),
                                    rho=(1.0, 1.0) if model == 'color' else (1.0,),
                                    alpha0=4 / 9 if ndim == 2 else 1 / 3, sigma=0.005, beta=0.7,
                                    steps=100, write=50))
    return out


def drop_3d():
    """scripts/ci_smoke.py drop: 12^3 color D3Q19 MRT, 40 steps."""
    n = 12
    z, y, x = np.mgrid[0:n, 0:n, 0:n]
    g = np.where((x - 5.5) ** 2 + (y - 5.5) ** 2 + (z - 5.5) ** 2 <= 9, 100, 0).astype(np.uint8)
    return dict(name='drop-3d', geometry=g, labels={0: ('VD', 0, 0, 0), 100: ('VD', 0, 0, 1)},
                model='color', collision='MRT', tau=(1.0, 1.0), rho=(1.0, 1.0), alpha0=1 / 3,
                sigma=0.005, beta=0.7, steps=40, write=20)


def wall_color_3d(tau1=0.7, collision='MRT'):
    """Two-phase channel with an obstacle, SD walls at 60 degrees, GV in x per phase."""
    nx, ny, nz = 12, 10, 8
    g = np.full((nz, ny, nx), 75, np.uint8)
    g[:, 0, :] = 255
    g[:, -1, :] = 255
    g[3:5, 4:6, 3:6] = 255
    blk = g[2:6, 2:8, 7:11]
    blk[blk == 75] = 76
    return dict(name=f'wall-color-3d-{collision}-{tau1}', geometry=g,
                labels={75: ('GV', 2e-6, 1, 0), 76: ('GV', 2e-6, 1, 1), 255: ('SD', 60.0, 0, 0)},
                model='color', collision=collision, tau=(1.0, tau1), rho=(1.0, 1.0), alpha0=1 / 3,
                sigma=1e-3, beta=0.7, steps=200, write=200)


def wall_color_2d(collision='MRT'):
    """D2Q9 drop between SD walls (45 degrees) with a BB block."""
    nx, ny = 20, 16
    g = np.zeros((ny, nx), np.uint8)
    g[0, :] = 255
    g[-1, :] = 255
    g[6:9, 12:15] = 254
    yy, xx = np.mgrid[0:ny, 0:nx]
    g[((xx - 6) ** 2 + (yy - 7) ** 2 <= 9) & (g == 0)] = 100
    return dict(name=f'wall-color-2d-{collision}', geometry=g,
                labels={0: ('VD', 0, 0, 0), 100: ('VD', 0, 0, 1), 255: ('SD', 45.0, 0, 0),
                        254: ('BB', 0.0, 0, 0)},
                model='color', collision=collision, tau=(1.0, 0.8), rho=(1.0, 1.0), alpha0=4 / 9,
                sigma=5e-3, beta=0.7, steps=300, write=300)


def porous_scsp(collision='MRT', n=(16, 16, 12), seed=7):
    """Small Gaussian-filtered porous medium, single phase, GV in x."""
    from lbflow_b200.geometry import porous_medium
    nx, ny, nz = n
    fluid = porous_medium((nz, ny, nx), sigma=2.0, porosity=0.35, seed=seed)
    g = np.where(fluid, 75, 255).astype(np.uint8)
    return dict(name=f'porous-scsp-{collision}', geometry=g,
                labels={75: ('GV', 1e-5, 1, 0), 255: ('SD', 90.0, 0, 0)},
                model='scsp', collision=collision, tau=(1.0,), rho=(1.0,), steps=300, write=300)


def porous_scsp_2d(collision='MRT'):
    from lbflow_b200.geometry import porous_medium
    fluid = porous_medium((1, 40, 48), sigma=2.0, porosity=0.5, seed=3)[0]
    g = np.where(fluid, 75, 255).astype(np.uint8)
    return dict(name=f'porous-scsp-2d-{collision}', geometry=g,
                labels={75: ('GV', 1e-5, 1, 0), 255: ('BB', 0.0, 0, 0)},
                model='scsp', collision=collision, tau=(0.9,), rho=(1.0,), steps=400, write=400)


def _boundary_channel(name, shape, axis, lo, hi, walls, collision, tau=(1.0,), wall_type='SD', steps=300):
    """A channel along `axis` (0 = x, 1 = y, 2 = z) with Zou-He boundary planes:
    `lo` / `hi` = (type, value, dir) on the first / last plane across the axis,
    solid planes at both ends of the `walls` axis, VD inside."""
    g = np.full(shape, 75, np.uint8)
    nd = len(shape)

    def sl(ax, i):
        idx = [slice(None)] * nd
        idx[nd - 1 - ax] = i
        return tuple(idx)
    g[sl(axis, 0)] = 50
    g[sl(axis, -1)] = 200
    g[sl(walls, 0)] = 255
    g[sl(walls, -1)] = 255
    labels = {75: ('VD', 0, 0, 0), 50: (lo[0], lo[1], lo[2], 0), 200: (hi[0], hi[1], hi[2], 0),
              255: (wall_type, 90.0 if wall_type == 'SD' else 0.0, 0, 0)}
    return dict(name=name, geometry=g, labels=labels, model='scsp', collision=collision, tau=tau,
                rho=(1.0,), steps=steps, write=steps)


def zou_he_cases():
    """Pressure (PB) and velocity (VB) boundaries, SCSP::zouHeBoundary
    (scsp.cpp:188-275), on every axis and both signs, D2Q9 and D3Q19, the
    pressure channel of scripts/porous_media.py:257-279 in small, and a porous
    medium whose inlet plane mixes PB voxels with bounce-back links."""
    dp = 1 + 3 * 1e-4
    out = [
        _boundary_channel('pb-channel-d3-MRT', (3, 8, 17), 0, ('PB', dp, 1), ('PB', 1.0, 2), 1, 'MRT'),
        _boundary_channel('pb-channel-d3-SRT', (3, 8, 17), 0, ('PB', dp, 1), ('PB', 1.0, 2), 1, 'SRT',
                          tau=(0.8,)),
        _boundary_channel('vb-channel-d3-MRT', (3, 8, 17), 0, ('VB', 1e-3, 1), ('PB', 1.0, 2), 1, 'MRT'),
        _boundary_channel('vb-channel-y-d3-SRT', (3, 17, 8), 1, ('PB', 1.0, 3), ('VB', 1e-3, 4), 0, 'SRT',
                          tau=(0.7,)),
        _boundary_channel('pb-channel-z-d3-MRT', (17, 8, 4), 2, ('PB', dp, 5), ('PB', 1.0, 6), 1, 'MRT',
                          tau=(1.3,)),
        _boundary_channel('pb-channel-d2-MRT', (10, 24), 0, ('PB', dp, 1), ('PB', 1.0, 3), 1, 'MRT'),
        _boundary_channel('vb-channel-y-d2-SRT', (24, 10), 1, ('PB', 1.0, 2), ('VB', 5e-4, 4), 0, 'SRT',
                          tau=(0.9,), wall_type='BB'),
    ]
    c = porous_scsp('MRT')
    g = c['geometry'].copy()
    g[:, :, 0][g[:, :, 0] == 75] = 50
    g[:, :, -1][g[:, :, -1] == 75] = 200
    c.update(name='pb-porous-d3-MRT', geometry=g,
             labels={75: ('VD', 0, 0, 0), 50: ('PB', dp, 1, 0), 200: ('PB', 1.0, 2, 0),
                     255: ('SD', 90.0, 0, 0)})
    out.append(c)
    return out


def entry_case(ratio=1.5, ndim=2, h=16, nx=None, steps=8000, write=2000, collision='MRT', tau=(1.0, 1.0)):
    """The capillary-entry slit of scripts/porous_media.py:154-182 (entry_cases,
    legacy walls): phase 0 fills x < h and is pushed by a PB inlet (density
    1 + 3 dp, phase 0, direction +x) into a slit of phase 1 held by a PB outlet
    (density 1, phase 1, direction -x); SD walls at 60 degrees; dp = ratio
    times the sharp entry pressure 2 sigma cos 60 / h (4 sigma ... in 3D)."""
    import math
    nx = nx or 4 * h + 1
    sigma = 0.005 * 16 / h if h != 16 else 0.005
    pc = (2 if ndim == 2 else 4) * sigma * math.cos(math.radians(60)) / h
    dp = ratio * pc
    shape = (h + 2, nx) if ndim == 2 else (h + 2, h + 2, nx)
    g = np.full(shape, 100, np.uint8)
    xs = np.arange(nx)
    g[..., xs < h] = 0
    g[..., 0] = 50
    g[..., -1] = 200
    if ndim == 2:
        g[0, :] = 255
        g[-1, :] = 255
    else:
        g[:, 0, :] = 255
        g[:, -1, :] = 255
        g[0, :, :] = 255
        g[-1, :, :] = 255
    name = 'entry-' + ('d3-' if ndim == 3 else '') + f'h{h}-ratio{ratio}-{collision}'
    return dict(name=name, geometry=g,
                labels={50: ('PB', 1 + 3 * dp, 1, 0), 200: ('PB', 1.0, 3 if ndim == 2 else 2, 1),
                        0: ('VD', 0, 0, 0), 100: ('VD', 0, 0, 1), 255: ('SD', 60.0, 0, 0)},
                model='color', collision=collision, tau=tau, rho=(1.0, 1.0),
                alpha0=4 / 9 if ndim == 2 else 1 / 3, sigma=sigma, beta=0.7, steps=steps, write=write,
                height=h, pressure_ratio=ratio, sharp_entry_pressure=pc, pressure_drop=dp)


def color_zou_he_cases():
    """Two-phase Zou-He boundaries, ColorFluid::zouHeBoundary
    (colorfluid.cpp:638-734): the entry slit in 2D and 3D, a VB inlet with
    unequal viscosities (per-node MRT rates), and an SRT channel along -y."""
    out = [entry_case(1.5, 2, steps=400, write=400),
           entry_case(0.5, 2, collision='SRT', tau=(1.0, 0.8), steps=400, write=400),
           entry_case(1.5, 3, h=6, nx=25, steps=200, write=200)]
    c = entry_case(1.5, 2, h=8, nx=33, steps=300, write=300, tau=(1.0, 0.7))
    c['labels'] = dict(c['labels'])
    c['labels'][50] = ('VB', 2e-3, 1, 0)
    c['name'] = 'vb-color-d2-h8-MRT'
    out.append(c)
    # Along -y in 3D: VB (phase 1) on the y = ny-1 plane pushing into phase 0,
    # PB (phase 0) on y = 0; SD walls on the x planes.
    nx, ny, nz = 8, 20, 4
    g = np.full((nz, ny, nx), 0, np.uint8)
    g[:, ny // 2:, :] = 100
    g[:, 0, :] = 50
    g[:, -1, :] = 200
    g[:, :, 0] = 255
    g[:, :, -1] = 255
    out.append(dict(name='vb-color-y-d3-SRT', geometry=g,
                    labels={50: ('PB', 1.0, 3, 0), 200: ('VB', 1e-3, 4, 1), 0: ('VD', 0, 0, 0),
                            100: ('VD', 0, 0, 1), 255: ('SD', 90.0, 0, 0)},
                    model='color', collision='SRT', tau=(1.0, 1.0), rho=(1.0, 1.0), alpha0=1 / 3,
                    sigma=0.003, beta=0.7, steps=200, write=200))
    return out


def film_cases():
    """Half-permeable films (HF; simulator.cpp:418-421, colorfluid.cpp:155-158,
    752-765): a film voxel lets its own phase through and bounces the other
    back, and holds only its own phase.  A D2Q9 channel driven by GV forces
    through a phase-0 film, and a D3Q19 tube after the reference's HalfFilm
    sample: a film of each phase across the inlet side, VB inlets per phase,
    a PB outlet, unequal densities and viscosities."""
    nx, ny = 24, 12
    g = np.full((ny, nx), 0, np.uint8)
    g[:, nx // 2:] = 100
    g[:, 8:10] = 25
    g[0, :] = 255
    g[-1, :] = 255
    d2 = dict(name='film-d2-MRT', geometry=g,
              labels={0: ('GV', 2e-5, 1, 0), 100: ('GV', 2e-5, 1, 1), 25: ('HF', 0, 0, 0),
                      255: ('SD', 90.0, 0, 0)},
              model='color', collision='MRT', tau=(1.0, 0.8), rho=(1.0, 1.0), alpha0=4 / 9,
              sigma=5e-3, beta=0.7, steps=300, write=300)
    nx, ny, nz = 8, 6, 24
    g = np.full((nz, ny, nx), 0, np.uint8)
    g[:, :, nx // 2:] = 100
    g[0, :, :nx // 2] = 50
    g[0, :, nx // 2:] = 150
    g[3:5, :, :nx // 2] = 25
    g[3:5, :, nx // 2:] = 125
    g[-1] = 200
    g[:, 0, :] = 255
    g[:, -1, :] = 255
    d3 = dict(name='film-d3-MRT', geometry=g,
              labels={0: ('VD', 0, 0, 0), 25: ('HF', 0, 0, 0), 50: ('VB', 1e-3, 5, 0),
                      100: ('VD', 0, 0, 1), 125: ('HF', 0, 0, 1), 150: ('VB', 1e-3, 5, 1),
                      200: ('PB', 1.0, 6, 0), 255: ('SD', 90.0, 0, 0)},
              model='color', collision='MRT', tau=(0.57, 1.2154), rho=(1.0, 0.831683168), alpha0=1 / 3,
              sigma=0.0859, beta=0.7, steps=200, write=200)
    return [d2, d3]


def pressure_report_channel():
    """scripts/porous_media.py:257-279 (pressure_study): a 16-wide slit between
    SD walls, PB inlet 1 + 3e-5 and outlet 1 along x, MRT tau 1, 6000 steps,
    reports every 2000 steps, latticeLen 1e-6 so that K is in lattice units.
    The reference accepts it when the reported pressure drop and K are within
    2e-4 of dp (nx - 3) / (nx - 1) and (h^3/12 + h/24) / (h + 2)."""
    h, nx, nz, dp = 16, 65, 4, 1e-5
    g = np.full((nz, h + 2, nx), 75, np.uint8)
    g[:, :, 0] = 50
    g[:, :, -1] = 200
    g[:, 0, :] = 255
    g[:, -1, :] = 255
    return dict(name='pressure-channel-report', geometry=g,
                labels={50: ('PB', 1 + 3 * dp, 1, 0), 200: ('PB', 1.0, 2, 0), 75: ('VD', 0, 0, 0),
                        255: ('SD', 90.0, 0, 0)},
                model='scsp', collision='MRT', tau=(1.0,), rho=(1.0,), steps=6000, write=2000,
                stop_error=1e-12, lattice_len=1e-6, h=h, dp=dp)


def golden_cases():
    """The cases whose reference outputs are committed under tests/golden/."""
    return ([channel_config1(), channel_mrt(), drop_3d(), wall_color_3d(0.7, 'MRT'),
             wall_color_3d(1.0, 'SRT'), wall_color_2d('MRT'), wall_color_2d('SRT'),
             porous_scsp('MRT'), porous_scsp('SRT'), porous_scsp_2d('MRT')] + force_cases()
            + zou_he_cases() + color_zou_he_cases() + film_cases())


def prm_text(case, grid_file='geometry.raw', out='field', report_dir=0):
    """An input.prm for the case, in the form scripts/benchmarks.py writes (:73-101)."""
    g = case['geometry']
    ndim = 2 if g.ndim == 2 else 3
    if ndim == 2:
        ny, nx = g.shape
        dims = f'{ny} {nx}'
    else:
        nz, ny, nx = g.shape
        dims = f'{nz} {ny} {nx}'
    color = case['model'] == 'color'
    lines = [
        f'gridFile "{grid_file}";', f'dimension {dims};', f'directions {9 if ndim == 2 else 19};',
        'fileType "uint8";', f'latticeLen {case.get("lattice_len", 1)};', 'startTime 0;', f'endTime {case["steps"]};',
        f'writeInterval {case["write"]};', f'reportInterval {case.get("report", case["write"])};',
        f'restartInterval {case.get("restart", case["steps"])};',
        f'stopError {case.get("stop_error", 1e-8)};', f'outPath "{out}";', 'logPath ".";',
        f'reportDir {report_dir};', f'reportSlice 1 {nx - 2};',
        f'fluidModel "{case["model"]}";', f'equilModel "{case["collision"]}";',
        'rexlationTime ' + ' '.join(format(t, '.17g') for t in case['tau']) + ';',
        'latticeSpeed 1;', f'alpha0 {format(case.get("alpha0", 1 / 3), ".17g")};',
        'density ' + ' '.join(map(str, case['rho'])) + ';', 'contactAngle 90;',
        f'surfaceTension {case.get("sigma", 0.005)};', f'interfaceThickness {case.get("beta", 0.7)};',
        'wallGradient "legacy";', 'viscosityInterpolation "arithmetic";',
    ]
    for k, (t, v, d, ph) in sorted(case['labels'].items()):
        val = 'N/A' if t in ('VD', 'BB') else format(v, '.17g') if t in ('GV', 'PB', 'VB') else format(v, 'g')
        dr = str(d) if t in ('GV', 'PB', 'VB') else 'N/A'
        p = str(ph) if t in ('VD', 'GV', 'PB', 'VB', 'HF') else 'N/A'
        lines.append(f'{k} "{t}" "{val}" "{dr}" "{p}"')
    if not color:
        pass
    return '\n'.join(lines) + '\n'
