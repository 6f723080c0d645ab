"""Host-side pieces of the learned warm start (no GPU): input features, target
scaling, network size, and the cold-start fallback of the convergence loop
driven by a scripted engine."""
import math

import numpy as np
import pytest
import torch


def test_network_size_and_spec():
    from lbflow_b200 import warmstart as ws
    net = ws.WarmStartNet()
    n = sum(p.numel() for p in net.parameters())
    assert 1.5e6 <= n <= 2.0e6
    # Every gathered channel count is a multiple of 8 (the kernels' 16-byte pieces).
    for name, kind, cin, cout in ws._spec():
        assert cin % 8 == 0, name
        if name != 'head':
            assert cout % 8 == 0, name


def test_features_periodic_and_signed():
    from lbflow_b200 import warmstart as ws
    rng = np.random.default_rng(0)
    fl = torch.from_numpy(rng.random((1, 16, 12, 20)) < 0.4)
    f = ws.features(fl).float()
    assert f.shape == (1, 16, 12, 20, 8)
    assert torch.equal(f[..., 0], fl.float())
    sdf = f[..., 1]
    assert torch.all(sdf[fl] > 0) and torch.all(sdf[~fl] < 0)
    # A pore voxel with a solid face neighbour is at chessboard distance 1.
    solid = ~fl[0]
    near = torch.zeros_like(solid)
    for ax in range(3):
        for s in (1, -1):
            near |= torch.roll(solid, s, ax)
    assert torch.allclose(sdf[0][fl[0] & near], torch.tensor(1 / 8.0))
    # Translation equivariance under periodic shifts.
    g = ws.features(torch.roll(fl, (3, -2, 5), (1, 2, 3))).float()
    assert torch.equal(g, torch.roll(f, (3, -2, 5), (1, 2, 3)))
    assert torch.allclose(f[..., 4], fl.float().mean(), atol=2e-3)   # bf16 features


def test_target_scaling():
    from lbflow_b200 import warmstart as ws
    rho = np.full((4, 4, 4), 1.0 + 3 * 1e-5 * 2.0)
    rho[0, 0, 0] = 0.0                      # solid voxel
    u = np.zeros((3, 4, 4, 4))
    u[0] = 0.5 * 1e-5 / ((1.0 - 0.5) / 3)  # k_x = 0.5 at tau = 1, g = 1e-5
    t = ws.targets(rho, u, 1.0, 1e-5)
    assert t.shape == (4, 4, 4, 4)
    assert np.allclose(t[..., 0], 0.5) and np.allclose(t[1:, ..., 3], 2.0)
    assert t[0, 0, 0, 3] == 0.0


class ScriptedEngine:
    """Stands in for lbflow_b200.Engine: residuals follow a script per start."""

    dims, N = 3, 1000

    def __init__(self, warm_script, cold_script, warm_raises_at=None):
        self.scripts = {'warm': warm_script, 'cold': cold_script}
        self.mode = None
        self.k = 0
        self.raise_at = warm_raises_at
        self.starts = []

    def warm(self):
        self.mode, self.k = 'warm', 0
        self.starts.append('warm')

    def initialize(self):
        self.mode, self.k = 'cold', 0
        self.starts.append('cold')

    def step(self, n, macros=False, adjacent=False):
        if macros:
            self.k += 1

    def synchronize(self):
        pass

    def check(self):
        if self.mode == 'warm' and self.raise_at is not None and self.k >= self.raise_at:
            raise RuntimeError('device error word')

    def _res(self):
        sc = self.scripts[self.mode]
        return sc[min(self.k - 1, len(sc) - 1)]

    def convergence(self, first=False):
        r = self._res()
        return np.array([r * r * 1.0, 1.0, r * r * 1.0, 0, 0, 0])

    def flux_sums(self):
        return np.zeros(9)


def test_converge_keeps_a_good_warm_start():
    from lbflow_b200.permeability import converge
    e = ScriptedEngine([1e-3, 1e-4, 1e-5, 5e-7, 4e-7, 3e-7, 2e-7], [1.0])
    r = converge(e, 1.0, 1e-5, report=10, warm=e.warm)
    assert r['converged'] and not r['fallback'] and e.starts == ['warm']
    assert r['steps'] == 60      # first report + 5 residual reports, the last 3 below tol


def test_converge_falls_back_when_warm_start_stalls():
    from lbflow_b200.permeability import converge
    stall = [1e-2] * 20
    cold = [1e-1, 1e-3, 1e-5, 5e-7, 4e-7, 3e-7]
    e = ScriptedEngine(stall, cold)
    r = converge(e, 1.0, 1e-5, report=10, warm=e.warm, patience=5)
    assert r['fallback'] and e.starts == ['warm', 'cold'] and r['converged']
    # 1 first report + 6 reports without a new minimum, then the cold run's 6.
    assert r['steps'] == (1 + 1 + 5) * 10 + 6 * 10


def test_converge_falls_back_on_device_error():
    from lbflow_b200.permeability import converge
    e = ScriptedEngine([1e-3] * 10, [1e-1, 1e-3, 5e-7, 4e-7, 3e-7], warm_raises_at=2)
    r = converge(e, 1.0, 1e-5, report=10, warm=e.warm)
    assert r['fallback'] and r['converged'] and e.starts == ['warm', 'cold']


def test_cold_start_never_falls_back():
    from lbflow_b200.permeability import converge
    e = ScriptedEngine([1.0], [1e-2] * 12)
    r = converge(e, 1.0, 1e-5, report=10, max_steps=120)
    assert not r['converged'] and not r['fallback'] and e.starts == ['cold']


def test_stall_near_tolerance_is_not_a_fallback():
    from lbflow_b200.permeability import converge
    floor = [1e-3, 1e-4, 2e-6] + [2e-6] * 20     # a storage-precision floor just above tol
    e = ScriptedEngine(floor, [1.0])
    r = converge(e, 1.0, 1e-5, report=10, tol=1e-6, warm=e.warm, max_steps=200)
    assert not r['fallback'] and e.starts == ['warm']
    assert math.isclose(r['steps'], 200)


def test_darcy_pressure_layered_medium():
    """Series layers along x: the conservative flux is uniform at the harmonic
    mean mobility and the pressure gradient is g - q / M(x)."""
    from lbflow_b200 import warmstart as ws
    g, b = 1e-5, 4
    D, H, W = 8, 8, 128
    x = (torch.arange(W, dtype=torch.float64) + 0.5) / W
    M = 1.0 + 0.6 * torch.sin(2 * math.pi * x)                     # voxel mobility along x
    mob = ws._block_mean(M.expand(D, H, W)[..., None], b)[..., 0]
    phi = ws.darcy_pressure(mob, g, b, face='harmonic')
    mf = 2 * mob * torch.roll(mob, -1, 2) / (mob + torch.roll(mob, -1, 2))
    face = mf * (g - (torch.roll(phi, -1, 2) - phi) / b)            # x flux through each + face
    assert float(face.std() / face.mean()) < 1e-8
    qh = g / float((1.0 / M).mean())
    assert abs(float(face.mean()) - qh) < 0.02 * qh
    xc = (torch.arange(W // b, dtype=torch.float64) + 0.5) * b
    prof = torch.cumsum(g - qh / M, 0)
    ref = prof[(xc - 0.5).long()]
    ref = ref - ref.mean()
    got = phi[0, 0]
    assert float((got - ref).norm() / ref.norm()) < 0.05
    assert torch.allclose(phi[1, 1], phi[0, 0])                    # uniform across y, z
    # The flux form gives the same pressure from the local response M g.
    q = torch.zeros(D // b, H // b, W // b, 3, dtype=torch.float64)
    q[..., 0] = mob * g
    phi2 = ws.darcy_pressure_from_flux(q, mob, b, face='harmonic')
    assert float((phi2 - phi).norm() / phi.norm()) < 0.05


def test_darcy_pressure_removes_divergence_3d():
    from lbflow_b200 import warmstart as ws
    gen = torch.Generator().manual_seed(3)
    q = torch.rand(6, 8, 10, 3, generator=gen, dtype=torch.float64) * 1e-5
    mob = 0.5 + torch.rand(6, 8, 10, generator=gen, dtype=torch.float64)
    b = 8
    phi = ws.darcy_pressure_from_flux(q, mob, b, face='harmonic')
    div = torch.zeros_like(mob)
    for c, ax in enumerate((2, 1, 0)):
        nb = torch.roll(mob, -1, ax)
        mf = 2 * mob * nb / (mob + nb)
        face = 0.5 * (q[..., c] + torch.roll(q[..., c], -1, ax)) - mf * (torch.roll(phi, -1, ax) - phi) / b
        div += (face - torch.roll(face, 1, ax)) / b
    assert float(div.abs().max()) < 1e-6 * float(q.abs().max()) / b     # CG stops at 1e-8 relative
    assert abs(float(phi.mean())) < 1e-18


def test_upsample_periodic_reproduces_linear_and_constant_fields():
    from lbflow_b200 import warmstart as ws
    phi = torch.full((3, 4, 5), 2.5, dtype=torch.float64)
    up = ws._upsample_periodic(phi, 4)
    assert up.shape == (12, 16, 20) and torch.allclose(up, torch.full_like(up, 2.5))
    # A periodic cosine along x sampled at block centres interpolates close to the voxel values.
    w, b = 16, 4
    xc = (torch.arange(w, dtype=torch.float64) + 0.5) * b - 0.5
    phi = torch.cos(2 * math.pi * xc / (w * b)).expand(2, 2, w).contiguous()
    up = ws._upsample_periodic(phi, b)
    xv = torch.arange(w * b, dtype=torch.float64)
    assert float((up[0, 0] - torch.cos(2 * math.pi * xv / (w * b))).abs().max()) < 0.02


def test_smooth121_removes_grid_scale_mode():
    from lbflow_b200 import warmstart as ws
    D, H, W = 8, 6, 10
    z, y, x = torch.meshgrid(torch.arange(D), torch.arange(H), torch.arange(W), indexing='ij')
    m = torch.ones(D, H, W, dtype=torch.float64)
    stag = ((-1.0) ** (x + y + z)).double()
    assert float(ws._smooth121(stag, m).abs().max()) < 1e-12
    smooth = torch.cos(2 * math.pi * x.double() / W)
    expect = smooth * (0.5 + 0.5 * math.cos(2 * math.pi / W))
    assert float((ws._smooth121(smooth, m) - expect).abs().max()) < 1e-12
    # Solid voxels stay zero and a constant field over the pores is kept.
    m[2:4, 2:4, 2:4] = 0
    out = ws._smooth121(torch.full((D, H, W), 3.0, dtype=torch.float64), m)
    assert torch.allclose(out[m > 0], torch.tensor(3.0, dtype=torch.float64)) and float(out[m == 0].abs().max()) == 0


def test_multigrid_transfers_are_adjoint_and_solver_converges():
    """The V-cycle's restriction is the adjoint of its prolongation / 8 (so the
    preconditioner is symmetric), and the preconditioned solve of a
    high-contrast mobility field converges in a few dozen iterations."""
    from lbflow_b200 import warmstart as ws
    gen = torch.Generator().manual_seed(1)
    e = torch.randn(4, 6, 8, generator=gen, dtype=torch.float64)
    r = torch.randn(8, 12, 16, generator=gen, dtype=torch.float64)
    assert math.isclose(float((ws._prolong(e) * r).sum()), float(8 * (e * ws._restrict(r)).sum()), rel_tol=1e-12)
    mob = torch.exp(2.0 * torch.randn(16, 16, 32, generator=gen, dtype=torch.float64))
    mob[torch.rand(16, 16, 32, generator=gen) < 0.3] = 1e-4
    phi = ws.darcy_pressure(mob, 1e-5, 2, rtol=1e-8)
    assert ws._solve_periodic.iterations < 120
    mf = ws._face_mobility(mob)
    rhs = 1e-5 * (mf[0] - torch.roll(mf[0], 1, 2)) / 2
    res = ws._apply(phi, mf, 2.0) - (rhs - rhs.mean())
    assert float(res.norm() / rhs.norm()) < 1e-7


def test_block_mobility_of_uniform_and_pressure_driven_flow():
    """The accelerator's estimator: M = q / (g - dphi/dx) along x, exact for
    a uniform flux under a linear pressure ramp (periodic wrap excluded)."""
    from lbflow_b200 import warmstart as ws
    b, g = 2, 1e-5
    nb = (3, 4, 6)
    s = torch.zeros(*nb, 5, dtype=torch.float64)
    s[..., 4] = b ** 3
    s[..., 0] = b ** 3                       # rho = 1: no pressure gradient
    s[..., 1] = 2.5e-6 * b ** 3               # q_x = 2.5e-6
    mob, cnt, phi = ws.block_mobility(s, g, b)
    assert torch.allclose(mob, torch.full(nb, 2.5e-6 / g, dtype=torch.float64))
    assert torch.equal(cnt, s[..., 4]) and torch.all(phi == 0)
    # Pressure rising along x by dp per block: drive = g - dp / b.
    dp = 3e-6
    x = torch.arange(nb[2], dtype=torch.float64)
    rho = 1.0 + 3.0 * dp * x
    s[..., 0] = rho * b ** 3
    mob, _, _ = ws.block_mobility(s, g, b)
    inner = mob[..., 1:-1]
    assert torch.allclose(inner, torch.full_like(inner, 2.5e-6 / (g - dp / b)))


def test_block_sums_dense_layout():
    from lbflow_b200 import warmstart as ws
    rng = np.random.default_rng(1)
    fl = torch.from_numpy(rng.random((4, 6, 8)) < 0.5)
    rho = torch.from_numpy(1 + rng.random((4, 6, 8)) * 1e-3) * fl
    u = torch.from_numpy(rng.standard_normal((3, 4, 6, 8))) * fl
    s = ws.block_sums_dense(rho, u, fl, 2)
    assert s.shape == (2, 3, 4, 5)
    blk = (slice(2, 4), slice(0, 2), slice(4, 6))
    assert torch.isclose(s[1, 0, 2, 0], rho[blk].sum())
    assert torch.isclose(s[1, 0, 2, 2], u[1][blk].sum())
    assert s[1, 0, 2, 4] == fl[blk].sum()


def test_mobility_network_shape_and_targets():
    from lbflow_b200 import warmstart as ws
    net = ws.MobilityNet()
    assert net.norm.tolist() == [0.0, 1.0]
    assert set(net.state_dict()) == set(ws.WarmStartNet().state_dict()) | {'norm'}
    rng = np.random.default_rng(2)
    fl = torch.from_numpy(rng.random((4, 4, 4)) < 0.6)
    u = torch.zeros(3, 4, 4, 4, dtype=torch.float64)
    u[0] = 1e-6 * fl
    t, w = ws.mobility_targets(torch.ones(4, 4, 4, dtype=torch.float64) * fl, u, fl, 1.0, 1e-5)
    assert t.shape == (2, 2, 2) and w.shape == (2, 2, 2)
    # Blocks with fluid: q = 1e-6 * count / 8, M = q / g, target log(M nu).
    for idx in np.ndindex(2, 2, 2):
        if w[idx] > 0:
            want = math.log(1e-6 * float(w[idx]) / 8 / 1e-5 / 6)
            assert abs(float(t[idx]) - want) < 1e-5
