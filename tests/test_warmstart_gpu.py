"""The learned warm start on the GPU.

 - The whole network (forward and backward through the tcgen05 kernels)
   against the same network in torch FP64 on the CPU, with activations
   rounded to bf16 where the GPU stores them.
 - lbf_initialize_equilibrium reproduces the fields it is given.
 - Starting from a converged solution converges at once to the same K; the
   trained operator (when its weights are present) reaches the K band in
   fewer steps than the start from rest.
"""
from pathlib import Path

import numpy as np
import pytest
import torch
import torch.nn.functional as F

pytestmark = pytest.mark.gpu

LABELS = {75: ('GV', 1e-5, 1, 0), 255: ('SD', 90.0, 0, 0)}
WEIGHTS = Path(__file__).resolve().parent.parent / 'lbflow_b200' / 'weights' / 'warmstart.pt'


def _cf(x):
    return x.permute(0, 4, 1, 2, 3)


def _cl(x):
    return x.permute(0, 2, 3, 4, 1)


def _bf(x):
    """bf16 rounding of a stored activation, identity for the gradient."""
    return x + (x.to(torch.bfloat16).double() - x).detach()


def ref_forward(net, x):
    from lbflow_b200.warmstart import SLOPE
    P = {n[:-2]: (getattr(net, n[:-2] + '_w').detach().cpu().to(torch.bfloat16).double().requires_grad_(True),
                  getattr(net, n[:-2] + '_b').detach().cpu().double().requires_grad_(True))
         for n, _ in net.named_parameters() if n.endswith('_w')}

    def c3(name, x, skip=None, act=True):
        w, b = P[name]
        if skip is not None:
            x = torch.cat([x, skip], -1)
        y = F.conv3d(F.pad(_cf(x), (1, 1, 1, 1, 1, 1), mode='circular'), w, b)
        return _bf(_cl(F.leaky_relu(y, SLOPE) if act else y))

    def d2(name, x):
        w, b = P[name]
        return _bf(_cl(F.leaky_relu(F.conv3d(_cf(x), w, b, stride=2), SLOPE)))

    def u2(name, x):
        w, b = P[name]
        return _bf(_cl(F.leaky_relu(F.conv_transpose3d(_cf(x), w, b, stride=2), SLOPE)))

    e1 = c3('enc1b', c3('enc1a', x))
    e2 = c3('enc2b', c3('enc2a', d2('down1', e1)))
    e3 = c3('enc3b', c3('enc3a', d2('down2', e2)))
    m = c3('midb', c3('mida', d2('down3', e3)))
    d3 = c3('dec3b', c3('dec3a', u2('up3', m), skip=e3))
    d2_ = c3('dec2b', c3('dec2a', u2('up2', d3), skip=e2))
    d1 = c3('dec1b', c3('dec1a', u2('up1', d2_), skip=e1))
    return c3('head', d1, act=False), P


def _rel(a, b):
    return float((a - b).detach().norm() / b.detach().norm().clamp(min=1e-300))


def _linear_ref(kind, x, w, b):
    """FP64 oracle of one layer without its activation (channels-last in/out)."""
    if kind == 'conv3':
        return _cl(F.conv3d(F.pad(_cf(x), (1, 1, 1, 1, 1, 1), mode='circular'), w, b))
    if kind == 'down2':
        return _cl(F.conv3d(_cf(x), w, b, stride=2))
    return _cl(F.conv_transpose3d(_cf(x), w, b, stride=2))


@pytest.fixture
def recorded_network(monkeypatch):
    """A random network run forward and backward on the GPU with every layer
    call recorded: its inputs, weights, output and the gradient arriving at
    the output."""
    from lbflow_b200 import conv
    from lbflow_b200 import warmstart as ws
    calls = []

    def wrap(kind, fn):
        def run(x, w, b, slope=None, x1=None):
            y = fn(x, w, b, slope, x1=x1) if kind == 'conv3' else fn(x, w, b, slope)
            rec = dict(kind=kind, x0=x.detach(), x1=None if x1 is None else x1.detach(), w=w, b=b, slope=slope,
                       y=y.detach())
            y.register_hook(lambda g, rec=rec: rec.__setitem__('gy', g.detach()))
            calls.append(rec)
            return y
        return run

    monkeypatch.setattr(conv, 'conv3', wrap('conv3', conv.conv3))
    monkeypatch.setattr(conv, 'down2', wrap('down2', conv.down2))
    monkeypatch.setattr(conv, 'up2', wrap('up2', conv.up2))
    torch.manual_seed(0)
    net = ws.WarmStartNet(seed=3).cuda()
    with torch.no_grad():
        for n, p in net.named_parameters():
            if n.endswith('_b'):
                p.copy_(0.05 * torch.randn_like(p))   # exercise every bias path
    rng = np.random.default_rng(1)
    fl = torch.from_numpy(rng.random((2, 16, 16, 24)) < 0.35)
    x = ws.features(fl.cuda())
    y = net(x)
    R = torch.randn(y.shape).to(torch.bfloat16)
    (y.float() * R.cuda().float()).sum().backward()
    conv.check()
    monkeypatch.undo()
    return net, x, y, R, calls


def test_network_layers_teacher_forced(recorded_network):
    """Every layer call of a forward and backward pass of the operator,
    checked against the FP64 oracle on that call's own GPU inputs: the output
    to one bf16 rounding, the weight and bias gradients to FP32 accumulation
    and the data gradient to one bf16 rounding.  The backward oracle takes
    the incoming gradient times the leaky-ReLU slope rounded to bf16, as the
    GPU stores it."""
    from lbflow_b200 import conv
    net, _, _, _, calls = recorded_network
    assert len(calls) == 21
    for k, c in enumerate(calls):
        x = c['x0'] if c['x1'] is None else torch.cat([c['x0'], c['x1']], -1)
        xd = x.double().cpu()
        wd = c['w'].detach().cpu().to(torch.bfloat16).double()
        bd = c['b'].detach().cpu().double()
        pre = _linear_ref(c['kind'], xd, wd, bd)
        yref = F.leaky_relu(pre, c['slope']) if c['slope'] is not None else pre
        y = c['y'].double().cpu()
        scale = yref.abs().max().item()
        assert torch.all((y - yref).abs() <= 2.0 ** -8 * yref.abs() + 1e-5 * scale), (k, c['kind'])
        # Backward of this call alone, on the GPU, with the recorded incoming gradient.
        x0 = c['x0'].clone().requires_grad_(True)
        x1 = None if c['x1'] is None else c['x1'].clone().requires_grad_(True)
        w = c['w'].detach().clone().requires_grad_(True)
        b = c['b'].detach().clone().requires_grad_(True)
        fn = {'conv3': conv.conv3, 'down2': conv.down2, 'up2': conv.up2}[c['kind']]
        yy = fn(x0, w, b, c['slope'], x1=x1) if c['kind'] == 'conv3' else fn(x0, w, b, c['slope'])
        ins = [t for t in (x0, x1) if t is not None]
        grads = torch.autograd.grad(yy, ins + [w, b], c['gy'])
        conv.check()
        gy = c['gy'].float().cpu()
        if c['slope'] is not None:
            gy = gy * torch.where(c['y'].cpu() > 0, 1.0, c['slope'])
        dpre = gy.to(torch.bfloat16).double()
        xr = xd.clone().requires_grad_(True)
        wr = wd.clone().requires_grad_(True)
        br = bd.clone().requires_grad_(True)
        gx_r, gw_r, gb_r = torch.autograd.grad(_linear_ref(c['kind'], xr, wr, br), [xr, wr, br], dpre)
        gx = torch.cat([g.double().cpu() for g in grads[:len(ins)]], -1)
        gscale = gx_r.abs().max().item()
        assert torch.all((gx - gx_r).abs() <= 2.0 ** -8 * gx_r.abs() + 1e-5 * gscale), (k, c['kind'], 'dX')
        for g, r, what in ((grads[-2], gw_r, 'dW'), (grads[-1], gb_r, 'db')):
            err = (g.double().cpu() - r).abs().max().item()
            assert err <= 2e-5 * r.abs().max().item(), (k, c['kind'], what, err)


def test_network_end_to_end_against_fp64_oracle(recorded_network):
    """The whole pass against the FP64 network with bf16-rounded activations.
    With random weights the bf16 network is sensitive to rounding: FP32
    instead of FP64 accumulation flips single bf16 roundings, and these grow
    through 21 layers.  An FP32-accumulating emulation on the CPU shows the
    same spread (output 0.6%, weight gradients 4-16% relative L2), so the
    bounds here are directional; the per-call check above is the tight one."""
    net, x, y, R, _ = recorded_network
    yr, P = ref_forward(net, x.cpu().double())
    (yr * R.double()).sum().backward()
    e = _rel(y.double().cpu(), yr.detach())
    print(f'output rel L2 {e:.2e}')
    assert e < 2e-2
    for name, (w, b) in P.items():
        gw = getattr(net, name + '_w').grad.double().cpu()
        cos = float((gw * w.grad).sum() / (gw.norm() * w.grad.norm()))
        print(f'{name:6s} weight grad rel L2 {_rel(gw, w.grad):.2e}  cos {cos:.5f}')
        assert _rel(gw, w.grad) < 0.3 and cos > 0.97, name


@pytest.mark.parametrize('storage,tol', [('fp64', 1e-12), ('fp32', 1e-6)])
def test_initialize_equilibrium_reproduces_fields(storage, tol):
    from lbflow_b200 import Engine
    from lbflow_b200.geometry import porous_medium
    fluid = porous_medium((16, 16, 24), sigma=2.0, porosity=0.35, seed=5)
    geom = np.where(fluid, 75, 255).astype(np.uint8)
    rng = np.random.default_rng(2)
    f = np.zeros(fluid.shape + (4,), np.float32)
    f[..., :3] = (rng.standard_normal(fluid.shape + (3,)) * 1e-3).astype(np.float32)
    f[..., 3] = (1.0 + rng.standard_normal(fluid.shape) * 1e-3).astype(np.float32)
    dev = torch.from_numpy(f).cuda()
    torch.cuda.synchronize()
    with Engine(geom, LABELS, collision='MRT', tau=(1.0,), storage=storage) as e:
        e.initialize_equilibrium(dev)
        e.check()
        rho, _, u = e.macros()
    fl = fluid
    assert np.all(np.abs(rho[fl] - f[..., 3][fl]) <= tol * 1e-1 + 1e-15)
    for d in range(3):
        assert np.all(np.abs(u[d][fl] - f[..., d][fl]) <= tol * 1e-3 + 1e-15), d
    assert np.all(rho[~fl] == 0)


def test_warm_start_from_converged_field_converges_at_once():
    from lbflow_b200 import Engine
    from lbflow_b200.geometry import porous_medium
    from lbflow_b200.permeability import converge
    fluid = porous_medium((24, 24, 32), sigma=2.5, porosity=0.3, seed=8)
    geom = np.where(fluid, 75, 255).astype(np.uint8)
    with Engine(geom, LABELS, collision='MRT', tau=(0.8,)) as e:
        cold = converge(e, 0.8, 1e-5, report=500, tol=1e-8)
        rho, _, u = e.macros()
    assert cold['converged']
    fields = np.concatenate([np.moveaxis(u, 0, -1), rho[..., None]], -1).astype(np.float32)
    dev = torch.from_numpy(fields).cuda().contiguous()
    torch.cuda.synchronize()
    with Engine(geom, LABELS, collision='MRT', tau=(0.8,)) as e:
        warm = converge(e, 0.8, 1e-5, report=500, tol=1e-8,
                        warm=lambda: e.initialize_equilibrium(dev))
    print(f"cold {cold['steps']} steps, warm {warm['steps']} steps")
    assert warm['converged'] and not warm['fallback']
    assert abs(warm['K'] - cold['K']) <= 1e-6 * abs(cold['K'])
    # At the first report the warm start is already at the steady K; the
    # start from rest is still far from it.  (Reaching tol = 1e-8 takes a
    # while either way: the equilibrium start lacks the non-equilibrium
    # populations and its small acoustic transient must decay.)
    Kc, Kw = cold['history'][0][3], warm['history'][0][3]
    assert abs(Kw - cold['K']) <= 1e-4 * abs(cold['K']) < abs(Kc - cold['K'])


@pytest.mark.skipif(not WEIGHTS.exists(), reason='trained warm-start weights not present')
def test_trained_operator_starts_closer_to_the_steady_state():
    """The trained operator on a medium it was not trained on: the run started
    from its prediction is much closer to the steady permeability at the
    first report than the run from rest (which overshoots by tens of percent
    during the viscous transient), and ends at the same K."""
    from lbflow_b200 import Engine
    from lbflow_b200 import warmstart as ws
    from lbflow_b200.geometry import porous_medium
    from lbflow_b200.permeability import converge
    net, _ = ws.load(WEIGHTS)
    fluid = porous_medium((64, 64, 64), sigma=3.0, porosity=0.25, seed=987654)   # not a training seed
    geom = np.where(fluid, 75, 255).astype(np.uint8)
    fl = torch.from_numpy(fluid).cuda()
    runs = {}
    for mode in ('cold', 'warm'):
        with Engine(geom, LABELS, collision='MRT', tau=(1.0,)) as e:
            warm = (lambda: ws.warm_start(e, net, fl, 1.0, 1e-5, mode='none')) if mode == 'warm' else None
            runs[mode] = converge(e, 1.0, 1e-5, report=250, tol=1e-6, max_steps=40000, warm=warm)
    K = runs['cold']['K']
    ec = abs(runs['cold']['history'][0][3] - K) / K
    ew = abs(runs['warm']['history'][0][3] - K) / K
    print(f'K error at the first report: from rest {ec:.3e}, from the operator {ew:.3e}')
    assert ew < 0.5 * ec
    assert abs(runs['warm']['K'] - K) <= 1e-4 * abs(K) and not runs['warm']['fallback']


MOB_WEIGHTS = WEIGHTS.parent / 'mobility.pt'


@pytest.mark.skipif(not MOB_WEIGHTS.exists(), reason='trained block-mobility weights not present')
def test_learned_mobility_start_reaches_the_band_sooner_than_rest():
    """The learned start (block mobilities from the trained network, the
    block Darcy pressure at t = 0) on a medium of the cube recipe that no
    training medium used: fewer steps to K within 1e-3 of the converged value
    than LBFlow's start from rest, the same converged K, no fallback.  The
    run with the in-run correction (DarcyAccelerator, no network) is timed
    beside them and printed: it reaches the band sooner than either start."""
    from lbflow_b200 import Engine
    from lbflow_b200 import warmstart as ws
    from lbflow_b200.geometry import porous_medium
    from lbflow_b200.permeability import converge, time_to_band
    net, _ = ws.load_mobility(MOB_WEIGHTS)
    fluid = porous_medium((128, 128, 128), sigma=3.0, porosity=0.22, seed=424242)
    geom = np.where(fluid, 75, 255).astype(np.uint8)
    fl = torch.from_numpy(fluid).cuda()
    runs = {}
    for mode in ('cold', 'learned', 'correction'):
        with Engine(geom, LABELS, collision='MRT', tau=(1.0,)) as e:
            warm = (lambda: ws.mobility_start(e, net, fl, 1.0, 1e-5)) if mode == 'learned' else None
            acc = ws.DarcyAccelerator(e, fl, 1e-5, block=2, at=(500,)) if mode == 'correction' else None
            runs[mode] = converge(e, 1.0, 1e-5, report=250, tol=1e-6, max_steps=200000, warm=warm,
                                  accelerate=acc)
    K = runs['cold']['K']
    band = {m: time_to_band(r['history'], K) for m, r in runs.items()}
    print('steps to the 1e-3 band: ' + ', '.join(f'{m} {b[0] if b else None}' for m, b in band.items()))
    assert runs['learned']['converged'] and not runs['learned']['fallback']
    assert abs(runs['learned']['K'] - K) <= 1e-5 * abs(K)
    assert band['learned'] is not None and band['learned'][0] < band['cold'][0]


def test_block_sums_match_dense_macros():
    from lbflow_b200 import Engine
    from lbflow_b200.geometry import porous_medium
    fluid = porous_medium((16, 24, 32), sigma=2.0, porosity=0.3, seed=4)
    geom = np.where(fluid, 75, 255).astype(np.uint8)
    with Engine(geom, LABELS, collision='MRT', tau=(0.9,)) as e:
        e.initialize()
        e.step(200, macros=True)
        rho, _, u = e.macros()
        s = e.block_sums(8)
    assert s.shape == (2, 3, 4, 5)
    blk = lambda a: a.reshape(2, 8, 3, 8, 4, 8).sum(axis=(1, 3, 5))
    assert np.array_equal(s[..., 4], blk(fluid.astype(float)))
    assert np.allclose(s[..., 0], blk(rho), rtol=1e-13, atol=0)
    for c in range(3):
        assert np.allclose(s[..., 1 + c], blk(u[c]), rtol=1e-11, atol=1e-20)


@pytest.mark.parametrize('storage,tol', [('fp64', 1e-15), ('fp32', 1e-9), ('bfp16', 1e-7)])
def test_add_density_shifts_populations(storage, tol):
    from lbflow_b200 import Engine
    from lbflow_b200.geometry import porous_medium
    fluid = porous_medium((16, 16, 24), sigma=2.0, porosity=0.35, seed=6)
    geom = np.where(fluid, 75, 255).astype(np.uint8)
    rng = np.random.default_rng(3)
    drho = (rng.standard_normal(fluid.shape) * 1e-4).astype(np.float32)
    w = np.array([12] + [2] * 6 + [1] * 12) / 36.0
    with Engine(geom, LABELS, collision='MRT', tau=(1.0,), storage=storage) as e:
        e.initialize()
        e.step(30)
        f0 = e.populations()
        d = torch.from_numpy(drho).cuda().contiguous()
        torch.cuda.synchronize()
        e.add_density(d)
        f1 = e.populations()
        e.check()
    expect = f0 + w[None, :, None, None, None] * np.where(fluid, drho, 0.0)[None, None]
    assert np.max(np.abs(f1[:, :, fluid] - expect[:, :, fluid])) <= tol + 1e-6 * tol
    assert np.all(f1[:, :, ~fluid] == 0)


@pytest.mark.parametrize('shape,b', [((32, 32, 32), 2), ((24, 48, 16), 4)])
def test_darcy_solver_cuda_matches_torch(shape, b):
    """The library's multigrid-CG block pressure solve (lbf_darcy_pressure)
    against the torch reference solve of the same discrete problem."""
    from lbflow_b200 import warmstart as ws
    gen = torch.Generator().manual_seed(5)
    # Porous-like mobility: log-normal, with many near-solid blocks.
    mob = torch.exp(2.0 * torch.randn(shape, generator=gen, dtype=torch.float64))
    mob[torch.rand(shape, generator=gen) < 0.3] = 1e-4
    ref = ws.darcy_pressure(mob, 1e-5, b, rtol=1e-10)
    phi, it = ws.darcy_pressure_device(mob.cuda(), 1e-5, b, rtol=1e-9, max_iter=500)
    print(f'{shape} b={b}: {it} iterations')
    assert it < 500
    # The CUDA solve keeps face mobilities in FP32: agreement to ~1e-6.
    assert float((phi.cpu() - ref).norm() / ref.norm()) < 1e-5
    assert abs(float(phi.mean())) < 1e-12 * float(ref.abs().max())


def test_accelerator_shortens_the_run_and_keeps_the_answer():
    """One block Darcy correction after 500 steps: the run reaches K within
    1e-3 of the converged value sooner than from rest, and converges to the
    same K."""
    from lbflow_b200 import Engine
    from lbflow_b200 import warmstart as ws
    from lbflow_b200.geometry import porous_medium
    from lbflow_b200.permeability import converge, time_to_band
    fluid = porous_medium((64, 64, 64), sigma=3.0, porosity=0.22, seed=11)
    geom = np.where(fluid, 75, 255).astype(np.uint8)
    fl = torch.from_numpy(fluid).cuda()
    runs = {}
    for mode in ('cold', 'acc'):
        with Engine(geom, LABELS, collision='MRT', tau=(1.0,)) as e:
            acc = ws.DarcyAccelerator(e, fl, 1e-5, block=2, at=(500,)) if mode == 'acc' else None
            runs[mode] = converge(e, 1.0, 1e-5, report=250, tol=1e-6, accelerate=acc)
            if acc is not None:
                assert acc.applied == [500] and acc.iterations[0] < 200
    K = runs['cold']['K']
    assert runs['acc']['converged'] and abs(runs['acc']['K'] - K) <= 1e-5 * abs(K)
    tc = time_to_band(runs['cold']['history'], K)
    ta = time_to_band(runs['acc']['history'], K)
    print(f'steps to the 1e-3 band: from rest {tc[0]}, with the correction {ta[0]}')
    assert ta[0] < tc[0]
