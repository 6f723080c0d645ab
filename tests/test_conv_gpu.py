"""Tensor-core convolutions of the warm-start operator against torch's CPU
FP64 convolutions (the oracle for this dense part; LBFlow has no network).

Inputs and weights are rounded to bf16 first, so the oracle sees exactly the
operands the tensor cores multiply.  Tolerances: bf16 outputs carry one bf16
rounding (relative 2^-9) on top of FP32 accumulation; FP32 weight gradients
only the accumulation (relative 1e-5 of the largest entry).
"""
import pytest
import torch
import torch.nn.functional as F

pytestmark = pytest.mark.gpu

DIMS = (2, 6, 10, 12)     # batch, z, y, x: 1440 GEMM rows, not a multiple of the 128-row tile


def _rand(*shape, scale=1.0, seed=0):
    g = torch.Generator().manual_seed(seed)
    return (torch.randn(*shape, generator=g) * scale).to(torch.bfloat16)


def _cf(x):   # channels-last -> channels-first
    return x.permute(0, 4, 1, 2, 3)


def _cl(x):
    return x.permute(0, 2, 3, 4, 1)


def ref_conv3(x, w, b, slope):
    y = F.conv3d(F.pad(_cf(x), (1, 1, 1, 1, 1, 1), mode='circular'), w, b)
    return _cl(F.leaky_relu(y, slope) if slope is not None else y)


def ref_down2(x, w, b, slope):
    y = F.conv3d(_cf(x), w, b, stride=2)
    return _cl(F.leaky_relu(y, slope) if slope is not None else y)


def ref_up2(x, w, b, slope):
    y = F.conv_transpose3d(_cf(x), w, b, stride=2)
    return _cl(F.leaky_relu(y, slope) if slope is not None else y)


def _close_bf16(y, ref):
    y = y.double().cpu()
    scale = ref.abs().max().item()
    err = (y - ref).abs()
    bound = 2.0 ** -8 * ref.abs() + 1e-5 * scale
    assert torch.all(err <= bound), f'max err {err.max().item():.3e} (scale {scale:.3e})'


def _close_rel(a, ref, rel):
    a = a.double().cpu()
    scale = ref.abs().max().item()
    err = (a - ref).abs().max().item()
    assert err <= rel * scale, f'max err {err:.3e} vs {rel:.1e} * {scale:.3e}'


def _setup(cin, cout, k, transposed=False, seed=1):
    wshape = (cin, cout, k, k, k) if transposed else (cout, cin, k, k, k)
    fan = cin * k ** 3
    w = _rand(*wshape, scale=fan ** -0.5, seed=seed).float()
    b = _rand(cout, scale=0.1, seed=seed + 1).float()
    return w, b


@pytest.mark.parametrize('cin,cout', [(8, 16), (16, 16), (32, 64), (64, 128), (128, 64), (16, 8)])
@pytest.mark.parametrize('slope', [None, 0.1])
def test_conv3_forward(cin, cout, slope):
    from lbflow_b200 import conv
    x = _rand(*DIMS, cin, seed=3)
    w, b = _setup(cin, cout, 3)
    y = conv.conv3(x.cuda(), w.cuda(), b.cuda(), slope)
    conv.check()
    _close_bf16(y, ref_conv3(x.double(), w.bfloat16().double(), b.double(), slope))


def test_conv3_two_sources():
    from lbflow_b200 import conv
    x0, x1 = _rand(*DIMS, 32, seed=4), _rand(*DIMS, 16, seed=5)
    w, b = _setup(48, 32, 3)
    y = conv.conv3(x0.cuda(), w.cuda(), b.cuda(), 0.1, x1=x1.cuda())
    conv.check()
    ref = ref_conv3(torch.cat([x0, x1], -1).double(), w.bfloat16().double(), b.double(), 0.1)
    _close_bf16(y, ref)


@pytest.mark.parametrize('cin,cout', [(16, 32), (64, 128)])
def test_down2_up2_forward(cin, cout):
    from lbflow_b200 import conv
    x = _rand(2, 8, 12, 16, cin, seed=6)
    w, b = _setup(cin, cout, 2)
    y = conv.down2(x.cuda(), w.cuda(), b.cuda(), 0.1)
    conv.check()
    _close_bf16(y, ref_down2(x.double(), w.bfloat16().double(), b.double(), 0.1))
    xc = _rand(2, 4, 6, 8, cout, seed=7)
    wu, bu = _setup(cout, cin, 2, transposed=True)
    yu = conv.up2(xc.cuda(), wu.cuda(), bu.cuda(), None)
    conv.check()
    _close_bf16(yu, ref_up2(xc.double(), wu.bfloat16().double(), bu.double(), None))


def _grads(op, ref, x, w, b, slope, seed=11, **kw):
    """Gradients of sum(y * R) through our kernels and through FP64 autograd."""
    xg = x.cuda().requires_grad_(True)
    wg = w.cuda().requires_grad_(True)
    bg = b.cuda().requires_grad_(True)
    y = op(xg, wg, bg, slope, **kw)
    R = _rand(*y.shape, seed=seed)
    (y.float() * R.cuda().float()).sum().backward()
    from lbflow_b200 import conv
    conv.check()
    xr = x.double().requires_grad_(True)
    wr = w.bfloat16().double().requires_grad_(True)
    br = b.double().requires_grad_(True)
    yr = ref(xr, wr, br, slope)
    (yr * R.double()).sum().backward()
    return (xg.grad, wg.grad, bg.grad), (xr.grad, wr.grad, br.grad)


@pytest.mark.parametrize('cin,cout', [(16, 16), (32, 64), (64, 128), (128, 32)])
def test_conv3_gradients_linear(cin, cout):
    """Without the activation the data gradient carries one bf16 rounding and
    the weight gradient only FP32 accumulation."""
    from lbflow_b200 import conv
    x = _rand(*DIMS, cin, seed=8)
    w, b = _setup(cin, cout, 3)
    (gx, gw, gb), (rx, rw, rb) = _grads(conv.conv3, ref_conv3, x, w, b, None)
    _close_bf16(gx, rx)
    _close_rel(gw, rw, 1e-5)
    _close_rel(gb, rb, 1e-5)


def test_conv3_gradients_leaky_relu_large_grid():
    """Leaky ReLU mask in the backward pass; a grid of 65,536 rows splits the
    weight-gradient reduction over many CTAs."""
    from lbflow_b200 import conv
    x = _rand(2, 16, 32, 64, 32, seed=9)
    w, b = _setup(32, 64, 3)
    (gx, gw, gb), (rx, rw, rb) = _grads(conv.conv3, ref_conv3, x, w, b, 0.1)
    # dY * mask is rounded to bf16 before the convolutions: relative 2^-9 per entry.
    _close_rel(gx, rx, 8e-3)
    _close_rel(gw, rw, 4e-3)
    _close_rel(gb, rb, 4e-3)


@pytest.mark.parametrize('cin,cout', [(16, 32), (64, 128)])
def test_down2_gradients(cin, cout):
    from lbflow_b200 import conv
    x = _rand(2, 8, 12, 16, cin, seed=12)
    w, b = _setup(cin, cout, 2)
    (gx, gw, gb), (rx, rw, rb) = _grads(conv.down2, ref_down2, x, w, b, None)
    _close_bf16(gx, rx)
    _close_rel(gw, rw, 1e-5)
    _close_rel(gb, rb, 1e-5)


@pytest.mark.parametrize('cin,cout', [(32, 16), (128, 64)])
def test_up2_gradients(cin, cout):
    from lbflow_b200 import conv
    x = _rand(2, 4, 6, 8, cin, seed=13)
    w, b = _setup(cin, cout, 2, transposed=True)
    (gx, gw, gb), (rx, rw, rb) = _grads(conv.up2, ref_up2, x, w, b, None)
    _close_bf16(gx, rx)
    _close_rel(gw, rw, 1e-5)
    _close_rel(gb, rb, 1e-5)


def test_conv3_two_source_gradients():
    from lbflow_b200 import conv
    x0, x1 = _rand(*DIMS, 16, seed=14), _rand(*DIMS, 16, seed=15)
    w, b = _setup(32, 16, 3)
    x0g, x1g = x0.cuda().requires_grad_(True), x1.cuda().requires_grad_(True)
    wg, bg = w.cuda().requires_grad_(True), b.cuda().requires_grad_(True)
    y = conv.conv3(x0g, wg, bg, None, x1=x1g)
    R = _rand(*y.shape, seed=16)
    (y.float() * R.cuda().float()).sum().backward()
    conv.check()
    xr = torch.cat([x0, x1], -1).double().requires_grad_(True)
    wr = w.bfloat16().double().requires_grad_(True)
    yr = ref_conv3(xr, wr, b.double(), None)
    (yr * R.double()).sum().backward()
    _close_bf16(torch.cat([x0g.grad, x1g.grad], -1), xr.grad)
    _close_rel(wg.grad, wr.grad, 1e-5)
