"""Tensor-core 3D convolutions of the learned warm start as torch autograd
Functions (ctypes binding of include/lbflow_operator.h).

Activations are channels-last bf16 tensors (batch, z, y, x, channel) whose
channel counts are multiples of 8; weights are fp32 parameters in torch's
layout, rounded to bf16 and packed into the kernels' K-major matrices at
every call.  Forward convolutions, data gradients and weight gradients all
run in the library's tcgen05 kernels; torch supplies device memory, the
stream, the leaky-ReLU mask of the backward pass and bias sums.  There is no
fallback: without the CUDA library every call raises.

Three operators:
  conv3  3x3x3 convolution with periodic wrap (one or two concatenated inputs)
  down2  2x2x2 convolution with stride 2 (halves the grid)
  up2    2x2x2 transposed convolution with stride 2 (doubles the grid)
"""
import ctypes

import torch

from . import LbfError, library

U32, I32, P = ctypes.c_uint32, ctypes.c_int32, ctypes.c_void_p
OUT_BF16, OUT_F32, OUT_SCATTER2 = 0, 1, 2
ERR_MMA_TIMEOUT = 1 << 8


class _Gather(ctypes.Structure):
    _fields_ = [('src0', P), ('src1', P), ('c0', U32), ('c1', U32), ('batch', U32),
                ('in_d', U32), ('in_h', U32), ('in_w', U32), ('out_d', U32), ('out_h', U32), ('out_w', U32),
                ('ksize', U32), ('stride', U32), ('pad', I32)]


class _Igemm(ctypes.Structure):
    _fields_ = [('a', _Gather), ('weight', P), ('n', U32), ('n_pad', U32), ('k_pad', U32), ('bias', P),
                ('out', P), ('out_mode', U32), ('out_ld', U32), ('act', U32), ('slope', ctypes.c_float),
                ('err', P)]


class _Wgrad(ctypes.Structure):
    _fields_ = [('a', _Gather), ('b', P), ('cb', U32), ('out', P), ('workspace', P),
                ('workspace_bytes', ctypes.c_size_t), ('err', P)]


_SIGS = False
_ERR = {}


def _lib():
    global _SIGS
    lib = library()
    if not _SIGS:
        lib.lbf_igemm_run.restype = ctypes.c_int
        lib.lbf_igemm_run.argtypes = [ctypes.POINTER(_Igemm), P]
        lib.lbf_wgrad_run.restype = ctypes.c_int
        lib.lbf_wgrad_run.argtypes = [ctypes.POINTER(_Wgrad), P]
        lib.lbf_wgrad_workspace.restype = ctypes.c_size_t
        lib.lbf_wgrad_workspace.argtypes = [ctypes.POINTER(_Wgrad)]
        lib.lbf_operator_info.restype = None
        lib.lbf_operator_info.argtypes = [ctypes.POINTER(U32)]
        _SIGS = True
    return lib


def error_word(device):
    """The device error word the kernels of this device report into."""
    key = torch.device(device).index or 0
    if key not in _ERR:
        _ERR[key] = torch.zeros(1, dtype=torch.int32, device=device)
    return _ERR[key]


def check(device=None):
    """Raise if a kernel on `device` recorded a tensor-core wait timeout."""
    dev = device if device is not None else torch.device('cuda', torch.cuda.current_device())
    w = int(error_word(dev).item())
    if w:
        raise LbfError(-4, f'tensor-core kernel error word {w:#x} (MMA wait timed out)')


def _stream(t):
    return ctypes.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)


def _ck(rc):
    if rc != 0:
        raise LbfError(rc, library().lbf_last_error(None).decode())


def _pad16(n):
    for p in (16, 32, 64):
        if n <= p:
            return p
    return (n + 127) // 128 * 128


def _pad64(k):
    return (k + 63) // 64 * 64


def _gather(src0, src1, ksize, stride, pad, out_dims):
    assert src0.dtype == torch.bfloat16 and src0.is_contiguous() and src0.dim() == 5
    B, D, H, W, c0 = src0.shape
    c1 = 0
    if src1 is not None:
        assert src1.dtype == torch.bfloat16 and src1.is_contiguous() and src1.shape[:4] == src0.shape[:4]
        c1 = src1.shape[4]
    return _Gather(src0.data_ptr(), src1.data_ptr() if src1 is not None else None, c0, c1, B, D, H, W,
                   *out_dims, ksize, stride, pad)


def pack_weight(mat):
    """(n, k) matrix -> zero-padded bf16 [n_pad][k_pad] (the kernels' K-major B)."""
    n, k = mat.shape
    out = torch.zeros(_pad16(n), _pad64(k), dtype=torch.bfloat16, device=mat.device)
    out[:n, :k] = mat
    return out


def igemm(src0, src1, ksize, stride, pad, out_dims, wmat, bias=None, mode=OUT_BF16, out=None, out_ld=None,
          act=False, slope=0.0):
    """out[row][n] = act(sum_k A[row][k] wmat[n][k] + bias) on the tensor cores.

    wmat: (n, k) with k = ksize^3 * channels (tap-major), any float dtype."""
    lib = _lib()
    n, k = wmat.shape
    wp = pack_weight(wmat)
    g = _gather(src0, src1, ksize, stride, pad, out_dims)
    assert k == ksize ** 3 * (g.c0 + g.c1)
    B = src0.shape[0]
    if out is None:
        if mode == OUT_SCATTER2:
            ld = n // 8
            out = torch.empty(B, 2 * out_dims[0], 2 * out_dims[1], 2 * out_dims[2], ld, dtype=torch.bfloat16,
                              device=src0.device)
        else:
            ld = n
            out = torch.empty(B, *out_dims, n, dtype=torch.float32 if mode == OUT_F32 else torch.bfloat16,
                              device=src0.device)
        out_ld = ld
    b = bias.float().contiguous() if bias is not None else None
    d = _Igemm(g, wp.data_ptr(), n, wp.shape[0], wp.shape[1], b.data_ptr() if b is not None else None,
               out.data_ptr(), mode, out_ld, 1 if act else 0, float(slope), error_word(src0.device).data_ptr())
    _ck(lib.lbf_igemm_run(ctypes.byref(d), _stream(src0)))
    return out


def wgrad(src0, src1, ksize, stride, pad, out_dims, b):
    """out[i][j] = sum_row A[row][i] b[row][j] (fp32), i = tap * channels + channel."""
    lib = _lib()
    g = _gather(src0, src1, ksize, stride, pad, out_dims)
    assert b.dtype == torch.bfloat16 and b.is_contiguous()
    cb = b.shape[-1]
    assert b.numel() == g.batch * g.out_d * g.out_h * g.out_w * cb
    mtot = ksize ** 3 * (g.c0 + g.c1)
    out = torch.empty(mtot, cb, dtype=torch.float32, device=b.device)
    d = _Wgrad(g, b.data_ptr(), cb, out.data_ptr(), None, 0, error_word(b.device).data_ptr())
    nbytes = lib.lbf_wgrad_workspace(ctypes.byref(d))
    if nbytes == 0:
        _ck(-1)
    ws = torch.empty(nbytes // 4 + 1, dtype=torch.float32, device=b.device)
    d.workspace = ws.data_ptr()
    d.workspace_bytes = nbytes
    _ck(lib.lbf_wgrad_run(ctypes.byref(d), _stream(b)))
    return out


def _lrelu_grad(gy, y, slope):
    return (gy.float() * torch.where(y > 0, 1.0, slope)).to(torch.bfloat16).contiguous()


class Conv3(torch.autograd.Function):
    """3x3x3 periodic convolution of cat(x0, x1) (x1 optional) + bias, then
    leaky ReLU when slope is not None.  weight: (Cout, C0 + C1, 3, 3, 3)."""

    @staticmethod
    def forward(ctx, x0, x1, weight, bias, slope):
        dims = tuple(x0.shape[1:4])
        cout = weight.shape[0]
        wmat = weight.permute(0, 2, 3, 4, 1).reshape(cout, -1)
        y = igemm(x0, x1, 3, 1, 1, dims, wmat, bias, act=slope is not None, slope=slope or 0.0)
        ctx.save_for_backward(x0, x1, weight, y)
        ctx.slope = slope
        return y

    @staticmethod
    def backward(ctx, gy):
        x0, x1, weight, y = ctx.saved_tensors
        gy = _lrelu_grad(gy, y, ctx.slope) if ctx.slope is not None else gy.to(torch.bfloat16).contiguous()
        dims = tuple(x0.shape[1:4])
        cout, cin = weight.shape[:2]
        gx0 = gx1 = gw = gb = None
        if ctx.needs_input_grad[0] or ctx.needs_input_grad[1]:
            # dX[i] = sum_d dY[i + d - 1] W[:, :, 2 - d]: a periodic convolution of dY
            # with the flipped, transposed kernel.
            wt = weight.flip(2, 3, 4).transpose(0, 1)              # (Cin, Cout, 3, 3, 3)
            gx = igemm(gy, None, 3, 1, 1, dims, wt.permute(0, 2, 3, 4, 1).reshape(cin, -1))
            c0 = x0.shape[-1]
            gx0 = gx[..., :c0].contiguous() if x1 is not None else gx
            gx1 = gx[..., c0:].contiguous() if x1 is not None else None
        if ctx.needs_input_grad[2]:
            m = wgrad(x0, x1, 3, 1, 1, dims, gy)                   # (27 * Cin, Cout)
            gw = m.reshape(3, 3, 3, cin, cout).permute(4, 3, 0, 1, 2).contiguous()
        if ctx.needs_input_grad[3]:
            gb = gy.float().sum(dim=(0, 1, 2, 3))
        return gx0, gx1, gw, gb, None


class Down2(torch.autograd.Function):
    """2x2x2 stride-2 convolution + bias (+ leaky ReLU).  weight: (Cout, Cin, 2, 2, 2)."""

    @staticmethod
    def forward(ctx, x, weight, bias, slope):
        dims = tuple(d // 2 for d in x.shape[1:4])
        cout = weight.shape[0]
        y = igemm(x, None, 2, 2, 0, dims, weight.permute(0, 2, 3, 4, 1).reshape(cout, -1), bias,
                  act=slope is not None, slope=slope or 0.0)
        ctx.save_for_backward(x, weight, y)
        ctx.slope = slope
        return y

    @staticmethod
    def backward(ctx, gy):
        x, weight, y = ctx.saved_tensors
        gy = _lrelu_grad(gy, y, ctx.slope) if ctx.slope is not None else gy.to(torch.bfloat16).contiguous()
        cdims = tuple(gy.shape[1:4])
        cout, cin = weight.shape[:2]
        gx = gw = gb = None
        if ctx.needs_input_grad[0]:
            # dX[2c + d][ci] = sum_co dY[c][co] W[co, ci, d]: scatter into the 8 fine voxels.
            wm = weight.permute(2, 3, 4, 1, 0).reshape(8 * cin, cout)
            gx = igemm(gy, None, 1, 1, 0, cdims, wm, mode=OUT_SCATTER2)
        if ctx.needs_input_grad[1]:
            m = wgrad(x, None, 2, 2, 0, cdims, gy)                 # (8 * Cin, Cout)
            gw = m.reshape(2, 2, 2, cin, cout).permute(4, 3, 0, 1, 2).contiguous()
        if ctx.needs_input_grad[2]:
            gb = gy.float().sum(dim=(0, 1, 2, 3))
        return gx, gw, gb, None


class Up2(torch.autograd.Function):
    """2x2x2 stride-2 transposed convolution + bias (+ leaky ReLU).
    weight: (Cin, Cout, 2, 2, 2) as torch's conv_transpose3d."""

    @staticmethod
    def forward(ctx, x, weight, bias, slope):
        cdims = tuple(x.shape[1:4])
        cin, cout = weight.shape[:2]
        wm = weight.permute(2, 3, 4, 1, 0).reshape(8 * cout, cin)   # n = tap * Cout + co
        y = igemm(x, None, 1, 1, 0, cdims, wm, bias, mode=OUT_SCATTER2, act=slope is not None,
                  slope=slope or 0.0)
        ctx.save_for_backward(x, weight, y)
        ctx.slope = slope
        return y

    @staticmethod
    def backward(ctx, gy):
        x, weight, y = ctx.saved_tensors
        gy = _lrelu_grad(gy, y, ctx.slope) if ctx.slope is not None else gy.to(torch.bfloat16).contiguous()
        cdims = tuple(x.shape[1:4])
        cin, cout = weight.shape[:2]
        gx = gw = gb = None
        if ctx.needs_input_grad[0]:
            # dX[c][ci] = sum_{d, co} dY[2c + d][co] W[ci, co, d]: a stride-2 gather of dY.
            wm = weight.permute(0, 2, 3, 4, 1).reshape(cin, 8 * cout)
            gx = igemm(gy, None, 2, 2, 0, cdims, wm)
        if ctx.needs_input_grad[1]:
            m = wgrad(gy, None, 2, 2, 0, cdims, x)                 # (8 * Cout, Cin)
            gw = m.reshape(2, 2, 2, cout, cin).permute(4, 3, 0, 1, 2).contiguous()
        if ctx.needs_input_grad[2]:
            gb = gy.float().sum(dim=(0, 1, 2, 3))
        return gx, gw, gb, None


def conv3(x0, weight, bias, slope=None, x1=None):
    return Conv3.apply(x0, x1, weight, bias, slope)


def down2(x, weight, bias, slope=None):
    return Down2.apply(x, weight, bias, slope)


def up2(x, weight, bias, slope=None):
    return Up2.apply(x, weight, bias, slope)


def conv3_f32(x, weight, bias):
    """3x3x3 periodic convolution with an fp32 output (the operator's head)."""
    dims = tuple(x.shape[1:4])
    cout = weight.shape[0]
    return igemm(x, None, 3, 1, 1, dims, weight.permute(0, 2, 3, 4, 1).reshape(cout, -1), bias, mode=OUT_F32)


def info():
    lib = _lib()
    out = (U32 * 4)()
    lib.lbf_operator_info(out)
    return dict(tile_rows=out[0], k_per_stage=out[1], stages=out[2], threads=out[3])
