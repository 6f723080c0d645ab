"""Learned warm start: a 3D convolutional neural operator that predicts the
steady flow of a periodic porous medium under a body force, used as the
initial state of the lattice Boltzmann run.

LBFlow always starts from rest (SCSP::initialize, solver/src/lbm/scsp.cpp:
116-134) and steps until its velocity residual falls below stopError
(Simulator::updateConvergence, simulator.cpp:248-325).  Here the network maps
the voxel geometry to the steady velocity and density; the engine starts from
the equilibrium populations of that prediction (lbf_initialize_equilibrium)
and the unchanged step loop and stopping rule take it from there, so the
converged answer is the solver's, not the network's.  If the residual stalls
or blows up the run restarts from rest (the cold-start fallback).

Scaling.  In the creeping-flow regime of these runs (Re << 1) the steady
velocity is linear in the force: u = (g / nu) k(x) with nu = (tau - 1/2)/3,
and the density deviation is rho - rho0 = 3 g pi(x).  The network predicts
the geometry-only fields k (whose mean over all voxels is the permeability K
of scripts/rock_workflow.py:60-66) and pi, normalised by constants stored
with the weights, so one network serves every tau and force magnitude.  The
force must lie along +x; other directions are handled by the caller
permuting axes.

Network (about 1.8M parameters, bf16 activations, fp32 master weights):
a 4-level U-Net on channels-last tensors whose every convolution, data
gradient and weight gradient runs in the tcgen05 kernels of conv.py.
Channels 16-32-64-128; per level two periodic 3x3x3 convolutions with leaky
ReLU, 2x2x2 stride-2 convolutions down, 2x2x2 stride-2 transposed
convolutions up, skip connections concatenated inside the decoder's first
convolution, and a linear 3x3x3 head.  Grid edges must be multiples of 8.
"""
import math
import time

import numpy as np
import torch

from . import conv

CH = (16, 32, 64, 128)
IN_CH = 8          # input features (5 used, zero padded to a multiple of 8)
OUT_CH = 8         # head channels: k_x, k_y, k_z, pi, 4 unused
SLOPE = 0.1
DIST_MAX = 12      # chessboard distances are capped here


def _spec():
    c1, c2, c3, c4 = CH
    s = [('enc1a', 'c3', IN_CH, c1), ('enc1b', 'c3', c1, c1), ('down1', 'd2', c1, c2),
         ('enc2a', 'c3', c2, c2), ('enc2b', 'c3', c2, c2), ('down2', 'd2', c2, c3),
         ('enc3a', 'c3', c3, c3), ('enc3b', 'c3', c3, c3), ('down3', 'd2', c3, c4),
         ('mida', 'c3', c4, c4), ('midb', 'c3', c4, c4),
         ('up3', 'u2', c4, c3), ('dec3a', 'c3', 2 * c3, c3), ('dec3b', 'c3', c3, c3),
         ('up2', 'u2', c3, c2), ('dec2a', 'c3', 2 * c2, c2), ('dec2b', 'c3', c2, c2),
         ('up1', 'u2', c2, c1), ('dec1a', 'c3', 2 * c1, c1), ('dec1b', 'c3', c1, c1),
         ('head', 'c3', c1, OUT_CH)]
    return s


class WarmStartNet(torch.nn.Module):
    def __init__(self, seed=0):
        super().__init__()
        g = torch.Generator().manual_seed(seed)
        self.kinds = {}
        for name, kind, cin, cout in _spec():
            if kind == 'u2':
                w = torch.randn(cin, cout, 2, 2, 2, generator=g) * math.sqrt(2.0 / cin)
            else:
                k = 3 if kind == 'c3' else 2
                w = torch.randn(cout, cin, k, k, k, generator=g) * math.sqrt(2.0 / (cin * k ** 3))
            if name == 'head':
                w *= 0.1
            self.register_parameter(name + '_w', torch.nn.Parameter(w))
            self.register_parameter(name + '_b', torch.nn.Parameter(torch.zeros(cout)))
            self.kinds[name] = kind
        # Normalisation of the targets (set from the training data).
        self.register_buffer('scale', torch.ones(4))

    def _p(self, name):
        return getattr(self, name + '_w'), getattr(self, name + '_b')

    def _c3(self, name, x, skip=None, act=True):
        w, b = self._p(name)
        return conv.conv3(x, w, b, SLOPE if act else None, x1=skip)

    def forward(self, x):
        """x: (B, D, H, W, 8) bf16 features -> (B, D, H, W, 8) bf16 outputs."""
        e1 = self._c3('enc1b', self._c3('enc1a', x))
        e2 = conv.down2(e1, *self._p('down1'), SLOPE)
        e2 = self._c3('enc2b', self._c3('enc2a', e2))
        e3 = conv.down2(e2, *self._p('down2'), SLOPE)
        e3 = self._c3('enc3b', self._c3('enc3a', e3))
        m = conv.down2(e3, *self._p('down3'), SLOPE)
        m = self._c3('midb', self._c3('mida', m))
        d3 = conv.up2(m, *self._p('up3'), SLOPE)
        d3 = self._c3('dec3b', self._c3('dec3a', d3, skip=e3))
        d2 = conv.up2(d3, *self._p('up2'), SLOPE)
        d2 = self._c3('dec2b', self._c3('dec2a', d2, skip=e2))
        d1 = conv.up2(d2, *self._p('up1'), SLOPE)
        d1 = self._c3('dec1b', self._c3('dec1a', d1, skip=e1))
        return self._c3('head', d1, act=False)

    def flops(self, voxels):
        """Forward FLOPs (2 x multiply-adds) of one sample of `voxels` voxels."""
        total = 0
        level = {'enc1': 1, 'dec1': 1, 'enc2': 8, 'dec2': 8, 'enc3': 64, 'dec3': 64, 'mid': 512,
                 'down1': 8, 'down2': 64, 'down3': 512, 'up3': 512, 'up2': 64, 'up1': 8, 'head': 1}
        for name, kind, cin, cout in _spec():
            key = next(k for k in level if name.startswith(k))
            rows = voxels / level[key]
            taps = {'c3': 27, 'd2': 8, 'u2': 8}[kind]
            total += 2 * rows * taps * cin * cout
        return total


def _periodic_pool(x, k, mode):
    p = k // 2
    xp = torch.nn.functional.pad(x, (p, p, p, p, p, p), mode='circular')
    if mode == 'max':
        return torch.nn.functional.max_pool3d(xp, k, stride=1)
    return torch.nn.functional.avg_pool3d(xp, k, stride=1)


def features(fluid):
    """Input features of (B, D, H, W) fluid masks (bool or 0/1, any device):
    mask, signed chessboard distance / 8 (positive in pores), its squared
    positive part / 64, porosity of the surrounding 9^3 box, global porosity.
    Returns (B, D, H, W, 8) bf16, channels-last, on the masks' device."""
    m = fluid.float().unsqueeze(1)                      # (B, 1, D, H, W)
    solid = 1.0 - m
    dist_f = torch.zeros_like(m)
    dist_s = torch.zeros_like(m)
    cur_s, cur_f = solid, m
    for _ in range(DIST_MAX):
        dist_f += 1.0 - cur_s                           # pores not yet reached by the dilated solid
        dist_s += 1.0 - cur_f
        cur_s = _periodic_pool(cur_s, 3, 'max')
        cur_f = _periodic_pool(cur_f, 3, 'max')
    sdf = (dist_f - dist_s) / 8.0
    por = _periodic_pool(m, 9, 'avg')
    glob = m.mean(dim=(2, 3, 4), keepdim=True).expand_as(m)
    z = torch.zeros_like(m)
    f = torch.cat([m, sdf, torch.clamp(sdf, min=0) ** 2, por, glob, z, z, z], dim=1)
    return f.permute(0, 2, 3, 4, 1).contiguous().to(torch.bfloat16)


def targets(rho, u, tau, g, rho0=1.0):
    """Geometry-only fields of a steady solution: k = u nu / g (3 components)
    and pi = (rho - rho0) / (3 g), stacked as (D, H, W, 4) float32."""
    nu = (tau - 0.5) / 3.0
    k = np.moveaxis(u, 0, -1) * (nu / g)
    pi = (rho - rho0) / (3.0 * g)
    pi = np.where(rho > 0, pi, 0.0)
    return np.concatenate([k, pi[..., None]], axis=-1).astype(np.float32)


def _block_mean(x, b):
    """Means over b^3 blocks of a (D, H, W, C) field -> (D/b, H/b, W/b, C)."""
    D, H, W, C = x.shape
    return x.reshape(D // b, b, H // b, b, W // b, b, C).mean(dim=(1, 3, 5))


def _shift(x, s, axis):
    return torch.roll(x, s, dims=axis)


_AXES = (2, 1, 0)            # x, y, z components live on grid axes W, H, D


def _face_mobility(mob, face='geometric'):
    """Mobility on the + faces of each block along x, y, z: the geometric mean
    of the two blocks (the effective-medium value for random media, between
    the series (harmonic) and parallel (arithmetic) bounds), or either bound."""
    out = []
    for ax in _AXES:
        nb = _shift(mob, -1, ax)
        if face == 'geometric':
            out.append(torch.sqrt(mob * nb))
        elif face == 'arithmetic':
            out.append(0.5 * (mob + nb))
        else:
            out.append(2.0 * mob * nb / (mob + nb))
    return out


def _apply(phi, mf, h):
    """Variable-coefficient periodic Laplacian sum_faces M_f (phi_nb - phi) / h^2."""
    out = torch.zeros_like(phi)
    for c, ax in enumerate(_AXES):
        f = mf[c] * (_shift(phi, -1, ax) - phi)                     # at face i + 1/2
        out += f - _shift(f, 1, ax)
    return out / (h * h)


def _diag(mf, h):
    d = torch.zeros_like(mf[0])
    for c, ax in enumerate(_AXES):
        d -= mf[c] + _shift(mf[c], 1, ax)
    return d / (h * h)


def _coarsen_faces(mf):
    """Face mobilities of the 2x-coarser grid: the mean of the four fine faces
    on each coarse interface (flux-consistent for a linear pressure)."""
    out = []
    for c, ax in enumerate(_AXES):
        m = mf[c]
        # The fine faces on coarse interfaces have an odd index along ax.
        m = torch.index_select(m, ax, torch.arange(1, m.shape[ax], 2, device=m.device))
        for o in _AXES:
            if o == ax:
                continue
            shp = list(m.shape)
            shp[o:o + 1] = [shp[o] // 2, 2]
            m = m.reshape(shp).mean(dim=o + 1)
        out.append(m)
    return out


def _prolong(e):
    """Periodic trilinear prolongation of cell-centred values to the 2x-finer
    grid: fine cell 2i takes 3/4 e_i + 1/4 e_(i-1), fine cell 2i+1 takes
    3/4 e_i + 1/4 e_(i+1), along each axis."""
    for ax in (0, 1, 2):
        lo = 0.75 * e + 0.25 * _shift(e, 1, ax)
        hi = 0.75 * e + 0.25 * _shift(e, -1, ax)
        e = torch.stack([lo, hi], dim=ax + 1).flatten(ax, ax + 1)
    return e


def _restrict(r):
    """Adjoint of _prolong divided by 8: weights 1/8, 3/8, 3/8, 1/8 of the fine
    cells 2i-1 .. 2i+2 along each axis (so the V-cycle stays symmetric)."""
    for ax in (0, 1, 2):
        n = r.shape[ax] // 2
        ev = torch.index_select(r, ax, torch.arange(0, 2 * n, 2, device=r.device))
        od = torch.index_select(r, ax, torch.arange(1, 2 * n, 2, device=r.device))
        r = 0.375 * (ev + od) + 0.125 * (_shift(od, 1, ax) + _shift(ev, -1, ax))
    return r


class _Multigrid:
    """Symmetric V-cycle for the periodic variable-coefficient Laplacian
    (damped Jacobi, trilinear prolongation, its adjoint as restriction, face
    mobilities averaged over coarse interfaces, a dense pseudo-inverse on the
    coarsest grid), the conjugate-gradient preconditioner.  FP32."""

    def __init__(self, mf, h, nu=2, omega=0.7, max_coarse=512):
        mf = [m.float() for m in mf]
        self.levels = []
        while True:
            self.levels.append((mf, h, _diag(mf, h)))
            shape = mf[0].shape
            if mf[0].numel() <= max_coarse or any(n % 2 for n in shape):
                break
            mf, h = _coarsen_faces(mf), 2 * h
        cmf, ch, _ = self.levels[-1]
        shape = cmf[0].shape
        n = cmf[0].numel()
        eye = torch.eye(n, dtype=torch.float64, device=cmf[0].device).reshape(n, *shape)
        A = torch.stack([_apply(eye[k], [m.double() for m in cmf], ch).reshape(-1) for k in range(n)], dim=1)
        self.coarse_inv = torch.linalg.pinv(A).float()
        self.coarse_shape = shape
        self.nu, self.omega = nu, omega

    def _smooth(self, x, r, lvl, sweeps):
        mf, h, dg = self.levels[lvl]
        for _ in range(sweeps):
            x = x + self.omega * (r - _apply(x, mf, h)) / dg
        return x

    def _cycle(self, r, lvl):
        mf, h, _ = self.levels[lvl]
        if lvl == len(self.levels) - 1:
            x = (self.coarse_inv @ (r - r.mean()).reshape(-1)).reshape(self.coarse_shape)
            return x - x.mean()
        x = self._smooth(torch.zeros_like(r), r, lvl, self.nu)
        rc = _restrict(r - _apply(x, mf, h))
        x = x + _prolong(self._cycle(rc - rc.mean(), lvl + 1))
        return self._smooth(x, r, lvl, self.nu)

    def __call__(self, r):
        return self._cycle(r.float(), 0).double()


def _solve_periodic(rhs, mf, b, iters=200, rtol=1e-8):
    """Solve  sum_faces M_f (phi_nb - phi) / b^2 = rhs  on a periodic block
    grid by conjugate gradients (FP64) preconditioned with a multigrid
    V-cycle, robust to the orders-of-magnitude mobility contrast of a porous
    medium.  Zero-mean phi.  The iteration count is left in
    _solve_periodic.iterations."""
    rhs = rhs - rhs.mean()
    phi = torch.zeros_like(rhs)
    nrm = rhs.norm()
    _solve_periodic.iterations = 0
    if nrm == 0:
        return phi
    M = _Multigrid(mf, float(b))
    r = rhs.clone()
    z = M(r)
    p = z.clone()
    rz = (r * z).sum()
    for it in range(iters):
        Ap = _apply(p, mf, float(b))
        alpha = rz / (p * Ap).sum()
        phi = phi + alpha * p
        r = r - alpha * Ap
        _solve_periodic.iterations = it + 1
        if r.norm() <= rtol * nrm:
            break
        z = M(r)
        rz_new = (r * z).sum()
        p = z + (rz_new / rz) * p
        rz = rz_new
    return phi - phi.mean()


def darcy_pressure(mob, g, b, rtol=1e-8, face='geometric'):
    """Large-scale pressure of the upscaled (Darcy) problem on b^3 blocks.

    mob: (d, h, w) block mobility M (Darcy flux per unit driving force,
    isotropic); the block flux F = M_f (g x_hat - grad phi) across every face
    is conserved:  div(M grad phi) = g dM/dx.  phi is the pressure over rho0
    (p / rho0), zero mean, FP64.  This is the pressure field that the
    lattice Boltzmann run otherwise builds up by slow pressure diffusion
    across the whole domain.  The torch implementation here is the reference
    of the library's CUDA solve (darcy_pressure_device)."""
    mob = mob.double().clamp(min=1e-30)
    mf = _face_mobility(mob, face)
    rhs = g * (mf[0] - _shift(mf[0], 1, _AXES[0])) / b
    return _solve_periodic(rhs, mf, b, rtol=rtol)


def darcy_pressure_device(mob, g, b, rtol=1e-3, max_iter=200):
    """darcy_pressure (geometric face means) by the library's CUDA solver
    (lbf_darcy_pressure: multigrid-preconditioned conjugate gradients) on a
    CUDA tensor of block mobilities; returns (phi, iterations)."""
    import ctypes
    from . import LbfError, library
    lib = library()
    mob = mob.double().contiguous()
    phi = torch.empty_like(mob)
    it = ctypes.c_uint32(0)
    nz, ny, nx = mob.shape
    rc = lib.lbf_darcy_pressure(ctypes.c_void_p(mob.data_ptr()), nz, ny, nx, float(b), float(g), float(rtol),
                                int(max_iter), ctypes.c_void_p(phi.data_ptr()), ctypes.byref(it),
                                ctypes.c_void_p(torch.cuda.current_stream(mob.device).cuda_stream))
    if rc != 0:
        raise LbfError(rc, lib.lbf_last_error(None).decode())
    return phi, int(it.value)


def darcy_pressure_from_flux(q, mob, b, face='geometric'):
    """Coarse pressure that makes a block-averaged flux field conservative:
    q (d, h, w, 3) block-mean velocity, face flux = mean of the two blocks;
    solves div(M grad phi) = div q so that q - M grad(phi) is divergence-free."""
    q = q.double()
    mob = mob.double().clamp(min=1e-30)
    div = torch.zeros_like(mob)
    for c, ax in enumerate(_AXES):
        flux = 0.5 * (q[..., c] + _shift(q[..., c], -1, ax))
        div += (flux - _shift(flux, 1, ax)) / b
    return _solve_periodic(div, _face_mobility(mob, face), b)


def _upsample_periodic(phi, b):
    """Trilinear interpolation of block-centre values to voxel centres, periodic."""
    x = phi[None, None]
    x = torch.nn.functional.pad(x, (1, 1, 1, 1, 1, 1), mode='circular')
    d, h, w = phi.shape
    up = torch.nn.functional.interpolate(x, scale_factor=b, mode='trilinear', align_corners=False)
    # Padding by one block shifts the interpolated grid by b voxels.
    return up[0, 0, b:b + d * b, b:b + h * b, b:b + w * b]


def _pore_block_mean(x, m, b):
    """Pore-weighted block means of a (D, H, W) field (zero where a block has no pores)."""
    num = _block_mean((x * m)[..., None], b)[..., 0]
    den = _block_mean(m[..., None], b)[..., 0]
    return torch.where(den > 0, num / den.clamp(min=1e-30), torch.zeros_like(num))


def _smooth121(x, m):
    """Mask-normalised [1, 2, 1] / 4 filter along each axis (periodic) of a
    (D, H, W) field over the pores m: removes the grid-scale (Nyquist)
    component of a predicted field, which the lattice Boltzmann run would
    otherwise carry as a slowly decaying staggered mode."""
    num, den = x * m, m.clone()
    for ax in (0, 1, 2):
        num = 0.25 * (_shift(num, 1, ax) + 2.0 * num + _shift(num, -1, ax))
        den = 0.25 * (_shift(den, 1, ax) + 2.0 * den + _shift(den, -1, ax))
    return torch.where(den > 0, num / den.clamp(min=1e-30), torch.zeros_like(num)) * m


def predict(net, fluid, tau, g, rho0=1.0, block=8, mode='darcy', velocity=False, smooth=True):
    """Warm-start fields (D, H, W, 4) float32 on the GPU: velocity x, y, z and
    density for force g along +x and relaxation time tau.

    mode 'none':  velocity and density deviation 3 g pi straight from the network.
    mode 'darcy': the network's pi keeps only its structure below the block
                  scale; the block-scale pressure comes from darcy_pressure
                  with block mobilities = block means of the network's k_x / nu.
    mode 'flux':  the network's density plus the pressure that makes its
                  block fluxes conservative (darcy_pressure_from_flux).
    velocity=False (the default) starts from rest with the predicted density
    only: the velocity relaxes to the pressure within the viscous transient
    of a pore, so a predicted velocity adds nothing to the start, while its
    residual imperfections excite a period-2 staggered mode that keeps
    LBFlow's adjacent-step residual above 1e-6 (measured on the 256^3 cube:
    never converged in 150,000 steps with it, 95,000 steps without).
    smooth: [1, 2, 1] filter of the predicted fields (_smooth121)."""
    with torch.no_grad():
        f = features(fluid.unsqueeze(0))
        y = net(f)[0, ..., :4].float() * net.scale
        m = fluid.double()
        nu = (tau - 0.5) / 3.0
        yd = y.double()
        if smooth:
            yd = torch.stack([_smooth121(yd[..., c], m) for c in range(4)], dim=-1)
        out = torch.empty(*fluid.shape, 4, dtype=torch.float32, device=fluid.device)
        out[..., :3] = (yd[..., :3] * (g / nu) * m[..., None]).float()
        pi = yd[..., 3] * m
        if mode == 'darcy' and block:
            pi = pi - _upsample_periodic(_pore_block_mean(pi, m, block), block) * m
            mob = _block_mean(out[..., :1].double(), block)[..., 0] / g
            mob = torch.clamp(mob, min=1e-3 * float(mob.clamp(min=0).mean()) + 1e-30)
            phi = darcy_pressure(mob, g, block, rtol=1e-4)
            drho = 3.0 * g * pi + 3.0 * rho0 * _upsample_periodic(phi, block) * m
        elif mode == 'flux' and block:
            q = _block_mean(out[..., :3].double(), block)
            mob = torch.clamp(q[..., 0] / g, min=1e-3 * float(q[..., 0].clamp(min=0).mean() / g) + 1e-30)
            phi = darcy_pressure_from_flux(q, mob, block)
            drho = 3.0 * g * pi + 3.0 * rho0 * _upsample_periodic(phi, block) * m
        else:
            drho = 3.0 * g * pi
        if not velocity:
            out[..., :3] = 0.0
        # Zero-mean density deviation over the pores (mass of the rest state).
        drho = drho - drho.sum() / m.sum().clamp(min=1.0) * m
        out[..., 3] = (rho0 + drho).float()
        conv.check(fluid.device)
        return out.contiguous()


def warm_start(engine, net, fluid, tau, g, rho0=1.0, block=8, mode='darcy', velocity=False, smooth=True):
    """Initialise `engine` from the network's prediction; returns the fields."""
    fields = predict(net, fluid, tau, g, rho0, block, mode, velocity, smooth)
    torch.cuda.current_stream(fluid.device).synchronize()
    engine.initialize_equilibrium(fields)
    return fields


def block_mobility(s, g, b, rho0=1.0):
    """Block mobility of a running state from its block sums s (d, h, w, 5) =
    (sum rho, sum u_x, sum u_y, sum u_z, fluid voxels) over b^3 blocks: with
    the block flux q = sum u / b^3, the block pressure phi = (rho_b - rho0) /
    (3 rho0) and the driving force per unit mass g x_hat - grad phi (central
    differences), the least-squares M of q = M (g x_hat - grad phi) over the
    three components.  Returns (M, fluid voxels, phi); M is 0 where the drive
    vanishes."""
    cnt = s[..., 4]
    rho_b = torch.where(cnt > 0, s[..., 0] / cnt.clamp(min=1.0), torch.full_like(cnt, rho0))
    q = s[..., 1:4] / float(b ** 3)
    phi = (rho_b - rho0) / (3.0 * rho0)
    drive = []
    for c, ax in enumerate(_AXES):
        grad = (_shift(phi, -1, ax) - _shift(phi, 1, ax)) / (2.0 * b)
        drive.append((g if c == 0 else 0.0) - grad)
    num = sum(q[..., c] * drive[c] for c in range(3))
    den = sum(d * d for d in drive)
    mob = torch.where(den > 0, num / den.clamp(min=1e-300), torch.zeros_like(num))
    return mob, cnt, phi


def block_sums_dense(rho, u, fluid, b):
    """block_sums of dense fields: rho (D, H, W), u (3, D, H, W) (zero on
    solids), fluid (D, H, W) -> (D/b, H/b, W/b, 5) float64."""
    m = fluid.double()
    parts = [rho.double() * m, u[0].double(), u[1].double(), u[2].double(), m]
    return torch.stack([_block_mean(x[..., None], b)[..., 0] * float(b ** 3) for x in parts], dim=-1)


class DarcyAccelerator:
    """Block-scale pressure correction of a running single-phase engine.

    After the fast viscous transient the flow in each b^3 block is the local
    Darcy response  q = M (g x_hat - grad phi)  to the current pressure phi,
    while phi itself still creeps towards steady state by pressure diffusion
    across the domain -- the slowest modes of the run.  At each report step
    in `at` the accelerator reads the block sums (lbf_block_sums, kept on the
    device), estimates M per block from q and the block pressure gradient
    (least squares over the three components), solves the upscaled problem
    for the steady block pressure (darcy_pressure_device, geometric face
    means) and adds the difference as a density change at unchanged momentum
    (lbf_add_density).  Mass is conserved and the lattice Boltzmann fixed
    point is unchanged, so the converged answer is the solver's own; only
    the slow modes are shortened.  3-D, force along +x; grid edges must be
    multiples of the block edge."""

    def __init__(self, engine, fluid, g, rho0=1.0, block=2, at=(500,), rtol=1e-3, face='geometric', omega=1.0):
        """at: report steps to correct at, each an int (uses `block`) or a
        (step, block) pair.  rtol: relative residual at which the block
        pressure solve stops (the mobility estimate is far coarser).  face:
        block-face mobility average; omega: fraction of the pressure
        difference applied."""
        self.engine, self.g, self.rho0 = engine, g, rho0
        self.fluid = fluid.double()
        self.at = {}
        for item in at:
            t, b = item if isinstance(item, (tuple, list)) else (item, block)
            self.at[int(t)] = int(b)
        self.rtol, self.face, self.omega = rtol, face, omega
        self.applied = []
        self.iterations = []
        self.phases = []          # per correction: seconds of each phase (synchronised)
        self.seconds = 0.0

    def __call__(self, t):
        if t not in self.at:
            return False
        t0 = time.perf_counter()
        self.apply(self.at[t])
        torch.cuda.synchronize(self.fluid.device)
        self.seconds += time.perf_counter() - t0
        self.applied.append(t)
        return True

    def apply(self, b):
        g, rho0 = self.g, self.rho0
        dev = self.fluid.device
        D, H, W = self.fluid.shape
        marks = [('start', time.perf_counter())]

        def mark(name):
            torch.cuda.synchronize(dev)
            marks.append((name, time.perf_counter()))

        s = torch.empty(D // b, H // b, W // b, 5, dtype=torch.float64, device=dev)
        self.engine.block_sums(b, out=s)
        mark('block_sums')
        mob, cnt, phi = block_mobility(s, g, b, rho0)
        mob = torch.clamp(mob, min=1e-3 * float(mob.clamp(min=0).mean()) + 1e-30)
        mark('mobility')
        if mob.is_cuda and self.face == 'geometric':
            target, it = darcy_pressure_device(mob, g, b, rtol=self.rtol)
        else:
            target = darcy_pressure(mob, g, b, rtol=self.rtol, face=self.face)
            it = _solve_periodic.iterations
        self.iterations.append(it)
        mark('solve')
        porous = cnt > 0
        cur = phi - (phi * porous).sum() / porous.sum().clamp(min=1)
        dphi = self.omega * (target - cur) * porous
        drho = 3.0 * rho0 * _upsample_periodic(dphi, b) * self.fluid
        drho = drho - drho.sum() / self.fluid.sum().clamp(min=1.0) * self.fluid
        mark('density_field')
        self.engine.add_density(drho.float().contiguous())
        mark('add_density')
        self.phases.append({n: round(t - marks[k][1], 4) for k, (n, t) in enumerate(marks[1:])})


def save(net, path, meta=None):
    torch.save({'state': {k: v.detach().cpu() for k, v in net.state_dict().items()}, 'ch': CH,
                'meta': meta or {}}, path)


def load(path, device='cuda'):
    ck = torch.load(path, map_location='cpu', weights_only=False)
    if tuple(ck['ch']) != CH:
        raise ValueError(f'weights are for channels {ck["ch"]}, this network has {CH}')
    net = WarmStartNet()
    net.load_state_dict(ck['state'])
    return net.to(device), ck.get('meta', {})


# ------------------------------------------------------ learned mobility --
# The block Darcy correction (DarcyAccelerator) has to wait a few hundred
# steps of the run from rest before it can estimate each block's mobility
# from the developed local flow.  The mobility of a block is a local,
# geometry-only property (at fixed viscosity), so a convolutional network
# can predict it from the voxels at t = 0; the upscaled Darcy problem (the
# library's CUDA solve) then supplies the domain-scale coupling that a local
# network cannot see, and the run starts with its block-scale pressure in
# place.  Targets are the accelerator's own estimates after MOB_STEPS steps
# from rest, the state it corrects from.

MOB_BLOCK = 2
MOB_STEPS = 500


class MobilityNet(WarmStartNet):
    """WarmStartNet whose head channel 0 is the log block mobility
    log(M nu) (M of block_mobility, nu = (tau - 1/2)/3) of the MOB_BLOCK^3
    block a voxel lies in, normalised by `norm` = (mean, std); the block
    value is the mean over its voxels."""

    def __init__(self, seed=0):
        super().__init__(seed)
        self.register_buffer('norm', torch.tensor([0.0, 1.0]))

    def blocks(self, x, b=MOB_BLOCK):
        """x: (B, D, H, W, 8) features -> (B, D/b, H/b, W/b) normalised log mobility (float32)."""
        y = self(x)[..., 0].float()
        B, D, H, W = y.shape
        return y.reshape(B, D // b, b, H // b, b, W // b, b).mean(dim=(2, 4, 6))


def mobility_targets(rho, u, fluid, tau, g, b=MOB_BLOCK, rho0=1.0):
    """Training target of one medium from its state after MOB_STEPS steps:
    log(M nu) per block and the block's fluid voxel count as its weight
    (float32, (D/b, H/b, W/b) each), M clamped below as the accelerator
    clamps it."""
    s = block_sums_dense(rho, u, fluid, b)
    mob, cnt, _ = block_mobility(s, g, b, rho0)
    mob = torch.clamp(mob, min=1e-3 * float(mob.clamp(min=0).mean()) + 1e-30)
    nu = (tau - 0.5) / 3.0
    return torch.log(mob * nu).float(), cnt.float()


def _augment_blocks(feat, targ, wt, gen, b=MOB_BLOCK):
    """Periodic shifts by whole blocks, y/z mirrors and the y<->z swap (the
    block mobility is a scalar, so these leave it unchanged)."""
    dims = feat.shape[1:4]
    sh = [int(torch.randint(0, d // b, (1,), generator=gen)) for d in dims]
    feat = torch.roll(feat, [v * b for v in sh], dims=(1, 2, 3))
    targ = torch.roll(targ, sh, dims=(1, 2, 3))
    wt = torch.roll(wt, sh, dims=(1, 2, 3))
    for ax in (1, 2):
        if torch.rand(1, generator=gen).item() < 0.5:
            feat, targ, wt = feat.flip(ax), targ.flip(ax), wt.flip(ax)
    if dims[0] == dims[1] and torch.rand(1, generator=gen).item() < 0.5:
        feat, targ, wt = feat.transpose(1, 2), targ.transpose(1, 2), wt.transpose(1, 2)
    return feat.contiguous(), targ.contiguous(), wt.contiguous()


def train_mobility(net, samples, iters=3000, lr=2e-3, batch_voxels=2 * 96 ** 3, seed=0, log=None):
    """samples: list of (fluid (D,H,W) bool cuda, log-mobility target and
    weight, both (D/b,H/b,W/b) float cuda).  Weighted mean-square error of
    the normalised block log mobility, AdamW with a cosine schedule; every
    convolution and gradient on the tensor-core kernels.  Returns the loss
    history."""
    dev = samples[0][0].device
    w_all = torch.cat([w.reshape(-1) for _, _, w in samples]).double()
    t_all = torch.cat([t.reshape(-1) for _, t, _ in samples]).double()
    mu = float((w_all * t_all).sum() / w_all.sum())
    sd = float(torch.sqrt((w_all * (t_all - mu) ** 2).sum() / w_all.sum()).clamp(min=1e-6))
    net.norm.copy_(torch.tensor([mu, sd]))
    by_shape = {}
    for i, (fl, _, _) in enumerate(samples):
        by_shape.setdefault(tuple(fl.shape), []).append(i)
    shapes = sorted(by_shape)
    feats = [features(fl.unsqueeze(0))[0] for fl, _, _ in samples]
    opt = torch.optim.AdamW(net.parameters(), lr=lr, weight_decay=1e-4)
    gen = torch.Generator().manual_seed(seed)
    hist = []
    t0 = time.perf_counter()
    for it in range(iters):
        for gparam in opt.param_groups:
            gparam['lr'] = lr * 0.5 * (1 + math.cos(math.pi * it / iters))
        shp = shapes[int(torch.randint(0, len(shapes), (1,), generator=gen))]
        pool = by_shape[shp]
        nb = max(1, min(len(pool), batch_voxels // int(np.prod(shp))))
        pick = [pool[int(j)] for j in torch.randint(0, len(pool), (nb,), generator=gen)]
        fb, tb, wb = [], [], []
        for j in pick:
            f, t, w = _augment_blocks(feats[j].unsqueeze(0), samples[j][1].unsqueeze(0),
                                      samples[j][2].unsqueeze(0), gen)
            fb.append(f)
            tb.append(t)
            wb.append(w)
        fb, tb, wb = torch.cat(fb), (torch.cat(tb) - mu) / sd, torch.cat(wb)
        y = net.blocks(fb)
        loss = (((y - tb) ** 2) * wb).sum() / wb.sum()
        opt.zero_grad(set_to_none=True)
        loss.backward()
        torch.nn.utils.clip_grad_norm_(net.parameters(), 1.0)
        opt.step()
        if it % 50 == 0 or it == iters - 1:
            lv = float(loss.detach())
            hist.append((it, lv, time.perf_counter() - t0))
            if log:
                log(f'iter {it} loss {lv:.4e} shape {shp} batch {nb} {time.perf_counter() - t0:.1f}s')
    conv.check(dev)
    return hist


def predict_mobility(net, fluid, tau, b=MOB_BLOCK):
    """Block mobilities M (D/b, H/b, W/b) float64 of a fluid mask for
    relaxation time tau, from the network (blocks without fluid get 0)."""
    with torch.no_grad():
        y = net.blocks(features(fluid.unsqueeze(0)), b)[0].double()
        nu = (tau - 0.5) / 3.0
        mob = torch.exp(y * float(net.norm[1]) + float(net.norm[0])) / nu
        cnt = _block_mean(fluid.double()[..., None], b)[..., 0]
        return torch.where(cnt > 0, mob, torch.zeros_like(mob))


def evaluate_mobility(net, samples, tau=1.0):
    """Per medium: weighted RMS error and correlation of the predicted log
    block mobility against the target."""
    out = []
    for fl, t, w in samples:
        p = torch.log((predict_mobility(net, fl, tau) * ((tau - 0.5) / 3.0)).clamp(min=1e-300)).float()
        m = w > 0
        d = (p - t)[m]
        ww = w[m]
        rms = float(torch.sqrt((ww * d * d).sum() / ww.sum()))
        pc, tc = p[m] - (ww * p[m]).sum() / ww.sum(), t[m] - (ww * t[m]).sum() / ww.sum()
        corr = float((ww * pc * tc).sum() / torch.sqrt((ww * pc * pc).sum() * (ww * tc * tc).sum()).clamp(min=1e-30))
        out.append(dict(log_mob_rms=rms, log_mob_corr=corr))
    return out


def mobility_start(engine, net, fluid, tau, g, rho0=1.0, block=MOB_BLOCK, rtol=1e-3):
    """Start `engine` (single phase, force g along +x) with the block Darcy
    pressure of the predicted block mobilities: the same upscaled problem
    and density change as DarcyAccelerator, applied at t = 0 to the rest
    state, velocity at rest.  Returns the CG iterations of the solve."""
    mob = predict_mobility(net, fluid, tau, block)
    porous = mob > 0
    mob = torch.clamp(mob, min=1e-3 * float(mob.clamp(min=0).mean()) + 1e-30)
    target, it = darcy_pressure_device(mob, g, block, rtol=rtol)
    m = fluid.double()
    drho = 3.0 * rho0 * _upsample_periodic(target * porous, block) * m
    drho = drho - drho.sum() / m.sum().clamp(min=1.0) * m
    fields = torch.zeros(*fluid.shape, 4, dtype=torch.float32, device=fluid.device)
    fields[..., 3] = (rho0 + drho).float()
    torch.cuda.current_stream(fluid.device).synchronize()
    engine.initialize_equilibrium(fields.contiguous())
    return it


def save_mobility(net, path, meta=None):
    torch.save({'state': {k: v.detach().cpu() for k, v in net.state_dict().items()}, 'ch': CH,
                'kind': 'mobility', 'meta': meta or {}}, path)


def load_mobility(path, device='cuda'):
    ck = torch.load(path, map_location='cpu', weights_only=False)
    if tuple(ck['ch']) != CH or ck.get('kind') != 'mobility':
        raise ValueError(f'{path} does not hold block-mobility weights for channels {CH}')
    net = MobilityNet()
    net.load_state_dict(ck['state'])
    return net.to(device), ck.get('meta', {})


# ----------------------------------------------------------------- training --

def _augment(feat, targ, gen):
    """Random periodic shift, y/z mirrors and the y<->z swap (symmetries of a
    periodic medium under a force along x)."""
    dims = feat.shape[1:4]
    shifts = [int(torch.randint(0, d, (1,), generator=gen)) for d in dims]
    feat = torch.roll(feat, shifts, dims=(1, 2, 3))
    targ = torch.roll(targ, shifts, dims=(1, 2, 3))
    if torch.rand(1, generator=gen).item() < 0.5:          # mirror z: k_z -> -k_z
        feat, targ = feat.flip(1), targ.flip(1)
        targ = targ * torch.tensor([1, 1, -1, 1.0], device=targ.device)
    if torch.rand(1, generator=gen).item() < 0.5:          # mirror y: k_y -> -k_y
        feat, targ = feat.flip(2), targ.flip(2)
        targ = targ * torch.tensor([1, -1, 1, 1.0], device=targ.device)
    if dims[0] == dims[1] and torch.rand(1, generator=gen).item() < 0.5:   # swap z and y
        feat = feat.transpose(1, 2)
        targ = targ.transpose(1, 2)[..., [0, 2, 1, 3]]
    return feat.contiguous(), targ.contiguous()


def train(net, samples, iters=2000, lr=2e-3, batch_voxels=2 * 64 ** 3, seed=0, log=None, weights=(1, 0.5, 0.5, 2)):
    """samples: list of (fluid mask (D,H,W) bool cuda, target (D,H,W,4) float cuda).
    Minimises the normalised mean-square error over pore voxels with AdamW and
    a cosine learning-rate schedule.  Returns the loss history."""
    dev = samples[0][0].device
    # Normalisation: RMS of each target channel over pores.
    num = torch.zeros(4, dtype=torch.float64, device=dev)
    cnt = 0.0
    for fl, t in samples:
        num += (t[fl].double() ** 2).sum(0)
        cnt += float(fl.sum())
    scale = torch.sqrt(num / max(cnt, 1.0)).float().clamp(min=1e-6)
    net.scale.copy_(scale)
    by_shape = {}
    for i, (fl, _) in enumerate(samples):
        by_shape.setdefault(tuple(fl.shape), []).append(i)
    shapes = sorted(by_shape)
    feats = [features(fl.unsqueeze(0))[0] for fl, _ in samples]
    opt = torch.optim.AdamW(net.parameters(), lr=lr, weight_decay=1e-4)
    gen = torch.Generator().manual_seed(seed)
    wts = torch.tensor(weights, dtype=torch.float32, device=dev)
    hist = []
    t0 = time.perf_counter()
    for it in range(iters):
        for gparam in opt.param_groups:
            gparam['lr'] = lr * 0.5 * (1 + math.cos(math.pi * it / iters))
        shp = shapes[int(torch.randint(0, len(shapes), (1,), generator=gen))]
        pool = by_shape[shp]
        nb = max(1, min(len(pool), batch_voxels // int(np.prod(shp))))
        pick = [pool[int(j)] for j in torch.randint(0, len(pool), (nb,), generator=gen)]
        fb, tb = [], []
        for j in pick:
            f, t = _augment(feats[j].unsqueeze(0), samples[j][1].unsqueeze(0), gen)
            fb.append(f)
            tb.append(t)
        fb = torch.cat(fb)
        tb = torch.cat(tb) / scale
        mask = fb[..., 0].float().unsqueeze(-1)
        y = net(fb)[..., :4].float()
        loss = (((y - tb) ** 2) * mask * wts).sum() / (mask.sum() * wts.sum())
        opt.zero_grad(set_to_none=True)
        loss.backward()
        torch.nn.utils.clip_grad_norm_(net.parameters(), 1.0)
        opt.step()
        if it % 50 == 0 or it == iters - 1:
            lv = float(loss.detach())
            hist.append((it, lv, time.perf_counter() - t0))
            if log:
                log(f'iter {it} loss {lv:.4e} shape {shp} batch {nb} {time.perf_counter() - t0:.1f}s')
    conv.check(dev)
    return hist


def evaluate(net, samples):
    """Relative L2 error of the predicted k and pi over pores, and of the
    predicted permeability, per sample."""
    out = []
    with torch.no_grad():
        for fl, t in samples:
            y = net(features(fl.unsqueeze(0)))[0, ..., :4].float() * net.scale
            m = fl.float()
            ek = torch.sqrt((((y[..., :3] - t[..., :3]) ** 2).sum(-1) * m).sum() / ((t[..., :3] ** 2).sum(-1) * m).sum())
            ep = torch.sqrt((((y[..., 3] - t[..., 3]) ** 2) * m).sum() / ((t[..., 3] ** 2) * m).sum().clamp(min=1e-30))
            Kp = float((y[..., 0] * m).mean())
            Kt = float(t[..., 0].mean())
            out.append(dict(k_rel_l2=float(ek), pi_rel_l2=float(ep), K_pred=Kp, K_true=Kt,
                            K_rel_err=abs(Kp - Kt) / max(abs(Kt), 1e-30)))
    return out
