"""Test harness for the adjoint: a torch.autograd.Function around the C-ABI
adjoint, and an independent FP64 reference of the same forward model written
with torch tensors (on the CPU or a GPU), whose autograd gradient is the FP64
reference gradient.

Forward model: nsteps x {movemark (RK4, markmart.c:73-115); ronurecalc}, with
the grid velocity v = sum_m a_m (vx_m, vy_m); output the final node temperatures
tk = sum_i w_i T_i / sum_i w_i (markmart.c:899-906, 988-991).
"""
from __future__ import annotations

import numpy as np
import torch

from i2elvis_planet_b200 import lib


class MarkerStepFn(torch.autograd.Function):
    """tk = F(T0, amps) on the GPU; backward runs i2g_adjoint_backward."""

    @staticmethod
    def forward(ctx, T0, amps, run):
        ms, inst = run["ms"], run["inst"]
        ms.set_markers(inst.x, inst.y, T0.detach().cpu().numpy(), inst.eta, inst.mtype)
        ms.set_nodes(**inst.nodes)
        tk = ms.adjoint_forward(amps.detach().cpu().numpy(), run["nsteps"], inst.timestep, inst.timesum,
                                run.get("every", 5))
        ctx.run = run
        return torch.from_numpy(tk)

    @staticmethod
    def backward(ctx, g):
        dT, da = ctx.run["ms"].adjoint_backward(g.detach().cpu().numpy())
        return torch.from_numpy(dT), torch.from_numpy(da), None


def setup_run(inst, precision, nsteps, every=5):
    ms = lib.MarkerStep.from_instance(inst, precision=precision)
    ms.adjoint_setup(inst.mode_vx, inst.mode_vy)
    return {"ms": ms, "inst": inst, "nsteps": nsteps, "every": every}


# ---------------------------------------------------------------- torch FP64 reference
def _cell(g, x):
    """largest m in [0, n-2] with g[m] <= x (m1serch/m2serch, markmart.c:1051-1088)"""
    m = torch.searchsorted(g, x.detach(), right=True) - 1
    return m.clamp(0, g.numel() - 2)


def _interp_v(inst, vxf, vyf, x, y, sig=None):
    """allinterv() (markmart.c:1378-1453) with autograd through positions and fields.
    sig (int64 per marker, optional) accumulates the stencil cells the call picks."""
    gx = torch.as_tensor(inst.gx, device=x.device)
    gy = torch.as_tensor(inst.gy, device=x.device)
    nx, ny = gx.numel(), gy.numel()
    xc = x.clamp(0.0, inst.xsize)
    yc = y.clamp(0.0, inst.ysize)
    m10 = _cell(gx, xc)
    m20 = _cell(gy, yc)
    xmid = 0.5 * (gx[1:] + gx[:-1])
    ymid = 0.5 * (gy[1:] + gy[:-1])
    # vx: basic columns, staggered rows
    m2 = (m20 - (yc.detach() < ymid[m20]).long()).clamp(0, ny - 3)
    x0, x1 = gx[m10], gx[m10 + 1]
    y0, y1 = ymid[m2], ymid[m2 + 1]
    wx1 = (xc - x0) / (x1 - x0)
    wy1 = (yc - y0) / (y1 - y0)
    wx0, wy0 = 1 - wx1, 1 - wy1
    i00 = m10 * ny + m2
    vx = (wx0 * wy0 * vxf[i00] + wx0 * wy1 * vxf[i00 + 1] + wx1 * wy0 * vxf[i00 + ny] +
          wx1 * wy1 * vxf[i00 + ny + 1])
    # vy: staggered columns, basic rows
    m1 = (m10 - (xc.detach() < xmid[m10]).long()).clamp(0, nx - 3)
    x0, x1 = xmid[m1], xmid[m1 + 1]
    y0, y1 = gy[m20], gy[m20 + 1]
    wx1 = (xc - x0) / (x1 - x0)
    wy1 = (yc - y0) / (y1 - y0)
    wx0, wy0 = 1 - wx1, 1 - wy1
    i00 = m1 * ny + m20
    vy = (wx0 * wy0 * vyf[i00] + wx0 * wy1 * vyf[i00 + 1] + wx1 * wy0 * vyf[i00 + ny] +
          wx1 * wy1 * vyf[i00 + ny + 1])
    if sig is not None:
        sig.mul_(1000003).add_(((m10 * ny + m20) * ny + m2) * nx + m1)
    return vx, vy


def _positions(inst, amps, nsteps, sig=None):
    dev = amps.device
    mvx = torch.as_tensor(inst.mode_vx, device=dev)
    mvy = torch.as_tensor(inst.mode_vy, device=dev)
    vxf = amps @ mvx
    vyf = amps @ mvy
    x = torch.as_tensor(inst.x, device=dev).clone()
    y = torch.as_tensor(inst.y, device=dev).clone()
    dt = inst.timestep
    for _ in range(nsteps):
        k1x, k1y = _interp_v(inst, vxf, vyf, x, y, sig)
        k2x, k2y = _interp_v(inst, vxf, vyf, x + k1x * dt / 2.0, y + k1y * dt / 2.0, sig)
        k3x, k3y = _interp_v(inst, vxf, vyf, x + k2x * dt / 2.0, y + k2y * dt / 2.0, sig)
        k4x, k4y = _interp_v(inst, vxf, vyf, x + k3x * dt, y + k3y * dt, sig)
        x = x + dt * (k1x + 2.0 * k2x + 2.0 * k3x + k4x) / 6.0
        y = y + dt * (k1y + 2.0 * k2y + 2.0 * k3y + k4y) / 6.0
    return x, y


def stencil_signature(inst, amps: torch.Tensor, nsteps: int):
    """Per marker, a hash of every stencil cell its RK4 stages pick and of its
    final cell, and that final cell: two runs whose signatures differ for a
    marker took different branches of the piecewise-bilinear model for it."""
    with torch.no_grad():
        sig = torch.zeros(inst.marknum, dtype=torch.int64, device=amps.device)
        x, y = _positions(inst, amps, nsteps, sig)
        gx = torch.as_tensor(inst.gx, device=amps.device)
        gy = torch.as_tensor(inst.gy, device=amps.device)
        m10, m20 = _cell(gx, x.clamp(0.0, inst.xsize)), _cell(gy, y.clamp(0.0, inst.ysize))
        inside = (x > 0) & (y > 0) & (x < inst.xsize) & (y < inst.ysize)
        sig.mul_(1000003).add_((m10 * gy.numel() + m20) * 2 + inside.long())
        return sig, m10 * (gy.numel() - 1) + m20


def reference_tk(inst, T0: torch.Tensor, amps: torch.Tensor, nsteps: int) -> torch.Tensor:
    """The forward model in torch FP64: RK4 positions, then the final averaging
    (on the device of amps)."""
    dev = amps.device
    x, y = _positions(inst, amps, nsteps)
    L = inst.xsize
    inside = (x > 0) & (y > 0) & (x < L) & (y < inst.ysize) & (T0 > 0)
    mtype = torch.as_tensor(inst.mtype.astype(np.int64), device=dev)
    T = torch.where(mtype < 2, torch.full_like(T0, inst.scal["tmp_ambient"]), T0)
    gx = torch.as_tensor(inst.gx, device=dev)
    gy = torch.as_tensor(inst.gy, device=dev)
    ny = gy.numel()
    m10 = _cell(gx, x)
    m20 = _cell(gy, y)
    wx1 = (x - gx[m10]) / (gx[m10 + 1] - gx[m10])
    wy1 = (y - gy[m20]) / (gy[m20 + 1] - gy[m20])
    wx0, wy0 = 1 - wx1, 1 - wy1
    nn = inst.nodenum
    num = torch.zeros(nn, dtype=torch.float64, device=dev)
    den = torch.zeros(nn, dtype=torch.float64, device=dev)
    mask = inside.double()
    for a, wa in ((0, wx0), (1, wx1)):
        for b, wb in ((0, wy0), (1, wy1)):
            idx = (m10 + a) * ny + m20 + b
            w = wa * wb * mask
            num = num.index_add(0, idx, w * T)
            den = den.index_add(0, idx, w)
    tk0 = torch.as_tensor(inst.nodes["tk"], device=dev)
    return torch.where(den > 0, num / torch.where(den > 0, den, torch.ones_like(den)), tk0)
