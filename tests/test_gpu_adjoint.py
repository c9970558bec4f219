"""Adjoint of the marker step through the C ABI, wrapped in a
torch.autograd.Function: checked against the FP64 reference gradient (torch
autograd of an independent FP64 implementation of the same forward model) and
against central finite differences (h = 1e-6 relative) at the 201x201 /
640,000-marker / 20-step configuration, checkpoint every 5 steps.

The forward model is piecewise bilinear: a marker whose RK4 stages pick another
stencil cell between the +h and -h runs adds an O(1) kink term to the
difference quotient.  The finite-difference checks therefore use the kink-free
subset of the loss: the nodes that no such marker reaches (found by comparing
every marker's stencil signature across the runs in the torch reference).  On
that subset the quotient is a plain derivative and agrees with the adjoint to
1e-5 (in practice ~1e-9)."""
import time

import numpy as np
import pytest
import torch

import marker_autograd as ma
from i2elvis_planet_b200 import abi, synth

pytestmark = pytest.mark.gpu


def target(inst):
    gx, gy = np.meshgrid(inst.gx, inst.gy, indexing="ij")
    L = inst.xsize
    return (900.0 + 600.0 * np.sin(np.pi * gx / L) * np.cos(2 * np.pi * gy / L)).reshape(-1)


def loss_and_grads(run, inst, T0, amps, tgt, mask=None):
    T = torch.as_tensor(T0).clone().requires_grad_(True)
    a = torch.as_tensor(amps).clone().requires_grad_(True)
    tk = ma.MarkerStepFn.apply(T, a, run)
    r2 = (tk - torch.as_tensor(tgt)) ** 2
    L = (r2 * torch.as_tensor(mask)).sum() if mask is not None else r2.sum()
    L.backward()
    return float(L.detach()), T.grad.numpy().copy(), a.grad.numpy().copy()


def loss_only(run, inst, T0, amps, tgt, mask=None):
    ms = run["ms"]
    ms.set_markers(inst.x, inst.y, T0, inst.eta, inst.mtype)
    ms.set_nodes(**inst.nodes)
    tk = ms.adjoint_forward(amps, run["nsteps"], inst.timestep, inst.timesum, run["every"])
    r2 = (tk - tgt) ** 2
    return float((r2 * mask).sum() if mask is not None else r2.sum())


def device():
    return torch.device("cuda") if torch.cuda.is_available() else torch.device("cpu")


def kink_free_mask(inst, nsteps, hrel):
    """1 on the nodes no marker reaches whose stencils differ between the base and
    any +-h run of any mode; 0 on the rest."""
    d = device()
    base, cell0 = ma.stencil_signature(inst, torch.as_tensor(inst.amps, device=d), nsteps)
    cells = []
    for m in range(inst.amps.size):
        for sgn in (1.0, -1.0):
            a = inst.amps.copy()
            a[m] += sgn * hrel * abs(inst.amps[m])
            sig, cell = ma.stencil_signature(inst, torch.as_tensor(a, device=d), nsteps)
            moved = sig != base
            cells += [cell[moved], cell0[moved]]
    cells = torch.unique(torch.cat(cells)).cpu().numpy()
    ny = inst.ynumy
    m1, m2 = np.divmod(cells, ny - 1)
    mask = np.ones(inst.nodenum)
    for a in (0, 1):
        for b in (0, 1):
            mask[(m1 + a) * ny + m2 + b] = 0.0
    return mask, cells.size


def fd_amps(run, inst, tgt, mask, hrel):
    fd = np.zeros(inst.amps.size)
    for m in range(inst.amps.size):
        h = hrel * abs(inst.amps[m])
        ap = inst.amps.copy(); ap[m] += h
        am = inst.amps.copy(); am[m] -= h
        fd[m] = (loss_only(run, inst, inst.T, ap, tgt, mask) - loss_only(run, inst, inst.T, am, tgt, mask)) / (2 * h)
    return fd


def test_fp64_adjoint_matches_reference_gradient():
    inst = synth.make_config("c5", n=41, nsteps=6)
    tgt = target(inst)
    run = ma.setup_run(inst, abi.PREC_FP64, nsteps=6, every=2)
    L, gT, ga = loss_and_grads(run, inst, inst.T, inst.amps, tgt)
    T = torch.as_tensor(inst.T).clone().requires_grad_(True)
    a = torch.as_tensor(inst.amps).clone().requires_grad_(True)
    Lr = ((ma.reference_tk(inst, T, a, 6) - torch.as_tensor(tgt)) ** 2).sum()
    Lr.backward()
    assert abs(L - float(Lr)) <= 1e-11 * abs(float(Lr))
    np.testing.assert_allclose(ga, a.grad.numpy(), rtol=1e-8, atol=1e-8 * np.abs(a.grad.numpy()).max())
    assert np.abs(gT - T.grad.numpy()).max() <= 1e-9 * np.abs(T.grad.numpy()).max()
    run["ms"].close()


def test_c5_fp64_adjoint_matches_reference_gradient():
    """The whole C5 configuration against the torch FP64 reference gradient."""
    inst = synth.make_config("c5")
    tgt = target(inst)
    run = ma.setup_run(inst, abi.PREC_FP64, nsteps=20, every=5)
    L, gT, ga = loss_and_grads(run, inst, inst.T, inst.amps, tgt)
    d = device()
    T = torch.as_tensor(inst.T, device=d).clone().requires_grad_(True)
    a = torch.as_tensor(inst.amps, device=d).clone().requires_grad_(True)
    Lr = ((ma.reference_tk(inst, T, a, 20) - torch.as_tensor(tgt, device=d)) ** 2).sum()
    Lr.backward()
    gar, gTr = a.grad.cpu().numpy(), T.grad.cpu().numpy()
    assert abs(L - float(Lr.detach())) <= 1e-11 * abs(float(Lr.detach()))
    assert np.abs(ga - gar).max() <= 1e-8 * np.abs(gar).max()
    assert np.abs(gT - gTr).max() <= 1e-9 * np.abs(gTr).max()
    run["ms"].close()


def test_c5_adjoint_matches_finite_differences():
    inst = synth.make_config("c5")
    tgt = target(inst)
    hrel = 1e-6
    mask, ncells = kink_free_mask(inst, 20, hrel)
    assert (mask == 0).sum() < 0.1 * mask.size  # the kinks touch few nodes
    run = ma.setup_run(inst, abi.PREC_FP64, nsteps=20, every=5)
    t0 = time.perf_counter()
    L, gT, ga = loss_and_grads(run, inst, inst.T, inst.amps, tgt, mask)
    t_adj = time.perf_counter() - t0
    fd = fd_amps(run, inst, tgt, mask, hrel)
    rel = np.abs(fd - ga) / np.abs(fd).max()
    print(f"kink-free subset: {int((mask == 0).sum())} of {mask.size} nodes left out ({ncells} cells); "
          f"FD vs adjoint normwise per mode {rel.tolist()}")
    assert rel.max() <= 1e-5, rel
    # temperatures: the loss is quadratic in T0, central differences are exact up to rounding
    for i in np.nonzero(inst.mtype == 5)[0][:3]:
        Tp = inst.T.copy(); Tp[i] += 1.0
        Tm = inst.T.copy(); Tm[i] -= 1.0
        dd = (loss_only(run, inst, Tp, inst.amps, tgt, mask) - loss_only(run, inst, Tm, inst.amps, tgt, mask)) / 2.0
        assert abs(dd - gT[i]) <= 1e-6 * max(abs(dd), abs(gT).max() * 1e-3)
    run["ms"].close()
    print(f"adjoint forward+backward {t_adj:.3f} s")


def test_c5_mixed_adjoint_matches_finite_differences():
    """The mixed form's adjoint against the derivative of the loss (central
    differences of the FP64 forward on the kink-free subset; the mixed forward's
    own FP32 rounding, ~1e-7, would swamp a 1e-6 quotient)."""
    inst = synth.make_config("c5")
    tgt = target(inst)
    mask, _ = kink_free_mask(inst, 20, 1e-6)
    r64 = ma.setup_run(inst, abi.PREC_FP64, nsteps=20, every=5)
    fd = fd_amps(r64, inst, tgt, mask, 1e-6)
    rmx = ma.setup_run(inst, abi.PREC_MIXED, nsteps=20, every=5)
    _, _, gamx = loss_and_grads(rmx, inst, inst.T, inst.amps, tgt, mask)
    rel = np.abs(gamx - fd) / np.abs(fd).max()
    assert rel.max() <= 1e-5, rel
    r64["ms"].close()
    rmx["ms"].close()


def test_mixed_adjoint_close_to_fp64():
    inst = synth.make_config("c5")
    tgt = target(inst)
    r64 = ma.setup_run(inst, abi.PREC_FP64, nsteps=20, every=5)
    rmx = ma.setup_run(inst, abi.PREC_MIXED, nsteps=20, every=5)
    _, gT64, ga64 = loss_and_grads(r64, inst, inst.T, inst.amps, tgt)
    _, gTmx, gamx = loss_and_grads(rmx, inst, inst.T, inst.amps, tgt)
    assert np.abs(gamx - ga64).max() <= 1e-5 * np.abs(ga64).max()
    assert np.abs(gTmx - gT64).max() <= 1e-5 * np.abs(gT64).max()
    r64["ms"].close()
    rmx["ms"].close()
