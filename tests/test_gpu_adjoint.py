"""Adjoint of the marker step through the C ABI, wrapped in a
torch.autograd.Function: checked against the FP64 reference gradient (torch
autograd of an independent FP64 implementation of the same forward model) and
against central finite differences (h = 1e-6 relative) at the 201x201 /
640,000-marker / 20-step configuration, checkpoint every 5 steps."""
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


def loss_and_grads(run, inst, T0, amps, tgt):
    T = torch.as_tensor(T0).clone().requires_grad_(True)
    a = torch.as_tensor(amps).clone().requires_grad_(True)
    tk = ma.MarkerStepFn.apply(T, a, run)
    L = ((tk - torch.as_tensor(tgt)) ** 2).sum()
    L.backward()
    return float(L.detach()), T.grad.numpy().copy(), a.grad.numpy().copy()


def loss_only(run, inst, T0, amps, tgt):
    ms = run["ms"]
    ms.set_markers(inst.x, inst.y, T0, inst.eta, inst.mtype)
    ms.set_nodes(**inst.nodes)
    tk = ms.adjoint_forward(amps, run["nsteps"], inst.timestep, inst.timesum, run["every"])
    return float(((tk - tgt) ** 2).sum())


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


def test_c5_adjoint_matches_finite_differences():
    inst = synth.make_config("c5")
    tgt = target(inst)
    run = ma.setup_run(inst, abi.PREC_FP64, nsteps=20, every=5)
    t0 = time.perf_counter()
    L, gT, ga = loss_and_grads(run, inst, inst.T, inst.amps, tgt)
    t_adj = time.perf_counter() - t0
    rels = {}
    for hrel in (1e-6, 1e-7):
        fd = np.zeros_like(ga)
        for m in range(ga.size):
            h = hrel * abs(inst.amps[m])
            ap = inst.amps.copy(); ap[m] += h
            am = inst.amps.copy(); am[m] -= h
            fd[m] = (loss_only(run, inst, inst.T, ap, tgt) - loss_only(run, inst, inst.T, am, tgt)) / (2 * h)
        rels[hrel] = np.abs(fd - ga) / np.abs(fd).max()
    print("FD vs adjoint, normwise per mode:", {k: v.tolist() for k, v in rels.items()})
    # The interpolant is piecewise bilinear: a marker that crosses a cell face or a
    # staggered midline between the +h and -h runs adds an O(1) kink term to the
    # difference quotient, so the residual shrinks with h (the exact check is the
    # FP64 reference gradient above): within 2e-5 normwise at h = 1e-6 and within
    # 1e-5 at h = 1e-7.
    assert rels[1e-6].max() <= 2e-5, rels
    assert rels[1e-7].max() <= 1e-5, rels
    # temperatures: the loss is quadratic in T0, central differences are exact up to rounding
    for i in np.nonzero(inst.mtype == 5)[0][:3]:
        Tp = inst.T.copy(); Tp[i] += 1.0
        Tm = inst.T.copy(); Tm[i] -= 1.0
        d = (loss_only(run, inst, Tp, inst.amps, tgt) - loss_only(run, inst, Tm, inst.amps, tgt)) / 2.0
        assert abs(d - gT[i]) <= 1e-6 * max(abs(d), abs(gT).max() * 1e-3)
    run["ms"].close()
    print(f"adjoint forward+backward {t_adj:.3f} s")


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
