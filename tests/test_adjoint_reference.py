"""The torch FP64 reference of the adjoint's forward model agrees with the
oracle (the sequential restatement pinned to the compiled reference): positions
after several RK4 steps and the final node temperatures."""
import numpy as np
import torch

import marker_autograd as ma
from i2elvis_planet_b200 import synth
from oracle import oracle


def small_c5(n=41, nsteps=4):
    return synth.make_config("c5", n=n, nsteps=nsteps)


def test_reference_forward_matches_oracle():
    inst = small_c5()
    T0 = torch.as_tensor(inst.T)
    amps = torch.as_tensor(inst.amps)
    tk = ma.reference_tk(inst, T0, amps, inst.nsteps).numpy()
    s = oracle.Oracle(inst).run(order=oracle.ORDER_CELL)
    err = np.abs(tk - s.nodes["tk"]).max() / np.abs(s.nodes["tk"]).max()
    assert err < 1e-12, err


def test_reference_gradient_is_linear_in_T0():
    """dL/dT0 of L = sum (tk - tgt)^2 at T0 and at 2*T0 - tgt-independent parts: the
    loss is quadratic in T0, so central differences in T0 are exact."""
    inst = small_c5(n=21, nsteps=2)
    T0 = torch.as_tensor(inst.T).clone().requires_grad_(True)
    amps = torch.as_tensor(inst.amps)
    tgt = torch.linspace(100.0, 1500.0, inst.nodenum, dtype=torch.float64)
    L = ((ma.reference_tk(inst, T0, amps, inst.nsteps) - tgt) ** 2).sum()
    L.backward()
    i = int(np.argmax(inst.mtype != 0))
    h = 1.0
    with torch.no_grad():
        Tp = T0.detach().clone(); Tp[i] += h
        Tm = T0.detach().clone(); Tm[i] -= h
        Lp = ((ma.reference_tk(inst, Tp, amps, inst.nsteps) - tgt) ** 2).sum()
        Lm = ((ma.reference_tk(inst, Tm, amps, inst.nsteps) - tgt) ** 2).sum()
    fd = float((Lp - Lm) / (2 * h))
    assert abs(fd - float(T0.grad[i])) <= 1e-8 * max(abs(fd), 1.0)
