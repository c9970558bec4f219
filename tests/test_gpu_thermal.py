"""Parity of the CUDA marker temperature update (titerate(), heatmart.c:514-697)
with the oracle and the compiled reference.

Bars (FP64 form): with heatdif = 0 every marker temperature is bit-identical to the
oracle and to the reference (FP64 storage); with heatdif != 0 the diffusion step
takes exp() from CUDA's libdevice, which can differ from the host libm in the last
bit, so temperatures agree to 1e-13 relative.  Mixed form: within 1e-6 relative of
the FP64 form.
"""
import hashlib
import os

import numpy as np
import pytest

import variants
from i2elvis_planet_b200 import abi, lib, synth
from oracle import oracle

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL_EXP = 1e-13  # last-bit exp differences, relative to max |T|


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def gpu_thermal(inst, tk_new, heatdif, precision=abi.PREC_FP64, pass_fields=True):
    ms = lib.MarkerStep.from_instance(inst, precision=precision)
    n = inst.nodes
    if pass_fields:
        ms.titerate_markers(tk_new, n["tk"], heatdif, inst.timestep, kt=n["kt"], cp=n["cp"], ro=n["ro"])
    else:
        ms.set_nodes(kt=n["kt"], cp=n["cp"], ro=n["ro"])
        ms.titerate_markers(tk_new, n["tk"], heatdif, inst.timestep)
    T = ms.get_markers(fields=("T",))["T"]
    ms.close()
    return T


def oracle_thermal(inst, tk_new, heatdif):
    o = oracle.Oracle(inst)
    s = o.initial_state()
    o.titerate_markers(s, tk_new, heatdif, inst.timestep, order=oracle.ORDER_CELL)
    return s.T


@pytest.mark.parametrize("name", variants.THERMAL_NAMES)
def test_titerate_fp64_matches_oracle_and_reference(name):
    inst, tk_new, heatdif = variants.thermal_variant(name)
    T = gpu_thermal(inst, tk_new, heatdif)
    ref = oracle_thermal(inst, tk_new, heatdif)
    g = np.load(os.path.join(GOLD, f"titerate_{name}_ref64.npz"))
    if heatdif == 0:
        np.testing.assert_array_equal(T, ref)
        assert digest(T) == str(g["digest_T"])
    else:
        assert rel(T, ref) <= TOL_EXP
        assert rel(T[::int(g["stride"])], g["m_T"]) <= TOL_EXP


def test_titerate_device_node_fields():
    """kt, cp, ro left NULL: the context's node fields (here from i2g_set_nodes)."""
    inst, tk_new, heatdif = variants.thermal_variant("thermal")
    a = gpu_thermal(inst, tk_new, heatdif, pass_fields=True)
    b = gpu_thermal(inst, tk_new, heatdif, pass_fields=False)
    np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("name", ("thermal", "thermal_strong"))
def test_titerate_mixed_within_1e6_of_fp64(name):
    inst, tk_new, heatdif = variants.thermal_variant(name)
    t64 = gpu_thermal(inst, tk_new, heatdif)
    tmx = gpu_thermal(inst, tk_new, heatdif, precision=abi.PREC_MIXED)
    assert rel(tmx, t64) <= 1e-6


@pytest.mark.parametrize("moved", ("after_ronurecalc", "after_movemark"))
def test_titerate_in_the_time_loop(moved):
    """titerate between ronurecalc and the next movemark (the reference's order,
    i2mart.c:94-146) sums in the ranking ronurecalc left; right after a movemark
    the markers are ranked first.  Markers in random storage order, three steps."""
    inst = synth.make_config("c1", permute=True)
    f = synth.thermal_fields(inst, fluid_frac=0.05, cold_frac=0.02)
    ms = lib.MarkerStep.from_instance(inst, precision=abi.PREC_FP64)
    ms.set_reorder_interval(3)
    o = oracle.Oracle(inst)
    s = o.initial_state()
    ts = inst.timesum
    for step in range(3):
        ms.movemark(inst.timestep, ts)
        o.movemark(s, inst.timestep, ts)
        s.eta[:] = inst.eta
        if moved == "after_ronurecalc":
            ms.ronurecalc(ts)
            o.ronurecalc(s, ts, order=oracle.ORDER_CELL)
        s.nodes.update({k: inst.nodes[k] for k in ("tk", "kt", "cp", "ro")})
        ms.titerate_markers(f["tk_new"], inst.nodes["tk"], 1.0, inst.timestep, kt=inst.nodes["kt"],
                            cp=inst.nodes["cp"], ro=inst.nodes["ro"])
        o.titerate_markers(s, f["tk_new"], 1.0, inst.timestep, order=oracle.ORDER_CELL)
        ts += inst.timestep
    mk = ms.get_markers(fields=("x", "y", "T"))
    ms.close()
    np.testing.assert_array_equal(mk["x"], s.x)
    np.testing.assert_array_equal(mk["y"], s.y)
    assert rel(mk["T"], s.T) <= TOL_EXP


def test_titerate_errors():
    inst, tk_new, heatdif = variants.thermal_variant("thermal")
    ms = lib.MarkerStep.from_instance(inst, upload=False)
    with pytest.raises(lib.I2GError) as e:
        ms.titerate_markers(tk_new, inst.nodes["tk"], heatdif, inst.timestep)
    assert e.value.status == abi.ESTATE
    ms.close()
    ms = lib.MarkerStep.from_instance(inst)
    with pytest.raises(lib.I2GError) as e:
        ms.titerate_markers(tk_new, None, heatdif, inst.timestep)
    assert e.value.status == abi.EINVAL
    with pytest.raises(lib.I2GError) as e:
        ms.titerate_markers(tk_new, inst.nodes["tk"], float("nan"), inst.timestep)
    assert e.value.status == abi.EINVAL
    ms.close()


def test_titerate_device_arrays_match_host_arrays():
    """i2g_titerate_markers_dev reads device arrays in place: same result."""
    import torch
    inst, tk_new, heatdif = variants.thermal_variant("thermal")
    a = gpu_thermal(inst, tk_new, heatdif)
    ms = lib.MarkerStep.from_instance(inst)
    dev = {k: torch.tensor(v, dtype=torch.float64, device="cuda") for k, v in
           (("tn", tk_new), ("to", inst.nodes["tk"]), ("kt", inst.nodes["kt"]), ("cp", inst.nodes["cp"]),
            ("ro", inst.nodes["ro"]))}
    torch.cuda.synchronize()
    ms.titerate_markers_dev(dev["tn"], dev["to"], heatdif, inst.timestep, kt=dev["kt"], cp=dev["cp"], ro=dev["ro"])
    b = ms.get_markers(fields=("T",))["T"]
    ms.close()
    np.testing.assert_array_equal(a, b)
