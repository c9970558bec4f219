"""i2g_interp_tnode: allintert() (markmart.c:1687-1745) at every device-resident
marker, against the oracle's restatement, bit for bit in both precision forms
(the kernel is FP64, in the reference's order of operations), with markers on
grid lines, on and outside the box edges, on a uniform and a nonuniform grid and
after the markers moved."""
import numpy as np
import pytest

import variants
from i2elvis_planet_b200 import abi, lib
from oracle import oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["edges", "outgrid2", "nonuniform"])
@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_MIXED])
def test_interp_tnode_matches_oracle(name, precision):
    inst = variants.variant(name)
    ms = lib.MarkerStep.from_instance(inst, precision=precision)
    ms.movemark(inst.timestep, inst.timesum)
    ms.ronurecalc(inst.timesum)
    tk = ms.get_nodes()["tk"]
    tk2 = tk + 5.0 * np.sin(np.arange(tk.size) * 0.37)
    out, out2 = ms.interp_tnode(tk, tk2)
    mk = ms.get_markers()
    ms.close()
    o = oracle.Oracle(inst)
    s = o.initial_state()
    s.x, s.y = mk["x"], mk["y"]
    ref, ref2 = o.interp_tnode(s, tk, tk2)
    np.testing.assert_array_equal(out, ref)
    np.testing.assert_array_equal(out2, ref2)
    assert ((mk["x"] < 0) | (mk["x"] > inst.xsize)).any() or name != "outgrid2"


def test_interp_tnode_arguments():
    """A constant field comes back at every marker (to rounding); a missing field or
    output is I2G_EINVAL."""
    inst = variants.variant("default")
    ms = lib.MarkerStep.from_instance(inst, precision=abi.PREC_MIXED)
    out, out2 = ms.interp_tnode(np.full(inst.nodenum, 500.0))
    assert out2 is None and np.abs(out - 500.0).max() <= 1e-12 * 500.0
    assert ms.lib.i2g_interp_tnode(ms.h, None, None, None, None) == abi.EINVAL
    ms.close()
