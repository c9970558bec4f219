"""The headline configuration: 1001 x 1001 nodes, 6 x 6 markers per cell (36M
markers), viscosity 1e18-1e24 Pa s, 8 extra stream-function modes, markers in
random storage order.

  * the mixed form over the workload's 10 steps against the FP64 form from the
    same seeded state: every node field within 1e-6 normwise (max|d| / max|ref|);
  * the FP64 form against the oracle (the reference's loop restated, summed in
    the cell-sorted order) over one step of a seeded 2M-marker subset on the full
    grid: markers bit for bit, the node fields without a libm call between marker
    and node bit for bit, the others within 1e-12.
"""
import numpy as np
import pytest

from i2elvis_planet_b200 import abi, lib, synth
from oracle import oracle

pytestmark = pytest.mark.gpu

EXACT_NODE = ("ro", "et", "cp", "ht", "tk", "po")


def normwise(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.fixture(scope="module")
def c3():
    return synth.make_config("c3")


def test_c3_mixed_within_1e6_of_fp64(c3):
    assert c3.marknum == 36_000_000 and c3.nsteps == 10
    m64, n64, ms = lib.run_instance(c3, precision=abi.PREC_FP64, track_tmax=False)
    ms.close()
    mmx, nmx, ms = lib.run_instance(c3, precision=abi.PREC_MIXED, track_tmax=False)
    assert ms.fused_info()["fused_moves"] == 10
    ms.close()
    errs = {k: normwise(nmx[k], n64[k]) for k in synth.NODE_OUT}
    for k, e in errs.items():
        assert e <= 1e-6, (k, errs)
    cell = c3.gx[1] - c3.gx[0]
    assert np.abs(mmx["x"] - m64["x"]).max() <= 1e-6 * cell
    assert np.abs(mmx["y"] - m64["y"]).max() <= 1e-6 * cell
    np.testing.assert_array_equal(mmx["T"], m64["T"])


def test_c3_fp64_matches_oracle_on_a_subset(c3):
    idx = np.sort(np.argsort(synth.rng_u64(2718, 1, c3.marknum), kind="stable")[:2_000_000])
    sub = synth.subset(c3, idx)
    sub.nsteps = 1
    mk, nodes, ms = lib.run_instance(sub, precision=abi.PREC_FP64, track_tmax=True)
    ms.close()
    s = oracle.Oracle(sub).run(order=oracle.ORDER_CELL)
    for f in ("x", "y", "T", "p", "tmax"):
        np.testing.assert_array_equal(mk[f], getattr(s, f), err_msg=f)
    for k in EXACT_NODE:
        np.testing.assert_array_equal(nodes[k], s.nodes[k], err_msg=k)
    for k in ("nu", "nd", "kt"):
        assert normwise(nodes[k], s.nodes[k]) <= 1e-12, k
