"""The C host shim (include/i2g_shim.c) as a drop-in for movemark() and
ronurecalc(): the reference's own time loop and globals, compiled from its
unmodified sources (oracle/ref_harness.c, the i2mart.c:107-153 order), with the
shim's two calls in place of the reference's (oracle/_ref/dropin32: the FP64
form; dropin32m: the mixed form), against the reference build (ref32) after the
same steps.  Both keep the markers in the reference's single-precision storage.

  * FP64 form: marker positions, temperatures, pressures and maximum temperatures
    bit for bit; node fields within 1e-12 (the reference sums in marker storage
    order, the shim's library in cell order);
  * mixed form: positions within two single-precision units; node fields within
    1e-6 of the field's largest value at 99.9% of the nodes and within 1e-4 at
    all: a position that rounds to the other single-precision neighbour can put
    a marker on the other side of the radmax circle (markmart.c:335-340), which
    changes its viscosity by orders of magnitude.

With densimod 2 (the P-T table path) the shim hands the reference's td[][][][]
table and melting switches to the library once and the eps[] melt state around
every ronurecalc; the marker types the library flips come back into markt[].
"""
import numpy as np
import pytest

import variants
from i2elvis_planet_b200 import synth
from oracle import refio

pytestmark = pytest.mark.gpu


def normwise(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.fixture(scope="module")
def case():
    inst = synth.make_config("c1", nsteps=3)
    return inst, refio.run_reference(inst, "ref32", nsteps=3)


def test_dropin_fp64_matches_the_reference_build(case):
    inst, ref = case
    got = refio.run_reference(inst, "dropin32", nsteps=3)
    for f in ("x", "y", "T", "p", "tmax"):
        np.testing.assert_array_equal(getattr(got, f), getattr(ref, f), err_msg=f)
    for k in synth.NODE_OUT:
        assert normwise(got.nodes[k], ref.nodes[k]) <= 1e-12, k


def test_dropin_mixed_close_to_the_reference_build(case):
    inst, ref = case
    got = refio.run_reference(inst, "dropin32m", nsteps=3)
    for f in ("x", "y"):
        a, b = getattr(got, f), getattr(ref, f)
        ulp = np.spacing(np.abs(b).astype(np.float32)).astype(np.float64)
        assert (np.abs(a - b) <= 2 * ulp).all(), f
    for k in synth.NODE_OUT:
        a, b = got.nodes[k], ref.nodes[k]
        d = np.abs(a - b) / max(np.abs(b).max(), 1e-300)
        assert (d <= 1e-6).mean() >= 0.999 and d.max() <= 1e-4, (k, d.max(), int((d > 1e-6).sum()))


def test_dropin_table_path_matches_the_reference_build():
    inst = variants.variant("td")
    ref = refio.run_reference(inst, "ref32")
    got = refio.run_reference(inst, "dropin32")
    for f in ("x", "y", "T", "p", "tmax"):
        np.testing.assert_array_equal(getattr(got, f), getattr(ref, f), err_msg=f)
    np.testing.assert_array_equal(got.mtype, ref.mtype)
    assert (ref.mtype != inst.mtype).sum() > 100
    np.testing.assert_allclose(got.melt, ref.melt, rtol=1e-12, atol=0)
    for k in synth.NODE_OUT:
        if k in variants.DEVIATIONS["td"]:
            continue
        assert normwise(got.nodes[k], ref.nodes[k]) <= 1e-12, k


def test_dropin_resident_markers_match(case):
    """The shim with resident markers (-DI2G_SHIM_RESIDENT: markers go up only
    when the host flagged a change, the host arrays are brought current on
    i2g_shim_sync_host) gives the FP64 drop-in's results bit for bit; the
    harness re-injects eta between the calls (sync, write, flag)."""
    inst, ref = case
    a = refio.run_reference(inst, "dropin32", nsteps=3)
    b = refio.run_reference(inst, "dropin32r", nsteps=3)
    for f in ("x", "y", "T", "eta", "p", "tmax", "por"):
        np.testing.assert_array_equal(getattr(b, f), getattr(a, f), err_msg=f)
    np.testing.assert_array_equal(b.mtype, a.mtype)
    for k in synth.NODE_OUT:
        np.testing.assert_array_equal(b.nodes[k], a.nodes[k], err_msg=k)


@pytest.mark.parametrize("name", ["mag_dynamo0", "mag_dynamo1"])
def test_dropin_magnetisation_matches_the_reference_build(name):
    """markmg_old / markmg_time (markmart.c:651-744) through the shim: the host's
    arrays go up with the markers and come back after ronurecalc, equal to the
    reference build's; the resident shim brings them back on sync."""
    inst = variants.variant(name)
    ref = refio.run_reference(inst, "ref32")
    for build in ("dropin32", "dropin32r"):
        got = refio.run_reference(inst, build)
        np.testing.assert_array_equal(got.mg_old, ref.mg_old, err_msg=build)
        np.testing.assert_array_equal(got.mg_time, ref.mg_time, err_msg=build)
        for f in ("x", "y", "T", "p"):
            np.testing.assert_array_equal(getattr(got, f), getattr(ref, f), err_msg=(build, f))
    assert (ref.mg_old != inst.mg_old).sum() > 0
