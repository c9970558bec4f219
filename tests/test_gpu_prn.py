"""The device codec of the output file's marker section (i2g_write_prn_markers,
i2g_read_prn_markers) against the reference's saver()/loader() and the numpy
restatement pinned to them (oracle/prn.py, tests/test_prn_codec.py): bit for bit."""
import hashlib
import os

import numpy as np
import pytest

import variants
from i2elvis_planet_b200 import abi, lib, synth
from oracle import prn, refio

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def context(inst, precision=abi.PREC_FP64):
    ms = lib.MarkerStep.from_instance(inst, precision=precision)
    ms.set_marker_extras(tmax=inst.tmax, hi=inst.hi, por=inst.por)
    return ms


def extras(inst):
    return dict(gr=inst.gr, acc=inst.acc, mg_old=inst.mg_old, mg_time=inst.mg_time)


def test_write_matches_saver():
    inst = variants.prn_instance()
    g = np.load(os.path.join(GOLD, "prn_ref32.npz"))
    ms = context(inst)
    b = ms.write_prn(**extras(inst)) + bytes(abi.PRN_RECORD_BYTES)
    assert digest(np.frombuffer(b, np.uint8)) == str(g["section_digest"])
    ms.close()


def test_read_matches_loader():
    inst = variants.prn_instance()
    g = np.load(os.path.join(GOLD, "prn_ref32.npz"))
    src = context(inst)
    data = src.write_prn(**extras(inst))
    src.close()
    ms = lib.MarkerStep.from_instance(inst, upload=False)
    ms.set_grid(inst.gx, inst.gy, **inst.grid)
    got = ms.read_prn(data)
    mk = ms.get_markers(fields=("x", "y", "T", "eta", "type"), with_tmax=True)
    for k in ("x", "y", "T", "eta", "tmax"):
        assert digest(mk[k]) == str(g[f"digest_{k}"]), k
    assert digest(mk["type"]) == str(g["digest_mtype"])
    assert digest(got["gr"].astype(np.float64)) == str(g["digest_gr"])
    assert digest(got["acc"].astype(np.float64)) == str(g["digest_acc"])
    assert digest(got["mg_time"]) == str(g["digest_mg_time"])
    assert digest(got["mg_old"]) == str(g["digest_mg_old"])
    # write -> read -> write is the identity on the section
    assert ms.write_prn(**extras(inst)) == data
    ms.close()


@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_MIXED], ids=["fp64", "mixed"])
def test_write_after_steps_matches_restatement(precision):
    """After three steps of the c1 workload (markers in cell order on the device),
    the section equals the restatement packed from the caller-order state."""
    inst = synth.make_config("c1", nsteps=3)
    n = inst.marknum
    inst.gr, inst.acc = 10.0 * synth.rng_uniform(8, 1, n), 5.0 * synth.rng_uniform(8, 2, n)
    mk, _, ms = lib.run_instance(inst, precision=precision)
    b = ms.write_prn(**extras(inst))
    want = prn.pack_markers(dict(x=mk["x"], y=mk["y"], T=mk["T"], eta=mk["eta"], tmax=mk["tmax"], gr=inst.gr,
                                 acc=inst.acc), None, None, mk["type"])
    assert b == want
    ms.close()


def test_shim_section_matches_saver():
    """The C shim's i2g_shim_save_markers in the drop-in build writes the same
    section as the reference's saver() (oracle/ref_harness.c mode 2)."""
    inst = variants.prn_instance()
    r = refio.run_reference(inst, "dropin32", prn=True)
    assert r.shim_prn_markers == r.prn_markers
