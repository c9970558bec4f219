"""The marker section of the reference's binary output file (saver()/loader(),
loadmart.c:521-535, 795-808): the numpy restatement in oracle/prn.py is pinned to
the compiled reference (tests/golden/prn_ref32.npz, made by make_golden.py from
saver() writing the file and loader() reading it back), so that it can check the
library's device codec (tests/test_gpu_prn.py)."""
import hashlib
import os

import numpy as np

import variants
from oracle import prn

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def golden():
    return np.load(os.path.join(GOLD, "prn_ref32.npz"))


def section(inst):
    f = dict(x=inst.x, y=inst.y, T=inst.T, eta=inst.eta, hi=inst.hi, por=inst.por, gr=inst.gr, tmax=inst.tmax,
             acc=inst.acc)
    # saver() writes markers 0..marknum: the record past the last marker holds the
    # arrays' zero-initialised entries
    return prn.pack_markers(f, inst.mg_old, inst.mg_time, inst.mtype) + bytes(prn.RECORD.itemsize)


def test_writer_matches_saver():
    inst = variants.prn_instance()
    g = golden()
    b = section(inst)
    assert len(b) == int(g["section_bytes"])
    assert digest(np.frombuffer(b, np.uint8)) == str(g["section_digest"])


def test_reader_matches_loader():
    inst = variants.prn_instance()
    g = golden()
    u = prn.unpack_markers(section(inst)[:-prn.RECORD.itemsize])
    for k in ("x", "y", "T", "eta", "por", "tmax", "gr", "acc", "mg_time", "mg_old"):
        assert digest(u[k]) == str(g[f"digest_{k}"]), k
    assert digest(u["type"]) == str(g["digest_mtype"])


def test_char_conversion_edges():
    v = np.array([0.0, -0.9, 127.9, 128.0, 255.0, 256.0, -129.0, 3e9, -3e9, np.nan, np.inf, -1.0])
    np.testing.assert_array_equal(prn.to_char(v), np.array([0, 0, 127, -128, -1, 0, 127, 0, 0, 0, 0, -1], np.int8))
