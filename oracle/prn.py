"""TEST INFRASTRUCTURE ONLY: numpy restatement of the marker section of the
reference's binary output file, the checker for the library's device codec
(i2g_write_prn_markers / i2g_read_prn_markers).

saver() (loadmart.c:795-808) writes, for markers 0..marknum, nine 4-byte floats
(markx, marky, markk, markv, markhi, markpor, markgr, marktmax, markacc) and three
single bytes (markmg_old, markmg_time converted to char, markt), 39 bytes per
marker without padding.  loader() (loadmart.c:521-535) reads the nine floats
back, then stores the float it read last (markacc) in markmg_old (converted to
char) and in markmg_time, and the third byte in markt; the two magnetisation
bytes of the file are read and dropped.
"""
from __future__ import annotations

import numpy as np

RECORD = np.dtype([("f", "<f4", (9,)), ("b", "i1", (3,))])
assert RECORD.itemsize == 39
FLOATS = ("x", "y", "T", "eta", "hi", "por", "gr", "tmax", "acc")


def to_char(v) -> np.ndarray:
    """C's conversion of a floating value to char as x86-64 compilers emit it: the
    low byte of the 32-bit truncation (cvttss2si / cvttsd2si), whose result for
    NaN and values outside the int range is INT_MIN (low byte 0).  The C standard
    leaves out-of-range conversions undefined; this is what the reference builds do."""
    v = np.asarray(v, dtype=np.float64)
    ok = (v > -2147483649.0) & (v < 2147483648.0)
    i = np.where(ok, np.trunc(np.where(ok, v, 0.0)), -2147483648.0).astype(np.int64)
    return (i & 0xFF).astype(np.uint8).view(np.int8)


def pack_markers(fields: dict, mg_old, mg_time, mtype) -> bytes:
    """The saver() records of the given markers (float fields in FLOATS order)."""
    n = len(mtype)
    rec = np.zeros(n, dtype=RECORD)
    for k, name in enumerate(FLOATS):
        a = fields.get(name)
        rec["f"][:, k] = np.zeros(n, np.float32) if a is None else np.asarray(a).astype(np.float32)
    rec["b"][:, 0] = np.zeros(n, np.int8) if mg_old is None else np.asarray(mg_old, dtype=np.int8)
    rec["b"][:, 1] = np.zeros(n, np.int8) if mg_time is None else to_char(mg_time)
    rec["b"][:, 2] = np.asarray(mtype, dtype=np.int8)
    return rec.tobytes()


def unpack_markers(buf: bytes) -> dict:
    """The arrays loader() fills from saver() records (FP32 fields widened)."""
    rec = np.frombuffer(buf, dtype=RECORD)
    out = {name: rec["f"][:, k].astype(np.float64) for k, name in enumerate(FLOATS)}
    acc = rec["f"][:, 8]
    out["mg_old"] = to_char(acc)
    out["mg_time"] = acc.astype(np.float64)
    out["type"] = rec["b"][:, 2].copy()
    return out
