"""ctypes mirror of include/i2g.h (struct layouts and constants)."""
from __future__ import annotations

import ctypes as C

import numpy as np

ABI_VERSION = 1
MAXTYPES = 200

OK, EINVAL, ECAPACITY, ECUDA, ETIMEOUT, EUNSUPPORTED, ENOMEM, ESTATE = range(8)
STATUS_NAMES = {0: "I2G_OK", 1: "I2G_EINVAL", 2: "I2G_ECAPACITY", 3: "I2G_ECUDA", 4: "I2G_ETIMEOUT",
                5: "I2G_EUNSUPPORTED", 6: "I2G_ENOMEM", 7: "I2G_ESTATE"}

PREC_FP64 = 0
PREC_MIXED = 1
MOVE_UPDATE_VISC = 0x1
AVG_TRACK_TMAX = 0x1

_TYPE_FIELDS = ("marknu", "markdh", "markdv", "markss", "markmm", "markll", "marka0", "marka1",
                "markb0", "markb1", "marke0", "marke1", "markro", "markaa", "markbb", "markcp",
                "markkt", "markht", "markkf", "markkp", "markn0", "markn1", "marks0", "marks1")


class Types(C.Structure):
    _fields_ = [(f, C.c_double * MAXTYPES) for f in _TYPE_FIELDS] + [("markim", C.c_int32 * MAXTYPES)]


class Params(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int32), ("precision", C.c_int32),
        ("xnumx", C.c_int64), ("ynumy", C.c_int64), ("max_markers", C.c_int64),
        ("xsize", C.c_double), ("ysize", C.c_double),
        ("markmod", C.c_int32), ("outgrid", C.c_int32), ("intermod", C.c_int32), ("intermod1", C.c_int32),
        ("gridmod", C.c_int32), ("densimod", C.c_int32), ("viscmod", C.c_int32), ("dynamo", C.c_int32),
        ("nubeg", C.c_double), ("nuend", C.c_double), ("nucontr", C.c_double),
        ("tmp_ambient", C.c_double), ("M_init", C.c_double), ("M_acc", C.c_double),
        ("core_form_time", C.c_double), ("k_cutoff", C.c_double),
        ("al2627_init", C.c_double), ("fe6056_init", C.c_double), ("relax_time", C.c_double),
        ("por_init", C.c_double),
        ("xmelt_si", C.c_double), ("xmelt_fe", C.c_double), ("xmelt_ice", C.c_double),
        ("device", C.c_int32), ("reserved", C.c_int32 * 7),
    ]


class TdTable(C.Structure):
    """i2g_td_table: the densimod 2 P-T table (the reference's td[][][][] layout)."""
    _fields_ = [("td", C.POINTER(C.c_double)), ("tkdim", C.c_int32), ("pbdim", C.c_int32),
                ("tknum", C.c_int32), ("pbnum", C.c_int32),
                ("tkmin", C.c_double), ("pbmin", C.c_double), ("tkstp", C.c_double), ("pbstp", C.c_double),
                ("si_melting", C.c_int32), ("fe_melting", C.c_int32), ("ice_melting", C.c_int32),
                ("reserved", C.c_int32)]


def td_table_from_dict(td: dict):
    """(TdTable, the array it points at) for a synth.td_table dict; keep both alive."""
    arr = np.ascontiguousarray(td["td"], dtype=np.float64)
    assert arr.ndim == 4 and arr.shape[2:] == (2, 5)
    t = TdTable()
    t.td = arr.ctypes.data_as(C.POINTER(C.c_double))
    t.tkdim, t.pbdim = arr.shape[0], arr.shape[1]
    t.tknum, t.pbnum = int(td["tknum"]), int(td["pbnum"])
    t.tkmin, t.pbmin, t.tkstp, t.pbstp = (float(td[k]) for k in ("tkmin", "pbmin", "tkstp", "pbstp"))
    t.si_melting, t.fe_melting, t.ice_melting = (int(td[k]) for k in ("si_melting", "fe_melting", "ice_melting"))
    return t, arr


def melt_state_from_instance(inst) -> np.ndarray:
    """eps[21], eps[22], eps[50], eps[51], eps[52], eps[53] at the start of a run."""
    s = inst.scal
    return np.array([s["eps21"], 0.0, s["eps50"], 0.0, s["eps52"], 0.0])


class Stats(C.Structure):
    _fields_ = [("numin", C.c_double), ("numax", C.c_double), ("marknum", C.c_int64),
                ("nodenum", C.c_int64), ("markers_averaged", C.c_int64), ("sorts", C.c_int64)]


PHASES = ("movemark", "cell_sort", "contrib", "cell_sums", "node_loop")


class Tune(C.Structure):
    _fields_ = [("tile_cols", C.c_int32), ("move_ctas_per_sm", C.c_int32), ("avg_ctas_per_sm", C.c_int32),
                ("ms_per_step", C.c_double), ("candidates", C.c_int32), ("strategy", C.c_int32)]


BATCH_FUSED, BATCH_STREAMS = 0, 1
PRN_RECORD_BYTES = 39  # I2G_PRN_RECORD_BYTES


class FusedStats(C.Structure):
    _fields_ = [("enabled", C.c_int32), ("bucket_places", C.c_int32), ("type_slots", C.c_int32),
                ("uniform_grid", C.c_int32), ("fused_moves", C.c_int64), ("bucket_growths", C.c_int64)]


class Profile(C.Structure):
    _fields_ = [("ms", C.c_double * len(PHASES)), ("calls", C.c_int64 * len(PHASES)), ("launches", C.c_int64)]


def params_from_instance(inst, precision: int = PREC_FP64, max_markers: int | None = None,
                         device: int = 0) -> Params:
    p = Params()
    p.abi_version = ABI_VERSION
    p.precision = precision
    p.xnumx, p.ynumy = inst.xnumx, inst.ynumy
    p.max_markers = inst.marknum if max_markers is None else max_markers
    p.xsize, p.ysize = inst.xsize, inst.ysize
    for k in ("markmod", "outgrid", "intermod", "intermod1", "gridmod", "densimod", "viscmod", "dynamo"):
        setattr(p, k, int(inst.flags[k]))
    s = inst.scal
    for k in ("nubeg", "nuend", "nucontr", "tmp_ambient", "M_init", "M_acc", "core_form_time", "k_cutoff",
              "al2627_init", "fe6056_init", "relax_time", "por_init"):
        setattr(p, k, float(s[k]))
    p.xmelt_si, p.xmelt_fe, p.xmelt_ice = s["eps21"], s["eps50"], s["eps52"]
    p.device = device
    return p


def types_from_instance(inst) -> Types:
    t = Types()
    for k in _TYPE_FIELDS:
        getattr(t, k)[:] = np.asarray(inst.types[k], dtype=np.float64).tolist()
    t.markim[:] = [int(v) for v in inst.markim]
    return t


def dptr(a: np.ndarray | None):
    """double* of a contiguous float64 array (or NULL)."""
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


def i8ptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.int8 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_int8))
