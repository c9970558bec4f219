"""ctypes binding of libi2g.so and a thin host-side mirror of the reference calls.

The reference drives the marker step as ``movemark()`` then ``ronurecalc()``
(i2mart.c:107, 146) over process globals.  :class:`MarkerStep` keeps that shape:
it owns one context, takes the reference's arrays (node layout ``m1*ynumy+m2``,
marker arrays in the reference's order) and exposes ``movemark(timestep)`` and
``ronurecalc(timesum)``.  Errors raise :class:`I2GError` carrying the ABI status
instead of the reference's printf()+exit().

The library is built in-tree (``i2elvis_planet_b200/libi2g.so``) and loading it
fails loudly if it is missing; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import abi
from .synth import GRID_FIELDS, NODE_OUT, Instance

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libi2g.so")

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_i8p = C.POINTER(C.c_int8)
_cp = C.c_void_p

# name -> (restype, argtypes); declarations of include/i2g.h
PROTOTYPES = {
    "i2g_strerror": (C.c_char_p, [C.c_int]),
    "i2g_last_error": (C.c_char_p, [_cp]),
    "i2g_abi_version": (C.c_int, []),
    "i2g_create": (C.c_int, [C.POINTER(_cp), C.POINTER(abi.Params), C.POINTER(abi.Types)]),
    "i2g_destroy": (C.c_int, [_cp]),
    "i2g_set_types": (C.c_int, [_cp, C.POINTER(abi.Types)]),
    "i2g_set_grid": (C.c_int, [_cp] + [_dp] * 13),
    "i2g_set_nodes": (C.c_int, [_cp] + [_dp] * 9),
    "i2g_get_nodes": (C.c_int, [_cp] + [_dp] * 9),
    "i2g_set_markers": (C.c_int, [_cp, C.c_int64, _dp, _dp, _dp, _dp, _i8p]),
    "i2g_set_marker_extras": (C.c_int, [_cp, _dp, _dp, _dp]),
    "i2g_get_markers": (C.c_int, [_cp, C.c_int64, _dp, _dp, _dp, _dp, _dp, _dp, _i8p]),
    "i2g_set_markers_dev": (C.c_int, [_cp, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "i2g_get_markers_dev": (C.c_int, [_cp, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "i2g_get_nodes_dev": (C.c_int, [_cp] + [C.c_void_p] * 9),
    "i2g_set_markers_f32": (C.c_int, [_cp, C.c_int64, _fp, _fp, _fp, _fp, C.c_char_p]),
    "i2g_get_markers_f32": (C.c_int, [_cp, C.c_int64, _fp, _fp, _fp, _fp, _fp]),
    "i2g_movemark": (C.c_int, [_cp, C.c_double, C.c_double, C.c_uint32]),
    "i2g_ronurecalc": (C.c_int, [_cp, C.c_double, C.c_uint32]),
    "i2g_step": (C.c_int, [_cp, C.c_double, C.c_double, C.c_int32, C.c_uint32, C.c_uint32]),
    "i2g_set_reorder_interval": (C.c_int, [_cp, C.c_int32]),
    "i2g_set_fused": (C.c_int, [_cp, C.c_int]),
    "i2g_fused_info": (C.c_int, [_cp, C.POINTER(abi.FusedStats)]),
    "i2g_set_td_table": (C.c_int, [_cp, C.POINTER(abi.TdTable)]),
    "i2g_set_timestep": (C.c_int, [_cp, C.c_double]),
    "i2g_get_marker_extras": (C.c_int, [_cp, C.c_int64, _dp, _dp, _dp]),
    "i2g_set_marker_mag": (C.c_int, [_cp, _i8p, _dp]),
    "i2g_get_marker_mag": (C.c_int, [_cp, C.c_int64, _i8p, _dp]),
    "i2g_write_prn_markers": (C.c_int, [_cp, C.c_int64, _fp, _fp, C.c_char_p, _dp, C.c_void_p]),
    "i2g_read_prn_markers": (C.c_int, [_cp, C.c_int64, C.c_void_p, _fp, _fp, C.c_void_p, _dp]),
    "i2g_set_melt_state": (C.c_int, [_cp, _dp]),
    "i2g_get_melt_state": (C.c_int, [_cp, _dp]),
    "i2g_interp_tnode": (C.c_int, [_cp, _dp, _dp, _dp, _dp]),
    "i2g_titerate_markers": (C.c_int, [_cp, _dp, _dp, _dp, _dp, _dp, C.c_double, C.c_double]),
    "i2g_titerate_markers_dev": (C.c_int, [_cp, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.c_double, C.c_double]),
    "i2g_stream": (C.c_void_p, [_cp]),
    "i2g_set_stream": (C.c_int, [_cp, C.c_void_p]),
    "i2g_sync": (C.c_int, [_cp]),
    "i2g_get_stats": (C.c_int, [_cp, C.POINTER(abi.Stats)]),
    "i2g_profile_enable": (C.c_int, [_cp, C.c_int]),
    "i2g_profile_read": (C.c_int, [_cp, C.POINTER(abi.Profile), C.c_int]),
    "i2g_adjoint_setup": (C.c_int, [_cp, C.c_int32, _dp, _dp]),
    "i2g_adjoint_forward": (C.c_int, [_cp, _dp, C.c_int32, C.c_double, C.c_double, C.c_int32, _dp]),
    "i2g_adjoint_backward": (C.c_int, [_cp, _dp, _dp, _dp]),
    "i2g_batch_create": (C.c_int, [C.POINTER(_cp), C.POINTER(_cp), C.c_int32]),
    "i2g_batch_destroy": (C.c_int, [_cp]),
    "i2g_batch_step": (C.c_int, [_cp, _dp, _dp, C.c_int32, C.c_uint32]),
    "i2g_batch_autotune": (C.c_int, [_cp, _dp, _dp, C.c_int32, C.POINTER(abi.Tune)]),
    "i2g_batch_set_tune": (C.c_int, [_cp, C.POINTER(abi.Tune)]),
    "i2g_batch_set_graphs": (C.c_int, [_cp, C.c_int]),
    "i2g_batch_stream": (C.c_void_p, [_cp]),
    "i2g_batch_sync": (C.c_int, [_cp]),
    "i2g_static_max_markers": (C.c_int64, []),
    "i2g_static_max_lines": (C.c_int64, []),
    # all array arguments are device addresses
    "i2g_ronurecalc_static": (C.c_int, [C.POINTER(abi.Params), C.POINTER(abi.Types)] + [_cp] * 11 +
                              [C.c_int64] + [_cp] * 5 + [C.c_double] + [_cp] * 9 + [_cp]),
}

_lib = None


class I2GError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str = ""):
        self.status = status
        super().__init__(f"{where}: {abi.STATUS_NAMES.get(status, status)} ({msg})")


def load(path: str = LIB_PATH):
    """Load libi2g.so (build it first with i2elvis_planet_b200.build)."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} not built: run `python -m i2elvis_planet_b200.build`")
        L = C.CDLL(path)
        for name, (res, args) in PROTOTYPES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _d(a):
    return abi.dptr(a) if a is not None else None


class MarkerStep:
    """One planetesimal instance on the GPU: the reference's movemark()/ronurecalc() pair."""

    def __init__(self, params: abi.Params, types: abi.Types):
        self.lib = load()
        self.params = params
        self.types = types
        h = C.c_void_p()
        self._check(self.lib.i2g_create(C.byref(h), C.byref(params), C.byref(types)), "i2g_create", None)
        self.h = h
        self.n = 0
        self.nodenum = params.xnumx * params.ynumy

    @classmethod
    def from_instance(cls, inst: Instance, precision: int = abi.PREC_FP64, device: int = 0,
                      max_markers: int | None = None, upload: bool = True) -> "MarkerStep":
        ms = cls(abi.params_from_instance(inst, precision=precision, device=device, max_markers=max_markers),
                 abi.types_from_instance(inst))
        if inst.td is not None:
            ms.set_td_table(inst.td)
        if upload:
            ms.set_grid(inst.gx, inst.gy, **inst.grid)
            ms.set_nodes(**inst.nodes)
            ms.set_markers(inst.x, inst.y, inst.T, inst.eta, inst.mtype)
        return ms

    # -- error handling
    def _check(self, rc: int, where: str, h=...):
        if rc != 0:
            hh = self.h if h is ... else h
            msg = self.lib.i2g_last_error(hh).decode() if hh else ""
            raise I2GError(rc, where, msg)

    def close(self):
        if getattr(self, "h", None):
            self.lib.i2g_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- state transfer (host arrays, caller order)
    def set_grid(self, gx, gy, **fields):
        keep = {k: (np.ascontiguousarray(fields[k], dtype=np.float64) if fields.get(k) is not None else None)
                for k in GRID_FIELDS}
        gx = np.ascontiguousarray(gx, dtype=np.float64)
        gy = np.ascontiguousarray(gy, dtype=np.float64)
        self._check(self.lib.i2g_set_grid(self.h, _d(gx), _d(gy), *[_d(keep[k]) for k in GRID_FIELDS]),
                    "i2g_set_grid")

    def set_nodes(self, **fields):
        keep = {k: (np.ascontiguousarray(fields[k], dtype=np.float64) if fields.get(k) is not None else None)
                for k in NODE_OUT}
        self._check(self.lib.i2g_set_nodes(self.h, *[_d(keep[k]) for k in NODE_OUT]), "i2g_set_nodes")

    def get_nodes(self) -> dict:
        out = {k: np.empty(self.nodenum) for k in NODE_OUT}
        self._check(self.lib.i2g_get_nodes(self.h, *[_d(out[k]) for k in NODE_OUT]), "i2g_get_nodes")
        return out

    def set_markers(self, x, y, T, eta, mtype):
        x, y, T, eta = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, T, eta))
        mtype = np.ascontiguousarray(mtype, dtype=np.int8)
        self._check(self.lib.i2g_set_markers(self.h, x.size, _d(x), _d(y), _d(T), _d(eta), abi.i8ptr(mtype)),
                    "i2g_set_markers")
        self.n = x.size

    def set_marker_extras(self, tmax=None, hi=None, por=None):
        a = [np.ascontiguousarray(v, dtype=np.float64) if v is not None else None for v in (tmax, hi, por)]
        self._check(self.lib.i2g_set_marker_extras(self.h, *[_d(v) for v in a]), "i2g_set_marker_extras")

    def get_markers(self, fields=("x", "y", "T", "eta", "p"), with_tmax: bool = False) -> dict:
        out = {k: np.empty(self.n) for k in fields}
        tmax = np.empty(self.n) if with_tmax else None
        mt = np.empty(self.n, dtype=np.int8) if "type" in fields else None
        self._check(self.lib.i2g_get_markers(self.h, self.n, *[_d(out.get(k)) for k in ("x", "y", "T", "eta", "p")],
                                             _d(tmax), abi.i8ptr(mt) if mt is not None else None),
                    "i2g_get_markers")
        if with_tmax:
            out["tmax"] = tmax
        if mt is not None:
            out["type"] = mt
        return out

    # -- the two reference calls
    def movemark(self, timestep: float, timesum: float = 0.0, update_visc: bool = False):
        """movemark() (markmart.c:3-188)."""
        self._check(self.lib.i2g_movemark(self.h, timestep, timesum, abi.MOVE_UPDATE_VISC if update_visc else 0),
                    "i2g_movemark")

    def ronurecalc(self, timesum: float, track_tmax: bool = False):
        """ronurecalc() without its closing tkrecalc() (markmart.c:192-1009)."""
        self._check(self.lib.i2g_ronurecalc(self.h, timesum, abi.AVG_TRACK_TMAX if track_tmax else 0),
                    "i2g_ronurecalc")

    def step(self, timestep: float, timesum: float, nsteps: int, update_visc: bool = False,
             track_tmax: bool = False):
        self._check(self.lib.i2g_step(self.h, timestep, timesum, nsteps,
                                      abi.MOVE_UPDATE_VISC if update_visc else 0,
                                      abi.AVG_TRACK_TMAX if track_tmax else 0), "i2g_step")

    def set_reorder_interval(self, every: int):
        """Averaging calls between moves of the marker records into cell order."""
        self._check(self.lib.i2g_set_reorder_interval(self.h, int(every)), "i2g_set_reorder_interval")

    def set_td_table(self, td: dict):
        """densimod 2: the P-T table (a synth.td_table dict, the reference's td layout)."""
        t, arr = abi.td_table_from_dict(td)
        self._check(self.lib.i2g_set_td_table(self.h, C.byref(t)), "i2g_set_td_table")
        del arr

    def set_marker_mag(self, mg_old, mg_time):
        """Magnetisation state and time (markmg_old, markmg_time): produced from now on."""
        a = np.ascontiguousarray(mg_old, dtype=np.int8)
        b = np.ascontiguousarray(mg_time, dtype=np.float64)
        self._check(self.lib.i2g_set_marker_mag(self.h, abi.i8ptr(a), abi.dptr(b)), "i2g_set_marker_mag")

    def get_marker_mag(self):
        a = np.empty(self.n, dtype=np.int8)
        b = np.empty(self.n)
        self._check(self.lib.i2g_get_marker_mag(self.h, self.n, abi.i8ptr(a), abi.dptr(b)), "i2g_get_marker_mag")
        return a, b

    def get_por(self) -> np.ndarray:
        out = np.empty(self.n)
        self._check(self.lib.i2g_get_marker_extras(self.h, self.n, None, None, abi.dptr(out)), "i2g_get_marker_extras")
        return out

    def set_timestep(self, timestep: float):
        """The global timestep the next ronurecalc's porosity sintering reads."""
        self._check(self.lib.i2g_set_timestep(self.h, timestep), "i2g_set_timestep")

    def set_melt_state(self, eps6):
        """eps[21], eps[22], eps[50], eps[51], eps[52], eps[53] (the melt state meltpart1 leaves)."""
        a = np.ascontiguousarray(eps6, dtype=np.float64)
        assert a.size == 6
        self._check(self.lib.i2g_set_melt_state(self.h, abi.dptr(a)), "i2g_set_melt_state")

    def get_melt_state(self) -> np.ndarray:
        a = np.empty(6)
        self._check(self.lib.i2g_get_melt_state(self.h, abi.dptr(a)), "i2g_get_melt_state")
        return a

    # -- the marker section of the reference's binary output file
    def write_prn(self, gr=None, acc=None, mg_old=None, mg_time=None, out: np.ndarray | None = None):
        """saver()'s marker records (loadmart.c:795-808) of markers 0..n-1: bytes, or
        written into ``out`` (a uint8 array of 39 n bytes, e.g. pinned) and returned."""
        n = self.n
        f32 = [np.ascontiguousarray(a, dtype=np.float32) if a is not None else None for a in (gr, acc)]
        mgo = np.ascontiguousarray(mg_old, dtype=np.int8) if mg_old is not None else None
        mgt = np.ascontiguousarray(mg_time, dtype=np.float64) if mg_time is not None else None
        given = out is not None
        if not given:
            out = np.empty(abi.PRN_RECORD_BYTES * n, dtype=np.uint8)
        assert out.dtype == np.uint8 and out.size == abi.PRN_RECORD_BYTES * n and out.flags.c_contiguous
        fp = [a.ctypes.data_as(C.POINTER(C.c_float)) if a is not None else None for a in f32]
        self._check(self.lib.i2g_write_prn_markers(self.h, n, fp[0], fp[1],
                                                   mgo.ctypes.data_as(C.c_char_p) if mgo is not None else None,
                                                   _d(mgt), out.ctypes.data_as(C.c_void_p)),
                    "i2g_write_prn_markers")
        return out if given else out.tobytes()

    def read_prn(self, data: bytes) -> dict:
        """loader() (loadmart.c:521-535) of n records into this context; returns the
        fields the library does not keep (gr, acc, mg_old, mg_time) as loader() sets them."""
        buf = data if isinstance(data, np.ndarray) else np.frombuffer(data, dtype=np.uint8)
        n = buf.size // abi.PRN_RECORD_BYTES
        assert n * abi.PRN_RECORD_BYTES == buf.size and buf.dtype == np.uint8
        gr, acc = np.empty(n, np.float32), np.empty(n, np.float32)
        mgo, mgt = np.empty(n, np.int8), np.empty(n)
        self._check(self.lib.i2g_read_prn_markers(self.h, n, buf.ctypes.data_as(C.c_void_p),
                                                  gr.ctypes.data_as(C.POINTER(C.c_float)),
                                                  acc.ctypes.data_as(C.POINTER(C.c_float)),
                                                  mgo.ctypes.data_as(C.c_void_p), _d(mgt)),
                    "i2g_read_prn_markers")
        self.n = n
        return dict(gr=gr, acc=acc, mg_old=mgo, mg_time=mgt)

    def set_fused(self, enable: bool):
        """The mixed form's fused movemark + averaging (on by default)."""
        self._check(self.lib.i2g_set_fused(self.h, int(bool(enable))), "i2g_set_fused")

    def fused_info(self) -> dict:
        f = abi.FusedStats()
        self._check(self.lib.i2g_fused_info(self.h, C.byref(f)), "i2g_fused_info")
        return {k: int(getattr(f, k)) for k, _ in abi.FusedStats._fields_}

    def interp_tnode(self, tk, tk2=None):
        """allintert() (markmart.c:1687-1745) at every marker: the node temperature
        tk (and tk2) interpolated at the marker's position, in the caller's order."""
        tk = np.ascontiguousarray(tk, dtype=np.float64)
        t2 = None if tk2 is None else np.ascontiguousarray(tk2, dtype=np.float64)
        for a in (tk, t2):
            if a is not None and a.size != self.nodenum:
                raise ValueError("node arrays need xnumx * ynumy values")
        n = self.n
        out = np.empty(n)
        out2 = None if t2 is None else np.empty(n)
        self._check(self.lib.i2g_interp_tnode(self.h, _d(tk), _d(t2), _d(out), _d(out2)), "i2g_interp_tnode")
        return out, out2

    def titerate_markers(self, tk_new, tk_old, heatdif: float, timestep: float, kt=None, cp=None, ro=None):
        """titerate()'s marker temperature update (heatmart.c:514-697) after the
        caller's thermal solve: node T after (tk_new) and before (tk_old) it; kt, cp,
        ro replace the context's node fields when given."""
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (tk_new, tk_old, kt, cp, ro)]
        for a in arrs:
            if a is not None and a.size != self.nodenum:
                raise ValueError("node arrays need xnumx * ynumy values")
        self._check(self.lib.i2g_titerate_markers(self.h, *[_d(a) for a in arrs], float(heatdif), float(timestep)),
                    "i2g_titerate_markers")

    def titerate_markers_dev(self, tk_new, tk_old, heatdif: float, timestep: float, kt=None, cp=None, ro=None):
        """The same from device tensors (torch, float64, contiguous, on this context's
        device), read in place on the context's stream."""
        ptrs = []
        for a in (tk_new, tk_old, kt, cp, ro):
            if a is None:
                ptrs.append(None)
                continue
            if not (a.is_cuda and a.dtype.is_floating_point and a.element_size() == 8 and a.is_contiguous()
                    and a.numel() == self.nodenum):
                raise ValueError("device node arrays: contiguous float64 CUDA tensors of xnumx * ynumy values")
            ptrs.append(C.c_void_p(a.data_ptr()))
        self._check(self.lib.i2g_titerate_markers_dev(self.h, *ptrs, float(heatdif), float(timestep)),
                    "i2g_titerate_markers_dev")

    def sync(self):
        self._check(self.lib.i2g_sync(self.h), "i2g_sync")

    def stream(self) -> int:
        return int(self.lib.i2g_stream(self.h) or 0)

    def profile_enable(self, on: bool = True):
        self._check(self.lib.i2g_profile_enable(self.h, int(on)), "i2g_profile_enable")

    def profile_read(self, reset: bool = False) -> dict:
        p = abi.Profile()
        self._check(self.lib.i2g_profile_read(self.h, C.byref(p), int(reset)), "i2g_profile_read")
        return {"ms": dict(zip(abi.PHASES, list(p.ms))), "calls": dict(zip(abi.PHASES, list(p.calls))),
                "launches": int(p.launches)}

    # -- adjoint (gradients w.r.t. initial marker temperatures and mode amplitudes)
    def adjoint_setup(self, mode_vx: np.ndarray, mode_vy: np.ndarray):
        mvx = np.ascontiguousarray(mode_vx, dtype=np.float64)
        mvy = np.ascontiguousarray(mode_vy, dtype=np.float64)
        self.nmodes = mvx.shape[0]
        self._check(self.lib.i2g_adjoint_setup(self.h, self.nmodes, _d(mvx), _d(mvy)), "i2g_adjoint_setup")

    def adjoint_forward(self, amps, nsteps: int, timestep: float, timesum: float, ckpt_every: int = 5) -> np.ndarray:
        a = np.ascontiguousarray(amps, dtype=np.float64)
        tk = np.empty(self.nodenum)
        self._check(self.lib.i2g_adjoint_forward(self.h, _d(a), nsteps, timestep, timesum, ckpt_every, _d(tk)),
                    "i2g_adjoint_forward")
        return tk

    def adjoint_backward(self, dL_dtk: np.ndarray):
        g = np.ascontiguousarray(dL_dtk, dtype=np.float64)
        dT = np.empty(self.n)
        da = np.empty(self.nmodes)
        self._check(self.lib.i2g_adjoint_backward(self.h, _d(g), _d(dT), _d(da)), "i2g_adjoint_backward")
        return dT, da

    def stats(self) -> abi.Stats:
        s = abi.Stats()
        self._check(self.lib.i2g_get_stats(self.h, C.byref(s)), "i2g_get_stats")
        return s


class Batch:
    """Many instances stepped together (i2g_batch_*): fused (one launch per phase
    over all instances, each step replayed from a CUDA graph) or streams (every
    instance's own step on its own stream, side by side)."""

    def __init__(self, steps: list):
        self.lib = load()
        self.steps = steps  # MarkerStep objects (kept alive by the batch)
        arr = (C.c_void_p * len(steps))(*[m.h.value for m in steps])
        h = C.c_void_p()
        rc = self.lib.i2g_batch_create(C.byref(h), arr, len(steps))
        if rc:
            raise I2GError(rc, "i2g_batch_create")
        self.h = h

    def step(self, timestep: np.ndarray, timesum: np.ndarray, nsteps: int, track_tmax: bool = False):
        """Advance every instance nsteps; timesum (float64 array) is updated in place."""
        dt = np.ascontiguousarray(timestep, dtype=np.float64)
        assert timesum.dtype == np.float64 and timesum.flags.c_contiguous
        rc = self.lib.i2g_batch_step(self.h, abi.dptr(dt), abi.dptr(timesum), nsteps,
                                     abi.AVG_TRACK_TMAX if track_tmax else 0)
        if rc:
            raise I2GError(rc, "i2g_batch_step")

    def autotune(self, timestep: np.ndarray, timesum: np.ndarray, steps_per_candidate: int = 2) -> dict:
        dt = np.ascontiguousarray(timestep, dtype=np.float64)
        t = abi.Tune()
        rc = self.lib.i2g_batch_autotune(self.h, abi.dptr(dt), abi.dptr(timesum), steps_per_candidate, C.byref(t))
        if rc:
            raise I2GError(rc, "i2g_batch_autotune")
        return {"tile_cols": t.tile_cols, "move_ctas_per_sm": t.move_ctas_per_sm,
                "avg_ctas_per_sm": t.avg_ctas_per_sm, "ms_per_step": t.ms_per_step, "candidates": t.candidates,
                "strategy": "streams" if t.strategy == abi.BATCH_STREAMS else "fused"}

    def set_tune(self, tile_cols: int = 16, move_ctas_per_sm: int = 8, avg_ctas_per_sm: int = 2,
                 strategy: int = abi.BATCH_FUSED):
        t = abi.Tune(tile_cols, move_ctas_per_sm, avg_ctas_per_sm, 0.0, 0, strategy)
        rc = self.lib.i2g_batch_set_tune(self.h, C.byref(t))
        if rc:
            raise I2GError(rc, "i2g_batch_set_tune")

    def set_graphs(self, enable: bool):
        """Replay the streams strategy's steps from a CUDA graph where it can (default on)."""
        rc = self.lib.i2g_batch_set_graphs(self.h, 1 if enable else 0)
        if rc:
            raise I2GError(rc, "i2g_batch_set_graphs")

    def stream(self) -> int:
        return int(self.lib.i2g_batch_stream(self.h) or 0)

    def sync(self):
        rc = self.lib.i2g_batch_sync(self.h)
        if rc:
            raise I2GError(rc, "i2g_batch_sync")

    def close(self):
        if getattr(self, "h", None):
            self.lib.i2g_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run_instance(inst: Instance, precision: int = abi.PREC_FP64, nsteps: int | None = None,
                 eta_reinject: bool = True, update_visc: bool = False, track_tmax: bool = True):
    """The harness loop on the GPU: nsteps x {movemark; ronurecalc; timesum += dt}.

    With ``eta_reinject`` the per-marker viscosity is left as set (the reference
    harness re-writes it after each movemark); ``update_visc`` stores movemark's
    viscalc() result instead.  Returns (markers dict, nodes dict, MarkerStep)."""
    ms = MarkerStep.from_instance(inst, precision=precision)
    por = inst.por if np.any(inst.por) else None
    if track_tmax or np.any(inst.hi) or por is not None:
        ms.set_marker_extras(tmax=inst.tmax if track_tmax else None, hi=inst.hi if np.any(inst.hi) else None,
                             por=por)
    if inst.mg_old is not None:
        ms.set_marker_mag(inst.mg_old, inst.mg_time)
    timesum = inst.timesum
    for _ in range(inst.nsteps if nsteps is None else nsteps):
        ms.movemark(inst.timestep, timesum, update_visc=update_visc)
        ms.ronurecalc(timesum, track_tmax=track_tmax)
        timesum += inst.timestep
    mk = ms.get_markers(fields=("x", "y", "T", "eta", "p", "type"), with_tmax=track_tmax)
    if por is not None:
        mk["por"] = ms.get_por()
    if inst.mg_old is not None:
        mk["mg_old"], mk["mg_time"] = ms.get_marker_mag()
    return mk, ms.get_nodes(), ms
