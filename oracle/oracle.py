"""TEST INFRASTRUCTURE ONLY: ctypes binding of the oracle (oracle/liboracle.so).

The oracle restates movemark()/ronurecalc() and titerate()'s marker temperature
update sequentially in C (oracle/i2g_oracle.c).
Only tests, the smoke check and the bench's CPU-baseline legs may use it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

from i2elvis_planet_b200 import abi
from i2elvis_planet_b200.synth import NODE_OUT, Instance

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
ORDER_REFERENCE = 0
ORDER_CELL = 1


class Grid(C.Structure):
    _fields_ = [("xnumx", C.c_int64), ("ynumy", C.c_int64)] + [
        (k, C.POINTER(C.c_double)) for k in
        ("gx", "gy", "vx", "vy", "pr", "exx", "eyy", "exy", "sxx", "syy", "sxy", "ga", "mu")]


class Nodes(C.Structure):
    _fields_ = [(k, C.POINTER(C.c_double)) for k in NODE_OUT]


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        P = C.POINTER
        dp = P(C.c_double)
        L.ora_m1serch.restype = C.c_int64
        L.ora_m1serch.argtypes = [dp, C.c_int64, C.c_double]
        L.ora_fdweight1.argtypes = [C.c_double, C.c_double, C.c_double, dp, dp]
        L.ora_allinterv.argtypes = [P(abi.Params), P(Grid), C.c_double, C.c_double, dp, dp]
        L.ora_allintere.argtypes = [P(abi.Params), P(Grid), C.c_double, C.c_double, dp, P(C.c_int64)]
        L.ora_cell_key.restype = C.c_int64
        L.ora_cell_key.argtypes = [P(abi.Params), P(Grid), C.c_double, C.c_double]
        L.ora_radiogenic.restype = C.c_double
        L.ora_radiogenic.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double]
        L.ora_movemark.restype = C.c_int
        L.ora_movemark.argtypes = [P(abi.Params), P(abi.Types), P(Grid), C.c_int64, dp, dp, dp, dp, dp,
                                   P(C.c_int8), dp, C.c_double, C.c_double, C.c_uint32]
        L.ora_ronurecalc.restype = C.c_int
        L.ora_ronurecalc.argtypes = [P(abi.Params), P(abi.Types), P(Grid), C.c_int64, dp, dp, dp, dp,
                                     P(C.c_int8), dp, dp, dp, C.c_double, C.c_uint32, C.c_int,
                                     P(abi.TdTable), dp, P(SinterArgs), P(Nodes), dp]
        L.ora_interp_tnode.restype = None
        L.ora_interp_tnode.argtypes = [P(abi.Params), P(Grid), C.c_int64, dp, dp, dp, dp, dp, dp]
        L.ora_titerate_markers.restype = C.c_int
        L.ora_titerate_markers.argtypes = [P(abi.Params), P(Grid), C.c_int64, dp, dp, dp, P(C.c_int8), dp, dp,
                                           dp, dp, dp, C.c_double, C.c_double, C.c_int]
        _lib = L
    return _lib


class SinterArgs(C.Structure):
    """ora_sinter_args: the timestep the sintering reads, FP32 porosity storage, gave-up
    flag; markmg_old, markmg_time and the carried magnetisation time."""
    _fields_ = [("timestep", C.c_double), ("f32", C.c_int), ("stuck", C.c_int),
                ("mg_old", C.POINTER(C.c_int8)), ("mg_time", C.POINTER(C.c_double)), ("mag_time", C.c_double)]


@dataclass
class State:
    """Marker and node state the oracle evolves (caller marker order)."""
    x: np.ndarray
    y: np.ndarray
    T: np.ndarray
    eta: np.ndarray
    p: np.ndarray
    mtype: np.ndarray
    tmax: np.ndarray
    nodes: dict
    numin: float = 0.0
    numax: float = 0.0
    melt: np.ndarray | None = None  # eps[21], eps[22], eps[50], eps[51], eps[52], eps[53]
    por: np.ndarray | None = None
    mg_old: np.ndarray | None = None   # markmg_old
    mg_time: np.ndarray | None = None  # markmg_time
    mag_time: float = -1.0             # ronurecalc()'s carried magnetisation time


class Oracle:
    def __init__(self, inst: Instance):
        self.inst = inst
        self.P = abi.params_from_instance(inst)
        self.T = abi.types_from_instance(inst)
        self._keep = {k: np.ascontiguousarray(v, dtype=np.float64) for k, v in inst.grid.items()}
        self._hi = np.ascontiguousarray(inst.hi, dtype=np.float64)
        self._gx = np.ascontiguousarray(inst.gx, dtype=np.float64)
        self._gy = np.ascontiguousarray(inst.gy, dtype=np.float64)
        self.td = abi.td_table_from_dict(inst.td) if inst.td is not None else None
        self.G = Grid(inst.xnumx, inst.ynumy, abi.dptr(self._gx), abi.dptr(self._gy),
                      *[abi.dptr(self._keep[k]) for k in
                        ("vx", "vy", "pr", "exx", "eyy", "exy", "sxx", "syy", "sxy", "ga", "mu")])

    def set_velocity(self, vx: np.ndarray, vy: np.ndarray) -> None:
        self._keep["vx"] = np.ascontiguousarray(vx, dtype=np.float64)
        self._keep["vy"] = np.ascontiguousarray(vy, dtype=np.float64)
        self.G.vx = abi.dptr(self._keep["vx"])
        self.G.vy = abi.dptr(self._keep["vy"])

    def initial_state(self) -> State:
        i = self.inst
        return State(x=i.x.copy(), y=i.y.copy(), T=i.T.copy(), eta=i.eta.copy(), p=np.zeros(i.marknum),
                     mtype=i.mtype.copy(), tmax=i.tmax.copy(), nodes={k: v.copy() for k, v in i.nodes.items()},
                     melt=abi.melt_state_from_instance(i), por=np.ascontiguousarray(i.por, dtype=np.float64).copy(),
                     mg_old=(np.full(i.marknum, 3, np.int8) if i.mg_old is None else
                             np.ascontiguousarray(i.mg_old, dtype=np.int8).copy()),
                     mg_time=(np.full(i.marknum, -1.0) if i.mg_time is None else
                              np.ascontiguousarray(i.mg_time, dtype=np.float64).copy()))

    def movemark(self, s: State, timestep: float, timesum: float, flags: int = 0) -> None:
        rc = lib().ora_movemark(C.byref(self.P), C.byref(self.T), C.byref(self.G), s.x.size, abi.dptr(s.x),
                                abi.dptr(s.y), abi.dptr(s.T), abi.dptr(s.eta), abi.dptr(s.p), abi.i8ptr(s.mtype),
                                abi.dptr(self._hi), timestep, timesum, flags)
        if rc:
            raise RuntimeError(f"ora_movemark: {abi.STATUS_NAMES.get(rc, rc)}")

    def ronurecalc(self, s: State, timesum: float, order: int = ORDER_REFERENCE, track_tmax: bool = True,
                   timestep: float | None = None) -> None:
        """timestep: the global the porosity sintering reads (default: the instance's)."""
        nd = Nodes(*[abi.dptr(s.nodes[k]) for k in NODE_OUT])
        mm = np.zeros(2)
        sa = SinterArgs(self.inst.timestep if timestep is None else timestep, 0, 0,
                        abi.i8ptr(s.mg_old) if s.mg_old is not None else None,
                        abi.dptr(s.mg_time) if s.mg_time is not None else None, s.mag_time)
        rc = lib().ora_ronurecalc(C.byref(self.P), C.byref(self.T), C.byref(self.G), s.x.size, abi.dptr(s.x),
                                  abi.dptr(s.y), abi.dptr(s.T), abi.dptr(s.eta), abi.i8ptr(s.mtype),
                                  abi.dptr(self._hi), abi.dptr(s.tmax) if track_tmax else None,
                                  abi.dptr(s.por) if s.por is not None else None, timesum, 0,
                                  order, C.byref(self.td[0]) if self.td is not None else None,
                                  abi.dptr(s.melt) if s.melt is not None else None, C.byref(sa),
                                  C.byref(nd), abi.dptr(mm))
        if rc:
            raise RuntimeError(f"ora_ronurecalc: {abi.STATUS_NAMES.get(rc, rc)}")
        s.numin, s.numax = float(mm[0]), float(mm[1])
        s.mag_time = float(sa.mag_time)

    def run(self, nsteps: int | None = None, order: int = ORDER_REFERENCE, eta_reinject: bool = True,
            move_flags: int = 0) -> State:
        """nsteps x {movemark; re-inject eta; ronurecalc; timesum += timestep}."""
        inst = self.inst
        s = self.initial_state()
        eta0 = inst.eta.copy()
        timesum = inst.timesum
        for _ in range(inst.nsteps if nsteps is None else nsteps):
            self.movemark(s, inst.timestep, timesum, move_flags)
            if eta_reinject:
                s.eta[:] = eta0
            self.ronurecalc(s, timesum, order)
            timesum += inst.timestep
        return s

    def titerate_markers(self, s: State, tk_new: np.ndarray, heatdif: float, timestep: float,
                         order: int = ORDER_REFERENCE) -> None:
        """The marker temperature update of titerate() (heatmart.c:514-697) on s.T:
        node T before the solve s.nodes['tk'], after it tk_new; s.nodes kt, cp, ro."""
        tn = np.ascontiguousarray(tk_new, dtype=np.float64)
        to, kt, cp, ro = (np.ascontiguousarray(s.nodes[k], dtype=np.float64) for k in ("tk", "kt", "cp", "ro"))
        rc = lib().ora_titerate_markers(C.byref(self.P), C.byref(self.G), s.x.size, abi.dptr(s.x), abi.dptr(s.y),
                                        abi.dptr(s.T), abi.i8ptr(s.mtype), abi.dptr(tn), abi.dptr(to),
                                        abi.dptr(kt), abi.dptr(cp), abi.dptr(ro), heatdif, timestep, order)
        if rc:
            raise RuntimeError(f"ora_titerate_markers: {abi.STATUS_NAMES.get(rc, rc)}")

    def interp_tnode(self, s: State, tk: np.ndarray, tk2: np.ndarray | None = None):
        """allintert() (markmart.c:1687-1745) at every marker of s: eps[2] from tk and
        eps[3] from tk2, the point clamped to the box."""
        tk = np.ascontiguousarray(tk, dtype=np.float64)
        out = np.empty(s.x.size)
        out2 = np.empty(s.x.size) if tk2 is not None else None
        t2 = np.ascontiguousarray(tk2, dtype=np.float64) if tk2 is not None else None
        lib().ora_interp_tnode(C.byref(self.P), C.byref(self.G), s.x.size, abi.dptr(s.x), abi.dptr(s.y),
                               abi.dptr(tk), abi.dptr(t2) if t2 is not None else None, abi.dptr(out),
                               abi.dptr(out2) if out2 is not None else None)
        return out, out2

    # -- single-point helpers for known-answer tests
    def m1serch(self, g: np.ndarray, x: float) -> int:
        g = np.ascontiguousarray(g, dtype=np.float64)
        return int(lib().ora_m1serch(abi.dptr(g), g.size, x))

    def allinterv(self, x: float, y: float):
        a, b = C.c_double(), C.c_double()
        lib().ora_allinterv(C.byref(self.P), C.byref(self.G), x, y, C.byref(a), C.byref(b))
        return a.value, b.value

    def cell_key(self, x: float, y: float) -> int:
        return int(lib().ora_cell_key(C.byref(self.P), C.byref(self.G), x, y))


def radiogenic(mtype: int, timesum: float, al: float, fe: float) -> float:
    return float(lib().ora_radiogenic(mtype, timesum, al, fe))
