"""TEST INFRASTRUCTURE ONLY: run the compiled reference marker step on a synthetic instance.

``oracle/_ref/ref32`` and ``oracle/_ref/ref64`` are built by ``make -C oracle ref``
from the unmodified reference sources (see oracle/ref_harness.c).  This module
writes their input file, runs them and reads their output.  Only tests, the
smoke check and the bench's CPU-baseline legs use it.

File layout (all little-endian):

input  ``int64 hdr[32]``: magic, xnumx, ynumy, marknum, nsteps, markmod, outgrid,
       intermod, intermod1, gridmod, densimod, viscmod, dynamo, reinject_eta,
       mnumx, mnumy, printmod;
       ``double scal[64]``: xsize, ysize, timestep, timesum, nubeg, nuend, nucontr,
       tmp_ambient, M_init, M_acc, core_form_time, k_cutoff, al2627_init,
       fe6056_init, relax_time, por_init, eps21, eps50, eps52;
       24 per-type tables ``double[200]`` (synth.TYPE_TABLES order), ``int64 markim[200]``;
       ``gx[xnumx]``, ``gy[ynumy]``; 20 node arrays (GRID_FIELDS then NODE_OUT);
       markers x, y, T, eta, hi, por, tmax, mgtime (double) and type, mgold (int8);
       mode 1 (hdr[17], titerate's marker update): heatdif in scal[19], then tk_new[nodenum];
       densimod 2 table (hdr[18] = 1): hdr[19..23] = si_melting, fe_melting, ice_melting,
       tknum, pbnum, scal[20..23] = tkmin, pbmin, tkstp, pbstp, then per [tk][pb][db] node
       (density g/cm^3, enthalpy kcal/kg).
output ``int64 hdr[8]`` (magic, marknum, nodenum, nsteps, sizeof marker float);
       markers x, y, T, eta, p, por, tmax, mgtime (double), type, mgold (int8);
       9 node arrays (NODE_OUT); per-step (movemark, ronurecalc) seconds; tkrecalc seconds;
       eps[21], eps[22], eps[50], eps[51], eps[52], eps[53] after the last step.
"""
from __future__ import annotations

import os
import subprocess
import tempfile
from dataclasses import dataclass

import numpy as np

from i2elvis_planet_b200.synth import GRID_FIELDS, NODE_OUT, TYPE_TABLES, Instance

MAGIC = 0x31473249
HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")


def ref_binary(kind: str) -> str:
    """Path of the compiled reference (kind 'ref32' or 'ref64'); raises if it was not built."""
    p = os.path.join(REF_DIR, kind)
    if not os.path.exists(p):
        raise FileNotFoundError(f"{p} missing: run `make -C oracle ref` where the reference tree is present")
    return p


def write_input(inst: Instance, path: str, nsteps: int | None = None, reinject: bool = True,
                titerate: tuple | None = None, prn: bool = False, interp_tk2: np.ndarray | None = None) -> None:
    """``titerate`` = (tk_new, heatdif): write a mode-1 input (one titerate() call
    whose solve yields tk_new; the node T before it is inst.nodes['tk']).  ``prn``:
    a mode-2 input (saver() writes the output file, loader() reads it back).
    ``interp_tk2``: a mode-3 input (allintert() at every marker, tk from
    inst.nodes['tk'] and this tk2)."""
    f = inst.flags
    s = inst.scal
    hdr = np.zeros(32, dtype=np.int64)
    hdr[:18] = [MAGIC, inst.xnumx, inst.ynumy, inst.marknum, inst.nsteps if nsteps is None else nsteps,
                f["markmod"], f["outgrid"], f["intermod"], f["intermod1"], f["gridmod"], f["densimod"],
                f["viscmod"], f["dynamo"], int(reinject), inst.mnumx, inst.mnumy, 0,
                1 if titerate is not None else (2 if prn else (3 if interp_tk2 is not None else 0))]
    if inst.gr is not None or inst.acc is not None:
        hdr[24] = 1
    td = inst.td
    if td is not None:
        tab = np.asarray(td["td"], dtype=np.float64)
        hdr[18:24] = [1, td["si_melting"], td["fe_melting"], td["ice_melting"], td["tknum"], td["pbnum"]]
    scal = np.zeros(64)
    scal[:20] = [inst.xsize, inst.ysize, inst.timestep, inst.timesum, s["nubeg"], s["nuend"], s["nucontr"],
                 s["tmp_ambient"], s["M_init"], s["M_acc"], s["core_form_time"], s["k_cutoff"],
                 s["al2627_init"], s["fe6056_init"], s["relax_time"], s["por_init"], s["eps21"],
                 s["eps50"], s["eps52"], titerate[1] if titerate is not None else 0.0]
    if td is not None:
        scal[20:24] = [td["tkmin"], td["pbmin"], td["tkstp"], td["pbstp"]]
    with open(path, "wb") as fo:
        fo.write(hdr.tobytes())
        fo.write(scal.tobytes())
        for k in TYPE_TABLES:
            fo.write(np.asarray(inst.types[k], dtype=np.float64).tobytes())
        fo.write(np.asarray(inst.markim, dtype=np.int64).tobytes())
        fo.write(np.asarray(inst.gx, dtype=np.float64).tobytes())
        fo.write(np.asarray(inst.gy, dtype=np.float64).tobytes())
        for k in GRID_FIELDS:
            fo.write(np.asarray(inst.grid[k], dtype=np.float64).tobytes())
        for k in NODE_OUT:
            fo.write(np.asarray(inst.nodes[k], dtype=np.float64).tobytes())
        n = inst.marknum
        for a in (inst.x, inst.y, inst.T, inst.eta, inst.hi, inst.por, inst.tmax):
            fo.write(np.asarray(a, dtype=np.float64).tobytes())
        mgt = np.full(n, -1.0) if inst.mg_time is None else inst.mg_time
        mgo = np.full(n, 3, dtype=np.int8) if inst.mg_old is None else inst.mg_old
        fo.write(np.asarray(mgt, dtype=np.float64).tobytes())   # markmg_time
        fo.write(np.asarray(inst.mtype, dtype=np.int8).tobytes())
        fo.write(np.asarray(mgo, dtype=np.int8).tobytes())      # markmg_old
        if titerate is not None:
            fo.write(np.asarray(titerate[0], dtype=np.float64).tobytes())
        if interp_tk2 is not None:
            fo.write(np.asarray(interp_tk2, dtype=np.float64).tobytes())
        if hdr[24]:
            for a in (inst.gr, inst.acc):
                fo.write(np.asarray(np.zeros(n) if a is None else a, dtype=np.float64).tobytes())
        if td is not None:
            fo.write(np.ascontiguousarray(tab[:td["tknum"], :td["pbnum"], :, :2]).tobytes())


@dataclass
class RefResult:
    x: np.ndarray
    y: np.ndarray
    T: np.ndarray
    eta: np.ndarray
    p: np.ndarray
    por: np.ndarray
    tmax: np.ndarray
    mtype: np.ndarray
    nodes: dict
    t_move: np.ndarray
    t_avg: np.ndarray
    t_tkrecalc: float
    marker_bytes: int
    melt: np.ndarray | None = None  # eps[21], eps[22], eps[50], eps[51], eps[52], eps[53] at the end
    mg_time: np.ndarray | None = None
    mg_old: np.ndarray | None = None
    gr: np.ndarray | None = None
    acc: np.ndarray | None = None
    prn_markers: bytes | None = None  # the marker section of saver()'s file (mode 2)
    shim_prn_markers: bytes | None = None  # the C shim's section of the same markers (drop-in builds)
    interp: tuple | None = None  # allintert()'s eps[2], eps[3] at every marker (mode 3)


def read_output(path: str) -> RefResult:
    raw = np.fromfile(path, dtype=np.uint8)
    off = 0

    def take(dtype, count):
        nonlocal off
        nb = np.dtype(dtype).itemsize * count
        a = raw[off:off + nb].view(dtype).copy()
        off += nb
        return a

    hdr = take(np.int64, 8)
    if hdr[0] != MAGIC:
        raise ValueError("bad reference output")
    n, nn, ns, mb = (int(v) for v in hdr[1:5])
    mk = [take(np.float64, n) for _ in range(8)]
    mtype = take(np.int8, n)
    mgold = take(np.int8, n)
    nodes = {k: take(np.float64, nn) for k in NODE_OUT}
    tim = take(np.float64, 2 * ns).reshape(ns, 2) if ns else np.zeros((0, 2))
    tkr = float(take(np.float64, 1)[0])
    melt = take(np.float64, 6)
    gr = take(np.float64, n)
    acc = take(np.float64, n)
    r = RefResult(x=mk[0], y=mk[1], T=mk[2], eta=mk[3], p=mk[4], por=mk[5], tmax=mk[6], mtype=mtype,
                  nodes=nodes, t_move=tim[:, 0], t_avg=tim[:, 1], t_tkrecalc=tkr, marker_bytes=mb, melt=melt,
                  mg_time=mk[7], mg_old=mgold, gr=gr, acc=acc)
    if int(hdr[5]) == 3:  # allintert() at every marker: eps[2], eps[3]
        r.interp = (take(np.float64, n), take(np.float64, n))
    return r


def run_reference(inst: Instance, kind: str = "ref64", nsteps: int | None = None, reinject: bool = True,
                  workdir: str | None = None, timeout: float = 3600.0, titerate: tuple | None = None,
                  prn: bool = False, interp_tk2: np.ndarray | None = None) -> RefResult:
    """Run the compiled reference for ``nsteps`` marker steps on ``inst`` and return its state;
    with ``titerate`` = (tk_new, heatdif), one titerate() call instead (mode 1); with
    ``prn``, saver() then loader() instead (mode 2): the state is what loader() read,
    ``prn_markers`` the marker section of the file (the last marknum + 1 records)."""
    exe = ref_binary(kind)
    with tempfile.TemporaryDirectory(dir=workdir) as td:
        fin = os.path.join(td, "in.i2gin")
        fout = os.path.join(td, "out.i2gout")
        write_input(inst, fin, nsteps=nsteps, reinject=reinject, titerate=titerate, prn=prn, interp_tk2=interp_tk2)
        subprocess.run([exe, fin, fout], check=True, timeout=timeout, stdout=subprocess.DEVNULL, cwd=td)
        r = read_output(fout)
        if prn:
            with open(os.path.join(td, "out.prn"), "rb") as f:
                data = f.read()
            r.prn_markers = data[len(data) - PRN_RECORD_BYTES * (inst.marknum + 1):]
            shim = os.path.join(td, "shim.prn")
            if os.path.exists(shim):
                with open(shim, "rb") as f:
                    r.shim_prn_markers = f.read()
        return r


PRN_RECORD_BYTES = 39  # loadmart.c:795-808: nine 4-byte floats and three bytes per marker
