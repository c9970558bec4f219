"""Generate the golden fixtures from the compiled, unmodified reference.

Run where the reference tree is present (it builds oracle/_ref first):

    python tests/golden/make_golden.py

For every parity variant (tests/golden/variants.py) and for the 101x101 'c1'
workload it runs ``oracle/_ref/ref64`` (reference source, FP64 marker storage)
and, for 'default' and 'c1', ``oracle/_ref/ref32`` (reference storage), then
stores in ``tests/golden/<name>_<kind>.npz``:

* a SHA-256 digest of every full output array (bit-exact pins),
* every node output field (tolerance comparisons),
* every 16th marker of each marker output (spot values),
* a digest of the inputs, so a change of the synthetic generator is caught.

For the thermal cases (variants.THERMAL_NAMES) it runs the reference's
titerate() once (oracle/ref_harness.c mode 1) and stores the marker temperature
digest and spot values in ``tests/golden/titerate_<name>_<kind>.npz``; for three
parity variants it calls allintert() at every marker (mode 3) and stores the
digests of eps[2] and eps[3] in ``tests/golden/interp_ref64.npz``.
"""
from __future__ import annotations

import hashlib
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from i2elvis_planet_b200 import synth  # noqa: E402
from oracle import refio  # noqa: E402
import variants  # noqa: E402

MARKER_OUT = ("x", "y", "T", "eta", "p", "tmax")
STRIDE = 16


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def input_digest(inst: synth.Instance) -> str:
    h = hashlib.sha256()
    for a in (inst.gx, inst.gy, inst.x, inst.y, inst.T, inst.eta, inst.mtype, inst.hi):
        h.update(np.ascontiguousarray(a).tobytes())
    if np.any(inst.por):
        h.update(np.ascontiguousarray(inst.por).tobytes())
    if inst.mg_old is not None:
        h.update(np.ascontiguousarray(inst.mg_old).tobytes())
        h.update(np.ascontiguousarray(inst.mg_time).tobytes())
        h.update(repr((inst.flags["dynamo"], inst.timesum)).encode())
    for k in synth.GRID_FIELDS:
        h.update(np.ascontiguousarray(inst.grid[k]).tobytes())
    for k in synth.NODE_OUT:
        h.update(np.ascontiguousarray(inst.nodes[k]).tobytes())
    if inst.td is not None:
        h.update(np.ascontiguousarray(inst.td["td"]).tobytes())
        h.update(repr(sorted((k, v) for k, v in inst.td.items() if k != "td")).encode())
    return h.hexdigest()


def save(name: str, kind: str, inst: synth.Instance, r: refio.RefResult, node_fields=synth.NODE_OUT) -> None:
    out = {"input_digest": np.array(input_digest(inst)), "stride": np.array(STRIDE)}
    for f in MARKER_OUT:
        a = getattr(r, f)
        out[f"digest_{f}"] = np.array(digest(a))
        out[f"m_{f}"] = a[::STRIDE].copy()
    if inst.mg_old is not None:
        # magnetisation state and time (markmart.c:651-744)
        out["digest_mg_old"] = np.array(digest(r.mg_old))
        out["digest_mg_time"] = np.array(digest(r.mg_time))
    if np.any(inst.por):
        out["digest_por"] = np.array(digest(r.por))
        out["m_por"] = r.por[::STRIDE].copy()
    if inst.td is not None:
        # the table path changes marker types and leaves a melt state (markmart.c:2180-2181, 287)
        out["digest_type"] = np.array(digest(r.mtype))
        out["m_type"] = r.mtype[::STRIDE].copy()
        out["melt"] = r.melt
    for k in synth.NODE_OUT:
        out[f"digest_{k}"] = np.array(digest(r.nodes[k]))
    for k in node_fields:
        out[f"n_{k}"] = r.nodes[k]
    np.savez_compressed(os.path.join(HERE, f"{name}_{kind}.npz"), **out)


INTERP_NAMES = ("edges", "outgrid2", "nonuniform")


def interp_tk2(inst: synth.Instance) -> np.ndarray:
    """The second node field of the allintert() fixtures: tk with a seeded ripple."""
    tk = np.asarray(inst.nodes["tk"], dtype=np.float64)
    return tk + 5.0 * np.sin(np.arange(tk.size) * 0.37)


def main() -> None:
    """All fixtures; with --only a,b only those parity variants."""
    only = None
    if "--only" in sys.argv:
        only = set(sys.argv[sys.argv.index("--only") + 1].split(","))
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)
    for name in variants.NAMES:
        if only is not None and name not in only:
            continue
        inst = variants.variant(name)
        mf = variants.move_flags(inst)
        r = refio.run_reference(inst, "ref64", reinject=not mf)
        save(name, "ref64", inst, r)
        if name == "default":
            save(name, "ref32", inst, refio.run_reference(inst, "ref32"))
        print("golden", name)
    if only is None or "prn" in only:
        # saver() writes the output file, loader() reads it back (oracle/ref_harness.c mode 2)
        inst = variants.prn_instance()
        r = refio.run_reference(inst, "ref32", prn=True)
        out = {"input_digest": np.array(input_digest(inst)), "section_digest": np.array(digest(
            np.frombuffer(r.prn_markers, np.uint8))), "section_bytes": np.array(len(r.prn_markers))}
        for k in ("x", "y", "T", "eta", "por", "tmax", "gr", "acc", "mg_time", "mg_old", "mtype"):
            out[f"digest_{k}"] = np.array(digest(getattr(r, k)))
        np.savez_compressed(os.path.join(HERE, "prn_ref32.npz"), **out)
        print("golden prn")
    if only is None or "interp" in only:
        # allintert() at every marker (oracle/ref_harness.c mode 3), markers on grid
        # lines, on and outside the box edges, a nonuniform grid
        out = {}
        for name in INTERP_NAMES:
            inst = variants.variant(name)
            tk2 = interp_tk2(inst)
            r = refio.run_reference(inst, "ref64", interp_tk2=tk2)
            h = hashlib.sha256(input_digest(inst).encode())
            h.update(np.ascontiguousarray(tk2).tobytes())
            out[f"input_digest_{name}"] = np.array(h.hexdigest())
            out[f"digest_eps2_{name}"] = np.array(digest(r.interp[0]))
            out[f"digest_eps3_{name}"] = np.array(digest(r.interp[1]))
            out[f"m_eps2_{name}"] = r.interp[0][::STRIDE].copy()
        np.savez_compressed(os.path.join(HERE, "interp_ref64.npz"), **out)
        print("golden interp")
    if only is not None:
        return
    c1 = synth.make_config("c1")
    save("c1", "ref64", c1, refio.run_reference(c1, "ref64"), node_fields=("ro", "nu", "tk"))
    save("c1", "ref32", c1, refio.run_reference(c1, "ref32"), node_fields=("ro", "nu", "tk"))
    print("golden c1")
    for name in variants.THERMAL_NAMES:
        inst, tk_new, heatdif = variants.thermal_variant(name)
        for kind in ("ref64", "ref32") if name == "thermal" else ("ref64",):
            r = refio.run_reference(inst, kind, titerate=(tk_new, heatdif))
            h = hashlib.sha256(input_digest(inst).encode())
            h.update(np.ascontiguousarray(tk_new).tobytes())
            np.savez_compressed(os.path.join(HERE, f"titerate_{name}_{kind}.npz"),
                                input_digest=np.array(h.hexdigest()), stride=np.array(STRIDE),
                                heatdif=np.array(heatdif), digest_T=np.array(digest(r.T)), m_T=r.T[::STRIDE].copy())
        print("golden titerate", name)


if __name__ == "__main__":
    main()
