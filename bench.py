"""Throughput of the B200 marker step (movemark + ronurecalc) in marker updates/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload c3|c2|c1] [--precision mixed|fp64]

Default workload: 1001x1001 nodes, 6x6 markers per cell (36,000,000 markers), 8
extra stream-function modes, viscosity 1e18-1e24 Pa s, markers in random storage
order; mixed precision.  A step is one movemark() + ronurecalc() over every marker
(the reference harness loop of i2mart.c:107-153 without the solvers).  Inputs are
resident in HBM when the timed region starts and are larger than L2 (no flush).

N > 1 (torchrun): every rank runs its own planetesimal (seed + rank) with no
collective on the data path (weak scaling); value = all ranks' marker updates /
the slowest rank's device time.

--impl reference: the reference's own C marker step (oracle/_ref/ref32, built from
the unmodified sources) on the host cores: the workload's markers split into
disjoint slices, one process per core, each on the full grid, so that every step
updates every marker of the workload.

The JSON line carries, besides throughput: the roofline of the dominant kernel,
the reference loop timed on one host core (cpu_baseline), the same step end to end
through the C ABI with host buffers (e2e), and the mixed form's error against the
FP64 form and against the reference's C loop (error).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "marker updates/s (RK4 advect + M2N avg): mixed vs FP64 on B200 @1e-6 rel err"
FALLBACK_HBM_GBS = 6650.0
# algorithmic bytes (FP64 storage layout): per marker read x,y,T,eta (4x8) + type (1),
# write x,y,p (3x8); per node read vx,vy,pr (3x8), write ro,nu,nd,et,cp,kt,ht,tk (8x8)
B_MARKER = 57
B_NODE = 88
# per-kernel share of those bytes, per marker / per node (the shares sum to
# B_MARKER, B_NODE; sort traffic, the sorted copy and the payload are overhead)
KERNEL_BYTES = {
    "movemark": ("k_move", 41.0, 24.0),       # read x,y,type; write x,y,p | read vx,vy,pr
    "cell_sort": ("k_fixup", 0.0, 0.0),       # cell ranking: no algorithmic bytes
    # read T,eta (x,y,type counted under movemark); on the benchmark's constant-property
    # calls the phase runs k_contrib_const, the record-moving k_contrib every 32nd call
    "contrib": ("k_contrib_const", 16.0, 0.0),
    "cell_sums": ("k_cellsums", 0.0, 0.0),    # payload -> cell corner sums: intermediate only
    "node_loop": ("k_nodesums", 0.0, 64.0),   # write ro,nu,nd,et,cp,kt,ht,tk
}
# the mixed form's fused step: movemark with the averaging records reads every
# marker input and writes every marker output; the cell sums with the node loop
# write the node fields
FUSED_KERNEL_BYTES = {
    "movemark": ("k_move_fused", 57.0, 24.0),  # read x,y,T,eta,type; write x,y,p | read vx,vy,pr
    "cell_sort": ("k_fixup", 0.0, 0.0),        # the periodic reorder
    "contrib": ("k_fused_begin", 0.0, 0.0),
    "cell_sums": ("k_cellnodes", 0.0, 64.0),   # buckets -> node fields ro,nu,nd,et,cp,kt,ht,tk
    "node_loop": ("k_fused_clamp", 0.0, 0.0),
}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def profile_traffic(kernel: str):
    """DRAM bytes per marker of `kernel` from a committed ncu summary (profiles/)."""
    d = os.path.join(ROOT, "profiles")
    if not os.path.isdir(d):
        return None
    for fn in sorted(os.listdir(d)):
        # <kernel>_<workload>_<precision>.txt
        if not fn.endswith(".txt") or fn.rsplit("_", 2)[0] != kernel:
            continue
        for line in open(os.path.join(d, fn)):
            if line.startswith("dram_bytes_per_marker:"):
                return float(line.split(":")[1])
    return None


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons of the GPU, polled through NVML
    every 2 ms from a thread while the block runs (read-only queries); falls back
    to `nvidia-smi -lms 200` when NVML is unavailable."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.p = None
        self.fn = None
        self.nv = None
        self.sm, self.smax, self.reasons = [], [], set()

    def _handle(self, nv):
        try:
            import torch
            bus = torch.cuda.get_device_properties(self.index).pci_bus_id
            dom = torch.cuda.get_device_properties(self.index).pci_domain_id
            dv = torch.cuda.get_device_properties(self.index).pci_device_id
            return nv.nvmlDeviceGetHandleByPciBusId(f"{dom:08x}:{bus:02x}:{dv:02x}.0".encode())
        except Exception:
            return nv.nvmlDeviceGetHandleByIndex(self.index)

    def _poll(self):
        nv, h = self.nv, self.h
        bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        smax = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        while not self.stop.is_set():
            try:
                self.sm.append(float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)))
                self.smax.append(float(smax))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                for n, b in bits.items():
                    if r & b:
                        self.reasons.add(n)
            except Exception:
                pass
            self.stop.wait(0.002)

    def __enter__(self):
        try:
            import threading
            import pynvml as nv
            nv.nvmlInit()
            self.nv, self.h = nv, self._handle(nv)
            self.stop = threading.Event()
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
            # NVML's first queries can take longer than a short timed region:
            # return once the poller has its first sample
            t0 = time.time()
            while not self.sm and time.time() - t0 < 2.0:
                time.sleep(0.001)
            return self
        except Exception:
            self.nv = None
        try:
            self.fn = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False).name
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=open(self.fn, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.nv is not None:
            self.stop.set()
            self.t.join(timeout=5)
            try:
                self.nv.nvmlShutdown()
            except Exception:
                pass
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()

    def summary(self) -> dict:
        if self.nv is None and self.fn and os.path.exists(self.fn):
            for line in open(self.fn):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    self.sm.append(float(f[1]))
                    self.smax.append(float(f[2]))
                except ValueError:
                    continue
                for n, v in zip(self.NAMES, f[5:9]):
                    if v.lower() == "active":
                        self.reasons.add(n)
            os.unlink(self.fn)
        if not self.sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(self.sm), "sm_max_mhz": max(self.smax), "reasons": sorted(self.reasons),
                "samples": len(self.sm), "source": "nvml" if self.nv is not None else "nvidia-smi"}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def reduce_job(units: float, ms: float, device) -> tuple:
    """(sum of every rank's units, the slowest rank's milliseconds) over the process
    group; the values themselves without one.  Every rank calls it once, in the
    same place, so the collectives line up."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(units), float(ms)
    u = torch.tensor([float(units)], dtype=torch.float64, device=device)
    m = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    dist.all_reduce(m, op=dist.ReduceOp.MAX)
    return float(u.item()), float(m.item())


def build_instance(workload: str, rank: int, table: bool = False):
    """The named workload; table: the same markers on the densimod 2 P-T table
    path (synth.with_table: seeded table, silicate, crust and wet types)."""
    from i2elvis_planet_b200 import synth
    inst = synth.make_config(workload, instance=rank)
    return synth.with_table(inst) if table else inst


def cpu_baseline(inst, sample: int, nsteps: int = 2) -> dict:
    """The reference's marker step (oracle/_ref/ref32, unmodified source) on 1 host
    core over a bounded sample of the workload's markers, full grid."""
    from i2elvis_planet_b200 import synth
    from oracle import refio
    s = synth.subset(inst, np.arange(min(sample, inst.marknum)))
    kind = "reference"
    try:
        refio.ref_binary("ref32")
        r = refio.run_reference(s, "ref32", nsteps=nsteps)
        per = [a + b for a, b in zip(r.t_move, r.t_avg)]
        t = statistics.median(per)
    except FileNotFoundError:
        # prebuilt reference absent: the oracle's sequential C restatement
        from oracle import oracle
        kind = "port"
        o = oracle.Oracle(s)
        st = o.initial_state()
        per = []
        for _ in range(nsteps):
            t0 = time.perf_counter()
            o.movemark(st, s.timestep, s.timesum)
            o.ronurecalc(st, s.timesum)
            per.append(time.perf_counter() - t0)
        t = statistics.median(per)
    return {"value": s.marknum / t, "unit": "marker updates/s", "cores": 1, "kind": kind,
            "sample": f"{s.marknum} of the {inst.marknum} {inst.name} markers on the full "
                      f"{inst.xnumx}x{inst.ynumy} grid, median of {nsteps} steps, 1 process"}


def field_errors(got: dict, ref: dict, keys) -> dict:
    """Per field: max|d| / max|ref| and ||d||_2 / ||ref||_2."""
    out = {}
    for k in keys:
        a, b = np.asarray(got[k], dtype=np.float64), np.asarray(ref[k], dtype=np.float64)
        d = a - b
        out[k] = {"max_rel": float(np.abs(d).max() / max(np.abs(b).max(), 1e-300)),
                  "l2_rel": float(np.linalg.norm(d) / max(np.linalg.norm(b), 1e-300))}
    return out


def error_report(inst) -> dict:
    """The mixed form's error on the benchmark's own instance, outside the timed
    region: (1) against the FP64 form (the reference's arithmetic operation by
    operation, bit-identical to the oracle) over the workload's steps from the
    same seeded state, every node field and the marker positions; (2) against the
    reference's own C loop (oracle/_ref/ref64: the unmodified sources with FP64
    marker storage) over 2 steps of every marker of a 200 x 200-cell window of the
    workload, on the full grid, at the nodes inside the window."""
    from i2elvis_planet_b200 import abi, lib, synth
    nsteps = inst.nsteps
    runs = {}
    for name, prec in (("fp64", abi.PREC_FP64), ("mixed", abi.PREC_MIXED)):
        mk, nodes, ms = lib.run_instance(inst, precision=prec, track_tmax=False)
        fused = ms.fused_info()["fused_moves"] if prec == abi.PREC_MIXED else 0
        ms.close()
        runs[name] = (mk, nodes, fused)
    (m64, n64, _), (mmx, nmx, fused) = runs["fp64"], runs["mixed"]
    cell = inst.gx[1] - inst.gx[0]
    out = {"vs_fp64": {"steps": nsteps, "markers": inst.marknum, "fused_moves": fused,
                       "nodes": field_errors(nmx, n64, synth.NODE_OUT),
                       "marker_max_abs_dx_m": float(np.abs(mmx["x"] - m64["x"]).max()),
                       "marker_max_abs_dy_m": float(np.abs(mmx["y"] - m64["y"]).max()),
                       "marker_max_abs_dxy_cells": float(max(np.abs(mmx["x"] - m64["x"]).max(),
                                                             np.abs(mmx["y"] - m64["y"]).max()) / cell),
                       "marker_T_max_rel": float(np.abs(mmx["T"] - m64["T"]).max() / np.abs(m64["T"]).max()),
                       "marker_p_max_rel": float(np.abs(mmx["p"] - m64["p"]).max() / np.abs(m64["p"]).max())}}
    worst = max(v["max_rel"] for v in out["vs_fp64"]["nodes"].values())
    out["vs_fp64"]["worst_node_max_rel"] = worst
    del runs, m64, n64, mmx, nmx
    try:
        from oracle import refio
        refio.ref_binary("ref64")
        # every marker of a window of cells across the disk edge (air, silicate
        # and iron), on the full grid; nodes compared three cells inside the
        # window, where no marker of the window's surroundings would reach
        n1 = inst.xnumx - 1
        w = max(8, min(200, n1 // 5))
        a0, b0 = (3 * n1) // 10, n1 // 10
        cx = np.floor((inst.x - inst.gx[0]) / cell).astype(np.int64)
        cy = np.floor((inst.y - inst.gy[0]) / cell).astype(np.int64)
        idx = np.nonzero((cx >= a0) & (cx < a0 + w) & (cy >= b0) & (cy < b0 + w))[0]
        sub = synth.subset(inst, idx)
        r = refio.run_reference(sub, "ref64", nsteps=2)
        mk, nodes, ms = lib.run_instance(sub, precision=abi.PREC_MIXED, nsteps=2, track_tmax=False)
        ms.close()
        m1, m2 = np.meshgrid(np.arange(inst.xnumx), np.arange(inst.ynumy), indexing="ij")
        inner = ((m1 >= a0 + 3) & (m1 <= a0 + w - 3) & (m2 >= b0 + 3) & (m2 <= b0 + w - 3)).reshape(-1)
        out["vs_reference_c"] = {"binary": "ref64 (unmodified reference sources, FP64 marker storage)",
                                 "steps": 2, "markers": int(sub.marknum),
                                 "window_cells": f"[{a0}, {a0 + w}) x [{b0}, {b0 + w})",
                                 "nodes": field_errors({k: v[inner] for k, v in nodes.items()},
                                                       {k: v[inner] for k, v in r.nodes.items()}, synth.NODE_OUT),
                                 "marker_max_abs_dxy_cells": float(max(np.abs(mk["x"] - r.x).max(),
                                                                       np.abs(mk["y"] - r.y).max()) / cell)}
        out["vs_reference_c"]["worst_node_max_rel"] = max(
            v["max_rel"] for v in out["vs_reference_c"]["nodes"].values())
    except FileNotFoundError as e:
        out["vs_reference_c"] = {"unavailable": str(e)}
    return out


def run_reference_arm(args) -> None:
    """The reference's own C marker step (oracle/_ref/ref32, the unmodified sources,
    FP32 marker storage) over the whole configuration: the workload's markers are
    split into disjoint slices, one process per slice, every process on the full
    grid, so every step updates every marker of the configuration once.  The
    reference loop is serial (OpenMP is commented out in i2mart.c:6-8), so the
    slices run side by side on the host's cores; a step's time is its slowest
    process."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    from i2elvis_planet_b200 import synth
    from oracle import refio
    inst = build_instance(args.workload, 0, args.table)
    try:
        exe = refio.ref_binary("ref32")
    except FileNotFoundError as e:
        print(json.dumps({"impl": "reference", "unavailable": f"reference build missing: {e}"}))
        return
    try:
        import psutil
        avail = psutil.virtual_memory().available
    except Exception:
        avail = 32 << 30
    n = inst.marknum
    cores = os.cpu_count() or 1
    nproc = max(1, min(cores, args.ref_procs))
    # resident set of one process: the grid arrays (~1.6 GB at 1001^2) + ~120 B per marker
    while nproc > 1 and nproc * (1.6e9 + 120.0 * (n / nproc)) > 0.6 * avail:
        nproc -= 1
    bounds = np.linspace(0, n, nproc + 1).astype(np.int64)
    nsteps = args.warmup + args.steps
    td = tempfile.mkdtemp(prefix="i2gref_")
    procs = []
    try:
        for p in range(nproc):
            s = synth.subset(inst, np.arange(bounds[p], bounds[p + 1]))
            fin = os.path.join(td, f"in{p}.i2gin")
            refio.write_input(s, fin, nsteps=nsteps)
            procs.append((fin, os.path.join(td, f"out{p}.i2gout")))
            del s
        t0 = time.time()
        running = [subprocess.Popen([exe, fi, fo], stdout=subprocess.DEVNULL) for fi, fo in procs]
        rcs = [p.wait() for p in running]
        wall = time.time() - t0
        if any(rcs):
            print(json.dumps({"impl": "reference", "unavailable": f"reference process failed: {rcs}"}))
            return
        outs = [refio.read_output(fo) for _, fo in procs]
    finally:
        for f in os.listdir(td):
            os.unlink(os.path.join(td, f))
        os.rmdir(td)
    step_t = np.array([[o.t_move[k] + o.t_avg[k] for k in range(nsteps)] for o in outs])  # [proc, step]
    timed = step_t[:, args.warmup:]
    per_step = timed.max(axis=0)  # slowest process per step
    total = float(per_step.sum())
    value = n * args.steps / total
    out = {
        "metric": METRIC, "value": value, "unit": "marker updates/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 storage, f64 math",
        "data": "synthetic", "impl": "reference",
        "config": {"workload": f"{inst.name}: {inst.xnumx}x{inst.ynumy} nodes, {n} markers",
                   "markers_per_process": int(bounds[1] - bounds[0]), "processes": nproc,
                   "slices": "disjoint, together every marker of the workload", "wall_s": round(wall, 1)},
        "cpu_baseline": {"value": value, "unit": "marker updates/s", "cores": nproc, "kind": "reference",
                         "sample": f"all {n} markers of {inst.name} per step, {nproc} processes of "
                                   f"~{n // nproc} markers each on the full grid"},
        "e2e": {"value": value, "unit": "marker updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))


def prn_leg(ms, inst, reps: int = 3) -> dict:
    """The output file's marker section through the C ABI (pinned host buffer,
    host wall time per call, best of reps): saver()'s records from the
    device-resident markers, then loader()'s records back into the context."""
    import torch
    n = inst.marknum
    gr = torch.zeros(n, dtype=torch.float32, pin_memory=True).numpy()
    acc = torch.zeros(n, dtype=torch.float32, pin_memory=True).numpy()
    out = torch.empty(39 * n, dtype=torch.uint8, pin_memory=True).numpy()
    wt, rt = [], []
    for _ in range(reps):
        t0 = time.perf_counter()
        ms.write_prn(gr=gr, acc=acc, out=out)
        wt.append(time.perf_counter() - t0)
    for _ in range(reps):
        t0 = time.perf_counter()
        ms.read_prn(out)
        rt.append(time.perf_counter() - t0)
    nb = out.size
    return {"records": n, "bytes": nb, "write_ms": 1e3 * min(wt), "read_ms": 1e3 * min(rt),
            "write_gbs": nb / min(wt) / 1e9, "read_gbs": nb / min(rt) / 1e9,
            "note": "host wall time per call, pinned host buffers, PCIe copy included"}


def thermal_leg(ms, inst, stream, reps: int = 5) -> dict:
    """titerate()'s marker temperature update (heatmart.c:514-697) on the
    device-resident markers after a thermal solve (synth.thermal_fields: a smooth
    node T change), node arrays on the device, CUDA events on the context's
    stream, best of reps; with the subgrid diffusion (heatdif 1) and without."""
    import torch
    from i2elvis_planet_b200 import synth
    import copy
    probe = copy.copy(inst)  # thermal_fields replaces arrays and node fields, never writes into them
    probe.nodes = dict(inst.nodes)
    f = synth.thermal_fields(probe)
    dev = torch.device("cuda", torch.cuda.current_device())
    tn = torch.as_tensor(f["tk_new"], device=dev)
    to = torch.as_tensor(f["tk_old"], device=dev)
    kt, cp, ro = (torch.as_tensor(probe.nodes[k], device=dev) for k in ("kt", "cp", "ro"))
    out = {}
    for hd in (0.0, 1.0):
        best = 1e30
        for _ in range(reps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            ms.titerate_markers_dev(tn, to, hd, inst.timestep, kt, cp, ro)
            e1.record(stream)
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        out[f"heatdif_{int(hd)}_ms"] = best
    return out


def run_ours(args) -> None:
    import torch
    import torch.distributed as dist

    from i2elvis_planet_b200 import abi, lib, synth

    ws, rank, local = dist_env()
    if ws > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()
    prec = abi.PREC_MIXED if args.precision == "mixed" else abi.PREC_FP64
    inst = build_instance(args.workload, rank, args.table)
    nm, nn = inst.marknum, inst.nodenum
    ms = lib.MarkerStep.from_instance(inst, precision=prec, device=dev)
    stream = torch.cuda.ExternalStream(ms.stream(), device=dev)
    timesum = inst.timesum
    for _ in range(args.warmup):
        ms.movemark(inst.timestep, timesum)
        ms.ronurecalc(timesum)
        timesum += inst.timestep
    ms.sync()
    ms.profile_enable(True)
    ms.profile_read(reset=True)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            ms.movemark(inst.timestep, timesum)
            ms.ronurecalc(timesum)
            timesum += inst.timestep
        e1.record(stream)
        torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    ms_total = e0.elapsed_time(e1)
    prof = ms.profile_read(reset=True)
    ms.profile_enable(False)
    fused = ms.fused_info()["fused_moves"] > 0
    units, ms_max = reduce_job(nm * args.steps, ms_total, "cuda")
    value = units / (ms_max / 1e3)

    # roofline of the dominant kernel (phase with the most device time)
    peak, peak_kind = peaks()
    dom = max(prof["ms"], key=lambda k: prof["ms"][k])
    kname, bm, bn = (FUSED_KERNEL_BYTES if fused else KERNEL_BYTES)[dom]
    calls = max(1, prof["calls"][dom])
    per_launch_ms = prof["ms"][dom] / calls
    alg = bm * nm + bn * nn
    achieved = alg / (per_launch_ms / 1e3) / 1e9 if alg else 0.0
    tr = profile_traffic(kname)
    step_bytes = B_MARKER * nm + B_NODE * nn
    step_gbs = step_bytes / (ms_total / args.steps / 1e3) / 1e9

    # end to end through the C ABI with pinned host buffers (the drop-in call sequence)
    e2e = run_e2e(ms, inst, args, stream) if args.e2e_steps > 0 else None

    cpu = None
    if rank == 0 and ws == 1 and not args.skip_cpu_baseline:
        cpu = cpu_baseline(inst, args.cpu_sample)
    fused_stats = ms.fused_info()
    prn = prn_leg(ms, inst) if args.prn else None
    thermal = thermal_leg(ms, inst, stream) if args.thermal else None
    ms.close()
    err = None
    if rank == 0 and ws == 1 and not args.skip_error and prec == abi.PREC_MIXED:
        err = error_report(inst)

    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": "marker updates/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "mixed (f32 weights/products, f64 coords/sums)" if prec == abi.PREC_MIXED else "f64",
            "data": "synthetic",
            "config": {"workload": f"{inst.name}: {inst.xnumx}x{inst.ynumy} nodes, {inst.mnumx}x{inst.mnumy} "
                                   f"markers/cell, {nm} markers, random storage order",
                       "markers_per_gpu": nm, "nodes_per_gpu": nn, "precision": args.precision,
                       "parallelism": f"{ws} independent instances" if ws > 1 else "single instance",
                       "l2": "inputs larger than L2 (no flush): "
                             f"{step_bytes / 1e9:.2f} GB algorithmic per step vs 126 MB L2"},
            "roofline": {"bound": "hbm", "kernel": kname, "phase": dom, "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                         "traffic": (tr * nm if tr is not None else None),
                         "algorithmic_bytes_per_launch": alg,
                         "per_launch_ms": per_launch_ms},
            "step_roofline": {"bytes_per_step": step_bytes, "achieved": step_gbs, "peak": peak,
                              "frac": step_gbs / peak, "unit": "GB/s"},
            "phases_ms_per_step": {k: v / args.steps for k, v in prof["ms"].items()},
            "gpu_launches": prof["launches"],
            "clocks": clk.summary(),
            "e2e": e2e,
            "cpu_baseline": cpu,
            "fused": fused_stats,
            "error": err,
        }
        if args.table:
            out["config"]["densimod"] = 2
            out["config"]["table"] = "seeded 350x350 P-T table, Herzberg solidus, water-ice melting"
        if prn is not None:
            out["prn"] = prn
        if thermal is not None:
            out["titerate_markers"] = thermal
        print(json.dumps(out))
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_batch(args) -> None:
    """Batched workload: 64 planetesimals (grids 101^2..401^2, 3x3..6x6 markers per
    cell, disk radius 50-250 km, vmax 1e-10..1e-8 m/s), mixed precision; the
    autotuner picks during warm-up between one launch per phase over all instances
    (graph replay per step, launch shape tuned) and every instance's own step on
    its own stream.  N ranks: every rank steps its own 64 (weak scaling)."""
    import torch
    import torch.distributed as dist

    from i2elvis_planet_b200 import abi, lib, synth

    ws, rank, local = dist_env()
    if ws > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=900),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()
    prec = abi.PREC_MIXED if args.precision == "mixed" else abi.PREC_FP64
    insts = synth.make_batch(args.ninst, seed_instance0=args.ninst * rank)
    nm = sum(i.marknum for i in insts)
    nn = sum(i.nodenum for i in insts)
    steps = [lib.MarkerStep.from_instance(i, precision=prec, device=dev) for i in insts]
    b = lib.Batch(steps)
    dt = np.array([i.timestep for i in insts])
    ts = np.array([i.timesum for i in insts])
    tune = b.autotune(dt, ts, steps_per_candidate=2)
    b.step(dt, ts, args.warmup)
    b.sync()
    for m in steps:
        m.profile_read(reset=True)
    stream = torch.cuda.ExternalStream(b.stream(), device=dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev) as clk:
        e0.record(stream)
        b.step(dt, ts, args.steps)
        e1.record(stream)
        torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    ms_total = e0.elapsed_time(e1)
    units, ms_max = reduce_job(nm * args.steps, ms_total, "cuda")
    peak, peak_kind = peaks()
    step_bytes = B_MARKER * nm + B_NODE * nn
    step_gbs = step_bytes / (ms_total / args.steps / 1e3) / 1e9
    if rank == 0:
        out = {
            "metric": METRIC, "value": units / (ms_max / 1e3), "unit": "marker updates/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "mixed (f32 weights/products, f64 coords/sums)" if prec == abi.PREC_MIXED else "f64",
            "data": "synthetic",
            "config": {"workload": f"batched: {len(insts)} planetesimals, grids "
                                   f"{min(i.xnumx for i in insts)}^2..{max(i.xnumx for i in insts)}^2, "
                                   f"{nm} markers per GPU",
                       "markers_per_gpu": nm, "nodes_per_gpu": nn, "precision": args.precision,
                       "launch_shape": tune, "parallelism": f"{ws} x {len(insts)} independent instances",
                       "l2": f"inputs larger than L2 (no flush): {step_bytes / 1e9:.2f} GB algorithmic per step"},
            "step_roofline": {"bytes_per_step": step_bytes, "achieved": step_gbs, "peak": peak,
                              "frac": step_gbs / peak, "unit": "GB/s", "peak_source": peak_kind},
            "gpu_launches": (sum(m.profile_read(reset=True)["launches"] for m in steps)
                             if tune["strategy"] == "streams" else 11 * args.steps),
            "clocks": clk.summary(),
        }
        print(json.dumps(out))
    b.close()
    for m in steps:
        m.close()
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_adjoint_bench(args) -> None:
    """Adjoint workload: 201x201 nodes, 4x4 markers per cell (640,000 markers), 8
    stream-function modes, 20 steps, checkpoint every 5.  Reports the forward
    throughput and the cost of the backward pass relative to the forward."""
    import torch

    from i2elvis_planet_b200 import abi, lib, synth

    torch.cuda.set_device(0)
    prec = abi.PREC_MIXED if args.precision == "mixed" else abi.PREC_FP64
    inst = synth.make_config("c5")
    nsteps, every = 20, 5
    ms = lib.MarkerStep.from_instance(inst, precision=prec)
    ms.adjoint_setup(inst.mode_vx, inst.mode_vy)
    stream = torch.cuda.ExternalStream(ms.stream())
    g = np.ones(inst.nodenum)

    def once():
        ms.set_markers(inst.x, inst.y, inst.T, inst.eta, inst.mtype)
        ms.sync()
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record(stream)
        ms.adjoint_forward(inst.amps, nsteps, inst.timestep, inst.timesum, every)
        e1.record(stream)
        ms.adjoint_backward(g)
        e2.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), e1.elapsed_time(e2)

    for _ in range(args.warmup):
        once()
    f, b = zip(*[once() for _ in range(args.steps)])
    fwd, bwd = statistics.median(f), statistics.median(b)
    out = {"metric": "adjoint cost: backward / forward device time", "value": bwd / fwd, "unit": "ratio",
           "higher_is_better": False, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
           "dtype": args.precision, "data": "synthetic",
           "config": {"workload": f"c5: {inst.xnumx}x{inst.ynumy} nodes, {inst.marknum} markers, {nsteps} steps, "
                                  f"checkpoint every {every}, 8 modes"},
           "forward_ms": fwd, "backward_ms": bwd,
           "forward_marker_updates_per_s": inst.marknum * nsteps / (fwd / 1e3)}
    print(json.dumps(out))
    ms.close()


def run_e2e(ms, inst, args, stream) -> dict:
    """The drop-in call sequence with host buffers, every step: grid (vx, vy, pr)
    and markers (x, y, T, eta, type) host->device from pinned memory, movemark +
    ronurecalc, then markers (x, y, T, p) and all nine node fields device->host.
    Markers cross in the reference's own FP32 storage (headmart.c:122-125)
    through i2g_set_markers_f32 / i2g_get_markers_f32, as a reference host would
    pass them; node fields are FP64 (headmart.c:87-99)."""
    import ctypes as C

    import torch

    from i2elvis_planet_b200 import abi
    nm, nn = inst.marknum, inst.nodenum

    def pinned(a, dtype):
        t = torch.empty(a.shape[0], dtype=dtype, pin_memory=True)
        t.numpy()[:] = a
        return t.numpy()

    fx, fy, fT, fe = (pinned(a.astype(np.float32), torch.float32) for a in (inst.x, inst.y, inst.T, inst.eta))
    ht = pinned(inst.mtype, torch.int8)
    gvx, gvy, gpr = (pinned(inst.grid[k], torch.float64) for k in ("vx", "vy", "pr"))
    ox, oy, oT, op = (pinned(np.zeros(nm, np.float32), torch.float32) for _ in range(4))
    nodes = [pinned(np.zeros(nn), torch.float64) for _ in range(9)]
    d = abi.dptr
    fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
    L = ms.lib
    h2d = 8 * (inst.xnumx + inst.ynumy) + 3 * 8 * nn + (4 * 4 + 1) * nm
    d2h = 4 * 4 * nm + 9 * 8 * nn

    def one(timesum):
        ms._check(L.i2g_set_grid(ms.h, d(inst.gx), d(inst.gy), d(gvx), d(gvy), d(gpr), *([None] * 8)), "set_grid")
        ms._check(L.i2g_set_markers_f32(ms.h, nm, fp(fx), fp(fy), fp(fT), fp(fe), ht.ctypes.data_as(C.c_char_p)),
                  "set_markers_f32")
        ms._check(L.i2g_movemark(ms.h, inst.timestep, timesum, 0), "movemark")
        ms._check(L.i2g_ronurecalc(ms.h, timesum, 0), "ronurecalc")
        ms._check(L.i2g_get_markers_f32(ms.h, nm, fp(ox), fp(oy), fp(oT), None, fp(op)), "get_markers_f32")
        ms._check(L.i2g_get_nodes(ms.h, *[d(a) for a in nodes]), "get_nodes")

    def resident(timesum):
        # markers resident on the device (the shim's I2G_SHIM_RESIDENT mode): per
        # step the Stokes solve's vx, vy, pr go up and the node fields come down
        ms._check(L.i2g_set_grid(ms.h, d(inst.gx), d(inst.gy), d(gvx), d(gvy), d(gpr), *([None] * 8)), "set_grid")
        ms._check(L.i2g_movemark(ms.h, inst.timestep, timesum, 0), "movemark")
        ms._check(L.i2g_ronurecalc(ms.h, timesum, 0), "ronurecalc")
        ms._check(L.i2g_get_nodes(ms.h, *[d(a) for a in nodes]), "get_nodes")

    def timed(fn):
        fn(inst.timesum)  # warm-up
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e0.record(stream)
        for s in range(args.e2e_steps):
            fn(inst.timesum + s * inst.timestep)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), time.perf_counter() - t0

    dev_ms, wall = timed(one)
    rdev_ms, rwall = timed(resident)
    h2d_r = 8 * (inst.xnumx + inst.ynumy) + 3 * 8 * nn
    d2h_r = 9 * 8 * nn
    return {"value": nm * args.e2e_steps / (dev_ms / 1e3), "unit": "marker updates/s",
            "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "steps": args.e2e_steps,
            "ms_per_step": dev_ms / args.e2e_steps, "host_wall_ms_per_step": 1e3 * wall / args.e2e_steps,
            "host_arrays": "markers FP32 (reference storage), nodes FP64, pinned",
            "resident": {"value": nm * args.e2e_steps / (rdev_ms / 1e3), "unit": "marker updates/s",
                         "h2d_bytes_per_step": h2d_r, "d2h_bytes_per_step": d2h_r,
                         "ms_per_step": rdev_ms / args.e2e_steps,
                         "host_wall_ms_per_step": 1e3 * rwall / args.e2e_steps,
                         "host_arrays": "markers resident on the device; grid vx, vy, pr up and the nine "
                                        "node fields down every step, FP64, pinned"}}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c3", choices=["c1", "c2", "c3", "c4", "c5", "p6"])
    ap.add_argument("--ninst", type=int, default=64)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--cpu-sample", type=int, default=2_000_000)
    ap.add_argument("--skip-cpu-baseline", action="store_true")
    ap.add_argument("--skip-error", action="store_true",
                    help="leave out the mixed-vs-FP64 and mixed-vs-reference error report")
    ap.add_argument("--ref-procs", type=int, default=32)
    ap.add_argument("--table", action="store_true",
                    help="densimod 2: the workload's markers on the P-T table path (seeded table)")
    ap.add_argument("--prn", action="store_true",
                    help="also time the output file's marker section (device codec) at the workload")
    ap.add_argument("--thermal", action="store_true",
                    help="also time titerate()'s marker temperature update at the workload")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        run_reference_arm(args)
    elif args.workload == "c4":
        # the streams strategy runs 64 streams side by side: give the process
        # the most host-to-device work queues (a per-process setting, read when
        # CUDA initialises in this process)
        os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
        run_batch(args)
    elif args.workload == "c5":
        run_adjoint_bench(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
