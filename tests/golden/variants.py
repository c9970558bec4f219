"""Small parity cases that exercise every supported branch of the marker step.

Each variant is the 21x21 'micro' planetesimal with one reference mode switched
or one kind of edge input planted.  make_golden.py runs the compiled reference on
each and stores its outputs; the CPU tests pin the oracle to them and the GPU
tests compare the CUDA path with both.
"""
from __future__ import annotations

import numpy as np

from i2elvis_planet_b200 import synth


def _base(nsteps=2, seed_instance=0, **kw):
    return synth.make_config("micro", instance=seed_instance, nsteps=nsteps, **kw)


def _edge_markers(inst, rng_stream=11):
    """Plant markers exactly on grid lines, on cell midlines, on the box edges and
    outside the box (the bisection tie-break of markmart.c:1061, the staggered-stencil
    switch of markmart.c:1406/1431/1514 and the clamps of markmart.c:1389)."""
    gx, gy = inst.gx, inst.gy
    L = inst.xsize
    pts = []
    for m in (0, 1, 5, 10, gx.size - 2, gx.size - 1):
        pts.append((gx[m], gy[min(m + 1, gy.size - 1)] * 0.999))
        pts.append(((gx[m] + gx[min(m + 1, gx.size - 1)]) / 2.0, gy[3]))
        pts.append((gx[4], (gy[m] + gy[min(m + 1, gy.size - 1)]) / 2.0))
    pts += [(0.0, 0.0), (L, L), (0.0, L / 3), (L, L / 2), (-1e3, L / 2), (L + 5e3, L / 3), (L / 2, -2e3),
            (L / 3, L + 1e3), (-1e3, -1e3)]
    pts = np.array(pts)
    k = pts.shape[0]
    idx = np.arange(k) * (inst.marknum // k)
    inst.x[idx] = pts[:, 0]
    inst.y[idx] = pts[:, 1]
    return inst


def with_table(i, hirschmann=False):
    """densimod 2 on instance i (synth.with_table)."""
    return synth.with_table(i, hirschmann=hirschmann)


def variant(name: str) -> synth.Instance:
    if name == "default":
        return _base()
    if name == "euler":
        i = _base()
        i.flags["markmod"] = 1
        return i
    if name == "visc0":
        i = _base()
        i.flags["viscmod"] = 0
        return i
    if name == "visc2":
        i = _base()
        i.flags["viscmod"] = 2
        i.scal["nucontr"] = 1e-3   # contrast limit from the top (markmart.c:1002)
        return i
    if name == "dens1":
        i = _base()
        i.flags["densimod"] = 1
        for t in (0, 5, 7):
            i.types["markaa"][t] = 3e-5
            i.types["markbb"][t] = 2e-5
            i.types["markkf"][t] = 150.0
            i.types["markkp"][t] = 2e-6
        return i
    if name == "edges":
        i = _edge_markers(_base())
        i.flags["outgrid"] = 0
        # wall outflow: add a uniform drift so markers leave the box
        i.grid["vx"] = i.grid["vx"] + 0.6e-9
        i.grid["vy"] = i.grid["vy"] - 0.4e-9
        return i
    if name == "outgrid1":
        i = _edge_markers(_base())
        i.flags["outgrid"] = 1
        i.grid["vx"] = i.grid["vx"] + 0.6e-9
        return i
    if name == "outgrid2":
        i = _edge_markers(_base())
        i.flags["outgrid"] = 2
        i.grid["vy"] = i.grid["vy"] + 0.5e-9
        return i
    if name == "strain":
        # nonzero strain-rate/stress fields, ductile/brittle/Peierls parameters and
        # viscosity recomputed by movemark (UPDATE_VISC) and by ronurecalc for eta <= 0
        i = _base()
        n = i.nodenum
        gx, gy = np.meshgrid(i.gx, i.gy, indexing="ij")
        s = (np.sin(2 * np.pi * gx / i.xsize) * np.cos(np.pi * gy / i.ysize)).reshape(-1)
        c = (np.cos(3 * np.pi * gx / i.xsize) * np.sin(2 * np.pi * gy / i.ysize)).reshape(-1)
        i.grid["exx"] = 1e-14 * s
        i.grid["eyy"] = -1e-14 * s
        i.grid["exy"] = 3e-15 * c
        i.grid["sxx"] = 2e7 * s
        i.grid["syy"] = -2e7 * s
        i.grid["sxy"] = 5e6 * c + 1e6
        i.grid["ga"] = 0.05 + 0.01 * c
        T = i.types
        # silicate: power law with P-T dependence (branch D) + brittle
        T["marknu"][5] = 3.98e16; T["markdh"][5] = 5.32e5; T["markdv"][5] = 0.8
        T["markss"][5] = 3e7; T["markmm"][5] = 3.5; T["markll"][5] = 1.0
        T["marka0"][5] = 1e8; T["markb0"][5] = 0.3; T["marks0"][5] = 0.0; T["marks1"][5] = 9.1e9
        # iron: Newtonian P-T dependent (branch B) + Peierls
        T["marknu"][7] = 1.26e11; T["markdh"][7] = 5.32e5; T["markdv"][7] = 0.1
        T["marks0"][7] = 6.3e-5; T["marks1"][7] = 9.1e9
        # air: constant Newtonian (branch A)
        T["marknu"][0] = 1e19
        i.flags["viscmod"] = 1
        i.flags["_update_visc"] = 1
        i.hi[::11] = 0.995   # recent impact: reduced brittle strength (markmart.c:1886-1889)
        return i
    if name == "strain_reinject":
        # re-injected zero viscosity makes ronurecalc call viscalc itself (markmart.c:321-334)
        i = variant("strain")
        i.flags.pop("_update_visc")
        i.eta[::7] = 0.0
        return i
    if name == "mu":
        i = _base()
        mu = np.zeros(i.nodenum)
        mu[::17] = 3e21
        i.grid["mu"] = mu
        i.nodes["nu"][:] = 1e21
        i.nodes["nd"][:] = 2e21
        i.nodes["tk"][:] = 999.0
        return i
    if name == "gridmod2":
        i = _base()
        i.flags["gridmod"] = 2
        return i
    if name == "molten":
        # molten silicate / iron / chondritic types with the conductivity branch of
        # markmart.c:509-610 active (timesum > core_form_time) and stale melt fractions
        i = _base()
        u = synth.rng_uniform(777, 1, i.marknum)
        inside = i.mtype != 0
        i.mtype[inside & (u < 0.15)] = 25
        i.mtype[inside & (u >= 0.15) & (u < 0.25)] = 15
        i.mtype[inside & (u >= 0.25) & (u < 0.3)] = 8
        T = i.types
        for t in (25, 15, 8):
            T["markro"][t] = {25: 2900.0, 15: 3000.0, 8: 7500.0}[t]
            T["markkt"][t] = 3.0
            T["markbb"][t] = 3e-5
        T["markbb"][5] = 3e-5
        T["markbb"][7] = 1e-5
        i.grid["ga"] = np.full(i.nodenum, 0.08)
        i.scal["core_form_time"] = 0.0
        i.scal["eps21"] = 0.5
        i.scal["eps50"] = 0.0
        return i
    if name == "molten_fe":
        i = variant("molten")
        i.scal["eps21"] = 0.8
        i.scal["eps50"] = 1.0
        return i
    if name in ("td", "td_hirschmann"):
        return with_table(_base(), hirschmann=name == "td_hirschmann")
    if name == "porous":
        # porous solid silicate: cold pressing below 700 K and hot sintering above
        # (markmart.c:362-466), both porosity regimes (above and below 10 %), and
        # porosity outside the range the branch takes
        i = _base()
        u = synth.rng_uniform(780, 1, i.marknum)
        sil = i.mtype == 5
        i.por = np.where(sil, 0.02 + 0.9 * u, 0.0)
        i.mtype[sil & (u > 0.8)] = 6
        hot = sil & (synth.rng_uniform(780, 2, i.marknum) < 0.5)
        i.T[hot] = 700.0 + 900.0 * synth.rng_uniform(780, 3, int(hot.sum()))
        i.scal["por_init"] = 0.5
        i.timestep = 3.15576e13  # 1 Myr: porosity changes of a few percent at the hot end
        return i
    if name in ("mag_dynamo0", "mag_dynamo1"):
        # magnetisation (markmart.c:651-744): silicate temperatures across the
        # Curie points of magnetite (851.16 K) and hematite (948.16 K), every
        # previous state 0..3, the dynamo off or on; the first processed marker
        # (air) assigns the carried magnetisation time
        # one step with the dynamo on: the first step is where new magnetisation
        # times are assigned (after it the states are 1 or 2 and assign nothing)
        i = _base(nsteps=1 if name == "mag_dynamo1" else 2)
        n = i.marknum
        sil = i.mtype == 5
        i.mtype[sil & (synth.rng_uniform(782, 1, n) < 0.3)] = 6
        hot = np.isin(i.mtype, (5, 6))
        i.T[hot] = 700.0 + 400.0 * synth.rng_uniform(782, 2, int(hot.sum()))
        i.mg_old = (4.0 * synth.rng_uniform(782, 3, n)).astype(np.int8)
        i.mg_time = 10.0 * synth.rng_uniform(782, 4, n)
        i.flags["dynamo"] = 1 if name == "mag_dynamo1" else 0
        i.timesum = 3.15576e13 * 2.5  # 2.5 Myr
        assert i.mtype[0] == 0
        return i
    if name == "unlisted_type":
        # rock types 1 and 3 are outside the radiogenic-heating lists of
        # markmart.c:749-837; the reference keeps the previous marker's heating for
        # them, this build uses 0 (only 'ht' may differ, and only where they contribute)
        i = _base()
        u = synth.rng_uniform(778, 1, i.marknum)
        i.mtype[(i.mtype == 0) & (u < 0.3)] = 1
        i.mtype[(i.mtype == 5) & (u < 0.1)] = 3
        return i
    if name == "markim":
        i = _base()
        i.markim[7] = 1
        return i
    if name == "nonuniform":
        i = _base()
        n = i.xnumx
        t = np.linspace(0.0, 1.0, n)
        g = i.xsize * (t + 0.08 * np.sin(2 * np.pi * t))
        g[0], g[-1] = 0.0, i.xsize
        i.gx = g.copy()
        i.gy = (i.ysize * (t - 0.05 * np.sin(2 * np.pi * t)))
        i.gy[0], i.gy[-1] = 0.0, i.ysize
        modes = i.modes
        mvx, mvy = synth.stream_velocity(i.gx, i.gy, modes, i.amps)
        i.grid["vx"] = i.amps @ mvx
        i.grid["vy"] = i.amps @ mvy
        return i
    raise KeyError(name)


NAMES = ("default", "euler", "visc0", "visc2", "dens1", "edges", "outgrid1", "outgrid2", "strain",
         "strain_reinject", "mu",
         "gridmod2", "molten", "molten_fe", "markim", "nonuniform", "unlisted_type", "td", "td_hirschmann",
         "porous", "mag_dynamo0", "mag_dynamo1")

# fields in which a variant legitimately differs from the reference (declared deviations)
DEVIATIONS = {"unlisted_type": ("ht",), "td": ("ht",), "td_hirschmann": ("ht",)}  # crust types 11/12/31/32


def move_flags(inst) -> int:
    return 1 if inst.flags.get("_update_visc") else 0


# -- titerate()'s marker temperature update (heatmart.c:514-697) ---------------
def thermal_variant(name: str):
    """(instance, tk_new, heatdif) of a thermal-update case: node T before the
    solve in inst.nodes['tk'], after it tk_new (synth.thermal_fields)."""
    if name == "thermal":
        i = _base()
        f = synth.thermal_fields(i, fluid_frac=0.1, cold_frac=0.05)
        return i, f["tk_new"], 1.0
    if name == "thermal_nodif":
        i = _base()
        f = synth.thermal_fields(i, fluid_frac=0.1, cold_frac=0.05)
        return i, f["tk_new"], 0.0
    if name == "thermal_edges":
        # markers on grid lines, cell midlines, the box edges and outside it: the
        # strict inside test of heatmart.c:527/541 and the search tie-break
        i = _edge_markers(_base())
        f = synth.thermal_fields(i, fluid_frac=0.1, cold_frac=0.05)
        return i, f["tk_new"], 1.0
    if name == "thermal_strong":
        # nonuniform grid, large diffusion exponent (the -150 floor of heatmart.c:593)
        i = variant("nonuniform")
        f = synth.thermal_fields(i, fluid_frac=0.05, cold_frac=0.1, dT=200.0)
        return i, f["tk_new"], 5e4
    raise KeyError(name)


THERMAL_NAMES = ("thermal", "thermal_nodif", "thermal_edges", "thermal_strong")


# -- the marker section of the reference's output file (saver/loader) ---------------
def prn_instance():
    """The micro planetesimal with every field the output file carries set:
    grain size, accretion time (also what loader() puts into the magnetisation
    fields), magnetisation state and time across the char range and beyond it,
    maximum temperature, impact time and porosity."""
    i = _base()
    n = i.marknum
    i.gr = 100.0 * synth.rng_uniform(5, 1, n)
    i.acc = 300.0 * synth.rng_uniform(5, 2, n) - 50.0
    i.mg_time = 400.0 * synth.rng_uniform(5, 3, n) - 200.0
    i.mg_time[::97] = 3e9          # beyond the int range
    i.mg_old = (4.0 * synth.rng_uniform(5, 4, n)).astype(np.int8)
    i.tmax = i.T + 5.0
    i.hi = synth.rng_uniform(5, 5, n)
    i.por = np.where(i.mtype == 5, 0.9 + 0.1 * synth.rng_uniform(5, 6, n), 0.0)
    return i
