"""The mixed form's fused step: movemark with every marker's averaging record
into the buckets of its new cell, then one kernel that sums the buckets and
finishes the nodes.  Its sums are exact (the terms rounded to a quantum fixed per
call), so node fields do not depend on the order the records arrive in.

Bars (every call through the C ABI):
  * node fields within 1e-6 normwise (max|d| / max|ref|) of the FP64 form and of
    the general mixed path (canonical-order sums; its w0 = 1 - w1 is rounded to
    FP32, the fused records' is exact, so the two differ at the 1e-7 level);
  * marker positions within 1e-6 of a cell of the general mixed path (the same
    up to rounding: on a uniform grid the fused step finds cells by arithmetic),
    temperatures equal;
  * node fields bitwise equal across runs and across a permuted marker order.
"""
import numpy as np
import pytest

import variants
from i2elvis_planet_b200 import abi, lib, synth

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-6
TOL_GENERAL = 1e-6


def normwise(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def run(inst, precision=abi.PREC_MIXED, fused=True, nsteps=None, update_visc=False):
    ms = lib.MarkerStep.from_instance(inst, precision=precision)
    ms.set_fused(fused)
    ms.set_marker_extras(tmax=inst.tmax, hi=inst.hi if np.any(inst.hi) else None)
    ts = inst.timesum
    for _ in range(inst.nsteps if nsteps is None else nsteps):
        ms.movemark(inst.timestep, ts, update_visc=update_visc)
        ms.ronurecalc(ts, track_tmax=True)
        ts += inst.timestep
    mk = ms.get_markers(with_tmax=True)
    nodes = ms.get_nodes()
    info = ms.fused_info()
    st = ms.stats()
    ms.close()
    return mk, nodes, info, st


def check_against(inst, nsteps=None, update_visc=False, expect_fused=True, tol_general=TOL_GENERAL):
    mk, nodes, info, st = run(inst, nsteps=nsteps, update_visc=update_visc)
    assert (info["fused_moves"] > 0) == expect_fused, info
    mg, ng, ig, sg = run(inst, fused=False, nsteps=nsteps, update_visc=update_visc)
    assert ig["fused_moves"] == 0
    m64, n64, _, _ = run(inst, precision=abi.PREC_FP64, nsteps=nsteps, update_visc=update_visc)
    # markers: on a uniform grid the fused step finds cells and offsets by
    # arithmetic and takes the later RK4 stages from the quarter-cell forms
    # instead of the stencil tables, so positions and pressure agree with the
    # general mixed path to rounding; temperatures are the same except where a
    # rounding puts a marker on the other side of the box edge
    cell = min(np.diff(inst.gx).min(), np.diff(inst.gy).min())
    for f in ("x", "y"):
        assert np.abs(mk[f] - mg[f]).max() <= 1e-6 * cell, f
    assert normwise(mk["p"], mg["p"]) <= 1e-6
    edge = np.minimum.reduce([np.abs(mg["x"]), np.abs(mg["y"]), np.abs(mg["x"] - inst.xsize),
                              np.abs(mg["y"] - inst.ysize)]) <= 1e-6 * cell
    for f in ("T", "tmax"):
        bad = mk[f] != mg[f]
        assert not bad.any() or edge[bad].all(), f
    for k in synth.NODE_OUT:
        assert normwise(nodes[k], ng[k]) <= tol_general, (k, normwise(nodes[k], ng[k]))
        assert normwise(nodes[k], n64[k]) <= TOL_FP64, (k, normwise(nodes[k], n64[k]))
    assert st.markers_averaged == sg.markers_averaged
    assert st.numin == sg.numin or abs(st.numin - sg.numin) <= tol_general * abs(sg.numin)
    return mk, nodes, info


def test_fused_c1_and_c2():
    """C1 (101^2, one step) and C2 (401^2, ten steps): the fused path runs (the
    grid is uniform, three rock types) and agrees with the general mixed path and
    the FP64 form."""
    _, _, info = check_against(synth.make_config("c1"))
    assert info["uniform_grid"] == 1 and info["type_slots"] == 3
    check_against(synth.make_config("c2"), nsteps=4)


@pytest.mark.parametrize("name", ["default", "edges", "outgrid1", "outgrid2", "gridmod2", "nonuniform", "euler", "markim",
                                  "visc0", "visc2", "mu", "strain_reinject"])
def test_fused_variants(name):
    """The parity variants the fused path takes: markers on grid lines and box
    edges, outgrid 1/2, gridmod 2, a nonuniform grid (line tables instead of
    arithmetic), Euler steps, viscmod 0/2, a viscosity override, markers without
    their own viscosity (viscalc at the new position)."""
    inst = variants.variant(name)
    if name == "outgrid2":
        # outgrid 2 zeroes the velocity along a wall once a marker is outside
        # (markmart.c:101-105); a marker planted exactly on a wall, where the flow
        # has vx ~ 0, leaves or stays by the sign of a rounding-level velocity,
        # which two different FP32 evaluations need not share.  Here the wall
        # markers start 1e-3 of a cell outside (the FP64 parity tests keep them on
        # the wall, bit for bit against the reference).
        d = 1e-3 * min(np.diff(inst.gx).min(), np.diff(inst.gy).min())
        for a, L in (("x", inst.xsize), ("y", inst.ysize)):
            v = getattr(inst, a)
            v[v == 0.0] = -d
            v[v == L] = L + d
    check_against(inst, update_visc=bool(variants.move_flags(inst)))


def test_fused_strain_update():
    """movemark's viscosity update (strain rates and stresses set) on the fused path."""
    inst = variants.variant("strain")
    check_against(inst, update_visc=True)


def test_fused_bitwise_across_runs_and_storage_order():
    """Exact sums: the same node fields, bit for bit, for two runs and for the
    markers handed over in another order."""
    inst = synth.make_config("c1", nsteps=3)
    _, n1, _, _ = run(inst)
    _, n2, _, _ = run(inst)
    perm = np.argsort(synth.rng_u64(77, 3, inst.marknum), kind="stable")
    m3, n3, _, _ = run(synth.subset(inst, perm))
    m1, _, _, _ = run(inst)
    for k in synth.NODE_OUT:
        np.testing.assert_array_equal(n2[k], n1[k], err_msg=k)
        np.testing.assert_array_equal(n3[k], n1[k], err_msg=k)
    np.testing.assert_array_equal(m3["x"], m1["x"][perm])


def test_fused_reset_waits_for_ronurecalc():
    """The sticky-air temperature reset belongs to ronurecalc: after a fused
    movemark the markers still hold their temperatures; after the ronurecalc
    they hold what the general path gives."""
    inst = synth.make_config("micro", nsteps=1)
    air = inst.mtype < 2
    inst.T[air] = 400.0  # air away from the ambient 150 K
    outs = []
    for fused in (True, False):
        ms = lib.MarkerStep.from_instance(inst, precision=abi.PREC_MIXED)
        ms.set_fused(fused)
        ms.movemark(inst.timestep, inst.timesum)
        before = ms.get_markers(fields=("T",))["T"]
        ms.movemark(inst.timestep, inst.timesum)
        ms.ronurecalc(inst.timesum)
        after = ms.get_markers(fields=("T",))["T"]
        outs.append((before, after, ms.get_nodes(), ms.fused_info()))
        ms.close()
    (b1, a1, n1, i1), (b0, a0, n0, _) = outs
    assert i1["fused_moves"] == 2
    np.testing.assert_array_equal(b1, b0)
    np.testing.assert_array_equal(a1, a0)
    assert (a1[air] != b1[air]).any()
    for k in synth.NODE_OUT:
        assert normwise(n1[k], n0[k]) <= TOL_GENERAL, k


def converging(inst, frac=0.9):
    """A velocity field that carries every marker frac of the way to the box
    centre in one step: thousands of markers end in a few cells."""
    g = dict(inst.grid)
    n = inst.xnumx
    xm = np.concatenate([0.5 * (inst.gx[1:] + inst.gx[:-1]), [inst.gx[-1]]])
    ym = np.concatenate([0.5 * (inst.gy[1:] + inst.gy[:-1]), [inst.gy[-1]]])
    X = np.repeat(inst.gx, n).reshape(n, n)   # vx nodes: (gx[m1], ymid[m2])
    Ym = np.tile(ym, n).reshape(n, n)
    Xm = np.repeat(xm, n).reshape(n, n)       # vy nodes: (xmid[m1], gy[m2])
    Y = np.tile(inst.gy, n).reshape(n, n)
    c = inst.xsize / 2
    g["vx"] = (-frac * (X - c) / inst.timestep).reshape(-1)
    g["vy"] = (-frac * (Y - c) / inst.timestep).reshape(-1)
    del Ym, Xm
    out = inst.copy()
    out.grid = g
    return out


def test_fused_full_buckets_overflow_then_grow():
    """Markers crowding into a few cells overflow their buckets: the overflow list
    keeps the sums exact (within the bars), and the next movemark enlarges the
    buckets."""
    inst = converging(synth.make_config("micro", nsteps=1))
    mk, nodes, info = check_against(inst, nsteps=2)
    assert info["bucket_growths"] >= 1, info


def test_fused_sparse_nodes_take_the_guard():
    """One marker per cell near its upper corner, and 1000 markers crowded into
    one cell: the crowded cell sets a coarse quantum for the call, and the nodes
    of the left column and the bottom row see weights of about 1e-5 only, which
    that quantum resolves to less than 1e-9; they are recomputed with quanta of
    their own."""
    inst = synth.make_config("micro", nsteps=1)
    n = inst.xnumx - 1
    m1 = np.repeat(np.arange(n), n)
    m2 = np.tile(np.arange(n), n)
    u = synth.rng_uniform(4242, 1, n * n + 1000)
    w = synth.rng_uniform(4242, 2, 1000)
    dx = inst.gx[1] - inst.gx[0]
    sub = synth.subset(inst, np.arange(n * n + 1000))
    x = inst.gx[m1] + (1.0 - 1e-5 * (1 + u[:n * n])) * dx
    y = inst.gy[m2] + (1.0 - 1e-5 * (2 - u[:n * n])) * dx
    cx = inst.gx[10] + (0.05 + 0.9 * u[n * n:]) * dx
    cy = inst.gy[12] + (0.05 + 0.9 * w) * dx
    sub.x = np.concatenate([x, cx])
    sub.y = np.concatenate([y, cy])
    sub.grid = dict(inst.grid)
    sub.grid["vx"] = np.zeros_like(inst.grid["vx"])
    sub.grid["vy"] = np.zeros_like(inst.grid["vy"])
    check_against(sub)


def test_fused_more_types_take_the_general_path():
    """Five averaged rock types are more than the fused path's four slots."""
    inst = synth.make_config("micro", nsteps=1)
    inst.mtype = inst.mtype.copy()
    inst.mtype[::7] = 9
    inst.mtype[::11] = 1
    assert len(set(int(t) for t in inst.mtype if t < 50)) == 5
    check_against(inst, expect_fused=False)
