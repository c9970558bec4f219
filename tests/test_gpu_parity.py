"""Parity of the CUDA marker step with the compiled reference and the oracle.

Every call goes through the C ABI (libi2g.so via ctypes).  Bars:
  * FP64 form, marker outputs (x, y, T, p, tmax): bit-identical to the reference
    built with FP64 marker storage (SHA-256 of the full arrays in the fixtures);
    viscosity from viscalc() within 1e-12 (libm pow/exp/log differ in the last bit).
  * FP64 form, node fields: bit-identical to the oracle summed in the CUDA order
    for every field without a transcendental function; <= 1e-12 relative to the
    reference (summation order) for all.
  * Mixed form: node fields within 1e-6 normwise (max|d| / max|ref|) of the FP64 form.
"""
import hashlib
import os

import numpy as np
import pytest

import variants
from i2elvis_planet_b200 import abi, lib, synth
from oracle import oracle

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
EXACT_NODE = ("ro", "et", "cp", "ht", "tk", "po")   # no libm call between marker and node
TOL_NODE = 1e-12
# The table path (densimod 2) adds to the expansion term a central difference of
# latent heats over 0.1 % of the pressure (markmart.c:2213-2221): one unit in the
# last place of a solidus fit (libm pow/log) grows about 1e5-fold there.
TOL_TABLE = {"et": 1e-9}


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def gold(name, kind="ref64"):
    return np.load(os.path.join(GOLD, f"{name}_{kind}.npz"))


def normwise(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def run_gpu(inst, precision=abi.PREC_FP64, with_melt=False):
    mf = variants.move_flags(inst)
    mk, nodes, ms = lib.run_instance(inst, precision=precision, update_visc=bool(mf), track_tmax=True)
    melt = ms.get_melt_state()
    ms.close()
    return (mk, nodes, melt) if with_melt else (mk, nodes)


@pytest.mark.parametrize("name", variants.NAMES)
def test_fp64_matches_reference_and_oracle(name):
    inst = variants.variant(name)
    g = gold(name)
    mk, nodes, melt = run_gpu(inst, with_melt=True)
    # markers: bit-exact (positions, pressure, temperature, max temperature)
    for f in ("x", "y", "T", "p", "tmax"):
        assert digest(mk[f]) == str(g[f"digest_{f}"]), f
    if "digest_mg_old" in g:
        # magnetisation state and time (markmart.c:651-744), with the carried time
        assert digest(mk["mg_old"]) == str(g["digest_mg_old"])
        assert digest(mk["mg_time"]) == str(g["digest_mg_time"])
    if "digest_por" in g:
        # porosity after cold pressing and sintering (markmart.c:362-466): the
        # grain-size Newton iteration calls pow, whose last bit may differ from libm's
        st = int(g["stride"])
        assert np.abs(mk["por"][::st] - g["m_por"]).max() <= 1e-12
    table = "digest_type" in g
    if table:
        # densimod 2: the melt flips of the marker types, and the melt state the last
        # table marker leaves (the libm of the solidus fits may differ in the last bit)
        assert digest(mk["type"]) == str(g["digest_type"])
        assert np.abs(melt - g["melt"]).max() <= 1e-12 * max(np.abs(g["melt"]).max(), 1.0)
    if name.startswith("strain"):
        ref = g["m_eta"]
        assert normwise(mk["eta"][::int(g["stride"])], ref) <= TOL_NODE
    else:
        assert digest(mk["eta"]) == str(g["digest_eta"])
    dev = variants.DEVIATIONS.get(name, ())
    for k in synth.NODE_OUT:
        if k in dev:
            continue
        tol = TOL_TABLE.get(k, TOL_NODE) if table else TOL_NODE
        assert normwise(nodes[k], g[f"n_{k}"]) <= tol, k
    # node fields: bit-exact against the oracle in the same summation order
    mf = variants.move_flags(inst)
    s = oracle.Oracle(inst).run(order=oracle.ORDER_CELL, eta_reinject=not mf, move_flags=mf)
    exact = ("tk", "po") if table else EXACT_NODE  # the table path calls pow/exp/log for ro, cp, et
    for k in exact:
        np.testing.assert_array_equal(nodes[k], s.nodes[k], err_msg=k)
    for k in synth.NODE_OUT:
        tol = TOL_TABLE.get(k, TOL_NODE) if table else TOL_NODE
        assert normwise(nodes[k], s.nodes[k]) <= tol, k


def test_c1_fp64_matches_reference():
    inst = synth.make_config("c1")
    g = gold("c1")
    mk, nodes = run_gpu(inst)
    for f in ("x", "y", "T", "p", "tmax", "eta"):
        assert digest(mk[f]) == str(g[f"digest_{f}"]), f
    for k in ("ro", "nu", "tk"):
        assert normwise(nodes[k], g[f"n_{k}"]) <= TOL_NODE, k


def test_c1_reference_storage_error():
    """Against the reference's own float-storage build the FP64 path differs only by
    single-precision rounding of positions (about 1e-7 of the box)."""
    inst = synth.make_config("c1")
    g32 = gold("c1", "ref32")
    mk, nodes = run_gpu(inst)
    st = int(g32["stride"])
    assert np.abs(mk["x"][::st] - g32["m_x"]).max() / inst.xsize < 1e-6
    for k in ("ro", "tk"):
        assert normwise(nodes[k], g32[f"n_{k}"]) < 1e-3


def mixed_table_close(nm, n64, types_m, types_64):
    """The mixed form on the table path.  A marker whose temperature lies within
    the FP32 pressure's reach of its solidus (about 1e-4 K) can flip type in one
    form and not the other, which moves its conductivity as a whole; and near zero
    pressure the latent-heat expansion term (a central difference over 0.1 % of
    the pressure, markmart.c:2213-2221) is rounding noise of the enthalpy
    difference in either form.  At most 1e-4 of the markers differ in type; 99.5 %
    of the nodes stay within 1e-6 of the field's largest value."""
    assert (types_m != types_64).mean() <= 1e-4
    for k in synth.NODE_OUT:
        d = np.abs(nm[k] - n64[k]) / max(np.abs(n64[k]).max(), 1e-300)
        assert (d <= 1e-6).mean() >= 0.995, (k, d.max(), int((d > 1e-6).sum()))


@pytest.mark.parametrize("name", ["default", "edges", "molten", "nonuniform", "td", "td_hirschmann", "porous",
                                  "mag_dynamo1"])
def test_mixed_within_1e6_of_fp64(name):
    inst = variants.variant(name)
    mk64, n64 = run_gpu(inst)
    mkm, nmx = run_gpu(inst, precision=abi.PREC_MIXED)
    if inst.td is not None:
        mixed_table_close(nmx, n64, mkm["type"], mk64["type"])
        return
    for k in synth.NODE_OUT:
        assert normwise(nmx[k], n64[k]) <= 1e-6, (k, normwise(nmx[k], n64[k]))


def test_c2_mixed_vs_fp64_ten_steps():
    inst = synth.make_config("c2")
    mk64, n64 = run_gpu(inst)
    mkmx, nmx = run_gpu(inst, precision=abi.PREC_MIXED)
    for k in synth.NODE_OUT:
        assert normwise(nmx[k], n64[k]) <= 1e-6, (k, normwise(nmx[k], n64[k]))
    assert np.abs(mkmx["x"] - mk64["x"]).max() / inst.xsize < 1e-6


def test_c2_fp64_matches_oracle_ten_steps():
    inst = synth.make_config("c2")
    mk, nodes = run_gpu(inst)
    s = oracle.Oracle(inst).run(order=oracle.ORDER_CELL)
    for f in ("x", "y", "T", "p", "tmax"):
        np.testing.assert_array_equal(mk[f], getattr(s, f), err_msg=f)
    for k in EXACT_NODE:
        np.testing.assert_array_equal(nodes[k], s.nodes[k], err_msg=k)
    for k in ("nu", "nd", "kt"):
        assert normwise(nodes[k], s.nodes[k]) <= TOL_NODE, k


def test_deterministic_runs_and_storage_order():
    """Bitwise-identical output across runs; a permuted marker storage order moves
    only rounding (the within-cell order follows the caller index)."""
    inst = synth.make_config("c1")
    mk1, n1 = run_gpu(inst)
    mk2, n2 = run_gpu(inst)
    for k in synth.NODE_OUT:
        np.testing.assert_array_equal(n1[k], n2[k])
    perm = np.argsort(synth.rng_u64(5, 5, inst.marknum), kind="stable")
    p = synth.subset(inst, perm)
    mk3, n3 = run_gpu(p)
    np.testing.assert_array_equal(mk3["x"], mk1["x"][perm])
    for k in synth.NODE_OUT:
        assert normwise(n3[k], n1[k]) <= 1e-13, k


def test_uniform_velocity_is_translation():
    """A uniform velocity field moves every marker by dt*v: bit-identical to the
    oracle's arithmetic and within 1e-14 of the box size of the exact translation (the bilinear
    weights of a constant field sum to one up to rounding)."""
    inst = synth.make_config("micro", nsteps=1)
    inst.grid["vx"][:] = 1e-9
    inst.grid["vy"][:] = -0.5e-9
    inst.flags["outgrid"] = 0
    ms = lib.MarkerStep.from_instance(inst)
    ms.movemark(inst.timestep, inst.timesum)
    mk = ms.get_markers()
    ms.close()
    o = oracle.Oracle(inst)
    s = o.initial_state()
    o.movemark(s, inst.timestep, inst.timesum)
    np.testing.assert_array_equal(mk["x"], s.x)
    np.testing.assert_array_equal(mk["y"], s.y)
    tol = 1e-14 * inst.xsize
    np.testing.assert_allclose(mk["x"], inst.x + inst.timestep * 1e-9, rtol=0, atol=tol)
    np.testing.assert_allclose(mk["y"], inst.y + inst.timestep * -0.5e-9, rtol=0, atol=tol)


def test_constant_property_partition_of_unity():
    inst = synth.make_config("micro", nsteps=1)
    inst.mtype[:] = 5
    inst.T[:] = 1000.0
    _, nodes = run_gpu(inst)
    np.testing.assert_allclose(nodes["ro"], 3300.0, rtol=1e-14)
    np.testing.assert_allclose(nodes["tk"], 1000.0, rtol=1e-14)


def test_errors_are_status_codes():
    inst = synth.make_config("micro")
    ms = lib.MarkerStep.from_instance(inst, upload=False)
    with pytest.raises(lib.I2GError) as e:
        ms.movemark(inst.timestep)
    assert e.value.status == abi.ESTATE
    ms.set_grid(inst.gx, inst.gy, **inst.grid)
    bad = inst.mtype.copy()
    bad[3] = 100
    with pytest.raises(lib.I2GError) as e:
        ms.set_markers(inst.x, inst.y, inst.T, inst.eta, bad)
    assert e.value.status == abi.EUNSUPPORTED
    bad[3] = -2
    with pytest.raises(lib.I2GError) as e:
        ms.set_markers(inst.x, inst.y, inst.T, inst.eta, bad)
    assert e.value.status == abi.EINVAL and "marker 3" in str(e.value)
    with pytest.raises(lib.I2GError) as e:  # a rejected set leaves no markers
        ms.movemark(inst.timestep)
    assert e.value.status == abi.ESTATE
    big = np.zeros(inst.marknum + 1)
    with pytest.raises(lib.I2GError) as e:
        ms.set_markers(big, big, big, big, np.zeros(big.size, np.int8))
    assert e.value.status == abi.ECAPACITY
    gx = inst.gx.copy()
    gx[5] = gx[4]
    with pytest.raises(lib.I2GError) as e:
        ms.set_grid(gx, inst.gy, **inst.grid)
    assert e.value.status == abi.EINVAL
    ms.close()


def test_reference_storage_entry_points():
    """i2g_set_markers_f32 / i2g_get_markers_f32 take the reference's own float
    marker arrays (headmart.c:122-125)."""
    import ctypes as C
    inst = synth.make_config("micro", nsteps=1)
    ms = lib.MarkerStep.from_instance(inst, upload=False)
    ms.set_grid(inst.gx, inst.gy, **inst.grid)
    f = [np.ascontiguousarray(a, dtype=np.float32) for a in (inst.x, inst.y, inst.T, inst.eta)]
    t = np.ascontiguousarray(inst.mtype, dtype=np.int8)
    fp = C.POINTER(C.c_float)
    rc = ms.lib.i2g_set_markers_f32(ms.h, inst.marknum, *[a.ctypes.data_as(fp) for a in f],
                                    t.ctypes.data_as(C.c_char_p))
    assert rc == 0
    ms.n = inst.marknum
    out = [np.empty(inst.marknum, np.float32) for _ in range(5)]
    assert ms.lib.i2g_get_markers_f32(ms.h, inst.marknum, *[a.ctypes.data_as(fp) for a in out]) == 0
    np.testing.assert_array_equal(out[0], f[0])
    np.testing.assert_array_equal(out[2], f[2])
    ms.close()


@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_MIXED], ids=["fp64", "mixed"])
def test_reorder_interval_does_not_change_results(precision):
    """The averaging moves the marker records into cell order only every
    i2g_set_reorder_interval calls and otherwise scatters their contributions in
    place; the sums see the same order either way, so every output is bitwise
    the same for every interval (markers in random storage order, tmax tracked,
    and ronurecalc called twice in a row once)."""
    inst = synth.make_config("c1", permute=True)
    outs = []
    for every in (1, 3, 8):
        ms = lib.MarkerStep.from_instance(inst, precision=precision)
        ms.set_reorder_interval(every)
        ms.set_marker_extras(tmax=inst.tmax)
        ts = inst.timesum
        for s in range(7):
            ms.movemark(inst.timestep, ts)
            ms.ronurecalc(ts, track_tmax=True)
            if s == 4:
                ms.ronurecalc(ts, track_tmax=True)
            ts += inst.timestep
        outs.append((ms.get_markers(fields=("x", "y", "T", "eta", "p"), with_tmax=True), ms.get_nodes(),
                     ms.stats()))
        ms.close()
    (m0, n0, s0) = outs[0]
    for mk, nodes, st in outs[1:]:
        for f in ("x", "y", "T", "eta", "p", "tmax"):
            np.testing.assert_array_equal(mk[f], m0[f], err_msg=f)
        for k in synth.NODE_OUT:
            np.testing.assert_array_equal(nodes[k], n0[k], err_msg=k)
        assert st.markers_averaged == s0.markers_averaged
    with pytest.raises(lib.I2GError):
        lib.MarkerStep.from_instance(synth.make_config("micro"), upload=False).set_reorder_interval(0)


@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_MIXED])
def test_constant_property_path_matches_general_model(precision):
    """A call whose rock properties are per-type constants (densimod 0, no markkf /
    markkp terms, no porosity, before core formation) runs the lean contributions
    kernel, which hands the markers with eta <= 0 (viscosity from viscalc) to the
    general model in a second launch.  Reorder interval 1 runs the general model on
    every call; every output must be bitwise the same, and the lean path must have
    run (one launch more per call)."""
    inst = variants.variant("strain_reinject")
    assert (inst.eta <= 0).any()
    outs, launches = [], []
    for every in (1, 8):
        ms = lib.MarkerStep.from_instance(inst, precision=precision)
        ms.set_fused(False)  # the general path's own kernels (the fused path is tested apart)
        ms.set_reorder_interval(every)
        ms.set_marker_extras(tmax=inst.tmax, hi=inst.hi)
        ms.profile_enable(True)
        ts = inst.timesum
        per_call = []
        for _ in range(3):
            ms.profile_read(reset=True)
            ms.movemark(inst.timestep, ts)
            ms.ronurecalc(ts, track_tmax=True)
            per_call.append(ms.profile_read(reset=True)["launches"])
            ts += inst.timestep
        outs.append((ms.get_markers(fields=("x", "y", "T", "eta", "p"), with_tmax=True), ms.get_nodes()))
        launches.append(per_call)
        ms.close()
    assert launches[1] == [n + 1 for n in launches[0]], launches
    (m0, n0), (m1, n1) = outs
    for f in ("x", "y", "T", "eta", "p", "tmax"):
        np.testing.assert_array_equal(m1[f], m0[f], err_msg=f)
    for k in synth.NODE_OUT:
        np.testing.assert_array_equal(n1[k], n0[k], err_msg=k)


def crowded_instance():
    """The 21x21 micro case with markers crowded into a few cells: about 1000, 150,
    56 and 40 markers in four cells (the other cells keep ~16), so the within-cell
    ranking runs every layout it has (half-warp pairs up to 48 markers, a whole
    warp up to 64, shared memory up to 256, global memory beyond)."""
    inst = synth.make_config("micro", nsteps=2)
    u = synth.rng_uniform(9191, 1, inst.marknum)
    w = synth.rng_uniform(9191, 2, inst.marknum)
    x, y = inst.x.copy(), inst.y.copy()
    start = 0
    for (c1, c2), k in (((2, 2), 1000), ((5, 5), 150), ((8, 8), 56), ((10, 10), 40)):
        sl = slice(start, start + k)
        x[sl] = inst.gx[c1] + (0.05 + 0.9 * u[sl]) * (inst.gx[c1 + 1] - inst.gx[c1])
        y[sl] = inst.gy[c2] + (0.05 + 0.9 * w[sl]) * (inst.gy[c2 + 1] - inst.gy[c2])
        start += k
    inst.x, inst.y = x, y
    return inst


def test_crowded_cells_match_oracle():
    inst = crowded_instance()
    mk, nodes = run_gpu(inst)
    s = oracle.Oracle(inst).run(order=oracle.ORDER_CELL)
    for f in ("x", "y", "T", "p", "tmax"):
        np.testing.assert_array_equal(mk[f], getattr(s, f), err_msg=f)
    for k in EXACT_NODE:
        np.testing.assert_array_equal(nodes[k], s.nodes[k], err_msg=k)
    for k in ("nu", "nd", "kt"):
        assert normwise(nodes[k], s.nodes[k]) <= TOL_NODE, k
    mkm, nm = run_gpu(inst, precision=abi.PREC_MIXED)
    for k in synth.NODE_OUT:
        assert normwise(nm[k], nodes[k]) <= 1e-6, k
    # the crowding held through both steps
    o = oracle.Oracle(inst)
    counts = np.bincount([o.cell_key(a, b) for a, b in zip(s.x, s.y)], minlength=20 * 20)
    assert counts.max() > 256 and ((counts > 64) & (counts <= 256)).any() and ((counts > 48) & (counts <= 64)).any()


def test_table_path_c1_three_steps_matches_oracle():
    """densimod 2 at the 101x101 workload (90,000 markers) over three steps: marker
    types, melt state and nodes against the oracle, in both forms."""
    inst = variants.with_table(synth.make_config("c1", nsteps=3))
    s = oracle.Oracle(inst).run(order=oracle.ORDER_CELL)
    mk, nodes, melt = run_gpu(inst, with_melt=True)
    np.testing.assert_array_equal(mk["type"], s.mtype)
    assert (mk["type"] != inst.mtype).sum() > 1000
    assert np.abs(melt - s.melt).max() <= 1e-12 * max(np.abs(s.melt).max(), 1.0)
    for k in synth.NODE_OUT:
        assert normwise(nodes[k], s.nodes[k]) <= TOL_TABLE.get(k, TOL_NODE), k
    mkm, nm, meltm = run_gpu(inst, precision=abi.PREC_MIXED, with_melt=True)
    mixed_table_close(nm, s.nodes, mkm["type"], s.mtype)


def test_table_path_needs_its_table_and_carries_the_melt_state():
    inst = variants.variant("td")
    ms = lib.MarkerStep(abi.params_from_instance(inst), abi.types_from_instance(inst))
    ms.set_grid(inst.gx, inst.gy, **inst.grid)
    ms.set_nodes(**inst.nodes)
    ms.set_markers(inst.x, inst.y, inst.T, inst.eta, inst.mtype)
    with pytest.raises(lib.I2GError) as e:
        ms.ronurecalc(inst.timesum)
    assert e.value.status == abi.ESTATE
    ms.set_td_table(inst.td)
    np.testing.assert_array_equal(ms.get_melt_state(), [0.5, 0, 0, 0, 0, 0])
    ms.set_melt_state([0.45, 1.0, 0.0, 0.0, 0.0, 0.0])
    ms.ronurecalc(inst.timesum)
    a = ms.get_nodes()
    after = ms.get_melt_state()
    assert 0 < after[0] < 1
    # the starting melt state reaches the molten markers before the first table marker only
    o = oracle.Oracle(inst)
    st = o.initial_state()
    st.melt[:] = [0.45, 1.0, 0.0, 0.0, 0.0, 0.0]
    o.ronurecalc(st, inst.timesum, order=oracle.ORDER_CELL)
    for k in synth.NODE_OUT:
        assert normwise(a[k], st.nodes[k]) <= TOL_TABLE.get(k, TOL_NODE), k
    np.testing.assert_allclose(after, st.melt, rtol=1e-12, atol=0)
    ms.close()


def test_porosity_c1_matches_oracle():
    """Cold pressing and sintering at the 101x101 workload over three steps: the
    porosity every marker ends with and the nodes, against the oracle."""
    inst = synth.make_config("c1", nsteps=3)
    u = synth.rng_uniform(781, 1, inst.marknum)
    sil = inst.mtype == 5
    inst.por = np.where(sil, 0.02 + 0.9 * u, 0.0)
    hot = sil & (synth.rng_uniform(781, 2, inst.marknum) < 0.5)
    inst.T[hot] = 700.0 + 900.0 * synth.rng_uniform(781, 3, int(hot.sum()))
    inst.scal["por_init"] = 0.5
    s = oracle.Oracle(inst).run(order=oracle.ORDER_CELL)
    mk, nodes = run_gpu(inst)
    assert (s.por != inst.por).sum() > 1000
    assert np.abs(mk["por"] - s.por).max() <= 1e-12
    for k in synth.NODE_OUT:
        assert normwise(nodes[k], s.nodes[k]) <= TOL_NODE, k


def test_magnetisation_c1_matches_oracle():
    """Magnetisation at the 101x101 workload over three steps, dynamo on: the
    states and times of every marker against the oracle, in both forms (the
    states depend on temperature thresholds the mixed form also meets exactly:
    temperatures are FP64 in both)."""
    inst = synth.make_config("c1", nsteps=3)
    n = inst.marknum
    hot = np.isin(inst.mtype, (5, 6))
    inst.T[hot] = 700.0 + 400.0 * synth.rng_uniform(783, 1, int(hot.sum()))
    inst.mg_old = (4.0 * synth.rng_uniform(783, 2, n)).astype(np.int8)
    inst.mg_time = 10.0 * synth.rng_uniform(783, 3, n)
    inst.flags["dynamo"] = 1
    inst.timesum = 3.15576e13 * 2.5
    s = oracle.Oracle(inst).run(order=oracle.ORDER_CELL)
    for prec in (abi.PREC_FP64, abi.PREC_MIXED):
        mk, nodes = run_gpu(inst, precision=prec)
        np.testing.assert_array_equal(mk["mg_old"], s.mg_old)
        np.testing.assert_array_equal(mk["mg_time"], s.mg_time)
