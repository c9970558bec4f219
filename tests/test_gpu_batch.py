"""The batched step (one launch per phase over many instances, replayed from a
CUDA graph) reproduces each instance's own single-context result bit for bit,
whatever launch shape the autotuner picks."""
import numpy as np
import pytest

from i2elvis_planet_b200 import abi, lib, synth

pytestmark = pytest.mark.gpu


def small_batch():
    out = []
    for i, (n, k, r) in enumerate([(31, 3, 120e3), (47, 5, 200e3), (23, 4, 80e3), (61, 6, 230e3)]):
        out.append(synth.make_instance(f"b{i}", n=n, k=k, nsteps=3, seed=5000 + i, r_disk=r,
                                       vmax=10.0 ** (-9.5 + 0.5 * i), extra_modes=2))
    return out


def single(inst, precision, nsteps, fused=False):
    """One context's own steps; fused=False keeps the mixed form on the general
    path, whose kernels the fused batch strategy runs over all instances."""
    ms = lib.MarkerStep.from_instance(inst, precision=precision)
    ms.set_fused(fused)
    ts = inst.timesum
    for _ in range(nsteps):
        ms.movemark(inst.timestep, ts)
        ms.ronurecalc(ts)
        ts += inst.timestep
    mk, nd = ms.get_markers(), ms.get_nodes()
    ms.close()
    return mk, nd


@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_MIXED])
def test_batch_equals_single_instances(precision):
    insts = small_batch()
    steps = [lib.MarkerStep.from_instance(i, precision=precision) for i in insts]
    b = lib.Batch(steps)
    dt = np.array([i.timestep for i in insts])
    ts = np.array([i.timesum for i in insts])
    b.step(dt, ts, 3)
    b.sync()
    for inst, ms in zip(insts, steps):
        mk, nd = single(inst, precision, 3)
        mk_b, nd_b = ms.get_markers(), ms.get_nodes()
        for f in ("x", "y", "T", "p"):
            np.testing.assert_array_equal(mk_b[f], mk[f], err_msg=f)
        for kf in synth.NODE_OUT:
            np.testing.assert_array_equal(nd_b[kf], nd[kf], err_msg=kf)
    np.testing.assert_allclose(ts, [i.timesum + 3 * i.timestep for i in insts], rtol=1e-15)
    b.close()


def test_launch_shape_does_not_change_results():
    insts = small_batch()
    res = []
    for shape in [(8, 4, 1), (32, 16, 2)]:
        steps = [lib.MarkerStep.from_instance(i, precision=abi.PREC_MIXED) for i in insts]
        b = lib.Batch(steps)
        b.set_tune(*shape)
        dt = np.array([i.timestep for i in insts])
        ts = np.array([i.timesum for i in insts])
        b.step(dt, ts, 2)
        b.sync()
        res.append([ms.get_nodes() for ms in steps])
        b.close()
    for a, c in zip(res[0], res[1]):
        for kf in synth.NODE_OUT:
            np.testing.assert_array_equal(a[kf], c[kf])


def test_autotune_picks_a_shape_and_keeps_stepping():
    insts = small_batch()
    steps = [lib.MarkerStep.from_instance(i, precision=abi.PREC_MIXED) for i in insts]
    b = lib.Batch(steps)
    dt = np.array([i.timestep for i in insts])
    ts = np.array([i.timesum for i in insts])
    t = b.autotune(dt, ts, steps_per_candidate=1)
    assert t["candidates"] == 19 and t["tile_cols"] in (8, 16, 32) and t["ms_per_step"] > 0
    assert t["strategy"] in ("fused", "streams")
    # 19 candidates x (1 warm + 2 timed) steps advanced the instances
    np.testing.assert_allclose(ts, [i.timesum + 57 * i.timestep for i in insts], rtol=1e-13)
    b.step(dt, ts, 1)
    b.sync()
    b.close()


@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_MIXED])
def test_streams_strategy_equals_fused(precision):
    """Each instance on its own stream through the single-context step gives the
    fused batch's results bit for bit, and the two strategies can alternate."""
    insts = small_batch()
    out = []
    for plan in ([abi.BATCH_FUSED] * 3, [abi.BATCH_STREAMS] * 3,
                 [abi.BATCH_STREAMS, abi.BATCH_FUSED, abi.BATCH_STREAMS]):
        steps = [lib.MarkerStep.from_instance(i, precision=precision) for i in insts]
        for ms in steps:
            ms.set_fused(False)
        b = lib.Batch(steps)
        dt = np.array([i.timestep for i in insts])
        ts = np.array([i.timesum for i in insts])
        for strategy in plan:
            b.set_tune(strategy=strategy)
            b.step(dt, ts, 1)
        b.sync()
        out.append(([ms.get_markers() for ms in steps], [ms.get_nodes() for ms in steps]))
        np.testing.assert_allclose(ts, [i.timesum + 3 * i.timestep for i in insts], rtol=1e-15)
        b.close()
    for mk, nd in out[1:]:
        for a, c in zip(out[0][0], mk):
            for f in ("x", "y", "T", "p"):
                np.testing.assert_array_equal(a[f], c[f], err_msg=f)
        for a, c in zip(out[0][1], nd):
            for kf in synth.NODE_OUT:
                np.testing.assert_array_equal(a[kf], c[kf], err_msg=kf)


def test_streams_strategy_takes_the_fused_step():
    """The streams strategy steps every context through its own calls, so the
    mixed contexts take the fused movemark + averaging: the same results, bit for
    bit, as each context stepped alone."""
    insts = small_batch()
    steps = [lib.MarkerStep.from_instance(i, precision=abi.PREC_MIXED) for i in insts]
    b = lib.Batch(steps)
    b.set_tune(strategy=abi.BATCH_STREAMS)
    dt = np.array([i.timestep for i in insts])
    ts = np.array([i.timesum for i in insts])
    b.step(dt, ts, 3)
    b.sync()
    for inst, ms in zip(insts, steps):
        assert ms.fused_info()["fused_moves"] == 3
        mk, nd = single(inst, abi.PREC_MIXED, 3, fused=True)
        mk_b, nd_b = ms.get_markers(), ms.get_nodes()
        for f in ("x", "y", "T", "p"):
            np.testing.assert_array_equal(mk_b[f], mk[f], err_msg=f)
        for kf in synth.NODE_OUT:
            np.testing.assert_array_equal(nd_b[kf], nd[kf], err_msg=kf)
    b.close()


def test_c4_instances_match_oracle():
    """The 64 instances of the batched workload (grids 101..401, 115M markers)
    stepped together in the FP64 form; four of them, spread over the grid sizes,
    against the oracle (bit for bit where no libm call intervenes)."""
    from oracle import oracle
    nsteps = 2
    insts = synth.make_batch(64, nsteps=nsteps)
    steps = [lib.MarkerStep.from_instance(i, precision=abi.PREC_FP64) for i in insts]
    b = lib.Batch(steps)
    dt = np.array([i.timestep for i in insts])
    ts = np.array([i.timesum for i in insts])
    b.step(dt, ts, nsteps)
    b.sync()
    for k in (0, 21, 42, 63):
        inst = insts[k]
        s = oracle.Oracle(inst).run(order=oracle.ORDER_CELL)
        mk, nd = steps[k].get_markers(), steps[k].get_nodes()
        for f in ("x", "y", "T", "p"):
            np.testing.assert_array_equal(mk[f], getattr(s, f), err_msg=f"instance {k} {f}")
        for kf in ("ro", "et", "cp", "ht", "tk", "po"):
            np.testing.assert_array_equal(nd[kf], s.nodes[kf], err_msg=f"instance {k} {kf}")
        for kf in ("nu", "nd", "kt"):
            d = np.abs(nd[kf] - s.nodes[kf]).max() / np.abs(s.nodes[kf]).max()
            assert d <= 1e-12, (k, kf, d)
    b.close()
    for ms in steps:
        ms.close()


def test_streams_graph_equals_direct_launches():
    """The streams strategy replayed from a CUDA graph (mixed form, every
    instance on the fused step, per-step constants from the device table) gives
    bit for bit what launching every step from the host gives, and what each
    context stepping alone gives: across the record moves every 32nd step,
    calls of several lengths and tmax tracking."""
    insts = small_batch()
    res = []
    for graphs in (True, False):
        steps = [lib.MarkerStep.from_instance(i, precision=abi.PREC_MIXED) for i in insts]
        for ms, i in zip(steps, insts):
            ms.set_marker_extras(tmax=i.tmax)
        b = lib.Batch(steps)
        b.set_tune(strategy=abi.BATCH_STREAMS)
        b.set_graphs(graphs)
        dt = np.array([i.timestep for i in insts])
        ts = np.array([i.timesum for i in insts])
        for n in (1, 7, 30, 2):
            b.step(dt, ts, n, track_tmax=True)
        b.sync()
        assert sum(ms.fused_info()["fused_moves"] for ms in steps) >= 40 * len(insts)
        res.append(([ms.get_markers(with_tmax=True) for ms in steps], [ms.get_nodes() for ms in steps], ts.copy()))
        b.close()
        for ms in steps:
            ms.close()
    (mk_g, nd_g, ts_g), (mk_d, nd_d, ts_d) = res
    np.testing.assert_array_equal(ts_g, ts_d)
    for k, inst in enumerate(insts):
        for f in ("x", "y", "T", "eta", "p", "tmax"):
            np.testing.assert_array_equal(mk_g[k][f], mk_d[k][f], err_msg=f"instance {k} {f}")
        for kf in synth.NODE_OUT:
            np.testing.assert_array_equal(nd_g[k][kf], nd_d[k][kf], err_msg=f"instance {k} {kf}")
        mk, nd = single(inst, abi.PREC_MIXED, 40, fused=True)
        for f in ("x", "y", "T", "p"):
            np.testing.assert_array_equal(mk_g[k][f], mk[f], err_msg=f"instance {k} {f} vs single")
        for kf in synth.NODE_OUT:
            np.testing.assert_array_equal(nd_g[k][kf], nd[kf], err_msg=f"instance {k} {kf} vs single")
