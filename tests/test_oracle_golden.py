"""The oracle is pinned to the compiled reference: its outputs match the golden
fixtures (made by tests/golden/make_golden.py from the unmodified reference built
with FP64 marker storage) bit for bit."""
import hashlib
import os

import numpy as np
import pytest

import variants
from i2elvis_planet_b200 import synth
from oracle import oracle

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
MARKER_OUT = ("x", "y", "T", "eta", "p", "tmax")


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def load(name, kind="ref64"):
    return np.load(os.path.join(GOLD, f"{name}_{kind}.npz"))


def input_digest(inst):
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


@pytest.mark.parametrize("name", variants.NAMES)
def test_oracle_matches_reference_bitwise(name):
    inst = variants.variant(name)
    g = load(name)
    assert str(g["input_digest"]) == input_digest(inst), "synthetic generator drifted from the fixtures"
    mf = variants.move_flags(inst)
    s = oracle.Oracle(inst).run(eta_reinject=not mf, move_flags=mf)
    dev = variants.DEVIATIONS.get(name, ())
    for f in MARKER_OUT:
        assert digest(getattr(s, f)) == str(g[f"digest_{f}"]), f
    if "digest_por" in g:  # porosity after cold pressing and sintering
        assert digest(s.por) == str(g["digest_por"])
    if "digest_mg_old" in g:  # magnetisation state and time
        assert digest(s.mg_old) == str(g["digest_mg_old"])
        assert digest(s.mg_time) == str(g["digest_mg_time"])
    if "digest_type" in g:  # the table path flips types and leaves a melt state
        assert digest(s.mtype) == str(g["digest_type"])
        np.testing.assert_array_equal(s.melt, g["melt"])
    for k in synth.NODE_OUT:
        if k in dev:
            continue
        assert digest(s.nodes[k]) == str(g[f"digest_{k}"]), k


def test_table_path_exercises_its_branches():
    """The densimod 2 cases reach every branch they are there for: types flip both
    ways, the last table marker leaves a partial melt behind, and the crust-type
    'ht' deviation is confined to nodes those markers reach."""
    inst = variants.variant("td")
    g = load("td")
    s = oracle.Oracle(inst).run()
    assert ((inst.mtype < 20) & (s.mtype > 20)).any() and ((inst.mtype > 20) & (s.mtype < 20)).any()
    assert 0 < g["melt"][0] < 1
    diff = s.nodes["ht"] != g["n_ht"]
    o = oracle.Oracle(inst)
    ny = inst.ynumy
    touched = np.zeros(inst.nodenum, bool)
    for i in np.nonzero(np.isin(s.mtype, (11, 12, 31, 32)) | np.isin(inst.mtype, (11, 12, 31, 32)))[0]:
        key = o.cell_key(s.x[i], s.y[i])
        m1, m2 = divmod(key, ny - 1)
        for a in (0, 1):
            for b in (0, 1):
                touched[(m1 + a) * ny + m2 + b] = True
    assert not (diff & ~touched).any()


def test_declared_deviation_is_confined():
    """Unlisted rock types: the reference reuses the previous marker's radiogenic
    heating (markmart.c:749-837 leave mht unset); this build uses 0.  Only 'ht'
    differs, and only at nodes that such markers reach."""
    inst = variants.variant("unlisted_type")
    g = load("unlisted_type")
    s = oracle.Oracle(inst).run()
    diff = s.nodes["ht"] != g["n_ht"]
    assert diff.any()
    # every differing node has an unlisted-type marker within one cell
    o = oracle.Oracle(inst)
    ny = inst.ynumy
    touched = np.zeros(inst.nodenum, bool)
    for i in np.nonzero(np.isin(inst.mtype, (1, 3)))[0]:
        key = o.cell_key(s.x[i], s.y[i])
        m1, m2 = divmod(key, ny - 1)
        for a in (0, 1):
            for b in (0, 1):
                touched[(m1 + a) * ny + m2 + b] = True
    assert not (diff & ~touched).any()


def test_c1_oracle_matches_reference():
    inst = synth.make_config("c1")
    g = load("c1")
    assert str(g["input_digest"]) == input_digest(inst)
    s = oracle.Oracle(inst).run()
    for f in MARKER_OUT:
        assert digest(getattr(s, f)) == str(g[f"digest_{f}"]), f
    for k in synth.NODE_OUT:
        assert digest(s.nodes[k]) == str(g[f"digest_{k}"]), k


def test_cell_order_summation_close_to_reference():
    """Summing each node's markers cell by cell (the CUDA order) changes only
    rounding: <= 1e-13 relative on every node field."""
    inst = variants.variant("default")
    g = load("default")
    s = oracle.Oracle(inst).run(order=oracle.ORDER_CELL)
    for k in synth.NODE_OUT:
        ref = g[f"n_{k}"]
        err = np.abs(s.nodes[k] - ref) / np.maximum(np.abs(ref).max(), 1e-300)
        assert err.max() <= 1e-13, (k, err.max())


def test_ref32_storage_error_is_single_precision():
    """The reference's own storage (float markers) differs from FP64 storage by
    single-precision rounding; recorded to bound what 'matches the reference C loop'
    can mean for an FP64 path."""
    g64, g32 = load("default"), load("default", "ref32")
    for f in ("x", "y"):
        rel = np.abs(g64[f"m_{f}"] - g32[f"m_{f}"]) / 5e5
        assert rel.max() < 1e-6
    for k in ("ro", "tk"):
        a, b = g64[f"n_{k}"], g32[f"n_{k}"]
        assert np.abs(a - b).max() / np.abs(a).max() < 1e-4


# -- titerate()'s marker temperature update ---------------------------------------
def thermal_input_digest(inst, tk_new):
    h = hashlib.sha256(input_digest(inst).encode())
    h.update(np.ascontiguousarray(tk_new).tobytes())
    return h.hexdigest()


def oracle_thermal(name, order=oracle.ORDER_REFERENCE):
    inst, tk_new, heatdif = variants.thermal_variant(name)
    o = oracle.Oracle(inst)
    s = o.initial_state()
    o.titerate_markers(s, tk_new, heatdif, inst.timestep, order=order)
    return inst, tk_new, s


@pytest.mark.parametrize("name", variants.THERMAL_NAMES)
def test_titerate_oracle_matches_reference_bitwise(name):
    """The oracle's marker temperature update equals the reference's titerate()
    (FP64 storage) bit for bit: fluid reset, cold reset, subgrid diffusion with its
    -150 floor, node averages and antidiffusion in marker order."""
    inst, tk_new, s = oracle_thermal(name)
    g = load(f"titerate_{name}")
    assert str(g["input_digest"]) == thermal_input_digest(inst, tk_new), "synthetic generator drifted"
    assert digest(s.T) == str(g["digest_T"])
    np.testing.assert_array_equal(s.T[::int(g["stride"])], g["m_T"])


@pytest.mark.parametrize("name", ("thermal", "thermal_strong"))
def test_titerate_cell_order_close_to_reference(name):
    """The antidiffusion node sums in the CUDA order change only rounding."""
    inst, tk_new, s = oracle_thermal(name, oracle.ORDER_CELL)
    g = load(f"titerate_{name}")
    ref = g["m_T"]
    got = s.T[::int(g["stride"])]
    assert np.abs(got - ref).max() / np.abs(ref).max() <= 1e-14


def test_titerate_ref32_storage_error():
    """Reference storage keeps marker T in single precision: within 1e-6 relative."""
    g64, g32 = load("titerate_thermal"), load("titerate_thermal", "ref32")
    a, b = g64["m_T"], g32["m_T"]
    assert 0 < np.abs(a - b).max() / np.abs(a).max() < 1e-6


def test_titerate_cases_cover_their_branches():
    """Each thermal case reaches the branches it is there for."""
    inst, tk_new, hd = variants.thermal_variant("thermal")
    inside = (inst.x > 0) & (inst.y > 0) & (inst.x < inst.xsize) & (inst.y < inst.ysize)
    assert ((inst.mtype >= 50) & inside).sum() > 100             # fluid markers
    assert ((inst.T <= 0) & (inst.mtype < 50) & inside).sum() > 50  # cold resets
    inst, _, _ = variants.thermal_variant("thermal_edges")
    assert (~((inst.x > 0) & (inst.y > 0) & (inst.x < inst.xsize) & (inst.y < inst.ysize))).sum() >= 5
    inst, tk_new, hd = variants.thermal_variant("thermal_strong")
    dx = np.diff(inst.gx).min()
    kappa = (inst.nodes["kt"] / inst.nodes["ro"] / inst.nodes["cp"]).max()
    assert hd * kappa * 4.0 / dx ** 2 * inst.timestep > 150.0    # the exponent floor applies


def test_interp_tnode_known_answers():
    """allintert() (markmart.c:1687-1745) in the oracle: a node temperature that is
    bilinear in x and y on every cell is reproduced at any point inside the box
    (the weights are the cell's linear ones), points outside are clamped to the
    box first (markmart.c:1697-1698), and the optional second field follows the
    same weights."""
    inst = variants.variant("nonuniform")
    o = oracle.Oracle(inst)
    s = o.initial_state()
    gx, gy = np.meshgrid(inst.gx, inst.gy, indexing="ij")
    tk = (300.0 + 2e-3 * gx + 5e-3 * gy + 1e-9 * gx * gy).reshape(-1)
    tk2 = 2.0 * tk
    rng = np.random.default_rng(5)
    s.x = rng.uniform(-0.1, 1.1, s.x.size) * inst.xsize
    s.y = rng.uniform(-0.1, 1.1, s.y.size) * inst.ysize
    out, out2 = o.interp_tnode(s, tk, tk2)
    xc = np.clip(s.x, 0.0, inst.xsize)
    yc = np.clip(s.y, 0.0, inst.ysize)
    exact = 300.0 + 2e-3 * xc + 5e-3 * yc + 1e-9 * xc * yc
    assert np.abs(out - exact).max() <= 1e-10 * np.abs(exact).max()
    np.testing.assert_array_equal(out2, 2.0 * out)


@pytest.mark.parametrize("name", ("edges", "outgrid2", "nonuniform"))
def test_interp_tnode_matches_reference_bitwise(name):
    """The oracle's allintert() at every marker equals the reference's own
    allintert() (oracle/ref_harness.c mode 3, FP64 storage) bit for bit: markers
    on grid lines, on and outside the box edges, a nonuniform grid; tk2 is tk with
    a seeded ripple (tests/golden/make_golden.py)."""
    inst = variants.variant(name)
    tk = np.asarray(inst.nodes["tk"], dtype=np.float64)
    tk2 = tk + 5.0 * np.sin(np.arange(tk.size) * 0.37)
    g = np.load(os.path.join(GOLD, "interp_ref64.npz"))
    h = hashlib.sha256(input_digest(inst).encode())
    h.update(np.ascontiguousarray(tk2).tobytes())
    assert str(g[f"input_digest_{name}"]) == h.hexdigest(), "synthetic generator drifted"
    o = oracle.Oracle(inst)
    e2, e3 = o.interp_tnode(o.initial_state(), tk, tk2)
    assert digest(e2) == str(g[f"digest_eps2_{name}"])
    assert digest(e3) == str(g[f"digest_eps3_{name}"])
