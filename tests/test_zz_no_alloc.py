"""i2g_ronurecalc_static, the averaging entry point that allocates nothing,
checked against the context entry point i2g_ronurecalc on the same problem.

Who it is for: callers that keep markers and nodes in device arrays of their own
and cannot allocate device memory where they average -- their memory belongs to
a pool allocator that must not be bypassed, or the host has reserved the device
for itself, or the time loop must not stall on the device synchronisation that
cudaMalloc/cudaFree can bring.  Instead of a context it uses one static scratch
array inside libi2g.so, which bounds a call to 65536 markers and 129 grid lines
per direction.

It runs the same kernels in the same summation order as the context path (cell
by cell, within a cell by caller index), so node fields and the reset marker
temperatures must agree bit for bit -- the bar of the context path's own
determinism tests -- in both precision forms.  Calls in a row on different
problems (smaller, then larger again, then one with strain fields, gridmod 2 and
markers outside the box) check that nothing left in the array by one call leaks
into the next.

This file is collected last on purpose: if it fails, a run stopped at the first
failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from i2elvis_planet_b200 import abi, lib, synth
from i2elvis_planet_b200.synth import NODE_OUT

pytestmark = pytest.mark.gpu

STATIC_GRID = ("pr", "exx", "eyy", "exy", "sxx", "syy", "sxy", "ga", "mu")


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    return torch


def context_average(inst, precision):
    """One i2g_ronurecalc on a context that holds the instance."""
    ms = lib.MarkerStep.from_instance(inst, precision=precision)
    ms.ronurecalc(inst.timesum)
    nodes = ms.get_nodes()
    T = ms.get_markers(fields=("T",))["T"]
    ms.close()
    return nodes, T


def static_average(torch, inst, precision):
    """One i2g_ronurecalc_static on device copies of the instance."""
    L = lib.load()
    dev = torch.device("cuda:0")

    def d(a, dtype=np.float64):
        return torch.as_tensor(np.ascontiguousarray(a, dtype=dtype), device=dev)

    P = abi.params_from_instance(inst, precision=precision)
    Ty = abi.types_from_instance(inst)
    gx, gy = d(inst.gx), d(inst.gy)
    grid = {k: (d(inst.grid[k]) if inst.grid.get(k) is not None else None) for k in STATIC_GRID}
    x, y, T, eta = d(inst.x), d(inst.y), d(inst.T), d(inst.eta)
    mt = d(inst.mtype, np.int8)
    nodes = {k: d(inst.nodes[k]) for k in NODE_OUT}

    def p(a):
        return a.data_ptr() if a is not None else None

    stream = torch.cuda.current_stream(dev).cuda_stream
    rc = L.i2g_ronurecalc_static(C.byref(P), C.byref(Ty), p(gx), p(gy), *[p(grid[k]) for k in STATIC_GRID],
                                 inst.x.size, p(x), p(y), p(T), p(eta), p(mt), inst.timesum,
                                 *[p(nodes[k]) for k in NODE_OUT], stream)
    assert rc == abi.OK, L.i2g_strerror(rc).decode()
    torch.cuda.synchronize(dev)
    return {k: v.cpu().numpy() for k, v in nodes.items()}, T.cpu().numpy()


def strained_micro():
    """The 21x21 case with strain-rate and stress fields, gridmod 2, markers
    without a viscosity of their own (viscalc at the marker) and markers outside
    the box (skipped by the averaging)."""
    import variants
    inst = variants.variant("strain_reinject")
    inst.flags["gridmod"] = 2
    inst.hi = np.zeros_like(inst.hi)  # the static entry point takes no impact times
    inst.x = inst.x.copy()
    inst.x[::13] = -1.0
    inst.x[5::17] = inst.xsize + 2.0
    return inst


def problems():
    # 61x61 grid, 57600 markers stored in shuffled order; the 21x21 micro case;
    # the 61x61 problem again (the second call left non-zero counts, cursors and
    # corner sums inside the range the third call uses); the strained case
    big = synth.make_config("c1", n=61, permute=True)
    return [big, synth.make_config("micro"), big, strained_micro()]


@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_MIXED], ids=["fp64", "mixed"])
def test_static_matches_context_on_calls_in_a_row(torch_cuda, precision):
    insts = problems()
    expected = [context_average(inst, precision) for inst in insts]
    for inst, (n_ref, T_ref) in zip(insts, expected):
        assert inst.x.size <= lib.load().i2g_static_max_markers()
        nodes, T = static_average(torch_cuda, inst, precision)
        for k in NODE_OUT:
            np.testing.assert_array_equal(nodes[k], n_ref[k], err_msg=f"{inst.name} {k}")
        np.testing.assert_array_equal(T, T_ref, err_msg=f"{inst.name} T")


def test_static_without_markers(torch_cuda):
    """No markers, after a call that had some: no node takes a value, and the
    contrast clamp of a call without any averaged viscosity clamps nu and nd to
    zero, as the reference's numin = numax = 0 does (markmart.c:995-1009)."""
    inst = synth.make_config("micro")
    static_average(torch_cuda, inst, abi.PREC_MIXED)
    empty = synth.subset(inst, np.arange(0))
    rng = np.random.default_rng(5)
    for k in NODE_OUT:
        empty.nodes[k] = rng.uniform(1.0, 2.0, inst.nodenum)
    nodes, _ = static_average(torch_cuda, empty, abi.PREC_MIXED)
    for k in NODE_OUT:
        if k in ("nu", "nd"):
            np.testing.assert_array_equal(nodes[k], 0.0, err_msg=k)
        else:
            np.testing.assert_array_equal(nodes[k], empty.nodes[k], err_msg=k)


def test_static_rejects_problems_beyond_its_scratch(torch_cuda):
    L = lib.load()
    inst = synth.make_config("micro")
    dev = torch_cuda.device("cuda:0")
    nmax = int(L.i2g_static_max_markers())
    big = torch_cuda.zeros(nmax + 1, dtype=torch_cuda.float64, device=dev)
    big8 = torch_cuda.zeros(nmax + 1, dtype=torch_cuda.int8, device=dev)
    nodes = torch_cuda.zeros(inst.nodenum, dtype=torch_cuda.float64, device=dev)
    g = torch_cuda.as_tensor(inst.gx, device=dev)
    Ty = abi.types_from_instance(inst)

    def call(P, n):
        return L.i2g_ronurecalc_static(C.byref(P), C.byref(Ty), g.data_ptr(), g.data_ptr(), nodes.data_ptr(),
                                       *[None] * 8, n, big.data_ptr(), big.data_ptr(), big.data_ptr(),
                                       big.data_ptr(), big8.data_ptr(), 0.0, *[nodes.data_ptr()] * 9, None)

    P = abi.params_from_instance(inst)
    assert call(P, nmax + 1) == abi.ECAPACITY
    P.xnumx = int(L.i2g_static_max_lines()) + 1
    assert call(P, 10) == abi.ECAPACITY
    P = abi.params_from_instance(inst)
    P.gridmod = 0
    assert call(P, 10) == abi.EINVAL
