"""Failure paths, made on the host (no GPU fault): device memory running out at
each allocation of a context (I2G_FAIL_ALLOC_AT=k fails the k-th allocation as an
exhausted cudaMalloc would), a failing CUDA runtime (I2G_FAIL_CUDA=1), and
batches built from inconsistent contexts.  Every failure comes back as a status
code, leaves the context destroyable, and leaks no device memory."""
import ctypes as C
import gc
import os

import numpy as np
import pytest

from i2elvis_planet_b200 import abi, lib, synth

pytestmark = pytest.mark.gpu


@pytest.fixture
def env():
    keep = {k: os.environ.get(k) for k in ("I2G_FAIL_ALLOC_AT", "I2G_FAIL_CUDA")}
    yield os.environ
    for k, v in keep.items():
        if v is None:
            os.environ.pop(k, None)
        else:
            os.environ[k] = v


def free_bytes():
    import torch
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


def full_setup(inst, precision):
    """create, upload, one movemark + ronurecalc (the fused buckets are allocated there)"""
    ms = None
    try:
        ms = lib.MarkerStep(abi.params_from_instance(inst, precision=precision), abi.types_from_instance(inst))
        ms.set_grid(inst.gx, inst.gy, **inst.grid)
        ms.set_nodes(**inst.nodes)
        ms.set_markers(inst.x, inst.y, inst.T, inst.eta, inst.mtype)
        ms.movemark(inst.timestep, inst.timesum)
        ms.ronurecalc(inst.timesum)
        return None
    except lib.I2GError as e:
        return e
    finally:
        if ms is not None:
            ms.close()


@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_MIXED], ids=["fp64", "mixed"])
def test_every_allocation_failure_is_enomem_and_leaks_nothing(env, precision):
    inst = synth.make_config("micro")
    assert full_setup(inst, precision) is None  # warm the runtime and module loads
    free0 = free_bytes()
    failures = 0
    for k in range(1, 400):
        env["I2G_FAIL_ALLOC_AT"] = str(k)
        err = full_setup(inst, precision)
        gc.collect()
        if err is None:
            break
        assert err.status == abi.ENOMEM, (k, err)
        # i2g_create frees its context on failure and returns only the status
        assert "injected" in str(err) or "i2g_create" in str(err), err
        failures += 1
    else:
        pytest.fail("the set-up never completed")
    del env["I2G_FAIL_ALLOC_AT"]
    assert failures >= 20  # every device array of a context was hit
    assert abs(free_bytes() - free0) <= 2 << 20


def test_cuda_failure_is_ecuda_and_the_context_survives(env):
    inst = synth.make_config("micro")
    ms = lib.MarkerStep.from_instance(inst, precision=abi.PREC_MIXED)
    env["I2G_FAIL_CUDA"] = "1"
    for call in (lambda: ms.movemark(inst.timestep, inst.timesum), lambda: ms.ronurecalc(inst.timesum),
                 lambda: ms.get_markers()):
        with pytest.raises(lib.I2GError) as e:
            call()
        assert e.value.status == abi.ECUDA
        assert "injected" in str(e.value)
    del env["I2G_FAIL_CUDA"]
    ms.movemark(inst.timestep, inst.timesum)
    ms.ronurecalc(inst.timesum)
    assert np.isfinite(ms.get_nodes()["ro"]).all()
    ms.close()


def test_batches_of_inconsistent_contexts_are_rejected():
    L = lib.load()
    a = synth.make_config("micro")
    ok1 = lib.MarkerStep.from_instance(a, precision=abi.PREC_MIXED)
    ok2 = lib.MarkerStep.from_instance(a, precision=abi.PREC_MIXED)
    other = lib.MarkerStep.from_instance(a, precision=abi.PREC_FP64)
    empty = lib.MarkerStep.from_instance(a, precision=abi.PREC_MIXED, upload=False)

    def create(hs):
        arr = (C.c_void_p * len(hs))(*hs)
        b = C.c_void_p()
        rc = L.i2g_batch_create(C.byref(b), arr, len(hs))
        if rc == abi.OK:
            L.i2g_batch_destroy(b)
        return rc

    assert create([ok1.h.value, ok1.h.value]) == abi.EINVAL      # the same instance twice
    assert create([ok1.h.value, other.h.value]) == abi.EINVAL    # mixed and FP64 forms
    assert create([ok1.h.value, None]) == abi.ESTATE             # a missing instance
    assert create([ok1.h.value, empty.h.value]) == abi.ESTATE    # an instance without grid and markers
    assert create([ok1.h.value, ok2.h.value]) == abi.OK
    b = lib.Batch([ok1, ok2])
    dt = np.array([a.timestep] * 2)
    ts = np.array([a.timesum] * 2)
    assert L.i2g_batch_step(b.h, None, abi.dptr(ts), 1, 0) == abi.EINVAL
    assert L.i2g_batch_step(b.h, abi.dptr(dt), abi.dptr(ts), -1, 0) == abi.EINVAL
    assert L.i2g_batch_step(b.h, abi.dptr(dt), abi.dptr(ts), 1, 1 << 30) == abi.EINVAL
    b.step(dt, ts, 1)
    b.close()
    for m in (ok1, ok2, other, empty):
        m.close()
