"""Host-side checks of the C ABI that need no GPU: the library loads, exports every
entry point declared in include/i2g.h, and rejects bad parameters before it touches
a device."""
import ctypes as C
import os
import re
import subprocess

import pytest

from i2elvis_planet_b200 import abi, lib, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "i2g.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(i2g_\w+)\s*\(", src)))


@pytest.fixture(scope="module")
def libi2g():
    if not os.path.exists(lib.LIB_PATH):
        from i2elvis_planet_b200 import build
        build.build()
    return lib.load()


def test_every_declared_symbol_is_exported(libi2g):
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(libi2g, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", lib.LIB_PATH], capture_output=True, text=True).stdout
    for n in names:
        assert re.search(rf"\bT {n}$", out, flags=re.M), n


def test_bindings_cover_the_header():
    assert set(declared_functions()) == set(lib.PROTOTYPES)


def test_struct_layouts_match_header():
    # i2g_types: 24 tables of 200 doubles + 200 int32
    assert C.sizeof(abi.Types) == 24 * 200 * 8 + 200 * 4
    assert C.sizeof(abi.Params) % 8 == 0
    assert abi.Params.device.offset + 4 + 7 * 4 == C.sizeof(abi.Params)


def test_status_strings(libi2g):
    assert libi2g.i2g_abi_version() == abi.ABI_VERSION
    for code, name in abi.STATUS_NAMES.items():
        assert libi2g.i2g_strerror(code)


def _params(**over):
    inst = synth.make_config("micro")
    p = abi.params_from_instance(inst)
    for k, v in over.items():
        setattr(p, k, v)
    return p, abi.types_from_instance(inst)


@pytest.mark.parametrize("field,value,status", [
    ("abi_version", 99, abi.EINVAL),
    ("xnumx", 2, abi.EINVAL),
    ("precision", 7, abi.EINVAL),
    ("gridmod", -1, abi.EINVAL),
    ("nubeg", 0.0, abi.EINVAL),
    ("intermod", 1, abi.EUNSUPPORTED),
    ("intermod1", 2, abi.EUNSUPPORTED),
    ("densimod", 3, abi.EUNSUPPORTED),
    ("viscmod", 3, abi.EUNSUPPORTED),
])
def test_create_rejects_bad_params_before_any_device_work(libi2g, field, value, status):
    p, t = _params(**{field: value})
    h = C.c_void_p()
    assert libi2g.i2g_create(C.byref(h), C.byref(p), C.byref(t)) == status
    assert not h.value


def test_create_without_device_fails_loudly(libi2g):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    p, t = _params()
    h = C.c_void_p()
    assert libi2g.i2g_create(C.byref(h), C.byref(p), C.byref(t)) == abi.ECUDA


@pytest.mark.skipif(subprocess.run(["which", "gcc"], capture_output=True).returncode != 0, reason="needs gcc")
def test_struct_layouts_match_the_c_compiler(tmp_path):
    """Every field offset and the size of each ctypes mirror equal what a C
    compiler makes of include/i2g.h."""
    mirrors = {"i2g_types": abi.Types, "i2g_params": abi.Params, "i2g_stats": abi.Stats, "i2g_tune": abi.Tune,
               "i2g_profile": abi.Profile, "i2g_fused_stats": abi.FusedStats, "i2g_td_table": abi.TdTable}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "i2g.h"', 'int main(void) {']
    for cname, cls in mirrors.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ['return 0;', '}']
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = {}
    for line in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines():
        cname, key, val = line.split()
        got[(cname, key)] = int(val)
    for cname, cls in mirrors.items():
        assert got[(cname, "size")] == C.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert got[(cname, fname)] == getattr(cls, fname).offset, (cname, fname)
