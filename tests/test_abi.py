"""The C ABI library builds, loads without a GPU and exports what include/pybasin_b200.h declares."""

from __future__ import annotations

import ctypes
import re
import subprocess
from pathlib import Path

import pytest

from pybasin_b200 import _lib as L
from pybasin_b200 import build as B

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "pybasin_b200.h"


def declared_functions() -> list[str]:
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(pb_[a-z_0-9]+)\s*\(", text, re.M)))


def test_library_builds_and_loads():
    path = B.build()
    assert path.exists()
    lib = L.load()
    assert lib.pb_abi_version() == 102


def test_every_declared_symbol_is_exported():
    B.build()
    lib = ctypes.CDLL(str(B.lib_path()))
    names = declared_functions()
    assert set(L.EXPORTED_SYMBOLS) <= set(names)
    for n in names:
        assert hasattr(lib, n), f"{n} declared in {HEADER.name} but not exported"


def test_error_strings_without_gpu():
    lib = L.load()
    assert lib.pb_error_string(0) == b"success"
    assert b"invalid" in lib.pb_error_string(-5)


def test_invalid_arguments_are_rejected_without_launching():
    lib = L.load()
    assert lib.pb_solve_batch(None, None) == L.PB_EINVAL
    a = L.SolveArgs()
    a.dim = 2
    a.n_traj = 4
    a.n_ic = 4
    a.n_save = 1
    assert lib.pb_solve_batch(ctypes.byref(a), None) == L.PB_EINVAL  # null y0/params/save_ts
    assert lib.pb_label_nearest(None, 1, 1, None, 0, None, 1, None, None, 1, None, None, None) == L.PB_EINVAL


def test_solve_args_layout_matches_header():
    """offsetof/sizeof of pb_solve_args from the C compiler equal the ctypes mirror."""
    fields = [f[0] for f in L.SolveArgs._fields_]
    prog = ["#include <stdio.h>", "#include <stddef.h>", '#include "pybasin_b200.h"', "int main(void){"]
    prog.append('printf("size %zu\\n", sizeof(pb_solve_args));')
    for f in fields:
        prog.append(f'printf("{f} %zu\\n", offsetof(pb_solve_args, {f}));')
    prog.append("return 0;}")
    tmp = ROOT / "pybasin_b200" / "_lib"
    tmp.mkdir(exist_ok=True)
    src = tmp / "abi_layout.c"
    exe = tmp / "abi_layout"
    src.write_text("\n".join(prog))
    cc = "/usr/bin/gcc" if Path("/usr/bin/gcc").exists() else "gcc"
    try:
        subprocess.run([cc, "-I", str(ROOT / "include"), "-o", str(exe), str(src)], check=True)
    except (FileNotFoundError, subprocess.CalledProcessError) as e:  # pragma: no cover
        pytest.skip(f"no C compiler: {e}")
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = dict(line.split() for line in out if line.strip())
    assert int(got["size"]) == ctypes.sizeof(L.SolveArgs)
    for f in fields:
        assert int(got[f]) == getattr(L.SolveArgs, f).offset, f


def test_occupancy_query_needs_a_device_or_reports_error():
    lib = L.load()
    bps = ctypes.c_int32(0)
    sms = ctypes.c_int32(0)
    rc = lib.pb_query_occupancy(L.SYS_DUFFING, 2, L.PREC_MIXED, L.SCHED_QUEUE, 128, ctypes.byref(bps), ctypes.byref(sms))
    assert rc in (L.PB_SUCCESS, L.PB_ECUDA)
    assert lib.pb_query_occupancy(99, 2, 0, 0, 128, None, None) == L.PB_EINVALID_ODE


def test_scratch_size_and_noalloc_bound_the_feature_count_first():
    """A feature count beyond the fixed arrays of pb_solve_args is refused before the
    scratch layout walks those arrays (no GPU involved)."""
    lib = L.load()
    a = L.SolveArgs()
    a.dim = 2
    a.n_traj = 4
    a.n_ic = 4
    a.n_save = 8
    a.n_features = L.MAX_FEATURES + 1
    assert lib.pb_solve_scratch_bytes(ctypes.byref(a)) == -1
    assert lib.pb_solve_batch_noalloc(ctypes.byref(a), None) == L.PB_EINVAL
    a.n_features = -1
    assert lib.pb_solve_scratch_bytes(ctypes.byref(a)) == -1
    assert lib.pb_solve_batch_noalloc(ctypes.byref(a), None) == L.PB_EINVAL
