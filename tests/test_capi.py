"""The C ABI library loads without a GPU and exports every symbol that
include/kapsel_gpu.h declares; host-only helpers are checked against the
oracle (no device calls)."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "kapsel_gpu.h")


def declared_symbols():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(kapsel_\w+)\s*\(", txt)))


@pytest.fixture(scope="module")
def lib():
    import kapsel_old_b200 as kg

    if not os.path.exists(kg.LIB_PATH):
        from kapsel_old_b200 import build

        build.build()
    return ctypes.CDLL(kg.LIB_PATH)


def test_exports_every_declared_symbol(lib):
    syms = declared_symbols()
    assert len(syms) >= 25
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_strerror_and_params_default(lib):
    import kapsel_old_b200 as kg

    L = kg.load_library()
    assert L.kapsel_gpu_strerror(0) == b"ok"
    assert b"invalid" in L.kapsel_gpu_strerror(-1)
    p = kg._Params()
    L.kapsel_params_default(ctypes.byref(p))
    assert list(p.np_xyz) == [6, 6, 6] and p.dt == 0.01 and p.a == 5.0 and p.rotation == 1


def test_thermostat_stream_matches_reference_mt19937(lib):
    from oracle import spm

    L = lib
    L.kapsel_thermostat_normals.argtypes = [ctypes.c_uint, ctypes.c_longlong, ctypes.c_longlong,
                                            ctypes.POINTER(ctypes.c_double)]
    out = np.zeros(600)
    assert L.kapsel_thermostat_normals(0, 0, 600, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))) == 0
    g = spm.MT19937Gauss(0)
    ref = g.normals6(100).reshape(-1)
    assert np.array_equal(out, ref)
    skip = np.zeros(12)
    assert L.kapsel_thermostat_normals(0, 588, 12, skip.ctypes.data_as(ctypes.POINTER(ctypes.c_double))) == 0
    assert np.array_equal(skip, ref[588:])


def test_sekibun_matches_oracle(lib):
    from oracle import spm

    L = lib
    L.kapsel_sekibun_cells.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                       ctypes.POINTER(ctypes.c_int), ctypes.c_int]
    for a, counts in ((5.0, 1935), (4.0, 1309), (6.0, 2801), (10.0, 8709)):
        n = L.kapsel_sekibun_cells(a, 2.0, 1.0, None, 0)
        assert n == counts
        buf = (ctypes.c_int * (3 * n))()
        assert L.kapsel_sekibun_cells(a, 2.0, 1.0, buf, n) == n
        mine = np.frombuffer(buf, dtype=np.int32).reshape(n, 3)
        cfg = {"np_xyz": (6, 6, 6), "particles": [], "a": a, "a_xi": 2.0}
        assert np.array_equal(mine, spm.sekibun_cells(spm.Params(cfg)))


def test_invalid_arguments_rejected_without_gpu(lib):
    import kapsel_old_b200 as kg

    L = kg.load_library()
    assert L.kapsel_gpu_create(None, None) == -1
    p = kg._Params()
    L.kapsel_params_default(ctypes.byref(p))
    p.np_xyz[0] = 3  # grids are 16..256 per axis
    h = ctypes.c_void_p()
    assert L.kapsel_gpu_create(ctypes.byref(p), ctypes.byref(h)) == -1
    p.np_xyz[0] = 9  # 512-point lines are beyond the in-kernel transforms
    assert L.kapsel_gpu_create(ctypes.byref(p), ctypes.byref(h)) == -1
    # NaN, Inf and out-of-range physical parameters are refused before any
    # device call (the reference would run on and produce NaN fields)
    for name, value in (("dt", float("nan")), ("dx", float("nan")), ("eta", -1.0), ("kbt", float("nan")),
                        ("kbt", -1e-3), ("mass_ratio", 0.0), ("gravity_g", float("inf")), ("a", float("nan"))):
        q = kg._Params()
        L.kapsel_params_default(ctypes.byref(q))
        setattr(q, name, value)
        assert L.kapsel_gpu_create(ctypes.byref(q), ctypes.byref(h)) == -1, name


C_CALLER = r"""
#include <stdio.h>
#include <string.h>
#include "kapsel_gpu.h"

/* A plain C caller of the C ABI: the calls that need no GPU. */
int main(void) {
  kapsel_params p;
  kapsel_ctx *ctx = NULL;
  kapsel_udf *u = NULL;
  kapsel_params_default(&p);
  if (p.np_xyz[0] != 6 || !(p.dt > 0.0)) return 1;
  p.dt = -1.0;
  if (kapsel_gpu_create(&p, &ctx) != KAPSEL_EINVAL || ctx != NULL) return 2;
  if (strlen(kapsel_gpu_strerror(KAPSEL_ETIMEOUT)) == 0) return 3;
  if (kapsel_udf_read("/nonexistent/input.udf", &u) == 0) return 4;
  printf("ok\n");
  return 0;
}
"""


def test_header_is_a_plain_c_interface(tmp_path):
    """include/kapsel_gpu.h compiles as strict C99 (no C++ in the interface)
    and a C program links against the library and calls it; the calls used
    here need no GPU."""
    import shutil
    import subprocess

    import kapsel_old_b200 as kg

    cc = shutil.which("gcc") or shutil.which("cc")
    if not cc:
        pytest.skip("no C compiler")
    src = tmp_path / "caller.c"
    src.write_text(C_CALLER)
    exe = tmp_path / "caller"
    libdir = os.path.dirname(kg.LIB_PATH)
    inc = os.path.join(os.path.dirname(libdir), "include")
    r = subprocess.run([cc, "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", inc, str(src), "-L", libdir,
                        "-lkapsel_gpu", f"-Wl,-rpath,{libdir}", "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and r.stdout.strip() == "ok", (r.returncode, r.stdout, r.stderr)
