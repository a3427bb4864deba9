"""The engine library loads on a CPU-only host and exports the declared C ABI."""
import ctypes as C
import os
import re

import pytest

from fractura_b200 import _lib, abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            names += re.findall(r"AP_API\s+[\w\s\*]+?\b(ap_\w+)\s*\(", text)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "ap_render_pass" in names and "ap_histogram_cdf" in names
    assert set(_lib.EXPORTS) <= set(names)


def test_library_exports_every_declared_symbol():
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("engine library not built")
    L = C.CDLL(_lib.LIB_PATH)
    for name in declared_functions():
        assert hasattr(L, name), name


def test_abi_version_and_struct_layout():
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("engine library not built")
    L = _lib.load()
    assert L.ap_abi_version() == abi.AP_ABI_VERSION
    assert (C.sizeof(abi.ApFrameParams), C.sizeof(abi.ApFrameBuffers), C.sizeof(abi.ApTileDesc),
            C.sizeof(abi.ApGradView), C.sizeof(abi.ApStrictView)) == c_struct_sizes()


def c_struct_sizes(tmp_dir=None):
    """sizeof() of the header's structs as the C compiler lays them out."""
    import subprocess
    import tempfile
    d = tmp_dir or tempfile.mkdtemp()
    src = os.path.join(d, "sz.c")
    exe = os.path.join(d, "sz")
    with open(src, "w") as f:
        f.write('#include <stdio.h>\n#include "apeiron_b200.h"\n'
                'int main(void){printf("%zu %zu %zu %zu %zu", sizeof(ApFrameParams), sizeof(ApFrameBuffers),'
                ' sizeof(ApTileDesc), sizeof(ApGradView), sizeof(ApStrictView)); return 0;}\n')
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), src, "-o", exe], check=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split()
    return tuple(int(x) for x in out)


def test_oracle_sees_same_layout():
    import oracle
    assert oracle.lib().apo_abi_version() == abi.AP_ABI_VERSION


def test_invalid_arguments_rejected_without_gpu():
    """Validation happens before any CUDA call, so it is testable on a CPU host."""
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("engine library not built")
    L = _lib.load()
    p = abi.new_params(width=0, height=10)
    b = abi.ApFrameBuffers()
    assert L.ap_render_pass(C.byref(p), C.byref(b), None) == abi.AP_E_INVALID
    assert b"geometry" in L.ap_last_error()
    p = abi.new_params(width=8, height=8, max_iter=10, fractal_type=7)
    assert L.ap_render_pass(C.byref(p), C.byref(b), None) == abi.AP_E_INVALID
    assert L.ap_edge_detect(None, None, 4, 4, 0.35, None) == abi.AP_E_INVALID
    assert L.ap_histogram_cdf(None, 4, 4, 10, 65536, None, None, None) == abi.AP_E_INVALID


def test_batch_plan_checks_tiles_without_gpu():
    """ap_batch_plan is host code: it numbers the patches and rejects tiles that are not
    coarse perturbation passes on packed inputs."""
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("engine library not built")
    import numpy as np
    L = _lib.load()
    arr = (abi.ApTileDesc * 2)()
    for q, (w, h) in enumerate(((40, 20), (16, 16))):
        arr[q].p = abi.new_params(width=w, height=h, max_iter=100, tier=abi.AP_TIER_PERTURB,
                                  mode=abi.AP_MODE_COARSE, flags=abi.AP_FLAG_NO_RGB, ref_len=10)
        arr[q].orbit_packed = C.c_void_p(64)
        arr[q].iter_map = C.c_void_p(128)
    first = np.zeros(3, np.int64)
    assert L.ap_batch_plan(C.byref(arr), 2, 16, 16, first.ctypes.data_as(C.c_void_p)) == 0
    assert list(first) == [0, 3 * 2, 3 * 2 + 1]
    assert L.ap_batch_plan(C.byref(arr), 2, 16, 8, first.ctypes.data_as(C.c_void_p)) != 0  # 128 px
    arr[1].p.tier = abi.AP_TIER_FP64
    assert L.ap_batch_plan(C.byref(arr), 2, 16, 16, first.ctypes.data_as(C.c_void_p)) != 0
    assert b"tile 1" in L.ap_last_error()
