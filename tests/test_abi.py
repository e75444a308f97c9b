"""The C ABI library without a GPU: it loads, exports every function declared in
include/chswe.h, its swe_cfg layout matches the header, and calls that need a
device fail loudly (no CPU fallback)."""
import ctypes
import os
import re
import subprocess
import tempfile

import pytest

from tests.conftest import ROOT, gpu_available

HEADER = os.path.join(ROOT, "include", "chswe.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(swe_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_function(lib_built):
    lib = ctypes.CDLL(lib_built)
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    from ch_swe_b200 import _lib
    assert set(names) == set(_lib.EXPORTED)


def test_cfg_struct_layout_matches_header():
    from ch_swe_b200._lib import SweCfg
    prog = r'''
#include <stdio.h>
#include <stddef.h>
#include "chswe.h"
int main(void){
  printf("%zu %zu %zu %zu %zu %zu %zu\n", sizeof(swe_cfg), offsetof(swe_cfg, radius), offsetof(swe_cfg, grav),
         offsetof(swe_cfg, omega), offsetof(swe_cfg, rotation_axis), offsetof(swe_cfg, coriolis_constant),
         offsetof(swe_cfg, h_mean));
  return 0; }
'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        exe = os.path.join(d, "t")
        open(c, "w").write(prog)
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        got = [int(x) for x in subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()]
    want = [ctypes.sizeof(SweCfg), SweCfg.radius.offset, SweCfg.grav.offset, SweCfg.omega.offset,
            SweCfg.rotation_axis.offset, SweCfg.coriolis_constant.offset, SweCfg.h_mean.offset]
    assert got == want


def test_defaults_are_the_reference_constants(lib_built):
    from ch_swe_b200 import _lib
    cfg = _lib.SweCfg()
    assert _lib.load().swe_cfg_default(ctypes.byref(cfg)) == 0
    assert cfg.radius == 0.6371229e7 and cfg.grav == 9.80616
    assert abs(cfg.omega - 2 * 3.141592653589793 / 86164.0) < 1e-18
    assert list(cfg.rotation_axis) == [0.0, 0.0, 1.0]


def test_invalid_configurations_rejected(lib_built):
    from ch_swe_b200 import _lib
    L = _lib.load()
    cfg = _lib.SweCfg()
    L.swe_cfg_default(ctypes.byref(cfg))
    ctx = ctypes.c_void_p()
    for field, bad in (("N", 4), ("n_members", 0), ("precision", 7), ("operator_kind", 3)):
        c2 = _lib.SweCfg()
        ctypes.memmove(ctypes.byref(c2), ctypes.byref(cfg), ctypes.sizeof(cfg))
        setattr(c2, field, bad)
        assert L.swe_ctx_create(ctypes.byref(c2), ctypes.byref(ctx)) == -1


@pytest.mark.skipif(gpu_available(), reason="checks the no-device error path")
def test_no_device_fails_loudly(lib_built):
    from ch_swe_b200 import SweError, create_domain
    with pytest.raises(SweError):
        create_domain(16)


def test_ah_domain_validation():
    """The Ah and C staggerings are built for the linear operator, C for SBP 4-2
    (checked before any device call)."""
    import pytest
    from ch_swe_b200 import create_domain
    from ch_swe_b200.swm import state_shapes
    with pytest.raises(ValueError):
        create_domain(16, horizontal_staggering="Ah", operator="advective")
    with pytest.raises(ValueError):
        create_domain(16, horizontal_staggering="C", operator="advective")
    with pytest.raises(ValueError):
        create_domain(16, horizontal_staggering="C", sbp_order=21)
    with pytest.raises(ValueError):
        create_domain(16, horizontal_staggering="D")
    assert state_shapes(16, None, "C") == ((6, 16, 16), (6, 16, 17), (6, 17, 16))
    assert state_shapes(16, None, "Ah") == ((6, 17, 17),) * 3
    assert state_shapes(16, 2, "Ah")[1] == (2, 6, 17, 17)
