"""The allocation-free operator entry point, for host programs that cannot call
cudaMalloc (their device memory belongs to another runtime or a fixed pool):
``swe_operator_apply_noalloc`` takes device pointers to the input and output
states and keeps every intermediate in a static device array of the library.

Checked through the C ABI against the context-based ``swe_operator_apply`` on
the same input, twice in a row (the static scratch keeps the previous call's
contents), within the FP64 tolerance of the other parity tests.  This file is
collected last so that a run stopping at the first failure has already run
every other test; it also passes when run alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from tests.conftest import gpu_available

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-12


@pytest.fixture(scope="module", autouse=True)
def _need_gpu(lib_built):
    if not gpu_available():
        pytest.fail("no CUDA device: the -m gpu tests need a B200")


def _rel(a, b):
    s = np.abs(b).max()
    return np.abs(a - b).max() / (s if s > 0 else 1.0)


def _cfg(dom):
    from ch_swe_b200 import _lib
    cfg = _lib.SweCfg()
    _lib.check(_lib.load().swe_cfg_default(ctypes.byref(cfg)))
    cfg.N = dom.N
    cfg.precision = _lib.SWE_FP64
    cfg.n_members = 1
    cfg.radius, cfg.grav, cfg.omega = dom.planet_radius, dom.grav, dom.omega
    for k in range(3):
        cfg.rotation_axis[k] = dom.rotation_axis[k]
    cfg.coriolis_constant = int(dom.coriolis_constant)
    cfg.h_mean = dom.h_mean
    return cfg


@pytest.mark.parametrize("N,axis", [(16, (0.0, 0.0, 1.0)), (64, (0.4, -0.2, 0.9))])
def test_noalloc_apply_matches_context_apply_twice(N, axis):
    import torch
    from ch_swe_b200 import _lib, create_domain, create_stvec_swm, create_swm_operator, state_shapes
    dom = create_domain(N, h_mean=750.0, rotation_axis=axis)
    op = create_swm_operator(dom.grav, {"swm_operator_type": "linear_swm_operator", "h_mean": 750.0}, dom)
    cfg = _cfg(dom)
    L = _lib.load()
    rng = np.random.default_rng(N)
    for call in range(2):
        h, u, v = (rng.standard_normal(s) for s in state_shapes(N))
        x = create_stvec_swm(dom).upload(h, u, v)
        ref_out = create_stvec_swm(dom)
        op.apply(ref_out, x, dom)
        ref = ref_out.download()
        out = create_stvec_swm(dom)
        dom.synchronize()
        xin, _, _, _ = x.device_view()
        yout, _, _, _ = out.device_view()
        rc = L.swe_operator_apply_noalloc(ctypes.byref(cfg), xin, yout, None)
        assert rc == 0, _lib.ERRORS.get(rc, rc)
        torch.cuda.synchronize()
        got = out.download()
        for g, r, name in zip(got, ref, "huv"):
            assert _rel(g, r) < FP64_RTOL, (call, name, _rel(g, r))


def test_noalloc_rejects_cube_above_limit():
    from ch_swe_b200 import _lib
    cfg = _lib.SweCfg()
    L = _lib.load()
    _lib.check(L.swe_cfg_default(ctypes.byref(cfg)))
    cfg.N = _lib.SWE_NOALLOC_MAX_N + 1
    dummy = ctypes.c_void_p(16)
    assert L.swe_operator_apply_noalloc(ctypes.byref(cfg), dummy, ctypes.c_void_p(32), None) == _lib.SWE_ETOOBIG
