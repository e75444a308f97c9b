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
import os
import subprocess
import sys

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


def test_noalloc_larger_then_smaller_cube():
    """N = 64 and then N = 16: the second call reuses parts of the array that the first
    wrote in another layout."""
    import torch
    from ch_swe_b200 import _lib, create_domain, create_stvec_swm, create_swm_operator, state_shapes
    L = _lib.load()
    for N in (64, 16):
        dom = create_domain(N, h_mean=900.0)
        op = create_swm_operator(dom.grav, {"swm_operator_type": "linear_swm_operator", "h_mean": 900.0}, dom)
        cfg = _cfg(dom)
        rng = np.random.default_rng(1000 + N)
        h, u, v = (rng.standard_normal(s) for s in state_shapes(N))
        x = create_stvec_swm(dom).upload(h, u, v)
        ref_out = create_stvec_swm(dom)
        op.apply(ref_out, x, dom)
        ref = ref_out.download()
        out = create_stvec_swm(dom)
        dom.synchronize()
        rc = L.swe_operator_apply_noalloc(ctypes.byref(cfg), x.device_view()[0], out.device_view()[0], None)
        assert rc == 0, _lib.ERRORS.get(rc, rc)
        torch.cuda.synchronize()
        for g, r, name in zip(out.download(), ref, "huv"):
            assert _rel(g, r) < FP64_RTOL, (N, name, _rel(g, r))
        dom.destroy()


_FRESH = r"""
import ctypes, sys
import numpy as np
import torch
sys.path.insert(0, sys.argv[1])
from ch_swe_b200 import _lib, state_shapes
N = 24
L = _lib.load()
cfg = _lib.SweCfg()
_lib.check(L.swe_cfg_default(ctypes.byref(cfg)))
cfg.N = N
cfg.h_mean = 800.0
rng = np.random.default_rng(5)
h, u, v = (rng.standard_normal(s) for s in state_shapes(N))
# the caller's own device buffers in the documented layout: [field][panel][N+9 rows][pitch],
# point (i, j) at row j+3, column i+3, zero margins
P = (N + 1 + 8 + 7) // 8 * 8
box = np.zeros((3, 6, N + 9, P))
box[0, :, 4:N + 5, 4:N + 5] = h
box[1, :, 4:N + 5, 4:N + 4] = u
box[2, :, 4:N + 4, 4:N + 5] = v
xin = torch.tensor(box, device="cuda")
yout = torch.zeros_like(xin)
rc = L.swe_operator_apply_noalloc(ctypes.byref(cfg), ctypes.c_void_p(xin.data_ptr()), ctypes.c_void_p(yout.data_ptr()), None)
assert rc == 0, rc
torch.cuda.synchronize()
got = yout.cpu().numpy()
# the reference afterwards: the context-based apply
from ch_swe_b200 import create_domain, create_stvec_swm, create_swm_operator
dom = create_domain(N, h_mean=800.0)
op = create_swm_operator(dom.grav, {"swm_operator_type": "linear_swm_operator", "h_mean": 800.0}, dom)
x = create_stvec_swm(dom).upload(h, u, v)
y = create_stvec_swm(dom)
op.apply(y, x, dom)
rh, ru, rv = y.download()
for g, r in ((got[0, :, 4:N + 5, 4:N + 5], rh), (got[1, :, 4:N + 5, 4:N + 4], ru), (got[2, :, 4:N + 4, 4:N + 5], rv)):
    err = np.abs(g - r).max() / np.abs(r).max()
    assert err < 1e-12, err
print("fresh-process noalloc ok")
"""


def test_noalloc_first_call_in_fresh_process():
    """The first call on a device in a process that never created a context (the case
    the entry point exists for): it looks up the array, uploads the edge tables and
    opts the kernels in to their shared memory itself."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", _FRESH, root], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "fresh-process noalloc ok" in r.stdout


def test_noalloc_rejects_cube_above_limit():
    from ch_swe_b200 import _lib
    cfg = _lib.SweCfg()
    L = _lib.load()
    _lib.check(L.swe_cfg_default(ctypes.byref(cfg)))
    cfg.N = _lib.SWE_NOALLOC_MAX_N + 1
    dummy = ctypes.c_void_p(16)
    assert L.swe_operator_apply_noalloc(ctypes.byref(cfg), dummy, ctypes.c_void_p(32), None) == _lib.SWE_ETOOBIG
