"""The C-grid operators of the oracle (grad_c_sbp_sat_42, div_c_sbp_sat_42,
co2contra_c_sbp42_new: h on the cell centres, u on the x points, v on the y points),
pinned by properties of the discretisation that a wrong halo sign, swap or offset
breaks: the gradient of a constant vanishes; the SBP-SAT adjointness
<grad h, u>_x,y + <h, div u>_o = 0 holds to rounding for any fields; co2contra is
symmetric in the SBP inner product; and div(co2contra(grad h)) converges to the
Laplacian of the first spherical harmonic, -2 z / a^2."""
import numpy as np
import pytest

from oracle.oracle import EARTH_RADIUS, Oracle


@pytest.fixture(scope="module")
def orc(oracle_built):
    return Oracle(16)


def test_grad_of_constant_vanishes(orc):
    so, _, _ = orc.c_shapes()
    gx, gy = orc.c_grad(np.full(so, 7.5))
    assert np.abs(gx).max() < 1e-20 and np.abs(gy).max() < 1e-20


def test_sbp_sat_adjointness_any_fields(orc):
    rng = np.random.default_rng(3)
    so, sx, sy = orc.c_shapes()
    h, u, v = rng.standard_normal(so), rng.standard_normal(sx), rng.standard_normal(sy)
    gx, gy = orc.c_grad(h)
    d = orc.c_div(u, v)
    wo, wx, wy = orc.c_weights(0), orc.c_weights(1), orc.c_weights(2)
    a = (wx * gx * u).sum() + (wy * gy * v).sum()
    b = (wo * h * d).sum()
    assert abs(a + b) < 1e-12 * abs(a)


def test_co2contra_symmetric(orc):
    rng = np.random.default_rng(4)
    _, sx, sy = orc.c_shapes()
    u1, v1, u2, v2 = rng.standard_normal(sx), rng.standard_normal(sy), rng.standard_normal(sx), rng.standard_normal(sy)
    t1 = orc.c_co2contra(u1, v1)
    t2 = orc.c_co2contra(u2, v2)
    wx, wy = orc.c_weights(1), orc.c_weights(2)
    a = (wx * u2 * t1[0]).sum() + (wy * v2 * t1[1]).sum()
    b = (wx * u1 * t2[0]).sum() + (wy * v1 * t2[1]).sum()
    assert abs(a - b) < 1e-13 * abs(a)


def test_laplacian_of_first_harmonic_converges():
    """div(co2contra(grad z)) -> -2 z / a^2: about order 1.4 in the mean square (the closure
    rows of the composed first differences are first order) and above 2 away from the
    panel edges."""
    from ch_swe_b200.testcases import mesh_geometry
    rms, inner = [], []
    for N in (16, 32, 64):
        o = Oracle(N)
        r, _, _ = mesh_geometry(N, "o")
        z = r[..., 2] / np.linalg.norm(r, axis=-1)
        gx, gy = o.c_grad(z)
        ut, vt = o.c_co2contra(gx, gy)
        lap = o.c_div(ut, vt)
        exact = -2.0 * z / EARTH_RADIUS ** 2
        e = np.abs(lap - exact) / np.abs(exact).max()
        rms.append(np.sqrt((e ** 2).mean()))
        inner.append(e[:, 5:-5, 5:-5].max())
    r_rms = [np.log2(rms[k] / rms[k + 1]) for k in range(2)]
    r_in = [np.log2(inner[k] / inner[k + 1]) for k in range(2)]
    assert min(r_rms) > 1.3 and min(r_in) > 2.0, (rms, inner)
    assert inner[-1] < 1e-6
